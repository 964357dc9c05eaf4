// dem_slab.cuh -- kernels of the spatial (z-slab) decomposition of one
// system.
//
// A slab is a context that holds the arrays of every particle of the system
// (indexed by the system's own particle numbers) but advances only the
// particles of its cell layers [z0, z1) (DevParams::slab_c0/slab_c1): the
// relink keeps only its own cells' lists, the test kernel takes only its own
// particles as "i", the fold kernel folds and integrates only its own
// particles.  The sweep's half-shell (src/MForces.f90:199-272, offsets with
// kx + Nx*(ky + Ny*kz) > 0) reaches one layer up, so before the test a slab
// receives the layer above it (the ghost layer: its cells' lists in list
// order, the particles' pass copies, cells and current history rows); after
// the pair kernel it returns the "j" results it computed for those ghosts,
// and the records of theirs it matched, to their owner; after the fold it
// hands the particles that left its layers, with everything they own, to the
// slab they entered.  The slab below sends the cells of its top layer's
// particles, so that records whose partner sits there are judged adjacent or
// not exactly as the whole system would (partner_adjacent).
//
// Every exchange is a packed buffer of fixed-size records: a 16-byte header
// {what, count, record bytes, extra words}, `extra` int32 words, then
// `count` records of {int32 particle, int32 pad x3, columns}.  A column is
// an array of the context indexed (row, particle): element bytes `elem`
// (a multiple of 4) at base + row * stride + particle * elem.
#pragma once
#include "dem_pass.cuh"

namespace dem {

constexpr int SLAB_MAXC = 48;
constexpr int SLAB_HEAD = 16;  // bytes of the buffer header
constexpr int SLAB_ID = 16;    // bytes of a record's particle field

struct SlabCols {
  int n;         // columns
  int rec;       // bytes per record (SLAB_ID + the columns)
  int overflow;  // more than SLAB_MAXC columns were asked for
  const char* src[SLAB_MAXC];
  char* dst[SLAB_MAXC];
  long long stride[SLAB_MAXC];
  int elem[SLAB_MAXC];
  int rows[SLAB_MAXC];
  int off[SLAB_MAXC];  // byte offset of the column in the record
};

// The particles of cells [c_begin, c_begin + ncells), walking each list
// (any order across cells); *count must be 0 on entry.  A walk longer than n
// or a list longer than the room sets *err.
__global__ void k_slab_layer(const int* __restrict__ head, const int* __restrict__ next,
                             int c_begin, int ncells, int n, int* __restrict__ out,
                             int* __restrict__ count, int cap, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncells) return;
  int g = 0;
  for (int q = head[c_begin + i]; q != -1; q = next[q]) {
    if (++g > n || q < 0 || q >= n) {
      atomicExch(err, 1);
      return;
    }
    const int at = atomicAdd(count, 1);
    if (at < cap) out[at] = q;
    else atomicExch(err, 1);
  }
}

// Pack (list != NULL: the particles list[0..count)) or unpack (list ==
// NULL: the particles named in the records) the columns of C, one thread
// per 4-byte word of a record.  Unpacking also stamps stamp[p] = epoch and
// lists the particles in ids_out (each NULL: not done).
__global__ void k_slab_cols(SlabCols C, const int* __restrict__ list, int count, char* buf,
                            int* __restrict__ stamp, int epoch, int* __restrict__ ids_out) {
  const long long words = C.rec / 4;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= words * count) return;
  const int item = (int)(t / words);
  const int byte = (int)(t % words) * 4;
  char* rec = buf + (size_t)item * C.rec;
  const bool pack = list != nullptr;
  const int p = pack ? list[item] : *(const int*)rec;
  if (byte < SLAB_ID) {
    if (byte == 0) {
      if (pack) {
        *(int*)rec = p;
      } else {
        if (stamp) stamp[p] = epoch;
        if (ids_out) ids_out[item] = p;
      }
    }
    return;
  }
  int k = 0;
  while (k + 1 < C.n && C.off[k + 1] <= byte) k++;
  const int within = byte - C.off[k];
  const int row = within / C.elem[k];
  const int w = within % C.elem[k];
  const long long at = (long long)row * C.stride[k] + (long long)p * C.elem[k] + w;
  if (pack) *(int*)(rec + byte) = *(const int*)(C.src[k] + at);
  else *(int*)(C.dst[k] + at) = *(const int*)(rec + byte);
}

// *out = max(*out, v[ids[i]]) over the items (the fullest history table or
// result list of an exchange: the records carry that many slots)
__global__ void k_slab_max_of(const int* __restrict__ ids, int count, const int* __restrict__ v,
                              int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) atomicMax(out, v[ids[i]]);
}

// dst[i] = max(dst[i], src[i]) (rebuild stamps of a layer)
__global__ void k_slab_max(int* __restrict__ dst, const int* __restrict__ src, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m && src[i] > dst[i]) dst[i] = src[i];
}

// The "j" results (in_cap slots of `rec` bytes, layout [slot * stride + q])
// and matched-record bits of the ghosts ids[0..count), one record each:
// {q, count, matched, 0, slots...}; the ghosts' counts and bits are reset
// here (their owner folds them).
__global__ void k_slab_jhalf_pack(const int* __restrict__ ids, int count, int* __restrict__ in_cnt,
                                  const char* __restrict__ in_rec, int slots, int stride, int rec,
                                  unsigned* __restrict__ matched, char* __restrict__ buf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int q = ids[i];
  const int m = min(in_cnt[q], slots);
  int* h = (int*)(buf + (size_t)i * (SLAB_ID + (size_t)slots * rec));
  h[0] = q;
  h[1] = m;
  h[2] = (int)matched[q];
  h[3] = 0;
  char* d = (char*)(h + 4);
  for (int e = 0; e < m; e++) {
    const int* s = (const int*)(in_rec + ((size_t)e * stride + q) * rec);
    for (int w = 0; w < rec / 4; w++) ((int*)(d + (size_t)e * rec))[w] = s[w];
  }
  in_cnt[q] = 0;
  matched[q] = 0u;
}

// Append received "j" results after the owner's own (the fold orders them by
// sweep key) and OR the matched bits in; too many for the room sets the
// incoming overflow (the pass is then an error of the decomposition).
__global__ void k_slab_jhalf_unpack(const char* __restrict__ buf, int count, int* __restrict__ in_cnt,
                                    char* __restrict__ in_rec, int in_cap, int slots, int stride,
                                    int rec, unsigned* __restrict__ matched, Counters* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int* h = (const int*)(buf + (size_t)i * (SLAB_ID + (size_t)slots * rec));
  const int q = h[0], m = h[1];
  matched[q] |= (unsigned)h[2];
  const int base = in_cnt[q];
  const char* s = (const char*)(h + 4);
  for (int e = 0; e < m; e++) {
    if (base + e >= in_cap) {
      atomicMax(&cnt->need_in, base + m);
      atomicExch(&cnt->in_overflow, 1);
      atomicExch(&cnt->abort, 1);
      break;
    }
    int* d = (int*)(in_rec + ((size_t)(base + e) * stride + q) * rec);
    for (int w = 0; w < rec / 4; w++) d[w] = ((const int*)(s + (size_t)e * rec))[w];
  }
  in_cnt[q] = min(base + m, in_cap);
}

// Particles of the slab [c0, c1) (by cell_cur) whose next cell lies in
// [t0, t1) (the layer just above or just below): they leave for that slab.
// A next cell outside the slab and outside both neighbour layers (a jump of
// more than one layer) sets *err.
__global__ void k_slab_leavers(int n, const int* __restrict__ cell_cur,
                               const int* __restrict__ cell_nxt, int c0, int c1, int t0, int t1,
                               int u0, int u1, int* __restrict__ out, int* __restrict__ count,
                               int cap, int* __restrict__ err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int c = cell_cur[p];
  if (c < c0 || c >= c1) return;
  const int d = cell_nxt[p];
  if (d >= c0 && d < c1) return;
  if (d >= t0 && d < t1) {
    const int at = atomicAdd(count, 1);
    if (at < cap) out[at] = p;
    else atomicExch(err, 1);
  } else if (!(d >= u0 && d < u1)) {
    atomicExch(err, 2);
  }
}

// After a leaver was handed on: both of its cell entries name the cell it
// entered, so this slab never takes it for one of its own again.
__global__ void k_slab_depart(const int* __restrict__ ids, int count, int* __restrict__ cell_cur,
                              const int* __restrict__ cell_nxt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) cell_cur[ids[i]] = cell_nxt[ids[i]];
}

// A particle handed over by a neighbour slab enters its new cell's list at
// the next relink (RedistributeParticles3D's AddParticle, as the fold does
// for a particle of this slab that changed cell).
__global__ void k_slab_arrive(const int* __restrict__ ids, int count, CellLists L, Counters* cnt,
                              int par_cur, int par_nxt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int p = ids[i];
  L.mflag[p] = 0;
  note_cell(L, cnt, par_nxt, p, L.cell[par_cur][p], L.cell[par_nxt][p]);
}

}  // namespace dem
