// UpdateParticleList (src/MDEM.f90:612-671) on the device: particles that
// left the box are removed, highest index first, and the last particle takes
// the place of each one.  The removals are rare and inherently ordered (each
// one renumbers the current last particle), so one thread block applies them
// one after another; inside a removal the block works in parallel over the
// particles of the removed particle's 27-cell neighbourhood.
//
// The contact tables keep the reference's record set exactly:
//  * RemoveParticleFromContactList (src/MContacts.f90:579-633): records
//    "j -> i" of the neighbours j are dropped, and all records owned by i;
//  * ChangeIndexInContactList (src/MContacts.f90:173-252): a neighbour j
//    whose highest partner is NP (the last element of its ordered list) gets
//    partner i instead (j < i), or hands the record to i as "i -> j" (j > i);
//    i takes over NP's wall records.
// Records are looked up by exact partner match, and exported ordered by
// partner, which is the reference's ordered list.
#pragma once

#include "dem_kernels.cuh"

namespace dem {

constexpr int RM_THREADS = 512;
constexpr int RM_NB_CAP = 4096;  // particles of one 27-cell neighbourhood

// status words of a removal launch
constexpr int RM_OK = 0;
constexpr int RM_NEED_CAPACITY = 1;  // particle i would inherit more records than fit
constexpr int RM_NB_OVERFLOW = 2;    // a neighbourhood holds more than RM_NB_CAP particles
constexpr int RM_LIST_ERROR = 3;     // cell lists inconsistent

struct RemovalArgs {
  const DevParams* PT;
  StateArrays P;
  double* radius;
  int* comp;
  double* ring;
  int ring_slots;
  int ring_stride;  // the particle count the ring is laid out for
  CellLists L;
  int par;          // L.cell[par] = CellIndex
  History H;        // the live records
  // FP32 record values of the mixed mode (null in FP64 mode)
  float4 *ha, *hb;
  float* hc;
  float4 *wa, *wb;
  float* wc;
  int nw;
  int* list;    // escaped particles, -1 once removed
  int n_list;
  int* state;   // [0] particle count, [1] status, [2] capacity asked for,
                // [3] removals, [4] swaps, [5] records renamed or moved,
                // [8 + k] particles of component k removed
};
constexpr int RM_STATE_WORDS = 32;

// escaped particles: any coordinate outside [-L/2, L/2] (src/MDEM.f90:624-625)
__global__ void k_escape_list(const DevParams* __restrict__ PT, int n, StateArrays Q,
                              int* __restrict__ list, int* __restrict__ count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const DevParams& P = PT[0];
  const double x[3] = {Q.px[p], Q.py[p], Q.pz[p]};
  bool out = false;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double h = 0.5 * P.lbox[d];
    out = out || (x[d] > h) || (x[d] < -h);
  }
  if (out) list[atomicAdd(count, 1)] = p;
}

__device__ __forceinline__ void rm_copy_record(const RemovalArgs& A, size_t from, size_t to) {
  A.H.key[to] = A.H.key[from];
  if (A.ha) {
    A.ha[to] = A.ha[from];
    A.hb[to] = A.hb[from];
    A.hc[to] = A.hc[from];
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) A.H.val[to * 3 + k] = A.H.val[from * 3 + k];
  }
}

// drop record r of owner j (the later records move up one slot)
__device__ __forceinline__ void rm_drop_record(const RemovalArgs& A, int j, int r) {
  const int c = A.H.cnt[j];
  for (int s = r + 1; s < c; s++) rm_copy_record(A, hslot(A.H, j, s), hslot(A.H, j, s - 1));
  A.H.cnt[j] = c - 1;
}

// slot of the highest partner of owner j (-1: no records)
__device__ __forceinline__ int rm_top_record(const RemovalArgs& A, int j) {
  const int c = A.H.cnt[j];
  int best = -1, key = -1;
  for (int r = 0; r < c; r++) {
    const int k = A.H.key[hslot(A.H, j, r)];
    if (k > key) {
      key = k;
      best = r;
    }
  }
  return best;
}

// the MonteCarlo neighbour cells of cell c (NeighbourCells3D with MonteCarlo,
// src/MCells.f90:353-375, 424-476), the cell itself first; returns the count
__device__ int rm_neighbour_cells(const DevParams& P, int c, int* cells) {
  int ix, iy, iz;
  cell_coords(P, c, ix, iy, iz);
  const int I[3] = {ix, iy, iz};
  const int N[3] = {P.nx, P.ny, P.nz};
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {  // VerifyPBC (src/MCells.f90:1030-1040)
    lo[d] = -1;
    hi[d] = 1;
    if (!P.pbc[d]) {
      if (I[d] == 0) lo[d] = 0;
      if (I[d] == N[d] - 1) hi[d] = 0;
    }
  }
  int m = 0;
  cells[m++] = c;
  for (int kz = lo[2]; kz <= hi[2]; kz++)
    for (int ky = lo[1]; ky <= hi[1]; ky++)
      for (int kx = lo[0]; kx <= hi[0]; kx++) {
        if (kx == 0 && ky == 0 && kz == 0) continue;
        int j[3] = {ix + kx, iy + ky, iz + kz};
#pragma unroll
        for (int d = 0; d < 3; d++)  // ApplyPBC (src/MCells.f90:1044-1052)
          if (P.pbc[d]) {
            if (j[d] == N[d]) j[d] = 0;
            if (j[d] == -1) j[d] = N[d] - 1;
          }
        cells[m++] = P.coff + j[0] + P.nx * (j[1] + P.ny * j[2]);
      }
  return m;
}

__global__ void __launch_bounds__(RM_THREADS, 1) k_remove(RemovalArgs A) {
  __shared__ int s_cells[27];
  __shared__ int s_cnt[27];
  __shared__ int s_off[28];
  __shared__ int s_nb[RM_NB_CAP];
  __shared__ int s_red[RM_THREADS / 32];
  __shared__ int s_i, s_slot, s_m, s_ncell, s_app, s_need, s_stop;
  const DevParams& P = A.PT[0];
  const int t = threadIdx.x;
  const int lane = t & 31, wid = t >> 5;
  const int n_max = A.ring_stride;  // bound for every list walk
  for (;;) {
    // ---- the highest escaped index still present
    int best = -1, best_k = -1;
    for (int k = t; k < A.n_list; k += RM_THREADS) {
      const int v = A.list[k];
      if (v > best) {
        best = v;
        best_k = k;
      }
    }
    int wb = __reduce_max_sync(0xffffffffu, best);
    if (lane == 0) s_red[wid] = wb;
    __syncthreads();
    if (t == 0) {
      int m = -1;
      for (int w = 0; w < RM_THREADS / 32; w++) m = max(m, s_red[w]);
      s_i = m;
      s_stop = 0;
    }
    __syncthreads();
    const int i = s_i;
    if (i < 0) return;
    if (best == i && best_k >= 0) s_slot = best_k;  // one thread holds it
    const int NP = A.state[0] - 1;
    const int iCell = A.L.cell[A.par][i];
    // ---- AllNeighbourParticles (src/MCells.f90:833-860): the neighbourhood
    // of iCell before i leaves it; one thread per cell walks its list
    if (t == 0) s_ncell = rm_neighbour_cells(P, iCell, s_cells);
    __syncthreads();
    if (t < s_ncell) {
      int k = 0;
      for (int q = A.L.head[s_cells[t]]; q != -1 && k <= n_max; q = A.L.next[q]) k++;
      s_cnt[t] = k;
    }
    __syncthreads();
    if (t == 0) {
      int o = 0;
      for (int k = 0; k < s_ncell; k++) {
        s_off[k] = o;
        o += s_cnt[k];
      }
      s_off[s_ncell] = o;
      s_m = o;
      if (o > RM_NB_CAP) {
        A.state[1] = RM_NB_OVERFLOW;
        s_stop = 1;
      }
    }
    __syncthreads();
    if (s_stop) return;
    if (t < s_ncell) {
      int k = s_off[t];
      for (int q = A.L.head[s_cells[t]]; q != -1 && k < s_off[t + 1]; q = A.L.next[q])
        s_nb[k++] = q;
    }
    if (t == 0) s_need = 0;
    __syncthreads();
    const int m = s_m;
    // ---- capacity: the records i inherits from its neighbours j > i
    if (i != NP) {
      int need = 0;
      for (int k = t; k < m; k += RM_THREADS) {
        const int j = s_nb[k];
        if (j > i && j != NP) {
          const int r = rm_top_record(A, j);
          if (r >= 0 && A.H.key[hslot(A.H, j, r)] == NP) need++;
        }
      }
      need = __reduce_add_sync(0xffffffffu, need);
      if (lane == 0 && need) atomicAdd(&s_need, need);
    }
    __syncthreads();
    if (s_need > A.H.cap) {
      if (t == 0) {
        A.state[1] = RM_NEED_CAPACITY;
        A.state[2] = s_need;
      }
      return;  // nothing of this removal has been applied
    }
    // ---- RemoveParticleFromCell (src/MCells.f90:702-724)
    if (t == 0) {
      A.list[s_slot] = -1;
      A.state[8 + A.comp[i]] += 1;  // Component(Index)%Number - 1
      int q = A.L.head[iCell];
      if (q == i) {
        A.L.head[iCell] = A.L.next[i];
      } else {
        int guard = 0;
        while (q != -1 && A.L.next[q] != i && ++guard <= n_max) q = A.L.next[q];
        if (q == -1 || guard > n_max) {
          A.state[1] = RM_LIST_ERROR;
          s_stop = 1;
        } else {
          A.L.next[q] = A.L.next[i];
        }
      }
    }
    // ---- RemoveParticleFromContactList: "j -> i" records of the neighbours
    for (int k = t; k < m; k += RM_THREADS) {
      const int j = s_nb[k];
      if (j == i) continue;
      const int c = A.H.cnt[j];
      for (int r = 0; r < c; r++)
        if (A.H.key[hslot(A.H, j, r)] == i) {
          rm_drop_record(A, j, r);
          break;
        }
    }
    __syncthreads();
    if (s_stop) return;
    if (t == 0) {
      A.H.cnt[i] = 0;
      for (int w = 0; w < A.nw; w++) A.H.wflag[(size_t)i * A.nw + w] = 0;
      s_app = 0;
    }
    __syncthreads();
    if (i != NP) {
      // ---- Particle(i) = Particle(NP); Previous(:,i) = Previous(:,NP)
      double* const f[15] = {A.P.px, A.P.py, A.P.pz, A.P.vx, A.P.vy, A.P.vz, A.P.wx, A.P.wy,
                             A.P.wz, A.P.ax, A.P.ay, A.P.az, A.P.lx, A.P.ly, A.P.lz};
      if (t < 15) f[t][i] = f[t][NP];
      if (t == 15) A.radius[i] = A.radius[NP];
      if (t == 16) A.comp[i] = A.comp[NP];
      const int nring = A.ring_slots * 9;
      for (int k = t; k < nring; k += RM_THREADS) {
        double* r = A.ring + (size_t)k * A.ring_stride;
        r[i] = r[NP];
      }
      // ---- ReplaceParticleIndexInCell (src/MCells.f90:728-743)
      if (t == 0) {
        const int cNP = A.L.cell[A.par][NP];
        int q = A.L.head[cNP];
        if (q == NP) {
          A.L.head[cNP] = i;
        } else {
          int guard = 0;
          while (q != -1 && A.L.next[q] != NP && ++guard <= n_max) q = A.L.next[q];
          if (q == -1 || guard > n_max) {
            A.state[1] = RM_LIST_ERROR;
            s_stop = 1;
          } else {
            A.L.next[q] = i;
          }
        }
        A.L.next[i] = A.L.next[NP];
        A.L.cell[A.par][i] = cNP;
      }
      // ---- ChangeIndexInContactList, NP -> i
      for (int k = t; k < m; k += RM_THREADS) {
        const int j = s_nb[k];
        if (j == i || j == NP) continue;
        const int r = rm_top_record(A, j);
        if (r < 0) continue;
        const size_t sl = hslot(A.H, j, r);
        if (A.H.key[sl] != NP) continue;
        if (j < i) {
          A.H.key[sl] = i;
        } else {
          const int d = atomicAdd(&s_app, 1);
          const size_t to = hslot(A.H, i, d);
          rm_copy_record(A, sl, to);
          A.H.key[to] = j;
          rm_drop_record(A, j, r);
        }
        atomicAdd(&A.state[5], 1);
      }
      __syncthreads();
      if (s_stop) return;
      if (t == 0) {
        A.H.cnt[i] = s_app;
        A.H.cnt[NP] = 0;
        A.state[4] += 1;
      }
      for (int w = t; w < A.nw; w += RM_THREADS) {
        const size_t a = (size_t)i * A.nw + w, b = (size_t)NP * A.nw + w;
        A.H.wflag[a] = A.H.wflag[b];
        A.H.wflag[b] = 0;
        if (A.wa) {
          A.wa[a] = A.wa[b];
          A.wb[a] = A.wb[b];
          A.wc[a] = A.wc[b];
        } else {
#pragma unroll
          for (int k = 0; k < 3; k++) A.H.wval[a * 3 + k] = A.H.wval[b * 3 + k];
        }
      }
    }
    if (t == 0) {
      A.state[0] = NP;
      A.state[3] += 1;
    }
    __syncthreads();
  }
}

// the ring laid out for `nd` particles from a layout for `ns` (nd <= ns)
__global__ void k_ring_restride(const double* __restrict__ src, double* __restrict__ dst,
                                int slots9, int ns, int nd) {
  const size_t total = (size_t)slots9 * nd;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const size_t b = k / nd, i = k - b * nd;
    dst[k] = src[b * ns + i];
  }
}

}  // namespace dem

namespace dem {

// ---------------------------------------------------------------------------
// Pouring (PourParticle, src/MDEM.f90:412-532): the candidate points of all
// attempts (drawn on the host from the reference's generator) are tested at
// once, one warp per attempt; the host takes the first that fits.

struct PourTest {
  const DevParams* PT;
  const double* px;
  const double* py;
  const double* pz;
  const int* comp;
  CellLists L;
  const double2* cand;  // (x, y) of every attempt
  double z;             // pHalfLbox(3) - Ri
  double Ri;            // the largest component radius
  int ibig;             // its component (maxloc)
  int n_att;
  int n;                // particles (bound of every list walk)
  int* fits;            // [n_att] 1: no particle or wall overlaps the sphere
};

__global__ void __launch_bounds__(128) k_pour_test(PourTest T) {
  __shared__ int s_cells[4][27];
  __shared__ int s_nc[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int a = blockIdx.x * 4 + wid;
  if (a >= T.n_att) return;
  const DevParams& P = T.PT[0];
  const double2 c2 = T.cand[a];
  const double x[3] = {c2.x, c2.y, T.z};
  if (lane == 0) s_nc[wid] = rm_neighbour_cells(P, current_cell(P, x[0], x[1], x[2]), s_cells[wid]);
  __syncwarp();
  bool clash = false;
  if (lane < s_nc[wid]) {
    int guard = 0;
    for (int q = T.L.head[s_cells[wid][lane]]; q != -1 && !clash && ++guard <= T.n;
         q = T.L.next[q]) {
      // Rij is integer(ib) in PourParticle: each component is truncated
      const int r0 = (int)(T.px[q] - x[0]), r1 = (int)(T.py[q] - x[1]),
                r2 = (int)(T.pz[q] - x[2]);
      const int s = r0 * r0 + r1 * r1 + r2 * r2;
      clash = !((double)s > P.min_dij_sq[T.ibig * NCM + T.comp[q]]);
    }
  }
  if (lane < P.nw) {
    double Dij, Nij[3], Qji[3];
    clash = clash || overlap_wall(P, P.walls[lane], x, T.Ri, Dij, Nij, Qji);
  }
  clash = __any_sync(0xffffffffu, clash);
  if (lane == 0) T.fits[a] = clash ? 0 : 1;
}

// InsertParticle (src/MDEM.f90:536-561) at index n (the ring already laid
// out for n + 1 particles, its new entries zero)
struct InsertArgs {
  const DevParams* PT;
  StateArrays P;
  double* radius;
  int* comp;
  CellLists L;
  int par;
  History H0, H1;
  int nw;
  int n;
  int comp_new;
  double pos[3], vel_z, radius_new;
};

__global__ void k_insert(InsertArgs A) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const DevParams& P = A.PT[0];
  const int i = A.n;
  double* const f[15] = {A.P.px, A.P.py, A.P.pz, A.P.vx, A.P.vy, A.P.vz, A.P.wx, A.P.wy,
                         A.P.wz, A.P.ax, A.P.ay, A.P.az, A.P.lx, A.P.ly, A.P.lz};
  for (int k = 0; k < 15; k++) f[k][i] = 0.0;
  A.P.px[i] = A.pos[0];
  A.P.py[i] = A.pos[1];
  A.P.pz[i] = A.pos[2];
  A.P.vz[i] = A.vel_z;
  A.radius[i] = A.radius_new;
  A.comp[i] = A.comp_new;
  // CellIndex(NP) and AddParticle (prepend, src/MCells.f90:684-698); the
  // prepared transition sees the new particle staying in its cell
  const int c = current_cell(P, A.pos[0], A.pos[1], A.pos[2]);
  A.L.next[i] = A.L.head[c];
  A.L.head[c] = i;
  A.L.cell[A.par][i] = c;
  A.L.cell[A.par ^ 1][i] = c;
  A.L.mflag[i] = 0;
  A.H0.cnt[i] = 0;
  A.H1.cnt[i] = 0;
  for (int w = 0; w < A.nw; w++) {
    A.H0.wflag[(size_t)i * A.nw + w] = 0;
    A.H1.wflag[(size_t)i * A.nw + w] = 0;
  }
}

// the ring laid out for nd > ns particles (entries of the new particles zero)
__global__ void k_ring_widen(const double* __restrict__ src, double* __restrict__ dst, int slots9,
                             int ns, int nd) {
  const size_t total = (size_t)slots9 * nd;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const size_t b = k / nd, i = k - b * nd;
    dst[k] = i < (size_t)ns ? src[b * ns + i] : 0.0;
  }
}

}  // namespace dem
