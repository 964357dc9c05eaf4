// dem_pass.cuh -- device helpers shared by the FP64 and the mixed force
// passes: the per-block counters, the ordered fold, the AB/AM epilogues and the
// cell transition (RedistributeParticles3D's bookkeeping) for the next pass.
//
// A force pass is three kernels.  The test kernel (one thread per particle,
// in original index order) applies the reference's overlap test to the
// particle's candidate row (the partners it meets as "i") and lists its
// contacts; the pair kernel evaluates every listed contact once and hands its
// "i" half to the contact's place in the list and its "j" half to the
// partner; the fold kernel (one thread per particle) builds the particle's
// block of the sweep, adds the received halves and the block in the sweep's
// order and finishes with the integrator step of the pass (AB predictor or
// AM corrector).  Its epilogue also hashes the particle's next
// position into its cell and, when the cell changes, records the move for
// the next relink: the arrival list of the new cell and the dirty list of
// both cells.  Every such side effect is idempotent, so a pass that was
// stopped by a table overflow can be launched again after the tables grow.
#pragma once
#include <cstring>

#include "dem_device.cuh"

namespace dem {

__device__ __forceinline__ void mark_dirty(const CellLists& L, Counters* cnt, int par, int c) {
  if (atomicExch(&L.dflag[c], 1) == 0) {
    const int k = atomicAdd(&cnt->n_dirty[par], 1);
    L.dlist[par][k] = c;
  }
}

// Cell of particle p under the next assignment; a particle that changes cell
// is pushed once onto its new cell's arrival list.
__device__ __forceinline__ void note_cell(const CellLists& L, Counters* cnt, int par, int p,
                                          int c_old, int c_new) {
  L.cell[par][p] = c_new;
  if (c_new != c_old) {
    if (atomicExch(&L.mflag[p], 1) == 0) {
      L.mnext[p] = L.next[p];  // the relink walks the old list past p with it
      L.arr_next[p] = atomicExch(&L.arr_head[c_new], p);
      atomicAdd(&cnt->movers_pending, 1ull);
    }
    mark_dirty(L, cnt, par, c_old);
    mark_dirty(L, cnt, par, c_new);
  }
}

// squared minimum-image displacement between two positions of a particle
template <class BoxT>
__device__ __forceinline__ double disp2(const BoxT& P, const double a[3], const double b[3]) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double d = a[k] - b[k];
    if (P.pbc[k]) d = d - P.lbox[k] * rint(d * P.inv_lbox[k]);
    s = s + d * d;
  }
  return s;
}

// Largest displacement of the warp into the pass maximum (FP32 rounded up;
// non-negative floats order like their bit patterns).
__device__ __forceinline__ void publish_disp(Counters* cnt, double d2) {
  const unsigned bits = __float_as_uint(__double2float_ru(sqrt(d2)));
  const unsigned m = __reduce_max_sync(0xffffffffu, bits);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&cnt->disp_max, m);
}

// Per-warp pass statistics: one atomic per counter per warp.
__device__ __forceinline__ void publish_counts(Counters* cnt, bool update, unsigned n_col,
                                               unsigned n_pc, unsigned n_wc, unsigned need) {
  const unsigned FULL = 0xffffffffu;
  n_col = __reduce_add_sync(FULL, n_col);
  n_pc = __reduce_add_sync(FULL, n_pc);
  n_wc = __reduce_add_sync(FULL, n_wc);
  need = __reduce_max_sync(FULL, need);
  if ((threadIdx.x & 31) == 0) {
    if (need) atomicMax(&cnt->need_capacity, (int)need);
    if (n_col) atomicAdd(update ? &cnt->ncol_pending : &cnt->ncol, (unsigned long long)n_col);
    if (n_pc) atomicAdd(&cnt->pair_contacts, (unsigned long long)n_pc);
    if (n_wc) atomicAdd(&cnt->wall_contacts, (unsigned long long)n_wc);
  }
}

// The same statistics summed over the block first (one atomic per counter
// per block of at most 256 threads), together with the largest number of
// "j" records a particle received.  All threads of the block call.
__device__ __forceinline__ void publish_counts_block(Counters* cnt, bool update, unsigned n_col,
                                                     unsigned n_pc, unsigned n_wc,
                                                     unsigned need, unsigned need_in) {
  const unsigned FULL = 0xffffffffu;
  __shared__ unsigned s_c[8][5];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned v[5] = {__reduce_add_sync(FULL, n_col), __reduce_add_sync(FULL, n_pc),
                         __reduce_add_sync(FULL, n_wc), __reduce_max_sync(FULL, need),
                         __reduce_max_sync(FULL, need_in)};
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 5; k++) s_c[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t[5] = {0u, 0u, 0u, 0u, 0u};
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      t[0] += s_c[w][0];
      t[1] += s_c[w][1];
      t[2] += s_c[w][2];
      t[3] = t[3] > s_c[w][3] ? t[3] : s_c[w][3];
      t[4] = t[4] > s_c[w][4] ? t[4] : s_c[w][4];
    }
    if (t[0]) atomicAdd(update ? &cnt->ncol_pending : &cnt->ncol, (unsigned long long)t[0]);
    if (t[1]) atomicAdd(&cnt->pair_contacts, (unsigned long long)t[1]);
    if (t[2]) atomicAdd(&cnt->wall_contacts, (unsigned long long)t[2]);
    if (t[3]) atomicMax(&cnt->need_capacity, (int)t[3]);
    if (t[4]) atomicMax(&cnt->need_in, (int)t[4]);
  }
}

// The largest displacement of the block into the pass maximum (one atomic
// per block of at most 256 threads).  All threads of the block call.
__device__ __forceinline__ void publish_disp_block(Counters* cnt, double d2) {
  __shared__ unsigned s_d[8];
  const unsigned bits = __float_as_uint(__double2float_ru(sqrt(d2)));
  const unsigned m = __reduce_max_sync(0xffffffffu, bits);
  if ((threadIdx.x & 31) == 0) s_d[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = 0u;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = t > s_d[w] ? t : s_d[w];
    if (t) atomicMax(&cnt->disp_max, t);
  }
}

// Slot of partner `hi` among the records of `lo`; -1: no record.
__device__ __forceinline__ int find_record(const History& H, int lo, int hi) {
  const int c = H.cnt[lo];
  for (int r = 0; r < c; r++)
    if (H.key[hslot(H, lo, r)] == hi) return r;
  return -1;
}

// The "j" results a particle received in this pass, in the order of the
// givers' blocks in the sweep (their keys), with the particle's own block
// (key_p) at its place: the order in which ComputeAccelerations adds them to
// Force(p) and Torque(p) (src/MForces.f90:254-259, 319-320).  key_of(e)
// returns the key of record e; own() and add(e) fold.  The keys of the first
// 8 records are kept in registers; records past those are rare.
template <class KeyOf, class Own, class Add>
__device__ __forceinline__ void fold_in_order(int ni, unsigned long long key_p, KeyOf&& key_of,
                                              Own&& own, Add&& add) {
  unsigned long long kr[8];
#pragma unroll
  for (int e = 0; e < 8; e++) kr[e] = e < ni ? key_of(e) : ~0ull;
  bool own_done = false;
  unsigned long long lo = 0ull;  // every key >= lo is still to be folded
  for (int t = 0; t < ni; t++) {
    int best = -1;
    unsigned long long km = ~0ull;
#pragma unroll
    for (int e = 0; e < 8; e++)
      if (e < ni && kr[e] >= lo && kr[e] < km) {
        km = kr[e];
        best = e;
      }
    for (int e = 8; e < ni; e++) {
      const unsigned long long k = key_of(e);
      if (k >= lo && k < km) {
        km = k;
        best = e;
      }
    }
    if (!own_done && key_p < km) {
      own();
      own_done = true;
    }
    add(best);
    lo = km + 1ull;
  }
  if (!own_done) own();
}

template <class T>
__device__ __forceinline__ T mk_v4(double a, double b, double c, double d);
template <>
__device__ __forceinline__ double4 mk_v4<double4>(double a, double b, double c, double d) {
  return make_double4(a, b, c, d);
}
template <>
__device__ __forceinline__ float4 mk_v4<float4>(double a, double b, double c, double d) {
  return make_float4((float)a, (float)b, (float)c, (float)d);
}
template <class T>
__device__ __forceinline__ T mk_w2(double a, double b);
template <>
__device__ __forceinline__ double2 mk_w2<double2>(double a, double b) {
  return make_double2(a, b);
}
template <>
__device__ __forceinline__ float2 mk_w2<float2>(double a, double b) {
  return make_float2((float)a, (float)b);
}

__device__ __forceinline__ void prefetch_l2(const void* ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// The state the integrator epilogue of particle p will read, requested into
// L2 at the start of the fold kernel so that those reads overlap the fold
// (they do not depend on it).  mixed: the FP64 velocities of Particle
// (predictor) or Predicted (corrector) come from the state arrays.
template <int EPI, class V4, class W2>
__device__ __forceinline__ void prefetch_epilogue(const PassArgs<V4, W2>& A, const DevParams& P,
                                                  int p, bool mixed) {
  if (EPI == EPI_STORE) return;
  const size_t n = (size_t)A.n;
  if (EPI == EPI_PREDICT) {
    for (int k = 0; k < P.nprev; k++) {
      const double* rg = A.ring + (size_t)A.rm.phys[k] * 9 * n + p;
#pragma unroll
      for (int d = 0; d < 9; d++) prefetch_l2(rg + d * n);
    }
    if (mixed) {
      const double* v[6] = {A.part.vx, A.part.vy, A.part.vz, A.part.wx, A.part.wy, A.part.wz};
#pragma unroll
      for (int d = 0; d < 6; d++) prefetch_l2(v[d] + p);
    }
  } else {
    if (A.amsum)
#pragma unroll
      for (int d = 0; d < 9; d++) prefetch_l2(A.amsum + d * n + p);
    const double* q[9] = {A.part.px, A.part.py, A.part.pz, A.part.vx, A.part.vy,
                          A.part.vz, A.part.wx, A.part.wy, A.part.wz};
#pragma unroll
    for (int d = 0; d < 9; d++) prefetch_l2(q[d] + p);
    if (mixed) {
      prefetch_l2(A.pred.vx + p);
      prefetch_l2(A.pred.vy + p);
      prefetch_l2(A.pred.vz + p);
    }
  }
}

// The integrator part of a pass, after a = F/m and alpha = T/I
// (src/MForces.f90:330-333):
//  EPI_STORE   a, alpha -> tgt;
//  EPI_PREDICT the AB predictor of MoveParticles (src/MDEM.f90:296-331) from
//              x(t) = xp, v(t) = vp, w(t) = wp and the ring, (v,a,alpha)(t)
//              into the spare ring slot; the prediction is the next pass's
//              position;
//  EPI_CORRECT the AM corrector (src/MDEM.f90:340-367) with v~ = vp; the new
//              x(t+dt) is the next pass's position.
// d2 receives the squared displacement from this pass's position to the next.
template <int EPI, class V4, class W2>
__device__ __forceinline__ void epilogue(const PassArgs<V4, W2>& A, const DevParams& P, int p,
                                         const double xp[3], double Rp, const double vp[3],
                                         const double wp[3], const double acc[3],
                                         const double alp[3], int c_cur, double& d2) {
  const Box& B = P.box;
  const size_t n = (size_t)A.n;
  if (EPI == EPI_STORE) {
    A.tgt.ax[p] = acc[0]; A.tgt.ay[p] = acc[1]; A.tgt.az[p] = acc[2];
    A.tgt.lx[p] = alp[0]; A.tgt.ly[p] = alp[1]; A.tgt.lz[p] = alp[2];
    return;
  }
  double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
  if (EPI == EPI_CORRECT && A.amsum) {
    // sum_k AM(k)*Previous(ipc(k)) over the rotated ring, as the predictor
    // pass formed it (same terms, same order)
#pragma unroll
    for (int d = 0; d < 3; d++) sv[d] = A.amsum[d * n + p];
#pragma unroll
    for (int d = 0; d < 3; d++) sa[d] = A.amsum[(3 + d) * n + p];
#pragma unroll
    for (int d = 0; d < 3; d++) sl[d] = A.amsum[(6 + d) * n + p];
  } else {
    // the predictor also forms the corrector's sums: after the ring rotation
    // its slot k is this pass's (v, a, alpha) for k = 0, else the slot k-1
    // read here
    const bool am = EPI == EPI_PREDICT && A.amsum && P.nprev > 0;
    double mv[3], ma[3], ml[3];
    if (am) {
#pragma unroll
      for (int d = 0; d < 3; d++) mv[d] = 0.0 + P.am[0] * vp[d];
#pragma unroll
      for (int d = 0; d < 3; d++) ma[d] = 0.0 + P.am[0] * acc[d];
#pragma unroll
      for (int d = 0; d < 3; d++) ml[d] = 0.0 + P.am[0] * alp[d];
    }
    for (int k = 0; k < P.nprev; k++) {
      const double C = EPI == EPI_PREDICT ? P.ab[k] : P.am[k];
      const double* rg = A.ring + (size_t)A.rm.phys[k] * 9 * n + p;
      double t[9];
#pragma unroll
      for (int d = 0; d < 9; d++) t[d] = rg[d * n];
#pragma unroll
      for (int d = 0; d < 3; d++) sv[d] = sv[d] + C * t[d];
#pragma unroll
      for (int d = 0; d < 3; d++) sa[d] = sa[d] + C * t[3 + d];
#pragma unroll
      for (int d = 0; d < 3; d++) sl[d] = sl[d] + C * t[6 + d];
      if (am && k + 1 < P.nprev) {
        const double M = P.am[k + 1];
#pragma unroll
        for (int d = 0; d < 3; d++) mv[d] = mv[d] + M * t[d];
#pragma unroll
        for (int d = 0; d < 3; d++) ma[d] = ma[d] + M * t[3 + d];
#pragma unroll
        for (int d = 0; d < 3; d++) ml[d] = ml[d] + M * t[6 + d];
      }
    }
    if (am) {
#pragma unroll
      for (int d = 0; d < 3; d++) A.amsum[d * n + p] = mv[d];
#pragma unroll
      for (int d = 0; d < 3; d++) A.amsum[(3 + d) * n + p] = ma[d];
#pragma unroll
      for (int d = 0; d < 3; d++) A.amsum[(6 + d) * n + p] = ml[d];
    }
  }
  double x[3], v[3], w[3];
  if (EPI == EPI_PREDICT) {
    const StateArrays& Q = A.part;
    const StateArrays& R = A.pred;
    // (with A.lazy, a and alpha stay in the new ring slot only)
    if (!A.lazy || P.nprev == 0) {
      Q.ax[p] = acc[0]; Q.ay[p] = acc[1]; Q.az[p] = acc[2];
      Q.lx[p] = alp[0]; Q.ly[p] = alp[1]; Q.lz[p] = alp[2];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = xp[d] + P.ab0 * vp[d] + sv[d];
#pragma unroll
    for (int d = 0; d < 3; d++) v[d] = vp[d] + P.ab0 * acc[d] + sa[d];
#pragma unroll
    for (int d = 0; d < 3; d++) w[d] = wp[d] + P.ab0 * alp[d] + sl[d];
#pragma unroll
    for (int d = 0; d < 3; d++)
      if (B.pbc[d]) x[d] = x[d] - B.lbox[d] * fnint(x[d] * B.inv_lbox[d]);
    // (with A.lazy, Predicted x stays in the position copy Xn, and with
    // FP64 copies Predicted v, w stay in v4n, w2n; the mixed corrector reads
    // Predicted v, and its FP32 copies do not hold v, w exactly)
    if (!A.lazy) {
      R.px[p] = x[0]; R.py[p] = x[1]; R.pz[p] = x[2];
    }
    if (!A.lazy || sizeof(V4) != sizeof(double4)) {
      R.vx[p] = v[0]; R.vy[p] = v[1]; R.vz[p] = v[2];
      R.wx[p] = w[0]; R.wy[p] = w[1]; R.wz[p] = w[2];
    }
    if (P.nprev > 0) {
      double* rg = A.ring + (size_t)A.rm.phys[P.nprev] * 9 * n + p;
#pragma unroll
      for (int d = 0; d < 3; d++) rg[d * n] = vp[d];
#pragma unroll
      for (int d = 0; d < 3; d++) rg[(3 + d) * n] = acc[d];
#pragma unroll
      for (int d = 0; d < 3; d++) rg[(6 + d) * n] = alp[d];
    }
  } else {
    const StateArrays& Q = A.part;
    const StateArrays& R = A.pred;
    R.ax[p] = acc[0]; R.ay[p] = acc[1]; R.az[p] = acc[2];
    R.lx[p] = alp[0]; R.ly[p] = alp[1]; R.lz[p] = alp[2];
    x[0] = Q.px[p]; x[1] = Q.py[p]; x[2] = Q.pz[p];
    v[0] = Q.vx[p]; v[1] = Q.vy[p]; v[2] = Q.vz[p];
    w[0] = Q.wx[p]; w[1] = Q.wy[p]; w[2] = Q.wz[p];
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = x[d] + P.am0 * vp[d] + sv[d];
#pragma unroll
    for (int d = 0; d < 3; d++) v[d] = v[d] + P.am0 * acc[d] + sa[d];
#pragma unroll
    for (int d = 0; d < 3; d++) w[d] = w[d] + P.am0 * alp[d] + sl[d];
#pragma unroll
    for (int d = 0; d < 3; d++)
      if (B.pbc[d]) x[d] = x[d] - B.lbox[d] * fnint(x[d] * B.inv_lbox[d]);
    Q.px[p] = x[0]; Q.py[p] = x[1]; Q.pz[p] = x[2];
    Q.vx[p] = v[0]; Q.vy[p] = v[1]; Q.vz[p] = v[2];
    Q.wx[p] = w[0]; Q.wy[p] = w[1]; Q.wz[p] = w[2];
    bool out = false;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double h = 0.5 * B.lbox[d];
      out = out || (x[d] > h) || (x[d] < -h);
    }
    if (out) atomicAdd(&A.cnt->escaped, 1ull);
  }
  // the next pass's copies, cell and displacement
  A.Xn[p] = make_double4(x[0], x[1], x[2], Rp);
  A.v4n[p] = mk_v4<V4>(v[0], v[1], v[2], w[0]);
  A.w2n[p] = mk_w2<W2>(w[1], w[2]);
  note_cell(A.L, A.cnt, A.par_nxt, p, c_cur, current_cell(P, x[0], x[1], x[2]));
  d2 = disp2(B, x, xp);
  if (!isfinite(x[0] + x[1] + x[2])) {
    // a diverged state would put every particle into one cell; stop here
    atomicExch(&A.cnt->nonfinite, 1);
    set_abort(A.cnt, A.tag);
  }
}

// First statement of every kernel of a force pass (relink, test, pair,
// fold).  A kernel launched with programmatic stream serialization may be
// scheduled while the kernel before it in the stream is still running; it
// waits here until that kernel has completed and its writes are visible, and
// then allows the next kernel of the pass to be scheduled (whose blocks take
// the SM slots this kernel's last blocks free, and wait in turn).  Without
// that launch attribute both instructions return at once.  Nothing a pass
// kernel reads or writes is touched before the wait.
__device__ __forceinline__ void pass_kernel_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Host side: launch a pass kernel on `st`, with programmatic stream
// serialization when `early` (the kernel must begin with pass_kernel_entry).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pass(bool early, void (*kernel)(KArgs...), unsigned grid, unsigned block,
                               cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = early ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

__device__ __forceinline__ void set_abort(Counters* cnt, int tag) {
  atomicCAS(&cnt->abort_tag, 0, tag + 1);
  atomicExch(&cnt->abort, 1);
}

}  // namespace dem
