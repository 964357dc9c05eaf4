// dem_kernels.cuh -- sm_100a kernels of the FP64 DEM step.
//
// K1  cell rebuild = counting sort of particles by cell hash into traversal
//     order (k_assign -> scan -> k_scatter -> k_cellsort -> k_gather).
//     Within a cell the order is exactly the reference's linked-list order:
//     RedistributeParticles3D (src/MCells.f90:607-643) walks particles in
//     index order and prepends every particle that changed cell
//     (TransferParticle, :747-774), so a cell lists first the particles that
//     entered it during this pass (highest index first) and then the ones that
//     stayed, in their previous order.  The sort key encodes exactly that.
// K2+K4 force kernel: one thread per particle in traversal order gathers its
//     contacts (no atomics), evaluates every pair in the reference's
//     orientation ("i" = the particle visited first) and adds the
//     contributions in the order of the reference's cell sweep, so that the
//     forces are bit-identical to ComputeAccelerations (src/MForces.f90:
//     145-335).  The AB predictor / AM corrector (src/MDEM.f90:296-365) run in
//     the same kernel's epilogue.
// K3  history: records owned by imin are double-buffered; a pass that updates
//     them writes a fresh table (new/updated contacts + records of pairs that
//     the sweep did not visit, as the reference keeps those untouched).
#pragma once
#include "dem_device.cuh"

namespace dem {

// ---------------------------------------------------------------------------
// warp helpers
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// K1: cell rebuild

// One thread per current slot: new cell, mover flag, sort key, slot in cell.
__global__ void k_assign(const DevParams* __restrict__ Pp, int n, int initial,
                         const double* __restrict__ px, const double* __restrict__ py,
                         const double* __restrict__ pz, const int* __restrict__ order,
                         const int* __restrict__ old_cell, int* __restrict__ cell_cnt,
                         int* __restrict__ a_cell, int* __restrict__ a_loc,
                         unsigned* __restrict__ a_key, int* __restrict__ a_orig,
                         Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0 && cnt->ncol_pending) {
    // the previous history-updating pass completed: its Ncol counts
    cnt->ncol += cnt->ncol_pending;
    cnt->ncol_pending = 0;
  }
  unsigned long long mv = 0;
  if (s < n) {
    const DevParams& P = *Pp;
    int orig = initial ? s : order[s];
    int c = current_cell(P, px[orig], py[orig], pz[orig]);
    int old = initial ? -1 : old_cell[s];
    bool mover = c != old;
    unsigned key = mover ? (unsigned)(n - 1 - orig) : (unsigned)(n + s);
    int loc = atomicAdd(&cell_cnt[c], 1);
    a_cell[s] = c;
    a_loc[s] = loc;
    a_key[s] = key;
    a_orig[s] = orig;
    mv = mover ? 1ull : 0ull;
  }
  mv = warp_sum_u64(mv);
  if ((threadIdx.x & 31) == 0 && mv) atomicAdd(&cnt->movers, mv);
}

// k_assign for the context path: also marks the old and new cell of every
// particle that changed cell (their neighbourhoods' candidate rows are
// rebuilt) and tracks the largest squared displacement since the last full
// candidate-list rebuild.
__global__ void k_assign_track(const DevParams* __restrict__ Pp, int n,
                               const double* __restrict__ px, const double* __restrict__ py,
                               const double* __restrict__ pz, const int* __restrict__ order,
                               const int* __restrict__ old_cell, int* __restrict__ cell_cnt,
                               int* __restrict__ a_cell, int* __restrict__ a_loc,
                               unsigned* __restrict__ a_key, int* __restrict__ a_orig,
                               ContactLists L, Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0 && cnt->ncol_pending) {
    cnt->ncol += cnt->ncol_pending;
    cnt->ncol_pending = 0;
  }
  unsigned long long mv = 0;
  double d2 = 0.0;
  if (s < n) {
    const DevParams& P = *Pp;
    const int orig = order[s];
    const double x = px[orig], y = py[orig], z = pz[orig];
    const int c = current_cell(P, x, y, z);
    const int old = old_cell[s];
    const bool mover = c != old;
    const unsigned key = mover ? (unsigned)(n - 1 - orig) : (unsigned)(n + s);
    const int loc = atomicAdd(&cell_cnt[c], 1);
    a_cell[s] = c;
    a_loc[s] = loc;
    a_key[s] = key;
    a_orig[s] = orig;
    if (mover) {
      L.dirty[c] = 1;
      L.dirty[old] = 1;
      mv = 1ull;
    }
    const double4 r = L.ref_pos[orig];
    const double dx = x - r.x, dy = y - r.y, dz = z - r.z;
    d2 = dx * dx + dy * dy + dz * dz;
    if (!(d2 <= 1e300)) d2 = 1e300;  // NaN-safe: any invalid state forces a rebuild
  }
  mv = warp_sum_u64(mv);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d2 = fmax(d2, __shfl_down_sync(0xffffffffu, d2, o));
  if ((threadIdx.x & 31) == 0) {
    if (mv) atomicAdd(&cnt->movers, mv);
    if (d2 > 0.0) atomicMax(&cnt->max_disp2, (unsigned long long)__double_as_longlong(d2));
  }
}

// exclusive scan, phase 1: tiles of 4*blockDim elements
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh_warp, int& total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    int w = lane < nw ? sh_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) sh_warp[lane] = w;
  }
  __syncthreads();
  int warp_prefix = warp > 0 ? sh_warp[warp - 1] : 0;
  total = sh_warp[(blockDim.x >> 5) - 1];
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const int* __restrict__ in, int m,
                                                             int* __restrict__ out,
                                                             int* __restrict__ bsum,
                                                             const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  __shared__ int sh[32];
  int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  int t = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < m ? in[base + k] : 0;
    t += v[k];
  }
  int total;
  int ex = block_exclusive_scan(t, sh, total);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < m) out[base + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// phase 2: one block scans the tile sums in chunks (carry kept in a register)
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_bsums(int* __restrict__ bsum, int nb,
                                                             int* __restrict__ out, int m,
                                                             const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  __shared__ int sh[32];
  int carry = 0;
  for (int b0 = 0; b0 < nb; b0 += SCAN_THREADS) {
    int i = b0 + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    int total;
    int ex = block_exclusive_scan(v, sh, total);
    if (i < nb) bsum[i] = ex + carry;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[m] = carry;
}

// phase 3: add tile offsets
__global__ void k_scan_add(int* __restrict__ out, int m, const int* __restrict__ bsum,
                           const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] += bsum[i / SCAN_TILE];
}

__global__ void k_scatter(int n, const int* __restrict__ a_cell, const int* __restrict__ a_loc,
                          const unsigned* __restrict__ a_key, const int* __restrict__ a_orig,
                          const int* __restrict__ cell_start, unsigned* __restrict__ t_key,
                          int* __restrict__ t_orig, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int d = cell_start[a_cell[s]] + a_loc[s];
  t_key[d] = a_key[s];
  t_orig[d] = a_orig[s];
}

// One thread per cell: order the members by key (insertion sort; the keys
// are unique and nearly always already sorted), publish order/cell maps.
__global__ void k_cellsort(int ncell, const int* __restrict__ cell_start,
                           unsigned* __restrict__ t_key, int* __restrict__ t_orig,
                           int* __restrict__ order, int* __restrict__ slot_cell,
                           int* __restrict__ cell_of_orig, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int b = cell_start[c], e = cell_start[c + 1];
  for (int i = b + 1; i < e; i++) {
    unsigned k = t_key[i];
    int o = t_orig[i];
    int j = i - 1;
    while (j >= b && t_key[j] > k) {
      t_key[j + 1] = t_key[j];
      t_orig[j + 1] = t_orig[j];
      j--;
    }
    t_key[j + 1] = k;
    t_orig[j + 1] = o;
  }
  for (int i = b; i < e; i++) {
    int o = t_orig[i];
    order[i] = o;
    slot_cell[i] = c;
    cell_of_orig[o] = c;
  }
}

// Copy the source state into traversal order (the "SoA reorder").
template <bool PP>
__global__ void k_gather(const DevParams* __restrict__ Pp, int n, StateArrays src,
                         const double* __restrict__ radius, const int* __restrict__ comp,
                         SortedArrays S, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int o = S.orig[t];
  double R;
  if (PP) {
    R = radius[o];
  } else {
    int k = comp[o];
    S.comp[t] = k;
    R = Pp->comp_radius[k];
  }
  S.pos[t] = make_double4(src.px[o], src.py[o], src.pz[o], R);
  S.v4[t] = make_double4(src.vx[o], src.vy[o], src.vz[o], src.wx[o]);
  S.w2[t] = make_double2(src.wy[o], src.wz[o]);
}

// ---------------------------------------------------------------------------
// material helpers

template <bool PP>
struct Material;

template <>
struct Material<false> {
  __device__ __forceinline__ static void pair(const DevParams& P, int ca, double, int cb, double,
                                              PairPar& pp) {
    int k = ca * NCM + cb;
    pp.min_dij = P.min_dij[k];
    pp.min_dij_sq = P.min_dij_sq[k];
    pp.kn = P.kn[k];
    pp.yn = P.yn[k];
    pp.kt = P.kt[k];
    pp.yt = P.yt[k];
    pp.mu_sq = P.mu_sq[k];
  }
  __device__ __forceinline__ static double min_dij_sq(const DevParams& P, int ca, double, int cb,
                                                      double) {
    return P.min_dij_sq[ca * NCM + cb];
  }
  __device__ __forceinline__ static void wall(const DevParams& P, int ca, double, int w,
                                              PairPar& pp) {
    int k = ca * NWM + w;
    pp.kn = P.knw[k];
    pp.yn = P.ynw[k];
    pp.kt = P.ktw[k];
    pp.yt = P.ytw[k];
    pp.mu_sq = P.muw_sq[k];
  }
  __device__ __forceinline__ static void self(const DevParams& P, int ca, double, double& inv_m,
                                              double& inv_i, double& eff_m) {
    inv_m = P.comp_inv_mass[ca];
    inv_i = P.comp_inv_inertia[ca];
    eff_m = P.comp_eff_mass[ca];
  }
};

template <>
struct Material<true> {
  __device__ __forceinline__ static double mass(const DevParams& P, double R) {
    return P.pp_mass_coef * ((R * R) * R);
  }
  __device__ __forceinline__ static void pair(const DevParams& P, int, double Ra, int, double Rb,
                                              PairPar& pp) {
    double ma = mass(P, Ra), mb = mass(P, Rb);
    double meff = (ma * mb) / (ma + mb);
    pp.min_dij = Ra + Rb;
    pp.min_dij_sq = pp.min_dij * pp.min_dij;
    pp.kn = P.pp_kn;
    pp.yn = P.pp_gamma_n * sqrt(meff * P.pp_kn);
    pp.kt = P.pp_kt;
    pp.yt = P.pp_gamma_t * sqrt(meff * P.pp_kt);
    pp.mu_sq = P.pp_mu_sq;
  }
  __device__ __forceinline__ static double min_dij_sq(const DevParams&, int, double Ra, int,
                                                      double Rb) {
    double d = Ra + Rb;
    return d * d;
  }
  __device__ __forceinline__ static void wall(const DevParams& P, int, double Ra, int w,
                                              PairPar& pp) {
    double m = mass(P, Ra);
    pp.kn = P.pp_knw[w];
    pp.yn = P.pp_gamma_nw[w] * sqrt(m * P.pp_knw[w]);
    pp.kt = P.pp_ktw[w];
    pp.yt = P.pp_gamma_tw[w] * sqrt(m * P.pp_ktw[w]);
    pp.mu_sq = P.pp_muw_sq[w];
  }
  __device__ __forceinline__ static void self(const DevParams& P, int, double R, double& inv_m,
                                              double& inv_i, double& eff_m) {
    double m = mass(P, R);
    inv_m = 1.0 / m;
    inv_i = 1.0 / ((0.4 * m) * (R * R));
    eff_m = (m * (P.pp_density - P.pp_fluid_density)) / P.pp_density;
  }
};

// ---------------------------------------------------------------------------
// history access

__device__ __forceinline__ int hist_find(const History& H, int owner, int partner) {
  int c = H.cnt[owner];
  const int* k = H.key + (size_t)owner * H.cap;
  for (int r = 0; r < c; r++)
    if (k[r] == partner) return r;
  return -1;
}

__device__ __forceinline__ void hist_read(const History& H, int owner, int r, double ft[3],
                                          double vt[3]) {
  const double2* v = H.val + ((size_t)owner * H.cap + r) * 3;
  double2 a = v[0], b = v[1], c = v[2];
  ft[0] = a.x; ft[1] = a.y; ft[2] = b.x;
  vt[0] = b.y; vt[1] = c.x; vt[2] = c.y;
}

__device__ __forceinline__ void hist_write(const History& H, int owner, int r, int partner,
                                           const double ft[3], const double vt[3]) {
  H.key[(size_t)owner * H.cap + r] = partner;
  double2* v = H.val + ((size_t)owner * H.cap + r) * 3;
  v[0] = make_double2(ft[0], ft[1]);
  v[1] = make_double2(ft[2], vt[0]);
  v[2] = make_double2(vt[1], vt[2]);
}

// ---------------------------------------------------------------------------
// K2+K4: force kernel (FP64, exact order)


// SWEEP = false: particles whose contact-list row is valid; SWEEP = true:
// the (rare) particles whose row overflowed, which sweep the cells here.
template <bool PP, int EPI, bool SWEEP>
__global__ void __launch_bounds__(128, SWEEP ? 1 : 4) k_force_fp64(ForceArgs A) {
  if (A.cnt->abort) return;
  if (SWEEP && A.cnt->list_overflow == 0) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long n_col = 0, n_pc = 0, n_wc = 0;
  int need = 0;
  const int4 meta = s < A.n ? A.cl_meta[s] : make_int4(0, 0, 0, 0);
  if (!SWEEP && s == 0) clear_rebuild_trigger(A);
  if (s < A.n && (meta.x < 0) == SWEEP) {
    const DevParams& P = *A.P;
    const SortedArrays& S = A.S;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int c = S.cell[s];
    const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
    const double4 p4 = S.pos[s];
    const double xp[3] = {p4.x, p4.y, p4.z};
    const double Rp = p4.w;
    const double4 pv4 = S.v4[s];
    const double2 pw2 = S.w2[s];
    const double vp[3] = {pv4.x, pv4.y, pv4.z};
    const double wp[3] = {pv4.w, pw2.x, pw2.y};
    const int orig = S.orig[s];
    const int cp = PP ? 0 : S.comp[s];
    double inv_m, inv_i, eff_m;
    Material<PP>::self(P, cp, Rp, inv_m, inv_i, eff_m);
    const double half_dt = A.half_dt;
    const bool update = A.update != 0;
    int hw_n = 0;
    bool overflow = false;

    double iF[3], iT[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 3; k++) iF[k] = eff_m * P.gravity[k];

    auto record = [&](int partner, const double ft[3], const double vt[3]) {
      if (hw_n < A.Hw.cap)
        hist_write(A.Hw, orig, hw_n, partner, ft, vt);
      else
        overflow = true;
      hw_n++;
    };

    // p is "i", slot t is "j" (src/MForces.f90:199-272)
    auto visit_i = [&](int t) {
      const double4 q4 = S.pos[t];
      double Rij[3] = {q4.x - xp[0], q4.y - xp[1], q4.z - xp[2]};
#pragma unroll
      for (int k = 0; k < 3; k++)
        if (P.pbc[k]) Rij[k] = Rij[k] - P.lbox[k] * fnint(Rij[k] * P.inv_lbox[k]);
      const double DijSq = sumsq3(Rij);
      const int cq = PP ? 0 : S.comp[t];
      const double Delta = Material<PP>::min_dij_sq(P, cp, Rp, cq, q4.w) - DijSq;
      if (Delta > 0.0) {
        PairPar pp;
        Material<PP>::pair(P, cp, Rp, cq, q4.w, pp);
        const int qo = S.orig[t];
        const double4 qv4 = S.v4[t];
        const double2 qw2 = S.w2[t];
        const double vq[3] = {qv4.x, qv4.y, qv4.z};
        const double wq[3] = {qv4.w, qw2.x, qw2.y};
        const int lo = orig < qo ? orig : qo, hi = orig < qo ? qo : orig;
        double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
        int r = hist_find(A.Hr, lo, hi);
        bool contacting = r >= 0;
        if (contacting) hist_read(A.Hr, lo, r, FT0, VT0);
        if (!contacting) n_col++;
        n_pc++;
        ContactOut o;
        pair_contact(Rij, DijSq, Delta, pp, Rp, vp, wp, q4.w, vq, wq, half_dt, contacting, FT0,
                     VT0, o);
#pragma unroll
        for (int k = 0; k < 3; k++) iF[k] = iF[k] + o.FN[k] + o.FT[k];
        double RN[3], tq[3];
#pragma unroll
        for (int k = 0; k < 3; k++) RN[k] = Rp * o.N[k];
        cross3(RN, o.FT, tq);
#pragma unroll
        for (int k = 0; k < 3; k++) iT[k] = iT[k] + tq[k];
        if (update && orig < qo) record(qo, o.FT, o.VT);
      }
    };

    // ---- loop 1: own cell after p, then the half-shell cells in the order
    // of the FirstNeighbour list (reverse of AddAllNeighbours3D insertion)
    walk_as_i<SWEEP>(A, meta, s, orig, c, cx, cy, cz, visit_i);

    // ---- walls (src/MForces.f90:274-314)
    for (int w = 0; w < P.nw; w++) {
      const dem_wall& W = P.walls[w];
      const int wi = orig * P.nw + w;
      bool contacting = A.Hr.wflag[wi] != 0;
      double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
      if (contacting) {
        const double2* v = A.Hr.wval + (size_t)wi * 3;
        double2 a = v[0], b = v[1], d = v[2];
        FT0[0] = a.x; FT0[1] = a.y; FT0[2] = b.x;
        VT0[0] = b.y; VT0[1] = d.x; VT0[2] = d.y;
      }
      double Dij, Nij[3], Qji[3];
      bool ov = false;
      if (W.shape == DEM_WALL_RECTANGLE) ov = overlap_rect(P, W, xp, Rp, Dij, Nij, Qji);
      if (ov) {
        n_wc++;
        const double Delta = Rp * Rp - Dij * Dij;
        const double dn = Dij - Rp;
        double DispN[3], wqv[3], Vij[3], ro[3], cr[3], VijC[3], Rw[3];
#pragma unroll
        for (int k = 0; k < 3; k++) DispN[k] = dn * Nij[k];
        cross3(W.omega, Qji, wqv);
#pragma unroll
        for (int k = 0; k < 3; k++) Vij[k] = W.velocity[k] + wqv[k] - vp[k];
#pragma unroll
        for (int k = 0; k < 3; k++) ro[k] = Rp * wp[k];
        cross3(ro, Nij, cr);
#pragma unroll
        for (int k = 0; k < 3; k++) VijC[k] = Vij[k] - cr[k];
#pragma unroll
        for (int k = 0; k < 3; k++) Rw[k] = W.position[k] + Qji[k] - xp[k];
        PairPar pp;
        Material<PP>::wall(P, cp, Rp, w, pp);
        ContactOut o;
        common_calc(Rw, Nij, DispN, Vij, VijC, Delta, half_dt, contacting, FT0, VT0, pp.kn, pp.yn,
                    pp.kt, pp.yt, pp.mu_sq, o);
#pragma unroll
        for (int k = 0; k < 3; k++) iF[k] = iF[k] + o.FN[k] + o.FT[k];
        double RN[3], tq[3];
#pragma unroll
        for (int k = 0; k < 3; k++) RN[k] = Rp * o.N[k];
        cross3(RN, o.FT, tq);
#pragma unroll
        for (int k = 0; k < 3; k++) iT[k] = iT[k] + tq[k];
        atomicAdd(&A.cnt->wall_fn[w], sqrt(sumsq3(o.FN)));
        if (update) {
          A.Hw.wflag[wi] = 1;
          double2* v = A.Hw.wval + (size_t)wi * 3;
          v[0] = make_double2(o.FT[0], o.FT[1]);
          v[1] = make_double2(o.FT[2], o.VT[0]);
          v[2] = make_double2(o.VT[1], o.VT[2]);
        }
      } else if (update) {
        A.Hw.wflag[wi] = 0;
      }
    }

    // ---- loop 2: p as "j"; contributions in traversal order of the "i"
    // particle, own block (Force(i) = Force(i) + iForce) at p's position.
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    auto visit_j = [&](int t) {
      const double4 q4 = S.pos[t];
      double Rij[3] = {xp[0] - q4.x, xp[1] - q4.y, xp[2] - q4.z};
#pragma unroll
      for (int k = 0; k < 3; k++)
        if (P.pbc[k]) Rij[k] = Rij[k] - P.lbox[k] * fnint(Rij[k] * P.inv_lbox[k]);
      const double DijSq = sumsq3(Rij);
      const int cq = PP ? 0 : S.comp[t];
      const double Delta = Material<PP>::min_dij_sq(P, cq, q4.w, cp, Rp) - DijSq;
      if (Delta > 0.0) {
        PairPar pp;
        Material<PP>::pair(P, cq, q4.w, cp, Rp, pp);
        const int qo = S.orig[t];
        const double4 qv4 = S.v4[t];
        const double2 qw2 = S.w2[t];
        const double vq[3] = {qv4.x, qv4.y, qv4.z};
        const double wq[3] = {qv4.w, qw2.x, qw2.y};
        const int lo = orig < qo ? orig : qo, hi = orig < qo ? qo : orig;
        double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
        int r = hist_find(A.Hr, lo, hi);
        bool contacting = r >= 0;
        if (contacting) hist_read(A.Hr, lo, r, FT0, VT0);
        ContactOut o;
        pair_contact(Rij, DijSq, Delta, pp, q4.w, vq, wq, Rp, vp, wp, half_dt, contacting, FT0,
                     VT0, o);
#pragma unroll
        for (int k = 0; k < 3; k++) F[k] = F[k] - o.FN[k] - o.FT[k];
#pragma unroll
        for (int k = 0; k < 3; k++) T[k] = T[k] + Rp * o.NxFT[k];
        if (update && orig < qo) record(qo, o.FT, o.VT);
      }
    };
    walk_as_j<SWEEP>(A, meta, s, orig, c, cx, cy, cz, visit_j, [&]() {
#pragma unroll
      for (int k = 0; k < 3; k++) F[k] = F[k] + iF[k];
#pragma unroll
      for (int k = 0; k < 3; k++) T[k] = T[k] + iT[k];
    });

    // ---- records of pairs the sweep did not visit are kept as they were
    if (update) {
      const int nold = A.Hr.cnt[orig];
      for (int r = 0; r < nold; r++) {
        const int q2 = A.Hr.key[(size_t)orig * A.Hr.cap + r];
        if (!cells_adjacent(P, c, A.cell_of_orig[q2])) {
          double ft[3], vt[3];
          hist_read(A.Hr, orig, r, ft, vt);
          record(q2, ft, vt);
        }
      }
      A.Hw.cnt[orig] = hw_n < A.Hw.cap ? hw_n : A.Hw.cap;
      if (overflow) {
        // the pass is re-run with larger tables; stop everything after it
        atomicExch(&A.cnt->overflow, 1);
        atomicCAS(&A.cnt->abort_tag, 0, A.tag + 1);
        atomicExch(&A.cnt->abort, 1);
      }
      need = hw_n;
    }

    // ---- a = F/m, alpha = T/I (src/MForces.f90:330-333) + epilogue
    double acc[3], alp[3];
#pragma unroll
    for (int k = 0; k < 3; k++) acc[k] = F[k] * inv_m;
#pragma unroll
    for (int k = 0; k < 3; k++) alp[k] = T[k] * inv_i;

    if (EPI == EPI_STORE) {
      A.tgt.ax[orig] = acc[0]; A.tgt.ay[orig] = acc[1]; A.tgt.az[orig] = acc[2];
      A.tgt.lx[orig] = alp[0]; A.tgt.ly[orig] = alp[1]; A.tgt.lz[orig] = alp[2];
    } else if (EPI == EPI_PREDICT) {
      // src/MDEM.f90:296-331: AB predictor from x(t), v(t), w(t) (the values
      // this pass gathered) and the ring, then store (v,a,alpha)(t).
      const StateArrays& Q = A.part;
      const StateArrays& R = A.pred;
      Q.ax[orig] = acc[0]; Q.ay[orig] = acc[1]; Q.az[orig] = acc[2];
      Q.lx[orig] = alp[0]; Q.ly[orig] = alp[1]; Q.lz[orig] = alp[2];
      double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
      const size_t n = (size_t)A.n;
      for (int k = 0; k < P.nprev; k++) {
        const double ABk = P.ab[k];
        const double* rg = A.ring + (size_t)A.rm.phys[k] * 9 * n + orig;
#pragma unroll
        for (int d = 0; d < 3; d++) sv[d] = sv[d] + ABk * rg[d * n];
#pragma unroll
        for (int d = 0; d < 3; d++) sa[d] = sa[d] + ABk * rg[(3 + d) * n];
#pragma unroll
        for (int d = 0; d < 3; d++) sl[d] = sl[d] + ABk * rg[(6 + d) * n];
      }
      double xr[3], vr[3], wr[3];
#pragma unroll
      for (int d = 0; d < 3; d++) xr[d] = xp[d] + P.ab0 * vp[d] + sv[d];
#pragma unroll
      for (int d = 0; d < 3; d++) vr[d] = vp[d] + P.ab0 * acc[d] + sa[d];
#pragma unroll
      for (int d = 0; d < 3; d++) wr[d] = wp[d] + P.ab0 * alp[d] + sl[d];
#pragma unroll
      for (int d = 0; d < 3; d++)
        if (P.pbc[d]) xr[d] = xr[d] - P.lbox[d] * fnint(xr[d] * P.inv_lbox[d]);
      R.px[orig] = xr[0]; R.py[orig] = xr[1]; R.pz[orig] = xr[2];
      R.vx[orig] = vr[0]; R.vy[orig] = vr[1]; R.vz[orig] = vr[2];
      R.wx[orig] = wr[0]; R.wy[orig] = wr[1]; R.wz[orig] = wr[2];
      if (P.nprev > 0) {
        double* rg = A.ring + (size_t)A.rm.phys[P.nprev] * 9 * n + orig;
#pragma unroll
        for (int d = 0; d < 3; d++) rg[d * n] = vp[d];
#pragma unroll
        for (int d = 0; d < 3; d++) rg[(3 + d) * n] = acc[d];
#pragma unroll
        for (int d = 0; d < 3; d++) rg[(6 + d) * n] = alp[d];
      }
    } else {  // EPI_CORRECT, src/MDEM.f90:340-367
      const StateArrays& Q = A.part;
      const StateArrays& R = A.pred;
      R.ax[orig] = acc[0]; R.ay[orig] = acc[1]; R.az[orig] = acc[2];
      R.lx[orig] = alp[0]; R.ly[orig] = alp[1]; R.lz[orig] = alp[2];
      double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
      const size_t n = (size_t)A.n;
      for (int k = 0; k < P.nprev; k++) {
        const double AMk = P.am[k];
        const double* rg = A.ring + (size_t)A.rm.phys[k] * 9 * n + orig;
#pragma unroll
        for (int d = 0; d < 3; d++) sv[d] = sv[d] + AMk * rg[d * n];
#pragma unroll
        for (int d = 0; d < 3; d++) sa[d] = sa[d] + AMk * rg[(3 + d) * n];
#pragma unroll
        for (int d = 0; d < 3; d++) sl[d] = sl[d] + AMk * rg[(6 + d) * n];
      }
      double x[3] = {Q.px[orig], Q.py[orig], Q.pz[orig]};
      double v[3] = {Q.vx[orig], Q.vy[orig], Q.vz[orig]};
      double w[3] = {Q.wx[orig], Q.wy[orig], Q.wz[orig]};
#pragma unroll
      for (int d = 0; d < 3; d++) x[d] = x[d] + P.am0 * vp[d] + sv[d];
#pragma unroll
      for (int d = 0; d < 3; d++) v[d] = v[d] + P.am0 * acc[d] + sa[d];
#pragma unroll
      for (int d = 0; d < 3; d++) w[d] = w[d] + P.am0 * alp[d] + sl[d];
#pragma unroll
      for (int d = 0; d < 3; d++)
        if (P.pbc[d]) x[d] = x[d] - P.lbox[d] * fnint(x[d] * P.inv_lbox[d]);
      Q.px[orig] = x[0]; Q.py[orig] = x[1]; Q.pz[orig] = x[2];
      Q.vx[orig] = v[0]; Q.vy[orig] = v[1]; Q.vz[orig] = v[2];
      Q.wx[orig] = w[0]; Q.wy[orig] = w[1]; Q.wz[orig] = w[2];
      bool out = false;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double h = 0.5 * P.lbox[d];
        out = out || (x[d] > h) || (x[d] < -h);
      }
      if (out) atomicAdd(&A.cnt->escaped, 1ull);
    }
  }
  n_col = warp_sum_u64(n_col);
  n_pc = warp_sum_u64(n_pc);
  n_wc = warp_sum_u64(n_wc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) need = max(need, __shfl_down_sync(0xffffffffu, need, o));
  if ((threadIdx.x & 31) == 0) {
    if (need) atomicMax(&A.cnt->need_capacity, need);
    if (n_col) atomicAdd(A.update ? &A.cnt->ncol_pending : &A.cnt->ncol, n_col);
    if (n_pc) atomicAdd(&A.cnt->pair_contacts, n_pc);
    if (n_wc) atomicAdd(&A.cnt->wall_contacts, n_wc);
  }
}

// ---------------------------------------------------------------------------
// small per-particle kernels (original index order)

// K2 screening: candidate lists.  For every particle whose row must be
// (re)built -- all particles on a full rebuild, else those whose 27-cell
// neighbourhood gained or lost a particle in this pass, and rows that
// overflowed -- sweep the cells exactly as ComputeAccelerations does
// (src/MForces.f90:173-272) and keep, in sweep order, the particles within
// MinDij + skin.  The force kernels apply the exact FP64 overlap test to these
// candidates, so contact sets, orientation and order stay the reference's.
// Every thread also publishes its particle's slot for the orig -> slot map.
struct ScreenRange {
  int b, e, code;  // code: bit 0..5 image (2 bits per axis, biased by 1), bit 6: p is "j"
};

__device__ __forceinline__ int range_code(int wx, int wy, int wz, bool p_is_j) {
  return (wx + 1) | ((wy + 1) << 2) | ((wz + 1) << 4) | (p_is_j ? 64 : 0);
}

template <bool PP>
__global__ void __launch_bounds__(256, 4) k_screen(const DevParams* __restrict__ Pp, int n,
                                                   const double4* __restrict__ pos,
                                                   const int* __restrict__ comp,
                                                   const int* __restrict__ slot_cell,
                                                   const int* __restrict__ order,
                                                   const int* __restrict__ cs, ContactLists L,
                                                   Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const DevParams& P = *Pp;
  const int orig = order[s];
  L.slot_of_orig[orig] = s;
  const int c = slot_cell[s];
  const bool full = rebuild_due(P, cnt);
  if (!full && !L.repair[c] && L.meta[orig].x >= 0) return;

  const int nx = P.nx, ny = P.ny;
  const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
  // ---- the ranges, in sweep order: loop 1, then loop 2
  ScreenRange R[29];
  int nr = 0, own_j = -1;
  sweep_cells_as_i(P, cs, s, c, cx, cy, cz, [&](int b, int e, int wx, int wy, int wz) {
    R[nr++] = ScreenRange{b, e, range_code(wx, wy, wz, false)};
  });
  const int nr1 = nr;
  sweep_cells_as_j(
      P, cs, s, c, cx, cy, cz,
      [&](int b, int e, int wx, int wy, int wz) {
        R[nr++] = ScreenRange{b, e, range_code(wx, wy, wz, true)};
      },
      [&]() { own_j = nr - 1; });

  // ---- one loop over all candidates
  const double4 p4 = pos[s];
  if (full) L.ref_pos[orig] = p4;
  const int cp = PP ? 0 : comp[s];
  const double skin = P.vl_skin;
  const double maxd = sqrt(P.max_min_dij_sq) + skin;
  const double maxsq = maxd * maxd;
  int* out = L.slot + (size_t)orig * KC;
  int m = 0, n1 = 0, n2b = 0;
  for (int r = 0; r < nr; r++) {
    const ScreenRange rr = R[r];
    const bool pj = rr.code & 64;
    const int sg = pj ? -1 : 1;
    const int nxi = sg * -(((rr.code) & 3) - 1);
    const int nyi = sg * -(((rr.code >> 2) & 3) - 1);
    const int nzi = sg * -(((rr.code >> 4) & 3) - 1);
    for (int t = rr.b; t < rr.e; t++) {
      const double4 q4 = pos[t];
      double Rij[3];
      Rij[0] = pj ? p4.x - q4.x : q4.x - p4.x;
      Rij[0] = min_image(Rij[0], P.pbc[0], P.lbox[0], P.inv_lbox[0], nxi);
      if (Rij[0] * Rij[0] >= maxsq) continue;
      Rij[1] = pj ? p4.y - q4.y : q4.y - p4.y;
      Rij[1] = min_image(Rij[1], P.pbc[1], P.lbox[1], P.inv_lbox[1], nyi);
      Rij[2] = pj ? p4.z - q4.z : q4.z - p4.z;
      Rij[2] = min_image(Rij[2], P.pbc[2], P.lbox[2], P.inv_lbox[2], nzi);
      const double DijSq = sumsq3(Rij);
      const int cq = PP ? 0 : comp[t];
      // candidates: within MinDij + skin (a superset of the exact overlaps)
      double md = PP ? p4.w + q4.w : sqrt(Material<PP>::min_dij_sq(P, cp, p4.w, cq, q4.w));
      md = md + skin;
      if (md * md - DijSq > 0.0) {
        if (m < KC) out[m] = order[t];
        m++;
      }
    }
    if (r == nr1 - 1) n1 = m;
    if (r == own_j) n2b = m - n1;
  }
  L.meta[orig] = m <= KC ? make_int4(n1, n2b, m - n1 - n2b, 0) : make_int4(-1, 0, 0, 0);
  if (m > KC) atomicAdd(&cnt->list_overflow, 1);
}

// This pass's exact contact rows: the candidates of every particle that
// pass the overlap test DeltaDijSq > 0 of the force kernels (same operations,
// src/MForces.f90:209-224), in candidate order, as traversal slots.  A light
// kernel, so that the heavy contact arithmetic only meets real contacts.
template <bool PP>
__global__ void __launch_bounds__(256) k_filter(const DevParams* __restrict__ Pp, int n,
                                                const double4* __restrict__ pos,
                                                const int* __restrict__ comp,
                                                const int* __restrict__ order, ContactLists L,
                                                const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const DevParams& P = *Pp;
  const int orig = order[s];
  const int4 meta = L.meta[orig];
  if (meta.x < 0) {
    L.xmeta[s] = meta;  // overflowed row: the force kernel sweeps the cells
    return;
  }
  const double4 p4 = pos[s];
  const int cp = PP ? 0 : comp[s];
  const int* in = L.slot + (size_t)orig * KC;
  int* out = L.xslot + (size_t)s * KC;
  const int total = meta.x + meta.y + meta.z;
  int m = 0, n1 = 0, n2b = 0;
  for (int k = 0; k < total; k++) {
    const int t = L.slot_of_orig[in[k]];
    const double4 q4 = pos[t];
    const bool pj = k >= meta.x;  // loop 2: p is "j", Rij = xp - xq
    double Rij[3] = {pj ? p4.x - q4.x : q4.x - p4.x, pj ? p4.y - q4.y : q4.y - p4.y,
                     pj ? p4.z - q4.z : q4.z - p4.z};
#pragma unroll
    for (int d = 0; d < 3; d++)
      if (P.pbc[d]) Rij[d] = Rij[d] - P.lbox[d] * fnint(Rij[d] * P.inv_lbox[d]);
    const double DijSq = sumsq3(Rij);
    const int cq = PP ? 0 : comp[t];
    const double Delta = pj ? Material<PP>::min_dij_sq(P, cq, q4.w, cp, p4.w) - DijSq
                            : Material<PP>::min_dij_sq(P, cp, p4.w, cq, q4.w) - DijSq;
    if (Delta > 0.0) out[m++] = t;
    if (k == meta.x - 1) n1 = m;
    if (k == meta.x + meta.y - 1) n2b = m - n1;
  }
  if (meta.x == 0) n1 = 0;
  if (meta.y == 0) n2b = 0;
  L.xmeta[s] = make_int4(n1, n2b, m - n1 - n2b, 0);
}

// A particle entered or left each dirty cell: the rows of every particle in
// its 27-cell neighbourhood are rebuilt in this pass.
__global__ void k_mark_repair(const DevParams* __restrict__ Pp, ContactLists L,
                              const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const DevParams& P = *Pp;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.ncell || !L.dirty[c]) return;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
  int xi, xf, yi, yf, zi, zf;
  axis_range(cx, nx, P.pbc[0], xi, xf);
  axis_range(cy, ny, P.pbc[1], yi, yf);
  axis_range(cz, nz, P.pbc[2], zi, zf);
  for (int kz = zi; kz <= zf; kz++)
    for (int ky = yi; ky <= yf; ky++)
      for (int kx = xi; kx <= xf; kx++) {
        const int jx = axis_wrap(cx + kx, nx, P.pbc[0]);
        const int jy = axis_wrap(cy + ky, ny, P.pbc[1]);
        const int jz = axis_wrap(cz + kz, nz, P.pbc[2]);
        L.repair[jx + nx * (jy + ny * jz)] = 1;
      }
}

// AB predictor (src/MDEM.f90:297-331) as a streaming pass over particles in
// index order: Predicted = x(t) + AB0*v + sum_k AB(k)*Previous(ipc(k)), PBC
// wrap, then (v, a, alpha)(t) into the spare ring slot (the slot the
// reference's cshift makes ipc(1)).
__global__ void __launch_bounds__(256) k_predict(const DevParams* __restrict__ Pp, int n,
                                                 StateArrays Q, StateArrays R,
                                                 double* __restrict__ ring, RingMap rm,
                                                 const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevParams& P = *Pp;
  const size_t N = (size_t)n;
  const double x[3] = {Q.px[i], Q.py[i], Q.pz[i]};
  const double v[3] = {Q.vx[i], Q.vy[i], Q.vz[i]};
  const double w[3] = {Q.wx[i], Q.wy[i], Q.wz[i]};
  const double a[3] = {Q.ax[i], Q.ay[i], Q.az[i]};
  const double l[3] = {Q.lx[i], Q.ly[i], Q.lz[i]};
  double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < P.nprev; k++) {
    const double ABk = P.ab[k];
    const double* rg = ring + (size_t)rm.phys[k] * 9 * N + i;
#pragma unroll
    for (int d = 0; d < 3; d++) sv[d] = sv[d] + ABk * rg[d * N];
#pragma unroll
    for (int d = 0; d < 3; d++) sa[d] = sa[d] + ABk * rg[(3 + d) * N];
#pragma unroll
    for (int d = 0; d < 3; d++) sl[d] = sl[d] + ABk * rg[(6 + d) * N];
  }
  double xr[3], vr[3], wr[3];
#pragma unroll
  for (int d = 0; d < 3; d++) xr[d] = x[d] + P.ab0 * v[d] + sv[d];
#pragma unroll
  for (int d = 0; d < 3; d++) vr[d] = v[d] + P.ab0 * a[d] + sa[d];
#pragma unroll
  for (int d = 0; d < 3; d++) wr[d] = w[d] + P.ab0 * l[d] + sl[d];
#pragma unroll
  for (int d = 0; d < 3; d++)
    if (P.pbc[d]) xr[d] = xr[d] - P.lbox[d] * fnint(xr[d] * P.inv_lbox[d]);
  R.px[i] = xr[0]; R.py[i] = xr[1]; R.pz[i] = xr[2];
  R.vx[i] = vr[0]; R.vy[i] = vr[1]; R.vz[i] = vr[2];
  R.wx[i] = wr[0]; R.wy[i] = wr[1]; R.wz[i] = wr[2];
  if (P.nprev > 0) {
    double* rg = ring + (size_t)rm.phys[P.nprev] * 9 * N + i;
#pragma unroll
    for (int d = 0; d < 3; d++) rg[d * N] = v[d];
#pragma unroll
    for (int d = 0; d < 3; d++) rg[(3 + d) * N] = a[d];
#pragma unroll
    for (int d = 0; d < 3; d++) rg[(6 + d) * N] = l[d];
  }
}

// AM corrector (src/MDEM.f90:340-367) as a streaming pass: x = x + AM0*v~ +
// sum_k AM(k)*Previous(ipc(k)) (ipc after the shift), likewise v and omega,
// PBC wrap; counts the particles that left the box (src/MDEM.f90:624-625).
__global__ void __launch_bounds__(256) k_correct(const DevParams* __restrict__ Pp, int n,
                                                 StateArrays Q, StateArrays R,
                                                 const double* __restrict__ ring, RingMap rm,
                                                 Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool out = false;
  if (i < n) {
    const DevParams& P = *Pp;
    const size_t N = (size_t)n;
    double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < P.nprev; k++) {
      const double AMk = P.am[k];
      const double* rg = ring + (size_t)rm.phys[k] * 9 * N + i;
#pragma unroll
      for (int d = 0; d < 3; d++) sv[d] = sv[d] + AMk * rg[d * N];
#pragma unroll
      for (int d = 0; d < 3; d++) sa[d] = sa[d] + AMk * rg[(3 + d) * N];
#pragma unroll
      for (int d = 0; d < 3; d++) sl[d] = sl[d] + AMk * rg[(6 + d) * N];
    }
    const double vp[3] = {R.vx[i], R.vy[i], R.vz[i]};
    const double ap[3] = {R.ax[i], R.ay[i], R.az[i]};
    const double lp[3] = {R.lx[i], R.ly[i], R.lz[i]};
    double x[3] = {Q.px[i], Q.py[i], Q.pz[i]};
    double v[3] = {Q.vx[i], Q.vy[i], Q.vz[i]};
    double w[3] = {Q.wx[i], Q.wy[i], Q.wz[i]};
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = x[d] + P.am0 * vp[d] + sv[d];
#pragma unroll
    for (int d = 0; d < 3; d++) v[d] = v[d] + P.am0 * ap[d] + sa[d];
#pragma unroll
    for (int d = 0; d < 3; d++) w[d] = w[d] + P.am0 * lp[d] + sl[d];
#pragma unroll
    for (int d = 0; d < 3; d++)
      if (P.pbc[d]) x[d] = x[d] - P.lbox[d] * fnint(x[d] * P.inv_lbox[d]);
    Q.px[i] = x[0]; Q.py[i] = x[1]; Q.pz[i] = x[2];
    Q.vx[i] = v[0]; Q.vy[i] = v[1]; Q.vz[i] = v[2];
    Q.wx[i] = w[0]; Q.wy[i] = w[1]; Q.wz[i] = w[2];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double h = 0.5 * P.lbox[d];
      out = out || (x[d] > h) || (x[d] < -h);
    }
  }
  const unsigned long long e = warp_sum_u64(out ? 1ull : 0ull);
  if ((threadIdx.x & 31) == 0 && e) atomicAdd(&cnt->escaped, e);
}

// ring store of MoveParticlesEuler (src/MDEM.f90:266-271): (v,a,alpha) -> slot
__global__ void k_ring_store(int n, StateArrays Q, double* __restrict__ ring, int slot,
                             const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* rg = ring + (size_t)slot * 9 * n + i;
  rg[0 * (size_t)n] = Q.vx[i]; rg[1 * (size_t)n] = Q.vy[i]; rg[2 * (size_t)n] = Q.vz[i];
  rg[3 * (size_t)n] = Q.ax[i]; rg[4 * (size_t)n] = Q.ay[i]; rg[5 * (size_t)n] = Q.az[i];
  rg[6 * (size_t)n] = Q.lx[i]; rg[7 * (size_t)n] = Q.ly[i]; rg[8 * (size_t)n] = Q.lz[i];
}

// explicit Euler update (src/MDEM.f90:240-252)
__global__ void k_euler_update(int n, StateArrays Q, double dt, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double h2 = 0.5 * (dt * dt);
  Q.px[i] = Q.px[i] + Q.vx[i] * dt + Q.ax[i] * h2;
  Q.py[i] = Q.py[i] + Q.vy[i] * dt + Q.ay[i] * h2;
  Q.pz[i] = Q.pz[i] + Q.vz[i] * dt + Q.az[i] * h2;
  Q.vx[i] = Q.vx[i] + Q.ax[i] * dt;
  Q.vy[i] = Q.vy[i] + Q.ay[i] * dt;
  Q.vz[i] = Q.vz[i] + Q.az[i] * dt;
  Q.wx[i] = Q.wx[i] + Q.lx[i] * dt;
  Q.wy[i] = Q.wy[i] + Q.ly[i] * dt;
  Q.wz[i] = Q.wz[i] + Q.lz[i] * dt;
}

// ApplyPeriodicBoundaryConditions (src/MDEM.f90:373-388)
__global__ void k_apply_pbc(const DevParams* __restrict__ Pp, int n, StateArrays Q,
                            const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevParams& P = *Pp;
  double* p[3] = {Q.px, Q.py, Q.pz};
#pragma unroll
  for (int d = 0; d < 3; d++)
    if (P.pbc[d]) {
      double x = p[d][i];
      p[d][i] = x - P.lbox[d] * fnint(x * P.inv_lbox[d]);
    }
}

// rows of 3 doubles (host layout) <-> SoA state arrays
__global__ void k_rows_to_soa(int n, const double* __restrict__ rows, double* __restrict__ x,
                              double* __restrict__ y, double* __restrict__ z) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = rows[3 * (size_t)i];
  y[i] = rows[3 * (size_t)i + 1];
  z[i] = rows[3 * (size_t)i + 2];
}
__global__ void k_soa_to_rows(int n, const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, double* __restrict__ rows) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rows[3 * (size_t)i] = x[i];
  rows[3 * (size_t)i + 1] = y[i];
  rows[3 * (size_t)i + 2] = z[i];
}

// copy history records into a table with a larger capacity
__global__ void k_hist_regrow(int n, History src, History dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = src.cnt[i];
  dst.cnt[i] = c;
  for (int r = 0; r < c; r++) {
    dst.key[(size_t)i * dst.cap + r] = src.key[(size_t)i * src.cap + r];
    for (int k = 0; k < 3; k++)
      dst.val[((size_t)i * dst.cap + r) * 3 + k] = src.val[((size_t)i * src.cap + r) * 3 + k];
  }
}

// observables: per-block partial sums (fixed order), reduced on the host
template <bool PP>
__global__ void k_observables(const DevParams* __restrict__ Pp, int n, StateArrays Q,
                              const double* __restrict__ radius, const int* __restrict__ comp,
                              double* __restrict__ partial /* [grid][8] */) {
  const DevParams& P = *Pp;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double R, m, I;
    if (PP) {
      R = radius[i];
      m = P.pp_mass_coef * ((R * R) * R);
    } else {
      int k = comp[i];
      R = P.comp_radius[k];
      m = 1.0 / P.comp_inv_mass[k];
    }
    I = (0.4 * m) * (R * R);
    if (!PP) I = 1.0 / P.comp_inv_inertia[comp[i]];
    double v[3] = {Q.vx[i], Q.vy[i], Q.vz[i]};
    double w[3] = {Q.wx[i], Q.wy[i], Q.wz[i]};
    double x[3] = {Q.px[i], Q.py[i], Q.pz[i]};
    acc[0] += m * sumsq3(v) + I * sumsq3(w);
    acc[1] -= m * dot3(x, P.gravity);
    acc[2] += 4.0 / 3.0 * 3.14159265358979323846 * R * R * R;
    acc[3] += m * v[0];
    acc[4] += m * v[1];
    acc[5] += m * v[2];
  }
  __shared__ double sh[8][256];
  for (int k = 0; k < 8; k++) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 8; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 8; k++) partial[blockIdx.x * 8 + k] = sh[k][0];
}

}  // namespace dem
