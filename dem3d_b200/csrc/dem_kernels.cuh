// dem_kernels.cuh -- sm_100a kernels of the DEM step (FP64 pass kernel and
// the precision-independent cell-list, candidate-row and integrator kernels).
//
// K1  cell lists: the reference's linked lists (src/MCells.f90), kept in its
//     order.  The initial distribution (DistributeParticles3D) is a counting
//     sort by cell with every cell in decreasing index, then linked.  Each
//     later pass relinks only the cells that gained or lost a particle
//     (RedistributeParticles3D, src/MCells.f90:607-643: the movers are
//     prepended in increasing index order, so a cell lists the particles that
//     entered it in this pass, highest index first, then the ones that
//     stayed, in their previous order).
// K2  candidate rows: for every particle, the partners within MinDij + skin
//     in the order the reference's sweep meets them (src/MForces.f90:173-272),
//     rebuilt by one warp per particle around relinked cells, and for every
//     particle when the accumulated displacement bound reaches 0.4 skin.
// K2+K4 pass kernel: one thread per particle (original index order) applies
//     the reference's overlap test to its candidates, evaluates every contact
//     in the reference's orientation ("i" = the particle visited first) and
//     adds the contributions in the order of the sweep, so that the forces
//     are bit-identical to ComputeAccelerations (src/MForces.f90:145-335).
//     The AB predictor / AM corrector (src/MDEM.f90:296-365) run in its
//     epilogue, which also hashes the next position into its cell.
// K3  history: records owned by imin are double-buffered; a pass that updates
//     them writes a fresh table (new/updated contacts + records of pairs that
//     the sweep did not visit, as the reference keeps those untouched).
#pragma once
#include "dem_pass.cuh"

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
__global__ void k_assign(const DevParams* __restrict__ PT, const int* __restrict__ sysid, int n,
                         int initial, const double* __restrict__ px,
                         const double* __restrict__ py, const double* __restrict__ pz,
                         const int* __restrict__ order,
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
    int orig = initial ? s : order[s];
    const DevParams& P = sys_params(PT, sysid, orig);
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

__device__ __forceinline__ void hist_read(const History& H, int owner, int r, double ft[3],
                                          double vt[3]) {
  const double2* v = H.val + hslot(H, owner, r) * 3;
  double2 a = v[0], b = v[1], c = v[2];
  ft[0] = a.x; ft[1] = a.y; ft[2] = b.x;
  vt[0] = b.y; vt[1] = c.x; vt[2] = c.y;
}

__device__ __forceinline__ void hist_write(const History& H, int owner, int r, int partner,
                                           const double ft[3], const double vt[3]) {
  H.key[hslot(H, owner, r)] = partner;
  double2* v = H.val + hslot(H, owner, r) * 3;
  v[0] = make_double2(ft[0], ft[1]);
  v[1] = make_double2(ft[2], vt[0]);
  v[2] = make_double2(vt[1], vt[2]);
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
__global__ void k_apply_pbc(const DevParams* __restrict__ PT, const int* __restrict__ sysid,
                            int n, StateArrays Q, const Counters* __restrict__ cnt) {
  if (cnt->abort) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevParams& P = sys_params(PT, sysid, i);
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
    dst.key[hslot(dst, i, r)] = src.key[hslot(src, i, r)];
    for (int k = 0; k < 3; k++) dst.val[hslot(dst, i, r) * 3 + k] = src.val[hslot(src, i, r) * 3 + k];
  }
}

// Canonical tables: every pair record moved to the table of its smaller
// index (the reference's owner, imin), as particle removal expects them
// (src/MContacts.f90:173-252, 579-633).  dst counts start at zero; the
// records of a table come in no particular order (lookups go by partner).
// status[0]: a table would overflow, status[1]: largest count asked for.
// FP32 record values of the mixed mode move with them (sa.. -> da.., or
// null in FP64 mode).
__global__ void k_hist_canon(int n, History src, History dst, const float4* __restrict__ sa,
                             const float4* __restrict__ sb, const float* __restrict__ sc,
                             float4* __restrict__ da, float4* __restrict__ db,
                             float* __restrict__ dc, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = src.cnt[i];
  for (int r = 0; r < c; r++) {
    const size_t from = hslot(src, i, r);
    const int q = src.key[from];
    const bool move = q >= 0 && q < i;
    const int o = move ? q : i;
    const int s = atomicAdd(&dst.cnt[o], 1);
    if (s >= dst.cap) {
      atomicExch(&status[0], 1);
      atomicMax(&status[1], s + 1);
      continue;
    }
    const size_t to = hslot(dst, o, s);
    dst.key[to] = move ? i : q;
    if (sa) {
      da[to] = sa[from];
      db[to] = sb[from];
      dc[to] = sc[from];
    } else {
#pragma unroll
      for (int k = 0; k < 3; k++) dst.val[to * 3 + k] = src.val[from * 3 + k];
    }
  }
}

// observables: per-block partial sums (fixed order), reduced on the host
template <bool PP>
__global__ void k_observables(const DevParams* __restrict__ PT, const int* __restrict__ sysid,
                              int n, StateArrays Q, const double* __restrict__ radius,
                              const int* __restrict__ comp,
                              double* __restrict__ partial /* [grid][8] */) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const DevParams& P = sys_params(PT, sysid, i);
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


// ---------------------------------------------------------------------------
// K1: linked cell lists

// DistributeParticles3D (src/MCells.f90:542-564): every particle is prepended
// to its cell in index order; the counting sort gives each cell in
// decreasing index, which is linked here.  head[] starts at -1.
__global__ void k_link_init(int n, const int* __restrict__ order,
                            const int* __restrict__ slot_cell, const int* __restrict__ cell_start,
                            int* __restrict__ head, int* __restrict__ next,
                            int* __restrict__ cell_of) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int p = order[s], c = slot_cell[s];
  next[p] = s + 1 < cell_start[c + 1] ? order[s + 1] : -1;
  if (s == cell_start[c]) head[c] = p;
  cell_of[p] = c;
}

// Forget a prepared cell transition (arrival lists and dirty flags of
// dirty list `par`); the count itself is reset by the host afterwards.
__global__ void k_discard(CellLists L, int par, const Counters* __restrict__ cnt) {
  const int m = cnt->n_dirty[par];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int c = L.dlist[par][i];
    L.arr_head[c] = -1;
    L.dflag[c] = 0;
  }
}

// Copies of a state for the pass kernel (positions + radius, velocities) by
// original index, the cell of every particle under the next assignment and
// the displacement from the last pass's positions `Xlast` (NULL: none).
template <class V4, class W2>
__global__ void __launch_bounds__(256) k_prepare(const DevParams* __restrict__ PT,
                                                 const int* __restrict__ sysid, int n,
                                                 StateArrays src, const double* __restrict__ radius,
                                                 double4* X, V4* __restrict__ v4,
                                                 W2* __restrict__ w2, const double4* Xlast,
                                                 const int* __restrict__ cell_cur, CellLists L,
                                                 int par, Counters* cnt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (p < n) {
    const DevParams& P = sys_params(PT, sysid, p);
    const double x[3] = {src.px[p], src.py[p], src.pz[p]};
    if (Xlast) {
      const double4 o = Xlast[p];
      const double y[3] = {o.x, o.y, o.z};
      d2 = disp2(P, x, y);
      if (!(d2 <= 1e300)) d2 = 1e300;  // a non-finite state forces a full rebuild
    }
    if (!isfinite(x[0] + x[1] + x[2])) {
      atomicExch(&cnt->nonfinite, 1);
      atomicExch(&cnt->abort, 1);
    }
    X[p] = make_double4(x[0], x[1], x[2], radius[p]);
    v4[p] = mk_v4<V4>(src.vx[p], src.vy[p], src.vz[p], src.wx[p]);
    w2[p] = mk_w2<W2>(src.wy[p], src.wz[p]);
    L.mflag[p] = 0;
    note_cell(L, cnt, par, p, cell_cur[p], current_cell(P, x[0], x[1], x[2]));
  }
  publish_disp(cnt, d2);
}

// Relink (RedistributeParticles3D's list updates, src/MCells.f90:607-643):
// one thread per dirty cell of list `par` drops the particles that left it
// (TransferParticle's unlink, :747-774) and prepends its arrivals in
// decreasing index (AddParticle, :684-698, applied in increasing index
// order), then marks its 27-cell neighbourhood for candidate-row repair.
// The walk over the old list follows a leaver's successor saved when it
// moved (mnext), so no thread reads a link that another thread rewrites.
// Thread 0 also closes the previous pass's bookkeeping and decides whether
// this pass rebuilds every candidate row.
__global__ void k_relink(const DevParams* __restrict__ PT, const int* __restrict__ cellsys,
                         CellLists L, int par, int n, int update, int stop_tag, Counters* cnt) {
  if (cnt->abort) return;
  // inside a captured chunk, particles that left the box in the last step
  // stop the chunk before this step (the host runs UpdateParticleList); the
  // count is final here (written by the previous kernel), so every block
  // takes the same branch
  if (stop_tag >= 0 && cnt->escaped != 0ull) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      cnt->escape_stop = 1;
      set_abort(cnt, stop_tag);
    }
    return;
  }
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    const DevParams& P = PT[0];  // the integrator settings are shared
    cnt->n_repair = 0;
    cnt->n_dirty[par ^ 1] = 0;
    cnt->movers = cnt->movers_pending;
    cnt->movers_pending = 0ull;
    if (cnt->ncol_pending) {  // the previous history-updating pass completed
      cnt->ncol += cnt->ncol_pending;
      cnt->ncol_pending = 0ull;
    }
    cnt->pair_contacts = 0ull;
    cnt->wall_contacts = 0ull;
    if (update) {
      cnt->need_capacity = 0;
      cnt->need_in = 0;
    }
    else cnt->escaped = 0ull;  // escapes are counted by the current step's corrector
    const double d = (double)__uint_as_float(cnt->disp_max);
    cnt->disp_max = 0u;
    const double acc = cnt->disp_acc + d;
    const int full = cnt->force_full != 0 || !(acc <= P.vl_thr);
    cnt->full_due = full;
    cnt->disp_acc = full ? 0.0 : acc;
    if (full) cnt->force_full = 0;
  }
  const int m = cnt->n_dirty[par];
  const int* __restrict__ cell_new = L.cell[par];
  for (int i = tid; i < m; i += gridDim.x * blockDim.x) {
    const int c = L.dlist[par][i];
    // 1. unlink the leavers
    int prev = -1, first = -1, q = L.head[c];
    int guard = 0;
    while (q != -1) {
      if (++guard > n) {
        atomicExch(&cnt->list_error, 1);
        atomicExch(&cnt->abort, 1);
        return;
      }
      const bool stays = cell_new[q] == c;
      const int nq = stays ? L.next[q] : L.mnext[q];
      if (stays) {
        if (prev == -1) first = q;
        else L.next[prev] = q;
        prev = q;
      }
      q = nq;
    }
    if (prev != -1) L.next[prev] = -1;
    // 2. prepend the arrivals, highest index first
    int sh = -1, tail = -1, a = L.arr_head[c];
    guard = 0;
    while (a != -1) {
      if (++guard > n) {
        atomicExch(&cnt->list_error, 1);
        atomicExch(&cnt->abort, 1);
        return;
      }
      const int an = L.arr_next[a];
      L.mflag[a] = 0;
      if (sh == -1) {
        sh = tail = a;
        L.next[a] = -1;
      } else if (a > sh) {
        L.next[a] = sh;
        sh = a;
      } else {
        int q2 = sh;
        for (int g2 = 0; L.next[q2] != -1 && L.next[q2] > a && g2 < guard; g2++) q2 = L.next[q2];
        L.next[a] = L.next[q2];
        L.next[q2] = a;
        if (L.next[a] == -1) tail = a;
      }
      a = an;
    }
    L.arr_head[c] = -1;
    if (sh != -1) {
      L.next[tail] = first;
      first = sh;
    }
    L.head[c] = first;
    L.dflag[c] = 0;
    // 3. the rows of every particle around c are rebuilt in this pass: the
    // 27 flag exchanges are issued together, then one append per cell
    const DevParams& P = sys_params(PT, cellsys, c);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int cl = c - P.coff;
    const int cx = cl % nx, cy = (cl / nx) % ny, cz = cl / (nx * ny);
    int jcs[27];
    unsigned fresh = 0u;
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const int jx = cx + o % 3 - 1, jy = cy + (o / 3) % 3 - 1, jz = cz + o / 9 - 1;
      const bool ok = (P.pbc[0] || (jx >= 0 && jx < nx)) && (P.pbc[1] || (jy >= 0 && jy < ny)) &&
                      (P.pbc[2] || (jz >= 0 && jz < nz));
      jcs[o] = ok ? P.coff + axis_wrap(jx, nx, P.pbc[0]) +
                        nx * (axis_wrap(jy, ny, P.pbc[1]) + ny * axis_wrap(jz, nz, P.pbc[2]))
                  : -1;
    }
#pragma unroll
    for (int o = 0; o < 27; o++)
      if (jcs[o] >= 0 && atomicExch(&L.rflag[jcs[o]], 1) == 0) fresh |= 1u << o;
    if (fresh) {
      int k = atomicAdd(&cnt->n_repair, __popc(fresh));
#pragma unroll
      for (int o = 0; o < 27; o++)
        if ((fresh >> o) & 1u) L.rlist[k++] = jcs[o];
    }
  }
}

// ---------------------------------------------------------------------------
// K2: candidate rows

// The row of particle p (cell c), built by one warp.  Lane L < 27 owns the
// neighbour cell at offset (L%3-1, L/3%3-1, L/9-1); lane 13 (own cell) walks
// the part of the list after p, lane 27 the part before p (p's rank).  The
// row holds the partners the sweep meets with p as "i": the own cell after p,
// then the half-shell cells (offset index kx + Nx*(ky + Ny*kz) > 0,
// AddAllNeighbours3D src/MCells.f90:456) in FirstNeighbour order, i.e.
// descending (kz, ky, kx) -- NeighbourParticles' list (src/MCells.f90:
// 793-829) from p on.
template <bool PP>
__device__ __forceinline__ void build_row(const DevParams& P, int n, int p, int c,
                                          const double4* __restrict__ X,
                                          const int* __restrict__ comp,
                                          const int* __restrict__ head,
                                          const int* __restrict__ next, const Rows& R,
                                          Counters* cnt, int tag) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int cl = c - P.coff;
  const int cx = cl % nx, cy = (cl / nx) % ny, cz = cl / (nx * ny);
  const double4 p4 = X[p];
  const int cp = PP ? 0 : comp[p];
  int start = -1, order = 1 << 20;
  bool walk = false;
  if (lane < 27) {
    const int d[3] = {lane % 3 - 1, (lane / 3) % 3 - 1, lane / 9 - 1};
    const int cc[3] = {cx, cy, cz};
    const int N[3] = {nx, ny, nz};
    bool ok = true;
    int w[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      int j = cc[k] + d[k];
      if (P.pbc[k]) {
        if (j == N[k]) j = 0;
        if (j == -1) j = N[k] - 1;
      } else if (j < 0 || j >= N[k]) {
        ok = false;
      }
      w[k] = j;
    }
    const int lex = d[0] + 3 * d[1] + 9 * d[2];
    if (lane == 13) {
      start = next[p];
      order = 0;
      walk = true;
    } else if (ok && lex > 0) {
      start = head[P.coff + w[0] + nx * (w[1] + ny * w[2])];
      order = 1 + (13 - lex);
      walk = true;
    }
  }
  const double skin = P.vl_skin;
  auto is_cand = [&](int q) -> bool {
    const double4 q4 = X[q];
    double Rij[3] = {q4.x - p4.x, q4.y - p4.y, q4.z - p4.z};
#pragma unroll
    for (int k = 0; k < 3; k++) Rij[k] = min_image_exact(Rij[k], P.box, k);
    const double DijSq = sumsq3(Rij);
    double md;
    if (PP) md = p4.w + q4.w;
    else md = sqrt(Material<PP>::min_dij_sq(P, cp, p4.w, comp[q], q4.w));
    md = md + skin;
    return md * md - DijSq > 0.0;
  };
  // pass 1: walk and count; the first 8 list elements and their test
  // results stay in registers for pass 2.  Lane 27 counts the list before p.
  int count = 0, walked = 0;
  unsigned hits = 0u;
  int cache[8];
  bool bad = false;
  int q = start;
#pragma unroll
  for (int i = 0; i < 8; i++) cache[i] = -1;
  if (walk) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (q != -1) {
        cache[i] = q;
        walked = i + 1;
        if (is_cand(q)) {
          hits |= 1u << i;
          count++;
        }
        q = next[q];
      }
    }
  }
  const int resume = q;  // first element not cached (-1: none)
  {
    int guard = 0;
    if (walk) {
      while (q != -1) {
        if (++guard > n) {
          bad = true;
          break;
        }
        if (is_cand(q)) count++;
        q = next[q];
      }
    } else if (lane == 27) {
      q = head[c];
      while (q != p) {
        if (q == -1 || ++guard > n) {
          bad = true;
          break;
        }
        count++;
        q = next[q];
      }
    }
  }
  if (__any_sync(FULL, bad)) {
    if (lane == 0) {
      atomicExch(&cnt->list_error, 1);
      set_abort(cnt, tag);
    }
    return;
  }
  int off = 0, m = 0;
  for (int l = 0; l < 27; l++) {
    const int ol = __shfl_sync(FULL, order, l);
    const int cl2 = __shfl_sync(FULL, walk ? count : 0, l);
    if (ol < order) off += cl2;
    m += cl2;
  }
  const int rank = __shfl_sync(FULL, count, 27);
  if (m > R.kc) {
    if (lane == 0) {
      atomicMax(&cnt->need_kc, m);
      atomicExch(&cnt->row_overflow, 1);
      set_abort(cnt, tag);
      R.meta[p] = 0;
    }
    return;
  }
  // pass 2: write (the cached part, then the rest of the list)
  if (walk) {
    int k = off;
#pragma unroll
    for (int i = 0; i < 8; i++)
      if (i < walked && ((hits >> i) & 1u)) R.cand[(size_t)(k++) * n + p] = cache[i];
    int q2 = resume;
    while (q2 != -1) {
      if (is_cand(q2)) R.cand[(size_t)(k++) * n + p] = q2;
      q2 = next[q2];
    }
  }
  if (lane == 0) {
    R.meta[p] = m;
    R.rank[p] = rank;
  }
}

// Candidate rows of the pass: every row when the pass is due for a full
// rebuild (one warp per particle), else the rows of the particles of every
// repair cell (one warp per cell).  The repair flags of the listed cells are
// cleared in every case (also when a stopped sequence skips the work).
template <bool PP>
__global__ void __launch_bounds__(256) k_screen(const DevParams* __restrict__ PT,
                                                const int* __restrict__ sysid,
                                                const int* __restrict__ cellsys, int n,
                                                const double4* __restrict__ X,
                                                const int* __restrict__ comp,
                                                const int* __restrict__ cell_cur, CellLists L,
                                                Rows R, Counters* cnt, int tag) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool skip = cnt->abort != 0;
  const bool full = cnt->full_due != 0;
  const int m = cnt->n_repair;
  for (int r = warp; r < m; r += nwarps) {
    const int c = L.rlist[r];
    if (!skip && !full) {
      int p = L.head[c], guard = 0;
      while (p != -1) {
        if (++guard > n) {
          if (lane == 0) {
            atomicExch(&cnt->list_error, 1);
            set_abort(cnt, tag);
          }
          break;
        }
        build_row<PP>(sys_params(PT, cellsys, c), n, p, c, X, comp, L.head, L.next, R, cnt,
                      tag);
        p = L.next[p];
      }
    }
    if (lane == 0) L.rflag[c] = 0;
  }
  if (!skip && full)
    for (int p = warp; p < n; p += nwarps)
      build_row<PP>(sys_params(PT, sysid, p), n, p, cell_cur[p], X, comp, L.head, L.next, R, cnt,
                    tag);
}

// ---------------------------------------------------------------------------
// K2+K4: the FP64 force pass (exact order), two kernels.
//
// k_contact_fp64: one thread per particle p, as "i" of its row: the overlap
//   test over the row, every contact evaluated once (one lane per contact),
//   the "i" part folded by p in row order (iForce, iTorque), then p's walls
//   and drag -- p's whole block of the sweep.  The "j" part of each contact
//   (FN, FT, Nij x FT) goes to the partner's incoming records with p's sweep
//   key.  The history record of the pair is looked up in p's table, then in
//   the partner's, and rewritten into p's new table.
// k_fold_fp64: one thread per particle: its incoming "j" results and its own
//   block added in sweep order (Force(j) = Force(j) - FN - FT,
//   Torque(j) = Torque(j) + Rj*Nij_x_FT, Force(i) = Force(i) + iForce,
//   src/MForces.f90:254-259, 319-320), a = F/m, alpha = T/I, then the
//   integrator epilogue.

// record keys of the owner kept in shared memory by the contact kernels
constexpr int KREG = 8;

// Owner data handed to the lane that computes one of its contacts.
struct OwnerF64 {
  double x, y, z, R, vx, vy, vz, wx, wy, wz;
  int p, cp, sys, pad;
  unsigned long long key;
};

// MINB: resident blocks of 128 threads per SM the kernel is compiled for
// (registers per thread <= 65536 / (128 * MINB)); the autotuner picks one.
template <bool PP, int MINB>
__global__ void __launch_bounds__(128, MINB) k_contact_fp64(PassArgs<double4, double2> A) {
  // per warp: the current 32 contacts (candidate index, owner lane), their
  // "i" results FN, FT, VT, torque term (12 doubles), the owners' first
  // record keys, record counts and the records their contacts matched
  __shared__ int s_k[4][32], s_o[4][32], s_q[4][32];
  __shared__ int s_hk[4][KREG][32], s_hc[4][32];
  __shared__ unsigned s_match[4][32];
  __shared__ double s_r[12][4][32];
  __shared__ double s_w[NWM][128];  // |FN| of each wall contact
  __shared__ int s_abort;
  // one decision for the whole block (it meets a block barrier later)
  if (threadIdx.x == 0) s_abort = A.cnt->abort;
  __syncthreads();
  if (s_abort) return;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int w = 0; w < A.nw_max; w++) s_w[w][threadIdx.x] = 0.0;
  const int p0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = p0 < A.n;
  const int p = valid ? p0 : 0;
  const DevParams& P = sys_params(A.P, A.sysid, p);  // this particle's system
  const Box& B = P.box;
  const int n = A.n;
  unsigned n_col = 0, n_pc = 0, n_wc = 0;
  int need = 0, need_in = 0;
  bool in_over = false;

  const int c = A.cell_cur[p];
  const double4 p4 = A.X[p];
  const double xp[3] = {p4.x, p4.y, p4.z};
  const double Rp = p4.w;
  const double4 pv4 = A.v4[p];
  const double2 pw2 = A.w2[p];
  const double vp[3] = {pv4.x, pv4.y, pv4.z};
  const double wp[3] = {pv4.w, pw2.x, pw2.y};
  const int cp = PP ? 0 : A.comp[p];
  double inv_m, inv_i, eff_m;
  Material<PP>::self(P, cp, Rp, inv_m, inv_i, eff_m);
  const int n1 = A.meta[p] & META_MASK;
  const unsigned long long key_p = sweep_key(c, A.rank[p]);
  const double half_dt = A.half_dt;
  const bool update = A.update != 0;
  int hw_n = 0;
  bool overflow = false;
  const int hc = valid ? A.Hr.cnt[p] : 0;
#pragma unroll
  for (int r = 0; r < KREG; r++) s_hk[wid][r][lane] = r < hc ? A.Hr.key[hslot(A.Hr, p, r)] : -1;
  s_hc[wid][lane] = hc;
  s_match[wid][lane] = 0u;
  __syncwarp();

  double iF[3], iT[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 3; k++) iF[k] = eff_m * P.gravity[k];

  auto record = [&](int partner, const double ft[3], const double vt[3]) {
    if (hw_n < A.Hw.cap)
      hist_write(A.Hw, p, hw_n, partner, ft, vt);
    else
      overflow = true;
    hw_n++;
  };
  // Rij = x_j - x_i (minimum image, src/MForces.f90:209-217)
  auto geometry = [&](const Box& Bx, const double xo[3], const double4& q4,
                      double Rij[3]) -> double {
    Rij[0] = q4.x - xo[0];
    Rij[1] = q4.y - xo[1];
    Rij[2] = q4.z - xo[2];
#pragma unroll
    for (int k = 0; k < 3; k++) Rij[k] = min_image_exact(Rij[k], Bx, k);
    return sumsq3(Rij);
  };
  // the overlap test DeltaDijSq = MinDijSq - DijSq > 0 (src/MForces.f90:218-224)
  auto test = [&](int, int q, const double4& q4) -> bool {
    double Rij[3];
    const double DijSq = geometry(B, xp, q4, Rij);
    const int cq = PP ? 0 : A.comp[q];
    return Material<PP>::min_dij_sq(P, cp, Rp, cq, q4.w) - DijSq > 0.0;
  };
  // one contact of owner `o` ("i") with candidate k ("j"), computed by this
  // lane (src/MForces.f90:199-252)
  auto compute = [&](const OwnerF64& o, int oo, int k, int slot) {
    const int q = __ldg(A.cand + (size_t)k * n + o.p);
    const int s_in = atomicAdd(&A.in_cnt[q], 1);  // q's "j" record (returns early)
    const double4 q4 = A.X[q];
    const double2 qw2 = A.w2[q];
    const double4 qv4 = A.v4[q];
    const double xo[3] = {o.x, o.y, o.z};
    double Rij[3];
    const DevParams& PO = A.P[o.sys];  // the owner's system (a warp may span two)
    const double DijSq = geometry(PO.box, xo, q4, Rij);
    const int cq = PP ? 0 : A.comp[q];
    const double Delta = Material<PP>::min_dij_sq(PO, o.cp, o.R, cq, q4.w) - DijSq;
    PairPar pp;
    Material<PP>::pair(PO, o.cp, o.R, cq, q4.w, pp);
    const double va[3] = {o.vx, o.vy, o.vz}, wa[3] = {o.wx, o.wy, o.wz};
    const double vb[3] = {qv4.x, qv4.y, qv4.z}, wb[3] = {qv4.w, qw2.x, qw2.y};
    // VerifyPairContact: the owner's records, then the partner's
    double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
    const int oc = s_hc[wid][oo];
    int r = -1;
#pragma unroll
    for (int rr = 0; rr < KREG; rr++)
      if (rr < oc && s_hk[wid][rr][oo] == q) r = rr;
    for (int rr = KREG; r < 0 && rr < oc; rr++)
      if (A.Hr.key[hslot(A.Hr, o.p, rr)] == q) r = rr;
    bool contacting = r >= 0;
    if (contacting) {
      hist_read(A.Hr, o.p, r, FT0, VT0);
      if (r < 32) atomicOr(&s_match[wid][oo], 1u << r);
    } else {
      const int r2 = find_record(A.Hr, q, o.p);
      contacting = r2 >= 0;
      if (contacting) hist_read(A.Hr, q, r2, FT0, VT0);
    }
    if (!contacting) n_col++;
    n_pc++;
    ContactOut out;
    pair_contact(Rij, DijSq, Delta, pp, o.R, va, wa, q4.w, vb, wb, half_dt, contacting, FT0, VT0,
                 out);
    // "j" side into q's incoming records
    if (s_in < A.in_cap) {
      InRec64* rec = (InRec64*)A.in_rec + (size_t)s_in * A.in_stride + q;
      rec->a = make_double2(__longlong_as_double((long long)o.key), out.FN[0]);
      rec->b = make_double2(out.FN[1], out.FN[2]);
      rec->c = make_double2(out.FT[0], out.FT[1]);
      rec->d = make_double2(out.FT[2], out.NxFT[0]);
      rec->e = make_double2(out.NxFT[1], out.NxFT[2]);
    } else {
      in_over = true;
    }
    need_in = need_in > s_in + 1 ? need_in : s_in + 1;
    // "i" side to the owner (iTorque + (Ri*Nij) x FT)
    double RN[3], tq[3];
#pragma unroll
    for (int d = 0; d < 3; d++) RN[d] = o.R * out.N[d];
    cross3(RN, out.FT, tq);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      s_r[d][wid][slot] = out.FN[d];
      s_r[3 + d][wid][slot] = out.FT[d];
      s_r[6 + d][wid][slot] = out.VT[d];
      s_r[9 + d][wid][slot] = tq[d];
    }
    s_q[wid][slot] = q;
  };
  // the owner adds one contact (iForce = iForce + FN + FT) and stores its record
  auto accum = [&](int slot, int) {
    double FN[3], FT[3], VT[3], tq[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      FN[d] = s_r[d][wid][slot];
      FT[d] = s_r[3 + d][wid][slot];
      VT[d] = s_r[6 + d][wid][slot];
      tq[d] = s_r[9 + d][wid][slot];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) iF[d] = iF[d] + FN[d] + FT[d];
#pragma unroll
    for (int d = 0; d < 3; d++) iT[d] = iT[d] + tq[d];
    if (update) record(s_q[wid][slot], FT, VT);
  };
  const OwnerF64 me{xp[0], xp[1], xp[2], Rp, vp[0], vp[1], vp[2], wp[0], wp[1], wp[2],
                    p, cp, A.sysid ? A.sysid[p] : 0, 0, key_p};
  contact_loop(A.cand, A.X, n, p, valid, n1, me, s_k[wid], s_o[wid], test, compute, accum);

  if (valid) {
    // ---- walls (src/MForces.f90:274-314)
    for (int w = 0; w < P.nw; w++) {
      const dem_wall& W = P.walls[w];
      const int wi = p * P.nw + w;
      bool contacting = A.Hr.wflag[wi] != 0;
      double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
      if (contacting) {
        const double2* v = A.Hr.wval + (size_t)wi * 3;
        double2 a = v[0], b = v[1], d = v[2];
        FT0[0] = a.x; FT0[1] = a.y; FT0[2] = b.x;
        VT0[0] = b.y; VT0[1] = d.x; VT0[2] = d.y;
      }
      double Dij, Nij[3], Qji[3];
      const bool ov = overlap_wall(P, W, xp, Rp, Dij, Nij, Qji);
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
        s_w[w][threadIdx.x] = sqrt(sumsq3(o.FN));
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
    if (A.drag) {  // iForce = iForce + DragForce(iPart) (src/MForces.f90:316)
#pragma unroll
      for (int k = 0; k < 3; k++) iF[k] = iF[k] + A.drag[(size_t)3 * p + k];
    }
    Own64* ow = (Own64*)A.own + p;
    ow->a = make_double2(iF[0], iF[1]);
    ow->b = make_double2(iF[2], iT[0]);
    ow->c = make_double2(iT[1], iT[2]);
    // ---- the records this particle holds and no contact of the pass
    // matched: kept if the sweep did not visit the pair (its cells are not
    // neighbours, or the partner index lies past the last particle, a record
    // that particle removal left behind), else the contact ended
    // (RemovePairContact) or the other particle evaluated it
    if (update) {
      const unsigned matched = s_match[wid][lane];
      for (int r = 0; r < hc; r++) {
        if (r < 32 && ((matched >> r) & 1u)) continue;
        const int q2 = A.Hr.key[hslot(A.Hr, p, r)];
        if (q2 >= A.n || !cells_adjacent(P, c, A.cell_cur[q2])) {
          double ft[3], vt[3];
          hist_read(A.Hr, p, r, ft, vt);
          record(q2, ft, vt);
        }
      }
      A.Hw.cnt[p] = hw_n < A.Hw.cap ? hw_n : A.Hw.cap;
      need = hw_n;
    }
  }
  if (A.nw_max > 0) wall_partials(s_w, A.nw_max, A.wall_part);
  // a table that overflowed: the pass is launched again with larger tables;
  // stop what follows
  if (overflow) {
    atomicExch(&A.cnt->overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  if (in_over) {
    atomicExch(&A.cnt->in_overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  publish_counts_block(A.cnt, A.update != 0, n_col, n_pc, n_wc, (unsigned)need,
                       (unsigned)need_in);
}

// The fold kernel: Force and Torque of every particle in sweep order, a =
// F/m, alpha = T/I (src/MForces.f90:330-333), then the integrator epilogue.
template <bool PP, int EPI, int MINB>
__global__ void __launch_bounds__(128, MINB) k_fold_fp64(PassArgs<double4, double2> A) {
  __shared__ int s_abort;
  // one decision for the whole block (it meets a block barrier at the end)
  if (threadIdx.x == 0) s_abort = A.cnt->abort;
  __syncthreads();
  if (s_abort) return;
  const int p0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = p0 < A.n;
  const int p = valid ? p0 : 0;
  double d2 = 0.0;
  if (valid) {
    const DevParams& P = sys_params(A.P, A.sysid, p);
    const int c = A.cell_cur[p];
    const unsigned long long key_p = sweep_key(c, A.rank[p]);
    const int ni = A.in_cnt[p];
    A.in_cnt[p] = 0;  // for the next pass's contact kernel
    const double4 p4 = A.X[p];
    const double xp[3] = {p4.x, p4.y, p4.z};
    const double Rp = p4.w;
    const int cp = PP ? 0 : A.comp[p];
    double inv_m, inv_i, eff_m;
    Material<PP>::self(P, cp, Rp, inv_m, inv_i, eff_m);
    const Own64 ow = ((const Own64*)A.own)[p];
    const InRec64* in = (const InRec64*)A.in_rec + p;
    const size_t st = (size_t)A.in_stride;
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    fold_in_order(
        ni, key_p,
        [&](int e) {
          return (unsigned long long)__double_as_longlong(((const double*)(in + e * st))[0]);
        },
        [&]() {
          const double iF[3] = {ow.a.x, ow.a.y, ow.b.x}, iT[3] = {ow.b.y, ow.c.x, ow.c.y};
#pragma unroll
          for (int k = 0; k < 3; k++) F[k] = F[k] + iF[k];
#pragma unroll
          for (int k = 0; k < 3; k++) T[k] = T[k] + iT[k];
        },
        [&](int e) {
          const InRec64 r = in[e * st];
          const double FN[3] = {r.a.y, r.b.x, r.b.y}, FT[3] = {r.c.x, r.c.y, r.d.x};
          const double NxFT[3] = {r.d.y, r.e.x, r.e.y};
#pragma unroll
          for (int k = 0; k < 3; k++) F[k] = F[k] - FN[k] - FT[k];
#pragma unroll
          for (int k = 0; k < 3; k++) T[k] = T[k] + Rp * NxFT[k];
        });
    if (EPI == EPI_STORE && A.amsum) {
      const size_t n3 = (size_t)3 * A.n;
#pragma unroll
      for (int k = 0; k < 3; k++) A.amsum[(size_t)3 * p + k] = F[k];
#pragma unroll
      for (int k = 0; k < 3; k++) A.amsum[n3 + (size_t)3 * p + k] = T[k];
    }
    double acc[3], alp[3];
#pragma unroll
    for (int k = 0; k < 3; k++) acc[k] = F[k] * inv_m;
#pragma unroll
    for (int k = 0; k < 3; k++) alp[k] = T[k] * inv_i;
    const double4 pv4 = A.v4[p];
    const double2 pw2 = A.w2[p];
    const double vp[3] = {pv4.x, pv4.y, pv4.z};
    const double wp[3] = {pv4.w, pw2.x, pw2.y};
    epilogue<EPI>(A, P, p, xp, Rp, vp, wp, acc, alp, c, d2);
  }
  if (EPI != EPI_STORE) publish_disp_block(A.cnt, d2);
}

}  // namespace dem
