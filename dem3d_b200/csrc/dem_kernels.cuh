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
#include "dem_test.cuh"

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

// The values the predictor passes leave out (PassArgs::lazy) written back:
// Particle a, alpha from the ring slot ipc(1) (nprev > 0), Predicted x from
// the Predicted side's position copy and, with FP64 copies (EXACT),
// Predicted v, w from its velocity copies.  Plain copies: the bits are the
// ones the predictor computed.
template <bool EXACT, class V4, class W2>
__global__ void k_settle_state(int n, StateArrays Q, StateArrays R, const double* __restrict__ ring,
                               int slot0, int nprev, const double4* __restrict__ X1,
                               const V4* __restrict__ v41, const W2* __restrict__ w21) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (nprev > 0) {
    const double* rg = ring + (size_t)slot0 * 9 * n + i;
    Q.ax[i] = rg[3 * (size_t)n]; Q.ay[i] = rg[4 * (size_t)n]; Q.az[i] = rg[5 * (size_t)n];
    Q.lx[i] = rg[6 * (size_t)n]; Q.ly[i] = rg[7 * (size_t)n]; Q.lz[i] = rg[8 * (size_t)n];
  }
  const double4 x = X1[i];
  R.px[i] = x.x; R.py[i] = x.y; R.pz[i] = x.z;
  if (EXACT) {
    const V4 v = v41[i];
    const W2 w = w21[i];
    R.vx[i] = (double)v.x; R.vy[i] = (double)v.y; R.vz[i] = (double)v.z;
    R.wx[i] = (double)v.w; R.wy[i] = (double)w.x; R.wz[i] = (double)w.y;
  }
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

// ---------------------------------------------------------------------------
// Storage in cell order (dem_set_reorder): the permutation pi (new place s
// holds the particle stored at pi[s]) is the cells' lists in cell order.

// pi[cell_start[c] + k] = the k-th particle of cell c's list
__global__ void k_reorder_fill(CellLists L, int ncell, const int* __restrict__ cell_start,
                               int* __restrict__ pi, int n, int* __restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int k = cell_start[c];
  const int end = cell_start[c + 1];
  for (int q = L.head[c]; q != -1; q = L.next[q]) {
    if (k >= end || k >= n || q < 0 || q >= n) {
      atomicExch(err, 1);
      return;
    }
    pi[k++] = q;
  }
  if (k != end) atomicExch(err, 1);
}

// the list length of every cell (the slots record it)
__global__ void k_reorder_counts(const CellLists L, int ncell, int* __restrict__ cnt,
                                 int* __restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int m = L.slot_n[c];
  if (m < 0) atomicExch(err, 1);
  cnt[c] = m < 0 ? 0 : m;
}

__global__ void k_iota(int n, int* __restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

__global__ void k_inverse(int n, const int* __restrict__ pi, int* __restrict__ inv) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) inv[pi[s]] = s;
}

// dst row r, place s <- base row r, place pi[s] (elem bytes, a multiple of 4)
__global__ void k_gather_col(const char* __restrict__ base, int elem, int rows, long long stride,
                             int n, const int* __restrict__ pi, char* __restrict__ dst) {
  const long long words = (long long)elem / 4;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= words * n * rows) return;
  const int w = (int)(t % words);
  const long long rs = t / words;
  const int s = (int)(rs % n), r = (int)(rs / n);
  ((int*)(dst + ((long long)r * n + s) * elem))[w] =
      ((const int*)(base + (long long)r * stride + (long long)pi[s] * elem))[w];
}

__global__ void k_scatter_col(char* __restrict__ base, int elem, int rows, long long stride, int n,
                              const char* __restrict__ src) {
  const long long words = (long long)elem / 4;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= words * n * rows) return;
  const int w = (int)(t % words);
  const long long rs = t / words;
  const int s = (int)(rs % n), r = (int)(rs / n);
  ((int*)(base + (long long)r * stride + (long long)s * elem))[w] =
      ((const int*)(src + ((long long)r * n + s) * elem))[w];
}

// stored particle numbers in a[0..m) renamed by inv (other values kept)
__global__ void k_remap(int* __restrict__ a, long long m, const int* __restrict__ inv, int n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int v = a[i];
  if (v >= 0 && v < n) a[i] = inv[v];
}

// The slots of cells [c_begin, c_begin + ncells) from their lists (after
// the lists were built or changed outside the relink).
__global__ void k_cell_slots(CellLists L, int c_begin, int ncells, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ncells) copy_slots(L, c_begin + i, L.head[c_begin + i], n);
}

__global__ void k_relink(const DevParams* __restrict__ PT, const int* __restrict__ cellsys,
                         CellLists L, int par, int n, int update, int stop_tag, Counters* cnt) {
  pass_kernel_entry();
  relink_body(PT, cellsys, L, par, n, update, stop_tag, cnt, blockIdx.x * blockDim.x + threadIdx.x,
              gridDim.x * blockDim.x);
}

// ---------------------------------------------------------------------------
// K2+K4: a force pass is three kernels.
//
// k_test (both precisions): one thread per particle as "i" of its row
//   applies the reference's overlap test DeltaDijSq = MinDijSq - DijSq > 0
//   (src/MForces.f90:218-224, exact FP64) to its candidates and writes its
//   contacts to the pass's contact list, together and in row order.
// k_pair_fp64 / k_pair_mixed: one thread per contact of the list evaluates
//   it once (src/MForces.f90:199-252, CommonCalculations :339-387) with the
//   pair's history record (looked up in i's table, then j's), writes the "i"
//   half at the contact's place in the list, the "j" half to j's incoming
//   records with i's sweep key, and the updated record into i's new table at
//   the contact's rank among i's contacts.
// k_fold_fp64 / k_fold_mixed: one thread per particle p builds its block of
//   the sweep (iForce = m_eff*g, the "i" halves of its contacts in row order,
//   its walls, its drag; src/MForces.f90:190-316), keeps the records no
//   contact visited, adds the block and the "j" halves it received in sweep
//   order (Force(j) = Force(j) - FN - FT, Torque(j) + Rj*Nij_x_FT,
//   Force(i) = Force(i) + iForce; :254-259, 319-320), forms a = F/m,
//   alpha = T/I (:330-333) and runs the integrator epilogue.

// BS threads per block.  STRIDE: grid-stride over blocks of BS particles (a
// grid smaller than the particle count gives each thread several particles);
// else one block of particles per block.
// (register budget: 7 blocks of 128 threads per SM, 28 warps, as the
// kernel fits in 72 registers)
template <bool PP, int BS, bool STRIDE>
__global__ void __launch_bounds__(BS, 7 * 128 / BS) k_test(TestArgs A) {
  pass_kernel_entry();
  if (!STRIDE) {
    test_body<PP>(A, blockIdx.x);
    return;
  }
  const int nvb = (A.n + BS - 1) / BS;
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) test_body<PP>(A, vb);
}

// record keys read before the record count is known (speculatively, within
// the table's capacity)
constexpr int KSPEC = 2;

// The pair kernel (FP64): one thread per contact, grid-stride over the list.
// (Body for block `vblock` of a grid of `vgrid` blocks.)
template <bool PP>
__device__ __forceinline__ void pair_fp64_body(const PassArgs<double4, double2>& A, int vblock,
                                               int vgrid) {
  __shared__ int s_abort;
  if (threadIdx.x == 0) s_abort = A.cnt->abort;
  __syncthreads();
  if (s_abort) return;
  const int total = A.cnt->n_contacts;
  if (vblock == 0 && threadIdx.x == 0) {
    // the pass's pair contacts: the length of its contact list
    atomicAdd(&A.cnt->pair_contacts, (unsigned long long)total);
    atomicMax(&A.cnt->need_cl, total);
  }
  const bool update = A.update != 0;
  const double half_dt = A.half_dt;
  unsigned n_col = 0;
  int need = 0, need_in = 0;
  bool overflow = false, in_over = false;
  for (int s = vblock * blockDim.x + threadIdx.x; s < total; s += vgrid * blockDim.x) {
    const int2 e = A.clist[s];
    const int p = e.x, q = e.y;
    const int s_in = atomicAdd(&A.in_cnt[q], 1);  // q's "j" record (returns early)
    const int ord = s - A.cstart[p];
    const int hc = A.Hr.cnt[p];
    int kspec[KSPEC];
#pragma unroll
    for (int r = 0; r < KSPEC; r++) kspec[r] = r < A.Hr.cap ? A.Hr.key[hslot(A.Hr, p, r)] : -1;
    const DevParams& P = sys_params(A.P, A.sysid, p);
    const double4 p4 = A.X[p], q4 = A.X[q];
    const double4 pv4 = A.v4[p], qv4 = A.v4[q];
    const double2 pw2 = A.w2[p], qw2 = A.w2[q];
    const int cp = PP ? 0 : A.comp[p], cq = PP ? 0 : A.comp[q];
    // Rij = x_j - x_i (minimum image, src/MForces.f90:209-217)
    double Rij[3] = {q4.x - p4.x, q4.y - p4.y, q4.z - p4.z};
#pragma unroll
    for (int k = 0; k < 3; k++) Rij[k] = min_image_exact(Rij[k], P.box, k);
    const double DijSq = sumsq3(Rij);
    const double Delta = Material<PP>::min_dij_sq(P, cp, p4.w, cq, q4.w) - DijSq;
    PairPar pp;
    Material<PP>::pair(P, cp, p4.w, cq, q4.w, pp);
    const double va[3] = {pv4.x, pv4.y, pv4.z}, wa[3] = {pv4.w, pw2.x, pw2.y};
    const double vb[3] = {qv4.x, qv4.y, qv4.z}, wb[3] = {qv4.w, qw2.x, qw2.y};
    // VerifyPairContact: i's records, then j's
    int r = -1;
#pragma unroll
    for (int rr = 0; rr < KSPEC; rr++)
      if (r < 0 && rr < hc && kspec[rr] == q) r = rr;
    for (int rr = KSPEC; r < 0 && rr < hc; rr++)
      if (A.Hr.key[hslot(A.Hr, p, rr)] == q) r = rr;
    double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
    bool contacting = r >= 0;
    if (contacting) {
      hist_read(A.Hr, p, r, FT0, VT0);
      if (r < 32) atomicOr(&A.matched[p], 1u << r);
    } else {
      const int r2 = find_record(A.Hr, q, p);
      contacting = r2 >= 0;
      if (contacting) hist_read(A.Hr, q, r2, FT0, VT0);
    }
    if (!contacting) n_col++;
    ContactOut out;
    pair_contact(Rij, DijSq, Delta, pp, p4.w, va, wa, q4.w, vb, wb, half_dt, contacting, FT0, VT0,
                 out);
    // "j" half into q's incoming records
    if (s_in < A.in_cap) {
      InRec64* rec = (InRec64*)A.in_rec + (size_t)s_in * A.in_stride + q;
      rec->a = make_double2(__longlong_as_double((long long)sweep_key(A.cell_cur[p], A.rank[p])),
                            out.FN[0]);
      rec->b = make_double2(out.FN[1], out.FN[2]);
      rec->c = make_double2(out.FT[0], out.FT[1]);
      rec->d = make_double2(out.FT[2], out.NxFT[0]);
      rec->e = make_double2(out.NxFT[1], out.NxFT[2]);
    } else {
      in_over = true;
    }
    need_in = need_in > s_in + 1 ? need_in : s_in + 1;
    // "i" half at the contact's place (iTorque + (Ri*Nij) x FT)
    double RN[3], tq[3];
#pragma unroll
    for (int d = 0; d < 3; d++) RN[d] = p4.w * out.N[d];
    cross3(RN, out.FT, tq);
    IRec64* ir = (IRec64*)A.irec + s;
    ir->a = make_double2(out.FN[0], out.FN[1]);
    ir->b = make_double2(out.FN[2], out.FT[0]);
    ir->c = make_double2(out.FT[1], out.FT[2]);
    ir->d = make_double2(tq[0], tq[1]);
    ir->e = make_double2(tq[2], 0.0);
    // UpdatePairContact: the record goes to i's new table, in row order
    if (update) {
      if (ord < A.Hw.cap) hist_write(A.Hw, p, ord, q, out.FT, out.VT);
      else overflow = true;
      need = need > ord + 1 ? need : ord + 1;
    }
  }
  if (overflow) {
    atomicExch(&A.cnt->overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  if (in_over) {
    atomicExch(&A.cnt->in_overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  publish_counts_block(A.cnt, update, n_col, 0u, 0u, (unsigned)need, (unsigned)need_in);
}

template <bool PP, int MINB>
__global__ void __launch_bounds__(128, MINB) k_pair_fp64(PassArgs<double4, double2> A) {
  pass_kernel_entry();
  pair_fp64_body<PP>(A, blockIdx.x, gridDim.x);
}

// The fold kernel (FP64): p's block of the sweep, its Force and Torque in
// sweep order, a = F/m, alpha = T/I, then the integrator epilogue.  WALLS:
// some system has walls.
template <bool PP, int EPI, bool WALLS>
__device__ __forceinline__ void fold_fp64_body(const PassArgs<double4, double2>& A, int vblock) {
  __shared__ double s_w[WALLS ? NWM : 1][128];  // |FN| of each wall contact
  __shared__ int s_abort;
  // one decision for the whole block (it meets block barriers later)
  if (threadIdx.x == 0) s_abort = A.cnt->abort;
  __syncthreads();
  if (s_abort) return;
  if (WALLS)
    for (int w = 0; w < A.nw_max; w++) s_w[w][threadIdx.x] = 0.0;
  if (vblock == 0 && threadIdx.x == 0) atomicAdd(&A.cnt->pass_id, 1);  // this pass is done
  const int p0 = vblock * blockDim.x + threadIdx.x;
  const int p = p0 < A.n ? p0 : 0;
  // (a slab of a decomposition advances only its own particles)
  const bool valid = p0 < A.n && in_slab(sys_params(A.P, A.sysid, p), A.cell_cur[p]);
  const bool update = A.update != 0;
  unsigned n_wc = 0;
  int need = 0;
  bool overflow = false;
  double d2 = 0.0;
  if (valid) {
    const DevParams& P = sys_params(A.P, A.sysid, p);
    prefetch_epilogue<EPI>(A, P, p, false);
    const int c = A.cell_cur[p];
    const unsigned long long key_p = sweep_key(c, A.rank[p]);
    const int ni = A.in_cnt[p];
    if (ni) A.in_cnt[p] = 0;  // for the next pass's pair kernel
    const unsigned matched = A.matched[p];
    if (matched) A.matched[p] = 0u;
    const int nc = A.ccount[p];
    const int st0 = A.cstart[p];
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
    // ---- p's block: gravity, its contacts as "i" in row order
    double iF[3], iT[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 3; k++) iF[k] = eff_m * P.gravity[k];
    const IRec64* ir = (const IRec64*)A.irec + st0;
    for (int k = 0; k < nc; k++) {
      const IRec64 r = ir[k];
      const double FN[3] = {r.a.x, r.a.y, r.b.x}, FT[3] = {r.b.y, r.c.x, r.c.y};
      const double tq[3] = {r.d.x, r.d.y, r.e.x};
#pragma unroll
      for (int d = 0; d < 3; d++) iF[d] = iF[d] + FN[d] + FT[d];
#pragma unroll
      for (int d = 0; d < 3; d++) iT[d] = iT[d] + tq[d];
    }
    int hw_n = nc;  // the pair kernel wrote the records of the contacts
    // ---- walls (src/MForces.f90:274-314)
    if (WALLS) {
      const double half_dt = A.half_dt;
      for (int w = 0; w < P.nw; w++) {
        const dem_wall& W = P.walls[w];
        const int wi = p * P.nw + w;
        bool contacting = A.Hr.wflag[wi] != 0;
        double FT0[3] = {0.0, 0.0, 0.0}, VT0[3] = {0.0, 0.0, 0.0};
        if (contacting) {
          const double2* v = A.Hr.wval + (size_t)wi * 3;
          double2 a = v[0], b = v[1], dd = v[2];
          FT0[0] = a.x; FT0[1] = a.y; FT0[2] = b.x;
          VT0[0] = b.y; VT0[1] = dd.x; VT0[2] = dd.y;
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
          common_calc(Rw, Nij, DispN, Vij, VijC, Delta, half_dt, contacting, FT0, VT0, pp.kn,
                      pp.yn, pp.kt, pp.yt, pp.mu_sq, o);
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
    }
    if (A.drag) {  // iForce = iForce + DragForce(iPart) (src/MForces.f90:316)
#pragma unroll
      for (int k = 0; k < 3; k++) iF[k] = iF[k] + A.drag[(size_t)3 * p + k];
    }
    // ---- the records p holds that no contact matched: kept if the sweep
    // did not visit the pair (its cells are not neighbours, or the partner
    // index lies past the last particle, a record that particle removal left
    // behind), else the contact ended (RemovePairContact) or the other
    // particle evaluated it
    if (update) {
      const int hc = A.Hr.cnt[p];
      for (int r = 0; r < hc; r++) {
        if (r < 32 && ((matched >> r) & 1u)) continue;
        const int q2 = A.Hr.key[hslot(A.Hr, p, r)];
        if (q2 >= A.n || !partner_adjacent(A, P, c, q2)) {
          if (hw_n < A.Hw.cap) {
            double ft[3], vt[3];
            hist_read(A.Hr, p, r, ft, vt);
            hist_write(A.Hw, p, hw_n, q2, ft, vt);
          } else {
            overflow = true;
          }
          hw_n++;
        }
      }
      A.Hw.cnt[p] = hw_n < A.Hw.cap ? hw_n : A.Hw.cap;
      if (hw_n > A.Hw.cap) overflow = true;
      need = hw_n;
    }
    // ---- Force and Torque in sweep order
    const InRec64* in = (const InRec64*)A.in_rec + p;
    const size_t st = (size_t)A.in_stride;
    double F[3] = {0.0, 0.0, 0.0}, T[3] = {0.0, 0.0, 0.0};
    fold_in_order(
        ni, key_p,
        [&](int e) {
          return (unsigned long long)__double_as_longlong(((const double*)(in + e * st))[0]);
        },
        [&]() {
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
    epilogue<EPI>(A, P, p, xp, Rp, vp, wp, acc, alp, c, d2);
  }
  if (WALLS && A.nw_max > 0) wall_partials(s_w, A.nw_max, A.wall_part, vblock);
  if (overflow) {
    atomicExch(&A.cnt->overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  publish_counts_block(A.cnt, update, 0u, 0u, n_wc, (unsigned)need, 0u);
  if (EPI != EPI_STORE) publish_disp_block(A.cnt, d2);
}

// (STRIDE: grid-stride over blocks of 128 particles, like k_test.  Register
// budget without walls: 6 blocks of 128 per SM, 80 registers; the predictor
// spills a little there and still runs faster than at 5 blocks, 135 against
// 146 us per launch at 1M spheres.)
template <bool PP, int EPI, bool WALLS, bool STRIDE>
__global__ void __launch_bounds__(128, WALLS ? 4 : 6) k_fold_fp64(PassArgs<double4, double2> A) {
  pass_kernel_entry();
  if (!STRIDE) {
    fold_fp64_body<PP, EPI, WALLS>(A, blockIdx.x);
    return;
  }
  const int nvb = (A.n + 127) / 128;
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
    fold_fp64_body<PP, EPI, WALLS>(A, vb);
    __syncthreads();  // the block's shared arrays are reused by the next block of particles
  }
}

// ---------------------------------------------------------------------------
// The persistent chunk kernel (FP64): npass force passes (prog[0..npass))
// in one cooperative launch of blocks of 128 threads, as many as fit on the
// GPU at once.  Every pass runs its four phases in the order of the
// separate kernels, each phase over the whole grid (the relink over all
// threads, the test and fold over blocks of 128 particles grid-stride, the
// pair kernel grid-stride over the contact list), with a grid-wide barrier
// after each.  The results are those of the separate kernels: the same
// bodies, the same contact list contents (its order is free), the same sums.
// Rows are read coherently (written by earlier passes of the same launch).
using ChunkPass64 = ChunkPass<double4, double2, NoView>;

template <bool PP, bool WALLS>
__global__ void __launch_bounds__(128, 4) k_chunk_fp64(const ChunkPass64* __restrict__ prog,
                                                       int npass, GridSync g) {
  __shared__ ChunkPass64 sp;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  for (int k = 0; k < npass; k++) {
    load_pass(sp, prog + k);
    const RelinkArgs& R = sp.rl;
    relink_body(R.PT, R.cellsys, R.L, R.par, R.n, R.update, R.stop_tag, R.cnt, tid, nthreads);
    if (!grid_sync(g)) return;
    const int nvb = (sp.t.n + 127) / 128;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) test_body<PP, false>(sp.t, vb);
    if (!grid_sync(g)) return;
    pair_fp64_body<PP>(sp.a, blockIdx.x, gridDim.x);
    if (!grid_sync(g)) return;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
      if (sp.epi == EPI_PREDICT) fold_fp64_body<PP, EPI_PREDICT, WALLS>(sp.a, vb);
      else fold_fp64_body<PP, EPI_CORRECT, WALLS>(sp.a, vb);
      __syncthreads();
    }
    if (!grid_sync(g)) return;  // (also: every block is done with sp)
  }
}

}  // namespace dem
