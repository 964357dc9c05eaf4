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
// (The body of k_relink; tid / nthreads: this thread's index in the grid and
// the grid's thread count, so that a persistent kernel can run it too.)
__device__ __forceinline__ void relink_body(const DevParams* __restrict__ PT,
                                            const int* __restrict__ cellsys, const CellLists& L,
                                            int par, int n, int update, int stop_tag,
                                            Counters* cnt, int tid, int nthreads) {
  if (cnt->abort) return;
  // inside a captured chunk, particles that left the box in the last step
  // stop the chunk before this step (the host runs UpdateParticleList); the
  // count is final here (written by the previous kernel), so every block
  // takes the same branch
  if (stop_tag >= 0 && cnt->escaped != 0ull) {
    if (tid == 0) {
      cnt->escape_stop = 1;
      set_abort(cnt, stop_tag);
    }
    return;
  }
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
    cnt->n_contacts = 0;  // the contact list of this pass starts empty
    if (update) {
      cnt->need_capacity = 0;
      cnt->need_in = 0;
      cnt->need_cl = 0;
    } else {
      cnt->escaped = 0ull;  // escapes are counted by the current step's corrector
    }
    const double d = (double)__uint_as_float(cnt->disp_max);
    cnt->disp_max = 0u;
    const double acc = cnt->disp_acc + d;
    const int full = cnt->force_full != 0 || !(acc <= P.vl_thr);
    cnt->full_due = full;
    cnt->disp_acc = full ? 0.0 : acc;
    if (full) cnt->force_full = 0;
  }
  const int m = cnt->n_dirty[par];
  const int stamp = cnt->pass_id + 1;  // fold kernels advance pass_id, not this one
  const int* __restrict__ cell_new = L.cell[par];
  for (int i = tid; i < m; i += nthreads) {
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
    // 3. the rows of every particle around c are rebuilt in this pass (by
    // the test kernel): the 27 cells are stamped with the pass
    const DevParams& P = sys_params(PT, cellsys, c);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int cl = c - P.coff;
    const int cx = cl % nx, cy = (cl / nx) % ny, cz = cl / (nx * ny);
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const int jx = cx + o % 3 - 1, jy = cy + (o / 3) % 3 - 1, jz = cz + o / 9 - 1;
      const bool ok = (P.pbc[0] || (jx >= 0 && jx < nx)) && (P.pbc[1] || (jy >= 0 && jy < ny)) &&
                      (P.pbc[2] || (jz >= 0 && jz < nz));
      if (ok)
        L.rflag[P.coff + axis_wrap(jx, nx, P.pbc[0]) +
                nx * (axis_wrap(jy, ny, P.pbc[1]) + ny * axis_wrap(jz, nz, P.pbc[2]))] = stamp;
    }
  }
}

__global__ void k_relink(const DevParams* __restrict__ PT, const int* __restrict__ cellsys,
                         CellLists L, int par, int n, int update, int stop_tag, Counters* cnt) {
  relink_body(PT, cellsys, L, par, n, update, stop_tag, cnt, blockIdx.x * blockDim.x + threadIdx.x,
              gridDim.x * blockDim.x);
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

// Arguments of the test kernel (the same for both precisions).
struct TestArgs {
  const DevParams* P;
  const int* sysid;
  int n;
  const int* cell_cur;  // cell of every particle in this pass
  CellLists L;
  Rows R;
  const double4* X;
  const int* comp;
  const int* cand;
  const int* meta;
  int2* clist;
  int* cstart;
  int* ccount;
  int cl_cap;
  Counters* cnt;
  int tag;
};

// First, the candidate rows of the warp's particles that this pass rebuilds
// (every row on a full rebuild, else the rows of the particles whose cell the
// relink stamped with this pass) are built, one particle at a time by the
// whole warp (build_row).  (No block barriers: every warp runs on its own.
// The pass's contact count and the list length it needs come from the pair
// kernel, or from here when the list overflows.)
// (The body of k_test for block `vblock`, so that a persistent kernel can
// run it too.)
template <bool PP>
__device__ __forceinline__ void test_body(const TestArgs& A, int vblock) {
  if (A.cnt->abort) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int p0 = vblock * blockDim.x + threadIdx.x;
  const bool valid = p0 < A.n;
  const int p = valid ? p0 : 0;
  const int n = A.n;
  {
    const bool full = A.cnt->full_due != 0;
    const int stamp = A.cnt->pass_id + 1;
    const int cp0 = A.cell_cur[p];
    unsigned todo = __ballot_sync(FULL, valid && (full || A.L.rflag[cp0] == stamp));
    while (todo) {
      const int l = __ffs(todo) - 1;
      todo &= todo - 1u;
      const int pl = __shfl_sync(FULL, p, l);
      const int cl = __shfl_sync(FULL, cp0, l);
      build_row<PP>(sys_params(A.P, A.sysid, pl), n, pl, cl, A.X, A.comp, A.L.head, A.L.next,
                    A.R, A.cnt, A.tag);
    }
    __syncwarp();  // the rows written by the warp are visible to their owners
  }
  // the first candidates are read before the row length is known (every
  // row holds at least 4 entries' room)
  int q0[4];
#pragma unroll
  for (int u = 0; u < 4; u++) q0[u] = __ldg(A.cand + (size_t)u * n + p);
  const DevParams& P = sys_params(A.P, A.sysid, p);
  const double4 p4 = A.X[p];
  const int cp = PP ? 0 : A.comp[p];
  const int m = valid ? (A.meta[p] & META_MASK) : 0;
  // contact bit masks of the row, 64 candidates per window (windows past
  // the first only for rows longer than 64)
  unsigned long long mask0 = 0ull;
  unsigned long long more[(KC_MAX + 1) / 64 - 1];
  int total = 0;
  for (int base = 0; base < m; base += 64) {
    unsigned long long mask = 0ull;
    const int end = m < base + 64 ? m : base + 64;
#pragma unroll 1
    for (int b = base; b < end; b += 4) {
      int q[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        q[u] = b + u < end ? (b == 0 ? q0[u] : __ldg(A.cand + (size_t)(b + u) * n + p)) : -1;
      double4 xq[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        xq[u] = q[u] >= 0 ? A.X[q[u]] : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (q[u] < 0) continue;
        double Rij[3] = {xq[u].x - p4.x, xq[u].y - p4.y, xq[u].z - p4.z};
#pragma unroll
        for (int k = 0; k < 3; k++) Rij[k] = min_image_exact(Rij[k], P.box, k);
        const double DijSq = sumsq3(Rij);
        const int cq = PP ? 0 : A.comp[q[u]];
        if (Material<PP>::min_dij_sq(P, cp, p4.w, cq, xq[u].w) - DijSq > 0.0)
          mask |= 1ull << (b + u - base);
      }
    }
    total += __popcll(mask);
    if (base == 0) mask0 = mask;
    else more[base / 64 - 1] = mask;
  }
  // one allocation per warp; a particle's contacts are contiguous
  int incl = total;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const int wsum = __shfl_sync(FULL, incl, 31);
  int wbase = 0;
  if (lane == 31 && wsum > 0) wbase = atomicAdd(&A.cnt->n_contacts, wsum);
  wbase = __shfl_sync(FULL, wbase, 31);
  const int start = wbase + incl - total;
  if (valid) {
    A.cstart[p] = start;
    A.ccount[p] = total;
  }
  if (start + total > A.cl_cap) {
    // the list is grown and the pass launched again
    atomicMax(&A.cnt->need_cl, start + total);
    atomicExch(&A.cnt->cl_overflow, 1);
    set_abort(A.cnt, A.tag);
  } else if (total > 0) {
    int s = start;
    for (int base = 0; base < m; base += 64) {
      unsigned long long mask = base == 0 ? mask0 : more[base / 64 - 1];
      while (mask) {
        const int k = base + __ffsll((long long)mask) - 1;
        mask &= mask - 1ull;
        A.clist[s++] = make_int2(p, __ldg(A.cand + (size_t)k * n + p));
      }
    }
  }
}

template <bool PP>
__global__ void __launch_bounds__(128) k_test(TestArgs A) {
  test_body<PP>(A, blockIdx.x);
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
  const bool valid = p0 < A.n;
  const int p = valid ? p0 : 0;
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
        if (q2 >= A.n || !cells_adjacent(P, c, A.cell_cur[q2])) {
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

template <bool PP, int EPI, bool WALLS>
__global__ void __launch_bounds__(128, WALLS ? 4 : 5) k_fold_fp64(PassArgs<double4, double2> A) {
  fold_fp64_body<PP, EPI, WALLS>(A, blockIdx.x);
}

}  // namespace dem
