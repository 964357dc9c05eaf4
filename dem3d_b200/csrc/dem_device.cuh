// dem_device.cuh -- device-side data layout and the exact FP64 pair model.
//
// Everything in this header that touches a floating-point value reproduces the
// reference's Fortran expression operation by operation (the file is compiled
// with -fmad=false so that no multiply-add is fused), which is what lets the
// FP64 path match the CPU oracle bit for bit.
#pragma once
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dem3d_b200.h"

namespace dem {

constexpr int NCM = DEM_MAX_COMPONENTS;
constexpr int NWM = DEM_MAX_WALLS;

// Parameters resident in device memory (one copy per context).
struct DevParams {
  int nc, nw;
  int pbc[3];
  int nx, ny, nz, ncell;
  int nprev;
  int pad_;
  double lbox[3], inv_lbox[3], gravity[3];
  double nxbylx, nybyly, nzbylz, nxby2, nyby2, nzby2;
  double ab0, am0, ab[3], am[3];
  double max_min_dij_sq;  // largest MinDijSq of any pair (screening early-out)
  double vl_skin;         // candidate-list skin (added to MinDij)
  double vl_thr2;         // (skin/4)^2: displacement that forces a full rebuild
  double comp_radius[NCM], comp_inv_mass[NCM], comp_inv_inertia[NCM], comp_eff_mass[NCM];
  double min_dij[NCM * NCM], min_dij_sq[NCM * NCM];
  double kn[NCM * NCM], yn[NCM * NCM], kt[NCM * NCM], yt[NCM * NCM], mu_sq[NCM * NCM];
  double knw[NCM * NWM], ynw[NCM * NWM], ktw[NCM * NWM], ytw[NCM * NWM], muw_sq[NCM * NWM];
  double pp_mass_coef, pp_density, pp_fluid_density;
  double pp_kn, pp_kt, pp_gamma_n, pp_gamma_t, pp_mu_sq;
  double pp_knw[NWM], pp_ktw[NWM], pp_gamma_nw[NWM], pp_gamma_tw[NWM], pp_muw_sq[NWM];
  dem_wall walls[NWM];
};

// Per-particle master state in original index order (SoA, FP64).
struct StateArrays {
  double *px, *py, *pz, *vx, *vy, *vz, *wx, *wy, *wz, *ax, *ay, *az, *lx, *ly, *lz;
};

// Device counters (one cache line each is not needed: low traffic).
struct Counters {
  unsigned long long ncol;
  unsigned long long ncol_pending;  // Ncol of the last history-updating pass
  unsigned long long pair_contacts;
  unsigned long long wall_contacts;
  unsigned long long movers;
  unsigned long long escaped;
  int overflow;      // a particle needed more pair records than the capacity
  int need_capacity; // largest record count requested
  int abort;         // nonzero: later kernels of a captured sequence do nothing
  int abort_tag;     // 1 + index (within a captured chunk) of the failing step
  int list_overflow; // particles of this pass whose contact-list row overflowed
  int force_rebuild; // rebuild every candidate list in the next pass
  unsigned long long max_disp2;  // bits of the largest squared displacement since
                                 // the last full candidate-list rebuild
  double wall_fn[NWM];
};

// Contact history, one table per buffer: records owned by imin.
struct History {
  int* cnt;       // [n] records owned by particle
  int* key;       // [n*cap] partner (imax)
  double2* val;   // [n*cap*3] (ft.x,ft.y) (ft.z,vt.x) (vt.y,vt.z)
  int* wflag;     // [n*nw] wall record present
  double2* wval;  // [n*nw*3]
  int cap;
};

// Sorted (cell/traversal order) copies used by the force kernel.
struct SortedArrays {
  double4* pos;  // x, y, z, radius
  double4* v4;   // vx, vy, vz, wx
  double2* w2;   // wy, wz
  int* comp;     // component (table mode)
  int* orig;     // slot -> original index (also "order")
  int* cell;     // slot -> cell
};

constexpr int EPI_STORE = 0;    // store a/alpha into the target arrays only
constexpr int EPI_PREDICT = 1;  // MoveParticles predictor (pass 1)
constexpr int EPI_CORRECT = 2;  // MoveParticles corrector (pass 2)

struct RingMap {
  int phys[5];  // phys[k] = physical slot of logical ipc(k+1); phys[nprev] = spare
};

// Candidate lists, one row of KC entries per particle (indexed by original
// index): the particles within MinDij + skin, as original indices, first the
// "p is i" partners in the order of p's neighbour list, then the "p is j"
// partners in sweep order.  meta = (n1, n2 before p's own block, n2 after
// it, 0); n1 = -1 when the row overflowed or was never built (the force
// kernel then sweeps the cells itself for that particle).  A row stays valid
// while no cell of its 27-cell neighbourhood gains or loses a particle (the
// relative order of the others in the cell lists is unchanged) and no
// particle has moved skin/4 since the last full rebuild.
constexpr int KC = 32;
struct ContactLists {
  int* slot;          // [n*KC] candidate original indices
  int4* meta;         // [n]
  int* slot_of_orig;  // [n] traversal slot of every particle (this pass)
  double4* ref_pos;   // [n] positions at the last full rebuild
  unsigned char* dirty;   // [ncell] a particle entered/left the cell this pass
  unsigned char* repair;  // [ncell] rows of this cell's particles are rebuilt
  // this pass's exact contacts, filtered from the candidates: rows indexed by
  // traversal slot holding traversal slots, same order and meta layout
  int* xslot;   // [n*KC]
  int4* xmeta;  // [n]
};

struct ForceArgs {
  const DevParams* P;
  int n;
  SortedArrays S;
  const int* cell_start;
  const int* cell_of_orig;
  const int* cl_slot;
  const int4* cl_meta;
  const int* slot_of_orig;
  History Hr, Hw;
  int update;
  double half_dt;
  StateArrays tgt;   // where a/alpha go (EPI_STORE)
  StateArrays part;  // Particle
  StateArrays pred;  // Predicted
  double* ring;      // [(slot*9 + comp)*n + orig]
  RingMap rm;
  Counters* cnt;
  int tag;  // index of this step within a captured chunk
};

// ------------------------------------------------------------------------
// exact helpers (left-to-right sums as gfortran evaluates sum/dot_product)

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  double c = 0.0;
  c = c + a[0] * b[0];
  c = c + a[1] * b[1];
  c = c + a[2] * b[2];
  return c;
}
__device__ __forceinline__ double sumsq3(const double a[3]) {
  double c = 0.0;
  c = c + a[0] * a[0];
  c = c + a[1] * a[1];
  c = c + a[2] * a[2];
  return c;
}
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
  double c0 = a[1] * b[2] - a[2] * b[1];
  double c1 = a[2] * b[0] - a[0] * b[2];
  double c2 = a[0] * b[1] - a[1] * b[0];
  c[0] = c0;
  c[1] = c1;
  c[2] = c2;
}
// Fortran nint to default integer, then back to real(8)
__device__ __forceinline__ double fnint(double x) { return (double)(int)round(x); }

__device__ __forceinline__ void change_plane(const double V[3], const double N[3], double out[3]) {
  // ChangePlane, src/MForces.f90:391-406
  double d = dot3(V, N);
  double P[3];
#pragma unroll
  for (int k = 0; k < 3; k++) P[k] = V[k] - d * N[k];
  double NormSq = sumsq3(P);
  if (NormSq != 0.0) {
    double f = sqrt(sumsq3(V) / NormSq);
#pragma unroll
    for (int k = 0; k < 3; k++) out[k] = f * P[k];
  } else {
    out[0] = out[1] = out[2] = 0.0;
  }
}

struct PairPar {
  double min_dij, min_dij_sq, kn, yn, kt, yt, mu_sq;
};

// Result of CommonCalculations for one contact, in the orientation used.
struct ContactOut {
  double FN[3], FT[3], VT[3], N[3], NxFT[3];
};

// CommonCalculations (src/MForces.f90:339-387) given the contact geometry.
// Vij is the centre relative velocity (used only for the new-contact
// PartialDt), VijC the contact relative velocity.
__device__ __forceinline__ void common_calc(const double Rij[3], const double Nij[3],
                                            const double DispN[3], const double Vij[3],
                                            const double VijC[3], double DeltaDijSq,
                                            double half_dt, bool contacting,
                                            const double FT0[3], const double VT0in[3],
                                            double Kn, double Yn, double Kt, double Yt,
                                            double MuSq, ContactOut& o) {
  double VijN[3];
  double d = dot3(VijC, Nij);
#pragma unroll
  for (int k = 0; k < 3; k++) VijN[k] = d * Nij[k];
#pragma unroll
  for (int k = 0; k < 3; k++) o.VT[k] = VijC[k] - VijN[k];
#pragma unroll
  for (int k = 0; k < 3; k++) o.FN[k] = Kn * DispN[k] + Yn * VijN[k];
  if (contacting) {
    double VT0[3], cp[3], dD[3], dV[3];
    change_plane(VT0in, Nij, VT0);
#pragma unroll
    for (int k = 0; k < 3; k++) dD[k] = half_dt * (VT0[k] + o.VT[k]);
#pragma unroll
    for (int k = 0; k < 3; k++) dV[k] = o.VT[k] - VT0[k];
    change_plane(FT0, Nij, cp);
#pragma unroll
    for (int k = 0; k < 3; k++) o.FT[k] = cp[k] + Kt * dD[k] + Yt * dV[k];
  } else {
    double PartialDt;
    double VijSq = sumsq3(Vij);
    if (VijSq > 0.0) {
      double RijVij = dot3(Rij, Vij);
      double a = 2.0 * half_dt;
      double b = (RijVij + sqrt(RijVij * RijVij + VijSq * DeltaDijSq)) / VijSq;
      PartialDt = b < a ? b : a;
    } else {
      PartialDt = 0.0;
    }
    double f = Kt * PartialDt + Yt;
#pragma unroll
    for (int k = 0; k < 3; k++) o.FT[k] = f * o.VT[k];
  }
  double MuNormForceNSq = MuSq * sumsq3(o.FN);
  double NormForceTSq = sumsq3(o.FT);
  if (NormForceTSq > MuNormForceNSq) {
    double f = sqrt(MuNormForceNSq / NormForceTSq);
#pragma unroll
    for (int k = 0; k < 3; k++) o.FT[k] = f * o.FT[k];
  }
#pragma unroll
  for (int k = 0; k < 3; k++) o.N[k] = Nij[k];
  cross3(Nij, o.FT, o.NxFT);
}

// The particle-particle branch of ComputeAccelerations (src/MForces.f90:
// 230-252) for an overlapping pair, "i" = a, "j" = b, Rij = xb - xa (minimum
// image), already tested DeltaDijSq > 0.
__device__ __forceinline__ void pair_contact(const double Rij[3], double DijSq,
                                             double DeltaDijSq, const PairPar& pp,
                                             double Ra, const double va[3], const double wa[3],
                                             double Rb, const double vb[3], const double wb[3],
                                             double half_dt, bool contacting,
                                             const double FT0[3], const double VT0[3],
                                             ContactOut& o) {
  double Dij = sqrt(DijSq);
  double Nij[3], DispN[3], Vij[3], ws[3], cr[3], VijC[3];
#pragma unroll
  for (int k = 0; k < 3; k++) Nij[k] = Rij[k] / Dij;
  double dn = Dij - pp.min_dij;
#pragma unroll
  for (int k = 0; k < 3; k++) DispN[k] = dn * Nij[k];
#pragma unroll
  for (int k = 0; k < 3; k++) Vij[k] = vb[k] - va[k];
#pragma unroll
  for (int k = 0; k < 3; k++) ws[k] = Ra * wa[k] + Rb * wb[k];
  cross3(ws, Nij, cr);
#pragma unroll
  for (int k = 0; k < 3; k++) VijC[k] = Vij[k] - cr[k];
  common_calc(Rij, Nij, DispN, Vij, VijC, DeltaDijSq, half_dt, contacting, FT0, VT0, pp.kn,
              pp.yn, pp.kt, pp.yt, pp.mu_sq, o);
}

// Rectangle branch of Overlap (src/MConfig.f90:709-749).
__device__ __forceinline__ bool overlap_rect(const DevParams& P, const dem_wall& w,
                                             const double x[3], double Ri, double& Dij,
                                             double Nij[3], double Qji[3]) {
  double Rij[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    Rij[k] = w.position[k] - x[k];
    if (P.pbc[k]) Rij[k] = Rij[k] - P.lbox[k] * fnint(Rij[k] * P.inv_lbox[k]);
  }
  double AlphaN = dot3(Rij, w.n);
  double absAlphaN = fabs(AlphaN);
  bool ov = absAlphaN < Ri;
  if (ov) {
    double AlphaU = dot3(Rij, w.u);
    double AlphaW = dot3(Rij, w.w);
    double absAlphaU = fabs(AlphaU);
    double absAlphaW = fabs(AlphaW);
    ov = (absAlphaU < w.l1 + Ri) && (absAlphaW < w.l2 + Ri);
    if (ov) {
      if (absAlphaU < w.l1 && absAlphaW < w.l2) {
        double s = copysign(1.0, AlphaN);
#pragma unroll
        for (int k = 0; k < 3; k++) Nij[k] = s * w.n[k];
        Dij = absAlphaN;
#pragma unroll
        for (int k = 0; k < 3; k++) Qji[k] = -(AlphaU * w.u[k] + AlphaW * w.w[k]);
      } else {
        double mu = -w.l1, mw = -w.l2;
        AlphaU = AlphaU < w.l1 ? AlphaU : w.l1;
        AlphaU = mu > AlphaU ? mu : AlphaU;
        AlphaW = AlphaW < w.l2 ? AlphaW : w.l2;
        AlphaW = mw > AlphaW ? mw : AlphaW;
#pragma unroll
        for (int k = 0; k < 3; k++) Qji[k] = -(AlphaU * w.u[k] + AlphaW * w.w[k]);
#pragma unroll
        for (int k = 0; k < 3; k++) Nij[k] = Rij[k] + Qji[k];
        double DijSq = sumsq3(Nij);
        ov = DijSq < Ri * Ri;
        if (ov) {
          Dij = sqrt(DijSq);
#pragma unroll
          for (int k = 0; k < 3; k++) Nij[k] = Nij[k] / Dij;
        }
      }
    }
  }
  return ov;
}

// CurrentCell3D (src/MCells.f90:498-513), 0-based.
__device__ __forceinline__ int current_cell(const DevParams& P, double x, double y, double z) {
  int ix = (int)(P.nxbylx * x + P.nxby2);
  int iy = (int)(P.nybyly * y + P.nyby2);
  int iz = (int)(P.nzbylz * z + P.nzby2);
  ix = ix < P.nx - 1 ? ix : P.nx - 1;
  iy = iy < P.ny - 1 ? iy : P.ny - 1;
  iz = iz < P.nz - 1 ? iz : P.nz - 1;
  ix = ix > 0 ? ix : 0;
  iy = iy > 0 ? iy : 0;
  iz = iz > 0 ? iz : 0;
  return ix + (iy + iz * P.ny) * P.nx;
}

// Are two cells neighbours in the sweep sense (same cell, or one in the
// other's half-shell list)?  With >= 3 cells along every periodic axis this
// is plain adjacency with wrap-around (VerifyPBC/ApplyPBC, src/MCells.f90:
// 1030-1052).
__device__ __forceinline__ bool cells_adjacent(const DevParams& P, int a, int b) {
  int ax = a % P.nx, ay = (a / P.nx) % P.ny, az = a / (P.nx * P.ny);
  int bx = b % P.nx, by = (b / P.nx) % P.ny, bz = b / (P.nx * P.ny);
  int d[3] = {bx - ax, by - ay, bz - az};
  int N[3] = {P.nx, P.ny, P.nz};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    int x = d[k] < 0 ? -d[k] : d[k];
    if (x > 1 && !(P.pbc[k] && x == N[k] - 1)) return false;
  }
  return true;
}

// axis helper: neighbour offsets of a cell coordinate, trimmed like VerifyPBC
__device__ __forceinline__ void axis_range(int i, int N, int pbc, int& lo, int& hi) {
  lo = -1;
  hi = 1;
  if (!pbc) {
    if (i == 0) lo = 0;
    if (i == N - 1) hi = 0;
  }
}
__device__ __forceinline__ int axis_wrap(int j, int N, int pbc) {
  if (pbc) {
    if (j == N) j = 0;
    if (j == -1) j = N - 1;
  }
  return j;
}
// offsets of one axis in ascending order of the wrapped cell coordinate
__device__ __forceinline__ int axis_sorted(int i, int N, int pbc, int off[3]) {
  int lo, hi;
  axis_range(i, N, pbc, lo, hi);
  int m = 0;
  if (pbc && i == 0) {  // -1 wraps to N-1 (largest)
    off[m++] = 0;
    off[m++] = 1;
    off[m++] = -1;
  } else if (pbc && i == N - 1) {  // +1 wraps to 0 (smallest)
    off[m++] = 1;
    off[m++] = -1;
    off[m++] = 0;
  } else {
    for (int k = lo; k <= hi; k++) off[m++] = k;
  }
  return m;
}


// ------------------------------------------------------------------------
// the reference's cell sweep (ComputeAccelerations, src/MForces.f90:173-324)
// seen from one particle p at traversal slot s of cell c = (cx, cy, cz)

// Loop 1 ("p is i"): the neighbour list of p's block is the rest of its own
// cell, then the half-shell cells in the order of the FirstNeighbour list,
// which AddAllNeighbours3D (src/MCells.f90:424-476) builds by prepending in
// kz, ky, kx loop order with kx + Nx*(ky + Ny*kz) > 0 (so: reverse order).
template <class Visit>
__device__ __forceinline__ void sweep_as_i(const DevParams& P, const int* __restrict__ cs, int s,
                                           int c, int cx, int cy, int cz, Visit&& visit) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int e = cs[c + 1];
  for (int t = s + 1; t < e; t++) visit(t);
  int xi, xf, yi, yf, zi, zf;
  axis_range(cx, nx, P.pbc[0], xi, xf);
  axis_range(cy, ny, P.pbc[1], yi, yf);
  axis_range(cz, nz, P.pbc[2], zi, zf);
  for (int kz = zf; kz >= zi; kz--) {
    const int jz = axis_wrap(cz + kz, nz, P.pbc[2]);
    for (int ky = yf; ky >= yi; ky--) {
      const int jy = axis_wrap(cy + ky, ny, P.pbc[1]);
      for (int kx = xf; kx >= xi; kx--) {
        if (kx + nx * (ky + ny * kz) <= 0) continue;
        const int jx = axis_wrap(cx + kx, nx, P.pbc[0]);
        const int jc = jx + nx * (jy + ny * jz);
        const int b = cs[jc], e2 = cs[jc + 1];
        for (int t = b; t < e2; t++) visit(t);
      }
    }
  }
}

// Loop 2 ("p is j"): every particle q whose block lists p -- the earlier
// members of p's cell and the members of the cells whose half shell holds
// p's cell -- in the order the sweep reaches q (ascending cell index, then
// list order); own() is called where p's own block ends (Force(i) =
// Force(i) + iForce, src/MForces.f90:319-320).
template <class Visit, class Own>
__device__ __forceinline__ void sweep_as_j(const DevParams& P, const int* __restrict__ cs, int s,
                                           int c, int cx, int cy, int cz, Visit&& visit,
                                           Own&& own) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int ox[3], oy[3], oz[3];
  const int mx = axis_sorted(cx, nx, P.pbc[0], ox);
  const int my = axis_sorted(cy, ny, P.pbc[1], oy);
  const int mz = axis_sorted(cz, nz, P.pbc[2], oz);
  for (int a = 0; a < mz; a++) {
    const int dz = oz[a];
    const int jz = axis_wrap(cz + dz, nz, P.pbc[2]);
    for (int b = 0; b < my; b++) {
      const int dy = oy[b];
      const int jy = axis_wrap(cy + dy, ny, P.pbc[1]);
      for (int d = 0; d < mx; d++) {
        const int dx = ox[d];
        if (dx == 0 && dy == 0 && dz == 0) {
          for (int t = cs[c]; t < s; t++) visit(t);
          own();
          continue;
        }
        // p's cell is in the half shell of the cell at offset (dx,dy,dz)
        if (-dx + nx * (-dy + ny * -dz) <= 0) continue;
        const int jx = axis_wrap(cx + dx, nx, P.pbc[0]);
        const int jc = jx + nx * (jy + ny * jz);
        const int b0 = cs[jc], e2 = cs[jc + 1];
        for (int t = b0; t < e2; t++) visit(t);
      }
    }
  }
}

// The same two sweeps, also telling the visitor how the neighbour cell was
// reached: w = (+1 | -1 | 0) per axis when the cell index wrapped past the
// upper | lower edge of a periodic axis.
__device__ __forceinline__ int axis_wrap_w(int j, int N, int pbc, int& w) {
  w = 0;
  if (pbc) {
    if (j == N) { j = 0; w = 1; }
    if (j == -1) { j = N - 1; w = -1; }
  }
  return j;
}

template <class Visit>
__device__ __forceinline__ void sweep_as_i_w(const DevParams& P, const int* __restrict__ cs,
                                             int s, int c, int cx, int cy, int cz,
                                             Visit&& visit) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int e = cs[c + 1];
  for (int t = s + 1; t < e; t++) visit(t, 0, 0, 0);
  int xi, xf, yi, yf, zi, zf;
  axis_range(cx, nx, P.pbc[0], xi, xf);
  axis_range(cy, ny, P.pbc[1], yi, yf);
  axis_range(cz, nz, P.pbc[2], zi, zf);
  for (int kz = zf; kz >= zi; kz--) {
    int wz;
    const int jz = axis_wrap_w(cz + kz, nz, P.pbc[2], wz);
    for (int ky = yf; ky >= yi; ky--) {
      int wy;
      const int jy = axis_wrap_w(cy + ky, ny, P.pbc[1], wy);
      for (int kx = xf; kx >= xi; kx--) {
        if (kx + nx * (ky + ny * kz) <= 0) continue;
        int wx;
        const int jx = axis_wrap_w(cx + kx, nx, P.pbc[0], wx);
        const int jc = jx + nx * (jy + ny * jz);
        const int b = cs[jc], e2 = cs[jc + 1];
        for (int t = b; t < e2; t++) visit(t, wx, wy, wz);
      }
    }
  }
}

template <class Visit, class Own>
__device__ __forceinline__ void sweep_as_j_w(const DevParams& P, const int* __restrict__ cs,
                                             int s, int c, int cx, int cy, int cz, Visit&& visit,
                                             Own&& own) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int ox[3], oy[3], oz[3];
  const int mx = axis_sorted(cx, nx, P.pbc[0], ox);
  const int my = axis_sorted(cy, ny, P.pbc[1], oy);
  const int mz = axis_sorted(cz, nz, P.pbc[2], oz);
  for (int a = 0; a < mz; a++) {
    const int dz = oz[a];
    int wz;
    const int jz = axis_wrap_w(cz + dz, nz, P.pbc[2], wz);
    for (int b = 0; b < my; b++) {
      const int dy = oy[b];
      int wy;
      const int jy = axis_wrap_w(cy + dy, ny, P.pbc[1], wy);
      for (int d = 0; d < mx; d++) {
        const int dx = ox[d];
        if (dx == 0 && dy == 0 && dz == 0) {
          for (int t = cs[c]; t < s; t++) visit(t, 0, 0, 0);
          own();
          continue;
        }
        if (-dx + nx * (-dy + ny * -dz) <= 0) continue;
        int wx;
        const int jx = axis_wrap_w(cx + dx, nx, P.pbc[0], wx);
        const int jc = jx + nx * (jy + ny * jz);
        const int b0 = cs[jc], e2 = cs[jc + 1];
        for (int t = b0; t < e2; t++) visit(t, wx, wy, wz);
      }
    }
  }
}

// The two sweeps as slot ranges: emit(b, e, wx, wy, wz) per visited cell
// (own cell: the part after / before p), own() right after p's own range in
// loop 2.
template <class Emit>
__device__ __forceinline__ void sweep_cells_as_i(const DevParams& P, const int* __restrict__ cs,
                                                 int s, int c, int cx, int cy, int cz,
                                                 Emit&& emit) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  emit(s + 1, cs[c + 1], 0, 0, 0);
  int xi, xf, yi, yf, zi, zf;
  axis_range(cx, nx, P.pbc[0], xi, xf);
  axis_range(cy, ny, P.pbc[1], yi, yf);
  axis_range(cz, nz, P.pbc[2], zi, zf);
  for (int kz = zf; kz >= zi; kz--) {
    int wz;
    const int jz = axis_wrap_w(cz + kz, nz, P.pbc[2], wz);
    for (int ky = yf; ky >= yi; ky--) {
      int wy;
      const int jy = axis_wrap_w(cy + ky, ny, P.pbc[1], wy);
      for (int kx = xf; kx >= xi; kx--) {
        if (kx + nx * (ky + ny * kz) <= 0) continue;
        int wx;
        const int jx = axis_wrap_w(cx + kx, nx, P.pbc[0], wx);
        const int jc = jx + nx * (jy + ny * jz);
        emit(cs[jc], cs[jc + 1], wx, wy, wz);
      }
    }
  }
}

template <class Emit, class Own>
__device__ __forceinline__ void sweep_cells_as_j(const DevParams& P, const int* __restrict__ cs,
                                                 int s, int c, int cx, int cy, int cz, Emit&& emit,
                                                 Own&& own) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  int ox[3], oy[3], oz[3];
  const int mx = axis_sorted(cx, nx, P.pbc[0], ox);
  const int my = axis_sorted(cy, ny, P.pbc[1], oy);
  const int mz = axis_sorted(cz, nz, P.pbc[2], oz);
  for (int a = 0; a < mz; a++) {
    const int dz = oz[a];
    int wz;
    const int jz = axis_wrap_w(cz + dz, nz, P.pbc[2], wz);
    for (int b = 0; b < my; b++) {
      const int dy = oy[b];
      int wy;
      const int jy = axis_wrap_w(cy + dy, ny, P.pbc[1], wy);
      for (int d = 0; d < mx; d++) {
        const int dx = ox[d];
        if (dx == 0 && dy == 0 && dz == 0) {
          emit(cs[c], s, 0, 0, 0);
          own();
          continue;
        }
        if (-dx + nx * (-dy + ny * -dz) <= 0) continue;
        int wx;
        const int jx = axis_wrap_w(cx + dx, nx, P.pbc[0], wx);
        const int jc = jx + nx * (jy + ny * jz);
        emit(cs[jc], cs[jc + 1], wx, wy, wz);
      }
    }
  }
}

// Minimum image of one component exactly as Rij(k) - Lbox(k)*nint(Rij(k)*
// InvLbox(k)) (src/MForces.f90:212-214), given the image n the cell sweep
// implies: if |Rij - n*L| < 0.49*L then nint(Rij/L) == n (the margin covers
// the rounding of Rij*InvLbox), so Rij - L*n is the reference's value bit for
// bit; otherwise the formula itself is evaluated.
__device__ __forceinline__ double min_image(double r, int pbc, double L, double iL, int n) {
  if (!pbc) return r;
  const double d = r - L * (double)n;
  if (fabs(d) < 0.49 * L) return d;
  return r - L * fnint(r * iL);
}

// Loop 1 / loop 2 driven by the screening kernel's contact list when the
// particle's row did not overflow, else by the full sweep (same order).
// Full candidate-list rebuild due in this pass: requested by the host (new
// state or cells) or some particle moved more than skin/4 since the last one.
__device__ __forceinline__ bool rebuild_due(const DevParams& P, const Counters* cnt) {
  return cnt->force_rebuild != 0 ||
         __longlong_as_double((long long)cnt->max_disp2) > P.vl_thr2;
}

// Called by one thread of the force kernel (after the screening kernel has
// read the trigger): the rebuild of this pass is done.
__device__ __forceinline__ void clear_rebuild_trigger(const ForceArgs& A) {
  if (rebuild_due(*A.P, A.cnt)) {
    A.cnt->force_rebuild = 0;
    A.cnt->max_disp2 = 0ull;
  }
}

template <bool SWEEP, class Visit>
__device__ __forceinline__ void walk_as_i(const ForceArgs& A, int4 meta, int s, int orig, int c,
                                          int cx, int cy, int cz, Visit&& visit) {
  if (!SWEEP) {
    const int* l = A.cl_slot + (size_t)s * KC;
    for (int k = 0; k < meta.x; k++) visit(l[k]);
  } else {
    sweep_as_i(*A.P, A.cell_start, s, c, cx, cy, cz, visit);
  }
}

template <bool SWEEP, class Visit, class Own>
__device__ __forceinline__ void walk_as_j(const ForceArgs& A, int4 meta, int s, int orig, int c,
                                          int cx, int cy, int cz, Visit&& visit, Own&& own) {
  if (!SWEEP) {
    const int* l = A.cl_slot + (size_t)s * KC + meta.x;
    for (int k = 0; k < meta.y; k++) visit(l[k]);
    own();
    for (int k = meta.y; k < meta.y + meta.z; k++) visit(l[k]);
  } else {
    sweep_as_j(*A.P, A.cell_start, s, c, cx, cy, cz, visit, own);
  }
}

}  // namespace dem
