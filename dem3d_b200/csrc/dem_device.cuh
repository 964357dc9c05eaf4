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

// Periodic box of a system.
struct Box {
  double lbox[3], inv_lbox[3];
  double half_lim[3];  // 0.49 lbox: |r| below it has nint(r/L) = 0 exactly
  int pbc[3];
};

// Minimum image of one component, Rij(k) - Lbox(k)*nint(Rij(k)*InvLbox(k))
// (src/MForces.f90:212-214), bit for bit: when |r| < 0.49 L the nint is 0
// and the expression is r itself, so the formula is only evaluated for
// pairs that straddle the periodic boundary.
__device__ __forceinline__ double min_image_exact(double r, const Box& B, int k) {
  if (B.pbc[k] && !(fabs(r) < B.half_lim[k]))
    r = r - B.lbox[k] * (double)(int)round(r * B.inv_lbox[k]);
  return r;
}

// Parameters of one system, resident in device memory (a context holds a
// table of them: one per independent system of an ensemble, all sharing the
// integrator settings).  Cells and particles of system s are numbered
// globally from coff / poff.
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
  double cutoff;          // CutOff = 2 * largest radius (cell size floor)
  double vl_skin;         // candidate-row skin (added to MinDij)
  double vl_thr;          // accumulated displacement bound that forces a full rebuild
  double inv_nx, inv_ny;  // 1/Nx, 1/Ny (cell coordinates without integer division)
  Box box;                // lbox, inv_lbox, pbc again, with the minimum-image shortcut bound
  int coff, poff, np;     // first cell, first particle, particles of this system
  int sys;                // index of this system
  // cells whose particles this context advances: [slab_c0, slab_c1), a
  // range of whole z-layers (cells are numbered x + Nx*(y + Ny*z)); every
  // cell of the system unless the context is one slab of a decomposition
  int slab_c0, slab_c1;
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

// Device counters and status words of a context.
struct Counters {
  unsigned long long ncol;
  unsigned long long ncol_pending;  // Ncol of the last history-updating pass
  unsigned long long pair_contacts;
  unsigned long long wall_contacts;
  unsigned long long movers;          // particles that changed cell in the last relink
  unsigned long long escaped;
  unsigned long long movers_pending;  // particles pushed as arrivals for the next relink
  int overflow;      // a particle needed more pair records than the capacity
  int need_capacity; // largest record count requested
  int abort;         // nonzero: later kernels of a captured sequence do nothing
  int abort_tag;     // 1 + 2*(step within a captured chunk) + pass of the failing pass
  int n_dirty[2];    // cells in dirty list b (transition to cell assignment b)
  int n_repair;      // cells whose particles' candidate rows are rebuilt this pass
  int full_due;      // this pass rebuilds every candidate row
  int force_full;    // the next pass must rebuild every row (new state, grown rows)
  int row_overflow;  // a candidate row needed more than kc entries
  int need_kc;       // longest candidate row requested
  int in_overflow;   // a particle received more "j" contact results than fit
  int need_in;       // most "j" contact results of one particle in the last step
  int cl_overflow;   // the pass found more contacts than the contact list holds
  int need_cl;       // most contacts of one pass in the last step
  int n_contacts;    // length of this pass's contact list
  int list_error;    // a cell-list walk exceeded its bound (corrupt lists)
  int nonfinite;     // a particle position became NaN or infinite
  unsigned int disp_max;  // FP32 bits (rounded up) of the largest displacement of one pass
  double disp_acc;   // sum of disp_max since the last full rebuild
  int escape_stop;   // a captured chunk stopped before a step: particles had left the box
  int pass_id;       // force passes completed; a cell stamped pass_id + 1 has rows to rebuild
  int barrier_timeout;  // a grid-wide barrier of a persistent launch gave up waiting
  int n_mlist[2];  // entries of CellLists::mlist recorded by the relinks of even / odd stamps
};

// Contact history, one table per buffer, stored slot major (record r of
// particle i at r*n + i), so that the first records of neighbouring particles
// share cache lines.  The record of a pair (the reference's node keyed by
// (imin, imax), src/MContacts.f90:329-437) sits in the table of one of its
// two particles: after a history-updating pass, the one that evaluated the
// contact as "i"; after an import or before a removal, imin.  A lookup tries
// the evaluating particle's table, then the partner's; a pair has at most one
// record.
struct History {
  int* cnt;       // [n] records held by particle
  int* key;       // [cap*n] partner
  double2* val;   // [cap*n*3] (ft.x,ft.y) (ft.z,vt.x) (vt.y,vt.z)
  int* wflag;     // [n*nw] wall record present
  double2* wval;  // [n*nw*3]
  int cap;
  int n;          // particles (rows of every slot)
};
__device__ __host__ __forceinline__ size_t hslot(const History& H, int i, int r) {
  return (size_t)r * (size_t)H.n + (size_t)i;
}

// Traversal-order arrays of the counting sort that builds the initial cell
// lists (DistributeParticles3D) and serves the allocation-free entry point.
struct SortedArrays {
  int* orig;     // slot -> original index (also "order")
  int* cell;     // slot -> cell
};

constexpr int EPI_STORE = 0;    // store a/alpha into the target arrays only
constexpr int EPI_PREDICT = 1;  // MoveParticles predictor (pass 1)
constexpr int EPI_CORRECT = 2;  // MoveParticles corrector (pass 2)

struct RingMap {
  int phys[5];  // phys[k] = physical slot of logical ipc(k+1); phys[nprev] = spare
};

// The reference's linked cell lists (FirstParticle/NextParticle of MCells),
// kept in its order: a cell's list holds the particles that entered it in
// the last redistribution in decreasing index, then the others in their
// previous order.  Between passes only the cells that gained or lost a
// particle are relinked.
struct CellLists {
  int* head;      // [ncell] first particle of the cell's list, -1 = empty
  int* next;      // [n] next particle of the same list, -1 = end
  int* cell[2];   // [n] cell of every particle under assignment b
  int* arr_head;  // [ncell] particles entering the cell at the next relink, -1 = none
  int* arr_next;  // [n]
  int* mflag;     // [n] particle already pushed as an arrival
  int* mnext;     // [n] a mover's successor in the list it leaves
  int* dflag;     // [ncell] cell already in a dirty list
  int* rflag;     // [ncell] stamp: pass_id + 1 when the cell's rows are rebuilt in that pass
  int* dlist[2];  // [ncell] cells that gain or lose a particle on the way to assignment b
  int* rlist;     // [ncell] (unused: the stamps replace a repair list)
  // the particles that left or entered a cell in the relink of the pass
  // with stamp s: mlist[(s & 1) * mcap + k], k < Counters::n_mlist[s & 1]
  // (more than mcap: not all recorded); dstamp[c] = s when that relink
  // rewrote cell c's list
  int* mlist;
  int* dstamp;
  int mcap;
  // each cell's list copied in order into SLOT_CAP slots ([cell*SLOT_CAP +
  // k]) and its length (slot_n > SLOT_CAP: only the first SLOT_CAP are
  // copied; -1: not current): the candidate rows read a neighbour cell with
  // independent loads instead of walking its links one after the other
  int* slot;
  int* slot_n;
  // the reference's index of the particle stored at each place, when the
  // storage is kept in cell order (the relink orders arrivals by it); NULL:
  // stored in the reference's order
  const int* gid;
};
constexpr int SLOT_CAP = 32;
// movers one relink records for the test kernel's row check (more: every
// stamped row is rebuilt)
constexpr int MLIST_CAP = 4096;

// Candidate rows, column-major (cand[k*n + p]): the particles within
// MinDij + skin of particle p that the sweep visits with p as "i" (loop jj
// of src/MForces.f90:199-272: the rest of p's cell list, then the half-shell
// cells in FirstNeighbour order), as original indices, in that order.
// meta = the row length; rank = p's position in its cell's list, which with
// the cell gives the place of p's block in the sweep.  A row stays valid
// while no cell of its 27-cell neighbourhood gains or loses a particle and
// no particle has moved skin/2 since the last full rebuild.
struct Rows {
  int* cand;
  int* meta;
  int* rank;
  int kc;
};
constexpr int META_BITS = 10;
constexpr int META_MASK = (1 << META_BITS) - 1;
constexpr int KC_MAX = META_MASK;

// Place of particle i's block in ComputeAccelerations' sweep (cells in
// increasing index, then the cell's list order): contributions to a
// particle's Force and Torque arrive in the order of these keys.
__device__ __forceinline__ unsigned long long sweep_key(int cell, int rank) {
  return ((unsigned long long)(unsigned)cell << 32) | (unsigned)rank;
}

// Contact results handed from the pair kernel to the fold kernel.
//  - "j" side: what particle j adds for one contact that particle i
//    evaluated (Force(j) - FN - FT, Torque(j) + Rj*(Nij x FT)), with i's sweep
//    key; record s of particle j at s*stride + j.
//  - "i" side: what particle i adds for the same contact (iForce + FN + FT,
//    iTorque + (Ri*Nij) x FT), at the contact's place in the contact list.
struct alignas(16) InRec64 {
  double2 a, b, c, d, e;  // (key, FN.x) (FN.y, FN.z) (FT.x, FT.y) (FT.z, NxFT.x) (NxFT.y, NxFT.z)
};
struct alignas(16) InRec32 {
  float4 a, b, c;  // (key lo, key hi, FN.x, FN.y) (FN.z, FT.xyz) (NxFT.xyz, 0)
};
struct alignas(16) IRec64 {
  double2 a, b, c, d, e;  // (FN.x, FN.y) (FN.z, FT.x) (FT.y, FT.z) (tq.x, tq.y) (tq.z, 0)
};
struct alignas(16) IRec32 {
  float4 a, b, c;  // (FN.xyz, FT.x) (FT.yz, tq.xy) (tq.z, 0, 0, 0); FT = FT + FT remainder
};

// Arguments of the two kernels of a force pass (contact kernel, fold
// kernel).  V4/W2 are the velocity copies the pass reads for partners
// (double in FP64 mode, float in mixed mode).
template <class V4, class W2>
struct PassArgs {
  const DevParams* P;   // system table
  const int* sysid;     // system of every particle (NULL: one system)
  int n;
  const double4* X;   // this pass's positions (x, y, z, R) by original index
  const V4* v4;       // vx, vy, vz, wx
  const W2* w2;       // wy, wz
  const int* comp;
  const int* cand;
  const int* meta;
  const int* cell_cur;  // cell of every particle in this pass
  CellLists L;          // next assignment: L.cell[par_nxt]
  int par_nxt;
  History Hr, Hw;
  int update;
  double half_dt;
  StateArrays tgt;   // where a/alpha go (EPI_STORE)
  StateArrays part;  // Particle
  StateArrays pred;  // Predicted
  double4* Xn;       // positions of the next pass (written by the epilogue)
  V4* v4n;
  W2* w2n;
  double* ring;      // [(slot*9 + comp)*n + orig]
  RingMap rm;
  Counters* cnt;
  int tag;  // 2*(step within a captured chunk) + pass
  const double* drag;  // [3n] fluid drag of every sphere (NULL: no fluid)
  // 1: the AB predictor leaves out the values that only export calls read
  // and that other arrays of the step already hold: Particle a, alpha (the
  // ring slot it writes holds them), Predicted x (the next pass's position
  // copy) and, with FP64 velocity copies, Predicted v, w.  The host writes
  // them back (k_settle_state) before a call reads or changes particle data.
  int lazy;
  // EPI_PREDICT/EPI_CORRECT: the corrector's ring sums sum_k AM(k)*
  // Previous(ipc(k)) (v, a, alpha: [9][n]), formed by the predictor pass,
  // which holds every term of them.  EPI_STORE: ComputeAccelerations'
  // Force(i) and Torque(i) before the division by mass and inertia
  // (src/MForces.f90:319-333) as amsum[3p+k], then amsum[3n+3p+k]; NULL: not
  // kept
  double* amsum;
  const int* rank;
  // test kernel -> pair kernel -> fold kernel: the pass's contact list
  // (pair (i, j) per contact, the contacts of each "i" together and in row
  // order: clist[cstart[i] .. + ccount[i])), the "i" results of every
  // contact (IRec64 / IRec32 [cl_cap]), the "j" results of every particle
  // (count, records InRec64 / InRec32 [in_cap][in_stride]) and the records
  // of each particle's table that a contact matched (bit r: record r); the
  // fold kernel resets the counts and the matched bits
  int2* clist;
  int* cstart;
  int* ccount;
  void* irec;
  int cl_cap;
  int* in_cnt;
  void* in_rec;
  int in_cap, in_stride;
  unsigned* matched;
  // normal force on each wall, summed per block of the fold kernel in a
  // fixed order ([block][DEM_MAX_WALLS]); nw_max: walls of the system with
  // the most
  double* wall_part;
  int nw_max;
  // a slab of a decomposition: the partner cells it knows this pass are its
  // own slab's and those stamped gepoch in gstamp (the ghost layers it
  // received); NULL: every cell is known
  const int* gstamp;
  int gepoch;
};


// The |FN| of every wall contact of a block of 128 particles, summed in a
// fixed order (lanes of warp 0 over the four warps, then a shuffle tree):
// s_w[w][thread] holds each thread's value; the sums go to row `block` of
// out.  All threads of the block call.
template <class T>
__device__ __forceinline__ void wall_partials(const T (*s_w)[128], int nw_max, double* out,
                                              int block) {
  __syncthreads();
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    for (int w = 0; w < nw_max; w++) {
      double v = (double)s_w[w][l];
      v = v + (double)s_w[w][l + 32];
      v = v + (double)s_w[w][l + 64];
      v = v + (double)s_w[w][l + 96];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
      if (l == 0) out[(size_t)block * NWM + w] = v;
    }
  }
}

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

// Wij of Overlap (src/MConfig.f90:797-819): the unit radial direction of the
// particle from the cone axis.  For a particle exactly on the axis (AlphaW =
// 0) the reference draws a random unit vector; here the coordinate axis
// least aligned with U, made orthogonal to U, is taken instead (the oracle
// does the same).
__device__ __forceinline__ void cone_radial(const double RijW[3], double AlphaW, const double U[3],
                                            double W[3]) {
  if (AlphaW == 0.0) {
    int k0 = 0;
    for (int k = 1; k < 3; k++)
      if (fabs(U[k]) < fabs(U[k0])) k0 = k;
    double e[3] = {0.0, 0.0, 0.0};
    e[k0] = 1.0;
    const double WdotU = dot3(e, U);
#pragma unroll
    for (int k = 0; k < 3; k++) W[k] = e[k] - WdotU * U[k];
    const double nn = sqrt(sumsq3(W));
#pragma unroll
    for (int k = 0; k < 3; k++) W[k] = W[k] / nn;
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++) W[k] = RijW[k] / AlphaW;
  }
}

// Overlap's Cone branch (src/MConfig.f90:751-793): conic frustum with half
// length L1 along U, radii L2 and L3 at its two ends; the auxiliary
// quantities of ConfigureWalls (src/MConfig.f90:661-684) for radius Ri.
__device__ __forceinline__ bool overlap_cone(const DevParams& P, const dem_wall& w,
                                             const double x[3], double Ri, double& Dij,
                                             double Nij[3], double Qji[3]) {
  double Rij[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    Rij[k] = w.position[k] - x[k];
    if (P.pbc[k]) Rij[k] = Rij[k] - P.lbox[k] * fnint(Rij[k] * P.inv_lbox[k]);
  }
  const double L_2 = w.l1, L = 2.0 * L_2, Ra = w.l2, Rp = w.l3;
  const double Aux = sqrt(L * L + (Rp - Ra) * (Rp - Ra));
  const double Rap = Aux, SinTheta = L / Aux, CosTheta = (Rp - Ra) / Aux;
  const double MaxAlphaU = L_2 + Ri;
  double mn = (Ra < Rp ? Ra : Rp) - Ri;
  mn = 0.0 > mn ? 0.0 : mn;
  const double MinAlphaWSq = mn * mn;
  const double mx = (Ra > Rp ? Ra : Rp) + Ri;
  const double MaxAlphaWSq = mx * mx;
  const double AlphaU = dot3(Rij, w.u);
  bool ov = fabs(AlphaU) < MaxAlphaU;
  if (!ov) return false;
  double RijW[3];
#pragma unroll
  for (int k = 0; k < 3; k++) RijW[k] = Rij[k] - AlphaU * w.u[k];
  const double AlphaWSq = sumsq3(RijW);
  ov = (AlphaWSq >= MinAlphaWSq) && (AlphaWSq < MaxAlphaWSq);
  if (!ov) return false;
  const double AlphaW = sqrt(AlphaWSq);
  const double Lby2_AlphaU = w.l1 - AlphaU;
  const double Ra_AlphaW = w.l2 - AlphaW;
  double Lambda = Lby2_AlphaU * SinTheta - Ra_AlphaW * CosTheta;
  double W[3];
  cone_radial(RijW, AlphaW, w.u, W);
  if (Lambda >= 0.0 && Lambda <= Rap) {
    const double SignedDij = -(Lby2_AlphaU * CosTheta + Ra_AlphaW * SinTheta);
    Dij = fabs(SignedDij);
    ov = Dij < Ri;
    if (ov) {
#pragma unroll
      for (int k = 0; k < 3; k++) Nij[k] = SinTheta * W[k] + CosTheta * w.u[k];
#pragma unroll
      for (int k = 0; k < 3; k++) Qji[k] = SignedDij * Nij[k] - Rij[k];
#pragma unroll
      for (int k = 0; k < 3; k++) Nij[k] = (Qji[k] + Rij[k]) / Dij;
    }
  } else {
    const double t = Lambda < Rap ? Lambda : Rap;
    Lambda = 0.0 > t ? 0.0 : t;
    const double a = SinTheta * Lambda - Lby2_AlphaU;
    const double b = CosTheta * Lambda + Ra_AlphaW;
#pragma unroll
    for (int k = 0; k < 3; k++) Nij[k] = a * w.u[k] - b * W[k];
    const double DijSq = sumsq3(Nij);
    ov = DijSq < Ri * Ri;
    if (ov) {
      Dij = sqrt(DijSq);
#pragma unroll
      for (int k = 0; k < 3; k++) Qji[k] = Nij[k] - Rij[k];
#pragma unroll
      for (int k = 0; k < 3; k++) Nij[k] = Nij[k] / Dij;
    }
  }
  return ov;
}

// Overlap (src/MConfig.f90:692-822): Rectangle or Cone.  CONE = false
// compiles the rectangle branch only, for kernels launched on systems without
// cone walls (the cone branch costs registers wherever it is compiled in).
template <bool CONE = true>
__device__ __forceinline__ bool overlap_wall(const DevParams& P, const dem_wall& w,
                                             const double x[3], double Ri, double& Dij,
                                             double Nij[3], double Qji[3]) {
  if (w.shape == DEM_WALL_RECTANGLE) return overlap_rect(P, w, x, Ri, Dij, Nij, Qji);
  if (!CONE || w.shape != DEM_WALL_CONE) return false;
  return overlap_cone(P, w, x, Ri, Dij, Nij, Qji);
}

// System parameters of particle p (or of cell c with a cell->system map).
__device__ __forceinline__ const DevParams& sys_params(const DevParams* T, const int* sid, int i) {
  return T[sid ? sid[i] : 0];
}

// CurrentCell3D (src/MCells.f90:498-513), 0-based, as a global cell index.
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
  return P.coff + ix + (iy + iz * P.ny) * P.nx;
}

// Are two cells neighbours in the sweep sense (same cell, or one in the
// other's half-shell list)?  With >= 3 cells along every periodic axis this
// is plain adjacency with wrap-around (VerifyPBC/ApplyPBC, src/MCells.f90:
// 1030-1052).
// q = c / d and c - q*d for 0 <= c < 2^31, d >= 1, from a reciprocal (one
// correction step makes it exact)
__device__ __forceinline__ int div_fast(int c, int d, double inv_d, int& rem) {
  int q = (int)((double)c * inv_d);
  int r = c - q * d;
  if (r >= d) {
    q++;
    r -= d;
  } else if (r < 0) {
    q--;
    r += d;
  }
  rem = r;
  return q;
}
// coordinates of global cell c of system P
__device__ __forceinline__ void cell_coords(const DevParams& P, int c, int& x, int& y, int& z) {
  const int t = div_fast(c - P.coff, P.nx, P.inv_nx, x);
  z = div_fast(t, P.ny, P.inv_ny, y);
}

// Are two cells neighbours in the sweep sense (same cell, or one in the
// other's half-shell list)?  With >= 3 cells along every periodic axis this
// is plain adjacency with wrap-around (VerifyPBC/ApplyPBC, src/MCells.f90:
// 1030-1052).
__device__ __forceinline__ bool in_slab(const DevParams& P, int c) {
  return c >= P.slab_c0 && c < P.slab_c1;
}

__device__ __forceinline__ bool cells_adjacent(const DevParams& P, int a, int b) {
  int ax, ay, az, bx, by, bz;
  cell_coords(P, a, ax, ay, az);
  cell_coords(P, b, bx, by, bz);
  int d[3] = {bx - ax, by - ay, bz - az};
  int N[3] = {P.nx, P.ny, P.nz};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    int x = d[k] < 0 ? -d[k] : d[k];
    if (x > 1 && !(P.pbc[k] && x == N[k] - 1)) return false;
  }
  return true;
}

// Whether a history record's partner q sits in a cell adjacent to cell c
// (the sweep visits the pair, src/MForces.f90:199-272), for records the
// pass did not match.  A slab trusts only the cells it knows this pass; a
// partner anywhere else is not adjacent to any of its cells.
template <class PA>
__device__ __forceinline__ bool partner_adjacent(const PA& A, const DevParams& P, int c, int q) {
  const int cq = A.cell_cur[q];
  if (A.gstamp && !in_slab(P, cq) && A.gstamp[q] != A.gepoch) return false;
  return cells_adjacent(P, c, cq);
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
}  // namespace dem
