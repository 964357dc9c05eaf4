/*
 * dem_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * A serial FP64 restatement of DEM3D's per-step path, written to follow the
 * reference Fortran line by line so that the CUDA library can be checked
 * against it bit for bit.  It is used by tests/, by __graft_entry__.smoke()
 * and by bench.py's CPU-baseline leg, never by the product library.
 *
 * Parity status: the reference (Fortran 90) cannot be compiled in this
 * environment (no Fortran compiler) and ships no test vectors or outputs, so
 * this restatement is pinned by known-answer tests derived from the
 * reference's own model (analytic binary collision: restitution coefficient
 * and contact duration implied by the damping rule of src/DEM.f90:288-298,
 * Coulomb sliding limit src/MForces.f90:372-378, wall geometry
 * src/MConfig.f90:717-749, cell hashing src/MCells.f90:498-513) rather than
 * by reference outputs: parity with the reference binary is unpinned.
 *
 * Data structures are the reference's: AoS particles (TParticle,
 * src/MDimension3D.f90:28-35), singly linked cell lists with prepend
 * (src/MCells.f90:19-27,666-698), singly linked sorted contact lists per
 * particle (src/MContacts.f90:21-33) with the module cursors imin/imax/
 * CurrentPair/PreviousPair (src/MContacts.f90:35-37), the ABM ring
 * Previous(NPrev,NP) with ipc and cshift (src/MDEM.f90:14-24,266,326).
 *
 * Documented deviations (each switchable so small cases stay literal):
 *  - Neighbour(MaxNeighbours=50) (src/MForces.f90:27,33) is a growable
 *    buffer here: the reference overflows it without a check at large
 *    cells; for cells with <=50 neighbours the two are identical;
 *  - MaxNCell (src/MForces.f90:28) is a parameter (30000 in the reference);
 *  - n_components == 0 selects per-particle radii (continuous
 *    polydispersity), each particle acting as its own component with the
 *    reference's pair-combination rules (src/DEM.f90:259-327);
 *  - particle indices are 0-based.
 * Compile with -ffp-contract=off: the reference's arithmetic is reproduced
 * operation by operation and no fused multiply-add may be formed.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/dem3d_b200.h"

#define NCM DEM_MAX_COMPONENTS
#define NWM DEM_MAX_WALLS

typedef struct {
  int32_t index; /* component index (TParticle%Index) */
  double pos[3], vel[3], acc[3], omega[3], alpha[3];
  double radius; /* per-particle mode only */
} OParticle;

typedef struct CNode {
  int32_t index;
  struct CNode* next;
} CNode;

typedef struct {
  CNode* first_particle;
  CNode* first_neighbour;
} OCell;

typedef struct Partner {
  int32_t index;
  double v1[3], v2[3];
  struct Partner* next;
} Partner;

typedef struct {
  Partner* first_partner;
  Partner* first_wall;
} OMain;

typedef struct {
  double v[3], a[3], al[3];
} OPrev;

typedef struct orc_ctx {
  dem_params p;
  int32_t n;
  int32_t nalloc;  /* rows of the arrays (n shrinks when particles leave) */
  OParticle* part;
  OParticle* pred;
  OPrev* prev; /* [nprev][n] */
  int32_t ipc[4];
  int32_t nprev;
  double AB0, AM0, AB[3], AM[3];
  double inv_lbox[3];
  double time;
  /* MCells module variables (src/MCells.f90:36-43) */
  int32_t Nx, Ny, Nz, Nt, Nxm1, Nym1, Nzm1;
  double NxByLx, NyByLy, NzByLz, NxBy2, NyBy2, NzBy2;
  OCell* cell;
  int32_t* cell_index; /* CellIndex (src/MForces.f90:31) */
  int32_t cells_ready;
  /* MContacts */
  OMain* mainp;
  Partner* current_pair;
  Partner* previous_pair;
  int32_t imin, imax, iwall;
  /* MForces scratch */
  int32_t* neighbour;
  int32_t neighbour_cap;
  int32_t literal_neighbour_cap; /* 0 = growable, else hard cap (reference: 50) */
  int32_t literal_removal;       /* 1: renamed records appended as the reference does */
  double* force;
  double* torque;
  /* MForces module variables (src/MForces.f90:36-44) */
  double Ri, Rj, Rij[3], DijSq, Dij, Nij[3], Qji[3], Vij[3], VijC[3], iForce[3];
  double ijForceN[3], ijForceT[3], iTorque[3], Nij_x_ijForceT[3], ijDispN[3];
  double VijT[3], ijForceT0[3], ijDeltaDT[3], ijDeltaVT[3], VijT0[3];
  double DeltaDijSq, HalfTimeStep;
  int Contacting;
  int64_t ncol;
  double wall_fn[NWM];
  int64_t last_pairs, last_walls;  /* overlapping pairs of the last force pass */
  int moving;               /* WallsInMovement */
  int removal;              /* run() calls UpdateParticleList after each step */
  int pouring;              /* run() calls PouringAttempt before each step */
  int fluid;                /* FluidFlow */
  dem_fluid fl;
  double fl_area, fl_dz, fl_vf0, fl_h2, fl_mh2;  /* InitializeFluid */
  double* vf;               /* Vf(0:NL) */
  double* ef;               /* Ef(0:NL) */
  dem_pouring pour;
  dem_rng rng;              /* ranf's state (src/MUtil.f90:10-11) */
  int32_t comp_count[NCM];  /* Component(:)%Number */
  int64_t removal_count, removal_swaps, removal_moved;  /* test diagnostics */
  dem_wall_motion wm[NWM];  /* WM(j) */
  char err[256];
} orc_ctx;

/* ------------------------------------------------------------------ */
/* small vector helpers: dot_product/sum as left-to-right sums          */

static inline double dot3(const double* a, const double* b) {
  /* dot_product(a,b) via DotProduct (src/MDimension3D.f90:75-82) */
  double c = 0.0;
  c = c + a[0] * b[0];
  c = c + a[1] * b[1];
  c = c + a[2] * b[2];
  return c;
}

static inline double sumsq3(const double* a) {
  double c = 0.0;
  c = c + a[0] * a[0];
  c = c + a[1] * a[1];
  c = c + a[2] * a[2];
  return c;
}

static inline void cross3(const double* a, const double* b, double* c) {
  /* CrossProduct, src/MDimension3D.f90:86-95 */
  double c0 = a[1] * b[2] - a[2] * b[1];
  double c1 = a[2] * b[0] - a[0] * b[2];
  double c2 = a[0] * b[1] - a[1] * b[0];
  c[0] = c0;
  c[1] = c1;
  c[2] = c2;
}

/* Fortran nint: round half away from zero to default integer */
static inline double fnint(double x) { return (double)(int32_t)lround(x); }

static void set_err(orc_ctx* c, const char* m) {
  snprintf(c->err, sizeof(c->err), "%s", m);
}

/* ------------------------------------------------------------------ */
/* material helpers: component tables or per-particle radius            */

static inline double o_radius(const orc_ctx* c, const OParticle* q) {
  return c->p.n_components > 0 ? c->p.comp_radius[q->index] : q->radius;
}
static inline double o_mass_pp(const orc_ctx* c, const OParticle* q) {
  double R = q->radius;
  return c->p.pp_mass_coef * ((R * R) * R);
}
static inline double o_inv_mass(const orc_ctx* c, const OParticle* q) {
  if (c->p.n_components > 0) return c->p.comp_inv_mass[q->index];
  return 1.0 / o_mass_pp(c, q);
}
static inline double o_inv_inertia(const orc_ctx* c, const OParticle* q) {
  if (c->p.n_components > 0) return c->p.comp_inv_inertia[q->index];
  double m = o_mass_pp(c, q);
  double R = q->radius;
  return 1.0 / ((0.4 * m) * (R * R));
}
static inline double o_eff_mass(const orc_ctx* c, const OParticle* q) {
  if (c->p.n_components > 0) return c->p.comp_eff_mass[q->index];
  double m = o_mass_pp(c, q);
  return (m * (c->p.pp_density - c->p.pp_fluid_density)) / c->p.pp_density;
}

typedef struct {
  double min_dij, min_dij_sq, kn, yn, kt, yt, mu_sq;
} PairPar;

static inline void o_pair_params(const orc_ctx* c, const OParticle* a,
                                 const OParticle* b, PairPar* pp) {
  if (c->p.n_components > 0) {
    int k = a->index * NCM + b->index;
    pp->min_dij = c->p.min_dij[k];
    pp->min_dij_sq = c->p.min_dij_sq[k];
    pp->kn = c->p.kn[k];
    pp->yn = c->p.yn[k];
    pp->kt = c->p.kt[k];
    pp->yt = c->p.yt[k];
    pp->mu_sq = c->p.mu_sq[k];
  } else {
    double ma = o_mass_pp(c, a), mb = o_mass_pp(c, b);
    double meff = (ma * mb) / (ma + mb);
    pp->min_dij = a->radius + b->radius;
    pp->min_dij_sq = pp->min_dij * pp->min_dij;
    pp->kn = c->p.pp_kn;
    pp->yn = c->p.pp_gamma_n * sqrt(meff * c->p.pp_kn);
    pp->kt = c->p.pp_kt;
    pp->yt = c->p.pp_gamma_t * sqrt(meff * c->p.pp_kt);
    pp->mu_sq = c->p.pp_mu_sq;
  }
}

static inline void o_wall_params(const orc_ctx* c, const OParticle* a, int w,
                                 PairPar* pp) {
  if (c->p.n_components > 0) {
    int k = a->index * NWM + w;
    pp->kn = c->p.knw[k];
    pp->yn = c->p.ynw[k];
    pp->kt = c->p.ktw[k];
    pp->yt = c->p.ytw[k];
    pp->mu_sq = c->p.muw_sq[k];
  } else {
    double m = o_mass_pp(c, a);
    pp->kn = c->p.pp_knw[w];
    pp->yn = c->p.pp_gamma_nw[w] * sqrt(m * c->p.pp_knw[w]);
    pp->kt = c->p.pp_ktw[w];
    pp->yt = c->p.pp_gamma_tw[w] * sqrt(m * c->p.pp_ktw[w]);
    pp->mu_sq = c->p.pp_muw_sq[w];
  }
}

/* ------------------------------------------------------------------ */
/* MCells                                                               */

/* InitCellStructure3D, src/MCells.f90:155-227 */
static void init_cell_structure(orc_ctx* c, double Lx, double Ly, double Lz,
                                double CutOff, int32_t MaxNCell) {
  int32_t Nx4 = (int32_t)(Lx / CutOff);
  int32_t Ny4 = (int32_t)(Ly / CutOff);
  int32_t Nz4 = (int32_t)(Lz / CutOff);
  int64_t N4 = (int64_t)Nx4 * Ny4 * Nz4;
  if (N4 > MaxNCell) {
    double LCell = pow(Lx * Ly * Lz / (double)MaxNCell, 1.0 / 3.0);
    c->Nx = (int32_t)(Lx / LCell);
    c->Ny = (int32_t)(Ly / LCell);
    c->Nz = (int32_t)(Lz / LCell);
    c->Nt = c->Nx * c->Ny * c->Nz;
  } else {
    c->Nx = Nx4;
    c->Ny = Ny4;
    c->Nz = Nz4;
    c->Nt = (int32_t)N4;
  }
  c->NxByLx = (double)c->Nx / Lx;
  c->NyByLy = (double)c->Ny / Ly;
  c->NzByLz = (double)c->Nz / Lz;
  c->NxBy2 = (double)c->Nx * 0.5;
  c->NyBy2 = (double)c->Ny * 0.5;
  c->NzBy2 = (double)c->Nz * 0.5;
  c->Nxm1 = c->Nx - 1;
  c->Nym1 = c->Ny - 1;
  c->Nzm1 = c->Nz - 1;
  c->cell = (OCell*)calloc((size_t)c->Nt, sizeof(OCell));
}

/* VerifyPBC, src/MCells.f90:1030-1040 */
static void verify_pbc(int32_t* ini, int32_t* fin, int32_t i, int32_t MCell, int pbc) {
  *ini = -1;
  *fin = +1;
  if (!pbc) {
    if (i == 0) *ini = 0;
    if (i == MCell - 1) *fin = 0;
  }
}

/* ApplyPBC, src/MCells.f90:1044-1052 */
static void apply_pbc(int32_t* j, int32_t MCell, int pbc) {
  if (pbc) {
    if (*j == MCell) *j = 0;
    if (*j == -1) *j = MCell - 1;
  }
}

/* AddNeighbour, src/MCells.f90:666-680 (prepend) */
static void add_neighbour(orc_ctx* c, int32_t jCell, int32_t iCell) {
  CNode* cur = (CNode*)malloc(sizeof(CNode));
  cur->index = jCell;
  cur->next = c->cell[iCell].first_neighbour;
  c->cell[iCell].first_neighbour = cur;
}

/* AddAllNeighbours3D with MC = .false., src/MCells.f90:424-476 */
static void add_all_neighbours(orc_ctx* c, int32_t iCell, int32_t ix, int32_t iy,
                               int32_t iz, int32_t xi, int32_t xf, int32_t yi,
                               int32_t yf, int32_t zi, int32_t zf) {
  const int* P = c->p.pbc;
  for (int32_t kz = zi; kz <= zf; kz++) {
    int32_t jz = iz + kz;
    apply_pbc(&jz, c->Nz, P[2]);
    for (int32_t ky = yi; ky <= yf; ky++) {
      int32_t jy = iy + ky;
      apply_pbc(&jy, c->Ny, P[1]);
      for (int32_t kx = xi; kx <= xf; kx++) {
        int32_t kCell = kx + c->Nx * (ky + c->Ny * kz);
        if (kCell > 0) {
          int32_t jx = ix + kx;
          apply_pbc(&jx, c->Nx, P[0]);
          int32_t jCell = jx + c->Nx * (jy + c->Ny * jz);
          add_neighbour(c, jCell, iCell);
        }
      }
    }
  }
}

/* FullNeighbourCells3D(MolecularDynamics,...), src/MCells.f90:276-327 */
static void full_neighbour_cells(orc_ctx* c) {
  int32_t xi, xf, yi, yf, zi, zf;
  for (int32_t iz = 0; iz <= c->Nzm1; iz++) {
    verify_pbc(&zi, &zf, iz, c->Nz, c->p.pbc[2]);
    for (int32_t iy = 0; iy <= c->Nym1; iy++) {
      verify_pbc(&yi, &yf, iy, c->Ny, c->p.pbc[1]);
      for (int32_t ix = 0; ix <= c->Nxm1; ix++) {
        verify_pbc(&xi, &xf, ix, c->Nx, c->p.pbc[0]);
        int32_t iCell = ix + c->Nx * (iy + c->Ny * iz);
        add_all_neighbours(c, iCell, ix, iy, iz, xi, xf, yi, yf, zi, zf);
      }
    }
  }
}

/* CurrentCell3D, src/MCells.f90:498-513 (0-based result) */
static inline int32_t current_cell(const orc_ctx* c, double x, double y, double z) {
  int32_t ix = (int32_t)(c->NxByLx * x + c->NxBy2);
  int32_t iy = (int32_t)(c->NyByLy * y + c->NyBy2);
  int32_t iz = (int32_t)(c->NzByLz * z + c->NzBy2);
  ix = ix < c->Nxm1 ? ix : c->Nxm1;
  iy = iy < c->Nym1 ? iy : c->Nym1;
  iz = iz < c->Nzm1 ? iz : c->Nzm1;
  ix = ix > 0 ? ix : 0;
  iy = iy > 0 ? iy : 0;
  iz = iz > 0 ? iz : 0;
  return ix + (iy + iz * c->Ny) * c->Nx;
}

/* AddParticle, src/MCells.f90:684-698 (prepend) */
static void add_particle(orc_ctx* c, int32_t i, int32_t iCell) {
  CNode* cur = (CNode*)malloc(sizeof(CNode));
  cur->index = i;
  cur->next = c->cell[iCell].first_particle;
  c->cell[iCell].first_particle = cur;
}

/* TransferParticle, src/MCells.f90:747-774 */
static void transfer_particle(orc_ctx* c, int32_t i, int32_t iCell, int32_t jCell) {
  CNode* cur = c->cell[iCell].first_particle;
  CNode* aux;
  if (cur->index == i) {
    c->cell[iCell].first_particle = cur->next;
    aux = cur;
  } else {
    while (cur->next->index != i) cur = cur->next;
    aux = cur->next;
    cur->next = aux->next;
  }
  aux->next = c->cell[jCell].first_particle;
  c->cell[jCell].first_particle = aux;
}

/* DistributeParticles3D, src/MCells.f90:542-564 */
static void distribute_particles(orc_ctx* c) {
  for (int32_t i = 0; i < c->n; i++)
    c->cell_index[i] = current_cell(c, c->part[i].pos[0], c->part[i].pos[1], c->part[i].pos[2]);
  for (int32_t i = 0; i < c->n; i++) add_particle(c, i, c->cell_index[i]);
}

/* RedistributeParticles3D, src/MCells.f90:607-643 */
static void redistribute_particles(orc_ctx* c, const OParticle* P) {
  for (int32_t i = 0; i < c->n; i++) {
    int32_t Old = c->cell_index[i];
    int32_t New = current_cell(c, P[i].pos[0], P[i].pos[1], P[i].pos[2]);
    if (New != Old) {
      transfer_particle(c, i, Old, New);
      c->cell_index[i] = New;
    }
  }
}

static int ensure_neighbour(orc_ctx* c, int32_t need) {
  if (need <= c->neighbour_cap) return 1;
  if (c->literal_neighbour_cap > 0) return 0;
  int32_t cap = c->neighbour_cap ? c->neighbour_cap : 64;
  while (cap < need) cap *= 2;
  c->neighbour = (int32_t*)realloc(c->neighbour, sizeof(int32_t) * (size_t)cap);
  c->neighbour_cap = cap;
  return 1;
}

/* NeighbourParticles, src/MCells.f90:793-829 */
static int neighbour_particles(orc_ctx* c, int32_t iCell, int32_t* npcc, int32_t* npsc) {
  int32_t nic = 0;
  for (CNode* p = c->cell[iCell].first_particle; p; p = p->next) {
    if (!ensure_neighbour(c, nic + 1)) return 0;
    c->neighbour[nic++] = p->index;
  }
  int32_t non = nic;
  if (nic != 0) {
    for (CNode* cc = c->cell[iCell].first_neighbour; cc; cc = cc->next) {
      for (CNode* p = c->cell[cc->index].first_particle; p; p = p->next) {
        if (!ensure_neighbour(c, non + 1)) return 0;
        c->neighbour[non++] = p->index;
      }
    }
  }
  *npcc = nic;
  *npsc = non;
  return 1;
}

static void destroy_cells(orc_ctx* c) {
  if (!c->cell) return;
  for (int32_t i = 0; i < c->Nt; i++) {
    CNode* p = c->cell[i].first_neighbour;
    while (p) { CNode* a = p; p = p->next; free(a); }
    p = c->cell[i].first_particle;
    while (p) { CNode* a = p; p = p->next; free(a); }
    c->cell[i].first_neighbour = NULL;
    c->cell[i].first_particle = NULL;
  }
}

static void clear_cell_particles(orc_ctx* c) {
  for (int32_t i = 0; i < c->Nt; i++) {
    CNode* p = c->cell[i].first_particle;
    while (p) { CNode* a = p; p = p->next; free(a); }
    c->cell[i].first_particle = NULL;
  }
}

/* ------------------------------------------------------------------ */
/* MContacts                                                            */

/* VerifyPairContact, src/MContacts.f90:329-373 */
static void verify_pair_contact(orc_ctx* c, int32_t i, int32_t j, int* contacting,
                                double* v1, double* v2) {
  c->imin = i < j ? i : j;
  c->imax = i < j ? j : i;
  c->current_pair = c->mainp[c->imin].first_partner;
  *contacting = c->current_pair != NULL;
  if (*contacting) {
    c->previous_pair = c->current_pair;
    while (c->current_pair->index < c->imax && c->current_pair->next) {
      c->previous_pair = c->current_pair;
      c->current_pair = c->current_pair->next;
    }
    *contacting = c->current_pair->index == c->imax;
    if (*contacting) {
      memcpy(v1, c->current_pair->v1, sizeof(double) * 3);
      memcpy(v2, c->current_pair->v2, sizeof(double) * 3);
    } else {
      v1[0] = v1[1] = v1[2] = 0.0;
      v2[0] = v2[1] = v2[2] = 0.0;
    }
  } else {
    v1[0] = v1[1] = v1[2] = 0.0;
    v2[0] = v2[1] = v2[2] = 0.0;
  }
}

/* UpdatePairContact / UpdateWallContact, src/MContacts.f90:377-423,489-535 */
static void update_contact(orc_ctx* c, const double* v1, const double* v2,
                           int contacting, int key, Partner** head) {
  if (contacting) {
    memcpy(c->current_pair->v1, v1, sizeof(double) * 3);
    memcpy(c->current_pair->v2, v2, sizeof(double) * 3);
  } else {
    Partner* aux = (Partner*)malloc(sizeof(Partner));
    aux->index = key;
    memcpy(aux->v1, v1, sizeof(double) * 3);
    memcpy(aux->v2, v2, sizeof(double) * 3);
    aux->next = NULL;
    if (c->current_pair) {
      if (c->current_pair->index < key) {
        c->current_pair->next = aux;
      } else {
        aux->next = c->current_pair;
        if (c->current_pair->index == c->previous_pair->index)
          *head = aux;
        else
          c->previous_pair->next = aux;
      }
    } else {
      *head = aux;
    }
  }
}

/* RemovePairContact / RemoveWallContact, src/MContacts.f90:427-437,539-549 */
static void remove_contact(orc_ctx* c, int key, Partner** head) {
  if (c->previous_pair->index == key)
    *head = c->current_pair->next;
  else
    c->previous_pair->next = c->current_pair->next;
  free(c->current_pair);
}

/* VerifyWallContact, src/MContacts.f90:441-485 */
static void verify_wall_contact(orc_ctx* c, int32_t i, int32_t w, int* contacting,
                                double* v1, double* v2) {
  c->imin = i;
  c->iwall = w;
  c->current_pair = c->mainp[c->imin].first_wall;
  *contacting = c->current_pair != NULL;
  if (*contacting) {
    c->previous_pair = c->current_pair;
    while (c->current_pair->index < c->iwall && c->current_pair->next) {
      c->previous_pair = c->current_pair;
      c->current_pair = c->current_pair->next;
    }
    *contacting = c->current_pair->index == c->iwall;
    if (*contacting) {
      memcpy(v1, c->current_pair->v1, sizeof(double) * 3);
      memcpy(v2, c->current_pair->v2, sizeof(double) * 3);
    } else {
      v1[0] = v1[1] = v1[2] = 0.0;
      v2[0] = v2[1] = v2[2] = 0.0;
    }
  } else {
    v1[0] = v1[1] = v1[2] = 0.0;
    v2[0] = v2[1] = v2[2] = 0.0;
  }
}

static void destroy_contacts(orc_ctx* c) {
  if (!c->mainp) return;
  for (int32_t i = 0; i < c->n; i++) {
    Partner* p = c->mainp[i].first_partner;
    while (p) { Partner* a = p; p = p->next; free(a); }
    p = c->mainp[i].first_wall;
    while (p) { Partner* a = p; p = p->next; free(a); }
    c->mainp[i].first_partner = NULL;
    c->mainp[i].first_wall = NULL;
  }
}

/* sorted insert used by set_contacts (ReadContactList builds sorted lists) */
static void insert_sorted(Partner** head, int32_t key, const double* v1, const double* v2) {
  Partner* aux = (Partner*)malloc(sizeof(Partner));
  aux->index = key;
  memcpy(aux->v1, v1, sizeof(double) * 3);
  memcpy(aux->v2, v2, sizeof(double) * 3);
  Partner** pp = head;
  while (*pp && (*pp)->index < key) pp = &(*pp)->next;
  aux->next = *pp;
  *pp = aux;
}

/* ------------------------------------------------------------------ */
/* MForces                                                              */

/* ChangePlane, src/MForces.f90:391-406 */
static void change_plane(const double* V, const double* N, double* out) {
  double d = dot3(V, N);
  double P[3];
  for (int k = 0; k < 3; k++) P[k] = V[k] - d * N[k];
  double NormSq = sumsq3(P);
  if (NormSq != 0.0) {
    double f = sqrt(sumsq3(V) / NormSq);
    for (int k = 0; k < 3; k++) out[k] = f * P[k];
  } else {
    out[0] = out[1] = out[2] = 0.0;
  }
}

/* CommonCalculations, src/MForces.f90:339-387 */
static void common_calculations(orc_ctx* c, const double* Rij, double Kn, double Yn,
                                double Kt, double Yt, double MuSq) {
  double VijN[3];
  double d = dot3(c->VijC, c->Nij);
  for (int k = 0; k < 3; k++) VijN[k] = d * c->Nij[k];
  for (int k = 0; k < 3; k++) c->VijT[k] = c->VijC[k] - VijN[k];
  for (int k = 0; k < 3; k++) c->ijForceN[k] = Kn * c->ijDispN[k] + Yn * VijN[k];
  if (c->Contacting) {
    double t[3];
    change_plane(c->VijT0, c->Nij, t);
    memcpy(c->VijT0, t, sizeof(t));
    for (int k = 0; k < 3; k++) c->ijDeltaDT[k] = c->HalfTimeStep * (c->VijT0[k] + c->VijT[k]);
    for (int k = 0; k < 3; k++) c->ijDeltaVT[k] = c->VijT[k] - c->VijT0[k];
    double cp[3];
    change_plane(c->ijForceT0, c->Nij, cp);
    for (int k = 0; k < 3; k++)
      c->ijForceT[k] = cp[k] + Kt * c->ijDeltaDT[k] + Yt * c->ijDeltaVT[k];
  } else {
    double PartialDt;
    double VijSq = sumsq3(c->Vij);
    if (VijSq > 0.0) {
      double RijVij = dot3(Rij, c->Vij);
      double a = 2.0 * c->HalfTimeStep;
      double b = (RijVij + sqrt(RijVij * RijVij + VijSq * c->DeltaDijSq)) / VijSq;
      PartialDt = b < a ? b : a;
    } else {
      PartialDt = 0.0;
    }
    double f = Kt * PartialDt + Yt;
    for (int k = 0; k < 3; k++) c->ijForceT[k] = f * c->VijT[k];
  }
  double MuNormForceNSq = MuSq * sumsq3(c->ijForceN);
  double NormForceTSq = sumsq3(c->ijForceT);
  if (NormForceTSq > MuNormForceNSq) {
    double f = sqrt(MuNormForceNSq / NormForceTSq);
    for (int k = 0; k < 3; k++) c->ijForceT[k] = f * c->ijForceT[k];
  }
  for (int k = 0; k < 3; k++) c->iForce[k] = c->iForce[k] + c->ijForceN[k] + c->ijForceT[k];
  cross3(c->Nij, c->ijForceT, c->Nij_x_ijForceT);
  double RN[3], tq[3];
  for (int k = 0; k < 3; k++) RN[k] = c->Ri * c->Nij[k];
  cross3(RN, c->ijForceT, tq);
  for (int k = 0; k < 3; k++) c->iTorque[k] = c->iTorque[k] + tq[k];
}

/* Wij of Overlap (src/MConfig.f90:797-819); on the axis (AlphaW = 0) the
 * reference draws a random unit vector: here the coordinate axis least
 * aligned with U, made orthogonal to U (the library does the same). */
static void cone_radial(const double RijW[3], double AlphaW, const double U[3], double W[3]) {
  if (AlphaW == 0.0) {
    int k0 = 0;
    for (int k = 1; k < 3; k++)
      if (fabs(U[k]) < fabs(U[k0])) k0 = k;
    double e[3] = {0.0, 0.0, 0.0};
    e[k0] = 1.0;
    double WdotU = dot3(e, U);
    for (int k = 0; k < 3; k++) W[k] = e[k] - WdotU * U[k];
    double nn = sqrt(sumsq3(W));
    for (int k = 0; k < 3; k++) W[k] = W[k] / nn;
  } else {
    for (int k = 0; k < 3; k++) W[k] = RijW[k] / AlphaW;
  }
}

/* Overlap, src/MConfig.f90:692-822: Rectangle (:717-749) and Cone (:751-793,
 * with the auxiliary quantities of ConfigureWalls, :661-684, for radius Ri) */
static int overlap_wall(const orc_ctx* c, const OParticle* ip, const dem_wall* w,
                        double Ri, double* Dij, double* Nij, double* Qji) {
  double Rij[3];
  for (int k = 0; k < 3; k++) {
    Rij[k] = w->position[k] - ip->pos[k];
    if (c->p.pbc[k]) Rij[k] = Rij[k] - c->p.lbox[k] * fnint(Rij[k] * c->inv_lbox[k]);
  }
  int ov = 0;
  if (w->shape == DEM_WALL_RECTANGLE) {
    double AlphaN = dot3(Rij, w->n);
    double absAlphaN = fabs(AlphaN);
    ov = absAlphaN < Ri;
    if (ov) {
      double AlphaU = dot3(Rij, w->u);
      double AlphaW = dot3(Rij, w->w);
      double absAlphaU = fabs(AlphaU);
      double absAlphaW = fabs(AlphaW);
      ov = (absAlphaU < w->l1 + Ri) && (absAlphaW < w->l2 + Ri);
      if (ov) {
        if (absAlphaU < w->l1 && absAlphaW < w->l2) {
          double s = copysign(1.0, AlphaN);
          for (int k = 0; k < 3; k++) Nij[k] = s * w->n[k];
          *Dij = absAlphaN;
          for (int k = 0; k < 3; k++) Qji[k] = -(AlphaU * w->u[k] + AlphaW * w->w[k]);
        } else {
          double mu = -w->l1, mw = -w->l2;
          AlphaU = AlphaU < w->l1 ? AlphaU : w->l1;
          AlphaU = mu > AlphaU ? mu : AlphaU;
          AlphaW = AlphaW < w->l2 ? AlphaW : w->l2;
          AlphaW = mw > AlphaW ? mw : AlphaW;
          for (int k = 0; k < 3; k++) Qji[k] = -(AlphaU * w->u[k] + AlphaW * w->w[k]);
          for (int k = 0; k < 3; k++) Nij[k] = Rij[k] + Qji[k];
          double DijSq = sumsq3(Nij);
          ov = DijSq < Ri * Ri;
          if (ov) {
            *Dij = sqrt(DijSq);
            for (int k = 0; k < 3; k++) Nij[k] = Nij[k] / *Dij;
          }
        }
      }
    }
  } else if (w->shape == DEM_WALL_CONE) {
    double L_2 = w->l1, L = 2.0 * L_2, Ra = w->l2, Rp = w->l3;
    double Aux = sqrt(L * L + (Rp - Ra) * (Rp - Ra));
    double Rap = Aux, SinTheta = L / Aux, CosTheta = (Rp - Ra) / Aux;
    double MaxAlphaU = L_2 + Ri;
    double mn = (Ra < Rp ? Ra : Rp) - Ri;
    mn = 0.0 > mn ? 0.0 : mn;
    double MinAlphaWSq = mn * mn;
    double mx = (Ra > Rp ? Ra : Rp) + Ri;
    double MaxAlphaWSq = mx * mx;
    double AlphaU = dot3(Rij, w->u);
    ov = fabs(AlphaU) < MaxAlphaU;
    if (ov) {
      double RijW[3];
      for (int k = 0; k < 3; k++) RijW[k] = Rij[k] - AlphaU * w->u[k];
      double AlphaWSq = sumsq3(RijW);
      ov = (AlphaWSq >= MinAlphaWSq) && (AlphaWSq < MaxAlphaWSq);
      if (ov) {
        double AlphaW = sqrt(AlphaWSq);
        double Lby2_AlphaU = w->l1 - AlphaU;
        double Ra_AlphaW = w->l2 - AlphaW;
        double Lambda = Lby2_AlphaU * SinTheta - Ra_AlphaW * CosTheta;
        double W[3];
        cone_radial(RijW, AlphaW, w->u, W);
        if (Lambda >= 0.0 && Lambda <= Rap) {
          double SignedDij = -(Lby2_AlphaU * CosTheta + Ra_AlphaW * SinTheta);
          *Dij = fabs(SignedDij);
          ov = *Dij < Ri;
          if (ov) {
            for (int k = 0; k < 3; k++) Nij[k] = SinTheta * W[k] + CosTheta * w->u[k];
            for (int k = 0; k < 3; k++) Qji[k] = SignedDij * Nij[k] - Rij[k];
            for (int k = 0; k < 3; k++) Nij[k] = (Qji[k] + Rij[k]) / *Dij;
          }
        } else {
          double t = Lambda < Rap ? Lambda : Rap;
          Lambda = 0.0 > t ? 0.0 : t;
          double a = SinTheta * Lambda - Lby2_AlphaU;
          double b = CosTheta * Lambda + Ra_AlphaW;
          for (int k = 0; k < 3; k++) Nij[k] = a * w->u[k] - b * W[k];
          double DijSq = sumsq3(Nij);
          ov = DijSq < Ri * Ri;
          if (ov) {
            *Dij = sqrt(DijSq);
            for (int k = 0; k < 3; k++) Qji[k] = Nij[k] - Rij[k];
            for (int k = 0; k < 3; k++) Nij[k] = Nij[k] / *Dij;
          }
        }
      }
    }
  }
  return ov;
}

/* ------------------------------------------------------------------ */
/* mFluid                                                                */

static const double FL_PI = 3.1415926535897932384626433832795; /* src/MUtil.f90 */

/* UpdateVelocityField (src/mFluid.f90:96-139) */
static void update_velocity_field(orc_ctx* c, const OParticle* P) {
  for (int32_t k = 0; k <= c->fl.levels; k++) {
    const double Zk = c->fl_mh2 + (double)k * c->fl_dz;
    double SumA = 0.0, SumB = 0.0, SumC = 0.0;
    for (int32_t i = 0; i < c->n; i++) {
      const int32_t ind = P[i].index;
      const double d = Zk - P[i].pos[2];
      const double Diff2 = d * d;
      const double R = c->p.comp_radius[ind];
      const double R2 = R * R;
      if (Diff2 < R2) {
        const double Ai = FL_PI * (R2 - Diff2);
        SumA = SumA + Ai;
        const double DensAi = Ai * c->fl.comp_density[ind];
        SumB = SumB + DensAi * P[i].vel[2];
        SumC = SumC + DensAi;
      }
    }
    if (SumA == 0.0) {
      c->vf[k] = c->fl_vf0;
      c->ef[k] = 1.0;
    } else {
      const double Es = SumA / c->fl_area;
      c->ef[k] = 1.0 - Es;
      const double Vs = SumB / SumC;
      c->vf[k] = (c->fl_vf0 - Es * Vs) / c->ef[k];
    }
  }
}

/* DragForce (src/mFluid.f90:143-197).  The level index is kept inside
 * 0..NL-1 (the reference would read past Vf(NL) for a sphere above the box). */
static void drag_force(const orc_ctx* c, const OParticle* ip, double FD[3]) {
  const double Zi = ip->pos[2];
  const double jr = (Zi + c->fl_h2) / c->fl_dz;
  int32_t j = (int32_t)jr;
  if (j < 0) j = 0;
  if (j > c->fl.levels - 1) j = c->fl.levels - 1;
  double Vfz = c->vf[j];
  Vfz = Vfz + (jr - (double)j) * (c->vf[j + 1] - Vfz);
  double Efz = c->ef[j];
  Efz = Efz + (jr - (double)j) * (c->ef[j + 1] - Efz);
  double Vr[3] = {-ip->vel[0], -ip->vel[1], -ip->vel[2]};
  Vr[2] = Vfz + Vr[2];
  const double Vra = sqrt((Vr[0] * Vr[0] + Vr[1] * Vr[1]) + Vr[2] * Vr[2]);
  if (Vra > 0.0) {
    const double Ri = c->p.comp_radius[ip->index];
    const double Re = 2.0 * Efz * Ri * Vra * c->fl.density / c->fl.viscosity;
    double n = 3.6, n0 = n + 1.0, x = 0.0;
    for (int it = 0; fabs(n - n0) > 1.e-8 && it < 1000; it++) {
      n0 = n;
      x = Re / pow(Efz, n);
      const double x75 = pow(x, 0.75);
      n = (4.8 + 0.42 * x75) / (1.0 + 0.175 * x75);
    }
    double a = 0.63 + 4.8 / sqrt(x);
    const double Cd1 = a * a;
    a = 0.63 + 4.8 / sqrt(Re);
    const double CD = a * a;
    const double fi = (Cd1 / CD) * pow(Efz, 2.0 * (1.0 - n));
    const double s = CD * (FL_PI / 2.0) * Ri * Ri * c->fl.density * Vra;
    for (int k = 0; k < 3; k++) FD[k] = s * Vr[k] * fi;
  } else {
    FD[0] = FD[1] = FD[2] = 0.0;
  }
}

/* ComputeAccelerations, src/MForces.f90:145-335 */
static int compute_accelerations(orc_ctx* c, OParticle* P, double TimeStep, int Update) {
  const int32_t n = c->n;
  c->HalfTimeStep = 0.5 * TimeStep;
  redistribute_particles(c, P);
  memset(c->force, 0, sizeof(double) * 3 * (size_t)n);
  memset(c->torque, 0, sizeof(double) * 3 * (size_t)n);
  for (int w = 0; w < NWM; w++) c->wall_fn[w] = 0.0;
  c->last_pairs = 0;
  c->last_walls = 0;
  if (c->fluid) update_velocity_field(c, P);
  for (int32_t iCell = 0; iCell < c->Nt; iCell++) {
    int32_t NPCC, NPSC;
    if (!neighbour_particles(c, iCell, &NPCC, &NPSC)) {
      set_err(c, "Neighbour buffer overflow (literal MaxNeighbours)");
      return DEM_ERR_CAPACITY;
    }
    for (int32_t ii = 0; ii < NPCC; ii++) {
      int32_t i = c->neighbour[ii];
      const OParticle iPart = P[i];
      c->Ri = o_radius(c, &iPart);
      double em = o_eff_mass(c, &iPart);
      for (int k = 0; k < 3; k++) c->iForce[k] = em * c->p.gravity[k];
      c->iTorque[0] = c->iTorque[1] = c->iTorque[2] = 0.0;
      for (int32_t jj = ii + 1; jj < NPSC; jj++) {
        int32_t j = c->neighbour[jj];
        const OParticle jPart = P[j];
        c->Rj = o_radius(c, &jPart);
        for (int k = 0; k < 3; k++) {
          c->Rij[k] = jPart.pos[k] - iPart.pos[k];
          if (c->p.pbc[k])
            c->Rij[k] = c->Rij[k] - c->p.lbox[k] * fnint(c->Rij[k] * c->inv_lbox[k]);
        }
        c->DijSq = sumsq3(c->Rij);
        verify_pair_contact(c, i, j, &c->Contacting, c->ijForceT0, c->VijT0);
        PairPar pp;
        o_pair_params(c, &iPart, &jPart, &pp);
        c->DeltaDijSq = pp.min_dij_sq - c->DijSq;
        if (c->DeltaDijSq > 0.0) {
          if (!c->Contacting) c->ncol = c->ncol + 1;
          c->last_pairs++;
          c->Dij = sqrt(c->DijSq);
          for (int k = 0; k < 3; k++) c->Nij[k] = c->Rij[k] / c->Dij;
          double dn = c->Dij - pp.min_dij;
          for (int k = 0; k < 3; k++) c->ijDispN[k] = dn * c->Nij[k];
          for (int k = 0; k < 3; k++) c->Vij[k] = jPart.vel[k] - iPart.vel[k];
          double wsum[3], cr[3];
          for (int k = 0; k < 3; k++) wsum[k] = c->Ri * iPart.omega[k] + c->Rj * jPart.omega[k];
          cross3(wsum, c->Nij, cr);
          for (int k = 0; k < 3; k++) c->VijC[k] = c->Vij[k] - cr[k];
          common_calculations(c, c->Rij, pp.kn, pp.yn, pp.kt, pp.yt, pp.mu_sq);
          for (int k = 0; k < 3; k++)
            c->force[3 * j + k] = c->force[3 * j + k] - c->ijForceN[k] - c->ijForceT[k];
          for (int k = 0; k < 3; k++)
            c->torque[3 * j + k] = c->torque[3 * j + k] + c->Rj * c->Nij_x_ijForceT[k];
          if (Update)
            update_contact(c, c->ijForceT, c->VijT, c->Contacting, c->imax,
                           &c->mainp[c->imin].first_partner);
        } else {
          if (c->Contacting && Update) remove_contact(c, c->imax, &c->mainp[c->imin].first_partner);
        }
      }
      for (int32_t w = 0; w < c->p.n_walls; w++) {
        const dem_wall* jWall = &c->p.walls[w];
        verify_wall_contact(c, i, w, &c->Contacting, c->ijForceT0, c->VijT0);
        if (overlap_wall(c, &iPart, jWall, c->Ri, &c->Dij, c->Nij, c->Qji)) {
          c->DeltaDijSq = c->Ri * c->Ri - c->Dij * c->Dij;
          c->last_walls++;
          double dn = c->Dij - c->Ri;
          for (int k = 0; k < 3; k++) c->ijDispN[k] = dn * c->Nij[k];
          double wq[3];
          cross3(jWall->omega, c->Qji, wq);
          for (int k = 0; k < 3; k++) c->Vij[k] = jWall->velocity[k] + wq[k] - iPart.vel[k];
          double ro[3], cr[3];
          for (int k = 0; k < 3; k++) ro[k] = c->Ri * iPart.omega[k];
          cross3(ro, c->Nij, cr);
          for (int k = 0; k < 3; k++) c->VijC[k] = c->Vij[k] - cr[k];
          double Rw[3];
          for (int k = 0; k < 3; k++) Rw[k] = jWall->position[k] + c->Qji[k] - iPart.pos[k];
          PairPar pp;
          o_wall_params(c, &iPart, w, &pp);
          common_calculations(c, Rw, pp.kn, pp.yn, pp.kt, pp.yt, pp.mu_sq);
          c->wall_fn[w] += sqrt(sumsq3(c->ijForceN));
          if (Update)
            update_contact(c, c->ijForceT, c->VijT, c->Contacting, c->iwall,
                           &c->mainp[c->imin].first_wall);
        } else {
          if (c->Contacting && Update) remove_contact(c, c->iwall, &c->mainp[c->imin].first_wall);
        }
      }
      if (c->fluid) { /* iForce = iForce + DragForce(iPart), src/MForces.f90:316 */
        double FD[3];
        drag_force(c, &iPart, FD);
        for (int k = 0; k < 3; k++) c->iForce[k] = c->iForce[k] + FD[k];
      }
      for (int k = 0; k < 3; k++) c->force[3 * i + k] = c->force[3 * i + k] + c->iForce[k];
      for (int k = 0; k < 3; k++) c->torque[3 * i + k] = c->torque[3 * i + k] + c->iTorque[k];
    }
  }
  for (int32_t i = 0; i < n; i++) {
    double im = o_inv_mass(c, &P[i]);
    double ii = o_inv_inertia(c, &P[i]);
    for (int k = 0; k < 3; k++) P[i].acc[k] = c->force[3 * i + k] * im;
    for (int k = 0; k < 3; k++) P[i].alpha[k] = c->torque[3 * i + k] * ii;
  }
  return DEM_OK;
}

/* ------------------------------------------------------------------ */
/* MDEM                                                                 */

/* ApplyPeriodicBoundaryConditions, src/MDEM.f90:373-388 */
static void apply_pbc_particles(orc_ctx* c, OParticle* P) {
  for (int k = 0; k < 3; k++) {
    if (c->p.pbc[k]) {
      for (int32_t i = 0; i < c->n; i++) {
        double pos = P[i].pos[k];
        P[i].pos[k] = pos - c->p.lbox[k] * fnint(pos * c->inv_lbox[k]);
      }
    }
  }
}

static inline OPrev* prev_at(orc_ctx* c, int32_t slot1 /* 1-based */, int32_t i) {
  return &c->prev[(size_t)(slot1 - 1) * (size_t)c->nalloc + (size_t)i];
}

/* ipc = cshift(ipc, shift=-1) */
static void cshift_ipc(orc_ctx* c) {
  if (c->nprev <= 0) return;
  int32_t last = c->ipc[c->nprev - 1];
  for (int k = c->nprev - 1; k > 0; k--) c->ipc[k] = c->ipc[k - 1];
  c->ipc[0] = last;
}

/* Euler, src/MDEM.f90:227-254 */
static int euler(orc_ctx* c, double TimeStep) {
  double TimeStepSqBy2 = 0.5 * (TimeStep * TimeStep);
  int st = compute_accelerations(c, c->part, TimeStep, 1);
  if (st) return st;
  for (int32_t i = 0; i < c->n; i++) {
    OParticle* q = &c->part[i];
    for (int k = 0; k < 3; k++)
      q->pos[k] = q->pos[k] + q->vel[k] * TimeStep + q->acc[k] * TimeStepSqBy2;
    for (int k = 0; k < 3; k++) q->vel[k] = q->vel[k] + q->acc[k] * TimeStep;
    for (int k = 0; k < 3; k++) q->omega[k] = q->omega[k] + q->alpha[k] * TimeStep;
  }
  return DEM_OK;
}

/* MoveWalls, src/MDEM.f90:392-408 (Pi as in src/MUtil.f90) */
static void move_walls(orc_ctx* c, double Time) {
  const double Pi = 3.1415926535897932384626433832795;
  const double TwoPi = 2.0 * Pi;
  for (int32_t j = 0; j < c->p.n_walls; j++) {
    const dem_wall_motion* m = &c->wm[j];
    for (int k = 0; k < 3; k++) {
      double Phase = m->two_pi_frequency[k] * Time + m->phase_angle[k];
      Phase = Phase - TwoPi * (double)(int)(Phase / TwoPi);
      c->p.walls[j].position[k] = m->constant_factor[k] + m->amplitude[k] * cos(Phase);
      c->p.walls[j].velocity[k] = m->velocity_amplitude[k] * sin(Phase);
    }
  }
}

/* MoveParticlesEuler, src/MDEM.f90:258-281 */
static int move_particles_euler(orc_ctx* c) {
  double NewTimeStep = c->p.time_step / (double)c->p.euler_intervals;
  cshift_ipc(c);
  if (c->nprev > 0) {
    for (int32_t i = 0; i < c->n; i++) {
      OPrev* pv = prev_at(c, c->ipc[0], i);
      memcpy(pv->v, c->part[i].vel, sizeof(double) * 3);
      memcpy(pv->a, c->part[i].acc, sizeof(double) * 3);
      memcpy(pv->al, c->part[i].alpha, sizeof(double) * 3);
    }
  }
  for (int32_t s = 0; s < c->p.euler_intervals; s++) {
    int st = euler(c, NewTimeStep);
    if (st) return st;
    c->time = c->time + NewTimeStep;
    if (c->moving) move_walls(c, c->time);
  }
  apply_pbc_particles(c, c->part);
  return DEM_OK;
}

/* MoveParticles, src/MDEM.f90:285-369 */
static int move_particles(orc_ctx* c, int32_t step) {
  int st = compute_accelerations(c, c->part, c->p.time_step, 1);
  if (st) return st;
  for (int32_t i = 0; i < c->n; i++) {
    double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < c->nprev; k++) {
      double ABk = c->AB[k];
      OPrev* pv = prev_at(c, c->ipc[k], i);
      for (int d = 0; d < 3; d++) sv[d] = sv[d] + ABk * pv->v[d];
      for (int d = 0; d < 3; d++) sa[d] = sa[d] + ABk * pv->a[d];
      for (int d = 0; d < 3; d++) sl[d] = sl[d] + ABk * pv->al[d];
    }
    OParticle* q = &c->part[i];
    OParticle* r = &c->pred[i];
    for (int d = 0; d < 3; d++) r->pos[d] = q->pos[d] + c->AB0 * q->vel[d] + sv[d];
    for (int d = 0; d < 3; d++) r->vel[d] = q->vel[d] + c->AB0 * q->acc[d] + sa[d];
    for (int d = 0; d < 3; d++) r->omega[d] = q->omega[d] + c->AB0 * q->alpha[d] + sl[d];
  }
  apply_pbc_particles(c, c->pred);
  cshift_ipc(c);
  if (c->nprev > 0) {
    for (int32_t i = 0; i < c->n; i++) {
      OPrev* pv = prev_at(c, c->ipc[0], i);
      memcpy(pv->v, c->part[i].vel, sizeof(double) * 3);
      memcpy(pv->a, c->part[i].acc, sizeof(double) * 3);
      memcpy(pv->al, c->part[i].alpha, sizeof(double) * 3);
    }
  }
  c->time = (double)step * c->p.time_step;
  if (c->moving) move_walls(c, c->time);
  st = compute_accelerations(c, c->pred, c->p.time_step, 0);
  if (st) return st;
  for (int32_t i = 0; i < c->n; i++) {
    double sv[3] = {0.0, 0.0, 0.0}, sa[3] = {0.0, 0.0, 0.0}, sl[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < c->nprev; k++) {
      double AMk = c->AM[k];
      OPrev* pv = prev_at(c, c->ipc[k], i);
      for (int d = 0; d < 3; d++) sv[d] = sv[d] + AMk * pv->v[d];
      for (int d = 0; d < 3; d++) sa[d] = sa[d] + AMk * pv->a[d];
      for (int d = 0; d < 3; d++) sl[d] = sl[d] + AMk * pv->al[d];
    }
    OParticle* q = &c->part[i];
    OParticle* r = &c->pred[i];
    for (int d = 0; d < 3; d++) q->pos[d] = q->pos[d] + c->AM0 * r->vel[d] + sv[d];
    for (int d = 0; d < 3; d++) q->vel[d] = q->vel[d] + c->AM0 * r->acc[d] + sa[d];
    for (int d = 0; d < 3; d++) q->omega[d] = q->omega[d] + c->AM0 * r->alpha[d] + sl[d];
  }
  apply_pbc_particles(c, c->part);
  return DEM_OK;
}

/* ------------------------------------------------------------------ */
/* UpdateParticleList (src/MDEM.f90:612-671): particles that left the   */
/* box are removed; the last particle takes the place of each one.      */

/* AllNeighbourParticles (src/MCells.f90:833-860) over the MonteCarlo list
 * of iCell (NeighbourCells3D with MonteCarlo, :353-375, AddAllNeighbours3D
 * :424-476): the particles of iCell, then of each neighbour cell in list
 * order -- AddNeighbour prepends (:666-680), so the list runs opposite to
 * the loops that build it. */
static int32_t all_neighbour_particles(orc_ctx* c, int32_t iCell, int32_t** out) {
  int32_t iz = iCell / (c->Nx * c->Ny);
  int32_t iy = iCell / c->Nx - iz * c->Ny;
  int32_t ix = iCell - (iy + iz * c->Ny) * c->Nx;
  const int pbc[3] = {c->p.pbc[0], c->p.pbc[1], c->p.pbc[2]};
  const int32_t N[3] = {c->Nx, c->Ny, c->Nz};
  const int32_t I[3] = {ix, iy, iz};
  int32_t lo[3], hi[3];
  for (int d = 0; d < 3; d++) { /* VerifyPBC, :1030-1040 */
    lo[d] = -1;
    hi[d] = 1;
    if (!pbc[d]) {
      if (I[d] == 0) lo[d] = 0;
      if (I[d] == N[d] - 1) hi[d] = 0;
    }
  }
  int32_t built[26], nb_cells = 0;
  for (int32_t kz = lo[2]; kz <= hi[2]; kz++)
    for (int32_t ky = lo[1]; ky <= hi[1]; ky++)
      for (int32_t kx = lo[0]; kx <= hi[0]; kx++) {
        if (kx == 0 && ky == 0 && kz == 0) continue;
        int32_t j[3] = {ix + kx, iy + ky, iz + kz};
        for (int d = 0; d < 3; d++) /* ApplyPBC, :1044-1052 */
          if (pbc[d]) {
            if (j[d] == N[d]) j[d] = 0;
            if (j[d] == -1) j[d] = N[d] - 1;
          }
        built[nb_cells++] = j[0] + c->Nx * (j[1] + c->Ny * j[2]);
      }
  int32_t cells[27], m = 0;
  cells[m++] = iCell;
  for (int32_t k = nb_cells - 1; k >= 0; k--) cells[m++] = built[k];
  int32_t cnt = 0;
  for (int k = 0; k < m; k++)
    for (CNode* q = c->cell[cells[k]].first_particle; q; q = q->next) cnt++;
  int32_t* nb = (int32_t*)malloc(sizeof(int32_t) * (size_t)(cnt > 0 ? cnt : 1));
  cnt = 0;
  for (int k = 0; k < m; k++)
    for (CNode* q = c->cell[cells[k]].first_particle; q; q = q->next) nb[cnt++] = q->index;
  *out = nb;
  return cnt;
}

/* RemoveParticleFromCell (src/MCells.f90:702-724) */
static void remove_particle_from_cell(orc_ctx* c, int32_t i, int32_t iCell) {
  CNode* cur = c->cell[iCell].first_particle;
  if (cur->index == i) {
    c->cell[iCell].first_particle = cur->next;
    free(cur);
  } else {
    while (cur->next->index != i) cur = cur->next;
    CNode* aux = cur->next;
    cur->next = aux->next;
    free(aux);
  }
}

/* ReplaceParticleIndexInCell (src/MCells.f90:728-743) */
static void replace_particle_index_in_cell(orc_ctx* c, int32_t i, int32_t iCell, int32_t j) {
  CNode* cur = c->cell[iCell].first_particle;
  while (cur->index != i) cur = cur->next;
  cur->index = j;
}

static void free_partners(Partner* p) {
  while (p) { Partner* a = p; p = p->next; free(a); }
}

/* RemoveParticleFromContactList (src/MContacts.f90:579-633) */
static void remove_particle_from_contact_list(orc_ctx* c, int32_t i, int32_t npsc,
                                              const int32_t* nb) {
  for (int32_t jj = 0; jj < npsc; jj++) {
    int32_t j = nb[jj];
    Partner* cur = c->mainp[j].first_partner;
    if (!cur) continue;
    Partner* prev = cur;
    while (cur->index < i && cur->next) {
      prev = cur;
      cur = cur->next;
    }
    if (cur->index == i) {
      if (prev->index == i) c->mainp[j].first_partner = cur->next;
      else prev->next = cur->next;
      free(cur);
    }
  }
  free_partners(c->mainp[i].first_partner);
  free_partners(c->mainp[i].first_wall);
  c->mainp[i].first_partner = NULL;
  c->mainp[i].first_wall = NULL;
}

/* ChangeIndexInContactList (src/MContacts.f90:173-252), NP -> i.  One
 * deliberate deviation: the records that particle i inherits as main
 * particle (partners j > i of NP) are inserted in index order, where the
 * reference appends them in neighbour order (:225-241).  An appended list can
 * be out of order, and the reference's ordered search (VerifyPairContact,
 * src/MContacts.f90:329-372) then misses some of its records; keeping the
 * list ordered keeps every record reachable. */
static void change_index_in_contact_list(orc_ctx* c, int32_t NP, int32_t i, int32_t npsc,
                                         const int32_t* nb, int64_t* moved) {
  Partner* first = NULL;
  for (int32_t jj = 0; jj < npsc; jj++) {
    int32_t j = nb[jj];
    Partner* cur = c->mainp[j].first_partner;
    if (!cur) continue;
    if (j < i) {
      Partner *prev = NULL, *point = NULL;
      while (cur->next) {
        prev = cur;
        if (cur->index < i) point = cur;
        cur = cur->next;
      }
      if (cur->index == NP) {
        (*moved)++;
        if (prev) {
          prev->next = cur->next;
          cur->index = i;
          if (point) {
            cur->next = point->next;
            point->next = cur;
          } else {
            cur->next = c->mainp[j].first_partner;
            c->mainp[j].first_partner = cur;
          }
        } else {
          cur->index = i;
        }
      }
    } else {
      Partner* prev = NULL;
      while (cur->next) {
        prev = cur;
        cur = cur->next;
      }
      if (cur->index == NP) {
        (*moved)++;
        cur->index = j;
        if (prev) prev->next = NULL;
        else c->mainp[j].first_partner = NULL;
        Partner** at = &first;
        if (c->literal_removal) {
          /* the reference's append in neighbour order (src/MContacts.f90:225-241) */
          while (*at) at = &(*at)->next;
        } else {
          /* ordered insert into i's new list (see above) */
          while (*at && (*at)->index < j) at = &(*at)->next;
        }
        cur->next = *at;
        *at = cur;
      }
    }
  }
  c->mainp[i].first_partner = first;
  c->mainp[i].first_wall = c->mainp[NP].first_wall;
  c->mainp[NP].first_wall = NULL;
  /* NP's own partner list is not carried over; it lies beyond the new NP */
  free_partners(c->mainp[NP].first_partner);
  c->mainp[NP].first_partner = NULL;
}

static int update_particle_list(orc_ctx* c, int64_t* removed) {
  int64_t nrem = 0;
  for (int32_t i = c->n - 1; i >= 0; i--) {
    const OParticle* q = &c->part[i];
    int out = 0;
    for (int k = 0; k < 3; k++) {
      const double h = 0.5 * c->p.lbox[k];
      if (q->pos[k] > h || q->pos[k] < -h) out = 1;
    }
    if (!out) continue;
    if (c->p.n_components > 0) c->comp_count[q->index]--;
    int32_t iCell = c->cell_index[i];
    int32_t* nb = NULL;
    int32_t npsc = all_neighbour_particles(c, iCell, &nb);
    remove_particle_from_cell(c, i, iCell);
    remove_particle_from_contact_list(c, i, npsc, nb);
    int32_t NP = c->n - 1;
    if (i != NP) {
      c->part[i] = c->part[NP];
      c->pred[i].index = c->part[NP].index;
      c->pred[i].radius = c->part[NP].radius;
      for (int32_t k = 1; k <= c->nprev; k++) *prev_at(c, k, i) = *prev_at(c, k, NP);
      replace_particle_index_in_cell(c, NP, c->cell_index[NP], i);
      c->cell_index[i] = c->cell_index[NP];
      change_index_in_contact_list(c, NP, i, npsc, nb, &c->removal_moved);
      c->removal_swaps++;
    }
    free(nb);
    c->n = NP;
    nrem++;
  }
  c->removal_count += nrem;
  if (removed) *removed = nrem;
  return DEM_OK;
}

/* ------------------------------------------------------------------ */
/* Pouring (PourParticle / InsertParticle, src/MDEM.f90:412-561)         */

/* ranf (src/MUtil.f90:17-48): Marsaglia shift register combined with the
 * Park-Miller generator (Schrage's method).  aam is computed in default
 * (single) precision, as nearest(1.0,-1.0)/IM is, then widened. */
static double ranf(dem_rng* r) {
  const int32_t IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836;
  if (r->dummy <= 0 || r->iiy < 0) {
    volatile float one_minus = nextafterf(1.0f, -1.0f);
    volatile float a = one_minus / (float)IM;
    int32_t ad = r->dummy < 0 ? -r->dummy : r->dummy;
    r->aam = (double)a;
    r->iiy = (888889999 ^ ad) | 1;
    r->iix = 777755555 ^ ad;
    r->dummy = ad + 1;
  }
  uint32_t x = (uint32_t)r->iix;
  x ^= x << 13; /* ishft(iix,13) */
  x ^= x >> 17; /* ishft(iix,-17): logical shift */
  x ^= x << 5;
  r->iix = (int32_t)x;
  r->iik = r->iiy / IQ;
  r->iiy = IA * (r->iiy - r->iik * IQ) - IR * r->iik;
  if (r->iiy < 0) r->iiy += IM;
  return r->aam * (double)((IM & (r->iix ^ r->iiy)) | 1);
}

/* room for `cap` particles (ResizeVariables grows MaxNP, src/MDEM.f90:565-608) */
static void reserve_particles(orc_ctx* c, int32_t cap) {
  if (cap <= c->nalloc) return;
  size_t N = (size_t)cap, n = (size_t)c->n;
  c->part = (OParticle*)realloc(c->part, N * sizeof(OParticle));
  c->pred = (OParticle*)realloc(c->pred, N * sizeof(OParticle));
  c->cell_index = (int32_t*)realloc(c->cell_index, N * sizeof(int32_t));
  c->mainp = (OMain*)realloc(c->mainp, N * sizeof(OMain));
  memset(c->mainp + n, 0, (N - n) * sizeof(OMain));
  c->force = (double*)realloc(c->force, 3 * N * sizeof(double));
  c->torque = (double*)realloc(c->torque, 3 * N * sizeof(double));
  int32_t slots = c->nprev > 0 ? c->nprev : 1;
  OPrev* pv = (OPrev*)calloc(N * (size_t)slots, sizeof(OPrev));
  for (int32_t k = 0; k < c->nprev; k++)
    memcpy(pv + (size_t)k * N, c->prev + (size_t)k * c->nalloc, n * sizeof(OPrev));
  free(c->prev);
  c->prev = pv;
  c->nalloc = cap;
}

/* InsertParticle (src/MDEM.f90:536-561) */
static void insert_particle(orc_ctx* c, const OParticle* part) {
  if (c->n == c->nalloc) {
    int32_t grown = (int32_t)(1.05 * (double)c->nalloc);
    reserve_particles(c, grown > c->nalloc + 1 ? grown : c->nalloc + 1);
  }
  int32_t NP = c->n;
  c->n = NP + 1;
  c->comp_count[part->index]++;
  c->part[NP] = *part;
  c->pred[NP].index = part->index;
  c->pred[NP].radius = part->radius;
  for (int32_t k = 1; k <= c->nprev; k++) memset(prev_at(c, k, NP), 0, sizeof(OPrev));
  c->cell_index[NP] = current_cell(c, part->pos[0], part->pos[1], part->pos[2]);
  add_particle(c, NP, c->cell_index[NP]);
  c->mainp[NP].first_partner = NULL;
  c->mainp[NP].first_wall = NULL;
}

/* PourParticle (src/MDEM.f90:412-532).  As in the reference, every attempt
 * tests the largest component's radius (the "<test>" lines), and the
 * particle-particle test squares the separation converted to integer(ib):
 * Rij is declared integer there, so each component is truncated. */
static int pour_particle(orc_ctx* c, int32_t* inserted) {
  *inserted = 0;
  const dem_pouring* P = &c->pour;
  const int32_t NC = c->p.n_components;
  int32_t not_reached[NCM], nnr = 0;
  for (int32_t k = 0; k < NC; k++)
    if (c->comp_count[k] < P->target_number[k]) not_reached[nnr++] = k;
  if (nnr == 0) return DEM_OK;
  int32_t j = (int32_t)((double)nnr * ranf(&c->rng));
  OParticle iPart;
  memset(&iPart, 0, sizeof(iPart));
  iPart.index = not_reached[j];
  int32_t iBig = 0;
  for (int32_t k = 1; k < NC; k++)
    if (c->p.comp_radius[k] > c->p.comp_radius[iBig]) iBig = k;
  const double Ri = c->p.comp_radius[iBig];
  const double Di = 2.0 * Ri;
  iPart.pos[2] = 0.5 * c->p.lbox[2] - Ri;
  const double TwoPi = 2.0 * 3.1415926535897932384626433832795;
  int possible = 0;
  int32_t attempt = 0;
  while (!possible && attempt < P->max_attempts) {
    possible = 1;
    attempt++;
    if (P->shape == DEM_POUR_RECTANGLE) {
      for (int k = 0; k < 2; k++) iPart.pos[k] = (P->size[k] - Di) * (ranf(&c->rng) - 0.5);
    } else {
      double Rad = 0.5 * ranf(&c->rng) * (P->size[0] - Di);
      double Angle = TwoPi * ranf(&c->rng);
      iPart.pos[0] = Rad * sin(Angle);
      iPart.pos[1] = Rad * cos(Angle);
    }
    int32_t iCell = current_cell(c, iPart.pos[0], iPart.pos[1], iPart.pos[2]);
    int32_t* nb = NULL;
    int32_t npsc = all_neighbour_particles(c, iCell, &nb);
    for (int32_t jj = 0; possible && jj < npsc; jj++) {
      const OParticle* jPart = &c->part[nb[jj]];
      int32_t R[3];
      for (int k = 0; k < 3; k++) R[k] = (int32_t)(jPart->pos[k] - iPart.pos[k]);
      int32_t s = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
      possible = (double)s > c->p.min_dij_sq[iBig * NCM + jPart->index];
    }
    free(nb);
    for (int32_t w = 0; possible && w < c->p.n_walls; w++) {
      double Dij, Nij[3], Qji[3];
      possible = !overlap_wall(c, &iPart, &c->p.walls[w], Ri, &Dij, Nij, Qji);
    }
  }
  if (possible) {
    iPart.vel[2] = P->velocity_z;
    insert_particle(c, &iPart);
    *inserted = 1;
  }
  return DEM_OK;
}

/* ------------------------------------------------------------------ */
/* public API (mirrors include/dem3d_b200.h with an orc_ prefix)        */

const char* orc_last_error(const orc_ctx* c) { return c ? c->err : "null context"; }

int orc_create(const dem_params* p, orc_ctx** out) {
  if (!p || !out) return DEM_ERR_INVALID;
  if (p->method_order < 1 || p->method_order > 4) return DEM_ERR_INVALID;
  if (p->n_walls < 0 || p->n_walls > NWM) return DEM_ERR_INVALID;
  if (p->n_components < 0 || p->n_components > NCM) return DEM_ERR_INVALID;
  if (p->euler_intervals < 1) return DEM_ERR_INVALID;
  for (int w = 0; w < p->n_walls; w++)
    if (p->walls[w].shape != DEM_WALL_RECTANGLE && p->walls[w].shape != DEM_WALL_CONE)
      return DEM_ERR_UNSUPPORTED;
  orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
  c->removal = 1; /* the main loop always calls UpdateParticleList (src/DEM.f90:96) */
  c->rng.iix = -1;  /* src/MUtil.f90:11 */
  c->rng.iiy = -1;
  c->p = *p;
  for (int k = 0; k < 3; k++) c->inv_lbox[k] = 1.0 / p->lbox[k];
  /* InitializeAuxiliaries, src/MDEM.f90:110-162 */
  c->nprev = p->method_order - 1;
  double dt = p->time_step;
  switch (p->method_order) {
    case 4: {
      double Aux = dt / 24.0;
      c->AB0 = 55.0 * Aux; c->AM0 = 9.0 * Aux;
      c->AB[0] = -59.0 * Aux; c->AM[0] = 19.0 * Aux;
      c->AB[1] = 37.0 * Aux; c->AM[1] = -5.0 * Aux;
      c->AB[2] = -9.0 * Aux; c->AM[2] = 1.0 * Aux;
    } break;
    case 3: {
      double Aux = dt / 12.0;
      c->AB0 = 23.0 * Aux; c->AM0 = 5.0 * Aux;
      c->AB[0] = -16.0 * Aux; c->AM[0] = 8.0 * Aux;
      c->AB[1] = 5.0 * Aux; c->AM[1] = -1.0 * Aux;
    } break;
    case 2:
      c->AB0 = 1.5 * dt; c->AM0 = 0.5 * dt;
      c->AB[0] = -0.5 * dt; c->AM[0] = 0.5 * dt;
      break;
    default:
      c->AB0 = dt; c->AM0 = dt;
  }
  /* InitializeCellList, src/MForces.f90:91-106 */
  double rmax = 0.0;
  if (p->n_components > 0) {
    for (int i = 0; i < p->n_components; i++)
      rmax = p->comp_radius[i] > rmax ? p->comp_radius[i] : rmax;
  } else {
    rmax = p->pp_rmax;
  }
  double CutOff = 2.0 * rmax;
  if (!(CutOff > 0.0)) { free(c); return DEM_ERR_INVALID; }
  init_cell_structure(c, p->lbox[0], p->lbox[1], p->lbox[2], CutOff,
                      p->max_ncell > 0 ? p->max_ncell : 30000);
  if (c->Nx < 1 || c->Ny < 1 || c->Nz < 1) { free(c->cell); free(c); return DEM_ERR_INVALID; }
  full_neighbour_cells(c);
  *out = c;
  return DEM_OK;
}

void orc_destroy(orc_ctx* c) {
  if (!c) return;
  destroy_cells(c);
  free(c->cell);
  destroy_contacts(c);
  free(c->mainp);
  free(c->part);
  free(c->pred);
  free(c->prev);
  free(c->cell_index);
  free(c->neighbour);
  free(c->force);
  free(c->torque);
  free(c->vf);
  free(c->ef);
  free(c);
}

/* test hook: the reference's unordered append in ChangeIndexInContactList */
int orc_set_literal_removal(orc_ctx* c, int32_t on) {
  c->literal_removal = on != 0;
  return DEM_OK;
}

int orc_set_literal_neighbour_cap(orc_ctx* c, int32_t cap) {
  c->literal_neighbour_cap = cap;
  if (cap > 0) {
    c->neighbour = (int32_t*)realloc(c->neighbour, sizeof(int32_t) * (size_t)cap);
    c->neighbour_cap = cap;
  }
  return DEM_OK;
}

int orc_set_state(orc_ctx* c, int32_t n, const int32_t* comp, const double* radius,
                  const double* pos, const double* vel, const double* omega,
                  const double* acc, const double* alpha) {
  if (n < 0 || !pos || !vel || !omega) return DEM_ERR_INVALID;
  if (c->p.n_components > 0 && !comp) return DEM_ERR_INVALID;
  if (c->p.n_components == 0 && !radius) return DEM_ERR_INVALID;
  clear_cell_particles(c);
  destroy_contacts(c);
  free(c->mainp);
  free(c->part);
  free(c->pred);
  free(c->prev);
  free(c->cell_index);
  free(c->force);
  free(c->torque);
  c->n = n;
  c->nalloc = n;
  size_t N = (size_t)(n > 0 ? n : 1);
  c->part = (OParticle*)calloc(N, sizeof(OParticle));
  c->pred = (OParticle*)calloc(N, sizeof(OParticle));
  c->prev = (OPrev*)calloc(N * (size_t)(c->nprev > 0 ? c->nprev : 1), sizeof(OPrev));
  c->cell_index = (int32_t*)calloc(N, sizeof(int32_t));
  c->mainp = (OMain*)calloc(N, sizeof(OMain));
  c->force = (double*)calloc(3 * N, sizeof(double));
  c->torque = (double*)calloc(3 * N, sizeof(double));
  for (int32_t i = 0; i < n; i++) {
    OParticle* q = &c->part[i];
    q->index = comp ? comp[i] : 0;
    if (c->p.n_components > 0 && (q->index < 0 || q->index >= c->p.n_components))
      return DEM_ERR_INVALID;
    q->radius = radius ? radius[i] : 0.0;
    for (int k = 0; k < 3; k++) {
      q->pos[k] = pos[3 * i + k];
      q->vel[k] = vel[3 * i + k];
      q->omega[k] = omega[3 * i + k];
      q->acc[k] = acc ? acc[3 * i + k] : 0.0;
      q->alpha[k] = alpha ? alpha[3 * i + k] : 0.0;
    }
    c->pred[i].index = q->index;
    c->pred[i].radius = q->radius;
  }
  memset(c->comp_count, 0, sizeof(c->comp_count));
  if (c->p.n_components > 0)
    for (int32_t i = 0; i < n; i++) c->comp_count[c->part[i].index]++;
  for (int k = 0; k < c->nprev; k++) c->ipc[k] = k + 1;
  c->ncol = 0;
  c->cells_ready = 0;
  c->time = 0.0;
  return DEM_OK;
}

static void copy_out(const OParticle* P, int32_t n, double* pos, double* vel, double* omega,
                     double* acc, double* alpha) {
  for (int32_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      if (pos) pos[3 * i + k] = P[i].pos[k];
      if (vel) vel[3 * i + k] = P[i].vel[k];
      if (omega) omega[3 * i + k] = P[i].omega[k];
      if (acc) acc[3 * i + k] = P[i].acc[k];
      if (alpha) alpha[3 * i + k] = P[i].alpha[k];
    }
}

int orc_get_state(orc_ctx* c, double* pos, double* vel, double* omega, double* acc,
                  double* alpha) {
  copy_out(c->part, c->n, pos, vel, omega, acc, alpha);
  return DEM_OK;
}

int orc_update_state(orc_ctx* c, const double* pos, const double* vel, const double* omega,
                     const double* acc, const double* alpha) {
  const double* in[5] = {pos, vel, omega, acc, alpha};
  for (int32_t i = 0; i < c->n; i++) {
    OParticle* q = &c->part[i];
    double* f[5] = {q->pos, q->vel, q->omega, q->acc, q->alpha};
    for (int a = 0; a < 5; a++)
      if (in[a])
        for (int k = 0; k < 3; k++) f[a][k] = in[a][3 * i + k];
  }
  return DEM_OK;
}

int orc_get_predicted(orc_ctx* c, double* pos, double* vel, double* omega, double* acc,
                      double* alpha) {
  copy_out(c->pred, c->n, pos, vel, omega, acc, alpha);
  return DEM_OK;
}

int orc_get_n(orc_ctx* c, int32_t* n) { *n = c->n; return DEM_OK; }

int orc_set_wall_motion(orc_ctx* c, const dem_wall_motion* m) {
  if (!c) return DEM_ERR_INVALID;
  if (!m) { c->moving = 0; return DEM_OK; }
  for (int32_t j = 0; j < c->p.n_walls; j++) c->wm[j] = m[j];
  c->moving = 1;
  return DEM_OK;
}

int orc_get_walls(orc_ctx* c, dem_wall* walls) {
  if (!c || !walls) return DEM_ERR_INVALID;
  for (int32_t j = 0; j < c->p.n_walls; j++) walls[j] = c->p.walls[j];
  return DEM_OK;
}

int orc_set_integration(orc_ctx* c, const double* previous, const int32_t* ipc) {
  for (int k = 0; k < c->nprev; k++) {
    c->ipc[k] = ipc[k];
    for (int32_t i = 0; i < c->n; i++) {
      OPrev* pv = &c->prev[(size_t)k * c->nalloc + i];
      const double* s = previous + ((size_t)k * c->n + i) * 9;
      memcpy(pv->v, s, 24);
      memcpy(pv->a, s + 3, 24);
      memcpy(pv->al, s + 6, 24);
    }
  }
  return DEM_OK;
}

int orc_get_integration(orc_ctx* c, double* previous, int32_t* ipc) {
  for (int k = 0; k < c->nprev; k++) {
    if (ipc) ipc[k] = c->ipc[k];
    if (previous)
      for (int32_t i = 0; i < c->n; i++) {
        const OPrev* pv = &c->prev[(size_t)k * c->nalloc + i];
        double* d = previous + ((size_t)k * c->n + i) * 9;
        memcpy(d, pv->v, 24);
        memcpy(d + 3, pv->a, 24);
        memcpy(d + 6, pv->al, 24);
      }
  }
  return DEM_OK;
}

int orc_set_contacts(orc_ctx* c, int64_t m, const int32_t* imin, const int32_t* imax,
                     const double* ft, const double* vt, int64_t mw, const int32_t* ip,
                     const int32_t* iw, const double* ftw, const double* vtw) {
  destroy_contacts(c);
  for (int64_t r = 0; r < m; r++) {
    /* a partner past the last particle is a record left by particle removal */
    if (imin[r] < 0 || imin[r] >= c->n || imin[r] >= imax[r]) return DEM_ERR_INVALID;
    insert_sorted(&c->mainp[imin[r]].first_partner, imax[r], ft + 3 * r, vt + 3 * r);
  }
  for (int64_t r = 0; r < mw; r++) {
    if (ip[r] < 0 || ip[r] >= c->n || iw[r] < 0 || iw[r] >= c->p.n_walls) return DEM_ERR_INVALID;
    insert_sorted(&c->mainp[ip[r]].first_wall, iw[r], ftw + 3 * r, vtw + 3 * r);
  }
  return DEM_OK;
}

int orc_count_contacts(orc_ctx* c, int64_t* np, int64_t* nw) {
  int64_t a = 0, b = 0;
  for (int32_t i = 0; i < c->n; i++) {
    for (Partner* p = c->mainp[i].first_partner; p; p = p->next) a++;
    for (Partner* p = c->mainp[i].first_wall; p; p = p->next) b++;
  }
  if (np) *np = a;
  if (nw) *nw = b;
  return DEM_OK;
}

int orc_get_contacts(orc_ctx* c, int64_t cap, int32_t* imin, int32_t* imax, double* ft,
                     double* vt, int64_t capw, int32_t* ip, int32_t* iw, double* ftw,
                     double* vtw) {
  int64_t a = 0, b = 0;
  for (int32_t i = 0; i < c->n; i++) {
    for (Partner* p = c->mainp[i].first_partner; p; p = p->next) {
      if (a >= cap) return DEM_ERR_CAPACITY;
      imin[a] = i;
      imax[a] = p->index;
      memcpy(ft + 3 * a, p->v1, 24);
      memcpy(vt + 3 * a, p->v2, 24);
      a++;
    }
    for (Partner* p = c->mainp[i].first_wall; p; p = p->next) {
      if (b >= capw) return DEM_ERR_CAPACITY;
      ip[b] = i;
      iw[b] = p->index;
      memcpy(ftw + 3 * b, p->v1, 24);
      memcpy(vtw + 3 * b, p->v2, 24);
      b++;
    }
  }
  return DEM_OK;
}

int orc_initialize_cell_distribution(orc_ctx* c) {
  clear_cell_particles(c);
  distribute_particles(c);
  c->cells_ready = 1;
  return DEM_OK;
}

int orc_get_grid(orc_ctx* c, int32_t* nxyz) {
  nxyz[0] = c->Nx;
  nxyz[1] = c->Ny;
  nxyz[2] = c->Nz;
  return DEM_OK;
}

int orc_get_cell_count(orc_ctx* c, int32_t* ncell) {
  *ncell = c->Nt;
  return DEM_OK;
}

int orc_get_cells(orc_ctx* c, int32_t* cell_index, int32_t* traversal, int32_t* cell_start) {
  if (cell_index) memcpy(cell_index, c->cell_index, sizeof(int32_t) * (size_t)c->n);
  int32_t k = 0;
  for (int32_t i = 0; i < c->Nt; i++) {
    if (cell_start) cell_start[i] = k;
    for (CNode* p = c->cell[i].first_particle; p; p = p->next) {
      if (traversal) traversal[k] = p->index;
      k++;
    }
  }
  if (cell_start) cell_start[c->Nt] = k;
  return DEM_OK;
}

/* ReadCellDistribution (src/MForces.f90:121-131): CellIndex from the
 * positions, then the lists as stored (ReadCellStructure, src/MCells.f90:
 * 988-1026).  The lists must hold every particle once, in its own cell. */
int orc_set_cells(orc_ctx* c, const int32_t* traversal, const int32_t* cell_start) {
  if (!c || !traversal || !cell_start) return DEM_ERR_INVALID;
  if (cell_start[0] != 0 || cell_start[c->Nt] != c->n) return DEM_ERR_INVALID;
  for (int32_t i = 0; i < c->n; i++)
    c->cell_index[i] = current_cell(c, c->part[i].pos[0], c->part[i].pos[1], c->part[i].pos[2]);
  char* seen = (char*)calloc((size_t)(c->n > 0 ? c->n : 1), 1);
  int bad = 0;
  for (int32_t cc = 0; cc < c->Nt && !bad; cc++) {
    if (cell_start[cc + 1] < cell_start[cc]) { bad = 1; break; }
    for (int32_t k = cell_start[cc]; k < cell_start[cc + 1]; k++) {
      int32_t q = traversal[k];
      if (q < 0 || q >= c->n || seen[q] || c->cell_index[q] != cc) { bad = 1; break; }
      seen[q] = 1;
    }
  }
  free(seen);
  if (bad) return DEM_ERR_INVALID;
  clear_cell_particles(c);
  for (int32_t cc = 0; cc < c->Nt; cc++)
    for (int32_t k = cell_start[cc + 1] - 1; k >= cell_start[cc]; k--)
      add_particle(c, traversal[k], cc);  /* prepending in reverse keeps the order */
  c->cells_ready = 1;
  return DEM_OK;
}

/* FluidFlow and InitializeFluid (src/mFluid.f90:72-92) */
int orc_set_fluid(orc_ctx* c, const dem_fluid* f) {
  if (!c) return DEM_ERR_INVALID;
  free(c->vf);
  free(c->ef);
  c->vf = c->ef = NULL;
  c->fluid = 0;
  if (!f) return DEM_OK;
  if (c->p.n_components <= 0) return DEM_ERR_UNSUPPORTED;
  if (f->levels < 1 || !(f->viscosity > 0.0)) return DEM_ERR_INVALID;
  c->fl = *f;
  c->fl_area = c->p.lbox[0] * c->p.lbox[1];
  c->fl_dz = c->p.lbox[2] / (double)f->levels;
  c->fl_vf0 = f->flow_rate / c->fl_area;
  c->fl_h2 = c->p.lbox[2] / 2.0;
  c->fl_mh2 = -c->fl_h2;
  c->vf = (double*)calloc((size_t)f->levels + 1, sizeof(double));
  c->ef = (double*)calloc((size_t)f->levels + 1, sizeof(double));
  c->fluid = 1;
  return DEM_OK;
}

int orc_set_pouring(orc_ctx* c, const dem_pouring* p) {
  if (!c) return DEM_ERR_INVALID;
  if (!p) { c->pouring = 0; return DEM_OK; }
  if (c->p.n_components <= 0) return DEM_ERR_UNSUPPORTED;
  if (p->interval < 1 || p->max_attempts < 0 ||
      (p->shape != DEM_POUR_RECTANGLE && p->shape != DEM_POUR_CIRCLE))
    return DEM_ERR_INVALID;
  c->pour = *p;
  c->pouring = 1;
  return DEM_OK;
}

int orc_pour_particle(orc_ctx* c, int32_t* inserted) {
  if (!c || !c->cells_ready) return DEM_ERR_STATE;
  int32_t ins = 0;
  int st = pour_particle(c, &ins);
  if (inserted) *inserted = ins;
  return st;
}

int orc_set_rng(orc_ctx* c, const dem_rng* r) {
  if (!c || !r) return DEM_ERR_INVALID;
  c->rng = *r;
  return DEM_OK;
}

/* test hook: `count` successive ranf values from state r (r advances) */
int orc_ranf(dem_rng* r, int32_t count, double* out) {
  for (int32_t k = 0; k < count; k++) out[k] = ranf(r);
  return DEM_OK;
}

int orc_get_rng(orc_ctx* c, dem_rng* r) {
  if (!c || !r) return DEM_ERR_INVALID;
  *r = c->rng;
  return DEM_OK;
}

int orc_update_particle_list(orc_ctx* c, int64_t* removed) {
  if (!c || !c->cells_ready) return DEM_ERR_STATE;
  return update_particle_list(c, removed);
}

int orc_set_particle_removal(orc_ctx* c, int32_t enable) {
  if (!c) return DEM_ERR_INVALID;
  c->removal = enable != 0;
  return DEM_OK;
}

int orc_get_components(orc_ctx* c, int32_t* comp) {
  if (!c || !comp) return DEM_ERR_INVALID;
  for (int32_t i = 0; i < c->n; i++) comp[i] = c->part[i].index;
  return DEM_OK;
}

/* test diagnostics: removals, swaps with the last particle, records renamed */
int orc_get_removal_stats(orc_ctx* c, int64_t* stats) {
  stats[0] = c->removal_count;
  stats[1] = c->removal_swaps;
  stats[2] = c->removal_moved;
  return DEM_OK;
}

int orc_set_ncol(orc_ctx* c, int64_t ncol) {
  if (!c || ncol < 0) return DEM_ERR_INVALID;
  c->ncol = ncol;
  return DEM_OK;
}

int orc_compute_accelerations(orc_ctx* c, int32_t use_predicted, double time_step,
                              int32_t update) {
  if (!c->cells_ready) return DEM_ERR_STATE;
  return compute_accelerations(c, use_predicted ? c->pred : c->part, time_step, update);
}

/* ComputeAccelerations' Force and Torque arrays (src/MForces.f90:154,
 * summed at :319-320), rows of three as the pass left them */
int orc_compute_forces(orc_ctx* c, int32_t use_predicted, double time_step, int32_t update,
                       double* force, double* torque) {
  if (!force || !torque) return DEM_ERR_INVALID;
  int st = orc_compute_accelerations(c, use_predicted, time_step, update);
  if (st) return st;
  memcpy(force, c->force, sizeof(double) * 3 * (size_t)c->n);
  memcpy(torque, c->torque, sizeof(double) * 3 * (size_t)c->n);
  return DEM_OK;
}

int orc_move_particles(orc_ctx* c, int32_t step) {
  if (!c->cells_ready) return DEM_ERR_STATE;
  return move_particles(c, step);
}

int orc_move_particles_euler(orc_ctx* c) {
  if (!c->cells_ready) return DEM_ERR_STATE;
  return move_particles_euler(c);
}

/* the time loop of src/DEM.f90:85-99 (no pouring / periodic tasks) */
int orc_run(orc_ctx* c, int32_t first_step, int32_t last_step) {
  if (!c->cells_ready) return DEM_ERR_STATE;
  int32_t s0 = first_step;
  if (first_step == 1) {
    for (int32_t s = 1; s <= c->p.method_order - 1; s++) {
      int st = move_particles_euler(c);
      if (st) return st;
    }
    s0 = c->p.method_order;
  }
  for (int32_t s = s0; s <= last_step; s++) {
    if (c->pouring && s % c->pour.interval == 0) { /* PouringAttempt (src/DEM.f90:115-123) */
      int32_t ins;
      pour_particle(c, &ins);
    }
    int st = move_particles(c, s);
    if (st) return st;
    if (c->removal) update_particle_list(c, NULL);
  }
  return DEM_OK;
}

int orc_get_ncol(orc_ctx* c, int64_t* ncol) { *ncol = c->ncol; return DEM_OK; }

/* particles outside +-L/2 (UpdateParticleList test, src/MDEM.f90:624-625) */
int orc_get_escaped(orc_ctx* c, int64_t* count) {
  int64_t k = 0;
  for (int32_t i = 0; i < c->n; i++) {
    int out = 0;
    for (int d = 0; d < 3; d++) {
      double h = 0.5 * c->p.lbox[d];
      if (c->part[i].pos[d] > h || c->part[i].pos[d] < -h) out = 1;
    }
    k += out;
  }
  *count = k;
  return DEM_OK;
}

/* Area of a wall that the spheres can press on: a rectangle's extent along
 * each in-plane axis (the box axis it runs along) up to the box length there,
 * or a cone's lateral area. */
static double o_wall_area(const dem_wall* W, const double* L) {
  if (W->shape == DEM_WALL_RECTANGLE) {
    int ku = 0, kw = 0;
    for (int j = 1; j < 3; j++) {
      if (fabs(W->u[j]) > fabs(W->u[ku])) ku = j;
      if (fabs(W->w[j]) > fabs(W->w[kw])) kw = j;
    }
    double a = 2.0 * W->l1 < L[ku] ? 2.0 * W->l1 : L[ku];
    double b = 2.0 * W->l2 < L[kw] ? 2.0 * W->l2 : L[kw];
    return a * b;
  }
  if (W->shape == DEM_WALL_CONE) {
    double len = 2.0 * W->l1, dr = W->l3 - W->l2;
    return 3.14159265358979323846 * (W->l2 + W->l3) * sqrt(len * len + dr * dr);
  }
  return 0.0;
}

/* KineticEnergy / PotentialEnergy (src/MDEM.f90:183-213) + extras: solid
 * fraction (of the bed's lower 0.8*H, H = twice the mean centre height above
 * the lowest rectangle wall facing z, for a system with gravity along -z and
 * no periodicity in z; else of the box), contacts of the last force pass,
 * wall forces and pressures */
int orc_get_observables(orc_ctx* c, dem_observables* o) {
  memset(o, 0, sizeof(*o));
  const double pi = 3.14159265358979323846;
  double Ek = 0.0, Ep = 0.0;
  for (int32_t i = 0; i < c->n; i++) {
    const OParticle* q = &c->part[i];
    double m = 1.0 / o_inv_mass(c, q);
    double I = 1.0 / o_inv_inertia(c, q);
    if (c->p.n_components == 0) {
      m = o_mass_pp(c, q);
      double R = q->radius;
      I = (0.4 * m) * (R * R);
    }
    Ek = Ek + m * sumsq3(q->vel) + I * sumsq3(q->omega);
    Ep = Ep - m * dot3(q->pos, c->p.gravity);
    for (int d = 0; d < 3; d++) o->momentum[d] += m * q->vel[d];
  }
  o->kinetic_energy = 0.5 * Ek;
  o->potential_energy = Ep;
  double solid = 0.0, region = 0.0;
  if (!(c->p.gravity[2] < 0.0) || c->p.pbc[2] || c->n == 0) {
    for (int32_t i = 0; i < c->n; i++) {
      double R = o_radius(c, &c->part[i]);
      solid += 4.0 / 3.0 * pi * R * R * R;
    }
    region = c->n ? c->p.lbox[0] * c->p.lbox[1] * c->p.lbox[2] : 0.0;
  } else {
    double base = -0.5 * c->p.lbox[2];
    int floor = 0;
    for (int w = 0; w < c->p.n_walls; w++) {
      const dem_wall* W = &c->p.walls[w];
      if (W->shape == DEM_WALL_RECTANGLE && fabs(W->n[2]) > 0.99 &&
          (!floor || W->position[2] < base)) {
        base = W->position[2];
        floor = 1;
      }
    }
    double mean = 0.0;
    for (int32_t i = 0; i < c->n; i++) mean += c->part[i].pos[2] - base;
    double h = 2.0 * (mean / c->n);
    double top = 0.8 * h;
    for (int32_t i = 0; i < c->n; i++)
      if (c->part[i].pos[2] - base < top) {
        double R = o_radius(c, &c->part[i]);
        solid += 4.0 / 3.0 * pi * R * R * R;
      }
    region = c->p.lbox[0] * c->p.lbox[1] * top;
    o->bed_height = h;
  }
  o->packing_fraction = region > 0.0 ? solid / region : 0.0;
  int64_t np, nw;
  orc_count_contacts(c, &np, &nw);
  o->n_pair_records = np;
  o->n_pair_contacts = c->last_pairs;
  o->n_wall_contacts = c->last_walls;
  o->mean_coordination = c->n ? 2.0 * (double)c->last_pairs / (double)c->n : 0.0;
  for (int w = 0; w < NWM; w++) o->wall_normal_force[w] = c->wall_fn[w];
  for (int w = 0; w < c->p.n_walls; w++) {
    double a = o_wall_area(&c->p.walls[w], c->p.lbox);
    o->wall_pressure[w] = a > 0.0 ? o->wall_normal_force[w] / a : 0.0;
  }
  return DEM_OK;
}
