/*
 * dem3d_b200.h -- C-ABI of the B200-native DEM step (cell lists -> contact
 * search + tangential history -> spring-dashpot/Coulomb forces -> ABM4).
 *
 * Drop-in boundary for the per-step path of DEM3D (Fortran 90).  Every entry
 * point below names the reference routine it replaces.  Conventions:
 *   - plain C types only (no CUDA or torch types); host pointers everywhere;
 *     the library copies host arrays in and out and never keeps a caller
 *     pointer after a call returns;
 *   - particle indices are 0-based (the reference is 1-based; every ordering
 *     rule of the reference is invariant under that shift);
 *   - vectors of n particles are laid out as n rows of 3 doubles (x,y,z),
 *     i.e. the contiguous copy of Particle(1:n)%Position(1:3);
 *   - every call returns an int status: DEM_OK (0) or a negative DEM_ERR_*;
 *     dem_last_error() gives a one-line description.  Nothing calls exit().
 *   - one host thread per context; calls are synchronous on return.
 *   - all quantities are in the reference's reduced units (after
 *     ScaleVariables, src/DEM.f90:807-866).
 */
#ifndef DEM3D_B200_H
#define DEM3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_MAX_COMPONENTS 16
#define DEM_MAX_WALLS 8

/* status codes */
#define DEM_OK 0
#define DEM_ERR_INVALID (-1)      /* bad argument / inconsistent parameters */
#define DEM_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define DEM_ERR_CAPACITY (-3)     /* a device buffer could not be grown */
#define DEM_ERR_UNSUPPORTED (-5)  /* valid for the reference, not supported here */
#define DEM_ERR_STATE (-6)        /* call out of order (e.g. no state set) */
#define DEM_ERR_NO_DEVICE (-7)    /* no CUDA device / extension not usable */

/* wall shapes (src/MConfig.f90:44-45) */
#define DEM_WALL_RECTANGLE 1
#define DEM_WALL_CONE 2

/* precision modes */
#define DEM_PREC_FP64 0   /* plain FP64: bit-exact with the oracle */
#define DEM_PREC_MIXED 1  /* FP32 contact arithmetic, FP64 positions/ABM */

/* TWall, src/MDimension3D.f90:45-59 (L1..L3 already halved as in
 * ReadSpecifications, src/DEM.f90:477-479; n = u x w). */
typedef struct dem_wall {
  int32_t shape;
  int32_t order;
  double l1, l2, l3;
  double u[3], w[3], n[3];
  double position[3], velocity[3], omega[3];
} dem_wall;

/*
 * Scaled run parameters.  Two ways to give material properties:
 *  - n_components >= 1: the reference's component tables (MForces module
 *    variables src/MForces.f90:13-24 after InitializeForce :54-87), indexed
 *    [ci*DEM_MAX_COMPONENTS + cj] and [ci*DEM_MAX_WALLS + w];
 *  - n_components == 0: per-particle radius (continuous polydispersity, an
 *    extension: the reference only has discrete components).  Each particle
 *    is its own component of one material; pair tables are formed on the fly
 *    with the reference's own combination rules (src/DEM.f90:259-327):
 *      m = mass_coef*R^3, I = 0.4*m*R^2, Meff = mi*mj/(mi+mj),
 *      Yn = gamma_n*sqrt(Meff*kn), Yt = gamma_t*sqrt(Meff*kt),
 *      MinDij = Ri+Rj; walls use Meff = mi.
 */
typedef struct dem_params {
  int32_t n_components;    /* NC (0 = per-particle radius mode) */
  int32_t n_walls;         /* NW <= DEM_MAX_WALLS */
  int32_t pbc[3];          /* PBC(1:3) */
  int32_t method_order;    /* MethodOrder, 1..4 */
  int32_t euler_intervals; /* NumberOfEulerIntervals */
  int32_t max_ncell;       /* MaxNCell (30000 in src/MForces.f90:28) */
  int32_t precision;       /* DEM_PREC_* */
  int32_t hist_capacity;   /* initial pair records per particle (0 = 16) */
  double lbox[3];          /* Lbox */
  double gravity[3];       /* Gravity */
  double time_step;        /* TimeStep */
  /* component tables (n_components >= 1) */
  double comp_radius[DEM_MAX_COMPONENTS];
  double comp_inv_mass[DEM_MAX_COMPONENTS];
  double comp_inv_inertia[DEM_MAX_COMPONENTS];
  double comp_eff_mass[DEM_MAX_COMPONENTS];
  double min_dij[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double min_dij_sq[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double kn[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double yn[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double kt[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double yt[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double mu_sq[DEM_MAX_COMPONENTS * DEM_MAX_COMPONENTS];
  double knw[DEM_MAX_COMPONENTS * DEM_MAX_WALLS];
  double ynw[DEM_MAX_COMPONENTS * DEM_MAX_WALLS];
  double ktw[DEM_MAX_COMPONENTS * DEM_MAX_WALLS];
  double ytw[DEM_MAX_COMPONENTS * DEM_MAX_WALLS];
  double muw_sq[DEM_MAX_COMPONENTS * DEM_MAX_WALLS];
  /* per-particle mode (n_components == 0) */
  double pp_mass_coef;      /* 4/3*pi*density */
  double pp_density;        /* for EffectiveMass = m*(rho - rho_f)/rho */
  double pp_fluid_density;
  double pp_rmax;           /* largest radius (cell CutOff = 2*rmax) */
  double pp_kn, pp_kt, pp_gamma_n, pp_gamma_t, pp_mu_sq;
  double pp_knw[DEM_MAX_WALLS], pp_ktw[DEM_MAX_WALLS];
  double pp_gamma_nw[DEM_MAX_WALLS], pp_gamma_tw[DEM_MAX_WALLS];
  double pp_muw_sq[DEM_MAX_WALLS];
  dem_wall walls[DEM_MAX_WALLS];
} dem_params;

/* Observables (K5).  kinetic/potential: src/MDEM.f90:183-213; the others
 * have no counterpart in the reference and are defined here.  Ensembles: sums
 * over all systems, fractions as ratios of sums. */
typedef struct dem_observables {
  double kinetic_energy;
  double potential_energy;
  double mean_coordination;   /* 2*(pair contacts of the last force pass)/N */
  /* Solid fraction.  A system with gravity along -z and no periodicity in z
   * holds a bed: its base is the lowest rectangle wall facing z (else the
   * box bottom), its filled height H is twice the mean height of the sphere
   * centres above the base, and the fraction is the volume of the spheres
   * whose centres lie in the lower 0.8*H, over Lx*Ly*0.8*H.  Otherwise: the
   * volume of all spheres over the box volume. */
  double packing_fraction;
  double wall_normal_force[DEM_MAX_WALLS]; /* sum of |FN| on each wall, last force pass */
  double momentum[3];
  int64_t n_pair_contacts;    /* overlapping pairs in the last force pass */
  int64_t n_wall_contacts;    /* overlapping sphere-wall pairs in the last force pass */
  /* wall_normal_force over the wall's area: a rectangle's extent along each
   * of its in-plane axes up to the box length along that axis, a cone's
   * lateral area */
  double wall_pressure[DEM_MAX_WALLS];
  double bed_height;          /* H above (mean over the systems with a bed; 0: none) */
  int64_t n_pair_records;     /* pair history records held (the contacts of the
                                 last updating pass and the records it kept) */
} dem_observables;

/* TWallMovement (src/MDEM.f90:39-45) of one wall, in reduced units (as
 * after ScaleVariables, src/DEM.f90:841-847): position = constant_factor +
 * amplitude*cos(phase), velocity = velocity_amplitude*sin(phase), phase =
 * two_pi_frequency*Time + phase_angle (per component). */
typedef struct dem_wall_motion {
  double constant_factor[3];
  double amplitude[3];
  double velocity_amplitude[3];
  double two_pi_frequency[3];
  double phase_angle[3];
} dem_wall_motion;

/* Pouring (PouringAttempt/PourParticle, src/DEM.f90:115-123,
 * src/MDEM.f90:412-532): every `interval` steps one sphere of a component
 * still below its target count is dropped at a random point of the pouring
 * surface just under the top of the box, if it overlaps nothing there. */
#define DEM_POUR_RECTANGLE 1 /* Rect (src/MDEM.f90:34) */
#define DEM_POUR_CIRCLE 2    /* Circle */
typedef struct dem_pouring {
  int32_t interval;     /* IPouring = max(1, nint(PouringInterval/TimeStep)) */
  int32_t shape;        /* PouringShape */
  int32_t max_attempts; /* MaxAttempts */
  int32_t target_number[DEM_MAX_COMPONENTS]; /* TargetNumber(1:NC) */
  double size[2];       /* PouringSize (simulation units): sides, or diameter */
  double velocity_z;    /* velocity of a new sphere: -1e-4*LengthScale/TimeScale */
} dem_pouring;

/* State of ranf (src/MUtil.f90:10-11): Dummy (the seed, negative to start),
 * the Marsaglia and Park-Miller words iix, iiy, iik and the scale aam. */
typedef struct dem_rng {
  double aam;
  int32_t dummy, iix, iiy, iik;
} dem_rng;

/* Fluid drag (mFluid, src/mFluid.f90): a one-dimensional upward flow through
 * the bed, its velocity and porosity averaged over NL+1 horizontal levels
 * (UpdateVelocityField, :96-139), drives a drag force on every sphere
 * (DragForce, :143-197).  Simulation units (after ScaleFluidProperties). */
typedef struct dem_fluid {
  double viscosity;                        /* FluidViscosity */
  double flow_rate;                        /* FluidFlowRate */
  double density;                          /* FluidDensity */
  double comp_density[DEM_MAX_COMPONENTS]; /* Component(:)%Density */
  int32_t levels;                          /* NL */
  int32_t pad_;
} dem_fluid;

typedef struct dem_ctx dem_ctx;

/* Library build/version string (also proves the .so loads). */
const char* dem_version(void);
/* Select the CUDA device for contexts created afterwards by this thread
 * (the library carries its own CUDA runtime). */
int dem_select_device(int32_t device);

/* Parameters + cell grid set-up.  Replaces InitializeAuxiliaries
 * (src/MDEM.f90:110-162: ABM coefficients, InitializeCellList
 * src/MForces.f90:91-106, InitializeForce :54-87). */
int dem_create(const dem_params* params, dem_ctx** out);
/* An ensemble of n_systems independent systems in one context (no
 * counterpart in the reference, which runs one system per process): every
 * system has its own box, walls, cell grid and material parameters; the
 * integrator (method_order, euler_intervals, time_step) and the precision are
 * shared.  Every stage of a step runs as one launch over all systems.
 * Particles are concatenated by system (sizes from dem_set_system_counts,
 * called before dem_set_state); particle and cell numbers are global, so a
 * system's particle i is global index offset_s + i.  dem_get_grid returns
 * system 0's grid; contacts, Ncol and observables cover all systems. */
int dem_create_ensemble(const dem_params* params, int32_t n_systems, dem_ctx** out);
int dem_set_system_counts(dem_ctx* ctx, const int32_t* counts);
/* FinalizeDEM, src/MDEM.f90:166-179. */
void dem_destroy(dem_ctx* ctx);
const char* dem_last_error(const dem_ctx* ctx);

/* Particle state (Particle(1:n), src/MConfig.f90:68 / TParticle
 * src/MDimension3D.f90:28-35).  comp: component index per particle (0-based,
 * table mode) or NULL; radius: per-particle radius (per-particle mode) or
 * NULL.  acc/alpha may be NULL (zero).  Resets the ABM ring to zeros with
 * ipc = 1..NPrev (InitializeIntegrationVariables, src/MDEM.f90:93-106), the
 * contact lists to empty (InitializeContacts, src/MContacts.f90:43-49) and
 * Ncol to 0. */
int dem_set_state(dem_ctx* ctx, int32_t n, const int32_t* comp,
                  const double* radius, const double* pos, const double* vel,
                  const double* omega, const double* acc, const double* alpha);
int dem_get_state(dem_ctx* ctx, double* pos, double* vel, double* omega,
                  double* acc, double* alpha);
/* Overwrite Particle(1:n) (same n, any array may be NULL = keep) without
 * touching the ABM ring, the contact lists or the cell lists: what a driver
 * that keeps Particle in host memory calls before each step. */
int dem_update_state(dem_ctx* ctx, const double* pos, const double* vel,
                     const double* omega, const double* acc, const double* alpha);
/* Predicted(1:n) of MDEM (src/MDEM.f90:20). */
int dem_get_predicted(dem_ctx* ctx, double* pos, double* vel, double* omega,
                      double* acc, double* alpha);
int dem_get_n(dem_ctx* ctx, int32_t* n);

/* ABM ring Previous(NPrev,n) + ipc(NPrev) (src/MDEM.f90:19-22), as
 * previous[(k*n + i)*9 + {v0..2,a0..2,alpha0..2}] with k the PHYSICAL slot
 * 0..NPrev-1 and ipc 1-based as in the reference.  Same record order as
 * Save/ReadIntegrationVariables (src/MDEM.f90:52-89). */
int dem_set_integration(dem_ctx* ctx, const double* previous, const int32_t* ipc);
int dem_get_integration(dem_ctx* ctx, double* previous, int32_t* ipc);

/* Contact history (MainParticle lists, src/MContacts.f90:21-33).  Pair
 * records (imin < imax) and wall records (particle, wall), Vector1 = ft
 * (previous tangential force), Vector2 = vt (previous tangential contact
 * velocity).  get_* returns them sorted by key like the reference's lists
 * (SaveContactList, src/MContacts.f90:75-117).  imax may exceed n - 1: a
 * record that particle removal left behind, as in the reference. */
int dem_set_contacts(dem_ctx* ctx, int64_t m, const int32_t* imin,
                     const int32_t* imax, const double* ft, const double* vt,
                     int64_t mw, const int32_t* ip, const int32_t* iw,
                     const double* ftw, const double* vtw);
int dem_count_contacts(dem_ctx* ctx, int64_t* n_pair, int64_t* n_wall);
int dem_get_contacts(dem_ctx* ctx, int64_t cap, int32_t* imin, int32_t* imax,
                     double* ft, double* vt, int64_t capw, int32_t* ip,
                     int32_t* iw, double* ftw, double* vtw);

/* InitializeCellDistribution (src/MForces.f90:110-117 ->
 * DistributeParticles3D src/MCells.f90:542-564). */
int dem_initialize_cell_distribution(dem_ctx* ctx);
/* Cell grid: Nx,Ny,Nz (InitCellStructure3D src/MCells.f90:155-227). */
int dem_get_grid(dem_ctx* ctx, int32_t* nxyz);
/* Cells of the context: Nx*Ny*Nz, summed over the systems of an ensemble. */
int dem_get_cell_count(dem_ctx* ctx, int32_t* ncell);
/* CellIndex(1:n) (0-based cells) and the particles of every cell in list
 * order (the traversal order of ComputeAccelerations): traversal[n],
 * cell_start[ncell+1], ncell from dem_get_cell_count. */
int dem_get_cells(dem_ctx* ctx, int32_t* cell_index, int32_t* traversal,
                  int32_t* cell_start);
/* ReadCellDistribution (src/MForces.f90:121-131, ReadCellStructure
 * src/MCells.f90:988-1026): CellIndex from the positions and the cell lists
 * as saved (the layout dem_get_cells returns), instead of a fresh
 * distribution.  Every particle must appear once, in the cell its position
 * hashes to (DEM_ERR_INVALID otherwise). */
int dem_set_cells(dem_ctx* ctx, const int32_t* traversal, const int32_t* cell_start);

/* ComputeAccelerations(Particle or Predicted, NP, TimeStep, Update)
 * (src/MForces.f90:145-335), including RedistributeParticles3D. */
int dem_compute_accelerations(dem_ctx* ctx, int32_t use_predicted,
                              double time_step, int32_t update);
/* The same pass, also returning its Force(NP,3) and Torque(NP,3) arrays
 * (src/MForces.f90:154, summed at :319-320 before the division by mass and
 * inertia at :330-333; gravity and fluid drag included) as rows of three:
 * force[3*i + k], torque[3*i + k] for i < n.  Mixed precision returns its
 * FP32 sums widened. */
int dem_compute_forces(dem_ctx* ctx, int32_t use_predicted, double time_step,
                       int32_t update, double* force, double* torque);
/* MoveParticles(step) (src/MDEM.f90:285-369): force pass @x(t) with history
 * update, AB predictor, ring store, force pass @prediction, AM corrector. */
int dem_move_particles(dem_ctx* ctx, int32_t step);
/* MoveParticlesEuler (src/MDEM.f90:258-281). */
int dem_move_particles_euler(dem_ctx* ctx);
/* The time loop of src/DEM.f90:85-99 without pouring/reporting: if
 * first_step == 1 the MethodOrder-1 Euler start-up steps run first, then
 * MoveParticles(step) for step = max(first_step,MethodOrder) .. last_step.
 * Steps are replayed from CUDA graphs. */
int dem_run(dem_ctx* ctx, int32_t first_step, int32_t last_step);
/* dem_run bracketed by CUDA events on the context's stream; device_ms is the
 * elapsed device time (host synchronisation gaps between replays included). */
int dem_run_timed(dem_ctx* ctx, int32_t first_step, int32_t last_step, double* device_ms);

/* WallsInMovement = YES with WM(1:NW) (src/DEM.f90:714-733): after every
 * Euler sub-step and after every predictor the library evaluates MoveWalls
 * (src/MDEM.f90:392-408) on the host (so positions match a CPU build bit for
 * bit) and moves every wall.  motion: NW records, or NULL to stop moving
 * them.  Contexts with one system only. */
int dem_set_wall_motion(dem_ctx* ctx, const dem_wall_motion* motion);
/* Wall(1:NW) as the last pass saw them (system 0). */
int dem_get_walls(dem_ctx* ctx, dem_wall* walls);

/* UpdateParticleList (src/MDEM.f90:612-671): every particle outside
 * [-L/2, L/2] is removed, highest index first; the last particle takes its
 * place (Particle, Previous, cell lists, contact records renamed as
 * RemoveParticleFromContactList/ChangeIndexInContactList do,
 * src/MContacts.f90:173-252, 579-633).  removed: how many left.  The
 * particle count shrinks (dem_get_n); dem_get_components gives the new
 * Particle%Index order.  Contexts with one system only. */
int dem_update_particle_list(dem_ctx* ctx, int64_t* removed);
/* Whether dem_run calls UpdateParticleList after every step, as the
 * reference's main loop does (src/DEM.f90:94-98).  On by default for
 * single-system contexts; off means escapes are only counted. */
int dem_set_particle_removal(dem_ctx* ctx, int32_t enable);
/* Particle%Index - 1 of every particle (changes when particles are removed). */
int dem_get_components(dem_ctx* ctx, int32_t* comp);
/* Removals so far: {particles removed, swaps with the last particle,
 * contact records renamed or handed over}. */
int dem_get_removal_stats(dem_ctx* ctx, int64_t* stats);

/* Pouring for dem_run (NULL: off).  Single-system contexts with a component
 * table.  The per-particle arrays grow to hold every component's target. */
int dem_set_pouring(dem_ctx* ctx, const dem_pouring* pouring);
/* PourParticle once (inserted: 1 if a sphere went in, else 0). */
int dem_pour_particle(dem_ctx* ctx, int32_t* inserted);
/* The generator state, as SaveState/ReadState keep it (src/DEM.f90:995-999). */
int dem_set_rng(dem_ctx* ctx, const dem_rng* rng);
int dem_get_rng(dem_ctx* ctx, dem_rng* rng);

/* FluidFlow with its settings (NULL: off).  Single-system contexts with a
 * component table; InitializeFluid (src/mFluid.f90:72-92) is done here. */
int dem_set_fluid(dem_ctx* ctx, const dem_fluid* fluid);

/* Ncol (src/MForces.f90:47,227). */
int dem_get_ncol(dem_ctx* ctx, int64_t* ncol);
/* Ncol read back from a state file (ReadState, src/DEM.f90:1109). */
int dem_set_ncol(dem_ctx* ctx, int64_t ncol);
/* Particles that left the box (UpdateParticleList test src/MDEM.f90:624-625)
 * after the last corrector; removal itself is not done by this library. */
int dem_get_escaped(dem_ctx* ctx, int64_t* count);
int dem_get_observables(dem_ctx* ctx, dem_observables* out);

/* Instrumentation: per-kernel CUDA-event timing on the context's stream and
 * a count of kernels launched since the last reset. */
int dem_set_profiling(dem_ctx* ctx, int32_t enable);
int dem_get_kernel_stats(dem_ctx* ctx, int32_t idx, char* name, int32_t name_cap,
                         int64_t* launches, double* total_ms);
int dem_reset_kernel_stats(dem_ctx* ctx);
int dem_get_launch_count(dem_ctx* ctx, int64_t* launches);
/* CUDA-event timer on the context's stream: start, then stop -> ms. */
int dem_timer_start(dem_ctx* ctx);
int dem_timer_stop(dem_ctx* ctx, double* ms);
/* cudaStream_t of the context, as an opaque pointer (for event timing). */
int dem_get_stream(dem_ctx* ctx, void** stream);
/* Mean pair contacts per particle of the last force pass and the device
 * bytes the last pass touched by design (for roofline accounting). */
int dem_get_pass_stats(dem_ctx* ctx, int64_t* pair_contacts, int64_t* wall_contacts,
                       int64_t* movers, int32_t* hist_capacity);
/* Candidate rows of the last pass: total entries over all particles and the
 * row capacity (for byte accounting). */
int dem_get_row_stats(dem_ctx* ctx, int64_t* candidates, int32_t* row_capacity);

/* Tuning (no counterpart in the reference).  skin_factor: candidate-row skin
 * as a fraction of CutOff (0.05 by default; larger = longer rows, fewer full
 * row rebuilds); pass_variant: the contact kernel's block budget, compiled
 * for 4 (0, default), 3 (1) or 5 (2) resident blocks of 128 threads per SM
 * (fewer registers per thread, more warps to hide memory latency).  Neither
 * changes any result: the rows stay complete and in sweep order, and the
 * arithmetic is the same code. */
int dem_set_tuning(dem_ctx* ctx, double skin_factor, int32_t pass_variant);
int dem_get_tuning(dem_ctx* ctx, double* skin_factor, int32_t* pass_variant);
/* Launch shape (no counterpart in the reference; changes no result: the
 * same bodies run over the same particles and contacts, and every sum keeps
 * its order).
 *  - launch_mode: how dem_run issues its 4-step chunks.  0 (default): a
 *    CUDA graph of the chunk's kernels (relink, test, pair, fold per force
 *    pass: 8 launches per step).  1: one persistent cooperative launch per
 *    chunk, as many blocks of 128 threads as fit on the GPU at once, which
 *    step through the 8 passes' phases with grid-wide barriers between them
 *    (every wait bounded: see dem_set_persistent_barrier).  Chunks with
 *    moving walls, fluid drag or kernel profiling run as graphs.
 *  - test_block: threads per block of the test kernel (64, 128 or 256).
 *  - particles_per_thread: particles each thread of the test and fold
 *    kernels takes in turn (1, 2 or 4): the grid holds 1/particles_per_thread
 *    of the blocks and strides over them.
 *  - pair_waves: the pair kernel's grid, in waves of the blocks an SM holds
 *    (1, 2 or 4; contacts per thread = contacts / grid threads). */
int dem_set_launch_shape(dem_ctx* ctx, int32_t launch_mode, int32_t test_block,
                         int32_t particles_per_thread, int32_t pair_waves);
int dem_get_launch_shape(dem_ctx* ctx, int32_t* launch_mode, int32_t* test_block,
                         int32_t* particles_per_thread, int32_t* pair_waves);
/* Early launch (no counterpart in the reference; changes no result): with
 * on != 0 (the default) the test, pair and fold kernels of a force pass are
 * launched with programmatic stream serialization, so that each is
 * scheduled while the kernel ahead of it finishes and starts its work the
 * moment that kernel's writes are visible.  *on (get) may be NULL. */
int dem_set_early_launch(dem_ctx* ctx, int32_t on);
int dem_get_early_launch(dem_ctx* ctx, int32_t* on);
/* Grid-wide barriers of persistent chunks: every wait gives up after
 * timeout_ms (default 2000), after which the chunk ends early, dem_run
 * returns DEM_ERR_STATE and the state must be set again.  extra_blocks > 0
 * is for tests only: every barrier then waits for that many blocks more
 * than were launched, so the first wait runs out.  *blocks (may be NULL):
 * blocks of the last persistent launch. */
int dem_set_persistent_barrier(dem_ctx* ctx, double timeout_ms, int32_t extra_blocks);
int dem_get_persistent_blocks(dem_ctx* ctx, int32_t* blocks);

/* Autotuner: advances the run from first_step through DEM_AUTOTUNE_TRIALS
 * trials, each one untimed 4-step chunk and steps_per_trial timed steps
 * (rounded up to whole 4-step chunks), one knob at a time from the default
 * launch shape: trials 0-8 the skin (0.025 / 0.05 / 0.1) x the three pair
 * variants; from the best of those, 9-10 particles_per_thread 2 and 4,
 * 11-12 test_block 64 and 256, 13-14 pair_waves 1 and 4, 15 launch_mode 1
 * (trial time -1 where a chunk could not run persistent).  Each stage keeps
 * a value only if it beat the best time so far.  Returns the last step
 * advanced and the trial times (trial_ms may be NULL).  The trajectory is
 * the one dem_run would produce. */
#define DEM_AUTOTUNE_TRIALS 16
int dem_autotune(dem_ctx* ctx, int32_t first_step, int32_t steps_per_trial,
                 int32_t* last_step, double* trial_ms);

/* Storage in cell order (no counterpart in the reference; changes no
 * result).  With every_steps > 0, dem_run permutes the particles' arrays
 * into the cells' list order before its first step and then every
 * every_steps steps (state, Predicted, ABM ring, pass copies, history
 * tables, cell lists, with every stored particle number renamed), so that
 * the gathers of neighbouring spheres read neighbouring memory again after
 * the spheres have moved.  The reference's numbering is kept alongside for
 * the one rule of the step that depends on it (a cell's arrivals enter its
 * list in decreasing index) and is restored before any call that reads or
 * writes particle data or renumbers particles (states, contacts, cells,
 * forces, removal, pouring).  0 (default): never.  *reorders: permutations
 * done so far. */
int dem_set_reorder(dem_ctx* ctx, int32_t every_steps);
int dem_get_reorder(dem_ctx* ctx, int32_t* every_steps, int64_t* reorders);

/* Spatial decomposition of one system into z-slabs (no counterpart in the
 * reference; its thesis names spatial decomposition as the way to run it in
 * parallel).  Each slab is a context holding every particle's arrays (the
 * system's own particle numbers) that advances only the particles in its
 * cell layers [z0, z1); it is set up from the whole state like any context
 * (dem_set_state, dem_set_integration, dem_set_contacts, dem_set_ncol,
 * dem_initialize_cell_distribution), then dem_slab_set_range.  A
 * MoveParticles step is, for pass 0 (history update + AB predictor) and
 * pass 1 (AM corrector), on every slab in turn:
 *   - dem_slab_displacement: the largest displacement of the pass before,
 *     read from every slab, their maximum written back to every slab;
 *   - phase DEM_SLAB_RELINK; then from the slab above each slab
 *     DEM_SLAB_GHOSTS (its bottom layer's lists, pass copies, cells and
 *     history rows) and from the slab below DEM_SLAB_LOWER (its top layer's
 *     cells);
 *   - phase DEM_SLAB_TEST_PAIR; then to the slab above DEM_SLAB_JHALVES (the
 *     results for its particles computed here, and its records matched);
 *   - phase DEM_SLAB_FOLD; then DEM_SLAB_MIGRATE_UP / _DOWN to the slabs
 *     above / below (the particles that entered their layers, with their
 *     state, ABM ring and history);
 *   - phase DEM_SLAB_FINISH.
 * Every exchange is a device buffer written by dem_slab_pack on the sending
 * slab (*bytes: its size; DEM_ERR_CAPACITY with *bytes set when cap is too
 * small) and read by dem_slab_unpack on the receiving one; between them it
 * travels by any device copy (cudaMemcpy on one GPU, a send/receive between
 * GPUs).  The particles each slab advances at the end are dem_slab_owned's;
 * their states equal the undivided system's bit for bit.  Slabs hold at
 * least two layers; a pass whose tables overflow is an error. */
#define DEM_SLAB_RELINK 0
#define DEM_SLAB_TEST_PAIR 1
#define DEM_SLAB_FOLD 2
#define DEM_SLAB_FINISH 3
#define DEM_SLAB_GHOSTS 0
#define DEM_SLAB_LOWER 1
#define DEM_SLAB_JHALVES 2
#define DEM_SLAB_MIGRATE_UP 3
#define DEM_SLAB_MIGRATE_DOWN 4
int dem_slab_set_range(dem_ctx* ctx, int32_t z0, int32_t z1);
int dem_slab_phase(dem_ctx* ctx, int32_t step, int32_t pass, int32_t phase);
int dem_slab_pack(dem_ctx* ctx, int32_t what, void* buf, int64_t cap, int64_t* bytes);
int dem_slab_unpack(dem_ctx* ctx, int32_t what, const void* buf, int64_t bytes);
int dem_slab_displacement(dem_ctx* ctx, uint32_t* bits_out, const uint32_t* bits_in);
int dem_slab_owned(dem_ctx* ctx, int32_t* owned);

/* Allocation-free cell distribution.  No counterpart in the reference: it
 * serves callers that may not allocate device memory while they run: a host
 * application whose device memory is all handed out by its own pool or
 * framework (a cudaMalloc behind its back breaks its budget and fragments
 * its pool), or a service that forbids allocation after start-up (cudaMalloc
 * and cudaFree synchronise the device and can take milliseconds).  It
 * computes what
 * dem_initialize_cell_distribution computes (the cell of every particle and
 * the particles of every cell in list order) for one particle set, without a
 * context and without calling cudaMalloc/cudaFree or any allocating library:
 * its working memory is one static device array of about 14 MB that every
 * GPU which loads the library keeps until the process exits.
 *  - d_pos: device array of n rows (x,y,z); d_cell_index[n], d_traversal[n]
 *    and d_cell_start[ncell+1] are device outputs (ncell from
 *    dem_get_grid's formula, also returned in *ncell_out if not NULL);
 *  - limits: n <= DEM_NOALLOC_MAX_PARTICLES and
 *    ncell <= DEM_NOALLOC_MAX_CELLS, else DEM_ERR_CAPACITY (with a message
 *    in err, if given); the other checks of dem_create apply;
 *  - stream: a cudaStream_t (NULL = the default stream); the call waits for
 *    its own work before returning;
 *  - every call looks up the array's device address on the current device
 *    (cudaGetSymbolAddress, a host-side query); the first call on a device
 *    also loads the library's device code there, so on each device make
 *    that first call before any stream capture;
 *  - all calls share the one array: calls that overlap on the GPU (other
 *    threads, other streams) race and must be serialised by the caller. */
#define DEM_NOALLOC_MAX_PARTICLES 262144
#define DEM_NOALLOC_MAX_CELLS 262144
int dem_distribute_particles_noalloc(const dem_params* params, int32_t n, const double* d_pos,
                                     int32_t* d_cell_index, int32_t* d_traversal,
                                     int32_t* d_cell_start, int32_t* ncell_out, void* stream,
                                     char* err, int32_t err_cap);

#ifdef __cplusplus
}
#endif

#endif /* DEM3D_B200_H */
