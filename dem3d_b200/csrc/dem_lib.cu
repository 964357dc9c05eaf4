// dem_lib.cu -- C-ABI of the B200 DEM step (include/dem3d_b200.h).
//
// Host orchestration of the device kernels in dem_kernels.cuh: context and
// device memory, the two force passes of MoveParticles, the Euler start-up,
// CUDA-graph replay of whole steps, contact-history import/export and the
// instrumentation used by the benchmark.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dem_kernels.cuh"
#include "dem_mixed.cuh"
#include "dem_remove.cuh"
#include "dem_fluid.cuh"
#include "dem_slab.cuh"

using namespace dem;

#define DEM_VERSION_STR "dem3d_b200 0.1 (sm_100a)"

namespace {

struct KernelStat {
  std::string name;
  long long launches = 0;
  double total_ms = 0.0;
};

struct PendingEvent {
  int stat;
  cudaEvent_t e0, e1;
};

}  // namespace

struct dem_ctx {
  dem_params params{};  // of system 0 (shared integrator settings)
  DevParams hp{};       // system 0
  DevParams* dp = nullptr;  // device table, one entry per system
  int nsys = 1;
  std::vector<DevParams> hsys;        // host copies of the table
  std::vector<dem_params> sys_params; // the parameters each system was created with
  std::vector<int> counts;            // particles per system (ensembles)
  int ncell_total = 0;
  int* cellsys = nullptr;  // [ncell_total] system of every cell (ensembles only)
  int* sysid = nullptr;    // [n] system of every particle (ensembles only)
  int n = 0;
  int ncap = 0;       // rows allocated for every per-particle array (>= n)
  int ncap_hint = 0;  // capacity the next dem_set_state allocates at least
  int nprev = 0;
  bool state_set = false;
  bool cells_ready = false;
  bool pp = false;  // per-particle radius mode
  int precision = DEM_PREC_FP64;
  cudaStream_t stream = nullptr;
  int device = 0;

  StateArrays P{}, Pr{};
  double* state_block = nullptr;  // all 30 state arrays
  double* ring = nullptr;
  double* radius = nullptr;
  int* comp = nullptr;

  // initial distribution (counting sort) buffers
  SortedArrays S{};
  int* cell_start = nullptr;
  int* cell_cnt = nullptr;
  int *a_cell = nullptr, *a_loc = nullptr, *a_orig = nullptr, *t_orig = nullptr;
  unsigned *a_key = nullptr, *t_key = nullptr;
  int* scan_bsum = nullptr;
  int n_tiles = 0;

  // linked cell lists, candidate rows and the per-pass copies of the two
  // sides (0 = Particle, 1 = Predicted): positions + radius, velocities
  // (double4/double2 in FP64 mode, float4/float2 in mixed mode)
  CellLists L{};
  Rows rows{};
  int kc = 32;
  double4* X[2] = {nullptr, nullptr};
  void* v4[2] = {nullptr, nullptr};
  void* w2[2] = {nullptr, nullptr};
  // moving walls (WallsInMovement): MoveWalls is evaluated on the host; in a
  // captured chunk the walls of step k come from pinned slot k, which the
  // host fills before every replay
  std::vector<dem_wall_motion> wm;
  dem_wall* wall_slots = nullptr;  // pinned, [5][NWM]: 4 chunk slots + staging
  bool capturing = false;
  bool walls_moved = false;  // MoveWalls has run at least once (at `time`)
  // UpdateParticleList after every step of dem_run (single-system contexts);
  // captured chunks then stop before a step that follows escapes
  bool removal = true;
  bool stop_on_escape = false;
  // pouring (PouringAttempt before every step of dem_run) and ranf's state
  bool pouring = false;
  dem_pouring pour{};
  dem_rng rng{0.0, 0, -1, -1, 0};
  std::vector<int> comp_count;  // Component(:)%Number
  // fluid drag (FluidFlow): level tables Vf/Ef and the drag of every sphere
  bool fluid = false;
  FluidArgs fa{};
  double* fl_vf = nullptr;  // [2*(NL+1)]: Vf then Ef
  double* drag = nullptr;   // [3*ncap]
  int drag_cap = 0;
  double* amsum = nullptr;  // [9*ncap] corrector ring sums (predictor -> corrector)
  int amsum_cap = 0;
  // test -> pair -> fold kernels of a pass: the contact list (cl_cap
  // contacts, their "i" results IRec64/IRec32), each particle's place in
  // it, the "j" results per particle (count, in_cap records of
  // InRec64/InRec32 laid out for pass_cap rows) and the matched record bits
  int2* clist = nullptr;
  void* irec = nullptr;
  int cl_cap = 0;
  int* cstart = nullptr;
  int* ccount = nullptr;
  unsigned* matched = nullptr;
  int* in_cnt = nullptr;
  void* in_rec = nullptr;
  double* wall_part = nullptr;  // [contact-kernel blocks][NWM] wall normal forces
  int nw_max = 0;               // walls of the system with the most
  int in_cap = 4;
  int pass_cap = 0;
  double2* pour_cand = nullptr;  // candidate points of one PourParticle call
  int* pour_fits = nullptr;
  int pour_cap = 0;
  int* rm_buf = nullptr;  // escaped list + status words of the removal kernel
  int rm_cap = 0;
  long long rm_stats[3] = {0, 0, 0};  // removals, swaps, records renamed or moved
  int pass_variant = 0;  // pair kernel compiled for 4 (0), 3 (1) or 5 (2) blocks per SM
  // launch shape (dem_set_launch_shape): threads per block of the test
  // kernel, particles per thread of the test and fold kernels, the pair
  // kernel's grid in waves of resident blocks, and 4-step chunks as one
  // persistent launch (1) or replayed graphs (0)
  int test_block = 128;
  int ppt = 1;
  int pair_waves = 2;
  int launch_mode = 0;
  // the test, pair and fold kernels of a pass launched with programmatic
  // stream serialization (dem_set_early_launch), so that each is scheduled
  // while the kernel ahead of it finishes
  int early_launch = 1;
  // persistent chunks: while `recording`, the pass launchers append the
  // passes of a chunk to rec (relink arguments wait in rec_rl for their
  // pass) instead of launching; each rotation phase keeps its chunk's
  // passes in device memory (prog[phase], prog_n passes)
  bool recording = false;
  RelinkArgs rec_rl{};
  std::vector<unsigned char> rec;
  int rec_n = 0;
  void* prog[20] = {};
  int prog_n[20] = {};
  bool prog_valid = false;
  unsigned* bar = nullptr;  // grid barrier: arrival count, generation
  unsigned long long bar_limit_ns = 2000000000ull;
  int bar_extra = 0;        // blocks a test adds to every barrier (0: none)
  int chunk_blocks = 0;     // blocks of the last persistent launch
  // one slab of a spatial decomposition (dem_slab_set_range): the context
  // holds every particle's arrays but advances only the particles of its
  // cell layers; gstamp[p] == gepoch marks the ghosts it received this pass
  bool slab = false;
  int* gstamp = nullptr;
  int gepoch = 0;
  int slab_z0 = 0, slab_z1 = 0;
  int* slab_list = nullptr;   // particles of a layer / migrants (scratch, [ncap])
  int* slab_ghosts = nullptr; // the ghosts received this pass
  int n_ghosts = 0;
  int* slab_count = nullptr;  // device counters of the list kernels
  RingMap slab_rm{};          // the ring map of the pass in progress
  // storage in cell order (dem_set_reorder): every reorder_every steps of
  // dem_run the particle arrays are permuted into the cells' list order;
  // gid[s] is the reference's index of the particle stored at s (L.gid);
  // calls that read or write particle data restore the reference's order
  int reorder_every = 0;
  long long since_reorder = 0;
  long long reorders = 0;
  bool permuted = false;
  // the passes' predictors left Particle a, alpha in the ring slot ipc(1)
  // and Predicted x (v, w: FP64) in the Predicted side's pass copies
  // (PassArgs::lazy); settle_state writes them back
  bool lazy_state = false;
  int* gid = nullptr;
  int gid_cap = 0;
  bool has_cone = false; // some wall of some system is a cone
  double skin_factor = 0.05;  // candidate-row skin / CutOff
  int par = 0;         // L.cell[par] is the assignment the lists hold
  int prepared = -1;   // side whose copies + next assignment are ready (-1: none)
  int last_side = -1;  // side of the last pass (its copies are intact)

  History H[2]{};
  int hcur = 0;  // H[hcur] holds the current records
  int hcap = 16;

  MixedBuffers M{};

  Counters* cnt = nullptr;
  Counters* hcnt = nullptr;  // pinned host mirror
  double* obs_partial = nullptr;

  double* staging = nullptr;  // 15*n doubles, rows layout for host I/O
  double* force_out = nullptr;  // set during dem_compute_forces: Force, Torque rows
  cudaEvent_t timer[2] = {nullptr, nullptr};

  int ringmap[5] = {0, 1, 2, 3, 4};
  double time = 0.0;

  // graphs: one per (phase of the ring/history rotation)
  cudaGraphExec_t graph[20] = {};
  int graph_steps = 0;
  long long graph_kernels = 0;  // kernels in one captured chunk
  bool graph_valid = false;

  bool prof = false;
  std::vector<KernelStat> stats;
  std::vector<PendingEvent> pending;
  std::vector<cudaEvent_t> event_pool;
  long long launches = 0;
  long long last_pairs = 0, last_walls = 0, last_movers = 0;

  std::string err;
};

namespace {

int fail(dem_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(dem_ctx* c, cudaError_t e, const char* where) {
  std::string m = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  return fail(c, DEM_ERR_CUDA, m);
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);    \
  } while (0)

// settle: write back what the predictors left out (settle_state) first
int restore_order(dem_ctx* c, bool settle = true);
int settle_state(dem_ctx* c);

// calls that read or write particle data see the reference's order
#define RESTORE_ORDER                \
  do {                               \
    int st_ = restore_order(c);      \
    if (st_) return st_;             \
  } while (0)

int stat_index(dem_ctx* c, const char* name) {
  for (size_t i = 0; i < c->stats.size(); i++)
    if (c->stats[i].name == name) return (int)i;
  c->stats.push_back(KernelStat{name});
  return (int)c->stats.size() - 1;
}

cudaEvent_t get_event(dem_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// launch with optional event timing
template <typename... KArgs, typename... Args>
void launch(dem_ctx* c, const char* name, void (*kernel)(KArgs...), unsigned grid, unsigned block,
            Args... args) {
  if (grid == 0) return;
  if (c->prof) {
    PendingEvent pe;
    pe.stat = stat_index(c, name);
    pe.e0 = get_event(c);
    pe.e1 = get_event(c);
    cudaEventRecord(pe.e0, c->stream);
    kernel<<<grid, block, 0, c->stream>>>(args...);
    cudaEventRecord(pe.e1, c->stream);
    c->pending.push_back(pe);
  } else {
    kernel<<<grid, block, 0, c->stream>>>(args...);
  }
  c->launches++;
}

// launch of a test, pair or fold kernel: early (programmatic stream
// serialization) when the context allows it and no kernel is being timed
// on its own
template <typename... KArgs, typename... Args>
void launch_early(dem_ctx* c, bool early, const char* name, void (*kernel)(KArgs...),
                  unsigned grid, unsigned block, Args... args) {
  if (grid == 0) return;
  if (c->prof || !early) {
    launch(c, name, kernel, grid, block, args...);
    return;
  }
  launch_pass(true, kernel, grid, block, c->stream, args...);
  c->launches++;
}

// launch with dynamic shared memory (opt-in raised once per kernel)
template <typename... KArgs, typename... Args>
void launch_sm(dem_ctx* c, const char* name, void (*kernel)(KArgs...), unsigned grid,
               unsigned block, int smem, Args... args) {
  if (grid == 0) return;
  static thread_local std::vector<const void*> raised;
  if (std::find(raised.begin(), raised.end(), (const void*)kernel) == raised.end()) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    raised.push_back((const void*)kernel);
  }
  if (c->prof) {
    PendingEvent pe;
    pe.stat = stat_index(c, name);
    pe.e0 = get_event(c);
    pe.e1 = get_event(c);
    cudaEventRecord(pe.e0, c->stream);
    kernel<<<grid, block, smem, c->stream>>>(args...);
    cudaEventRecord(pe.e1, c->stream);
    c->pending.push_back(pe);
  } else {
    kernel<<<grid, block, smem, c->stream>>>(args...);
  }
  c->launches++;
}

// run fn (which launches exactly one kernel on the context stream) with the
// same event timing as launch()
template <class Fn>
void timed(dem_ctx* c, const char* name, Fn&& fn) {
  if (c->prof) {
    PendingEvent pe;
    pe.stat = stat_index(c, name);
    pe.e0 = get_event(c);
    pe.e1 = get_event(c);
    cudaEventRecord(pe.e0, c->stream);
    fn();
    cudaEventRecord(pe.e1, c->stream);
    c->pending.push_back(pe);
  } else {
    fn();
  }
  c->launches++;
}

void resolve_events(dem_ctx* c) {
  if (c->pending.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto& pe : c->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pe.e0, pe.e1);
    c->stats[pe.stat].launches++;
    c->stats[pe.stat].total_ms += ms;
    c->event_pool.push_back(pe.e0);
    c->event_pool.push_back(pe.e1);
  }
  c->pending.clear();
}

unsigned blocks_for(long long n, int b) { return (unsigned)((n + b - 1) / b); }

void free_lists(dem_ctx* c) {
  CellLists& L = c->L;
  int** f[] = {&L.head,  &L.next,  &L.cell[0], &L.cell[1], &L.arr_head, &L.arr_next, &L.mflag,
               &L.mnext, &L.dflag, &L.rflag,   &L.dlist[0], &L.dlist[1],  &L.rlist,
               &L.slot,  &L.slot_n, &L.mlist, &L.dstamp};
  for (int** q : f) {
    cudaFree(*q);
    *q = nullptr;
  }
  cudaFree(c->rows.cand);
  cudaFree(c->rows.meta);
  cudaFree(c->rows.rank);
  c->rows = Rows{};
  cudaFree(c->in_cnt);
  cudaFree(c->in_rec);
  cudaFree(c->wall_part);
  cudaFree(c->clist);
  cudaFree(c->irec);
  cudaFree(c->cstart);
  cudaFree(c->ccount);
  cudaFree(c->matched);
  c->in_cnt = nullptr;
  c->in_rec = nullptr;
  c->wall_part = nullptr;
  c->clist = nullptr;
  c->irec = nullptr;
  c->cstart = nullptr;
  c->ccount = nullptr;
  c->matched = nullptr;
  c->cl_cap = 0;
  c->pass_cap = 0;
  for (int b = 0; b < 2; b++) {
    cudaFree(c->X[b]);
    cudaFree(c->v4[b]);
    cudaFree(c->w2[b]);
    c->X[b] = nullptr;
    c->v4[b] = c->w2[b] = nullptr;
  }
}

void free_state(dem_ctx* c) {
  cudaFree(c->sysid);
  c->sysid = nullptr;
  cudaFree(c->gid);
  c->gid = nullptr;
  c->gid_cap = 0;
  c->L.gid = nullptr;
  c->permuted = false;
  c->lazy_state = false;
  cudaFree(c->staging);
  c->staging = nullptr;
  cudaFree(c->state_block);
  cudaFree(c->ring);
  cudaFree(c->radius);
  cudaFree(c->comp);
  cudaFree(c->S.orig);
  cudaFree(c->S.cell);
  cudaFree(c->a_cell);
  cudaFree(c->a_loc);
  cudaFree(c->a_orig);
  cudaFree(c->t_orig);
  cudaFree(c->a_key);
  cudaFree(c->t_key);
  free_lists(c);
  for (int b = 0; b < 2; b++) {
    cudaFree(c->H[b].cnt);
    cudaFree(c->H[b].key);
    cudaFree(c->H[b].val);
    cudaFree(c->H[b].wflag);
    cudaFree(c->H[b].wval);
    c->H[b] = History{};
  }
  mixed_free(c->M);
  c->state_block = c->ring = c->radius = nullptr;
  c->comp = nullptr;
  c->S = SortedArrays{};
  c->a_cell = c->a_loc = c->a_orig = c->t_orig = nullptr;
  c->a_key = c->t_key = nullptr;
}

void drop_graphs(dem_ctx* c) {
  for (auto& g : c->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  c->graph_valid = false;
  // the recorded chunks hold the same pointers and rotation phases
  for (int k = 0; k < 20; k++) {
    if (c->prog[k]) cudaFree(c->prog[k]);
    c->prog[k] = nullptr;
    c->prog_n[k] = 0;
  }
  c->prog_valid = false;
}

// tables laid out for the allocated capacity (record r of particle i at
// r*ncap + i), so the particle count can change without moving records
int alloc_history(dem_ctx* c, History& H, int cap) {
  size_t n = (size_t)std::max(c->ncap, 1);
  int nw = std::max(c->params.n_walls, 1);
  H.cap = cap;
  H.n = (int)n;
  CK(cudaMalloc(&H.cnt, n * sizeof(int)));
  CK(cudaMalloc(&H.key, n * cap * sizeof(int)));
  CK(cudaMalloc(&H.val, n * cap * 3 * sizeof(double2)));
  CK(cudaMalloc(&H.wflag, n * nw * sizeof(int)));
  CK(cudaMalloc(&H.wval, n * nw * 3 * sizeof(double2)));
  CK(cudaMemsetAsync(H.cnt, 0, n * sizeof(int), c->stream));
  CK(cudaMemsetAsync(H.key, 0xFF, n * cap * sizeof(int), c->stream));
  CK(cudaMemsetAsync(H.wflag, 0, n * nw * sizeof(int), c->stream));
  return DEM_OK;
}

// grow both history tables, keeping the current records
int grow_history(dem_ctx* c, int need) {
  int cap = c->hcap;
  while (cap < need) cap *= 2;
  History nh[2];
  for (int b = 0; b < 2; b++) {
    int st = alloc_history(c, nh[b], cap);
    if (st) return st;
  }
  History& cur = c->H[c->hcur];
  launch(c, "hist_regrow", k_hist_regrow, blocks_for(c->n, 256), 256, c->n, cur, nh[c->hcur]);
  // wall records are particle major (i*nw + w): the first n rows move as they are
  size_t n = (size_t)std::max(std::min(c->n, cur.n), 1);
  int nw = std::max(c->params.n_walls, 1);
  CK(cudaMemcpyAsync(nh[c->hcur].wflag, cur.wflag, n * nw * sizeof(int), cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(nh[c->hcur].wval, cur.wval, n * nw * 3 * sizeof(double2),
                     cudaMemcpyDeviceToDevice, c->stream));
  if (c->precision == DEM_PREC_MIXED &&
      !mixed_regrow(c->M, c->n, c->ncap, cap, c->hcur, cur, c->stream))
    return fail(c, DEM_ERR_CAPACITY, "mixed history regrow failed");
  CK(cudaStreamSynchronize(c->stream));
  for (int b = 0; b < 2; b++) {
    cudaFree(c->H[b].cnt);
    cudaFree(c->H[b].key);
    cudaFree(c->H[b].val);
    cudaFree(c->H[b].wflag);
    cudaFree(c->H[b].wval);
    c->H[b] = nh[b];
  }
  c->hcap = cap;
  drop_graphs(c);
  return DEM_OK;
}

StateArrays make_state(double* base, size_t n);
int ensure_drag(dem_ctx* c);

// Room for `newcap` particles in every per-particle array (the values of the
// current n particles are kept; the per-pass copies, the candidate rows and
// the prepared cell transition are rebuilt by the next pass).
int grow_capacity(dem_ctx* c, int newcap) {
  if (newcap <= c->ncap) return DEM_OK;
  {
    int st = settle_state(c);  // (the ring and the copies are not kept)
    if (st) return st;
  }
  CK(cudaStreamSynchronize(c->stream));
  drop_graphs(c);
  // (called in the reference's order: gid is the identity and is made again
  // for the new capacity at the next reorder)
  cudaFree(c->gid);
  c->gid = nullptr;
  c->gid_cap = 0;
  c->L.gid = nullptr;
  const size_t n = (size_t)c->n, N = (size_t)newcap;
  auto fresh = [&](auto*& p, size_t elems, size_t keep) -> cudaError_t {
    using T = std::remove_reference_t<decltype(*p)>;
    T* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(elems, 1));
    if (e != cudaSuccess) return e;
    if (keep) e = cudaMemcpyAsync(q, p, sizeof(T) * keep, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(p);
    p = q;
    return e;
  };
  // Particle keeps its values; Predicted is rebuilt by every step
  double* sb = nullptr;
  CK(cudaMalloc(&sb, sizeof(double) * 30 * N));
  CK(cudaMemsetAsync(sb, 0, sizeof(double) * 30 * N, c->stream));
  StateArrays nP = make_state(sb, N);
  double* const from[15] = {c->P.px, c->P.py, c->P.pz, c->P.vx, c->P.vy, c->P.vz, c->P.wx, c->P.wy,
                            c->P.wz, c->P.ax, c->P.ay, c->P.az, c->P.lx, c->P.ly, c->P.lz};
  double* const to[15] = {nP.px, nP.py, nP.pz, nP.vx, nP.vy, nP.vz, nP.wx, nP.wy,
                          nP.wz, nP.ax, nP.ay, nP.az, nP.lx, nP.ly, nP.lz};
  for (int k = 0; k < 15 && n; k++)
    CK(cudaMemcpyAsync(to[k], from[k], sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->state_block);
  c->state_block = sb;
  c->P = nP;
  c->Pr = make_state(sb + 15 * N, N);
  const size_t slots9 = 9 * (size_t)(c->nprev + 1);
  CK(fresh(c->staging, 15 * N, 0));
  CK(fresh(c->ring, slots9 * N, slots9 * n));  // laid out for n: the first slots9*n
  CK(fresh(c->radius, N, n));
  CK(fresh(c->comp, N, n));
  CK(fresh(c->S.orig, N, 0));
  CK(fresh(c->S.cell, N, 0));
  CK(fresh(c->a_cell, N, 0));
  CK(fresh(c->a_loc, N, 0));
  CK(fresh(c->a_orig, N, 0));
  CK(fresh(c->t_orig, N, 0));
  CK(fresh(c->a_key, N, 0));
  CK(fresh(c->t_key, N, 0));
  CellLists& L = c->L;
  CK(fresh(L.next, N, n));
  CK(fresh(L.cell[0], N, n));
  CK(fresh(L.cell[1], N, n));
  CK(fresh(L.arr_next, N, n));
  CK(fresh(L.mflag, N, n));
  CK(fresh(L.mnext, N, n));
  CK(fresh(c->rows.cand, N * (size_t)c->rows.kc, 0));
  CK(fresh(c->rows.meta, N, 0));
  CK(cudaMemsetAsync(c->rows.meta, 0, sizeof(int) * N, c->stream));
  CK(fresh(c->rows.rank, N, 0));
  CK(cudaMemsetAsync(c->rows.rank, 0, sizeof(int) * N, c->stream));
  if (N > n) CK(cudaMemsetAsync(L.mflag + n, 0, sizeof(int) * (N - n), c->stream));
  for (int b = 0; b < 2; b++) {
    CK(fresh(c->X[b], N, 0));
    if (c->precision == DEM_PREC_MIXED) {
      float4* v = (float4*)c->v4[b];
      float2* w = (float2*)c->w2[b];
      CK(fresh(v, N, 0));
      CK(fresh(w, N, 0));
      c->v4[b] = v;
      c->w2[b] = w;
    } else {
      double4* v = (double4*)c->v4[b];
      double2* w = (double2*)c->w2[b];
      CK(fresh(v, N, 0));
      CK(fresh(w, N, 0));
      c->v4[b] = v;
      c->w2[b] = w;
    }
  }
  // history tables laid out for the new capacity
  c->ncap = (int)N;
  int st = grow_history(c, c->hcap);
  if (st) return st;
  if (c->precision == DEM_PREC_MIXED && !mixed_grow_walls(c->M, c->n, c->ncap, c->hcur, c->stream))
    return fail(c, DEM_ERR_CUDA, "mixed wall records");
  const int one = 1;
  CK(cudaMemcpyAsync(&c->cnt->force_full, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  c->prepared = -1;
  c->last_side = -1;
  CK(cudaStreamSynchronize(c->stream));
  return ensure_drag(c);
}

StateArrays make_state(double* base, size_t n) {
  StateArrays s;
  double** f[15] = {&s.px, &s.py, &s.pz, &s.vx, &s.vy, &s.vz, &s.wx, &s.wy,
                    &s.wz, &s.ax, &s.ay, &s.az, &s.lx, &s.ly, &s.lz};
  for (int k = 0; k < 15; k++) *f[k] = base + (size_t)k * n;
  return s;
}

// ---------------------------------------------------------------------------
// K1: initial distribution (DistributeParticles3D) of the Particle positions

constexpr int LIST_BLOCKS = 148;      // relink / repair kernels (grid-stride)

// the slots of every cell from its list (after the lists were built or
// changed outside the relink: initial distribution, imported lists, removal,
// insertion)
void refresh_slots(dem_ctx* c) {
  launch(c, "cell_slots", k_cell_slots, blocks_for(c->ncell_total, 256), 256, c->L, 0,
         c->ncell_total, c->n);
}

int init_cells(dem_ctx* c) {
  const int n = c->n;
  const int ncell = c->ncell_total;
  CellLists& L = c->L;
  CK(cudaMemsetAsync(L.head, 0xFF, sizeof(int) * (size_t)ncell, c->stream));
  CK(cudaMemsetAsync(L.arr_head, 0xFF, sizeof(int) * (size_t)ncell, c->stream));
  CK(cudaMemsetAsync(L.dflag, 0, sizeof(int) * (size_t)ncell, c->stream));
  CK(cudaMemsetAsync(L.rflag, 0, sizeof(int) * (size_t)ncell, c->stream));
  CK(cudaMemsetAsync(L.dstamp, 0, sizeof(int) * (size_t)ncell, c->stream));
  if (n > 0) CK(cudaMemsetAsync(L.mflag, 0, sizeof(int) * (size_t)n, c->stream));
  CK(cudaMemsetAsync(c->cell_cnt, 0, sizeof(int) * (size_t)ncell, c->stream));
  if (n > 0) {
    launch(c, "cell_assign", k_assign, blocks_for(n, 256), 256, (const DevParams*)c->dp,
           (const int*)c->sysid, n, 1, (const double*)c->P.px, (const double*)c->P.py, (const double*)c->P.pz,
           (const int*)c->S.orig, (const int*)c->S.cell, c->cell_cnt, c->a_cell, c->a_loc,
           c->a_key, c->a_orig, c->cnt);
    launch(c, "scan_tiles", k_scan_tiles, (unsigned)c->n_tiles, SCAN_THREADS,
           (const int*)c->cell_cnt, ncell, c->cell_start, c->scan_bsum, (const Counters*)c->cnt);
    launch(c, "scan_bsums", k_scan_bsums, 1u, SCAN_THREADS, c->scan_bsum, c->n_tiles,
           c->cell_start, ncell, (const Counters*)c->cnt);
    launch(c, "scan_add", k_scan_add, blocks_for(ncell, 256), 256, c->cell_start, ncell,
           (const int*)c->scan_bsum, (const Counters*)c->cnt);
    launch(c, "cell_scatter", k_scatter, blocks_for(n, 256), 256, n, (const int*)c->a_cell,
           (const int*)c->a_loc, (const unsigned*)c->a_key, (const int*)c->a_orig,
           (const int*)c->cell_start, c->t_key, c->t_orig, (const Counters*)c->cnt);
    launch(c, "cell_sort", k_cellsort, blocks_for(ncell, 128), 128, ncell,
           (const int*)c->cell_start, c->t_key, c->t_orig, c->S.orig, c->S.cell, L.cell[c->par],
           (const Counters*)c->cnt);
    launch(c, "link_init", k_link_init, blocks_for(n, 256), 256, n, (const int*)c->S.orig,
           (const int*)c->S.cell, (const int*)c->cell_start, L.head, L.next, L.cell[c->par]);
  }
  refresh_slots(c);
  // no transition pending; the first pass builds every candidate row
  CK(cudaMemsetAsync(&c->cnt->n_dirty[0], 0, 3 * sizeof(int), c->stream));
  CK(cudaMemsetAsync(&c->cnt->movers_pending, 0, sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(&c->cnt->disp_max, 0, sizeof(unsigned), c->stream));
  CK(cudaMemsetAsync(&c->cnt->disp_acc, 0, sizeof(double), c->stream));
  const int one = 1;
  CK(cudaMemcpyAsync(&c->cnt->force_full, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  c->prepared = -1;
  c->last_side = -1;
  return DEM_OK;
}

// ---------------------------------------------------------------------------
// one pass: copies of the side (if not prepared), relink, candidate rows,
// pass kernel

// The predictors leave out Particle a, alpha and Predicted x (v, w with FP64
// copies) where other arrays hold them (PassArgs::lazy): not with fluid drag
// (its kernels read Predicted z and v) nor in a slab of a decomposition
// (ghost and result exchanges).
bool lazy_now(const dem_ctx* c) { return !c->fluid && !c->slab; }

template <class V4, class W2>
PassArgs<V4, W2> pass_args(dem_ctx* c, int side, bool update, double dt, const RingMap& rm,
                           int tag, const StateArrays& tgt) {
  PassArgs<V4, W2> A;
  A.P = c->dp;
  A.sysid = c->sysid;
  A.n = c->n;
  A.X = c->X[side];
  A.v4 = (const V4*)c->v4[side];
  A.w2 = (const W2*)c->w2[side];
  A.comp = c->comp;
  A.cand = c->rows.cand;
  A.meta = c->rows.meta;
  A.cell_cur = c->L.cell[c->par];
  A.L = c->L;
  A.par_nxt = c->par ^ 1;
  A.Hr = c->H[c->hcur];
  A.Hw = c->H[c->hcur ^ 1];
  A.update = update ? 1 : 0;
  A.half_dt = 0.5 * dt;
  A.tgt = tgt;
  A.part = c->P;
  A.pred = c->Pr;
  A.Xn = c->X[side ^ 1];
  A.v4n = (V4*)c->v4[side ^ 1];
  A.w2n = (W2*)c->w2[side ^ 1];
  A.ring = c->ring;
  A.rm = rm;
  A.cnt = c->cnt;
  A.tag = tag;
  A.drag = c->fluid ? c->drag : nullptr;
  A.lazy = lazy_now(c) ? 1 : 0;
  A.amsum = c->amsum;
  A.rank = c->rows.rank;
  A.clist = c->clist;
  A.cstart = c->cstart;
  A.ccount = c->ccount;
  A.irec = c->irec;
  A.cl_cap = c->cl_cap;
  A.in_cnt = c->in_cnt;
  A.in_rec = c->in_rec;
  A.in_cap = c->in_cap;
  A.in_stride = c->pass_cap;
  A.matched = c->matched;
  A.wall_part = c->wall_part;
  A.nw_max = c->nw_max;
  A.gstamp = c->slab ? c->gstamp : nullptr;
  A.gepoch = c->gepoch;
  return A;
}

size_t in_rec_bytes(const dem_ctx* c) {
  return c->precision == DEM_PREC_MIXED ? sizeof(InRec32) : sizeof(InRec64);
}

// the "j" records of a pass laid out for in_cap records of pass_cap rows
int alloc_incoming(dem_ctx* c, int cap) {
  cudaFree(c->in_rec);
  c->in_rec = nullptr;
  CK(cudaMalloc(&c->in_rec, in_rec_bytes(c) * (size_t)cap * (size_t)c->pass_cap));
  c->in_cap = cap;
  return DEM_OK;
}

// the contact list of a pass and the "i" results of its contacts
int alloc_contacts(dem_ctx* c, int cap) {
  cudaFree(c->clist);
  cudaFree(c->irec);
  c->clist = nullptr;
  c->irec = nullptr;
  const size_t rb = c->precision == DEM_PREC_MIXED ? sizeof(IRec32) : sizeof(IRec64);
  CK(cudaMalloc(&c->clist, sizeof(int2) * (size_t)std::max(cap, 1)));
  CK(cudaMalloc(&c->irec, rb * (size_t)std::max(cap, 1)));
  c->cl_cap = cap;
  return DEM_OK;
}

// a longer contact list (it only lives within a pass)
int grow_contacts(dem_ctx* c, int need) {
  long long cap = std::max(c->cl_cap, 1024);
  while (cap < need) cap = cap * 3 / 2;
  if (cap > (1ll << 30)) return fail(c, DEM_ERR_CAPACITY, "contact list beyond 2^30 contacts");
  if (cap == c->cl_cap) return DEM_OK;
  CK(cudaStreamSynchronize(c->stream));
  int st = alloc_contacts(c, (int)cap);
  if (st) return st;
  drop_graphs(c);
  return DEM_OK;
}

// more "j" records per particle (the records only live within a pass)
int grow_incoming(dem_ctx* c, int need) {
  int cap = std::max(c->in_cap, 1);
  while (cap < need) cap *= 2;
  if (cap == c->in_cap) return DEM_OK;
  CK(cudaStreamSynchronize(c->stream));
  int st = alloc_incoming(c, cap);
  if (st) return st;
  drop_graphs(c);
  return DEM_OK;
}

// room for the two-kernel handover of a pass (counts start at zero)
int ensure_pass_buffers(dem_ctx* c) {
  const int N = std::max(c->ncap, 1);
  if (c->pass_cap >= N) return DEM_OK;
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->in_cnt);
  cudaFree(c->wall_part);
  cudaFree(c->cstart);
  cudaFree(c->ccount);
  cudaFree(c->matched);
  c->in_cnt = nullptr;
  c->wall_part = nullptr;
  c->cstart = c->ccount = nullptr;
  c->matched = nullptr;
  c->pass_cap = N;
  CK(cudaMalloc(&c->in_cnt, sizeof(int) * (size_t)N));
  CK(cudaMemset(c->in_cnt, 0, sizeof(int) * (size_t)N));
  CK(cudaMalloc(&c->matched, sizeof(unsigned) * (size_t)N));
  CK(cudaMemset(c->matched, 0, sizeof(unsigned) * (size_t)N));
  CK(cudaMalloc(&c->cstart, sizeof(int) * (size_t)N));
  CK(cudaMalloc(&c->ccount, sizeof(int) * (size_t)N));
  if (c->cl_cap < 2 * N) {
    int st = alloc_contacts(c, 2 * N);
    if (st) return st;
  }
  const size_t parts = (size_t)blocks_for(N, 128) * NWM;
  CK(cudaMalloc(&c->wall_part, sizeof(double) * parts));
  CK(cudaMemset(c->wall_part, 0, sizeof(double) * parts));
  drop_graphs(c);
  return alloc_incoming(c, c->in_cap);
}

// room for the drag of every sphere and the corrector ring sums (outside
// graph capture)
int ensure_drag(dem_ctx* c) {
  {
    int st = ensure_pass_buffers(c);
    if (st) return st;
  }
  if (c->nprev > 0 && c->amsum_cap < std::max(c->ncap, 1)) {
    cudaFree(c->amsum);
    c->amsum = nullptr;
    c->amsum_cap = 0;
    CK(cudaMalloc(&c->amsum, sizeof(double) * 9 * (size_t)std::max(c->ncap, 1)));
    c->amsum_cap = std::max(c->ncap, 1);
  }
  if (!c->fluid || c->drag_cap >= std::max(c->ncap, 1)) return DEM_OK;
  cudaFree(c->drag);
  c->drag = nullptr;
  c->drag_cap = 0;
  CK(cudaMalloc(&c->drag, sizeof(double) * 3 * (size_t)std::max(c->ncap, 1)));
  c->drag_cap = std::max(c->ncap, 1);
  return DEM_OK;
}

// UpdateVelocityField + DragForce for the state the pass evaluates
void fluid_prepare(dem_ctx* c, int side) {
  if (!c->fluid || c->n == 0) return;
  const StateArrays& Q = side ? c->Pr : c->P;
  const int nl1 = c->fa.levels + 1;
  launch(c, "fluid_levels", k_fluid_levels, (unsigned)nl1, (unsigned)FLUID_THREADS, c->fa, c->n,
         (const double*)Q.pz, (const double*)Q.vz, (const int*)c->comp, c->fl_vf, c->fl_vf + nl1,
         (const Counters*)c->cnt);
  launch(c, "fluid_drag", k_fluid_drag, blocks_for(c->n, 256), 256u, c->fa, c->n, Q,
         (const int*)c->comp, (const double*)c->fl_vf, (const double*)(c->fl_vf + nl1), c->drag,
         (const Counters*)c->cnt);
}

// part: 0 = the whole pass, 1 = the test and pair kernels, 2 = the fold
// kernel (a slab of a decomposition exchanges data in between)
// early_ok: the operation ahead of this pass's test kernel in the stream is
// the pass's relink (or a fluid kernel after it), so the test, pair and fold
// kernels may be launched early; not after the status resets of a repeated
// pass, nor between the exchanges of a slab
void launch_pass_kernel(dem_ctx* c, int side, bool update, double dt, int epi, const RingMap& rm,
                        int tag, int part = 0, bool early_ok = true) {
  if (c->n == 0) return;
  const bool early = early_ok && c->early_launch && !c->slab && part == 0;
  const StateArrays& tgt = side ? c->Pr : c->P;
  // the test kernel: the contact list of the pass
  TestArgs T;
  T.P = c->dp;
  T.sysid = c->sysid;
  T.n = c->n;
  T.cell_cur = c->L.cell[c->par];
  T.L = c->L;
  T.R = c->rows;
  T.X = c->X[side];
  T.comp = c->comp;
  T.cand = c->rows.cand;
  T.meta = c->rows.meta;
  T.clist = c->clist;
  T.cstart = c->cstart;
  T.ccount = c->ccount;
  T.cl_cap = c->cl_cap;
  T.cnt = c->cnt;
  T.tag = tag;
  T.slab_c0 = c->slab ? c->hsys[0].slab_c0 : 0;
  T.slab_span = c->slab ? (unsigned)(c->hsys[0].slab_c1 - c->hsys[0].slab_c0) : 0xffffffffu;
  T.fine = c->slab ? 0 : 1;  // (a slab's stamps of its ghost layer come by exchange)
  const bool walls = c->nw_max > 0;
  if (c->recording) {
    // a pass of a persistent chunk: appended, not launched
    auto add = [&](const auto& cp) {
      const size_t at = c->rec.size();
      c->rec.resize(at + sizeof(cp));
      std::memcpy(c->rec.data() + at, &cp, sizeof(cp));
      c->rec_n++;
    };
    if (c->precision == DEM_PREC_MIXED) {
      ChunkPass<float4, float2, MixedView> cp{};
      cp.rl = c->rec_rl;
      cp.t = T;
      cp.a = pass_args<float4, float2>(c, side, update, dt, rm, tag, tgt);
      cp.v = mixed_view(c->M, c->hcur);
      cp.epi = epi;
      add(cp);
    } else {
      ChunkPass<double4, double2, NoView> cp{};
      cp.rl = c->rec_rl;
      cp.t = T;
      cp.a = pass_args<double4, double2>(c, side, update, dt, rm, tag, tgt);
      cp.epi = epi;
      add(cp);
    }
    return;
  }
  // test kernel: test_block threads per block; with ppt > 1 the grid holds
  // 1/ppt of the blocks and strides over them
  if (part != 2) {
    const int bs = c->test_block;
    const unsigned nvb = blocks_for(c->n, bs);
    const bool stride = c->ppt > 1;
    const unsigned g = stride ? (nvb + c->ppt - 1) / c->ppt : nvb;
#define TK(PPV, BS, S) launch_early(c, early, "test", k_test<PPV, BS, S>, g, BS, T)
#define TCASE(PPV)                    \
  do {                                \
    if (bs == 64) {                   \
      if (stride) TK(PPV, 64, true);  \
      else TK(PPV, 64, false);        \
    } else if (bs == 256) {           \
      if (stride) TK(PPV, 256, true); \
      else TK(PPV, 256, false);       \
    } else {                          \
      if (stride) TK(PPV, 128, true); \
      else TK(PPV, 128, false);       \
    }                                 \
  } while (0)
    if (c->pp) TCASE(true);
    else TCASE(false);
#undef TCASE
#undef TK
  }
  const int mb = c->pass_variant == 1 ? 3 : c->pass_variant == 2 ? 5 : 4;
  // the pair kernel loops over the list: pair_waves waves of the blocks its
  // register budget lets an SM hold (at least mb per SM)
  const unsigned pair_blocks = (unsigned)(148 * c->pair_waves * std::max(mb, 6));
  if (c->precision == DEM_PREC_MIXED) {
    auto A = pass_args<float4, float2>(c, side, update, dt, rm, tag, tgt);
    if (epi == EPI_STORE) A.amsum = c->force_out;
    for (int k = 0; k < 2; k++) {
      if ((k == 0 && part == 2) || (k == 1 && part == 1)) continue;
      timed(c, k ? "fold_mixed" : "pair_mixed", [&]() {
        mixed_pass(c->M, c->pp, epi, c->pass_variant, walls, c->has_cone, A, c->hcur, c->stream,
                   k, pair_blocks, c->ppt, early && !c->prof);
      });  // (timed counts the launch)
    }
    return;
  }
  auto A = pass_args<double4, double2>(c, side, update, dt, rm, tag, tgt);
  if (epi == EPI_STORE) A.amsum = c->force_out;
#define PAIR_CASE(PPV, MB) \
  launch_early(c, early, "pair_fp64", k_pair_fp64<PPV, MB>, pair_blocks, 128, A)
  if (part == 2) {
  } else if (mb == 3) {
    if (c->pp) PAIR_CASE(true, 3);
    else PAIR_CASE(false, 3);
  } else if (mb == 5) {
    if (c->pp) PAIR_CASE(true, 5);
    else PAIR_CASE(false, 5);
  } else {
    if (c->pp) PAIR_CASE(true, 4);
    else PAIR_CASE(false, 4);
  }
#undef PAIR_CASE
  if (part == 1) return;
  // fold kernel: blocks of 128 particles (ppt > 1: grid-stride, not for the
  // Euler start-up's EPI_STORE)
  const unsigned nvb = blocks_for(c->n, 128);
  const bool stride = c->ppt > 1 && epi != EPI_STORE;
  const unsigned g = stride ? (nvb + c->ppt - 1) / c->ppt : nvb;
#define FK(PPV, E, W, S) \
  launch_early(c, early, "fold_fp64", k_fold_fp64<PPV, E, W, S>, g, 128, A)
#define FOLD_CASE(PPV, W)                     \
  do {                                        \
    if (epi == EPI_PREDICT) {                 \
      if (stride) FK(PPV, EPI_PREDICT, W, true); \
      else FK(PPV, EPI_PREDICT, W, false);    \
    } else if (epi == EPI_CORRECT) {          \
      if (stride) FK(PPV, EPI_CORRECT, W, true); \
      else FK(PPV, EPI_CORRECT, W, false);    \
    } else {                                  \
      FK(PPV, EPI_STORE, W, false);           \
    }                                         \
  } while (0)
  if (walls) {
    if (c->pp) FOLD_CASE(true, true);
    else FOLD_CASE(false, true);
  } else {
    if (c->pp) FOLD_CASE(true, false);
    else FOLD_CASE(false, false);
  }
#undef FOLD_CASE
#undef FK
}

// Copies of `side` for the pass kernel and the cell transition towards its
// positions (after forgetting a transition prepared for the other side).
int prepare_side(dem_ctx* c, int side) {
  if (side == 1) {  // Predicted's copies are made from Predicted
    int st = settle_state(c);
    if (st) return st;
  }
  const int nxt = c->par ^ 1;
  launch(c, "discard", k_discard, (unsigned)LIST_BLOCKS, 256, c->L, nxt, (const Counters*)c->cnt);
  CK(cudaMemsetAsync(&c->cnt->n_dirty[nxt], 0, sizeof(int), c->stream));
  if (c->n > 0) {
    const StateArrays& src = side ? c->Pr : c->P;
    const double4* Xlast = c->last_side >= 0 ? c->X[c->last_side] : nullptr;
    if (c->precision == DEM_PREC_MIXED)
      launch(c, "prepare", k_prepare<float4, float2>, blocks_for(c->n, 256), 256,
             (const DevParams*)c->dp, (const int*)c->sysid, c->n, src, (const double*)c->radius, c->X[side],
             (float4*)c->v4[side], (float2*)c->w2[side], Xlast, (const int*)c->L.cell[c->par],
             c->L, nxt, c->cnt);
    else
      launch(c, "prepare", k_prepare<double4, double2>, blocks_for(c->n, 256), 256,
             (const DevParams*)c->dp, (const int*)c->sysid, c->n, src, (const double*)c->radius, c->X[side],
             (double4*)c->v4[side], (double2*)c->w2[side], Xlast, (const int*)c->L.cell[c->par],
             c->L, nxt, c->cnt);
  }
  c->prepared = side;
  return DEM_OK;
}

// relink towards the prepared assignment (the candidate rows around the
// relinked cells are rebuilt by the test kernel)
void pass_lists(dem_ctx* c, int side, bool update, int tag) {
  (void)side;
  const int b = c->par ^ 1;
  const int stop_tag = c->capturing && c->stop_on_escape && update ? tag : -1;
  if (c->recording) {
    c->rec_rl = RelinkArgs{c->dp, c->cellsys, c->L, b, c->n, update ? 1 : 0, stop_tag, c->cnt};
  } else {
    launch(c, "relink", k_relink, (unsigned)LIST_BLOCKS, 256, (const DevParams*)c->dp,
           (const int*)c->cellsys, c->L, b, c->n, update ? 1 : 0, stop_tag, c->cnt);
  }
  c->par = b;
}

RingMap current_map(dem_ctx* c) {
  RingMap rm;
  for (int k = 0; k < 5; k++) rm.phys[k] = c->ringmap[k];
  return rm;
}

// ipc = cshift(ipc,-1) with the spare slot becoming ipc(1)
void rotate_ring(dem_ctx* c) {
  int np = c->nprev;
  if (np <= 0) return;
  int spare = c->ringmap[np];
  int oldest = c->ringmap[np - 1];
  for (int k = np - 1; k > 0; k--) c->ringmap[k] = c->ringmap[k - 1];
  c->ringmap[0] = spare;
  c->ringmap[np] = oldest;
}

// the rotation after a step's predictor pass: its ring slot becomes ipc(1),
// and a lazy predictor (PassArgs::lazy) left a, alpha there
void abm_rotate(dem_ctx* c) {
  rotate_ring(c);
  if (lazy_now(c)) c->lazy_state = true;
}

// Particle a, alpha and Predicted x (v, w: FP64) written back from the
// arrays the lazy predictors left them in; before anything reads or changes
// particle data, grows or renumbers it, or runs an Euler step
int settle_state(dem_ctx* c) {
  if (!c->lazy_state) return DEM_OK;
  if (c->capturing || c->recording)
    return fail(c, DEM_ERR_STATE, "state written back inside a captured chunk");
  const int n = c->n;
  if (n > 0) {
    const int slot0 = c->nprev > 0 ? c->ringmap[0] : 0;
    if (c->precision == DEM_PREC_MIXED)
      launch(c, "settle_state", k_settle_state<false, float4, float2>, blocks_for(n, 256), 256, n,
             c->P, c->Pr, (const double*)c->ring, slot0, c->nprev, (const double4*)c->X[1],
             (const float4*)c->v4[1], (const float2*)c->w2[1]);
    else
      launch(c, "settle_state", k_settle_state<true, double4, double2>, blocks_for(n, 256), 256,
             n, c->P, c->Pr, (const double*)c->ring, slot0, c->nprev, (const double4*)c->X[1],
             (const double4*)c->v4[1], (const double2*)c->w2[1]);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "settle_state");
  }
  c->lazy_state = false;
  return DEM_OK;
}

int read_counters(dem_ctx* c) {
  CK(cudaMemcpyAsync(c->hcnt, c->cnt, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->last_pairs = (long long)c->hcnt->pair_contacts;
  c->last_walls = (long long)c->hcnt->wall_contacts;
  c->last_movers = (long long)c->hcnt->movers;
  return DEM_OK;
}

// forget a stopped pass: status words, its partial counts and its Ncol
int clear_abort(dem_ctx* c) {
  Counters* d = c->cnt;
  CK(cudaMemsetAsync(&d->ncol_pending, 0, sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(&d->pair_contacts, 0, 2 * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(&d->overflow, 0, 4 * sizeof(int), c->stream));
  // row_overflow .. n_contacts
  CK(cudaMemsetAsync(&d->row_overflow, 0, 7 * sizeof(int), c->stream));
  // the stopped pair kernel may have counted "j" records and matched records
  if (c->pass_cap > 0) {
    CK(cudaMemsetAsync(c->in_cnt, 0, sizeof(int) * (size_t)c->pass_cap, c->stream));
    CK(cudaMemsetAsync(c->matched, 0, sizeof(unsigned) * (size_t)c->pass_cap, c->stream));
  }
  return DEM_OK;
}

// longer candidate rows: the rows are rebuilt by the next full rebuild
int grow_rows(dem_ctx* c, int need) {
  if (need > KC_MAX) return fail(c, DEM_ERR_CAPACITY, "candidate rows longer than 1023");
  int kc = std::max(need, c->kc + c->kc / 2);
  kc = std::min((kc + 7) / 8 * 8, KC_MAX);
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->rows.cand);
  c->rows.cand = nullptr;
  CK(cudaMalloc(&c->rows.cand, sizeof(int) * (size_t)std::max(c->n, 1) * kc));
  c->kc = kc;
  c->rows.kc = kc;
  drop_graphs(c);
  return DEM_OK;
}

// A pass whose relink ran and whose rows or pass kernel stopped (capacity):
// grow what overflowed and launch the rest of the pass again.  The pass
// kernel only writes fresh outputs and idempotent transition records, so a
// launch that stopped half way can be repeated.
int finish_pass(dem_ctx* c, int side, bool update, double dt, int epi, const RingMap& rm,
                int tag) {
  for (int attempt = 0;; attempt++) {
    int st = read_counters(c);
    if (st) return st;
    const Counters h = *c->hcnt;
    if (!h.abort) return DEM_OK;
    if (h.nonfinite) return fail(c, DEM_ERR_STATE, "a particle position is not finite");
    if (h.list_error) return fail(c, DEM_ERR_STATE, "cell lists inconsistent (walk bound hit)");
    if (attempt >= 8) return fail(c, DEM_ERR_CAPACITY, "capacity cannot be grown");
    st = clear_abort(c);
    if (st) return st;
    if (h.overflow) {
      st = grow_history(c, std::max(h.need_capacity, c->hcap + 1));
      if (st) return st;
    }
    if (h.in_overflow) {
      st = grow_incoming(c, std::max(h.need_in, c->in_cap + 1));
      if (st) return st;
    }
    if (h.cl_overflow) {
      st = grow_contacts(c, std::max(h.need_cl, c->cl_cap + 1));
      if (st) return st;
    }
    if (h.row_overflow) {
      st = grow_rows(c, h.need_kc);
      if (st) return st;
      const int one = 1;
      CK(cudaMemcpyAsync(&c->cnt->full_due, &one, sizeof(int), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaMemsetAsync(&c->cnt->disp_acc, 0, sizeof(double), c->stream));
    }
    launch_pass_kernel(c, side, update, dt, epi, rm, tag, 0, false);
  }
}

// One force pass (ComputeAccelerations) on `side` (0 = Particle, 1 =
// Predicted) with the integrator epilogue `epi`.  check: recover from a
// capacity overflow here (not possible inside a captured graph).
int force_pass(dem_ctx* c, int side, bool update, double dt, int epi, const RingMap& rm,
               bool check, int tag) {
  if (c->prepared != side) {
    int st = prepare_side(c, side);
    if (st) return st;
  }
  pass_lists(c, side, update, tag);
  fluid_prepare(c, side);
  launch_pass_kernel(c, side, update, dt, epi, rm, tag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "pass kernel launch");
  if (check) {
    int st = finish_pass(c, side, update, dt, epi, rm, tag);
    if (st) return st;
  }
  c->last_side = side;
  c->prepared = epi == EPI_PREDICT ? 1 : epi == EPI_CORRECT ? 0 : -1;
  if (update) c->hcur ^= 1;
  return DEM_OK;
}

// Pair records into the tables of their imin (the current records go to the
// other buffer, which becomes current); the wall records are copied along.
int canonical_history(dem_ctx* c) {
  const int n = c->n;
  if (n == 0) return DEM_OK;
  const bool mixed = c->precision == DEM_PREC_MIXED;
  // two status words past the removal's own (state[0..8+NCM) of k_remove)
  static_assert(8 + NCM + 2 <= RM_STATE_WORDS, "status words");
  int* status = c->rm_buf + RM_STATE_WORDS - 2;
  for (int attempt = 0;; attempt++) {
    const int cur = c->hcur, nxt = cur ^ 1;
    History& S = c->H[cur];
    History& D = c->H[nxt];
    CK(cudaMemsetAsync(status, 0, 2 * sizeof(int), c->stream));
    CK(cudaMemsetAsync(D.cnt, 0, sizeof(int) * (size_t)n, c->stream));
    launch(c, "hist_canon", k_hist_canon, blocks_for(n, 256), 256, n, S, D,
           (const float4*)(mixed ? c->M.ha[cur] : nullptr),
           (const float4*)(mixed ? c->M.hb[cur] : nullptr),
           (const float*)(mixed ? c->M.hc[cur] : nullptr), mixed ? c->M.ha[nxt] : nullptr,
           mixed ? c->M.hb[nxt] : nullptr, mixed ? c->M.hc[nxt] : nullptr, status);
    int hs[2] = {0, 0};
    CK(cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hs[0]) {
      if (attempt >= 4) return fail(c, DEM_ERR_CAPACITY, "history tables cannot be grown");
      int st = grow_history(c, hs[1] + 2);
      if (st) return st;
      continue;
    }
    const size_t w = (size_t)n * (size_t)std::max(c->params.n_walls, 1);
    CK(cudaMemcpyAsync(D.wflag, S.wflag, sizeof(int) * w, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(D.wval, S.wval, sizeof(double2) * 3 * w, cudaMemcpyDeviceToDevice,
                       c->stream));
    if (mixed) {
      CK(cudaMemcpyAsync(c->M.wa[nxt], c->M.wa[cur], sizeof(float4) * w,
                         cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(c->M.wb[nxt], c->M.wb[cur], sizeof(float4) * w,
                         cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(c->M.wc[nxt], c->M.wc[cur], sizeof(float) * w, cudaMemcpyDeviceToDevice,
                         c->stream));
    }
    c->hcur = nxt;
    drop_graphs(c);
    return DEM_OK;
  }
}

// UpdateParticleList (src/MDEM.f90:612-671): the escaped particles are
// listed by one grid-wide kernel, then removed by k_remove (one block, in
// decreasing index).  A removal that would overflow the history tables asks
// for capacity before it changes anything; the tables grow and the kernel
// carries on.  Afterwards the ring is laid out for the new particle count
// (the history tables are laid out for the capacity and stay), and the next
// pass rebuilds every candidate row.
int update_particle_list_impl(dem_ctx* c, int64_t* removed) {
  if (removed) *removed = 0;
  RESTORE_ORDER;
  if (c->nsys > 1) return fail(c, DEM_ERR_UNSUPPORTED, "particle removal needs one system");
  const int n0 = c->n;
  if (n0 == 0) return DEM_OK;
  CK(cudaStreamSynchronize(c->stream));
  if (c->rm_cap < n0) {
    cudaFree(c->rm_buf);
    c->rm_buf = nullptr;
    CK(cudaMalloc(&c->rm_buf, sizeof(int) * ((size_t)n0 + RM_STATE_WORDS)));
    c->rm_cap = n0;
  }
  int* state = c->rm_buf;  // status words, then the list
  int* list = c->rm_buf + RM_STATE_WORDS;
  int hs[RM_STATE_WORDS] = {n0};  // [7]: escaped count
  CK(cudaMemcpyAsync(state, hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream));
  launch(c, "escape_list", k_escape_list, blocks_for(n0, 256), 256, (const DevParams*)c->dp, n0,
         c->P, list, state + 7);
  CK(cudaMemcpyAsync(hs, state, sizeof(hs), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int n_list = hs[7];
  if (n_list > 0) {
    int st = canonical_history(c);
    if (st) return st;
    for (int attempt = 0;; attempt++) {
      RemovalArgs A;
      A.PT = c->dp;
      A.P = c->P;
      A.radius = c->radius;
      A.comp = c->comp;
      A.ring = c->ring;
      A.ring_slots = c->nprev + 1;
      A.ring_stride = n0;
      A.L = c->L;
      A.par = c->par;
      A.H = c->H[c->hcur];
      const bool mixed = c->precision == DEM_PREC_MIXED;
      A.ha = mixed ? c->M.ha[c->hcur] : nullptr;
      A.hb = mixed ? c->M.hb[c->hcur] : nullptr;
      A.hc = mixed ? c->M.hc[c->hcur] : nullptr;
      A.wa = mixed ? c->M.wa[c->hcur] : nullptr;
      A.wb = mixed ? c->M.wb[c->hcur] : nullptr;
      A.wc = mixed ? c->M.wc[c->hcur] : nullptr;
      A.nw = c->params.n_walls;
      A.list = list;
      A.n_list = n_list;
      A.state = state;
      launch(c, "remove", k_remove, 1u, (unsigned)RM_THREADS, A);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(hs, state, sizeof(hs), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (hs[1] == RM_OK) break;
      if (hs[1] == RM_NEED_CAPACITY && attempt < 8) {
        int st = grow_history(c, hs[2] + 2);  // same particle count: same layout
        if (st) return st;
        const int zero = 0;
        CK(cudaMemcpyAsync(state + 1, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        continue;
      }
      if (hs[1] == RM_NB_OVERFLOW)
        return fail(c, DEM_ERR_CAPACITY, "a removed particle's neighbourhood is too crowded");
      return fail(c, DEM_ERR_STATE, "cell lists inconsistent during particle removal");
    }
  }
  const int n1 = hs[0];
  if (!c->pp)
    for (size_t k = 0; k < c->comp_count.size(); k++) c->comp_count[k] -= hs[8 + k];
  c->rm_stats[0] += hs[3];
  c->rm_stats[1] += hs[4];
  c->rm_stats[2] += hs[5];
  if (n1 != n0) {
    // the ring and the history tables laid out for n1 particles
    const int slots9 = 9 * (c->nprev + 1);
    double* nr = nullptr;
    CK(cudaMalloc(&nr, sizeof(double) * (size_t)slots9 * (size_t)std::max(n1, 1)));
    if (n1 > 0)
      launch(c, "ring_restride", k_ring_restride, 592u, 256u, (const double*)c->ring, nr, slots9,
             n0, n1);
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(c->ring);
    c->ring = nr;
    c->n = n1;  // the history tables keep their layout (stride = capacity)
  }
  CK(cudaMemsetAsync(&c->cnt->escaped, 0, sizeof(unsigned long long), c->stream));
  const int one = 1;
  CK(cudaMemcpyAsync(&c->cnt->force_full, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  refresh_slots(c);
  // the cell transition towards the current positions, for the new numbering
  c->last_side = -1;
  int st = prepare_side(c, 0);
  if (st) return st;
  drop_graphs(c);
  if (removed) *removed = n0 - n1;
  CK(cudaGetLastError());
  return read_counters(c);
}

// ranf (src/MUtil.f90:17-48): Marsaglia shift register combined with the
// Park-Miller generator (Schrage's method); aam in single precision, as
// nearest(1.0,-1.0)/IM is computed, then widened.
double ranf_host(dem_rng& r) {
  const int32_t IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836;
  if (r.dummy <= 0 || r.iiy < 0) {
    volatile float one_minus = std::nextafter(1.0f, -1.0f);
    volatile float a = one_minus / (float)IM;
    const int32_t ad = r.dummy < 0 ? -r.dummy : r.dummy;
    r.aam = (double)a;
    r.iiy = (888889999 ^ ad) | 1;
    r.iix = 777755555 ^ ad;
    r.dummy = ad + 1;
  }
  uint32_t x = (uint32_t)r.iix;
  x ^= x << 13;
  x ^= x >> 17;  // ishft(iix,-17) is a logical shift
  x ^= x << 5;
  r.iix = (int32_t)x;
  r.iik = r.iiy / IQ;
  r.iiy = IA * (r.iiy - r.iik * IQ) - IR * r.iik;
  if (r.iiy < 0) r.iiy += IM;
  return r.aam * (double)((IM & (r.iix ^ r.iiy)) | 1);
}

// the point of one pouring attempt (src/MDEM.f90:455-472)
void pour_point(const dem_pouring& P, double Di, dem_rng& r, double& x, double& y) {
  if (P.shape == DEM_POUR_RECTANGLE) {
    x = (P.size[0] - Di) * (ranf_host(r) - 0.5);
    y = (P.size[1] - Di) * (ranf_host(r) - 0.5);
  } else {
    const double TwoPi = 2.0 * 3.1415926535897932384626433832795;
    const double Rad = 0.5 * ranf_host(r) * (P.size[0] - Di);
    const double Angle = TwoPi * ranf_host(r);
    x = Rad * sin(Angle);
    y = Rad * cos(Angle);
  }
}

// rows the per-particle arrays need while pouring: every component up to its
// target (removals only lower the counts)
int pour_capacity(const dem_ctx* c, const std::vector<int>& counts, int n) {
  if (!c->pouring) return n;
  long long tot = 0;
  for (int k = 0; k < c->params.n_components; k++)
    tot += std::max(counts[(size_t)k], c->pour.target_number[k]);
  return (int)std::min<long long>(std::max<long long>(tot, n), (1 << 30) - 1);
}

bool pour_active(const dem_ctx* c) {
  if (!c->pouring) return false;
  for (int k = 0; k < c->params.n_components; k++)
    if (c->comp_count[(size_t)k] < c->pour.target_number[k]) return true;
  return false;
}

// PourParticle (src/MDEM.f90:412-532) with InsertParticle (:536-561).  The
// points of all MaxAttempts attempts are drawn on the host from a copy of the
// generator and tested at once on the device (k_pour_test); the generator
// then advances over the attempts the reference makes (up to the first point
// that fits), and the sphere goes in at index n.
int pour_particle_impl(dem_ctx* c, int32_t* inserted) {
  if (inserted) *inserted = 0;
  RESTORE_ORDER;
  if (!pour_active(c)) return DEM_OK;
  const dem_pouring& Pp = c->pour;
  const int NC = c->params.n_components;
  int not_reached[NCM], nnr = 0;
  for (int k = 0; k < NC; k++)
    if (c->comp_count[(size_t)k] < Pp.target_number[k]) not_reached[nnr++] = k;
  const int j = (int)((double)nnr * ranf_host(c->rng));
  const int comp = not_reached[j];
  int ibig = 0;  // maxloc(Component%Radius)
  for (int k = 1; k < NC; k++)
    if (c->params.comp_radius[k] > c->params.comp_radius[ibig]) ibig = k;
  const double Ri = c->params.comp_radius[ibig], Di = 2.0 * Ri;
  const double z = 0.5 * c->params.lbox[2] - Ri;
  const int na = Pp.max_attempts;
  if (na <= 0) return DEM_OK;
  std::vector<double2> cand((size_t)na);
  dem_rng r = c->rng;
  for (int a = 0; a < na; a++) pour_point(Pp, Di, r, cand[(size_t)a].x, cand[(size_t)a].y);
  if (c->pour_cap < na) {
    cudaFree(c->pour_cand);
    cudaFree(c->pour_fits);
    c->pour_cand = nullptr;
    c->pour_fits = nullptr;
    CK(cudaMalloc(&c->pour_cand, sizeof(double2) * (size_t)na));
    CK(cudaMalloc(&c->pour_fits, sizeof(int) * (size_t)na));
    c->pour_cap = na;
  }
  CK(cudaMemcpyAsync(c->pour_cand, cand.data(), sizeof(double2) * (size_t)na,
                     cudaMemcpyHostToDevice, c->stream));
  PourTest T;
  T.PT = c->dp;
  T.px = c->P.px;
  T.py = c->P.py;
  T.pz = c->P.pz;
  T.comp = c->comp;
  T.L = c->L;
  T.cand = c->pour_cand;
  T.z = z;
  T.Ri = Ri;
  T.ibig = ibig;
  T.n_att = na;
  T.n = c->n;
  T.fits = c->pour_fits;
  launch(c, "pour_test", k_pour_test, (unsigned)((na + 3) / 4), 128u, T);
  std::vector<int> fits((size_t)na);
  CK(cudaMemcpyAsync(fits.data(), c->pour_fits, sizeof(int) * (size_t)na, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int first = -1;
  for (int a = 0; a < na && first < 0; a++)
    if (fits[(size_t)a]) first = a;
  const int used = first >= 0 ? first + 1 : na;
  for (int a = 0; a < used; a++) {
    double x, y;
    pour_point(Pp, Di, c->rng, x, y);
  }
  if (first < 0) return DEM_OK;
  // InsertParticle at index n
  const int n0 = c->n;
  if (n0 + 1 > c->ncap) {
    int st = grow_capacity(c, std::max(c->ncap + 1, (int)(1.05 * (double)c->ncap)));
    if (st) return st;
  }
  const int slots9 = 9 * (c->nprev + 1);
  double* nr = nullptr;
  CK(cudaMalloc(&nr, sizeof(double) * (size_t)slots9 * (size_t)c->ncap));
  launch(c, "ring_widen", k_ring_widen, 592u, 256u, (const double*)c->ring, nr, slots9, n0,
         n0 + 1);
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->ring);
  c->ring = nr;
  InsertArgs A;
  A.PT = c->dp;
  A.P = c->P;
  A.radius = c->radius;
  A.comp = c->comp;
  A.L = c->L;
  A.par = c->par;
  A.H0 = c->H[0];
  A.H1 = c->H[1];
  A.nw = c->params.n_walls;
  A.n = n0;
  A.comp_new = comp;
  A.pos[0] = cand[(size_t)first].x;
  A.pos[1] = cand[(size_t)first].y;
  A.pos[2] = z;
  A.vel_z = Pp.velocity_z;
  A.radius_new = c->params.comp_radius[comp];
  launch(c, "insert", k_insert, 1u, 32u, A);  // (in mixed mode too: the wall flags and
                                              // record counts live in the key tables)
  c->n = n0 + 1;
  refresh_slots(c);
  c->comp_count[(size_t)comp]++;
  const int one = 1;
  CK(cudaMemcpyAsync(&c->cnt->force_full, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  c->prepared = -1;
  c->last_side = -1;
  drop_graphs(c);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  if (inserted) *inserted = 1;
  return DEM_OK;
}

// MoveWalls (src/MDEM.f90:392-408) at Time, into walls[0:NW) of system 0.
void move_walls_host(const dem_ctx* c, double Time, dem_wall* walls) {
  const double Pi = 3.1415926535897932384626433832795;  // src/MUtil.f90
  const double TwoPi = 2.0 * Pi;
  for (size_t j = 0; j < c->wm.size(); j++) {
    const dem_wall_motion& m = c->wm[j];
    for (int k = 0; k < 3; k++) {
      double Phase = m.two_pi_frequency[k] * Time + m.phase_angle[k];
      Phase = Phase - TwoPi * (double)(int)(Phase / TwoPi);
      walls[j].position[k] = m.constant_factor[k] + m.amplitude[k] * cos(Phase);
      walls[j].velocity[k] = m.velocity_amplitude[k] * sin(Phase);
    }
  }
}

// if (WallsInMovement) call MoveWalls(Time): the walls at c->time into the
// device table (from slot k of the chunk while a chunk is being captured).
int apply_walls(dem_ctx* c, int k) {
  if (c->wm.empty()) return DEM_OK;
  const size_t nb = sizeof(dem_wall) * c->wm.size();
  dem_wall* dst = reinterpret_cast<dem_wall*>(reinterpret_cast<char*>(c->dp) +
                                              offsetof(DevParams, walls));  // system 0
  c->walls_moved = true;
  if (c->capturing) {
    CK(cudaMemcpyAsync(dst, c->wall_slots + (size_t)k * NWM, nb, cudaMemcpyHostToDevice,
                       c->stream));
    return DEM_OK;
  }
  dem_wall* w = c->wall_slots + (size_t)4 * NWM;  // staging, not a chunk slot
  CK(cudaStreamSynchronize(c->stream));  // the previous upload has been read
  for (size_t j = 0; j < c->wm.size(); j++) w[j] = c->hsys[0].walls[j];
  move_walls_host(c, c->time, w);
  CK(cudaMemcpyAsync(dst, w, nb, cudaMemcpyHostToDevice, c->stream));
  return DEM_OK;
}

// the host copy of system 0's walls follows the device one (before any
// upload of the parameter table, and for dem_get_walls)
void sync_host_walls(dem_ctx* c) {
  if (c->wm.empty() || !c->walls_moved) return;
  move_walls_host(c, c->time, c->hsys[0].walls);
  c->hp = c->hsys[0];
}

// the walls of the G steps of the chunk that starts at `step` into the slots
void fill_wall_slots(dem_ctx* c, int step, int G) {
  if (c->wm.empty()) return;
  for (int k = 0; k < G; k++) {
    dem_wall* w = c->wall_slots + (size_t)k * NWM;
    for (size_t j = 0; j < c->wm.size(); j++) w[j] = c->hsys[0].walls[j];
    move_walls_host(c, (double)(step + k) * c->params.time_step, w);
  }
}

int validate_ready(dem_ctx* c) {
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no particle state set");
  if (!c->cells_ready)
    return fail(c, DEM_ERR_STATE, "cell distribution not initialised (call "
                                  "dem_initialize_cell_distribution)");
  return DEM_OK;
}

// MoveParticles(step) (src/MDEM.f90:285-369); tags 2k (pass 1), 2k+1 (pass 2)
int move_particles_impl(dem_ctx* c, int step, bool check, int k) {
  RingMap rm = current_map(c);
  // force pass @ x(t) with history update, a(t) -> Particle, AB predictor
  int st = force_pass(c, 0, true, c->params.time_step, EPI_PREDICT, rm, check, 2 * k);
  if (st) return st;
  abm_rotate(c);
  c->time = (double)step * c->params.time_step;
  st = apply_walls(c, k);
  if (st) return st;
  rm = current_map(c);
  // force pass @ prediction, history read only, AM corrector
  return force_pass(c, 1, false, c->params.time_step, EPI_CORRECT, rm, check, 2 * k + 1);
}

// MoveParticlesEuler (src/MDEM.f90:258-281)
int move_particles_euler_impl(dem_ctx* c) {
  int st0 = settle_state(c);  // the ring store reads Particle a, alpha
  if (st0) return st0;
  const int n = c->n;
  const double dt = c->params.time_step / (double)c->params.euler_intervals;
  if (c->nprev > 0) {
    int spare = c->ringmap[c->nprev];
    launch(c, "ring_store", k_ring_store, blocks_for(n, 256), 256, n, c->P, c->ring, spare,
           (const Counters*)c->cnt);
    rotate_ring(c);
  }
  RingMap rm = current_map(c);
  for (int s = 0; s < c->params.euler_intervals; s++) {
    int st = force_pass(c, 0, true, dt, EPI_STORE, rm, true, 0);
    if (st) return st;
    launch(c, "euler_update", k_euler_update, blocks_for(n, 256), 256, n, c->P, dt,
           (const Counters*)c->cnt);
    c->prepared = -1;
    c->time = c->time + dt;
    st = apply_walls(c, 0);
    if (st) return st;
  }
  launch(c, "apply_pbc", k_apply_pbc, blocks_for(n, 256), 256, (const DevParams*)c->dp,
         (const int*)c->sysid, n, c->P,
         (const Counters*)c->cnt);
  c->prepared = -1;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "euler");
  return DEM_OK;
}

// Capture `steps` MoveParticles steps (no host checks) into one graph; the
// host bookkeeping is left as it was.
int capture_steps(dem_ctx* c, int steps, cudaGraphExec_t* out) {
  cudaGraph_t g;
  bool prof = c->prof;
  c->prof = false;
  long long l0 = c->launches;
  int rm[5];
  std::memcpy(rm, c->ringmap, sizeof(rm));
  const int hc = c->hcur, par = c->par, prep = c->prepared, last = c->last_side;
  const double t = c->time;
  const bool lazy = c->lazy_state;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int st = DEM_OK;
  c->capturing = true;
  for (int k = 0; k < steps && !st; k++) st = move_particles_impl(c, 0, false, k);
  c->capturing = false;
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  c->prof = prof;
  c->graph_kernels = c->launches - l0;
  c->launches = l0;
  std::memcpy(c->ringmap, rm, sizeof(rm));
  c->hcur = hc;
  c->par = par;
  c->prepared = prep;
  c->last_side = last;
  c->time = t;
  c->lazy_state = lazy;
  if (st) return st;
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  return DEM_OK;
}

// A chunk runs as one persistent launch when its steps hold nothing but
// force passes: no wall motion (a host copy per step), no fluid drag (two
// more kernels per pass), no per-kernel event timing.
bool chunk_persistent(const dem_ctx* c) {
  return c->launch_mode == 1 && c->wm.empty() && !c->fluid && !c->prof;
}

// Record `steps` MoveParticles steps as the passes of one persistent chunk
// into prog[phase] (the host bookkeeping is left as it was, as by
// capture_steps).  Recording launches nothing.
int record_chunk(dem_ctx* c, int steps, int phase) {
  const long long l0 = c->launches;
  int rm[5];
  std::memcpy(rm, c->ringmap, sizeof(rm));
  const int hc = c->hcur, par = c->par, prep = c->prepared, last = c->last_side;
  const double t = c->time;
  const bool lazy = c->lazy_state;
  c->rec.clear();
  c->rec_n = 0;
  c->recording = true;
  c->capturing = true;
  int st = DEM_OK;
  for (int k = 0; k < steps && !st; k++) st = move_particles_impl(c, 0, false, k);
  c->recording = false;
  c->capturing = false;
  const bool clean = c->launches == l0;
  c->launches = l0;
  std::memcpy(c->ringmap, rm, sizeof(rm));
  c->hcur = hc;
  c->par = par;
  c->prepared = prep;
  c->last_side = last;
  c->time = t;
  c->lazy_state = lazy;
  if (st) return st;
  if (!clean || c->rec_n != 2 * steps)
    return fail(c, DEM_ERR_STATE, "a persistent chunk held work other than its force passes");
  CK(cudaMalloc(&c->prog[phase], c->rec.size()));
  CK(cudaMemcpy(c->prog[phase], c->rec.data(), c->rec.size(), cudaMemcpyHostToDevice));
  c->prog_n[phase] = c->rec_n;
  return DEM_OK;
}

// the FP64 chunk kernel for this context as a cooperative launch of at
// most `want` blocks (as many as fit on the device at once)
template <class K>
cudaError_t coop_launch64(K k, const ChunkPass64* prog, int npass, GridSync g, int want,
                          cudaStream_t st, int* blocks_out) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 128, 0);
  const int nb = std::min(want, per * sms);
  if (nb <= 0) return cudaErrorLaunchOutOfResources;
  g.expected += (unsigned)nb;  // (on entry: the blocks a test adds to every barrier)
  void* args[] = {(void*)&prog, (void*)&npass, (void*)&g};
  if (blocks_out) *blocks_out = nb;
  return cudaLaunchCooperativeKernel((const void*)k, dim3(nb), dim3(128), args, 0, st);
}

// Launch the recorded chunk of rotation phase `phase`.
int launch_chunk(dem_ctx* c, int phase) {
  if (!c->bar) {
    CK(cudaMalloc(&c->bar, 2 * sizeof(unsigned)));
    CK(cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned), c->stream));
  }
  GridSync g{c->bar, c->bar + 1, c->cnt, c->bar_limit_ns, (unsigned)c->bar_extra};
  const int want = std::max(1, (int)blocks_for(c->n, 128));
  const bool walls = c->nw_max > 0;
  cudaError_t e;
  if (c->precision == DEM_PREC_MIXED) {
    e = mixed_chunk(c->pp, walls, c->has_cone,
                    (const ChunkPass<float4, float2, MixedView>*)c->prog[phase], c->prog_n[phase],
                    g, want, c->stream, &c->chunk_blocks);
  } else {
    const ChunkPass64* prog = (const ChunkPass64*)c->prog[phase];
    const int np = c->prog_n[phase];
    if (walls) {
      e = c->pp ? coop_launch64(k_chunk_fp64<true, true>, prog, np, g, want, c->stream,
                                &c->chunk_blocks)
                : coop_launch64(k_chunk_fp64<false, true>, prog, np, g, want, c->stream,
                                &c->chunk_blocks);
    } else {
      e = c->pp ? coop_launch64(k_chunk_fp64<true, false>, prog, np, g, want, c->stream,
                                &c->chunk_blocks)
                : coop_launch64(k_chunk_fp64<false, false>, prog, np, g, want, c->stream,
                                &c->chunk_blocks);
    }
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "persistent chunk launch");
  c->launches += 1;
  return DEM_OK;
}


// ---------------------------------------------------------------------------
// Slabs of a spatial decomposition (dem_slab_*): column tables and layers.

void slab_col(SlabCols& C, const void* base, int elem, int rows, long long stride) {
  if (C.n >= SLAB_MAXC) {
    C.overflow = 1;
    return;
  }
  const int k = C.n++;
  C.src[k] = (const char*)base;
  C.dst[k] = (char*)base;
  C.elem[k] = elem;
  C.rows[k] = rows;
  C.stride[k] = stride;
  C.off[k] = C.rec;
  C.rec += elem * rows;
}

SlabCols slab_cols_begin() {
  SlabCols C{};
  C.rec = SLAB_ID;
  return C;
}

// the history rows of table b (counts, partners, values; FP32 values in
// mixed mode), and with walls the wall rows
// (rows: the record slots carried, at most the capacity; a particle's
// records past its count are not read)
void slab_hist_cols(const dem_ctx* c, SlabCols& C, int b, bool walls, int rows) {
  const History& H = c->H[b];
  const long long N = H.n;
  const bool mixed = c->precision == DEM_PREC_MIXED;
  rows = std::min(rows, H.cap);
  slab_col(C, H.cnt, 4, 1, 0);
  if (rows > 0) {
    slab_col(C, H.key, 4, rows, N * 4);
    if (mixed) {
      slab_col(C, c->M.ha[b], 16, rows, N * 16);
      slab_col(C, c->M.hb[b], 16, rows, N * 16);
      slab_col(C, c->M.hc[b], 4, rows, N * 4);
    } else {
      slab_col(C, H.val, 48, rows, N * 48);
    }
  }
  if (!walls) return;
  const int nw = std::max(c->params.n_walls, 1);
  slab_col(C, H.wflag, 4 * nw, 1, 0);
  if (mixed) {
    slab_col(C, c->M.wa[b], 16 * nw, 1, 0);
    slab_col(C, c->M.wb[b], 16 * nw, 1, 0);
    slab_col(C, c->M.wc[b], 4 * nw, 1, 0);
  } else {
    slab_col(C, H.wval, 48 * nw, 1, 0);
  }
}

// what a slab needs of a ghost for the pass on `side`: list link, pass
// copies, cell, current history rows
SlabCols slab_ghost_cols(const dem_ctx* c, int side, int hrows) {
  const bool mixed = c->precision == DEM_PREC_MIXED;
  SlabCols C = slab_cols_begin();
  slab_col(C, c->L.next, 4, 1, 0);
  slab_col(C, c->X[side], 32, 1, 0);
  slab_col(C, c->v4[side], mixed ? 16 : 32, 1, 0);
  slab_col(C, c->w2[side], mixed ? 8 : 16, 1, 0);
  slab_col(C, c->L.cell[c->par], 4, 1, 0);
  slab_hist_cols(c, C, c->hcur, false, hrows);
  return C;
}

// everything a particle owns: state, Predicted, ABM ring, corrector sums,
// pass copies of both sides, both cell entries, both history tables
SlabCols slab_full_cols(const dem_ctx* c) {
  const bool mixed = c->precision == DEM_PREC_MIXED;
  const long long N = c->ncap, n = c->n;
  SlabCols C = slab_cols_begin();
  slab_col(C, c->state_block, 8, 30, N * 8);
  if (c->nprev > 0) slab_col(C, c->ring, 8, 9 * (c->nprev + 1), n * 8);
  if (c->amsum) slab_col(C, c->amsum, 8, 9, n * 8);
  for (int b = 0; b < 2; b++) {
    slab_col(C, c->X[b], 32, 1, 0);
    slab_col(C, c->v4[b], mixed ? 16 : 32, 1, 0);
    slab_col(C, c->w2[b], mixed ? 8 : 16, 1, 0);
    slab_col(C, c->L.cell[b], 4, 1, 0);
  }
  for (int b = 0; b < 2; b++) slab_hist_cols(c, C, b, true, c->H[b].cap);
  return C;
}

int slab_nxy(const dem_ctx* c) { return c->hsys[0].nx * c->hsys[0].ny; }
int slab_nz(const dem_ctx* c) { return c->hsys[0].nz; }
// first cell of layer z (taken modulo Nz)
int slab_layer(const dem_ctx* c, int z) {
  const int nz = slab_nz(c);
  return c->hsys[0].coff + ((z % nz + nz) % nz) * slab_nxy(c);
}
// whether the slab has a layer above / below it (periodic z: always)
bool slab_has_up(const dem_ctx* c) { return c->hsys[0].pbc[2] || c->slab_z1 < slab_nz(c); }
bool slab_has_down(const dem_ctx* c) { return c->hsys[0].pbc[2] || c->slab_z0 > 0; }

// the particles of layer z into c->slab_list; returns their count
int slab_list_layer(dem_ctx* c, int z, int* count) {
  CK(cudaMemsetAsync(c->slab_count, 0, 2 * sizeof(int), c->stream));
  const int nxy = slab_nxy(c);
  launch(c, "slab_layer", k_slab_layer, blocks_for(nxy, 128), 128, (const int*)c->L.head,
         (const int*)c->L.next, slab_layer(c, z), nxy, c->n, c->slab_list, c->slab_count, c->ncap,
         c->slab_count + 1);
  int h[2];
  CK(cudaMemcpyAsync(h, c->slab_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h[1]) return fail(c, DEM_ERR_STATE, "slab: a cell list of a boundary layer is inconsistent");
  *count = h[0];
  return DEM_OK;
}

// the largest v[p] over the particles of c->slab_list[0..count)
int slab_max_over(dem_ctx* c, int count, const int* v, int* out) {
  *out = 0;
  if (count == 0) return DEM_OK;
  CK(cudaMemsetAsync(c->slab_count + 2, 0, sizeof(int), c->stream));
  launch(c, "slab_max_of", k_slab_max_of, blocks_for(count, 256), 256, (const int*)c->slab_list,
         count, v, c->slab_count + 2);
  CK(cudaMemcpyAsync(out, c->slab_count + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DEM_OK;
}

// the header and records of a packed exchange
int slab_write(dem_ctx* c, int what, const SlabCols& C, int count, const std::vector<int>& extra,
               void* buf, int64_t cap, int64_t* bytes) {
  if (C.overflow) return fail(c, DEM_ERR_STATE, "slab: too many particle arrays");
  const int64_t head = SLAB_HEAD + 4 * (int64_t)extra.size();
  const int64_t body = (head + 15) / 16 * 16;
  const int64_t total = body + (int64_t)count * C.rec;
  *bytes = total;
  if (total > cap) return fail(c, DEM_ERR_CAPACITY, "slab: the exchange buffer is too small");
  std::vector<int> h(4 + extra.size());
  h[0] = what;
  h[1] = count;
  h[2] = C.rec;
  h[3] = (int)extra.size();
  std::copy(extra.begin(), extra.end(), h.begin() + 4);
  CK(cudaMemcpyAsync(buf, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (count > 0) {
    const long long thr = (long long)count * (C.rec / 4);
    launch(c, "slab_cols", k_slab_cols, (unsigned)((thr + 255) / 256), 256, C,
           (const int*)c->slab_list, count, (char*)buf + body, (int*)nullptr, 0, (int*)nullptr);
  }
  CK(cudaStreamSynchronize(c->stream));  // the header's host copy is read
  return DEM_OK;
}

// the header of a received exchange (host copy) and where its records start
int slab_read_head(dem_ctx* c, const void* buf, int64_t bytes, int what, std::vector<int>& h,
                   int64_t* body) {
  int h4[4];
  if (bytes < SLAB_HEAD) return fail(c, DEM_ERR_INVALID, "slab: short exchange buffer");
  CK(cudaMemcpy(h4, buf, sizeof(h4), cudaMemcpyDeviceToHost));
  if (h4[0] != what || h4[1] < 0 || h4[3] < 0)
    return fail(c, DEM_ERR_INVALID, "slab: the buffer holds another exchange");
  h.assign(4 + (size_t)h4[3], 0);
  CK(cudaMemcpy(h.data(), buf, h.size() * sizeof(int), cudaMemcpyDeviceToHost));
  *body = (SLAB_HEAD + 4 * (int64_t)h4[3] + 15) / 16 * 16;
  if (*body + (int64_t)h4[1] * h4[2] > bytes)
    return fail(c, DEM_ERR_INVALID, "slab: truncated exchange buffer");
  return DEM_OK;
}

// ---------------------------------------------------------------------------
// Storage in cell order (dem_set_reorder).

// Permute every particle array: place s takes the particle stored at pi[s]
// (pi a device array of n places); the stored particle numbers (cell
// lists, slots, arrival lists, history partners, candidate rows) are
// renamed.
int permute_particles(dem_ctx* c, const int* pi) {
  const int n = c->n;
  if (n == 0) return DEM_OK;
  SlabCols C = slab_full_cols(c);
  auto col = [&](const void* base, int elem) { slab_col(C, base, elem, 1, 0); };
  col(c->comp, 4);
  col(c->radius, 8);
  col(c->gid, 4);
  if (c->sysid) col(c->sysid, 4);
  col(c->L.next, 4);
  col(c->L.arr_next, 4);
  col(c->L.mflag, 4);
  col(c->L.mnext, 4);
  col(c->rows.meta, 4);
  col(c->rows.rank, 4);
  // the candidate rows move with their particles and are renamed below:
  // the same partners in the same order, so no row is rebuilt
  slab_col(C, c->rows.cand, 4, c->rows.kc, (long long)n * 4);
  col(c->in_cnt, 4);
  col(c->matched, 4);
  if (C.overflow) return fail(c, DEM_ERR_STATE, "reorder: too many particle arrays");
  size_t most = 0;
  for (int k = 0; k < C.n; k++) most = std::max(most, (size_t)C.elem[k] * C.rows[k] * (size_t)n);
  char* tmp = nullptr;
  int* inv = nullptr;
  CK(cudaMalloc(&tmp, most));
  CK(cudaMalloc(&inv, sizeof(int) * (size_t)n));
  for (int k = 0; k < C.n; k++) {
    const long long thr = (long long)C.elem[k] / 4 * n * C.rows[k];
    const unsigned g = (unsigned)((thr + 255) / 256);
    launch(c, "reorder_gather", k_gather_col, g, 256u, C.src[k], C.elem[k], C.rows[k],
           C.stride[k], n, pi, tmp);
    launch(c, "reorder_scatter", k_scatter_col, g, 256u, C.dst[k], C.elem[k], C.rows[k],
           C.stride[k], n, (const char*)tmp);
  }
  launch(c, "inverse", k_inverse, blocks_for(n, 256), 256, n, pi, inv);
  auto remap = [&](int* a, long long m) {
    if (m > 0)
      launch(c, "remap", k_remap, (unsigned)((m + 255) / 256), 256u, a, m, (const int*)inv, n);
  };
  const long long nc = c->ncell_total;
  remap(c->L.next, n);
  remap(c->L.arr_next, n);
  remap(c->L.mnext, n);
  remap(c->L.head, nc);
  remap(c->L.arr_head, nc);
  remap(c->L.slot, nc * SLOT_CAP);
  for (int b = 0; b < 2; b++) remap(c->H[b].key, (long long)c->H[b].cap * c->H[b].n);
  remap(c->rows.cand, (long long)c->rows.kc * n);
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(tmp);
  cudaFree(inv);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "reorder");
  return DEM_OK;
}

// gid for the whole capacity, the identity while the storage is in the
// reference's order (the relink reads it through L.gid, so a new array
// means new graphs)
int ensure_gid(dem_ctx* c) {
  if (c->gid && c->gid_cap >= c->ncap) return DEM_OK;
  if (c->permuted) return fail(c, DEM_ERR_STATE, "reorder: capacity changed while permuted");
  cudaFree(c->gid);
  c->gid = nullptr;
  const int cap = std::max(c->ncap, 1);
  CK(cudaMalloc(&c->gid, sizeof(int) * (size_t)cap));
  launch(c, "iota", k_iota, blocks_for(cap, 256), 256, cap, c->gid);
  c->gid_cap = cap;
  c->L.gid = c->gid;
  drop_graphs(c);
  return DEM_OK;
}

// the particles into the cells' list order (cell by cell, each list in
// order): gathers from one cell's particles then read neighbouring memory
int reorder_by_cell(dem_ctx* c) {
  const int n = c->n, nc = c->ncell_total;
  if (n == 0) return DEM_OK;
  {
    int st = ensure_gid(c);
    if (st) return st;
  }
  int* pi = nullptr;
  CK(cudaMalloc(&pi, sizeof(int) * (size_t)n));
  int* dev_err = nullptr;
  CK(cudaMalloc(&dev_err, sizeof(int)));
  CK(cudaMemsetAsync(dev_err, 0, sizeof(int), c->stream));
  launch(c, "reorder_counts", k_reorder_counts, blocks_for(nc, 256), 256, c->L, nc, c->cell_cnt,
         dev_err);
  launch(c, "scan_tiles", k_scan_tiles, (unsigned)c->n_tiles, SCAN_THREADS,
         (const int*)c->cell_cnt, nc, c->cell_start, c->scan_bsum, (const Counters*)c->cnt);
  launch(c, "scan_bsums", k_scan_bsums, 1u, SCAN_THREADS, c->scan_bsum, c->n_tiles,
         c->cell_start, nc, (const Counters*)c->cnt);
  launch(c, "scan_add", k_scan_add, blocks_for(nc, 256), 256, c->cell_start, nc,
         (const int*)c->scan_bsum, (const Counters*)c->cnt);
  launch(c, "reorder_fill", k_reorder_fill, blocks_for(nc, 256), 256, c->L, nc,
         (const int*)c->cell_start, pi, n, dev_err);
  int h_err = 0, total = 0;
  CK(cudaMemcpyAsync(&h_err, dev_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&total, c->cell_start + nc, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(dev_err);
  int st = DEM_OK;
  if (h_err || total != n) st = fail(c, DEM_ERR_STATE, "reorder: cell lists inconsistent");
  else st = permute_particles(c, pi);
  cudaFree(pi);
  if (st) return st;
  c->permuted = true;
  c->reorders++;
  return DEM_OK;
}

// back to the reference's order (place g holds the particle numbered g)
int restore_order(dem_ctx* c, bool settle) {
  if (settle) {
    int st = settle_state(c);
    if (st) return st;
  }
  if (!c->permuted) return DEM_OK;
  const int n = c->n;
  int* pi = nullptr;
  CK(cudaMalloc(&pi, sizeof(int) * (size_t)std::max(n, 1)));
  if (n > 0) launch(c, "inverse", k_inverse, blocks_for(n, 256), 256, n, (const int*)c->gid, pi);
  int st = permute_particles(c, pi);
  cudaFree(pi);
  if (st) return st;
  c->permuted = false;
  return DEM_OK;
}


}  // namespace

// ===========================================================================
// C-ABI

extern "C" {

const char* dem_version(void) { return DEM_VERSION_STR; }

int dem_select_device(int32_t device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DEM_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return DEM_ERR_INVALID;
  return cudaSetDevice(device) == cudaSuccess ? DEM_OK : DEM_ERR_CUDA;
}

const char* dem_last_error(const dem_ctx* c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"

namespace {

// DevParams of one system: scaled parameters, ABM coefficients
// (InitializeAuxiliaries, src/MDEM.f90:110-162), the cell grid
// (InitCellStructure3D, src/MCells.f90:155-227) and the force tables
// (InitializeForce, src/MForces.f90:54-87).
int build_system(const dem_params* p, DevParams& h) {
  if (p->method_order < 1 || p->method_order > 4) return DEM_ERR_INVALID;
  if (p->n_walls < 0 || p->n_walls > NWM) return DEM_ERR_INVALID;
  if (p->n_components < 0 || p->n_components > NCM) return DEM_ERR_INVALID;
  if (p->euler_intervals < 1) return DEM_ERR_INVALID;
  if (p->precision != DEM_PREC_FP64 && p->precision != DEM_PREC_MIXED) return DEM_ERR_INVALID;
  if (p->precision == DEM_PREC_MIXED && !mixed_available()) return DEM_ERR_UNSUPPORTED;
  for (int w = 0; w < p->n_walls; w++)
    if (p->walls[w].shape != DEM_WALL_RECTANGLE && p->walls[w].shape != DEM_WALL_CONE)
      return DEM_ERR_UNSUPPORTED;
  h = DevParams{};
  h.nc = p->n_components;
  h.nw = p->n_walls;
  for (int k = 0; k < 3; k++) {
    h.pbc[k] = p->pbc[k] ? 1 : 0;
    h.lbox[k] = p->lbox[k];
    h.inv_lbox[k] = 1.0 / p->lbox[k];  // ScaleVariables, src/DEM.f90:825
    h.gravity[k] = p->gravity[k];
  }
  h.nprev = p->method_order - 1;
  // ABM coefficients, src/MDEM.f90:127-154
  double dt = p->time_step;
  switch (p->method_order) {
    case 4: {
      double Aux = dt / 24.0;
      h.ab0 = 55.0 * Aux; h.am0 = 9.0 * Aux;
      h.ab[0] = -59.0 * Aux; h.am[0] = 19.0 * Aux;
      h.ab[1] = 37.0 * Aux; h.am[1] = -5.0 * Aux;
      h.ab[2] = -9.0 * Aux; h.am[2] = 1.0 * Aux;
    } break;
    case 3: {
      double Aux = dt / 12.0;
      h.ab0 = 23.0 * Aux; h.am0 = 5.0 * Aux;
      h.ab[0] = -16.0 * Aux; h.am[0] = 8.0 * Aux;
      h.ab[1] = 5.0 * Aux; h.am[1] = -1.0 * Aux;
    } break;
    case 2:
      h.ab0 = 1.5 * dt; h.am0 = 0.5 * dt;
      h.ab[0] = -0.5 * dt; h.am[0] = 0.5 * dt;
      break;
    default:
      h.ab0 = dt; h.am0 = dt;
  }
  // cell grid, InitCellStructure3D (src/MCells.f90:155-227) with
  // CutOff = 2*maxval(Component%Radius) (src/MForces.f90:96)
  double rmax = 0.0;
  if (p->n_components > 0) {
    for (int i = 0; i < p->n_components; i++) rmax = std::max(rmax, p->comp_radius[i]);
  } else {
    rmax = p->pp_rmax;
  }
  double CutOff = 2.0 * rmax;
  if (!(CutOff > 0.0)) {
    return DEM_ERR_INVALID;
  }
  int MaxNCell = p->max_ncell > 0 ? p->max_ncell : 30000;
  double Lx = p->lbox[0], Ly = p->lbox[1], Lz = p->lbox[2];
  int Nx4 = (int)(Lx / CutOff), Ny4 = (int)(Ly / CutOff), Nz4 = (int)(Lz / CutOff);
  long long N4 = (long long)Nx4 * Ny4 * Nz4;
  int Nx, Ny, Nz;
  if (N4 > MaxNCell) {
    double LCell = std::pow(Lx * Ly * Lz / (double)MaxNCell, 1.0 / 3.0);
    Nx = (int)(Lx / LCell);
    Ny = (int)(Ly / LCell);
    Nz = (int)(Lz / LCell);
  } else {
    Nx = Nx4;
    Ny = Ny4;
    Nz = Nz4;
  }
  int N[3] = {Nx, Ny, Nz};
  for (int k = 0; k < 3; k++) {
    if (N[k] < 1) {
      return DEM_ERR_INVALID;
    }
    // with 1 or 2 cells along a periodic axis the reference lists a cell
    // twice in a half shell (duplicate pair visits); not reproduced here
    if (p->pbc[k] && N[k] < 3) {
      return DEM_ERR_UNSUPPORTED;
    }
  }
  h.nx = Nx;
  h.ny = Ny;
  h.nz = Nz;
  h.ncell = Nx * Ny * Nz;
  h.nxbylx = (double)Nx / Lx;
  h.nybyly = (double)Ny / Ly;
  h.nzbylz = (double)Nz / Lz;
  h.nxby2 = (double)Nx * 0.5;
  h.nyby2 = (double)Ny * 0.5;
  h.nzby2 = (double)Nz * 0.5;
  h.inv_nx = 1.0 / (double)Nx;
  h.inv_ny = 1.0 / (double)Ny;
  // material tables
  for (int i = 0; i < NCM; i++) {
    h.comp_radius[i] = p->comp_radius[i];
    h.comp_inv_mass[i] = p->comp_inv_mass[i];
    h.comp_inv_inertia[i] = p->comp_inv_inertia[i];
    h.comp_eff_mass[i] = p->comp_eff_mass[i];
  }
  std::memcpy(h.min_dij, p->min_dij, sizeof(h.min_dij));
  std::memcpy(h.min_dij_sq, p->min_dij_sq, sizeof(h.min_dij_sq));
  std::memcpy(h.kn, p->kn, sizeof(h.kn));
  std::memcpy(h.yn, p->yn, sizeof(h.yn));
  std::memcpy(h.kt, p->kt, sizeof(h.kt));
  std::memcpy(h.yt, p->yt, sizeof(h.yt));
  std::memcpy(h.mu_sq, p->mu_sq, sizeof(h.mu_sq));
  std::memcpy(h.knw, p->knw, sizeof(h.knw));
  std::memcpy(h.ynw, p->ynw, sizeof(h.ynw));
  std::memcpy(h.ktw, p->ktw, sizeof(h.ktw));
  std::memcpy(h.ytw, p->ytw, sizeof(h.ytw));
  std::memcpy(h.muw_sq, p->muw_sq, sizeof(h.muw_sq));
  // largest MinDijSq of any pair, for the screening early-out
  h.max_min_dij_sq = 0.0;
  if (p->n_components > 0) {
    for (int i = 0; i < p->n_components; i++)
      for (int j = 0; j < p->n_components; j++)
        h.max_min_dij_sq = std::max(h.max_min_dij_sq, p->min_dij_sq[i * NCM + j]);
  } else {
    double d = p->pp_rmax + p->pp_rmax;  // Ri + Rj <= rmax + rmax after rounding
    h.max_min_dij_sq = d * d;
  }
  {
    // candidate rows keep the partners within MinDij + skin; a pair absent
    // from them moved closer by at most twice the largest displacement since
    // the rows were built, so the rows are complete while the accumulated
    // displacement bound stays below skin/2 (0.4 skin keeps a margin)
    h.cutoff = CutOff;
    h.vl_skin = 0.05 * CutOff;
    h.vl_thr = 0.4 * h.vl_skin;
  }
  h.pp_mass_coef = p->pp_mass_coef;
  h.pp_density = p->pp_density;
  h.pp_fluid_density = p->pp_fluid_density;
  h.pp_kn = p->pp_kn;
  h.pp_kt = p->pp_kt;
  h.pp_gamma_n = p->pp_gamma_n;
  h.pp_gamma_t = p->pp_gamma_t;
  h.pp_mu_sq = p->pp_mu_sq;
  for (int w = 0; w < NWM; w++) {
    h.pp_knw[w] = p->pp_knw[w];
    h.pp_ktw[w] = p->pp_ktw[w];
    h.pp_gamma_nw[w] = p->pp_gamma_nw[w];
    h.pp_gamma_tw[w] = p->pp_gamma_tw[w];
    h.pp_muw_sq[w] = p->pp_muw_sq[w];
    h.walls[w] = p->walls[w];
  }

  for (int k = 0; k < 3; k++) {
    h.box.lbox[k] = h.lbox[k];
    h.box.inv_lbox[k] = h.inv_lbox[k];
    h.box.half_lim[k] = 0.49 * h.lbox[k];
    h.box.pbc[k] = h.pbc[k];
  }
  return DEM_OK;
}

}  // namespace

extern "C" {

int dem_create(const dem_params* p, dem_ctx** out) { return dem_create_ensemble(p, 1, out); }

int dem_create_ensemble(const dem_params* ps, int32_t nsys, dem_ctx** out) {
  if (!ps || !out || nsys < 1) return DEM_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DEM_ERR_NO_DEVICE;
  }
  std::vector<DevParams> hs((size_t)nsys);
  long long ncell = 0;
  for (int s = 0; s < nsys; s++) {
    const dem_params* p = ps + s;
    // the systems share the integrator and the precision
    if (p->method_order != ps->method_order || p->euler_intervals != ps->euler_intervals ||
        p->time_step != ps->time_step || p->precision != ps->precision ||
        (p->n_components == 0) != (ps->n_components == 0))
      return DEM_ERR_INVALID;
    int st = build_system(p, hs[(size_t)s]);
    if (st) return st;
    hs[(size_t)s].coff = (int)ncell;
    hs[(size_t)s].sys = s;
    hs[(size_t)s].slab_c0 = (int)ncell;
    hs[(size_t)s].slab_c1 = (int)ncell + hs[(size_t)s].ncell;
    ncell += hs[(size_t)s].ncell;
    if (ncell >= (1LL << 30)) return DEM_ERR_INVALID;
  }
  const dem_params* p = ps;
  dem_ctx* c = new dem_ctx();
  c->params = *p;
  c->pp = p->n_components == 0;
  c->precision = p->precision;
  c->nprev = p->method_order - 1;
  c->hcap = p->hist_capacity > 0 ? p->hist_capacity : 16;
  c->nsys = nsys;
  c->removal = nsys == 1;
  for (int s = 0; s < nsys; s++) {
    c->nw_max = std::max(c->nw_max, ps[s].n_walls);
    for (int w = 0; w < ps[s].n_walls; w++)
      if (ps[s].walls[w].shape == DEM_WALL_CONE) c->has_cone = true;
  }
  c->hsys = hs;
  c->hp = hs[0];
  c->ncell_total = (int)ncell;
  c->sys_params.assign(ps, ps + nsys);
  cudaGetDevice(&c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return DEM_ERR_CUDA;
  }
  const size_t NC = (size_t)c->ncell_total;
  cudaError_t e = cudaMalloc(&c->dp, sizeof(DevParams) * (size_t)nsys);
  if (e == cudaSuccess)
    e = cudaMemcpy(c->dp, hs.data(), sizeof(DevParams) * (size_t)nsys, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nsys > 1) {
    std::vector<int> cs(NC);
    for (int s = 0; s < nsys; s++)
      for (int k = 0; k < hs[(size_t)s].ncell; k++) cs[(size_t)hs[(size_t)s].coff + k] = s;
    e = cudaMalloc(&c->cellsys, sizeof(int) * NC);
    if (e == cudaSuccess) e = cudaMemcpy(c->cellsys, cs.data(), sizeof(int) * NC, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&c->cnt, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->cnt, 0, sizeof(Counters), c->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&c->hcnt, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMalloc(&c->cell_start, sizeof(int) * (NC + 1));
  if (e == cudaSuccess) e = cudaMalloc(&c->cell_cnt, sizeof(int) * NC);
  c->n_tiles = (int)((NC + SCAN_TILE - 1) / SCAN_TILE);
  if (e == cudaSuccess) e = cudaMalloc(&c->scan_bsum, sizeof(int) * (size_t)c->n_tiles);
  if (e == cudaSuccess) e = cudaMalloc(&c->obs_partial, sizeof(double) * 8 * 1184);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    c->err = std::string("dem_create: ") + cudaGetErrorString(e);
    dem_destroy(c);
    return DEM_ERR_CUDA;
  }
  std::memset(c->hcnt, 0, sizeof(Counters));
  *out = c;
  return DEM_OK;
}

int dem_set_system_counts(dem_ctx* c, const int32_t* counts) {
  if (!c || !counts) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  long long off = 0;
  for (int s = 0; s < c->nsys; s++) {
    if (counts[s] < 0) return fail(c, DEM_ERR_INVALID, "negative system size");
    c->hsys[(size_t)s].poff = (int)off;
    c->hsys[(size_t)s].np = counts[s];
    off += counts[s];
    if (off >= (1LL << 30)) return fail(c, DEM_ERR_INVALID, "too many particles");
  }
  c->counts.assign(counts, counts + c->nsys);
  sync_host_walls(c);
  c->hp = c->hsys[0];
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(c->dp, c->hsys.data(), sizeof(DevParams) * (size_t)c->nsys,
                cudaMemcpyHostToDevice));
  return DEM_OK;
}

void dem_destroy(dem_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  free_state(c);
  cudaFree(c->bar);
  cudaFree(c->gid);
  cudaFree(c->gstamp);
  cudaFree(c->slab_list);
  cudaFree(c->slab_ghosts);
  cudaFree(c->slab_count);
  cudaFree(c->dp);
  cudaFree(c->rm_buf);
  cudaFree(c->pour_cand);
  cudaFree(c->pour_fits);
  cudaFree(c->fl_vf);
  cudaFree(c->drag);
  cudaFree(c->amsum);
  if (c->wall_slots) cudaFreeHost(c->wall_slots);
  cudaFree(c->cellsys);
  cudaFree(c->cnt);
  if (c->hcnt) cudaFreeHost(c->hcnt);
  cudaFree(c->cell_start);
  cudaFree(c->cell_cnt);
  cudaFree(c->scan_bsum);
  cudaFree(c->obs_partial);
  for (auto& pe : c->pending) {
    cudaEventDestroy(pe.e0);
    cudaEventDestroy(pe.e1);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  for (auto e : c->timer)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

static int put_state_arrays(dem_ctx* c, const StateArrays& s, const double* pos,
                            const double* vel, const double* omega, const double* acc,
                            const double* alpha);

int dem_set_state(dem_ctx* c, int32_t n, const int32_t* comp, const double* radius,
                  const double* pos, const double* vel, const double* omega, const double* acc,
                  const double* alpha) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (n < 0 || !pos || !vel || !omega) return fail(c, DEM_ERR_INVALID, "bad state arrays");
  if (!c->pp && !comp) return fail(c, DEM_ERR_INVALID, "component indices required");
  if (c->pp && !radius) return fail(c, DEM_ERR_INVALID, "per-particle radii required");
  if (n >= (1 << 30)) return fail(c, DEM_ERR_INVALID, "too many particles");
  // system of every particle (an ensemble's particles are concatenated by system)
  std::vector<int> sid;
  if (c->nsys > 1) {
    if ((int)c->counts.size() != c->nsys)
      return fail(c, DEM_ERR_STATE, "ensemble: call dem_set_system_counts first");
    long long tot = 0;
    for (int k : c->counts) tot += k;
    if (tot != n) return fail(c, DEM_ERR_INVALID, "n differs from the sum of the system sizes");
    sid.resize((size_t)n);
    for (int s = 0, i = 0; s < c->nsys; s++)
      for (int k = 0; k < c->counts[(size_t)s]; k++) sid[(size_t)i++] = s;
  }
  auto sys_of = [&](int i) -> const dem_params& {
    return c->sys_params[sid.empty() ? 0 : (size_t)sid[(size_t)i]];
  };
  if (!c->pp)
    for (int i = 0; i < n; i++)
      if (comp[i] < 0 || comp[i] >= sys_of(i).n_components)
        return fail(c, DEM_ERR_INVALID, "component index out of range");
  if (c->pp)
    for (int i = 0; i < n; i++)
      if (!(radius[i] > 0.0) || radius[i] > sys_of(i).pp_rmax)
        return fail(c, DEM_ERR_INVALID, "radius must lie in (0, pp_rmax]");
  CK(cudaStreamSynchronize(c->stream));
  drop_graphs(c);
  free_state(c);
  c->n = n;
  // Component(:)%Number, and room for pouring up to the targets
  c->comp_count.assign((size_t)std::max(c->params.n_components, 0), 0);
  if (!c->pp && c->nsys == 1)
    for (int i = 0; i < n; i++) c->comp_count[(size_t)comp[i]]++;
  size_t N = (size_t)std::max(std::max(std::max(n, c->ncap_hint), pour_capacity(c, c->comp_count, n)), 1);
  c->ncap = (int)N;
  CK(cudaMalloc(&c->state_block, sizeof(double) * 30 * N));
  CK(cudaMalloc(&c->staging, sizeof(double) * 15 * N));
  CK(cudaMemsetAsync(c->state_block, 0, sizeof(double) * 30 * N, c->stream));
  c->P = make_state(c->state_block, N);
  c->Pr = make_state(c->state_block + 15 * N, N);
  int slots = c->nprev + 1;
  CK(cudaMalloc(&c->ring, sizeof(double) * 9 * N * slots));
  CK(cudaMemsetAsync(c->ring, 0, sizeof(double) * 9 * N * slots, c->stream));
  CK(cudaMalloc(&c->radius, sizeof(double) * N));
  CK(cudaMalloc(&c->comp, sizeof(int) * N));
  CK(cudaMalloc(&c->S.orig, sizeof(int) * N));
  CK(cudaMalloc(&c->S.cell, sizeof(int) * N));
  CK(cudaMalloc(&c->a_cell, sizeof(int) * N));
  CK(cudaMalloc(&c->a_loc, sizeof(int) * N));
  CK(cudaMalloc(&c->a_orig, sizeof(int) * N));
  CK(cudaMalloc(&c->t_orig, sizeof(int) * N));
  CK(cudaMalloc(&c->a_key, sizeof(unsigned) * N));
  CK(cudaMalloc(&c->t_key, sizeof(unsigned) * N));
  {
    const size_t NC = (size_t)c->ncell_total;
    CellLists& L = c->L;
    CK(cudaMalloc(&L.head, sizeof(int) * NC));
    CK(cudaMalloc(&L.next, sizeof(int) * N));
    CK(cudaMalloc(&L.cell[0], sizeof(int) * N));
    CK(cudaMalloc(&L.cell[1], sizeof(int) * N));
    CK(cudaMalloc(&L.arr_head, sizeof(int) * NC));
    CK(cudaMalloc(&L.arr_next, sizeof(int) * N));
    CK(cudaMalloc(&L.mflag, sizeof(int) * N));
    CK(cudaMalloc(&L.mnext, sizeof(int) * N));
    CK(cudaMalloc(&L.dflag, sizeof(int) * NC));
    CK(cudaMalloc(&L.rflag, sizeof(int) * NC));
    CK(cudaMalloc(&L.dlist[0], sizeof(int) * NC));
    CK(cudaMalloc(&L.dlist[1], sizeof(int) * NC));
    CK(cudaMalloc(&L.rlist, sizeof(int) * NC));
    CK(cudaMalloc(&L.slot, sizeof(int) * NC * SLOT_CAP));
    CK(cudaMalloc(&L.slot_n, sizeof(int) * NC));
    CK(cudaMemsetAsync(L.slot_n, 0xFF, sizeof(int) * NC, c->stream));
    L.mcap = MLIST_CAP;
    CK(cudaMalloc(&L.mlist, sizeof(int) * 2 * (size_t)MLIST_CAP));
    CK(cudaMalloc(&L.dstamp, sizeof(int) * NC));
    CK(cudaMemsetAsync(L.dstamp, 0, sizeof(int) * NC, c->stream));
    CK(cudaMalloc(&c->rows.cand, sizeof(int) * N * (size_t)c->kc));
    CK(cudaMalloc(&c->rows.meta, sizeof(int) * N));
    CK(cudaMemsetAsync(c->rows.meta, 0, sizeof(int) * N, c->stream));
    CK(cudaMalloc(&c->rows.rank, sizeof(int) * N));
    CK(cudaMemsetAsync(c->rows.rank, 0, sizeof(int) * N, c->stream));
    c->rows.kc = c->kc;
    const bool mixed = c->precision == DEM_PREC_MIXED;
    for (int b = 0; b < 2; b++) {
      CK(cudaMalloc(&c->X[b], sizeof(double4) * N));
      CK(cudaMalloc(&c->v4[b], (mixed ? sizeof(float4) : sizeof(double4)) * N));
      CK(cudaMalloc(&c->w2[b], (mixed ? sizeof(float2) : sizeof(double2)) * N));
    }
    c->par = 0;
  }
  for (int b = 0; b < 2; b++) {
    int st = alloc_history(c, c->H[b], c->hcap);
    if (st) return st;
  }
  c->hcur = 0;
  if (c->precision == DEM_PREC_MIXED) {
    if (!mixed_alloc(c->M, c->ncap, c->params.n_walls, c->hcap))
      return fail(c, DEM_ERR_CUDA, "mixed alloc");
  }
  // host -> device (positions etc. are n x 3 rows)
  {
    int st = put_state_arrays(c, c->P, pos, vel, omega, acc, alpha);
    if (st) return st;
  }
  std::vector<int> ci(N, 0);
  std::vector<double> rr(N, 0.0);
  for (int i = 0; i < n; i++) {
    ci[i] = comp ? comp[i] : 0;
    rr[i] = radius ? radius[i] : sys_of(i).comp_radius[ci[i]];
  }
  if (!sid.empty()) {
    CK(cudaMalloc(&c->sysid, sizeof(int) * N));
    CK(cudaMemcpy(c->sysid, sid.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->comp, ci.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->radius, rr.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  CK(cudaMemsetAsync(c->cnt, 0, sizeof(Counters), c->stream));
  for (int k = 0; k < 5; k++) c->ringmap[k] = k;
  CK(cudaStreamSynchronize(c->stream));
  c->state_set = true;
  {
    int st = ensure_drag(c);
    if (st) return st;
  }
  c->cells_ready = false;
  sync_host_walls(c);  // walls keep their place; their motion restarts at Time = 0
  c->walls_moved = false;
  c->time = 0.0;
  return DEM_OK;
}

static int get_state_arrays(dem_ctx* c, const StateArrays& s, double* pos, double* vel,
                            double* omega, double* acc, double* alpha) {
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  const int n = c->n;
  if (n == 0) return DEM_OK;
  double* outs[5] = {pos, vel, omega, acc, alpha};
  double* const* src = &s.px;  // 15 consecutive pointers in StateArrays
  for (int a = 0; a < 5; a++) {
    if (!outs[a]) continue;
    double* stg = c->staging + (size_t)a * 3 * n;
    launch(c, "soa_to_rows", k_soa_to_rows, blocks_for(n, 256), 256, n,
           (const double*)src[3 * a], (const double*)src[3 * a + 1], (const double*)src[3 * a + 2],
           stg);
    CK(cudaMemcpyAsync(outs[a], stg, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return DEM_OK;
}

static int put_state_arrays(dem_ctx* c, const StateArrays& s, const double* pos,
                            const double* vel, const double* omega, const double* acc,
                            const double* alpha) {
  const int n = c->n;
  if (n == 0) return DEM_OK;
  const double* ins[5] = {pos, vel, omega, acc, alpha};
  double* const* dst = &s.px;
  for (int a = 0; a < 5; a++) {
    if (!ins[a]) continue;
    double* stg = c->staging + (size_t)a * 3 * n;
    CK(cudaMemcpyAsync(stg, ins[a], sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    launch(c, "rows_to_soa", k_rows_to_soa, blocks_for(n, 256), 256, n, (const double*)stg,
           dst[3 * a], dst[3 * a + 1], dst[3 * a + 2]);
  }
  CK(cudaStreamSynchronize(c->stream));
  return DEM_OK;
}

int dem_update_state(dem_ctx* c, const double* pos, const double* vel, const double* omega,
                     const double* acc, const double* alpha) {
  if (!c) return DEM_ERR_INVALID;
  {
    // positions and velocities only: a and alpha may stay where the
    // predictor left them
    int st_ = restore_order(c, acc || alpha);
    if (st_) return st_;
  }
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  // the Particle copies of the pass kernel are stale from here on
  if (c->prepared == 0) c->prepared = -1;
  return put_state_arrays(c, c->P, pos, vel, omega, acc, alpha);
}

int dem_timer_start(dem_ctx* c) {
  if (!c) return DEM_ERR_INVALID;
  for (auto& e : c->timer)
    if (!e) CK(cudaEventCreate(&e));
  CK(cudaEventRecord(c->timer[0], c->stream));
  return DEM_OK;
}

int dem_timer_stop(dem_ctx* c, double* ms) {
  if (!c || !ms || !c->timer[0]) return DEM_ERR_INVALID;
  CK(cudaEventRecord(c->timer[1], c->stream));
  CK(cudaEventSynchronize(c->timer[1]));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, c->timer[0], c->timer[1]));
  *ms = f;
  return DEM_OK;
}

int dem_get_state(dem_ctx* c, double* pos, double* vel, double* omega, double* acc,
                  double* alpha) {
  if (!c) return DEM_ERR_INVALID;
  {
    int st_ = restore_order(c, acc || alpha);
    if (st_) return st_;
  }
  return get_state_arrays(c, c->P, pos, vel, omega, acc, alpha);
}

int dem_get_predicted(dem_ctx* c, double* pos, double* vel, double* omega, double* acc,
                      double* alpha) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  return get_state_arrays(c, c->Pr, pos, vel, omega, acc, alpha);
}

int dem_get_n(dem_ctx* c, int32_t* n) {
  if (!c || !n) return DEM_ERR_INVALID;
  *n = c->n;
  return DEM_OK;
}

int dem_set_integration(dem_ctx* c, const double* previous, const int32_t* ipc) {
  if (!c || !previous || !ipc) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  size_t N = (size_t)std::max(c->n, 1);
  // logical slot k (ipc(k+1)) -> physical slot k; spare = nprev
  std::vector<double> tmp(9 * N * (c->nprev + 1), 0.0);
  for (int k = 0; k < c->nprev; k++) {
    int src = ipc[k] - 1;
    if (src < 0 || src >= c->nprev) return fail(c, DEM_ERR_INVALID, "bad ipc");
    for (int i = 0; i < c->n; i++)
      for (int d = 0; d < 9; d++)
        tmp[((size_t)k * 9 + d) * N + i] = previous[((size_t)src * c->n + i) * 9 + d];
  }
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(c->ring, tmp.data(), sizeof(double) * tmp.size(), cudaMemcpyHostToDevice));
  for (int k = 0; k < 5; k++) c->ringmap[k] = k;
  drop_graphs(c);
  return DEM_OK;
}

int dem_get_integration(dem_ctx* c, double* previous, int32_t* ipc) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  size_t N = (size_t)std::max(c->n, 1);
  std::vector<double> tmp(9 * N * (c->nprev + 1));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(tmp.data(), c->ring, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost));
  // exported in canonical form: physical slot k = logical ipc(k+1)
  for (int k = 0; k < c->nprev; k++) {
    if (ipc) ipc[k] = k + 1;
    if (previous) {
      int ph = c->ringmap[k];
      for (int i = 0; i < c->n; i++)
        for (int d = 0; d < 9; d++)
          previous[((size_t)k * c->n + i) * 9 + d] = tmp[((size_t)ph * 9 + d) * N + i];
    }
  }
  return DEM_OK;
}

int dem_set_contacts(dem_ctx* c, int64_t m, const int32_t* imin, const int32_t* imax,
                     const double* ft, const double* vt, int64_t mw, const int32_t* ip,
                     const int32_t* iw, const double* ftw, const double* vtw) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  const int n = c->n;
  size_t N = (size_t)std::max(n, 1);
  int nw = std::max(c->params.n_walls, 1);
  std::vector<int> cnt(N, 0);
  for (int64_t r = 0; r < m; r++) {
    // a partner past the last particle is a record that particle removal
    // left behind (never looked up again); the owner must exist
    if (imin[r] < 0 || imin[r] >= n || imin[r] >= imax[r])
      return fail(c, DEM_ERR_INVALID, "bad pair record (need 0 <= imin < n, imin < imax)");
    cnt[imin[r]]++;
  }
  int need = 0;
  for (int i = 0; i < n; i++) need = std::max(need, cnt[i]);
  CK(cudaStreamSynchronize(c->stream));
  if (need > c->hcap) {
    int st = grow_history(c, need);
    if (st) return st;
  }
  const int cap = c->hcap;
  const size_t S = (size_t)c->H[c->hcur].n;  // slot stride of the tables
  cnt.assign(S, 0);
  std::vector<int> key(S * cap, -1);
  std::vector<double2> val(S * cap * 3);
  // records kept sorted by partner as the reference lists are
  std::vector<int64_t> idx(m);
  for (int64_t r = 0; r < m; r++) idx[r] = r;
  std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
    return imin[a] != imin[b] ? imin[a] < imin[b] : imax[a] < imax[b];
  });
  for (int64_t q = 0; q < m; q++) {
    int64_t r = idx[q];
    int o = imin[r], k = cnt[o]++;
    key[(size_t)k * S + o] = imax[r];  // slot major
    double2* v = &val[((size_t)k * S + o) * 3];
    v[0] = make_double2(ft[3 * r], ft[3 * r + 1]);
    v[1] = make_double2(ft[3 * r + 2], vt[3 * r]);
    v[2] = make_double2(vt[3 * r + 1], vt[3 * r + 2]);
  }
  std::vector<int> wf(N * nw, 0);
  std::vector<double2> wv(N * nw * 3);
  for (int64_t r = 0; r < mw; r++) {
    if (ip[r] < 0 || ip[r] >= n || iw[r] < 0 || iw[r] >= c->params.n_walls)
      return fail(c, DEM_ERR_INVALID, "bad wall record");
    size_t wi = (size_t)ip[r] * c->params.n_walls + iw[r];
    wf[wi] = 1;
    wv[wi * 3 + 0] = make_double2(ftw[3 * r], ftw[3 * r + 1]);
    wv[wi * 3 + 1] = make_double2(ftw[3 * r + 2], vtw[3 * r]);
    wv[wi * 3 + 2] = make_double2(vtw[3 * r + 1], vtw[3 * r + 2]);
  }
  History& H = c->H[c->hcur];
  CK(cudaMemcpy(H.cnt, cnt.data(), sizeof(int) * S, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(H.key, key.data(), sizeof(int) * key.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(H.val, val.data(), sizeof(double2) * val.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(H.wflag, wf.data(), sizeof(int) * wf.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(H.wval, wv.data(), sizeof(double2) * wv.size(), cudaMemcpyHostToDevice));
  if (c->precision == DEM_PREC_MIXED) mixed_import_history(c->M, H, n, c->params.n_walls, c->hcur, c->stream);
  drop_graphs(c);
  return DEM_OK;
}

namespace {
struct HostHist {
  std::vector<int> cnt, key, wf;
  std::vector<double2> val, wv;
};
int download_history(dem_ctx* c, HostHist& h) {
  int nw = std::max(c->params.n_walls, 1);
  History H = c->H[c->hcur];
  size_t N = (size_t)H.n;  // slot stride (the allocated capacity)
  if (c->precision == DEM_PREC_MIXED) {
    // the mixed path keeps FP32 records; export them widened
    H = c->H[c->hcur];
    mixed_export_history(c->M, H, c->n, c->params.n_walls, c->hcur, c->stream);
  }
  CK(cudaStreamSynchronize(c->stream));
  h.cnt.resize(N);
  h.key.resize(N * H.cap);
  h.val.resize(N * H.cap * 3);
  h.wf.resize(N * nw);
  h.wv.resize(N * nw * 3);
  CK(cudaMemcpy(h.cnt.data(), H.cnt, sizeof(int) * N, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.key.data(), H.key, sizeof(int) * h.key.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.val.data(), H.val, sizeof(double2) * h.val.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.wf.data(), H.wflag, sizeof(int) * h.wf.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.wv.data(), H.wval, sizeof(double2) * h.wv.size(), cudaMemcpyDeviceToHost));
  return DEM_OK;
}
}  // namespace

int dem_count_contacts(dem_ctx* c, int64_t* n_pair, int64_t* n_wall) {
  if (!c) return DEM_ERR_INVALID;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  HostHist h;
  int st = download_history(c, h);
  if (st) return st;
  int64_t a = 0, b = 0;
  for (int i = 0; i < c->n; i++) a += h.cnt[i];
  for (int i = 0; i < c->n * c->params.n_walls; i++) b += h.wf[i] != 0;
  if (n_pair) *n_pair = a;
  if (n_wall) *n_wall = b;
  return DEM_OK;
}

int dem_get_contacts(dem_ctx* c, int64_t cap, int32_t* imin, int32_t* imax, double* ft,
                     double* vt, int64_t capw, int32_t* ip, int32_t* iw, double* ftw,
                     double* vtw) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  HostHist h;
  int st = download_history(c, h);
  if (st) return st;
  const size_t N = (size_t)c->H[c->hcur].n;  // slot stride
  // a record sits with either particle of its pair: export it as the
  // reference's node (imin, imax), all nodes ordered by imin, then imax
  struct Rec {
    int lo, hi;
    size_t slot;
  };
  std::vector<Rec> recs;
  for (int i = 0; i < c->n; i++)
    for (int r = 0; r < h.cnt[i]; r++) {
      const size_t sl = (size_t)r * N + i;
      const int k = h.key[sl];
      recs.push_back(k < i ? Rec{k, i, sl} : Rec{i, k, sl});
    }
  std::sort(recs.begin(), recs.end(),
            [](const Rec& x, const Rec& y) { return x.lo != y.lo ? x.lo < y.lo : x.hi < y.hi; });
  if ((int64_t)recs.size() > cap) return fail(c, DEM_ERR_INVALID, "pair record buffer too small");
  int64_t a = 0, b = 0;
  for (const Rec& q : recs) {
    imin[a] = q.lo;
    imax[a] = q.hi;
    const double2* v = &h.val[q.slot * 3];
    ft[3 * a] = v[0].x; ft[3 * a + 1] = v[0].y; ft[3 * a + 2] = v[1].x;
    vt[3 * a] = v[1].y; vt[3 * a + 1] = v[2].x; vt[3 * a + 2] = v[2].y;
    a++;
  }
  for (int i = 0; i < c->n; i++)
    for (int w = 0; w < c->params.n_walls; w++) {
      size_t wi = (size_t)i * c->params.n_walls + w;
      if (!h.wf[wi]) continue;
      if (b >= capw) return fail(c, DEM_ERR_INVALID, "wall record buffer too small");
      ip[b] = i;
      iw[b] = w;
      const double2* v = &h.wv[wi * 3];
      ftw[3 * b] = v[0].x; ftw[3 * b + 1] = v[0].y; ftw[3 * b + 2] = v[1].x;
      vtw[3 * b] = v[1].y; vtw[3 * b + 1] = v[2].x; vtw[3 * b + 2] = v[2].y;
      b++;
    }
  return DEM_OK;
}

int dem_initialize_cell_distribution(dem_ctx* c) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  int st = init_cells(c);
  if (st) return st;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->cells_ready = true;
  return DEM_OK;
}

int dem_get_grid(dem_ctx* c, int32_t* nxyz) {
  if (!c || !nxyz) return DEM_ERR_INVALID;
  nxyz[0] = c->hp.nx;
  nxyz[1] = c->hp.ny;
  nxyz[2] = c->hp.nz;
  return DEM_OK;
}

int dem_get_cell_count(dem_ctx* c, int32_t* ncell) {
  if (!c || !ncell) return DEM_ERR_INVALID;
  *ncell = c->ncell_total;
  return DEM_OK;
}

int dem_get_cells(dem_ctx* c, int32_t* cell_index, int32_t* traversal, int32_t* cell_start) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  int st = validate_ready(c);
  if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  const int n = c->n, ncell = c->ncell_total;
  std::vector<int> cell((size_t)std::max(n, 1)), next((size_t)std::max(n, 1)), head((size_t)ncell);
  if (n > 0) {
    CK(cudaMemcpy(cell.data(), c->L.cell[c->par], sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(next.data(), c->L.next, sizeof(int) * n, cudaMemcpyDeviceToHost));
  }
  CK(cudaMemcpy(head.data(), c->L.head, sizeof(int) * ncell, cudaMemcpyDeviceToHost));
  if (cell_index && n > 0) std::memcpy(cell_index, cell.data(), sizeof(int) * n);
  // the lists in cell order = the traversal order of ComputeAccelerations
  int k = 0;
  for (int cc = 0; cc < ncell; cc++) {
    if (cell_start) cell_start[cc] = k;
    for (int q = head[cc], guard = 0; q != -1; q = next[q]) {
      if (++guard > n || q < 0 || q >= n || k >= n)
        return fail(c, DEM_ERR_STATE, "cell lists inconsistent");
      if (traversal) traversal[k] = q;
      k++;
    }
  }
  if (cell_start) cell_start[ncell] = k;
  if (k != n) return fail(c, DEM_ERR_STATE, "cell lists do not hold every particle");
  return DEM_OK;
}

// ReadCellDistribution (src/MForces.f90:121-131): CellIndex from the
// positions, then the lists as stored (ReadCellStructure, src/MCells.f90:
// 988-1026), so that a resumed run walks the cells in the order the saved run
// would have.  The lists must hold every particle once, in its own cell.
int dem_set_cells(dem_ctx* c, const int32_t* traversal, const int32_t* cell_start) {
  if (!c || !traversal || !cell_start) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  const int n = c->n, ncell = c->ncell_total;
  if (cell_start[0] != 0 || cell_start[ncell] != n)
    return fail(c, DEM_ERR_INVALID, "cell_start must run from 0 to n");
  drop_graphs(c);
  c->cells_ready = false;
  int st = init_cells(c);  // CellIndex, flags and counters as a fresh distribution
  if (st) return st;
  std::vector<int> cell((size_t)std::max(n, 1));
  if (n > 0)
    CK(cudaMemcpyAsync(cell.data(), c->L.cell[c->par], sizeof(int) * n, cudaMemcpyDeviceToHost,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int> head((size_t)ncell, -1), next((size_t)std::max(n, 1), -1);
  std::vector<char> seen((size_t)std::max(n, 1), 0);
  for (int cc = 0; cc < ncell; cc++) {
    const int a = cell_start[cc], b = cell_start[cc + 1];
    if (b < a) return fail(c, DEM_ERR_INVALID, "cell_start decreases");
    for (int k = a; k < b; k++) {
      const int q = traversal[k];
      if (q < 0 || q >= n || seen[(size_t)q] || cell[(size_t)q] != cc)
        return fail(c, DEM_ERR_INVALID, "cell lists must hold every particle once, in its cell");
      seen[(size_t)q] = 1;
      next[(size_t)q] = k + 1 < b ? traversal[k + 1] : -1;
    }
    if (b > a) head[(size_t)cc] = traversal[a];
  }
  CK(cudaMemcpyAsync(c->L.head, head.data(), sizeof(int) * (size_t)ncell, cudaMemcpyHostToDevice,
                     c->stream));
  if (n > 0)
    CK(cudaMemcpyAsync(c->L.next, next.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  refresh_slots(c);
  c->cells_ready = true;
  return DEM_OK;
}

// Ncol as read from a state file (ReadState, src/DEM.f90:1109)
int dem_set_ncol(dem_ctx* c, int64_t ncol) {
  if (!c || ncol < 0) return DEM_ERR_INVALID;
  CK(cudaStreamSynchronize(c->stream));
  const unsigned long long v[2] = {(unsigned long long)ncol, 0ull};  // ncol, ncol_pending
  CK(cudaMemcpy(&c->cnt->ncol, v, sizeof(v), cudaMemcpyHostToDevice));
  c->hcnt->ncol = v[0];
  c->hcnt->ncol_pending = 0;
  return DEM_OK;
}

int dem_compute_accelerations(dem_ctx* c, int32_t use_predicted, double time_step,
                              int32_t update) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  st = force_pass(c, use_predicted ? 1 : 0, update != 0, time_step, EPI_STORE, current_map(c),
                  true, 0);
  if (st) return st;
  CK(cudaGetLastError());
  st = read_counters(c);
  return st;
}

// ComputeAccelerations with its Force and Torque arrays (src/MForces.f90:154,
// summed at :319-320 and divided at :330-333) copied out as rows of three.
// The pass kernel writes them into the host I/O staging buffer, which holds
// 15 doubles per particle.
int dem_compute_forces(dem_ctx* c, int32_t use_predicted, double time_step, int32_t update,
                       double* force, double* torque) {
  if (!c || !force || !torque) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  int st = validate_ready(c);
  if (st) return st;
  c->force_out = c->staging;
  st = force_pass(c, use_predicted ? 1 : 0, update != 0, time_step, EPI_STORE, current_map(c),
                  true, 0);
  c->force_out = nullptr;
  if (st) return st;
  CK(cudaGetLastError());
  st = read_counters(c);
  if (st) return st;
  const size_t n3 = (size_t)3 * c->n;
  if (n3 == 0) return DEM_OK;
  CK(cudaMemcpyAsync(force, c->staging, sizeof(double) * n3, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(torque, c->staging + n3, sizeof(double) * n3, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DEM_OK;
}

int dem_move_particles(dem_ctx* c, int32_t step) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  st = move_particles_impl(c, step, true, 0);
  if (st) return st;
  CK(cudaGetLastError());
  return read_counters(c);
}

int dem_move_particles_euler(dem_ctx* c) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  st = move_particles_euler_impl(c);
  if (st) return st;
  return read_counters(c);
}

// The main loop.  Steps are replayed from CUDA graphs of G = 4 steps (the
// period of the ring rotation (<= 4 slots) and of the history double buffer);
// every kernel in a graph first checks the abort word.  Before each replay
// the history tables are grown if the last updating pass came within
// HEADROOM records of the capacity.  If a pass inside a replay still
// overflows, it records its step index and every later kernel of the replay
// does nothing: the host advances its bookkeeping to that step, grows the
// tables and re-runs that step synchronously (the failed pass is re-runnable:
// it only wrote fresh outputs).
int dem_run(dem_ctx* c, int32_t first_step, int32_t last_step) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  int s0 = first_step;
  // the main loop calls UpdateParticleList after every step (src/DEM.f90:96),
  // the Euler start-up does not
  const bool removal = c->removal && c->nsys == 1;
  c->stop_on_escape = removal;
  // fresh: the host mirror of the counters was read after the last pass
  auto remove_escaped = [&](bool fresh = false) -> int {
    if (!removal) return DEM_OK;
    if (!fresh) {
      int s = read_counters(c);
      if (s) return s;
    }
    return c->hcnt->escaped ? update_particle_list_impl(c, nullptr) : DEM_OK;
  };
  if (first_step == 1) {
    for (int s = 1; s <= c->params.method_order - 1; s++) {
      st = move_particles_euler_impl(c);
      if (st) return st;
    }
    s0 = c->params.method_order;
  } else {
    st = remove_escaped();  // escapes left by a step run through another call
    if (st) return st;
  }
  int step = s0;
  const int G = 4;
  const int HEADROOM = 2;
  const double dt = c->params.time_step;
  int poured_step = s0 - 1;
  while (step <= last_step) {
    int remaining = last_step - step + 1;
    // PouringAttempt(Step) (src/DEM.f90:95, 115-123); a chunk holds no other
    // pouring step, so those steps run one at a time
    bool pour_inside = false;
    if (pour_active(c)) {
      if (step % c->pour.interval == 0 && poured_step != step) {
        st = pour_particle_impl(c, nullptr);
        if (st) return st;
      }
      for (int k = 1; k < G; k++)
        if ((step + k) % c->pour.interval == 0) pour_inside = true;
    }
    poured_step = step;
    // the storage back into cell order every reorder_every steps
    if (c->reorder_every > 0 && !c->slab && c->since_reorder >= c->reorder_every) {
      st = reorder_by_cell(c);
      if (st) return st;
      c->since_reorder = 0;
    }
    if (remaining < G || c->prof || pour_inside) {
      st = move_particles_impl(c, step, true, 0);
      if (st) return st;
      st = remove_escaped();
      if (st) return st;
      step++;
      c->since_reorder++;
      continue;
    }
    st = read_counters(c);
    if (st) return st;
    if (c->hcnt->need_capacity + HEADROOM > c->hcap) {
      st = grow_history(c, c->hcnt->need_capacity + HEADROOM);
      if (st) return st;
    }
    if (c->hcnt->need_in + HEADROOM > c->in_cap) {
      st = grow_incoming(c, c->hcnt->need_in + HEADROOM);
      if (st) return st;
    }
    if (c->hcnt->need_cl + c->hcnt->need_cl / 16 > c->cl_cap) {
      st = grow_contacts(c, c->hcnt->need_cl + c->hcnt->need_cl / 8);
      if (st) return st;
    }
    // a graph starts from prepared Particle copies
    if (c->prepared != 0) {
      st = prepare_side(c, 0);
      if (st) return st;
    }
    // one graph (or recorded persistent chunk) per rotation phase (ring
    // spare slot, history parity, list parity)
    int phase = (c->nprev > 0 ? c->ringmap[c->nprev] : 0) * 4 + c->hcur * 2 + c->par;
    if (chunk_persistent(c)) {
      if (!c->prog[phase]) {
        st = record_chunk(c, G, phase);
        if (st) return st;
      }
      st = launch_chunk(c, phase);
      if (st) return st;
    } else {
      if (!c->graph_valid) {
        for (auto& g : c->graph) g = nullptr;
        c->graph_valid = true;
      }
      if (!c->graph[phase]) {
        st = capture_steps(c, G, &c->graph[phase]);
        if (st) return st;
      }
      fill_wall_slots(c, step, G);  // the previous replay has completed
      CK(cudaGraphLaunch(c->graph[phase], c->stream));
      c->launches += c->graph_kernels;
    }
    st = read_counters(c);
    if (st) return st;
    if (c->hcnt->barrier_timeout) {
      // the chunk stopped part-way: the barrier words and flags are reset,
      // the state is left as it is and must be set again
      CK(cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned), c->stream));
      CK(cudaMemsetAsync(&c->cnt->barrier_timeout, 0, sizeof(int), c->stream));
      CK(cudaMemsetAsync(&c->cnt->abort, 0, 2 * sizeof(int), c->stream));  // abort, abort_tag
      CK(cudaStreamSynchronize(c->stream));
      c->cells_ready = false;
      drop_graphs(c);
      return fail(c, DEM_ERR_STATE,
                  "persistent chunk: a grid-wide barrier timed out; the state is part-way "
                  "through the chunk (set it again)");
    }
    int done = G, failed_pass = -1;
    bool escape_stop = false;
    if (c->hcnt->abort) {
      const int tag = c->hcnt->abort_tag - 1;  // 2*(step in chunk) + pass
      if (c->hcnt->nonfinite) return fail(c, DEM_ERR_STATE, "a particle position is not finite");
      if (c->hcnt->list_error) return fail(c, DEM_ERR_STATE, "cell lists inconsistent");
      if (tag < 0 || tag >= 2 * G) return fail(c, DEM_ERR_STATE, "bad abort tag");
      done = tag / 2;
      escape_stop = c->hcnt->escape_stop != 0;
      // an escape stop happens before the step starts: nothing to finish
      failed_pass = escape_stop ? -1 : tag % 2;
    }
    for (int k = 0; k < done; k++) {
      abm_rotate(c);
      c->hcur ^= 1;
    }
    if (done > 0) {
      c->prepared = 0;
      c->last_side = 1;
    }
    step += done;
    c->since_reorder += done;
    c->time = (double)(step - 1) * dt;
    if (escape_stop) {
      // the replay's later wall copies ran: back to the walls of step-1
      st = apply_walls(c, 0);
      if (st) return st;
      CK(cudaMemsetAsync(&c->cnt->abort, 0, 2 * sizeof(int), c->stream));  // abort, abort_tag
      CK(cudaMemsetAsync(&c->cnt->escape_stop, 0, sizeof(int), c->stream));
      st = update_particle_list_impl(c, nullptr);
      if (st) return st;
      continue;
    }
    if (failed_pass >= 0) {
      // the replay's later wall uploads ran: back to the walls of step-1
      st = apply_walls(c, 0);
      if (st) return st;
      // the failed step: its first pass ran up to the failure (relink done),
      // or its first pass completed and its second one failed
      c->par ^= 1;
      if (failed_pass == 0) {
        RingMap rm = current_map(c);
        st = finish_pass(c, 0, true, dt, EPI_PREDICT, rm, 0);
        if (st) return st;
        c->last_side = 0;
        c->prepared = 1;
        c->hcur ^= 1;
        abm_rotate(c);
        c->time = (double)step * dt;
        st = apply_walls(c, 0);
        if (st) return st;
        rm = current_map(c);
        st = force_pass(c, 1, false, dt, EPI_CORRECT, rm, true, 1);
        if (st) return st;
      } else {
        c->last_side = 0;
        c->prepared = 1;
        c->hcur ^= 1;
        abm_rotate(c);
        c->time = (double)step * dt;
        st = apply_walls(c, 0);
        if (st) return st;
        c->par ^= 1;
        RingMap rm = current_map(c);
        st = finish_pass(c, 1, false, dt, EPI_CORRECT, rm, 1);
        if (st) return st;
        c->last_side = 1;
        c->prepared = 0;
      }
      step++;
    }
    st = remove_escaped(failed_pass < 0);  // escapes of the chunk's last step
    if (st) return st;
  }
  CK(cudaGetLastError());
  return DEM_OK;
}

int dem_run_timed(dem_ctx* c, int32_t first_step, int32_t last_step, double* device_ms) {
  if (!c || !device_ms) return DEM_ERR_INVALID;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaEventRecord(e0, c->stream));
  int st = dem_run(c, first_step, last_step);
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *device_ms = ms;
  return st;
}

int dem_get_ncol(dem_ctx* c, int64_t* ncol) {
  if (!c || !ncol) return DEM_ERR_INVALID;
  int st = read_counters(c);
  if (st) return st;
  // the last history-updating pass completed (no abort is pending after an
  // API call returns), so its count is part of Ncol
  *ncol = (int64_t)(c->hcnt->ncol + c->hcnt->ncol_pending);
  return DEM_OK;
}

int dem_set_fluid(dem_ctx* c, const dem_fluid* f) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  drop_graphs(c);
  if (!f) {
    c->fluid = false;
    return DEM_OK;
  }
  if (c->nsys > 1 || c->pp)
    return fail(c, DEM_ERR_UNSUPPORTED, "fluid flow needs one system with a component table");
  if (f->levels < 1 || !(f->viscosity > 0.0))
    return fail(c, DEM_ERR_INVALID, "fluid: NL >= 1 and a positive viscosity");
  // InitializeFluid (src/mFluid.f90:72-92)
  FluidArgs& F = c->fa;
  F.levels = f->levels;
  F.area = c->params.lbox[0] * c->params.lbox[1];
  F.dz = c->params.lbox[2] / (double)f->levels;
  F.vf0 = f->flow_rate / F.area;
  F.h2 = c->params.lbox[2] / 2.0;
  F.density = f->density;
  F.viscosity = f->viscosity;
  for (int k = 0; k < NCM; k++) {
    F.comp_density[k] = f->comp_density[k];
    F.comp_radius[k] = c->params.comp_radius[k];
  }
  cudaFree(c->fl_vf);
  c->fl_vf = nullptr;
  CK(cudaMalloc(&c->fl_vf, sizeof(double) * 2 * (size_t)(f->levels + 1)));
  c->fluid = true;
  return ensure_drag(c);
}

int dem_set_pouring(dem_ctx* c, const dem_pouring* p) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!p) {
    c->pouring = false;
    drop_graphs(c);
    return DEM_OK;
  }
  if (c->nsys > 1 || c->pp)
    return fail(c, DEM_ERR_UNSUPPORTED, "pouring needs one system with a component table");
  if (p->interval < 1 || p->max_attempts < 0 ||
      (p->shape != DEM_POUR_RECTANGLE && p->shape != DEM_POUR_CIRCLE))
    return fail(c, DEM_ERR_INVALID, "pouring: interval >= 1, attempts >= 0, known shape");
  for (int k = 0; k < c->params.n_components; k++)
    if (p->target_number[k] < 0) return fail(c, DEM_ERR_INVALID, "negative target number");
  c->pour = *p;
  c->pouring = true;
  drop_graphs(c);
  if (c->state_set) {
    const int need = pour_capacity(c, c->comp_count, c->n);
    if (need > c->ncap) return grow_capacity(c, need);
  }
  return DEM_OK;
}

int dem_pour_particle(dem_ctx* c, int32_t* inserted) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  return pour_particle_impl(c, inserted);
}

int dem_set_rng(dem_ctx* c, const dem_rng* r) {
  if (!c || !r) return DEM_ERR_INVALID;
  c->rng = *r;
  return DEM_OK;
}

int dem_get_rng(dem_ctx* c, dem_rng* r) {
  if (!c || !r) return DEM_ERR_INVALID;
  *r = c->rng;
  return DEM_OK;
}

int dem_update_particle_list(dem_ctx* c, int64_t* removed) {
  if (!c) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  return update_particle_list_impl(c, removed);
}

int dem_set_particle_removal(dem_ctx* c, int32_t enable) {
  if (!c) return DEM_ERR_INVALID;
  if (enable && c->nsys > 1)
    return fail(c, DEM_ERR_UNSUPPORTED, "particle removal needs a single-system context");
  c->removal = enable != 0;
  drop_graphs(c);
  return DEM_OK;
}

int dem_get_components(dem_ctx* c, int32_t* comp) {
  if (!c || !comp) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  CK(cudaStreamSynchronize(c->stream));
  if (c->n > 0) CK(cudaMemcpy(comp, c->comp, sizeof(int) * (size_t)c->n, cudaMemcpyDeviceToHost));
  return DEM_OK;
}

int dem_get_removal_stats(dem_ctx* c, int64_t* stats) {
  if (!c || !stats) return DEM_ERR_INVALID;
  for (int k = 0; k < 3; k++) stats[k] = c->rm_stats[k];
  return DEM_OK;
}

int dem_set_wall_motion(dem_ctx* c, const dem_wall_motion* motion) {
  if (!c) return DEM_ERR_INVALID;
  if (c->nsys > 1) return fail(c, DEM_ERR_UNSUPPORTED, "moving walls need a single-system context");
  drop_graphs(c);
  sync_host_walls(c);  // walls stay where the last motion left them
  c->walls_moved = false;
  if (!motion) {
    c->wm.clear();
    return DEM_OK;
  }
  const int nw = c->params.n_walls;
  for (int j = 0; j < nw; j++)
    for (int k = 0; k < 3; k++) {
      const dem_wall_motion& m = motion[j];
      if (!std::isfinite(m.constant_factor[k]) || !std::isfinite(m.amplitude[k]) ||
          !std::isfinite(m.velocity_amplitude[k]) || !std::isfinite(m.two_pi_frequency[k]) ||
          !std::isfinite(m.phase_angle[k]) || m.two_pi_frequency[k] < 0.0)
        return fail(c, DEM_ERR_INVALID, "wall motion must be finite with frequency >= 0");
    }
  if (!c->wall_slots) CK(cudaMallocHost(&c->wall_slots, sizeof(dem_wall) * NWM * 5));
  c->wm.assign(motion, motion + nw);
  return DEM_OK;
}

int dem_get_walls(dem_ctx* c, dem_wall* walls) {
  if (!c || !walls) return DEM_ERR_INVALID;
  sync_host_walls(c);
  for (int j = 0; j < c->params.n_walls; j++) walls[j] = c->hsys[0].walls[j];
  return DEM_OK;
}

int dem_get_escaped(dem_ctx* c, int64_t* count) {
  if (!c || !count) return DEM_ERR_INVALID;
  int st = read_counters(c);
  if (st) return st;
  *count = (int64_t)c->hcnt->escaped;
  return DEM_OK;
}

}  // extern "C"

namespace {

// Area of a wall that the spheres of a box can press on: a rectangle's
// extent along each in-plane axis (the box axis it runs along) up to the box
// length there, or a cone's lateral area.
double wall_area(const dem_wall& W, const double* L) {
  auto axis = [](const double* v) {
    int k = 0;
    for (int j = 1; j < 3; j++)
      if (std::fabs(v[j]) > std::fabs(v[k])) k = j;
    return k;
  };
  if (W.shape == DEM_WALL_RECTANGLE)
    return std::min(2.0 * W.l1, L[axis(W.u)]) * std::min(2.0 * W.l2, L[axis(W.w)]);
  if (W.shape == DEM_WALL_CONE) {
    const double len = 2.0 * W.l1, dr = W.l3 - W.l2;
    return 3.14159265358979323846 * (W.l2 + W.l3) * std::sqrt(len * len + dr * dr);
  }
  return 0.0;
}

// Solid volume and region volume of one system (see dem_observables): the
// bed's lower 0.8*H for a system with gravity along -z and no periodicity
// in z, else the whole box.  Returns whether the system has a bed (h = H).
bool solid_fraction(const dem_params& q, const double* z, const double* R, int n,
                    double& solid, double& region, double& h) {
  const double pi = 3.14159265358979323846;
  solid = 0.0;
  h = 0.0;
  if (!(q.gravity[2] < 0.0) || q.pbc[2] || n == 0) {
    for (int i = 0; i < n; i++) solid += 4.0 / 3.0 * pi * R[i] * R[i] * R[i];
    region = n ? q.lbox[0] * q.lbox[1] * q.lbox[2] : 0.0;
    return false;
  }
  double base = -0.5 * q.lbox[2];
  bool floor = false;
  for (int w = 0; w < q.n_walls; w++) {
    const dem_wall& W = q.walls[w];
    if (W.shape == DEM_WALL_RECTANGLE && std::fabs(W.n[2]) > 0.99 &&
        (!floor || W.position[2] < base)) {
      base = W.position[2];
      floor = true;
    }
  }
  double mean = 0.0;
  for (int i = 0; i < n; i++) mean += z[i] - base;
  h = 2.0 * (mean / n);
  const double top = 0.8 * h;
  for (int i = 0; i < n; i++)
    if (z[i] - base < top) solid += 4.0 / 3.0 * pi * R[i] * R[i] * R[i];
  region = q.lbox[0] * q.lbox[1] * top;
  return true;
}

}  // namespace

extern "C" {

int dem_get_observables(dem_ctx* c, dem_observables* o) {
  if (!c || !o) return DEM_ERR_INVALID;
  if (!c->state_set) return fail(c, DEM_ERR_STATE, "no state");
  std::memset(o, 0, sizeof(*o));
  const int grid = 148 * 4;
  if (c->n > 0) {
    if (c->pp)
      launch(c, "observables", k_observables<true>, grid, 256, (const DevParams*)c->dp,
             (const int*)c->sysid, c->n, c->P,
             (const double*)c->radius, (const int*)c->comp, c->obs_partial);
    else
      launch(c, "observables", k_observables<false>, grid, 256, (const DevParams*)c->dp,
             (const int*)c->sysid, c->n,
             c->P, (const double*)c->radius, (const int*)c->comp, c->obs_partial);
  }
  std::vector<double> part((size_t)grid * 8, 0.0);
  CK(cudaStreamSynchronize(c->stream));
  if (c->n > 0)
    CK(cudaMemcpy(part.data(), c->obs_partial, sizeof(double) * part.size(), cudaMemcpyDeviceToHost));
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < grid; b++)
    for (int k = 0; k < 8; k++) acc[k] += part[(size_t)b * 8 + k];
  o->kinetic_energy = 0.5 * acc[0];
  o->potential_energy = acc[1];
  o->momentum[0] = acc[3];
  o->momentum[1] = acc[4];
  o->momentum[2] = acc[5];
  // solid fraction (bed or whole box) and bed height, per system, in index
  // order on the host
  {
    std::vector<double> z((size_t)std::max(c->n, 1)), rad((size_t)std::max(c->n, 1));
    if (c->n > 0) {
      CK(cudaMemcpy(z.data(), c->P.pz, sizeof(double) * c->n, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(rad.data(), c->radius, sizeof(double) * c->n, cudaMemcpyDeviceToHost));
    }
    double solid = 0.0, region = 0.0, hsum = 0.0;
    int nbed = 0;
    for (int s = 0, off = 0; s < c->nsys; s++) {
      const int cnt = c->nsys > 1 ? c->counts[(size_t)s] : c->n;
      const dem_params& q = c->sys_params[(size_t)s];
      double so = 0.0, re = 0.0, h = 0.0;
      const bool bed = solid_fraction(q, z.data() + off, rad.data() + off, cnt, so, re, h);
      solid += so;
      region += re;
      if (bed) {
        hsum += h;
        nbed++;
      }
      off += cnt;
    }
    o->packing_fraction = region > 0.0 ? solid / region : 0.0;
    o->bed_height = nbed ? hsum / nbed : 0.0;
  }
  int64_t np = 0, nw = 0;
  int st = dem_count_contacts(c, &np, &nw);
  if (st) return st;
  o->n_pair_records = np;
  st = read_counters(c);
  if (st) return st;
  o->n_pair_contacts = (int64_t)c->hcnt->pair_contacts;
  o->n_wall_contacts = (int64_t)c->hcnt->wall_contacts;
  o->mean_coordination = c->n ? 2.0 * (double)o->n_pair_contacts / (double)c->n : 0.0;
  // wall normal forces of the last contact kernel: block sums in block order
  if (c->n > 0 && c->nw_max > 0) {
    const size_t nb = blocks_for(c->n, 128);
    std::vector<double> part(nb * NWM);
    CK(cudaMemcpy(part.data(), c->wall_part, sizeof(double) * part.size(),
                  cudaMemcpyDeviceToHost));
    for (size_t b = 0; b < nb; b++)
      for (int w = 0; w < c->nw_max; w++) o->wall_normal_force[w] += part[b * NWM + w];
  }
  for (int w = 0; w < c->nw_max; w++) {
    double area = 0.0;
    for (const dem_params& q : c->sys_params)
      if (w < q.n_walls) area += wall_area(q.walls[w], q.lbox);
    o->wall_pressure[w] = area > 0.0 ? o->wall_normal_force[w] / area : 0.0;
  }
  return DEM_OK;
}

int dem_set_profiling(dem_ctx* c, int32_t enable) {
  if (!c) return DEM_ERR_INVALID;
  resolve_events(c);
  c->prof = enable != 0;
  return DEM_OK;
}

int dem_get_kernel_stats(dem_ctx* c, int32_t idx, char* name, int32_t name_cap,
                         int64_t* launches, double* total_ms) {
  if (!c) return DEM_ERR_INVALID;
  resolve_events(c);
  if (idx < 0 || idx >= (int)c->stats.size()) return DEM_ERR_INVALID;
  if (name && name_cap > 0) {
    std::snprintf(name, (size_t)name_cap, "%s", c->stats[idx].name.c_str());
  }
  if (launches) *launches = c->stats[idx].launches;
  if (total_ms) *total_ms = c->stats[idx].total_ms;
  return DEM_OK;
}

int dem_reset_kernel_stats(dem_ctx* c) {
  if (!c) return DEM_ERR_INVALID;
  resolve_events(c);
  c->stats.clear();
  c->launches = 0;
  return DEM_OK;
}

int dem_get_launch_count(dem_ctx* c, int64_t* launches) {
  if (!c || !launches) return DEM_ERR_INVALID;
  *launches = c->launches;
  return DEM_OK;
}

int dem_get_stream(dem_ctx* c, void** stream) {
  if (!c || !stream) return DEM_ERR_INVALID;
  *stream = (void*)c->stream;
  return DEM_OK;
}

int dem_get_pass_stats(dem_ctx* c, int64_t* pair_contacts, int64_t* wall_contacts,
                       int64_t* movers, int32_t* hist_capacity) {
  if (!c) return DEM_ERR_INVALID;
  int st = read_counters(c);
  if (st) return st;
  if (pair_contacts) *pair_contacts = c->last_pairs;
  if (wall_contacts) *wall_contacts = c->last_walls;
  if (movers) *movers = c->last_movers;
  if (hist_capacity) *hist_capacity = c->hcap;
  return DEM_OK;
}

int dem_set_tuning(dem_ctx* c, double skin_factor, int32_t pass_variant) {
  if (!c) return DEM_ERR_INVALID;
  if (!(skin_factor > 0.0 && skin_factor <= 0.5) || pass_variant < 0 || pass_variant > 2)
    return fail(c, DEM_ERR_INVALID, "skin factor must lie in (0, 0.5], variant in {0, 1, 2}");
  CK(cudaStreamSynchronize(c->stream));
  if (skin_factor != c->skin_factor) {
    sync_host_walls(c);
    for (DevParams& h : c->hsys) {
      h.vl_skin = skin_factor * h.cutoff;
      h.vl_thr = 0.4 * h.vl_skin;
    }
    c->hp = c->hsys[0];
    CK(cudaMemcpy(c->dp, c->hsys.data(), sizeof(DevParams) * (size_t)c->nsys,
                  cudaMemcpyHostToDevice));
    // rows built with the old skin are rebuilt by the next pass
    const int one = 1;
    CK(cudaMemcpy(&c->cnt->force_full, &one, sizeof(int), cudaMemcpyHostToDevice));
    c->skin_factor = skin_factor;
  }
  if (pass_variant != c->pass_variant) {
    c->pass_variant = pass_variant;
    drop_graphs(c);
  }
  return DEM_OK;
}

int dem_get_tuning(dem_ctx* c, double* skin_factor, int32_t* pass_variant) {
  if (!c) return DEM_ERR_INVALID;
  if (skin_factor) *skin_factor = c->skin_factor;
  if (pass_variant) *pass_variant = c->pass_variant;
  return DEM_OK;
}

int dem_set_launch_shape(dem_ctx* c, int32_t launch_mode, int32_t test_block,
                         int32_t particles_per_thread, int32_t pair_waves) {
  if (!c) return DEM_ERR_INVALID;
  auto one_of = [](int v, int a, int b, int d) { return v == a || v == b || v == d; };
  if ((launch_mode != 0 && launch_mode != 1) || !one_of(test_block, 64, 128, 256) ||
      !one_of(particles_per_thread, 1, 2, 4) || !one_of(pair_waves, 1, 2, 4))
    return fail(c, DEM_ERR_INVALID,
                "launch shape: mode in {0, 1}, test_block in {64, 128, 256}, "
                "particles_per_thread in {1, 2, 4}, pair_waves in {1, 2, 4}");
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  if (launch_mode != c->launch_mode || test_block != c->test_block ||
      particles_per_thread != c->ppt || pair_waves != c->pair_waves)
    drop_graphs(c);
  c->launch_mode = launch_mode;
  c->test_block = test_block;
  c->ppt = particles_per_thread;
  c->pair_waves = pair_waves;
  return DEM_OK;
}

int dem_set_early_launch(dem_ctx* c, int32_t on) {
  if (!c) return DEM_ERR_INVALID;
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  if ((on != 0) != (c->early_launch != 0)) drop_graphs(c);
  c->early_launch = on != 0;
  return DEM_OK;
}

int dem_get_early_launch(dem_ctx* c, int32_t* on) {
  if (!c) return DEM_ERR_INVALID;
  if (on) *on = c->early_launch;
  return DEM_OK;
}

int dem_get_launch_shape(dem_ctx* c, int32_t* launch_mode, int32_t* test_block,
                         int32_t* particles_per_thread, int32_t* pair_waves) {
  if (!c) return DEM_ERR_INVALID;
  if (launch_mode) *launch_mode = c->launch_mode;
  if (test_block) *test_block = c->test_block;
  if (particles_per_thread) *particles_per_thread = c->ppt;
  if (pair_waves) *pair_waves = c->pair_waves;
  return DEM_OK;
}

int dem_set_persistent_barrier(dem_ctx* c, double timeout_ms, int32_t extra_blocks) {
  if (!c) return DEM_ERR_INVALID;
  if (!(timeout_ms > 0.0 && timeout_ms <= 60000.0) || extra_blocks < 0 || extra_blocks > 1024)
    return fail(c, DEM_ERR_INVALID, "barrier timeout in (0, 60000] ms, extra blocks in [0, 1024]");
  c->bar_limit_ns = (unsigned long long)(timeout_ms * 1e6);
  c->bar_extra = extra_blocks;
  return DEM_OK;
}

int dem_get_persistent_blocks(dem_ctx* c, int32_t* blocks) {
  if (!c) return DEM_ERR_INVALID;
  if (blocks) *blocks = c->chunk_blocks;
  return DEM_OK;
}

int dem_autotune(dem_ctx* c, int32_t first_step, int32_t steps_per_trial, int32_t* last_step,
                 double* trial_ms) {
  if (!c || steps_per_trial < 4) return DEM_ERR_INVALID;
  int st = validate_ready(c);
  if (st) return st;
  const double skins[3] = {0.025, 0.05, 0.1};
  const int timed_steps = (steps_per_trial + 3) / 4 * 4;  // whole chunks
  int step = first_step;
  double best_ms = 1e300;
  // one trial: an untimed chunk takes the graph capture (or the chunk's
  // recording) and the forced full rebuild, then the timed steps
  auto trial = [&](int t, double& ms) -> int {
    int s2 = dem_run(c, step, step + 3);
    if (s2) return s2;
    step += 4;
    s2 = dem_run_timed(c, step, step + timed_steps - 1, &ms);
    if (s2) return s2;
    step += timed_steps;
    if (trial_ms) trial_ms[t] = ms;
    return DEM_OK;
  };
  int mode = 0, tb = 128, ppt = 1, waves = 2;
  st = dem_set_launch_shape(c, mode, tb, ppt, waves);
  if (st) return st;
  // skin x pair variant
  int best = 0;
  for (int t = 0; t < 9; t++) {
    st = dem_set_tuning(c, skins[t / 3], t % 3);
    if (st) return st;
    double ms = 0.0;
    st = trial(t, ms);
    if (st) return st;
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  st = dem_set_tuning(c, skins[best / 3], best % 3);
  if (st) return st;
  // then one launch-shape knob at a time
  struct Knob {
    int* var;
    int values[2];
  } knobs[3] = {{&ppt, {2, 4}}, {&tb, {64, 256}}, {&waves, {1, 4}}};
  int t = 9;
  for (const Knob& k : knobs) {
    const int keep = *k.var;
    int chosen = keep;
    for (int v : k.values) {
      *k.var = v;
      st = dem_set_launch_shape(c, mode, tb, ppt, waves);
      if (st) return st;
      double ms = 0.0;
      st = trial(t++, ms);
      if (st) return st;
      if (ms < best_ms) {
        best_ms = ms;
        chosen = v;
      }
    }
    *k.var = chosen;
  }
  // persistent chunks
  st = dem_set_launch_shape(c, 1, tb, ppt, waves);
  if (st) return st;
  if (chunk_persistent(c)) {
    double ms = 0.0;
    st = trial(t, ms);
    if (st) return st;
    if (ms < best_ms) {
      best_ms = ms;
      mode = 1;
    }
  } else if (trial_ms) {
    trial_ms[t] = -1.0;
  }
  st = dem_set_launch_shape(c, mode, tb, ppt, waves);
  if (st) return st;
  if (last_step) *last_step = step - 1;
  return DEM_OK;
}

int dem_slab_set_range(dem_ctx* c, int32_t z0, int32_t z1) {
  if (!c) return DEM_ERR_INVALID;
  RESTORE_ORDER;
  int st = validate_ready(c);
  if (st) return st;
  if (c->nsys != 1 || c->fluid || !c->wm.empty() || c->pouring)
    return fail(c, DEM_ERR_INVALID,
                "slab: one system without fluid drag, wall motion or pouring");
  const int nz = slab_nz(c);
  if (z0 < 0 || z1 > nz || z0 >= z1)
    return fail(c, DEM_ERR_INVALID, "slab: the layers must satisfy 0 <= z0 < z1 <= Nz");
  if (z1 - z0 < 2 && !(z0 == 0 && z1 == nz))
    return fail(c, DEM_ERR_INVALID, "slab: a slab holds at least two cell layers");
  CK(cudaStreamSynchronize(c->stream));
  DevParams& h = c->hsys[0];
  h.slab_c0 = h.coff + z0 * slab_nxy(c);
  h.slab_c1 = h.coff + z1 * slab_nxy(c);
  c->hp = h;
  CK(cudaMemcpy(c->dp, c->hsys.data(), sizeof(DevParams), cudaMemcpyHostToDevice));
  c->slab = !(z0 == 0 && z1 == nz);
  c->slab_z0 = z0;
  c->slab_z1 = z1;
  c->removal = false;  // particles leave a slab for its neighbour, not the system
  if (!c->gstamp) {
    CK(cudaMalloc(&c->gstamp, sizeof(int) * (size_t)std::max(c->ncap, 1)));
    CK(cudaMalloc(&c->slab_list, sizeof(int) * (size_t)std::max(c->ncap, slab_nxy(c))));
    CK(cudaMalloc(&c->slab_ghosts, sizeof(int) * (size_t)std::max(c->ncap, 1)));
    CK(cudaMalloc(&c->slab_count, sizeof(int) * 4));
  }
  CK(cudaMemset(c->gstamp, 0xFF, sizeof(int) * (size_t)std::max(c->ncap, 1)));
  c->n_ghosts = 0;
  drop_graphs(c);
  // room for the "j" results a slab receives as well as its own: the
  // exchange cannot grow it in the middle of a pass
  return grow_incoming(c, 16);
}

int dem_slab_phase(dem_ctx* c, int32_t step, int32_t pass, int32_t phase) {
  if (!c) return DEM_ERR_INVALID;
  if (!c->slab && !(c->slab_z1 > c->slab_z0))
    return fail(c, DEM_ERR_STATE, "slab: dem_slab_set_range first");
  if (pass < 0 || pass > 1 || phase < 0 || phase > 3)
    return fail(c, DEM_ERR_INVALID, "slab: pass in {0, 1}, phase in 0..3");
  const int side = pass;
  const bool update = pass == 0;
  const int epi = pass == 0 ? EPI_PREDICT : EPI_CORRECT;
  const double dt = c->params.time_step;
  int st = DEM_OK;
  switch (phase) {
    case DEM_SLAB_RELINK:
      st = ensure_drag(c);
      if (st) return st;
      c->slab_rm = current_map(c);
      if (c->prepared != side) {
        st = prepare_side(c, side);
        if (st) return st;
      }
      c->gepoch++;
      c->n_ghosts = 0;
      pass_lists(c, side, update, pass);
      break;
    case DEM_SLAB_TEST_PAIR:
      launch_pass_kernel(c, side, update, dt, epi, c->slab_rm, pass, 1);
      break;
    case DEM_SLAB_FOLD:
      launch_pass_kernel(c, side, update, dt, epi, c->slab_rm, pass, 2);
      break;
    default: {  // DEM_SLAB_FINISH
      st = read_counters(c);
      if (st) return st;
      const Counters& h = *c->hcnt;
      if (h.abort) {
        if (h.nonfinite) return fail(c, DEM_ERR_STATE, "a particle position is not finite");
        if (h.list_error) return fail(c, DEM_ERR_STATE, "cell lists inconsistent");
        return fail(c, DEM_ERR_CAPACITY,
                    "slab: a table overflowed in the pass (reserve more room: history "
                    "capacity, incoming results, rows)");
      }
      c->last_side = side;
      c->prepared = epi == EPI_PREDICT ? 1 : 0;
      if (update) c->hcur ^= 1;
      if (pass == 0) {
        abm_rotate(c);
        c->time = (double)step * dt;
        st = apply_walls(c, 0);
        if (st) return st;
      }
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "slab phase");
  return DEM_OK;
}

int dem_slab_pack(dem_ctx* c, int32_t what, void* buf, int64_t cap, int64_t* bytes) {
  if (!c || !buf || !bytes) return DEM_ERR_INVALID;
  if (!c->slab) return fail(c, DEM_ERR_STATE, "slab: dem_slab_set_range first");
  int count = 0;
  int st = DEM_OK;
  std::vector<int> extra;
  switch (what) {
    case DEM_SLAB_GHOSTS: {
      // this slab's bottom layer, for the slab below: its cells' lists,
      // the stamps of the layer below it (the receiver's top layer), and
      // its particles' pass data
      if (!slab_has_down(c)) return slab_write(c, what, slab_cols_begin(), 0, {}, buf, cap, bytes);
      const int nxy = slab_nxy(c);
      const int cb = slab_layer(c, c->slab_z0), cr = slab_layer(c, c->slab_z0 - 1);
      extra.resize(2 + 2 * (size_t)nxy);
      extra[0] = cb;
      CK(cudaMemcpyAsync(extra.data() + 2, c->L.head + cb, sizeof(int) * nxy,
                         cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(extra.data() + 2 + nxy, c->L.rflag + cr, sizeof(int) * nxy,
                         cudaMemcpyDeviceToHost, c->stream));
      st = slab_list_layer(c, c->slab_z0, &count);
      if (st) return st;
      // the records carry as many history slots as the fullest table needs
      int hrows = 0;
      st = slab_max_over(c, count, c->H[c->hcur].cnt, &hrows);
      if (st) return st;
      extra[1] = hrows;
      return slab_write(c, what, slab_ghost_cols(c, c->prepared, hrows), count, extra, buf, cap,
                        bytes);
    }
    case DEM_SLAB_LOWER: {
      // the cells of this slab's top layer's particles, for the slab above
      if (!slab_has_up(c)) return slab_write(c, what, slab_cols_begin(), 0, {}, buf, cap, bytes);
      st = slab_list_layer(c, c->slab_z1 - 1, &count);
      if (st) return st;
      SlabCols C = slab_cols_begin();
      slab_col(C, c->L.cell[c->par], 4, 1, 0);
      extra.push_back(slab_layer(c, c->slab_z1 - 1));
      return slab_write(c, what, C, count, extra, buf, cap, bytes);
    }
    case DEM_SLAB_JHALVES: {
      // the "j" results and matched bits of the ghosts received this pass,
      // for their owner (the slab above)
      const int rec = (int)in_rec_bytes(c);
      // as many result slots as the ghost with the most results
      int slots = 0;
      if (c->n_ghosts > 0) {
        CK(cudaMemcpyAsync(c->slab_list, c->slab_ghosts, sizeof(int) * (size_t)c->n_ghosts,
                           cudaMemcpyDeviceToDevice, c->stream));
        int st2 = slab_max_over(c, c->n_ghosts, c->in_cnt, &slots);
        if (st2) return st2;
        slots = std::min(slots, c->in_cap);
      }
      const int64_t item = SLAB_ID + (int64_t)slots * rec;
      const int64_t total = SLAB_HEAD + 16 + (int64_t)c->n_ghosts * item;
      *bytes = total;
      if (total > cap) return fail(c, DEM_ERR_CAPACITY, "slab: the exchange buffer is too small");
      int h[8] = {what, c->n_ghosts, (int)item, 4, slots, rec, 0, 0};
      CK(cudaMemcpyAsync(buf, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
      launch(c, "slab_jhalf_pack", k_slab_jhalf_pack, blocks_for(c->n_ghosts, 128), 128,
             (const int*)c->slab_ghosts, c->n_ghosts, c->in_cnt, (const char*)c->in_rec,
             slots, c->pass_cap, rec, c->matched, (char*)buf + SLAB_HEAD + 16);
      CK(cudaStreamSynchronize(c->stream));
      return DEM_OK;
    }
    case DEM_SLAB_MIGRATE_UP:
    case DEM_SLAB_MIGRATE_DOWN: {
      // the particles that entered the layer just above (below) this slab
      const bool up = what == DEM_SLAB_MIGRATE_UP;
      if (!(up ? slab_has_up(c) : slab_has_down(c)))
        return slab_write(c, what, slab_cols_begin(), 0, {}, buf, cap, bytes);
      const int nxy = slab_nxy(c);
      const int tu = slab_layer(c, c->slab_z1), td = slab_layer(c, c->slab_z0 - 1);
      const int t0 = up ? tu : td, u0 = up ? td : tu;
      const int b = c->par ^ 1;  // the next assignment
      CK(cudaMemsetAsync(c->slab_count, 0, 2 * sizeof(int), c->stream));
      launch(c, "slab_leavers", k_slab_leavers, blocks_for(c->n, 256), 256, c->n,
             (const int*)c->L.cell[c->par], (const int*)c->L.cell[b], c->hsys[0].slab_c0,
             c->hsys[0].slab_c1, t0, t0 + nxy, (slab_has_up(c) && slab_has_down(c)) ? u0 : 0,
             (slab_has_up(c) && slab_has_down(c)) ? u0 + nxy : 0, c->slab_list, c->slab_count,
             c->ncap, c->slab_count + 1);
      int hc[2];
      CK(cudaMemcpyAsync(hc, c->slab_count, sizeof(hc), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (hc[1] == 2)
        return fail(c, DEM_ERR_STATE, "slab: a particle moved more than one cell layer in a pass");
      if (hc[1]) return fail(c, DEM_ERR_STATE, "slab: leaver list overflow");
      count = hc[0];
      st = slab_write(c, what, slab_full_cols(c), count, {}, buf, cap, bytes);
      if (st) return st;
      // handed on: both cell entries name the cell it entered
      launch(c, "slab_depart", k_slab_depart, blocks_for(count, 128), 128,
             (const int*)c->slab_list, count, c->L.cell[c->par], (const int*)c->L.cell[b]);
      CK(cudaStreamSynchronize(c->stream));
      return DEM_OK;
    }
    default:
      return fail(c, DEM_ERR_INVALID, "slab: unknown exchange");
  }
}

int dem_slab_unpack(dem_ctx* c, int32_t what, const void* buf, int64_t bytes) {
  if (!c || !buf) return DEM_ERR_INVALID;
  if (!c->slab) return fail(c, DEM_ERR_STATE, "slab: dem_slab_set_range first");
  std::vector<int> h;
  int64_t body = 0;
  int st = slab_read_head(c, buf, bytes, what, h, &body);
  if (st) return st;
  const int count = h[1], rec = h[2];
  const char* recs = (const char*)buf + body;
  switch (what) {
    case DEM_SLAB_GHOSTS: {
      if (count == 0 && h[3] == 0) return DEM_OK;
      const int nxy = slab_nxy(c);
      if (h[3] != 2 + 2 * nxy || h[4] != slab_layer(c, c->slab_z1))
        return fail(c, DEM_ERR_INVALID, "slab: ghosts from a slab that is not the one above");
      const int* ex = h.data() + 4;
      const SlabCols C = slab_ghost_cols(c, c->prepared, ex[1]);
      if (rec != C.rec) return fail(c, DEM_ERR_INVALID, "slab: ghosts with another layout");
      CK(cudaMemcpyAsync(c->L.head + ex[0], ex + 2, sizeof(int) * nxy, cudaMemcpyHostToDevice,
                         c->stream));
      // stamps: rows of this slab's top layer whose neighbourhood changed
      CK(cudaMemcpyAsync(c->slab_list, ex + 2 + nxy, sizeof(int) * nxy, cudaMemcpyHostToDevice,
                         c->stream));
      launch(c, "slab_max", k_slab_max, blocks_for(nxy, 256), 256,
             c->L.rflag + slab_layer(c, c->slab_z1 - 1), (const int*)c->slab_list, nxy);
      if (count > 0) {
        const long long thr = (long long)count * (rec / 4);
        launch(c, "slab_cols", k_slab_cols, (unsigned)((thr + 255) / 256), 256, C,
               (const int*)nullptr, count, (char*)recs, c->gstamp, c->gepoch, c->slab_ghosts);
      }
      // the ghost cells' slots from the lists just received
      launch(c, "cell_slots", k_cell_slots, blocks_for(nxy, 256), 256, c->L, ex[0], nxy, c->n);
      c->n_ghosts = count;
      break;
    }
    case DEM_SLAB_LOWER: {
      if (count == 0) return DEM_OK;
      SlabCols C = slab_cols_begin();
      slab_col(C, c->L.cell[c->par], 4, 1, 0);
      if (h[3] != 1 || h[4] != slab_layer(c, c->slab_z0 - 1) || rec != C.rec)
        return fail(c, DEM_ERR_INVALID, "slab: cells from a slab that is not the one below");
      const long long thr = (long long)count * (rec / 4);
      launch(c, "slab_cols", k_slab_cols, (unsigned)((thr + 255) / 256), 256, C,
             (const int*)nullptr, count, (char*)recs, c->gstamp, c->gepoch, (int*)nullptr);
      break;
    }
    case DEM_SLAB_JHALVES: {
      if (count == 0) return DEM_OK;
      const int slots = h[4], r = h[5];
      if (r != (int)in_rec_bytes(c) || slots > c->in_cap || rec != SLAB_ID + slots * r)
        return fail(c, DEM_ERR_INVALID, "slab: results from a slab with another layout");
      launch(c, "slab_jhalf_unpack", k_slab_jhalf_unpack, blocks_for(count, 128), 128, recs,
             count, c->in_cnt, (char*)c->in_rec, c->in_cap, slots, c->pass_cap, r, c->matched,
             c->cnt);
      break;
    }
    case DEM_SLAB_MIGRATE_UP:
    case DEM_SLAB_MIGRATE_DOWN: {
      if (count == 0) return DEM_OK;
      const SlabCols C = slab_full_cols(c);
      if (rec != C.rec) return fail(c, DEM_ERR_INVALID, "slab: particles with another layout");
      const long long thr = (long long)count * (rec / 4);
      launch(c, "slab_cols", k_slab_cols, (unsigned)((thr + 255) / 256), 256, C,
             (const int*)nullptr, count, (char*)recs, (int*)nullptr, 0, c->slab_list);
      launch(c, "slab_arrive", k_slab_arrive, blocks_for(count, 128), 128,
             (const int*)c->slab_list, count, c->L, c->cnt, c->par, c->par ^ 1);
      break;
    }
    default:
      return fail(c, DEM_ERR_INVALID, "slab: unknown exchange");
  }
  CK(cudaStreamSynchronize(c->stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "slab unpack");
  return DEM_OK;
}

int dem_slab_displacement(dem_ctx* c, uint32_t* bits_out, const uint32_t* bits_in) {
  if (!c) return DEM_ERR_INVALID;
  CK(cudaStreamSynchronize(c->stream));
  if (bits_out) CK(cudaMemcpy(bits_out, &c->cnt->disp_max, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (bits_in) CK(cudaMemcpy(&c->cnt->disp_max, bits_in, sizeof(uint32_t), cudaMemcpyHostToDevice));
  return DEM_OK;
}

int dem_slab_owned(dem_ctx* c, int32_t* owned) {
  if (!c || !owned) return DEM_ERR_INVALID;
  if (!c->cells_ready) return fail(c, DEM_ERR_STATE, "cell distribution not initialised");
  std::vector<int> cell((size_t)c->n);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(cell.data(), c->L.cell[c->par], sizeof(int) * (size_t)c->n,
                cudaMemcpyDeviceToHost));
  const int c0 = c->hsys[0].slab_c0, c1 = c->hsys[0].slab_c1;
  for (int i = 0; i < c->n; i++) owned[i] = cell[(size_t)i] >= c0 && cell[(size_t)i] < c1;
  return DEM_OK;
}

int dem_set_reorder(dem_ctx* c, int32_t every_steps) {
  if (!c) return DEM_ERR_INVALID;
  if (every_steps < 0) return fail(c, DEM_ERR_INVALID, "reorder: steps must be >= 0");
  if (every_steps > 0 && c->slab)
    return fail(c, DEM_ERR_INVALID, "reorder: a slab keeps the system's own order");
  RESTORE_ORDER;
  c->reorder_every = every_steps;
  c->since_reorder = every_steps;  // the next dem_run starts with a reorder
  return DEM_OK;
}

int dem_get_reorder(dem_ctx* c, int32_t* every_steps, int64_t* reorders) {
  if (!c) return DEM_ERR_INVALID;
  if (every_steps) *every_steps = c->reorder_every;
  if (reorders) *reorders = c->reorders;
  return DEM_OK;
}

int dem_get_row_stats(dem_ctx* c, int64_t* candidates, int32_t* row_capacity) {
  if (!c) return DEM_ERR_INVALID;
  if (row_capacity) *row_capacity = c->kc;
  if (candidates) {
    *candidates = 0;
    if (c->state_set && c->n > 0) {
      std::vector<int> meta((size_t)c->n);
      CK(cudaStreamSynchronize(c->stream));
      CK(cudaMemcpy(meta.data(), c->rows.meta, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
      int64_t t = 0;
      for (int m : meta) t += m & META_MASK;
      *candidates = t;
    }
  }
  return DEM_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free cell distribution (dem_distribute_particles_noalloc).
//
// For callers that may not allocate device memory: the working memory of the
// counting sort lives in one file-scope device array of fixed size instead
// of per-context buffers.  Host code only ever sees the array's host-side
// stand-in symbol, which is not a device address; every call looks the
// device address up on the current device with cudaGetSymbolAddress (a
// host-side query), so no address outlives a device reset or belongs to
// another context.

namespace {

constexpr int NA_MAXN = DEM_NOALLOC_MAX_PARTICLES;
constexpr int NA_MAXC = DEM_NOALLOC_MAX_CELLS;
constexpr int NA_TILES = (NA_MAXC + SCAN_TILE - 1) / SCAN_TILE;

struct NoAllocScratch {
  DevParams params;
  Counters counters;
  int cell_cnt[NA_MAXC];
  int bsum[NA_TILES + 1];
  int a_cell[NA_MAXN];
  int a_loc[NA_MAXN];
  int a_orig[NA_MAXN];
  int t_orig[NA_MAXN];
  int slot_cell[NA_MAXN];
  unsigned a_key[NA_MAXN];
  unsigned t_key[NA_MAXN];
  double px[NA_MAXN];
  double py[NA_MAXN];
  double pz[NA_MAXN];
};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

extern "C" int dem_distribute_particles_noalloc(const dem_params* p, int32_t n,
                                                const double* d_pos, int32_t* d_cell_index,
                                                int32_t* d_traversal, int32_t* d_cell_start,
                                                int32_t* ncell_out, void* stream, char* err,
                                                int32_t err_cap) {
  auto say = [&](int code, const char* msg) {
    if (err && err_cap > 0) std::snprintf(err, (size_t)err_cap, "%s", msg);
    return code;
  };
  if (!p || n < 0) return say(DEM_ERR_INVALID, "null parameters or negative n");
  if (n > NA_MAXN) {
    char m[160];
    std::snprintf(m, sizeof(m),
                  "n = %d exceeds DEM_NOALLOC_MAX_PARTICLES = %d (use a context instead)", n,
                  NA_MAXN);
    return say(DEM_ERR_CAPACITY, m);
  }
  if (n > 0 && (!d_pos || !d_cell_index || !d_traversal)) return say(DEM_ERR_INVALID, "null array");
  if (!d_cell_start) return say(DEM_ERR_INVALID, "null cell_start");
  // cell grid: InitCellStructure3D (src/MCells.f90:155-227), CutOff = 2*max R
  double rmax = 0.0;
  if (p->n_components > 0) {
    if (p->n_components > NCM) return say(DEM_ERR_INVALID, "too many components");
    for (int i = 0; i < p->n_components; i++) rmax = std::max(rmax, p->comp_radius[i]);
  } else {
    rmax = p->pp_rmax;
  }
  const double CutOff = 2.0 * rmax;
  if (!(CutOff > 0.0)) return say(DEM_ERR_INVALID, "radius must be positive");
  const int MaxNCell = p->max_ncell > 0 ? p->max_ncell : 30000;
  const double Lx = p->lbox[0], Ly = p->lbox[1], Lz = p->lbox[2];
  const int Nx4 = (int)(Lx / CutOff), Ny4 = (int)(Ly / CutOff), Nz4 = (int)(Lz / CutOff);
  int N[3];
  if ((long long)Nx4 * Ny4 * Nz4 > MaxNCell) {
    const double LCell = std::pow(Lx * Ly * Lz / (double)MaxNCell, 1.0 / 3.0);
    N[0] = (int)(Lx / LCell);
    N[1] = (int)(Ly / LCell);
    N[2] = (int)(Lz / LCell);
  } else {
    N[0] = Nx4;
    N[1] = Ny4;
    N[2] = Nz4;
  }
  for (int k = 0; k < 3; k++) {
    if (N[k] < 1) return say(DEM_ERR_INVALID, "box smaller than one cell");
    if (p->pbc[k] && N[k] < 3)
      return say(DEM_ERR_UNSUPPORTED, "fewer than 3 cells along a periodic axis");
  }
  const long long ncell_ll = (long long)N[0] * N[1] * N[2];
  if (ncell_ll > NA_MAXC) {
    char m[160];
    std::snprintf(m, sizeof(m),
                  "%lld cells exceed DEM_NOALLOC_MAX_CELLS = %d (use a context instead)",
                  ncell_ll, NA_MAXC);
    return say(DEM_ERR_CAPACITY, m);
  }
  const int ncell = (int)ncell_ll;
  if (ncell_out) *ncell_out = ncell;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return say(DEM_ERR_NO_DEVICE, "no usable CUDA device");
  }
  // the array's device address on the current device (the first call on a
  // device also loads the device code there)
  void* base = nullptr;
  {
    cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (e != cudaSuccess || !base) {
      cudaGetLastError();
      return say(DEM_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
  }
  NoAllocScratch* S = (NoAllocScratch*)base;  // device addresses only
  DevParams* dp = &S->params;
  Counters* cnt = &S->counters;
  cudaStream_t st = (cudaStream_t)stream;

  DevParams h{};
  h.nx = N[0];
  h.ny = N[1];
  h.nz = N[2];
  h.ncell = ncell;
  h.nxbylx = (double)N[0] / Lx;
  h.nybyly = (double)N[1] / Ly;
  h.nzbylz = (double)N[2] / Lz;
  h.nxby2 = (double)N[0] * 0.5;
  h.nyby2 = (double)N[1] * 0.5;
  h.nzby2 = (double)N[2] * 0.5;
  for (int k = 0; k < 3; k++) h.pbc[k] = p->pbc[k] ? 1 : 0;

  // the array keeps the previous call's contents: reset what must start at 0
  cudaError_t e = cudaMemcpyAsync(dp, &h, sizeof(DevParams), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(Counters), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(S->cell_cnt, 0, sizeof(int) * (size_t)ncell, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return say(DEM_ERR_CUDA, cudaGetErrorString(e));
  }
  const int ntiles = (ncell + SCAN_TILE - 1) / SCAN_TILE;
  if (n > 0) {
    k_rows_to_soa<<<blocks_for(n, 256), 256, 0, st>>>(n, d_pos, S->px, S->py, S->pz);
    // DistributeParticles3D: every particle enters its cell in index order
    k_assign<<<blocks_for(n, 256), 256, 0, st>>>(dp, nullptr, n, 1, S->px, S->py, S->pz, d_traversal,
                                                   S->slot_cell, S->cell_cnt, S->a_cell, S->a_loc,
                                                   S->a_key, S->a_orig, cnt);
  }
  k_scan_tiles<<<ntiles, SCAN_THREADS, 0, st>>>(S->cell_cnt, ncell, d_cell_start, S->bsum, cnt);
  k_scan_bsums<<<1, SCAN_THREADS, 0, st>>>(S->bsum, ntiles, d_cell_start, ncell, cnt);
  k_scan_add<<<blocks_for(ncell, 256), 256, 0, st>>>(d_cell_start, ncell, S->bsum, cnt);
  if (n > 0) {
    k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(n, S->a_cell, S->a_loc, S->a_key, S->a_orig,
                                                   d_cell_start, S->t_key, S->t_orig, cnt);
    k_cellsort<<<blocks_for(ncell, 128), 128, 0, st>>>(ncell, d_cell_start, S->t_key, S->t_orig,
                                                        d_traversal, S->slot_cell, d_cell_index,
                                                        cnt);
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return say(DEM_ERR_CUDA, cudaGetErrorString(e));
  return DEM_OK;
}
