// dem_test.cuh -- the precision-independent parts of a force pass: the
// relink of the cell lists, the candidate rows and the exact overlap test.
// Both translation units include them (the FP64 one, compiled with IEEE
// square root, and the mixed one, compiled with approximate division and
// square root), so every floating-point operation here is written with an
// explicitly rounded intrinsic (__dadd_rn, __dsub_rn, __dmul_rn,
// __dsqrt_rn), which no compiler flag changes: the candidate rows and the
// contact lists are the same bits in either unit, and equal to the
// reference's (src/MForces.f90:218-224 tests DeltaDijSq = MinDijSq - DijSq
// > 0 in FP64).
#pragma once
#include "dem_pass.cuh"

namespace dem {

// min_image_exact, sumsq3 and the pair's MinDijSq with every operation
// rounded on its own (no contraction into fused multiply-adds)
__device__ __forceinline__ double min_image_rn(double r, const Box& B, int k) {
  if (B.pbc[k] && !(fabs(r) < B.half_lim[k]))
    r = __dsub_rn(r, __dmul_rn(B.lbox[k], (double)(int)round(__dmul_rn(r, B.inv_lbox[k]))));
  return r;
}
__device__ __forceinline__ double sumsq3_rn(const double a[3]) {
  double c = 0.0;
  c = __dadd_rn(c, __dmul_rn(a[0], a[0]));
  c = __dadd_rn(c, __dmul_rn(a[1], a[1]));
  c = __dadd_rn(c, __dmul_rn(a[2], a[2]));
  return c;
}
// MinDijSq of a pair: the material table (components ca, cb), or (Ra + Rb)^2
// for per-particle radii (PP)
template <bool PP>
__device__ __forceinline__ double min_dij_sq_rn(const DevParams& P, int ca, double Ra, int cb,
                                                double Rb) {
  if (PP) {
    const double d = __dadd_rn(Ra, Rb);
    return __dmul_rn(d, d);
  }
  return P.min_dij_sq[ca * NCM + cb];
}

// Copy cell c's list into its slots (the first SLOT_CAP entries) and record
// its length; a walk longer than n (corrupt links) records -1.
__device__ __forceinline__ void copy_slots(const CellLists& L, int c, int first, int n) {
  int k = 0;
  for (int q = first; q != -1; q = L.next[q]) {
    if (k >= n) {
      k = -1;
      break;
    }
    if (k < SLOT_CAP) L.slot[(size_t)c * SLOT_CAP + k] = q;
    k++;
  }
  L.slot_n[c] = k;
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
  // (the status words, the dirty-cell count and the pass number requested
  // together)
  const int abort0 = cnt->abort;
  const unsigned long long escaped = cnt->escaped;
  const int m = cnt->n_dirty[par];
  const int stamp = cnt->pass_id + 1;  // fold kernels advance pass_id, not this one
  if (abort0) return;
  // inside a captured chunk, particles that left the box in the last step
  // stop the chunk before this step (the host runs UpdateParticleList); the
  // count is final here (written by the previous kernel), so every block
  // takes the same branch
  if (stop_tag >= 0 && escaped != 0ull) {
    if (tid == 0) {
      cnt->escape_stop = 1;
      set_abort(cnt, stop_tag);
    }
    return;
  }
  if (tid == 0) {
    const DevParams& P = PT[0];  // the integrator settings are shared
    cnt->n_repair = 0;
    cnt->n_mlist[(stamp & 1) ^ 1] = 0;  // for the next pass's relink
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
  const int* __restrict__ cell_new = L.cell[par];
  // a particle that leaves or enters a cell, for the test kernel's row check
  auto record = [&](int x) {
    const int k = atomicAdd(&cnt->n_mlist[stamp & 1], 1);
    if (k < L.mcap) L.mlist[(size_t)(stamp & 1) * L.mcap + k] = x;
  };
  for (int i = tid; i < m; i += nthreads) {
    const int c = L.dlist[par][i];
    const DevParams& P = sys_params(PT, cellsys, c);
    if (!in_slab(P, c)) {
      // a cell another slab advances (a particle of this slab left for it):
      // its list here is not kept; only the transition is forgotten
      for (int a = L.arr_head[c], g2 = 0; a != -1 && g2 < n; a = L.arr_next[a], g2++)
        L.mflag[a] = 0;
      L.arr_head[c] = -1;
      L.dflag[c] = 0;
      continue;
    }
    // 1. unlink the leavers.  The old list is in the cell's slots when it
    // fits there (independent loads); else it is walked link by link (a
    // leaver's successor saved when it moved: its own link may be rewritten
    // by the thread of the cell it entered)
    int prev = -1, first = -1;
    int guard = 0;
    const int len = L.slot_n[c];
    const bool from_slots = len >= 0 && len <= SLOT_CAP;
    int old[SLOT_CAP];
    unsigned stay = 0u;  // bit k: old element k stays
    if (from_slots) {
      const int* sl = L.slot + (size_t)c * SLOT_CAP;
#pragma unroll 4
      for (int k = 0; k < len; k++) old[k] = sl[k];
#pragma unroll 4
      for (int k = 0; k < len; k++)
        if (cell_new[old[k]] == c) stay |= 1u << k;
      for (int k = 0; k < len; k++) {
        if (!((stay >> k) & 1u)) {
          record(old[k]);
          continue;
        }
        if (prev == -1) first = old[k];
        else L.next[prev] = old[k];
        prev = old[k];
      }
    } else {
      int q = L.head[c];
      while (q != -1) {
        if (++guard > n) {
          atomicExch(&cnt->list_error, 1);
          atomicExch(&cnt->abort, 1);
          return;
        }
        const bool stays = cell_new[q] == c;
        const int nq = stays ? L.next[q] : L.mnext[q];
        if (!stays) record(q);
        if (stays) {
          if (prev == -1) first = q;
          else L.next[prev] = q;
          prev = q;
        }
        q = nq;
      }
    }
    if (prev != -1) L.next[prev] = -1;
    // 2. prepend the arrivals, highest index first (the reference's index:
    // gid when the storage is in cell order)
    auto G = [&](int x) { return L.gid ? L.gid[x] : x; };
    int sh = -1, tail = -1, a = L.arr_head[c];
    guard = 0;
    while (a != -1) {
      if (++guard > n) {
        atomicExch(&cnt->list_error, 1);
        atomicExch(&cnt->abort, 1);
        return;
      }
      const int an = L.arr_next[a];  // (guard: arrivals so far)
      L.mflag[a] = 0;
      record(a);
      if (sh == -1) {
        sh = tail = a;
        L.next[a] = -1;
      } else if (G(a) > G(sh)) {
        L.next[a] = sh;
        sh = a;
      } else {
        int q2 = sh;
        for (int g2 = 0; L.next[q2] != -1 && G(L.next[q2]) > G(a) && g2 < guard; g2++)
          q2 = L.next[q2];
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
    L.dstamp[c] = stamp;
    if (from_slots) {
      // the new list's slots: the arrivals (this thread linked them), then
      // the stayers in their old order
      int k = 0;
      int x = sh;
      for (int t = 0; t < guard; t++) {
        if (k < SLOT_CAP) L.slot[(size_t)c * SLOT_CAP + k] = x;
        k++;
        x = L.next[x];
      }
      for (int j = 0; j < len; j++)
        if ((stay >> j) & 1u) {
          if (k < SLOT_CAP) L.slot[(size_t)c * SLOT_CAP + k] = old[j];
          k++;
        }
      L.slot_n[c] = k;
    } else {
      copy_slots(L, c, first, n);
    }
    // 3. the rows that read c are rebuilt in this pass (by the test
    // kernel): a row of a particle in cell b holds the rest of b's list and
    // the half-shell cells b + o, kx + Nx*(ky + Ny*kz) > 0, so c is read by
    // the rows of c itself and of c + o' for the 13 offsets o' with
    // kx + Nx*(ky + Ny*kz) < 0; those 14 cells are stamped with the pass
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int cl = c - P.coff;
    const int cx = cl % nx, cy = (cl / nx) % ny, cz = cl / (nx * ny);
#pragma unroll
    for (int o = 0; o < 14; o++) {
      const int jx = cx + o % 3 - 1, jy = cy + (o / 3) % 3 - 1, jz = cz + o / 9 - 1;
      const bool ok = (P.pbc[0] || (jx >= 0 && jx < nx)) && (P.pbc[1] || (jy >= 0 && jy < ny)) &&
                      (P.pbc[2] || (jz >= 0 && jz < nz));
      if (ok)
        L.rflag[P.coff + axis_wrap(jx, nx, P.pbc[0]) +
                nx * (axis_wrap(jy, ny, P.pbc[1]) + ny * axis_wrap(jz, nz, P.pbc[2]))] = stamp;
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
                                          const int* __restrict__ comp, const CellLists& L,
                                          const Rows& R, Counters* cnt, int tag) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int cl = c - P.coff;
  const int cx = cl % nx, cy = (cl / nx) % ny, cz = cl / (nx * ny);
  const double4 p4 = X[p];
  const int cp = PP ? 0 : comp[p];
  int cw = -1, order = 1 << 20;  // the lane's cell, its place in the row
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
      cw = c;
      order = 0;
      walk = true;
    } else if (ok && lex > 0) {
      cw = P.coff + w[0] + nx * (w[1] + ny * w[2]);
      order = 1 + (13 - lex);
      walk = true;
    }
  } else if (lane == 27) {
    cw = c;
  }
  const double skin = P.vl_skin;
  auto is_cand = [&](int q) -> bool {
    const double4 q4 = X[q];
    double Rij[3] = {__dsub_rn(q4.x, p4.x), __dsub_rn(q4.y, p4.y), __dsub_rn(q4.z, p4.z)};
#pragma unroll
    for (int k = 0; k < 3; k++) Rij[k] = min_image_rn(Rij[k], P.box, k);
    const double DijSq = sumsq3_rn(Rij);
    double md;
    if (PP) md = __dadd_rn(p4.w, q4.w);
    else md = __dsqrt_rn(min_dij_sq_rn<PP>(P, cp, p4.w, comp[q], q4.w));
    md = __dadd_rn(md, skin);
    return __dsub_rn(__dmul_rn(md, md), DijSq) > 0.0;
  };
  // the lane's cell read from its slots when its whole list is there
  // (independent loads), else by walking its links
  const int len = cw >= 0 ? L.slot_n[cw] : -1;
  const bool arr = len >= 0 && len <= SLOT_CAP;
  const int* sl = L.slot + (size_t)(cw >= 0 ? cw : 0) * SLOT_CAP;
  // pass 1: count the candidates; lane 13 (own cell after p) and lane 27
  // (p's rank: the list before p) first find p in its cell.  Slots: the hits
  // are a bit mask for pass 2; links: the first 8 elements and their test
  // results stay in registers for pass 2.
  int count = 0, walked = 0;
  unsigned hits = 0u;
  int cache[8];
  bool bad = false;
  int q = -1;
#pragma unroll
  for (int i = 0; i < 8; i++) cache[i] = -1;
  if (arr) {
    int k0 = 0;
    if (lane == 13 || lane == 27) {
      int r = 0;
      while (r < len && sl[r] != p) r++;
      if (r == len) bad = true;
      if (lane == 27) count = r;
      k0 = r + 1;
    }
    if (walk && !bad) {
#pragma unroll 4
      for (int k = k0; k < len; k++)
        if (is_cand(sl[k])) {
          hits |= 1u << k;
          count++;
        }
    }
  } else if (cw >= 0) {
    q = lane == 13 ? L.next[p] : L.head[cw];
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
          q = L.next[q];
        }
      }
    }
  }
  const int resume = q;  // (links) first element not cached (-1: none)
  if (!arr && cw >= 0) {
    int guard = 0;
    if (walk) {
      while (q != -1) {
        if (++guard > n) {
          bad = true;
          break;
        }
        if (is_cand(q)) count++;
        q = L.next[q];
      }
    } else if (lane == 27) {
      while (q != p) {
        if (q == -1 || ++guard > n) {
          bad = true;
          break;
        }
        count++;
        q = L.next[q];
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
  // pass 2: write (slots: the hits; links: the cached part, then the rest)
  if (walk) {
    int k = off;
    if (arr) {
      unsigned h = hits;
      while (h) {
        const int j = __ffs(h) - 1;
        h &= h - 1u;
        R.cand[(size_t)(k++) * n + p] = sl[j];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i < walked && ((hits >> i) & 1u)) R.cand[(size_t)(k++) * n + p] = cache[i];
      int q2 = resume;
      while (q2 != -1) {
        if (is_cand(q2)) R.cand[(size_t)(k++) * n + p] = q2;
        q2 = L.next[q2];
      }
    }
  }
  if (lane == 0) {
    R.meta[p] = m;
    R.rank[p] = rank;
  }
}


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
  // the cells whose particles are tested: [slab_c0, slab_c0 + slab_span)
  // (a slab of a decomposition, or every cell)
  int slab_c0;
  unsigned slab_span;
  // 1: a stamped row is rebuilt only when a particle that changed cell is
  // near it (row_stays); 0: every stamped row is rebuilt
  int fine;
};

// Whether the row of particle pl (cell cl), stamped because a cell it reads
// was relinked, can stay as it is; called by the whole warp together.  A
// relink keeps the stayers of a list in their order and puts the arrivals
// first, so the row changes only if a particle that left or entered one of
// those cells is within MinDij + skin of pl; one farther than that can come
// no closer than MinDij + 0.2 skin before the next full rebuild (every
// particle moves at most 0.4 skin in between), so a stale entry for it in
// the row is tested and rejected, and its absence changes no contact.  The
// lanes check the pass's movers 32 at a time (a margin errs towards
// rebuilding); when none is near, the row stays, and if pl's own cell was
// relinked its rank (its place in the list) is rewritten from the slots.
template <bool PP>
__device__ __forceinline__ bool row_stays(const TestArgs& A, int pl, int cl, const double4& p4,
                                          int cp, int stamp, int n, int lane) {
  const unsigned FULL = 0xffffffffu;
  const int b = stamp & 1;
  const int nm = A.cnt->n_mlist[b];
  if (nm > A.L.mcap) return false;
  const DevParams& P = sys_params(A.P, A.sysid, pl);
  const double skin = P.vl_skin;
  const int* ml = A.L.mlist + (size_t)b * A.L.mcap;
  bool near = false;
  for (int k = lane; k < nm && !near; k += 32) {
    const int q = ml[k];
    if ((unsigned)q >= (unsigned)n) {
      near = true;
      break;
    }
    const double4 q4 = A.X[q];
    double Rij[3] = {__dsub_rn(q4.x, p4.x), __dsub_rn(q4.y, p4.y), __dsub_rn(q4.z, p4.z)};
#pragma unroll
    for (int d = 0; d < 3; d++) Rij[d] = min_image_rn(Rij[d], P.box, d);
    const double DijSq = sumsq3_rn(Rij);
    double md;
    if (PP) md = __dadd_rn(p4.w, q4.w);
    else md = __dsqrt_rn(min_dij_sq_rn<PP>(P, cp, p4.w, A.comp[q], q4.w));
    md = __dadd_rn(__dadd_rn(md, skin), __dadd_rn(1.0e-9, __dmul_rn(1.0e-9, md)));
    if (!(__dsub_rn(__dmul_rn(md, md), DijSq) < 0.0)) near = true;
  }
  if (__any_sync(FULL, near)) return false;
  if (A.L.dstamp[cl] == stamp) {
    const int len = A.L.slot_n[cl];
    if (len < 0 || len > SLOT_CAP) return false;
    const bool hit = lane < len && A.L.slot[(size_t)cl * SLOT_CAP + lane] == pl;
    const unsigned h = __ballot_sync(FULL, hit);
    if (!h) return false;
    if (lane == 0) A.R.rank[pl] = __ffs(h) - 1;
  }
  return true;
}

// First, the candidate rows of the warp's particles that this pass rebuilds
// (every row on a full rebuild, else the rows of the particles whose cell the
// relink stamped with this pass) are built, one particle at a time by the
// whole warp (build_row).  Then every particle tests its row, and the block
// takes room for its contacts in the list with one atomic (two block
// barriers, which every thread of the block meets).  (The pass's contact
// count and the list length it needs come from the pair kernel, or from
// here when the list overflows.)
// (The body of k_test for block `vblock`, so that a persistent kernel can
// run it too.  NC: candidates read through the non-coherent path, which
// needs the rows unchanged for the whole launch except by the warp that
// reads them; a kernel that runs several passes reads them coherently.)
template <bool NC>
__device__ __forceinline__ int ld_row(const int* a) {
  return NC ? __ldg(a) : *a;
}

template <bool PP, bool NC = true>
__device__ __forceinline__ void test_body(const TestArgs& A, int vblock) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int p0 = vblock * blockDim.x + threadIdx.x;
  const bool valid0 = p0 < A.n;
  const int p = valid0 ? p0 : 0;
  const int n = A.n;
  // the abort word, the pass's rebuild decision, the particle's cell, own
  // data, row length and first candidates are requested together (the first
  // candidates before the row length is known: every row holds at least 4
  // entries' room); nothing is written once the abort word is seen (the
  // block still meets its barrier), and a warp whose rows were rebuilt reads
  // them again
  const bool live = A.cnt->abort == 0;
  const bool full = A.cnt->full_due != 0;
  const int stamp = A.cnt->pass_id + 1;
  const int cp0 = A.cell_cur[p];
  // (a slab of a decomposition tests only its own particles)
  const bool valid = valid0 && (unsigned)(cp0 - A.slab_c0) < A.slab_span;
  const double4 p4 = A.X[p];
  const int cp = PP ? 0 : A.comp[p];
  int q0[4];
#pragma unroll
  for (int u = 0; u < 4; u++) q0[u] = ld_row<NC>(A.cand + (size_t)u * n + p);
  int meta = A.meta[p];
  {
    bool stale = live && valid && (full || A.L.rflag[cp0] == stamp);
    if (!full && A.fine) {
      // the stamped rows checked against the pass's movers, one at a time
      // by the whole warp
      unsigned chk = __ballot_sync(FULL, stale);
      while (chk) {
        const int l = __ffs(chk) - 1;
        chk &= chk - 1u;
        const int pl = __shfl_sync(FULL, p, l);
        const int cl = __shfl_sync(FULL, cp0, l);
        const int cpl = __shfl_sync(FULL, cp, l);
        const double4 pl4 = make_double4(__shfl_sync(FULL, p4.x, l), __shfl_sync(FULL, p4.y, l),
                                         __shfl_sync(FULL, p4.z, l), __shfl_sync(FULL, p4.w, l));
        const bool keep = row_stays<PP>(A, pl, cl, pl4, cpl, stamp, n, lane);
        if (lane == l && keep) stale = false;
      }
    }
    unsigned todo = __ballot_sync(FULL, stale);
    if (todo) {
      while (todo) {
        const int l = __ffs(todo) - 1;
        todo &= todo - 1u;
        const int pl = __shfl_sync(FULL, p, l);
        const int cl = __shfl_sync(FULL, cp0, l);
        build_row<PP>(sys_params(A.P, A.sysid, pl), n, pl, cl, A.X, A.comp, A.L, A.R, A.cnt,
                      A.tag);
      }
      __syncwarp();  // the rows written by the warp are visible to their owners
#pragma unroll
      for (int u = 0; u < 4; u++) q0[u] = A.cand[(size_t)u * n + p];
      meta = A.meta[p];
    }
  }
  const DevParams& P = sys_params(A.P, A.sysid, p);
  const int m = live && valid ? (meta & META_MASK) : 0;
  // contact bit masks of the row, 64 candidates per window (windows past
  // the first only for rows longer than 64)
  unsigned long long mask0 = 0ull;
  unsigned long long more[(KC_MAX + 1) / 64 - 1];
  int total = 0;
  // the next group's candidates are requested with this group's positions:
  // one round trip per group of 4 after the first
  int qn[4];
#pragma unroll
  for (int u = 0; u < 4; u++) qn[u] = q0[u];
  for (int base = 0; base < m; base += 64) {
    unsigned long long mask = 0ull;
    const int end = m < base + 64 ? m : base + 64;
#pragma unroll 1
    for (int b = base; b < end; b += 4) {
      int q[4];
#pragma unroll
      for (int u = 0; u < 4; u++) q[u] = b + u < end ? qn[u] : -1;
#pragma unroll
      for (int u = 0; u < 4; u++)
        qn[u] = b + 4 + u < m ? ld_row<NC>(A.cand + (size_t)(b + 4 + u) * n + p) : -1;
      double4 xq[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        xq[u] = q[u] >= 0 ? A.X[q[u]] : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (q[u] < 0) continue;
        double Rij[3] = {__dsub_rn(xq[u].x, p4.x), __dsub_rn(xq[u].y, p4.y),
                         __dsub_rn(xq[u].z, p4.z)};
#pragma unroll
        for (int k = 0; k < 3; k++) Rij[k] = min_image_rn(Rij[k], P.box, k);
        const double DijSq = sumsq3_rn(Rij);
        const int cq = PP ? 0 : A.comp[q[u]];
        if (__dsub_rn(min_dij_sq_rn<PP>(P, cp, p4.w, cq, xq[u].w), DijSq) > 0.0)
          mask |= 1ull << (b + u - base);
      }
    }
    total += __popcll(mask);
    if (base == 0) mask0 = mask;
    else more[base / 64 - 1] = mask;
  }
  // one allocation per block (the warps' sums through shared memory, one
  // atomic on the pass's list length); a particle's contacts are contiguous
  int incl = total;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  __shared__ int s_wsum[8];  // blocks of at most 256 threads
  __shared__ int s_base;
  const int warp = threadIdx.x >> 5;
  if (lane == 31) s_wsum[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      const int t = s_wsum[w];
      s_wsum[w] = acc;
      acc += t;
    }
    s_base = acc > 0 ? atomicAdd(&A.cnt->n_contacts, acc) : 0;
  }
  __syncthreads();
  const int start = s_base + s_wsum[warp] + incl - total;
  if (live && valid) {
    A.cstart[p] = start;
    A.ccount[p] = total;
  }
  if (!live) return;
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
        A.clist[s++] = make_int2(p, ld_row<NC>(A.cand + (size_t)k * n + p));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent launches: a 4-step chunk (8 force passes) as one cooperative
// launch whose blocks step through every pass's phases (relink, test, pair,
// fold), separated by grid-wide barriers.

// Arguments of a relink (k_relink's parameters)
struct RelinkArgs {
  const DevParams* PT;
  const int* cellsys;
  CellLists L;
  int par, n, update, stop_tag;
  Counters* cnt;
};

// A grid-wide barrier over `expected` blocks (gridDim.x of a cooperative
// launch, so that every block is resident): an arrival counter and a
// generation word.  A block that waits longer than limit_ns nanoseconds
// (%globaltimer) sets cnt->barrier_timeout and cnt->abort and reports
// failure; its caller then returns, and the blocks still waiting give up in
// turn, so the launch always ends.
struct GridSync {
  unsigned* count;
  unsigned* gen;
  Counters* cnt;
  unsigned long long limit_ns;
  unsigned expected;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

// All threads of every block call; returns false after a timeout.  The
// block's thread 0 arrives with an acquire-release add (after the block
// barrier, so it releases the whole block's writes); the last to arrive
// resets the count and publishes the next generation with a release add;
// the others poll the generation with acquire loads.
__device__ __forceinline__ bool grid_sync(const GridSync& g) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned gen0 = ld_acquire_u32(g.gen);  // cannot advance before this block arrives
    unsigned prev;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;"
                 : "=r"(prev)
                 : "l"(g.count)
                 : "memory");
    if (prev == g.expected - 1u) {
      *(volatile unsigned*)g.count = 0u;
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.gen) : "memory");
    } else {
      const unsigned long long t0 = global_ns();
      while (ld_acquire_u32(g.gen) == gen0) {
        if (global_ns() - t0 > g.limit_ns) {
          atomicExch(&g.cnt->barrier_timeout, 1);
          atomicExch(&g.cnt->abort, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct NoView {};

// One force pass of a chunk: its relink, test and pass arguments, the
// integrator epilogue (EPI_PREDICT / EPI_CORRECT) and, for the mixed path,
// the FP32 record arrays it reads and writes.  16-byte aligned: blocks copy
// it into shared memory as int4.
template <class V4, class W2, class View>
struct alignas(16) ChunkPass {
  RelinkArgs rl;
  TestArgs t;
  PassArgs<V4, W2> a;
  View v;
  int epi;
};

// the pass `src` into the block's shared copy `dst`
template <class CP>
__device__ __forceinline__ void load_pass(CP& dst, const CP* __restrict__ src) {
  static_assert(sizeof(CP) % 16 == 0, "ChunkPass size");
  const int4* a = reinterpret_cast<const int4*>(src);
  int4* b = reinterpret_cast<int4*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(CP) / 16); i += blockDim.x) b[i] = a[i];
  __syncthreads();
}

}  // namespace dem
