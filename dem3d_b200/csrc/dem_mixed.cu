// dem_mixed.cu -- mixed-precision force path (DEM_PREC_MIXED).
//
// Same sweep, same pair sets, same history semantics and summation order as
// the FP64 kernel; what changes is the arithmetic of a contact:
//  - the candidate test DeltaDijSq = MinDijSq - DijSq stays FP64 (from FP64
//    positions), so the contact-pair set equals the FP64 one;
//  - the overlap is formed as delta = DeltaDijSq / (MinDij + Dij), which
//    keeps its relative digits in FP32 (MinDij - Dij itself would cancel);
//  - everything downstream (normal, relative velocity, spring-dashpot,
//    tangential spring, Coulomb cap, torques, per-particle sums) is FP32;
//  - the tangential spring is carried as an FP32 pair (hi, lo) and each
//    increment is added with a compensated (Kahan/TwoSum) sum;
//  - velocities are gathered as FP32 copies; positions, the ABM ring and
//    the predictor/corrector stay FP64.
// This translation unit is compiled without multiply-add contraction (every
// kernel that inlines the same code then rounds alike), with the hardware's
// approximate FP32 division and square root.
#include "dem_mixed.cuh"
#include "dem_test.cuh"

namespace dem {

namespace {

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 mk(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return mk(s * a.x, s * a.y, s * a.z); }
// (dot and cross products and the two-term combinations below use explicit
// fused multiply-adds: one rounding per term, whatever kernel inlines them)
__device__ __forceinline__ float dot(F3 a, F3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return mk(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
// s*a + t*b
__device__ __forceinline__ F3 comb(float s, F3 a, float t, F3 b) {
  return mk(__fmaf_rn(s, a.x, __fmul_rn(t, b.x)), __fmaf_rn(s, a.y, __fmul_rn(t, b.y)),
            __fmaf_rn(s, a.z, __fmul_rn(t, b.z)));
}
// a - s*b
__device__ __forceinline__ F3 sub_scaled(F3 a, float s, F3 b) {
  return mk(__fmaf_rn(-s, b.x, a.x), __fmaf_rn(-s, b.y, a.y), __fmaf_rn(-s, b.z, a.z));
}
// FP64 sums of a particle's FP32 contributions (exact terms, one rounding
// per addition at FP64: the net force of a packing, where contact forces
// nearly cancel, keeps the contact forces' own accuracy)
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, F3 b) {
  return D3{a.x + (double)b.x, a.y + (double)b.y, a.z + (double)b.z};
}
__device__ __forceinline__ D3 operator-(D3 a, F3 b) {
  return D3{a.x - (double)b.x, a.y - (double)b.y, a.z - (double)b.z};
}

struct MPair {
  float min_dij, kn, yn, kt, yt, mu_sq;
};

template <bool PP>
struct MMat;

template <>
struct MMat<false> {
  __device__ __forceinline__ static double min_dij_sq(const DevParams& P, int ca, double, int cb,
                                                      double) {
    return P.min_dij_sq[ca * NCM + cb];
  }
  __device__ __forceinline__ static void pair(const DevParams& P, int ca, float, int cb, float,
                                              MPair& m) {
    int k = ca * NCM + cb;
    m.min_dij = (float)P.min_dij[k];
    m.kn = (float)P.kn[k];
    m.yn = (float)P.yn[k];
    m.kt = (float)P.kt[k];
    m.yt = (float)P.yt[k];
    m.mu_sq = (float)P.mu_sq[k];
  }
  __device__ __forceinline__ static void wall(const DevParams& P, int ca, float, int w, MPair& m) {
    int k = ca * NWM + w;
    m.kn = (float)P.knw[k];
    m.yn = (float)P.ynw[k];
    m.kt = (float)P.ktw[k];
    m.yt = (float)P.ytw[k];
    m.mu_sq = (float)P.muw_sq[k];
  }
  __device__ __forceinline__ static void self(const DevParams& P, int ca, float, float& im,
                                              float& ii, float& em) {
    im = (float)P.comp_inv_mass[ca];
    ii = (float)P.comp_inv_inertia[ca];
    em = (float)P.comp_eff_mass[ca];
  }
};

template <>
struct MMat<true> {
  __device__ __forceinline__ static double min_dij_sq(const DevParams&, int, double Ra, int,
                                                      double Rb) {
    double d = Ra + Rb;
    return d * d;
  }
  __device__ __forceinline__ static float mass(const DevParams& P, float R) {
    return (float)P.pp_mass_coef * (R * R * R);
  }
  __device__ __forceinline__ static void pair(const DevParams& P, int, float Ra, int, float Rb,
                                              MPair& m) {
    float ma = mass(P, Ra), mb = mass(P, Rb);
    float meff = ma * mb / (ma + mb);
    m.min_dij = Ra + Rb;
    m.kn = (float)P.pp_kn;
    m.kt = (float)P.pp_kt;
    m.yn = (float)P.pp_gamma_n * sqrtf(meff * m.kn);
    m.yt = (float)P.pp_gamma_t * sqrtf(meff * m.kt);
    m.mu_sq = (float)P.pp_mu_sq;
  }
  __device__ __forceinline__ static void wall(const DevParams& P, int, float Ra, int w, MPair& m) {
    float ma = mass(P, Ra);
    m.kn = (float)P.pp_knw[w];
    m.kt = (float)P.pp_ktw[w];
    m.yn = (float)P.pp_gamma_nw[w] * sqrtf(ma * m.kn);
    m.yt = (float)P.pp_gamma_tw[w] * sqrtf(ma * m.kt);
    m.mu_sq = (float)P.pp_muw_sq[w];
  }
  __device__ __forceinline__ static void self(const DevParams& P, int, float R, float& im,
                                              float& ii, float& em) {
    float m = mass(P, R);
    im = 1.0f / m;
    ii = 1.0f / (0.4f * m * (R * R));
    em = (float)((double)m * (P.pp_density - P.pp_fluid_density) / P.pp_density);
  }
};

__device__ __forceinline__ F3 change_plane_f(F3 V, F3 N) {
  F3 P = sub_scaled(V, dot(V, N), N);
  float ns = dot(P, P);
  if (ns != 0.0f) return sqrtf(dot(V, V) / ns) * P;
  return mk(0.f, 0.f, 0.f);
}

// TwoSum: s + e == a + b exactly
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  float bp = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

struct MOut {
  F3 FN, FT, FTlo, VT, N, NxFT;
};

// CommonCalculations (src/MForces.f90:339-387) in FP32 given the geometry.
__device__ __forceinline__ void common_mixed(F3 Rij, F3 N, F3 DispN, F3 Vij, F3 VijC,
                                             float DeltaDijSq, float half_dt, bool contacting,
                                             F3 ft0, F3 ft0lo, F3 vt0, const MPair& m, MOut& o) {
  F3 VijN = dot(VijC, N) * N;
  o.VT = VijC - VijN;
  o.FN = comb(m.kn, DispN, m.yn, VijN);
  if (contacting) {
    F3 VT0 = change_plane_f(vt0, N);
    F3 dD = half_dt * (VT0 + o.VT);
    F3 dV = o.VT - VT0;
    // rotate the compensated spring (hi + lo) onto the new contact plane
    F3 ph = sub_scaled(ft0, dot(ft0, N), N);
    F3 pl = sub_scaled(ft0lo, dot(ft0lo, N), N);
    float ns = dot(ph, ph);
    F3 hi = mk(0.f, 0.f, 0.f), lo = mk(0.f, 0.f, 0.f);
    if (ns != 0.0f) {
      float f = sqrtf(dot(ft0, ft0) / ns);
      hi = f * ph;
      lo = f * pl;
    }
    F3 inc = comb(m.kt, dD, m.yt, dV);
    float e;
    two_sum(hi.x, inc.x, o.FT.x, e);
    o.FTlo.x = lo.x + e;
    two_sum(hi.y, inc.y, o.FT.y, e);
    o.FTlo.y = lo.y + e;
    two_sum(hi.z, inc.z, o.FT.z, e);
    o.FTlo.z = lo.z + e;
  } else {
    float PartialDt;
    float VijSq = dot(Vij, Vij);
    if (VijSq > 0.0f) {
      // (R.V + sqrt((R.V)^2 + |V|^2 dD2)) / |V|^2; for approaching particles
      // (R.V < 0) the sum cancels, so use the equal form dD2 / (sqrt(..) - R.V)
      float RijVij = dot(Rij, Vij);
      float a = 2.0f * half_dt;
      float root = sqrtf(RijVij * RijVij + VijSq * DeltaDijSq);
      float b = RijVij >= 0.0f ? (RijVij + root) / VijSq : DeltaDijSq / (root - RijVij);
      PartialDt = b < a ? b : a;
    } else {
      PartialDt = 0.0f;
    }
    o.FT = (m.kt * PartialDt + m.yt) * o.VT;
    o.FTlo = mk(0.f, 0.f, 0.f);
  }
  float mun = m.mu_sq * dot(o.FN, o.FN);
  float nt = dot(o.FT, o.FT);
  if (nt > mun) {
    float g = sqrtf(mun / nt);
    o.FT = g * o.FT;
    o.FTlo = g * o.FTlo;
  }
  o.N = N;
  o.NxFT = cross(N, o.FT);
}

// pair branch (src/MForces.f90:230-252), "i" = a, "j" = b, Rij = xb - xa
__device__ __forceinline__ void mixed_pair(const double Rd[3], double DijSq, double Delta,
                                           const MPair& m, float Ra, F3 va, F3 wa, float Rb,
                                           F3 vb, F3 wb, float half_dt, bool contacting, F3 ft0,
                                           F3 ft0lo, F3 vt0, MOut& o) {
  const float D = sqrtf((float)DijSq);
  const float fDelta = (float)Delta;
  const float delta = fDelta / (m.min_dij + D);  // = MinDij - Dij, without cancellation
  const float rD = 1.0f / D;
  F3 Rij = mk((float)Rd[0], (float)Rd[1], (float)Rd[2]);
  F3 N = rD * Rij;
  F3 DispN = (-delta) * N;
  F3 Vij = vb - va;
  F3 ws = Ra * wa + Rb * wb;
  F3 VijC = Vij - cross(ws, N);
  common_mixed(Rij, N, DispN, Vij, VijC, fDelta, half_dt, contacting, ft0, ft0lo, vt0, m, o);
}

__device__ __forceinline__ void rec_read(const float4* a, const float4* b, const float* c,
                                         size_t i, F3& ft, F3& lo, F3& vt) {
  float4 x = a[i], y = b[i];
  ft = mk(x.x, x.y, x.z);
  vt = mk(x.w, y.x, y.y);
  lo = mk(y.z, y.w, c[i]);
}
__device__ __forceinline__ void rec_write(float4* a, float4* b, float* c, size_t i, F3 ft, F3 lo,
                                          F3 vt) {
  a[i] = make_float4(ft.x, ft.y, ft.z, vt.x);
  b[i] = make_float4(vt.y, vt.z, lo.x, lo.y);
  c[i] = lo.z;
}

// The mixed-precision force pass: the FP64 pass's structure (the same test
// kernel and contact list, exact FP64 overlap test, orientation, history
// semantics, each contact evaluated once, summation order), FP32 contact
// arithmetic, FP64 integrator epilogue.

constexpr int KSPEC = 2;  // record keys read before the record count is known

// The pair kernel: one thread per contact, grid-stride over the list.
// (Body for block `vblock` of a grid of `vgrid` blocks.)
template <bool PP>
__device__ __forceinline__ void pair_mixed_body(const PassArgs<float4, float2>& A,
                                                const MixedView& V, int vblock, int vgrid) {
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
  const float half_dt = (float)A.half_dt;
  const History& Hr = A.Hr;
  const History& Hw = A.Hw;
  unsigned n_col = 0;
  int need = 0, need_in = 0;
  bool overflow = false, in_over = false;
  const int stride = vgrid * blockDim.x;
  for (int s = vblock * blockDim.x + threadIdx.x; s < total; s += stride) {
    const int2 e = A.clist[s];
    const int p = e.x, q = e.y;
    // the next contact of this thread: its pair's data requested into L2
    // now, so that the next iteration's gathers overlap this one's work
    if (s + stride < total) {
      const int2 e2 = A.clist[s + stride];
      prefetch_l2(A.X + e2.x);
      prefetch_l2(A.X + e2.y);
      prefetch_l2(A.v4 + e2.x);
      prefetch_l2(A.v4 + e2.y);
      prefetch_l2(Hr.key + e2.x);
      prefetch_l2(A.in_cnt + e2.y);
    }
    const int s_in = atomicAdd(&A.in_cnt[q], 1);  // q's "j" record (returns early)
    const int ord = s - A.cstart[p];
    const int hc = Hr.cnt[p];
    int kspec[KSPEC];
#pragma unroll
    for (int r = 0; r < KSPEC; r++) kspec[r] = r < Hr.cap ? Hr.key[hslot(Hr, p, r)] : -1;
    const DevParams& P = sys_params(A.P, A.sysid, p);
    const double4 p4 = A.X[p], q4 = A.X[q];
    const float4 pv4 = A.v4[p], qv4 = A.v4[q];
    const float2 pw2 = A.w2[p], qw2 = A.w2[q];
    const int cp = PP ? 0 : A.comp[p], cq = PP ? 0 : A.comp[q];
    double Rij[3] = {q4.x - p4.x, q4.y - p4.y, q4.z - p4.z};
#pragma unroll
    for (int k = 0; k < 3; k++) Rij[k] = min_image_exact(Rij[k], P.box, k);
    const double DijSq = sumsq3(Rij);
    const double Delta = MMat<PP>::min_dij_sq(P, cp, p4.w, cq, q4.w) - DijSq;
    const float Ra = (float)p4.w, Rb = (float)q4.w;
    MPair m;
    MMat<PP>::pair(P, cp, Ra, cq, Rb, m);
    const F3 vo = mk(pv4.x, pv4.y, pv4.z), wo = mk(pv4.w, pw2.x, pw2.y);
    const F3 vq = mk(qv4.x, qv4.y, qv4.z), wq = mk(qv4.w, qw2.x, qw2.y);
    // i's records, then j's
    int r = -1;
#pragma unroll
    for (int rr = 0; rr < KSPEC; rr++)
      if (r < 0 && rr < hc && kspec[rr] == q) r = rr;
    for (int rr = KSPEC; r < 0 && rr < hc; rr++)
      if (Hr.key[hslot(Hr, p, rr)] == q) r = rr;
    F3 ft0 = mk(0.f, 0.f, 0.f), ft0lo = ft0, vt0 = ft0;
    bool contacting = r >= 0;
    if (contacting) {
      rec_read(V.ra, V.rb, V.rc, hslot(Hr, p, r), ft0, ft0lo, vt0);
      if (r < 32) atomicOr(&A.matched[p], 1u << r);
    } else {
      const int r2 = find_record(Hr, q, p);
      contacting = r2 >= 0;
      if (contacting) rec_read(V.ra, V.rb, V.rc, hslot(Hr, q, r2), ft0, ft0lo, vt0);
    }
    if (!contacting) n_col++;
    MOut out;
    mixed_pair(Rij, DijSq, Delta, m, Ra, vo, wo, Rb, vq, wq, half_dt, contacting, ft0, ft0lo,
               vt0, out);
    const F3 FTs = out.FT + out.FTlo;
    // "j" half into q's incoming records
    if (s_in < A.in_cap) {
      const unsigned long long key = sweep_key(A.cell_cur[p], A.rank[p]);
      InRec32* rec = (InRec32*)A.in_rec + (size_t)s_in * A.in_stride + q;
      rec->a = make_float4(__uint_as_float((unsigned)key), __uint_as_float((unsigned)(key >> 32)),
                           out.FN.x, out.FN.y);
      rec->b = make_float4(out.FN.z, FTs.x, FTs.y, FTs.z);
      rec->c = make_float4(out.NxFT.x, out.NxFT.y, out.NxFT.z, 0.f);
    } else {
      in_over = true;
    }
    need_in = need_in > s_in + 1 ? need_in : s_in + 1;
    // "i" half at the contact's place
    const F3 tq = cross(Ra * out.N, out.FT);
    IRec32* ir = (IRec32*)A.irec + s;
    ir->a = make_float4(out.FN.x, out.FN.y, out.FN.z, FTs.x);
    ir->b = make_float4(FTs.y, FTs.z, tq.x, tq.y);
    ir->c = make_float4(tq.z, 0.f, 0.f, 0.f);
    if (update) {
      if (ord < Hw.cap) {
        const size_t i = hslot(Hw, p, ord);
        Hw.key[i] = q;
        rec_write(V.wa, V.wb, V.wc, i, out.FT, out.FTlo, out.VT);
      } else {
        overflow = true;
      }
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
__global__ void __launch_bounds__(128, MINB) k_pair_mixed(PassArgs<float4, float2> A,
                                                          MixedView V) {
  pass_kernel_entry();
  pair_mixed_body<PP>(A, V, blockIdx.x, gridDim.x);
}

// The fold kernel: p's block of the sweep, Force and Torque in sweep order
// (FP32), a = F/m, alpha = T/I, then the FP64 integrator epilogue.  WALLS:
// some system has walls; CONE: some wall is a cone.  (Body for block
// `vblock` of particles.)
template <bool PP, int EPI, bool WALLS, bool CONE>
__device__ __forceinline__ void fold_mixed_body(const PassArgs<float4, float2>& A,
                                                const MixedView& V, int vblock) {
  __shared__ float s_w[WALLS ? NWM : 1][128];  // |FN| of each wall contact
  __shared__ int s_abort;
  // one decision for the whole block (it meets block barriers later)
  if (threadIdx.x == 0) s_abort = A.cnt->abort;
  __syncthreads();
  if (s_abort) return;
  if (WALLS)
    for (int w = 0; w < A.nw_max; w++) s_w[w][threadIdx.x] = 0.f;
  if (vblock == 0 && threadIdx.x == 0) atomicAdd(&A.cnt->pass_id, 1);  // this pass is done
  const int p0 = vblock * blockDim.x + threadIdx.x;
  const int p = p0 < A.n ? p0 : 0;
  // (a slab of a decomposition advances only its own particles)
  const bool valid = p0 < A.n && in_slab(sys_params(A.P, A.sysid, p), A.cell_cur[p]);
  const bool update = A.update != 0;
  const History& Hr = A.Hr;
  const History& Hw = A.Hw;
  unsigned n_wc = 0;
  int need = 0;
  bool overflow = false;
  double d2 = 0.0;
  if (valid) {
    const DevParams& P = sys_params(A.P, A.sysid, p);
    prefetch_epilogue<EPI>(A, P, p, true);
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
    const double Rpd = p4.w;
    const float Rp = (float)Rpd;
    const int cp = PP ? 0 : A.comp[p];
    float inv_m, inv_i, eff_m;
    MMat<PP>::self(P, cp, Rp, inv_m, inv_i, eff_m);
    // ---- p's block: gravity, its contacts as "i" in row order
    F3 iF = mk(eff_m * (float)P.gravity[0], eff_m * (float)P.gravity[1],
               eff_m * (float)P.gravity[2]);
    F3 iT = mk(0.f, 0.f, 0.f);
    const IRec32* ir = (const IRec32*)A.irec + st0;
    for (int k = 0; k < nc; k++) {
      const IRec32 r = ir[k];
      iF = iF + mk(r.a.x, r.a.y, r.a.z) + mk(r.a.w, r.b.x, r.b.y);
      iT = iT + mk(r.b.z, r.b.w, r.c.x);
    }
    int hw_n = nc;  // the pair kernel wrote the records of the contacts
    if (WALLS) {
      const float4 pv4 = A.v4[p];
      const float2 pw2 = A.w2[p];
      const F3 vp = mk(pv4.x, pv4.y, pv4.z);
      const F3 wp = mk(pv4.w, pw2.x, pw2.y);
      const float half_dt = (float)A.half_dt;
      for (int w = 0; w < P.nw; w++) {
        const dem_wall& W = P.walls[w];
        const size_t wi = (size_t)p * P.nw + w;
        const bool contacting = Hr.wflag[wi] != 0;
        F3 ft0 = mk(0.f, 0.f, 0.f), ft0lo = ft0, vt0 = ft0;
        if (contacting) rec_read(V.rwa, V.rwb, V.rwc, wi, ft0, ft0lo, vt0);
        double Dij, Nij[3], Qji[3];
        const bool ov = overlap_wall<CONE>(P, W, xp, Rpd, Dij, Nij, Qji);
        if (ov) {
          n_wc++;
          const double Delta = Rpd * Rpd - Dij * Dij;
          const float delta = (float)(Rpd - Dij);
          F3 N = mk((float)Nij[0], (float)Nij[1], (float)Nij[2]);
          F3 Q = mk((float)Qji[0], (float)Qji[1], (float)Qji[2]);
          F3 wv = mk((float)W.velocity[0], (float)W.velocity[1], (float)W.velocity[2]);
          F3 ww = mk((float)W.omega[0], (float)W.omega[1], (float)W.omega[2]);
          F3 Vij = (wv + cross(ww, Q)) - vp;
          F3 VijC = Vij - cross(Rp * wp, N);
          F3 Rw = mk((float)(W.position[0] + Qji[0] - xp[0]),
                     (float)(W.position[1] + Qji[1] - xp[1]),
                     (float)(W.position[2] + Qji[2] - xp[2]));
          MPair m;
          MMat<PP>::wall(P, cp, Rp, w, m);
          MOut o;
          common_mixed(Rw, N, (-delta) * N, Vij, VijC, (float)Delta, half_dt, contacting, ft0,
                       ft0lo, vt0, m, o);
          iF = iF + o.FN + (o.FT + o.FTlo);
          iT = iT + cross(Rp * o.N, o.FT);
          s_w[w][threadIdx.x] = sqrtf(dot(o.FN, o.FN));
          if (update) {
            Hw.wflag[wi] = 1;
            rec_write(V.wwa, V.wwb, V.wwc, wi, o.FT, o.FTlo, o.VT);
          }
        } else if (update) {
          Hw.wflag[wi] = 0;
        }
      }
    }
    if (A.drag)  // iForce = iForce + DragForce(iPart) (src/MForces.f90:316)
      iF = iF + mk((float)A.drag[(size_t)3 * p], (float)A.drag[(size_t)3 * p + 1],
                   (float)A.drag[(size_t)3 * p + 2]);
    if (update) {
      const int hc = Hr.cnt[p];
      for (int r = 0; r < hc; r++) {
        if (r < 32 && ((matched >> r) & 1u)) continue;
        const size_t i = hslot(Hr, p, r);
        const int q2 = Hr.key[i];
        if (q2 >= A.n || !partner_adjacent(A, P, c, q2)) {
          if (hw_n < Hw.cap) {
            F3 ft, lo, vt;
            rec_read(V.ra, V.rb, V.rc, i, ft, lo, vt);
            const size_t o = hslot(Hw, p, hw_n);
            Hw.key[o] = q2;
            rec_write(V.wa, V.wb, V.wc, o, ft, lo, vt);
          } else {
            overflow = true;
          }
          hw_n++;
        }
      }
      Hw.cnt[p] = hw_n < Hw.cap ? hw_n : Hw.cap;
      if (hw_n > Hw.cap) overflow = true;
      need = hw_n;
    }
    // ---- Force and Torque in sweep order
    const InRec32* in = (const InRec32*)A.in_rec + p;
    const size_t st = (size_t)A.in_stride;
    D3 F = D3{0.0, 0.0, 0.0}, T = D3{0.0, 0.0, 0.0};
    fold_in_order(
        ni, key_p,
        [&](int e) {
          const float2 k = *(const float2*)(in + e * st);
          return (unsigned long long)__float_as_uint(k.x) |
                 ((unsigned long long)__float_as_uint(k.y) << 32);
        },
        [&]() {
          F = F + iF;
          T = T + iT;
        },
        [&](int e) {
          const InRec32 r = in[e * st];
          const F3 FN = mk(r.a.z, r.a.w, r.b.x), FTs = mk(r.b.y, r.b.z, r.b.w);
          const F3 NxFT = mk(r.c.x, r.c.y, r.c.z);
          F = F - FN - FTs;
          T = T + Rp * NxFT;
        });
    if (EPI == EPI_STORE && A.amsum) {
      const size_t n3 = (size_t)3 * A.n, q = (size_t)3 * p;
      A.amsum[q] = F.x; A.amsum[q + 1] = F.y; A.amsum[q + 2] = F.z;
      A.amsum[n3 + q] = T.x; A.amsum[n3 + q + 1] = T.y; A.amsum[n3 + q + 2] = T.z;
    }
    const double acc[3] = {F.x * (double)inv_m, F.y * (double)inv_m, F.z * (double)inv_m};
    const double alp[3] = {T.x * (double)inv_i, T.y * (double)inv_i, T.z * (double)inv_i};
    // the integrator runs on FP64 velocities: Particle's for the predictor,
    // Predicted's for the corrector (the pass copies are FP32)
    double vd[3] = {0.0, 0.0, 0.0}, wd[3] = {0.0, 0.0, 0.0};
    if (EPI == EPI_PREDICT) {
      vd[0] = A.part.vx[p]; vd[1] = A.part.vy[p]; vd[2] = A.part.vz[p];
      wd[0] = A.part.wx[p]; wd[1] = A.part.wy[p]; wd[2] = A.part.wz[p];
    } else if (EPI == EPI_CORRECT) {
      vd[0] = A.pred.vx[p]; vd[1] = A.pred.vy[p]; vd[2] = A.pred.vz[p];
    }
    epilogue<EPI>(A, P, p, xp, Rpd, vd, wd, acc, alp, c, d2);
  }
  if (WALLS && A.nw_max > 0) wall_partials(s_w, A.nw_max, A.wall_part, vblock);
  if (overflow) {
    atomicExch(&A.cnt->overflow, 1);
    set_abort(A.cnt, A.tag);
  }
  publish_counts_block(A.cnt, update, 0u, 0u, n_wc, (unsigned)need, 0u);
  if (EPI != EPI_STORE) publish_disp_block(A.cnt, d2);
}

// (STRIDE: grid-stride over blocks of 128 particles.  Register budget: 6
// blocks of 128 per SM, 80 registers.  The predictor spills a few registers
// at that budget and still runs faster than at 5 blocks: 127.6 against
// 137.9 us per launch at 1M spheres, 611 against 695 us with walls at 4M.)
template <bool PP, int EPI, bool WALLS, bool CONE, bool STRIDE>
__global__ void __launch_bounds__(128, 6)
    k_fold_mixed(PassArgs<float4, float2> A, MixedView V) {
  pass_kernel_entry();
  if (!STRIDE) {
    fold_mixed_body<PP, EPI, WALLS, CONE>(A, V, blockIdx.x);
    return;
  }
  const int nvb = (A.n + 127) / 128;
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
    fold_mixed_body<PP, EPI, WALLS, CONE>(A, V, vb);
    __syncthreads();  // the block's shared arrays are reused by the next block of particles
  }
}

// The persistent chunk kernel (mixed): k_chunk_fp64's structure with the
// mixed pair and fold bodies.  The relink and test bodies are the FP64
// unit's code, written with explicitly rounded operations, so this unit's
// approximate division and square root do not reach them; this unit is
// compiled without contraction, so the inlined pair and fold bodies round
// exactly as in k_pair_mixed / k_fold_mixed.
using ChunkPassMx = ChunkPass<float4, float2, MixedView>;

template <bool PP, bool WALLS, bool CONE>
__global__ void __launch_bounds__(128, 4) k_chunk_mixed(const ChunkPassMx* __restrict__ prog,
                                                        int npass, GridSync g) {
  __shared__ ChunkPassMx sp;
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
    pair_mixed_body<PP>(sp.a, sp.v, blockIdx.x, gridDim.x);
    if (!grid_sync(g)) return;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
      if (sp.epi == EPI_PREDICT) fold_mixed_body<PP, EPI_PREDICT, WALLS, CONE>(sp.a, sp.v, vb);
      else fold_mixed_body<PP, EPI_CORRECT, WALLS, CONE>(sp.a, sp.v, vb);
      __syncthreads();
    }
    if (!grid_sync(g)) return;  // (also: every block is done with sp)
  }
}

// FP64 records <-> FP32 records
__global__ void k_hist_to_mixed(int n, History H, float4* a, float4* b, float* c, int nw,
                                float4* wa, float4* wb, float* wc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int r = 0; r < H.cnt[i]; r++) {
    const size_t k = hslot(H, i, r);
    double2 x = H.val[3 * k], y = H.val[3 * k + 1], z = H.val[3 * k + 2];
    a[k] = make_float4((float)x.x, (float)x.y, (float)y.x, (float)y.y);
    b[k] = make_float4((float)z.x, (float)z.y, 0.f, 0.f);
    c[k] = 0.f;
  }
  for (int w = 0; w < nw; w++) {
    size_t k = (size_t)i * nw + w;
    double2 x = H.wval[3 * k], y = H.wval[3 * k + 1], z = H.wval[3 * k + 2];
    wa[k] = make_float4((float)x.x, (float)x.y, (float)y.x, (float)y.y);
    wb[k] = make_float4((float)z.x, (float)z.y, 0.f, 0.f);
    wc[k] = 0.f;
  }
}

__global__ void k_hist_from_mixed(int n, History H, const float4* a, const float4* b,
                                  const float* c, int nw, const float4* wa, const float4* wb,
                                  const float* wc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int r = 0; r < H.cnt[i]; r++) {
    const size_t k = hslot(H, i, r);
    float4 x = a[k], y = b[k];
    H.val[3 * k] = make_double2((double)x.x + y.z, (double)x.y + y.w);
    H.val[3 * k + 1] = make_double2((double)x.z + c[k], (double)x.w);
    H.val[3 * k + 2] = make_double2((double)y.x, (double)y.y);
  }
  for (int w = 0; w < nw; w++) {
    size_t k = (size_t)i * nw + w;
    float4 x = wa[k], y = wb[k];
    H.wval[3 * k] = make_double2((double)x.x + y.z, (double)x.y + y.w);
    H.wval[3 * k + 1] = make_double2((double)x.z + wc[k], (double)x.w);
    H.wval[3 * k + 2] = make_double2((double)y.x, (double)y.y);
  }
}

__global__ void k_mixed_regrow(int n, int ns, int nd, const int* cnt, const float4* a,
                               const float4* b, const float* c, float4* na, float4* nb,
                               float* nc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int r = 0; r < cnt[i]; r++) {
    // slot-major: record r of particle i at r*stride + i, the old tables laid
    // out for ns rows, the new ones for nd
    const size_t s = (size_t)r * ns + i, d = (size_t)r * nd + i;
    na[d] = a[s];
    nb[d] = b[s];
    nc[d] = c[s];
  }
}

unsigned blocks(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// blocks of a cooperative launch of `k`: as many as fit on the device at
// once (occupancy x SMs), at most `want`
template <class K>
int coop_blocks(K k, int want) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 128, 0);
  const int most = per * sms;
  return want < most ? want : most;
}

template <class K>
cudaError_t launch_chunk(K k, const ChunkPassMx* prog, int npass, GridSync g, int want,
                         cudaStream_t st, int* blocks_out) {
  const int nb = coop_blocks(k, want);
  if (nb <= 0) return cudaErrorLaunchOutOfResources;
  g.expected += (unsigned)nb;  // (on entry: the blocks a test adds to every barrier)
  void* args[] = {(void*)&prog, (void*)&npass, (void*)&g};
  if (blocks_out) *blocks_out = nb;
  return cudaLaunchCooperativeKernel((const void*)k, dim3(nb), dim3(128), args, 0, st);
}

}  // namespace

bool mixed_available() { return true; }

bool mixed_alloc(MixedBuffers& M, int n, int nw, int cap) {
  mixed_free(M);
  size_t N = (size_t)(n > 0 ? n : 1);
  size_t W = N * (size_t)(nw > 0 ? nw : 1);
  M.n = n;
  M.nw = nw;
  M.cap = cap;
  bool ok = true;
  for (int b = 0; b < 2 && ok; b++) {
    ok = cudaMalloc(&M.ha[b], N * cap * sizeof(float4)) == cudaSuccess &&
         cudaMalloc(&M.hb[b], N * cap * sizeof(float4)) == cudaSuccess &&
         cudaMalloc(&M.hc[b], N * cap * sizeof(float)) == cudaSuccess &&
         cudaMalloc(&M.wa[b], W * sizeof(float4)) == cudaSuccess &&
         cudaMalloc(&M.wb[b], W * sizeof(float4)) == cudaSuccess &&
         cudaMalloc(&M.wc[b], W * sizeof(float)) == cudaSuccess;
  }
  M.ready = ok;
  return ok;
}

void mixed_free(MixedBuffers& M) {
  for (int b = 0; b < 2; b++) {
    cudaFree(M.ha[b]);
    cudaFree(M.hb[b]);
    cudaFree(M.hc[b]);
    cudaFree(M.wa[b]);
    cudaFree(M.wb[b]);
    cudaFree(M.wc[b]);
  }
  M = MixedBuffers{};
}

bool mixed_regrow(MixedBuffers& M, int n, int stride, int newcap, int cur, const History& old,
                  cudaStream_t st) {
  size_t N = (size_t)(stride > 0 ? stride : 1);
  float4 *na[2], *nb[2];
  float* nc[2];
  for (int b = 0; b < 2; b++) {
    if (cudaMalloc(&na[b], N * newcap * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&nb[b], N * newcap * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&nc[b], N * newcap * sizeof(float)) != cudaSuccess)
      return false;
  }
  if (n > 0)
    k_mixed_regrow<<<blocks(n, 256), 256, 0, st>>>(n, old.n, (int)N, old.cnt, M.ha[cur],
                                                    M.hb[cur], M.hc[cur], na[cur], nb[cur],
                                                    nc[cur]);
  cudaStreamSynchronize(st);
  for (int b = 0; b < 2; b++) {
    cudaFree(M.ha[b]);
    cudaFree(M.hb[b]);
    cudaFree(M.hc[b]);
    M.ha[b] = na[b];
    M.hb[b] = nb[b];
    M.hc[b] = nc[b];
  }
  M.cap = newcap;
  return true;
}

bool mixed_grow_walls(MixedBuffers& M, int n, int stride, int cur, cudaStream_t st) {
  const size_t W = (size_t)(stride > 0 ? stride : 1) * (size_t)(M.nw > 0 ? M.nw : 1);
  const size_t keep = (size_t)n * (size_t)(M.nw > 0 ? M.nw : 1);
  float4 *na[2], *nb[2];
  float* nc[2];
  for (int b = 0; b < 2; b++)
    if (cudaMalloc(&na[b], W * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&nb[b], W * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&nc[b], W * sizeof(float)) != cudaSuccess)
      return false;
  if (keep) {
    cudaMemcpyAsync(na[cur], M.wa[cur], keep * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(nb[cur], M.wb[cur], keep * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(nc[cur], M.wc[cur], keep * sizeof(float), cudaMemcpyDeviceToDevice, st);
  }
  cudaStreamSynchronize(st);
  for (int b = 0; b < 2; b++) {
    cudaFree(M.wa[b]);
    cudaFree(M.wb[b]);
    cudaFree(M.wc[b]);
    M.wa[b] = na[b];
    M.wb[b] = nb[b];
    M.wc[b] = nc[b];
  }
  M.n = stride;
  return true;
}

MixedView mixed_view(const MixedBuffers& M, int cur) {
  MixedView V;
  V.ra = M.ha[cur];
  V.rb = M.hb[cur];
  V.rc = M.hc[cur];
  V.wa = M.ha[cur ^ 1];
  V.wb = M.hb[cur ^ 1];
  V.wc = M.hc[cur ^ 1];
  V.rwa = M.wa[cur];
  V.rwb = M.wb[cur];
  V.rwc = M.wc[cur];
  V.wwa = M.wa[cur ^ 1];
  V.wwb = M.wb[cur ^ 1];
  V.wwc = M.wc[cur ^ 1];
  return V;
}

void mixed_pass(MixedBuffers& M, bool pp, int epi, int variant, bool walls, bool cone,
                const PassArgs<float4, float2>& A, int cur, cudaStream_t st, int part,
                unsigned pair_blocks, int ppt, bool early) {
  if (A.n == 0) return;
  const MixedView V = mixed_view(M, cur);
  if (part == 0) {
#define PCASE(PPV, MB) launch_pass(early, k_pair_mixed<PPV, MB>, pair_blocks, 128, st, A, V)
    if (variant == 1) {
      if (pp) PCASE(true, 3);
      else PCASE(false, 3);
    } else if (variant == 2) {
      if (pp) PCASE(true, 5);
      else PCASE(false, 5);
    } else {
      if (pp) PCASE(true, 4);
      else PCASE(false, 4);
    }
#undef PCASE
    return;
  }
  const unsigned nvb = blocks(A.n, 128);
  const bool stride = ppt > 1 && epi != EPI_STORE;
  const unsigned g = stride ? (nvb + ppt - 1) / ppt : nvb;
#define FK(PPV, E, W, CN, S) launch_pass(early, k_fold_mixed<PPV, E, W, CN, S>, g, 128, st, A, V)
#define FCASE(PPV, W, CN)                          \
  do {                                             \
    if (epi == EPI_PREDICT) {                      \
      if (stride) FK(PPV, EPI_PREDICT, W, CN, true); \
      else FK(PPV, EPI_PREDICT, W, CN, false);     \
    } else if (epi == EPI_CORRECT) {               \
      if (stride) FK(PPV, EPI_CORRECT, W, CN, true); \
      else FK(PPV, EPI_CORRECT, W, CN, false);     \
    } else {                                       \
      FK(PPV, EPI_STORE, W, CN, false);            \
    }                                              \
  } while (0)
  if (!walls) {
    if (pp) FCASE(true, false, false);
    else FCASE(false, false, false);
  } else if (cone) {
    if (pp) FCASE(true, true, true);
    else FCASE(false, true, true);
  } else {
    if (pp) FCASE(true, true, false);
    else FCASE(false, true, false);
  }
#undef FCASE
#undef FK
}

cudaError_t mixed_chunk(bool pp, bool walls, bool cone,
                        const ChunkPass<float4, float2, MixedView>* prog, int npass, GridSync g,
                        int want_blocks, cudaStream_t st, int* blocks_out) {
#define CCASE(PPV, W, CN) \
  return launch_chunk(k_chunk_mixed<PPV, W, CN>, prog, npass, g, want_blocks, st, blocks_out)
  if (!walls) {
    if (pp) CCASE(true, false, false);
    CCASE(false, false, false);
  }
  if (cone) {
    if (pp) CCASE(true, true, true);
    CCASE(false, true, true);
  }
  if (pp) CCASE(true, true, false);
  CCASE(false, true, false);
#undef CCASE
}

void mixed_import_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st) {
  if (n == 0) return;
  k_hist_to_mixed<<<blocks(n, 256), 256, 0, st>>>(n, H, M.ha[cur], M.hb[cur], M.hc[cur], nw,
                                                  M.wa[cur], M.wb[cur], M.wc[cur]);
}

void mixed_export_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st) {
  if (n == 0) return;
  k_hist_from_mixed<<<blocks(n, 256), 256, 0, st>>>(n, H, M.ha[cur], M.hb[cur], M.hc[cur], nw,
                                                    M.wa[cur], M.wb[cur], M.wc[cur]);
}

}  // namespace dem
