// dem_mixed.cuh -- interface of the mixed-precision (FP32 contact arithmetic)
// force path.  Implemented in dem_mixed.cu.
#pragma once
#include "dem_device.cuh"

namespace dem {

struct MixedBuffers {
  bool ready = false;
  int n = 0, nw = 0, cap = 0;
  // traversal-order copies: cell-origin-relative FP32 positions + radius,
  // FP32 velocities / angular velocities
  float4* rel = nullptr;  // x - ox, y - oy, z - oz, R
  float4* v4 = nullptr;   // vx, vy, vz, wx
  float2* w2 = nullptr;   // wy, wz
  // FP32 history (ft, vt) + Kahan compensation of the tangential spring,
  // double-buffered like the FP64 tables
  float4* hval[2] = {nullptr, nullptr};   // [n*cap*2]: (ft.xyz, c.x) (vt.xyz, c.y)
  float4* wval[2] = {nullptr, nullptr};   // [n*nw*2]
};

bool mixed_available();
bool mixed_alloc(MixedBuffers& M, int n, int nw, int cap);
void mixed_free(MixedBuffers& M);
bool mixed_regrow(MixedBuffers& M, int n, int newcap, int cur, const History& src_old);
void mixed_gather(MixedBuffers& M, bool pp, const DevParams* dp, int n, const StateArrays& src,
                  const double* radius, const int* comp, const SortedArrays& S, Counters* cnt,
                  cudaStream_t st);
void mixed_force(MixedBuffers& M, bool pp, int epi, const ForceArgs& A, int cur,
                 cudaStream_t st);
void mixed_import_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st);
void mixed_export_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st);

}  // namespace dem
