// dem_mixed.cuh -- interface of the mixed-precision (FP32 contact arithmetic)
// force path.  Implemented in dem_mixed.cu.
#pragma once
#include "dem_test.cuh"

namespace dem {

struct MixedBuffers {
  bool ready = false;
  int n = 0, nw = 0, cap = 0;
  // FP32 pair records (ft, vt, Kahan remainder of ft), double-buffered like
  // the key/count tables of History: a = (ft.xyz, vt.x), b = (vt.yz, lo.xy),
  // c = lo.z
  float4* ha[2] = {nullptr, nullptr};
  float4* hb[2] = {nullptr, nullptr};
  float* hc[2] = {nullptr, nullptr};
  // wall records, same packing, [n*nw]
  float4* wa[2] = {nullptr, nullptr};
  float4* wb[2] = {nullptr, nullptr};
  float* wc[2] = {nullptr, nullptr};
};

// The FP32 record arrays one pass reads (r*) and writes (w*): pair records
// (a, b, c of MixedBuffers) and wall records (wa, wb, wc)
struct MixedView {
  // history values [n*cap]: a = (ft.xyz, vt.x) b = (vt.yz, lo.xy) c = lo.z
  const float4* ra;
  const float4* rb;
  const float* rc;
  float4* wa;
  float4* wb;
  float* wc;
  // wall history values [n*nw], same packing
  const float4* rwa;
  const float4* rwb;
  const float* rwc;
  float4* wwa;
  float4* wwb;
  float* wwc;
};
MixedView mixed_view(const MixedBuffers& M, int cur);

bool mixed_available();
bool mixed_alloc(MixedBuffers& M, int n, int nw, int cap);
void mixed_free(MixedBuffers& M);
// the current records of `n` particles into tables of capacity newcap laid
// out for `stride` rows (old: the tables they come from, with their stride)
bool mixed_regrow(MixedBuffers& M, int n, int stride, int newcap, int cur, const History& old,
                  cudaStream_t st);
// the wall records of the first n particles into arrays for `stride` rows
bool mixed_grow_walls(MixedBuffers& M, int n, int stride, int cur, cudaStream_t st);
// One kernel of a force pass (FP32 contact arithmetic) on the context's
// stream: part 0 = the pair kernel (pair_blocks blocks of 128 threads over
// the contact list; variant: compiled for 4 (0), 3 (1) or 5 (2) resident
// blocks per SM), 1 = the fold kernel with epilogue `epi` (walls: some
// system has walls; cone: some wall is a cone; ppt > 1: the fold grid holds
// 1/ppt of the blocks of 128 particles and strides over them; early: launched
// with programmatic stream serialization).  The test kernel that builds the
// contact list is shared with the FP64 path.
void mixed_pass(MixedBuffers& M, bool pp, int epi, int variant, bool walls, bool cone,
                const PassArgs<float4, float2>& A, int cur, cudaStream_t st, int part,
                unsigned pair_blocks, int ppt, bool early);
// One persistent chunk (npass passes of prog, a device array) as a
// cooperative launch of at most want_blocks blocks of 128 threads (fewer if
// fewer fit on the device at once; the count in *blocks_out).  g.expected
// holds the blocks a test adds to every barrier (0 normally).
cudaError_t mixed_chunk(bool pp, bool walls, bool cone,
                        const ChunkPass<float4, float2, MixedView>* prog, int npass, GridSync g,
                        int want_blocks, cudaStream_t st, int* blocks_out);
void mixed_import_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st);
void mixed_export_history(MixedBuffers& M, const History& H, int n, int nw, int cur,
                          cudaStream_t st);

}  // namespace dem
