// dem_mixed.cu -- mixed-precision force path (placeholder until implemented).
#include "dem_mixed.cuh"

namespace dem {

bool mixed_available() { return false; }
bool mixed_alloc(MixedBuffers&, int, int, int) { return false; }
void mixed_free(MixedBuffers& M) { M = MixedBuffers{}; }
bool mixed_regrow(MixedBuffers&, int, int, int, const History&) { return false; }
void mixed_gather(MixedBuffers&, bool, const DevParams*, int, const StateArrays&, const double*,
                  const int*, const SortedArrays&, Counters*, cudaStream_t) {}
void mixed_force(MixedBuffers&, bool, int, const ForceArgs&, int, cudaStream_t) {}
void mixed_import_history(MixedBuffers&, const History&, int, int, int, cudaStream_t) {}
void mixed_export_history(MixedBuffers&, const History&, int, int, int, cudaStream_t) {}

}  // namespace dem
