// Launcher of the standalone Pareto filter (pareto.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace pmdd {
namespace dev {

// Device scratch a filter of n points of d objectives needs (bytes).
size_t pareto_scratch_bytes(int d, int64_t n);
// Maxima of in[0..n) (d int32 values per point) into out; *out_n (device) receives
// their count.  One block; n < 2^31; d in 1..8.
cudaError_t launch_pareto_filter(int d, const int32_t *in, int64_t n, void *scratch, int32_t *out, int64_t *out_n,
                                 cudaStream_t stream);

}  // namespace dev
}  // namespace pmdd
