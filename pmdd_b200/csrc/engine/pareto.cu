// Standalone Pareto filter of one int32 point set: the maxima under componentwise >=,
// one copy of each (ParetoFrontier::merge semantics, src/pmdd/enum/pareto_frontier.hpp:
// 237-303), by the block-wide sort-filter-skyline sweep of sfs.cuh.
#include "pareto.cuh"
#include "sfs.cuh"

namespace pmdd {
namespace dev {

template <int D>
__global__ void __launch_bounds__(SfsCfg<D, int32_t>::kThreads)
    pareto_filter_kernel(const int32_t *__restrict__ in, int64_t n, SfsScratch<int32_t> s, int32_t *__restrict__ out,
                         int64_t *__restrict__ out_n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int32_t k = sfs_block<D, int32_t>(smem_raw, in, n, s, out);
    if (threadIdx.x == 0) *out_n = k;
}

size_t pareto_scratch_bytes(int d, int64_t n) {
    const size_t pts = (static_cast<size_t>(n) * d * sizeof(int32_t) + 255) / 256 * 256;
    const size_t idx = (static_cast<size_t>(n) * sizeof(int32_t) + 255) / 256 * 256;
    return 2 * pts + 2 * idx;
}

SfsScratch<int32_t> pareto_scratch_layout(void *scratch, int d, int64_t n) {
    const size_t pts = (static_cast<size_t>(n) * d * sizeof(int32_t) + 255) / 256 * 256;
    const size_t idx = (static_cast<size_t>(n) * sizeof(int32_t) + 255) / 256 * 256;
    char *m = static_cast<char *>(scratch);
    SfsScratch<int32_t> s;
    s.P2 = reinterpret_cast<int32_t *>(m);
    s.SV = reinterpret_cast<int32_t *>(m + pts);
    s.I2 = reinterpret_cast<int32_t *>(m + 2 * pts);
    s.SVI = reinterpret_cast<int32_t *>(m + 2 * pts + idx);
    return s;
}

template <int D>
static cudaError_t launch_pareto_t(const int32_t *in, int64_t n, void *scratch, int32_t *out, int64_t *out_n,
                                   cudaStream_t stream) {
    using Cfg = SfsCfg<D, int32_t>;
    {
        const cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(pareto_filter_kernel<D>), Cfg::kSmem);
        if (e != cudaSuccess) return e;
    }
    pareto_filter_kernel<D><<<1, Cfg::kThreads, Cfg::kSmem, stream>>>(in, n, pareto_scratch_layout(scratch, D, n),
                                                                       out, out_n);
    return cudaGetLastError();
}

cudaError_t launch_pareto_filter(int d, const int32_t *in, int64_t n, void *scratch, int32_t *out, int64_t *out_n,
                                 cudaStream_t stream) {
    PMDD_DISPATCH_D(d, (launch_pareto_t<DD>(in, n, scratch, out, out_n, stream)));
}

}  // namespace dev
}  // namespace pmdd
