// The TSP MDD structure of n cities built on the device: see tspbuild.cuh.
#include <algorithm>
#include <climits>

#include "scan.cuh"
#include "tspbuild.cuh"

namespace pmdd {
namespace dev {

namespace {

constexpr int kTspThreads = 256;

int64_t choose(int n, int k) {
    if (k < 0 || k > n) return 0;
    int64_t c = 1;
    for (int i = 1; i <= k; ++i) c = c * (n - k + i) / i;
    return c;
}

int64_t dense_states(int n) { return (static_cast<int64_t>(1) << (n - 1)) * n; }

// Is dense state e = (S >> 1) * n + v a state (S, v) of layer l+1: |S| = l + 1, v != 0?
__device__ __forceinline__ bool layer_member(int64_t e, int n, int l, uint32_t *S_out, int *v_out) {
    const uint32_t Mp = static_cast<uint32_t>(e / n);
    const int v = static_cast<int>(e % n);
    const uint32_t S = (Mp << 1) | 1u;
    *S_out = S;
    *v_out = v;
    return v != 0 && ((S >> v) & 1u) && __popc(S) == l + 1;
}

// Parents of child (S, v) whose last city u passes the layer rule: u = 0 from layer 1,
// u != 0 after it.
__device__ __forceinline__ bool parent_city(int u, uint32_t Sp, int l) {
    return ((Sp >> u) & 1u) && (l == 1 ? u == 0 : u != 0);
}

__global__ void tsp_init_kernel(int32_t *idx, int64_t D) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < D;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        idx[e] = e == 0 ? 0 : -1;
}

__global__ void __launch_bounds__(kTspThreads) tsp_code_kernel(int n, int l, const int32_t *__restrict__ cur,
                                                               int32_t *__restrict__ next, int32_t *__restrict__ flag,
                                                               int64_t D, int64_t codes) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < D;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint32_t S;
        int v;
        if (!layer_member(e, n, l, &S, &v)) {
            next[e] = -1;
            continue;
        }
        const uint32_t Sp = S & ~(1u << v);
        int32_t best = INT_MAX;
        for (int u = 0; u < n; ++u) {
            if (!parent_city(u, Sp, l)) continue;
            const int32_t p = cur[static_cast<int64_t>(Sp >> 1) * n + u];
            if (p >= 0 && p < best) best = p;
        }
        if (best == INT_MAX) {  // no parent: cannot happen for a member state
            next[e] = -1;
            continue;
        }
        const int64_t code = static_cast<int64_t>(best) * n + v;
        next[e] = code < codes ? static_cast<int32_t>(code) : -1;
        if (code < codes) flag[code] = 1;
    }
}

// Exclusive scan of flag[0..m) in place by one block; *count receives the total, and
// *err is set when it differs from `expect`.
__global__ void __launch_bounds__(1024) tsp_rank_kernel(int32_t *flag, int64_t m, int32_t expect, int32_t *err) {
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t total;
    const int64_t chunk = (m + 1023) / 1024;
    const int64_t b = threadIdx.x * chunk, e = min(m, b + chunk);
    int32_t sum = 0;
    for (int64_t i = b; i < e; ++i) sum += flag[i];
    int32_t run = block_exclusive_scan<int32_t, 1024>(sum, warp_buf, &total);
    for (int64_t i = b; i < e; ++i) {
        const int32_t x = flag[i];
        flag[i] = run;
        run += x;
    }
    if (threadIdx.x == 0 && total != expect) atomicOr(err, 1);
}

__global__ void tsp_assign_kernel(int32_t *__restrict__ next, const int32_t *__restrict__ flag,
                                  int32_t *__restrict__ inv, int64_t D, int32_t width) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < D;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t code = next[e];
        if (code < 0) continue;
        const int32_t id = flag[code];
        next[e] = id;
        if (id >= 0 && id < width) inv[id] = static_cast<int32_t>(e);
    }
}

// Incoming arcs of every node of layer l+1: its parents in id order.
__global__ void __launch_bounds__(kTspThreads) tsp_fill_kernel(int n, int l, const int32_t *__restrict__ cur,
                                                               const int32_t *__restrict__ inv, int32_t width,
                                                               int32_t lo_prev, int32_t lo_next, int32_t arc_base,
                                                               int32_t deg, int32_t *__restrict__ in_off,
                                                               int32_t *__restrict__ arc_src,
                                                               int32_t *__restrict__ arc_w, int32_t *err) {
    for (int32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < width; id += gridDim.x * blockDim.x) {
        const int64_t e = inv[id];
        const uint32_t S = (static_cast<uint32_t>(e / n) << 1) | 1u;
        const int v = static_cast<int>(e % n);
        const uint32_t Sp = S & ~(1u << v);
        int32_t pid[kTspMaxCities], row[kTspMaxCities];
        int k = 0;
        for (int u = 0; u < n; ++u) {
            if (!parent_city(u, Sp, l)) continue;
            const int32_t p = cur[static_cast<int64_t>(Sp >> 1) * n + u];
            if (p < 0 || k >= deg) {
                atomicOr(err, 2);
                continue;
            }
            // insertion by parent id
            int q = k;
            while (q > 0 && pid[q - 1] > p) {
                pid[q] = pid[q - 1];
                row[q] = row[q - 1];
                --q;
            }
            pid[q] = p;
            row[q] = 1 + u * n + v;
            ++k;
        }
        if (k != deg) atomicOr(err, 2);
        const int32_t base = arc_base + id * deg;
        for (int q = 0; q < k; ++q) {
            arc_src[base + q] = lo_prev + pid[q];
            arc_w[base + q] = row[q];
        }
        in_off[lo_next + id + 1] = base + deg;
    }
}

// Arcs into the terminal (one per node of layer n, in id order) and the first two
// layers' arcs and offsets.
__global__ void tsp_ends_kernel(int n, const int32_t *__restrict__ inv_n, int32_t width_n, int32_t lo_n,
                                int32_t lo_term, int32_t arc_base, int32_t *__restrict__ in_off,
                                int32_t *__restrict__ arc_src, int32_t *__restrict__ arc_w) {
    for (int32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < width_n; id += gridDim.x * blockDim.x) {
        const int last = static_cast<int>(inv_n[id] % n);
        arc_src[arc_base + id] = lo_n + id;
        arc_w[arc_base + id] = 1 + last * n;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        in_off[0] = 0;  // the root
        in_off[1] = 0;
        in_off[2] = 1;  // ({0}, 0) from the root, weight row 0
        arc_src[0] = 0;
        arc_w[0] = 0;
        in_off[lo_term + 1] = arc_base + width_n;
    }
}

}  // namespace

TspShape tsp_shape(int n) {
    TspShape s;
    const int L = n + 2;
    std::vector<int64_t> size(L), indeg(L);
    size[0] = 1;
    indeg[0] = 0;
    size[1] = 1;
    indeg[1] = 1;
    for (int l = 2; l <= n; ++l) {
        size[l] = choose(n - 1, l - 1) * (l - 1);
        indeg[l] = l == 2 ? 1 : l - 2;
    }
    size[n + 1] = 1;
    indeg[n + 1] = size[n];
    s.layer_off.assign(L + 1, 0);
    s.arc_at.assign(L + 1, 0);
    for (int l = 0; l < L; ++l) {
        s.layer_off[l + 1] = s.layer_off[l] + static_cast<int32_t>(size[l]);
        s.arc_at[l + 1] = s.arc_at[l] + static_cast<int32_t>(size[l] * indeg[l]);
        s.max_width = std::max<int32_t>(s.max_width, static_cast<int32_t>(size[l]));
    }
    return s;
}

size_t tsp_scratch_bytes(int n) {
    const TspShape s = tsp_shape(n);
    const int64_t D = dense_states(n);
    auto al = [](int64_t ints) { return static_cast<size_t>((ints * 4 + 255) / 256 * 256); };
    return 2 * al(D) + al(static_cast<int64_t>(n) * s.max_width) + al(s.max_width);
}

cudaError_t launch_tsp_structure(int n, const TspShape &shape, int32_t *layer_offsets, int32_t *in_arc_offsets,
                                 int32_t *arc_src, int32_t *arc_weight, void *scratch, int32_t *err, int sms,
                                 cudaStream_t stream, int64_t *launches) {
    const int64_t D = dense_states(n);
    auto al = [](int64_t ints) { return static_cast<size_t>((ints * 4 + 255) / 256 * 256); };
    char *m = static_cast<char *>(scratch);
    int32_t *idx_a = reinterpret_cast<int32_t *>(m);
    int32_t *idx_b = reinterpret_cast<int32_t *>(m + al(D));
    int32_t *flag = reinterpret_cast<int32_t *>(m + 2 * al(D));
    int32_t *inv = reinterpret_cast<int32_t *>(m + 2 * al(D) + al(static_cast<int64_t>(n) * shape.max_width));
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((D + kTspThreads - 1) / kTspThreads,
                                                                          static_cast<int64_t>(sms) * 8)));
    cudaError_t e = cudaMemcpyAsync(layer_offsets, shape.layer_off.data(), sizeof(int32_t) * shape.layer_off.size(),
                                    cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
    tsp_init_kernel<<<grid, kTspThreads, 0, stream>>>(idx_a, D);
    int64_t nl = 1;
    int32_t *cur = idx_a, *next = idx_b;
    for (int l = 1; l < n; ++l) {
        const int32_t w_prev = shape.layer_off[l + 1] - shape.layer_off[l];
        const int32_t w_next = shape.layer_off[l + 2] - shape.layer_off[l + 1];
        const int64_t codes = static_cast<int64_t>(w_prev) * n;
        e = cudaMemsetAsync(flag, 0, sizeof(int32_t) * codes, stream);
        if (e != cudaSuccess) return e;
        tsp_code_kernel<<<grid, kTspThreads, 0, stream>>>(n, l, cur, next, flag, D, codes);
        tsp_rank_kernel<<<1, 1024, 0, stream>>>(flag, codes, w_next, err);
        tsp_assign_kernel<<<grid, kTspThreads, 0, stream>>>(next, flag, inv, D, w_next);
        const int32_t deg = l + 1 == 2 ? 1 : l - 1;
        const int fgrid = std::max(1, std::min((w_next + kTspThreads - 1) / kTspThreads, sms * 8));
        tsp_fill_kernel<<<fgrid, kTspThreads, 0, stream>>>(n, l, cur, inv, w_next, shape.layer_off[l],
                                                           shape.layer_off[l + 1], shape.arc_at[l + 1], deg,
                                                           in_arc_offsets, arc_src, arc_weight, err);
        nl += 4;
        std::swap(cur, next);
    }
    const int32_t w_n = shape.layer_off[n + 1] - shape.layer_off[n];
    const int egrid = std::max(1, std::min((w_n + kTspThreads - 1) / kTspThreads, sms * 8));
    tsp_ends_kernel<<<egrid, kTspThreads, 0, stream>>>(n, inv, w_n, shape.layer_off[n], shape.layer_off[n + 1],
                                                       shape.arc_at[n + 1], in_arc_offsets, arc_src, arc_weight);
    nl += 1;
    if (launches) *launches += nl;
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmdd
