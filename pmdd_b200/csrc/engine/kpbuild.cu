// Exact knapsack BDDs built on the device: see kpbuild.cuh for the construction.
#include <climits>

#include "kpbuild.cuh"
#include "scan.cuh"

namespace pmdd {
namespace dev {

namespace {

constexpr int NT = kKpThreads;

// In-place exclusive scan of a[0..m) by the whole block; returns the total (all threads).
__device__ int32_t block_scan_array(int32_t *a, int64_t m, int32_t *warp_buf, int32_t *total) {
    const int64_t chunk = (m + NT - 1) / NT;
    const int64_t b = threadIdx.x * chunk, e = min(m, b + chunk);
    int32_t sum = 0;
    for (int64_t i = b; i < e; ++i) sum += a[i];
    int32_t run = block_exclusive_scan<int32_t, NT>(sum, warp_buf, total);
    for (int64_t i = b; i < e; ++i) {
        const int32_t x = a[i];
        a[i] = run;
        run += x;
    }
    __syncthreads();
    return *total;
}

}  // namespace

__global__ void __launch_bounds__(NT) kp_reduce_kernel(const KpBuildJob *jobs) {
    const KpBuildJob &J = jobs[blockIdx.x];
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t total;
    __shared__ int32_t s_count;
    const int n = J.n, tid = threadIdx.x;
    const int64_t S = static_cast<int64_t>(J.cap) + 1;
    int32_t *key = J.tmp;              // [S]
    int32_t *flag = J.tmp + S;         // [2S]
    int32_t *remap_a = J.tmp + 3 * S;  // [S]
    int32_t *remap_b = J.tmp + 4 * S;  // [S]
    int32_t *st = J.tmp + 5 * S;       // [S] reachable states of a layer, ascending
    int32_t *r0j = J.tmp + 6 * S;      // [S]
    int32_t *r1j = J.tmp + 7 * S;      // [S]
    int32_t *head = J.tmp + 8 * S;     // [S]
    int32_t *minold = J.tmp + 9 * S;   // [S]

    // ---- top-down: reachable states and their first-seen numbering
    for (int64_t s = tid; s < S; s += NT) J.idx[s] = s == 0 ? 0 : -1;
    if (tid == 0) {
        J.width[0] = 1;
        J.width[n] = 1;
        *J.err = 0;
    }
    int32_t W = 1;
    for (int l = 0; l + 1 < n; ++l) {
        const int32_t *cur = J.idx + l * S;
        int32_t *nxt = J.idx + (l + 1) * S;
        const int32_t wl = J.w[l];
        for (int64_t f = tid; f < 2 * static_cast<int64_t>(W); f += NT) flag[f] = 0;
        __syncthreads();
        for (int64_t s = tid; s < S; s += NT) {
            int32_t k = INT_MAX;
            const int32_t a = cur[s];
            if (a >= 0) k = 2 * a;
            if (s >= wl) {
                const int32_t b = cur[s - wl];
                if (b >= 0) k = min(k, 2 * b + 1);
            }
            key[s] = k;
            if (k != INT_MAX) flag[k] = 1;
        }
        __syncthreads();
        W = block_scan_array(flag, 2 * static_cast<int64_t>(W), warp_buf, &total);
        for (int64_t s = tid; s < S; s += NT) nxt[s] = key[s] == INT_MAX ? -1 : flag[key[s]];
        if (tid == 0) J.width[l + 1] = W;
        __syncthreads();
    }

    // ---- bottom-up reduction
    int32_t *remap_next = remap_a, *remap_cur = remap_b;
    if (tid == 0) {
        remap_next[0] = 0;  // the terminal
        J.classes[n] = 1;
        J.arcs_into[0] = 0;
    }
    __syncthreads();
    for (int l = n - 1; l >= 0; --l) {
        const int32_t *cur = J.idx + l * S;
        const int32_t *nxt = l + 1 < n ? J.idx + (l + 1) * S : nullptr;
        const int32_t wl = J.w[l];
        const int32_t Wl = J.width[l];
        // a. reachable states in ascending order
        for (int64_t s = tid; s < S; s += NT) flag[s] = cur[s] >= 0 ? 1 : 0;
        __syncthreads();
        const int32_t cnt = block_scan_array(flag, S, warp_buf, &total);
        if (cnt != Wl && tid == 0) *J.err = 1;
        for (int64_t s = tid; s < S; s += NT)
            if (cur[s] >= 0 && flag[s] < Wl) st[flag[s]] = static_cast<int32_t>(s);
        __syncthreads();
        const int32_t Wc = min(cnt, Wl);
        // b. child classes of every state
        for (int32_t j = tid; j < Wc; j += NT) {
            const int32_t s = st[j];
            // both children of a reachable state are reachable (checked, never indexed at -1)
            int32_t c0old = nxt ? nxt[s] : 0, c1old = -1;
            if (static_cast<int64_t>(s) + wl <= J.cap) c1old = nxt ? nxt[s + wl] : 0;
            if (c0old < 0 || (c1old < 0 && static_cast<int64_t>(s) + wl <= J.cap)) {
                *J.err = 1;
                c0old = max(c0old, 0);
                c1old = static_cast<int64_t>(s) + wl <= J.cap ? max(c1old, 0) : -1;
            }
            r0j[j] = remap_next[c0old];
            r1j[j] = c1old >= 0 ? remap_next[c1old] : -1;
        }
        __syncthreads();
        // c. runs of equal (0-child, 1-child): one class each
        for (int32_t j = tid; j < Wc; j += NT) head[j] = (j == 0 || r0j[j] != r0j[j - 1] || r1j[j] != r1j[j - 1]) ? 1 : 0;
        __syncthreads();
        const int32_t K = block_scan_array(head, Wc, warp_buf, &total);
        int32_t *cnew = J.cls_new + l * S, *c0 = J.cls_c0 + l * S, *c1 = J.cls_c1 + l * S;
        for (int32_t c = tid; c < K; c += NT) minold[c] = INT_MAX;
        __syncthreads();
        // class of j = exclusive count of heads up to and including j, minus one
        for (int32_t j = tid; j < Wc; j += NT) {
            const bool h = j == 0 || r0j[j] != r0j[j - 1] || r1j[j] != r1j[j - 1];
            const int32_t c = head[j] + (h ? 0 : -1);
            atomicMin(&minold[c], cur[st[j]]);
            if (h) {
                c0[c] = r0j[j];
                c1[c] = r1j[j];
            }
        }
        __syncthreads();
        // d. number the classes by their first occurrence (smallest old index)
        for (int32_t x = tid; x < Wl; x += NT) flag[x] = 0;
        __syncthreads();
        for (int32_t c = tid; c < K; c += NT)
            if (minold[c] >= 0 && minold[c] < Wl) flag[minold[c]] = 1;
        __syncthreads();
        block_scan_array(flag, Wl, warp_buf, &total);
        for (int32_t c = tid; c < K; c += NT) cnew[c] = minold[c] >= 0 && minold[c] < Wl ? flag[minold[c]] : 0;
        __syncthreads();
        for (int32_t j = tid; j < Wc; j += NT) {
            const bool h = j == 0 || r0j[j] != r0j[j - 1] || r1j[j] != r1j[j - 1];
            const int32_t c = head[j] + (h ? 0 : -1);
            const int32_t old = cur[st[j]];
            if (old >= 0 && old < S) remap_cur[old] = cnew[c];
        }
        if (tid == 0) s_count = 0;
        __syncthreads();
        int32_t ones = 0;
        for (int32_t c = tid; c < K; c += NT) ones += c1[c] >= 0 ? 1 : 0;
        atomicAdd(&s_count, ones);
        __syncthreads();
        if (tid == 0) {
            J.classes[l] = K;
            J.arcs_into[l + 1] = K + s_count;
        }
        int32_t *t = remap_next;
        remap_next = remap_cur;
        remap_cur = t;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(NT) kp_flatten_kernel(const KpBuildJob *jobs) {
    extern __shared__ int32_t lo[];  // [n+2] layer offsets
    const KpBuildJob &J = jobs[blockIdx.x];
    __shared__ int32_t warp_buf[32];
    __shared__ int32_t total;
    const int n = J.n, d = J.nobjs, tid = threadIdx.x;
    const int64_t S = static_cast<int64_t>(J.cap) + 1;
    if (tid == 0) {
        int32_t acc = 0;
        for (int l = 0; l <= n; ++l) {
            lo[l] = acc;
            acc += J.classes[l];
        }
        lo[n + 1] = acc;
    }
    __syncthreads();
    for (int l = tid; l <= n + 1; l += NT) J.layer_offsets[l] = lo[l];
    for (int r = tid; r <= n; r += NT)
        for (int o = 0; o < d; ++o) J.weights[r * d + o] = r == 0 ? 0 : J.profit[o * n + (r - 1)];
    if (tid == 0) {
        J.in_arc_offsets[0] = 0;
        J.in_arc_offsets[1] = 0;  // the root has no incoming arcs
        J.min_weight[0] = 0;
    }
    int32_t *s1 = J.tmp, *e1 = J.tmp + S, *s0 = J.tmp + 2 * S, *e0 = J.tmp + 3 * S, *deg = J.tmp + 4 * S;
    int32_t arc_base = 0;
    __syncthreads();
    for (int l = 0; l < n; ++l) {
        const int32_t Kp = J.classes[l], Kc = J.classes[l + 1];
        const int32_t *cnew = J.cls_new + l * S, *c0 = J.cls_c0 + l * S, *c1 = J.cls_c1 + l * S;
        const int32_t wl = J.w[l];
        for (int32_t v = tid; v < Kc; v += NT) {
            s1[v] = -1;
            e1[v] = -1;
            s0[v] = -1;
            e0[v] = -1;
        }
        __syncthreads();
        // the parents of a child through one arc type are a run of classes in state order
        for (int32_t p = tid; p < Kp; p += NT) {
            const int32_t v1 = c1[p], v0 = c0[p];
            if (v1 >= 0 && v1 < Kc) {
                if (p == 0 || c1[p - 1] != v1) s1[v1] = p;
                if (p == Kp - 1 || c1[p + 1] != v1) e1[v1] = p;
            }
            if (v0 >= 0 && v0 < Kc) {
                if (p == 0 || c0[p - 1] != v0) s0[v0] = p;
                if (p == Kp - 1 || c0[p + 1] != v0) e0[v0] = p;
            }
        }
        __syncthreads();
        for (int32_t v = tid; v < Kc; v += NT)
            deg[v] = (s1[v] >= 0 ? e1[v] - s1[v] + 1 : 0) + (s0[v] >= 0 ? e0[v] - s0[v] + 1 : 0);
        __syncthreads();
        const int32_t layer_arcs = block_scan_array(deg, Kc, warp_buf, &total);
        for (int32_t v = tid; v < Kc; v += NT) {
            int32_t a = arc_base + deg[v];
            int32_t mw = INT_MAX;
#pragma unroll 1
            for (int t = 1; t >= 0; --t) {
                const int32_t sb = t ? s1[v] : s0[v], se = t ? e1[v] : e0[v];
                if (sb < 0) continue;
                const int32_t a0 = a;
                for (int32_t p = sb; p <= se; ++p) {
                    const int32_t u = cnew[p];
                    // insertion into [a0, a) kept ascending by parent id
                    int32_t q = a;
                    while (q > a0 && J.arc_src[q - 1] > lo[l] + u) {
                        J.arc_src[q] = J.arc_src[q - 1];
                        --q;
                    }
                    J.arc_src[q] = lo[l] + u;
                    J.arc_weight[a] = t ? 1 + l : 0;
                    mw = min(mw, J.min_weight[lo[l] + u] + (t ? wl : 0));
                    ++a;
                }
            }
            J.in_arc_offsets[lo[l + 1] + v + 1] = a;
            J.min_weight[lo[l + 1] + v] = mw == INT_MAX ? 0 : mw;
        }
        arc_base += layer_arcs;
        __syncthreads();
    }
    // min_weight order per layer (descending, ties by id): the reverse state order of the
    // classes, since a class's min_weight is its smallest reachable state
    for (int l = 0; l <= n; ++l) {
        const int32_t K = J.classes[l];
        if (l == n) {
            if (tid == 0) J.sd_order[lo[n]] = 0;
            break;
        }
        const int32_t *cnew = J.cls_new + l * S;
        for (int32_t p = tid; p < K; p += NT) {
            J.sd_order[lo[l] + (K - 1 - p)] = cnew[p];
            if (p + 1 < K && J.min_weight[lo[l] + cnew[p]] >= J.min_weight[lo[l] + cnew[p + 1]]) atomicMax(J.err, 2);
        }
    }
}

cudaError_t launch_kp_reduce(const KpBuildJob *jobs, int count, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    kp_reduce_kernel<<<count, NT, 0, stream>>>(jobs);
    return cudaGetLastError();
}

cudaError_t launch_kp_flatten(const KpBuildJob *jobs, int count, int max_layers, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const size_t smem = sizeof(int32_t) * (static_cast<size_t>(max_layers) + 2);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kp_flatten_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    kp_flatten_kernel<<<count, NT, smem, stream>>>(jobs);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace pmdd
