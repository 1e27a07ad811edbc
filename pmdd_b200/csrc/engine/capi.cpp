// extern "C" boundary of libpmdd_gpu.so (declared in include/pmdd.h).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <deque>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include "engine.hpp"
#include "kpbuild.cuh"
#include "tspbuild.cuh"
#include "pareto.cuh"
#include "pmdd.h"

namespace {

void write_err(char *err, size_t errlen, const std::string &msg) {
    if (err == nullptr || errlen == 0) return;
    const size_t n = std::min(errlen - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

// One engine per device for the one-shot, batch and resident entries, created on
// first use and kept for the life of the process (its arena is sized by
// PMDD_ARENA_BYTES, else PMDD_ARENA_FRACTION of the device's free memory, default a
// quarter).  `generation`
// changes whenever the engine is rebuilt after a CUDA failure, which invalidates
// resident DD sets made on the old one.
struct DeviceSlot {
    std::mutex mu;
    std::unique_ptr<pmdd::Engine> engine;
    uint64_t generation = 0;
};
std::mutex g_slots_mu;
std::unordered_map<int, std::unique_ptr<DeviceSlot>> g_slots;

DeviceSlot &slot_for(int device) {
    std::lock_guard<std::mutex> lk(g_slots_mu);
    auto &p = g_slots[device];
    if (!p) p.reset(new DeviceSlot);
    return *p;
}

int64_t default_arena_bytes(int device) {
    const char *env = std::getenv("PMDD_ARENA_BYTES");
    if (env && *env) {
        const long long v = std::atoll(env);
        if (v > 0) return v;
    }
    double frac = 0.25;
    const char *fenv = std::getenv("PMDD_ARENA_FRACTION");
    if (fenv && *fenv) {
        const double f = std::atof(fenv);
        if (f > 0.0 && f <= 0.95) frac = f;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    return static_cast<int64_t>(static_cast<double>(free_b) * frac);
}

// Caller holds slot.mu.
int ensure_engine(int device, DeviceSlot &slot, std::string *err) {
    if (slot.engine && slot.engine->ok()) {
        // the calling thread may have another device current
        if (!slot.engine->make_current()) {
            *err = slot.engine->error();
            return PMDD_ERR_CUDA;
        }
        return PMDD_OK;
    }
    slot.engine.reset(new pmdd::Engine(device, default_arena_bytes(device), 0));
    slot.generation++;
    if (!slot.engine->ok()) {
        *err = slot.engine->error();
        slot.engine.reset();
        return PMDD_ERR_NO_DEVICE;
    }
    return PMDD_OK;
}

int export_result(pmdd::Instance &I, pmdd_frontier *out, pmdd_stats *stats) {
    if (stats) *stats = I.stats;
    if (out) {
        out->nobjs = I.d;
        out->elem_bytes = static_cast<int32_t>(I.elem());
        out->num_points = I.result_n;
        out->points = nullptr;
        if (I.status == PMDD_OK) {
            const size_t bytes = std::max<size_t>(I.result.size(), 1);
            out->points = std::malloc(bytes);
            if (!out->points) return PMDD_ERR_OOM;
            if (!I.result.empty()) std::memcpy(out->points, I.result.data(), I.result.size());
        } else {
            out->num_points = 0;
        }
    }
    return I.status;
}

struct RunInfo {
    double device_elapsed_s = 0;
    int64_t launches = 0;
    double t_expand = 0, t_big = 0, t_rest = 0;  // kernel time of this call on the engine stream
    int64_t tile_launches = 0;
};

// Runs prepared requests to completion on the device's shared engine.  Caller holds
// slot.mu and has called ensure_engine.  With `ready`, request i is submitted only once
// ready(i) holds (its DD is being packed by other threads meanwhile); requests are
// submitted in order, and the engine steps on those already submitted.
int run_locked(DeviceSlot &slot, std::vector<std::unique_ptr<pmdd::Instance>> &reqs, RunInfo *info,
               std::string *err, const std::function<bool(size_t)> &ready = nullptr) {
    pmdd::Engine &E = *slot.engine;
    E.reset_mem_peak();  // the peak reported for this call is this call's
    const int64_t l0 = E.launches();
    const pmdd::KernelTimes k0 = E.kernel_times();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, E.stream());
    const size_t n = reqs.size();
    size_t next_submit = 0;
    auto submit_ready = [&]() {
        while (next_submit < n && (!ready || ready(next_submit))) {
            reqs[next_submit]->id = next_submit;
            E.submit(std::move(reqs[next_submit]));
            ++next_submit;
        }
    };
    size_t got = 0;
    int rc = PMDD_OK;
    while (got < n) {
        submit_ready();
        if (E.idle()) {  // every submitted request is done; the rest are still being packed
            std::this_thread::yield();
            continue;
        }
        const int r = E.step();
        while (!E.finished().empty()) {
            std::unique_ptr<pmdd::Instance> q = std::move(E.finished().front());
            E.finished().pop_front();
            const size_t at = static_cast<size_t>(q->id);
            reqs[at] = std::move(q);
            ++got;
        }
        if (r < 0) {
            *err = E.error();
            rc = PMDD_ERR_CUDA;
            break;
        }
    }
    if (rc == PMDD_OK) {
        cudaEventRecord(e1, E.stream());
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (info) {
            const pmdd::KernelTimes k1 = E.kernel_times();
            info->device_elapsed_s = ms * 1e-3;
            info->launches = E.launches() - l0;
            info->t_expand = k1.expand - k0.expand;
            info->t_big = k1.big - k0.big;
            info->t_rest = k1.rest - k0.rest;
            info->tile_launches = k1.tile_launches - k0.tile_launches;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != PMDD_OK) {
        // the engine is unusable: drop it so the next call starts clean
        for (auto &r : reqs)
            if (!r) r.reset(new pmdd::Instance);
        slot.engine.reset();
    }
    return rc;
}

// Validates every DD and lays it out, on the host threads; nothing is packed yet.
int prepare_all(const pmdd_dd *dds, int32_t count, const pmdd_options &o, bool with_out_csr,
                std::vector<std::unique_ptr<pmdd::Instance>> &reqs, int32_t *status, std::string *err) {
    reqs.resize(count);
    std::vector<int> rcs(count, PMDD_OK);
    std::vector<std::string> msgs(count);
    pmdd::parallel_for(count, pmdd::host_threads(), [&](int64_t i) {
        reqs[i].reset(new pmdd::Instance);
        rcs[i] = pmdd::prepare_instance(dds[i], o, static_cast<uint64_t>(i), reqs[i].get(), &msgs[i], with_out_csr,
                                        false);
    });
    for (int32_t i = 0; i < count; ++i) {
        if (rcs[i] != PMDD_OK) {
            *err = count > 1 ? "instance " + std::to_string(i) + ": " + msgs[i] : msgs[i];
            if (status) status[i] = rcs[i];
            return rcs[i];
        }
    }
    return PMDD_OK;
}

// Largest pinned staging the engine keeps for DD uploads; bigger sets are packed into
// per-instance pageable buffers instead.
constexpr size_t kMaxStagingBytes = size_t(4) << 30;

// Packs the prepared DDs, on the host threads, into the engine's pinned staging (one
// 256-byte aligned region per instance) so that each upload is one asynchronous DMA, or
// into per-instance host buffers when the staging cannot be had.  The caller holds
// slot.mu until the uploads have completed.
void pack_all(pmdd::Engine &E, const pmdd_dd *dds, std::vector<std::unique_ptr<pmdd::Instance>> &reqs) {
    const size_t n = reqs.size();
    std::vector<size_t> off(n + 1, 0);
    for (size_t i = 0; i < n; ++i) off[i + 1] = off[i] + ((reqs[i]->blob_bytes + 255) & ~static_cast<size_t>(255));
    unsigned char *st = off[n] > 0 && off[n] <= kMaxStagingBytes ? E.staging(off[n]) : nullptr;
    pmdd::parallel_for(static_cast<int64_t>(n), pmdd::host_threads(), [&](int64_t i) {
        pmdd::Instance &I = *reqs[i];
        if (st) {
            pmdd::pack_instance(dds[i], I, st + off[i]);
            I.blob_src = st + off[i];
        } else {
            I.blob.assign(I.blob_bytes, 0);
            pmdd::pack_instance(dds[i], I, I.blob.data());
        }
    });
}

// Packs (when `dds` is given) and runs prepared requests on the device's shared engine.
// The packing runs on host threads beside the engine: request i is submitted as soon as
// its DD sits in the pinned staging, so its upload and the first layers of the earlier
// requests overlap the packing of the later ones.
int run_on_device(int device, std::vector<std::unique_ptr<pmdd::Instance>> &reqs, RunInfo *info, std::string *err,
                  const pmdd_dd *dds = nullptr) {
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    const int rc = ensure_engine(device, slot, err);
    if (rc != PMDD_OK) return rc;
    if (!dds) return run_locked(slot, reqs, info, err);
    if (reqs.size() < 2) {
        pack_all(*slot.engine, dds, reqs);
        return run_locked(slot, reqs, info, err);
    }
    const size_t n = reqs.size();
    std::vector<size_t> off(n + 1, 0);
    for (size_t i = 0; i < n; ++i) off[i + 1] = off[i] + ((reqs[i]->blob_bytes + 255) & ~static_cast<size_t>(255));
    unsigned char *st = off[n] > 0 && off[n] <= kMaxStagingBytes ? slot.engine->staging(off[n]) : nullptr;
    std::vector<pmdd::Instance *> inst(n);
    for (size_t i = 0; i < n; ++i) inst[i] = reqs[i].get();
    std::unique_ptr<std::atomic<int>[]> packed(new std::atomic<int>[n]);
    for (size_t i = 0; i < n; ++i) packed[i].store(0, std::memory_order_relaxed);
    std::atomic<size_t> next(0);
    auto worker = [&]() {
        for (size_t i = next++; i < n; i = next++) {
            pmdd::Instance &I = *inst[i];
            if (st) {
                pmdd::pack_instance(dds[i], I, st + off[i]);
                I.blob_src = st + off[i];
            } else {
                I.blob.assign(I.blob_bytes, 0);
                pmdd::pack_instance(dds[i], I, I.blob.data());
            }
            packed[i].store(1, std::memory_order_release);
        }
    };
    const int threads = static_cast<int>(std::min<size_t>(static_cast<size_t>(pmdd::host_threads()), n));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    const int r = run_locked(slot, reqs, info, err,
                             [&](size_t i) { return packed[i].load(std::memory_order_acquire) != 0; });
    for (auto &th : pool) th.join();
    return r;
}

int collect_batch(std::vector<std::unique_ptr<pmdd::Instance>> &reqs, pmdd_frontier *outs, int32_t *status,
                  pmdd_stats *stats, const RunInfo &info, char *err, size_t errlen) {
    const int32_t count = static_cast<int32_t>(reqs.size());
    if (stats) {
        stats->device_elapsed_s = info.device_elapsed_s;
        stats->gpu_launches = info.launches;
        stats->kernel_expand_td_s = info.t_expand;
        stats->kernel_dominance_s = info.t_big;
        stats->kernel_total_s = info.t_expand + info.t_big + info.t_rest;
        stats->tile_launches = info.tile_launches;
    }
    int first_bad = PMDD_OK;
    for (int32_t i = 0; i < count; ++i) {
        pmdd_stats st;
        const int r = export_result(*reqs[i], outs ? &outs[i] : nullptr, &st);
        if (status) status[i] = r;
        if (r != PMDD_OK && first_bad == PMDD_OK) {
            first_bad = r;
            write_err(err, errlen, "instance " + std::to_string(i) + ": " + reqs[i]->error);
        }
        if (stats) {
            stats->work_candidates_total += st.work_candidates_total;
            stats->work_candidates_peak = std::max(stats->work_candidates_peak, st.work_candidates_peak);
            stats->work_frontier_survivors_total += st.work_frontier_survivors_total;
            stats->work_frontier_peak_points = std::max(stats->work_frontier_peak_points, st.work_frontier_peak_points);
            stats->work_join_products_total += st.work_join_products_total;
            stats->dominance_filtered_total += st.dominance_filtered_total;
            stats->work_tile_candidates_total += st.work_tile_candidates_total;
            stats->work_tile_survivors_total += st.work_tile_survivors_total;
            stats->work_stair_candidates_total += st.work_stair_candidates_total;
            stats->work_chained_layers += st.work_chained_layers;
            stats->gpu_mem_peak_used_bytes = std::max(stats->gpu_mem_peak_used_bytes, st.gpu_mem_peak_used_bytes);
            stats->gpu_mem_peak_reserved_bytes = st.gpu_mem_peak_reserved_bytes;
        }
    }
    return first_bad;
}

}  // namespace

extern "C" {

void pmdd_options_default(pmdd_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->method = 1;
    o->problem_type = 1;
    o->state_dominance = 0;
    o->maximization = 1;
    o->max_cand = 20000000LL;
    o->max_prod = 625000LL;
    o->device = 0;
}

void pmdd_frontier_free(pmdd_frontier *f) {
    if (!f) return;
    std::free(f->points);
    f->points = nullptr;
    f->num_points = 0;
}

int pmdd_enumerate(const pmdd_dd *dd, const pmdd_options *opts, pmdd_frontier *out, pmdd_stats *stats, char *err,
                   size_t errlen) {
    if (out) std::memset(out, 0, sizeof(*out));
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!dd) {
        write_err(err, errlen, "DD is NULL");
        return PMDD_ERR_INVALID;
    }
    pmdd_options o;
    if (opts) o = *opts;
    else pmdd_options_default(&o);
    std::vector<std::unique_ptr<pmdd::Instance>> reqs;
    std::string msg;
    const double t0 = pmdd::now_s();
    int rc = prepare_all(dd, 1, o, false, reqs, nullptr, &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    RunInfo info;
    rc = run_on_device(o.device, reqs, &info, &msg, dd);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    pmdd::Instance &I = *reqs[0];
    I.stats.wall_pack_transfer_s = I.admit_s - t0;
    I.stats.device_elapsed_s = info.device_elapsed_s;
    I.stats.gpu_launches = info.launches;
    I.stats.tile_launches = info.tile_launches;
    rc = export_result(I, out, stats);
    if (rc != PMDD_OK) write_err(err, errlen, I.error);
    return rc;
}

int pmdd_enumerate_batch(const pmdd_dd *dds, int32_t count, const pmdd_options *opts, pmdd_frontier *outs,
                         int32_t *status, pmdd_stats *stats, char *err, size_t errlen) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (count < 0 || (count > 0 && !dds)) {
        write_err(err, errlen, "invalid batch");
        return PMDD_ERR_INVALID;
    }
    pmdd_options o;
    if (opts) o = *opts;
    else pmdd_options_default(&o);
    if (outs)
        for (int32_t i = 0; i < count; ++i) std::memset(&outs[i], 0, sizeof(outs[i]));
    std::vector<std::unique_ptr<pmdd::Instance>> reqs;
    std::string msg;
    const auto t0 = std::chrono::steady_clock::now();
    int rc = prepare_all(dds, count, o, false, reqs, status, &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, count > 1 ? msg : "instance 0: " + msg);
        return rc;
    }
    const auto t1 = std::chrono::steady_clock::now();
    RunInfo info;
    rc = run_on_device(o.device, reqs, &info, &msg, dds);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    const auto t2 = std::chrono::steady_clock::now();
    rc = collect_batch(reqs, outs, status, stats, info, err, errlen);
    const char *tr = std::getenv("PMDD_TRACE");
    if (tr && tr[0] == '1') {
        const auto t3 = std::chrono::steady_clock::now();
        auto ms = [](std::chrono::steady_clock::duration d) { return std::chrono::duration<double, std::milli>(d).count(); };
        std::fprintf(stderr, "[pmdd batch] count=%d prepare_ms=%.1f run_ms=%.1f collect_ms=%.1f\n", count, ms(t1 - t0),
                     ms(t2 - t1), ms(t3 - t2));
    }
    return rc;
}

// ------------------------------------------------------- standalone filter
int pmdd_pareto_filter(const int32_t *points, int64_t num_points, int32_t nobjs, int32_t *out, int64_t *out_points,
                       int32_t device, char *err, size_t errlen) {
    if (out_points) *out_points = 0;
    if (nobjs < 1 || nobjs > 8 || num_points < 0 || num_points >= (static_cast<int64_t>(1) << 31) ||
        (num_points > 0 && (!points || !out)) || !out_points) {
        write_err(err, errlen, "invalid point set (nobjs 1..8, 0 <= num_points < 2^31, non-NULL buffers)");
        return PMDD_ERR_INVALID;
    }
    if (num_points == 0) return PMDD_OK;
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    std::string msg;
    if (ensure_engine(device, slot, &msg) != PMDD_OK) {
        write_err(err, errlen, msg);
        return PMDD_ERR_NO_DEVICE;
    }
    pmdd::Engine &E = *slot.engine;
    const size_t bytes = static_cast<size_t>(num_points) * nobjs * sizeof(int32_t);
    void *d_in = E.alloc(bytes), *d_out = E.alloc(bytes), *d_n = E.alloc(sizeof(int64_t));
    void *d_scratch = E.alloc(pmdd::dev::pareto_scratch_bytes(nobjs, num_points));
    int rc = PMDD_OK;
    if (!d_in || !d_out || !d_n || !d_scratch) {
        write_err(err, errlen, "point set does not fit the device memory budget");
        rc = PMDD_ERR_OOM;
    } else {
        cudaStream_t st = E.stream();
        cudaError_t e = cudaMemcpyAsync(d_in, points, bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = pmdd::dev::launch_pareto_filter(nobjs, static_cast<const int32_t *>(d_in), num_points, d_scratch,
                                                static_cast<int32_t *>(d_out), static_cast<int64_t *>(d_n), st);
        E.count_launches(1);
        int64_t n_out = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&n_out, d_n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && n_out > 0)
            e = cudaMemcpy(out, d_out, static_cast<size_t>(n_out) * nobjs * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            write_err(err, errlen, std::string("CUDA error: ") + cudaGetErrorString(e));
            rc = PMDD_ERR_CUDA;
        } else {
            *out_points = n_out;
        }
    }
    E.release(d_in);
    E.release(d_out);
    E.release(d_n);
    E.release(d_scratch);
    return rc;
}

// --------------------------------------------------------- resident DD sets
struct pmdd_resident {
    int device = 0;
    uint64_t generation = 0;
    int64_t bytes = 0;
    std::vector<std::unique_ptr<pmdd::Instance>> tmpl;  // prepared requests whose DD stays on the device
    std::vector<std::array<int64_t, 4>> widths;          // device-built DDs: original / reduced width and nodes
};

pmdd_resident *pmdd_resident_upload(const pmdd_dd *dds, int32_t count, int32_t device, char *err, size_t errlen) {
    if (count < 0 || (count > 0 && !dds)) {
        write_err(err, errlen, "invalid DD set");
        return nullptr;
    }
    std::unique_ptr<pmdd_resident> R(new pmdd_resident);
    R->device = device;
    pmdd_options o;
    pmdd_options_default(&o);
    std::string msg;
    if (prepare_all(dds, count, o, true, R->tmpl, nullptr, &msg) != PMDD_OK) {
        write_err(err, errlen, count > 1 ? msg : "instance 0: " + msg);
        return nullptr;
    }
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    if (ensure_engine(device, slot, &msg) != PMDD_OK) {
        write_err(err, errlen, msg);
        return nullptr;
    }
    R->generation = slot.generation;
    pack_all(*slot.engine, dds, R->tmpl);
    for (size_t i = 0; i < R->tmpl.size(); ++i) {
        pmdd::Instance &I = *R->tmpl[i];
        if (!slot.engine->upload_dd(I)) {
            for (size_t k = 0; k <= i; ++k) slot.engine->release_dd(*R->tmpl[k]);
            write_err(err, errlen, slot.engine->ok() ? "DD set does not fit the device memory budget"
                                                     : slot.engine->error());
            return nullptr;
        }
        R->bytes += static_cast<int64_t>(I.dev_bytes);
    }
    if (cudaStreamSynchronize(slot.engine->stream()) != cudaSuccess) {
        write_err(err, errlen, "DD upload failed");
        return nullptr;
    }
    for (auto &I : R->tmpl) {
        I->blob.clear();
        I->blob.shrink_to_fit();
        I->blob_src = nullptr;
        std::vector<int32_t>().swap(I->sd_order);
        std::vector<int32_t>().swap(I->sd_next);
    }
    return R.release();
}

int pmdd_resident_enumerate(pmdd_resident *R, const pmdd_options *opts, pmdd_frontier *outs, int32_t *status,
                            pmdd_stats *stats, char *err, size_t errlen) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!R) {
        write_err(err, errlen, "resident set is NULL");
        return PMDD_ERR_INVALID;
    }
    pmdd_options o;
    if (opts) o = *opts;
    else pmdd_options_default(&o);
    if (o.method != 1 && o.method != 3) {
        write_err(err, errlen, "method must be 1 (top-down) or 3 (coupled) on the GPU backend");
        return PMDD_ERR_INVALID;
    }
    DeviceSlot &slot = slot_for(R->device);
    std::lock_guard<std::mutex> lk(slot.mu);
    if (!slot.engine || !slot.engine->ok() || slot.generation != R->generation) {
        write_err(err, errlen, "resident DD set was invalidated by an engine restart");
        return PMDD_ERR_CUDA;
    }
    std::vector<std::unique_ptr<pmdd::Instance>> reqs;
    reqs.reserve(R->tmpl.size());
    for (size_t i = 0; i < R->tmpl.size(); ++i) {
        const pmdd::Instance &T = *R->tmpl[i];
        std::unique_ptr<pmdd::Instance> I(new pmdd::Instance);
        I->opts = o;
        I->d = T.d;
        I->wide = T.wide;
        I->L = T.L;
        I->N = T.N;
        I->A = T.A;
        I->K = T.K;
        I->layer_off = T.layer_off;
        I->arc_at_layer = T.arc_at_layer;
        I->off_layer = T.off_layer;
        I->off_in = T.off_in;
        I->off_src = T.off_src;
        I->off_w = T.off_w;
        I->off_weights = T.off_weights;
        I->off_minw = T.off_minw;
        I->blob_bytes = T.blob_bytes;
        I->dev_bytes = T.dev_bytes;
        I->dd = T.dd;
        I->d_in_off = T.d_in_off;
        I->d_arc_src = T.d_arc_src;
        I->d_arc_w = T.d_arc_w;
        I->d_weights = T.d_weights;
        I->has_sd_order = T.has_sd_order;
        I->sd_kind = T.sd_kind;
        I->state_words = T.state_words;
        I->off_sdord = T.off_sdord;
        I->off_sdnext = T.off_sdnext;
        I->off_state = T.off_state;
        I->d_sd_order = T.d_sd_order;
        I->d_sd_next = T.d_sd_next;
        I->d_state = T.d_state;
        I->d_out_off = T.d_out_off;
        I->d_out_head = T.d_out_head;
        I->d_out_w = T.d_out_w;
        I->d_cursor = T.d_cursor;
        I->external_dd = true;
        I->tsp = T.tsp;
        I->with_out_csr = T.with_out_csr;
        I->min_bytes = 0;  // the DD is resident already
        I->max_layer_arcs = T.max_layer_arcs;
        I->max_layer_nodes = T.max_layer_nodes;
        I->submit_s = pmdd::now_s();
        reqs.push_back(std::move(I));
    }
    RunInfo info;
    std::string msg;
    const int rc = run_locked(slot, reqs, &info, &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    for (int32_t i = 0; i < static_cast<int32_t>(reqs.size()); ++i)
        if (outs) std::memset(&outs[i], 0, sizeof(outs[i]));
    return collect_batch(reqs, outs, status, stats, info, err, errlen);
}

int64_t pmdd_resident_bytes(const pmdd_resident *R) { return R ? R->bytes : 0; }

void pmdd_resident_free(pmdd_resident *R) {
    if (!R) return;
    DeviceSlot &slot = slot_for(R->device);
    {
        std::lock_guard<std::mutex> lk(slot.mu);
        if (slot.engine && slot.generation == R->generation)
            for (auto &I : R->tmpl) slot.engine->release_dd(*I);
    }
    delete R;
}

// ------------------------------------------------- knapsack BDDs built on the device
namespace {
constexpr int32_t kBuildMaxItems = 4096;
constexpr int32_t kBuildMaxCap = 1 << 24;
constexpr int64_t kBuildScratchBytes = static_cast<int64_t>(2) << 30;  // per chunk of instances
}  // namespace

pmdd_resident *pmdd_resident_build_knapsack(const pmdd_knapsack *ks, int32_t count, int32_t device, char *err,
                                            size_t errlen) {
    if (count < 0 || (count > 0 && !ks)) {
        write_err(err, errlen, "invalid knapsack set");
        return nullptr;
    }
    for (int32_t i = 0; i < count; ++i) {
        const pmdd_knapsack &k = ks[i];
        std::string why;
        if (k.n < 1 || k.n > kBuildMaxItems) why = "n must be in 1..4096";
        else if (k.nobjs < 1 || k.nobjs > 8) why = "nobjs must be in 1..8";
        else if (!k.profits || !k.weights) why = "profits / weights pointer is NULL";
        else if (k.capacity < 0 || k.capacity > kBuildMaxCap) why = "capacity must be in 0..2^24";
        else
            for (int32_t j = 0; j < k.n && why.empty(); ++j)
                if (k.weights[j] < 0) why = "weights must be >= 0";
        if (!why.empty()) {
            write_err(err, errlen, "instance " + std::to_string(i) + ": " + why);
            return nullptr;
        }
    }
    std::unique_ptr<pmdd_resident> R(new pmdd_resident);
    R->device = device;
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    std::string msg;
    if (ensure_engine(device, slot, &msg) != PMDD_OK) {
        write_err(err, errlen, msg);
        return nullptr;
    }
    R->generation = slot.generation;
    pmdd::Engine &E = *slot.engine;
    cudaStream_t st = E.stream();
    std::vector<void *> temps;
    auto give_up = [&](const std::string &why) -> pmdd_resident * {
        cudaStreamSynchronize(st);
        for (void *p : temps) E.release(p);
        for (auto &I : R->tmpl)
            if (I->dd) E.release_dd(*I);
        write_err(err, errlen, why);
        return nullptr;
    };
    auto dev_alloc = [&](size_t bytes) -> void * {
        void *p = E.alloc(std::max<size_t>(bytes, 256));
        if (p) temps.push_back(p);
        return p;
    };
    // item weights and profits of every instance, one upload
    std::vector<size_t> in_off(count + 1, 0);
    for (int32_t i = 0; i < count; ++i) in_off[i + 1] = in_off[i] + static_cast<size_t>(ks[i].n) * (1 + ks[i].nobjs);
    std::vector<int32_t> hin(std::max<size_t>(in_off[count], 1));
    for (int32_t i = 0; i < count; ++i) {
        std::memcpy(&hin[in_off[i]], ks[i].weights, sizeof(int32_t) * ks[i].n);
        std::memcpy(&hin[in_off[i] + ks[i].n], ks[i].profits, sizeof(int32_t) * ks[i].n * ks[i].nobjs);
    }
    int32_t *d_in = static_cast<int32_t *>(dev_alloc(sizeof(int32_t) * hin.size()));
    if (!d_in) return give_up("knapsack inputs do not fit the device memory budget");
    if (cudaMemcpyAsync(d_in, hin.data(), sizeof(int32_t) * hin.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return give_up("knapsack input upload failed");
    auto scratch_bytes = [&](int32_t i) { return sizeof(int32_t) * pmdd::dev::kp_scratch_ints(ks[i].n, ks[i].capacity); };
    for (int32_t i0 = 0; i0 < count;) {
        int32_t i1 = i0;
        int64_t acc = 0;
        while (i1 < count && (i1 == i0 || acc + static_cast<int64_t>(scratch_bytes(i1)) <= kBuildScratchBytes)) {
            acc += static_cast<int64_t>(scratch_bytes(i1)) + 256;
            ++i1;
        }
        const int32_t m = i1 - i0;
        std::vector<size_t> hdr_off(m + 1, 0), scr_off(m + 1, 0);
        int max_layers = 0;
        for (int32_t k = 0; k < m; ++k) {
            const pmdd_knapsack &q = ks[i0 + k];
            hdr_off[k + 1] = hdr_off[k] + 3 * (static_cast<size_t>(q.n) + 1) + 1;
            scr_off[k + 1] = scr_off[k] + (scratch_bytes(i0 + k) + 255) / 256 * 64;  // ints, 256-byte aligned
            max_layers = std::max(max_layers, q.n + 1);
        }
        int32_t *d_scr = static_cast<int32_t *>(dev_alloc(sizeof(int32_t) * scr_off[m]));
        int32_t *d_hdr = static_cast<int32_t *>(dev_alloc(sizeof(int32_t) * hdr_off[m]));
        auto *d_jobs = static_cast<pmdd::dev::KpBuildJob *>(dev_alloc(sizeof(pmdd::dev::KpBuildJob) * m));
        if (!d_scr || !d_hdr || !d_jobs) return give_up("knapsack build scratch does not fit the device memory budget");
        std::vector<pmdd::dev::KpBuildJob> jobs(m);
        for (int32_t k = 0; k < m; ++k) {
            const pmdd_knapsack &q = ks[i0 + k];
            pmdd::dev::KpBuildJob &J = jobs[k];
            std::memset(&J, 0, sizeof(J));
            const int64_t S = static_cast<int64_t>(q.capacity) + 1, Lc = q.n + 1;
            J.n = q.n;
            J.cap = q.capacity;
            J.nobjs = q.nobjs;
            J.w = d_in + in_off[i0 + k];
            J.profit = d_in + in_off[i0 + k] + q.n;
            int32_t *base = d_scr + scr_off[k];
            J.idx = base;
            J.cls_new = base + Lc * S;
            J.cls_c0 = base + 2 * Lc * S;
            J.cls_c1 = base + 3 * Lc * S;
            J.tmp = base + 4 * Lc * S;
            int32_t *h = d_hdr + hdr_off[k];
            J.width = h;
            J.classes = h + Lc;
            J.arcs_into = h + 2 * Lc;
            J.err = h + 3 * Lc;
        }
        std::vector<int32_t> hhdr(hdr_off[m]);
        if (cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(jobs[0]) * m, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            pmdd::dev::launch_kp_reduce(d_jobs, m, st) != cudaSuccess ||
            cudaMemcpyAsync(hhdr.data(), d_hdr, sizeof(int32_t) * hhdr.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return give_up(std::string("knapsack build failed: ") + cudaGetErrorString(cudaGetLastError()));
        E.count_launches(1);
        for (int32_t k = 0; k < m; ++k) {
            const pmdd_knapsack &q = ks[i0 + k];
            const int32_t Lc = q.n + 1;
            const int32_t *h = hhdr.data() + hdr_off[k];
            if (h[3 * Lc] != 0) return give_up("knapsack build: inconsistent layer counts (internal)");
            std::vector<int32_t> layer_off(Lc + 1, 0), arc_at(Lc + 1, 0);
            int64_t ow = 0, on = 0, rw = 0, rn = 0;
            // header: width[Lc] | classes[Lc] | arcs_into[Lc] | err
            for (int32_t l = 0; l < Lc; ++l) {
                layer_off[l + 1] = layer_off[l] + h[Lc + l];
                arc_at[l + 1] = arc_at[l] + h[2 * Lc + l];
                ow = std::max<int64_t>(ow, h[l]);
                on += h[l];
                rw = std::max<int64_t>(rw, h[Lc + l]);
                rn += h[Lc + l];
            }
            // bound on |path sums| as prepare_instance computes it: a layer with a 1-arc adds
            // its largest |profit|
            int64_t bound = 0;
            for (int32_t l = 0; l < q.n; ++l) {
                if (q.weights[l] > q.capacity) continue;
                int64_t mx = 0;
                for (int o = 0; o < q.nobjs; ++o) mx = std::max<int64_t>(mx, std::llabs(static_cast<int64_t>(q.profits[o * q.n + l])));
                bound += mx;
            }
            std::unique_ptr<pmdd::Instance> I(new pmdd::Instance);
            pmdd_options_default(&I->opts);
            I->opts.problem_type = 1;
            I->id = static_cast<uint64_t>(i0 + k);
            pmdd::layout_built_knapsack(I.get(), q.nobjs, bound > static_cast<int64_t>(INT32_MAX), layer_off, arc_at,
                                        q.n + 1);
            I->dd = static_cast<unsigned char *>(E.alloc(I->dev_bytes));
            if (!I->dd) return give_up("built DD set does not fit the device memory budget");
            pmdd::dev::KpBuildJob &J = jobs[k];
            J.layer_offsets = reinterpret_cast<int32_t *>(I->dd + I->off_layer);
            J.in_arc_offsets = reinterpret_cast<int32_t *>(I->dd + I->off_in);
            J.arc_src = reinterpret_cast<int32_t *>(I->dd + I->off_src);
            J.arc_weight = reinterpret_cast<int32_t *>(I->dd + I->off_w);
            J.weights = reinterpret_cast<int32_t *>(I->dd + I->off_weights);
            J.min_weight = reinterpret_cast<int32_t *>(I->dd + I->off_minw);
            J.sd_order = reinterpret_cast<int32_t *>(I->dd + I->off_sdord);
            R->bytes += static_cast<int64_t>(I->dev_bytes);
            R->tmpl.push_back(std::move(I));
            R->widths.push_back({ow, on, rw, rn});
        }
        if (cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(jobs[0]) * m, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            pmdd::dev::launch_kp_flatten(d_jobs, m, max_layers, st) != cudaSuccess)
            return give_up(std::string("knapsack flatten failed: ") + cudaGetErrorString(cudaGetLastError()));
        E.count_launches(1);
        for (int32_t k = 0; k < m; ++k)
            if (!E.bind_dd(*R->tmpl[i0 + k])) return give_up(E.ok() ? "out-arc CSR failed" : E.error());
        if (cudaMemcpyAsync(hhdr.data(), d_hdr, sizeof(int32_t) * hhdr.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return give_up(std::string("knapsack build failed: ") + cudaGetErrorString(cudaGetLastError()));
        for (int32_t k = 0; k < m; ++k)
            if (hhdr[hdr_off[k] + 3 * (ks[i0 + k].n + 1)] != 0)
                return give_up("knapsack build: min_weight order check failed (internal)");
        E.release(d_scr);
        E.release(d_hdr);
        E.release(d_jobs);
        temps.erase(std::remove_if(temps.begin(), temps.end(),
                                   [&](void *p) { return p == d_scr || p == d_hdr || p == d_jobs; }),
                    temps.end());
        i0 = i1;
    }
    cudaStreamSynchronize(st);
    for (void *p : temps) E.release(p);
    return R.release();
}

pmdd_resident *pmdd_resident_build_tsp(const pmdd_tsp *ts, int32_t count, int32_t device, char *err, size_t errlen) {
    if (count < 0 || (count > 0 && !ts)) {
        write_err(err, errlen, "invalid TSP set");
        return nullptr;
    }
    for (int32_t i = 0; i < count; ++i) {
        std::string why;
        if (ts[i].n < pmdd::dev::kTspMinCities || ts[i].n > pmdd::dev::kTspMaxCities) why = "n must be in 2..20";
        else if (ts[i].nobjs < 1 || ts[i].nobjs > 8) why = "nobjs must be in 1..8";
        else if (!ts[i].cost) why = "cost pointer is NULL";
        if (!why.empty()) {
            write_err(err, errlen, "instance " + std::to_string(i) + ": " + why);
            return nullptr;
        }
    }
    std::unique_ptr<pmdd_resident> R(new pmdd_resident);
    R->device = device;
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    std::string msg;
    if (ensure_engine(device, slot, &msg) != PMDD_OK) {
        write_err(err, errlen, msg);
        return nullptr;
    }
    R->generation = slot.generation;
    pmdd::Engine &E = *slot.engine;
    pmdd_options o;
    pmdd_options_default(&o);
    o.problem_type = 3;
    for (int32_t i = 0; i < count; ++i) {
        const pmdd::TspStructure *S = E.tsp_structure(ts[i].n, &msg);
        std::unique_ptr<pmdd::Instance> I(new pmdd::Instance);
        if (S) pmdd::prepare_tsp_instance(*S, ts[i].nobjs, ts[i].cost, o, static_cast<uint64_t>(i), I.get());
        if (!S || !E.upload_dd(*I)) {
            if (I->dd) E.release_dd(*I);
            for (auto &T : R->tmpl) E.release_dd(*T);
            write_err(err, errlen, S ? "TSP set does not fit the device memory budget" : msg);
            return nullptr;
        }
        R->bytes += static_cast<int64_t>(I->dev_bytes);
        R->tmpl.push_back(std::move(I));
    }
    if (cudaStreamSynchronize(E.stream()) != cudaSuccess) {
        for (auto &T : R->tmpl) E.release_dd(*T);
        write_err(err, errlen, "TSP weight upload failed");
        return nullptr;
    }
    for (auto &I : R->tmpl) {
        I->blob.clear();
        I->blob.shrink_to_fit();
    }
    return R.release();
}

int pmdd_resident_dd_shape(const pmdd_resident *R, int32_t i, int32_t *shape, int64_t *widths) {
    if (!R || i < 0 || i >= static_cast<int32_t>(R->tmpl.size())) return PMDD_ERR_INVALID;
    const pmdd::Instance &T = *R->tmpl[i];
    if (shape) {
        shape[0] = T.d;
        shape[1] = T.L;
        shape[2] = T.N;
        shape[3] = T.A;
        shape[4] = T.K;
    }
    if (widths)
        for (int k = 0; k < 4; ++k) widths[k] = i < static_cast<int32_t>(R->widths.size()) ? R->widths[i][k] : -1;
    return PMDD_OK;
}

int pmdd_resident_dd_copy(pmdd_resident *R, int32_t i, int32_t *layer_offsets, int32_t *in_arc_offsets,
                          int32_t *arc_src, int32_t *arc_weight, int32_t *weights, int32_t *min_weight, char *err,
                          size_t errlen) {
    if (!R || i < 0 || i >= static_cast<int32_t>(R->tmpl.size()) || !layer_offsets || !in_arc_offsets ||
        !weights || ((!arc_src || !arc_weight) && R->tmpl[i]->A > 0)) {
        write_err(err, errlen, "invalid resident DD copy");
        return PMDD_ERR_INVALID;
    }
    DeviceSlot &slot = slot_for(R->device);
    std::lock_guard<std::mutex> lk(slot.mu);
    if (!slot.engine || !slot.engine->ok() || slot.generation != R->generation) {
        write_err(err, errlen, "resident DD set was invalidated by an engine restart");
        return PMDD_ERR_CUDA;
    }
    const pmdd::Instance &T = *R->tmpl[i];
    if (!slot.engine->make_current()) {
        write_err(err, errlen, slot.engine->error());
        return PMDD_ERR_CUDA;
    }
    cudaStream_t st = slot.engine->stream();
    auto get = [&](void *dst, const void *src, size_t bytes) {
        return bytes == 0 || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    };
    std::memcpy(layer_offsets, T.layer_off.data(), sizeof(int32_t) * (static_cast<size_t>(T.L) + 1));
    bool ok = get(in_arc_offsets, T.d_in_off, sizeof(int32_t) * (static_cast<size_t>(T.N) + 1)) &&
              get(arc_src, T.d_arc_src, sizeof(int32_t) * static_cast<size_t>(T.A)) &&
              get(arc_weight, T.d_arc_w, sizeof(int32_t) * static_cast<size_t>(T.A)) &&
              get(weights, T.d_weights, sizeof(int32_t) * static_cast<size_t>(T.K) * T.d);
    if (ok && min_weight && T.sd_kind == 1)
        ok = get(min_weight, T.dd + T.off_minw, sizeof(int32_t) * static_cast<size_t>(T.N));
    if (!ok || cudaStreamSynchronize(st) != cudaSuccess) {
        write_err(err, errlen, std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
        return PMDD_ERR_CUDA;
    }
    return PMDD_OK;
}

// ------------------------------------------------------------------ serving
// A server runs two lanes, each an engine of its own (memory budget, CUDA stream).
// Requests predicted to be small (heavy_request below: by DD arcs) go to the light lane, whose
// stream has the device's highest priority and which the caller's thread steps inside
// pmdd_server_run; the others go to the heavy lane, which a worker thread steps on its
// own whenever it has work.  A small request then waits neither for a step of a large
// one on the host nor behind its queued blocks on the GPU.  The heavy lane's engine is
// touched only by its worker: the caller posts submissions, cancellations and
// failure-injection settings as commands, and reads results and counters that the
// worker publishes after every step.  PMDD_SERVER_LANES=1 keeps a single lane.
namespace {

struct HeavyLane {
    std::unique_ptr<pmdd::Engine> engine;
    std::thread worker;
    std::mutex mu;                                   // guards everything below
    std::condition_variable wake;                    // the worker: commands, or stop
    std::condition_variable done;                    // the caller: a result, or idle
    std::vector<std::function<void(pmdd::Engine &)>> cmds;
    int64_t inbox_requests = 0;                      // submissions posted and not yet published
                                                     // as queued or running
    std::deque<std::unique_ptr<pmdd::Instance>> outbox;
    // published by the worker after each pass
    size_t queued = 0, running = 0;
    pmdd::Engine::Counters counters{};
    int64_t budget = 0, used = 0, peak = 0, growth = 0, injected = 0;
    bool stop = false, failed = false, working = false;
    std::string error;
    int64_t posted_requests = 0;                     // submissions among cmds (the worker's share)

    void post(std::function<void(pmdd::Engine &)> fn, bool request) {
        {
            std::lock_guard<std::mutex> lk(mu);
            cmds.push_back(std::move(fn));
            if (request) {
                ++inbox_requests;
                ++posted_requests;
            }
        }
        wake.notify_one();
    }
    bool busy_locked() const { return !cmds.empty() || working || queued + running > 0; }

    void publish_locked() {
        pmdd::Engine &E = *engine;
        while (!E.finished().empty()) {
            outbox.push_back(std::move(E.finished().front()));
            E.finished().pop_front();
        }
        queued = E.queued();
        running = E.running();
        counters = E.counters();
        budget = static_cast<int64_t>(E.arena().capacity());
        used = static_cast<int64_t>(E.arena().used());
        peak = static_cast<int64_t>(E.arena().peak());
        growth = E.reserved_growth();
        injected = E.arena().injected_failures();
    }

    void run_worker() {
        for (;;) {
            std::vector<std::function<void(pmdd::Engine &)>> batch;
            int64_t batch_requests = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                wake.wait(lk, [&] { return stop || !cmds.empty() || (!failed && !engine->idle()); });
                if (stop) return;
                batch.swap(cmds);
                batch_requests = posted_requests;
                posted_requests = 0;
                working = true;
            }
            for (auto &fn : batch) fn(*engine);
            int rc = 0;
            if (!failed && !engine->idle()) rc = engine->step();
            {
                std::lock_guard<std::mutex> lk(mu);
                if (rc < 0) {
                    failed = true;
                    error = engine->error();
                }
                publish_locked();
                inbox_requests -= batch_requests;  // now counted by the engine (or finished)
                working = false;
            }
            done.notify_all();
        }
    }

    ~HeavyLane() {
        if (worker.joinable()) {
            {
                std::lock_guard<std::mutex> lk(mu);
                stop = true;
            }
            wake.notify_all();
            worker.join();
        }
    }
};

}  // namespace

struct pmdd_server {
    std::unique_ptr<pmdd::Engine> engine;  // the light lane, or the only one
    std::unique_ptr<HeavyLane> heavy;      // nullptr: one lane
    std::deque<std::unique_ptr<pmdd::Instance>> ready;  // heavy-lane results handed over by run
    std::unordered_map<uint64_t, int> heavy_ids;
    uint64_t submitted = 0;
    int64_t heavy_arcs = int64_t(1) << 17;
};

namespace {

// A request goes to the heavy lane when its DD has more than srv->heavy_arcs arcs
// (PMDD_SERVER_HEAVY_ARCS, default 2^17).  On the served mix (knapsack n 20..60, set
// packing n 60..100, TSP 9..13 cities, three objectives) a request's lone latency grows
// with its arcs: the 2^17 limit leaves requests of at most ~3 ms alone in the light lane
// and sends the larger knapsacks (median ~6 ms alone, up to ~30 ms) to the heavy one.
bool heavy_request(const pmdd_server *srv, int64_t arcs) {
    return srv->heavy != nullptr && arcs > srv->heavy_arcs;
}

}  // namespace

pmdd_server *pmdd_server_create(int32_t device, int64_t budget_bytes, int32_t max_slots, char *err, size_t errlen) {
    std::unique_ptr<pmdd_server> s(new pmdd_server);
    if (budget_bytes <= 0) budget_bytes = default_arena_bytes(device);
    const char *lanes = std::getenv("PMDD_SERVER_LANES");
    // two lanes need a budget worth splitting (an engine takes at least 64 MB)
    const bool two = !(lanes && lanes[0] == '1') && budget_bytes >= (int64_t(512) << 20);
    const char *ha = std::getenv("PMDD_SERVER_HEAVY_ARCS");
    if (ha && *ha) s->heavy_arcs = std::max<long long>(0, std::atoll(ha));
    int prio_low = 0, prio_high = 0;
    if (two && (cudaSetDevice(device) != cudaSuccess ||
                cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess)) {
        write_err(err, errlen, std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError()));
        return nullptr;
    }
    // the light lane: a quarter of the budget, but at least half of it up to 512 MB
    const int64_t light = two ? std::max<int64_t>(budget_bytes / 4, std::min<int64_t>(budget_bytes / 2, int64_t(512) << 20))
                              : budget_bytes;
    s->engine.reset(new pmdd::Engine(device, light, max_slots, two ? prio_high : 0));
    if (!s->engine->ok()) {
        write_err(err, errlen, s->engine->error());
        return nullptr;
    }
    if (two) {
        s->heavy.reset(new HeavyLane);
        s->heavy->engine.reset(new pmdd::Engine(device, budget_bytes - light, max_slots, prio_low));
        if (!s->heavy->engine->ok()) {
            write_err(err, errlen, s->heavy->engine->error());
            return nullptr;
        }
        {
            std::lock_guard<std::mutex> lk(s->heavy->mu);
            s->heavy->publish_locked();
        }
        HeavyLane *h = s->heavy.get();
        h->worker = std::thread([h] { h->run_worker(); });
    }
    return s.release();
}

int pmdd_server_submit(pmdd_server *srv, const pmdd_dd *dd, const pmdd_options *opts, uint64_t req_id) {
    if (!srv || !dd) return PMDD_ERR_INVALID;
    pmdd_options o;
    if (opts) o = *opts;
    else pmdd_options_default(&o);
    std::unique_ptr<pmdd::Instance> I(new pmdd::Instance);
    std::string msg;
    const int rc = pmdd::prepare_instance(*dd, o, req_id, I.get(), &msg);
    if (rc != PMDD_OK) {
        I->id = req_id;
        I->status = rc;
        I->error = msg;
        srv->engine->finish_rejected(std::move(I));
        return rc;
    }
    if (heavy_request(srv, I->A)) {
        srv->heavy_ids[req_id] = 1;
        auto holder = std::make_shared<std::unique_ptr<pmdd::Instance>>(std::move(I));
        srv->heavy->post([holder](pmdd::Engine &E) { E.submit(std::move(*holder)); }, true);
    } else {
        srv->engine->submit(std::move(I));
    }
    srv->submitted++;
    return PMDD_OK;
}

namespace {

// A TSP request on one lane's engine (its shared n-city structure); the caller checked
// the arguments.
void submit_tsp_on(pmdd::Engine &E, int n, int nobjs, const int32_t *cost, const pmdd_options &o, uint64_t req_id) {
    std::string msg;
    const pmdd::TspStructure *S = E.tsp_structure(n, &msg);
    std::unique_ptr<pmdd::Instance> I(new pmdd::Instance);
    if (!S) {
        I->id = req_id;
        I->status = PMDD_ERR_OOM;
        I->error = msg;
        E.finish_rejected(std::move(I));
        return;
    }
    pmdd::prepare_tsp_instance(*S, nobjs, cost, o, req_id, I.get());
    E.submit(std::move(I));
}

}  // namespace

int pmdd_server_submit_tsp(pmdd_server *srv, const pmdd_tsp *t, const pmdd_options *opts, uint64_t req_id) {
    if (!srv || !t || !t->cost || t->n < pmdd::dev::kTspMinCities || t->n > pmdd::dev::kTspMaxCities ||
        t->nobjs < 1 || t->nobjs > 8)
        return PMDD_ERR_INVALID;
    pmdd_options o;
    if (opts) o = *opts;
    else pmdd_options_default(&o);
    o.problem_type = 3;
    if ((o.method != 1 && o.method != 3) || o.maximization == 0) return PMDD_ERR_INVALID;
    // arcs of the n-city MDD, about: layer l (1..n-1) holds C(n-1, l) visited sets times
    // l last cities, each state of layer l >= 2 with l - 1 parents
    int64_t arcs = 0;
    for (int l = 1; l < t->n; ++l) {
        int64_t c = 1;
        for (int k = 1; k <= l; ++k) c = c * (t->n - k) / k;  // C(n - 1, l), exact step by step
        arcs += c * l * std::max(1, l - 1);
    }
    if (heavy_request(srv, arcs)) {
        srv->heavy_ids[req_id] = 1;
        const int n = t->n, nobjs = t->nobjs;
        auto cost = std::make_shared<std::vector<int32_t>>(t->cost, t->cost + static_cast<size_t>(nobjs) * n * n);
        srv->heavy->post([n, nobjs, cost, o, req_id](pmdd::Engine &E) { submit_tsp_on(E, n, nobjs, cost->data(), o, req_id); },
                         true);
    } else {
        submit_tsp_on(*srv->engine, t->n, t->nobjs, t->cost, o, req_id);
    }
    srv->submitted++;
    return PMDD_OK;
}

int pmdd_server_prepare_tsp(pmdd_server *srv, int32_t n) {
    if (!srv || n < pmdd::dev::kTspMinCities || n > pmdd::dev::kTspMaxCities) return PMDD_ERR_INVALID;
    std::string msg;
    if (!srv->engine->tsp_structure(n, &msg)) return PMDD_ERR_OOM;
    if (srv->heavy) {  // built by the worker; waited for, so that the caller's clock starts after it
        auto rc = std::make_shared<std::atomic<int>>(-1);
        srv->heavy->post([n, rc](pmdd::Engine &E) {
            std::string m;
            rc->store(E.tsp_structure(n, &m) ? PMDD_OK : PMDD_ERR_OOM);
        }, false);
        HeavyLane &H = *srv->heavy;
        std::unique_lock<std::mutex> lk(H.mu);
        H.done.wait_for(lk, std::chrono::seconds(60), [&] { return rc->load() >= 0 || H.failed; });
        const int r = rc->load();
        if (r != PMDD_OK) return r < 0 ? PMDD_ERR_CUDA : r;
    }
    return PMDD_OK;
}

namespace {

// Moves the heavy lane's finished results to the caller's side (pmdd_server_run only,
// so that a result is pending until a run call has reported it, as in one lane).
size_t ready_results(pmdd_server *srv) {
    if (srv->heavy) {
        std::lock_guard<std::mutex> lk(srv->heavy->mu);
        while (!srv->heavy->outbox.empty()) {
            srv->ready.push_back(std::move(srv->heavy->outbox.front()));
            srv->heavy->outbox.pop_front();
        }
    }
    return srv->engine->finished().size() + srv->ready.size();
}

}  // namespace

int pmdd_server_run(pmdd_server *srv, int32_t max_steps) {
    if (!srv) return -1;
    int steps = 0;
    pmdd::Engine &E = *srv->engine;
    for (;;) {
        const size_t ready = ready_results(srv);
        if (ready > 0) return static_cast<int>(ready);
        if (srv->heavy) {
            std::lock_guard<std::mutex> lk(srv->heavy->mu);
            if (srv->heavy->failed) return -1;
        }
        if (max_steps > 0 && steps >= max_steps) return 0;
        if (!E.idle()) {
            if (E.step() < 0) return -1;
            ++steps;
            continue;
        }
        if (!srv->heavy) return 0;
        // the light lane is idle: wait a little for the heavy lane, so that the caller
        // comes back soon to submit what arrived meanwhile
        HeavyLane &H = *srv->heavy;
        std::unique_lock<std::mutex> lk(H.mu);
        if (H.outbox.empty() && !H.failed && H.busy_locked())
            H.done.wait_for(lk, std::chrono::milliseconds(2),
                            [&] { return !H.outbox.empty() || H.failed || !H.busy_locked(); });
        const bool got = !H.outbox.empty(), failed = H.failed, busy = H.busy_locked();
        lk.unlock();
        if (got) return static_cast<int>(ready_results(srv));
        if (failed) return -1;
        if (!busy || max_steps > 0) return 0;
    }
}

int pmdd_server_poll(pmdd_server *srv, pmdd_result *out) {
    if (!srv || !out) return 0;
    std::unique_ptr<pmdd::Instance> I;
    if (!srv->engine->finished().empty()) {
        I = std::move(srv->engine->finished().front());
        srv->engine->finished().pop_front();
    } else if (!srv->ready.empty()) {
        I = std::move(srv->ready.front());
        srv->ready.pop_front();
    }
    if (!I) return 0;
    srv->heavy_ids.erase(I->id);
    std::memset(out, 0, sizeof(*out));
    out->req_id = I->id;
    out->submit_s = I->submit_s;
    out->admit_s = I->admit_s;
    out->finish_s = I->finish_s;
    out->status = export_result(*I, &out->frontier, nullptr);
    write_err(out->error, sizeof(out->error), I->error);
    return 1;
}

int pmdd_server_cancel(pmdd_server *srv, uint64_t req_id) {
    if (!srv) return PMDD_ERR_INVALID;
    if (srv->heavy && srv->heavy_ids.count(req_id)) {
        srv->heavy->post([req_id](pmdd::Engine &E) { E.cancel(req_id); }, false);
        return PMDD_OK;
    }
    return srv->engine->cancel(req_id) ? PMDD_OK : PMDD_ERR_INVALID;
}

int pmdd_server_pending(const pmdd_server *srv) {
    if (!srv) return 0;
    size_t p = srv->engine->queued() + srv->engine->running();
    if (srv->heavy) {
        std::lock_guard<std::mutex> lk(srv->heavy->mu);
        // results the worker has finished count until a run call hands them over: they
        // arrive while the caller is away
        p += static_cast<size_t>(srv->heavy->inbox_requests) + srv->heavy->queued + srv->heavy->running +
             srv->heavy->outbox.size();
    }
    return static_cast<int>(p);
}

int pmdd_server_get_info(const pmdd_server *srv, pmdd_server_info *out) {
    if (!srv || !out) return PMDD_ERR_INVALID;
    const pmdd::Engine &E = *srv->engine;
    const pmdd::Engine::Counters &c = E.counters();
    std::memset(out, 0, sizeof(*out));
    out->submitted = static_cast<int64_t>(srv->submitted);
    out->admitted = c.admitted;
    out->completed = c.completed;
    out->failed = c.failed;
    out->rejected = c.rejected;
    out->cancelled = c.cancelled;
    out->queued = static_cast<int32_t>(E.queued());
    out->running = static_cast<int32_t>(E.running());
    out->queued_peak = static_cast<int32_t>(c.queued_peak);
    out->running_peak = static_cast<int32_t>(c.running_peak);
    out->budget_bytes = static_cast<int64_t>(E.arena().capacity());
    out->used_bytes = static_cast<int64_t>(E.arena().used());
    out->peak_used_bytes = static_cast<int64_t>(E.arena().peak());
    out->reserved_growth_bytes = E.reserved_growth();
    out->injected_alloc_failures = E.arena().injected_failures();
    if (srv->heavy) {  // both lanes: sums (peaks: the sum of the lanes' peaks)
        std::lock_guard<std::mutex> lk(srv->heavy->mu);
        const HeavyLane &H = *srv->heavy;
        out->admitted += H.counters.admitted;
        out->completed += H.counters.completed;
        out->failed += H.counters.failed;
        out->rejected += H.counters.rejected;
        out->cancelled += H.counters.cancelled;
        out->queued += static_cast<int32_t>(H.queued + static_cast<size_t>(H.inbox_requests));
        out->running += static_cast<int32_t>(H.running);
        out->queued_peak += static_cast<int32_t>(H.counters.queued_peak);
        out->running_peak += static_cast<int32_t>(H.counters.running_peak);
        out->budget_bytes += H.budget;
        out->used_bytes += H.used;
        out->peak_used_bytes += H.peak;
        out->reserved_growth_bytes += H.growth;
        out->injected_alloc_failures += H.injected;
    }
    return PMDD_OK;
}

int pmdd_server_inject_alloc_failures(pmdd_server *srv, int64_t after, int64_t count) {
    if (!srv || after < 0 || count < 0) return PMDD_ERR_INVALID;
    srv->engine->inject_alloc_failures(after, count);
    if (srv->heavy) {
        // commands run in order: the setting applies before any later submission
        srv->heavy->post([after, count](pmdd::Engine &E) { E.inject_alloc_failures(after, count); }, false);
    }
    return PMDD_OK;
}

void pmdd_server_destroy(pmdd_server *srv) { delete srv; }

const char *pmdd_version(void) { return "pmdd_b200 0.1 (sm_100a)"; }

int64_t pmdd_launch_count(void) { return pmdd::g_total_launches.load(); }

int64_t pmdd_tuned_mark_min(const char *path, int32_t nobjs, int32_t problem_type) {
    const auto table = pmdd::read_tuning(path ? std::string(path) : pmdd::default_tuning_path(), "big_mark_min");
    auto it = table.find({nobjs, problem_type});
    return it != table.end() ? it->second : 0;
}

int64_t pmdd_tuned_lex_pair_max(const char *path, int32_t nobjs, int32_t problem_type) {
    const auto table = pmdd::read_tuning(path ? std::string(path) : pmdd::default_tuning_path(), "lex_pair_max");
    auto it = table.find({nobjs, problem_type});
    return it != table.end() ? it->second : -1;
}

int64_t pmdd_tuned_tile_window_max(const char *path, int32_t nobjs, int32_t problem_type) {
    const auto table = pmdd::read_tuning(path ? std::string(path) : pmdd::default_tuning_path(), "tile_window_max");
    auto it = table.find({nobjs, problem_type});
    return it != table.end() ? it->second : -1;
}

}  // extern "C"
