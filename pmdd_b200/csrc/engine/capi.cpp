// extern "C" boundary of libpmdd_gpu.so (declared in include/pmdd.h).
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>

#include "engine.hpp"
#include "pmdd.h"

namespace {

void write_err(char *err, size_t errlen, const std::string &msg) {
    if (err == nullptr || errlen == 0) return;
    const size_t n = std::min(errlen - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

// One engine per device for the one-shot and batch entries, created on first use and
// kept for the life of the process (its arena is sized by PMDD_ARENA_BYTES, default a
// quarter of the device's free memory).
struct DeviceSlot {
    std::mutex mu;
    std::unique_ptr<pmdd::Engine> engine;
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
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    return static_cast<int64_t>(free_b / 4);
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

// Runs `n` prepared requests to completion on the device's shared engine.
int run_on_device(int device, std::vector<std::unique_ptr<pmdd::Instance>> &reqs, std::string *err) {
    DeviceSlot &slot = slot_for(device);
    std::lock_guard<std::mutex> lk(slot.mu);
    if (!slot.engine || !slot.engine->ok()) {
        slot.engine.reset(new pmdd::Engine(device, default_arena_bytes(device), 0));
        if (!slot.engine->ok()) {
            *err = slot.engine->error();
            slot.engine.reset();
            return PMDD_ERR_NO_DEVICE;
        }
    }
    pmdd::Engine &E = *slot.engine;
    std::unordered_map<uint64_t, size_t> index;
    for (size_t i = 0; i < reqs.size(); ++i) {
        reqs[i]->id = i;
        index[i] = i;
        E.submit(std::move(reqs[i]));
    }
    size_t got = 0;
    while (got < index.size()) {
        const int r = E.step();
        if (r < 0) {
            *err = E.error();
            // the engine is unusable: drop it so the next call starts clean
            for (auto &q : E.finished()) {
                const size_t k = index[q->id];
                reqs[k] = std::move(q);
            }
            E.finished().clear();
            slot.engine.reset();
            return PMDD_ERR_CUDA;
        }
        while (!E.finished().empty()) {
            std::unique_ptr<pmdd::Instance> q = std::move(E.finished().front());
            E.finished().pop_front();
            const size_t k = index[q->id];
            reqs[k] = std::move(q);
            ++got;
        }
    }
    return PMDD_OK;
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
    std::vector<std::unique_ptr<pmdd::Instance>> reqs(1);
    reqs[0].reset(new pmdd::Instance);
    std::string msg;
    const double t0 = pmdd::now_s();
    int rc = pmdd::prepare_instance(*dd, o, 0, reqs[0].get(), &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    rc = run_on_device(o.device, reqs, &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
    }
    pmdd::Instance &I = *reqs[0];
    I.stats.wall_pack_transfer_s = I.admit_s - t0;
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
    std::vector<std::unique_ptr<pmdd::Instance>> reqs(count);
    std::string msg;
    for (int32_t i = 0; i < count; ++i) {
        if (outs) std::memset(&outs[i], 0, sizeof(outs[i]));
        reqs[i].reset(new pmdd::Instance);
        const int rc = pmdd::prepare_instance(dds[i], o, static_cast<uint64_t>(i), reqs[i].get(), &msg);
        if (rc != PMDD_OK) {
            write_err(err, errlen, "instance " + std::to_string(i) + ": " + msg);
            if (status) status[i] = rc;
            return rc;
        }
    }
    int rc = run_on_device(o.device, reqs, &msg);
    if (rc != PMDD_OK) {
        write_err(err, errlen, msg);
        return rc;
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
            stats->kernel_total_s = std::max(stats->kernel_total_s, st.kernel_total_s);
            stats->work_candidates_total += st.work_candidates_total;
            stats->work_candidates_peak = std::max(stats->work_candidates_peak, st.work_candidates_peak);
            stats->work_frontier_survivors_total += st.work_frontier_survivors_total;
            stats->work_frontier_peak_points = std::max(stats->work_frontier_peak_points, st.work_frontier_peak_points);
            stats->work_join_products_total += st.work_join_products_total;
            stats->gpu_mem_peak_used_bytes = std::max(stats->gpu_mem_peak_used_bytes, st.gpu_mem_peak_used_bytes);
            stats->gpu_mem_peak_reserved_bytes = st.gpu_mem_peak_reserved_bytes;
        }
    }
    return first_bad;
}

// ------------------------------------------------------------------ serving
struct pmdd_server {
    std::unique_ptr<pmdd::Engine> engine;
    uint64_t submitted = 0;
};

pmdd_server *pmdd_server_create(int32_t device, int64_t budget_bytes, int32_t max_slots, char *err, size_t errlen) {
    std::unique_ptr<pmdd_server> s(new pmdd_server);
    if (budget_bytes <= 0) budget_bytes = default_arena_bytes(device);
    s->engine.reset(new pmdd::Engine(device, budget_bytes, max_slots));
    if (!s->engine->ok()) {
        write_err(err, errlen, s->engine->error());
        return nullptr;
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
        I->status = rc;
        I->error = msg;
        I->phase = pmdd::Instance::DONE;
        I->finish_s = pmdd::now_s();
        srv->engine->finished().push_back(std::move(I));
        return rc;
    }
    srv->engine->submit(std::move(I));
    srv->submitted++;
    return PMDD_OK;
}

int pmdd_server_run(pmdd_server *srv, int32_t max_steps) {
    if (!srv) return -1;
    int steps = 0;
    while ((max_steps <= 0 || steps < max_steps) && srv->engine->finished().empty() && !srv->engine->idle()) {
        if (srv->engine->step() < 0) return -1;
        ++steps;
    }
    return static_cast<int>(srv->engine->finished().size());
}

int pmdd_server_poll(pmdd_server *srv, pmdd_result *out) {
    if (!srv || !out || srv->engine->finished().empty()) return 0;
    std::unique_ptr<pmdd::Instance> I = std::move(srv->engine->finished().front());
    srv->engine->finished().pop_front();
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
    return srv->engine->cancel(req_id) ? PMDD_OK : PMDD_ERR_INVALID;
}

int pmdd_server_pending(const pmdd_server *srv) {
    if (!srv) return 0;
    return static_cast<int>(srv->engine->queued() + srv->engine->running());
}

void pmdd_server_destroy(pmdd_server *srv) { delete srv; }

const char *pmdd_version(void) { return "pmdd_b200 0.1 (sm_100a)"; }

int64_t pmdd_launch_count(void) { return pmdd::g_total_launches.load(); }

}  // extern "C"
