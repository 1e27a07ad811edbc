// Frontier and stats output, in the formats of the reference's writers
// (src/pmdd/util/output_utils.cpp:87-152 and :154-300), off the caller's thread.
//
// The reference pipes each frontier through `gzip -c` (one process per output file) and
// appends the stats record to a JSONL file from the enumerating thread.  Here the CSV is
// deflated in process by zlib and both writes run on a small pool of writer threads fed
// by a queue: a serving loop hands a result over (one copy of the points) and goes on.
// The CSV text is the reference's, byte for byte: one point per line, objectives as
// decimal integers separated by commas, '\n' line ends, points sorted ascending
// lexicographically first as the reference's main does (src/pmdd/main.cpp:267).
#include <zlib.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "pmdd_host.h"

namespace {

void write_err(char *err, size_t errlen, const std::string &msg) {
    if (err == nullptr || errlen == 0) return;
    const size_t n = std::min(errlen - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

template <typename T>
void sort_points(T *p, int64_t n, int d) {
    if (n < 2) return;
    std::vector<int64_t> idx(static_cast<size_t>(n));
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [p, d](int64_t a, int64_t b) {
        return std::lexicographical_compare(p + a * d, p + a * d + d, p + b * d, p + b * d + d);
    });
    std::vector<T> tmp(static_cast<size_t>(n) * d);
    for (int64_t i = 0; i < n; ++i) std::memcpy(&tmp[i * d], p + idx[i] * d, sizeof(T) * d);
    std::memcpy(p, tmp.data(), sizeof(T) * tmp.size());
}

// Decimal text of one value into buf (returns the length).
template <typename T>
int put_int(char *buf, T v) {
    char tmp[24];
    int k = 0;
    const bool neg = v < 0;
    unsigned long long u = neg ? 0ULL - static_cast<unsigned long long>(static_cast<long long>(v))
                               : static_cast<unsigned long long>(v);
    do {
        tmp[k++] = static_cast<char>('0' + u % 10);
        u /= 10;
    } while (u);
    int n = 0;
    if (neg) buf[n++] = '-';
    while (k) buf[n++] = tmp[--k];
    return n;
}

template <typename T>
bool write_csv_gz(const T *p, int64_t n, int d, const std::string &path, std::string *error) {
    gzFile f = gzopen(path.c_str(), "wb");
    if (!f) {
        *error = "could not open output";
        return false;
    }
    gzbuffer(f, 1 << 17);
    std::string chunk;
    chunk.reserve(1 << 16);
    char num[24];
    bool ok = true;
    for (int64_t i = 0; i < n && ok; ++i) {
        for (int o = 0; o < d; ++o) {
            if (o) chunk += ',';
            chunk.append(num, static_cast<size_t>(put_int(num, p[i * d + o])));
        }
        chunk += '\n';
        if (chunk.size() >= (1 << 16) - 256) {
            ok = gzwrite(f, chunk.data(), static_cast<unsigned>(chunk.size())) == static_cast<int>(chunk.size());
            chunk.clear();
        }
    }
    if (ok && !chunk.empty())
        ok = gzwrite(f, chunk.data(), static_cast<unsigned>(chunk.size())) == static_cast<int>(chunk.size());
    const bool closed = gzclose(f) == Z_OK;
    if (!ok || !closed) {
        *error = "failed while writing compressed frontier";
        return false;
    }
    return true;
}

bool write_any(std::vector<unsigned char> &pts, int64_t n, int d, int elem, bool sort, const std::string &path,
               std::string *error) {
    if (elem == 8) {
        int64_t *p = reinterpret_cast<int64_t *>(pts.data());
        if (sort) sort_points(p, n, d);
        return write_csv_gz(p, n, d, path, error);
    }
    int32_t *p = reinterpret_cast<int32_t *>(pts.data());
    if (sort) sort_points(p, n, d);
    return write_csv_gz(p, n, d, path, error);
}

std::mutex g_jsonl_mu;  // record appends from every writer are whole lines

bool append_jsonl(const std::string &path, const std::string &record, std::string *error) {
    std::lock_guard<std::mutex> lk(g_jsonl_mu);
    std::ofstream out(path.c_str(), std::ios::out | std::ios::app);
    if (!out.is_open()) {
        *error = "could not open output path " + path;
        return false;
    }
    out << record << '\n';
    out.flush();
    if (!out) {
        *error = "failed while appending to " + path;
        return false;
    }
    return true;
}

bool valid_shape(int64_t n, int32_t d, int32_t elem, const void *points, std::string *error) {
    if (n < 0 || d < 1 || d > 64 || (elem != 4 && elem != 8) || (n > 0 && points == nullptr)) {
        *error = "invalid frontier (count, objectives, element size or NULL points)";
        return false;
    }
    return true;
}

}  // namespace

struct pmdd_writer {
    struct Item {
        std::vector<unsigned char> pts;
        int64_t n = 0;
        int32_t d = 0, elem = 4;
        std::string csv, jsonl, record;
    };
    std::mutex mu;
    std::condition_variable cv_work, cv_idle;
    std::deque<Item> queue;
    int64_t busy = 0, failed = 0, written = 0;
    std::string first_error;
    bool stop = false;
    std::vector<std::thread> pool;

    void worker() {
        for (;;) {
            Item it;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [this] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                it = std::move(queue.front());
                queue.pop_front();
                ++busy;
            }
            std::string e;
            bool ok = true;
            if (!it.csv.empty()) ok = write_any(it.pts, it.n, it.d, it.elem, true, it.csv, &e);
            if (ok && !it.jsonl.empty()) ok = append_jsonl(it.jsonl, it.record, &e);
            {
                std::lock_guard<std::mutex> lk(mu);
                --busy;
                if (ok) ++written;
                else {
                    ++failed;
                    if (first_error.empty()) first_error = e;
                }
                if (busy == 0 && queue.empty()) cv_idle.notify_all();
            }
        }
    }
};

extern "C" {

int pmdd_write_frontier_csv_gz(const void *points, int64_t num_points, int32_t nobjs, int32_t elem_bytes,
                               int32_t sort, const char *path, char *err, size_t errlen) {
    std::string e;
    if (!valid_shape(num_points, nobjs, elem_bytes, points, &e) || path == nullptr || path[0] == '\0') {
        write_err(err, errlen, e.empty() ? "output path is empty" : e);
        return PMDD_ERR_INVALID;
    }
    std::vector<unsigned char> pts(static_cast<size_t>(num_points) * nobjs * elem_bytes);
    if (!pts.empty()) std::memcpy(pts.data(), points, pts.size());
    if (!write_any(pts, num_points, nobjs, elem_bytes, sort != 0, path, &e)) {
        write_err(err, errlen, e);
        return PMDD_ERR_IO;
    }
    return PMDD_OK;
}

pmdd_writer *pmdd_writer_create(int32_t threads, char *err, size_t errlen) {
    if (threads <= 0) threads = static_cast<int32_t>(std::max(1u, std::min(4u, std::thread::hardware_concurrency())));
    if (threads > 256) {
        write_err(err, errlen, "writer threads must be in 1..256");
        return nullptr;
    }
    pmdd_writer *w = new pmdd_writer;
    for (int32_t t = 0; t < threads; ++t) w->pool.emplace_back([w] { w->worker(); });
    return w;
}

int pmdd_writer_submit(pmdd_writer *w, const void *points, int64_t num_points, int32_t nobjs, int32_t elem_bytes,
                       const char *csv_gz_path, const char *jsonl_path, const char *jsonl_record) {
    std::string e;
    if (w == nullptr || !valid_shape(num_points, nobjs, elem_bytes, points, &e)) return PMDD_ERR_INVALID;
    const bool has_csv = csv_gz_path != nullptr && csv_gz_path[0] != '\0';
    const bool has_jsonl = jsonl_path != nullptr && jsonl_path[0] != '\0';
    if (!has_csv && !has_jsonl) return PMDD_ERR_INVALID;
    if (has_jsonl && (jsonl_record == nullptr || std::strchr(jsonl_record, '\n') != nullptr))
        return PMDD_ERR_INVALID;
    pmdd_writer::Item it;
    it.n = num_points;
    it.d = nobjs;
    it.elem = elem_bytes;
    if (has_csv) {
        it.csv = csv_gz_path;
        it.pts.resize(static_cast<size_t>(num_points) * nobjs * elem_bytes);
        if (!it.pts.empty()) std::memcpy(it.pts.data(), points, it.pts.size());
    }
    if (has_jsonl) {
        it.jsonl = jsonl_path;
        it.record = jsonl_record;
    }
    {
        std::lock_guard<std::mutex> lk(w->mu);
        if (w->stop) return PMDD_ERR_INVALID;
        w->queue.push_back(std::move(it));
    }
    w->cv_work.notify_one();
    return PMDD_OK;
}

int64_t pmdd_writer_pending(pmdd_writer *w) {
    if (w == nullptr) return 0;
    std::lock_guard<std::mutex> lk(w->mu);
    return static_cast<int64_t>(w->queue.size()) + w->busy;
}

int64_t pmdd_writer_flush(pmdd_writer *w, int64_t *written, char *err, size_t errlen) {
    if (w == nullptr) return 0;
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv_idle.wait(lk, [w] { return w->queue.empty() && w->busy == 0; });
    const int64_t failed = w->failed;
    if (written) *written = w->written;
    if (failed) write_err(err, errlen, w->first_error);
    w->failed = 0;
    w->written = 0;
    w->first_error.clear();
    return failed;
}

void pmdd_writer_destroy(pmdd_writer *w) {
    if (w == nullptr) return;
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->stop = true;
    }
    w->cv_work.notify_all();
    for (auto &t : w->pool) t.join();
    delete w;
}

}  // extern "C"
