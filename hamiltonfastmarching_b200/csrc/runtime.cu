// Per-thread stream selection, memory-pool policy and launch accounting of the library, plus the
// device-resident entry point of the C ABI.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "device_buffer.hpp"
#include "solver.hpp"

namespace hfm {

cudaStream_t &current_stream() {
    thread_local cudaStream_t s = nullptr;
    return s;
}

int &solver_share() {
    thread_local int share = 1;
    return share;
}

std::mutex &cooperative_mutex() {
    static std::mutex mu;
    return mu;
}

void keep_pool_cached() {
    // Once per device: keep freed blocks of the default pool cached instead of returning them at
    // every synchronisation, so repeated solves do not pay for new device mappings.
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[dev] = true;
}

// ---- staged transfers
namespace {

// Worker threads for the host-side parts of staged copies (one pool per process).
class CopyPool {
public:
    CopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        nworkers_ = std::max(1u, std::min(16u, hw ? hw / 2 : 4u));
        for (unsigned i = 0; i + 1 < nworkers_; ++i) threads_.emplace_back([this, i] { work(i + 1); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : threads_) t.join();
    }
    // dst[0:n) = src[0:n), split in nworkers_ parts; the caller copies part 0.
    void copy(char *dst, const char *src, size_t n) {
        std::unique_lock<std::mutex> call(call_mu_);  // one parallel copy at a time
        const size_t part = (n + nworkers_ - 1) / nworkers_;
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = dst; src_ = src; n_ = n; part_ = part;
            pending_ = nworkers_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(part, n));
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }

private:
    void work(unsigned idx) {
        unsigned long long seen = 0;
        for (;;) {
            char *d;
            const char *s;
            size_t n, part;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                d = dst_; s = src_; n = n_; part = part_;
            }
            const size_t b = std::min(n, (size_t)idx * part), e = std::min(n, b + part);
            if (e > b) std::memcpy(d + b, s + b, e - b);
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (--pending_ == 0) done_cv_.notify_all();
            }
        }
    }
    unsigned nworkers_ = 1;
    std::vector<std::thread> threads_;
    std::mutex mu_, call_mu_;
    std::condition_variable cv_, done_cv_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t n_ = 0, part_ = 0;
    unsigned pending_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

CopyPool &copy_pool() {
    static CopyPool *pool = new CopyPool();  // lives until exit (workers are never joined late)
    return *pool;
}

constexpr size_t kChunk = size_t(32) << 20;

// Two page-locked chunks and their completion events, per thread (kept for the thread's life).
struct Staging {
    char *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    bool ok = false;
    Staging() {
        ok = cudaHostAlloc((void **)&buf[0], kChunk, cudaHostAllocDefault) == cudaSuccess &&
             cudaHostAlloc((void **)&buf[1], kChunk, cudaHostAllocDefault) == cudaSuccess &&
             cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) cudaGetLastError();
    }
};

Staging &staging() {
    thread_local Staging *st = new Staging();  // released with the process
    return *st;
}

}  // namespace

void *pinned_words(size_t bytes) {
    static std::mutex mu;
    static char *pool = nullptr;
    static size_t used = 0;
    constexpr size_t kPool = size_t(64) << 10;
    std::lock_guard<std::mutex> lk(mu);
    if (!pool) HFM_CUDA(cudaHostAlloc((void **)&pool, kPool, cudaHostAllocDefault));
    const size_t n = (bytes + 15) & ~size_t(15);
    if (used + n > kPool) throw Error(HFM_ERR_NOMEM, "page-locked word pool spent");
    void *p = pool + used;
    used += n;
    return p;
}

void staging_warm_up() {
    staging();
    copy_pool();
}

void staged_upload(void *dst_dev, const void *src_host, size_t bytes, cudaStream_t s) {
    Staging &st = staging();
    if (bytes < kStagedMin || !st.ok) {
        HFM_CUDA(cudaMemcpyAsync(dst_dev, src_host, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    const char *src = static_cast<const char *>(src_host);
    char *dst = static_cast<char *>(dst_dev);
    for (size_t off = 0, i = 0; off < bytes; off += kChunk, ++i) {
        const int b = (int)(i & 1);
        const size_t len = std::min(kChunk, bytes - off);
        if (st.used[b]) HFM_CUDA(cudaEventSynchronize(st.ev[b]));  // the chunk's previous DMA is done
        copy_pool().copy(st.buf[b], src + off, len);
        HFM_CUDA(cudaMemcpyAsync(dst + off, st.buf[b], len, cudaMemcpyHostToDevice, s));
        HFM_CUDA(cudaEventRecord(st.ev[b], s));
        st.used[b] = true;
    }
}

void staged_download(void *dst_host, const void *src_dev, size_t bytes, cudaStream_t s) {
    Staging &st = staging();
    if (bytes < kStagedMin || !st.ok) {
        HFM_CUDA(cudaMemcpyAsync(dst_host, src_dev, bytes, cudaMemcpyDeviceToHost, s));
        HFM_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const char *src = static_cast<const char *>(src_dev);
    char *dst = static_cast<char *>(dst_host);
    const size_t nchunks = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t i) {
        const int b = (int)(i & 1);
        const size_t off = i * kChunk, len = std::min(kChunk, bytes - off);
        if (st.used[b]) HFM_CUDA(cudaEventSynchronize(st.ev[b]));
        HFM_CUDA(cudaMemcpyAsync(st.buf[b], src + off, len, cudaMemcpyDeviceToHost, s));
        HFM_CUDA(cudaEventRecord(st.ev[b], s));
        st.used[b] = true;
    };
    issue(0);
    for (size_t i = 0; i < nchunks; ++i) {
        const int b = (int)(i & 1);
        const size_t off = i * kChunk, len = std::min(kChunk, bytes - off);
        HFM_CUDA(cudaEventSynchronize(st.ev[b]));
        if (i + 1 < nchunks) issue(i + 1);  // the next chunk's DMA overlaps this chunk's host copy
        copy_pool().copy(dst + off, st.buf[b], len);
        st.used[b] = false;
    }
}

static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace hfm

using hfm::StreamScope;

extern "C" {

int hfm_kernel_launches(unsigned long long *count) {
    if (!count) return HFM_ERR_ARG;
    *count = hfm::g_launches.load();
    return HFM_OK;
}

int hfm_solve_riemann_device(const hfm_riemann_device_args *a, hfm_solve_stats *stats, char *err, size_t errcap) {
    auto fail = [&](int code, const char *m) {
        if (err && errcap) {
            std::strncpy(err, m, errcap - 1);
            err[errcap - 1] = 0;
        }
        return code;
    };
    if (!a || !a->metric || !a->values) return fail(HFM_ERR_ARG, "null argument");
    if (a->ndim != 2 && a->ndim != 3) return fail(HFM_ERR_VALUE, "ndim must be 2 or 3");
    if (a->precision != 64 && a->precision != 32) return fail(HFM_ERR_VALUE, "precision must be 64 or 32");
    if (a->nseeds < 1 || !a->seed_index || !a->seed_value) return fail(HFM_ERR_VALUE, "at least one seed is required");
    try {
        StreamScope scope(static_cast<cudaStream_t>(a->stream));
        hfm::EulerProblem p;
        p.ndim = a->ndim;
        int64_t N = 1;
        for (int i = 0; i < a->ndim; ++i) {
            if (a->dims[i] <= 0 || a->dims[i] > (1 << 30)) return fail(HFM_ERR_VALUE, "invalid dims");
            p.dims[i] = (int)a->dims[i];
            p.h[i] = a->grid_scale[i];
            if (!(p.h[i] > 0)) return fail(HFM_ERR_VALUE, "grid scales must be positive");
            N *= a->dims[i];
        }
        p.kind = hfm::StencilKind::RiemannPerCell;
        p.fp64 = a->precision == 64;
        p.dual = a->dual != 0;
        p.d_metric = a->metric;
        p.d_walls = a->walls;
        p.d_values_out = a->values;
        hfm::default_schedule(p);
        if (a->sweeps_per_tile > 0) p.sweeps_per_tile = a->sweeps_per_tile;
        std::vector<std::pair<int64_t, double>> seeds;
        for (int64_t i = 0; i < a->nseeds; ++i) {
            if (a->seed_index[i] < 0 || a->seed_index[i] >= N) return fail(HFM_ERR_VALUE, "seed index out of range");
            seeds.emplace_back(a->seed_index[i], a->seed_value[i]);
        }
        std::stable_sort(seeds.begin(), seeds.end(),
                         [](const std::pair<int64_t, double> &x, const std::pair<int64_t, double> &y) { return x.first < y.first; });
        for (size_t i = 0; i < seeds.size(); ++i)
            if (i == 0 || seeds[i].first != seeds[i - 1].first) {
                p.seed_index.push_back(seeds[i].first);
                p.seed_value.push_back(seeds[i].second);
            }
        hfm::EulerResult r;
        hfm::solve_eulerian(p, r);
        if (stats) {
            stats->n_accepted = r.n_accepted;
            stats->max_stencil_width = r.max_stencil_width;
            stats->stencil_ms = r.t_stencil_ms;
            stats->solve_ms = r.t_solve_ms;
            stats->rounds = r.rounds;
            stats->tile_activations = r.tile_activations;
            stats->local_solves = r.local_solves;
        }
        return HFM_OK;
    } catch (const hfm::Error &e) {
        return fail(e.code, e.what());
    } catch (const std::exception &e) {
        return fail(HFM_ERR_VALUE, e.what());
    }
}

}  // extern "C"
