// Request loop for serving solves: continuous batching over lanes, admission by device memory.
//
// The reference answers one Run(IO&) at a time (Headers/DispatchAndRun.h:224-244). Here a client
// submits filled stores; `lanes` worker threads each own a CUDA stream; a batch started while
// others run gives its persistent solver 1/lanes of the SMs, a batch started alone the whole GPU.
// A lane that is free takes, in arrival order, the waiting requests
// whose estimated device footprint fits in what the running batches leave of the memory budget
// (up to max_batch of them) and solves them as one batch (hfm_run_batch: instances of a family
// share a launch sequence). Requests that arrive while other batches are on the device are
// admitted by the next lane to free up, and their work overlaps with the running batches on the
// device. Results land in each request's own store; per-request submit / start / done times are
// kept for latency statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "device_buffer.hpp"
#include "io.hpp"
#include "store_handle.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    hfm_io *io = nullptr;
    size_t bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = HFM_OK;
    bool done = false;
};

// Device bytes of a request: per-cell solver state of its model and precision (stencil codes and
// weights or visibility words, values, the FP64 metric or speed field on upload, output staging),
// plus the tile lists and dependency graph, with a margin. Reads the store without marking keys.
size_t estimate_bytes(const hfm::Store &st) {
    size_t cells = 1;
    std::string model;
    bool fp64 = true;
    try {
        model = st.raw("model", false).str;
        const hfm::RawElement &d = st.raw("dims", false);
        for (size_t i = 0; i < d.count(); ++i) cells *= (size_t)std::max(1.0, d.ptr()[i]);
    } catch (...) {
        return size_t(1) << 20;  // the run reports the missing key
    }
    try {
        fp64 = st.raw("solverPrecision", false).str != "float32";
    } catch (...) {
    }
    const size_t r = fp64 ? 8 : 4;
    size_t per_cell;
    if (model == "Riemann3") per_cell = 48 + 6 * (4 + r) + r + 8 + 8 + 16;
    else if (model == "Riemann2") per_cell = 24 + 3 * (4 + r) + r + 8 + 8 + 16;
    else if (model == "Diagonal2" || model == "Diagonal3") per_cell = 24 + 3 * (4 + r) + r + 8 + 8 + 16;
    else if (model == "TTI3") per_cell = 112 + 200 + r + 8 + 8 + 16;
    else per_cell = 4 + r + r + 8 + 8 + 16;  // shared stencils: visibility, multiplier, values
    return cells * per_cell + (size_t(4) << 20);
}

}  // namespace

struct hfm_server {
    hfm_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::vector<std::thread> lanes;
    size_t budget = 0, in_use = 0, peak = 0;
    uint64_t next_ticket = 1;
    unsigned long long submitted = 0, completed = 0, batches = 0, max_batch_seen = 0;
    int running = 0;
    bool stop = false;
    Clock::time_point t0 = Clock::now();

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    void lane_main() {
        cudaStream_t stream = nullptr;
        const bool ok = cudaSetDevice(cfg.device) == cudaSuccess &&
                        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess;
        hfm::current_stream() = stream;
        std::vector<Request *> batch;
        std::vector<hfm_io *> ios;
        std::vector<int> codes;
        for (;;) {
            size_t bytes = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    return (stop && queue.empty()) || (!queue.empty() && in_use + queue.front()->bytes <= budget);
                });
                if (queue.empty()) break;  // stopping
                batch.clear();
                // leave a fair share of the waiting requests to the other free lanes
                const int free_lanes = std::max(1, cfg.lanes - running);
                const int limit = std::min<int>(cfg.max_batch, ((int)queue.size() + free_lanes - 1) / free_lanes);
                while (!queue.empty() && (int)batch.size() < limit &&
                       in_use + bytes + queue.front()->bytes <= budget) {
                    bytes += queue.front()->bytes;
                    batch.push_back(queue.front());
                    queue.pop_front();
                }
                in_use += bytes;
                peak = std::max(peak, in_use);
                ++running;
                // SM share of this batch's persistent solver: the whole GPU when it runs alone (low
                // load: the latency of a plain solve), 1/lanes when other batches are on the device
                // (their solvers then run side by side)
                hfm::solver_share() = running > 1 ? cfg.lanes : 1;
                const double t = now();
                for (Request *r : batch) r->t_start = t;
                if (!queue.empty()) cv_work.notify_one();  // leave the rest to another free lane
            }
            ios.clear();
            for (Request *r : batch) ios.push_back(r->io);
            codes.assign(batch.size(), HFM_ERR_CUDA);
            if (ok) {
                hfm_run_batch(ios.data(), (int)ios.size(), nullptr, codes.data());
                cudaStreamSynchronize(stream);
            } else {
                for (hfm_io *io : ios) io->last_error = "serving lane could not set up its CUDA stream";
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                const double t = now();
                for (size_t k = 0; k < batch.size(); ++k) {
                    batch[k]->status = codes[k];
                    batch[k]->t_done = t;
                    batch[k]->done = true;
                }
                in_use -= bytes;
                --running;
                completed += batch.size();
                ++batches;
                max_batch_seen = std::max<unsigned long long>(max_batch_seen, batch.size());
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

hfm_server *hfm_server_create(const hfm_server_config *cfg) {
    try {
        auto s = std::make_unique<hfm_server>();
        if (cfg) s->cfg = *cfg;
        if (s->cfg.lanes <= 0) s->cfg.lanes = 2;
        if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
        if (cudaSetDevice(s->cfg.device) != cudaSuccess) return nullptr;
        hfm::keep_pool_cached();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return nullptr;
        s->budget = s->cfg.hbm_budget_bytes > 0 ? (size_t)s->cfg.hbm_budget_bytes : (size_t)(0.8 * (double)free_b);
        for (int i = 0; i < s->cfg.lanes; ++i) s->lanes.emplace_back([p = s.get()] { p->lane_main(); });
        return s.release();
    } catch (...) {
        return nullptr;
    }
}

int hfm_server_submit(hfm_server *s, hfm_io *io, uint64_t *ticket) {
    if (!s || !io || !ticket) return HFM_ERR_ARG;
    try {
        auto r = std::make_unique<Request>();
        r->io = io;
        r->bytes = estimate_bytes(io->store);
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return HFM_ERR_ARG;
        if (r->bytes > s->budget) {
            io->last_error = "request exceeds the server's device memory budget";
            return HFM_ERR_NOMEM;
        }
        r->ticket = s->next_ticket++;
        r->t_submit = s->now();
        *ticket = r->ticket;
        s->queue.push_back(r.get());
        s->reqs.emplace(r->ticket, std::move(r));
        ++s->submitted;
    } catch (...) {
        return HFM_ERR_NOMEM;
    }
    s->cv_work.notify_one();
    return HFM_OK;
}

int hfm_server_wait(hfm_server *s, uint64_t ticket, double timeout_s, int *status) {
    if (!s) return HFM_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return HFM_ERR_ARG;
    Request *r = it->second.get();
    auto pred = [&] { return r->done; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return HFM_ERR_NOT_CONVERGED;
    if (status) *status = r->status;
    return HFM_OK;
}

int hfm_server_release(hfm_server *s, uint64_t ticket, double *times) {
    if (!s) return HFM_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || !it->second->done) return HFM_ERR_ARG;
    if (times) {
        times[0] = it->second->t_submit;
        times[1] = it->second->t_start;
        times[2] = it->second->t_done;
    }
    s->reqs.erase(it);
    return HFM_OK;
}

int hfm_server_get_stats(hfm_server *s, hfm_server_stats *st) {
    if (!s || !st) return HFM_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->batches = s->batches;
    st->max_batch = s->max_batch_seen;
    st->queued = s->queue.size();
    st->running_batches = (unsigned long long)s->running;
    st->budget_bytes = (double)s->budget;
    st->bytes_in_use = (double)s->in_use;
    st->peak_bytes = (double)s->peak;
    return HFM_OK;
}

void hfm_server_destroy(hfm_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (std::thread &t : s->lanes) t.join();
    delete s;
}

}  // extern "C"
