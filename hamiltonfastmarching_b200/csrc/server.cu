// Request loop for serving solves: continuous batching into resident persistent solvers, admission
// by device memory.
//
// The reference answers one Run(IO&) at a time (Headers/DispatchAndRun.h:224-244). Here clients
// submit filled stores and one scheduler thread owns the GPU work:
//   * a submitted request is parsed as hfm_run parses it (same keys, defaults and messages);
//   * a plain solve (arrival times only) of a Riemann2, Riemann3 or ReedsShepp2 family is admitted,
//     in arrival order, while its estimated device footprint fits in the memory budget and a slot
//     is free, into the resident solver of its family (resident.cuh): its stencils, visibility and
//     tile dependencies are built in the family's arena and its seed tiles join the running
//     solver's lists at the next slice;
//   * the resident solver runs in slices; a slice ends as soon as an instance converges, so each
//     request is released when its own tiles drain, or soon after a new request arrives (the
//     attention word, read by the solver between rounds), so that it is admitted while the others
//     keep running; families with work take turns (4 ms slices when more than one has work);
//   * other requests (geodesics, sensitivities, variations, stopping criteria, cached values,
//     exports of stencils or activeNeighs, TTI3 and the other models) run through hfm_run between
//     slices, one at a time.
// With max_batch = 1 every request runs through hfm_run, one at a time: the plain loop.
// Results land in each request's own store; per-request submit / start / done times are kept for
// latency statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "device_buffer.hpp"
#include "io.hpp"
#include "solver.hpp"
#include "store_handle.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    hfm_io *io = nullptr;
    size_t bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = HFM_OK;
    bool done = false, counted = false;
    std::unique_ptr<hfm::PreparedRun> prep;
    std::string family;
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

int error_code_of(const std::exception &e) {
    if (const auto *h = dynamic_cast<const hfm::Error *>(&e)) return h->code;
    if (dynamic_cast<const std::bad_alloc *>(&e)) return HFM_ERR_NOMEM;
    return HFM_ERR_VALUE;
}

}  // namespace

struct hfm_server {
    hfm_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;  // submitted, not yet taken by the scheduler
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::thread scheduler;
    size_t budget = 0, in_use = 0, peak = 0;
    uint64_t next_ticket = 1;
    unsigned long long submitted = 0, completed = 0, slices = 0, max_resident = 0, resident = 0;
    bool stop = false;
    bool started = false, start_ok = false;
    std::condition_variable cv_started;
    // attention word: raised by submit, read by the running solver (host memory mapped to the GPU)
    volatile unsigned *attn_host = nullptr;
    unsigned *attn_dev = nullptr;
    Clock::time_point t0 = Clock::now();

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    void complete(Request *r, int status) {
        {
            std::lock_guard<std::mutex> lk(mu);
            r->status = status;
            r->t_done = now();
            r->done = true;
            if (r->counted) in_use -= r->bytes;
            r->counted = false;
            ++completed;
        }
        cv_done.notify_all();
    }

    // A request through hfm_run (the ordinary single-solve path).
    void run_plain(Request *r) {
        if (r->prep) {  // hfm_run parses the store again: drop the output field the first parse made
            r->prep->fail();
            r->prep.reset();
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            r->t_start = now();
            in_use += r->bytes;
            r->counted = true;
            peak = std::max(peak, in_use);
        }
        const int rc = hfm_run(r->io, nullptr);
        complete(r, rc);
    }

    void scheduler_main() {
        cudaStream_t stream = nullptr;
        bool ok = cudaSetDevice(cfg.device) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess;
        unsigned *host_word = nullptr;
        if (ok) ok = cudaHostAlloc((void **)&host_word, sizeof(unsigned), cudaHostAllocMapped) == cudaSuccess;
        if (ok) {
            *host_word = 0u;
            ok = cudaHostGetDevicePointer((void **)&attn_dev, host_word, 0) == cudaSuccess;
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            attn_host = host_word;
            started = true;
            start_ok = ok;
        }
        cv_started.notify_all();
        if (!ok) {
            if (host_word) cudaFreeHost(host_word);
            if (stream) cudaStreamDestroy(stream);
            return;
        }
        hfm::current_stream() = stream;
        std::deque<Request *> waiting;  // parsed resident requests, not yet admitted
        std::map<std::string, std::unique_ptr<hfm::ResidentFamily>> fams;
        std::unordered_map<int64_t, Request *> running;
        size_t turn = 0;
        for (;;) {
            std::vector<Request *> incoming;
            bool busy = !waiting.empty();
            for (const auto &f : fams) busy = busy || f.second->has_work();
            {
                std::unique_lock<std::mutex> lk(mu);
                if (!busy) cv_work.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty() && !busy) break;
                incoming.assign(queue.begin(), queue.end());
                queue.clear();
                *attn_host = 0u;
            }
            // ---- parse: resident families wait for admission, the rest run now through hfm_run
            for (Request *r : incoming) {
                if (cfg.max_batch <= 1) {
                    run_plain(r);
                    continue;
                }
                r->io->last_error.clear();
                try {
                    r->prep = hfm::prepare_run(r->io);
                    r->family = r->prep->skip() ? std::string() : hfm::resident_family_key(r->prep->problem());
                } catch (const std::exception &e) {
                    r->io->last_error = e.what();
                    r->prep.reset();
                    complete(r, error_code_of(e));
                    continue;
                }
                if (r->family.empty()) run_plain(r);
                else waiting.push_back(r);
            }
            // ---- admission in arrival order, by memory budget and free slots
            while (!waiting.empty()) {
                Request *r = waiting.front();
                {
                    std::lock_guard<std::mutex> lk(mu);
                    if ((in_use > 0 && in_use + r->bytes > budget) || resident >= (unsigned long long)cfg.max_batch) break;
                    in_use += r->bytes;
                    r->counted = true;
                    peak = std::max(peak, in_use);
                }
                bool admitted = false;
                try {
                    auto &fam = fams[r->family];
                    if (!fam) fam = hfm::make_resident_family(r->prep->problem());
                    int mw = 0;
                    admitted = fam->admit(r->prep->problem(), (int64_t)r->ticket, &mw);
                } catch (const std::exception &e) {
                    waiting.pop_front();
                    r->io->last_error = e.what();
                    r->prep->fail();
                    r->prep.reset();
                    complete(r, error_code_of(e));
                    continue;
                }
                if (!admitted) {
                    std::lock_guard<std::mutex> lk(mu);
                    in_use -= r->bytes;
                    r->counted = false;
                    break;
                }
                waiting.pop_front();
                running[(int64_t)r->ticket] = r;
                std::lock_guard<std::mutex> lk(mu);
                r->t_start = now();
                ++resident;
                max_resident = std::max(max_resident, resident);
            }
            // ---- one slice of the next family with work
            std::vector<std::string> keys;
            for (const auto &f : fams)
                if (f.second->has_work()) keys.push_back(f.first);
            if (keys.empty()) continue;
            const std::string key = keys[turn++ % keys.size()];
            hfm::ResidentFamily &fam = *fams[key];
            std::vector<std::pair<int64_t, hfm::EulerResult>> done;
            int fail_code = HFM_OK;
            std::string fail_msg;
            try {
                fam.slice(attn_dev, 1.0, keys.size() > 1 ? 4.0 : 0.0);
                fam.collect(done);
            } catch (const std::exception &e) {
                fail_code = error_code_of(e);
                fail_msg = e.what();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                ++slices;
            }
            for (auto &d : done) {
                Request *r = running[d.first];
                running.erase(d.first);
                int rc = HFM_OK;
                try {
                    r->prep->finish(d.second);
                } catch (const std::exception &e) {
                    r->io->last_error = e.what();
                    r->prep->fail();
                    rc = error_code_of(e);
                }
                r->prep.reset();
                {
                    std::lock_guard<std::mutex> lk(mu);
                    --resident;
                }
                complete(r, rc);
            }
            if (fail_code != HFM_OK) {  // the family's solver failed: its requests fail with it
                std::vector<int64_t> lost;
                fam.abandon(lost);
                for (int64_t t : lost) {
                    Request *r = running[t];
                    running.erase(t);
                    r->io->last_error = fail_msg;
                    r->prep->fail();
                    r->prep.reset();
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        --resident;
                    }
                    complete(r, fail_code);
                }
                fams.erase(key);
            }
        }
        fams.clear();
        cudaStreamSynchronize(stream);
        cudaFreeHost(host_word);
        cudaStreamDestroy(stream);
    }
};

extern "C" {

hfm_server *hfm_server_create(const hfm_server_config *cfg) {
    try {
        auto s = std::make_unique<hfm_server>();
        if (cfg) s->cfg = *cfg;
        if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
        if (s->cfg.max_batch > 256) s->cfg.max_batch = 256;
        if (cudaSetDevice(s->cfg.device) != cudaSuccess) return nullptr;
        hfm::keep_pool_cached();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return nullptr;
        s->budget = s->cfg.hbm_budget_bytes > 0 ? (size_t)s->cfg.hbm_budget_bytes : (size_t)(0.8 * (double)free_b);
        s->scheduler = std::thread([p = s.get()] { p->scheduler_main(); });
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_started.wait(lk, [&] { return s->started; });
            if (!s->start_ok) {
                lk.unlock();
                s->scheduler.join();
                return nullptr;
            }
        }
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
        if (s->attn_host) *s->attn_host = 1u;  // a running slice ends soon so that it is admitted
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
    st->batches = s->slices;
    st->max_batch = s->max_resident;
    st->queued = s->queue.size();
    st->running_batches = s->resident;
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
    if (s->scheduler.joinable()) s->scheduler.join();
    delete s;
}

}  // extern "C"
