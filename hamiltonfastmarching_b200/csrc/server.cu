// Request loop for serving solves: continuous batching into resident persistent solvers, admission
// by device memory.
//
// The reference answers one Run(IO&) at a time (Headers/DispatchAndRun.h:224-244). Here clients
// submit filled stores; two threads own the work:
//   * the intake thread parses each request as hfm_run parses it (same keys, defaults and
//     messages) and, for a plain solve (arrival times only) of a Riemann2, Riemann3 or ReedsShepp2
//     family, uploads its large inputs (metric or speed multiplier, walls) to the device while the
//     solver runs, in arrival order and within a bound on staged bytes;
//   * the scheduler thread admits staged requests, in arrival order, while their estimated device
//     footprint fits in the memory budget and a slot is free: the instance is built in the arena of
//     its family's resident solver (resident.cuh) on a side stream, while a slice of the solver
//     runs on the SMs left free for it; the running slice is then interrupted (the attention word,
//     read by the solver between rounds) and the new instances' seed tiles join the lists;
//   * a slice ends as soon as an instance converges, so each request is released when its own
//     tiles drain; its values are copied out while the next slice runs; families with work take
//     turns (4 ms slices when more than one has work);
//   * other requests (geodesics, sensitivities, variations, stopping criteria, cached values,
//     exports of stencils or activeNeighs, TTI3 and the other models) run through hfm_run between
//     slices, one at a time.
// With max_batch = 1 every request runs through hfm_run, one at a time, unparsed by the intake
// thread: the plain loop. Results land in each request's own store; per-request submit / start /
// done times are kept for latency statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
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

// Age after which an admitted request's family takes the GPU ahead of the turn order.
constexpr double kStarveSeconds = 0.25;

struct Request {
    uint64_t ticket = 0;
    hfm_io *io = nullptr;
    size_t bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = HFM_OK;
    bool done = false, counted = false;
    std::unique_ptr<hfm::PreparedRun> prep;
    std::unique_ptr<hfm::StagedInputs> staged;  // device copies of its large inputs, until admission
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
    std::condition_variable cv_intake, cv_work, cv_done, cv_staged;
    std::deque<Request *> queue;  // submitted, not yet parsed by the intake thread
    std::deque<Request *> ready;  // parsed (and staged), not yet taken by the scheduler
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::thread intake, scheduler;
    size_t budget = 0, in_use = 0, peak = 0;
    size_t staged_bytes = 0, staged_cap = 0;  // device bytes of staged inputs not yet admitted
    uint64_t next_ticket = 1;
    unsigned long long submitted = 0, completed = 0, slices = 0, max_resident = 0, resident = 0;
    bool stop = false;
    bool started = false, start_ok = false;
    std::condition_variable cv_started;
    // attention word: raised by the scheduler to end a running slice (host memory mapped to the GPU)
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
        cv_work.notify_all();
    }

    // Frees a request's staged inputs (on the calling thread's current stream).
    void drop_staged(Request *r) {
        if (!r->staged) return;
        const size_t b = r->staged->bytes();
        r->staged.reset();
        {
            std::lock_guard<std::mutex> lk(mu);
            staged_bytes -= b;
        }
        cv_staged.notify_all();
    }

    // A request through hfm_run (the ordinary single-solve path).
    void run_plain(Request *r) {
        drop_staged(r);
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

    // Intake: parse in arrival order; stage the large inputs of resident-family requests.
    void intake_main() {
        cudaStream_t stream = nullptr;
        if (cudaSetDevice(cfg.device) != cudaSuccess ||
            cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
            stream = nullptr;
        hfm::current_stream() = stream;
        if (stream) hfm::staging_warm_up();
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_intake.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) break;  // stopping, nothing left
                r = queue.front();
                queue.pop_front();
            }
            if (cfg.max_batch > 1 && stream) {
                r->io->last_error.clear();
                try {
                    r->prep = hfm::prepare_run(r->io);
                    r->family = r->prep->skip() ? std::string() : hfm::resident_family_key(r->prep->problem());
                    if (!r->family.empty()) {
                        {
                            std::unique_lock<std::mutex> lk(mu);
                            cv_staged.wait(lk, [&] { return staged_bytes <= staged_cap; });
                        }
                        r->staged = hfm::stage_resident_inputs(r->prep->problem());
                        std::lock_guard<std::mutex> lk(mu);
                        staged_bytes += r->staged->bytes();
                    }
                } catch (const std::exception &e) {
                    r->io->last_error = e.what();
                    r->staged.reset();
                    if (r->prep) r->prep->fail();
                    r->prep.reset();
                    complete(r, error_code_of(e));
                    continue;
                }
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                ready.push_back(r);
            }
            cv_work.notify_all();
        }
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }

    void scheduler_main() {
        cudaStream_t stream = nullptr, side = nullptr;
        bool ok = cudaSetDevice(cfg.device) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) == cudaSuccess;
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
            if (side) cudaStreamDestroy(side);
            if (stream) cudaStreamDestroy(stream);
            return;
        }
        hfm::current_stream() = stream;
        hfm::staging_warm_up();
        // page-locked words of the families' solvers: set up now, before any slice runs
        try {
            hfm::pinned_words(0);
        } catch (...) {
        }
        std::deque<Request *> waiting;  // staged resident requests, not yet admitted (arrival order)
        std::deque<Request *> plain;    // requests for hfm_run
        std::map<std::string, std::unique_ptr<hfm::ResidentFamily>> fams;
        std::unordered_map<int64_t, Request *> running;  // admitted: prepared, in the lists or collected
        std::string cur;                // family whose slice is in flight ("" when none)
        Clock::time_point slice_t0{};
        std::string last;               // family of the previous slice (turns go in key order)
        // fails every admitted request of a family whose solver failed, and drops the family
        auto fail_family = [&](const std::string &key, int code, const std::string &msg) {
            std::vector<int64_t> lost;
            fams[key]->abandon(lost);
            for (int64_t t : lost) {
                Request *r = running[t];
                running.erase(t);
                r->io->last_error = msg;
                r->prep->fail();
                r->prep.reset();
                {
                    std::lock_guard<std::mutex> lk(mu);
                    --resident;
                }
                complete(r, code);
            }
            // nothing of the family's arena is in flight on either stream when it goes
            cudaStreamSynchronize(stream);
            cudaStreamSynchronize(side);
            hfm::StreamScope scope(side);
            fams.erase(key);
        };
        // Admits waiting requests in arrival order, by memory budget and free slots, at most `limit`
        // of them; each is built on the side stream. The family `running_key` has a slice in flight
        // and cannot grow its arena meanwhile: true when a request of it waits for that.
        auto admit_waiting = [&](const std::string &running_key, size_t limit) -> bool {
            for (size_t n = 0; n < limit && !waiting.empty(); ++n) {
                Request *r = waiting.front();
                {
                    std::lock_guard<std::mutex> lk(mu);
                    if ((in_use > 0 && in_use + r->bytes > budget) || resident >= (unsigned long long)cfg.max_batch)
                        return false;
                    in_use += r->bytes;
                    r->counted = true;
                    peak = std::max(peak, in_use);
                }
                hfm::ResidentFamily::Admit a = hfm::ResidentFamily::kNoSlot;
                try {
                    auto it = fams.find(r->family);
                    if (it == fams.end()) {
                        hfm::StreamScope scope(side);
                        auto fam = hfm::make_resident_family(r->prep->problem());
                        it = fams.emplace(r->family, std::move(fam)).first;
                    }
                    int mw = 0;
                    a = it->second->prepare(r->prep->problem(), (int64_t)r->ticket, r->staged.get(),
                                            r->family != running_key, side, &mw);
                } catch (const std::exception &e) {
                    waiting.pop_front();
                    {
                        hfm::StreamScope scope(side);
                        drop_staged(r);
                    }
                    r->io->last_error = e.what();
                    r->prep->fail();
                    r->prep.reset();
                    complete(r, error_code_of(e));
                    continue;
                }
                if (a != hfm::ResidentFamily::kPrepared) {
                    std::lock_guard<std::mutex> lk(mu);
                    in_use -= r->bytes;
                    r->counted = false;
                    return a == hfm::ResidentFamily::kNeedsGrow;
                }
                waiting.pop_front();
                {
                    hfm::StreamScope scope(side);
                    drop_staged(r);
                }
                running[(int64_t)r->ticket] = r;
                std::lock_guard<std::mutex> lk(mu);
                r->t_start = now();
                ++resident;
                max_resident = std::max(max_resident, resident);
            }
            return false;
        };
        for (;;) {
            // ---- requests from the intake thread
            {
                std::unique_lock<std::mutex> lk(mu);
                const bool idle = cur.empty() && waiting.empty() && plain.empty();
                if (idle) {
                    bool work = false;
                    for (const auto &f : fams) work = work || f.second->has_work() || f.second->has_pending();
                    if (!work) {
                        cv_work.wait(lk, [&] { return !ready.empty() || (stop && completed == submitted); });
                        if (ready.empty()) break;  // stopping: every request has completed
                    }
                }
                for (Request *r : ready) (r->prep && !r->family.empty() ? waiting : plain).push_back(r);
                ready.clear();
            }
            // ---- the slice in flight: new requests are built beside it (one per pass, so that its
            // end is seen soon); it is interrupted once prepared instances of its family wait (after
            // its minimum time), or, after 4 ms, when other work waits
            std::vector<std::pair<std::string, int64_t>> finished;
            if (!cur.empty()) {
                const bool want_stop = admit_waiting(cur, 1);
                hfm::ResidentFamily &F = *fams[cur];
                const double el = std::chrono::duration<double, std::milli>(Clock::now() - slice_t0).count();
                bool others = !plain.empty() || want_stop;
                for (const auto &f : fams)
                    if (f.first != cur) others = others || f.second->has_work() || f.second->has_pending();
                if (F.has_pending() || want_stop || (others && el >= 4.0)) *attn_host = 1u;
                if (!F.slice_done()) {
                    std::unique_lock<std::mutex> lk(mu);
                    cv_work.wait_for(lk, std::chrono::microseconds(200), [&] { return !ready.empty(); });
                    continue;
                }
                const std::string key = cur;
                cur.clear();
                std::vector<int64_t> done;
                try {
                    F.slice_end();
                    F.collect(done);
                } catch (const std::exception &e) {
                    fail_family(key, error_code_of(e), e.what());
                    done.clear();
                }
                {
                    std::lock_guard<std::mutex> lk(mu);
                    ++slices;
                }
                for (int64_t t : done) finished.emplace_back(key, t);
            }
            // ---- no slice in flight: admission (arenas may grow), single solves, the next slice
            if (cur.empty()) {
                admit_waiting(std::string(), waiting.size());
                while (!plain.empty()) {
                    Request *r = plain.front();
                    plain.pop_front();
                    run_plain(r);
                }
                std::vector<std::string> keys;
                for (const auto &f : fams)
                    if (f.second->has_work() || f.second->has_pending()) keys.push_back(f.first);
                if (!keys.empty()) {
                    // families take turns, the next after the previous slice's in key order (keys
                    // are sorted), so that small requests pass between the slices of large ones;
                    // but the family of the oldest admitted request goes first once that request
                    // has waited kStarveSeconds, so that a large request is not slowed without
                    // bound by the families that keep arriving after it
                    std::string key = keys.front();
                    for (const std::string &k : keys)
                        if (k > last) { key = k; break; }
                    double oldest = now() - kStarveSeconds;
                    for (const auto &kv : running) {
                        const Request *r = kv.second;
                        if (r->t_submit < oldest && std::binary_search(keys.begin(), keys.end(), r->family)) {
                            oldest = r->t_submit;
                            key = r->family;
                        }
                    }
                    last = key;
                    hfm::ResidentFamily &F = *fams[key];
                    try {
                        F.activate();
                        *attn_host = 0u;
                        if (F.has_work()) {
                            F.slice_begin(attn_dev, 1.0, keys.size() > 1 ? 4.0 : 0.0);
                            slice_t0 = Clock::now();
                            cur = key;
                        }
                    } catch (const std::exception &e) {
                        fail_family(key, error_code_of(e), e.what());
                    }
                    // instances without seeds converge at once
                    if (cur.empty() && fams.count(key)) {
                        std::vector<int64_t> done;
                        try {
                            fams[key]->collect(done);
                        } catch (const std::exception &e) {
                            fail_family(key, error_code_of(e), e.what());
                            done.clear();
                        }
                        for (int64_t t : done) finished.emplace_back(key, t);
                    }
                }
            }
            // ---- results of the converged instances, copied out while the next slice runs
            for (const auto &d : finished) {
                Request *r = running[d.second];
                running.erase(d.second);
                int rc = HFM_OK;
                hfm::EulerResult res;
                try {
                    fams.at(d.first)->finish(d.second, res, side);
                    r->prep->finish(res);
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
        }
        fams.clear();
        cudaStreamSynchronize(side);
        cudaStreamSynchronize(stream);
        {
            std::lock_guard<std::mutex> lk(mu);
            attn_host = nullptr;
        }
        cudaFreeHost(host_word);
        cudaStreamDestroy(side);
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
        // inputs staged ahead of admission: a quarter of the budget, at most 4 GiB
        s->staged_cap = std::min(s->budget / 4, size_t(4) << 30);
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
        s->intake = std::thread([p = s.get()] { p->intake_main(); });
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
    s->cv_intake.notify_one();
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
    s->cv_intake.notify_all();
    s->cv_work.notify_all();
    if (s->intake.joinable()) s->intake.join();
    if (s->scheduler.joinable()) s->scheduler.join();
    delete s;
}

}  // extern "C"
