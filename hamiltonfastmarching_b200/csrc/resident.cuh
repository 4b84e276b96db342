// Resident solver of the serving loop: instances of one model family (stencil shape and precision)
// live in a device arena and enter and leave one persistent solver between its slices.
//
// Included by eulerian.cu inside namespace hfm::detail, after the batch solver whose kernels it
// reuses (stencils, walls, visibility, seeds, tile dependencies, process_tile).
//
// The reference answers one Run(IO&) at a time (Headers/DispatchAndRun.h:224-244), each a fast
// marching front (Headers/Base/Implementation/HamiltonFastMarching.hxx:59-183). Here every admitted
// instance owns a range of the arena's global tile space (its stencil codes and weights or its
// visibility words and speed multipliers, its values, its scheduling words and its reverse tile
// dependencies), so a running solver takes new instances at its next slice and releases each one
// as soon as its own tiles drain: no instance waits for a larger one admitted with it.
//
// Scheduling: the batch solver's value-ordered bands, kept per instance. Round r solves, for each
// instance i, the active tiles whose key is at most (smallest key of i) + delta_i; delta_i starts
// from the spread of i's first wake-up keys and doubles (halves) when i solved fewer (more) tiles
// than [lo, hi] x the resident warps in the round before, as it would alone: a small instance takes
// all its tiles each round while a large one keeps its own band. Per instance,
// the statistics rows (smallest and largest wake-up key, tiles solved) and the count of its tiles
// in each list are kept by the list pushes; an instance whose count in the next list is zero has
// converged. A slice ends when an instance converges (so it is released at once), when no tile is
// left, or when the host has raised the attention word (requests wait for admission) and the
// slice has run its minimum time, or at its time limit when other families wait.

constexpr int kMaxResident = 256;  // instance slots of a family (per-instance statistics rows)
constexpr int kAdmissionSms = 8;   // SMs' worth of capacity a slice leaves to admission kernels
constexpr int kSliceCarveoutPct = 100;  // shared-memory carveout of a slice's SMs, percent of the maximum

// A request's large inputs on the device: the FP64 metric (Riemann models) or speed multiplier
// (shared-stencil models) in the input's row-major order, and the walls as bytes.
struct StagedImpl final : StagedInputs {
    DeviceBuffer<double> field;
    DeviceBuffer<uint8_t> walls;
    cudaEvent_t ready = nullptr;  // recorded after the uploads, on the staging stream
    size_t nbytes = 0;
    size_t bytes() const override { return nbytes; }
    ~StagedImpl() override {
        // the buffers are freed on the destroying thread's stream, after the uploads
        if (ready) {
            cudaStreamWaitEvent(current_stream(), ready, 0);
            cudaEventDestroy(ready);
        }
    }
};

inline std::unique_ptr<StagedInputs> stage_inputs_impl(const EulerProblem &p) {
    cudaStream_t s = current_stream();
    auto st = std::make_unique<StagedImpl>();
    const long long N = (long long)p.dims[0] * p.dims[1] * p.dims[2];
    if (p.kind == StencilKind::RiemannPerCell) {
        const int NS = p.ndim * (p.ndim + 1) / 2;
        const size_t rows = p.metric_constant ? 1 : (size_t)N;
        st->field.alloc(rows * NS);
        staged_upload(st->field.get(), p.metric_ptr ? p.metric_ptr : p.metric.data(), rows * NS * sizeof(double), s);
        st->nbytes += rows * NS * sizeof(double);
    } else {
        const long long nm[4] = {1, p.dims[2], (long long)p.dims[0] * p.dims[1], N};
        const long long len = nm[std::min(3, std::max(0, p.mult_depth))];
        st->field.alloc(len);
        staged_upload(st->field.get(), p.mult_ptr ? p.mult_ptr : p.mult.data(), len * sizeof(double), s);
        st->nbytes += len * sizeof(double);
    }
    if (!p.walls.empty() || p.walls_f64) {
        st->walls.alloc(N);
        if (!p.walls.empty()) {
            staged_upload(st->walls.get(), p.walls.data(), N, s);
        } else {
            DeviceBuffer<double> wf(N);
            staged_upload(wf.get(), p.walls_f64, N * sizeof(double), s);
            launch(walls_from_f64_kernel, nblocks(N, 256), 256, 0, s, N, (const double *)wf.get(), st->walls.get());
        }
        st->nbytes += N;
    }
    HFM_CUDA(cudaEventCreateWithFlags(&st->ready, cudaEventDisableTiming));
    HFM_CUDA(cudaEventRecord(st->ready, s));
    return st;
}

struct ServeCtl {
    long long round0;              // round at which the slice starts (lists and rows continue)
    const int *active;             // [nactive] instance slots with tiles in the lists
    int nactive;
    double *delta;                 // [kMaxResident] band width per slot, kept across slices
    unsigned *age;                 // [kMaxResident] rounds since admission
    unsigned *stop;                // [2] stop words by round parity: written by block 0 before a
                                   // barrier, read after it (block 0 can be one round ahead)
    long long *round_out;          // first round of the next slice, written at exit
    const volatile unsigned *attn; // host-mapped attention word (requests waiting), or null
    unsigned long long min_ns;     // attention is honoured once the slice has run this long
    unsigned long long max_ns;     // hard slice length (0: none)
    unsigned lo, hi;               // solved tiles per round and instance kept in [lo, hi]
    long long max_rounds;          // round cap of the slice
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void __launch_bounds__(kWarpsPerCta * 32, (fim_min_blocks<Real, NFWD, NSYM, KIND>()))
    fim_resident_kernel(Dev<Real> P, ServeCtl C) {
    __shared__ Real s_vals[kWarpsPerCta][64];
    __shared__ double s_delta[kMaxResident];
    __shared__ unsigned s_age[kMaxResident];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long kInfBits = 0x7ff0000000000000ull;
    for (int a = threadIdx.x; a < C.nactive; a += blockDim.x) {
        const int i = C.active[a];
        s_delta[i] = C.delta[i];
        s_age[i] = C.age[i];
    }
    __syncthreads();
    const unsigned long long t0 = global_ns();
    unsigned long long n_act = 0, n_solves = 0;
    StatAcc acc;
    int cnt_inst = -1;               // tiles solved by this warp in this round for instance cnt_inst
    unsigned long long cnt = 0;
    long long r = C.round0;
    bool ok = true;
    for (long long it = 0; it < C.max_rounds; ++it, ++r) {
        const int cur = (int)(r % 3), nxt = (int)((r + 1) % 3), old = (int)((r + 2) % 3);
        const int slot = (int)(r & 7), nslot = (int)((r + 1) & 7), rslot = (int)((r + 4) & 7);
        if (blockIdx.x == 0) {
            if (threadIdx.x == 0) {
                *P.count[old] = 0;
                *P.claim[old] = 0;
            }
            for (int a = threadIdx.x; a < C.nactive; a += blockDim.x) {
                const int i = C.active[a];
                unsigned long long *row = P.rstat + ((long long)rslot * P.nslots + i) * 4;
                row[0] = kInfBits;
                row[1] = 0ull;
                row[2] = 0ull;
                P.live[old * P.nslots + i] = 0u;
            }
        }
        const unsigned n = *(volatile unsigned *)P.count[cur];
        while (true) {
            unsigned i = 0;
            if (lane == 0) i = atomicAdd(P.claim[cur], 1u);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= n) break;
            const int T = P.list[cur][i];
            const int inst = P.tile_inst[T];
            unsigned long long kt = 0;
            int cls = 0;
            if (lane == 0) {
                P.flag[cur][T] = 0u;
                kt = *(volatile unsigned long long *)(P.key + T);
                const unsigned long long mk =
                    *(volatile unsigned long long *)(P.rstat + ((long long)slot * P.nslots + inst) * 4);
                cls = entry_class(P, T, kt, __longlong_as_double(mk) + s_delta[inst]);
            }
            kt = __shfl_sync(0xffffffffu, kt, 0);
            cls = __shfl_sync(0xffffffffu, cls, 0);
            if (cls == kEntryStale) continue;
            if (cls == kEntryCarried) {
                // not yet in its instance's band: carry to the next round with its key
                push_tiles(P, nxt, T, lane == 0, lane, inst);
                stat_add(P, acc, nslot, inst, kt, 0ull, lane);
                continue;
            }
            if (lane == 0) atomicExch(P.key + T, kInfBits);
            __threadfence();  // the key is cleared before the tile's pending cells are taken
            process_tile<Real, NFWD, NSYM, KIND>(P, T, s_vals[warp], lane, nxt, nslot, n_solves, acc);
            if (inst != cnt_inst) {
                if (cnt && lane == 0) atomicAdd(P.rstat + ((long long)slot * P.nslots + cnt_inst) * 4 + 2, cnt);
                cnt_inst = inst;
                cnt = 0;
            }
            ++cnt;
            ++n_act;
        }
        stat_flush(P, acc, lane);
        if (cnt && lane == 0) atomicAdd(P.rstat + ((long long)slot * P.nslots + cnt_inst) * 4 + 2, cnt);
        cnt_inst = -1;
        cnt = 0;
        // the stop decision is block 0's, published before the barrier so that every block reads
        // the same word after it
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long el = global_ns() - t0;
            const bool want = (C.max_ns && el >= C.max_ns) || (C.attn && *C.attn != 0u && el >= C.min_ns);
            ((volatile unsigned *)C.stop)[r & 1] = want ? 1u : 0u;
        }
        ok = grid_barrier(P.bar_count, P.bar_gen, gridDim.x, P.status, kBarrierPolls);
        if (!ok) break;
        if (*(volatile unsigned *)P.count[nxt] == 0u) { ++r; break; }  // every instance converged
        // per-instance band update, identical in every block; each slot is one thread's
        bool finished = false;
        {
            for (int a = threadIdx.x; a < C.nactive; a += blockDim.x) {
                const int i = C.active[a];
                if (*(volatile unsigned *)(P.live + nxt * P.nslots + i) == 0u) { finished = true; continue; }
                const unsigned long long *row = P.rstat + ((long long)slot * P.nslots + i) * 4;
                const unsigned long long np = *(volatile const unsigned long long *)(row + 2);
                if (s_age[i] == 0u) {
                    const unsigned long long *nrow = P.rstat + ((long long)nslot * P.nslots + i) * 4;
                    const double lo_k = __longlong_as_double(*(volatile const unsigned long long *)(nrow + 0));
                    const double hi_k = __longlong_as_double(*(volatile const unsigned long long *)(nrow + 1));
                    s_delta[i] = hi_k > lo_k ? 2.0 * (hi_k - lo_k) : Arith<double>::inf();
                } else if (np < C.lo) {
                    s_delta[i] *= 2.0;
                } else if (np > C.hi) {
                    s_delta[i] *= 0.5;
                }
                ++s_age[i];
            }
        }
        finished = __syncthreads_or(finished);
        if (finished || ((volatile unsigned *)C.stop)[r & 1]) { ++r; break; }
    }
    if (ok && blockIdx.x == 0 && threadIdx.x == 0) {
        *C.round_out = r;
        if (r - C.round0 >= C.max_rounds) atomicOr(P.status, (unsigned)kErrRoundCap);
    }
    if (ok && blockIdx.x == 0) {
        for (int a = threadIdx.x; a < C.nactive; a += blockDim.x) {
            const int i = C.active[a];
            C.delta[i] = s_delta[i];
            C.age[i] = s_age[i];
        }
    }
    if (lane == 0) atomicAdd(P.stats + 1, n_act);
#pragma unroll
    for (int o = 16; o; o >>= 1) n_solves += __shfl_xor_sync(0xffffffffu, n_solves, o);
    if (lane == 0) atomicAdd(P.stats + 2, n_solves);
}

// Seed tiles of a new instance into list `li`, with the statistics rows of round slot `slot`.
template <typename Real>
__global__ void inject_kernel(Dev<Real> P, int li, int slot, const int *seed_tiles, const unsigned long long *seed_masks,
                              int n) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= n) return;
    StatAcc acc;
    push_dependents(P, li, slot, seed_tiles[wid], seed_masks[wid], ~0ull, 0ull, 0ull, lane, acc);
    stat_flush(P, acc, lane);
}

// An instance's reverse dependency CSR (local tile ids) into the arena: per-tile entry ranges and
// global tile ids.
__global__ void deps_to_arena_kernel(long long nt, long long tile0, long long e0, const long long *rptr,
                                     long long *dep_beg, long long *dep_end) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nt) return;
    dep_beg[tile0 + t] = e0 + rptr[t];
    dep_end[tile0 + t] = e0 + rptr[t + 1];
}

__global__ void entries_to_arena_kernel(long long ne, long long tile0, const int *rtile, const unsigned long long *rmask,
                                        const unsigned long long *rdmask, int *dep_tile, unsigned long long *dep_mask,
                                        unsigned long long *dep_dmask) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= ne) return;
    dep_tile[j] = (int)(tile0 + rtile[j]);
    dep_mask[j] = rmask[j];
    dep_dmask[j] = rdmask[j];
}

// First-fit allocator of index ranges [0, cap).
class RangeAlloc {
public:
    void init(long long cap) {
        free_.clear();
        if (cap > 0) free_[0] = cap;
        cap_ = cap;
    }
    long long alloc(long long n) {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const long long at = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[at + n] = len - n;
            return at;
        }
        return -1;
    }
    void release(long long at, long long n) {
        if (n <= 0) return;
        auto it = free_.emplace(at, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    // grows the range to [0, cap): the new tail is free
    void grow(long long cap) {
        if (cap <= cap_) return;
        release(cap_, cap - cap_);
        cap_ = cap;
    }
    long long capacity() const { return cap_; }

private:
    std::map<long long, long long> free_;
    long long cap_ = 0;
};

template <typename Real, int NFWD, int NSYM, int KIND>
class Resident final : public ResidentFamily {
    static constexpr int ND = NFWD + NSYM, NB = NFWD + 2 * NSYM;
    static constexpr bool SHARE = is_share(KIND);
    static_assert(KIND != kKindTTI, "TTI3 is served through the single-solve path");

    struct Entry {
        int64_t ticket = 0;
        int slot = -1;
        GridGeom g{};
        long long tile0 = 0, nt = 0, e0 = 0, ne = 0, cls0 = 0, ncls = 0;
        long long round_in = 0, rounds = 0;
        int max_width = 0;
        double *h_out = nullptr;
        float setup_ms = 0;
        std::vector<int> seed_tiles;               // arena tiles holding seeds, with their cells
        std::vector<unsigned long long> seed_masks;
        std::chrono::steady_clock::time_point t_admit, t_solved;
    };

    // arena arrays
    long long cap_t_ = 0, cap_e_ = 0, cap_c_ = 0;  // tiles, dependency entries, stencil classes
    DeviceBuffer<unsigned> code_, vis_, tile_up_, flags_, live_, ctl_, age_;
    DeviceBuffer<Real> weight_, mult_, values_, cls_w_;
    DeviceBuffer<int8_t> cls_off_;
    DeviceBuffer<int> tile_inst_, lists_, dep_tile_, active_d_;
    DeviceBuffer<unsigned long long> key_, maxval_, dep_mask_, dep_dmask_, rstat_, stats_;
    DeviceBuffer<DirtyWake> dirty_;
    DeviceBuffer<long long> dep_beg_, dep_end_, round_out_;
    DeviceBuffer<double> delta_;
    DeviceBuffer<Inst> inst_;
    RangeAlloc tiles_, entries_, classes_;
    std::vector<int> free_slots_;
    std::map<int, Entry> pending_, active_;  // by slot: prepared, in the lists
    std::map<int64_t, Entry> collected_;      // by ticket: converged, result not yet copied out
    long long round_ = 0;
    bool in_slice_ = false;
    cudaEvent_t done_ev_ = nullptr;           // end of the running slice
    long long *h_ctl_ = nullptr;              // page-locked (pinned_words): round reached, status word
    std::unique_lock<std::mutex> coop_;       // the cooperative-launch lock, held during a slice
    struct Schedule {
        int sweeps = 2;
        double band_lo = 2.0, band_hi = 8.0;
        long long max_rounds = 1 << 20;
    } sched_;
    bool broken_ = false;

    static size_t bytes_per_tile() {
        const size_t per_cell = SHARE ? (4 + 2 * sizeof(Real)) : (ND * (4 + sizeof(Real)) + sizeof(Real));
        return 64 * per_cell + 4 + 8 * 3 + 4 + 12 + 12 + 16;
    }

    Dev<Real> global_view() {
        Dev<Real> P{};
        P.inst = inst_.get();
        P.ninst = kMaxResident;
        P.tile_inst = tile_inst_.get();
        P.ntile = cap_t_;
        P.ntc = cap_t_ * 64;
        P.sstride = cap_t_ * 64;
        P.ncells = cap_t_ * 64;
        P.values = values_.get();
        P.code = code_.get();
        P.weight = weight_.get();
        P.mult = mult_.get();
        P.vis = vis_.get();
        P.cls_off = cls_off_.get();
        P.cls_w = cls_w_.get();
        P.dep_ptr = dep_beg_.get();
        P.dep_end = dep_end_.get();
        P.dep_tile = dep_tile_.get();
        P.dep_mask = dep_mask_.get();
        P.dep_dmask = dep_dmask_.get();
        P.dirty = dirty_.get();
        P.key = key_.get();
        P.skip_settled = true;
        P.maxval = maxval_.get();
        P.rstat = rstat_.get();
        P.nslots = kMaxResident;
        P.live = live_.get();
        P.tile_up = tile_up_.get();
        for (int i = 0; i < 3; ++i) {
            P.list[i] = lists_.get() + i * cap_t_;
            P.flag[i] = flags_.get() + i * cap_t_;
            P.count[i] = ctl_.get() + i;
            P.claim[i] = ctl_.get() + 3 + i;
        }
        P.bar_count = ctl_.get() + 6;
        P.bar_gen = ctl_.get() + 7;
        P.status = ctl_.get() + 8;
        P.stats = stats_.get();
        P.max_rounds = (int)sched_.max_rounds;
        P.sweeps = sched_.sweeps;
        return P;
    }

    // Moves every arena array to capacities (tiles, entries, classes), keeping the contents.
    template <typename T>
    static void regrow(DeviceBuffer<T> &b, long long old_n, long long new_n, int planes, cudaStream_t s) {
        DeviceBuffer<T> nb((size_t)new_n * planes);
        HFM_CUDA(cudaMemsetAsync(nb.get(), 0, (size_t)new_n * planes * sizeof(T), s));
        if (b.get() && old_n > 0)
            for (int k = 0; k < planes; ++k)
                HFM_CUDA(cudaMemcpyAsync(nb.get() + (size_t)k * new_n, b.get() + (size_t)k * old_n,
                                         (size_t)old_n * sizeof(T), cudaMemcpyDeviceToDevice, s));
        b = std::move(nb);
    }

    void resize(long long ct, long long ce, long long cc, cudaStream_t s) {
        const long long ot = cap_t_, oe = cap_e_, oc = cap_c_;
        if (ct > ot) {
            if (!SHARE) {
                regrow(code_, ot * 64, ct * 64, ND, s);
                regrow(weight_, ot * 64, ct * 64, ND, s);
            } else {
                regrow(vis_, ot * 64, ct * 64, 1, s);
                regrow(mult_, ot * 64, ct * 64, 1, s);
            }
            regrow(values_, ot * 64, ct * 64, 1, s);
            regrow(tile_inst_, ot, ct, 1, s);
            regrow(dirty_, ot, ct, 1, s);
            regrow(key_, ot, ct, 1, s);
            regrow(maxval_, ot, ct, 1, s);
            regrow(tile_up_, ot, ct, 1, s);
            regrow(lists_, ot, ct, 3, s);
            regrow(flags_, ot, ct, 3, s);
            regrow(dep_beg_, ot, ct, 1, s);
            regrow(dep_end_, ot, ct, 1, s);
            tiles_.grow(ct);
            cap_t_ = ct;
        }
        if (ce > oe) {
            regrow(dep_tile_, oe, ce, 1, s);
            regrow(dep_mask_, oe, ce, 1, s);
            regrow(dep_dmask_, oe, ce, 1, s);
            entries_.grow(ce);
            cap_e_ = ce;
        }
        if (SHARE && cc > oc) {
            regrow(cls_off_, oc * ND * 3, cc * ND * 3, 1, s);
            regrow(cls_w_, oc * ND, cc * ND, 1, s);
            classes_.grow(cc);
            cap_c_ = cc;
        }
    }

    static long long pow2_at_least(long long n) {
        long long c = 1;
        while (c < n) c <<= 1;
        return c;
    }

public:
    // The family's schedule (local sweeps per activation, band limits) is the first request's.
    explicit Resident(const EulerProblem &first) {
        sched_.sweeps = first.sweeps_per_tile;
        sched_.band_lo = first.band_lo;
        sched_.band_hi = first.band_hi;
        sched_.max_rounds = first.max_rounds;
        cudaStream_t s = current_stream();
        inst_.alloc(kMaxResident);
        HFM_CUDA(cudaMemsetAsync(inst_.get(), 0, kMaxResident * sizeof(Inst), s));
        rstat_.alloc((size_t)8 * kMaxResident * 4);
        HFM_CUDA(cudaMemsetAsync(rstat_.get(), 0, (size_t)8 * kMaxResident * 4 * 8, s));
        live_.alloc(3 * kMaxResident);
        live_.zero(s);
        ctl_.alloc(16);
        ctl_.zero(s);
        stats_.alloc(4);
        stats_.zero(s);
        delta_.alloc(kMaxResident);
        age_.alloc(kMaxResident);
        age_.zero(s);
        active_d_.alloc(kMaxResident);
        round_out_.alloc(1);
        for (int i = kMaxResident - 1; i >= 0; --i) free_slots_.push_back(i);
        resize(1 << 15, 1 << 20, SHARE ? 1 << 10 : 0, s);
        h_ctl_ = static_cast<long long *>(pinned_words(2 * sizeof(long long)));
        h_ctl_[0] = h_ctl_[1] = 0;
    }

    size_t arena_bytes() const override {
        return (size_t)cap_t_ * bytes_per_tile() + (size_t)cap_e_ * 20 + (size_t)cap_c_ * ND * (3 + sizeof(Real));
    }

    bool has_work() const override { return !active_.empty(); }
    bool has_pending() const override { return !pending_.empty(); }
    int resident() const override { return (int)(active_.size() + pending_.size() + collected_.size()); }

    Admit prepare(const EulerProblem &p, int64_t ticket, const StagedInputs *staged_in, bool may_grow, cudaStream_t s,
                  int *max_width) override {
        if (broken_) throw Error(HFM_ERR_CUDA, "the resident solver of this family failed earlier");
        if (free_slots_.empty()) return kNoSlot;
        StreamScope scope(s);  // temporaries of the build are stream-ordered on `s`
        const StagedImpl *staged = dynamic_cast<const StagedImpl *>(staged_in);
        if (staged) HFM_CUDA(cudaStreamWaitEvent(s, staged->ready, 0));
        const GridGeom g = make_geom(p.ndim, p.dims, p.periodic, p.tile_shift[0] >= 0 ? p.tile_shift : nullptr);
        const long long nt = g.ntile, N = g.ncells;
        const long long ncls = SHARE ? p.nclass : 0;
        // room in the arena: grow it (doubling) if the tiles or classes do not fit
        long long tile0 = tiles_.alloc(nt);
        long long cls0 = SHARE ? classes_.alloc(ncls) : 0;
        if (tile0 < 0 || cls0 < 0) {
            if (tile0 >= 0) tiles_.release(tile0, nt);
            if (cls0 >= 0 && SHARE) classes_.release(cls0, ncls);
            if (!may_grow) return kNeedsGrow;
            resize(tile0 < 0 ? pow2_at_least(cap_t_ + nt) : cap_t_, cap_e_,
                   SHARE && cls0 < 0 ? pow2_at_least(cap_c_ + ncls) : cap_c_, s);
            tile0 = tiles_.alloc(nt);
            cls0 = SHARE ? classes_.alloc(ncls) : 0;
            if (tile0 < 0 || cls0 < 0) throw Error(HFM_ERR_NOMEM, "resident arena allocation failed");
        }
        Entry E;
        E.ticket = ticket;
        E.g = g;
        E.tile0 = tile0;
        E.nt = nt;
        E.cls0 = cls0;
        E.ncls = ncls;
        E.h_out = p.h_values_out;
        E.t_admit = std::chrono::steady_clock::now();
        bool grow_refused = false;
        auto undo = [&] {
            tiles_.release(tile0, nt);
            if (SHARE) classes_.release(cls0, ncls);
        };
        EventTimer tm;
        tm.start(s);
        try {
            // ---- local view of the instance's arena range (its own tile and cell numbering)
            Inst I{};
            I.g = g;
            for (int a = 0; a < 3; ++a) I.h[a] = p.h[a];
            I.dual = p.dual;
            I.metric_const = p.metric_constant;
            I.has_walls = (!p.walls.empty() || p.walls_f64) ? 1 : 0;
            I.mult_depth = p.mult_depth;
            I.mult_inverse = p.mult_inverse ? 1 : 0;
            DeviceBuffer<Inst> linst;
            linst.upload(&I, 1, s);
            DeviceBuffer<int> lzero(nt);
            lzero.zero(s);
            DeviceBuffer<unsigned> lstatus(1), maxw(1);
            lstatus.zero(s);
            maxw.zero(s);
            Dev<Real> V{};
            V.inst = linst.get();
            V.ninst = 1;
            V.tile_inst = lzero.get();
            V.ncells = N;
            V.ntile = nt;
            V.ntc = nt * 64;
            V.sstride = cap_t_ * 64;
            V.status = lstatus.get();
            V.values = values_.get() + tile0 * 64;
            if (!SHARE) {
                V.code = code_.get() + tile0 * 64;
                V.weight = weight_.get() + tile0 * 64;
            } else {
                V.vis = vis_.get() + tile0 * 64;
                V.mult = mult_.get() + tile0 * 64;
                V.cls_off = cls_off_.get() + cls0 * ND * 3;
                V.cls_w = cls_w_.get() + cls0 * ND;
            }
            // fresh scheduling words for the range
            launch(fill_kernel<Real>, std::min<unsigned>(nblocks(nt * 64, 256), 4096), 256, 0, s, V.values, nt * 64,
                   Arith<Real>::inf());
            launch(fill_kernel<DirtyWake>, nblocks(nt, 256), 256, 0, s, dirty_.get() + tile0, nt,
                   DirtyWake{0ull, kInfWake});
            HFM_CUDA(cudaMemsetAsync(tile_up_.get() + tile0, 0, nt * sizeof(unsigned), s));
            for (int l = 0; l < 3; ++l)
                HFM_CUDA(cudaMemsetAsync(flags_.get() + l * cap_t_ + tile0, 0, nt * sizeof(unsigned), s));
            launch(fill_kernel<unsigned long long>, nblocks(nt, 256), 256, 0, s, key_.get() + tile0, nt,
                   0x7ff0000000000000ull);
            launch(fill_kernel<unsigned long long>, nblocks(nt, 256), 256, 0, s, maxval_.get() + tile0, nt,
                   0x7ff0000000000000ull);

            // ---- stencils
            unsigned hmaxw = 0;
            DeviceBuffer<uint8_t> cls_en;
            if (!SHARE) {
                for (int k = 0; k < ND; ++k) {
                    HFM_CUDA(cudaMemsetAsync(V.code + (size_t)k * V.sstride, 0, nt * 64 * sizeof(unsigned), s));
                    HFM_CUDA(cudaMemsetAsync(V.weight + (size_t)k * V.sstride, 0, nt * 64 * sizeof(Real), s));
                }
                const int NS = p.ndim * (p.ndim + 1) / 2;
                DeviceBuffer<double> metric;
                const double *dmetric = staged ? staged->field.get() : nullptr;
                if (!dmetric) {
                    const size_t rows = p.metric_constant ? 1 : (size_t)N;
                    metric.alloc(rows * NS);
                    staged_upload(metric.get(), p.metric_ptr ? p.metric_ptr : p.metric.data(), rows * NS * sizeof(double),
                                  s);
                    dmetric = metric.get();
                }
                if (p.ndim == 2)
                    launch(riemann_stencil_kernel<2, Real>, nblocks(N, 128), 128, 0, s, V, dmetric, (int8_t *)nullptr,
                           (double *)nullptr);
                else
                    launch(riemann_stencil_kernel<3, Real>, nblocks(N, 128), 128, 0, s, V, dmetric, (int8_t *)nullptr,
                           (double *)nullptr);
                launch(width_kernel<Real, NSYM>, nblocks(N, 256), 256, 0, s, V, maxw.get());
                maxw.download(&hmaxw, 1, s);
            } else {
                std::vector<Real> hw(p.cls_w.begin(), p.cls_w.end());
                HFM_CUDA(cudaMemcpyAsync((void *)V.cls_off, p.cls_off.data(), p.cls_off.size(), cudaMemcpyHostToDevice, s));
                HFM_CUDA(cudaMemcpyAsync((void *)V.cls_w, hw.data(), hw.size() * sizeof(Real), cudaMemcpyHostToDevice, s));
                cls_en.upload(p.cls_enabled, s);
                const long long nm[4] = {1, g.dims[2], (long long)g.dims[0] * g.dims[1], g.ncells};
                const long long len = nm[std::min(3, std::max(0, p.mult_depth))];
                DeviceBuffer<double> mult_rm;
                const double *dmult = staged ? staged->field.get() : nullptr;
                if (!dmult) {
                    mult_rm.alloc(len);
                    staged_upload(mult_rm.get(), p.mult_ptr ? p.mult_ptr : p.mult.data(), len * sizeof(double), s);
                    dmult = mult_rm.get();
                }
                HFM_CUDA(cudaMemsetAsync(V.mult, 0, nt * 64 * sizeof(Real), s));
                HFM_CUDA(cudaMemsetAsync(V.vis, 0, nt * 64 * sizeof(unsigned), s));
                launch(mult_layout_kernel<Real>, nblocks(N, 256), 256, 0, s, V, dmult);
                int mw = 0;
                for (int cl = 0; cl < p.nclass; ++cl)
                    for (int k = 0; k < ND; ++k) {
                        if (p.cls_w[cl * ND + k] == 0.0) continue;
                        const int8_t *o = &p.cls_off[(cl * ND + k) * 3];
                        for (int si = 0; si < (k < NFWD ? 1 : 2); ++si) {
                            const int sl = k < NFWD ? k : NFWD + 2 * (k - NFWD) + si;
                            if (!p.cls_enabled[cl * NB + sl]) continue;
                            mw = std::max(mw, std::abs(o[0]) + std::abs(o[1]) + std::abs(o[2]));
                        }
                    }
                hmaxw = (unsigned)mw;
                maxw.upload(&hmaxw, 1, s);
                HFM_CUDA(cudaStreamSynchronize(s));  // the host staging of cls_w above
            }
            HFM_CUDA(cudaStreamSynchronize(s));
            E.max_width = (int)hmaxw;
            // ---- walls and visibility
            DeviceBuffer<uint8_t> walls;
            DeviceBuffer<int> wdist;
            DeviceBuffer<int8_t> wd8;
            if (I.has_walls) {
                const uint8_t *dwalls = staged && staged->walls.get() ? staged->walls.get() : nullptr;
                if (!dwalls) {
                    walls.alloc(N);
                    if (!p.walls.empty()) {
                        staged_upload(walls.get(), p.walls.data(), N, s);
                    } else {
                        DeviceBuffer<double> wf(N);
                        staged_upload(wf.get(), p.walls_f64, N * sizeof(double), s);
                        launch(walls_from_f64_kernel, nblocks(N, 256), 256, 0, s, N, (const double *)wf.get(), walls.get());
                    }
                    dwalls = walls.get();
                }
                wdist.alloc(N);
                wd8.alloc(N);
                launch(wall_init_kernel, nblocks(N, 256), 256, 0, s, N, dwalls, wdist.get());
                for (int a = 0; a < 3; ++a) {
                    if (g.dims[a] == 1) continue;
                    const long long nl = g.ncells / g.dims[a];
                    launch(wall_scan_kernel, nblocks(nl, 128), 128, 0, s, g, a, wdist.get());
                }
                launch(wall_cap_kernel<Real>, nblocks(N, 256), 256, 0, s, V, (const int *)wdist.get(),
                       (const unsigned *)maxw.get(), wd8.get());
            }
            launch(visibility_kernel<Real, NFWD, NSYM, KIND>, nblocks(nt * 64, 128), 128, 0, s, V,
                   (const int8_t *)wd8.get(), (const uint8_t *)cls_en.get());
            // ---- seeds (local indices) and their tiles
            std::vector<long long> hsi(p.seed_index.begin(), p.seed_index.end());
            for (long long x : hsi) {
                const int x2 = (int)(x % g.dims[2]);
                const long long rr = x / g.dims[2];
                const int x1 = (int)(rr % g.dims[1]), x0 = (int)(rr / g.dims[1]);
                const int T = (int)(tile0 + g.tile_of(x0, x1, x2));
                const int b = g.local_of(x0, x1, x2);
                auto it = std::find(E.seed_tiles.begin(), E.seed_tiles.end(), T);
                if (it == E.seed_tiles.end()) {
                    E.seed_tiles.push_back(T);
                    E.seed_masks.push_back(1ull << b);
                } else {
                    E.seed_masks[it - E.seed_tiles.begin()] |= 1ull << b;
                }
            }
            DeviceBuffer<long long> sidx;
            DeviceBuffer<double> sval;
            sidx.upload(hsi, s);
            sval.upload(p.seed_value, s);
            launch(seeds_kernel<Real, KIND>, nblocks((long long)hsi.size(), 128), 128, 0, s, V,
                   (const long long *)sidx.get(), (const double *)sval.get(), (int)hsi.size());
            // ---- reverse tile dependencies (local CSR), then into the arena's entry space
            DeviceBuffer<unsigned> dcnt(nt);
            // the dependency kernels hold shared-memory tables: they ask for the slice's carveout, so
            // that an SM running slice blocks is already split the way they want
            static std::once_flag deps_carveout;
            std::call_once(deps_carveout, [] {
                HFM_CUDA(cudaFuncSetAttribute(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapSmall, kDepWarpsSmall>,
                                              cudaFuncAttributePreferredSharedMemoryCarveout, kSliceCarveoutPct));
                HFM_CUDA(cudaFuncSetAttribute(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapLarge, kDepWarpsLarge>,
                                              cudaFuncAttributePreferredSharedMemoryCarveout, kSliceCarveoutPct));
            });
            auto deps_pass = [&](bool large, int pass, const long long *offs, int *src, int *dst, unsigned long long *msk,
                                 unsigned long long *dmsk) {
                if (large)
                    launch(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapLarge, kDepWarpsLarge>, nblocks(nt, kDepWarpsLarge),
                           kDepWarpsLarge * 32, 0, s, V, pass, dcnt.get(), offs, src, dst, msk, dmsk);
                else
                    launch(deps_kernel<Real, NFWD, NSYM, KIND, kDepCapSmall, kDepWarpsSmall>, nblocks(nt, kDepWarpsSmall),
                           kDepWarpsSmall * 32, 0, s, V, pass, dcnt.get(), offs, src, dst, msk, dmsk);
            };
            bool large = false;
            deps_pass(false, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
            unsigned st0 = 0;
            lstatus.download(&st0, 1, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            if (st0 & kErrSelling)
                throw Error(HFM_ERR_VALUE, "ObtuseSuperbase error : input must be positive definite (metric rejected by Selling)");
            if (st0 & kErrTableOverflow) {
                const unsigned keep = st0 & ~(unsigned)kErrTableOverflow;
                HFM_CUDA(cudaMemcpyAsync(lstatus.get(), &keep, sizeof(unsigned), cudaMemcpyHostToDevice, s));
                large = true;
                deps_pass(true, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
            }
            std::vector<unsigned> hc(nt);
            dcnt.download(hc.data(), nt, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            std::vector<long long> ho(nt + 1, 0);
            long long ne = 0;
            for (long long t = 0; t < nt; ++t) { ho[t] = ne; ne += hc[t]; }
            ho[nt] = ne;
            long long e0 = entries_.alloc(std::max(1ll, ne));
            if (e0 < 0) {
                if (!may_grow) {
                    grow_refused = true;
                    throw Error(HFM_ERR_NOMEM, "dependency entries do not fit while the solver runs");
                }
                resize(cap_t_, pow2_at_least(cap_e_ + ne), cap_c_, s);
                V.sstride = cap_t_ * 64;  // unchanged: only the entry space grew
                e0 = entries_.alloc(std::max(1ll, ne));
                if (e0 < 0) throw Error(HFM_ERR_NOMEM, "resident arena allocation failed");
            }
            E.e0 = e0;
            E.ne = std::max(1ll, ne);
            DeviceBuffer<long long> doff(nt + 1), rptr(nt + 1);
            doff.upload(ho, s);
            DeviceBuffer<int> rtile(std::max(1ll, ne));
            DeviceBuffer<unsigned long long> rmask(std::max(1ll, ne)), rdmask(std::max(1ll, ne));
            {
                DeviceBuffer<int> esrc(std::max(1ll, ne)), edst(std::max(1ll, ne));
                DeviceBuffer<unsigned long long> emsk(std::max(1ll, ne)), edmsk(std::max(1ll, ne));
                if (ne) deps_pass(large, 1, doff.get(), esrc.get(), edst.get(), emsk.get(), edmsk.get());
                DeviceBuffer<unsigned> rcnt(nt), cursor(nt);
                rcnt.zero(s);
                cursor.zero(s);
                if (ne) launch(dep_count_kernel, nblocks(ne, 256), 256, 0, s, ne, (const int *)esrc.get(), rcnt.get());
                std::vector<unsigned> hr(nt);
                rcnt.download(hr.data(), nt, s);
                HFM_CUDA(cudaStreamSynchronize(s));
                std::vector<long long> hrp(nt + 1, 0);
                long long tot = 0;
                for (long long t = 0; t < nt; ++t) { hrp[t] = tot; tot += hr[t]; }
                hrp[nt] = tot;
                rptr.upload(hrp, s);
                if (ne)
                    launch(dep_scatter_kernel, nblocks(ne, 256), 256, 0, s, ne, (const int *)esrc.get(),
                           (const int *)edst.get(), (const unsigned long long *)emsk.get(),
                           (const unsigned long long *)edmsk.get(), (const long long *)rptr.get(), cursor.get(),
                           rtile.get(), rmask.get(), rdmask.get());
            }
            launch(deps_to_arena_kernel, nblocks(nt, 256), 256, 0, s, nt, tile0, e0, (const long long *)rptr.get(),
                   dep_beg_.get(), dep_end_.get());
            if (ne)
                launch(entries_to_arena_kernel, nblocks(ne, 256), 256, 0, s, ne, tile0, (const int *)rtile.get(),
                       (const unsigned long long *)rmask.get(), (const unsigned long long *)rdmask.get(),
                       dep_tile_.get() + e0, dep_mask_.get() + e0, dep_dmask_.get() + e0);
            lstatus.download(&st0, 1, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            if (st0 & kErrTableOverflow) throw Error(HFM_ERR_UNSUPPORTED, "stencil too wide for the tile dependency table");
            // ---- the instance's slot: global instance entry, tile ownership, fresh statistics
            const int slot = free_slots_.back();
            free_slots_.pop_back();
            E.slot = slot;
            Inst GI = I;
            GI.tile0 = tile0;
            GI.cell0 = tile0 * 64;
            GI.cls0 = cls0;
            HFM_CUDA(cudaMemcpyAsync(inst_.get() + slot, &GI, sizeof(Inst), cudaMemcpyHostToDevice, s));
            launch(fill_kernel<int>, nblocks(nt, 256), 256, 0, s, tile_inst_.get() + tile0, nt, slot);
            std::vector<unsigned long long> rows(8 * 4);
            for (int k = 0; k < 8; ++k) { rows[4 * k] = 0x7ff0000000000000ull; rows[4 * k + 1] = rows[4 * k + 2] = rows[4 * k + 3] = 0; }
            for (int k = 0; k < 8; ++k)
                HFM_CUDA(cudaMemcpyAsync(rstat_.get() + ((size_t)k * kMaxResident + slot) * 4, &rows[4 * k],
                                         4 * sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
            for (int l = 0; l < 3; ++l)
                HFM_CUDA(cudaMemsetAsync(live_.get() + l * kMaxResident + slot, 0, sizeof(unsigned), s));
            const double inf = Arith<double>::inf();
            const unsigned zero = 0;
            HFM_CUDA(cudaMemcpyAsync(delta_.get() + slot, &inf, sizeof(double), cudaMemcpyHostToDevice, s));
            HFM_CUDA(cudaMemcpyAsync(age_.get() + slot, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, s));
            HFM_CUDA(cudaGetLastError());
            HFM_CUDA(cudaStreamSynchronize(s));
            E.setup_ms = tm.stop(s);
            if (max_width) *max_width = E.max_width;
            pending_.emplace(slot, std::move(E));
        } catch (...) {
            if (E.e0 || E.ne) entries_.release(E.e0, E.ne);
            undo();
            if (E.slot >= 0) free_slots_.push_back(E.slot);
            if (grow_refused) return kNeedsGrow;
            throw;
        }
        return kPrepared;
    }

    void activate() override {
        cudaStream_t s = current_stream();
        for (auto &kv : pending_) {
            Entry &E = kv.second;
            if (!E.seed_tiles.empty()) {
                DeviceBuffer<int> stile;
                DeviceBuffer<unsigned long long> smask;
                stile.upload(E.seed_tiles, s);
                smask.upload(E.seed_masks, s);
                launch(inject_kernel<Real>, nblocks((long long)E.seed_tiles.size() * 32, 128), 128, 0, s, global_view(),
                       (int)(round_ % 3), (int)(round_ & 7), (const int *)stile.get(),
                       (const unsigned long long *)smask.get(), (int)E.seed_tiles.size());
                E.round_in = round_;
            } else {
                E.round_in = -1;  // nothing to solve: released at the next collection
            }
            E.t_admit = std::chrono::steady_clock::now();
            active_.emplace(kv.first, std::move(E));
        }
        pending_.clear();
        HFM_CUDA(cudaGetLastError());
    }

    void slice_begin(const volatile unsigned *attn_dev, double min_ms, double max_ms) override {
        if (in_slice_) throw Error(HFM_ERR_CUDA, "resident solver: a slice is already running");
        cudaStream_t s = current_stream();
        std::vector<int> act;
        for (const auto &kv : active_)
            if (kv.second.round_in >= 0) act.push_back(kv.first);
        if (act.empty()) return;
        HFM_CUDA(cudaMemcpyAsync(active_d_.get(), act.data(), act.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        HFM_CUDA(cudaMemsetAsync(ctl_.get() + 9, 0, 2 * sizeof(unsigned), s));  // stop words
        Dev<Real> P = global_view();
        int dev = 0, nsm = 0, per_sm = 0;
        HFM_CUDA(cudaGetDevice(&dev));
        HFM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        // the SMs that run a slice keep shared memory for the admission kernels beside it (their
        // dependency tables): without this the carveout can be sized for the slice's blocks alone,
        // and an admission waits for the slice to end
        static std::once_flag carveout;
        std::call_once(carveout, [] {
            HFM_CUDA(cudaFuncSetAttribute(fim_resident_kernel<Real, NFWD, NSYM, KIND>,
                                          cudaFuncAttributePreferredSharedMemoryCarveout, kSliceCarveoutPct));
        });
        HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fim_resident_kernel<Real, NFWD, NSYM, KIND>,
                                                               kWarpsPerCta * 32, 0));
        if (per_sm < 1) throw Error(HFM_ERR_CUDA, "resident solver kernel cannot be resident");
        // the capacity of a few SMs stays free for the admission kernels issued while the slice runs
        const int grid = std::max(1, nsm * per_sm - std::min(kAdmissionSms * per_sm, nsm * per_sm / 2));
        // each instance keeps the band it would have alone: the tiles of a round are the union of
        // the instances' bands, so a large instance is not slowed by the small ones beside it
        const double nwarps = (double)grid * kWarpsPerCta;
        ServeCtl C{};
        C.round0 = round_;
        C.active = active_d_.get();
        C.nactive = (int)act.size();
        C.delta = delta_.get();
        C.age = age_.get();
        C.stop = ctl_.get() + 9;
        C.round_out = round_out_.get();
        C.attn = attn_dev;
        C.min_ns = (unsigned long long)(min_ms * 1e6);
        C.max_ns = (unsigned long long)(max_ms * 1e6);
        C.lo = (unsigned)std::max(1.0, sched_.band_lo * nwarps);
        C.hi = (unsigned)std::max(2.0, sched_.band_hi * nwarps);
        C.max_rounds = sched_.max_rounds;
        void *args[] = {&P, &C};
        if (!done_ev_) HFM_CUDA(cudaEventCreateWithFlags(&done_ev_, cudaEventDisableTiming));
        count_launch();
        coop_ = std::unique_lock<std::mutex>(cooperative_mutex());
        try {
            HFM_CUDA(cudaLaunchCooperativeKernel((void *)fim_resident_kernel<Real, NFWD, NSYM, KIND>, dim3(grid),
                                                 dim3(kWarpsPerCta * 32), args, 0, s));
        } catch (...) {
            coop_.unlock();
            throw;
        }
        try {
            HFM_CUDA(cudaMemcpyAsync(h_ctl_, round_out_.get(), sizeof(long long), cudaMemcpyDeviceToHost, s));
            HFM_CUDA(cudaMemcpyAsync(h_ctl_ + 1, ctl_.get() + 8, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            HFM_CUDA(cudaEventRecord(done_ev_, s));
        } catch (...) {
            cudaStreamSynchronize(s);  // the launched slice ends before its arrays can go
            broken_ = true;
            coop_.unlock();
            throw;
        }
        in_slice_ = true;
    }

    bool slice_done() override {
        if (!in_slice_) return true;
        const cudaError_t e = cudaEventQuery(done_ev_);
        if (e == cudaErrorNotReady) return false;
        return true;  // an error is reported by slice_end
    }

    void slice_end() override {
        if (!in_slice_) return;
        in_slice_ = false;
        const cudaError_t e = cudaEventSynchronize(done_ev_);
        coop_.unlock();
        if (e != cudaSuccess) {
            broken_ = true;
            throw Error(HFM_ERR_CUDA, std::string("resident solver: ") + cudaGetErrorString(e));
        }
        long long rout = 0;
        unsigned st = 0;
        std::memcpy(&rout, h_ctl_, sizeof(long long));
        std::memcpy(&st, h_ctl_ + 1, sizeof(unsigned));
        if (st & (kErrBarrierTimeout | kErrRoundCap)) {
            broken_ = true;
            throw Error(HFM_ERR_NOT_CONVERGED, st & kErrBarrierTimeout ? "resident solver: a grid barrier wait exceeded its limit"
                                                                      : "resident solver: round cap reached");
        }
        round_ = rout;
    }

    void collect(std::vector<int64_t> &done) override {
        if (active_.empty()) return;
        cudaStream_t s = current_stream();
        std::vector<unsigned> live(kMaxResident);
        HFM_CUDA(cudaMemcpyAsync(live.data(), live_.get() + (round_ % 3) * kMaxResident, kMaxResident * sizeof(unsigned),
                                 cudaMemcpyDeviceToHost, s));
        HFM_CUDA(cudaStreamSynchronize(s));
        for (auto it = active_.begin(); it != active_.end();) {
            Entry &E = it->second;
            if (E.round_in >= 0 && live[E.slot] != 0u) { ++it; continue; }
            E.rounds = E.round_in >= 0 ? round_ - E.round_in : 0;
            E.t_solved = std::chrono::steady_clock::now();
            done.push_back(E.ticket);
            collected_.emplace(E.ticket, std::move(E));
            it = active_.erase(it);
        }
    }

    void finish(int64_t ticket, EulerResult &res, cudaStream_t s) override {
        auto it = collected_.find(ticket);
        if (it == collected_.end()) throw Error(HFM_ERR_ARG, "resident solver: unknown instance");
        const Entry E = std::move(it->second);
        collected_.erase(it);
        auto release = [&] {
            tiles_.release(E.tile0, E.nt);
            if (SHARE) classes_.release(E.cls0, E.ncls);
            entries_.release(E.e0, E.ne);
            free_slots_.push_back(E.slot);
        };
        try {
            const long long n = E.g.ncells;
            const Real *src = values_.get() + E.tile0 * 64;
            double *dst = E.h_out;
            if (!dst) {
                res.values.resize(n);
                dst = res.values.data();
            }
            if (std::is_same<Real, double>::value) {
                if (n * sizeof(double) >= kStagedMin) staged_download(dst, src, n * sizeof(double), s);
                else HFM_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, s));
                HFM_CUDA(cudaStreamSynchronize(s));
            } else {
                std::vector<Real> tmp(n);
                if (n * sizeof(Real) >= kStagedMin) staged_download(tmp.data(), src, n * sizeof(Real), s);
                else HFM_CUDA(cudaMemcpyAsync(tmp.data(), src, n * sizeof(Real), cudaMemcpyDeviceToHost, s));
                HFM_CUDA(cudaStreamSynchronize(s));
                for (long long x = 0; x < n; ++x) dst[x] = (double)tmp[x];
            }
            long long reached = 0;
            for (long long x = 0; x < n; ++x) reached += dst[x] < Arith<double>::inf() ? 1 : 0;
            res.n_accepted = reached;
            res.max_stencil_width = E.max_width;
            res.t_stencil_ms = E.setup_ms;
            res.t_solve_ms = std::chrono::duration<double, std::milli>(E.t_solved - E.t_admit).count();
            res.rounds = E.rounds;
            res.t_total_ms = res.t_solve_ms;
        } catch (...) {
            release();
            throw;
        }
        release();
    }

    // Drops every instance (after a failure of the solver): their tickets are returned.
    void abandon(std::vector<int64_t> &tickets) override {
        auto drop = [&](const Entry &E) {
            tickets.push_back(E.ticket);
            tiles_.release(E.tile0, E.nt);
            if (SHARE) classes_.release(E.cls0, E.ncls);
            entries_.release(E.e0, E.ne);
            free_slots_.push_back(E.slot);
        };
        for (const auto &kv : pending_) drop(kv.second);
        for (const auto &kv : active_) drop(kv.second);
        for (const auto &kv : collected_) drop(kv.second);
        pending_.clear();
        active_.clear();
        collected_.clear();
    }

    ~Resident() override {
        if (in_slice_) {
            cudaEventSynchronize(done_ev_);
            in_slice_ = false;
            coop_.unlock();
        }
        if (done_ev_) cudaEventDestroy(done_ev_);  // h_ctl_ stays in the process's pool
    }
};

template <typename Real, int NFWD, int NSYM, int KIND>
std::unique_ptr<ResidentFamily> make_resident_impl(const EulerProblem &p) {
    return std::unique_ptr<ResidentFamily>(new Resident<Real, NFWD, NSYM, KIND>(p));
}
