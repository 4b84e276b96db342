// Per-thread stream selection, memory-pool policy and launch accounting of the library, plus the
// device-resident entry point of the C ABI.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

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

static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace hfm

namespace {

struct StreamScope {
    cudaStream_t saved;
    explicit StreamScope(cudaStream_t s) : saved(hfm::current_stream()) { hfm::current_stream() = s; }
    ~StreamScope() { hfm::current_stream() = saved; }
};

}  // namespace

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
