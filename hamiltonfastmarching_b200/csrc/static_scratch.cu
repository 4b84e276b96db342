// hfm_solve_riemann2_static_scratch: a Riemann2 FP64 solve that allocates no memory.
//
// Some callers cannot let a library allocate device memory: hosts whose allocator reserves the
// whole device up front (a framework's caching pool, or a fixed per-process memory budget) and
// leaves no room for cudaMalloc; latency-critical loops where cudaMalloc/cudaFree would
// synchronise the device and stall other streams; plugin hosts that forbid a library from changing
// its device footprint after start-up. For them this entry point keeps every intermediate array in
// one file-scope __device__ buffer of fixed size, created when the library is loaded and held by
// every GPU that loads it until the process exits. The caller passes the metric and receives the
// arrival times in its own device buffers.
//
// Limits: at most kMaxCells = 512*512 grid cells and kMaxSeeds = 1024 seeds (larger problems are
// rejected with HFM_ERR_VALUE); scratch size 9,453,824 bytes per device.
//
// The first call on a device looks up the device address of the buffer (cudaGetSymbolAddress)
// with that device current. Every call reads the convergence words back to the host and waits for
// its stream, so the entry point cannot be called inside a stream capture. All calls share the
// one buffer and it keeps the last call's contents: the arrays a call reads are fully rewritten by
// that call and the control words are cleared before use, but calls that overlap on the GPU
// (other threads, other streams) race on the buffer and must be serialised by the caller.
//
// Method: the same Selling stencils (selling.cuh) and the same Hopf-Lax update as the main path,
// iterated as chaotic Gauss-Seidel sweeps over all cells until no value changes; it reaches the
// same fixed point as the tiled solver (within 1e-10 relative). Repeated seeds keep their first
// value, as the main path does. Rounding can make a recomputed value land an ulp above the current
// one and such increases can cycle: once the sweeps have taken 2 increases per cell (plus 128),
// only decreases are taken, which terminates (the tiled solver's guard, per call instead of per
// tile). It calls no cudaMalloc, cudaFree or allocating routine.
#include <cstring>
#include <mutex>

#include "device_buffer.hpp"
#include "selling.cuh"

namespace hfm {
namespace static_scratch {

constexpr long long kMaxCells = 512LL * 512LL;
constexpr int kMaxSeeds = 1024;
constexpr size_t kCtrlBytes = 256;
constexpr size_t kSeedIdxOff = kCtrlBytes;
constexpr size_t kSeedValOff = kSeedIdxOff + kMaxSeeds * sizeof(long long);
constexpr size_t kCodeOff = kSeedValOff + kMaxSeeds * sizeof(double);
constexpr size_t kWeightOff = kCodeOff + 3 * kMaxCells * sizeof(unsigned);
constexpr size_t kScratchBytes = kWeightOff + 3 * kMaxCells * sizeof(double);
static_assert(kCodeOff % 256 == 0 && kWeightOff % 256 == 0, "scratch regions stay 256-byte aligned");

constexpr unsigned kPlus = 1u << 24, kMinus = 1u << 25, kFixed = 1u << 28;
constexpr unsigned kErrSellingBit = 8u;
constexpr int kSweepsPerCheck = 8;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct View {
    unsigned *changed;     // control word 0
    unsigned *status;      // control word 1
    unsigned *increases;   // control word 2: value increases taken since the start of the call
    const long long *seed_idx;
    const double *seed_val;
    unsigned *code;        // [3][N]
    double *weight;        // [3][N]
};

__host__ __device__ inline View view_of(unsigned char *base) {
    View v;
    v.changed = reinterpret_cast<unsigned *>(base);
    v.status = reinterpret_cast<unsigned *>(base) + 1;
    v.increases = reinterpret_cast<unsigned *>(base) + 2;
    v.seed_idx = reinterpret_cast<const long long *>(base + kSeedIdxOff);
    v.seed_val = reinterpret_cast<const double *>(base + kSeedValOff);
    v.code = reinterpret_cast<unsigned *>(base + kCodeOff);
    v.weight = reinterpret_cast<double *>(base + kWeightOff);
    return v;
}

__global__ void stencil_kernel(int nx, int ny, double h, const double *metric, int dual, unsigned char *base,
                               double *values) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long N = (long long)nx * ny;
    if (x >= N) return;
    const View V = view_of(base);
    const int i = (int)(x / ny), j = (int)(x % ny);
    double m[3] = {metric[3 * x], metric[3 * x + 1], metric[3 * x + 2]};
    const double hh[3] = {h, h, h};
    int off[6][3];
    double w[6];
    if (!riemann_stencil<2>(m, dual != 0, hh, off, w)) {
        atomicOr(V.status, kErrSellingBit);
        for (int k = 0; k < 3; ++k) { w[k] = 0.0; off[k][0] = off[k][1] = 0; }
    }
    for (int k = 0; k < 3; ++k) {
        unsigned c = (unsigned)(uint8_t)(int8_t)off[k][0] | ((unsigned)(uint8_t)(int8_t)off[k][1] << 8);
        if (w[k] != 0.0) {
            const int ip = i + off[k][0], jp = j + off[k][1], im = i - off[k][0], jm = j - off[k][1];
            if (ip >= 0 && ip < nx && jp >= 0 && jp < ny) c |= kPlus;
            if (im >= 0 && im < nx && jm >= 0 && jm < ny) c |= kMinus;
        }
        V.code[k * N + x] = c;
        V.weight[k * N + x] = w[k];
    }
    values[x] = Arith<double>::inf();
}

__global__ void seed_kernel(int n, long long N, unsigned char *base, double *values) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const View V = view_of(base);
    const long long x = V.seed_idx[s];
    values[x] = V.seed_val[s];
    V.code[x] |= kFixed;
}

// Hopf-Lax update over the 3 symmetric differences: candidates in increasing order, stop at the
// first one not below the running root, fast-marching accumulation order (EulerianStencil.hxx:30-72).
__device__ __forceinline__ double local_solve(const double (&v)[3], const double (&w)[3]) {
    using A = Arith<double>;
    unsigned taken = 0;
    double minVal = 0, a = 0, b = 0, c = -1, r = A::inf();
    for (int it = 0; it < 3; ++it) {
        double bv = A::inf(), bw = 0;
        int bk = -1;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (!((taken >> k) & 1u) && v[k] < bv) { bv = v[k]; bw = w[k]; bk = k; }
        if (bk < 0) break;
        if (it > 0 && !(bv < r)) break;
        if (it == 0) minVal = bv;
        const double dv = A::sub(bv, minVal), wv = A::mul(bw, dv);
        a = A::add(a, bw);
        b = A::add(b, wv);
        c = A::add(c, A::mul(wv, dv));
        if (a == 0.0) {
            r = A::inf();
        } else {
            const double d2 = A::sub(A::mul(b, b), A::mul(a, c));
            r = A::add(minVal, A::div(A::add(b, A::sqrt(0.0 < d2 ? d2 : 0.0)), a));
        }
        taken |= 1u << bk;
    }
    return r;
}

__global__ void sweep_kernel(int nx, int ny, int parity, int strict, unsigned char *base, double *values) {
    const long long N = (long long)nx * ny;
    const View V = view_of(base);
    bool changed = false;
    unsigned ups = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const long long x = (parity & 1) ? N - 1 - t : t;  // alternate the sweep direction
        const unsigned c0 = V.code[x];
        if (c0 & kFixed) continue;
        const int i = (int)(x / ny), j = (int)(x % ny);
        double v[3], w[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned c = V.code[k * N + x];
            const int o0 = (int)(int8_t)(c & 0xffu), o1 = (int)(int8_t)((c >> 8) & 0xffu);
            double val = Arith<double>::inf();
            if (c & kPlus) val = __ldcg(values + (long long)(i + o0) * ny + (j + o1));
            if (c & kMinus) {
                const double vv = __ldcg(values + (long long)(i - o0) * ny + (j - o1));
                if (vv < val) val = vv;
            }
            v[k] = val;
            w[k] = V.weight[k * N + x];
        }
        const double nv = local_solve(v, w);
        const double cur = __ldcg(values + x);
        if (strict ? nv < cur : nv != cur) {
            ups += nv > cur ? 1u : 0u;
            __stcg(values + x, nv);
            changed = true;
        }
    }
    if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) atomicOr(V.changed, 1u);
#pragma unroll
    for (int o = 16; o; o >>= 1) ups += __shfl_xor_sync(0xffffffffu, ups, o);
    if (ups && (threadIdx.x & 31) == 0) atomicAdd(V.increases, ups);
}

// Device address of the scratch buffer, looked up once per device with that device current.
unsigned char *scratch_address() {
    static std::mutex mu;
    static unsigned char *addr[64] = {nullptr};
    int dev = 0;
    HFM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(HFM_ERR_CUDA, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) throw Error(HFM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        addr[dev] = static_cast<unsigned char *>(p);
    }
    return addr[dev];
}

}  // namespace static_scratch
}  // namespace hfm

extern "C" int hfm_solve_riemann2_static_scratch(int64_t nx, int64_t ny, double grid_scale, const double *metric,
                                                 int dual, int64_t nseeds, const int64_t *seed_index,
                                                 const double *seed_value, double *values, void *stream,
                                                 char *err, size_t errcap) {
    using namespace hfm::static_scratch;
    auto fail = [&](int code, const std::string &m) {
        if (err && errcap) {
            std::strncpy(err, m.c_str(), errcap - 1);
            err[errcap - 1] = 0;
        }
        return code;
    };
    if (!metric || !values || !seed_index || !seed_value) return fail(HFM_ERR_ARG, "null argument");
    if (nx <= 0 || ny <= 0 || !(grid_scale > 0)) return fail(HFM_ERR_VALUE, "invalid grid");
    // each side first, so that the product below cannot overflow
    if (nx > kMaxCells || ny > kMaxCells || nx * ny > kMaxCells)
        return fail(HFM_ERR_VALUE, "grid of " + std::to_string(nx) + " x " + std::to_string(ny) + " cells exceeds the " +
                                       std::to_string(kMaxCells) + "-cell limit of the static-scratch entry point");
    if (nseeds < 1 || nseeds > kMaxSeeds)
        return fail(HFM_ERR_VALUE, "between 1 and " + std::to_string(kMaxSeeds) + " seeds are required");
    const long long N = nx * ny;
    for (int64_t s = 0; s < nseeds; ++s)
        if (seed_index[s] < 0 || seed_index[s] >= N) return fail(HFM_ERR_VALUE, "seed index out of range");
    // Repeated seed indices keep their first value (the main path's std::map semantics): a stable
    // insertion sort by index into fixed arrays, then the first entry of each run.
    long long sidx[kMaxSeeds];
    double sval[kMaxSeeds];
    int ns = 0;
    for (int64_t s = 0; s < nseeds; ++s) {
        const long long x = seed_index[s];
        int pos = ns;
        while (pos > 0 && sidx[pos - 1] > x) --pos;
        if (pos > 0 && sidx[pos - 1] == x) continue;  // an earlier seed holds this cell
        for (int k = ns; k > pos; --k) { sidx[k] = sidx[k - 1]; sval[k] = sval[k - 1]; }
        sidx[pos] = x;
        sval[pos] = seed_value[s];
        ++ns;
    }
    try {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        unsigned char *base = scratch_address();
        HFM_CUDA(cudaMemsetAsync(base, 0, kCtrlBytes, st));
        // pageable sources: each copy returns once the bytes are staged, so the arrays may go
        HFM_CUDA(cudaMemcpyAsync(base + kSeedIdxOff, sidx, ns * sizeof(long long), cudaMemcpyHostToDevice, st));
        HFM_CUDA(cudaMemcpyAsync(base + kSeedValOff, sval, ns * sizeof(double), cudaMemcpyHostToDevice, st));
        const unsigned blocks = (unsigned)((N + 255) / 256);
        hfm::launch(stencil_kernel, blocks, 256, 0, st, (int)nx, (int)ny, grid_scale, metric, dual, base, values);
        hfm::launch(seed_kernel, (unsigned)((ns + 127) / 128), 128, 0, st, ns, N, base, values);
        HFM_CUDA(cudaGetLastError());
        unsigned ctrl[3] = {0, 0, 0};
        const long long max_sweeps = 64 * (nx + ny) + 4096;
        const unsigned long long up_budget = 2ull * (unsigned long long)N + 128ull;
        bool converged = false, strict = false;
        for (long long sweep = 0; sweep < max_sweeps && !converged; sweep += kSweepsPerCheck) {
            HFM_CUDA(cudaMemsetAsync(base, 0, sizeof(unsigned), st));
            for (int k = 0; k < kSweepsPerCheck; ++k)
                hfm::launch(sweep_kernel, blocks < 1184u ? blocks : 1184u, 256, 0, st, (int)nx, (int)ny,
                            (int)(sweep + k), strict ? 1 : 0, base, values);
            HFM_CUDA(cudaMemcpyAsync(ctrl, base, sizeof(ctrl), cudaMemcpyDeviceToHost, st));
            HFM_CUDA(cudaStreamSynchronize(st));
            if (ctrl[1] & kErrSellingBit)
                return fail(HFM_ERR_VALUE, "ObtuseSuperbase error : input must be positive definite");
            converged = ctrl[0] == 0;
            strict = strict || ctrl[2] >= up_budget;
        }
        if (!converged) return fail(HFM_ERR_NOT_CONVERGED, "sweep cap reached before convergence");
        return HFM_OK;
    } catch (const hfm::Error &e) {
        return fail(e.code, e.what());
    }
}
