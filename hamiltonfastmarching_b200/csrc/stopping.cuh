// Stopping criteria on the device (stopAtDistance, nMaxAccepted, stopWhenAnyAccepted,
// stopWhenAllAccepted and their _Unoriented forms).
//
// Included by eulerian.cu inside namespace hfm::detail, after the solver kernels.
//
// The reference's fast marching stops at the first cell it pops that meets a criterion; that cell
// is counted in nAccepted but not accepted, and every cell not accepted keeps its tentative value
// (Headers/ExtraAlgorithms/CommonStoppingCriteria.h:58-93, HamiltonFastMarching.hxx:86-112). The
// accepted cells' values do not depend on later cells, so here the solve runs to the end and the
// stop is applied afterwards: cells are ordered by (value, index) as fast marching pops them; the
// stopping cell is the first in that order that meets a criterion (the M-th for nMaxAccepted, the
// first beyond the distance, the first or last target); the cells before it are the accepted ones;
// the others are solved once more from their accepted neighbours only (unreached if they have
// none). Fast marching pops cells of exactly equal values in its heap's order, which the (value,
// index) order follows only where values differ.

// Order-preserving 64-bit key of a double (negative values included).
__device__ __host__ __forceinline__ unsigned long long stop_key(double v) {
#ifdef __CUDA_ARCH__
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
#else
    unsigned long long b;
    std::memcpy(&b, &v, sizeof(b));
#endif
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Cells with a finite value and (key, index) <= (kkey, kidx) (kidx < 0: key < kkey only; kidx >= N:
// key <= kkey).
template <typename Real>
__global__ void stop_count_kernel(long long N, const Real *values, unsigned long long kkey, long long kidx,
                                  unsigned long long *out) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool in = false;
    if (x < N) {
        const double u = (double)values[x];
        if (u < Arith<double>::inf()) {
            const unsigned long long k = stop_key(u);
            in = k < kkey || (k == kkey && x <= kidx);
        }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    if ((threadIdx.x & 31) == 0 && bal) atomicAdd(out, (unsigned long long)__popc(bal));
}

// Smallest key (then index) among the finite cells with a value above d.
template <typename Real>
__global__ void stop_beyond_kernel(long long N, const Real *values, double d, unsigned long long *kmin) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double u = (double)values[x];
    if (u < Arith<double>::inf() && u > d) atomicMin(kmin, stop_key(u));
}
template <typename Real>
__global__ void stop_beyond_index_kernel(long long N, const Real *values, unsigned long long kkey,
                                         unsigned long long *imin) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double u = (double)values[x];
    if (u < Arith<double>::inf() && stop_key(u) == kkey) atomicMin(imin, (unsigned long long)x);
}

// Accepted cells (before the stopping cell) keep their value in vmask; the others read +inf there.
template <typename Real>
__global__ void stop_mask_kernel(long long N, const Real *values, unsigned long long kkey, long long kidx,
                                 uint8_t *acc, Real *vmask) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double u = (double)values[x];
    bool a = false;
    if (u < Arith<double>::inf()) {
        const unsigned long long k = stop_key(u);
        a = k < kkey || (k == kkey && x < kidx);
    }
    acc[x] = a;
    vmask[x] = a ? values[x] : Arith<Real>::inf();
}

// Tentative values of the cells not accepted: one local solve from the accepted neighbours
// (PM reads vmask); seeds keep their value, walls stay unreached.
template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void stop_tentative_kernel(Dev<Real> PM, const uint8_t *acc, Real *values) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= PM.ncells || acc[x]) return;
    const CellRef R = cell_ref(PM.inst, PM.ninst, x);
    const Inst &I = PM.inst[R.i];
    bool fixed, dead;
    cell_flags<Real, KIND>(PM, R.c, fixed, dead);
    if (fixed) return;
    if (dead) { values[x] = Arith<Real>::inf(); return; }
    values[x] = solve_cell<Real, NFWD, NSYM, KIND>(PM, I, R.c, R.x0, R.x1, R.x2, 0, 0, 0, nullptr, nullptr, nullptr);
}

__global__ void stop_select_kernel(long long N, const uint8_t *acc, const unsigned long long *masked,
                                   unsigned long long *active) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < N && !acc[x]) active[x] = masked[x];
}

// State of a stopped solve: the accepted mask and the masked values, for the activeNeighs of the
// cells not accepted.
template <typename Real>
struct Stopped {
    bool on = false;
    long long count = 0;  // nAccepted: accepted cells, plus the stopping cell
    DeviceBuffer<uint8_t> acc;
    DeviceBuffer<Real> vmask;
};

// Applies the stopping criteria of a single instance to the solved values (in place).
template <typename Real, int NFWD, int NSYM, int KIND>
void apply_stopping(const Dev<Real> &P, long long N, const EulerProblem &p, Real *values, Stopped<Real> &st,
                    cudaStream_t s) {
    DeviceBuffer<unsigned long long> cnt(2);
    auto count = [&](unsigned long long kkey, long long kidx) {
        cnt.zero(s);
        launch(stop_count_kernel<Real>, nblocks(N, 256), 256, 0, s, N, (const Real *)values, kkey, kidx, cnt.get());
        unsigned long long h = 0;
        cnt.download(&h, 1, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        return h;
    };
    const unsigned long long reached = count(~0ull, N);
    auto value_at = [&](long long x) {
        Real v;
        HFM_CUDA(cudaMemcpyAsync(&v, values + x, sizeof(Real), cudaMemcpyDeviceToHost, s));
        HFM_CUDA(cudaStreamSynchronize(s));
        return (double)v;
    };
    // stopping cell: the smallest (key, index) among the criteria; none: every reached cell
    bool stop = false;
    unsigned long long bkey = ~0ull;
    long long bidx = N;
    auto offer = [&](unsigned long long k, long long i) {
        if (!stop || k < bkey || (k == bkey && i < bidx)) { bkey = k; bidx = i; }
        stop = true;
    };
    if (p.stop_n_max > 0 && (unsigned long long)p.stop_n_max <= reached) {
        // the M-th cell: smallest key with at least M cells at or below it, then the index
        const unsigned long long M = (unsigned long long)p.stop_n_max;
        unsigned long long lo = 0, hi = ~0ull;
        while (lo < hi) {
            const unsigned long long mid = lo + (hi - lo) / 2;
            if (count(mid, N) >= M) hi = mid;
            else lo = mid + 1;
        }
        const unsigned long long below = count(lo, -1);
        long long ilo = 0, ihi = N - 1;
        while (ilo < ihi) {
            const long long mid = ilo + (ihi - ilo) / 2;
            if (count(lo, mid) - below >= M - below) ihi = mid;
            else ilo = mid + 1;
        }
        offer(lo, ilo);
    }
    for (long long t : p.stop_any) {
        const double v = value_at(t);
        if (v < Arith<double>::inf()) offer(stop_key(v), t);
    }
    if (!p.stop_all.empty()) {
        bool all = true;
        unsigned long long k = 0;
        long long i = -1;
        for (long long t : p.stop_all) {
            const double v = value_at(t);
            if (!(v < Arith<double>::inf())) { all = false; break; }
            const unsigned long long kt = stop_key(v);
            if (kt > k || (kt == k && t > i)) { k = kt; i = t; }
        }
        if (all) offer(k, i);
    }
    const long long nth = p.dims[2] > 0 ? p.dims[2] : 1;
    auto first_of_column = [&](long long xy, unsigned long long &k, long long &i) {
        bool any = false;
        for (long long th = 0; th < nth; ++th) {
            const long long x = xy * nth + th;
            const double v = value_at(x);
            if (!(v < Arith<double>::inf())) continue;
            const unsigned long long kt = stop_key(v);
            if (!any || kt < k || (kt == k && x < i)) { k = kt; i = x; }
            any = true;
        }
        return any;
    };
    for (long long xy : p.stop_any_u) {
        unsigned long long k;
        long long i;
        if (first_of_column(xy, k, i)) offer(k, i);
    }
    if (!p.stop_all_u.empty()) {
        bool all = true;
        unsigned long long k = 0;
        long long i = -1;
        for (long long xy : p.stop_all_u) {
            unsigned long long kt;
            long long it;
            if (!first_of_column(xy, kt, it)) { all = false; break; }
            if (kt > k || (kt == k && it > i)) { k = kt; i = it; }
        }
        if (all) offer(k, i);
    }
    if (p.has_stop_distance) {
        DeviceBuffer<unsigned long long> km(2);
        const unsigned long long init[2] = {~0ull, ~0ull};
        km.upload(init, 2, s);
        launch(stop_beyond_kernel<Real>, nblocks(N, 256), 256, 0, s, N, (const Real *)values, p.stop_distance, km.get());
        unsigned long long hk = 0;
        km.download(&hk, 1, s);
        HFM_CUDA(cudaStreamSynchronize(s));
        if (hk != ~0ull) {
            launch(stop_beyond_index_kernel<Real>, nblocks(N, 256), 256, 0, s, N, (const Real *)values, hk,
                   km.get() + 1);
            unsigned long long two[2];
            km.download(two, 2, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            offer(hk, (long long)two[1]);
        }
    }
    st.on = true;
    if (!stop) {
        st.count = (long long)reached;
        st.on = false;  // nothing to mask: every reached cell is accepted
        return;
    }
    st.count = (long long)count(bkey, bidx - 1) + 1;
    st.acc.alloc(N);
    st.vmask.alloc(N);
    launch(stop_mask_kernel<Real>, nblocks(N, 256), 256, 0, s, N, (const Real *)values, bkey, bidx, st.acc.get(),
           st.vmask.get());
    Dev<Real> PM = P;
    PM.values = st.vmask.get();
    launch(stop_tentative_kernel<Real, NFWD, NSYM, KIND>, nblocks(N, 128), 128, 0, s, PM,
           (const uint8_t *)st.acc.get(), values);
    HFM_CUDA(cudaGetLastError());
    HFM_CUDA(cudaStreamSynchronize(s));
}
