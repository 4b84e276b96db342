// Geodesic backtracking and the geodesic flow on the device.
//
// Included by eulerian.cu inside namespace hfm::detail, after the solver kernels (it uses Dev,
// Inst, solve_cell, cell_flags and the TTI path helpers).
//
// The reference extracts geodesics one tip at a time on the host with a std::map keyed by
// (value, index) (Headers/Base/Implementation/GeodesicDiscreteSolver.hxx:59-211). Tips are
// independent, so here one warp follows one tip: the pending (value, index, weight) entries of
// its tip live in the warp's shared memory, the largest one is found with a warp reduction, the
// Recompute of the extracted cell is done on the device from the arrival times still resident in
// HBM, and children are matched against the entries with a warp ballot. Running sums and the step
// bookkeeping are warp-uniform; the arithmetic keeps the reference's order and rounds every
// product and sum on its own (no contraction), so a geodesic follows the reference's to rounding.
// Warps loop over the tips of all instances of a batch (persistent grid).

constexpr int kGeoMaxFlow = 32;      // flow entries of one Recompute (two per difference, capped)
constexpr int kGeoWarps = 4;         // warps per CTA of the geodesic kernel
constexpr int kGeoCap = 256, kGeoStepCap = 64;          // shared-memory set / step list
constexpr int kGeoCapBig = 8192, kGeoStepCapBig = 512;  // global-memory rerun of overflowed tips
constexpr long long kGeoIndexBias = 1ll << 20;          // unwrapped indices packed as 3 x 21 bits

// Per-tip status bits.
enum : int {
    kGeoFailed = 1,         // the restart limit was reached (the reference's "extraction failed")
    kGeoPointOverflow = 2,  // more points than the tip's output capacity (rerun with more room)
    kGeoSetOverflow = 4,    // more pending entries than the warp's set holds (rerun in global memory)
    kGeoIterCap = 8,        // iteration limit of one pass reached
    kGeoRange = 16,         // an unwrapped index left the packable range
};

struct GeoTip {
    double p[3];        // dimensionless tip (cell i spans [i, i+1)); unoriented: (x, y) only
    double step, thr, vbound;  // geodesicStep, geodesicWeightThreshold, geodesicVolumeBound
    double causality;   // geodesicCausalityTolerance (ODE solver)
    long long out0;     // first point slot of this tip in the output
    int inst;           // instance of the batch
    int cap;            // output capacity in points
    int ndim;           // model dimension (2 or 3)
    int unoriented;     // choose the angle of smallest value (tips_Unoriented)
    int ode;            // geodesicSolver 'ODE' instead of 'Discrete'
    int nstat_max;      // ODE: stationarity limit, int(6 sqrt(D) / step)
    int nhist;          // ODE: length of the target-distance history, ceil(sqrt(D) / step)
    int table_log2;     // ODE: log2 of the per-tip visit-count table
};

struct GeoOut {
    int len;            // points written
    int status;         // kGeo* bits
    int restarts;       // restarts of the discrete solver
    int pad;
};

template <int CAP, int SCAP>
struct GeoSet {
    double val[CAP];
    double w[CAP];
    long long key[CAP];
    double sv[SCAP];        // step list: value of the extracted entry and the step of the mean
    double sd[SCAP][3];
    unsigned foff[kGeoMaxFlow];  // flow of the extracted cell
    double fw[kGeoMaxFlow];
    long long ckey[kGeoMaxFlow]; // its children: packed unwrapped index, pending slot or -1
    int cfound[kGeoMaxFlow];
};

__device__ __forceinline__ long long geo_pack(const int *ind) {
    return ((ind[0] + kGeoIndexBias) << 42) | ((ind[1] + kGeoIndexBias) << 21) | (ind[2] + kGeoIndexBias);
}
__device__ __forceinline__ void geo_unpack(long long k, int *ind) {
    const long long m = (1ll << 21) - 1;
    ind[0] = (int)(((k >> 42) & m) - kGeoIndexBias);
    ind[1] = (int)(((k >> 21) & m) - kGeoIndexBias);
    ind[2] = (int)((k & m) - kGeoIndexBias);
}
__device__ __forceinline__ bool geo_packable(const int *ind) {
    return ind[0] > -kGeoIndexBias && ind[0] < kGeoIndexBias && ind[1] > -kGeoIndexBias &&
           ind[1] < kGeoIndexBias && ind[2] > -kGeoIndexBias && ind[2] < kGeoIndexBias;
}

// Order-1 Recompute at cell (x0, x1, x2) of instance I (HamiltonFastMarching.hxx:187-272): the
// flow entries (packed offset, weight) in the reference's order, the recomputed value and the
// width. Stencils: the active differences (forward ones, then the +e / -e side of each symmetric
// one, as the activeNeighs bits), the quadratic update over them, weights w_i max(0, value - u_i)
// (EulerianStencil.hxx:157-229). TTI3: the Selling path at the extremum t, weights
// (sol - v) w(t) (TTI.hpp:278-389). Seeds, walls and unreached cells have no flow.
template <typename Real, int NFWD, int NSYM, int KIND>
__device__ int recompute_flow(const Dev<Real> &P, const Inst &I, int x0, int x1, int x2, unsigned *foff, double *fw,
                              double *value, double *width) {
    [[maybe_unused]] constexpr bool SHARE = is_share(KIND);
    constexpr int ND = NFWD + NSYM;
    using A = Arith<double>;
    const GridGeom &g = I.g;
    const long long c = (I.tile0 + g.tile_of(x0, x1, x2)) * 64 + g.local_of(x0, x1, x2);
    const Real *values = P.values + I.cell0;
    const double u = (double)values[g.lin(x0, x1, x2)];
    *value = u;
    *width = 0.0;
    bool fixed, dead;
    cell_flags<Real, KIND>(P, c, fixed, dead);
    if (fixed || dead || !(u < A::inf())) return 0;
    if constexpr (KIND == kKindShareS2) return 0;  // ReedsShepp3 geodesics are refused by the host
    if constexpr (KIND == kKindTTI) {
        double ta = 0.0;
        bool inner = false;
        solve_cell_tti<Real>(P, I, c, x0, x1, x2, 0, 0, 0, nullptr, &ta, &inner);
        if (!(ta < A::inf())) return 0;
        const TTICell &tc = P.tti[c];
        TTIPath path;
        if (!tti_path_at(tc, ta, path)) return 0;
        struct Cand {
            double v, wa, wb;
            unsigned off;
        } cand[6];
        for (int r = 0; r < 6; ++r) {
            double vs[2] = {A::inf(), A::inf()};
            for (int si = 0; si < 2; ++si) {
                const int s = si ? -1 : 1;
                const int y0 = x0 + s * path.off[r][0], y1 = x1 + s * path.off[r][1], y2 = x2 + s * path.off[r][2];
                if ((unsigned)y0 >= (unsigned)g.dims[0] || (unsigned)y1 >= (unsigned)g.dims[1] ||
                    (unsigned)y2 >= (unsigned)g.dims[2])
                    continue;
                vs[si] = (double)values[g.lin(y0, y1, y2)];
            }
            const bool plus = vs[0] < vs[1];  // the +e neighbour only when strictly smaller
            const int s = plus ? 1 : -1;
            Cand cd{plus ? vs[0] : vs[1], path.w0[r], path.w1[r],
                    pack_off(s * path.off[r][0], s * path.off[r][1], s * path.off[r][2])};
            int k = r - 1;
            while (k >= 0 && cand[k].v > cd.v) {
                cand[k + 1] = cand[k];
                --k;
            }
            cand[k + 1] = cd;
        }
        const double vmin = cand[0].v;
        if (!(vmin < A::inf())) return 0;
        double a = 0, b = 0, cc = -tti_multiplier(tc, dconst(ta)).v, sol = A::inf();
        int r = 0;
        for (; r < 6; ++r) {
            const double v = A::sub(cand[r].v, vmin);
            if (v >= sol) break;
            const double w = A::add(A::mul(A::sub(1.0, ta), cand[r].wa), A::mul(ta, cand[r].wb));
            const double wv = A::mul(w, v);
            a = A::add(a, w);
            b = A::add(b, wv);
            cc = A::add(cc, A::mul(wv, v));
            if (a <= 100 * fabs(cc) * 2.220446049250313e-16) continue;
            sol = A::div(A::add(b, A::sqrt(A::sub(A::mul(b, b), A::mul(a, cc)))), a);
        }
        double wsum = 0.0, wid = 0.0;
        for (int q = 0; q < r; ++q) {
            const double v = A::sub(cand[q].v, vmin);
            const double w0 = A::add(A::mul(A::sub(1.0, ta), cand[q].wa), A::mul(ta, cand[q].wb));
            const double d = A::mul(A::sub(sol, v), w0);
            foff[q] = cand[q].off;
            fw[q] = d > 0 ? d : 0.0;
            wsum = A::add(wsum, w0);
            wid = A::add(wid, fw[q]);
        }
        *value = A::add(sol, vmin);
        *width = A::div(wid, wsum);  // TTI.hpp:372-388
        return r;
    } else {
        unsigned used = 0, side = 0;
        solve_cell<Real, NFWD, NSYM, KIND>(P, I, c, x0, x1, x2, 0, 0, 0, nullptr, &used, &side);
        double m = 1.0;
        if (SHARE) m = (double)P.mult[c];
        double nv[kGeoMaxFlow], wts[kGeoMaxFlow];
        int n = 0;
        for (int k = 0; k < ND; ++k) {
            int o0, o1, o2;
            double wb;
            if (SHARE) {
                const int8_t *o = P.cls_off + ((I.cls0 + x2) * ND + k) * 3;
                o0 = o[0]; o1 = o[1]; o2 = o[2];
                wb = A::mul((double)P.cls_w[(I.cls0 + x2) * ND + k], A::mul(m, m));
            } else {
                const unsigned cd = P.code[k * P.sstride + c];
                o0 = off_c(cd, 0); o1 = off_c(cd, 1); o2 = off_c(cd, 2);
                wb = (double)P.weight[k * P.sstride + c];
            }
            // active sides of this difference, as the activeNeighs bits (active_kernel)
            unsigned act = 0;  // bit0: +e, bit1: -e
            if (k < NFWD) {
                if ((used >> k) & 1u) act = 1;
                else if (SHARE) {
                    for (int k2 = 0; k2 < NFWD; ++k2) {
                        if (!((used >> k2) & 1u)) continue;
                        const int8_t *o2p = P.cls_off + ((I.cls0 + x2) * ND + k2) * 3;
                        if (o2p[0] == o0 && o2p[1] == o1 && o2p[2] == o2) { act = 1; break; }
                    }
                }
            } else if ((used >> k) & 1u) {
                act = ((side >> (k - NFWD)) & 1u) ? 2u : 1u;
            }
            // a two-group stencil recomputes with the named group only
            if (KIND == kKindShare2 && (k < ND / 2 ? 0u : 1u) != ((used >> ND) & 1u)) act = 0;
            for (int si = 0; si < 2; ++si) {
                if (!((act >> si) & 1u) || n >= kGeoMaxFlow) continue;
                const int s = si ? -1 : 1;
                int y0 = x0 + s * o0, y1 = x1 + s * o1, y2 = x2 + s * o2;
                if (!g.wrap(y0, y1, y2)) continue;  // active neighbours are inside; kept as a guard
                nv[n] = (double)values[g.lin(y0, y1, y2)];
                wts[n] = wb;
                foff[n] = pack_off(s * o0, s * o1, s * o2);
                ++n;
            }
        }
        if (n == 0) return 0;
        // QuadraticMax over the active neighbours in this order (minVal = their smallest value)
        double mn = A::inf();
        for (int i = 0; i < n; ++i) mn = nv[i] < mn ? nv[i] : mn;
        double a = 0, b = 0, cc = -1;
        for (int i = 0; i < n; ++i) {
            const double v = A::sub(nv[i], mn);
            const double wv = A::mul(wts[i], v);
            a = A::add(a, wts[i]);
            b = A::add(b, wv);
            cc = A::add(cc, A::mul(wv, v));
        }
        double val = A::inf();
        if (a != 0.0) {
            const double d2 = A::sub(A::mul(b, b), A::mul(a, cc));
            val = A::add(mn, A::div(A::add(b, A::sqrt(0.0 < d2 ? d2 : 0.0)), a));
        }
        double wid = 0.0, wsum = 0.0;
        for (int i = 0; i < n; ++i) {
            const double d = A::sub(val, nv[i]);
            fw[i] = A::mul(wts[i], 0.0 < d ? d : 0.0);
            wid = A::add(wid, fw[i]);
        }
        for (int i = 0; i < n; ++i) wsum = A::add(wsum, wts[i]);
        if (wsum > 0) wid = A::div(wid, wsum);
        *value = val;
        *width = wid;
        return n;
    }
}

// Geodesic flow of every cell of a batch: sum of weight * offset over the Recompute flow
// (HamiltonFastMarching.hxx:363-378), dimensionless, [cell][ndim] at cell0 * ndim of each instance
// (the export is -ReDim of it, HFMInterface.hxx:541-553).
template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void geodesic_flow_kernel(Dev<Real> P, int ndim, double *out) {
    using A = Arith<double>;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const int ii = inst_of_cell(P.inst, P.ninst, x);
    const Inst &I = P.inst[ii];
    const GridGeom &g = I.g;
    const long long l = x - I.cell0;
    const int x2 = (int)(l % g.dims[2]);
    const long long r = l / g.dims[2];
    const int x1 = (int)(r % g.dims[1]);
    const int x0 = (int)(r / g.dims[1]);
    unsigned foff[kGeoMaxFlow];
    double fw[kGeoMaxFlow], v, wd;
    const int nf = recompute_flow<Real, NFWD, NSYM, KIND>(P, I, x0, x1, x2, foff, fw, &v, &wd);
    for (int a = 0; a < ndim; ++a) {
        double s = 0.0;
        for (int f = 0; f < nf; ++f) s = A::add(s, A::mul(fw[f], (double)off_c(foff[f], a)));
        out[x * ndim + a] = s;
    }
}

// Recompute flow of every cell of a batch, computed once before the geodesic launch (the
// discrete solver reads it at every extraction): nf[x] entries, entry f at foff/fw[f * N + x].
struct GeoRec {
    long long N;
    const uint8_t *nf;
    const unsigned *foff;
    const double *fw;
};

template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void geo_rec_kernel(Dev<Real> P, int maxf, uint8_t *nf, unsigned *foff, double *fw) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef C = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[C.i];
    unsigned o[kGeoMaxFlow];
    double w[kGeoMaxFlow], v, wd;
    int n = recompute_flow<Real, NFWD, NSYM, KIND>(P, I, C.x0, C.x1, C.x2, o, w, &v, &wd);
    n = n < maxf ? n : maxf;
    nf[x] = (uint8_t)n;
    for (int f = 0; f < n; ++f) {
        foff[f * P.ncells + x] = o[f];
        fw[f * P.ncells + x] = w[f];
    }
}

// Unit mass split among the 2^D grid neighbours of the tip, the extraction loop and the emission of
// points (GeodesicDiscreteSolver.hxx:59-211). Warp-uniform except where lane 0 writes. Returns 1
// if the mass spread beyond the volume bound (restart from the last point), 0 otherwise.
template <typename Real, int CAP, int SCAP, int D>
__device__ int geodesic_pass(const Dev<Real> &P, const Inst &I, const GeoRec &R, GeoSet<CAP, SCAP> &S, double *out,
                             int cap, int &len, int &status, double step, double thr, double vbound,
                             long long iter_cap) {
    using A = Arith<double>;
    const int lane = threadIdx.x & 31;
    const GridGeom &g = I.g;
    const Real *values = P.values + I.cell0;
    int n = 0;
    double ws = 0.0, is[3] = {0, 0, 0}, cs[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto sums = [&](double w, const int *ind) {
        ws = A::add(ws, w);
        for (int i = 0; i < D; ++i) is[i] = A::add(is[i], A::mul(w, (double)ind[i]));
        for (int i = 0; i < D; ++i)
            for (int j = 0; j <= i; ++j) cs[i][j] = A::add(cs[i][j], A::mul(w, A::mul((double)ind[i], (double)ind[j])));
    };
    auto emit = [&](const double *pt) -> bool {
        if (len >= cap) {
            status |= kGeoPointOverflow;
            return false;
        }
        if (lane == 0)
            for (int a = 0; a < D; ++a) out[(long long)len * D + a] = pt[a];
        ++len;
        return true;
    };
    double tip[3] = {0, 0, 0};
    __syncwarp();
    for (int a = 0; a < D; ++a) tip[a] = out[(long long)(len - 1) * D + a];
    int ref[3] = {0, 0, 0};
    double pref[3] = {0, 0, 0};
    for (int a = 0; a < D; ++a) {
        ref[a] = (int)floor(tip[a]);
        pref[a] = A::add((double)ref[a], 0.5);
    }
    for (int i = 0; i < (1 << D); ++i) {
        double weight = 1.0;
        int ind[3] = {0, 0, 0};
        for (int j = 0; j < D; ++j) {
            const double diff = A::sub(tip[j], pref[j]);
            ind[j] = ref[j];
            if (i & (1 << j)) {
                ind[j] += diff > 0 ? 1 : -1;
                weight = A::mul(weight, fabs(diff));
            } else {
                weight = A::mul(weight, A::sub(1.0, fabs(diff)));
            }
        }
        int q0 = ind[0], q1 = ind[1], q2 = ind[2];
        if (!g.wrap(q0, q1, q2)) continue;
        if (!geo_packable(ind)) { status |= kGeoRange; return 0; }
        if (lane == 0) {
            S.val[n] = (double)values[g.lin(q0, q1, q2)];
            S.key[n] = geo_pack(ind);
            S.w[n] = weight;
        }
        ++n;
        sums(weight, ind);
    }
    __syncwarp();
    if (ws == 0) return 0;
    double avg[3] = {0, 0, 0}, base[3] = {0, 0, 0};
    // a vector divided by a scalar is multiplied by the reciprocal, as in the reference's vector
    // types (FriendOperators.h:35, VectorType.h:37-41)
    {
        const double iw = A::div(1.0, ws);
        for (int a = 0; a < D; ++a) { avg[a] = A::mul(is[a], iw); base[a] = avg[a]; }
    }
    double stepNorm = 0.0;
    int nst = 0;
    double f0[3] = {0, 0, 0}, f1[3] = {0, 0, 0};  // steps beyond the list: sum of s and of s * value
    long long iters = 0;
    while (n > 0 && ws > 1e-5) {
        if (++iters > iter_cap) { status |= kGeoIterCap; return 0; }
        // entry of largest (value, index): lanes scan their slots, then a butterfly reduction
        double bv = -A::inf();
        long long bk = 0;
        int bs = -1;
        for (int j = lane; j < n; j += 32) {
            const double v = S.val[j];
            const long long k = S.key[j];
            if (bs < 0 || v > bv || (v == bv && k > bk)) { bv = v; bk = k; bs = j; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const long long ok = __shfl_xor_sync(0xffffffffu, bk, o);
            const int os = __shfl_xor_sync(0xffffffffu, bs, o);
            if (os >= 0 && (bs < 0 || ov > bv || (ov == bv && ok > bk))) { bv = ov; bk = ok; bs = os; }
        }
        const double ew = S.w[bs];
        __syncwarp();
        if (lane == 0) {
            S.val[bs] = S.val[n - 1];
            S.key[bs] = S.key[n - 1];
            S.w[bs] = S.w[n - 1];
        }
        --n;
        __syncwarp();
        if (ew == 0) continue;
        int ind[3];
        geo_unpack(bk, ind);
        sums(-ew, ind);
        int q0 = ind[0], q1 = ind[1], q2 = ind[2];
        // the extracted cell's flow, from the records computed for every cell before the launch
        // (entries are cells of the grid: a failed wrap is reported, not read)
        if (!g.wrap(q0, q1, q2)) { status |= kGeoRange; return 0; }
        const long long gx = I.cell0 + g.lin(q0, q1, q2);
        const int nf = R.nf[gx] < kGeoMaxFlow ? R.nf[gx] : kGeoMaxFlow;
        if (lane < nf) {
            S.foff[lane] = R.foff[lane * R.N + gx];
            S.fw[lane] = R.fw[lane * R.N + gx];
        }
        __syncwarp();
        double wSum = 0.0;
        for (int f = 0; f < nf; ++f) wSum = A::add(wSum, S.fw[f]);
        if (wSum == 0) continue;
        // children: lane f computes the index, key and value of child f (their loads overlap), one
        // pass over the pending entries finds those already there; they are then added in flow
        // order, as the reference does (the insertion threshold depends on the running sum)
        long long ckey = 0;
        double cval = 0.0;
        bool cok = true;
        if (lane < nf) {
            const unsigned oc = S.foff[lane];
            int c[3] = {ind[0] + off_c(oc, 0), ind[1] + off_c(oc, 1), ind[2] + off_c(oc, 2)};
            cok = geo_packable(c);
            if (cok) {
                ckey = geo_pack(c);
                cok = g.wrap(c[0], c[1], c[2]);  // flow neighbours are inside; kept as a guard
                if (cok) cval = (double)values[g.lin(c[0], c[1], c[2])];
            }
            S.ckey[lane] = ckey;
            S.cfound[lane] = -1;
        }
        if (__any_sync(0xffffffffu, !cok)) { status |= kGeoRange; return 0; }
        __syncwarp();
        for (int j = lane; j < n; j += 32) {
            const long long k = S.key[j];
            for (int f = 0; f < nf; ++f)
                if (S.ckey[f] == k) S.cfound[f] = j;
        }
        __syncwarp();
        for (int f = 0; f < nf; ++f) {
            const double w = A::div(A::mul(ew, S.fw[f]), wSum);
            const long long key = __shfl_sync(0xffffffffu, ckey, f);
            const double val = __shfl_sync(0xffffffffu, cval, f);
            const int found = S.cfound[f];
            __syncwarp();
            if (found >= 0) {
                if (lane == 0) S.w[found] = A::add(S.w[found], w);
            } else {
                if (w < A::mul(ws, thr)) continue;
                if (n >= CAP) { status |= kGeoSetOverflow; return 0; }
                if (lane == 0) {
                    S.val[n] = val;
                    S.key[n] = key;
                    S.w[n] = w;
                }
                // a later child with the same offset (repeated forward differences) adds to it
                if (lane > f && lane < nf && ckey == key) S.cfound[lane] = n;
                ++n;
            }
            __syncwarp();
            int c[3];
            geo_unpack(key, c);
            sums(w, c);
        }
        if (ws <= 0) {
            double pt[3];
            for (int a = 0; a < D; ++a) pt[a] = A::add(avg[a], 0.5);
            emit(pt);
            return 0;
        }
        double stp[3] = {0, 0, 0}, sq = 0.0;
        const double iw = A::div(1.0, ws);
        for (int a = 0; a < D; ++a) {
            const double old = avg[a];
            avg[a] = A::mul(is[a], iw);
            stp[a] = A::sub(avg[a], old);
        }
        for (int a = 0; a < D; ++a) sq = A::add(sq, A::mul(stp[a], stp[a]));
        if (nst < SCAP) {
            if (lane == 0) {
                S.sv[nst] = bv;
                for (int a = 0; a < 3; ++a) S.sd[nst][a] = stp[a];
            }
        } else {
            for (int a = 0; a < D; ++a) { f0[a] = A::add(f0[a], stp[a]); f1[a] = A::add(f1[a], A::mul(stp[a], bv)); }
        }
        ++nst;
        __syncwarp();
        stepNorm = A::add(stepNorm, A::sqrt(sq));
        if (n == 1) {  // mass concentrated at one point (a seed, or around a wall corner)
            if (nf == 0) break;
            double pt[3];
            for (int a = 0; a < D; ++a) { pt[a] = A::add(avg[a], 0.5); base[a] = avg[a]; }
            if (!emit(pt)) return 0;
            stepNorm = 0;
            nst = 0;
            for (int a = 0; a < 3; ++a) { f0[a] = 0; f1[a] = 0; }
            continue;
        }
        if (stepNorm < step && n > 1) continue;
        const double valInc = A::sub(S.sv[0], bv);
        if (valInc <= 0) continue;
        const double delta = A::div(valInc, (double)D);
        const double rden = A::div(1.0, A::add(valInc, delta));
        double pt[3];
        for (int a = 0; a < D; ++a) pt[a] = base[a];
        const int nl = nst < SCAP ? nst : SCAP;
        for (int k = 0; k < nl; ++k) {
            const double cf = A::add(A::sub(S.sv[k], bv), delta);
            for (int a = 0; a < D; ++a) pt[a] = A::add(pt[a], A::mul(A::mul(S.sd[k][a], cf), rden));
        }
        if (nst > SCAP)  // steps past the list, summed: sum s (v - value + delta) / den
            for (int a = 0; a < D; ++a)
                pt[a] = A::add(pt[a], A::mul(A::add(f1[a], A::mul(A::sub(delta, bv), f0[a])), rden));
        for (int a = 0; a < D; ++a) { pt[a] = A::add(pt[a], 0.5); base[a] = avg[a]; }
        if (!emit(pt)) return 0;
        stepNorm = 0;
        nst = 0;
        for (int a = 0; a < 3; ++a) { f0[a] = 0; f1[a] = 0; }
        // spread of the mass: det(covariance + Id) against the squared volume bound
        double V[3][3];
        for (int i = 0; i < D; ++i)
            for (int j = 0; j <= i; ++j) {
                V[i][j] = A::add(A::sub(A::mul(cs[i][j], iw), A::mul(A::mul(is[i], iw), A::mul(is[j], iw))),
                                 i == j ? 1.0 : 0.0);
                V[j][i] = V[i][j];
            }
        double det;
        if (D == 2) {
            det = A::sub(A::mul(V[0][0], V[1][1]), A::mul(V[1][0], V[0][1]));
        } else {
            const double m0 = A::sub(A::mul(V[1][1], V[2][2]), A::mul(V[1][2], V[2][1]));
            const double m1 = A::sub(A::mul(V[1][0], V[2][2]), A::mul(V[1][2], V[2][0]));
            const double m2 = A::sub(A::mul(V[1][0], V[2][1]), A::mul(V[1][1], V[2][0]));
            det = A::add(A::sub(A::mul(V[0][0], m0), A::mul(V[0][1], m1)), A::mul(V[0][2], m2));
        }
        if (det > A::mul(vbound, vbound)) {
            for (int a = 0; a < D; ++a) pt[a] = A::add(avg[a], 0.5);
            emit(pt);
            return 1;
        }
    }
    return 0;
}

// First point of a tip (warp-wide). tips_Unoriented: the angle (cell centre) of smallest value at
// the point (x, y), the last one on ties (HFMInterface.hxx:499-521); the first angle if (x, y) is
// outside the grid.
template <typename Real>
__device__ void geo_tip_start(const Dev<Real> &P, const Inst &I, const GeoTip &tp, double *tip) {
    using A = Arith<double>;
    const int lane = threadIdx.x & 31;
    const GridGeom &g = I.g;
    tip[0] = tp.p[0];
    tip[1] = tp.p[1];
    tip[2] = tp.p[2];
    if (!tp.unoriented) return;
    const Real *values = P.values + I.cell0;
    const double fx = floor(tip[0]), fy = floor(tip[1]);
    const bool inside = fx >= 0 && fy >= 0 && fx < g.dims[0] && fy < g.dims[1];
    double bv = A::inf();
    int bt = -1;
    if (inside)
        for (int th = lane; th < g.dims[2]; th += 32) {
            const double v = (double)values[g.lin((int)fx, (int)fy, th)];
            if (v <= bv) { bv = v; bt = th; }
        }
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int ot = __shfl_xor_sync(0xffffffffu, bt, o);
        if (ot >= 0 && (bt < 0 || ov < bv || (ov == bv && ot > bt))) { bv = ov; bt = ot; }
    }
    tip[2] = A::add((double)(bt < 0 ? 0 : bt), 0.5);
}

// One warp per tip, warps looping over the tips (GeodesicDiscreteSolver.hxx:41-55 for the restarts:
// after 5 restarts the volume bound grows by 1.3 per restart, 50 restarts mean failure). With
// GLOBAL the warps' sets live in `gsets` (one per warp of the grid) instead of shared memory.
template <typename Real, int CAP, int SCAP, bool GLOBAL, int D>
__global__ void __launch_bounds__(kGeoWarps * 32)
geodesic_kernel(Dev<Real> P, GeoRec R, const GeoTip *tips, int ntips, double *pts, GeoOut *outs,
                GeoSet<CAP, SCAP> *gsets) {
    using A = Arith<double>;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * kGeoWarps + wib, nw = (long long)gridDim.x * kGeoWarps;
    GeoSet<CAP, SCAP> *S;
    if constexpr (GLOBAL) {
        S = gsets + gw;
    } else {
        __shared__ GeoSet<CAP, SCAP> sets[kGeoWarps];
        S = sets + wib;
    }
    for (long long t = gw; t < ntips; t += nw) {
        const GeoTip tp = tips[t];
        const Inst &I = P.inst[tp.inst];
        const GridGeom &g = I.g;
        double *out = pts + tp.out0 * D;
        double tip[3];
        geo_tip_start<Real>(P, I, tp, tip);
        int len = 0, status = 0, restarts = 0;
        if (tp.cap < 1) {
            status |= kGeoPointOverflow;
        } else {
            if (lane == 0)
                for (int a = 0; a < D; ++a) out[a] = tip[a];
            len = 1;
            double vb = tp.vbound;
            const long long iter_cap = 64 * g.ncells + 4096;
            while (restarts < 50) {
                const int r = geodesic_pass<Real, CAP, SCAP, D>(P, I, R, *S, out, tp.cap, len, status, tp.step,
                                                               tp.thr, vb, iter_cap);
                if (!r || status) break;
                ++restarts;
                if (restarts >= 5) vb = A::mul(vb, 1.3);
            }
            if (restarts == 50) status |= kGeoFailed;
        }
        if (lane == 0) outs[t] = GeoOut{len, status, restarts, 0};
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------------
// ODE geodesic solver (Headers/Base/Implementation/GeodesicODESolver.hxx): a midpoint scheme on the
// geodesic flow interpolated from the 2^D cells around the point. It stops when the L-infinity
// distance to the seeds (capped at 6) is larger than it was ceil(sqrt(D)/step) steps before, and
// fails when a cell has been used more than int(6 sqrt(D)/step) times (stationarity). The counts
// live in a per-tip hash table in global memory (one per warp of the grid); the flow data of a
// cell is recomputed where the reference caches it (the same values). For the unit offsets used
// here the wall test of VisibleOffset reduces to "the target cell is not a wall".

constexpr short kOdeFar = 32767;
constexpr int kOdeTargetCap = 6;
constexpr int kOdeHistCap = 256;

// L-infinity distance to the seeds (LInfDistance, GeodesicODESolver.hxx:225-258): 0 at the seeds.
template <typename Real, int KIND>
__global__ void ode_target_init_kernel(Dev<Real> P, short *target) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    bool fixed, dead;
    cell_flags<Real, KIND>(P, R.c, fixed, dead);
    target[x] = fixed ? (short)0 : kOdeFar;
}

// The flow data the ODE solver reads at a cell (the reference's GeodesicFlow, cached per tip):
// rec[x][0..D) = sum of weight * offset over the Recompute flow, rec[x][D] = value, rec[x][D+1] =
// width. Computed once for every cell of the batch.
template <typename Real, int NFWD, int NSYM, int KIND>
__global__ void ode_cell_kernel(Dev<Real> P, int D, double *rec) {
    using A = Arith<double>;
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    unsigned foff[kGeoMaxFlow];
    double fw[kGeoMaxFlow], v, wd;
    const int nf = recompute_flow<Real, NFWD, NSYM, KIND>(P, I, R.x0, R.x1, R.x2, foff, fw, &v, &wd);
    double *o = rec + x * (D + 2);
    for (int a = 0; a < D; ++a) {
        double acc = 0.0;
        for (int f = 0; f < nf; ++f) acc = A::add(acc, A::mul(fw[f], (double)off_c(foff[f], a)));
        o[a] = acc;
    }
    o[D] = v;
    o[D + 1] = wd;
}

// One breadth-first level: an unassigned cell that is not a wall takes k + 1 if one of its 3^D - 1
// neighbours is at k (cells at the cap are not expanded).
template <typename Real>
__global__ void ode_target_step_kernel(Dev<Real> P, const int8_t *wd, int k, short *target) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= P.ncells || target[x] != kOdeFar) return;
    const CellRef R = cell_ref(P.inst, P.ninst, x);
    const Inst &I = P.inst[R.i];
    const GridGeom &g = I.g;
    if (wd && I.has_walls && wd[x] == 0) return;
    for (int o = 0; o < 27; ++o) {
        if (o == 13) continue;
        int y0 = R.x0 - (o / 9 - 1), y1 = R.x1 - ((o / 3) % 3 - 1), y2 = R.x2 - (o % 3 - 1);
        if (!g.wrap(y0, y1, y2)) continue;
        if (target[I.cell0 + g.lin(y0, y1, y2)] == (short)k) {
            target[x] = (short)(k + 1);
            return;
        }
    }
}

// GeodesicFlow at a point (GeodesicODESolver.hxx:53-154), warp-wide; lanes < 2^D each take one of
// the cells around the point. Returns the interpolated flow (uniform), the largest use count
// before this call among the cells (nstat) and their smallest target distance (tol).
template <typename Real>
__device__ void ode_flow_at(const Dev<Real> &P, const Inst &I, int D, const int8_t *wd, const short *target,
                            const double *rec, unsigned long long *keys, int *counts, int tmask, double causality,
                            const double *pt, double *flow, int &nstat, int &tol, int &status) {
    using A = Arith<double>;
    const int lane = threadIdx.x & 31;
    const GridGeom &g = I.g;
    int pi[3] = {0, 0, 0}, sg[3] = {0, 0, 0};
    double w[3] = {0, 0, 0};
    for (int j = 0; j < D; ++j) {
        pi[j] = (int)floor(pt[j]);
        w[j] = A::sub(A::sub(pt[j], (double)pi[j]), 0.5);
        sg[j] = w[j] > 0 ? 1 : -1;
        w[j] = fabs(w[j]);
    }
    bool valid = false;
    int ltol = 2147483647, lstat = 0;
    double val = A::inf(), wid = 0.0, fl[3] = {0, 0, 0}, weight = 0.0;
    if (lane < (1 << D)) {
        int q[3] = {pi[0], pi[1], pi[2]};
        for (int j = 0; j < D; ++j)
            if ((lane >> j) & 1) q[j] += sg[j];
        valid = g.wrap(q[0], q[1], q[2]);
        const long long y = valid ? g.lin(q[0], q[1], q[2]) : 0;
        if (valid && wd && I.has_walls && wd[I.cell0 + y] == 0) valid = false;
        if (valid) {
            ltol = target[I.cell0 + y];
            const double *r = rec + (I.cell0 + y) * (D + 2);
            for (int a = 0; a < D; ++a) fl[a] = r[a];
            val = r[D];
            wid = r[D + 1];
            // use count of the cell in this tip's table (open addressing, linear probing)
            unsigned h = (unsigned)((unsigned long long)(y + 1) * 0x9E3779B97F4A7C15ull >> 32) & (unsigned)tmask;
            int probes = 0;
            for (;;) {
                const unsigned long long prev = atomicCAS(keys + h, ~0ull, (unsigned long long)y);
                if (prev == ~0ull || prev == (unsigned long long)y) break;
                h = (h + 1) & (unsigned)tmask;
                if (++probes > (tmask >> 1)) { status |= kGeoSetOverflow; break; }
            }
            if (probes <= (tmask >> 1)) lstat = atomicAdd(counts + h, 1);
            weight = 1.0;
            for (int j = 0; j < D; ++j) weight = A::mul(weight, ((lane >> j) & 1) ? w[j] : A::sub(1.0, w[j]));
        }
    }
    status |= __reduce_or_sync(0xffffffffu, (unsigned)status);
    // reductions in the order of the cells (the reference's loops over i)
    tol = 2147483647;
    nstat = 0;
    double minVal = A::inf(), minWidth = 0.0;
    for (int i = 0; i < (1 << D); ++i) {
        const bool vi = __shfl_sync(0xffffffffu, valid, i);
        if (!vi) continue;
        tol = min(tol, __shfl_sync(0xffffffffu, ltol, i));
        nstat = max(nstat, __shfl_sync(0xffffffffu, lstat, i));
        const double wi = __shfl_sync(0xffffffffu, weight, i), v = __shfl_sync(0xffffffffu, val, i);
        const double wd_i = __shfl_sync(0xffffffffu, wid, i);
        if (wi > 0 && v < minVal) { minVal = v; minWidth = wd_i; }
    }
    flow[0] = flow[1] = flow[2] = 0.0;
    if (!(minVal < A::inf())) return;  // in a wall
    const double thr = A::add(minVal, A::mul(causality, minWidth));
    double ws = 0.0;
    for (int i = 0; i < (1 << D); ++i) {
        const bool vi = __shfl_sync(0xffffffffu, valid, i);
        const double wi = __shfl_sync(0xffffffffu, weight, i), v = __shfl_sync(0xffffffffu, val, i);
        double f[3];
        for (int a = 0; a < 3; ++a) f[a] = __shfl_sync(0xffffffffu, fl[a], i);
        if (!vi || !(wi > 0)) continue;
        if (v <= thr) {
            ws = A::add(ws, wi);
            for (int a = 0; a < D; ++a) flow[a] = A::add(flow[a], A::mul(wi, f[a]));
        }
    }
    if (ws > 0) {
        const double iw = A::div(1.0, ws);
        for (int a = 0; a < D; ++a) flow[a] = A::mul(flow[a], iw);
    }
}

// One warp per ODE tip (Run, GeodesicODESolver.hxx:159-212); the warp's count table has
// 2^table_log2 entries at keys/counts + warp * 2^table_log2.
template <typename Real>
__global__ void __launch_bounds__(kGeoWarps * 32)
geodesic_ode_kernel(Dev<Real> P, const GeoTip *tips, int ntips, double *pts, GeoOut *outs, const int8_t *wd,
                    const short *target, const double *rec, unsigned long long *tkeys, int *tcounts, int table_log2) {
    using A = Arith<double>;
    __shared__ int hist_s[kGeoWarps][kOdeHistCap];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long gw = (long long)blockIdx.x * kGeoWarps + wib, nw = (long long)gridDim.x * kGeoWarps;
    int *hist = hist_s[wib];
    for (long long t = gw; t < ntips; t += nw) {
        const GeoTip tp = tips[t];
        const Inst &I = P.inst[tp.inst];
        const int D = tp.ndim;
        double *out = pts + tp.out0 * D;
        double tip[3];
        geo_tip_start<Real>(P, I, tp, tip);
        int len = 0, status = 0, failed = 0;
        const int tl2 = min(tp.table_log2, table_log2);
        const int tmask = (1 << tl2) - 1;
        unsigned long long *keys = tkeys + (gw << table_log2);
        int *counts = tcounts + (gw << table_log2);
        for (int i = lane; i <= tmask; i += 32) { keys[i] = ~0ull; counts[i] = 0; }
        for (int i = lane; i < tp.nhist; i += 32) hist[i] = 2147483647;
        __syncwarp();
        __threadfence_block();
        if (tp.cap < 1 || tp.nhist > kOdeHistCap) {
            status |= kGeoPointOverflow;
        } else {
            if (lane == 0)
                for (int a = 0; a < D; ++a) out[a] = tip[a];
            len = 1;
            int head = 0;
            double p[3] = {tip[0], tip[1], tip[2]};
            for (;;) {
                double f[3];
                int nstat, tol;
                ode_flow_at<Real>(P, I, D, wd, target, rec, keys, counts, tmask, tp.causality, p, f, nstat, tol,
                                  status);
                if (status) break;
                int old = tol;
                if (tp.nhist > 0) {
                    __syncwarp();
                    old = hist[head];
                    __syncwarp();
                    if (lane == 0) hist[head] = tol;
                    head = head + 1 == tp.nhist ? 0 : head + 1;
                }
                if (old < tol) break;  // moving away from the seeds: done
                if (nstat > tp.nstat_max) { failed = 1; break; }
                double nrm = 0.0;
                for (int a = 0; a < D; ++a) nrm = A::add(nrm, A::mul(f[a], f[a]));
                nrm = A::sqrt(nrm);
                if (nrm == 0) break;  // at a seed
                const double half = A::mul(0.5, tp.step);
                double q[3] = {p[0], p[1], p[2]};
                const double inv = A::div(1.0, nrm);
                for (int a = 0; a < D; ++a) q[a] = A::add(p[a], A::mul(A::mul(half, f[a]), inv));
                ode_flow_at<Real>(P, I, D, wd, target, rec, keys, counts, tmask, tp.causality, q, f, nstat, tol,
                                  status);
                if (status) break;
                nrm = 0.0;
                for (int a = 0; a < D; ++a) nrm = A::add(nrm, A::mul(f[a], f[a]));
                nrm = A::sqrt(nrm);
                if (nrm == 0) break;
                if (len >= tp.cap) { status |= kGeoPointOverflow; break; }
                const double inv2 = A::div(1.0, nrm);
                for (int a = 0; a < D; ++a) p[a] = A::add(p[a], A::mul(A::mul(tp.step, f[a]), inv2));
                if (lane == 0)
                    for (int a = 0; a < D; ++a) out[(long long)len * D + a] = p[a];
                ++len;
            }
        }
        if (lane == 0) outs[t] = GeoOut{len, status | (failed ? kGeoFailed : 0), 0, 0};
        __syncwarp();
    }
}

// Gathers the points of each tip (len points of ndim values at out0) into a compact array.
__global__ void geodesic_compact_kernel(const double *pts, const GeoTip *tips, const GeoOut *outs,
                                        const long long *dst0, int ntips, double *dst) {
    for (int t = blockIdx.x; t < ntips; t += gridDim.x) {
        const long long n = (long long)outs[t].len * tips[t].ndim;
        const double *src = pts + tips[t].out0 * tips[t].ndim;
        double *d = dst + dst0[t];
        for (long long i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
    }
}

// Model dimensions a stencil family can have (the discrete kernel is compiled per dimension):
// two symmetric per-cell differences are Diagonal2, three Riemann2 or Diagonal3, six Riemann3; two
// shared axis differences are Isotropic2; every other family is three-dimensional.
template <int NFWD, int NSYM, int KIND>
constexpr bool geo_dim_ok(int d) {
    if (KIND == kKindRiemann && NFWD == 0 && NSYM == 2) return d == 2;
    if (KIND == kKindRiemann && NFWD == 0 && NSYM == 3) return true;
    if (is_share(KIND) && NFWD == 0 && NSYM == 2) return d == 2;
    return d == 3;
}

// Geodesics of the tips of every instance of a batch, on the arrival times resident in P.values,
// and the geodesic flow fields that were requested. A tip whose points or pending entries
// overflowed is run again with 8x the room (its set in global memory); three attempts at most.
template <typename Real, int NFWD, int NSYM, int KIND>
void run_geodesics(const Dev<Real> &P, const std::vector<Inst> &hinst, const std::vector<const EulerProblem *> &probs,
                   std::vector<EulerResult> &results, const int8_t *wd, cudaStream_t s) {
    const int ninst = (int)probs.size();
    bool any_flow = false;
    std::vector<GeoTip> tips;
    std::vector<int> group;  // 0: tips, 1: tips_Unoriented
    long long slots = 0;
    int ndim = 2;
    for (int i = 0; i < ninst; ++i) {
        const EulerProblem &p = *probs[i];
        ndim = p.ndim;
        any_flow |= p.want_geodesic_flow;
        long long extent = 0;
        for (int a = 0; a < p.ndim; ++a) extent += p.dims[a];
        const int cap = (int)std::min<long long>(1 << 24, std::max<long long>(256, (long long)(2.0 * extent / p.geo_step)));
        for (int gi = 0; gi < 2; ++gi) {
            const std::vector<double> &src = gi ? p.geo_tips_unoriented : p.geo_tips;
            const int w = gi ? 2 : p.ndim;
            for (size_t k = 0; k + w <= src.size(); k += w) {
                GeoTip t{};
                for (int a = 0; a < w; ++a) t.p[a] = src[k + a];
                t.step = p.geo_step;
                t.thr = p.geo_threshold;
                t.vbound = p.geo_volume_bound;
                t.out0 = slots;
                t.inst = i;
                t.cap = cap;
                t.ndim = p.ndim;
                t.unoriented = gi;
                t.ode = p.geo_ode ? 1 : 0;
                t.causality = p.geo_causality;
                if (p.geo_ode) {
                    const double sd = std::sqrt((double)p.ndim);
                    t.nstat_max = (int)(6 * sd / p.geo_step);
                    const double hl = sd / p.geo_step;
                    if (!(hl < kOdeHistCap))
                        throw Error(HFM_ERR_UNSUPPORTED, "geodesicStep too small for the ODE geodesic solver");
                    int nh = 0;
                    while (nh < hl) ++nh;
                    t.nhist = nh;
                    int l2 = 12;
                    while (l2 < 24 && (1ll << l2) < 2ll * cap) ++l2;
                    t.table_log2 = l2;
                }
                slots += cap;
                tips.push_back(t);
                group.push_back(gi);
            }
        }
    }
    const int ntips = (int)tips.size();
    if (ntips == 0 && !any_flow) return;
    EventTimer tm;
    tm.start(s);
    int dev = 0, nsm = 0;
    HFM_CUDA(cudaGetDevice(&dev));
    HFM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (any_flow) {
        DeviceBuffer<double> flow(P.ncells * ndim);
        launch(geodesic_flow_kernel<Real, NFWD, NSYM, KIND>, nblocks(P.ncells, 128), 128, 0, s, P, ndim, flow.get());
        HFM_CUDA(cudaGetLastError());
        for (int i = 0; i < ninst; ++i) {
            if (!probs[i]->want_geodesic_flow) continue;
            const long long n = hinst[i].g.ncells * ndim;
            results[i].geodesic_flow.resize(n);
            HFM_CUDA(cudaMemcpyAsync(results[i].geodesic_flow.data(), flow.get() + hinst[i].cell0 * ndim,
                                     n * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        HFM_CUDA(cudaStreamSynchronize(s));
    }
    if (ntips > 0) {
        std::vector<GeoOut> houts(ntips);
        std::vector<int> todo(ntips);
        for (int t = 0; t < ntips; ++t) todo[t] = t;
        std::vector<std::vector<double>> tip_pts(ntips);
        DeviceBuffer<short> target;  // L-infinity distance to the seeds (ODE tips)
        DeviceBuffer<double> orec;   // per-cell flow, value and width (ODE tips)
        // per-cell Recompute flow (discrete tips): at most one entry per forward difference and one
        // side per symmetric difference
        const int maxf = std::min(kGeoMaxFlow, KIND == kKindTTI ? 6 : NFWD + NSYM);
        DeviceBuffer<uint8_t> rnf;
        DeviceBuffer<unsigned> rfoff;
        DeviceBuffer<double> rfw;
        for (int attempt = 0; attempt < 3 && !todo.empty(); ++attempt) {
            bool big = false;
            if (attempt > 0) {
                long long sl = 0;
                for (int t : todo) {
                    const bool set_over = (houts[t].status & kGeoSetOverflow) != 0;
                    big |= set_over && !tips[t].ode;
                    if (set_over && tips[t].ode) tips[t].table_log2 = std::min(27, tips[t].table_log2 + 3);
                    if (houts[t].status & kGeoPointOverflow) tips[t].cap = (int)std::min<long long>(1 << 27, 8ll * tips[t].cap);
                    tips[t].out0 = sl;
                    sl += tips[t].cap;
                }
                slots = sl;
            }
            // discrete tips first, then ODE tips (one launch each)
            std::stable_partition(todo.begin(), todo.end(), [&](int t) { return !tips[t].ode; });
            std::vector<GeoTip> sub(todo.size());
            for (size_t k = 0; k < todo.size(); ++k) sub[k] = tips[todo[k]];
            const int nsub = (int)sub.size();
            int ndisc = 0;
            while (ndisc < nsub && !sub[ndisc].ode) ++ndisc;
            const int node = nsub - ndisc;
            DeviceBuffer<GeoTip> dtips(nsub);
            dtips.upload(sub.data(), nsub, s);
            DeviceBuffer<GeoOut> douts(nsub);
            DeviceBuffer<double> pts(slots * ndim);
            if (node > 0) {
                if (!target.get()) {
                    target.alloc(P.ncells);
                    launch(ode_target_init_kernel<Real, KIND>, nblocks(P.ncells, 256), 256, 0, s, P, target.get());
                    for (int k = 0; k < kOdeTargetCap; ++k)
                        launch(ode_target_step_kernel<Real>, nblocks(P.ncells, 256), 256, 0, s, P, wd, k, target.get());
                    orec.alloc((size_t)P.ncells * (ndim + 2));
                    launch(ode_cell_kernel<Real, NFWD, NSYM, KIND>, nblocks(P.ncells, 128), 128, 0, s, P, ndim, orec.get());
                    HFM_CUDA(cudaGetLastError());
                }
                int l2 = 0;
                for (int k = ndisc; k < nsub; ++k) l2 = std::max(l2, sub[k].table_log2);
                const int grid = std::max(1, std::min((node + kGeoWarps - 1) / kGeoWarps, nsm));
                const size_t entries = ((size_t)grid * kGeoWarps) << l2;
                DeviceBuffer<unsigned long long> tkeys(entries);
                DeviceBuffer<int> tcounts(entries);
                launch(geodesic_ode_kernel<Real>, grid, kGeoWarps * 32, 0, s, P, dtips.get() + ndisc, node, pts.get(),
                       douts.get() + ndisc, wd, (const short *)target.get(), (const double *)orec.get(), tkeys.get(),
                       tcounts.get(), l2);
                HFM_CUDA(cudaGetLastError());
                HFM_CUDA(cudaStreamSynchronize(s));
            }
            const int want_blocks = (ndisc + kGeoWarps - 1) / kGeoWarps;
            if (ndisc > 0 && !rnf.get()) {
                rnf.alloc(P.ncells);
                rfoff.alloc((size_t)maxf * P.ncells);
                rfw.alloc((size_t)maxf * P.ncells);
                launch(geo_rec_kernel<Real, NFWD, NSYM, KIND>, nblocks(P.ncells, 128), 128, 0, s, P, maxf, rnf.get(),
                       rfoff.get(), rfw.get());
                HFM_CUDA(cudaGetLastError());
            }
            const GeoRec R{P.ncells, rnf.get(), rfoff.get(), rfw.get()};
            if (ndisc > 0 && !big) {
                auto run = [&](auto kern) {
                    int per_sm = 0;
                    HFM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGeoWarps * 32, 0));
                    const int grid = std::max(1, std::min(want_blocks, nsm * std::max(1, per_sm)));
                    launch(kern, grid, kGeoWarps * 32, 0, s, P, R, dtips.get(), ndisc, pts.get(), douts.get(),
                           (GeoSet<kGeoCap, kGeoStepCap> *)nullptr);
                };
                if (ndim == 2) {
                    if constexpr (geo_dim_ok<NFWD, NSYM, KIND>(2))
                        run(geodesic_kernel<Real, kGeoCap, kGeoStepCap, false, 2>);
                } else if constexpr (geo_dim_ok<NFWD, NSYM, KIND>(3)) {
                    run(geodesic_kernel<Real, kGeoCap, kGeoStepCap, false, 3>);
                }
            } else if (ndisc > 0) {
                const int grid = std::max(1, std::min(want_blocks, 2 * nsm));
                DeviceBuffer<GeoSet<kGeoCapBig, kGeoStepCapBig>> gsets((size_t)grid * kGeoWarps);
                auto run = [&](auto kern) {
                    launch(kern, grid, kGeoWarps * 32, 0, s, P, R, dtips.get(), ndisc, pts.get(), douts.get(),
                           gsets.get());
                };
                if (ndim == 2) {
                    if constexpr (geo_dim_ok<NFWD, NSYM, KIND>(2))
                        run(geodesic_kernel<Real, kGeoCapBig, kGeoStepCapBig, true, 2>);
                } else if constexpr (geo_dim_ok<NFWD, NSYM, KIND>(3)) {
                    run(geodesic_kernel<Real, kGeoCapBig, kGeoStepCapBig, true, 3>);
                }
                HFM_CUDA(cudaStreamSynchronize(s));
            }
            HFM_CUDA(cudaGetLastError());
            std::vector<GeoOut> o(nsub);
            douts.download(o.data(), nsub, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            // compact the finished tips of this attempt and bring their points back
            std::vector<long long> d0(nsub, 0);
            long long tot = 0;
            for (int k = 0; k < nsub; ++k) {
                d0[k] = tot;
                tot += (long long)o[k].len * ndim;
            }
            DeviceBuffer<long long> dd0(nsub);
            dd0.upload(d0.data(), nsub, s);
            DeviceBuffer<double> cpt(std::max<long long>(tot, 1));
            launch(geodesic_compact_kernel, std::min(nsub, 4 * nsm), 128, 0, s, pts.get(), dtips.get(), douts.get(),
                   dd0.get(), nsub, cpt.get());
            HFM_CUDA(cudaGetLastError());
            std::vector<double> hp(tot);
            if (tot) cpt.download(hp.data(), tot, s);
            HFM_CUDA(cudaStreamSynchronize(s));
            std::vector<int> again;
            for (int k = 0; k < nsub; ++k) {
                const int t = todo[k];
                houts[t] = o[k];
                const bool rerun = (o[k].status & (kGeoPointOverflow | kGeoSetOverflow)) != 0;
                if (rerun && attempt < 2) {
                    again.push_back(t);
                    continue;
                }
                tip_pts[t].assign(hp.begin() + d0[k], hp.begin() + d0[k] + (long long)o[k].len * ndim);
            }
            todo.swap(again);
        }
        for (int t = 0; t < ntips; ++t) {  // in the order of the tips
            EulerResult &r = results[tips[t].inst];
            const int gi = group[t];
            r.geo_points[gi].insert(r.geo_points[gi].end(), tip_pts[t].begin(), tip_pts[t].end());
            r.geo_lengths[gi].push_back(houts[t].len);
            r.geo_status[gi].push_back(houts[t].status);
            r.geo_restarts[gi].push_back(houts[t].restarts);
        }
    }
    const float ms = tm.stop(s);
    for (int i = 0; i < ninst; ++i) results[i].t_geodesic_ms = ms;
}
