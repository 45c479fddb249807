// oza_tune_host.cpp -- C ABI of the accuracy tools (see oza_tune.cu):
// oza_block_error, oza_autotune_slices / oza_autotune_scheme (measured on a
// sampled block) and oza_slices_for_target / oza_scheme_for_target (from the
// calibrated tables of oza_slice_table.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "oza_capi.h"
#include "oza_kernels.h"
#include "oza_slice_table.h"

namespace oza {
cudaError_t launch_dd_block_gemm(const double* A, const double* B, int r, int c, size_t K, double* C,
                                 cudaStream_t st);
cudaError_t launch_gather_block(const double* A, const double* B, size_t M, size_t N, size_t K,
                                const long long* rows, int r, const long long* cols, int c, double* Ab, double* Bb,
                                cudaStream_t st);
}  // namespace oza

namespace {

oza_status_t tfail(oza_status_t st, const std::string& m) {
    oza::set_last_error(m.c_str());
    return st;
}

std::vector<long long> sample_indices(size_t n, int k, std::mt19937_64& rng) {
    std::vector<long long> idx;
    if ((size_t)k >= n) {
        idx.resize(n);
        std::iota(idx.begin(), idx.end(), 0ll);
        return idx;
    }
    std::vector<long long> all(n);
    std::iota(all.begin(), all.end(), 0ll);
    for (int i = 0; i < k; ++i) {   // partial Fisher-Yates
        std::uniform_int_distribution<size_t> d(i, n - 1);
        std::swap(all[i], all[d(rng)]);
    }
    idx.assign(all.begin(), all.begin() + k);
    std::sort(idx.begin(), idx.end());
    return idx;
}

// Max relative error of got against ref (absolute where ref is 0), as
// utils/matrix_compare.hpp:24-65 of the reference measures it.
double max_rel(const std::vector<double>& got, const std::vector<double>& ref) {
    double m = 0.0;
    for (size_t i = 0; i < ref.size(); ++i) {
        const double d = std::fabs(got[i] - ref[i]);
        const double r = ref[i] != 0.0 ? d / std::fabs(ref[i]) : d;
        if (!(r <= m)) m = r;   // NaN propagates as the maximum
    }
    return m;
}

// Device buffers of one sampled block and its double-double reference.
struct Block {
    oza_exec_t ex = nullptr;
    int r = 0, c = 0;
    size_t K = 0;
    std::vector<long long> rows, cols;
    void* d_idx = nullptr;
    double* Ab = nullptr;
    double* Bb = nullptr;
    double* Cb = nullptr;
    double* Rb = nullptr;
    std::vector<double> ref;
    double unit = 1.0;   // errors on this block are compared in units of this (a reference result's error)
    ~Block() {
        void* bufs[] = {d_idx, Ab, Bb, Cb, Rb};
        for (void* p : bufs)
            if (p) oza_executor_free(ex, p);
    }
};

oza_status_t make_block(oza_exec_t ex, const double* A, const double* B, size_t M, size_t N, size_t K, int block,
                        unsigned seed, Block& b) {
    if (block < 1) return tfail(OZA_INVALID_ARG, "block size must be >= 1");
    std::mt19937_64 rng(seed);
    b.ex = ex;
    b.K = K;
    b.rows = sample_indices(M, block, rng);
    b.cols = sample_indices(N, block, rng);
    b.r = (int)b.rows.size();
    b.c = (int)b.cols.size();
    const size_t nidx = b.rows.size() + b.cols.size();
    oza_status_t st;
    if ((st = oza_executor_alloc(ex, &b.d_idx, nidx * sizeof(long long))) != OZA_OK) return st;
    if ((st = oza_executor_alloc(ex, (void**)&b.Ab, (size_t)b.r * K * sizeof(double) + 8)) != OZA_OK) return st;
    if ((st = oza_executor_alloc(ex, (void**)&b.Bb, K * (size_t)b.c * sizeof(double) + 8)) != OZA_OK) return st;
    if ((st = oza_executor_alloc(ex, (void**)&b.Cb, (size_t)b.r * b.c * sizeof(double))) != OZA_OK) return st;
    if ((st = oza_executor_alloc(ex, (void**)&b.Rb, (size_t)b.r * b.c * sizeof(double))) != OZA_OK) return st;
    std::vector<long long> idx(b.rows);
    idx.insert(idx.end(), b.cols.begin(), b.cols.end());
    if ((st = oza_executor_copy(ex, b.d_idx, idx.data(), nidx * sizeof(long long), 1)) != OZA_OK) return st;
    const long long* drows = static_cast<const long long*>(b.d_idx);
    int dev = 0, prev = -1;
    if ((st = oza_executor_device(ex, &dev)) != OZA_OK) return st;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return tfail(OZA_CUDA_ERROR, "cudaSetDevice failed");
    cudaError_t e = oza::launch_gather_block(A, B, M, N, K, drows, b.r, drows + b.r, b.c, b.Ab, b.Bb, nullptr);
    if (e == cudaSuccess) e = oza::launch_dd_block_gemm(b.Ab, b.Bb, b.r, b.c, K, b.Rb, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) return tfail(OZA_CUDA_ERROR, std::string("sampled reference: ") + cudaGetErrorString(e));
    b.ref.resize((size_t)b.r * b.c);
    return oza_executor_copy(ex, b.ref.data(), b.Rb, b.ref.size() * sizeof(double), 2);
}

// Ozaki result on the block for one scheme / slice count, and its error.
oza_status_t block_trial(Block& b, int scheme, int slices, double* err) {
    oza_ws_t ws = nullptr;
    oza_status_t st = oza_ws_create(b.ex, scheme, (size_t)b.r, (size_t)b.c, b.K, slices, 0u, &ws);
    if (st != OZA_OK) return st;
    oza_timings_t t;   // synchronous
    st = oza_gemm(ws, b.Ab, b.Bb, b.Cb, &t);
    oza_ws_destroy(ws);
    if (st != OZA_OK) return st;
    std::vector<double> got(b.ref.size());
    st = oza_executor_copy(b.ex, got.data(), b.Cb, got.size() * sizeof(double), 2);
    if (st != OZA_OK) return st;
    *err = max_rel(got, b.ref);
    return OZA_OK;
}

// The largest sampled error over several blocks.
oza_status_t blocks_trial(Block* const* blocks, int nblocks, int scheme, int slices, double* err) {
    double worst = 0.0;
    for (int i = 0; i < nblocks; ++i) {
        double e = 0.0;
        const oza_status_t st = block_trial(*blocks[i], scheme, slices, &e);
        if (st != OZA_OK) return st;
        e /= blocks[i]->unit;
        if (!(e <= worst)) worst = e;   // NaN propagates
    }
    *err = worst;
    return OZA_OK;
}

// Smallest S in [1, smax] whose sampled error (the largest over the blocks)
// meets the target, by bisection on the (monotonically falling) error.
// *reached = false (and S = smax with its error) if even smax misses.
oza_status_t bisect_slices(Block* const* blocks, int nblocks, int scheme, int smax, double target, int* S,
                           double* err, bool* reached) {
    double err_hi = 0.0;
    oza_status_t st = blocks_trial(blocks, nblocks, scheme, smax, &err_hi);
    if (st != OZA_OK) return st;
    if (!(err_hi <= target)) {
        *S = smax;
        *err = err_hi;
        *reached = false;
        return OZA_OK;
    }
    int lo = 1, hi = smax;
    double best = err_hi;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        double e = 0.0;
        if ((st = blocks_trial(blocks, nblocks, scheme, mid, &e)) != OZA_OK) return st;
        if (e <= target) {
            hi = mid;
            best = e;
        } else {
            lo = mid + 1;
        }
    }
    *S = hi;
    *err = best;
    *reached = true;
    return OZA_OK;
}

// The error of an M x N device result C on the block's entries.
oza_status_t given_error(const Block& b, const double* C, size_t N, double* err) {
    std::vector<double> got((size_t)b.r * b.c);
    std::vector<double> row(N);
    for (int i = 0; i < b.r; ++i) {
        const oza_status_t st = oza_executor_copy(b.ex, row.data(), C + (size_t)b.rows[i] * N, N * sizeof(double), 2);
        if (st != OZA_OK) return st;
        for (int j = 0; j < b.c; ++j) got[(size_t)i * b.c + j] = row[b.cols[j]];
    }
    *err = max_rel(got, b.ref);
    return OZA_OK;
}

// INT8 GEMMs per Ozaki GEMM: S (Scheme II), S (S + 1) / 2 (Scheme I).
int gemm_count(int scheme, int S) { return scheme == OZA_SCHEME2 ? S : S * (S + 1) / 2; }

// Calibrated-table lookup (oza_slice_table.h) for a target, K and phi.
template <class Table>
int table_slices(const Table& tab, double target_rel_err, size_t K, double phi) {
    // Decade: the smallest d with 10^-d <= target (conservative), clamped to the table.
    int d = (int)std::ceil(-std::log10(target_rel_err) - 1e-9);
    if (d < kSliceTableDecadeMin) d = kSliceTableDecadeMin;
    if (d > kSliceTableDecadeMax) return 21;
    const int nk = (int)(sizeof(kSliceTableK) / sizeof(kSliceTableK[0]));
    const int np = (int)(sizeof(kSliceTablePhi) / sizeof(kSliceTablePhi[0]));
    int ki = 0;
    while (ki < nk - 1 && (size_t)kSliceTableK[ki] < K) ++ki;
    int extra = 0;   // beyond the last K: one more slice per factor 4
    for (size_t k = (size_t)kSliceTableK[nk - 1]; k < K; k *= 4) ++extra;
    int pi = 0;
    while (pi < np - 1 && kSliceTablePhi[pi] < phi) ++pi;
    // Monotone envelope: the measured maximum error is noisy in K and phi.
    int S = 1;
    for (int a = 0; a <= ki; ++a)
        for (int c = 0; c <= pi; ++c) S = std::max(S, (int)tab[a][c][d - kSliceTableDecadeMin]);
    S += extra;
    return S > 21 ? 21 : S;
}

// The scheme choice shared by oza_autotune_scheme and
// oza_autotune_scheme_like.  Errors are in each block's unit and compared
// with `target`; prepare(seed, block) samples a block.  Two independent
// blocks: a count is accepted only if it meets the target on both, so a count
// that just reaches it on one sample (the largest error over many outputs is
// heavy-tailed) is not taken.  Scheme II first (S INT8 GEMMs for S moduli);
// Scheme I (S (S + 1) / 2 GEMMs) where it is cheaper for the target or where
// Scheme II's 20 moduli miss it.  Scheme II's moduli are also capped by its
// INT32 bound.
template <class Prepare>
oza_status_t choose_scheme(const char* who, size_t K, double target, unsigned seed, Prepare prepare, int* scheme,
                           int* slices, double* achieved) {
    Block b0, b1;
    oza_status_t st = prepare(seed, b0);
    if (st == OZA_OK) st = prepare(seed ^ 0x5bd1e995u, b1);
    if (st != OZA_OK) return st;
    Block* blocks[2] = {&b0, &b1};
    int S2 = 20, S1 = 20;
    double e2 = 0.0, e1 = 0.0;
    bool r2 = false, r1 = false;
    const bool two_ok = (double)K * 125.0 * 125.0 < 2147483648.0;
    if (two_ok && (st = bisect_slices(blocks, 2, OZA_SCHEME2, 20, target, &S2, &e2, &r2)) != OZA_OK) return st;
    if (r2 && S2 == 20) {
        // Scheme II reaches the target only at its last modulus, with no count
        // left to add: confirm on four more blocks before taking it.
        for (unsigned k = 1; k <= 4 && r2; ++k) {
            Block extra;
            if ((st = prepare(seed + 0x9e3779b9u * k, extra)) != OZA_OK) return st;
            Block* one[1] = {&extra};
            double e = 0.0;
            if ((st = blocks_trial(one, 1, OZA_SCHEME2, 20, &e)) != OZA_OK) return st;
            if (!(e <= e2)) e2 = e;
            r2 = e2 <= target;
        }
    }
    int s1max = 20;
    if (r2)
        while (s1max > 0 && gemm_count(OZA_SCHEME1, s1max) >= S2) --s1max;   // only a cheaper Scheme I counts
    if (s1max > 0 && (st = bisect_slices(blocks, 2, OZA_SCHEME1, s1max, target, &S1, &e1, &r1)) != OZA_OK)
        return st;
    if (r1 || (!r2 && s1max > 0 && (!two_ok || e1 <= e2))) {
        *scheme = OZA_SCHEME1;
        *slices = S1;
        if (achieved) *achieved = e1;
    } else {
        *scheme = OZA_SCHEME2;
        *slices = S2;
        if (achieved) *achieved = e2;
    }
    if (!r1 && !r2) {
        char m[220];
        snprintf(m, sizeof(m), "%s: target %.3g not reached with 20 slices of either scheme "
                 "(sampled errors %.3g / %.3g)", who, target, e2, e1);
        return tfail(OZA_UNSUPPORTED, m);
    }
    return OZA_OK;
}

}  // namespace

extern "C" {

oza_status_t oza_block_error(oza_exec_t ex, const double* A, const double* B, const double* C, size_t M, size_t N,
                             size_t K, int block, unsigned seed, double* max_rel_err) {
    if (!ex || !A || !B || !C || !max_rel_err) return tfail(OZA_INVALID_ARG, "oza_block_error: null argument");
    if (M == 0 || N == 0) {
        *max_rel_err = 0.0;
        return OZA_OK;
    }
    Block b;
    oza_status_t st = make_block(ex, A, B, M, N, K, block, seed, b);
    if (st != OZA_OK) return st;
    return given_error(b, C, N, max_rel_err);
}

oza_status_t oza_autotune_slices(oza_exec_t ex, int scheme, size_t M, size_t N, size_t K, const double* A,
                                 const double* B, double target_rel_err, int block, unsigned seed, int* slices,
                                 double* achieved_err) {
    if (!ex || !A || !B || !slices) return tfail(OZA_INVALID_ARG, "oza_autotune_slices: null argument");
    if (scheme != OZA_SCHEME1 && scheme != OZA_SCHEME2) return tfail(OZA_INVALID_ARG, "oza_autotune_slices: scheme");
    if (!(target_rel_err > 0.0)) return tfail(OZA_INVALID_ARG, "oza_autotune_slices: target must be > 0");
    if (M == 0 || N == 0 || K == 0) {
        *slices = 1;
        if (achieved_err) *achieved_err = 0.0;
        return OZA_OK;
    }
    Block b;
    oza_status_t st = make_block(ex, A, B, M, N, K, block, seed, b);
    if (st != OZA_OK) return st;
    int S = 20;
    double e = 0.0;
    bool reached = false;
    Block* blocks[1] = {&b};
    if ((st = bisect_slices(blocks, 1, scheme, 20, target_rel_err, &S, &e, &reached)) != OZA_OK) return st;
    *slices = S;
    if (achieved_err) *achieved_err = e;
    if (!reached) {
        char m[160];
        snprintf(m, sizeof(m), "oza_autotune_slices: target %.3g not reached with 20 slices (sampled error %.3g)",
                 target_rel_err, e);
        return tfail(OZA_UNSUPPORTED, m);
    }
    return OZA_OK;
}

oza_status_t oza_autotune_scheme(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                                 double target_rel_err, int block, unsigned seed, int* scheme, int* slices,
                                 double* achieved_err) {
    if (!ex || !A || !B || !scheme || !slices) return tfail(OZA_INVALID_ARG, "oza_autotune_scheme: null argument");
    if (!(target_rel_err > 0.0)) return tfail(OZA_INVALID_ARG, "oza_autotune_scheme: target must be > 0");
    if (M == 0 || N == 0 || K == 0) {
        *scheme = OZA_SCHEME2;
        *slices = 1;
        if (achieved_err) *achieved_err = 0.0;
        return OZA_OK;
    }
    auto prepare = [&](unsigned sd, Block& b) { return make_block(ex, A, B, M, N, K, block, sd, b); };
    return choose_scheme("oza_autotune_scheme", K, target_rel_err, seed, prepare, scheme, slices, achieved_err);
}

oza_status_t oza_autotune_scheme_like(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                                      const double* C_ref, double factor, int block, unsigned seed, int* scheme,
                                      int* slices, double* achieved_ratio) {
    if (!ex || !A || !B || !C_ref || !scheme || !slices)
        return tfail(OZA_INVALID_ARG, "oza_autotune_scheme_like: null argument");
    if (!(factor > 0.0)) return tfail(OZA_INVALID_ARG, "oza_autotune_scheme_like: factor must be > 0");
    if (M == 0 || N == 0 || K == 0) {
        *scheme = OZA_SCHEME2;
        *slices = 1;
        if (achieved_ratio) *achieved_ratio = 0.0;
        return OZA_OK;
    }
    // Each block's errors in units of factor x the reference result's error
    // on that block (at least one unit roundoff, for blocks it gets exact).
    auto prepare = [&](unsigned sd, Block& b) {
        oza_status_t st = make_block(ex, A, B, M, N, K, block, sd, b);
        double e = 0.0;
        if (st == OZA_OK) st = given_error(b, C_ref, N, &e);
        if (st == OZA_OK) b.unit = factor * std::max(e, 0x1p-53);
        return st;
    };
    return choose_scheme("oza_autotune_scheme_like", K, 1.0, seed, prepare, scheme, slices, achieved_ratio);
}

oza_status_t oza_estimate_phi(oza_exec_t ex, size_t M, size_t N, size_t K, const double* A, const double* B,
                              int block, unsigned seed, double* phi) {
    if (!ex || !A || !B || !phi) return tfail(OZA_INVALID_ARG, "oza_estimate_phi: null argument");
    if (block < 1) return tfail(OZA_INVALID_ARG, "oza_estimate_phi: block size must be >= 1");
    *phi = 0.0;
    if (M == 0 || N == 0 || K == 0) return OZA_OK;
    std::mt19937_64 rng(seed);
    const std::vector<long long> rows = sample_indices(M, block, rng), cols = sample_indices(N, block, rng);
    const int r = (int)rows.size(), c = (int)cols.size();
    void* d_idx = nullptr;
    double *Ab = nullptr, *Bb = nullptr;
    oza_status_t st = oza_executor_alloc(ex, &d_idx, (size_t)(r + c) * sizeof(long long));
    if (st == OZA_OK) st = oza_executor_alloc(ex, (void**)&Ab, (size_t)r * K * sizeof(double) + 8);
    if (st == OZA_OK) st = oza_executor_alloc(ex, (void**)&Bb, K * (size_t)c * sizeof(double) + 8);
    std::vector<double> ha((size_t)r * K), hb(K * (size_t)c);
    if (st == OZA_OK) {
        std::vector<long long> idx(rows);
        idx.insert(idx.end(), cols.begin(), cols.end());
        st = oza_executor_copy(ex, d_idx, idx.data(), idx.size() * sizeof(long long), 1);
    }
    if (st == OZA_OK) {
        int dev = 0, prev = -1;
        st = oza_executor_device(ex, &dev);
        if (st == OZA_OK) {
            if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
            const long long* di = static_cast<const long long*>(d_idx);
            cudaError_t e = prev != dev ? cudaSetDevice(dev) : cudaSuccess;
            if (e == cudaSuccess) e = oza::launch_gather_block(A, B, M, N, K, di, r, di + r, c, Ab, Bb, nullptr);
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (prev >= 0 && prev != dev) cudaSetDevice(prev);
            if (e != cudaSuccess) st = tfail(OZA_CUDA_ERROR, std::string("oza_estimate_phi: ") + cudaGetErrorString(e));
        }
    }
    if (st == OZA_OK) st = oza_executor_copy(ex, ha.data(), Ab, ha.size() * sizeof(double), 2);
    if (st == OZA_OK) st = oza_executor_copy(ex, hb.data(), Bb, hb.size() * sizeof(double), 2);
    void* bufs[] = {d_idx, Ab, Bb};
    for (void* q : bufs)
        if (q) oza_executor_free(ex, q);
    if (st != OZA_OK) return st;
    // Pooled variance of ln|x| about each row's (A) and column's (B) own mean:
    // per-row and per-column scaling, which the step-1 shifts absorb, drops
    // out.  For (U - 0.5) exp(phi N(0,1)) it is 1 + phi^2 (ln|U - 0.5| has
    // variance 1), the family the calibrated tables were measured on.
    double ss = 0.0;
    long long dof = 0;
    auto strip = [&](const double* x, size_t n, size_t stride) {
        double sum = 0.0, sq = 0.0;
        long long cnt = 0;
        for (size_t i = 0; i < n; ++i) {
            const double v = x[i * stride];
            if (v == 0.0 || !std::isfinite(v)) continue;
            const double l = std::log(std::fabs(v));
            sum += l;
            sq += l * l;
            ++cnt;
        }
        if (cnt > 1) {
            ss += sq - sum * sum / (double)cnt;
            dof += cnt - 1;
        }
    };
    for (int i = 0; i < r; ++i) strip(ha.data() + (size_t)i * K, K, 1);
    for (int j = 0; j < c; ++j) strip(hb.data() + j, K, (size_t)c);
    const double var = dof > 0 ? ss / (double)dof : 0.0;
    *phi = var > 1.0 ? std::sqrt(var - 1.0) : 0.0;
    return OZA_OK;
}

int oza_slices_for_target(double target_rel_err, size_t K, double phi) {
    if (!(target_rel_err > 0.0) || K == 0 || !(phi >= 0.0)) return 0;
    return table_slices(kSliceTable, target_rel_err, K, phi);
}

int oza_scheme_for_target(double target_rel_err, size_t K, double phi, int* slices) {
    if (!slices || !(target_rel_err > 0.0) || K == 0 || !(phi >= 0.0)) return 0;
    const int s2 = (double)K * 125.0 * 125.0 < 2147483648.0 ? table_slices(kSliceTable, target_rel_err, K, phi) : 21;
    const int s1 = table_slices(kSliceTable1, target_rel_err, K, phi);
    // The cheaper in INT8 GEMMs of the schemes that reach the target (Scheme II
    // on a tie); Scheme I at 20 slices when neither does.
    if (s2 <= 20 && (s1 > 20 || gemm_count(OZA_SCHEME2, s2) <= gemm_count(OZA_SCHEME1, s1))) {
        *slices = s2;
        return OZA_SCHEME2;
    }
    *slices = s1;
    return OZA_SCHEME1;
}

}  // extern "C"
