/*
 * oza_oracle.c -- CPU restatement of the OzaBLAS Ozaki Scheme I / Scheme II
 * FP64-emulation pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the sm_100a
 * kernels in ozablas_b200/csrc.  Only the test suite, the smoke check and the
 * CPU-baseline leg of bench.py load it; the product library never links it and
 * has no CPU fallback.
 *
 * Every function states the reference routine it restates (paths relative to
 * the IlyaNyrkov/ozablas source tree).  The arithmetic is written from the
 * algorithm, in plain C with 64-bit indexing (the reference uses 32-bit `int`
 * index arithmetic, which overflows past 2^31 elements).
 *
 * Pinning: tests/test_oracle.py checks every stage of this file bit-exactly
 * against the reference's own kernel source compiled for the host
 * (oracle/ref_shim.cpp -> oracle/_ref/libozaref_cpu.so) and against the
 * committed fixtures in tests/golden/ that the reference produced.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OO_MAX_SLICES 20

/* ------------------------------------------------------------------------- */
/* CRT tables.                                                               */
/* The moduli are the reference's fixed list (src/common/crt_tables.hpp:13-16);
 * they must be identical for the residues to match.  The derived tables
 * (M, floor(M/2), M/m_i, (M/m_i)^-1 mod m_i; crt_tables.hpp:19-112) are
 * recomputed here from the moduli rather than transcribed.                  */
/* ------------------------------------------------------------------------- */
static const unsigned oo_moduli[OO_MAX_SLICES] = {
    251, 241, 239, 233, 229, 227, 223, 211, 199, 197,
    193, 191, 181, 179, 173, 167, 163, 157, 151, 149};

typedef struct { uint64_t w[4]; } u256;

static u256 u256_from(uint64_t v) { u256 r = {{v, 0, 0, 0}}; return r; }

static u256 u256_mul_small(u256 a, uint64_t b) {
    u256 r; unsigned __int128 carry = 0;
    for (int i = 0; i < 4; ++i) {
        unsigned __int128 p = (unsigned __int128)a.w[i] * b + carry;
        r.w[i] = (uint64_t)p; carry = p >> 64;
    }
    return r;
}

static uint64_t u256_mod_small(u256 a, uint64_t m) {
    unsigned __int128 rem = 0;
    for (int i = 3; i >= 0; --i) rem = ((rem << 64) | a.w[i]) % m;
    return (uint64_t)rem;
}

static int u256_ge(u256 a, u256 b) {
    for (int i = 3; i >= 0; --i) {
        if (a.w[i] > b.w[i]) return 1;
        if (a.w[i] < b.w[i]) return 0;
    }
    return 1;
}

static u256 u256_add(u256 a, u256 b) {
    u256 r; unsigned __int128 c = 0;
    for (int i = 0; i < 4; ++i) { c += (unsigned __int128)a.w[i] + b.w[i]; r.w[i] = (uint64_t)c; c >>= 64; }
    return r;
}

static u256 u256_sub(u256 a, u256 b) {   /* a - b, a >= b */
    u256 r; uint64_t borrow = 0;
    for (int i = 0; i < 4; ++i) {
        unsigned __int128 d = (unsigned __int128)a.w[i] - b.w[i] - borrow;
        r.w[i] = (uint64_t)d; borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return r;
}

/* Table for the first S moduli.  Fills M, floor(M/2), M/m_i and the inverse of
 * (M/m_i) modulo m_i (reference: crt_tables.hpp:19-112). */
void oo_crt_tables(int S, uint64_t M[4], uint64_t Mhalf[4],
                   uint64_t partial[OO_MAX_SLICES][4], uint64_t inv[OO_MAX_SLICES]) {
    u256 prod = u256_from(1);
    for (int i = 0; i < S; ++i) prod = u256_mul_small(prod, oo_moduli[i]);
    memcpy(M, prod.w, sizeof(prod.w));
    for (int i = 0; i < 4; ++i) Mhalf[i] = (prod.w[i] >> 1) | (i < 3 ? (prod.w[i + 1] << 63) : 0);
    for (int s = 0; s < S; ++s) {
        u256 p = u256_from(1);
        for (int i = 0; i < S; ++i) if (i != s) p = u256_mul_small(p, oo_moduli[i]);
        memcpy(partial[s], p.w, sizeof(p.w));
        uint64_t m = oo_moduli[s], r = u256_mod_small(p, m), x = 0;
        for (uint64_t c = 1; c < m; ++c) if ((r * c) % m == 1) { x = c; break; }
        inv[s] = x;
    }
}

unsigned oo_modulus(int s) { return oo_moduli[s]; }

/* Reference crt_math.hpp:73-80: d0 + ldexp(d1,64) + ldexp(d2,128) + ldexp(d3,192),
 * accumulated left to right from 0.0 with a rounding after each addition. */
static double oo_u256_to_double(u256 a) {
    double r = 0.0;
    r += (double)a.w[0];
    r += ldexp((double)a.w[1], 64);
    r += ldexp((double)a.w[2], 128);
    r += ldexp((double)a.w[3], 192);
    return r;
}

double oo_crt_M_double(int S) {
    uint64_t M[4], Mh[4], P[OO_MAX_SLICES][4], I[OO_MAX_SLICES];
    oo_crt_tables(S, M, Mh, P, I);
    u256 m; memcpy(m.w, M, sizeof(m.w));
    return oo_u256_to_double(m);
}

/* ------------------------------------------------------------------------- */
/* Step 1 parameters (src/pipeline/step1_statistics.hpp:12-20).              */
/* ------------------------------------------------------------------------- */
int oo_scheme1_beta(long K) {
    int beta = (int)floor((31.0 - log2((double)K)) / 2.0);
    return beta < 1 ? 1 : (beta > 7 ? 7 : beta);
}

/* K_param = floor(0.5*log2((M/2 - 1)/K)) with M rounded to double the way the
 * reference does it (src/cuda/pipeline.cu:196-198). */
int oo_scheme2_kparam(int S, long K) {
    double Md = oo_crt_M_double(S);
    double frac = (Md / 2.0 - 1.0) / (double)K;
    return (int)floor(0.5 * log2(frac));
}

/* frexp exponent of |v| (v != 0), i.e. e with |v| = f * 2^e, f in [0.5, 1). */
static int oo_frexp_exp(double v) { int e; frexp(v, &e); return e; }

/* shift[r] = offset - max_c e(A[r,c]); zero entries are skipped and the running
 * maximum starts at -1023 (step1_statistics.hpp:23-76, compute_row_shifts_A). */
void oo_row_shifts(const double* A, long rows, long cols, int offset, int32_t* shifts) {
    #pragma omp parallel for schedule(static)
    for (long r = 0; r < rows; ++r) {
        int mx = -1023;
        const double* row = A + r * cols;
        for (long c = 0; c < cols; ++c) {
            double v = fabs(row[c]);
            if (v > 0.0) { int e = oo_frexp_exp(v); if (e > mx) mx = e; }
        }
        shifts[r] = offset - mx;
    }
}

/* Column version for B (step1_statistics.hpp:78-99, compute_col_shifts_B). */
void oo_col_shifts(const double* B, long rows, long cols, int offset, int32_t* shifts) {
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    int* part = (int*)malloc(sizeof(int) * (size_t)cols * nthreads);
    for (long i = 0; i < cols * nthreads; ++i) part[i] = -1023;
    #pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int* mine = part + (size_t)t * cols;
        #pragma omp for schedule(static)
        for (long r = 0; r < rows; ++r) {
            const double* row = B + r * cols;
            for (long c = 0; c < cols; ++c) {
                double v = fabs(row[c]);
                if (v > 0.0) { int e = oo_frexp_exp(v); if (e > mine[c]) mine[c] = e; }
            }
        }
    }
    for (long c = 0; c < cols; ++c) {
        int mx = -1023;
        for (int t = 0; t < nthreads; ++t) if (part[(size_t)t * cols + c] > mx) mx = part[(size_t)t * cols + c];
        shifts[c] = offset - mx;
    }
    free(part);
}

/* ------------------------------------------------------------------------- */
/* Step 2.                                                                   */
/* ------------------------------------------------------------------------- */

/* Symmetric residue of the integer-valued double x modulo odd m, in
 * [-(m-1)/2, (m-1)/2].  The reference reaches the same value through two
 * branches (step2_slicing.hpp:29-38 on llrint(x) when |x| < 9e18, and
 * fmod(rint(x), m) with a Euclidean fix otherwise, :135-155); both are the
 * symmetric representative of the same integer, so one exact formula serves. */
static int8_t oo_symmetric_residue(double x, unsigned m) {
    double r = fmod(x, (double)m);          /* exact, sign of x */
    int ri = (int)r;
    if (ri < 0) ri += (int)m;
    if (ri > (int)(m >> 1)) ri -= (int)m;
    return (int8_t)ri;
}

/* Scheme II slicing (step2_slicing.hpp:211-307): x = rint(ldexp(v, shift)),
 * residue s = x mod m_s (symmetric).  out is [S][rows][cols].  per_row selects
 * whether shifts[] is indexed by row (A) or by column (B). */
void oo_slice2(const double* X, long rows, long cols, const int32_t* shifts, int per_row,
               int S, int8_t* out) {
    const size_t plane = (size_t)rows * cols;
    #pragma omp parallel for schedule(static)
    for (long r = 0; r < rows; ++r) {
        for (long c = 0; c < cols; ++c) {
            size_t idx = (size_t)r * cols + c;
            int sh = per_row ? shifts[r] : shifts[c];
            double x = rint(ldexp(X[idx], sh));
            for (int s = 0; s < S; ++s) out[(size_t)s * plane + idx] = oo_symmetric_residue(x, oo_moduli[s]);
        }
    }
}

/* double -> int8 the way the reference's `static_cast<int8_t>(double)`
 * executes on the GPU (step2_slicing.hpp:66,95): a saturating conversion to
 * int32 (truncation toward zero, NaN -> INT_MIN) whose low byte is kept.  For
 * finite inputs the special values occur only in Scheme I rows whose maximum
 * lies within 2^beta of the subnormal range (0 * inf = NaN -> 0, +inf -> -1,
 * -inf -> 0); every other slice value lies in [-64, 64].  (On an x86 host the
 * same C++ cast is undefined for these values and yields 0.) */
static int8_t oo_cvt_s8(double v) {
    int32_t i;
    if (v != v) i = INT32_MIN;
    else if (v >= 2147483647.0) i = INT32_MAX;
    else if (v <= -2147483648.0) i = INT32_MIN;
    else i = (int32_t)v;
    return (int8_t)(uint8_t)((uint32_t)i & 0xFFu);
}

/* Scheme I slicing (step2_slicing.hpp:44-100): with e = max exponent of the
 * row (A) / column (B), scale = 2^(e+1-beta); for s = 0..S-1,
 * sigma = 0.75*2^(e+1-beta+53-beta*s), a_s = (a + sigma) - sigma,
 * slice = int8(ldexp(a_s * 2^-(e+1-beta), beta*s)), a -= a_s.
 * neg_exp[] holds the shifts of step 1 (offset 0), so e = -neg_exp. */
void oo_slice1(const double* X, long rows, long cols, const int32_t* neg_exp, int per_row,
               int S, int beta, int8_t* out) {
    const size_t plane = (size_t)rows * cols;
    #pragma omp parallel for schedule(static)
    for (long r = 0; r < rows; ++r) {
        for (long c = 0; c < cols; ++c) {
            size_t idx = (size_t)r * cols + c;
            int e = -(per_row ? neg_exp[r] : neg_exp[c]);
            double scale = ldexp(1.0, e + 1 - beta);
            double inv_scale = ldexp(1.0, -(e + 1 - beta));
            double v = X[idx];
            for (int s = 0; s < S; ++s) {
                double sigma = 0.75 * ldexp(scale, 53 - beta * s);
                volatile double t = v + sigma;     /* no reassociation */
                double vs = t - sigma;
                double sl = ldexp(vs * inv_scale, beta * s);
                out[(size_t)s * plane + idx] = oo_cvt_s8(sl);
                v -= vs;
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Step 3: exact INT8 x INT8 -> INT32 GEMM, row-major A (MxK) and B (KxN).    */
/* Restates the product cuBLAS computes in src/cuda/pipeline.cu:117-124 and  */
/* :228-235 (exact while |C| < 2^31).  accumulate != 0 adds into C.          */
/* ------------------------------------------------------------------------- */
void oo_gemm_i8(const int8_t* A, const int8_t* B, long M, long N, long K, int32_t* C, int accumulate) {
    int8_t* Bt = (int8_t*)malloc((size_t)N * K);
    #pragma omp parallel for schedule(static)
    for (long j = 0; j < N; ++j)
        for (long k = 0; k < K; ++k) Bt[(size_t)j * K + k] = B[(size_t)k * N + j];
    #pragma omp parallel for schedule(dynamic, 4)
    for (long i = 0; i < M; ++i) {
        const int8_t* a = A + (size_t)i * K;
        for (long j = 0; j < N; ++j) {
            const int8_t* b = Bt + (size_t)j * K;
            int32_t acc = 0;
            for (long k = 0; k < K; ++k) acc += (int32_t)a[k] * (int32_t)b[k];
            size_t o = (size_t)i * N + j;
            C[o] = accumulate ? (int32_t)((uint32_t)C[o] + (uint32_t)acc) : acc;
        }
    }
    free(Bt);
}

/* ------------------------------------------------------------------------- */
/* Step 4.                                                                   */
/* ------------------------------------------------------------------------- */

/* Scheme II CRT reconstruction (step4_reconstruction.hpp:59-184):
 * c_s = ((C_s mod m_s) * inv_s) mod m_s, acc = sum c_s * M/m_s mod M, signed
 * map at floor(M/2), conversion by the 4-limb sum, scaling by
 * 2^-(shift_A[i] + shift_B[j]).  The 64-bit path the reference takes for
 * S <= 7 gives the same double (acc < 2^63 there, so the limb sum reduces to
 * one uint64 -> double conversion). */
void oo_reconstruct2(const int32_t* Ctc, const int32_t* sA, const int32_t* sB, long M, long N,
                     int S, double* C) {
    uint64_t Mw[4], Mh[4], P[OO_MAX_SLICES][4], I[OO_MAX_SLICES];
    oo_crt_tables(S, Mw, Mh, P, I);
    u256 Mu, Mhu; memcpy(Mu.w, Mw, 32); memcpy(Mhu.w, Mh, 32);
    const size_t plane = (size_t)M * N;
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        for (long j = 0; j < N; ++j) {
            size_t idx = (size_t)i * N + j;
            u256 acc = u256_from(0);
            for (int s = 0; s < S; ++s) {
                int32_t m = (int32_t)oo_moduli[s];
                int32_t rem = Ctc[(size_t)s * plane + idx] % m;
                if (rem < 0) rem += m;
                uint64_t cs = ((uint64_t)rem * I[s]) % (uint64_t)m;
                u256 ps; memcpy(ps.w, P[s], 32);
                acc = u256_add(acc, u256_mul_small(ps, cs));
                if (u256_ge(acc, Mu)) acc = u256_sub(acc, Mu);
            }
            double f;
            if (u256_ge(acc, Mhu)) f = -oo_u256_to_double(u256_sub(Mu, acc));
            else f = oo_u256_to_double(acc);
            C[idx] = ldexp(f, -(sA[i] + sB[j]));
        }
    }
}

/* Scheme I group reconstruction (step4_reconstruction.hpp:21-49):
 * C += double(C_g) * ldexp(2^(e_i+1-beta) * 2^(e_j+1-beta), 2*beta - beta*g).
 * The update is one fused multiply-add, which is what nvcc emits for the
 * reference's `C_out[idx] += val * scale` (the product is a power-of-two
 * scaling of an integer, so it is exact except in the subnormal range). */
void oo_reconstruct1_group(const int32_t* Cg, const int32_t* negA, const int32_t* negB, long M, long N,
                           int g, int beta, double* C) {
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        int ei = -negA[i];
        double ui = ldexp(1.0, ei + 1 - beta);
        for (long j = 0; j < N; ++j) {
            int ej = -negB[j];
            double vj = ldexp(1.0, ej + 1 - beta);
            double scale = ldexp(ui * vj, -beta * g + 2 * beta);
            size_t idx = (size_t)i * N + j;
            C[idx] = fma((double)Cg[idx], scale, C[idx]);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Full pipelines (src/cuda/pipeline.cu:40-167 and :173-265).  Intermediate  */
/* buffers are optional outputs (NULL = internal scratch).  Layouts are the  */
/* reference's: slices [S][rows][cols], C_tc [S][M][N] (Scheme II) and, for  */
/* Scheme I, [S][M][N] with plane g-2 holding group g.                       */
/* ------------------------------------------------------------------------- */
int oo_scheme2_gemm(const double* A, const double* B, long M, long N, long K, int S, double* C,
                    int32_t* shiftA, int32_t* shiftB, int8_t* Asl, int8_t* Bsl, int32_t* Ctc) {
    if (S < 1 || S > OO_MAX_SLICES) return -1;
    int32_t* sA = shiftA ? shiftA : (int32_t*)malloc(sizeof(int32_t) * M);
    int32_t* sB = shiftB ? shiftB : (int32_t*)malloc(sizeof(int32_t) * N);
    int8_t* as = Asl ? Asl : (int8_t*)malloc((size_t)S * M * K);
    int8_t* bs = Bsl ? Bsl : (int8_t*)malloc((size_t)S * K * N);
    int32_t* ct = Ctc ? Ctc : (int32_t*)malloc(sizeof(int32_t) * (size_t)S * M * N);
    int kp = oo_scheme2_kparam(S, K);
    oo_row_shifts(A, M, K, kp, sA);
    oo_col_shifts(B, K, N, kp, sB);
    oo_slice2(A, M, K, sA, 1, S, as);
    oo_slice2(B, K, N, sB, 0, S, bs);
    for (int s = 0; s < S; ++s)
        oo_gemm_i8(as + (size_t)s * M * K, bs + (size_t)s * K * N, M, N, K, ct + (size_t)s * M * N, 0);
    oo_reconstruct2(ct, sA, sB, M, N, S, C);
    if (!shiftA) free(sA);
    if (!shiftB) free(sB);
    if (!Asl) free(as);
    if (!Bsl) free(bs);
    if (!Ctc) free(ct);
    return 0;
}

int oo_scheme1_gemm(const double* A, const double* B, long M, long N, long K, int S, double* C,
                    int32_t* shiftA, int32_t* shiftB, int8_t* Asl, int8_t* Bsl, int32_t* Ctc) {
    if (S < 1) return -1;
    int32_t* sA = shiftA ? shiftA : (int32_t*)malloc(sizeof(int32_t) * M);
    int32_t* sB = shiftB ? shiftB : (int32_t*)malloc(sizeof(int32_t) * N);
    int8_t* as = Asl ? Asl : (int8_t*)malloc((size_t)S * M * K);
    int8_t* bs = Bsl ? Bsl : (int8_t*)malloc((size_t)S * K * N);
    int32_t* ct = Ctc ? Ctc : (int32_t*)malloc(sizeof(int32_t) * (size_t)S * M * N);
    int beta = oo_scheme1_beta(K);
    memset(C, 0, sizeof(double) * (size_t)M * N);
    oo_row_shifts(A, M, K, 0, sA);
    oo_col_shifts(B, K, N, 0, sB);
    oo_slice1(A, M, K, sA, 1, S, beta, as);
    oo_slice1(B, K, N, sB, 0, S, beta, bs);
    for (int g = 2; g <= S + 1; ++g) {
        int32_t* cg = ct + (size_t)(g - 2) * M * N;
        int first = 1;
        for (int s = 1; s <= g - 1; ++s) {
            int t = g - s;
            if (s > S || t > S) continue;
            oo_gemm_i8(as + (size_t)(s - 1) * M * K, bs + (size_t)(t - 1) * K * N, M, N, K, cg, !first);
            first = 0;
        }
        oo_reconstruct1_group(cg, sA, sB, M, N, g, beta, C);
    }
    if (!shiftA) free(sA);
    if (!shiftB) free(sB);
    if (!Asl) free(as);
    if (!Bsl) free(bs);
    if (!Ctc) free(ct);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Accuracy oracles.                                                          */
/* ------------------------------------------------------------------------- */

/* FP128 GEMM, one rounding to double at the end
 * (utils/matrix_reference.hpp:22-50). */
void oo_gemm_fp128(const double* A, const double* B, long M, long N, long K, double* C) {
    double* Bt = (double*)malloc(sizeof(double) * (size_t)N * K);
    #pragma omp parallel for schedule(static)
    for (long j = 0; j < N; ++j)
        for (long k = 0; k < K; ++k) Bt[(size_t)j * K + k] = B[(size_t)k * N + j];
    #pragma omp parallel for schedule(dynamic, 1)
    for (long i = 0; i < M; ++i)
        for (long j = 0; j < N; ++j) {
            __float128 s = 0;
            const double* a = A + (size_t)i * K;
            const double* b = Bt + (size_t)j * K;
            for (long k = 0; k < K; ++k) s += (__float128)a[k] * (__float128)b[k];
            C[(size_t)i * N + j] = (double)s;
        }
    free(Bt);
}

/* FP128 value of selected entries (i[t], j[t]); used for large shapes. */
void oo_gemm_fp128_sampled(const double* A, const double* B, long M, long N, long K,
                           const long* ii, const long* jj, long n, double* out) {
    (void)M;
    #pragma omp parallel for schedule(dynamic, 8)
    for (long t = 0; t < n; ++t) {
        __float128 s = 0;
        for (long k = 0; k < K; ++k) s += (__float128)A[(size_t)ii[t] * K + k] * (__float128)B[(size_t)k * N + jj[t]];
        out[t] = (double)s;
    }
}

/* Double-double GEMM (Dekker/Knuth error-free transformations), rounded to
 * double at the end: about 106-bit accumulation, much faster than FP128. */
void oo_gemm_dd(const double* A, const double* B, long M, long N, long K, double* C) {
    double* Bt = (double*)malloc(sizeof(double) * (size_t)N * K);
    #pragma omp parallel for schedule(static)
    for (long j = 0; j < N; ++j)
        for (long k = 0; k < K; ++k) Bt[(size_t)j * K + k] = B[(size_t)k * N + j];
    #pragma omp parallel for schedule(dynamic, 1)
    for (long i = 0; i < M; ++i)
        for (long j = 0; j < N; ++j) {
            double hi = 0.0, lo = 0.0;
            const double* a = A + (size_t)i * K;
            const double* b = Bt + (size_t)j * K;
            for (long k = 0; k < K; ++k) {
                double p = a[k] * b[k];
                double pe = fma(a[k], b[k], -p);          /* exact product error */
                double s = hi + p;                          /* two-sum */
                double bb = s - hi;
                double se = (hi - (s - bb)) + (p - bb);
                lo += se + pe;
                hi = s;
            }
            C[(size_t)i * N + j] = hi + lo;
        }
    free(Bt);
}

/* Plain FP64 GEMM with k-ordered accumulation (a CPU DGEMM stand-in). */
void oo_gemm_f64(const double* A, const double* B, long M, long N, long K, double* C) {
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        double* c = C + (size_t)i * N;
        for (long j = 0; j < N; ++j) c[j] = 0.0;
        for (long k = 0; k < K; ++k) {
            double a = A[(size_t)i * K + k];
            const double* b = B + (size_t)k * N;
            for (long j = 0; j < N; ++j) c[j] += a * b[j];
        }
    }
}

int oo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
