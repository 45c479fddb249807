// oza_kernels.cu -- sm_100a kernels of the Ozaki Scheme I / II FP64 GEMM.
//
//   step 1  k_stats_rows / k_stats_cols      max frexp exponent per row of A /
//                                            column of B (warp reductions over
//                                            coalesced loads)
//   step 2  k_slice_rows / k_slice_cols      INT8 slices (Scheme I) or symmetric
//                                            residues (Scheme II) written as
//                                            K-major, zero-padded planes
//   step 3  k_gemm_i8                        persistent warp-specialised
//                                            tcgen05 kind::i8 GEMM: TMA ->
//                                            128B-swizzled smem ring -> UMMA ->
//                                            INT32 accumulators in TMEM (double
//                                            buffered) -> epilogue warps
//   step 4  k_reconstruct2 / k_reconstruct1  exact CRT reconstruction (II) and
//                                            scaled group sum (I)
//
// Parity: every stage reproduces the reference pipeline bit for bit
// (src/pipeline/step1_statistics.hpp, step2_slicing.hpp,
// step4_reconstruction.hpp, src/cuda/pipeline.cu of IlyaNyrkov/ozablas); the
// tests compare each intermediate with the CPU oracle.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "oza_device.cuh"
#include "oza_kernels.h"

namespace oza {

__constant__ ModConst c_mod[kMaxSlices];
__constant__ CrtTable c_crt[kMaxSlices];

// The reference's moduli (src/common/crt_tables.hpp:13-16).  The residues are
// only comparable with the same list in the same order.
constexpr uint32_t kModuli[kMaxSlices] = {251, 241, 239, 233, 229, 227, 223, 211, 199, 197,
                                             193, 191, 181, 179, 173, 167, 163, 157, 151, 149};

// 3 M < 2^(32 NL) for the product M of the first S moduli (NL = ceil(S/4)
// 32-bit limbs of M): then T - q M (in [-M/2, 3M/2) for the quotient the CRT
// finish picks), its comparison with floor(M/2) and its correction by M are
// all signed values of NL limbs, so the finish can run on NL limbs, with T
// and q M taken modulo 2^(32 NL).  True for every S except 4 and 8.
__host__ __device__ constexpr bool crt_fits_nl(int S) {
    uint32_t w[6] = {1, 0, 0, 0, 0, 0};
    for (int i = 0; i <= S; ++i) {
        const uint64_t f = i < S ? kModuli[i] : 3u;
        uint64_t c = 0;
        for (int l = 0; l < 6; ++l) {
            const uint64_t v = (uint64_t)w[l] * f + c;
            w[l] = (uint32_t)v;
            c = v >> 32;
        }
    }
    for (int l = (S + 3) / 4; l < 6; ++l)
        if (w[l]) return false;
    return true;
}
static_assert(crt_fits_nl(16) && crt_fits_nl(20) && crt_fits_nl(12) && !crt_fits_nl(8) && !crt_fits_nl(4),
              "limb bound of the CRT finish");

// ---------------------------------------------------------------------------
// Host: constant tables
// ---------------------------------------------------------------------------
namespace {

// Little-endian multiword integer with 32-bit limbs.
struct Big {
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

Big big_from(uint32_t v) {
    Big b;
    b.w[0] = v;
    return b;
}

Big big_mul_small(const Big& a, uint32_t m) {
    Big r;
    uint64_t carry = 0;
    for (int i = 0; i < 8; ++i) {
        uint64_t p = (uint64_t)a.w[i] * m + carry;
        r.w[i] = (uint32_t)p;
        carry = p >> 32;
    }
    return r;
}

uint32_t big_mod_small(const Big& a, uint32_t m) {
    uint64_t rem = 0;
    for (int i = 7; i >= 0; --i) rem = ((rem << 32) | a.w[i]) % m;
    return (uint32_t)rem;
}

int32_t sym_rep(uint32_t r, uint32_t m) { return r > m / 2 ? (int32_t)r - (int32_t)m : (int32_t)r; }

uint32_t pow2_mod(int e, uint32_t m) {
    uint64_t r = 1 % m;
    for (int i = 0; i < e; ++i) r = (r * 2) % m;
    return (uint32_t)r;
}

std::mutex g_table_mu;
uint64_t g_table_done = 0;   // bit per device ordinal

}  // namespace

cudaError_t upload_tables() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_table_mu);
    if (dev < 64 && (g_table_done >> dev) & 1ull) return cudaSuccess;

    static ModConst mc[kMaxSlices];
    static CrtTable ct[kMaxSlices];
    for (int s = 0; s < kMaxSlices; ++s) {
        uint32_t m = kModuli[s];
        mc[s].m = m;
        mc[s].magic = (uint32_t)(((1ull << 39) + m - 1) / m);
        mc[s].c21 = sym_rep(pow2_mod(21, m), m);
        mc[s].c42 = sym_rep(pow2_mod(42, m), m);
        mc[s].c63 = sym_rep(pow2_mod(63, m), m);
        mc[s].magic32 = (uint32_t)(((1ull << 32) + m - 1) / m);
        mc[s].bh = (int32_t)(m * 1024 + (m - 1) / 2);
        mc[s].adj = (int32_t)(256 - (m - 1) / 2);
        mc[s].bhm = (uint32_t)mc[s].bh * mc[s].magic32;
        for (int w = 0; w < 4; ++w) {
            uint32_t word = 0;
            for (int b = 0; b < 4; ++b) {
                const int32_t c = sym_rep(pow2_mod(8 * (4 * w + b), m), m);
                word |= (uint32_t)(uint8_t)(int8_t)c << (8 * b);
            }
            mc[s].dig[w] = word;
        }
    }
    for (int S = 1; S <= kMaxSlices; ++S) {
        CrtTable& t = ct[S - 1];
        Big M = big_from(1);
        for (int i = 0; i < S; ++i) M = big_mul_small(M, kModuli[i]);
        for (int l = 0; l < 5; ++l) {
            t.M[l] = M.w[l];
            t.Mhalf[l] = (M.w[l] >> 1) | (M.w[l + 1] << 31);
        }
        int nl = 1;
        for (int l = 0; l < 5; ++l)
            if (M.w[l]) nl = l + 1;
        t.nlimbs = nl;
        // M / (product of the moduli in `skip`) as limbs
        auto cofactor = [&](std::initializer_list<int> skip, uint32_t (&out)[5]) {
            Big P = big_from(1);
            for (int j = 0; j < S; ++j)
                if (std::find(skip.begin(), skip.end(), j) == skip.end()) P = big_mul_small(P, kModuli[j]);
            for (int l = 0; l < 5; ++l) out[l] = P.w[l];
        };
        for (int i = 0; i < kMaxSlices; ++i) {
            if (i >= S) {
                for (int l = 0; l < 5; ++l) t.P[i][l] = 0;
                t.inv[i] = 0;
                t.c16inv[i] = 0;
                t.rinv[i] = 0.0;
                continue;
            }
            cofactor({i}, t.P[i]);
            Big P;
            for (int l = 0; l < 5; ++l) P.w[l] = t.P[i][l];
            uint32_t m = kModuli[i], r = big_mod_small(P, m), inv = 0;
            for (uint32_t c = 1; c < m; ++c)
                if ((uint64_t)r * c % m == 1) {
                    inv = c;
                    break;
                }
            t.inv[i] = inv;
            t.c16inv[i] = (uint32_t)((65536ull * inv) % m);
            t.rinv[i] = 1.0 / (double)m;
        }
        for (int q = 0; q < kMaxSlices / 3; ++q) {
            const int a = 3 * q, b = a + 1, c = a + 2;
            for (int l = 0; l < 5; ++l) t.TP[q][l] = 0;
            t.tk[q] = t.tab[q] = 0;
            t.trinv[q] = 0.0;
            if (c >= S) continue;
            const uint64_t ma = kModuli[a], mb = kModuli[b], mc = kModuli[c];
            cofactor({a, b, c}, t.TP[q]);
            t.tk[q] = (uint32_t)(mb * mc) | ((uint32_t)(ma * mc) << 16);
            t.tab[q] = (uint32_t)(ma * mb);
            t.trinv[q] = 1.0 / (double)(ma * mb * mc);
        }
        for (int l = 0; l < 5; ++l) t.DP[l] = 0;
        t.drinv = 0.0;
        if (S % 3 == 2) {
            cofactor({S - 2, S - 1}, t.DP);
            t.drinv = 1.0 / (double)((uint64_t)kModuli[S - 2] * kModuli[S - 1]);
        }
    }
    e = cudaMemcpyToSymbol(c_mod, mc, sizeof(mc));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_crt, ct, sizeof(ct));
    if (e != cudaSuccess) return e;
    if (dev < 64) g_table_done |= 1ull << dev;
    return cudaSuccess;
}

PairList make_pairs(int scheme, int slices, size_t K) {
    PairList p{};
    int n = 0, u = 0;
    // Scheme I: pairs per INT32 accumulator, from |slice| <= 2^(beta - 1)
    int per_unit = 1 << 30;
    if (scheme != 2 && K > 0) {
        int beta = (int)std::floor((31.0 - std::log2((double)K)) / 2.0);
        beta = beta < 1 ? 1 : (beta > 7 ? 7 : beta);
        const double bound = (double)K * std::ldexp(1.0, 2 * beta - 2);
        const double fit = std::floor(2147483647.0 / bound);
        per_unit = fit < 1.0 ? 1 : (fit > 1e9 ? 1 << 30 : (int)fit);
    }
    for (int g = 0; g < slices; ++g) {
        p.first_unit[g] = u;
        if (scheme == 2) {
            p.start[u++] = n;
            p.a[n] = (uint8_t)g;
            p.b[n] = (uint8_t)g;
            ++n;
        } else {
            // group g+2 (1-based slices s + t = g + 2), reference pipeline.cu:102-126
            const int G = g + 2;
            int in_unit = 0;
            for (int s = 1; s <= G - 1; ++s) {
                const int t = G - s;
                if (s > slices || t > slices) continue;
                if (in_unit == 0) p.start[u++] = n;
                p.a[n] = (uint8_t)(s - 1);
                p.b[n] = (uint8_t)(t - 1);
                ++n;
                if (++in_unit == per_unit) in_unit = 0;
            }
        }
    }
    p.first_unit[slices] = u;
    p.start[u] = n;
    p.num_groups = u;
    return p;
}

// ---------------------------------------------------------------------------
// Step 1: exponent statistics
// ---------------------------------------------------------------------------
constexpr unsigned long long kMagMask = 0x7FFFFFFFFFFFFFFFull;

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Maximum magnitude bit pattern of one row (one warp, all lanes get it).
__device__ __forceinline__ unsigned long long row_max_bits(const double* row, long long cols, int lane, bool vec2) {
    unsigned long long mx = 0;
    if (vec2) {
        const double2* row2 = reinterpret_cast<const double2*>(row);
        long long n2 = cols >> 1;
        for (long long k = lane; k < n2; k += 32) {
            double2 v = __ldg(row2 + k);
            unsigned long long a = (unsigned long long)__double_as_longlong(v.x) & kMagMask;
            unsigned long long b = (unsigned long long)__double_as_longlong(v.y) & kMagMask;
            mx = a > mx ? a : mx;
            mx = b > mx ? b : mx;
        }
        if ((cols & 1) && lane == 0) {
            unsigned long long a = (unsigned long long)__double_as_longlong(__ldg(row + cols - 1)) & kMagMask;
            mx = a > mx ? a : mx;
        }
    } else {
        for (long long k = lane; k < cols; k += 32) {
            unsigned long long a = (unsigned long long)__double_as_longlong(__ldg(row + k)) & kMagMask;
            mx = a > mx ? a : mx;
        }
    }
    return warp_max_u64(mx);
}

// One warp per row of A: shift[r] = offset - max frexp exponent (-1023 for an
// all-zero row).  Reference: compute_row_shifts_A, step1_statistics.hpp:23-76.
// The maximum exponent is taken from the maximum magnitude bit pattern, which
// orders like |x| for finite doubles.
__global__ void __launch_bounds__(256) k_stats_rows(const double* __restrict__ A, long long rows, long long cols,
                                                    int offset, int32_t* __restrict__ shift, bool vec2) {
    const int lane = threadIdx.x & 31;
    const long long warps_total = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
         r += warps_total) {
        const unsigned long long mx = row_max_bits(A + r * cols, cols, lane, vec2);
        if (lane == 0) shift[r] = offset - max_exp_from_bits(mx);
    }
}

// Column maxima of B (K x N) as magnitude bits, combined with atomicMax into
// colmax[] (zeroed beforehand; 0 encodes an all-zero column).  Block: 8 warps
// over the 64-column strip `strip`, each lane owning 2 adjacent columns; the
// block visits rows y0*8 + warp + i*ystride*8.  Reference:
// compute_col_shifts_B, step1_statistics.hpp:78-99.
__device__ __forceinline__ void stats_cols_block(const double* __restrict__ B, long long rows, long long cols,
                                                 unsigned long long* __restrict__ colmax, long long strip,
                                                 long long y0, long long ystride) {
    __shared__ unsigned long long part[8][64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long c0 = strip * 64 + 2 * lane;
    unsigned long long m0 = 0, m1 = 0;
    for (long long r = y0 * 8 + warp; r < rows; r += ystride * 8) {
        const double* row = B + r * cols;
        if (c0 < cols) {
            unsigned long long a = (unsigned long long)__double_as_longlong(__ldg(row + c0)) & kMagMask;
            m0 = a > m0 ? a : m0;
        }
        if (c0 + 1 < cols) {
            unsigned long long a = (unsigned long long)__double_as_longlong(__ldg(row + c0 + 1)) & kMagMask;
            m1 = a > m1 ? a : m1;
        }
    }
    part[warp][2 * lane] = m0;
    part[warp][2 * lane + 1] = m1;
    __syncthreads();
    if (threadIdx.x < 64) {
        unsigned long long m = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) m = part[w][threadIdx.x] > m ? part[w][threadIdx.x] : m;
        long long c = strip * 64 + threadIdx.x;
        if (c < cols && m != 0) atomicMax(colmax + c, m);
    }
}

__global__ void __launch_bounds__(256) k_stats_cols(const double* __restrict__ B, long long rows, long long cols,
                                                    unsigned long long* __restrict__ colmax) {
    stats_cols_block(B, rows, cols, colmax, blockIdx.x, blockIdx.y, gridDim.y);
}

// Position (row, chunk) of a grid-stride walk over rows x chunks, advanced by
// a fixed stride with one compare instead of a 64-bit division per step.
struct GridWalk {
    long long r, c, dr, dc, chunks;
    __device__ __forceinline__ GridWalk(long long start, long long stride, long long chunks_) : chunks(chunks_) {
        r = start / chunks;
        c = start - r * chunks;
        dr = stride / chunks;
        dc = stride - dr * chunks;
    }
    __device__ __forceinline__ void next() {
        r += dr;
        c += dc;
        if (c >= chunks) {
            c -= chunks;
            ++r;
        }
    }
};

// ---------------------------------------------------------------------------
// Step 2: slicing
// ---------------------------------------------------------------------------

// x * 2^sh exactly as ldexp rounds it.  A multiplication by an exact power of
// two rounds the same way; outside the normal exponent range fall back.
__device__ __forceinline__ double scale_pow2(double x, int sh, double p) {
    return (sh >= -1022 && sh <= 1023) ? x * p : ldexp(x, sh);
}

__device__ __forceinline__ double pow2_or_zero(int sh) {
    return (sh >= -1022 && sh <= 1023) ? __longlong_as_double((long long)(sh + 1023) << 52) : 0.0;
}

// Radix-2^21 digits of the integer-valued double x.  NARROW (|x| <= 2^62, which
// holds whenever K_param <= 62, i.e. always for S <= 16): one conversion to
// int64 and two's-complement digit fields d0, d1 in [0, 2^21), d2 signed.
// WIDE (|x| < 2^84): signed digits peeled off in double precision.
template <bool WIDE>
__device__ __forceinline__ void split21(double x, int& d0, int& d1, int& d2, int& d3) {
    if (!WIDE) {
        const long long t = __double2ll_rn(x);
        d0 = (int)(t & 0x1FFFFF);
        d1 = (int)((t >> 21) & 0x1FFFFF);
        d2 = (int)(t >> 42);
        d3 = 0;
        return;
    }
    double r = x;
    const double q3 = rint(r * 0x1p-63);
    r = r - q3 * 0x1p63;
    const double q2 = rint(r * 0x1p-42);
    r = r - q2 * 0x1p42;
    const double q1 = rint(r * 0x1p-21);
    r = r - q1 * 0x1p21;
    d3 = __double2int_rn(q3);
    d2 = __double2int_rn(q2);
    d1 = __double2int_rn(q1);
    d0 = __double2int_rn(r);
}

// Symmetric residue in [-(m-1)/2, (m-1)/2] of the integer with digits d (radix
// 2^21), modulo c_mod[s].m.  y = sum d_i * (2^(21 i) mod m) stays below 2^29
// in magnitude, the bias m * 2^22 makes it positive and below 2^31, and the
// magic-number division is exact there.  With s known at compile time the
// constants are instruction operands.
template <bool WIDE>
__device__ __forceinline__ int symmetric_residue(int s, int d0, int d1, int d2, int d3) {
    const ModConst& mc = c_mod[s];
    int y = d0 + d1 * mc.c21 + d2 * mc.c42;
    if (WIDE) y += d3 * mc.c63;
    const uint32_t u = (uint32_t)(y + (int)(mc.m << 22));
    const uint32_t r = u - div_small(u, mc.magic) * mc.m;
    return (int)r - ((r > (mc.m >> 1)) ? (int)mc.m : 0);
}

// (a * b) / 2^32 + c in one multiply (PTX mad.hi).
__device__ __forceinline__ uint32_t mulhi_add(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
    return (uint32_t)(a & 0xFF) | ((uint32_t)(b & 0xFF) << 8) | ((uint32_t)(c & 0xFF) << 16) |
           ((uint32_t)(d & 0xFF) << 24);
}

// double -> int8 exactly as the reference's `static_cast<int8_t>(double)`
// behaves on the GPU (step2_slicing.hpp:66,95): a saturating conversion to
// int32 (truncation toward zero, NaN -> INT_MIN) of which the low byte is
// kept.  In-range slice values (|v| <= 64) are unaffected; the special values
// arise only in Scheme I rows whose maximum lies within 2^beta of the
// subnormal range, where 2^-(e+1-beta) overflows to inf: NaN (0 * inf) -> 0,
// +inf -> -1, -inf -> 0.
__device__ __forceinline__ int cvt_s8(double v) {
    return (int)(int8_t)__double2int_rz(v);
}

// Scheme II residues of E (8 or 16) consecutive values: plane s of dst receives
// the E packed residues modulo m_s (reference slice_scheme2_A/B,
// step2_slicing.hpp:110-206: x = rint(ldexp(v, shift)), symmetric residues).
//
// NARROW (K_param <= 62, so |x| <= 2^62): x = sum_{i<8} d_i 256^i with signed
// byte digits d_i = byte_i(x + 0x8080...80) - 128, and
//   u = m 2^10 + (m-1)/2 + sum_i d_i (256^i mod m)       (two dp4a)
// lies in (0, 2^19).  With c = ceil(2^32/m) = (2^32 + e)/m, 0 <= e < m, the low
// word f = u c mod 2^32 equals (u mod m) 2^32/m + u e/m (as u e < 2^32), so
// floor(f m / 2^32) = u mod m exactly: one multiply for f and one mad.hi that
// also adds 256 - (m-1)/2, whose low byte is the symmetric residue (Lemire,
// Kaser and Kurz, "Faster remainder by direct computation", 2019).
// WIDE (|x| < 2^84): radix-2^21 digits and the magic division of
// symmetric_residue.
// Signed byte digits of x = rint(v 2^sh), |x| <= 2^62: x = sum_{i<8} d_i 256^i
// with d_i = byte_i(x + 0x8080...80) - 128, returned as the bytes of
// (x + 0x8080...80) ^ 0x8080...80 read as int8 (low word: d_0..d_3).
__device__ __forceinline__ void byte_digits(double v, int sh, double p, uint32_t& lo, uint32_t& hi) {
    const double x = rint(scale_pow2(v, sh, p));
    const unsigned long long t = (unsigned long long)__double2ll_rn(x);
    const unsigned long long w = (t + 0x8080808080808080ull) ^ 0x8080808080808080ull;
    lo = (uint32_t)w;
    hi = (uint32_t)(w >> 32);
}

// The same digits with no int64 conversion (whose conversion-unit cost bounds
// the tensor-core slicers): for finite v and a normal p = 2^sh with |y| =
// |v p| <= 2^62, y = yh + yl with yh = RN(y + 1.5 2^84) - 1.5 2^84 a multiple
// of 2^32 and yl = y - yh exact in [-2^31, 2^31]; each addition of a
// 1.5 2^k constant rounds an exact sum once, to the integer grid 2^(k-52)
// (round half to even; yh is even in units of 2^32, so rint(y) = yh +
// rint(yl)).  rint(yl) and yh / 2^32 are then the low words of yl + 1.5 2^52
// and yh 2^-32 + 1.5 2^52, the high word of the former giving yl's sign.
// FP64 pipe and integer ALU only; bit-identical to byte_digits there.
__device__ __forceinline__ void byte_digits_fp64(double v, double p, uint32_t& lo, uint32_t& hi) {
    const double y = __dmul_rn(v, p);
    const double yh = __dsub_rn(__dadd_rn(y, 0x1.8p84), 0x1.8p84);
    const double t = __dadd_rn(__dsub_rn(y, yh), 0x1.8p52);
    const double kc = __fma_rn(yh, 0x1p-32, 0x1.8p52);
    const uint32_t xl = (uint32_t)__double2loint(t);
    const uint32_t xh = (uint32_t)__double2loint(kc) + ((uint32_t)__double2hiint(t) - 0x43380000u);
    const unsigned long long x = ((unsigned long long)xh << 32) | xl;
    const unsigned long long w = (x + 0x8080808080808080ull) ^ 0x8080808080808080ull;
    lo = (uint32_t)w;
    hi = (uint32_t)(w >> 32);
}

// Rows / columns whose digits byte_digits_fp64 may form: all entries finite
// (maximum frexp exponent e <= 1024) and 2^sh a normal double.
__device__ __forceinline__ bool fp64_digits_ok(int e, int sh) { return e <= 1024 && sh >= -1022 && sh <= 1023; }

template <int S, bool WIDE, int E>
__device__ __forceinline__ void residuesE(const double (&v)[E], int sh, double p, int8_t* dst, size_t plane_stride) {
    if constexpr (!WIDE) {
        int dlo[E], dhi[E];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            uint32_t lo, hi;
            byte_digits(v[i], sh, p, lo, hi);
            dlo[i] = (int)lo;
            dhi[i] = (int)hi;
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const ModConst& mc = c_mod[s];
            uint32_t r[E];
#pragma unroll
            for (int i = 0; i < E; ++i) {
                const uint32_t u = (uint32_t)__dp4a(dhi[i], (int)mc.dig[1], __dp4a(dlo[i], (int)mc.dig[0], mc.bh));
                r[i] = mulhi_add(u * mc.magic32, mc.m, (uint32_t)mc.adj);
            }
            uint32_t wds[E / 4];
#pragma unroll
            for (int k = 0; k < E / 4; ++k)
                wds[k] = __byte_perm(__byte_perm(r[4 * k], r[4 * k + 1], 0x3340),
                                     __byte_perm(r[4 * k + 2], r[4 * k + 3], 0x3340), 0x5410);
            int8_t* o = dst + (size_t)s * plane_stride;
            if constexpr (E == 16) *reinterpret_cast<uint4*>(o) = make_uint4(wds[0], wds[1], wds[2], wds[3]);
            else *reinterpret_cast<uint2*>(o) = make_uint2(wds[0], wds[1]);
        }
    } else {
    int d0[E], d1[E], d2[E], d3[E];
#pragma unroll
    for (int i = 0; i < E; ++i) {
        const double x = rint(scale_pow2(v[i], sh, p));
        split21<true>(x, d0[i], d1[i], d2[i], d3[i]);
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int r[E];
#pragma unroll
        for (int i = 0; i < E; ++i) r[i] = symmetric_residue<true>(s, d0[i], d1[i], d2[i], d3[i]);
        int8_t* o = dst + (size_t)s * plane_stride;
        if constexpr (E == 16) {
            *reinterpret_cast<uint4*>(o) = make_uint4(pack4(r[0], r[1], r[2], r[3]), pack4(r[4], r[5], r[6], r[7]),
                                                      pack4(r[8], r[9], r[10], r[11]), pack4(r[12], r[13], r[14], r[15]));
        } else {
            *reinterpret_cast<uint2*>(o) = make_uint2(pack4(r[0], r[1], r[2], r[3]), pack4(r[4], r[5], r[6], r[7]));
        }
    }
    }
}

// Scheme I slices of 16 consecutive values of one row/column with max exponent
// e (reference slice_scheme1_A/B, step2_slicing.hpp:44-100).
__device__ __forceinline__ void slices16(const double (&vin)[16], int e, int beta, int S, uint4* dst,
                                         size_t plane_stride) {
    const double scale = ldexp(1.0, e + 1 - beta);
    const double inv_scale = ldexp(1.0, -(e + 1 - beta));
    double v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = vin[i];
    for (int s = 0; s < S; ++s) {
        const double sigma = 0.75 * ldexp(scale, 53 - beta * s);
        const double up = ldexp(1.0, beta * s);   // exact: slice values are small integers
        int r[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            double vs = __dsub_rn(__dadd_rn(v[i], sigma), sigma);
            double sl = __dmul_rn(__dmul_rn(vs, inv_scale), up);
            r[i] = cvt_s8(sl);
            v[i] = __dsub_rn(v[i], vs);
        }
        uint4 o;
        o.x = pack4(r[0], r[1], r[2], r[3]);
        o.y = pack4(r[4], r[5], r[6], r[7]);
        o.z = pack4(r[8], r[9], r[10], r[11]);
        o.w = pack4(r[12], r[13], r[14], r[15]);
        *reinterpret_cast<uint4*>(reinterpret_cast<int8_t*>(dst) + (size_t)s * plane_stride) = o;
    }
}

// An all-zero chunk (tile padding, or zeros in the data) has zero residues
// and zero Scheme I slices in every plane: store zero bytes and skip the
// arithmetic.  -0.0 counts as zero; NaN does not.
template <int E>
__device__ __forceinline__ bool store_if_zero(const double (&v)[E], int planes, int8_t* dst, size_t plane) {
    bool nz = false;
#pragma unroll
    for (int i = 0; i < E; ++i) nz = nz || (v[i] != 0.0);
    if (nz) return false;
    for (int s = 0; s < planes; ++s) {
        if constexpr (E == 16) *reinterpret_cast<uint4*>(dst + (size_t)s * plane) = make_uint4(0, 0, 0, 0);
        else *reinterpret_cast<uint2*>(dst + (size_t)s * plane) = make_uint2(0, 0);
    }
    return true;
}

// A (rows x cols, row-major) -> out[s][rows_p][cols_p].  One thread per E
// consecutive columns of a row (E = 8 for Scheme II, 8-byte stores per plane;
// 16 for Scheme I), coalesced.  Scheme II is instantiated per slice count SC
// (= S); Scheme I takes S at run time.  (r, ch) is the chunk's row and its
// index among the row's cols_p / E chunks.
template <int SCHEME, int SC, bool WIDE>
__device__ __forceinline__ void slice_rows_chunk(const double* __restrict__ A, long long rows, long long cols,
                                                 const int32_t* __restrict__ shift, int S, int beta,
                                                 int8_t* __restrict__ out, long long cols_p, size_t plane,
                                                 long long r, long long ch) {
    constexpr int E = SCHEME == 2 ? 8 : 16;
    const long long c0 = ch * E;
    // Rows past `rows` (tile padding) are not written: the products they feed
    // land in rows of the INT32 / coefficient planes that no later step reads.
    // The K padding of real rows is written as zeros.
    if (r >= rows) return;
    double v[E];
    const int sh = shift[r];
    const double* src = A + r * cols + c0;
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = (c0 + i < cols) ? __ldg(src + i) : 0.0;
    int8_t* dst = out + (size_t)r * cols_p + c0;
    if (store_if_zero<E>(v, SCHEME == 2 ? SC : S, dst, plane)) return;
    if (SCHEME == 2) {
        residuesE<SC, WIDE, E>(v, sh, pow2_or_zero(sh), dst, plane);
    } else {
        slices16(reinterpret_cast<const double(&)[16]>(v), -sh, beta, S, reinterpret_cast<uint4*>(dst), plane);
    }
}

template <int SCHEME, int SC, bool WIDE>
__global__ void __launch_bounds__(256, (SCHEME == 2 ? 3 : 1)) k_slice_rows(
    const double* __restrict__ A, long long rows, long long cols, const int32_t* __restrict__ shift, int S, int beta,
    int8_t* __restrict__ out, long long rows_p, long long cols_p, long long plane_rows) {
    constexpr int E = SCHEME == 2 ? 8 : 16;
    const size_t plane = (size_t)plane_rows * (size_t)cols_p;
    for (GridWalk w((long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, cols_p / E);
         w.r < rows; w.next())
        slice_rows_chunk<SCHEME, SC, WIDE>(A, rows, cols, shift, S, beta, out, cols_p, plane, w.r, w.c);
}

// B (K x N, row-major) -> out[s][Np][Kp], i.e. B^T, K-major.  Tile (bx, by) of
// 128 k x 32 n staged through shared memory; thread (n, kg) emits 16
// consecutive k of column n.  Also writes shift[n] = offset - max exponent of
// column n.
template <int SCHEME, int SC, bool WIDE>
__device__ __forceinline__ void slice_cols_tile(const double* __restrict__ B, long long K, long long N,
                                                const unsigned long long* __restrict__ colmax, int offset, int S,
                                                int beta, int32_t* __restrict__ shift, int8_t* __restrict__ out,
                                                long long Np, long long Kp, long long bx, long long by) {
    __shared__ double tile[128][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long n0 = bx * 32, k0 = by * 128;
    // Rows of B^T past N (tile padding) are not written: their products land in
    // columns of the INT32 / coefficient planes that no later step reads.
    if (n0 >= N) return;   // block-uniform
    // Load: warp w reads rows k0 + w + 8 i, 32 consecutive columns.
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        long long k = k0 + warp + 8 * i, n = n0 + lane;
        tile[warp + 8 * i][lane] = (k < K && n < N) ? __ldg(B + k * N + n) : 0.0;
    }
    __syncthreads();
    const long long n = n0 + lane;
    const int kg = warp;   // 16-row group
    if (n >= N) return;   // no barrier follows
    const int e = max_exp_from_bits(colmax[n]);
    const int sh = offset - e;
    if (by == 0 && kg == 0) shift[n] = sh;
    double v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = tile[kg * 16 + i][lane];
    const size_t plane = (size_t)Np * (size_t)Kp;
    int8_t* dst = out + (size_t)n * Kp + k0 + kg * 16;
    if (store_if_zero<16>(v, SCHEME == 2 ? SC : S, dst, plane)) return;
    if (SCHEME == 2) {
        residuesE<SC, WIDE, 16>(v, sh, pow2_or_zero(sh), dst, plane);
    } else {
        slices16(v, e, beta, S, reinterpret_cast<uint4*>(dst), plane);
    }
}

template <int SCHEME, int SC, bool WIDE>
__global__ void __launch_bounds__(256, (SCHEME == 2 ? 3 : 1)) k_slice_cols(const double* __restrict__ B, long long K, long long N,
                                                    const unsigned long long* __restrict__ colmax, int offset,
                                                    int S, int beta, int32_t* __restrict__ shift,
                                                    int8_t* __restrict__ out, long long Np, long long Kp) {
    slice_cols_tile<SCHEME, SC, WIDE>(B, K, N, colmax, offset, S, beta, shift, out, Np, Kp, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Step 2, Scheme II with S <= 16: digit products on the tensor cores
// ---------------------------------------------------------------------------
// The residue of x = sum_{i<8} d_i 256^i modulo m_s is the direct-remainder
// reduction of u_s = bh_s + sum_i d_i w_{s,i}, w_{s,i} = 256^i mod m_s (int8,
// symmetric), as in residuesE.  The sums over the digits form a small INT8
// matrix product.  Row t of the digit tile holds the 64 digit bytes of 8
// consecutive elements (element e at bytes 8e..8e+7); row 8s + e of the
// weight tile holds w_{s,0..7} at bytes 8e..8e+7 and zeros elsewhere, so
//   D[t][8s + e] = sum_i d_{t,e,i} w_{s,i}      (M = 128, N = 16 ceil(S/2), K = 64)
// comes out of two tcgen05.mma kind::i8 (K = 32 each) into TMEM.  Thread t
// reduces row t (one multiply-add and one mad.hi per residue) and stores 8
// residue bytes per plane.  The two dp4a per residue of the CUDA-core slicer
// move to the tensor pipe; the planes are bit-identical to it.
//
// One thread per tile row: 128 threads, warp w reads TMEM lanes 32w..32w+31;
// 128 TMEM columns per CTA.  Shared memory, 1024-byte aligned: the digit and
// weight tiles (128 rows x 128 B each, 128-byte swizzle, 64 B of each row
// used), then, for the column slicer, a 32-column x 128-k FP64 tile.  A CTA's
// dynamic shared memory (48 KB rows, 66 KB columns) keeps at most 4 (3) CTAs
// on an SM, so their TMEM stays within 512 columns and no allocation waits,
// and a slicer CTA never shares an SM with a GEMM CTA (198 KB).
constexpr int kMsThreads = 128;
constexpr int kMsTile = 128 * 128;   // one SW128 tile of 128 rows
constexpr uint32_t kMsTmemCols = 128;
constexpr int kMsF64Tile = 32 * 1024;
constexpr int kMsRowsSmem = 48 * 1024;
constexpr int kMsColsSmem = 2 * kMsTile + kMsF64Tile + 1024 /*align*/ + 64 /*barrier, slot, flag*/;
constexpr int kMsRowsPerSm = 4;   // CTAs resident per SM: launch bounds and shared memory
constexpr int kMsColsPerSm = 3;
static_assert(2 * kMsTile + 1024 + 64 <= kMsRowsSmem, "row slicer shared memory");
static_assert(5 * (kMsRowsSmem + 1024) > 228 * 1024 && 4 * (kMsColsSmem + 1024) > 228 * 1024,
              "at most 4 (rows) / 3 (columns) slicer CTAs per SM: TMEM 512 columns");

struct MsSmem {
    uint8_t* dig;           // digit tile
    uint8_t* wts;           // weight tile
    uint8_t* f64;           // FP64 tile (column slicer)
    uint64_t* bar;          // MMA completion
    uint32_t* tmem_slot;
    volatile int* abort;
};

__device__ __forceinline__ MsSmem ms_carve(uint8_t* raw, bool with_f64) {
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    MsSmem m;
    m.dig = base;
    m.wts = base + kMsTile;
    m.f64 = base + 2 * kMsTile;
    uint8_t* tail = m.f64 + (with_f64 ? kMsF64Tile : 0);
    m.bar = reinterpret_cast<uint64_t*>(tail);
    m.tmem_slot = reinterpret_cast<uint32_t*>(tail + 8);
    m.abort = reinterpret_cast<volatile int*>(tail + 12);
    return m;
}

// Row `row` of a 128-byte-swizzled tile: 16-byte chunk c at chunk c ^ (row % 8).
__device__ __forceinline__ uint8_t* sw128_row(uint8_t* tile, int row) {
    return tile + (row >> 3) * 1024 + (row & 7) * 128;
}

// Barrier, TMEM columns and the weight tile; returns the TMEM base address.
template <int S>
__device__ __forceinline__ uint32_t ms_setup(const MsSmem& m) {
    const int t = threadIdx.x;
    if (t == 0) {
        mbar_init(m.bar, 1);
        *m.abort = 0;
        fence_barrier_init();
    }
    if (t < 32) {
        tmem_alloc(m.tmem_slot, kMsTmemCols);
        tmem_relinquish();
    }
    const int s = t >> 3, e = t & 7;
    uint32_t lo = 0, hi = 0;
    if (s < S) {
        lo = c_mod[s].dig[0];
        hi = c_mod[s].dig[1];
    }
    uint8_t* row = sw128_row(m.wts, t);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (c == (e >> 1)) {
            if (e & 1) v.z = lo, v.w = hi;
            else v.x = lo, v.y = hi;
        }
        *reinterpret_cast<uint4*>(row + ((c ^ (t & 7)) << 4)) = v;
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *m.tmem_slot;
}

__device__ __forceinline__ void ms_put_digits(uint8_t* dig, int t, const uint32_t (&lo)[8], const uint32_t (&hi)[8]) {
    uint8_t* row = sw128_row(dig, t);
#pragma unroll
    for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(row + ((c ^ (t & 7)) << 4)) =
            make_uint4(lo[2 * c], hi[2 * c], lo[2 * c + 1], hi[2 * c + 1]);
}

// Thread 0 issues D = digits x weights^T (two K = 32 steps) and commits to
// the barrier; every warp then waits for it (bounded).  False if the wait gave up.
template <int S>
__device__ __forceinline__ bool ms_mma(const MsSmem& m, uint32_t tmem, uint32_t phase, int* err) {
    constexpr uint32_t idesc = umma_idesc_i8(128, 16 * ((S + 1) / 2));
    if (threadIdx.x == 0) {
        tc_fence_after();
        const uint64_t ad = umma_desc_sw128(smem_u32(m.dig));
        const uint64_t bd = umma_desc_sw128(smem_u32(m.wts));
        umma_i8(tmem, ad, bd, idesc, 0);
        umma_i8(tmem, ad + 2, bd + 2, idesc, 1);   // +32 bytes of K
        umma_commit(m.bar);
    }
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait(m.bar, phase, m.abort, err);
    ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
    tc_fence_after();
    return ok != 0;
}

// Residues of this thread's 8 elements from TMEM (column 8s + e holds
// u_s(e) - bh_s); stored (when `live`) as 8 bytes per plane at dst + s plane.
// Warp-collective: every lane calls it.
template <int S>
__device__ __forceinline__ void ms_store(uint32_t taddr, int8_t* dst, size_t plane, bool live) {
#pragma unroll
    for (int ch = 0; ch < (S + 3) / 4; ++ch) {
        uint32_t v[32];
        tmem_ld32(taddr + 32 * ch, v);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int s = 4 * ch + j;
            if (s < S) {
                const ModConst& mc = c_mod[s];
                uint32_t r[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) r[e] = mulhi_add(v[8 * j + e] * mc.magic32 + mc.bhm, mc.m, (uint32_t)mc.adj);
                const uint32_t w0 =
                    __byte_perm(__byte_perm(r[0], r[1], 0x3340), __byte_perm(r[2], r[3], 0x3340), 0x5410);
                const uint32_t w1 =
                    __byte_perm(__byte_perm(r[4], r[5], 0x3340), __byte_perm(r[6], r[7], 0x3340), 0x5410);
                if (live) *reinterpret_cast<uint2*>(dst + (size_t)s * plane) = make_uint2(w0, w1);
            }
        }
    }
}

// After the last round: if a wait gave up, let the pending MMA finish
// (bounded) before the TMEM columns are released.
__device__ __forceinline__ void ms_teardown(const MsSmem& m, uint32_t tmem, uint32_t pending_phase) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *m.abort) {
        volatile int no_abort = 0;
        mbar_wait(m.bar, pending_phase, &no_abort, nullptr);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, kMsTmemCols);
    }
}

// A (rows x cols, row-major) -> out[s][plane_rows][cols_p]: a grid-stride walk
// over (row, octet of columns), 128 octets per round.  Rows past `rows` are
// not written, the K padding of real rows is written as zeros (as k_slice_rows).
template <int S>
__global__ void __launch_bounds__(kMsThreads, kMsRowsPerSm)
    k_slice_rows_mma(const double* __restrict__ A, long long rows, long long cols, const int32_t* __restrict__ shift,
                     int offset, int8_t* __restrict__ out, long long cols_p, long long plane_rows, int* err) {
    extern __shared__ uint8_t ms_raw[];
    const MsSmem m = ms_carve(ms_raw, false);
    const uint32_t tmem = ms_setup<S>(m);
    const int t = threadIdx.x;
    const uint32_t taddr = tmem + ((uint32_t)(t & ~31) << 16);
    const size_t plane = (size_t)plane_rows * (size_t)cols_p;
    const long long octs = cols_p >> 3, total = rows * octs, stride = (long long)gridDim.x * kMsThreads;
    GridWalk w((long long)blockIdx.x * kMsThreads + t, stride, octs);
    // The octet of the next round is loaded while this round's MMA and
    // reduction run (one round ahead).
    double v[8];
    int sh = 0;
    auto fetch = [&](const GridWalk& at) {
        if (at.r < rows) {
            sh = shift[at.r];
            const long long c0 = at.c * 8;
            const double* src = A + at.r * cols + c0;
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = (c0 + i < cols) ? __ldg(src + i) : 0.0;
        } else {
            sh = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = 0.0;
        }
    };
    fetch(w);
    uint32_t phase = 0;
    bool ok = true;
    for (long long base = (long long)blockIdx.x * kMsThreads; base < total; base += stride) {
        const bool live = w.r < rows;
        int8_t* dst = out + w.r * cols_p + w.c * 8;
        uint32_t lo[8], hi[8];
        const double p = pow2_or_zero(sh);
        if (fp64_digits_ok(offset - sh, sh)) {
#pragma unroll
            for (int i = 0; i < 8; ++i) byte_digits_fp64(v[i], p, lo[i], hi[i]);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) byte_digits(v[i], sh, p, lo[i], hi[i]);
        }
        ms_put_digits(m.dig, t, lo, hi);
        w.next();
        fetch(w);
        fence_proxy_async_smem();
        tc_fence_before();
        if (!__syncthreads_and(ok)) break;
        ok = ms_mma<S>(m, tmem, phase, err);
        if (ok) ms_store<S>(taddr, dst, plane, live);
        phase ^= 1;
    }
    ms_teardown(m, tmem, phase ^ 1);
}

// B (K x N, row-major) -> out[s][Np][Kp] (B^T, K-major), and shift[n] =
// offset - max exponent of column n, as k_slice_cols.  Persistent over tiles
// of 128 k x 32 n: the tile is staged through shared memory (coalesced rows
// of B in, columns out), then 4 rounds in which thread t takes column
// 8q + t/16 of the tile and its k-octet t % 16, so a plane's stores are 128
// contiguous bytes per half-warp.  FP64 tile layout: column j is a 1 KB row of
// 64 16-byte chunks (k pairs), logical chunk L stored at L ^ ((L/8 ^ j) % 8),
// which keeps both the column-wise stores and the k-wise reads within 2x of
// conflict-free.
template <int S>
__global__ void __launch_bounds__(kMsThreads, kMsColsPerSm)
    k_slice_cols_mma(const double* __restrict__ B, long long K, long long N,
                     const unsigned long long* __restrict__ colmax, int offset, int32_t* __restrict__ shift,
                     int8_t* __restrict__ out, long long Np, long long Kp, int* err) {
    extern __shared__ uint8_t ms_raw[];
    const MsSmem m = ms_carve(ms_raw, true);
    const uint32_t tmem = ms_setup<S>(m);
    const int t = threadIdx.x;
    const uint32_t taddr = tmem + ((uint32_t)(t & ~31) << 16);
    const size_t plane = (size_t)Np * (size_t)Kp;
    const long long tn = (N + 31) / 32, tiles = tn * (Kp / 128);
    const int jl = t & 31, kl = t >> 5;   // staging: column jl, tile rows kl + 4i
    const int o = t & 15;                 // rounds: k-octet
    uint32_t phase = 0;
    bool ok = true;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long by = tile / tn, bx = tile - by * tn;
        const long long n0 = bx * 32, k0 = by * 128;
        if (!__syncthreads_and(ok)) break;   // also: the previous tile's reads of the FP64 tile are done
        {
            const long long n = n0 + jl;
            uint8_t* rowp = m.f64 + jl * 1024;
#pragma unroll 8
            for (int i = 0; i < 32; ++i) {
                const int kk = kl + 4 * i;
                const long long k = k0 + kk;
                const double x = (k < K && n < N) ? __ldg(B + k * N + n) : 0.0;
                const int L = kk >> 1;
                *reinterpret_cast<double*>(rowp + ((L ^ (((L >> 3) ^ jl) & 7)) << 4) + ((kk & 1) << 3)) = x;
            }
        }
        __syncthreads();
        for (int q = 0; q < 4; ++q) {
            const int j = 8 * q + (t >> 4);
            const long long n = n0 + j;
            const bool live = n < N;
            int sh = 0, e = 0;
            if (live) {
                e = max_exp_from_bits(colmax[n]);
                sh = offset - e;
                if (by == 0 && o == 0) shift[n] = sh;
            }
            const double p = pow2_or_zero(sh);
            const uint8_t* rowp = m.f64 + j * 1024;
            double x[8];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int L = 4 * o + c;
                const double2 d = *reinterpret_cast<const double2*>(rowp + ((L ^ (((L >> 3) ^ j) & 7)) << 4));
                x[2 * c] = d.x;
                x[2 * c + 1] = d.y;
            }
            uint32_t lo[8], hi[8];
            if (fp64_digits_ok(e, sh)) {
#pragma unroll
                for (int i = 0; i < 8; ++i) byte_digits_fp64(x[i], p, lo[i], hi[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) byte_digits(x[i], sh, p, lo[i], hi[i]);
            }
            ms_put_digits(m.dig, t, lo, hi);
            fence_proxy_async_smem();
            tc_fence_before();
            if (!__syncthreads_and(ok)) break;
            ok = ms_mma<S>(m, tmem, phase, err);
            if (ok) ms_store<S>(taddr, out + n * Kp + k0 + 8 * o, plane, live);
            phase ^= 1;
        }
    }
    ms_teardown(m, tmem, phase ^ 1);
}

// ---------------------------------------------------------------------------
// Exact CRT arithmetic (Scheme II step 4), shared by the fused GEMM epilogue
// and the standalone reconstruction kernel
// ---------------------------------------------------------------------------

// (C * inv_s) mod m_s in [0, m_s) for any int32 C: C = hi * 2^16 + lo,
// y = hi * ((2^16 inv) mod m) + lo * inv + m * 2^16 lies in (0, 2^31).
__device__ __forceinline__ uint32_t crt_coeff(int32_t C, uint32_t m, uint32_t magic, uint32_t inv,
                                              uint32_t c16inv) {
    const int hi = C >> 16;
    const int lo = C & 0xFFFF;
    const uint32_t u = (uint32_t)(hi * (int)c16inv + lo * (int)inv + (int)(m << 16));
    return u - div_small(u, magic) * m;
}

// Running state of one element: T = sum c_s * (M / m_s) as NL 64-bit column
// sums of 32-bit limb products (each product below 2^58, at most 20 of them),
// and an FP64 estimate of T / M: the sum of d / P over the terms d * (M / P)
// added, each d converted exactly (d < 2^32) and multiplied by 1 / P rounded
// to double.  T / M < S <= 20, so each of the at most 20 fused multiply-adds
// rounds by at most 2^-49, and the reciprocals' relative error of 2^-53 adds
// at most 20 * 2^-53: the estimate is within 2^-44 of T / M.  It runs on the
// FP64 pipe, beside the integer multiplies of the limbs.
template <int NL>
struct CrtAcc {
    unsigned long long a[NL];
    double q;
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int l = 0; l < NL; ++l) a[l] = 0ull;
        q = 0.0;
    }
    // d * W where W = M / P for the product P of the moduli d stands for, rinv = 1 / P
    __device__ __forceinline__ void add(const uint32_t (&W)[5], double rinv, uint32_t d) {
#pragma unroll
        for (int l = 0; l < NL; ++l) a[l] += (unsigned long long)d * W[l];
        // 2^52 + d exactly, minus 2^52: d as a double without a conversion instruction
        const double dd = __hiloint2double(0x43300000, (int)d) - 0x1p52;
        q = fma(dd, rinv, q);
    }
    // one residue s with coefficient c < m_s
    __device__ __forceinline__ void add(const CrtTable& T, int s, uint32_t c) { add(T.P[s], T.rinv[s], c); }
};

// r = x - y over N 32-bit limbs.  The whole borrow chain is one asm block: the
// carry flag does not survive between separate asm statements (the compiler
// may schedule its own carry-using adds in between).
template <int N>
__device__ __forceinline__ void mw_sub(uint32_t (&r)[N], const uint32_t (&x)[N], const uint32_t (&y)[N]);

template <>
__device__ __forceinline__ void mw_sub<1>(uint32_t (&r)[1], const uint32_t (&x)[1], const uint32_t (&y)[1]) {
    r[0] = x[0] - y[0];
}

template <>
__device__ __forceinline__ void mw_sub<2>(uint32_t (&r)[2], const uint32_t (&x)[2], const uint32_t (&y)[2]) {
    asm("sub.cc.u32 %0, %2, %4; subc.u32 %1, %3, %5;" : "=&r"(r[0]),"=&r"(r[1]) : "r"(x[0]),"r"(x[1]),"r"(y[0]),"r"(y[1]));
}

template <>
__device__ __forceinline__ void mw_sub<3>(uint32_t (&r)[3], const uint32_t (&x)[3], const uint32_t (&y)[3]) {
    asm("sub.cc.u32 %0, %3, %6; subc.cc.u32 %1, %4, %7; subc.u32 %2, %5, %8;" : "=&r"(r[0]),"=&r"(r[1]),"=&r"(r[2]) : "r"(x[0]),"r"(x[1]),"r"(x[2]),"r"(y[0]),"r"(y[1]),"r"(y[2]));
}

template <>
__device__ __forceinline__ void mw_sub<4>(uint32_t (&r)[4], const uint32_t (&x)[4], const uint32_t (&y)[4]) {
    asm("sub.cc.u32 %0, %4, %8; subc.cc.u32 %1, %5, %9; subc.cc.u32 %2, %6, %10; subc.u32 %3, %7, %11;" : "=&r"(r[0]),"=&r"(r[1]),"=&r"(r[2]),"=&r"(r[3]) : "r"(x[0]),"r"(x[1]),"r"(x[2]),"r"(x[3]),"r"(y[0]),"r"(y[1]),"r"(y[2]),"r"(y[3]));
}

template <>
__device__ __forceinline__ void mw_sub<5>(uint32_t (&r)[5], const uint32_t (&x)[5], const uint32_t (&y)[5]) {
    asm("sub.cc.u32 %0, %5, %10; subc.cc.u32 %1, %6, %11; subc.cc.u32 %2, %7, %12; subc.cc.u32 %3, %8, %13; subc.u32 %4, %9, %14;" : "=&r"(r[0]),"=&r"(r[1]),"=&r"(r[2]),"=&r"(r[3]),"=&r"(r[4]) : "r"(x[0]),"r"(x[1]),"r"(x[2]),"r"(x[3]),"r"(x[4]),"r"(y[0]),"r"(y[1]),"r"(y[2]),"r"(y[3]),"r"(y[4]));
}

template <>
__device__ __forceinline__ void mw_sub<6>(uint32_t (&r)[6], const uint32_t (&x)[6], const uint32_t (&y)[6]) {
    asm("sub.cc.u32 %0, %6, %12; subc.cc.u32 %1, %7, %13; subc.cc.u32 %2, %8, %14; subc.cc.u32 %3, %9, %15; subc.cc.u32 %4, %10, %16; subc.u32 %5, %11, %17;" : "=&r"(r[0]),"=&r"(r[1]),"=&r"(r[2]),"=&r"(r[3]),"=&r"(r[4]),"=&r"(r[5]) : "r"(x[0]),"r"(x[1]),"r"(x[2]),"r"(x[3]),"r"(x[4]),"r"(x[5]),"r"(y[0]),"r"(y[1]),"r"(y[2]),"r"(y[3]),"r"(y[4]),"r"(y[5]));
}

// x = T mod M mapped to [-(floor(M/2)+1), floor(M/2)) -- the reference's signed
// map at floor(M/2) -- then its magnitude converted as the reference does,
// d0 + d1 2^64 + d2 2^128 over 64-bit limbs with a rounding after each
// addition (crt_math.hpp:73-80), sign applied, scaled by 2^-esum
// (step4_reconstruction.hpp:59-184).
// FIT (crt_fits_nl(S)): the arithmetic runs on NL limbs, T and q M modulo
// 2^(32 NL); otherwise on NL + 1.  The same bits either way.
template <int NL, bool FIT = false>
__device__ __forceinline__ double crt_finish(const CrtTable& T, const CrtAcc<NL>& acc, int esum) {
    constexpr int L = FIT ? NL : NL + 1;
    uint32_t t[L];
    unsigned long long carry = 0;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        const unsigned long long v = acc.a[l] + carry;
        t[l] = (uint32_t)v;
        carry = v >> 32;
    }
    if constexpr (L > NL) t[NL] = (uint32_t)carry;
    // nearest quotient: with the estimate within 2^-44 of T / M,
    // floor(estimate + 1/2 - 2^-40) is q* or q* - 1, so V = T - q M is either
    // the answer or the answer + M (then V >= floor(M/2)).
    const uint32_t q = __double2uint_rz(acc.q + (0.5 - 0x1p-40));
    uint32_t qm[L];
    {
        unsigned long long c = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const unsigned long long v = (unsigned long long)q * (l < NL ? T.M[l] : 0u) + c;
            qm[l] = (uint32_t)v;
            c = v >> 32;
        }
    }
    uint32_t v[L], d[L], mh[L], m[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
        mh[l] = l < NL ? T.Mhalf[l] : 0u;
        m[l] = l < NL ? T.M[l] : 0u;
    }
    mw_sub<L>(v, t, qm);
    mw_sub<L>(d, v, mh);
    if ((int)d[L - 1] >= 0) {      // V >= floor(M/2): one M too many
        uint32_t w[L];
        mw_sub<L>(w, v, m);
#pragma unroll
        for (int l = 0; l < L; ++l) v[l] = w[l];
    }
    const bool neg = (int)v[L - 1] < 0;
    if (neg) {
        uint32_t z[L];
#pragma unroll
        for (int l = 0; l < L; ++l) z[l] = 0u;
        uint32_t w[L];
        mw_sub<L>(w, z, v);
#pragma unroll
        for (int l = 0; l < L; ++l) v[l] = w[l];
    }
    unsigned long long w0 = v[0];
    if constexpr (NL > 1) w0 |= (unsigned long long)v[1] << 32;
    double mag = __ull2double_rn(w0);
    if constexpr (NL > 2) {
        unsigned long long w1 = v[2];
        if constexpr (NL > 3) w1 |= (unsigned long long)v[3] << 32;
        mag = __dadd_rn(mag, __ull2double_rn(w1) * 0x1p64);
    }
    if constexpr (NL > 4) mag = __dadd_rn(mag, __ull2double_rn((unsigned long long)v[4]) * 0x1p128);
    const int e = -esum;
    return scale_pow2(neg ? -mag : mag, e, pow2_or_zero(e));
}

// ---------------------------------------------------------------------------
// Step 3: tcgen05 INT8 GEMM
// ---------------------------------------------------------------------------
// One persistent CTA per SM walks work units (group g, output tile 128 x 256)
// in group-major order, round-robin over CTAs (Scheme II: residue g,
// A_g * B_g^T; Scheme I: the slice pairs with s + t = g + 2).  Each unit
// accumulates into one of two TMEM accumulators, so the epilogue of one unit
// overlaps the MMAs of the next.  Group-major order keeps the CTAs on the
// same pair of planes at a time (L2-resident); a tile-major order made them
// drift across all S planes and re-read them from HBM (4.6x at 8192^3, S=16).
//   warp 0      TMA producer (4-stage ring of A 128x128 + B^T 256x128 int8 tiles)
//   warp 1      TMEM allocation, UMMA issue (one elected lane)
//   warps 2..   epilogue, EW warps; warp w reads TMEM lanes 32 (w % 4).. (its
//               lane quadrant): with EW = 4 all the tile's columns, with EW = 8
//               the column half (w - 2) / 4.  Four warps measured 1-2%
//               faster at large K (the epilogue hides behind a unit's MMAs);
//               units of few k-blocks, where the epilogue is the longer side,
//               take eight.
// Epilogues: kEpiI32 writes the INT32 group planes; kEpiCoef (Scheme II)
// reduces each residue product to its one-byte CRT coefficient and writes the
// byte planes, which k_crt_coef turns into FP64 C (a quarter of the INT32
// traffic, and the multiword CRT runs at full occupancy instead of in the
// epilogue warps, where it would stall the MMA pipeline).
template <int EW>
constexpr int gemm_threads() { return 64 + 32 * EW; }
// Units with fewer k-blocks of MMAs than this get 8 epilogue warps.
constexpr int kEpi8Below = 8;
constexpr int kStages = 4;
constexpr int kABytes = kTileM * kTileK;   // 16 KB per stage
constexpr int kBBytes = kTileN * kTileK;   // 32 KB per stage
constexpr uint32_t kAccCols = 256;         // TMEM column stride between the two accumulators
constexpr uint32_t kTmemCols = 2 * kAccCols;
constexpr int kEpiChunks = kTileN / 32;    // 32-column TMEM loads per tile row
static_assert(kTileN % 32 == 0 && kTileN <= (int)kAccCols, "tile width: a multiple of 32, at most 256");
constexpr int kGemmSmem = kStages * (kABytes + kBBytes) + 1024 /*align*/ + 256 /*barriers*/;
constexpr int kEpiI32 = 0;
constexpr int kEpiCoef = 1;

struct GemmArgs {
    int m_tiles, n_tiles, k_blocks, total_tiles, groups;
    int mt0;                      // first m-tile (row-chunked calls)
    uint32_t wait_hint;           // mbarrier suspend-time hint in ns (0: poll)
    int band;                     // m-tiles per rasterisation band
    long long Mp, Np;
    long long M, N;               // real extents (the epilogue skips padding)
    int* err;
    int32_t* ctc;                 // kEpiI32: [groups][Mp][Np]
    uint8_t* coef;                // kEpiCoef: [S][Mp][Np] CRT coefficient bytes
    int S;
};

// Tile t -> (mt, nt).  Tiles are walked in bands of `band` m-tiles, n-major
// inside a band, so the ~148 tiles in flight at once cover a band x (148/band)
// block: band * 1 MB of A and 148/band * 2 MB of B^T at K = 8192.
__device__ __forceinline__ void tile_coords(int t, const GemmArgs& a, int& mt, int& nt) {
    const int per_band = a.band * a.n_tiles;
    const int b = t / per_band;
    const int tb = t - b * per_band;
    const int rows = min(a.band, a.m_tiles - b * a.band);
    nt = tb / rows;
    mt = a.mt0 + b * a.band + (tb - nt * rows);
}

// One work unit's epilogue for one warp: 32 TMEM lanes (rows) x the 32-column
// chunks [c0, c1) of the accumulator at taddr, of output tile column nt.
template <int EPI>
__device__ __forceinline__ void epilogue_unit(int32_t* ctc, uint8_t* coef, long long Mp, long long Np, int S,
                                              uint32_t taddr, long long row, int grp, int nt, int c0, int c1) {
    if (EPI == kEpiI32) {
        int32_t* dst = ctc + (size_t)grp * Mp * Np + (size_t)row * Np + (size_t)nt * kTileN;
#pragma unroll 1
        for (int c = c0; c < c1; ++c) {
            uint32_t r[32];
            tmem_ld32(taddr + c * 32, r);
            tmem_ld_wait();
            int4* d4 = reinterpret_cast<int4*>(dst + c * 32);
#pragma unroll
            for (int v = 0; v < 8; ++v)
                d4[v] = make_int4((int)r[4 * v], (int)r[4 * v + 1], (int)r[4 * v + 2], (int)r[4 * v + 3]);
        }
    } else {
        // Scheme II: reduce each INT32 residue product to its CRT
        // coefficient ((C mod m_g) * inv_g) mod m_g, one byte.
        const ModConst mc = c_mod[grp];
        const uint32_t inv = c_crt[S - 1].inv[grp], c16 = c_crt[S - 1].c16inv[grp];
        uint8_t* dst = coef + (size_t)grp * Mp * Np + (size_t)row * Np + (size_t)nt * kTileN;
#pragma unroll 1
        for (int c = c0; c < c1; ++c) {
            uint32_t r[32];
            tmem_ld32(taddr + c * 32, r);
            tmem_ld_wait();
            uint32_t wds[8];
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                uint32_t b0 = crt_coeff((int32_t)r[4 * v], mc.m, mc.magic, inv, c16);
                uint32_t b1 = crt_coeff((int32_t)r[4 * v + 1], mc.m, mc.magic, inv, c16);
                uint32_t b2 = crt_coeff((int32_t)r[4 * v + 2], mc.m, mc.magic, inv, c16);
                uint32_t b3 = crt_coeff((int32_t)r[4 * v + 3], mc.m, mc.magic, inv, c16);
                wds[v] = b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
            }
            uint4* d4 = reinterpret_cast<uint4*>(dst + c * 32);
            d4[0] = make_uint4(wds[0], wds[1], wds[2], wds[3]);
            d4[1] = make_uint4(wds[4], wds[5], wds[6], wds[7]);
        }
    }
}

// One work unit of the one-CTA GEMM: output tile (mt, nt) of INT32 group grp,
// the sum over pairs [p0, p1) of A-plane x B-plane products over k_blocks.
struct GemmUnit {
    const CUtensorMap* tmA;
    const CUtensorMap* tmB;
    int p0, p1, grp, mt, nt, k_blocks, S;
    long long Mp, Np;
    long long M, N;               // real extents: padding rows and columns are never read
    int32_t* ctc;
    uint8_t* coef;
};

// Work units of one GEMM: group-major, tiles rasterised in bands.
struct SingleUnits {
    const CUtensorMap* tmA;
    const CUtensorMap* tmB;
    const PairList* pairs;
    const GemmArgs* a;
    __device__ __forceinline__ int count() const { return a->groups * a->total_tiles; }
    __device__ __forceinline__ void get(int u, GemmUnit& x) const {
        x.grp = u / a->total_tiles;
        tile_coords(u - x.grp * a->total_tiles, *a, x.mt, x.nt);
        x.tmA = tmA;
        x.tmB = tmB;
        x.p0 = pairs->start[x.grp];
        x.p1 = pairs->start[x.grp + 1];
        x.k_blocks = a->k_blocks;
        x.S = a->S;
        x.Mp = a->Mp;
        x.Np = a->Np;
        x.M = a->M;
        x.N = a->N;
        x.ctc = a->ctc;
        x.coef = a->coef;
    }
    __device__ __forceinline__ int a_plane(int p) const { return pairs->a[p]; }
    __device__ __forceinline__ int b_plane(int p) const { return pairs->b[p]; }
};

// Work units of a group of independent Scheme II GEMMs: an explicit list of
// (problem, mt, nt, modulus), one tensor-map pair and one coefficient buffer
// per problem.
struct GroupGemmProblem {
    long long Mp, Np, M, N;
    int k_blocks, S;
    uint8_t* coef;
};
struct GroupGemmArgs {
    const int4* units;
    int total_units;
    uint32_t wait_hint;
    const CUtensorMap* maps;   // [2 * problems]: A planes, then B^T planes
    const GroupGemmProblem* probs;
    int* err;
};
struct GroupUnits {
    const GroupGemmArgs* g;
    __device__ __forceinline__ int count() const { return g->total_units; }
    __device__ __forceinline__ void get(int u, GemmUnit& x) const {
        const int4 w = g->units[u];
        const GroupGemmProblem& pr = g->probs[w.x];
        x.tmA = g->maps + 2 * w.x;
        x.tmB = g->maps + 2 * w.x + 1;
        x.mt = w.y;
        x.nt = w.z;
        x.grp = w.w;
        x.p0 = w.w;
        x.p1 = w.w + 1;
        x.k_blocks = pr.k_blocks;
        x.S = pr.S;
        x.Mp = pr.Mp;
        x.Np = pr.Np;
        x.M = pr.M;
        x.N = pr.N;
        x.ctc = nullptr;
        x.coef = pr.coef;
    }
    __device__ __forceinline__ int a_plane(int p) const { return p; }
    __device__ __forceinline__ int b_plane(int p) const { return p; }
};

// Persistent, warp-specialised INT8 GEMM on one SM per CTA: warp 0 issues
// TMA loads into a kStages ring, warp 1 issues tcgen05 MMAs into one of two
// TMEM accumulators, warps 2-9 drain the other accumulator through the
// epilogue.  CTA c takes units c, c + grid, ...  Every wait is bounded.
template <int EPI, int EW, class Units>
__device__ __forceinline__ void gemm_i8_body(const Units& src, int* err, uint32_t hint) {
    static_assert(EW == 4 || EW == 8, "4 or 8 epilogue warps");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + kStages * kABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kStages * kBBytes);
    uint64_t* empty = full + kStages;
    uint64_t* acc_full = empty + kStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&acc_full[0], 1);
        mbar_init(&acc_full[1], 1);
        mbar_init(&acc_empty[0], EW);
        mbar_init(&acc_empty[1], EW);
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int total_units = src.count();

    if (warp == 0) {
        // ---------------- TMA producer (one lane) ----------------
        // The whole role runs in lane 0: no per-k-block reconvergence of the
        // warp, which would stall the issue stream between stages.
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            long long issued = 0;
            bool ok = true;
            const CUtensorMap* last_map = nullptr;
            for (int u = blockIdx.x; u < total_units && ok; u += gridDim.x) {
                GemmUnit x;
                src.get(u, x);
                if (x.tmA != last_map) {
                    tma_prefetch_desc(x.tmA);
                    tma_prefetch_desc(x.tmB);
                    last_map = x.tmA;
                }
                for (int p = x.p0; p < x.p1 && ok; ++p) {
                    const int arow = (int)(src.a_plane(p) * x.Mp + (long long)x.mt * kTileM);
                    const int brow = (int)(src.b_plane(p) * x.Np + (long long)x.nt * kTileN);
                    for (int kb = 0; kb < x.k_blocks; ++kb) {
                        if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, err, hint)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[stage], kABytes + kBBytes);
                        tma_load_2d(sA + stage * kABytes, x.tmA, &full[stage], kb * kTileK, arow);
                        tma_load_2d(sB + stage * kBBytes, x.tmB, &full[stage], kb * kTileK, brow);
                        ++issued;
                        if (++stage == kStages) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
            }
            if (!ok) {
                // Let the copies already issued land before the CTA leaves.
                long long n = issued < kStages ? issued : kStages;
                volatile int no_abort = 0;
                for (long long j = 0; j < n; ++j) {
                    long long idx = issued - 1 - j;
                    mbar_wait(&full[idx % kStages], (uint32_t)((idx / kStages) & 1), &no_abort, nullptr);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer (one lane) ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = umma_idesc_i8(kTileM, kTileN);
            int stage = 0;
            uint32_t phase = 0;
            int local = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < total_units && ok; u += gridDim.x, ++local) {
                GemmUnit x;
                src.get(u, x);
                const int acc = local & 1;
                const uint32_t acc_phase = (local >> 1) & 1;
                if (!mbar_wait(&acc_empty[acc], acc_phase ^ 1, abort_flag, err, hint)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem_base + acc * kAccCols;
                uint32_t accumulate = 0;
                for (int p = x.p0; p < x.p1 && ok; ++p) {
                    for (int kb = 0; kb < x.k_blocks; ++kb) {
                        if (!mbar_wait(&full[stage], phase, abort_flag, err, hint)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint64_t ad = umma_desc_sw128(smem_u32(sA + stage * kABytes));
                        const uint64_t bd = umma_desc_sw128(smem_u32(sB + stage * kBBytes));
#pragma unroll
                        for (int k = 0; k < kTileK / 32; ++k) {
                            // +32 bytes of K inside the swizzle row = +2 in 16-byte units
                            umma_i8(d, ad + 2 * k, bd + 2 * k, idesc, accumulate);
                            accumulate = 1;
                        }
                        umma_commit(&empty[stage]);
                        if (++stage == kStages) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                }
                if (!ok) break;
                umma_commit(&acc_full[acc]);
            }
            if (!ok) {
                // Wait for the MMAs already issued before TMEM is released.
                umma_commit(drain);
                volatile int no_abort = 0;
                mbar_wait(drain, 0, &no_abort, nullptr);
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        const int q = warp & 3;                 // TMEM lane quadrant this warp may access
        // 32-column chunks of this warp: all of them (4 warps) or one half (8 warps)
        const int half = (warp - 2) >> 2;
        const int c0 = EW == 8 ? half * ((kEpiChunks + 1) / 2) : 0;
        const int c1 = EW == 8 ? (half ? kEpiChunks : (kEpiChunks + 1) / 2) : kEpiChunks;
        const int row_local = q * 32 + lane;
        int local = 0;
        bool ok = true;
        for (int u = blockIdx.x; u < total_units && ok; u += gridDim.x, ++local) {
            GemmUnit x;
            src.get(u, x);
            const long long row = (long long)x.mt * kTileM + row_local;
            const int acc = local & 1;
            const uint32_t acc_phase = (local >> 1) & 1;
            int w = 1;
            if (lane == 0) w = mbar_wait(&acc_full[acc], acc_phase, abort_flag, err, hint);
            if (__shfl_sync(0xFFFFFFFFu, w, 0) == 0) {
                ok = false;
                continue;
            }
            tc_fence_after();
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + acc * kAccCols;
            // Skip this warp's quadrant when all its rows are tile padding, and
            // the 32-column chunks past N: no later step reads those entries.
            const long long cols_left = x.N - (long long)x.nt * kTileN;
            int ce = c1;
            if (cols_left < (long long)c1 * 32) ce = (int)((cols_left + 31) / 32);
            if ((long long)x.mt * kTileM + q * 32 >= x.M) ce = c0;
            if (ce > c0) epilogue_unit<EPI>(x.ctc, x.coef, x.Mp, x.Np, x.S, taddr, row, x.grp, x.nt, c0, ce);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[acc]);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, kTmemCols);
    }
}

template <int EPI, int EW>
__global__ void __launch_bounds__(gemm_threads<EW>(), 1)
    k_gemm_i8(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const __grid_constant__ PairList pairs, const __grid_constant__ GemmArgs args) {
    const SingleUnits src{&tmA, &tmB, &pairs, &args};
    gemm_i8_body<EPI, EW>(src, args.err, args.wait_hint);
}

// Grouped Scheme II GEMM over an explicit unit list (coefficient epilogue).
// Grouped problems are mostly of small K: eight epilogue warps.
__global__ void __launch_bounds__(gemm_threads<8>(), 1) k_group_gemm_i8(const __grid_constant__ GroupGemmArgs g) {
    const GroupUnits src{&g};
    gemm_i8_body<kEpiCoef, 8>(src, g.err, g.wait_hint);
}

// ---------------------------------------------------------------------------
// Step 4: reconstruction
// ---------------------------------------------------------------------------

// Scheme II step 4 from the coefficient byte planes [S][Mp][Np] written by the
// GEMM epilogue: one thread per 4 consecutive columns of a row (a warp reads
// 128 contiguous bytes per plane), exact CRT per element, FP64 C.  Residues
// are combined three at a time (CrtTable): the bytes of moduli a and b are
// interleaved with one byte permute per 2 elements and weighted by m_b m_c and
// m_a m_c in one dp2a; c_c m_a m_b is its accumulator.  With S fixed at
// compile time the table constants are instruction operands and the S loads
// are issued together.
template <int S>
__device__ __forceinline__ void crt_coef_chunk(const uint8_t* __restrict__ coef, long long Np, long long N,
                                               size_t plane, const int32_t* __restrict__ sA,
                                               const int32_t* __restrict__ sB, double* __restrict__ C,
                                               long long i, long long ch) {
    constexpr int NL = (S + 3) / 4;   // 32-bit limbs of M
    constexpr int NT = S / 3;         // residue triples
    const CrtTable& T = c_crt[S - 1];
    const long long j0 = ch << 2;
    const uint8_t* src = coef + (size_t)i * Np + j0;
    uint32_t w[S];
#pragma unroll
    for (int s = 0; s < S; ++s) w[s] = __ldg(reinterpret_cast<const uint32_t*>(src + (size_t)s * plane));
    CrtAcc<NL> st[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) st[e].zero();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const uint32_t wa = w[3 * t], wb = w[3 * t + 1], wc = w[3 * t + 2];
        const uint32_t x01 = __byte_perm(wa, wb, 0x5140);   // c_a0 c_b0 c_a1 c_b1
        const uint32_t x23 = __byte_perm(wa, wb, 0x7362);   // c_a2 c_b2 c_a3 c_b3
        const uint32_t k = T.tk[t], kab = T.tab[t];
        const uint32_t d0 = __dp2a_lo(k, x01, __byte_perm(wc, 0, 0x4440) * kab);
        const uint32_t d1 = __dp2a_hi(k, x01, __byte_perm(wc, 0, 0x4441) * kab);
        const uint32_t d2 = __dp2a_lo(k, x23, __byte_perm(wc, 0, 0x4442) * kab);
        const uint32_t d3 = __dp2a_hi(k, x23, __byte_perm(wc, 0, 0x4443) * kab);
        st[0].add(T.TP[t], T.trinv[t], d0);
        st[1].add(T.TP[t], T.trinv[t], d1);
        st[2].add(T.TP[t], T.trinv[t], d2);
        st[3].add(T.TP[t], T.trinv[t], d3);
    }
    if constexpr (S % 3 == 2) {
        const uint32_t ma = c_mod[S - 2].m, mb = c_mod[S - 1].m;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t d = ((w[S - 2] >> (8 * e)) & 0xFFu) * mb + ((w[S - 1] >> (8 * e)) & 0xFFu) * ma;
            st[e].add(T.DP, T.drinv, d);
        }
    } else if constexpr (S % 3 == 1) {
#pragma unroll
        for (int e = 0; e < 4; ++e) st[e].add(T, S - 1, (w[S - 1] >> (8 * e)) & 0xFFu);
    }
    const int sa = sA[i];
    double* crow = C + i * N;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const long long j = j0 + e;
        if (j < N) crow[j] = crt_finish<NL, crt_fits_nl(S)>(T, st[e], sa + sB[j]);
    }
}

template <int S>
__global__ void __launch_bounds__(128) k_crt_coef(const uint8_t* __restrict__ coef, long long Mp, long long Np,
                                                  long long M, long long N, const int32_t* __restrict__ sA,
                                                  const int32_t* __restrict__ sB, double* __restrict__ C) {
    const size_t plane = (size_t)Mp * (size_t)Np;
    for (GridWalk w((long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, (N + 3) >> 2);
         w.r < M; w.next())
        crt_coef_chunk<S>(coef, Np, N, plane, sA, sB, C, w.r, w.c);
}

template <int NL>
__global__ void __launch_bounds__(256) k_reconstruct2(const int32_t* __restrict__ ctc, long long Mp, long long Np,
                                                      long long M, long long N, int S,
                                                      const int32_t* __restrict__ sA,
                                                      const int32_t* __restrict__ sB, double* __restrict__ C) {
    const long long total = M * N;
    const size_t plane = (size_t)Mp * (size_t)Np;
    const CrtTable& T = c_crt[S - 1];
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const long long i = id / N, j = id - i * N;
        const int32_t* src = ctc + (size_t)i * Np + j;
        CrtAcc<NL> st;
        st.zero();
        for (int s = 0; s < S; ++s) {
            const uint32_t c = crt_coeff(__ldg(src + (size_t)s * plane), c_mod[s].m, c_mod[s].magic, T.inv[s],
                                         T.c16inv[s]);
            st.add(T, s, c);
        }
        C[id] = crt_finish<NL>(T, st, sA[i] + sB[j]);
    }
}

// Scheme I: C = sum over g = 2..S+1 (in that order) of double(C_g) * scale_g,
// each update one fused multiply-add from +0.0, which is the sequence of the
// reference's per-group launches (step4_reconstruction.hpp:21-49,
// pipeline.cu:102-135 after the memset at pipeline.cu:72).  scale_g is
// ldexp(u_i v_j, 2 beta - beta g) with u_i v_j an exact power of two (or 0 /
// inf at the exponent extremes); where u_i v_j is normal and the result stays
// normal that is the product with the exact power 2^(2 beta - beta g), and
// ldexp itself is called otherwise.  One thread per 4 consecutive columns of
// a row: one 16-byte load per group plane (all S issued together, S fixed at
// compile time), the scale exponents and powers computed once per row and
// column, 4 results per thread.
// ldexp for the rare scales that leave the normal range (kept out of line).
__device__ __noinline__ double ldexp_outlined(double x, int k) { return ldexp(x, k); }

template <int S>
__device__ __forceinline__ void reconstruct1_chunk(const int32_t* __restrict__ ctc, long long Np, long long N,
                                                   size_t plane, int beta, const int32_t* __restrict__ negA,
                                                   const int32_t* __restrict__ negB, double* __restrict__ C,
                                                   long long i, long long ch) {
    constexpr int kBatch = 4;   // group planes loaded together
    const long long j0 = ch << 2;
    const int4* src = reinterpret_cast<const int4*>(ctc + (size_t)i * Np + j0);
    const size_t plane4 = plane >> 2;
    int4 v[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch && b < S; ++b) v[b] = __ldg(src + b * plane4);
    const double ui = ldexp(1.0, -negA[i] + 1 - beta);
    double uv[4];
    int lim[4];   // smallest scale exponent k with uv * 2^k still normal (INT_MAX: never)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const long long j = j0 + e;
        uv[e] = __dmul_rn(ui, ldexp(1.0, (j < N ? -negB[j] : 0) + 1 - beta));
        const int E = (int)((unsigned long long)__double_as_longlong(uv[e]) >> 52) & 0x7FF;
        lim[e] = (E == 0 || E == 0x7FF) ? 0x7FFFFFFF : -1022 - (E - 1023);
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int g0 = 0; g0 < S; g0 += kBatch) {
        int4 nv[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b)
            if (g0 + kBatch + b < S) nv[b] = __ldg(src + (g0 + kBatch + b) * plane4);
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const int g = g0 + b;
            if (g >= S) break;
            const int k = -beta * g;   // 2 beta - beta (g + 2): plane g holds group g + 2
            const double p = __longlong_as_double((long long)(k + 1023) << 52);   // k in [-1022, 0]
            const int val[4] = {v[b].x, v[b].y, v[b].z, v[b].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double scale = k >= lim[e] ? __dmul_rn(uv[e], p) : ldexp_outlined(uv[e], k);
                acc[e] = __fma_rn((double)val[e], scale, acc[e]);
            }
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b)
            if (g0 + kBatch + b < S) v[b] = nv[b];
    }
    double* crow = C + i * N;
#pragma unroll
    for (int e = 0; e < 4; ++e)
        if (j0 + e < N) crow[j0 + e] = acc[e];
}

template <int S>
__global__ void __launch_bounds__(256) k_reconstruct1(const int32_t* __restrict__ ctc, long long Mp, long long Np,
                                                      long long M, long long N, int beta,
                                                      const int32_t* __restrict__ negA,
                                                      const int32_t* __restrict__ negB, double* __restrict__ C) {
    const size_t plane = (size_t)Mp * (size_t)Np;
    for (GridWalk w((long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, (N + 3) >> 2);
         w.r < M; w.next())
        reconstruct1_chunk<S>(ctc, Np, N, plane, beta, negA, negB, C, w.r, w.c);
}

// Scheme I step 4 where some groups were split over several INT32 planes
// (large K: make_pairs): group g's value is the exact sum of its planes
// [first[g], first[g + 1]), formed in 64 bits -- equal to the reference's
// INT32 group sum wherever that one does not overflow -- then the same
// scaled fused multiply-add in g order as k_reconstruct1.
struct UnitMap {
    int first[kMaxSlicesHost + 1];
};
__global__ void __launch_bounds__(256) k_reconstruct1_units(const int32_t* __restrict__ ctc, long long Mp,
                                                            long long Np, long long M, long long N, int S, int beta,
                                                            const int32_t* __restrict__ negA,
                                                            const int32_t* __restrict__ negB,
                                                            double* __restrict__ C, const __grid_constant__ UnitMap um) {
    const size_t plane4 = ((size_t)Mp * (size_t)Np) >> 2;
    for (GridWalk w((long long)blockIdx.x * blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x, (N + 3) >> 2);
         w.r < M; w.next()) {
        const long long i = w.r, j0 = w.c << 2;
        const int4* src = reinterpret_cast<const int4*>(ctc + (size_t)i * Np + j0);
        const double ui = ldexp(1.0, -negA[i] + 1 - beta);
        double uv[4], acc[4] = {0.0, 0.0, 0.0, 0.0};
        int lim[4];
        for (int e = 0; e < 4; ++e) {
            const long long j = j0 + e;
            uv[e] = __dmul_rn(ui, ldexp(1.0, (j < N ? -negB[j] : 0) + 1 - beta));
            const int E = (int)((unsigned long long)__double_as_longlong(uv[e]) >> 52) & 0x7FF;
            lim[e] = (E == 0 || E == 0x7FF) ? 0x7FFFFFFF : -1022 - (E - 1023);
        }
        for (int g = 0; g < S; ++g) {
            long long sum[4] = {0, 0, 0, 0};
            for (int u = um.first[g]; u < um.first[g + 1]; ++u) {
                const int4 v = __ldg(src + (size_t)u * plane4);
                sum[0] += v.x;
                sum[1] += v.y;
                sum[2] += v.z;
                sum[3] += v.w;
            }
            const int k = -beta * g;
            const double p = __longlong_as_double((long long)(k + 1023) << 52);
            for (int e = 0; e < 4; ++e) {
                const double scale = k >= lim[e] ? __dmul_rn(uv[e], p) : ldexp_outlined(uv[e], k);
                acc[e] = __fma_rn((double)sum[e], scale, acc[e]);
            }
        }
        double* crow = C + i * N;
        for (int e = 0; e < 4; ++e)
            if (j0 + e < N) crow[j0 + e] = acc[e];
    }
}

// Sum of planes [first, first + count) of ctc (Mp x Np) into dst (M x N,
// row-major), in two's-complement 32-bit arithmetic: the INT32 buffer the
// reference's consecutive GEMMs with beta = 1 leave.
__global__ void __launch_bounds__(256) k_sum_planes(const int32_t* __restrict__ ctc, long long Mp, long long Np,
                                                    long long M, long long N, int first, int count,
                                                    int32_t* __restrict__ dst) {
    const size_t plane = (size_t)Mp * (size_t)Np;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M * N;
         id += (long long)gridDim.x * blockDim.x) {
        const long long i = id / N, j = id - i * N;
        uint32_t s = 0;
        for (int u = first; u < first + count; ++u) s += (uint32_t)ctc[(size_t)u * plane + (size_t)i * Np + j];
        dst[id] = (int32_t)s;
    }
}

// ---------------------------------------------------------------------------
// Grouped Scheme II: steps 1, 2 and 4 of many independent GEMMs, one launch
// per stage (per slice-count class for the templated stages).  Block b of a
// launch works on problem ids[q] for start[q] <= b < start[q + 1], at local
// tile b - start[q]; the bodies are the single-GEMM kernels' own.
// ---------------------------------------------------------------------------
// Work per block of the grouped slicers: 4 chunks per thread (rows) and 2
// k-tiles per block (columns), so the block-to-problem search and the
// problem loads are amortised and loads of one chunk overlap the next.
constexpr int kGroupRowChunks = 4;
constexpr int kGroupColTiles = 2;

struct GroupProblemDev {
    const double* A;
    const double* B;
    double* C;
    long long M, N, K, Mp, Np, Kp;
    int S, k_param;
    int32_t* shiftA;
    int32_t* shiftB;
    unsigned long long* colmax;
    int8_t* a_planes;
    int8_t* b_planes;
    uint8_t* coef;
};

struct GroupLaunchDev {
    const int* ids;
    const long long* start;   // n + 1 entries
    int n;
};

// Largest q with start[q] <= b (block-uniform).
__device__ __forceinline__ int group_find(const GroupLaunchDev& L, long long b) {
    int lo = 0, hi = L.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(L.start + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// 8 rows per block, one warp per row.
__global__ void __launch_bounds__(256) k_group_stats_rows(const GroupProblemDev* __restrict__ probs,
                                                          const __grid_constant__ GroupLaunchDev L) {
    const int q = group_find(L, blockIdx.x);
    const GroupProblemDev& P = probs[L.ids[q]];
    const long long r = (blockIdx.x - L.start[q]) * 8 + (threadIdx.x >> 5);
    if (r >= P.M) return;
    const bool vec2 = ((reinterpret_cast<uintptr_t>(P.A) & 15) == 0) && (P.K % 2 == 0);
    const unsigned long long mx = row_max_bits(P.A + r * P.K, P.K, threadIdx.x & 31, vec2);
    if ((threadIdx.x & 31) == 0) P.shiftA[r] = P.k_param - max_exp_from_bits(mx);
}

// Tile (strip, y0) of ceil(N/64) x ceil(K/256) per problem.
__global__ void __launch_bounds__(256) k_group_stats_cols(const GroupProblemDev* __restrict__ probs,
                                                          const __grid_constant__ GroupLaunchDev L) {
    const int q = group_find(L, blockIdx.x);
    const GroupProblemDev& P = probs[L.ids[q]];
    const long long t = blockIdx.x - L.start[q];
    const long long strips = (P.N + 63) / 64, ny = (P.K + 255) / 256;
    stats_cols_block(P.B, P.K, P.N, P.colmax, t % strips, t / strips, ny);
}

// 256 chunks of 8 columns per block over the padded Mp x Kp.
template <int SC, bool WIDE>
__global__ void __launch_bounds__(256, 3) k_group_slice_rows(const GroupProblemDev* __restrict__ probs,
                                                             const __grid_constant__ GroupLaunchDev L) {
    const int q = group_find(L, blockIdx.x);
    const GroupProblemDev& P = probs[L.ids[q]];
    const long long total = P.M * (P.Kp / 8);   // real rows only (see slice_rows_chunk)
    const long long base = (blockIdx.x - L.start[q]) * (256 * kGroupRowChunks) + threadIdx.x;
#pragma unroll 1
    for (int r = 0; r < kGroupRowChunks; ++r) {
        const long long id = base + r * 256;
        if (id >= total) return;
        const long long cpr = P.Kp / 8;
        slice_rows_chunk<2, SC, WIDE>(P.A, P.M, P.K, P.shiftA, SC, 0, P.a_planes, P.Kp,
                                      (size_t)P.Mp * (size_t)P.Kp, id / cpr, id % cpr);
    }
}

// Tile (bx, by) of (Np/32) x (Kp/128) per problem.
template <int SC, bool WIDE>
__global__ void __launch_bounds__(256, 3) k_group_slice_cols(const GroupProblemDev* __restrict__ probs,
                                                             const __grid_constant__ GroupLaunchDev L) {
    const int q = group_find(L, blockIdx.x);
    const GroupProblemDev& P = probs[L.ids[q]];
    const long long t = blockIdx.x - L.start[q];
    const long long nx = (P.N + 31) / 32, ny = P.Kp / 128;   // real columns only (see slice_cols_tile)
#pragma unroll 1
    for (int r = 0; r < kGroupColTiles; ++r) {
        const long long by = (t / nx) * kGroupColTiles + r;
        if (by >= ny) return;   // block-uniform
        if (r) __syncthreads();  // the shared tile is reloaded
        slice_cols_tile<2, SC, WIDE>(P.B, P.K, P.N, P.colmax, P.k_param, SC, 0, P.shiftB, P.b_planes, P.Np, P.Kp,
                                     t % nx, by);
    }
}

// 256 chunks of 4 columns per block over M x N.
template <int S>
__global__ void __launch_bounds__(256) k_group_crt(const GroupProblemDev* __restrict__ probs,
                                                   const __grid_constant__ GroupLaunchDev L) {
    const int q = group_find(L, blockIdx.x);
    const GroupProblemDev& P = probs[L.ids[q]];
    const long long chunks = (P.N + 3) >> 2;
    const long long id = (blockIdx.x - L.start[q]) * 256 + threadIdx.x;
    if (id >= P.M * chunks) return;
    crt_coef_chunk<S>(P.coef, P.Np, P.N, (size_t)P.Mp * (size_t)P.Np, P.shiftA, P.shiftB, P.C, id / chunks,
                      id % chunks);
}

// ---------------------------------------------------------------------------
// Reference-layout copies of the intermediates (inspection mode only)
// ---------------------------------------------------------------------------
// B^T planes [S][Np][Kp] (K-major) -> the reference's B slices [S][K][N]
// (row-major, unpadded): 32 x 32 byte tiles through shared memory.
__global__ void __launch_bounds__(256) k_planes_to_kn(const int8_t* __restrict__ src, long long Np, long long Kp,
                                                      long long K, long long N, int8_t* __restrict__ dst) {
    __shared__ int8_t tile[32][33];
    const long long s = blockIdx.z;
    const long long n0 = (long long)blockIdx.x * 32, k0 = (long long)blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
    const int8_t* sp = src + (size_t)s * Np * Kp;
    int8_t* dp = dst + (size_t)s * K * N;
#pragma unroll
    for (int r = ty; r < 32; r += 8) {
        const long long n = n0 + r, k = k0 + tx;
        tile[r][tx] = (n < N && k < K) ? sp[(size_t)n * Kp + k] : 0;
    }
    __syncthreads();
#pragma unroll
    for (int r = ty; r < 32; r += 8) {
        const long long k = k0 + r, n = n0 + tx;
        if (k < K && n < N) dp[(size_t)k * N + n] = tile[tx][r];
    }
}

// ---------------------------------------------------------------------------
// Self-test of the bounded waits: thread 0 waits, through the same mbar_wait
// as the GEMM kernels, for a phase of an mbarrier that nothing arrives on.
// The wait gives up after limit_ns, raises the abort flag and writes the
// error code into *gerr; *status = 1 if the wait had (wrongly) succeeded.
// ---------------------------------------------------------------------------
__global__ void k_wait_probe(int* gerr, unsigned long long limit_ns, int* status) {
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) *status = mbar_wait(&bar, 0, &abort_flag, gerr, 0, limit_ns) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
namespace {

int grid_for(long long work, int per_block, int sms, int waves = 8) {
    long long b = (work + per_block - 1) / per_block;
    long long cap = (long long)sms * waves;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// K-major int8 planes [rows][Kp] as a 2D tensor with a (128 x box_rows) box
// and the 128-byte swizzle the UMMA descriptors expect.
bool make_plane_map(CUtensorMap* map, const int8_t* base, size_t rows, size_t Kp, int box_rows) {
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)Kp};
    cuuint32_t box[2] = {(cuuint32_t)kTileK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

cudaError_t launch_stats_rows(const double* A, size_t rows, size_t cols, int offset, int32_t* shift, int sms,
                              cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    bool vec2 = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (cols % 2 == 0);
    int grid = grid_for((long long)rows, 8, sms);
    k_stats_rows<<<grid, 256, 0, st>>>(A, (long long)rows, (long long)cols, offset, shift, vec2);
    return cudaGetLastError();
}

cudaError_t launch_stats_cols(const double* B, size_t rows, size_t cols, unsigned long long* colmax, int sms,
                              cudaStream_t st) {
    if (cols == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(colmax, 0, cols * sizeof(unsigned long long), st);
    if (e != cudaSuccess || rows == 0) return e;
    int gx = (int)((cols + 63) / 64);
    long long want = (long long)sms * 4 / gx;
    long long maxy = ((long long)rows + 63) / 64;
    int gy = (int)(want < 1 ? 1 : (want > maxy ? maxy : want));
    if (gy < 1) gy = 1;
    k_stats_cols<<<dim3(gx, gy), 256, 0, st>>>(B, (long long)rows, (long long)cols, colmax);
    return cudaGetLastError();
}

// Scheme II slicers are instantiated per slice count; WIDE digit splitting is
// needed only when K_param > 62, which requires S >= 17.
#define OZA_FOR_EACH_S(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) \
    X(16) X(17) X(18) X(19) X(20)

namespace {
int g_residue_slicer = 0;   // 0: tensor cores for kMmaSlicerMinS <= S <= 16, 1: CUDA cores only, 2: tensor cores for S <= 16
// Smallest S at which the default takes the tensor-core slicers.  Step 2 at
// 8192^3 / 4096^3 (ms, tensor / dp4a): S = 4 0.505 / 0.394, S = 8 0.712 /
// 0.714, S = 12 0.880 / 0.890, S = 16 1.109 / 1.197; at S = 2 (4096^3)
// 0.132 / 0.085.  Each MMA round has a fixed cost that a few moduli do not
// amortise.
constexpr int kMmaSlicerMinS = 12;
bool use_mma_slicer(int S) {
    return S <= 16 && (g_residue_slicer == 2 || (g_residue_slicer == 0 && S >= kMmaSlicerMinS));
}

template <int S>
cudaError_t launch_rows_mma(const double* A, long long R, long long C, const int32_t* shift, int offset, int8_t* out,
                            long long CP, long long PR, int sms, int* err, cudaStream_t st) {
    const long long rounds = (R * (CP / 8) + kMsThreads - 1) / kMsThreads;
    const long long cap = (long long)sms * kMsRowsPerSm;
    const int grid = (int)(rounds < cap ? rounds : cap);
    k_slice_rows_mma<S><<<grid, kMsThreads, kMsRowsSmem, st>>>(A, R, C, shift, offset, out, CP, PR, err);
    return cudaGetLastError();
}

template <int S>
cudaError_t launch_cols_mma(const double* B, long long K, long long N, const unsigned long long* colmax, int offset,
                            int32_t* shift, int8_t* out, long long Np, long long Kp, int* err, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_slice_cols_mma<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMsColsSmem);
    });
    if (attr != cudaSuccess) return attr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (N + 31) / 32 * (Kp / 128);
    const long long cap = (long long)sms * kMsColsPerSm;
    const int grid = (int)(tiles < cap ? tiles : cap);
    k_slice_cols_mma<S><<<grid, kMsThreads, kMsColsSmem, st>>>(B, K, N, colmax, offset, shift, out, Np, Kp, err);
    return cudaGetLastError();
}

#define OZA_FOR_EACH_S16(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)
}  // namespace

void set_residue_slicer(int mode) { g_residue_slicer = mode; }
int residue_slicer() { return g_residue_slicer; }

cudaError_t launch_slice_rows(int scheme, const double* A, size_t rows, size_t cols, const int32_t* shift, int S,
                              int beta, int k_param, int8_t* out, size_t rows_p, size_t cols_p, int sms,
                              cudaStream_t st, size_t plane_rows, int* err) {
    long long chunks = (long long)rows * (long long)(cols_p / (scheme == 2 ? 8 : 16));
    if (chunks == 0) return cudaSuccess;
    const int grid = grid_for(chunks, 256, sms);
    const long long R = (long long)rows, C = (long long)cols, RP = (long long)rows_p, CP = (long long)cols_p;
    const long long PR = plane_rows ? (long long)plane_rows : RP;
    if (scheme == 2 && k_param <= 62 && err && use_mma_slicer(S)) {
        switch (S) {
#define OZA_CASE(n) \
    case n: return launch_rows_mma<n>(A, R, C, shift, k_param, out, CP, PR, sms, err, st);
            OZA_FOR_EACH_S16(OZA_CASE)
#undef OZA_CASE
            default: return cudaErrorInvalidValue;
        }
    }
    if (scheme == 1) {
        k_slice_rows<1, 0, false><<<grid, 256, 0, st>>>(A, R, C, shift, S, beta, out, RP, CP, PR);
        return cudaGetLastError();
    }
    const bool wide = k_param > 62;
    if (wide && S < 17) return cudaErrorInvalidValue;   // K_param <= 61 for S <= 16
    switch (S) {
#define OZA_CASE(n)                                                                                   \
    case n:                                                                                           \
        if (wide) k_slice_rows<2, n, (n >= 17)><<<grid, 256, 0, st>>>(A, R, C, shift, n, 0, out, RP, CP, PR); \
        else k_slice_rows<2, n, false><<<grid, 256, 0, st>>>(A, R, C, shift, n, 0, out, RP, CP, PR);         \
        break;
        OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_slice_cols(int scheme, const double* B, size_t K, size_t N, const unsigned long long* colmax,
                              int offset, int S, int beta, int32_t* shift, int8_t* out, size_t Np, size_t Kp,
                              cudaStream_t st, int* err) {
    if (N == 0 || Kp == 0) return cudaSuccess;
    if (N > Np) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)((N + 31) / 32), (unsigned)(Kp / 128));
    const long long KK = (long long)K, NN = (long long)N, NP = (long long)Np, KP = (long long)Kp;
    if (scheme == 2 && offset <= 62 && err && use_mma_slicer(S)) {
        switch (S) {
#define OZA_CASE(n) \
    case n: return launch_cols_mma<n>(B, KK, NN, colmax, offset, shift, out, NP, KP, err, st);
            OZA_FOR_EACH_S16(OZA_CASE)
#undef OZA_CASE
            default: return cudaErrorInvalidValue;
        }
    }
    if (scheme == 1) {
        k_slice_cols<1, 0, false><<<grid, 256, 0, st>>>(B, KK, NN, colmax, offset, S, beta, shift, out, NP, KP);
        return cudaGetLastError();
    }
    const bool wide = offset > 62;
    if (wide && S < 17) return cudaErrorInvalidValue;
    switch (S) {
#define OZA_CASE(n)                                                                                          \
    case n:                                                                                                  \
        if (wide) k_slice_cols<2, n, (n >= 17)><<<grid, 256, 0, st>>>(B, KK, NN, colmax, offset, n, 0, shift, out, NP, KP); \
        else k_slice_cols<2, n, false><<<grid, 256, 0, st>>>(B, KK, NN, colmax, offset, n, 0, shift, out, NP, KP);         \
        break;
        OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int EPI, int EW>
static cudaError_t gemm_launch(const CUtensorMap& tmA, const CUtensorMap& tmB, const PairList& pairs,
                               const GemmArgs& a, int grid, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_gemm_i8<EPI, EW>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    });
    if (attr != cudaSuccess) return attr;
    k_gemm_i8<EPI, EW><<<grid, gemm_threads<EW>(), kGemmSmem, st>>>(tmA, tmB, pairs, a);
    return cudaGetLastError();
}

cudaError_t launch_gemm_i8(const GemmPlan& p, cudaStream_t st) {
    if (p.Mp % kTileM != 0 || p.Np % kTileN != 0 || p.Kp % kTileK != 0) return cudaErrorInvalidValue;
    CUtensorMap tmA, tmB;
    if (!make_plane_map(&tmA, p.a_planes, (size_t)p.planes * p.Mp, p.Kp, kTileM)) return cudaErrorInvalidValue;
    if (!make_plane_map(&tmB, p.b_planes, (size_t)p.planes * p.Np, p.Kp, kTileN)) return cudaErrorInvalidValue;
    GemmArgs a{};
    const int all_m_tiles = (int)(p.Mp / kTileM);
    if (p.m_tile_begin < 0 || p.m_tile_count < 0 || p.m_tile_begin + p.m_tile_count > all_m_tiles)
        return cudaErrorInvalidValue;
    a.mt0 = p.m_tile_begin;
    a.m_tiles = p.m_tile_count ? p.m_tile_count : all_m_tiles - p.m_tile_begin;
    a.n_tiles = (int)(p.Np / kTileN);
    a.k_blocks = (int)(p.Kp / kTileK);
    a.total_tiles = a.m_tiles * a.n_tiles;
    // Default band.  Scheme II: the m-tiles of 32 MiB of one A plane, at
    // least 16 (K = 8192: 32 m-tiles, 4096 rows).  The band of A stays in L2
    // while B's plane streams past once per band: at 8192^3, S = 16, bands of
    // 32 read 3.2 GB per launch against 5.3 GB for 16 (64: 10.9 GB), 1-2%
    // faster; at 16384 x 16384 x 1024 the whole M (128 m-tiles) is 2.4% faster
    // than 16.  Scheme I units read all slice pairs of a tile: 16 m-tiles.
    int band = p.band;
    if (band <= 0) {
        band = 16;
        if (p.coef) {
            const long long fit = (32ll << 20) / ((long long)kTileM * (long long)p.Kp);
            if (fit > band) band = (int)(fit < a.m_tiles ? fit : a.m_tiles);
        }
    }
    a.band = a.m_tiles < band ? a.m_tiles : band;
    a.groups = p.pairs.num_groups;
    a.Mp = (long long)p.Mp;
    a.Np = (long long)p.Np;
    a.M = (long long)(p.M ? p.M : p.Mp);
    a.N = (long long)(p.N ? p.N : p.Np);
    a.err = p.err;
    a.ctc = p.ctc;
    a.coef = p.coef;
    a.S = p.planes;
    a.wait_hint = p.wait_hint_ns;
    const long long units = (long long)a.total_tiles * a.groups;
    if (units == 0) return cudaSuccess;
    const int grid = (int)(units < p.sms ? units : p.sms);
    // k-blocks of MMAs per unit, averaged over the groups (Scheme I groups sum several pairs)
    const long long unit_kb = (long long)a.k_blocks * p.pairs.start[a.groups] / a.groups;
    if (unit_kb < kEpi8Below)
        return p.coef ? gemm_launch<kEpiCoef, 8>(tmA, tmB, p.pairs, a, grid, st)
                      : gemm_launch<kEpiI32, 8>(tmA, tmB, p.pairs, a, grid, st);
    return p.coef ? gemm_launch<kEpiCoef, 4>(tmA, tmB, p.pairs, a, grid, st)
                  : gemm_launch<kEpiI32, 4>(tmA, tmB, p.pairs, a, grid, st);
}

cudaError_t launch_reconstruct2(const int32_t* ctc, size_t Mp, size_t Np, size_t M, size_t N, int S,
                                const int32_t* shiftA, const int32_t* shiftB, double* C, cudaStream_t st) {
    long long total = (long long)M * (long long)N;
    if (total == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = grid_for(total, 256, sms, 16);
    // limbs of M: S <= 4 -> 1, <= 8 -> 2, <= 12 -> 3, <= 16 -> 4, else 5
    int nl = (S + 3) / 4;
    switch (nl) {
        case 1: k_reconstruct2<1><<<grid, 256, 0, st>>>(ctc, Mp, Np, M, N, S, shiftA, shiftB, C); break;
        case 2: k_reconstruct2<2><<<grid, 256, 0, st>>>(ctc, Mp, Np, M, N, S, shiftA, shiftB, C); break;
        case 3: k_reconstruct2<3><<<grid, 256, 0, st>>>(ctc, Mp, Np, M, N, S, shiftA, shiftB, C); break;
        case 4: k_reconstruct2<4><<<grid, 256, 0, st>>>(ctc, Mp, Np, M, N, S, shiftA, shiftB, C); break;
        default: k_reconstruct2<5><<<grid, 256, 0, st>>>(ctc, Mp, Np, M, N, S, shiftA, shiftB, C); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_crt_coef(const uint8_t* coef, size_t Mp, size_t Np, size_t M, size_t N, int S,
                            const int32_t* shiftA, const int32_t* shiftB, double* C, int sms, cudaStream_t st) {
    long long total = (long long)M * (long long)((N + 3) / 4);
    if (total == 0) return cudaSuccess;
    const int grid = grid_for(total, 128, sms, 32);
    const long long MP = (long long)Mp, NP = (long long)Np, MM = (long long)M, NN = (long long)N;
    switch (S) {
#define OZA_CASE(n) \
    case n: k_crt_coef<n><<<grid, 128, 0, st>>>(coef, MP, NP, MM, NN, shiftA, shiftB, C); break;
        OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_reconstruct1(const int32_t* ctc, size_t Mp, size_t Np, size_t M, size_t N, int S, int beta,
                                const int32_t* negA, const int32_t* negB, double* C, int sms, cudaStream_t st,
                                const PairList* units) {
    const long long total = (long long)M * (long long)((N + 3) / 4);
    if (total == 0) return cudaSuccess;
    if (Np % 4 != 0 || beta < 1 || beta * S > 1022) return cudaErrorInvalidValue;
    const int grid = grid_for(total, 256, sms, 16);
    const long long MP = (long long)Mp, NP = (long long)Np, MM = (long long)M, NN = (long long)N;
    if (units && units->num_groups != S) {
        if (S < 1 || S > kMaxSlicesHost || units->first_unit[S] != units->num_groups) return cudaErrorInvalidValue;
        UnitMap um{};
        for (int g = 0; g <= S; ++g) um.first[g] = units->first_unit[g];
        k_reconstruct1_units<<<grid, 256, 0, st>>>(ctc, MP, NP, MM, NN, S, beta, negA, negB, C, um);
        return cudaGetLastError();
    }
    switch (S) {
#define OZA_CASE(n) \
    case n: k_reconstruct1<n><<<grid, 256, 0, st>>>(ctc, MP, NP, MM, NN, beta, negA, negB, C); break;
        OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Grouped plan: device tables built once, replayed by every call
// ---------------------------------------------------------------------------
struct GroupPlan {
    struct Launch {
        GroupLaunchDev dev{};
        long long tiles = 0;
        int S = 0;
        bool wide = false;
        size_t ids_off = 0, start_off = 0;   // in the table image
    };
    std::vector<GroupProblemDev> probs;
    std::vector<uint8_t> image;           // host image of the device tables
    size_t probs_off = 0, gprobs_off = 0, maps_off = 0, units_off = 0;
    void* dev = nullptr;                  // owned table memory (group_plan_create only)
    GroupProblemDev* d_probs = nullptr;
    GroupGemmArgs gemm{};
    size_t table_bytes = 0;
    Launch rows, cols;
    std::vector<Launch> slr, slc, crt;
    std::vector<Launch*> all_launches() {
        std::vector<Launch*> v{&rows, &cols};
        for (auto* vec : {&slr, &slc, &crt})
            for (auto& L : *vec) v.push_back(&L);
        return v;
    }
};

namespace {

// Byte layout of the plan's device tables, built on the host in one buffer.
struct TableBuilder {
    std::vector<uint8_t> buf;
    TableBuilder() { buf.reserve(1 << 16); }
    size_t put(const void* src, size_t n, size_t align = 128) {
        size_t off = (buf.size() + align - 1) / align * align;
        buf.resize(off + n);
        if (n) std::memcpy(buf.data() + off, src, n);
        return off;
    }
};

}  // namespace

cudaError_t group_plan_prepare();

cudaError_t group_plan_build(const GroupProblem* in, int count, int* err, GroupPlan** out) {
    *out = nullptr;
    if (count <= 0) return cudaErrorInvalidValue;
    {
        const cudaError_t pe = group_plan_prepare();
        if (pe != cudaSuccess) return pe;
    }
    auto* gp = new (std::nothrow) GroupPlan();
    if (!gp) return cudaErrorMemoryAllocation;
    std::unique_ptr<GroupPlan> hold(gp);
    gp->probs.resize(count);
    std::vector<GroupGemmProblem> gprobs(count);
    std::vector<CUtensorMap> maps(2 * (size_t)count);
    std::vector<int4> units;
    for (int i = 0; i < count; ++i) {
        const GroupProblem& p = in[i];
        if (p.S < 1 || p.S > kMaxSlices || p.M == 0 || p.N == 0 || p.K == 0 || p.Mp % kTileM || p.Np % kTileN ||
            p.Kp % kTileK)
            return cudaErrorInvalidValue;
        if (p.k_param > 62 && p.S < 17) return cudaErrorInvalidValue;
        GroupProblemDev& d = gp->probs[i];
        d.A = p.A;
        d.B = p.B;
        d.C = p.C;
        d.M = (long long)p.M;
        d.N = (long long)p.N;
        d.K = (long long)p.K;
        d.Mp = (long long)p.Mp;
        d.Np = (long long)p.Np;
        d.Kp = (long long)p.Kp;
        d.S = p.S;
        d.k_param = p.k_param;
        d.shiftA = p.shiftA;
        d.shiftB = p.shiftB;
        d.colmax = p.colmax;
        d.a_planes = p.a_planes;
        d.b_planes = p.b_planes;
        d.coef = p.coef;
        gprobs[i] = GroupGemmProblem{d.Mp, d.Np, (long long)p.M, (long long)p.N, (int)(p.Kp / kTileK), p.S, p.coef};
        if (!make_plane_map(&maps[2 * i], p.a_planes, (size_t)p.S * p.Mp, p.Kp, kTileM) ||
            !make_plane_map(&maps[2 * i + 1], p.b_planes, (size_t)p.S * p.Np, p.Kp, kTileN))
            return cudaErrorInvalidValue;
        const int mt = (int)(p.Mp / kTileM), nt = (int)(p.Np / kTileN);
        for (int g = 0; g < p.S; ++g)
            for (int a = 0; a < mt; ++a)
                for (int b = 0; b < nt; ++b) units.push_back(make_int4(i, a, b, g));
    }
    // Longest units first (cost ~ k_blocks): CTA c takes units c, c + grid, ...,
    // so each round of `grid` units has near-equal cost.  Stable, so units of
    // one problem and modulus stay together for L2 reuse.
    {
        // Counting sort on k_blocks, descending, stable.
        int maxkb = 0;
        for (const auto& gpr : gprobs) maxkb = std::max(maxkb, gpr.k_blocks);
        std::vector<size_t> pos(maxkb + 2, 0);
        for (const int4& u : units) ++pos[maxkb - gprobs[u.x].k_blocks + 1];
        for (int b = 1; b <= maxkb + 1; ++b) pos[b] += pos[b - 1];
        std::vector<int4> sorted(units.size());
        for (const int4& u : units) sorted[pos[maxkb - gprobs[u.x].k_blocks]++] = u;
        units.swap(sorted);
    }

    // Per-stage block maps; the templated stages split by (S, wide) class.
    auto tiles_of = [&](const GroupProblemDev& d, int stage) -> long long {
        switch (stage) {
            case 0: return (d.M + 7) / 8;
            case 1: return ((d.N + 63) / 64) * ((d.K + 255) / 256);
            case 2: return (d.M * (d.Kp / 8) + 256 * kGroupRowChunks - 1) / (256 * kGroupRowChunks);
            case 3: return ((d.N + 31) / 32) * ((d.Kp / 128 + kGroupColTiles - 1) / kGroupColTiles);
            default: return (d.M * ((d.N + 3) / 4) + 255) / 256;
        }
    };
    std::vector<std::pair<int, bool>> classes;
    for (const auto& d : gp->probs) {
        std::pair<int, bool> c{d.S, d.k_param > 62};
        if (std::find(classes.begin(), classes.end(), c) == classes.end()) classes.push_back(c);
    }
    TableBuilder tb;
    gp->slr.resize(classes.size());
    gp->slc.resize(classes.size());
    gp->crt.resize(classes.size());
    auto add_launch = [&](GroupPlan::Launch& L, int stage, int S, bool wide, bool all) {
        std::vector<int> ids;
        std::vector<long long> start(1, 0);
        for (int i = 0; i < count; ++i) {
            const GroupProblemDev& d = gp->probs[i];
            if (!all && (d.S != S || (d.k_param > 62) != wide)) continue;
            ids.push_back(i);
            start.push_back(start.back() + tiles_of(d, stage));
        }
        L.dev.n = (int)ids.size();
        L.tiles = start.back();
        L.S = S;
        L.wide = wide;
        L.ids_off = tb.put(ids.data(), ids.size() * sizeof(int));
        L.start_off = tb.put(start.data(), start.size() * sizeof(long long));
    };
    add_launch(gp->rows, 0, 0, false, true);
    add_launch(gp->cols, 1, 0, false, true);
    for (size_t c = 0; c < classes.size(); ++c) {
        add_launch(gp->slr[c], 2, classes[c].first, classes[c].second, false);
        add_launch(gp->slc[c], 3, classes[c].first, classes[c].second, false);
        add_launch(gp->crt[c], 4, classes[c].first, classes[c].second, false);
    }
    for (const auto& L : {gp->rows.tiles, gp->cols.tiles})
        if (L > 0x7FFFFFFFll) return cudaErrorInvalidValue;
    for (size_t c = 0; c < classes.size(); ++c)
        if (gp->slr[c].tiles > 0x7FFFFFFFll || gp->slc[c].tiles > 0x7FFFFFFFll || gp->crt[c].tiles > 0x7FFFFFFFll)
            return cudaErrorInvalidValue;
    if (units.size() > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    gp->probs_off = tb.put(gp->probs.data(), gp->probs.size() * sizeof(GroupProblemDev));
    gp->gprobs_off = tb.put(gprobs.data(), gprobs.size() * sizeof(GroupGemmProblem));
    gp->maps_off = tb.put(maps.data(), maps.size() * sizeof(CUtensorMap), 128);
    gp->units_off = tb.put(units.data(), units.size() * sizeof(int4));
    gp->gemm.total_units = (int)units.size();
    gp->gemm.err = err;
    gp->image.swap(tb.buf);
    gp->table_bytes = gp->image.size();
    *out = hold.release();
    return cudaSuccess;
}

void group_plan_bind(GroupPlan* gp, void* dev) {
    uint8_t* base = static_cast<uint8_t*>(dev);
    for (GroupPlan::Launch* L : gp->all_launches()) {
        L->dev.ids = reinterpret_cast<const int*>(base + L->ids_off);
        L->dev.start = reinterpret_cast<const long long*>(base + L->start_off);
    }
    gp->d_probs = reinterpret_cast<GroupProblemDev*>(base + gp->probs_off);
    gp->gemm.units = reinterpret_cast<const int4*>(base + gp->units_off);
    gp->gemm.maps = reinterpret_cast<const CUtensorMap*>(base + gp->maps_off);
    gp->gemm.probs = reinterpret_cast<const GroupGemmProblem*>(base + gp->gprobs_off);
}

const void* group_plan_image(const GroupPlan* p) { return p->image.data(); }

cudaError_t group_plan_create(const GroupProblem* in, int count, int* err, GroupPlan** out) {
    GroupPlan* gp = nullptr;
    cudaError_t e = group_plan_build(in, count, err, &gp);
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&gp->dev, gp->table_bytes);
    if (e == cudaSuccess) e = cudaMemcpy(gp->dev, gp->image.data(), gp->table_bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        group_plan_destroy(gp);
        return e;
    }
    group_plan_bind(gp, gp->dev);
    *out = gp;
    return cudaSuccess;
}

void group_plan_destroy(GroupPlan* p) {
    if (!p) return;
    if (p->dev) cudaFree(p->dev);
    delete p;
}

cudaError_t group_plan_set_matrices(GroupPlan* p, const double* const* A, const double* const* B,
                                    double* const* C, cudaStream_t st) {
    bool changed = false;
    for (size_t i = 0; i < p->probs.size(); ++i) {
        GroupProblemDev& d = p->probs[i];
        if (d.A != A[i] || d.B != B[i] || d.C != C[i]) {
            d.A = A[i];
            d.B = B[i];
            d.C = C[i];
            changed = true;
        }
    }
    if (!changed) return cudaSuccess;
    // Pageable source: the copy is staged before this call returns.
    return cudaMemcpyAsync(p->d_probs, p->probs.data(), p->probs.size() * sizeof(GroupProblemDev),
                           cudaMemcpyHostToDevice, st);
}

size_t group_plan_units(const GroupPlan* p) { return (size_t)p->gemm.total_units; }
size_t group_plan_table_bytes(const GroupPlan* p) { return p->table_bytes; }
int group_plan_launches(const GroupPlan* p) { return 3 + 3 * (int)p->slr.size(); }

cudaError_t group_plan_prepare() {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_group_gemm_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    });
    return attr;
}

cudaError_t group_plan_launch(GroupPlan* p, unsigned long long* colmax, size_t colmax_count, int sms,
                              cudaStream_t st, cudaEvent_t* ev) {
    cudaError_t e = group_plan_prepare();
    if (e != cudaSuccess) return e;
#define OZA_TRY(x)                          \
    do {                                    \
        if ((e = (x)) != cudaSuccess) return e; \
    } while (0)
    if (ev) OZA_TRY(cudaEventRecord(ev[0], st));
    OZA_TRY(cudaMemsetAsync(colmax, 0, colmax_count * sizeof(unsigned long long), st));
    k_group_stats_rows<<<(unsigned)p->rows.tiles, 256, 0, st>>>(p->d_probs, p->rows.dev);
    k_group_stats_cols<<<(unsigned)p->cols.tiles, 256, 0, st>>>(p->d_probs, p->cols.dev);
    OZA_TRY(cudaGetLastError());
    if (ev) OZA_TRY(cudaEventRecord(ev[1], st));
    for (size_t c = 0; c < p->slr.size(); ++c) {
        const GroupPlan::Launch& R = p->slr[c];
        const GroupPlan::Launch& Cl = p->slc[c];
        switch (R.S) {
#define OZA_CASE(n)                                                                                         \
    case n:                                                                                                 \
        if (R.wide) {                                                                                       \
            k_group_slice_rows<n, (n >= 17)><<<(unsigned)R.tiles, 256, 0, st>>>(p->d_probs, R.dev);       \
            k_group_slice_cols<n, (n >= 17)><<<(unsigned)Cl.tiles, 256, 0, st>>>(p->d_probs, Cl.dev);     \
        } else {                                                                                            \
            k_group_slice_rows<n, false><<<(unsigned)R.tiles, 256, 0, st>>>(p->d_probs, R.dev);            \
            k_group_slice_cols<n, false><<<(unsigned)Cl.tiles, 256, 0, st>>>(p->d_probs, Cl.dev);          \
        }                                                                                                   \
        break;
            OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
            default: return cudaErrorInvalidValue;
        }
        OZA_TRY(cudaGetLastError());
    }
    if (ev) OZA_TRY(cudaEventRecord(ev[2], st));
    const int grid = p->gemm.total_units < sms ? p->gemm.total_units : sms;
    if (grid > 0) k_group_gemm_i8<<<grid, gemm_threads<8>(), kGemmSmem, st>>>(p->gemm);
    OZA_TRY(cudaGetLastError());
    if (ev) OZA_TRY(cudaEventRecord(ev[3], st));
    for (const GroupPlan::Launch& L : p->crt) {
        switch (L.S) {
#define OZA_CASE(n) \
    case n: k_group_crt<n><<<(unsigned)L.tiles, 256, 0, st>>>(p->d_probs, L.dev); break;
            OZA_FOR_EACH_S(OZA_CASE)
#undef OZA_CASE
            default: return cudaErrorInvalidValue;
        }
        OZA_TRY(cudaGetLastError());
    }
    if (ev) OZA_TRY(cudaEventRecord(ev[4], st));
#undef OZA_TRY
    return cudaSuccess;
}


cudaError_t launch_to_reference_layout(const int8_t* a_planes, const int8_t* b_planes, const int32_t* ctc, int S,
                                      int groups, size_t M, size_t N, size_t K, size_t Mp, size_t Np, size_t Kp,
                                      int8_t* a_ref, int8_t* b_ref, int32_t* c_ref, int c_first, int c_count,
                                      bool sum_planes, cudaStream_t st) {
    if (M == 0 || N == 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < S && K && e == cudaSuccess; ++s)
        e = cudaMemcpy2DAsync(a_ref + (size_t)s * M * K, K, a_planes + (size_t)s * Mp * Kp, Kp, K, M,
                              cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    if (K) {
        const dim3 grid((unsigned)((N + 31) / 32), (unsigned)((K + 31) / 32), (unsigned)S);
        k_planes_to_kn<<<grid, 256, 0, st>>>(b_planes, (long long)Np, (long long)Kp, (long long)K, (long long)N, b_ref);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (c_first < 0 || c_count < 0 || c_first + c_count > groups) return cudaErrorInvalidValue;
    if (sum_planes && c_count > 1) {
        k_sum_planes<<<grid_for((long long)(M * N), 256, 148, 8), 256, 0, st>>>(
            ctc, (long long)Mp, (long long)Np, (long long)M, (long long)N, c_first, c_count, c_ref);
        return cudaGetLastError();
    }
    for (int g = 0; g < c_count && e == cudaSuccess; ++g)
        e = cudaMemcpy2DAsync(c_ref + (size_t)g * M * N, N * sizeof(int32_t), ctc + (size_t)(c_first + g) * Mp * Np,
                              Np * sizeof(int32_t), N * sizeof(int32_t), M, cudaMemcpyDeviceToDevice, st);
    return e;
}

cudaError_t launch_wait_probe(int* gerr, unsigned long long limit_ns, int* status, cudaStream_t st) {
    k_wait_probe<<<1, 32, 0, st>>>(gerr, limit_ns, status);
    return cudaGetLastError();
}

}  // namespace oza
