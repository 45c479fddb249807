// oza_device.cuh -- sm_100a building blocks shared by the Ozaki kernels:
// mbarrier waits with a time bound, TMA tile loads, tcgen05 (UMMA) issue,
// TMEM allocation and TMEM -> register loads, and the per-modulus constants.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace oza {

constexpr int kMaxSlices = 20;

// Device error codes written to the workspace's error word.
enum DeviceError : int {
    kErrNone = 0,
    kErrWaitTimeout = 1,   // an mbarrier wait exceeded its time bound
};

// Per-modulus constants for the residue and CRT arithmetic (filled on the
// host per device by upload_tables() in oza_kernels.cu).  For modulus m (odd, 149..251):
//   magic  = ceil(2^39 / m): floor(u / m) == umulhi(u, magic) >> 7 for u < 2^31
//   c21/42/63 = 2^21, 2^42, 2^63 mod m, symmetric representatives
//   inv    = (M/m)^-1 mod m for the current slice count (per table row)
//   dig[w] = bytes 4w..4w+3 of (256^i mod m, symmetric, int8), i = 0..15
//   magic32 = ceil(2^32 / m): u mod m == umulhi(u * magic32 mod 2^32, m) for u < 2^32 / m
//   bh = m * 2^10 + (m-1)/2, adj = 256 - (m-1)/2 (direct-remainder residue reduction)
//   bhm = bh * magic32 mod 2^32 (the bias folded into the reduction's multiply)
struct ModConst {
    uint32_t m;
    uint32_t magic;
    int32_t c21, c42, c63;
    uint32_t magic32;
    int32_t bh, adj;
    uint32_t dig[4];
    uint32_t bhm;
};

// Scheme II CRT table for one slice count S.  T = sum_s c_s (M / m_s), with
// c_s = ((C_s mod m_s) inv_s) mod m_s the one-byte CRT coefficients, is formed
// three residues at a time: for a triple (a, b, c) of moduli,
//   c_a M/m_a + c_b M/m_b + c_c M/m_c = d (M / (m_a m_b m_c)),
//   d = c_a m_b m_c + c_b m_a m_c + c_c m_a m_b < 3 * 250 * 2^16 < 2^26,
// so each triple costs one 32 x 128-bit product instead of three.  The last
// S mod 3 residues form a pair (d = c_a m_b + c_b m_a) or stay single.
struct CrtTable {
    uint32_t M[5];            // M = prod m_i as 5 x 32-bit limbs (M < 2^153)
    uint32_t Mhalf[5];        // floor(M / 2)
    uint32_t P[kMaxSlices][5];  // M / m_i
    uint32_t inv[kMaxSlices];   // (M / m_i)^-1 mod m_i
    uint32_t c16inv[kMaxSlices];  // (2^16 * inv_i) mod m_i
    double rinv[kMaxSlices];      // 1 / m_i rounded to double, for the quotient estimate
    // Triples (3t, 3t+1, 3t+2), t < S / 3
    uint32_t TP[kMaxSlices / 3][5];           // M / (m_a m_b m_c)
    uint32_t tk[kMaxSlices / 3];              // (m_b m_c) | (m_a m_c) << 16: dp2a weights of c_a, c_b
    uint32_t tab[kMaxSlices / 3];             // m_a m_b: weight of c_c
    double trinv[kMaxSlices / 3];             // 1 / (m_a m_b m_c) rounded to double
    // The last two residues (S - 2, S - 1) when S mod 3 == 2
    uint32_t DP[5];                           // M / (m_{S-2} m_{S-1})
    double drinv;                             // 1 / (m_{S-2} m_{S-1}) rounded to double
    int nlimbs;                   // limbs of M that can be nonzero
};

// The tables themselves (__constant__ ModConst c_mod[], CrtTable c_crt[],
// index S-1) are defined in oza_kernels.cu, the only translation unit with
// device code.

// ---------------------------------------------------------------------------
// Small exact helpers
// ---------------------------------------------------------------------------

// floor(u / m) for 0 <= u < 2^31 and 128 <= m < 256 (Granlund-Montgomery,
// magic = ceil(2^39/m); the error term u/2^39 < 2^-8 < 1/m keeps it exact).
__device__ __forceinline__ uint32_t div_small(uint32_t u, uint32_t magic) {
    return __umulhi(u, magic) >> 7;
}

// frexp exponent from the magnitude bits of a nonzero finite double.
__device__ __forceinline__ int frexp_exp_bits(unsigned long long mag) {
    int E = (int)(mag >> 52);
    if (E > 0) return E - 1022;
    return -1010 - __clzll((long long)mag);   // subnormal
}

// Max exponent from a running maximum of magnitude bits.  The reference's
// running maximum starts at -1023 (step1_statistics.hpp:33,88), so an
// all-zero row and a row whose largest entry is a subnormal below 2^-1024
// (frexp exponent < -1023) both yield -1023.
__device__ __forceinline__ int max_exp_from_bits(unsigned long long mag) {
    if (mag == 0ull) return -1023;
    int e = frexp_exp_bits(mag);
    return e < -1023 ? -1023 : e;
}

// ---------------------------------------------------------------------------
// Shared-memory addresses, mbarriers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// The same with a suspend-time hint: the thread may sleep in hardware until
// the phase completes or about `hint_ns` pass, instead of re-polling.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Time bound of one wait.  A healthy wait in these kernels lasts microseconds;
// 2 s means a lost arrival.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// Bounded wait on phase `parity`.  Returns false if the bound expired or if
// another role of the CTA already gave up (*abort != 0); on expiry it raises
// *abort and records the error in the global error word.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort, int* gerr,
                                          uint32_t hint_ns = 0, uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (hint_ns ? mbar_try_wait_hint(bar, parity, hint_ns) : mbar_try_wait(bar, parity)) return true;
        if (hint_ns || (it & 63u) == 0) {
            if (*abort) return false;
            if (globaltimer_ns() - t0 > limit_ns) {
                *abort = 1;
                if (gerr) atomicExch(gerr, kErrWaitTimeout);
                return false;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// TMA
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// 2D tiled load, completion signalled on `bar` (complete_tx).  c0 is the
// innermost (byte) coordinate and must be a multiple of 16.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 / TMEM
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Make this thread's generic-proxy shared-memory writes visible to the async
// proxy (the tensor core reading an operand tile written with st.shared).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// UMMA shared-memory descriptor for a K-major tile written by TMA with the
// 128-byte swizzle: rows of 128 bytes, 8-row (1024 B) swizzle atoms stacked
// along M/N.  Start address in 16-byte units, LBO unused (1), SBO = 1024 B,
// descriptor version 1 (sm_100), layout type 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
    d |= static_cast<uint64_t>(1) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}

// Instruction descriptor for kind::i8: signed A and B, S32 accumulator,
// both operands K-major, tile M x N.
__host__ __device__ constexpr uint32_t umma_idesc_i8(int M, int N) {
    return (2u << 4)                                   // D format: S32
           | (1u << 7)                                 // A: signed 8-bit
           | (1u << 10)                                // B: signed 8-bit
           | (static_cast<uint32_t>(N >> 3) << 17)     // N / 8
           | (static_cast<uint32_t>(M >> 4) << 24);    // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, one elected thread issues.
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace oza
