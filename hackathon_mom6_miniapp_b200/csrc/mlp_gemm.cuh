// mlp_gemm.cuh -- BF16 tensor-core GEMM for the barotropic surrogate MLP on
// sm_100a: TMA-staged operand tiles, tcgen05.mma with the FP32 accumulator in
// tensor memory, and fused epilogues.
//
//   D[M x N] = A[M x K] * B[N x K]^T        (A, B bf16, row-major, K contiguous)
//
// One CTA computes a 128 x BN tile (BN <= 256, a multiple of 16) over the K
// range of its split (blockIdx.z).  Four warps: warp 0 allocates the
// accumulator columns in tensor memory and its lane 0 issues the TMA loads of
// each 64-wide K step into a ring of STAGES shared-memory stages (128-byte
// swizzle, the layout the MMA descriptors name); lane 0 of warp 1 issues four
// 128 x BN x 16 MMAs per stage and commits each stage back to the producer
// through an mbarrier; after the last commit all four warps read their 32
// accumulator rows out of tensor memory (tcgen05.ld) into the epilogue.
// Every wait is bounded: when a wait gives up the CTA records it in *err,
// stops issuing, waits (bounded) for its issued work and frees its tensor
// memory before it returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace mom6b {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmStages = 4, kGemmThreads = 128;
// Stages of the short-K layers (K <= 256): two fit twice per SM, so one
// CTA's epilogue overlaps the other's MMAs (2 x 256 TMEM columns = all 512).
constexpr int kGemmStagesShort = 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
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

// Wait for the phase with the given parity to complete; false after `budget`
// clock cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long budget)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > budget) return false;
    return true;
}

// 2-D tiled TMA load of box (x = inner coordinate, y) into shared memory,
// completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                           uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile stored by TMA with
// the 128-byte swizzle: rows of 64 bf16 (128 B), 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);          // start address
    d |= (uint64_t)1u << 16;                          // leading byte offset (unused, 16 B)
    d |= (uint64_t)(1024u >> 4) << 32;                // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                          // swizzle: 128 B
    return d;
}

// Instruction descriptor: bf16 x bf16 -> f32, both operands K-major, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n)
{
    return (1u << 4)                       // accumulator format: f32
           | (1u << 7)                     // A format: bf16
           | (1u << 10)                    // B format: bf16
           | ((uint32_t)(n >> 3) << 17)    // N / 8
           | ((uint32_t)(128 >> 4) << 24); // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive f32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Tensor-memory columns to allocate for BN accumulator columns (a power of 2, >= 32).
__host__ __device__ constexpr int tmem_cols_for(int bn)
{
    return bn <= 32 ? 32 : bn <= 64 ? 64 : bn <= 128 ? 128 : bn <= 256 ? 256 : 512;
}

// Clock cycles a wait may take before the CTA gives up (about a second).
constexpr long long kGemmWaitBudget = 2000000000LL;

// The GEMM main loop; leaves the accumulator in tensor memory and returns its
// base address in *tmem (all threads), or false when a wait gave up.  Epi is
// called by every thread with (row, first column, 16 values) for each of the
// BN / 16 column chunks of its row, then the tensor memory is freed.
template <int BN, int STAGES, class Epi>
__device__ __forceinline__ void gemm_tile(const CUtensorMap* mapA, const CUtensorMap* mapB,
                                          int M, int N, int K, int k_per_split, int* err,
                                          Epi&& epi)
{
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "MMA N must be 16..256, step 16");
    constexpr int A_BYTES = kGemmBM * kGemmBK * 2, B_BYTES = BN * kGemmBK * 2;
    constexpr int STAGE = A_BYTES + ((B_BYTES + 1023) / 1024) * 1024;
    constexpr int TCOLS = tmem_cols_for(BN);
    extern __shared__ __align__(1024) unsigned char gsm_raw[];
    // 1024-byte alignment of every stage (the swizzle atom)
    unsigned char* gsm = (unsigned char*)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;

    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    const int m0 = (int)blockIdx.x * kGemmBM, n0 = (int)blockIdx.y * BN;
    const int k0 = (int)blockIdx.z * k_per_split;
    const int k1 = min(K, k0 + k_per_split);
    const int nk = k1 > k0 ? (k1 - k0 + kGemmBK - 1) / kGemmBK : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (warp == 0 && lane == 0) {
        // producer: TMA loads of A rows [m0, m0+128) and B rows [n0, n0+BN)
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % STAGES, u = kt / STAGES;
            if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1), kGemmWaitBudget)) {
                s_fail = 1;
                break;
            }
            if (*(volatile int*)&s_fail) break;
            unsigned char* st = gsm + (size_t)s * STAGE;
            mbar_arrive_expect_tx(&full[s], (uint32_t)(A_BYTES + B_BYTES));
            tma_load_2d(st, mapA, k0 + kt * kGemmBK, m0, &full[s]);
            tma_load_2d(st + A_BYTES, mapB, k0 + kt * kGemmBK, n0, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        const uint32_t idesc = umma_idesc_bf16(BN);
        int issued = 0;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % STAGES, u = kt / STAGES;
            if (!mbar_wait(&full[s], (uint32_t)(u & 1), kGemmWaitBudget)) {
                s_fail = 1;
                break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(gsm + (size_t)s * STAGE);
            const uint32_t sb = sa + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < kGemmBK / 16; ++kk)
                umma_bf16(tmem, umma_desc_sw128(sa + kk * 32), umma_desc_sw128(sb + kk * 32),
                          idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            umma_commit(&empty[s]);
            ++issued;
        }
        umma_commit(&done);   // arrives when every issued MMA has completed
        (void)issued;
    }
    // every thread: wait for the accumulator
    const bool ok = mbar_wait(&done, 0u, 2 * kGemmWaitBudget);
    __syncthreads();
    tc_fence_after();
    if (!ok || s_fail) {
        if (threadIdx.x == 0) atomicExch(err, 1);
    } else if (nk > 0) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN / 16; ++c) {
            float v[16];
            tmem_ld16(tbase + (uint32_t)(c * 16), v);
            if (row < M && n0 + c * 16 < N) epi(row, n0 + c * 16, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TCOLS));
}

// Dynamic shared memory a gemm_tile<BN, STAGES> launch needs.
__host__ __device__ constexpr int gemm_smem_bytes(int bn, int stages)
{
    return stages * (kGemmBM * kGemmBK * 2 + ((bn * kGemmBK * 2 + 1023) / 1024) * 1024) + 1024;
}

} // namespace mom6b
