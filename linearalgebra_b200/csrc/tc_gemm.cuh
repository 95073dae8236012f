// Tensor-core (tcgen05) trailing update for the mixed-precision LU:
//
//     C[M x N] (fp32, row-major, ldc)  -=  A[M x K] * B[N x K]^T
//
// A and B are K-major operand copies (row stride K elements) in TF32 (fp32
// containers), BF16, FP16 or FP8-E4M3.  FP8 operands carry power-of-two
// scales, one per row of A and one per row of B (a row spans the whole K
// depth, so the scale is constant along the reduction); the epilogue applies
// C -= inv_sa[row] * inv_sb[col] * acc.  One CTA computes one 128 x 256 tile
// of C:
//   * warp 0 / lane 0 issues TMA loads of 128-byte-wide K slices of A and B
//     (128B swizzle) into a ring of shared-memory stages, completing on
//     mbarriers;
//   * warp 1 / lane 0 issues tcgen05.mma (M=128, N=256, 32 bytes of K per
//     instruction) accumulating in FP32 in tensor memory, and frees each
//     stage with tcgen05.commit;
//   * all four warps then read the accumulator from tensor memory
//     (tcgen05.ld, one row per thread) and write C - acc.
// With SPLIT3 the operands come in two parts each (x = big + small, big the
// TF32-truncated value) and the product is big*big + big*small + small*big,
// which recovers nearly FP32 accuracy from TF32 tensor cores (Ootomo &
// Yokota, IJHPCA 2022).
//
// Every mbarrier wait is bounded (2 s); on a timeout the kernel records an
// error in the device status block, waits (bounded) for its own copies in
// flight, releases its tensor memory and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cute/arch/mma_sm100_desc.hpp>

#include "common.cuh"

namespace b200la
{

enum TcKind : int
{
    TC_TF32 = 0,
    TC_BF16 = 1,
    TC_FP16 = 2,
    TC_FP8  = 3   // E4M3, kind::f8f6f4
};

constexpr int kTcBM        = 128;
constexpr int kTcBN        = 256;
constexpr int kTcAtomBytes = 128;                    // one 128B-swizzle atom of K per stage
constexpr int kTcTileA     = kTcBM * kTcAtomBytes;   // 16 KB: A slice of a stage
constexpr int kTcTileB     = kTcBN * kTcAtomBytes;   // 32 KB: B slice of a stage
constexpr int kTcPair      = kTcTileA + kTcTileB;    // one product's operands

template <int KIND> struct TcTraits;
template <> struct TcTraits<TC_TF32>
{
    static constexpr int      elem = 4;
    static constexpr uint32_t fmt  = 2;  // TF32
};
template <> struct TcTraits<TC_BF16>
{
    static constexpr int      elem = 2;
    static constexpr uint32_t fmt  = 1;  // BF16
};
template <> struct TcTraits<TC_FP16>
{
    static constexpr int      elem = 2;
    static constexpr uint32_t fmt  = 0;  // F16
};

template <> struct TcTraits<TC_FP8>
{
    static constexpr int      elem = 1;
    static constexpr uint32_t fmt  = 0;  // E4M3 (kind::f8f6f4 encoding)
};

__host__ __device__ constexpr int tc_elem_bytes(int kind)
{
    return kind == TC_TF32 ? 4 : (kind == TC_FP8 ? 1 : 2);
}

template <bool SPLIT3> constexpr int tc_stages() { return SPLIT3 ? 2 : 4; }
template <bool SPLIT3> constexpr int tc_stage_bytes() { return SPLIT3 ? 2 * kTcPair : kTcPair; }
template <bool SPLIT3> constexpr size_t tc_smem_bytes()
{
    // stages + 1 KB alignment slack + barriers/TMEM address
    return (size_t)tc_stages<SPLIT3>() * tc_stage_bytes<SPLIT3>() + 1024 + 256;
}

__device__ __forceinline__ void tma_load_2d(void* smem, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];" ::"r"(smem_u32(smem)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int KIND>
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
    uint32_t accumulate)
{
    if constexpr (KIND == TC_TF32)
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    }
    else if constexpr (KIND == TC_FP8)
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    }
    else
    {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Shared-memory matrix descriptor of a K-major tile stored as TMA writes it
// with 128B swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t tc_desc(uint32_t smem_addr)
{
    cute::UMMA::SmemDescriptor d;
    d.desc_                = 0;
    d.start_address_       = (uint16_t)((smem_addr & 0x3FFFF) >> 4);
    d.leading_byte_offset_ = 1;
    d.stride_byte_offset_  = 1024 >> 4;
    d.version_             = 1;
    d.base_offset_         = 0;
    d.lbo_mode_            = 0;
    d.layout_type_         = (uint8_t)cute::UMMA::LayoutType::SWIZZLE_128B;
    return d.desc_;
}

// Instruction descriptor (the bit layout of cute::UMMA::InstrDescriptor):
// F32 accumulate (bit 4), A/B formats (bits 7-9, 10-12), K-major A and B
// (bits 15, 16 = 0), N >> 3 (bits 17-22), M >> 4 (bits 24-28).
template <int KIND> __host__ __device__ constexpr uint32_t tc_idesc()
{
    return (1u << 4) | (TcTraits<KIND>::fmt << 7) | (TcTraits<KIND>::fmt << 10) |
           ((uint32_t)(kTcBN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
}
static_assert((tc_idesc<TC_TF32>() & ~(0x3Fu << 17)) == (0x8200910u & ~(0x3Fu << 17)),
    "TF32 instruction descriptor layout");

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i)
    {
        v[i] = __uint_as_float(r[i]);
    }
}

template <int KIND, bool SPLIT3>
__global__ void __launch_bounds__(128, 1) k_tc_update(const __grid_constant__ CUtensorMap tmA,
    const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmAs,
    const __grid_constant__ CUtensorMap tmBs, float* __restrict__ C, int64_t ldc, int M, int N, int K,
    DeviceStatus* __restrict__ st, const float* __restrict__ inv_sa, const float* __restrict__ inv_sb)
{
    constexpr int S   = tc_stages<SPLIT3>();
    constexpr int SB  = tc_stage_bytes<SPLIT3>();
    constexpr int EA  = kTcAtomBytes / TcTraits<KIND>::elem;  // K elements per stage
    constexpr uint32_t IDESC = tc_idesc<KIND>();

    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* tiles    = base;  // [S] x {A 16 KB, B 32 KB [, A_small, B_small]}
    uint64_t*      full     = reinterpret_cast<uint64_t*>(base + (size_t)S * SB);
    uint64_t*      empty    = full + S;
    uint64_t*      done     = empty + S;
    uint32_t*      tmem_ptr = reinterpret_cast<uint32_t*>(done + 1);
    int*           s_fail   = reinterpret_cast<int*>(tmem_ptr + 1);
    int*           s_issued = s_fail + 1;  // K slices whose loads were issued

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int m0   = blockIdx.y * kTcBM;
    const int n0   = blockIdx.x * kTcBN;
    const int natoms = K / EA;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < S; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *s_fail   = 0;
        *s_issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_ptr)),
            "r"(kTcBN)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_ptr;

    if (warp == 0 && lane == 0)
    {
        // producer: TMA loads of K slices into the stage ring
        for (int a = 0; a < natoms; ++a)
        {
            const int s = a % S;
            if (a >= S && !mbar_wait(&empty[s], ((a / S) - 1) & 1))
            {
                raise_error(st, DEV_WAIT_TIMEOUT, 10);
                atomicExch(s_fail, 1);
                break;
            }
            if (*reinterpret_cast<volatile int*>(s_fail))
            {
                break;
            }
            unsigned char* stage = tiles + (size_t)s * SB;
            mbar_expect_tx(&full[s], SB);
            tma_load_2d(stage, &tmA, a * EA, m0, &full[s]);
            tma_load_2d(stage + kTcTileA, &tmB, a * EA, n0, &full[s]);
            if constexpr (SPLIT3)
            {
                tma_load_2d(stage + kTcPair, &tmAs, a * EA, m0, &full[s]);
                tma_load_2d(stage + kTcPair + kTcTileA, &tmBs, a * EA, n0, &full[s]);
            }
            *reinterpret_cast<volatile int*>(s_issued) = a + 1;
        }
    }
    else if (warp == 1 && lane == 0)
    {
        // MMA issuer
        for (int a = 0; a < natoms; ++a)
        {
            const int s = a % S;
            if (!mbar_wait(&full[s], (a / S) & 1))
            {
                raise_error(st, DEV_WAIT_TIMEOUT, 11);
                atomicExch(s_fail, 1);
                break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(tiles + (size_t)s * SB);
            const uint32_t sb = sa + kTcTileA;
#pragma unroll
            for (int kk = 0; kk < kTcAtomBytes / 32; ++kk)
            {
                const uint64_t da = tc_desc(sa + kk * 32);
                const uint64_t db = tc_desc(sb + kk * 32);
                tc_mma<KIND>(tmem, da, db, IDESC, (a > 0 || kk > 0) ? 1u : 0u);
                if constexpr (SPLIT3)
                {
                    const uint64_t das = tc_desc(sa + kTcPair + kk * 32);
                    const uint64_t dbs = tc_desc(sa + kTcPair + kTcTileA + kk * 32);
                    tc_mma<KIND>(tmem, da, dbs, IDESC, 1u);
                    tc_mma<KIND>(tmem, das, db, IDESC, 1u);
                }
            }
            tc_commit(&empty[s]);
        }
        tc_commit(done);
    }
    __syncwarp();

    // while the MMAs run: pull this thread's row of the C tile into L2
    {
        const int r = m0 + warp * 32 + lane;
        if (r < M && n0 + kTcBN <= N && ((ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0))
        {
            const float* src = C + (size_t)r * ldc + n0;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(kTcBN * 4) : "memory");
        }
    }

    // epilogue: thread = one row of the tile, 32 columns per tensor-memory load
    const bool ok = mbar_wait(done, 0);
    if (!ok)
    {
        raise_error(st, DEV_WAIT_TIMEOUT, 12);
    }
    tc_fence_after();
    if (ok && !*reinterpret_cast<volatile int*>(s_fail))
    {
        const int  r      = m0 + warp * 32 + lane;
        const bool row_ok = r < M;
        float*     crow   = C + (size_t)(row_ok ? r : 0) * ldc;
        const bool vec    = ((ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
        // C of chunk j + 1 is loaded while chunk j is finished, so each
        // chunk's load latency overlaps the previous chunk's work
        float4 cv[8], cn[8];
        auto   fast_at = [&](int j) { return row_ok && vec && n0 + j * 32 + 32 <= N; };
        auto   load_c  = [&](int j, float4(&dst)[8]) {
            const float4* p = reinterpret_cast<const float4*>(crow + n0 + j * 32);
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                dst[q] = p[q];
            }
        };
        if (fast_at(0))
        {
            load_c(0, cv);
        }
#pragma unroll 1
        for (int j = 0; j < kTcBN / 32; ++j)
        {
            const int  c0   = n0 + j * 32;
            const bool fast = fast_at(j);
            if (j + 1 < kTcBN / 32 && fast_at(j + 1))
            {
                load_c(j + 1, cn);
            }
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * 32), v);
            if (row_ok)
            {
                if constexpr (KIND == TC_FP8)
                {
                    const float ra = inv_sa[r];
#pragma unroll
                    for (int q = 0; q < 32; ++q)
                    {
                        v[q] *= ra * (c0 + q < N ? inv_sb[c0 + q] : 0.f);
                    }
                }
                if (fast)
                {
                    float4* p = reinterpret_cast<float4*>(crow + c0);
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                    {
                        float4 x = cv[q];
                        x.x -= v[4 * q];
                        x.y -= v[4 * q + 1];
                        x.z -= v[4 * q + 2];
                        x.w -= v[4 * q + 3];
                        p[q] = x;
                    }
                }
                else
                {
#pragma unroll
                    for (int q = 0; q < 32; ++q)
                    {
                        if (c0 + q < N)
                        {
                            crow[c0 + q] -= v[q];
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                cv[q] = cn[q];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0 && lane == 0 && *reinterpret_cast<volatile int*>(s_fail))
    {
        // drain: wait (bounded) for the loads this CTA issued so no copy is
        // still writing shared memory when the CTA exits
        const int issued = *reinterpret_cast<volatile int*>(s_issued);
        for (int s = 0; s < S; ++s)
        {
            if (s < issued)
            {
                const int last_a = ((issued - 1 - s) / S) * S + s;
                mbar_wait(&full[s], (last_a / S) & 1);
            }
        }
    }
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcBN)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// Persistent form of the same update: one CTA per SM walks the 128 x 256
// tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (tile t covers rows
// (t % Mt) * 128 and columns (t / Mt) * 256), with two accumulators of 256
// TMEM columns so the epilogue of tile i runs while the MMAs of tile i + 1
// do:
//   * warp 0 / lane 0: TMA loads into the stage ring, across tiles;
//   * warp 1: allocates 512 TMEM columns; lane 0 issues the MMAs of tile i
//     into accumulator i % 2 once the epilogue has released it, and commits
//     the accumulator to acc_full[i % 2];
//   * warps 2..9: epilogue, two warps per TMEM lane quarter (warp w reads
//     TMEM lanes 32 (w % 4) ...; warps 2..5 take the tile's first 128
//     columns, 6..9 the last 128), C -= acc in 32-column chunks with the
//     next chunks' C loads in flight, then release the accumulator
//     (acc_empty, 256 arrivals); the C rows of the CTA's next tile are
//     prefetched into L2 when a tile's epilogue starts.
// The per-element arithmetic is that of k_tc_update.  Every wait is bounded;
// on a timeout the CTA records the error, stops issuing, drains its loads
// and MMAs in flight (bounded) and frees its tensor memory.
// ---------------------------------------------------------------------------
constexpr int kTcpThreads = 320;  // 2 producer/MMA warps + 8 epilogue warps
constexpr int kTcpEpiWarps = 8;

// Epilogue staging: each of the 8 epilogue warps turns its 32 rows x 32
// columns of the accumulator (thread = row, as tcgen05.ld delivers them)
// into row-contiguous pieces for coalesced C traffic.
constexpr int kTcpEpiLd = 33;
constexpr size_t kTcpEpiBytes = (size_t)8 * 32 * kTcpEpiLd * sizeof(float);

template <bool SPLIT3> constexpr size_t tcp_smem_bytes()
{
    return (size_t)tc_stages<SPLIT3>() * tc_stage_bytes<SPLIT3>() + 1024 + 256 + kTcpEpiBytes;
}

template <int KIND, bool SPLIT3>
__global__ void __launch_bounds__(kTcpThreads, 1) k_tc_update_persistent(const __grid_constant__ CUtensorMap tmA,
    const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmAs,
    const __grid_constant__ CUtensorMap tmBs, float* __restrict__ C, int64_t ldc, int M, int N, int K,
    DeviceStatus* __restrict__ st, const float* __restrict__ inv_sa, const float* __restrict__ inv_sb)
{
    constexpr int      S     = tc_stages<SPLIT3>();
    constexpr int      SB    = tc_stage_bytes<SPLIT3>();
    constexpr int      EA    = kTcAtomBytes / TcTraits<KIND>::elem;
    constexpr uint32_t IDESC = tc_idesc<KIND>();

    extern __shared__ __align__(1024) unsigned char tcp_smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(tcp_smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* tiles     = base;
    uint64_t*      full      = reinterpret_cast<uint64_t*>(base + (size_t)S * SB);
    uint64_t*      empty     = full + S;
    uint64_t*      acc_full  = empty + S;     // [2]
    uint64_t*      acc_empty = acc_full + 2;  // [2]
    uint64_t*      mma_done  = acc_empty + 2;
    uint32_t*      tmem_ptr  = reinterpret_cast<uint32_t*>(mma_done + 1);
    int*           s_fail    = reinterpret_cast<int*>(tmem_ptr + 1);
    int*           s_issued  = s_fail + 1;  // stage-ring loads issued
    float*         epi       = reinterpret_cast<float*>(base + (size_t)S * SB + 256);  // [8][32][kTcpEpiLd]

    const int warp   = threadIdx.x >> 5;
    const int lane   = threadIdx.x & 31;
    const int Mt     = (M + kTcBM - 1) / kTcBM;
    const int Nt     = (N + kTcBN - 1) / kTcBN;
    const int tiles_ = Mt * Nt;
    const int natoms = K / EA;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < S; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&acc_full[0], 1);
        mbar_init(&acc_full[1], 1);
        mbar_init(&acc_empty[0], 32 * kTcpEpiWarps);
        mbar_init(&acc_empty[1], 32 * kTcpEpiWarps);
        mbar_init(mma_done, 1);
        *s_fail   = 0;
        *s_issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_ptr)),
            "r"(2 * kTcBN)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_ptr;
    auto failed = [&]() { return *reinterpret_cast<volatile int*>(s_fail) != 0; };
    auto fail   = [&](int site) {
        raise_error(st, DEV_WAIT_TIMEOUT, site);
        atomicExch(s_fail, 1);
    };

    if (warp == 0)
    {
        if (lane == 0)
        {
            int it = 0;
            for (int t = blockIdx.x; t < tiles_ && !failed(); t += gridDim.x)
            {
                const int m0 = (t % Mt) * kTcBM;
                const int n0 = (t / Mt) * kTcBN;
                for (int a = 0; a < natoms; ++a, ++it)
                {
                    const int s = it % S;
                    if (it >= S && !mbar_wait(&empty[s], ((it / S) - 1) & 1))
                    {
                        fail(13);
                        break;
                    }
                    if (failed())
                    {
                        break;
                    }
                    unsigned char* stage = tiles + (size_t)s * SB;
                    mbar_expect_tx(&full[s], SB);
                    tma_load_2d(stage, &tmA, a * EA, m0, &full[s]);
                    tma_load_2d(stage + kTcTileA, &tmB, a * EA, n0, &full[s]);
                    if constexpr (SPLIT3)
                    {
                        tma_load_2d(stage + kTcPair, &tmAs, a * EA, m0, &full[s]);
                        tma_load_2d(stage + kTcPair + kTcTileA, &tmBs, a * EA, n0, &full[s]);
                    }
                    *reinterpret_cast<volatile int*>(s_issued) = it + 1;
                }
            }
        }
    }
    else if (warp == 1)
    {
        if (lane == 0)
        {
            int it = 0, ti = 0;
            for (int t = blockIdx.x; t < tiles_ && !failed(); t += gridDim.x, ++ti)
            {
                const int acc = ti & 1;
                if (ti >= 2 && !mbar_wait(&acc_empty[acc], ((ti >> 1) - 1) & 1))
                {
                    fail(14);
                    break;
                }
                tc_fence_after();
                const uint32_t d  = tmem + (uint32_t)(acc * kTcBN);
                bool           ok = true;
                for (int a = 0; a < natoms; ++a, ++it)
                {
                    const int s = it % S;
                    if (!mbar_wait(&full[s], (it / S) & 1))
                    {
                        fail(15);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(tiles + (size_t)s * SB);
                    const uint32_t sb = sa + kTcTileA;
#pragma unroll
                    for (int kk = 0; kk < kTcAtomBytes / 32; ++kk)
                    {
                        const uint64_t da = tc_desc(sa + kk * 32);
                        const uint64_t db = tc_desc(sb + kk * 32);
                        tc_mma<KIND>(d, da, db, IDESC, (a > 0 || kk > 0) ? 1u : 0u);
                        if constexpr (SPLIT3)
                        {
                            const uint64_t das = tc_desc(sa + kTcPair + kk * 32);
                            const uint64_t dbs = tc_desc(sa + kTcPair + kTcTileA + kk * 32);
                            tc_mma<KIND>(d, da, dbs, IDESC, 1u);
                            tc_mma<KIND>(d, das, db, IDESC, 1u);
                        }
                    }
                    tc_commit(&empty[s]);
                }
                if (!ok)
                {
                    break;
                }
                tc_commit(&acc_full[acc]);
            }
            tc_commit(mma_done);  // every MMA this thread issued has completed when this arrives
        }
    }
    else
    {
        // epilogue warps: TMEM lane quarter q = warp % 4, column half h
        const int  q   = warp & 3;
        const int  h   = (warp - 2) >> 2;
        const int  row = q * 32 + lane;
        const bool vec = ((ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
        constexpr int HC = kTcBN / 2;  // columns of a half
        auto prefetch_rows = [&](int t) {
            if (t >= tiles_)
            {
                return;
            }
            const int r  = (t % Mt) * kTcBM + row;
            const int n0 = (t / Mt) * kTcBN + h * HC;
            if (r < M && n0 + HC <= N && vec)
            {
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(C + (size_t)r * ldc + n0),
                    "r"(HC * 4)
                    : "memory");
            }
        };
        prefetch_rows(blockIdx.x);
        int ti = 0;
        for (int t = blockIdx.x; t < tiles_; t += gridDim.x, ++ti)
        {
            const int  acc = ti & 1;
            const bool got = __all_sync(0xffffffffu, mbar_wait(&acc_full[acc], (ti >> 1) & 1));
            if (!got)
            {
                if (lane == 0)
                {
                    fail(16);
                }
                break;
            }
            if (__any_sync(0xffffffffu, failed()))
            {
                break;
            }
            tc_fence_after();
            prefetch_rows(t + gridDim.x);
            const int  m0     = (t % Mt) * kTcBM;
            const int  n0     = (t / Mt) * kTcBN;
            const int  r      = m0 + row;
            const bool row_ok = r < M;
            // C traffic in row-contiguous pieces: lane (rr, c4) reads and writes
            // columns c4..c4+3 of the warp's rows rr, rr + 4, ..., rr + 28
            float*    S   = epi + (warp - 2) * 32 * kTcpEpiLd;
            const int rr  = lane >> 3;
            const int c4  = (lane & 7) * 4;
            const int wr0 = m0 + q * 32;  // the warp's first row
            float4    cv[8], cn[8], cn2[8];  // chunks j, j + 1, j + 2 of C in flight
            auto      load_c = [&](int j, float4(&dst)[8]) {
                const int c = n0 + j * 32 + c4;
#pragma unroll
                for (int i = 0; i < 8; ++i)
                {
                    const int rw = wr0 + rr + 4 * i;
                    if (rw < M && vec && c + 4 <= N)
                    {
                        dst[i] = *reinterpret_cast<const float4*>(C + (size_t)rw * ldc + c);
                    }
                    else
                    {
                        const float* pc = C + (size_t)(rw < M ? rw : 0) * ldc;
                        dst[i].x        = (rw < M && c < N) ? pc[c] : 0.f;
                        dst[i].y        = (rw < M && c + 1 < N) ? pc[c + 1] : 0.f;
                        dst[i].z        = (rw < M && c + 2 < N) ? pc[c + 2] : 0.f;
                        dst[i].w        = (rw < M && c + 3 < N) ? pc[c + 3] : 0.f;
                    }
                }
            };
            // this warp's chunks [j0, j0 + NJ); FP8 keeps one chunk ahead
            // (its scale loads need the registers), the others two
            constexpr int NJ    = HC / 32;
            constexpr int AHEAD = KIND == TC_FP8 ? 1 : 2;
            const int     j0    = h * NJ;
            load_c(j0, cv);
            if constexpr (AHEAD == 2)
            {
                load_c(j0 + 1, cn);
            }
#pragma unroll 1
            for (int j = j0; j < j0 + NJ; ++j)
            {
                const int c0 = n0 + j * 32;
                if constexpr (AHEAD == 2)
                {
                    if (j + 2 < j0 + NJ)
                    {
                        load_c(j + 2, cn2);
                    }
                }
                else
                {
                    if (j + 1 < j0 + NJ)
                    {
                        load_c(j + 1, cn);
                    }
                }
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * kTcBN + j * 32), v);
                if constexpr (KIND == TC_FP8)
                {
                    const float ra = row_ok ? inv_sa[r] : 0.f;
#pragma unroll
                    for (int qq = 0; qq < 32; ++qq)
                    {
                        v[qq] *= ra * (c0 + qq < N ? inv_sb[c0 + qq] : 0.f);
                    }
                }
#pragma unroll
                for (int qq = 0; qq < 32; ++qq)
                {
                    S[lane * kTcpEpiLd + qq] = v[qq];
                }
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 8; ++i)
                {
                    const int rl = rr + 4 * i;
                    const int rw = wr0 + rl;
                    const int c  = c0 + c4;
                    float4    x  = cv[i];
                    x.x -= S[rl * kTcpEpiLd + c4];
                    x.y -= S[rl * kTcpEpiLd + c4 + 1];
                    x.z -= S[rl * kTcpEpiLd + c4 + 2];
                    x.w -= S[rl * kTcpEpiLd + c4 + 3];
                    if (rw < M && vec && c + 4 <= N)
                    {
                        *reinterpret_cast<float4*>(C + (size_t)rw * ldc + c) = x;
                    }
                    else if (rw < M)
                    {
                        float* pc = C + (size_t)rw * ldc;
                        if (c < N)
                            pc[c] = x.x;
                        if (c + 1 < N)
                            pc[c + 1] = x.y;
                        if (c + 2 < N)
                            pc[c + 2] = x.z;
                        if (c + 3 < N)
                            pc[c + 3] = x.w;
                    }
                }
                __syncwarp();
#pragma unroll
                for (int qq = 0; qq < 8; ++qq)
                {
                    cv[qq] = cn[qq];
                    if constexpr (AHEAD == 2)
                    {
                        cn[qq] = cn2[qq];
                    }
                }
            }
            tc_fence_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[acc])) : "memory");
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 1 && lane == 0)
    {
        // every MMA issued has completed (bounded wait)
        mbar_wait(mma_done, 0);
    }
    if (warp == 0 && lane == 0 && failed())
    {
        // drain: the loads this CTA issued and nobody consumed
        const int issued = *reinterpret_cast<volatile int*>(s_issued);
        for (int s = 0; s < S; ++s)
        {
            if (s < issued)
            {
                const int last = ((issued - 1 - s) / S) * S + s;
                mbar_wait(&full[s], (last / S) & 1);
            }
        }
    }
    __syncthreads();
    if (warp == 1)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTcBN)
                     : "memory");
    }
}

}  // namespace b200la
