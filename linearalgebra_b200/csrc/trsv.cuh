// One-launch triangular solve for a single right-hand side, op(A) x = b
// with op = identity (lower or upper, unit or not), x overwritten in place.
//
// Row blocks of kTvRows rows are claimed by CTAs through an atomic ticket in
// solve order, so a CTA only ever waits for blocks claimed before its own
// (those CTAs are already running): no deadlock, whatever the residency.
// A CTA accumulates A[block, j] x_j for every solved block j as soon as
// block j's flag is set (bounded wait, 2 s), then solves its diagonal block
// with one warp and publishes x_block with a release store of its flag.
//
// TA is the matrix type (the factors: double or float), TX the vector and
// arithmetic type (double), so the same kernel solves with FP32 LU factors
// in FP64 for iterative refinement.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace b200la
{

constexpr int kTvRows    = 64;
constexpr int kTvThreads = 256;

struct TrsvSync
{
    int32_t  ticket;
    int32_t  pad[31];
    uint32_t flags[1];  // [nblocks], cleared per call
};

template <typename TA, typename TX>
__global__ void __launch_bounds__(kTvThreads) k_trsv_syncfree(const TA* __restrict__ a, int64_t lda,
    TX* __restrict__ x, int n, int upper, int unit, TrsvSync* sync, DeviceStatus* st,
    const DeviceStatus* gate)
{
    __shared__ TX  part[kTvRows][kTvThreads / kTvRows + 1];
    __shared__ TX  tri[kTvRows][kTvRows + 1];
    __shared__ TX  xst[2][kTvRows];
    __shared__ int s_blk, s_abort, s_ready;
    if (gate != nullptr && (ld_volatile_i32(&gate->error) != 0 || gate->first_zero >= 0))
    {
        return;
    }
    const int nb  = (n + kTvRows - 1) / kTvRows;
    const int tid = threadIdx.x;
    if (tid == 0)
    {
        s_blk   = atomicAdd(&sync->ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int t = s_blk;  // position in solve order
    if (t >= nb)
    {
        return;
    }
    const int blk = upper ? nb - 1 - t : t;
    const int r0  = blk * kTvRows;
    const int br  = min(kTvRows, n - r0);

    // ---- stage the diagonal block (only the selected triangle)
    for (int e = tid; e < kTvRows * kTvRows; e += kTvThreads)
    {
        const int i = e / kTvRows, j = e % kTvRows;
        TX        v = TX(0);
        if (i < br && j < br && (upper ? j >= i : j <= i) && !(unit && i == j))
        {
            v = (TX)a[(int64_t)(r0 + i) * lda + r0 + j];
        }
        tri[i][j] = v;
    }

    // ---- accumulate the solved blocks: thread = (row r, quarter q).  Warp 0
    // checks 32 flags at a time and publishes how many consecutive blocks
    // (in solve order) are ready; each ready block's x is staged in shared
    // memory once.
    const int r     = tid % kTvRows;
    const int q     = tid / kTvRows;
    TX        acc   = TX(0);
    int       ready = 0;
    for (int s = 0; s < t; ++s)
    {
        if (s >= ready)
        {
            if (tid < 32)
            {
                const uint64_t t0    = global_ns();
                uint32_t       polls = 0;
                int            got   = 0;
                for (;;)
                {
                    const int  ss   = s + tid;
                    const int  jb   = upper ? nb - 1 - ss : ss;
                    const bool set  = ss < t && ld_acquire_u32(&sync->flags[jb]) != 0;
                    const unsigned m = __ballot_sync(0xffffffffu, set);
                    got              = __ffs(~m) - 1;  // leading run of set flags
                    if (m == 0xffffffffu)
                    {
                        got = 32;
                    }
                    if (got > 0)
                    {
                        break;
                    }
                    if ((++polls & 255u) == 0 && global_ns() - t0 > kWaitLimitNs)
                    {
                        if (tid == 0)
                        {
                            raise_error(st, DEV_WAIT_TIMEOUT, 20);
                            s_abort = 1;
                        }
                        break;
                    }
                }
                if (tid == 0)
                {
                    s_ready = s + got;
                }
            }
            __syncthreads();
            if (s_abort)
            {
                return;
            }
            ready = s_ready;
        }
        const int jb = upper ? nb - 1 - s : s;
        const int c0 = jb * kTvRows;
        const int cw = min(kTvRows, n - c0);
        TX*       xs = xst[s & 1];
        if (tid < kTvRows)
        {
            xs[tid] = tid < cw ? __ldcg(x + c0 + tid) : TX(0);
        }
        __syncthreads();
        if (r < br)
        {
            const TA* arow = a + (int64_t)(r0 + r) * lda + c0;
            const int j0   = q * (kTvRows / 4);
#pragma unroll 4
            for (int j = j0; j < j0 + kTvRows / 4; ++j)
            {
                if (j < cw)
                {
                    acc = fma((TX)arow[j], xs[j], acc);
                }
            }
        }
    }
    part[r][q] = acc;
    __syncthreads();

    // ---- diagonal block: one warp, lane owns rows lane and lane + 32
    if (tid < 32)
    {
        const int lane = tid;
        TX        v0 = TX(0), v1 = TX(0);
        if (lane < br)
        {
            v0 = x[r0 + lane] - (part[lane][0] + part[lane][1] + part[lane][2] + part[lane][3]);
        }
        if (lane + 32 < br)
        {
            const int i = lane + 32;
            v1          = x[r0 + i] - (part[i][0] + part[i][1] + part[i][2] + part[i][3]);
        }
        if (!upper)
        {
            for (int p = 0; p < br; ++p)
            {
                TX xp;
                if (p < 32)
                {
                    TX mine = v0;
                    if (!unit && lane == p)
                    {
                        mine = v0 / tri[p][p];
                        v0   = mine;
                    }
                    xp = __shfl_sync(0xffffffffu, mine, p);
                }
                else
                {
                    TX mine = v1;
                    if (!unit && lane == p - 32)
                    {
                        mine = v1 / tri[p][p];
                        v1   = mine;
                    }
                    xp = __shfl_sync(0xffffffffu, mine, p - 32);
                }
                if (lane > p && lane < br)
                {
                    v0 = fma(-tri[lane][p], xp, v0);
                }
                if (lane + 32 > p && lane + 32 < br)
                {
                    v1 = fma(-tri[lane + 32][p], xp, v1);
                }
            }
        }
        else
        {
            for (int p = br - 1; p >= 0; --p)
            {
                TX xp;
                if (p < 32)
                {
                    TX mine = v0;
                    if (!unit && lane == p)
                    {
                        mine = v0 / tri[p][p];
                        v0   = mine;
                    }
                    xp = __shfl_sync(0xffffffffu, mine, p);
                }
                else
                {
                    TX mine = v1;
                    if (!unit && lane == p - 32)
                    {
                        mine = v1 / tri[p][p];
                        v1   = mine;
                    }
                    xp = __shfl_sync(0xffffffffu, mine, p - 32);
                }
                if (lane < p)
                {
                    v0 = fma(-tri[lane][p], xp, v0);
                }
                if (lane + 32 < p)
                {
                    v1 = fma(-tri[lane + 32][p], xp, v1);
                }
            }
        }
        if (lane < br)
        {
            x[r0 + lane] = v0;
        }
        if (lane + 32 < br)
        {
            x[r0 + lane + 32] = v1;
        }
        __syncwarp();
        if (lane == 0)
        {
            __threadfence();
            st_release_u32(&sync->flags[blk], 1u);
        }
    }
}

}  // namespace b200la
