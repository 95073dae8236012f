// Shared definitions for the B200 LU-solve kernels: status words, the
// workspace arena, bounded device-side waits and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

#include "../../include/b200la.h"

namespace b200la
{

// ---------------------------------------------------------------------------
// Device status block.  Every operation that can fail on the device carves
// one of these at offset 0 of its workspace.  Kernels only ever raise
// `error` (first error wins, atomicCAS from 0); the host reads the block back
// when it synchronizes (lu_decomposition) or on request
// (b200la_workspace_status).
// ---------------------------------------------------------------------------
enum DeviceError : int32_t
{
    DEV_OK           = 0,
    DEV_WAIT_TIMEOUT = 1,  // a bounded inter-CTA wait gave up
    DEV_BAD_PIVOT    = 2,  // a pivot entry outside [i+1, n] was supplied
    DEV_BAD_INPUT    = 3,  // a launch broke a kernel's precondition (the kernel skipped the work)
};

struct alignas(64) DeviceStatus
{
    int32_t error;       // DeviceError
    int32_t error_site;  // which wait / check raised it
    int64_t first_zero;  // 0-based index of the first exactly-zero pivot, -1 if none
    int64_t info;        // LAPACK-style info = first_zero + 1 (written at the end)
    int64_t pad[5];
};

// Wall-clock bound for every spin-wait on another CTA: 2 s.  A wait that
// runs out sets DeviceStatus::error and the kernel returns.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void raise_error(DeviceStatus* st, int32_t code, int32_t site)
{
    if (atomicCAS(&st->error, 0, code) == 0)
    {
        st->error_site = site;
    }
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int32_t ld_volatile_i32(const int32_t* p)
{
    return *reinterpret_cast<const volatile int32_t*>(p);
}

// ---------------------------------------------------------------------------
// Shared-memory mbarriers (TMA copies and tensor-core commits complete on
// them).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
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
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on an mbarrier phase; false when the 2 s limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity))
    {
        return true;
    }
    const uint64_t t0    = global_ns();
    uint32_t       polls = 0;
    while (!mbar_try_wait(bar, parity))
    {
        if ((++polls & 255u) == 0 && global_ns() - t0 > kWaitLimitNs)
        {
            return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Host-side workspace arena: the same carve order computes the size (base ==
// nullptr) and the real pointers, so size queries and carving cannot drift
// apart.  256-byte alignment for every carve (TMA and vector access safe).
// ---------------------------------------------------------------------------
class Arena
{
public:
    Arena() : base_(nullptr), cap_(0), sizing_(true) {}
    Arena(void* base, size_t cap) : base_(static_cast<unsigned char*>(base)), cap_(cap), sizing_(false) {}

    template <typename T> T* next(size_t count, size_t align = 256)
    {
        const size_t off = (off_ + align - 1) / align * align;
        off_             = off + sizeof(T) * count;
        if (sizing_)
        {
            return nullptr;
        }
        if (off_ > cap_)
        {
            overflow_ = true;
            return nullptr;
        }
        return reinterpret_cast<T*>(base_ + off);
    }
    size_t size() const { return off_; }
    bool   overflow() const { return overflow_; }

private:
    unsigned char* base_;
    size_t         cap_;
    size_t         off_      = 0;
    bool           sizing_;
    bool           overflow_ = false;
};

// Kernel classes of the launch recorder (b200la_profile_start/stop).
enum KernelClass : int
{
    KC_PANEL    = 0,
    KC_SWAP     = 1,
    KC_TRAILING = 2,
    KC_SOLVE    = 3,
    KC_GEMM     = 4,
    KC_MIXED    = 5,
    KC_RESIDUAL = 6,
    KC_BATCHED  = 7,
    KC_PREP     = 8,
    KC_SELECT   = 9,
    KC_INV_GEMM = 10,  // inversion: the blocked substitutions' GEMM updates
    KC_INV_AUX  = 11,  // inversion / determinant: identity, column gather, diagonal product
    KC_CHOL_UPD = 12,  // Cholesky: the trailing lower-triangle updates
    KC_CHOL_AUX = 13,  // Cholesky: diagonal blocks, panel solves, zeroing, transposition
    KC_TRANSPOSE = 14, // transpose and the out-of-place interop copy
    KC_COUNT    = 15
};

// Host helpers shared by the entry points (defined in runtime.cu).
void prof_begin(int cls, cudaStream_t s);  // records an event if class `cls` is being profiled
void prof_end(int cls, cudaStream_t s);    // closes it and counts one launch of the library
int  device_sm_count();
int  set_error(int status, const char* fmt, ...);
int  cuda_check(cudaError_t e, const char* what);

#define B200LA_CUDA(call)                                                                          \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
        {                                                                                          \
            return ::b200la::cuda_check(e_, #call);                                                \
        }                                                                                          \
    } while (0)

#define B200LA_LAUNCH_CHECK()                                                                      \
    do                                                                                             \
    {                                                                                              \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess)                                                                     \
        {                                                                                          \
            return ::b200la::cuda_check(e_, "kernel launch");                                      \
        }                                                                                          \
    } while (0)

}  // namespace b200la
