// transpose<T, B200>: the device-resident transpose and the row-major <->
// column-major interop of include/matrix_operation/transpose.h.
//
// transpose::apply(rows, columns, m, ...) turns the row-major rows x columns
// matrix in m into its row-major columns x rows transpose, in place.  The
// reference's CUDA_BLAS version (src/matrix_operation/gpu/cublas/
// transpose_cublas.cpp:25-57) runs an out-of-place cuBLAS geam into a
// scratch copy and copies it back (32 bytes of HBM traffic per 8-byte
// element); its NATIVE version (transpose_native.cpp) swaps 32 x 32 tile
// pairs for a square matrix and follows permutation cycles otherwise.
//
// Here:
//   square   k_transpose_square, in place without workspace: one CTA per
//            pair of mirrored 64 x 64 tiles (I, J), I >= J, both tiles staged
//            in shared memory, each written back as the other's transpose
//            (16 bytes of traffic per 8-byte element: one read, one write);
//   other    k_transpose_out from m into the workspace (rows x columns
//            elements), then one device-to-device copy back (32 bytes per
//            element, as the reference's path);
//   interop  b200la_{d,s}transpose_out: the out-of-place transpose into a
//            caller buffer, the same kernel, for callers that hold a
//            row-major matrix and need the column-major layout (or back)
//            without the in-place copy.
// Both kernels read and write whole 64-element rows of their tiles
// (coalesced) and read the staged tiles by columns through a padded
// row pitch (65 elements: no shared-memory bank conflicts).  The result is
// pure data movement, equal to the reference's bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace b200la
{
int require_sm100();

namespace tp
{

constexpr int kTile    = 64;
constexpr int kThreads = 256;
constexpr int kRowsPer = kThreads / kTile;  // tile rows one pass of the CTA covers

template <typename T> constexpr size_t pair_smem_bytes() { return sizeof(T) * 2 * kTile * (kTile + 1); }
template <typename T> constexpr size_t tile_smem_bytes() { return sizeof(T) * kTile * (kTile + 1); }

// Element copy global -> shared without a register round trip, so a CTA
// has all of its tile loads in flight before it waits.
template <int BYTES> __device__ __forceinline__ void cp_async(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Tile pair b of the lower triangle of tiles, row by row: (I, J), J <= I.
__device__ __forceinline__ void tri_pair(int64_t b, int64_t& I, int64_t& J)
{
    int64_t i = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (i * (i + 1) / 2 > b)
    {
        --i;
    }
    while ((i + 1) * (i + 2) / 2 <= b)
    {
        ++i;
    }
    I = i;
    J = b - i * (i + 1) / 2;
}

// Square n x n matrix, in place: tile (I, J) <- tile (J, I)^T and back.
template <typename T> __global__ void __launch_bounds__(kThreads) k_transpose_square(T* __restrict__ m, int64_t n)
{
    extern __shared__ __align__(16) unsigned char tp_smem[];
    T(*a)[kTile + 1] = reinterpret_cast<T(*)[kTile + 1]>(tp_smem);
    T(*b)[kTile + 1] = a + kTile;
    int64_t I, J;
    tri_pair(blockIdx.x, I, J);
    const int64_t r0 = I * kTile, c0 = J * kTile;
    const bool    diag = I == J;
    const int     c    = threadIdx.x % kTile;
    const int     rb   = threadIdx.x / kTile;
#pragma unroll
    for (int q = 0; q < kTile / kRowsPer; ++q)
    {
        const int r = rb + kRowsPer * q;
        if (r0 + r < n && c0 + c < n)
        {
            cp_async<sizeof(T)>(&a[r][c], m + (r0 + r) * n + c0 + c);
        }
        if (!diag && c0 + r < n && r0 + c < n)
        {
            cp_async<sizeof(T)>(&b[r][c], m + (c0 + r) * n + r0 + c);
        }
    }
    cp_async_wait_all();
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < kTile / kRowsPer; ++q)
    {
        const int r = rb + kRowsPer * q;
        if (diag)
        {
            if (r0 + r < n && r0 + c < n)
            {
                m[(r0 + r) * n + r0 + c] = a[c][r];
            }
            continue;
        }
        if (r0 + r < n && c0 + c < n)
        {
            m[(r0 + r) * n + c0 + c] = b[c][r];
        }
        if (c0 + r < n && r0 + c < n)
        {
            m[(c0 + r) * n + r0 + c] = a[c][r];
        }
    }
}

// dst (columns x rows, row-major) = src (rows x columns, row-major)^T; one
// CTA per 64 x 64 tile of src, tiles enumerated column tile fastest.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_transpose_out(const T* __restrict__ src, T* __restrict__ dst,
    int64_t rows, int64_t columns, int64_t col_tiles)
{
    extern __shared__ __align__(16) unsigned char tp_smem[];
    T(*a)[kTile + 1] = reinterpret_cast<T(*)[kTile + 1]>(tp_smem);
    const int64_t I  = blockIdx.x / col_tiles, J = blockIdx.x - (blockIdx.x / col_tiles) * col_tiles;
    const int64_t r0 = I * kTile, c0 = J * kTile;
    const int     c  = threadIdx.x % kTile;
    const int     rb = threadIdx.x / kTile;
#pragma unroll
    for (int q = 0; q < kTile / kRowsPer; ++q)
    {
        const int r = rb + kRowsPer * q;
        if (r0 + r < rows && c0 + c < columns)
        {
            cp_async<sizeof(T)>(&a[r][c], src + (r0 + r) * columns + c0 + c);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // dst row c0 + r (a column of src) holds src[r0 .. r0 + 64)[c0 + r]
#pragma unroll 4
    for (int q = 0; q < kTile / kRowsPer; ++q)
    {
        const int r = rb + kRowsPer * q;
        if (c0 + r < columns && r0 + c < rows)
        {
            dst[(c0 + r) * rows + r0 + c] = a[c][r];
        }
    }
}

template <typename T> int ensure_attributes()
{
    static std::mutex m;
    static bool       done[64] = {};
    int               dev      = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(m);
    if (dev >= 0 && dev < 64 && done[dev])
    {
        return B200LA_SUCCESS;
    }
    B200LA_CUDA(cudaFuncSetAttribute(k_transpose_square<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)pair_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_transpose_out<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)tile_smem_bytes<T>()));
    if (dev >= 0 && dev < 64)
    {
        done[dev] = true;
    }
    return B200LA_SUCCESS;
}

// Grids above this many CTAs are not needed for any matrix that fits a
// device (a 64 x 64 tile per CTA); larger requests are refused.
constexpr int64_t kMaxGrid = (int64_t)INT32_MAX;

template <typename T> size_t ws_size(int64_t rows, int64_t columns)
{
    if (rows <= 0 || columns <= 0 || rows == columns)
    {
        return 0;
    }
    Arena a;
    a.next<T>((size_t)rows * (size_t)columns);
    return a.size();
}

template <typename T> int check_shape(int64_t rows, int64_t columns)
{
    if (rows <= 0 || columns <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "transpose::apply: rows and columns must be positive");
    }
    const int64_t rt = (rows + kTile - 1) / kTile, ct = (columns + kTile - 1) / kTile;
    if (rt > kMaxGrid / ct)
    {
        return set_error(B200LA_NOT_SUPPORTED, "transpose: matrix too large");
    }
    return B200LA_SUCCESS;
}

template <typename T> int launch_out(const T* src, T* dst, int64_t rows, int64_t columns, cudaStream_t s)
{
    const int64_t rt = (rows + kTile - 1) / kTile, ct = (columns + kTile - 1) / kTile;
    prof_begin(KC_TRANSPOSE, s);
    k_transpose_out<T><<<(unsigned)(rt * ct), kThreads, tile_smem_bytes<T>(), s>>>(src, dst, rows, columns, ct);
    prof_end(KC_TRANSPOSE, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T> int transpose(int64_t rows, int64_t columns, T* m, void* ws, size_t bytes, void* stream)
{
    if (m == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "transpose::apply: m must not be null");
    }
    int st = check_shape<T>(rows, columns);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    const size_t need = ws_size<T>(rows, columns);
    if (need > 0 && (ws == nullptr || bytes < need))
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "transpose: workspace is null or too small (%zu < %zu bytes)",
            bytes, need);
    }
    st = require_sm100();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    st = ensure_attributes<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (rows == columns)
    {
        const int64_t t = (rows + kTile - 1) / kTile;
        prof_begin(KC_TRANSPOSE, s);
        k_transpose_square<T><<<(unsigned)(t * (t + 1) / 2), kThreads, pair_smem_bytes<T>(), s>>>(m, rows);
        prof_end(KC_TRANSPOSE, s);
        B200LA_LAUNCH_CHECK();
        return B200LA_SUCCESS;
    }
    Arena a(ws, bytes);
    T*    scratch = a.next<T>((size_t)rows * (size_t)columns);
    st            = launch_out<T>(m, scratch, rows, columns, s);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    B200LA_CUDA(cudaMemcpyAsync(m, scratch, sizeof(T) * (size_t)rows * (size_t)columns, cudaMemcpyDeviceToDevice, s));
    return B200LA_SUCCESS;
}

template <typename T> int transpose_out(int64_t rows, int64_t columns, const T* src, T* dst, void* stream)
{
    if (src == nullptr || dst == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "transpose: src and dst must not be null");
    }
    int st = check_shape<T>(rows, columns);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    const uintptr_t s0 = (uintptr_t)src, d0 = (uintptr_t)dst, len = sizeof(T) * (uintptr_t)rows * (uintptr_t)columns;
    if (s0 < d0 + len && d0 < s0 + len)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "transpose: src and dst must not overlap");
    }
    st = require_sm100();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    st = ensure_attributes<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return launch_out<T>(src, dst, rows, columns, static_cast<cudaStream_t>(stream));
}

}  // namespace tp
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dtranspose_workspace_size(int64_t rows, int64_t columns)
{
    return tp::ws_size<double>(rows, columns);
}
B200LA_API size_t b200la_stranspose_workspace_size(int64_t rows, int64_t columns)
{
    return tp::ws_size<float>(rows, columns);
}
B200LA_API int b200la_dtranspose(int64_t rows, int64_t columns, double* m, void* ws, size_t bytes, void* stream)
{
    return tp::transpose<double>(rows, columns, m, ws, bytes, stream);
}
B200LA_API int b200la_stranspose(int64_t rows, int64_t columns, float* m, void* ws, size_t bytes, void* stream)
{
    return tp::transpose<float>(rows, columns, m, ws, bytes, stream);
}
B200LA_API int b200la_dtranspose_out(int64_t rows, int64_t columns, const double* src, double* dst, void* stream)
{
    return tp::transpose_out<double>(rows, columns, src, dst, stream);
}
B200LA_API int b200la_stranspose_out(int64_t rows, int64_t columns, const float* src, float* dst, void* stream)
{
    return tp::transpose_out<float>(rows, columns, src, dst, stream);
}

}  // extern "C"
