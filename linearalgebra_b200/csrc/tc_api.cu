// Host side of the tcgen05 update: TMA tensor maps (driver entry point
// cuTensorMapEncodeTiled, resolved through the runtime so the library does not
// link libcuda directly) and launches.
#include <cuda.h>
#include <cuda_runtime.h>

#include <climits>
#include <cstdlib>
#include <mutex>

#include "tc_api.cuh"

namespace b200la
{
int require_sm100();

namespace
{
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static std::mutex    m;
    static EncodeTiledFn fn = nullptr;
    std::lock_guard<std::mutex> lock(m);
    if (fn == nullptr)
    {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
        {
            fn = reinterpret_cast<EncodeTiledFn>(p);
        }
    }
    return fn;
}

template <int KIND, bool SPLIT3> int set_attr_once()
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
    B200LA_CUDA(cudaFuncSetAttribute(k_tc_update<KIND, SPLIT3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)tc_smem_bytes<SPLIT3>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_tc_update_persistent<KIND, SPLIT3>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tcp_smem_bytes<SPLIT3>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_tc_update_persistent<KIND, SPLIT3>,
        cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (dev >= 0 && dev < 64)
    {
        done[dev] = true;
    }
    return B200LA_SUCCESS;
}
}  // namespace

int make_kmajor_map(CUtensorMap* map, const void* base, int kind, int64_t rows, int64_t k, int64_t ld,
    int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (fn == nullptr)
    {
        return set_error(B200LA_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
    }
    const int                elem  = tc_elem_bytes(kind);
    const CUtensorMapDataType dt   = kind == TC_TF32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                    : kind == TC_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                    : kind == TC_FP16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                      : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (ld * elem) % 16 != 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tensor-core operand not 16-byte aligned");
    }
    cuuint64_t dims[2]    = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * elem)};
    cuuint32_t box[2]     = {(cuuint32_t)(kTcAtomBytes / elem), (cuuint32_t)box_rows};
    cuuint32_t estr[2]    = {1, 1};
    const CUresult r = fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
    {
        return set_error(B200LA_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    }
    return B200LA_SUCCESS;
}

// B200LA_TC_PERSISTENT=0 launches one CTA per tile (k_tc_update) instead of
// the persistent kernel (same per-element arithmetic).
static bool tc_persistent_enabled()
{
    const char* e = getenv("B200LA_TC_PERSISTENT");
    return !(e != nullptr && e[0] == '0');
}

// Clusters of `cl` persistent-update CTAs that fit the device at once (0 if
// the query fails), per device.
template <int KIND, bool SPLIT3> int tc_active_clusters(int cl)
{
    static std::mutex m;
    static int        known[64][17] = {};
    int               dev           = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || cl < 2 || cl > 16)
    {
        return 0;
    }
    std::lock_guard<std::mutex> lock(m);
    if (known[dev][cl] == 0)
    {
        cudaLaunchConfig_t  cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim              = dim3(cl);
        cfg.blockDim             = dim3(kTcpThreads);
        cfg.dynamicSmemBytes     = tcp_smem_bytes<SPLIT3>();
        attr[0].id               = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs                = attr;
        cfg.numAttrs             = 1;
        int count                = 0;
        if (cudaOccupancyMaxActiveClusters(&count, (const void*)k_tc_update_persistent<KIND, SPLIT3>, &cfg) !=
            cudaSuccess)
        {
            cudaGetLastError();
            count = -1;
        }
        known[dev][cl] = count;
    }
    return known[dev][cl] > 0 ? known[dev][cl] : 0;
}

template <int KIND, bool SPLIT3>
static int launch_tc(const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& as, const CUtensorMap& bs,
    float* c, int64_t ldc, int m, int n, int k, DeviceStatus* st, const float* inv_sa, const float* inv_sb,
    cudaStream_t s, int max_ctas, int place_cluster)
{
    int rc = set_attr_once<KIND, SPLIT3>();
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    const int tiles = ((n + kTcBN - 1) / kTcBN) * ((m + kTcBM - 1) / kTcBM);
    if (tc_persistent_enabled())
    {
        const int sms = device_sm_count();
        // B200LA_TC_CTAS caps the persistent grid (the tests use it to make
        // every CTA walk many tiles)
        const char* cap = getenv("B200LA_TC_CTAS");
        if (cap != nullptr && atoi(cap) > 0)
        {
            max_ctas = max_ctas > 0 && max_ctas < atoi(cap) ? max_ctas : atoi(cap);
        }
        int g = max_ctas > 0 && max_ctas < sms ? max_ctas : sms;
        g             = g < tiles ? g : tiles;
        int ncl = 0;  // clusters of the placed launch
        if (place_cluster > 1)
        {
            const int cap = g / place_cluster;
            ncl           = tc_active_clusters<KIND, SPLIT3>(place_cluster) - 1;  // leave one GPC free
            ncl           = ncl < cap ? ncl : cap;
        }
        if (ncl >= 1)
        {
            cudaLaunchConfig_t  cfg = {};
            cudaLaunchAttribute attr[1];
            cfg.gridDim              = dim3(ncl * place_cluster);
            cfg.blockDim             = dim3(kTcpThreads);
            cfg.dynamicSmemBytes     = tcp_smem_bytes<SPLIT3>();
            cfg.stream               = s;
            attr[0].id               = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = place_cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs                = attr;
            cfg.numAttrs             = 1;
            prof_begin(KC_MIXED, s);
            B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_tc_update_persistent<KIND, SPLIT3>, a, b, as, bs, c, ldc, m, n,
                k, st, inv_sa, inv_sb));
            prof_end(KC_MIXED, s);
            return B200LA_SUCCESS;
        }
        prof_begin(KC_MIXED, s);
        k_tc_update_persistent<KIND, SPLIT3><<<g, kTcpThreads, tcp_smem_bytes<SPLIT3>(), s>>>(a, b, as, bs, c, ldc,
            m, n, k, st, inv_sa, inv_sb);
        prof_end(KC_MIXED, s);
        B200LA_LAUNCH_CHECK();
        return B200LA_SUCCESS;
    }
    dim3 grid((n + kTcBN - 1) / kTcBN, (m + kTcBM - 1) / kTcBM);
    prof_begin(KC_MIXED, s);
    k_tc_update<KIND, SPLIT3><<<grid, 128, tc_smem_bytes<SPLIT3>(), s>>>(a, b, as, bs, c, ldc, m, n, k, st, inv_sa,
        inv_sb);
    prof_end(KC_MIXED, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

int enqueue_tc_update(int kind, bool split3, const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& as,
    const CUtensorMap& bs, float* c, int64_t ldc, int m, int n, int k, DeviceStatus* st, cudaStream_t s,
    const float* inv_sa, const float* inv_sb, int max_ctas, int place_cluster)
{
    if (m <= 0 || n <= 0)
    {
        return B200LA_SUCCESS;
    }
    const int ea = kTcAtomBytes / tc_elem_bytes(kind);
    if (k <= 0 || k % ea != 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tensor-core update: depth %d is not a multiple of %d", k, ea);
    }
    if (kind == TC_TF32)
    {
        return split3 ? launch_tc<TC_TF32, true>(a, b, as, bs, c, ldc, m, n, k, st, nullptr, nullptr, s, max_ctas, place_cluster)
                      : launch_tc<TC_TF32, false>(a, b, as, bs, c, ldc, m, n, k, st, nullptr, nullptr, s, max_ctas, place_cluster);
    }
    if (split3)
    {
        return set_error(B200LA_NOT_SUPPORTED, "the three-term split is provided for TF32 only");
    }
    if (kind == TC_BF16)
    {
        return launch_tc<TC_BF16, false>(a, b, as, bs, c, ldc, m, n, k, st, nullptr, nullptr, s, max_ctas, place_cluster);
    }
    if (kind == TC_FP8)
    {
        if (inv_sa == nullptr || inv_sb == nullptr)
        {
            return set_error(B200LA_INVALID_ARGUMENT, "tensor-core update: FP8 operands need their scales");
        }
        return launch_tc<TC_FP8, false>(a, b, as, bs, c, ldc, m, n, k, st, inv_sa, inv_sb, s, max_ctas, place_cluster);
    }
    return launch_tc<TC_FP16, false>(a, b, as, bs, c, ldc, m, n, k, st, nullptr, nullptr, s, max_ctas, place_cluster);
}

}  // namespace b200la

using namespace b200la;

extern "C" B200LA_API int b200la_sgemm_tc_update(int kind, int split3, float* c, int64_t ldc, int64_t m,
    int64_t n, int64_t k, const void* a, const void* b, const void* a_small, const void* b_small,
    void* workspace, size_t workspace_bytes, void* stream)
{
    if (c == nullptr || a == nullptr || b == nullptr || (split3 && (a_small == nullptr || b_small == nullptr)))
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tc_update: null operand");
    }
    if (kind < TC_TF32 || kind > TC_FP16 || m <= 0 || n <= 0 || k <= 0 || ldc < n || m > INT_MAX / 2 ||
        n > INT_MAX / 2 || k > INT_MAX / 2)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tc_update: invalid kind or sizes");
    }
    if (workspace == nullptr || workspace_bytes < sizeof(DeviceStatus))
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "tc_update: needs %zu bytes of workspace",
            sizeof(DeviceStatus));
    }
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    CUtensorMap ma, mb, mas, mbs;
    if ((rc = make_kmajor_map(&ma, a, kind, m, k, k, kTcBM)) != B200LA_SUCCESS ||
        (rc = make_kmajor_map(&mb, b, kind, n, k, k, kTcBN)) != B200LA_SUCCESS)
    {
        return rc;
    }
    mas = ma;
    mbs = mb;
    if (split3 && ((rc = make_kmajor_map(&mas, a_small, kind, m, k, k, kTcBM)) != B200LA_SUCCESS ||
                      (rc = make_kmajor_map(&mbs, b_small, kind, n, k, k, kTcBN)) != B200LA_SUCCESS))
    {
        return rc;
    }
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    auto*        st = static_cast<DeviceStatus*>(workspace);
    B200LA_CUDA(cudaMemsetAsync(st, 0, sizeof(DeviceStatus), s));
    return enqueue_tc_update(kind, split3 != 0, ma, mb, mas, mbs, c, ldc, (int)m, (int)n, (int)k, st, s);
}

extern "C" B200LA_API size_t b200la_tc_update_workspace_size(void) { return sizeof(DeviceStatus); }

extern "C" B200LA_API int b200la_sgemm_tc_update_fp8(float* c, int64_t ldc, int64_t m, int64_t n, int64_t k,
    const void* a, const void* b, const float* a_inv_scale, const float* b_inv_scale, void* workspace,
    size_t workspace_bytes, void* stream)
{
    if (c == nullptr || a == nullptr || b == nullptr || a_inv_scale == nullptr || b_inv_scale == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tc_update_fp8: null operand");
    }
    if (m <= 0 || n <= 0 || k <= 0 || ldc < n || m > INT_MAX / 2 || n > INT_MAX / 2 || k > INT_MAX / 2)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "tc_update_fp8: invalid sizes");
    }
    if (workspace == nullptr || workspace_bytes < sizeof(DeviceStatus))
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "tc_update_fp8: needs %zu bytes of workspace",
            sizeof(DeviceStatus));
    }
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    CUtensorMap ma, mb;
    if ((rc = make_kmajor_map(&ma, a, TC_FP8, m, k, k, kTcBM)) != B200LA_SUCCESS ||
        (rc = make_kmajor_map(&mb, b, TC_FP8, n, k, k, kTcBN)) != B200LA_SUCCESS)
    {
        return rc;
    }
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    auto*        st = static_cast<DeviceStatus*>(workspace);
    B200LA_CUDA(cudaMemsetAsync(st, 0, sizeof(DeviceStatus), s));
    return enqueue_tc_update(TC_FP8, false, ma, mb, ma, mb, c, ldc, (int)m, (int)n, (int)k, st, s, a_inv_scale,
        b_inv_scale);
}
