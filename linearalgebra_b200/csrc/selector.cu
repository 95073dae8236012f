// Learned precision selector: a 12 -> 64 -> 64 -> 4 MLP (ReLU, softmax
// cross-entropy), FP32, with hand-written inference, training (forward +
// backward) and Adam kernels, and the kernels that gather the matrix
// statistics its features are made of.
//
// Parameter vector (5252 floats): W1[12][64] | b1[64] | W2[64][64] | b2[64] |
// W3[64][4] | b3[4]; y = relu(x W1 + b1), z = relu(y W2 + b2),
// logits = z W3 + b3.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace b200la
{
namespace
{
constexpr int kIn = 12, kH = 64, kOut = 4;
constexpr int kOffW1 = 0, kOffB1 = kIn * kH, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kOut, kParams = kOffB3 + kOut;
static_assert(kParams == 5252, "parameter count");
constexpr int kMlpThreads = 128;

__device__ __forceinline__ void mlp_forward(const float* p, const float* x, float* h1, float* h2, float* logits)
{
    for (int j = 0; j < kH; ++j)
    {
        float s = p[kOffB1 + j];
        for (int i = 0; i < kIn; ++i)
        {
            s = fmaf(x[i], p[kOffW1 + i * kH + j], s);
        }
        h1[j] = fmaxf(s, 0.f);
    }
    for (int j = 0; j < kH; ++j)
    {
        float s = p[kOffB2 + j];
        for (int i = 0; i < kH; ++i)
        {
            s = fmaf(h1[i], p[kOffW2 + i * kH + j], s);
        }
        h2[j] = fmaxf(s, 0.f);
    }
    for (int k = 0; k < kOut; ++k)
    {
        float s = p[kOffB3 + k];
        for (int i = 0; i < kH; ++i)
        {
            s = fmaf(h2[i], p[kOffW3 + i * kOut + k], s);
        }
        logits[k] = s;
    }
}

// probs[b][4] = softmax(MLP(x_b)), one thread per sample, parameters in
// shared memory.
__global__ void __launch_bounds__(kMlpThreads) k_mlp_forward(const float* __restrict__ params,
    const float* __restrict__ X, int batch, float* __restrict__ probs)
{
    __shared__ float p[kParams];
    for (int i = threadIdx.x; i < kParams; i += kMlpThreads)
    {
        p[i] = params[i];
    }
    __syncthreads();
    const int b = blockIdx.x * kMlpThreads + threadIdx.x;
    if (b >= batch)
    {
        return;
    }
    float x[kIn], h1[kH], h2[kH], lg[kOut];
    for (int i = 0; i < kIn; ++i)
    {
        x[i] = X[(size_t)b * kIn + i];
    }
    mlp_forward(p, x, h1, h2, lg);
    float m = lg[0];
    for (int k = 1; k < kOut; ++k)
    {
        m = fmaxf(m, lg[k]);
    }
    float z = 0.f;
    for (int k = 0; k < kOut; ++k)
    {
        lg[k] = expf(lg[k] - m);
        z += lg[k];
    }
    for (int k = 0; k < kOut; ++k)
    {
        probs[(size_t)b * kOut + k] = lg[k] / z;
    }
}

// Forward + backward of the summed softmax cross-entropy: grads +=
// d(loss_sum)/d(params), loss_sum += sum of the per-sample losses.  A CTA
// takes kGradSamples samples in two phases:
//   1. thread = sample: forward, softmax, and the backward deltas
//      dl = p - onehot(y), dh2 = (W3 dl) * [h2 > 0], dh1 = (W2 dh2) * [h1 > 0],
//      written with the activations to shared memory as [unit][sample]
//      (row stride kGradSamples + 1, so a warp reading one sample column of
//      consecutive units hits distinct banks);
//   2. thread = parameter (strided): dW1 = x^T dh1, dW2 = h1^T dh2,
//      dW3 = h2^T dl and the bias sums over the CTA's samples, in a fixed
//      order, then one global atomic add per parameter per CTA.
// Samples past `batch` contribute zeros.
constexpr int kGradSamples = 128;
constexpr int kGradLd      = kGradSamples + 1;
constexpr int kGradUnits   = kIn + kH + kH + kOut + kH + kH;  // x h1 h2 dl dh2 dh1
constexpr size_t grad_smem_bytes() { return sizeof(float) * ((size_t)kParams + (size_t)kGradUnits * kGradLd); }

__global__ void __launch_bounds__(kGradSamples) k_mlp_grad(const float* __restrict__ params,
    const float* __restrict__ X, const int32_t* __restrict__ labels, int batch, float* __restrict__ grads,
    float* __restrict__ loss_sum)
{
    extern __shared__ float gsm[];
    float* p   = gsm;
    float* xs  = p + kParams;           // [kIn][kGradLd]
    float* h1s = xs + kIn * kGradLd;    // [kH]
    float* h2s = h1s + kH * kGradLd;    // [kH]
    float* dls = h2s + kH * kGradLd;    // [kOut]
    float* d2s = dls + kOut * kGradLd;  // [kH] dh2
    float* d1s = d2s + kH * kGradLd;    // [kH] dh1
    const int t = threadIdx.x;
    for (int i = t; i < kParams; i += kGradSamples)
    {
        p[i] = params[i];
    }
    __syncthreads();

    // phase 1: thread = sample
    const int  b     = blockIdx.x * kGradSamples + t;
    const bool valid = b < batch;
    for (int i = 0; i < kIn; ++i)
    {
        xs[i * kGradLd + t] = valid ? X[(size_t)b * kIn + i] : 0.f;
    }
    for (int j = 0; j < kH; ++j)
    {
        float acc = p[kOffB1 + j];
        for (int i = 0; i < kIn; ++i)
        {
            acc = fmaf(xs[i * kGradLd + t], p[kOffW1 + i * kH + j], acc);
        }
        h1s[j * kGradLd + t] = valid ? fmaxf(acc, 0.f) : 0.f;
    }
    for (int j = 0; j < kH; ++j)
    {
        float acc = p[kOffB2 + j];
        for (int i = 0; i < kH; ++i)
        {
            acc = fmaf(h1s[i * kGradLd + t], p[kOffW2 + i * kH + j], acc);
        }
        h2s[j * kGradLd + t] = valid ? fmaxf(acc, 0.f) : 0.f;
    }
    float lg[kOut];
    for (int k = 0; k < kOut; ++k)
    {
        float acc = p[kOffB3 + k];
        for (int i = 0; i < kH; ++i)
        {
            acc = fmaf(h2s[i * kGradLd + t], p[kOffW3 + i * kOut + k], acc);
        }
        lg[k] = acc;
    }
    float m = lg[0];
    for (int k = 1; k < kOut; ++k)
    {
        m = fmaxf(m, lg[k]);
    }
    float z = 0.f;
    for (int k = 0; k < kOut; ++k)
    {
        lg[k] = expf(lg[k] - m);
        z += lg[k];
    }
    const int y    = valid ? labels[b] : 0;
    float     loss = valid ? -logf(fmaxf(lg[y] / z, 1e-30f)) : 0.f;
    for (int k = 0; k < kOut; ++k)
    {
        dls[k * kGradLd + t] = valid ? lg[k] / z - (k == y ? 1.f : 0.f) : 0.f;
    }
    for (int i = 0; i < kH; ++i)
    {
        float acc = 0.f;
        for (int k = 0; k < kOut; ++k)
        {
            acc = fmaf(p[kOffW3 + i * kOut + k], dls[k * kGradLd + t], acc);
        }
        d2s[i * kGradLd + t] = h2s[i * kGradLd + t] > 0.f ? acc : 0.f;
    }
    for (int i = 0; i < kH; ++i)
    {
        float acc = 0.f;
        for (int j = 0; j < kH; ++j)
        {
            acc = fmaf(p[kOffW2 + i * kH + j], d2s[j * kGradLd + t], acc);
        }
        d1s[i * kGradLd + t] = h1s[i * kGradLd + t] > 0.f ? acc : 0.f;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        loss += __shfl_down_sync(0xffffffffu, loss, off);
    }
    if ((t & 31) == 0 && loss != 0.f)
    {
        atomicAdd(loss_sum, loss);
    }
    __syncthreads();

    // phase 2: thread = parameter
    for (int q = t; q < kParams; q += kGradSamples)
    {
        const float* u;  // left factor row (nullptr: bias, sum of v)
        const float* v;
        if (q < kOffB1)
        {
            u = xs + (q / kH) * kGradLd;
            v = d1s + (q % kH) * kGradLd;
        }
        else if (q < kOffW2)
        {
            u = nullptr;
            v = d1s + (q - kOffB1) * kGradLd;
        }
        else if (q < kOffB2)
        {
            u = h1s + ((q - kOffW2) / kH) * kGradLd;
            v = d2s + ((q - kOffW2) % kH) * kGradLd;
        }
        else if (q < kOffW3)
        {
            u = nullptr;
            v = d2s + (q - kOffB2) * kGradLd;
        }
        else if (q < kOffB3)
        {
            u = h2s + ((q - kOffW3) / kOut) * kGradLd;
            v = dls + ((q - kOffW3) % kOut) * kGradLd;
        }
        else
        {
            u = nullptr;
            v = dls + (q - kOffB3) * kGradLd;
        }
        float acc = 0.f;
        if (u != nullptr)
        {
#pragma unroll 8
            for (int s2 = 0; s2 < kGradSamples; ++s2)
            {
                acc = fmaf(u[s2], v[s2], acc);
            }
        }
        else
        {
#pragma unroll 8
            for (int s2 = 0; s2 < kGradSamples; ++s2)
            {
                acc += v[s2];
            }
        }
        if (acc != 0.f)
        {
            atomicAdd(&grads[q], acc);
        }
    }
}

// Adam on the mean gradient (grads / batch); clears grads.
__global__ void k_adam(float* __restrict__ params, float* __restrict__ grads, float* __restrict__ m1,
    float* __restrict__ m2, float inv_batch, float lr, float beta1, float beta2, float eps, int step,
    float weight_decay)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams)
    {
        return;
    }
    const float gr = grads[i] * inv_batch + weight_decay * params[i];
    grads[i]       = 0.f;
    m1[i]          = beta1 * m1[i] + (1.f - beta1) * gr;
    m2[i]          = beta2 * m2[i] + (1.f - beta2) * gr * gr;
    const float mh = m1[i] / (1.f - powf(beta1, (float)step));
    const float vh = m2[i] / (1.f - powf(beta2, (float)step));
    params[i] -= lr * mh / (sqrtf(vh) + eps);
}

// ---- matrix statistics for the selector's features ------------------------
// Sixteen 64-bit words; non-negative doubles are kept as their bit patterns,
// whose unsigned order is the numeric order (atomicMax / atomicMin):
//   [0] ||A||_inf (max row sum of |a|)   [1] max |a_ij|   [2] sum a_ij^2
//   [3] max_i 1/(1+r_i), r_i = |a_ii| / sum_{j!=i} |a_ij|
//   [4] rows with r_i >= 1 (count)   [5] ||A||_1 (max column sum)
//   [6] min row sum   [7] min |a_ii|   [8] max |a_ii|   [9] sum |a_ij|
//   [10] min column sum   [11] sum |a_ii|
__device__ __forceinline__ void amax_d(unsigned long long* p, double v)
{
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void amin_d(unsigned long long* p, double v)
{
    atomicMin(p, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_stats_init(unsigned long long* out)
{
    const int i = threadIdx.x;
    if (i < 16)
    {
        out[i] = (i == 6 || i == 7 || i == 10) ? (unsigned long long)__double_as_longlong(INFINITY) : 0ull;
    }
}

// A warp per row: [0] [1] [2] [3] [4] [6] [7] [8] [9] [11].
__global__ void k_row_stats(const double* __restrict__ a, int n, unsigned long long* out)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n)
    {
        return;
    }
    const double* row = a + (int64_t)warp * n;
    double        s = 0.0, mx = 0.0, sq = 0.0;
    for (int j = lane; j < n; j += 32)
    {
        const double v = fabs(row[j]);
        s += v;
        mx = fmax(mx, v);
        sq = fma(v, v, sq);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        s += __shfl_down_sync(0xffffffffu, s, off);
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        sq += __shfl_down_sync(0xffffffffu, sq, off);
    }
    if (lane == 0)
    {
        amax_d(out + 0, s);
        amax_d(out + 1, mx);
        atomicAdd(reinterpret_cast<double*>(out + 2), sq);
        atomicAdd(reinterpret_cast<double*>(out + 9), s);
        const double d     = fabs(row[warp]);
        const double off   = s - d;
        const double ratio = off > 0 ? d / off : 1e30;
        amax_d(out + 3, 1.0 / (1.0 + ratio));
        if (ratio >= 1.0)
        {
            atomicAdd(out + 4, 1ull);
        }
        amin_d(out + 6, s);
        amin_d(out + 7, d);
        amax_d(out + 8, d);
        atomicAdd(reinterpret_cast<double*>(out + 11), d);
    }
}

// [5] [10]: column sums of |a|, 32 columns per CTA whose kColWarps warps
// split the rows (warp w takes rows w, w + kColWarps, ...; a warp reads 32
// consecutive entries of a row, 256 coalesced bytes), then the warps'
// partial sums are added in warp order in shared memory.  One thread per
// column walking all n rows left a few CTAs latency-bound on their loads.
constexpr int kColWarps = 32;

__global__ void __launch_bounds__(32 * kColWarps) k_col_stats(const double* __restrict__ a, int n,
    unsigned long long* out)
{
    __shared__ double part[kColWarps][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j    = blockIdx.x * 32 + lane;
    double    s    = 0.0;
    if (j < n)
    {
        for (int i = warp; i < n; i += kColWarps)
        {
            s += fabs(a[(int64_t)i * n + j]);
        }
    }
    part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && j < n)
    {
        double t = 0.0;
        for (int w = 0; w < kColWarps; ++w)
        {
            t += part[w][lane];
        }
        amax_d(out + 5, t);
        amin_d(out + 10, t);
    }
}

}  // namespace
int require_sm100();

int enqueue_mlp_forward(const float* params, const float* x, int batch, float* probs, cudaStream_t s)
{
    prof_begin(KC_SELECT, s);
    k_mlp_forward<<<(batch + kMlpThreads - 1) / kMlpThreads, kMlpThreads, 0, s>>>(params, x, batch, probs);
    prof_end(KC_SELECT, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// Resets the sixteen words and gathers A's statistics (row-major, lda = n).
int enqueue_matrix_stats(const double* a, int n, unsigned long long* out, cudaStream_t s)
{
    prof_begin(KC_SELECT, s);
    k_stats_init<<<1, 32, 0, s>>>(out);
    k_row_stats<<<(int)(((int64_t)n * 32 + 255) / 256), 256, 0, s>>>(a, n, out);
    k_col_stats<<<(n + 31) / 32, 32 * kColWarps, 0, s>>>(a, n, out);
    prof_end(KC_SELECT, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API int b200la_mlp_param_count(void) { return kParams; }

B200LA_API int b200la_mlp_forward(const float* params, const float* x, int64_t batch, float* probs, void* stream)
{
    if (!params || !x || !probs || batch <= 0 || batch > INT_MAX / 2)
        return set_error(B200LA_INVALID_ARGUMENT, "mlp_forward: invalid arguments");
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    return enqueue_mlp_forward(params, x, (int)batch, probs, static_cast<cudaStream_t>(stream));
}

B200LA_API int b200la_mlp_gradient(const float* params, const float* x, const int32_t* labels, int64_t batch,
    float* grads, float* loss_sum, void* stream)
{
    if (!params || !x || !labels || !grads || !loss_sum || batch <= 0 || batch > INT_MAX / 2)
        return set_error(B200LA_INVALID_ARGUMENT, "mlp_gradient: invalid arguments");
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static std::mutex attr_m;
    static bool       attr_done[64] = {};
    int               dev           = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lock(attr_m);
        if (dev < 0 || dev >= 64 || !attr_done[dev])
        {
            B200LA_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)grad_smem_bytes()));
            if (dev >= 0 && dev < 64)
                attr_done[dev] = true;
        }
    }
    prof_begin(KC_SELECT, s);
    k_mlp_grad<<<(int)((batch + kGradSamples - 1) / kGradSamples), kGradSamples, grad_smem_bytes(), s>>>(params, x,
        labels, (int)batch, grads, loss_sum);
    prof_end(KC_SELECT, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

B200LA_API int b200la_mlp_adam(float* params, float* grads, float* m1, float* m2, int64_t batch, float lr,
    float beta1, float beta2, float eps, int step, float weight_decay, void* stream)
{
    if (!params || !grads || !m1 || !m2 || batch <= 0 || step < 1)
        return set_error(B200LA_INVALID_ARGUMENT, "mlp_adam: invalid arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    prof_begin(KC_SELECT, s);
    k_adam<<<(kParams + 255) / 256, 256, 0, s>>>(params, grads, m1, m2, 1.f / (float)batch, lr, beta1, beta2, eps, step,
        weight_decay);
    prof_end(KC_SELECT, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

B200LA_API int b200la_matrix_stats(const double* a, int64_t n, unsigned long long* out, void* stream)
{
    if (!a || !out || n <= 0 || n > 65536)
        return set_error(B200LA_INVALID_ARGUMENT, "matrix_stats: invalid arguments");
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    return enqueue_matrix_stats(a, (int)n, out, static_cast<cudaStream_t>(stream));
}
}
