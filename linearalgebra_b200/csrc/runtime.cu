// Host runtime of the C ABI: per-thread error messages, CUDA error mapping
// and a per-device cache of the properties the launch planning needs.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace b200la
{
namespace
{
thread_local char g_last_error[512] = "";

struct DeviceInfo
{
    int  sm_count = 0;
    int  major    = 0;
    int  minor    = 0;
    bool coop     = false;
};

std::mutex g_dev_mutex;
DeviceInfo g_dev[64];

// Launch recorder: event pairs around the launches of the profiled kernel
// classes, plus a count of every kernel launch the library issues.
std::atomic<int64_t> g_launches{0};
std::atomic<int>     g_prof_mask{0};
std::mutex           g_prof_mutex;
struct EventPair
{
    cudaEvent_t a = nullptr, b = nullptr;
};
std::vector<EventPair> g_prof_events[KC_COUNT];
size_t                 g_prof_used[KC_COUNT] = {};
}  // namespace

void prof_begin(int cls, cudaStream_t s)
{
    if ((g_prof_mask.load(std::memory_order_relaxed) & (1 << cls)) == 0)
    {
        return;
    }
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    auto&                       v = g_prof_events[cls];
    if (g_prof_used[cls] == v.size())
    {
        EventPair e;
        if (cudaEventCreate(&e.a) != cudaSuccess || cudaEventCreate(&e.b) != cudaSuccess)
        {
            return;
        }
        v.push_back(e);
    }
    cudaEventRecord(v[g_prof_used[cls]].a, s);
}

void prof_end(int cls, cudaStream_t s)
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if ((g_prof_mask.load(std::memory_order_relaxed) & (1 << cls)) == 0)
    {
        return;
    }
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    if (g_prof_used[cls] < g_prof_events[cls].size())
    {
        cudaEventRecord(g_prof_events[cls][g_prof_used[cls]].b, s);
        ++g_prof_used[cls];
    }
}

int set_error(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_check(cudaError_t e, const char* what)
{
    return set_error(B200LA_CUDA_ERROR, "%s: %s (%s)", what, cudaGetErrorString(e),
        cudaGetErrorName(e));
}

static const DeviceInfo* current_device_info()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    {
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    DeviceInfo&                 d = g_dev[dev];
    if (d.sm_count == 0)
    {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        {
            return nullptr;
        }
        d.sm_count = prop.multiProcessorCount;
        d.major    = prop.major;
        d.minor    = prop.minor;
        int coop   = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        d.coop = coop != 0;
    }
    return &d;
}

int device_sm_count()
{
    const DeviceInfo* d = current_device_info();
    return d ? d->sm_count : 0;
}

// The kernels are built for sm_100a only: refuse anything else loudly
// instead of failing at the first launch.
int require_sm100()
{
    const DeviceInfo* d = current_device_info();
    if (d == nullptr)
    {
        return set_error(B200LA_CUDA_ERROR, "no CUDA device is current");
    }
    if (d->major != 10 || d->minor != 0)
    {
        return set_error(B200LA_NOT_SUPPORTED,
            "this library is built for sm_100a (B200); the current device is sm_%d%d", d->major,
            d->minor);
    }
    if (!d->coop)
    {
        return set_error(B200LA_NOT_SUPPORTED, "device lacks cooperative launch support");
    }
    return B200LA_SUCCESS;
}

}  // namespace b200la

extern "C" {

B200LA_API const char* b200la_last_error(void) { return b200la::g_last_error; }

B200LA_API const char* b200la_status_string(int status)
{
    switch (status)
    {
    case B200LA_SUCCESS: return "success";
    case B200LA_SINGULAR: return "singular: exact zero pivot";
    case B200LA_NOT_CONVERGED: return "refinement did not converge";
    case B200LA_INVALID_ARGUMENT: return "invalid argument";
    case B200LA_WORKSPACE_TOO_SMALL: return "workspace too small";
    case B200LA_CUDA_ERROR: return "CUDA error";
    case B200LA_DEVICE_TIMEOUT: return "device-side wait timed out";
    case B200LA_NOT_SUPPORTED: return "not supported";
    default: return "unknown status";
    }
}

B200LA_API int b200la_version(void) { return 100; }

B200LA_API int64_t b200la_launch_count(void) { return b200la::g_launches.load(); }

B200LA_API void b200la_profile_start(int class_mask)
{
    std::lock_guard<std::mutex> lock(b200la::g_prof_mutex);
    for (int c = 0; c < b200la::KC_COUNT; ++c)
    {
        b200la::g_prof_used[c] = 0;
    }
    b200la::g_prof_mask.store(class_mask);
}

B200LA_API int b200la_profile_stop(int kernel_class, double* total_ms, int64_t* launches)
{
    using namespace b200la;
    g_prof_mask.store(0);
    if (kernel_class < 0 || kernel_class >= KC_COUNT)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "profile_stop: bad kernel class");
    }
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    double                      sum = 0.0;
    for (size_t i = 0; i < g_prof_used[kernel_class]; ++i)
    {
        const EventPair& e = g_prof_events[kernel_class][i];
        if (cudaEventSynchronize(e.b) != cudaSuccess)
        {
            return cuda_check(cudaGetLastError(), "profile_stop");
        }
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess)
        {
            sum += ms;
        }
    }
    if (total_ms)
    {
        *total_ms = sum;
    }
    if (launches)
    {
        *launches = (int64_t)g_prof_used[kernel_class];
    }
    return B200LA_SUCCESS;
}
}
