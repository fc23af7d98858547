// Stream-ordered scratch memory for per-call temporaries (partial sums of
// source slices, sampled schedules, surrogate queues).
//
// The device's default memory pool returns every freed block to the driver
// at the next synchronisation (release threshold 0), so a call that
// allocates tens of MB of partial sums after a host sync pays for mapping
// fresh pages each time. The library keeps its own pool per device whose
// release threshold holds up to kRetainBytes across synchronisations;
// oskb_scratch_release() hands the cached blocks back.
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace oskb {
namespace {

constexpr int kMaxDevices = 64;
constexpr unsigned long long kRetainBytes = 4ULL << 30;

// Pools and SM counts are per device: one process may drive several GPUs
// from several host threads (one per device, as the reference's simulator
// does), so the tables are filled under a lock.
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[kMaxDevices] = {};
std::atomic<int> g_sms[kMaxDevices];

cudaMemPool_t pool_for_current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool[dev])
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        unsigned long long keep = kRetainBytes;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pool[dev] = p;
    }
    return g_pool[dev];
}

}  // namespace

int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        return -1;
    }
    return dev;
}

int device_sm_count()
{
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices) return 148;
    int n = g_sms[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
            cudaSuccess || n <= 0)
    {
        cudaGetLastError();
        return 148;
    }
    g_sms[dev].store(n, std::memory_order_relaxed);
    return n;
}

cudaError_t scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream)
{
    cudaMemPool_t p = pool_for_current_device();
    if (!p) return cudaMallocAsync(ptr, bytes, stream);
    return cudaMallocFromPoolAsync(ptr, bytes, p, stream);
}

cudaError_t scratch_free(void* ptr, cudaStream_t stream)
{
    return cudaFreeAsync(ptr, stream);
}

}  // namespace oskb

extern "C" int oskb_scratch_release(void)
{
    std::lock_guard<std::mutex> lock(oskb::g_pool_mutex);
    for (int d = 0; d < oskb::kMaxDevices; ++d)
    {
        if (!oskb::g_pool[d]) continue;
        cudaError_t e = cudaMemPoolTrimTo(oskb::g_pool[d], 0);
        if (e != cudaSuccess)
        {
            oskb::set_last_error("scratch_release", e);
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
    }
    return 0;
}
