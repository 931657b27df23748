// common.cpp -- host plumbing: errors, stream-ordered buffers, device properties.
#include "common.cuh"

#include <mutex>

namespace gtsc {

static thread_local std::string g_last_error;

void set_last_error(const std::string &m) { g_last_error = m; }
const std::string &last_error() { return g_last_error; }

void fail(gtsc_status code, const std::string &msg) { throw Error(code, msg); }

void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
            throw Error(GTSC_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
        throw Error(GTSC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// The default memory pool returns freed memory to the driver at every synchronisation unless its
// release threshold is raised; the encodings allocate and free column-sized buffers on every call,
// so keep what the pool has reserved (once per device).
static void keep_pool_memory()
{
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    for (int d : done)
        if (d == dev) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done.push_back(dev);
}

DevBuf dev_alloc(uint64_t bytes, cudaStream_t s)
{
    DevBuf b;
    b.bytes = bytes;
    if (bytes == 0) return b;
    keep_pool_memory();
    void *p = nullptr;
    // round up so that vector loads of a final partial chunk stay inside the allocation
    GTSC_CUDA(cudaMallocAsync(&p, (bytes + 63) & ~63ull, s));
    b.m = std::make_shared<DevMem>();
    b.m->p = (uint8_t *)p;
    b.m->s = s;
    return b;
}

int sm_count()
{
    static int count = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 148;
    });
    return count;
}

void d2h(void *dst, const void *src, uint64_t bytes, cudaStream_t s)
{
    if (!bytes) return;
    GTSC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    GTSC_CUDA(cudaStreamSynchronize(s));
}

}  // namespace gtsc
