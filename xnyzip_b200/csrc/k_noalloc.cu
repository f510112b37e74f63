// Allocation-free radix sort entry point.
//
// Some callers cannot allocate device memory while they run: a real-time loop that must not
// block on the CUDA allocator, or a plugin inside a host application that owns all of the
// device memory.  xnyz_sort_noalloc gives them the library's stable LSD radix sort (the one
// xnyz_stage_sort runs) with every scratch buffer taken from the fixed array below instead of
// a context workspace.  The caller passes only the keys (and optional payload), which are
// sorted in place.
//
// The scratch array is a file-scope device array of kNoAllocBytes (about 12.6 MB): every GPU
// that loads this part of the library holds it until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on each device looks the address
// up with cudaGetSymbolAddress (with that device current) and caches it; make that first call
// before any stream capture.  The cached address belongs to the device's primary context: after
// cudaDeviceReset it is stale, so do not call this entry point again in that process.  All
// calls share the array and it keeps the last call's contents: the digit histograms, tile
// counters and error word are cleared at the start of every call, and the look-back words are
// epoch-tagged.  Calls that overlap on the GPU (two streams, two host threads on one device)
// race on the array; serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/xnyz.h"
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace {

constexpr unsigned long long kNoAllocMaxKeys = 1ull << 20;
constexpr unsigned long long kTilesMax = kNoAllocMaxKeys / dev::kSortTile;
// byte offsets inside the scratch array
constexpr size_t kOffKeys = 0;
constexpr size_t kOffVals = kOffKeys + 8 * kNoAllocMaxKeys;
constexpr size_t kOffStatus = kOffVals + 4 * kNoAllocMaxKeys;
constexpr size_t kOffHist = kOffStatus + 8 * kTilesMax * 256;
constexpr size_t kOffCounters = kOffHist + 4 * 8 * 256;
constexpr size_t kOffErr = kOffCounters + 4 * 16;
constexpr size_t kNoAllocBytes = kOffErr + 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch[kMaxDevices] = {};
uint32_t g_epoch[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once per device).
cudaError_t scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

}  // namespace
}  // namespace xnyz

extern "C" xnyz_status xnyz_sort_noalloc(uint64_t* dev_keys, uint32_t* dev_payload, uint64_t n, int key_bits,
                                         void* stream) {
    using namespace xnyz;
    using namespace xnyz::dev;
    if (n > kNoAllocMaxKeys) return XNYZ_ERR_UNSUPPORTED;  // more keys than the fixed scratch holds
    if (!dev_keys && n) return XNYZ_ERR_INVALID_ARG;
    if (key_bits < 0 || key_bits > 64) return XNYZ_ERR_INVALID_ARG;
    const int passes = (key_bits + 7) / 8;
    if (n <= 1 || passes == 0) return XNYZ_OK;
    (void)cudaGetLastError();  // an earlier launch's error on this thread is not this call's failure
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return XNYZ_ERR_CUDA;
    unsigned char* s = nullptr;
    if (scratch_address(device, &s) != cudaSuccess) return XNYZ_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long* keys_alt = reinterpret_cast<unsigned long long*>(s + kOffKeys);
    uint32_t* vals_alt = reinterpret_cast<uint32_t*>(s + kOffVals);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(s + kOffStatus);
    uint32_t* hist = reinterpret_cast<uint32_t*>(s + kOffHist);
    uint32_t* counters = reinterpret_cast<uint32_t*>(s + kOffCounters);
    uint32_t* err = reinterpret_cast<uint32_t*>(s + kOffErr);
    // Clear what must start at zero: histograms, tile counters, the error word.
    if (cudaMemsetAsync(hist, 0, kOffErr + sizeof(uint32_t) - kOffHist, st) != cudaSuccess) return XNYZ_ERR_CUDA;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_epoch[device] + passes >= 16383) {
            if (cudaMemsetAsync(status, 0, 8 * kTilesMax * 256, st) != cudaSuccess) return XNYZ_ERR_CUDA;
            g_epoch[device] = 0;
        }
    }
    unsigned long long* kb[2] = {reinterpret_cast<unsigned long long*>(dev_keys), keys_alt};
    uint32_t* vb[2] = {dev_payload, dev_payload ? vals_alt : nullptr};
    launch_sort_histogram(kb[0], n, passes, hist, st);
    launch_sort_offsets(hist, passes, st);
    int cur = 0;
    for (int p = 0; p < passes; ++p) {
        uint32_t epoch;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            epoch = ++g_epoch[device];
        }
        launch_sort_pass(kb[cur], kb[cur ^ 1], vb[cur], vb[cur ^ 1], n, 8 * p, hist + 256 * p, status, epoch,
                         counters + p, err, st);
        cur ^= 1;
    }
    if (cudaGetLastError() != cudaSuccess) return XNYZ_ERR_CUDA;  // a launch was refused
    if (cur) {  // result in the scratch copy: back into the caller's arrays
        if (cudaMemcpyAsync(dev_keys, keys_alt, 8 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return XNYZ_ERR_CUDA;
        if (dev_payload &&
            cudaMemcpyAsync(dev_payload, vals_alt, 4 * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return XNYZ_ERR_CUDA;
    }
    uint32_t herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st) != cudaSuccess) return XNYZ_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return XNYZ_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess) return XNYZ_ERR_CUDA;
    return herr ? XNYZ_ERR_TIMEOUT : XNYZ_OK;
}
