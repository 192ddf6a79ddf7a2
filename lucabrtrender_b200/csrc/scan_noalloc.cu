// lrt_prefix_sum_noalloc: the prefix sum (the same single-pass decoupled
// look-back scan as lrt_prefix_sum) for callers that cannot allocate device
// memory -- a plugin inside a host application that owns every device
// allocation and its budget, or a frame-critical path where cudaMalloc would
// synchronise the device. The caller passes the input, output and total;
// the look-back status words live in a fixed array compiled into the library.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds its 128 KB until the process exits. In host code its name is
// only a host-side stand-in, so its device address is looked up once per
// device with cudaGetSymbolAddress (with that device current) and cached.
// That lookup happens on the first call on each device. Every call on a
// device shares the one array and leaves the last call's contents behind, so
// each call clears it first on its stream; calls whose work overlaps on the
// GPU (different streams, no ordering between them) race on it.
#include "../../include/lrt_raster.h"
#include "kernels.cuh"
#include "raster_common.cuh"

#include <mutex>

namespace {

// The scan's own scratch for the largest count (a 16-byte ticket header and
// one 8-byte status word per 4096-element partition), then 16 bytes holding
// this entry point's error word.
constexpr size_t kScanBytesMax = 16 + (size_t{LRT_PREFIX_SUM_NOALLOC_MAX} + 4095) / 4096 * 8;
constexpr size_t kNoAllocBytes = kScanBytesMax + 16;

static __device__ __align__(256) unsigned char g_scan_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch[kMaxDevices] = {};

// The device address of g_scan_scratch on the current device, looked up once.
cudaError_t scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[device] = p;
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

}  // namespace

extern "C" int lrt_prefix_sum_noalloc(const void* in, void* out, void* total, uint32_t count, void* streamPtr) {
    if (total == nullptr || (count > 0 && (in == nullptr || out == nullptr))) return LRT_INVALID_ARGUMENT;
    if (count > LRT_PREFIX_SUM_NOALLOC_MAX) return LRT_INVALID_ARGUMENT;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return LRT_DEVICE_FAILURE;
    void* scratch = nullptr;
    if (scratch_address(device, &scratch) != cudaSuccess) return LRT_DEVICE_FAILURE;
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    // The scan's scratch starts at the array's base (launch_exclusive_scan
    // clears the scan_scratch_bytes(count) <= kScanBytesMax it uses before
    // its kernel); the error word follows it.
    uint32_t* err = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(scratch) + kScanBytesMax);
    if (lrt::scan_scratch_bytes(count) > kScanBytesMax) return LRT_INTERNAL_ERROR;
    if (cudaMemsetAsync(err, 0, 4, stream) != cudaSuccess) return LRT_DEVICE_FAILURE;
    if (lrt::launch_exclusive_scan(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out),
                                   static_cast<uint32_t*>(total), count, scratch, err, stream) != cudaSuccess)
        return LRT_DEVICE_FAILURE;
    uint32_t status = 0;
    if (cudaMemcpyAsync(&status, err, 4, cudaMemcpyDeviceToHost, stream) != cudaSuccess) return LRT_DEVICE_FAILURE;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return LRT_DEVICE_FAILURE;
    if (status & lrt::kErrTimeout) return LRT_TIMEOUT;
    if (status & lrt::kErrTooManyPairs) return LRT_OVERFLOW;
    return LRT_OK;
}
