// Floodfill without any allocation: the scratch lives in a fixed-size array
// compiled into the library (see cubvh_floodfill_noalloc in
// include/cubvh_b200.h).
//
// Who needs this: callers that are not allowed to allocate GPU memory while
// they run, for example code executing inside another framework's memory
// pool or arena that forbids cudaMalloc/cudaFree (a stray allocation would
// synchronise the device or break the pool's accounting), or real-time loops
// that must not hit the allocator at all.  They still own and pass the input
// grid and the output labels; only the scratch comes from here.
//
// Cost: every GPU that loads this part of the library holds the array
// (kNoAllocScratchBytes) until the process exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/cubvh_b200.h"
#include "kernels.h"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;  // 32 MiB

// In host code this name is only a stand-in for the device array: its device
// address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_floodfill_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_addr[64] = {nullptr};  // device address of the array, per device ordinal

}  // namespace

namespace cubvh {

int floodfill_noalloc_scratch(void** ws, std::string& err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return CUBVH_ERR_CUDA; }
    if (dev < 0 || dev >= 64) { err = "device ordinal outside [0, 64)"; return CUBVH_ERR_INVALID; }
    // first call on this device: look up the array's device address with
    // this device current; later calls reuse it (so calls must not span a
    // cudaDeviceReset of the device, after which the array is reloaded)
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_floodfill_scratch);
        if (e != cudaSuccess) {
            err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return CUBVH_ERR_CUDA;
        }
        g_addr[dev] = p;
    }
    *ws = g_addr[dev];
    return CUBVH_OK;
}

int floodfill_noalloc_fits(int B, int H, int W, int D, std::string& err) {
    const size_t need = floodfill_workspace_bytes(B, H, W, D);
    if (need > kNoAllocScratchBytes) {
        err = "grid needs " + std::to_string(need) + " bytes of scratch but the no-allocation floodfill holds " +
              std::to_string(kNoAllocScratchBytes) + " (about 192^3 voxels); use cubvh_floodfill";
        return CUBVH_ERR_INVALID;
    }
    return CUBVH_OK;
}

int floodfill_noalloc(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels, cudaStream_t stream,
                      std::string& err) {
    int rc = floodfill_noalloc_fits(B, H, W, D, err);
    if (rc != CUBVH_OK) return rc;
    void* ws = nullptr;
    if ((rc = floodfill_noalloc_scratch(&ws, err)) != CUBVH_OK) return rc;
    // every buffer inside the scratch is written before it is read, and the
    // status word is zeroed by the launch itself: nothing carries over from
    // the previous call
    const cudaError_t e = launch_floodfill(grid, B, H, W, D, labels, ws, stream);
    if (e != cudaSuccess) { err = std::string("floodfill launch: ") + cudaGetErrorString(e); return CUBVH_ERR_CUDA; }
    return CUBVH_OK;
}

}  // namespace cubvh
