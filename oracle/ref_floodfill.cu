// TEST INFRASTRUCTURE ONLY.  Compiles the reference's own CUDA floodfill
// (ashawkey/cubvh include/gpu/floodfill.cuh, `_floodfill_batch`, :157-272) from
// the reference tree where it lies (oracle/Makefile, target `ref`), into
// oracle/_ref/libref_floodfill.so.  The tests use it to pin the floodfill
// oracle and the CUDA floodfill against the reference's own labels; bench.py's
// reference arm times it.  The cubvh_b200 package never loads it.
//
// The reference's Python entry (cubvh/api.py:128-139 -> src/api_gpu.cu:136-152)
// hands `_floodfill_batch` CUDA tensors although the function copies its input
// with cudaMemcpyHostToDevice and its output with cudaMemcpyDeviceToHost; this
// wrapper passes host buffers, which is the use those copy kinds declare.  The
// kernels and the iteration schedule are the reference's, unchanged.
#include <climits>
#include <cstdint>
#include <cstdio>  // the header calls printf without including it

#include "gpu/floodfill.cuh"  // found through -I<reference>/include

// grid: B*H*W*D bytes, each 0 (free) or 1 (blocked), in host memory.
// labels: B*H*W*D int32 in host memory.  Returns 0, or 1 for sizes outside
// int32 (the reference indexes with int), or 2 when a CUDA call failed.
extern "C" int ref_floodfill(const uint8_t* grid, int B, int H, int W, int D, int32_t* labels) {
    const long long n = (long long)B * H * W * D;
    // H*H + W*W + D*D is an int in the reference's iteration limit
    if (B <= 0 || H <= 0 || W <= 0 || D <= 0 || n > (long long)INT_MAX ||
        (long long)H * H + (long long)W * W + (long long)D * D > (long long)INT_MAX) return 1;
    // bytes 0/1 are valid bool objects
    _floodfill_batch(reinterpret_cast<const bool*>(grid), B, H, W, D, labels);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
