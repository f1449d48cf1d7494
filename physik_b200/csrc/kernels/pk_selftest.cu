// pk_selftest.cu -- a bounded wait of the grid exchange made to run out on purpose.
//
// Every PCG kernel here waits for the other blocks of its group through the arrival
// counter of count_exchange (pk_device.cuh); each wait gives up after a number of polls,
// sets the error flag and lets the kernel leave through its normal exit, so a lost block
// costs a timeout status instead of a hung GPU.  This launch checks that path on the
// device: `blocks` co-resident blocks (one cooperative launch) exchange two partial sums
// as a group of `blocks + missing` members.  With missing = 0 every block gets the exact
// group sums; with missing > 0 the counter can never reach its target, every wait stops
// after `limit` polls and every block reports the timeout.  No counterpart in the
// reference (its solver runs on one CPU thread and never waits).
#include <cuda_runtime.h>

#include "../../../include/pkcuda.h"
#include "pk_device.cuh"

namespace pk {
namespace {

__global__ void __launch_bounds__(128) exchange_wait_selftest_kernel(ExSlot* slots, unsigned* counter, GridSync* sync,
                                                                      int group, unsigned long long limit,
                                                                      double* out)
{
    __shared__ double sh[3 * 32];
    __shared__ int shi[32];
    // thread 0 holds the block's values (the exchange first sums over the block's threads)
    double v[2] = {threadIdx.x == 0 ? double(blockIdx.x + 1) : 0.0, threadIdx.x == 0 ? 1.0 : 0.0};
    int bad = 0;
    const bool ok = count_exchange<double, 2>(slots, counter, 0, group, sync, 1u, v, bad, sh, shi, limit);
    if (threadIdx.x == 0) {
        out[3 * blockIdx.x] = ok ? 1.0 : 0.0;
        out[3 * blockIdx.x + 1] = v[0];
        out[3 * blockIdx.x + 2] = v[1];
    }
}

}  // namespace
}  // namespace pk

extern "C" PKCUDA_API int pk_exchange_wait_selftest(int device, int blocks, int missing, unsigned long long limit,
                                                    double* out)
{
    if (blocks < 2 || blocks > 64 || missing < 0 || missing > 64 || !out || limit == 0) return PK_ERR_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return PK_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return PK_ERR_CUDA;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk::exchange_wait_selftest_kernel, 128, 0) !=
            cudaSuccess ||
        blocks > sms * per_sm)
        return PK_ERR_UNSUPPORTED;
    // Slots for both generation buffers of the larger of the grid and the group, the
    // counter and the sync word, the per-block results.
    const int members = blocks + missing;
    const size_t slot_bytes = 2 * sizeof(pk::ExSlot) * static_cast<size_t>(members);
    const size_t out_bytes = 3 * sizeof(double) * static_cast<size_t>(blocks);
    unsigned char* mem = nullptr;
    const size_t total = slot_bytes + 256 + out_bytes;
    if (cudaMalloc(&mem, total) != cudaSuccess) return PK_ERR_CUDA;
    int rc = PK_OK;
    pk::ExSlot* slots = reinterpret_cast<pk::ExSlot*>(mem);
    unsigned* counter = reinterpret_cast<unsigned*>(mem + slot_bytes);
    pk::GridSync* sync = reinterpret_cast<pk::GridSync*>(mem + slot_bytes + 128);
    double* d_out = reinterpret_cast<double*>(mem + slot_bytes + 256);
    if (cudaMemset(mem, 0, total) != cudaSuccess) rc = PK_ERR_CUDA;
    if (rc == PK_OK) {
        int group = members;
        void* args[] = {&slots, &counter, &sync, &group, &limit, &d_out};
        if (cudaLaunchCooperativeKernel((const void*)pk::exchange_wait_selftest_kernel, dim3(blocks), dim3(128), args,
                                        0, nullptr) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess)
            rc = PK_ERR_CUDA;
    }
    if (rc == PK_OK && cudaMemcpy(out, d_out, out_bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = PK_ERR_CUDA;
    int err = 0;
    if (rc == PK_OK && cudaMemcpy(&err, &sync->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = PK_ERR_CUDA;
    cudaFree(mem);
    if (rc == PK_OK && err) rc = PK_ERR_TIMEOUT;
    return rc;
}
