// pk_noalloc.cu -- the block-Jacobi PCG solve on caller-owned device buffers, with its
// working memory in a fixed array compiled into the library instead of allocated.
//
// Who needs it: callers that may not allocate device memory while they solve -- for
// example a game-engine plugin that runs the solve inside its frame loop under a fixed
// memory budget, or a host application that owns all device memory through its own
// pool and forbids anyone else's cudaMalloc.  They pass their inputs and outputs as
// device pointers; the CG vectors, partial sums, barrier word and statistics live in
// g_pcg_scratch below.
//
// Limits and sharing:
//   * g_pcg_scratch is kPcgScratchBytes (8 MiB) on every GPU that loads the library and
//     stays allocated until the process exits; systems of at most kNoAllocMaxRows rows
//     (32,768, in every precision) fit, larger ones are rejected with PK_ERR_UNSUPPORTED.
//   * All calls on a device share the one array and it keeps the last call's contents;
//     the call clears what must start at zero.  Calls whose GPU work overlaps (two
//     streams, or two host threads) race on it and corrupt each other.
//   * The first call on a device looks up the array's device address (a one-time set-up
//     per device, done with that device current).
//   * Every call synchronises its stream to return the statistics: it must not be called
//     while that stream is being captured into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>

#include "../../../include/pkcuda.h"
#include "pk_kernels.cuh"

namespace {

constexpr size_t kPcgScratchBytes = size_t(8) << 20;
constexpr int kNoAllocMaxRows = 32768;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_pcg_scratch[kPcgScratchBytes];

// Device address of g_pcg_scratch per device (host code may not use the symbol itself).
// Atomic slots: two host threads making their first call on one device at once both look
// the address up and store the same value.
std::atomic<void*> g_scratch_ptr[kMaxDevices] = {};

thread_local std::string g_noalloc_error;

int noalloc_fail(int code, const std::string& msg)
{
    g_noalloc_error = msg;
    return code;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Carves the scratch array: residual, product and search-direction records, partial
// sums, barrier word and statistics.
template <class Real, class Acc>
int run(int n, const int* row_start, const int* col, const void* values, const int* lt_start, const int* lt_row,
        const int* lt_block, const void* b, const void* minv, int max_iterations, double tolerance, void* x,
        pk_cg_result* out, cudaStream_t stream, unsigned char* scratch)
{
    const int grid_max = pk::pcg_max_grid<Real, Acc>(pk::kPcgThreads, false);
    if (grid_max <= 0) return noalloc_fail(PK_ERR_CUDA, "pk_pcg_noalloc: occupancy query failed");
    const int grid = std::max(1, std::min(grid_max, (n + 31) / 32));
    const size_t vec = align256(3 * sizeof(Real) * size_t(n));
    const size_t rec = align256(8 * sizeof(Real) * size_t(n));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = scratch + off;
        off += align256(bytes);
        return p;
    };
    Real* r = reinterpret_cast<Real*>(take(vec));
    Real* q = reinterpret_cast<Real*>(take(vec));
    Real* sd0 = reinterpret_cast<Real*>(take(rec));
    Real* sd1 = reinterpret_cast<Real*>(take(rec));
    Acc* part_a = reinterpret_cast<Acc*>(take(sizeof(Acc) * size_t(grid)));
    Acc* part_b = reinterpret_cast<Acc*>(take(2 * sizeof(Acc) * size_t(grid)));
    int* part_bad = reinterpret_cast<int*>(take(4 * sizeof(int) * size_t(grid)));
    unsigned char* zeroed = scratch + off;  // barrier and statistics start at zero
    pk::GridSync* sync = reinterpret_cast<pk::GridSync*>(take(sizeof(pk::GridSync)));
    pk::DevStats* stats = reinterpret_cast<pk::DevStats*>(take(sizeof(pk::DevStats)));
    if (off > kPcgScratchBytes) return noalloc_fail(PK_ERR_UNSUPPORTED, "pk_pcg_noalloc: scratch overflow");
    cudaError_t e = cudaMemsetAsync(zeroed, 0, size_t(scratch + off - zeroed), stream);
    if (e != cudaSuccess) return noalloc_fail(PK_ERR_CUDA, std::string("pk_pcg_noalloc: ") + cudaGetErrorString(e));

    pk::PcgArgs<Real, Acc> a{};
    a.a.n = n;
    a.a.row_start = row_start;
    a.a.col = col;
    a.a.values = static_cast<const Real*>(values);
    a.a.lt_start = lt_start;
    a.a.lt_row = lt_row;
    a.a.lt_block = lt_block;
    a.b = static_cast<const Real*>(b);
    a.minv = static_cast<const Real*>(minv);
    a.x = static_cast<Real*>(x);
    a.r = r;
    a.sd0 = sd0;
    a.sd1 = sd1;
    a.q = q;
    a.part_a = part_a;
    a.part_b = part_b;
    a.part_bad = part_bad;
    a.sync = sync;
    a.max_iterations = max_iterations;
    a.tolerance = static_cast<Acc>(static_cast<Real>(tolerance));
    a.skip_on_flags = 0;
    a.integrate = 0;
    a.flags = &stats->flags;
    a.stats = stats;
    a.ntiles = 0;  // unstaged SpMV: needs no tile list
    e = pk::launch_pcg_kernel<Real, Acc>(a, grid, pk::kPcgThreads, stream);
    if (e != cudaSuccess) return noalloc_fail(PK_ERR_CUDA, std::string("pk_pcg_noalloc: ") + cudaGetErrorString(e));
    pk::DevStats host{};
    e = cudaMemcpyAsync(&host, stats, sizeof(host), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return noalloc_fail(PK_ERR_CUDA, std::string("pk_pcg_noalloc: ") + cudaGetErrorString(e));
    out->iterations = host.iterations;
    out->converged = host.converged;
    out->residual_norm = host.residual_norm;
    out->have_solution = (host.flags & pk::kFlagInvalidRhs) ? 0 : 1;
    if (host.flags & pk::kFlagBarrierTimeout) return noalloc_fail(PK_ERR_TIMEOUT, "pk_pcg_noalloc: barrier timeout");
    return PK_OK;
}

}  // namespace

extern "C" {

PKCUDA_API const char* pk_pcg_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

PKCUDA_API int pk_pcg_noalloc(int precision, int n, const int* row_start, const int* col_index, const void* values,
                              const int* lt_start, const int* lt_row, const int* lt_block, const void* b,
                              const void* minv, int max_iterations, double tolerance, void* x, pk_cg_result* out,
                              void* stream)
{
    if (!out) return noalloc_fail(PK_ERR_ARG, "pk_pcg_noalloc: out is NULL");
    std::memset(out, 0, sizeof(*out));
    if (precision < PK_PREC_FP32 || precision > PK_PREC_FP64 || n < 0)
        return noalloc_fail(PK_ERR_ARG, "pk_pcg_noalloc: bad precision or size");
    if (n > kNoAllocMaxRows)
        return noalloc_fail(PK_ERR_UNSUPPORTED, "pk_pcg_noalloc: " + std::to_string(n) +
                                                    " rows exceed the fixed scratch limit of " +
                                                    std::to_string(kNoAllocMaxRows));
    if (n == 0) {
        out->converged = 1;
        return PK_OK;
    }
    // Every index array is read by the kernel whenever n > 0 (a matrix without
    // off-diagonal blocks still passes 1-element lt_row / lt_block buffers).
    if (!row_start || !col_index || !values || !lt_start || !lt_row || !lt_block || !b || !minv || !x)
        return noalloc_fail(PK_ERR_ARG, "pk_pcg_noalloc: NULL device pointer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(PK_ERR_NO_DEVICE, "pk_pcg_noalloc: no current CUDA device");
    void* slot = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!slot) {
        e = cudaGetSymbolAddress(&slot, g_pcg_scratch);
        if (e != cudaSuccess || !slot)
            return noalloc_fail(PK_ERR_CUDA, std::string("pk_pcg_noalloc: cudaGetSymbolAddress: ") +
                                                 cudaGetErrorString(e));
        g_scratch_ptr[dev].store(slot, std::memory_order_release);
    }
    unsigned char* scratch = static_cast<unsigned char*>(slot);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == PK_PREC_FP32)
        return run<float, float>(n, row_start, col_index, values, lt_start, lt_row, lt_block, b, minv,
                                 max_iterations, tolerance, x, out, st, scratch);
    if (precision == PK_PREC_MIXED)
        return run<float, double>(n, row_start, col_index, values, lt_start, lt_row, lt_block, b, minv,
                                  max_iterations, tolerance, x, out, st, scratch);
    return run<double, double>(n, row_start, col_index, values, lt_start, lt_row, lt_block, b, minv, max_iterations,
                               tolerance, x, out, st, scratch);
}

}  // extern "C"
