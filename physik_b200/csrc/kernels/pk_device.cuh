// pk_device.cuh -- device helpers shared by the kernel translation units: vector
// loads/stores, block and grid reductions in a fixed order, the bounded grid barrier of
// the cooperative PCG launch, and the mbarrier / TMA bulk-copy primitives.
// Everything here has internal linkage (one copy per translation unit).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pk_kernels.cuh"

namespace pk {
namespace {

constexpr unsigned long long kBarrierSpinLimit = 1ull << 24;  // ~seconds with back-off

template <class Real>
__device__ __forceinline__ Real qnan();
template <>
__device__ __forceinline__ float qnan<float>() { return __int_as_float(0x7fc00000); }
template <>
__device__ __forceinline__ double qnan<double>() { return __longlong_as_double(0x7ff8000000000000ll); }

template <class Real>
__device__ __forceinline__ V3<Real> ld3(const Real* p, int i)
{
    const Real* q = p + 3 * (size_t)i;
    return V3<Real>{__ldg(q), __ldg(q + 1), __ldg(q + 2)};
}
// Loads of data written earlier in the same launch by another block: bypass L1.
template <class Real>
__device__ __forceinline__ V3<Real> ldcg3(const Real* p, int i)
{
    const Real* q = p + 3 * (size_t)i;
    return V3<Real>{__ldcg(q), __ldcg(q + 1), __ldcg(q + 2)};
}
template <class Real>
__device__ __forceinline__ V3<Real> ldplain3(const Real* p, int i)
{
    const Real* q = p + 3 * (size_t)i;
    return V3<Real>{q[0], q[1], q[2]};
}
template <class Real>
__device__ __forceinline__ void st3(Real* p, int i, V3<Real> v)
{
    Real* q = p + 3 * (size_t)i;
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
}
template <class Real>
__device__ __forceinline__ M3<Real> ld9(const Real* p, size_t i)
{
    const Real* q = p + 9 * i;
    M3<Real> m;
    m.c[0] = V3<Real>{__ldg(q + 0), __ldg(q + 1), __ldg(q + 2)};
    m.c[1] = V3<Real>{__ldg(q + 3), __ldg(q + 4), __ldg(q + 5)};
    m.c[2] = V3<Real>{__ldg(q + 6), __ldg(q + 7), __ldg(q + 8)};
    return m;
}
template <class Real>
__device__ __forceinline__ void st9(Real* p, size_t i, const M3<Real>& m)
{
    Real* q = p + 9 * i;
    q[0] = m.c[0].x; q[1] = m.c[0].y; q[2] = m.c[0].z;
    q[3] = m.c[1].x; q[4] = m.c[1].y; q[5] = m.c[1].z;
    q[6] = m.c[2].x; q[7] = m.c[2].y; q[8] = m.c[2].z;
}
template <class Acc, class Real>
__device__ __forceinline__ Acc dot_acc(V3<Real> a, V3<Real> b)
{
    return Acc(a.x) * Acc(b.x) + Acc(a.y) * Acc(b.y) + Acc(a.z) * Acc(b.z);
}
// a + s*b evaluated in the accumulation type, rounded once to the storage type.
template <class Real, class Acc>
__device__ __forceinline__ V3<Real> axpy(V3<Real> a, Acc s, V3<Real> b)
{
    return V3<Real>{Real(Acc(a.x) + s * Acc(b.x)), Real(Acc(a.y) + s * Acc(b.y)), Real(Acc(a.z) + s * Acc(b.z))};
}
__device__ __forceinline__ bool acc_finite(float v) { return isfinite(v); }
__device__ __forceinline__ bool acc_finite(double v) { return isfinite(v); }

// ------------------------------------------------------------------ barrier
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// ------------------------------------------------------------------ TMA bulk copies
// One-dimensional bulk copies global -> shared (cp.async.bulk, no multicast) completing
// on an mbarrier with a transaction count.  Addresses and sizes are 16-byte multiples.
constexpr unsigned kMbarSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// Before an mbarrier's memory is initialised again (no thread may still wait on it).
__device__ __forceinline__ void mbar_inval(unsigned long long* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity; false after kMbarSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    for (unsigned i = 0; i < kMbarSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Sense-counting grid barrier for a cooperative launch.  Every wait is bounded: after
// kBarrierSpinLimit polls it records the timeout in sync->err and returns false, and
// every block also gives up as soon as it sees another block's timeout.
__device__ bool grid_barrier(GridSync* sync, int* s_flag)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned nblocks = gridDim.x;
        if (nblocks > 1) {
            const unsigned gen = ld_acquire(&sync->gen);
            const unsigned old = atom_add_acq_rel(&sync->arrive, 1u);
            if (old == nblocks - 1) {
                atomicExch(&sync->arrive, 0u);
                st_release(&sync->gen, gen + 1u);
            } else {
                unsigned long long spins = 0;
                while (ld_acquire(&sync->gen) == gen) {
                    if (++spins > kBarrierSpinLimit) {
                        atomicExch(&sync->err, 1);
                        ok = 0;
                        break;
                    }
                    if (spins > 32) __nanosleep(100);
                    if (*(volatile int*)&sync->err) {
                        ok = 0;
                        break;
                    }
                }
            }
        }
        if (*(volatile int*)&sync->err) ok = 0;
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// Block-wide sum of N values (fixed shuffle tree, then warp 0 in order): identical
// results on every run.  `sh` holds N*32 values.  Result valid in all threads.
template <class Acc, int N>
__device__ __forceinline__ void block_sum(Acc (&v)[N], Acc* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            Acc t = lane < nw ? sh[k * 32 + lane] : Acc(0);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
            if (lane == 0) sh[k * 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[k * 32];
    __syncthreads();
}

__device__ __forceinline__ int block_or(int v, int* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = __reduce_or_sync(0xffffffffu, (unsigned)v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    int t = 0;
    for (int w = 0; w < nw; ++w) t |= sh[w];
    __syncthreads();
    return t;
}

// Sum of the per-block partials part[i*stride + k] over all blocks, in a fixed order,
// evaluated identically by every block.
template <class Acc, int N>
__device__ __forceinline__ void grid_sum(const Acc* part, int stride, Acc (&out)[N], Acc* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            Acc t = Acc(0);
            for (int i = lane; i < (int)gridDim.x; i += 32) t += __ldcg(part + (size_t)i * stride + k);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
            if (lane == 0) sh[k * 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = sh[k * 32];
    __syncthreads();
}

__device__ __forceinline__ int grid_or(const int* part, int stride, int* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        int t = 0;
        for (int i = lane; i < (int)gridDim.x; i += 32) t |= __ldcg(part + (size_t)i * stride);
        t = (int)__reduce_or_sync(0xffffffffu, (unsigned)t);
        if (lane == 0) sh[0] = t;
    }
    __syncthreads();
    const int r = sh[0];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------------ block reduction
// Sum of N values and OR of one int over the block, in a fixed tree; valid in every
// thread.  `sh` holds (N+1)*32 values of Acc, `shi` 32 ints.
template <class Acc, int N>
__device__ __forceinline__ void block_sum_or(Acc (&v)[N], int& bad, Acc* sh, int* shi)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    bad = (int)__reduce_or_sync(0xffffffffu, (unsigned)bad);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) sh[k * 32 + warp] = v[k];
        shi[warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            Acc t = lane < nw ? sh[k * 32 + lane] : Acc(0);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
            v[k] = t;
        }
        int b = lane < nw ? shi[lane] : 0;
        b = (int)__reduce_or_sync(0xffffffffu, (unsigned)b);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < N; ++k) sh[N * 32 + k] = v[k];
            shi[0] = b;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[N * 32 + k];
    bad = shi[0];
    __syncthreads();
}

// Group exchange among the `members` blocks whose slots are slots[0 .. members) of each of
// the two generation buffers (buffer b at slots + b * stride): publishes this block's
// (number `me`) sums of v (N <= 2) and OR of bad, waits for every member's slot of
// generation `gen`, and returns the group-wide sums / OR, reduced in one fixed tree so
// every member gets identical values.  False when a wait gave up or a block reported a
// failure.  A group of one block is a block reduction.
template <class Acc, int N>
__device__ bool group_exchange(ExSlot* slots, int stride, int members, int me, GridSync* sync, unsigned gen,
                               Acc (&v)[N], int& bad, Acc* sh, int* shi)
{
    static_assert(N >= 1 && N <= 2, "two partials per slot");
    block_sum_or<Acc, N>(v, bad, sh, shi);
    if (members <= 1) return !*(volatile int*)&sync->err;
    const int G = members, tid = threadIdx.x;
    ExSlot* buf = slots + (gen & 1u) * (unsigned)stride;
    if (tid == 0) {
        ExSlot* my = buf + me;
        my->v0 = double(v[0]);
        my->v1 = N > 1 ? double(v[N - 1]) : 0.0;
        my->bad = bad;
        st_release(&my->gen, gen);  // cumulative: no separate fence
    }
    Acc pv[N];
#pragma unroll
    for (int k = 0; k < N; ++k) pv[k] = Acc(0);
    int pb = 0, fail = 0;
    for (int i = tid; i < G; i += blockDim.x) {
        const ExSlot* sl = buf + i;
        unsigned long long spins = 0;
        while (ld_acquire(&sl->gen) != gen) {
            if (++spins > kBarrierSpinLimit) {
                atomicExch(&sync->err, 1);
                fail = 1;
                break;
            }
            if ((spins & 1023u) == 0 && *(volatile int*)&sync->err) {
                fail = 1;
                break;
            }
        }
        if (fail) break;
        pv[0] += Acc(__ldcg(&sl->v0));
        if (N > 1) pv[N - 1] += Acc(__ldcg(&sl->v1));
        pb |= __ldcg(&sl->bad);
    }
    pb |= fail << 30;
    block_sum_or<Acc, N>(pv, pb, sh, shi);
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = pv[k];
    bad = pb & ~(1 << 30);
    return !(pb & (1 << 30)) && !*(volatile int*)&sync->err;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid exchange through one arrival counter (sync->arrive, zero at launch; exchanges
// numbered gen = 1, 2, ...): each block stores its partials in its slot of the buffer of
// the generation's parity and adds one to the counter with release semantics; the last
// warp of every block (in the part-resident kernel the producer warp, which has no row
// loads of its own in flight while it waits: polling from a warp with outstanding loads
// measured slower) waits (bounded) until the counter reaches gen * gridDim.x, then reads all
// slots -- lane i the slots i, i + 32, ... in order -- and reduces them in a fixed shuffle
// tree, so every block gets identical sums.  One poller warp per block on one address,
// instead of one poller per slot.  The parity buffers keep a block that runs ahead from
// overwriting a slot that another block has not read yet: to publish generation g + 2 it
// must have seen every block publish g + 1, which each does only after reading g.
//
// Split in two halves so a block can issue independent loads while it waits:
// count_publish reduces the block's partials and publishes them; count_finish waits and
// reduces.  count_exchange is both.  Shared scratch (sh: 3 x 32 Acc, shi: 32 ints, at
// most 16 warps): the warps' partials in sh[k * 32 + warp] / shi[warp], the group result
// in sh[64 + k] / shi[16], shi[17], so the result of one exchange and the partials of the
// next never share a word and neither half needs a barrier after its last read.  Within
// a group of more than one block only warp 0 needs the block's sums (to publish them):
// one block barrier, then warp 0 reduces the warp partials in the same fixed shuffle tree
// as block_sum_or; the barrier also orders every store the block made before it ahead
// of the release that publishes.
//
// A group is `size` consecutive blocks starting at block `first` that share one arrival
// counter `counter` (zero at launch); the whole grid is the group (0, gridDim.x).  Slots
// are indexed by block in both generation buffers of gridDim.x slots.
template <class Acc, int N>
__device__ __forceinline__ void count_publish(ExSlot* slots, unsigned* counter, int size, unsigned gen, Acc (&v)[N],
                                              int& bad, Acc* sh, int* shi)
{
    static_assert(N >= 1 && N <= 2, "two partials per slot");
    if (size <= 1) {  // no other block: every thread needs the block's sums
        block_sum_or<Acc, N>(v, bad, sh, shi);
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    bad = (int)__reduce_or_sync(0xffffffffu, (unsigned)bad);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) sh[k * 32 + warp] = v[k];
        shi[warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            Acc t = lane < nw ? sh[k * 32 + lane] : Acc(0);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
            v[k] = t;
        }
        int b = lane < nw ? shi[lane] : 0;
        b = (int)__reduce_or_sync(0xffffffffu, (unsigned)b);
        if (lane == 0) {
            ExSlot* my = slots + (gen & 1u) * (unsigned)gridDim.x + blockIdx.x;
            my->v0 = double(v[0]);
            my->v1 = N > 1 ? double(v[N - 1]) : 0.0;
            my->bad = b;
            // The release increment: a release is cumulative, so it also orders the
            // block's stores that the block barrier ordered before it (no separate fence).
            red_release_add(counter, 1u);
        }
    }
}

// `limit`: polls before the wait gives up (the wait self-test passes a small one).
template <class Acc, int N>
__device__ bool count_finish(ExSlot* slots, unsigned* counter, int first, int size, GridSync* sync, unsigned gen,
                             Acc (&v)[N], int& bad, Acc* sh, int* shi,
                             unsigned long long limit = kBarrierSpinLimit)
{
    const int G = gridDim.x, tid = threadIdx.x, lane = tid & 31;
    if (size <= 1) return !*(volatile int*)&sync->err;
    const ExSlot* buf = slots + (gen & 1u) * (unsigned)G + first;
    if ((tid >> 5) == (int)(blockDim.x >> 5) - 1) {
        const unsigned target = gen * (unsigned)size;
        int fail = 0;
        unsigned long long spins = 0;
        while ((int)(ld_acquire(counter) - target) < 0) {
            if (++spins > limit) {
                atomicExch(&sync->err, 1);
                fail = 1;
                break;
            }
            if ((spins & 1023u) == 0 && *(volatile int*)&sync->err) {
                fail = 1;
                break;
            }
        }
        fail = __any_sync(0xffffffffu, fail) ? 1 : 0;
        Acc pv[N];
#pragma unroll
        for (int k = 0; k < N; ++k) pv[k] = Acc(0);
        int pb = 0;
        if (!fail) {
            for (int i = lane; i < size; i += 32) {
                pv[0] += Acc(__ldcg(&buf[i].v0));
                if (N > 1) pv[N - 1] += Acc(__ldcg(&buf[i].v1));
                pb |= __ldcg(&buf[i].bad);
            }
        }
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) pv[k] += __shfl_xor_sync(0xffffffffu, pv[k], off);
        pb = (int)__reduce_or_sync(0xffffffffu, (unsigned)pb);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < N; ++k) sh[64 + k] = pv[k];
            shi[16] = pb;
            shi[17] = fail;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[64 + k];
    bad = shi[16];
    const int failed = shi[17];
    return !failed && !*(volatile int*)&sync->err;
}

template <class Acc, int N>
__device__ __forceinline__ bool count_exchange(ExSlot* slots, unsigned* counter, int first, int size, GridSync* sync,
                                               unsigned gen, Acc (&v)[N], int& bad, Acc* sh, int* shi,
                                               unsigned long long limit = kBarrierSpinLimit)
{
    count_publish<Acc, N>(slots, counter, size, gen, v, bad, sh, shi);
    return count_finish<Acc, N>(slots, counter, first, size, sync, gen, v, bad, sh, shi, limit);
}

// The whole grid as one group (slots: two buffers of gridDim.x).
template <class Acc, int N>
__device__ __forceinline__ bool grid_exchange(ExSlot* slots, GridSync* sync, unsigned gen, Acc (&v)[N], int& bad,
                                              Acc* sh, int* shi)
{
    return group_exchange<Acc, N>(slots, (int)gridDim.x, (int)gridDim.x, (int)blockIdx.x, sync, gen, v, bad, sh, shi);
}

}  // namespace
}  // namespace pk
