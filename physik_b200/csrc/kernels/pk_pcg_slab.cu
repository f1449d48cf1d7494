// pk_pcg_slab.cu -- the part-resident cooperative block-Jacobi PCG kernel.
//
// The same solve as the other PCG kernels (SolvePreconditionedConjugateGradient,
// src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241, with the SpMV of
// SparseBlockMatrix::Multiply, src/Math/SparseBlockMatrix.cpp:209-268, and
// World::IntegrateImplicitEuler, src/Core/World/World.cpp:644-695, fused at the end), for
// FP32 storage, laid out so that HBM only streams the matrix:
//
// * One block per part (pk_slab_plan.h).  The search directions d of the part's window
//   (its rows, then its halo) stay in shared memory for the whole solve.  At the start of
//   an iteration every block rebuilds its window as d = s + beta d: its own rows from the
//   s its threads keep in registers, the halo rows from the s the neighbouring parts
//   published (a part publishes only the rows some other window holds), so the SpMV
//   reads d only from shared memory.  A part's interior rows (no halo column) come first,
//   and a halo warp fills the halo rows while the consumers already stream the interior
//   tiles; a consumer waits for the halo only at the first tile whose header flags a
//   halo column.
// * Per-body solves run as one persistent launch: each block takes one part per round,
//   in order, from a round table the device rebuilds before every solve
//   (slab_schedule_kernel); a body of several parts is a group of consecutive blocks in
//   one round with its own exchange slots and counter.
// * The part's rows are streamed as tiles of full symmetric rows (upper blocks and the
//   transposes of the lower ones, 16-bit window columns) by one producer warp, one TMA
//   bulk copy per tile into a ring of stages, with an L2 evict-first policy so the
//   streamed matrix does not push the CG vectors out of L2.  The producer runs ahead
//   into the next iteration's first tiles while the block exchanges and updates.
// * Three consumer groups of four warps take every third ring position; four lanes per
//   row, up to four blocks per lane in flight.  Per row the products are summed lane by lane and then in a fixed shuffle tree,
//   the partial dot products of every phase in a fixed block tree, and the grid
//   exchange reduces the blocks' partials in one fixed tree that every block evaluates
//   identically: all blocks take the same decisions and a run repeats bit for bit.
//
// The symmetric stream form (pk_slab_plan.h) streams each block inside a sub-part once: a
// consumer group takes only its own sub-part's tiles, and per tile first evaluates every
// entry's product (a transposing entry also writes B^T d_r to its slot of the group's
// shared-memory ring), waits at the group's named barrier, then completes each row's q
// as its own sum plus its ring slots in order, and waits again before the next tile
// writes.  All sums keep one fixed order, so runs still repeat bit for bit.
//
// Each row's x, r and M^-1 live in tensor memory (TMEM) for the whole solve: the twelve
// consumer warps own rows t + 384k (t = their thread, k < 10), and warp w keeps row k at
// TMEM lane 32 (w % 4) + lane, columns 160 (w / 4) + 16k .. + 15, read and written with
// tcgen05.ld / tcgen05.st.  Only q (phase A -> phase B, other threads) and the published
// s go through global memory.  Every wait is bounded; a wait that gives up
// sets the error flag and the kernel leaves through its normal exit, after waiting
// (bounded) for its own bulk copies still in flight.  No TMA multicast is used.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pk_device.cuh"

namespace pk {
namespace {

__device__ __forceinline__ void mbar_arrive_slab(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ unsigned long long l2_evict_first_policy()
{
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Bulk copy global -> shared with an L2 cache-policy hint (no multicast).
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
                                              unsigned long long pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}

__device__ __forceinline__ V3<float> ldv4(const float* p)
{
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    return V3<float>{a.x, a.y, a.z};
}
__device__ __forceinline__ void stv4(float* p, V3<float> v)
{
    __stcg(reinterpret_cast<float4*>(p), make_float4(v.x, v.y, v.z, 0.f));
}
// ------------------------------------------------------------------ tensor memory
// One row record: 16 32-bit columns {x.xyz, r.xyz, M^-1 (9, column-major), unused}.  Each
// load / store is warp-wide (.sync.aligned) and waits for its own completion.
struct RowRec {
    unsigned w[16];
};
__device__ __forceinline__ void tmem_ld16(unsigned taddr, RowRec& r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3]), "=r"(r.w[4]), "=r"(r.w[5]), "=r"(r.w[6]),
          "=r"(r.w[7]), "=r"(r.w[8]), "=r"(r.w[9]), "=r"(r.w[10]), "=r"(r.w[11]), "=r"(r.w[12]), "=r"(r.w[13]),
          "=r"(r.w[14]), "=r"(r.w[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_st16(unsigned taddr, const RowRec& r)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n\t"
        "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
        "r"(r.w[0]), "r"(r.w[1]), "r"(r.w[2]), "r"(r.w[3]), "r"(r.w[4]), "r"(r.w[5]), "r"(r.w[6]), "r"(r.w[7]),
        "r"(r.w[8]), "r"(r.w[9]), "r"(r.w[10]), "r"(r.w[11]), "r"(r.w[12]), "r"(r.w[13]), "r"(r.w[14]), "r"(r.w[15])
        : "memory");
}
// x and r of a row record (its first 8 columns: x.xyz, r.xyz and two M^-1 words as they
// were), without waiting: the caller waits once (tmem_wait_st) before the next reads.
__device__ __forceinline__ void tmem_st8_nowait(unsigned taddr, const RowRec& r)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r.w[0]),
                 "r"(r.w[1]), "r"(r.w[2]), "r"(r.w[3]), "r"(r.w[4]), "r"(r.w[5]), "r"(r.w[6]), "r"(r.w[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ V3<float> rec3(const RowRec& r, int o)
{
    return V3<float>{__uint_as_float(r.w[o]), __uint_as_float(r.w[o + 1]), __uint_as_float(r.w[o + 2])};
}
__device__ __forceinline__ void put3(RowRec& r, int o, V3<float> v)
{
    r.w[o] = __float_as_uint(v.x);
    r.w[o + 1] = __float_as_uint(v.y);
    r.w[o + 2] = __float_as_uint(v.z);
}
__device__ __forceinline__ M3<float> rec_minv(const RowRec& r)
{
    M3<float> m;
    m.c[0] = rec3(r, 6);
    m.c[1] = rec3(r, 9);
    m.c[2] = rec3(r, 12);
    return m;
}

// Waits (bounded) until the shared-memory flag holds `want`; false when it gave up.
__device__ __forceinline__ bool wait_flag_shared(const int* flag, int want)
{
    for (unsigned long long spins = 0; *(const volatile int*)flag != want; ++spins) {
        if (spins > kBarrierSpinLimit) return false;
        __nanosleep(32);
    }
    __threadfence_block();
    return true;
}

// Named barrier of the consumer warps (the symmetric form's groups use 1 .. kSlabGroups).
constexpr unsigned kSlabOwnBar = 1 + kSlabGroups;

// alpha split into two floats, hi = float(alpha) and lo = float(alpha - hi), so that the
// FP32 updates x + alpha d and r - alpha q take two FMAs per component instead of the
// float -> double -> float round trip (24 conversions a row, which bound phase B: the
// conversion unit retires a quarter of a warp per cycle).  The result is within one
// float ulp of the FP64 update; with FP32 reductions lo is zero and is not applied.
template <class Acc>
struct SplitAlpha {
    float hi, lo;
    __device__ __forceinline__ explicit SplitAlpha(Acc a) : hi(float(a)), lo(float(a - Acc(float(a)))) {}
    __device__ __forceinline__ V3<float> axpy(V3<float> a, V3<float> b) const
    {
        V3<float> t{fmaf(hi, b.x, a.x), fmaf(hi, b.y, a.y), fmaf(hi, b.z, a.z)};
        if constexpr (sizeof(Acc) == 8) t = V3<float>{fmaf(lo, b.x, t.x), fmaf(lo, b.y, t.y), fmaf(lo, b.z, t.z)};
        return t;
    }
};

template <class Acc>
__global__ void __launch_bounds__(kSlabThreads, 1) pcg_slab_kernel(SlabPcgArgs<Acc> P)
{
    constexpr int S = kSlabStages;
    constexpr int LPR = kSlabLanesPerRow;
    extern __shared__ __align__(128) unsigned char dyn[];
    __shared__ __align__(8) unsigned long long full_bar[S];
    __shared__ __align__(8) unsigned long long empty_bar[S];
    __shared__ Acc sh_acc[3 * 32];
    __shared__ int sh_int[32];
    __shared__ int s_fail;
    __shared__ int s_bad;
    __shared__ int s_stop;  // a bulk copy may still be in flight: no further round
    __shared__ int s_halo_gen;  // the iteration whose window halo the halo warp has filled
    __shared__ unsigned s_tmem;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, blk = blockIdx.x;
    const bool producer = warp == kSlabConsumerWarps;
    const bool consumer = warp < kSlabConsumerWarps;
    const bool halo_warp = warp == kSlabConsumerWarps + 1;
    const int group = warp / kSlabGroupWarps;
    const int slot_row = ((warp % kSlabGroupWarps) * 32 + lane) / LPR;  // tile row of this lane
    const int sub = lane % LPR;
    float* win = reinterpret_cast<float*>(dyn);  // 3 floats per window row
    unsigned char* ring_base = dyn + kSlabRingOffset;
    const bool sym = P.sym != 0;
    const unsigned stage_bytes = sym ? (unsigned)kSymStageBytes : (unsigned)kSlabStageBytes;
    int4* table = reinterpret_cast<int4*>(dyn + (sym ? kSlabSymTableOffset : kSlabTableOffset));
    // symmetric form: this group's ring of transposed products (3 floats per slot)
    float* tp = reinterpret_cast<float*>(dyn + kSlabSymTpOffset) + (size_t)3 * kSymRingSlots * (size_t)(group < kSlabGroups ? group : 0);

    // Precompute failures upstream: every part reports zero statistics and nothing is solved.
    const unsigned in_flags = *(volatile unsigned*)P.flags;
    const bool skip = P.skip_on_flags && (in_flags & (kFlagPrecomputeFailed | kFlagSingularDiag));
    // Tensor memory for the rows' x, r, M^-1 (all 512 columns: one block per SM), held
    // across the rounds.
    if (!skip && warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();

    // One part per block and round (the coupled solve: one round).  A block takes its
    // rounds in order, so a group of round l starts once each of its blocks has finished its
    // parts of the earlier rounds: the group of the lowest unfinished round can always
    // proceed, and no group waits on a later one.
    bool bars_live = false;
    if (tid == 0) s_stop = 0;
    const int my_rounds = P.block_rounds ? min(P.rounds, __ldg(P.block_rounds + blk)) : P.rounds;
    for (int round = 0; round < my_rounds; ++round) {
    // The part: rows [row0, row0 + m) of the slab order, halo rows halo_src[halo0 ..
    // halo0 + h), tiles [tile0, tile0 + ntiles).  A part that does not fit the block's
    // tables (the host never builds one) is emptied and reports a breakdown.
    const size_t slot_of_part = (size_t)round * gridDim.x + (size_t)blk;
    int row0, m, halo0, h, tile0, ntiles, gfirst, gsize;
    {
        const int4 a = __ldg(reinterpret_cast<const int4*>(P.part_info) + 2 * slot_of_part);
        const int4 b = __ldg(reinterpret_cast<const int4*>(P.part_info) + 2 * slot_of_part + 1);
        row0 = a.x;
        m = a.y;
        halo0 = a.z;
        h = a.w;
        tile0 = b.x;
        ntiles = b.y;
        gfirst = b.z;  // this part's group: blocks [gfirst, gfirst + gsize) of the round
        gsize = b.w;
    }
    if (gfirst == kSlabNoGroup && gsize == 0) continue;  // no part for this block in this round
    // The previous round is done with the barriers and tables: the stage barriers start
    // again from phase 0 (the copies issued ahead have landed: see finish).
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            if (bars_live) {
                mbar_inval(&full_bar[s]);
                mbar_inval(&empty_bar[s]);
            }
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kSlabGroupWarps);
        }
        mbar_fence_init();
        s_fail = 0;
        s_bad = 0;
        s_halo_gen = 0;
    }
    bars_live = true;
    __syncthreads();
    // A group must hold this block; the coupled solve is one group of the whole grid.
    const bool group_ok = gfirst >= 0 && gsize >= 1 && gfirst + gsize <= (int)gridDim.x && blk >= gfirst &&
                          blk < gfirst + gsize && (P.grouped || (gfirst == 0 && gsize == (int)gridDim.x));
    int body = 0;
    if (P.grouped) {
        body = __ldg(P.part_body + slot_of_part);
        if ((unsigned)body >= (unsigned)P.nbodies) body = -1;
    }
    if (!group_ok || body < 0) {
        // Not a valid group (the host never builds one): the block works alone and fails.
        gfirst = blk;
        gsize = 1;
        body = 0;
        if (tid == 0) s_bad = 1;
    }
    // The round's exchange slots and its groups' arrival counters.
    ExSlot* const slots = P.slots + (size_t)round * 2 * gridDim.x;
    unsigned* const gcount = P.group_count + (size_t)round * gridDim.x + gfirst;
    BatchBodyStats* const bs = P.grouped ? P.body_stats + body : nullptr;
    const bool leader = P.grouped ? blk == gfirst : blk == 0;
    if (m < 0 || m > kSlabMaxRows || h < 0 || m + h > kSlabWinCap || row0 < 0 || row0 + m > P.n || ntiles < 0 ||
        ntiles > kSlabMaxTiles || halo0 < 0 || halo0 + h > P.halo_count || tile0 < 0 ||
        tile0 + ntiles > P.tile_count || (sym && ntiles % kSlabGroups != 0)) {
        m = h = ntiles = 0;
        row0 = 0;
        if (tid == 0) s_bad = 1;
    }
    const int wn = m + h;
    // Tile descriptors, checked once: a bad one (never built by the host) becomes an empty
    // tile and reports a breakdown.
    for (int i = tid; i < ntiles; i += blockDim.x) {
        int4 d = __ldg(P.tile_desc + tile0 + i);
        bool ok;
        if (sym) {
            // a tile of the group's sub-part, or an empty position (the group has no more)
            const int ne = (d.y - kSymHeaderBytes) / kSymEntryBytes;
            ok = (d.y == 0 && d.w == 0) ||
                 (d.x >= 0 && d.y >= kSymHeaderBytes && d.y <= kSymStageBytes && (d.y & 15) == 0 &&
                  d.y == kSymHeaderBytes + kSymEntryBytes * ne && ne <= kSymCapE && (ne & 7) == 0 && d.w >= 1 &&
                  d.w <= kSymRows && d.z >= 0 && d.z + d.w <= m &&
                  16ull * (unsigned long long)d.x + (unsigned long long)d.y <= P.stream_bytes);
        } else {
            const int ne = (d.y - kSlabHeaderBytes) / kSlabEntryBytes;
            ok = d.x >= 0 && d.y >= kSlabHeaderBytes && d.y <= kSlabStageBytes && (d.y & 15) == 0 &&
                 d.y == kSlabHeaderBytes + kSlabEntryBytes * ne && ne <= kSlabCapE && d.w >= 1 && d.w <= kSlabRows &&
                 d.z >= 0 && d.z + d.w <= m &&
                 16ull * (unsigned long long)d.x + (unsigned long long)d.y <= P.stream_bytes;
        }
        if (!ok) {
            d = make_int4(0, 0, 0, 0);
            s_bad = 1;
        }
        table[i] = d;
    }
    __syncthreads();

    if (skip) {
        if (leader && tid == 0) {
            if (P.grouped) {
                bs->iterations = 0;
                bs->converged = 0;
                bs->residual_norm = 0.0;
                bs->flags = 0;
            } else {
                P.stats->iterations = 0;
                P.stats->converged = 0;
                P.stats->residual_norm = 0.0;
            }
        }
        continue;
    }
    const bool row_owner = warp < kSlabConsumerWarps;  // the 384 threads of the per-row phases
    const int rt = tid;                                 // rows rt + 384 k
    const int krows = (m + kSlabRowThreads - 1) / kSlabRowThreads;
    const unsigned tmem_row0 =
        s_tmem + ((32u * (unsigned)(warp % 4)) << 16) + (unsigned)((warp / 4) * kSlabRowsPerThread * 16);
    const unsigned long long pol = l2_evict_first_policy();
    unsigned ring = 0;    // ring positions consumed so far (ntiles per iteration)
    unsigned issued = 0;  // ring positions issued by the producer (producer lane 0 only)
    unsigned xgen = 0;
    int hgen = 0;         // window passes so far (the halo flag's generation)

    // Phase A of the symmetric form, for one consumer group: its ring positions are
    // ring + group, ring + group + 3, ... (ntiles is a multiple of 3 and ring starts at 0,
    // so a position's group never changes).  Every warp of the group passes every
    // position and both named barriers, whatever happened (a wait that gave up only
    // empties its tile), so the barriers always complete.
    auto phase_a_sym = [&](Acc& dq, int& qbad) {
        // Two lanes per row: the group's 128 threads cover a whole tile (kSymRows rows) at
        // once; each lane takes every other entry of its row.
        constexpr int LS = 2;
        const float* wv = win;
        const int wmax = max(wn - 1, 0);
        const unsigned gbar = 1u + (unsigned)group;  // named barrier of this group (0 is __syncthreads)
        const int sr = ((warp % kSlabGroupWarps) * 32 + lane) / LS;  // tile row of this lane
        const int ls = lane % LS;
        for (unsigned p = ring + (unsigned)group; p < ring + (unsigned)ntiles; p += kSlabGroups) {
            const int s = (int)(p % S);
            const unsigned u = p / S;
            bool ok = mbar_wait(&full_bar[s], u & 1u);
            if (!ok) s_fail = 1;
            const int4 d = table[p - ring];
            ok = ok && d.y > 0;
            const unsigned char* st = ring_base + (size_t)s * stage_bytes;
            const int ne = ok ? (d.y - kSymHeaderBytes) / kSymEntryBytes : 0;
            const int rows = ok ? d.w : 0;
            const unsigned short* roff = reinterpret_cast<const unsigned short*>(st);
            const unsigned short* lbase = roff + (kSymRows + 1);
            const float* vals = reinterpret_cast<const float*>(st + kSymHeaderBytes);
            const unsigned short* lcol = reinterpret_cast<const unsigned short*>(st + kSymHeaderBytes + 36 * ne);
            const unsigned short* lslot = lcol + ne;
            const bool valid = sr < rows;
            int e0 = 0, e1 = 0;
            unsigned lb0 = 0u, lbn = 0u;
            V3<float> dr{0.f, 0.f, 0.f};
            if (valid) {
                e0 = min((int)roff[sr], ne);
                e1 = min((int)roff[sr + 1], ne);
                lb0 = lbase[sr];
                lbn = ((unsigned)lbase[sr + 1] - lb0) & (unsigned)(kSymRingSlots - 1);
                const int li = min(d.z + sr, wmax);
                dr = V3<float>{wv[3 * li], wv[3 * li + 1], wv[3 * li + 2]};
            }
            V3<float> acc{0.f, 0.f, 0.f};
            constexpr int kEntries = 4;
            for (int j0 = e0 + ls; j0 < e1; j0 += kEntries * LS) {
                int jj[kEntries];
                bool live[kEntries];
#pragma unroll
                for (int q = 0; q < kEntries; ++q) {
                    jj[q] = j0 + q * LS;
                    live[q] = jj[q] < e1;
                    if (!live[q]) jj[q] = j0;
                }
                float xv[kEntries][3], bv[kEntries][9];
                unsigned sl[kEntries];
#pragma unroll
                for (int q = 0; q < kEntries; ++q) {
                    const int c = 3 * min((int)lcol[jj[q]], wmax);
                    xv[q][0] = wv[c];
                    xv[q][1] = wv[c + 1];
                    xv[q][2] = wv[c + 2];
                    sl[q] = lslot[jj[q]];
#pragma unroll
                    for (int e = 0; e < 9; ++e) bv[q][e] = vals[9 * jj[q] + e];
                }
#pragma unroll
                for (int q = 0; q < kEntries; ++q) {
                    // Column-major block: element (i, c) is v[3c + i].
                    const float* v = bv[q];
                    if (live[q]) {
                        acc.x += v[0] * xv[q][0] + v[3] * xv[q][1] + v[6] * xv[q][2];
                        acc.y += v[1] * xv[q][0] + v[4] * xv[q][1] + v[7] * xv[q][2];
                        acc.z += v[2] * xv[q][0] + v[5] * xv[q][1] + v[8] * xv[q][2];
                        if (sl[q] != kSymNoSlot) {  // B^T d_r for the later row
                            float* t = tp + 3 * (sl[q] & (unsigned)(kSymRingSlots - 1));
                            t[0] = v[0] * dr.x + v[1] * dr.y + v[2] * dr.z;
                            t[1] = v[3] * dr.x + v[4] * dr.y + v[5] * dr.z;
                            t[2] = v[6] * dr.x + v[7] * dr.y + v[8] * dr.z;
                        }
                    }
                }
            }
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
            acc.z += __shfl_xor_sync(0xffffffffu, acc.z, 1);
            __syncwarp();
            if (lane == 0) mbar_arrive_slab(&empty_bar[s]);  // this warp is done with the stage
            asm volatile("bar.sync %0, %1;" ::"r"(gbar), "r"(32 * kSlabGroupWarps) : "memory");
            // q = own sum + the row's ring slots in slot order (the two lanes take alternate
            // slots, then one fixed shuffle).
            V3<float> ts{0.f, 0.f, 0.f};
            for (unsigned k = (unsigned)ls; k < lbn; k += LS) {
                const float* t = tp + 3 * ((lb0 + k) & (unsigned)(kSymRingSlots - 1));
                ts.x += t[0];
                ts.y += t[1];
                ts.z += t[2];
            }
            ts.x += __shfl_xor_sync(0xffffffffu, ts.x, 1);
            ts.y += __shfl_xor_sync(0xffffffffu, ts.y, 1);
            ts.z += __shfl_xor_sync(0xffffffffu, ts.z, 1);
            if (valid && ls == 0) {
                const V3<float> q{acc.x + ts.x, acc.y + ts.y, acc.z + ts.z};
                const int li = d.z + sr;
                stv4(P.qs + 4 * (size_t)(row0 + li), q);
                dq += dot_acc<Acc>(dr, q);
                if (!finite3(q)) qbad = 1;
            }
            // the next tile's products may overwrite slots read above
            asm volatile("bar.sync %0, %1;" ::"r"(gbar), "r"(32 * kSlabGroupWarps) : "memory");
        }
    };

    // Phase A: q = A d for the part's rows (d from the window), partial d.q.
    auto phase_a = [&](Acc& dq, int& qbad) {
        if (ntiles == 0) return;
        if (producer) {
            if (lane == 0) {
                // This iteration's tiles, then the next iteration's first ones.
                const unsigned end = ring + (unsigned)ntiles + (unsigned)min(S, ntiles);
                for (; issued < end; ++issued) {
                    const unsigned p = issued;
                    const int s = (int)(p % S);
                    const unsigned u = p / S;
                    if (u > 0 && !mbar_wait(&empty_bar[s], (u - 1) & 1u)) {
                        s_fail = 1;
                        break;
                    }
                    const int4 d = table[p % (unsigned)ntiles];
                    mbar_arrive_expect_tx(&full_bar[s], (unsigned)d.y);
                    if (d.y > 0)
                        bulk_g2s_hint(ring_base + (size_t)s * stage_bytes, P.stream + 16 * (size_t)d.x,
                                      (unsigned)d.y, &full_bar[s], pol);
                }
            }
            __syncwarp();
        } else if (consumer && sym) {
            phase_a_sym(dq, qbad);
        } else if (consumer) {
            const float* wv = win;
            const int wmax = max(wn - 1, 0);
            bool halo_in = false;
            const unsigned first = ring + (unsigned)((group - (int)(ring % kSlabGroups) + kSlabGroups) % kSlabGroups);
            for (unsigned p = first; p < ring + (unsigned)ntiles; p += kSlabGroups) {
                const int s = (int)(p % S);
                const unsigned u = p / S;
                if (!mbar_wait(&full_bar[s], u & 1u)) {
                    s_fail = 1;
                    break;
                }
                const int4 d = table[p - ring];
                const unsigned char* st = ring_base + (size_t)s * stage_bytes;
                const int ne = d.y > 0 ? (d.y - kSlabHeaderBytes) / kSlabEntryBytes : 0;
                const unsigned short* roff = reinterpret_cast<const unsigned short*>(st);
                // the first tile with a halo column waits until the halo warp has filled it
                if (!halo_in && d.y > 0 && roff[kSlabHaloWord] != 0) {
                    if (!wait_flag_shared(&s_halo_gen, hgen)) s_fail = 1;
                    halo_in = true;
                }
                const float* vals = reinterpret_cast<const float*>(st + kSlabHeaderBytes);
                const unsigned short* lcol = reinterpret_cast<const unsigned short*>(st + kSlabHeaderBytes + 36 * ne);
                const bool valid = slot_row < d.w;
                int e0 = 0, e1 = 0;
                if (valid) {
                    e0 = min((int)roff[slot_row], ne);
                    e1 = min((int)roff[slot_row + 1], ne);
                }
                V3<float> acc{0.f, 0.f, 0.f};
                // kEntries independent entries per lane per pass, every load issued before
                // the products; a dead slot re-reads the pass's first entry and adds nothing.
                constexpr int kEntries = 4;
                for (int j0 = e0 + sub; j0 < e1; j0 += kEntries * LPR) {
                    int jj[kEntries];
                    bool live[kEntries];
#pragma unroll
                    for (int q = 0; q < kEntries; ++q) {
                        jj[q] = j0 + q * LPR;
                        live[q] = jj[q] < e1;
                        if (!live[q]) jj[q] = j0;
                    }
                    float xv[kEntries][3], bv[kEntries][9];
#pragma unroll
                    for (int q = 0; q < kEntries; ++q) {
                        const int c = 3 * min((int)lcol[jj[q]], wmax);
                        xv[q][0] = wv[c];
                        xv[q][1] = wv[c + 1];
                        xv[q][2] = wv[c + 2];
#pragma unroll
                        for (int e = 0; e < 9; ++e) bv[q][e] = vals[9 * jj[q] + e];
                    }
#pragma unroll
                    for (int q = 0; q < kEntries; ++q) {
                        // Column-major block: element (i, c) is v[3c + i].
                        const float* v = bv[q];
                        if (live[q]) {
                            acc.x += v[0] * xv[q][0] + v[3] * xv[q][1] + v[6] * xv[q][2];
                            acc.y += v[1] * xv[q][0] + v[4] * xv[q][1] + v[7] * xv[q][2];
                            acc.z += v[2] * xv[q][0] + v[5] * xv[q][1] + v[8] * xv[q][2];
                        }
                    }
                }
#pragma unroll
                for (int off = LPR / 2; off > 0; off >>= 1) {
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
                    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive_slab(&empty_bar[s]);  // this warp is done with the stage
                if (valid && sub == 0) {
                    const int li = d.z + slot_row;
                    stv4(P.qs + 4 * (size_t)(row0 + li), acc);
                    dq += dot_acc<Acc>(V3<float>{wv[3 * li], wv[3 * li + 1], wv[3 * li + 2]}, acc);
                    if (!finite3(acc)) qbad = 1;
                }
            }
        }
        ring += (unsigned)ntiles;
    };

    // The s values of this thread's rows stay in registers for the next window pass; only
    // rows another part's window holds (expmask) are published to global memory.
    V3<float> sreg[kSlabRowsPerThread];
    unsigned expmask = 0u;
#pragma unroll
    for (int k = 0; k < kSlabRowsPerThread; ++k) {
        sreg[k] = V3<float>{0.f, 0.f, 0.f};
        const int i = rt + kSlabRowThreads * k;
        if (row_owner && k < krows && i < m && __ldg(P.exported + row0 + i)) expmask |= 1u << k;
    }
    unsigned fl = 0;
    int iterations = 0;
    bool converged = false;
    Acc residual = Acc(0);
    bool have_x = true;
    bool timed_out = false;
    Acc delta = Acc(0), rr = Acc(0), target = Acc(0);
    // The first ring positions of the solve, issued before the initial pass so that
    // iteration 0 starts on landed tiles (the stages are not touched until phase A).
    if (producer && lane == 0) {
        const unsigned end = (unsigned)min(S, ntiles);
        for (; issued < end; ++issued) {
            const int s = (int)issued;
            const int4 d = table[issued];
            mbar_arrive_expect_tx(&full_bar[s], (unsigned)d.y);
            if (d.y > 0)
                bulk_g2s_hint(ring_base + (size_t)s * stage_bytes, P.stream + 16 * (size_t)d.x, (unsigned)d.y,
                              &full_bar[s], pol);
        }
    }
    {
        // x = 0, r = b, M^-1 into tensor memory; s = M^-1 r published; d = 0 in the window;
        // r.s, |r|^2, finiteness.
        Acc v[2] = {Acc(0), Acc(0)};
        int bad = s_bad ? 4 : 0;
        if (row_owner) {
            // The rows' dynamic indices all in flight at once, then b and M^-1 of two rows
            // at a time (a tensor-memory store orders the loads after it).
            int cidx[kSlabRowsPerThread];
#pragma unroll
            for (int k = 0; k < kSlabRowsPerThread; ++k) {
                const int i = rt + kSlabRowThreads * k;
                int c = 0;
                if (k < krows && i < m) {
                    c = __ldg(P.perm + row0 + i);
                    if ((unsigned)c >= (unsigned)P.n) {
                        c = 0;
                        bad |= 4;
                    }
                }
                cidx[k] = c;
            }
#pragma unroll
            for (int k0 = 0; k0 < kSlabRowsPerThread; k0 += 2) {
                if (k0 >= krows) break;
                V3<float> brs[2]{};
                M3<float> mis[2]{};
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (k0 + u < krows && rt + kSlabRowThreads * (k0 + u) < m) {
                        brs[u] = ld3(P.b, cidx[k0 + u]);
                        mis[u] = ld9(P.minv, (size_t)cidx[k0 + u]);
                    }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                const int k = k0 + u;
                if (k >= krows) break;
                const int i = rt + kSlabRowThreads * k;
                RowRec rec{};
                if (i < m) {
                    const int g = row0 + i;
                    const V3<float> br = brs[u];
                    if (!finite3(br)) bad |= 1;
                    const M3<float> mi = mis[u];
                    const V3<float> sv = mul(mi, br);
                    if (!finite9(mi) || !finite3(sv)) bad |= 2;
                    put3(rec, 0, V3<float>{0.f, 0.f, 0.f});
                    put3(rec, 3, br);
                    put3(rec, 6, mi.c[0]);
                    put3(rec, 9, mi.c[1]);
                    put3(rec, 12, mi.c[2]);
                    sreg[k] = sv;
                    if ((expmask >> k) & 1u) stv4(P.ss + 4 * (size_t)g, sv);
                    v[0] += dot_acc<Acc>(br, sv);
                    v[1] += dot_acc<Acc>(br, br);
                }
                tmem_st16(tmem_row0 + 16u * (unsigned)k, rec);
                }
            }
        }
        for (int w = tid; w < 3 * wn; w += blockDim.x) win[w] = 0.f;
        if (!count_exchange<Acc, 2>(slots, gcount, gfirst, gsize, P.sync, ++xgen, v, bad, sh_acc, sh_int)) {
            timed_out = true;
            goto finish;
        }
        delta = v[0];
        rr = v[1];
        if (bad & 4) {  // a malformed layout: report, do not solve
            have_x = false;
            fl |= kFlagBreakdown;
            goto final_check;
        }
        if (bad & 1) {  // non-finite rhs: the reference clears x (the solve fails)
            have_x = false;
            fl |= kFlagInvalidRhs;
            goto final_check;
        }
        if (P.max_iterations <= 0 || !acc_finite(P.tolerance) || P.tolerance <= Acc(0)) {
            have_x = false;
            fl |= kFlagInvalidRhs;
            goto final_check;
        }
        if (bad & 2) goto final_check;  // preconditioner output not finite: x stays 0
        if (!acc_finite(delta) || delta < Acc(0)) goto final_check;
        target = P.tolerance * P.tolerance * delta;
        if (!acc_finite(target)) goto final_check;
    }
    if (delta <= target) {
        converged = true;
        residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
        goto final_check;
    }
    {
        Acc beta = Acc(0);
        for (int it = 0; it < P.max_iterations; ++it) {
            if (delta <= target) {
                converged = true;
                break;
            }
            // Window: d = s + beta d -- the part's own rows from their owners' registers,
            // the halo rows from the s their owners published.  Full form: the consumers
            // write the own rows and start on the part's interior tiles (interior rows come
            // first) while the halo warp fills the halo and then raises the halo flag.
            // Symmetric form: every thread takes halo rows, and a block barrier ends the pass.
            int hbad = 0;
            ++hgen;
            {
                const float bt = float(beta);
                if (row_owner) {
#pragma unroll
                    for (int k = 0; k < kSlabRowsPerThread; ++k) {
                        const int i = rt + kSlabRowThreads * k;
                        if (k < krows && i < m) {
                            float* d = win + 3 * i;
                            d[0] = sreg[k].x + d[0] * bt;
                            d[1] = sreg[k].y + d[1] * bt;
                            d[2] = sreg[k].z + d[2] * bt;
                        }
                    }
                }
                // kWinBatch halo entries per thread per pass: their indices, then their s
                // values are all in flight before any is used.
                constexpr int kWinBatch = 8;
                if (sym || halo_warp) {
                    const int step = sym ? (int)blockDim.x : 32;
                    for (int w0 = m + (sym ? tid : lane); w0 < wn; w0 += kWinBatch * step) {
                        int g[kWinBatch];
#pragma unroll
                        for (int k = 0; k < kWinBatch; ++k) {
                            const int w = w0 + k * step;
                            int gi = 0;
                            if (w < wn) gi = __ldg(P.halo_src + halo0 + (w - m));
                            if ((unsigned)gi >= (unsigned)P.n) {
                                gi = 0;
                                hbad = 1;
                            }
                            g[k] = gi;
                        }
                        float4 sv[kWinBatch];
#pragma unroll
                        for (int k = 0; k < kWinBatch; ++k)
                            sv[k] = __ldcg(reinterpret_cast<const float4*>(P.ss) + g[k]);
#pragma unroll
                        for (int k = 0; k < kWinBatch; ++k) {
                            const int w = w0 + k * step;
                            if (w < wn) {
                                float* d = win + 3 * w;
                                d[0] = sv[k].x + d[0] * bt;
                                d[1] = sv[k].y + d[1] * bt;
                                d[2] = sv[k].z + d[2] * bt;
                            }
                        }
                    }
                }
                if (!sym && halo_warp) {
                    __syncwarp();
                    if (lane == 0) {
                        __threadfence_block();
                        *(volatile int*)&s_halo_gen = hgen;
                    }
                }
            }
            if (sym)
                __syncthreads();
            else if (row_owner)  // every own row is written before a consumer reads it
                asm volatile("bar.sync %0, %1;" ::"r"(kSlabOwnBar), "r"(kSlabRowThreads) : "memory");
            Acc dq[1] = {Acc(0)};
            int qbad = 0;
            phase_a(dq[0], qbad);
            if (s_bad || hbad) qbad = 1;
            if (s_fail) {
                qbad = 1;
                atomicExch(&P.sync->err, 1);
            }
            count_publish<Acc, 1>(slots, gcount, gsize, ++xgen, dq, qbad, sh_acc, sh_int);
            // Phase B's q (written by other threads in phase A, visible after the publish's
            // block barrier) loads while the exchange completes.
            V3<float> qv[kSlabRowsPerThread];
#pragma unroll
            for (int k = 0; k < kSlabRowsPerThread; ++k) {
                const int i = rt + kSlabRowThreads * k;
                qv[k] = (row_owner && k < krows && i < m) ? ldv4(P.qs + 4 * (size_t)(row0 + i))
                                                          : V3<float>{0.f, 0.f, 0.f};
            }
            if (!count_finish<Acc, 1>(slots, gcount, gfirst, gsize, P.sync, xgen, dq, qbad, sh_acc, sh_int)) {
                timed_out = true;
                goto finish;
            }
            if (qbad) {
                fl |= kFlagBreakdown;
                break;
            }
            if (!acc_finite(dq[0]) || dq[0] <= Acc(0)) {
                fl |= kFlagBreakdown;
                break;
            }
            const Acc alpha = delta / dq[0];
            if (!acc_finite(alpha)) {
                fl |= kFlagBreakdown;
                break;
            }
            // Phase B: x += alpha d; r -= alpha q; s = M^-1 r; partials r.s and r.r.  x, r,
            // M^-1 from tensor memory; q was loaded while the exchange completed.
            Acc v[2] = {Acc(0), Acc(0)};
            int sbad = 0;
            if (row_owner) {
                const SplitAlpha<Acc> pa(alpha), na(-alpha);
                // Stores of x, r (8 columns) without waits: one wait after the loop.
#pragma unroll
                for (int k = 0; k < kSlabRowsPerThread; ++k) {
                    if (k >= krows) break;
                    const int i = rt + kSlabRowThreads * k;
                    RowRec rec;
                    tmem_ld16(tmem_row0 + 16u * (unsigned)k, rec);
                    if (i < m) {
                        const float* d = win + 3 * i;
                        const V3<float> xv = pa.axpy(rec3(rec, 0), V3<float>{d[0], d[1], d[2]});
                        const V3<float> rv = na.axpy(rec3(rec, 3), qv[k]);
                        const V3<float> sv = mul(rec_minv(rec), rv);
                        if (!finite3(sv)) sbad = 1;
                        sreg[k] = sv;
                        if ((expmask >> k) & 1u) stv4(P.ss + 4 * (size_t)(row0 + i), sv);
                        // r widened once for both dots
                        const Acc r0 = Acc(rv.x), r1 = Acc(rv.y), r2 = Acc(rv.z);
                        v[0] += r0 * Acc(sv.x) + r1 * Acc(sv.y) + r2 * Acc(sv.z);
                        v[1] += r0 * r0 + r1 * r1 + r2 * r2;
                        put3(rec, 0, xv);
                        put3(rec, 3, rv);
                    }
                    tmem_st8_nowait(tmem_row0 + 16u * (unsigned)k, rec);
                }
                tmem_wait_st();
            }
            if (!count_exchange<Acc, 2>(slots, gcount, gfirst, gsize, P.sync, ++xgen, v, sbad, sh_acc, sh_int)) {
                timed_out = true;
                goto finish;
            }
            rr = v[1];
            if (sbad) {
                fl |= kFlagBreakdown;
                break;
            }
            const Acc old = delta;
            delta = v[0];
            if (!acc_finite(delta) || !acc_finite(old) || old <= Acc(0)) {
                fl |= kFlagBreakdown;
                break;
            }
            beta = delta / old;
            if (!acc_finite(beta)) {
                fl |= kFlagBreakdown;
                break;
            }
            iterations = it + 1;
        }
        if (delta <= target) converged = true;
        residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
    }

final_check:
    // delta-v back in dynamic-row order; the solve succeeds when it is present and
    // finite; integration is all-or-nothing.
    // The thread's row and node indices and delta-v stay in registers for the integration
    // pass; row and node indices load all at once, node states two rows at a time.
    {
        int bad = 0;
        Acc none[1] = {Acc(0)};
        const V3<float> zero{0.f, 0.f, 0.f};
        int cidx[kSlabRowsPerThread], nidx[kSlabRowsPerThread];
        V3<float> dvs[kSlabRowsPerThread];
#pragma unroll
        for (int k = 0; k < kSlabRowsPerThread; ++k) {
            const int i = rt + kSlabRowThreads * k;
            cidx[k] = -1;
            nidx[k] = 0;
            dvs[k] = zero;
            if (row_owner && k < krows && i < m) {
                const int c = __ldg(P.perm + row0 + i);
                if ((unsigned)c >= (unsigned)P.n)
                    bad |= 1;
                else
                    cidx[k] = c;
            }
        }
        if (P.integrate) {
#pragma unroll
            for (int k = 0; k < kSlabRowsPerThread; ++k)
                if (cidx[k] >= 0) nidx[k] = __ldg(P.dyn_to_node + cidx[k]);
        }
        if (row_owner) {
#pragma unroll
            for (int k0 = 0; k0 < kSlabRowsPerThread; k0 += 2) {
                if (k0 >= krows) break;
                V3<float> xo[2] = {zero, zero}, vo[2] = {zero, zero};
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    if (P.integrate && cidx[k0 + u] >= 0) {
                        xo[u] = ldplain3(P.node_x, nidx[k0 + u]);
                        vo[u] = ldplain3(P.node_v, nidx[k0 + u]);
                    }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int k = k0 + u;
                    if (k >= krows) break;
                    RowRec rec;
                    tmem_ld16(tmem_row0 + 16u * (unsigned)k, rec);  // warp-wide
                    if (cidx[k] < 0) continue;
                    const V3<float> dv = have_x ? rec3(rec, 0) : zero;
                    dvs[k] = dv;
                    st3(P.x, cidx[k], dv);
                    if (!finite3(dv)) bad |= 1;
                    if (P.integrate) {
                        const V3<float> nv = vo[u] + dv;
                        const V3<float> nx = xo[u] + nv * P.dt;
                        if (!finite3(xo[u]) || !finite3(vo[u]) || !finite3(nv) || !finite3(nx)) bad |= 2;
                    }
                }
            }
        }
        if (!count_exchange<Acc, 1>(slots, gcount, gfirst, gsize, P.sync, ++xgen, none, bad, sh_acc, sh_int)) {
            timed_out = true;
            goto finish;
        }
        const bool solved = have_x && !(bad & 1);
        if (!have_x && !(fl & kFlagBreakdown)) fl |= kFlagInvalidRhs;
        if (have_x && (bad & 1)) fl |= kFlagNonFiniteDv;
        if (solved) fl |= kFlagSolved;
        if (solved && P.integrate) {
            if (bad & 2) {
                fl |= kFlagIntegrateAbort;
            } else {
#pragma unroll
                for (int k0 = 0; k0 < kSlabRowsPerThread; k0 += 2) {
                    V3<float> xo[2] = {zero, zero}, vo[2] = {zero, zero};
#pragma unroll
                    for (int u = 0; u < 2; ++u)
                        if (cidx[k0 + u] >= 0) {
                            vo[u] = ldplain3(P.node_v, nidx[k0 + u]);
                            xo[u] = ldplain3(P.node_x, nidx[k0 + u]);
                        }
#pragma unroll
                    for (int u = 0; u < 2; ++u)
                        if (cidx[k0 + u] >= 0) {
                            const V3<float> nv = vo[u] + dvs[k0 + u];
                            const V3<float> nx = xo[u] + nv * P.dt;
                            st3(P.node_v, nidx[k0 + u], nv);
                            st3(P.node_x, nidx[k0 + u], nx);
                        }
                }
                fl |= kFlagIntegrated;
            }
        }
        if (converged) fl |= kFlagConverged;
    }

finish:
    if (timed_out) fl |= kFlagBarrierTimeout;
    // Bulk copies issued ahead (the next iteration's first tiles) or cut short by a
    // timeout must land before the block exits: wait for the last S positions issued.
    if (producer && lane == 0) {
        for (unsigned k = 0; k < (unsigned)S && k < issued; ++k) {
            const unsigned p = issued - 1 - k;
            if (!mbar_wait(&full_bar[p % S], (p / S) & 1u)) s_stop = 1;
        }
    }
    // The next round rewrites the tensor memory once every warp's accesses are done.
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    if (leader && tid == 0 && P.grouped) {
        // Per body; world-wide: the largest iteration count and residual, the OR of the
        // failure flags and the AND of the success flags (missing: what some body lacks).
        bs->iterations = iterations;
        bs->converged = converged ? 1 : 0;
        bs->residual_norm = (double)residual;
        bs->flags = fl;
        atomicMax(&P.stats->iterations, iterations);
        if (residual >= Acc(0))  // non-negative doubles order like their bit patterns
            atomicMax(reinterpret_cast<unsigned long long*>(&P.stats->residual_norm),
                      (unsigned long long)__double_as_longlong((double)residual));
        atomicOr(P.flags, fl & ~(kFlagSolved | kFlagIntegrated | kFlagConverged));
        if (!(fl & kFlagSolved)) atomicOr(P.missing, kFlagSolved);
        if (!(fl & kFlagIntegrated)) atomicOr(P.missing, kFlagIntegrated);
        if (!(fl & kFlagConverged)) atomicOr(P.missing, kFlagConverged);
    } else if (leader && tid == 0) {
        P.stats->iterations = iterations;
        P.stats->converged = converged ? 1 : 0;
        P.stats->residual_norm = (double)residual;
        atomicOr(P.flags, fl);
    } else if (timed_out && tid == 0) {
        atomicOr(P.flags, kFlagBarrierTimeout);
    }
    if (s_stop) {  // read after the round's last block barrier: the same for every thread
        if (tid == 0) {
            atomicExch(&P.sync->err, 1);
            atomicOr(P.flags, kFlagBarrierTimeout);
        }
        break;
    }
    }  // rounds
    // Release the tensor memory once every warp's accesses are done.
    if (!skip) {
        tmem_fence_before();
        __syncthreads();
        if (warp == 0) {
            tmem_fence_after();
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(512u) : "memory");
        }
    }
}

// One block per tile: the tile's value area (9 floats per entry, a multiple of 4 floats
// starting on a 16-byte boundary) written in stream order with 16-byte stores, each float
// gathered from its upper block -- element j = 3 c + i of a transposed entry is element
// 3 i + c of the block; padding entries are zero.  A tile that does not match its entry
// list (the host never builds one) is left alone.
constexpr int kSlabFillThreads = 128;
__global__ void __launch_bounds__(kSlabFillThreads)
    slab_fill_kernel(const float* __restrict__ values, int nnz, const int4* __restrict__ tile_desc,
                     const int* __restrict__ tile_entry0, int ntiles, const unsigned* __restrict__ fill_src,
                     int nentries, float* __restrict__ out, unsigned long long out_floats, int header_bytes,
                     int entry_bytes)
{
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    const int4 d = __ldg(tile_desc + t);
    const int e0 = __ldg(tile_entry0 + t), e1 = __ldg(tile_entry0 + t + 1);
    const int ne = e1 - e0;
    const unsigned long long v0 = 4ull * (unsigned long long)d.x + (unsigned long long)(header_bytes / 4);
    if (e0 < 0 || ne <= 0 || e1 > nentries || d.x < 0 || (ne & 7) != 0 || d.y != header_bytes + entry_bytes * ne ||
        v0 + 9ull * (unsigned long long)ne > out_floats)
        return;
    float4* dst = reinterpret_cast<float4*>(out + v0);
    const unsigned* src = fill_src + e0;
    const int n4 = 9 * ne / 4;
    for (int f4 = threadIdx.x; f4 < n4; f4 += kSlabFillThreads) {
        float v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int f = 4 * f4 + q;
            const int e = f / 9, j = f - 9 * e;
            const unsigned s = __ldg(src + e);
            v[q] = 0.f;
            if (s != kSlabNoPos) {
                const unsigned k = s & ~kSlabLowerBit;
                const int jj = (s & kSlabLowerBit) ? 3 * (j % 3) + j / 3 : j;
                if (k < (unsigned)nnz) v[q] = __ldg(values + 9 * (size_t)k + jj);
            }
        }
        dst[f4] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// The round table of the per-body launch (SlabScheduleArgs).  Deterministic: fixed-order
// float sums, ties broken by index, so the same iteration counts build the same table; a
// body's result does not depend on the table.
__global__ void __launch_bounds__(kSlabSchedThreads) slab_schedule_kernel(SlabScheduleArgs A)
{
    __shared__ float load[kSlabSchedMaxGrid];
    __shared__ int count[kSlabSchedMaxGrid];
    __shared__ int order[kSlabSchedMaxSort];
    __shared__ float dur[kSlabSchedMaxSort];
    __shared__ int nparts[kSlabSchedMaxSort];  // then: the round the body went to
    __shared__ int first[kSlabSchedMaxSort];   // the first block it went to (-1: none)
    const int tid = threadIdx.x, lane = tid & 31, G = A.grid, nb = A.nbodies;
    if (G <= 0 || G > kSlabSchedMaxGrid || A.rounds < 1 || nb > kSlabSchedMaxSort) {
        if (tid == 0) atomicOr(A.flags, kFlagBreakdown);  // the host never builds such a table
        return;
    }
    // every entry idle; blocks free at time 0; each body's parts and estimated duration:
    // iterations x (c0 + row cost of its largest part)
    for (int i = tid; i < A.rounds * G; i += blockDim.x) {
        int* dst = A.out_info + (size_t)kSlabPartInts * i;
        for (int q = 0; q < kSlabPartInts; ++q) dst[q] = 0;
        dst[6] = kSlabNoGroup;
        A.out_body[i] = 0;
    }
    for (int b = tid; b < G; b += blockDim.x) {
        load[b] = 0.f;
        count[b] = 0;
    }
    for (int i = tid; i < nb; i += blockDim.x) {
        const int p0 = A.body_part0[i], k = A.body_parts[i];
        const int id = A.plan_body[p0];
        float it = float(A.max_iterations);
        if ((unsigned)id < (unsigned)A.nstats) {
            const BatchBodyStats st = A.body_stats[id];
            if (st.flags != 0u || st.iterations != 0) it = float(min(max(st.iterations, 0), A.max_iterations));
        }
        int rows = 0;
        for (int q = 0; q < k; ++q) rows = max(rows, A.plan_info[(size_t)kSlabPartInts * (p0 + q) + 1]);
        dur[i] = it * ((k > 1 ? kSlabSchedMultiUs : kSlabSchedSingleUs) + kSlabSchedRowUs * float(rows));
        nparts[i] = k;
        first[i] = -1;
    }
    __syncthreads();
    // bodies ranked by estimated work, duration x parts, largest first (ties: plan order):
    // a group needs several blocks free at once, which gets harder as the blocks fill
    for (int i = tid; i < nb; i += blockDim.x) {
        const float wi = dur[i] * float(nparts[i]);
        int rank = 0;
        for (int j = 0; j < nb; ++j) {
            const float wj = dur[j] * float(nparts[j]);
            rank += (wj > wi || (wj == wi && j < i)) ? 1 : 0;
        }
        order[rank] = i;
    }
    __syncthreads();
    // one warp places them, from shared memory only
    if (tid < 32) {
        for (int t = 0; t < nb; ++t) {
            const int i = order[t];
            const int k = nparts[i];
            // the window [b, b + k) that is free earliest and has a round left
            float best = INFINITY;
            int bb = 0x7fffffff;
            for (int b = lane; b + k <= G; b += 32) {
                float st = 0.f;
                int rd = 0;
                for (int q = b; q < b + k; ++q) {
                    st = fmaxf(st, load[q]);
                    rd = max(rd, count[q]);
                }
                if (rd < A.rounds && (st < best || (st == best && b < bb))) {
                    best = st;
                    bb = b;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bb, off);
                if (ob < best || (ob == best && oi < bb)) {
                    best = ob;
                    bb = oi;
                }
            }
            if (bb == 0x7fffffff) {  // no room: the host sized the table too small
                if (lane == 0) atomicOr(A.flags, kFlagBreakdown);
                break;
            }
            if (lane == 0) {
                int r = 0;
                for (int q = bb; q < bb + k; ++q) r = max(r, count[q]);
                for (int q = bb; q < bb + k; ++q) {
                    count[q] = r + 1;
                    load[q] = best + dur[i];
                }
                nparts[i] = r;  // k is not needed any more: the round
                first[i] = bb;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // the table entries of the placed bodies, in parallel
    for (int i = tid; i < nb; i += blockDim.x) {
        const int bb = first[i];
        if (bb < 0) continue;
        const int r = nparts[i], p0 = A.body_part0[i], k = A.body_parts[i];
        for (int q = 0; q < k; ++q) {
            const size_t e = (size_t)r * G + bb + q;
            int* dst = A.out_info + (size_t)kSlabPartInts * e;
            const int* src = A.plan_info + (size_t)kSlabPartInts * (p0 + q);
            for (int c = 0; c < 6; ++c) dst[c] = src[c];
            dst[6] = bb;  // the group: blocks [bb, bb + k) of round r
            dst[7] = k;
            A.out_body[e] = A.plan_body[p0 + q];
        }
    }
    for (int b = tid; b < G; b += blockDim.x) A.out_rounds[b] = count[b];
}

}  // namespace

// ------------------------------------------------------------------ launchers
cudaError_t launch_slab_schedule_kernel(const SlabScheduleArgs& args, cudaStream_t stream)
{
    slab_schedule_kernel<<<1, kSlabSchedThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

template <class Acc>
static cudaError_t slab_prepare()
{
    return cudaFuncSetAttribute(pcg_slab_kernel<Acc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(kSlabSmemBytes));
}

template <class Acc>
int pcg_slab_max_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (slab_prepare<Acc>() != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_slab_kernel<Acc>, kSlabThreads, kSlabSmemBytes) !=
        cudaSuccess)
        return 0;
    return sms * per_sm;
}

template <class Acc>
cudaError_t launch_pcg_slab_kernel(const SlabPcgArgs<Acc>& args, int grid, cudaStream_t stream)
{
    SlabPcgArgs<Acc> a = args;
    void* kargs[] = {&a};
    cudaError_t e = slab_prepare<Acc>();
    if (e != cudaSuccess) return e;
    // Each form asks only for its own shared memory: a larger request moves the SM's
    // carve-out towards shared memory and leaves less L1 (the full form at the symmetric
    // form's 217 KB instead of its own 193 KB measured ~1 us slower per iteration).
    const size_t smem = args.sym ? kSlabSymSmemBytes : kSlabFullSmemBytes;
    return cudaLaunchCooperativeKernel((const void*)pcg_slab_kernel<Acc>, dim3(grid), dim3(kSlabThreads), kargs, smem,
                                       stream);
}

cudaError_t launch_slab_fill_kernel(const float* values, int nnz, const int* tile_desc, const int* tile_entry0,
                                    int ntiles, const unsigned* fill_src, int nentries, float* out,
                                    unsigned long long out_floats, int sym, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    slab_fill_kernel<<<ntiles, kSlabFillThreads, 0, stream>>>(
        values, nnz, reinterpret_cast<const int4*>(tile_desc), tile_entry0, ntiles, fill_src, nentries, out, out_floats,
        sym ? kSymHeaderBytes : kSlabHeaderBytes, sym ? kSymEntryBytes : kSlabEntryBytes);
    return cudaGetLastError();
}

template cudaError_t launch_pcg_slab_kernel<float>(const SlabPcgArgs<float>&, int, cudaStream_t);
template cudaError_t launch_pcg_slab_kernel<double>(const SlabPcgArgs<double>&, int, cudaStream_t);
template int pcg_slab_max_grid<float>();
template int pcg_slab_max_grid<double>();

}  // namespace pk
