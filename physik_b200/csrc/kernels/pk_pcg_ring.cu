// pk_pcg_ring.cu -- the ring-staged cooperative block-Jacobi PCG kernel.
//
// The same solve as pk_pcg.cu (SolvePreconditionedConjugateGradient,
// src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241, on the upper-stored
// symmetric BSR of SparseBlockMatrix::Multiply, src/Math/SparseBlockMatrix.cpp:209-268,
// with World::IntegrateImplicitEuler, src/Core/World/World.cpp:644-695, fused at the end)
// and the same per-iteration phases:
//   A: d = s + beta*d, q = A d, partial d.q
//   B: x += alpha d, r -= alpha q, s = M^-1 r, partials r.s and r.r
// organised for B200 as a producer / consumer pipeline inside one block per SM:
//
// * Warp 12 is the producer.  For every tile of its block (tiles are dealt round-robin
//   over the grid, so the whole grid sweeps one wavefront through the matrix and a row's
//   transposed lower blocks, stored with rows a few planes earlier, are still in L2) it
//   streams the tile's row extents, upper blocks, columns and transposed index into the
//   next ring stage with TMA bulk copies completing on the stage's "full" mbarrier.  It
//   only issues copies: twelve stages keep ~180 KB of matrix in flight per SM.
// * Warps 0..11 are three consumer groups; group g takes ring positions p = g (mod 3).
//   Each row gets 4 lanes (8 in FP64), each lane up to 4 independent entries, so ~1,500
//   gathers of neighbour records and lower blocks are in flight per SM.  A group frees
//   a stage on its "empty" mbarrier; no consumer ever waits for another group.
// * A grid exchange replaces barrier + reduction: every block publishes its partials in
//   its own 32-byte slot with a release store of the exchange's generation, and polls
//   all slots in parallel (one thread per block).  The slot sums are reduced in one fixed
//   tree that every block evaluates identically, so all blocks take the same decisions
//   and a run repeats bit for bit.  Slots are double buffered by generation parity so a
//   block running ahead cannot overwrite partials another block has not read yet.
//
// Every wait is bounded (kMbarSpinLimit / kBarrierSpinLimit polls), after which the
// kernel records the failure and leaves through the same exit path; no __trap.  No TMA
// multicast is used.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pk_device.cuh"

namespace pk {
namespace {

// ------------------------------------------------------------------ barriers
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ------------------------------------------------------------------ records
template <class Real>
struct Rec {
    V3<Real> s, d;
};
// s and d of row c from its 8-value record (L1 bypassed: written by other blocks).  The
// vector load also fills the two padding slots, which are not used.
#pragma nv_diag_suppress 550
__device__ __forceinline__ Rec<float> ld_rec(const float* sd, int c)
{
    float a0, a1, a2, a3, a4, a5, a6, a7;
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(a4), "=f"(a5), "=f"(a6), "=f"(a7)
                 : "l"(sd + 8 * (size_t)c));
    return Rec<float>{V3<float>{a0, a1, a2}, V3<float>{a4, a5, a6}};
}
__device__ __forceinline__ Rec<double> ld_rec(const double* sd, int c)
{
    double a0, a1, a2, a3, a4, a5, a6, a7;
    const double* p = sd + 8 * (size_t)c;
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3) : "l"(p));
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a4), "=d"(a5), "=d"(a6), "=d"(a7) : "l"(p + 4));
    return Rec<double>{V3<double>{a0, a1, a2}, V3<double>{a4, a5, a6}};
}
#pragma nv_diag_default 550

// 16-byte {v.xyz, 0} stores / loads at element offset `off` of a 4- or 8-value slot.
__device__ __forceinline__ void st4(float* p, V3<float> v)
{
    __stcg(reinterpret_cast<float4*>(p), make_float4(v.x, v.y, v.z, 0.f));
}
__device__ __forceinline__ void st4(double* p, V3<double> v)
{
    __stcg(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
    __stcg(reinterpret_cast<double2*>(p) + 1, make_double2(v.z, 0.0));
}
__device__ __forceinline__ V3<float> ld4(const float* p)
{
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    return V3<float>{a.x, a.y, a.z};
}
__device__ __forceinline__ V3<double> ld4(const double* p)
{
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p)), b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return V3<double>{a.x, a.y, b.x};
}
template <class Real>
__device__ __forceinline__ M3<Real> sblock(const Real* p)
{
    M3<Real> B;
    B.c[0] = V3<Real>{p[0], p[1], p[2]};
    B.c[1] = V3<Real>{p[3], p[4], p[5]};
    B.c[2] = V3<Real>{p[6], p[7], p[8]};
    return B;
}

// ------------------------------------------------------------------ the kernel
template <class Real, class Acc>
__global__ void __launch_bounds__(kRingThreads, 1) pcg_ring_kernel(RingPcgArgs<Real, Acc> P)
{
    using T = RingTile<Real>;
    using LY = RingLayout<Real>;
    constexpr int S = T::kStages;
    constexpr int LPR = T::kLanesPerRow;
    constexpr int NE = sizeof(Real) == 8 ? 2 : 4;  // entries per lane per pass (in registers)
    static_assert(S % kRingGroups == 0, "a stage must always return to the same consumer group");
    extern __shared__ __align__(128) unsigned char dyn[];
    __shared__ __align__(8) unsigned long long full_bar[S];
    __shared__ __align__(8) unsigned long long empty_bar[S];
    __shared__ Acc sh_acc[3 * 32];
    __shared__ int sh_int[32];
    __shared__ int s_fail;
    __shared__ int s_bad_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, blk = blockIdx.x;
    const int my_tiles = blk < P.ntiles ? min((P.ntiles - 1 - blk) / G + 1, kRingMaxTilesPerBlock) : 0;
    const bool producer = warp == kRingConsumerWarps;
    const bool consumer = warp < kRingConsumerWarps;
    const int group = warp / kRingGroupWarps;
    const int slot_row = ((warp % kRingGroupWarps) * 32 + lane) / LPR;  // tile row of this lane
    const int sub = lane % LPR;                                          // entry lane within the row
    int* table = reinterpret_cast<int*>(dyn + LY::kTable);              // the block's tile descriptors

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kRingGroupWarps);
        }
        mbar_fence_init();
        s_fail = 0;
        s_bad_tile = 0;
    }
    // Descriptors of this block's tiles, checked once against the stage capacities; a bad
    // one (the host tiler never makes one) becomes an empty tile and reports a breakdown.
    for (int i = tid; i < my_tiles; i += blockDim.x) {
        const int4* dp = reinterpret_cast<const int4*>(P.desc + kRingDescInts * (size_t)(blk + i * G));
        int4 d0 = __ldg(dp), d1 = __ldg(dp + 1);
        const bool ok = d0.y > d0.x && d0.y - d0.x <= T::kRows && d0.x >= d0.z && d0.w > 0 &&
                        d0.w <= T::kRsCap && d0.y + 1 <= d0.z + d0.w && d1.y > 0 && d1.y <= T::kCapU &&
                        d1.w >= 0 && d1.w <= T::kCapL && ((d0.z | d0.w | d1.x | d1.y | d1.z | d1.w) & 3) == 0;
        if (!ok) {
            d0 = make_int4(0, 0, 0, 0);
            d1 = make_int4(0, 0, 0, 0);
            s_bad_tile = 1;
        }
        reinterpret_cast<int4*>(table)[2 * i] = d0;
        reinterpret_cast<int4*>(table)[2 * i + 1] = d1;
    }
    __syncthreads();

    const unsigned in_flags = *(volatile unsigned*)P.flags;
    if (P.skip_on_flags && (in_flags & (kFlagPrecomputeFailed | kFlagSingularDiag))) {
        if (blk == 0 && tid == 0) {
            P.stats->iterations = 0;
            P.stats->converged = 0;
            P.stats->residual_norm = 0.0;
        }
        return;
    }

    // Every row this block owns, in one fixed thread mapping (all per-row phases).
    auto for_rows = [&](auto&& f) {
        const int total = my_tiles * T::kRows;
        for (int slot = tid; slot < total; slot += blockDim.x) {
            const int i = slot / T::kRows;
            const int r = table[kRingDescInts * i] + (slot - i * T::kRows);
            if (r < table[kRingDescInts * i + 1]) f(r);
        }
    };

    unsigned ring = 0;  // ring positions used so far (same count in producer and consumers)
    unsigned xgen = 0;  // grid exchanges so far

    // Phase A of one iteration: q = A (s + beta d) for the block's tiles; d_next stored.
    auto phase_a = [&](const Real* sdcur, Real* sdnext, Real beta, Acc& dq, int& qbad) {
        if (producer) {
            if (lane == 0) {
                for (int i = 0; i < my_tiles; ++i) {
                    const unsigned p = ring + (unsigned)i;
                    const int s = (int)(p % S);
                    const unsigned u = p / S;
                    if (u > 0 && !mbar_wait(&empty_bar[s], (u - 1) & 1u)) {
                        s_fail = 1;
                        break;
                    }
                    const int4 d0 = reinterpret_cast<const int4*>(table)[2 * i];
                    const int4 d1 = reinterpret_cast<const int4*>(table)[2 * i + 1];
                    const int rs0 = d0.z, nrs = d0.w, k0 = d1.x, nk = d1.y, e0 = d1.z, ne = d1.w;
                    unsigned char* st = dyn + (size_t)s * LY::kBytes;
                    const unsigned tx = nk > 0 ? 8u * nrs + (unsigned(sizeof(Real)) * 9u + 4u) * nk + 8u * ne : 0u;
                    mbar_arrive_expect_tx(&full_bar[s], tx);
                    if (nk > 0) {
                        bulk_g2s(st + LY::kRs, P.a.row_start + rs0, 4u * nrs, &full_bar[s]);
                        bulk_g2s(st + LY::kLts, P.a.lt_start + rs0, 4u * nrs, &full_bar[s]);
                        bulk_g2s(st + LY::kVals, P.a.values + 9 * (size_t)k0, unsigned(sizeof(Real)) * 9u * nk,
                                 &full_bar[s]);
                        bulk_g2s(st + LY::kCol, P.a.col + k0, 4u * nk, &full_bar[s]);
                        if (ne > 0) {
                            bulk_g2s(st + LY::kLtr, P.a.lt_row + e0, 4u * ne, &full_bar[s]);
                            bulk_g2s(st + LY::kLtb, P.a.lt_block + e0, 4u * ne, &full_bar[s]);
                        }
                    }
                }
            }
            __syncwarp();
        } else if (consumer) {
            // Ring positions p = group (mod kRingGroups) of this phase.
            const unsigned first = ring + (unsigned)((group - (int)(ring % kRingGroups) + kRingGroups) % kRingGroups);
            for (unsigned p = first; p < ring + (unsigned)my_tiles; p += kRingGroups) {
                const int i = (int)(p - ring);
                const int s = (int)(p % S);
                const unsigned u = p / S;
                if (!mbar_wait(&full_bar[s], u & 1u)) {
                    s_fail = 1;
                    break;
                }
                const int4 d0 = reinterpret_cast<const int4*>(table)[2 * i];
                const int4 d1 = reinterpret_cast<const int4*>(table)[2 * i + 1];
                const unsigned char* st = dyn + (size_t)s * LY::kBytes;
                const int* rs = reinterpret_cast<const int*>(st + LY::kRs);
                const int* lts = reinterpret_cast<const int*>(st + LY::kLts);
                const Real* vals = reinterpret_cast<const Real*>(st + LY::kVals);
                const int* col = reinterpret_cast<const int*>(st + LY::kCol);
                const int* ltr = reinterpret_cast<const int*>(st + LY::kLtr);
                const int* ltb = reinterpret_cast<const int*>(st + LY::kLtb);
                const int nr = d0.y - d0.x;
                const bool valid = slot_row < nr;
                const int r = d0.x + slot_row;
                int ks = 0, nu = 0, ls = 0, tot = 0;
                if (valid) {
                    const int o = r - d0.z;  // inside [0, nrs - 1) by the descriptor check
                    ks = rs[o];
                    nu = rs[o + 1] - ks;
                    ls = lts[o];
                    tot = nu + (lts[o + 1] - ls);
                }
                Rec<Real> own{};
                if (valid && sub == 0) own = ld_rec(sdcur, r);
                V3<Real> acc{Real(0), Real(0), Real(0)};
                // Branch-free entries: an upper entry reads its block from the stage, a
                // transposed lower entry from global memory through the staged index, both
                // through one generic pointer; the transpose is a swap of three element
                // pairs.  Indices are clamped to the stage capacities and ranges; a bad one
                // reads a valid wrong entry and reports a breakdown.  Dead slots read the
                // stage's first block and this row's record and add nothing.
                for (int j0 = sub; j0 < tot; j0 += NE * LPR) {
                    const Real* bp[NE];
                    int c[NE];
                    bool tr[NE], live[NE];
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        const int j = j0 + q * LPR;
                        live[q] = j < tot;
                        tr[q] = j >= nu;
                        const int kk = min(max(ks + j - d1.x, 0), T::kCapU - 1);
                        const int ee = min(max(ls + (j - nu) - d1.z, 0), T::kCapL - 1);
                        int cc = live[q] ? *(tr[q] ? ltr + ee : col + kk) : r;
                        int kb = ltb[ee];
                        if ((unsigned)cc >= (unsigned)P.a.n) {
                            cc = 0;
                            qbad = 1;
                        }
                        const bool from_global = live[q] && tr[q];
                        if (from_global && (unsigned)kb >= (unsigned)P.nnz) {
                            kb = 0;
                            qbad = 1;
                        }
                        c[q] = cc;
                        bp[q] = from_global ? P.a.values + 9 * (size_t)kb : vals + 9 * kk;
                    }
                    Rec<Real> rc[NE];
                    Real bv[NE][9];
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        rc[q] = ld_rec(sdcur, c[q]);
#pragma unroll
                        for (int e = 0; e < 9; ++e) bv[q][e] = bp[q][e];
                    }
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        const V3<Real> xc = rc[q].s + rc[q].d * beta;
                        // Column-major block: element (i, m) is bv[3m + i]; the transpose swaps
                        // (0,1)/(1,0), (0,2)/(2,0), (1,2)/(2,1).
                        const Real* v = bv[q];
                        const Real a01 = tr[q] ? v[1] : v[3], a10 = tr[q] ? v[3] : v[1];
                        const Real a02 = tr[q] ? v[2] : v[6], a20 = tr[q] ? v[6] : v[2];
                        const Real a12 = tr[q] ? v[5] : v[7], a21 = tr[q] ? v[7] : v[5];
                        const V3<Real> y{v[0] * xc.x + a01 * xc.y + a02 * xc.z, a10 * xc.x + v[4] * xc.y + a12 * xc.z,
                                         a20 * xc.x + a21 * xc.y + v[8] * xc.z};
                        if (live[q]) acc = acc + y;
                    }
                }
#pragma unroll
                for (int off = LPR / 2; off > 0; off >>= 1) {
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
                    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[s]);  // this warp is done with the stage
                if (valid && sub == 0) {
                    const V3<Real> dn = own.s + own.d * beta;
                    st4(sdnext + 8 * (size_t)r + 4, dn);
                    st4(P.q4 + 4 * (size_t)r, acc);
                    dq += dot_acc<Acc>(dn, acc);
                    if (!finite3(acc)) qbad = 1;
                }
            }
        }
        ring += (unsigned)my_tiles;
    };

    unsigned fl = 0;
    int iterations = 0;
    bool converged = false;
    Acc residual = Acc(0);
    bool have_x = true;
    bool timed_out = false;

    Acc delta = Acc(0), rr = Acc(0), target = Acc(0);
    {
        // x = 0, r = b, s = M^-1 r, d = 0 (record sd0); delta = r.s, |r|^2, finiteness.
        Acc v[2] = {Acc(0), Acc(0)};
        int bad = 0;
        for_rows([&](int r) {
            const V3<Real> br = ld3(P.b, r);
            if (!finite3(br)) bad |= 1;
            const V3<Real> z{Real(0), Real(0), Real(0)};
            st3(P.x, r, z);
            st3(P.r, r, br);
            const M3<Real> mi = ld9(P.minv, (size_t)r);
            const V3<Real> s = mul(mi, br);
            if (!finite9(mi) || !finite3(s)) bad |= 2;
            st4(P.sd0 + 8 * (size_t)r, s);
            st4(P.sd0 + 8 * (size_t)r + 4, z);
            v[0] += dot_acc<Acc>(br, s);
            v[1] += dot_acc<Acc>(br, br);
        });
        if (!grid_exchange<Acc, 2>(P.slots, P.sync, ++xgen, v, bad, sh_acc, sh_int)) {
            timed_out = true;
            goto finish;
        }
        delta = v[0];
        rr = v[1];
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
        Real* sdcur = P.sd0;
        Real* sdnext = P.sd1;
        for (int it = 0; it < P.max_iterations; ++it) {
            if (delta <= target) {
                converged = true;
                break;
            }
            Acc dq[1] = {Acc(0)};
            int qbad = 0;
            phase_a(sdcur, sdnext, Real(beta), dq[0], qbad);
            if (s_bad_tile) qbad = 1;
            if (s_fail) {
                qbad = 1;
                atomicExch(&P.sync->err, 1);
            }
            if (!grid_exchange<Acc, 1>(P.slots, P.sync, ++xgen, dq, qbad, sh_acc, sh_int)) {
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
            // Phase B: x += alpha d; r -= alpha q; s = M^-1 r; partials r.s and r.r.  Two
            // rows per thread per pass, all loads of both issued before any store.
            Acc v[2] = {Acc(0), Acc(0)};
            int sbad = 0;
            {
                const int total = my_tiles * T::kRows, step = (int)blockDim.x;
                for (int s0 = tid; s0 < total; s0 += 2 * step) {
                    int rw[2];
                    bool ok[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int slot = s0 + h * step;
                        const int i = min(slot, total - 1) / T::kRows;
                        const int row = table[kRingDescInts * i] + (slot - i * T::kRows);
                        ok[h] = slot < total && row < table[kRingDescInts * i + 1];
                        rw[h] = ok[h] ? row : 0;
                    }
                    V3<Real> dn[2], q[2], xo[2], ro[2];
                    M3<Real> mi[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        dn[h] = ld4(sdnext + 8 * (size_t)rw[h] + 4);
                        q[h] = ld4(P.q4 + 4 * (size_t)rw[h]);
                        xo[h] = ldplain3(P.x, rw[h]);
                        ro[h] = ldplain3(P.r, rw[h]);
                        mi[h] = ld9(P.minv, (size_t)rw[h]);
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (!ok[h]) continue;
                        const V3<Real> xv = axpy<Real, Acc>(xo[h], alpha, dn[h]);
                        const V3<Real> rv = axpy<Real, Acc>(ro[h], -alpha, q[h]);
                        st3(P.x, rw[h], xv);
                        st3(P.r, rw[h], rv);
                        const V3<Real> sv = mul(mi[h], rv);
                        if (!finite3(sv)) sbad = 1;
                        st4(sdnext + 8 * (size_t)rw[h], sv);
                        v[0] += dot_acc<Acc>(rv, sv);
                        v[1] += dot_acc<Acc>(rv, rv);
                    }
                }
            }
            if (!grid_exchange<Acc, 2>(P.slots, P.sync, ++xgen, v, sbad, sh_acc, sh_int)) {
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
            Real* t = sdcur;
            sdcur = sdnext;
            sdnext = t;
            iterations = it + 1;
        }
        if (delta <= target) converged = true;
        residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
    }

final_check:
    // The solve succeeds when x is present and finite; integration is all-or-nothing.
    {
        int bad = 0;
        Acc none[1] = {Acc(0)};
        for_rows([&](int r) {
            const V3<Real> dv = have_x ? ldplain3(P.x, r) : V3<Real>{Real(0), Real(0), Real(0)};
            if (!finite3(dv)) bad |= 1;
            if (P.integrate) {
                const int node = __ldg(P.dyn_to_node + r);
                const V3<Real> xo = ldplain3(P.node_x, node), vo = ldplain3(P.node_v, node);
                const V3<Real> nv = vo + dv;
                const V3<Real> nx = xo + nv * P.dt;
                if (!finite3(xo) || !finite3(vo) || !finite3(nv) || !finite3(nx)) bad |= 2;
            }
        });
        if (!grid_exchange<Acc, 1>(P.slots, P.sync, ++xgen, none, bad, sh_acc, sh_int)) {
            timed_out = true;
            goto finish;
        }
        const bool solved = have_x && !(bad & 1);
        if (!have_x) fl |= kFlagInvalidRhs;
        if (have_x && (bad & 1)) fl |= kFlagNonFiniteDv;
        if (solved) fl |= kFlagSolved;
        if (solved && P.integrate) {
            if (bad & 2) {
                fl |= kFlagIntegrateAbort;
            } else {
                for_rows([&](int r) {
                    const int node = __ldg(P.dyn_to_node + r);
                    const V3<Real> dv = ldplain3(P.x, r);
                    const V3<Real> nv = ldplain3(P.node_v, node) + dv;
                    const V3<Real> nx = ldplain3(P.node_x, node) + nv * P.dt;
                    st3(P.node_v, node, nv);
                    st3(P.node_x, node, nx);
                });
                fl |= kFlagIntegrated;
            }
        }
        if (converged) fl |= kFlagConverged;
    }

finish:
    if (timed_out) {
        fl |= kFlagBarrierTimeout;
        // Let ring copies already issued land before the block exits (bounded waits).
        if (producer && lane == 0) {
            for (unsigned k = 0; k < (unsigned)S && k < ring; ++k) {
                const unsigned p = ring - 1 - k;
                (void)mbar_wait(&full_bar[p % S], (p / S) & 1u);
            }
        }
    }
    if (blk == 0 && tid == 0) {
        P.stats->iterations = iterations;
        P.stats->converged = converged ? 1 : 0;
        P.stats->residual_norm = (double)residual;
        atomicOr(P.flags, fl);
    } else if (timed_out && tid == 0) {
        atomicOr(P.flags, kFlagBarrierTimeout);
    }
}

}  // namespace

// ------------------------------------------------------------------ launchers
template <class Real, class Acc>
static cudaError_t ring_prepare()
{
    return cudaFuncSetAttribute(pcg_ring_kernel<Real, Acc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(RingLayout<Real>::kTotal));
}

template <class Real, class Acc>
int pcg_ring_max_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (ring_prepare<Real, Acc>() != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_ring_kernel<Real, Acc>, kRingThreads,
                                                      RingLayout<Real>::kTotal) != cudaSuccess)
        return 0;
    return sms * per_sm;
}

template <class Real, class Acc>
cudaError_t launch_pcg_ring_kernel(const RingPcgArgs<Real, Acc>& args, int grid, cudaStream_t stream)
{
    RingPcgArgs<Real, Acc> a = args;
    void* kargs[] = {&a};
    cudaError_t e = ring_prepare<Real, Acc>();
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel((const void*)pcg_ring_kernel<Real, Acc>, dim3(grid), dim3(kRingThreads), kargs,
                                       RingLayout<Real>::kTotal, stream);
}

template cudaError_t launch_pcg_ring_kernel<float, float>(const RingPcgArgs<float, float>&, int, cudaStream_t);
template cudaError_t launch_pcg_ring_kernel<float, double>(const RingPcgArgs<float, double>&, int, cudaStream_t);
template cudaError_t launch_pcg_ring_kernel<double, double>(const RingPcgArgs<double, double>&, int, cudaStream_t);
template int pcg_ring_max_grid<float, float>();
template int pcg_ring_max_grid<float, double>();
template int pcg_ring_max_grid<double, double>();

}  // namespace pk
