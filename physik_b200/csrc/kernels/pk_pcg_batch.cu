// pk_pcg_batch.cu -- batched block-Jacobi PCG: many independent bodies in one launch,
// each with its own CG scalars, stopping test, iteration count and all-or-nothing
// integration.
//
// Per body it is the solve of SolvePreconditionedConjugateGradient
// (src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:114-241) on the body's diagonal
// block of the upper-stored symmetric BSR (SparseBlockMatrix::Multiply,
// src/Math/SparseBlockMatrix.cpp:209-268), followed by World::IntegrateImplicitEuler
// (src/Core/World/World.cpp:644-695) -- what a reference World holding only that body
// computes.  (A reference World holding all bodies runs one coupled PCG with global
// scalars instead; that is the default, unbatched, path of this library.)
//
// Work layout: a body's dynamic rows are contiguous.  The host cuts every body into
// parts of about equal row count and gives each part one block; a body's parts are
// consecutive blocks, its "group".  Group members exchange partial dot products through
// generation-tagged slots (the same exchange as the ring-staged kernel, restricted to the
// group), so only blocks of one body ever wait for each other and a converged body's
// blocks simply finish.  A body of one part needs no exchange beyond its block.  The
// launch is cooperative so every group is co-resident.
//
// Per pass a block takes 64 rows (4 lanes per row, up to 4 independent entries per lane,
// every load of a pass issued before its products); the neighbours' {s, d} records and
// the transposed lower blocks are gathered from global memory.  Every wait is bounded;
// no __trap; no TMA.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pk_device.cuh"

namespace pk {
namespace {

template <class Real>
struct BRec {
    V3<Real> s, d;
};
#pragma nv_diag_suppress 550
__device__ __forceinline__ BRec<float> bld_rec(const float* sd, int c)
{
    float a0, a1, a2, a3, a4, a5, a6, a7;
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(a4), "=f"(a5), "=f"(a6), "=f"(a7)
                 : "l"(sd + 8 * (size_t)c));
    return BRec<float>{V3<float>{a0, a1, a2}, V3<float>{a4, a5, a6}};
}
__device__ __forceinline__ BRec<double> bld_rec(const double* sd, int c)
{
    double a0, a1, a2, a3, a4, a5, a6, a7;
    const double* p = sd + 8 * (size_t)c;
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3) : "l"(p));
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a4), "=d"(a5), "=d"(a6), "=d"(a7) : "l"(p + 4));
    return BRec<double>{V3<double>{a0, a1, a2}, V3<double>{a4, a5, a6}};
}
#pragma nv_diag_default 550
__device__ __forceinline__ void bst4(float* p, V3<float> v)
{
    __stcg(reinterpret_cast<float4*>(p), make_float4(v.x, v.y, v.z, 0.f));
}
__device__ __forceinline__ void bst4(double* p, V3<double> v)
{
    __stcg(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
    __stcg(reinterpret_cast<double2*>(p) + 1, make_double2(v.z, 0.0));
}
__device__ __forceinline__ V3<float> bld4(const float* p)
{
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    return V3<float>{a.x, a.y, a.z};
}
__device__ __forceinline__ V3<double> bld4(const double* p)
{
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p)), b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return V3<double>{a.x, a.y, b.x};
}

constexpr int kBatchLanesPerRow = 4;
constexpr int kBatchEntries = 4;  // entries per lane per pass

template <class Real, class Acc>
__global__ void __launch_bounds__(kBatchThreads, 2) pcg_batch_kernel(BatchPcgArgs<Real, Acc> P)
{
    constexpr int LPR = kBatchLanesPerRow, NE = kBatchEntries;
    constexpr int kRowsPerPass = kBatchThreads / LPR;
    __shared__ Acc sh_acc[3 * 32];
    __shared__ int sh_int[32];

    const int tid = threadIdx.x, sub = tid % LPR;
    const int4 pd = __ldg(reinterpret_cast<const int4*>(P.parts) + 2 * blockIdx.x);
    const int4 pg = __ldg(reinterpret_cast<const int4*>(P.parts) + 2 * blockIdx.x + 1);
    const int body = pd.x, r0 = pd.y, r1 = pd.z, me = pd.w;   // this part: rows [r0, r1) of body
    const int g0 = pg.x, members = pg.y;                      // the body's parts: blocks [g0, g0 + members)
    BatchBodyStats* bs = P.body_stats + body;
    ExSlot* slots = P.slots + g0;
    const int stride = (int)gridDim.x;
    const Real dt = P.dt;

    unsigned fl = 0;
    int iterations = 0;
    bool converged = false, have_x = true, timed_out = false;
    Acc residual = Acc(0), delta = Acc(0), rr = Acc(0), target = Acc(0);
    unsigned xgen = 0;

    const unsigned in_flags = *(volatile unsigned*)P.flags;
    if (P.skip_on_flags && (in_flags & (kFlagPrecomputeFailed | kFlagSingularDiag))) {
        if (me == 0 && tid == 0) {
            bs->iterations = 0;
            bs->converged = 0;
            bs->residual_norm = 0.0;
            bs->flags = 0;
        }
        return;
    }

    {
        // x = 0, r = b, s = M^-1 r, d = 0; delta = r.s, |r|^2, finiteness.
        Acc v[2] = {Acc(0), Acc(0)};
        int bad = 0;
        for (int r = r0 + tid; r < r1; r += blockDim.x) {
            const V3<Real> br = ld3(P.b, r);
            if (!finite3(br)) bad |= 1;
            const V3<Real> z{Real(0), Real(0), Real(0)};
            st3(P.x, r, z);
            st3(P.r, r, br);
            const M3<Real> mi = ld9(P.minv, (size_t)r);
            const V3<Real> s = mul(mi, br);
            if (!finite9(mi) || !finite3(s)) bad |= 2;
            bst4(P.sd0 + 8 * (size_t)r, s);
            bst4(P.sd0 + 8 * (size_t)r + 4, z);
            v[0] += dot_acc<Acc>(br, s);
            v[1] += dot_acc<Acc>(br, br);
        }
        if (!group_exchange<Acc, 2>(slots, stride, members, me, P.sync, ++xgen, v, bad, sh_acc, sh_int)) {
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
        if (bad & 2) goto final_check;
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
            // Phase A: d_next = s + beta d; q = A d_next; partial d_next . q
            Acc dq[1] = {Acc(0)};
            int qbad = 0;
            const Real rb = Real(beta);
            // The next pass's row extents are loaded while this pass's entries are in flight.
            auto extents = [&](int row, int4& e) {
                e = make_int4(0, 0, 0, 0);
                if (row < r1) {
                    e.x = __ldg(P.a.row_start + row);
                    e.y = __ldg(P.a.row_start + row + 1);
                    e.z = __ldg(P.a.lt_start + row);
                    e.w = __ldg(P.a.lt_start + row + 1);
                }
            };
            int4 ext_next;
            extents(r0 + tid / LPR, ext_next);
            for (int base = r0; base < r1; base += kRowsPerPass) {
                const int r = base + tid / LPR;
                const bool valid = r < r1;
                const int4 ext = ext_next;
                extents(r + kRowsPerPass, ext_next);
                const int ks = ext.x, nu = ext.y - ext.x, ls = ext.z, tot = nu + (ext.w - ext.z);
                V3<Real> acc{Real(0), Real(0), Real(0)};
                for (int j0 = sub; j0 < tot; j0 += NE * LPR) {
                    int c[NE], kb[NE];
                    bool tr[NE], live[NE];
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        const int j = j0 + q * LPR;
                        live[q] = j < tot;
                        tr[q] = j >= nu;
                        c[q] = r;
                        kb[q] = ks;  // the diagonal block: a valid address for dead slots
                        if (live[q] && !tr[q]) {
                            kb[q] = ks + j;
                            c[q] = __ldg(P.a.col + kb[q]);
                        } else if (live[q]) {
                            const int e = ls + (j - nu);
                            kb[q] = __ldg(P.a.lt_block + e);
                            c[q] = __ldg(P.a.lt_row + e);
                        }
                        if ((unsigned)c[q] >= (unsigned)P.a.n || (unsigned)kb[q] >= (unsigned)P.nnz) {
                            c[q] = r;
                            kb[q] = ks;
                            qbad = 1;
                        }
                    }
                    BRec<Real> rc[NE];
                    Real bv[NE][9];
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        rc[q] = bld_rec(sdcur, c[q]);
                        const Real* bp = P.a.values + 9 * (size_t)kb[q];
#pragma unroll
                        for (int e = 0; e < 9; ++e) bv[q][e] = __ldg(bp + e);
                    }
#pragma unroll
                    for (int q = 0; q < NE; ++q) {
                        const V3<Real> xc = rc[q].s + rc[q].d * rb;
                        // Column-major block: element (i, m) is bv[3m + i]; the transposed
                        // lower entry swaps (0,1)/(1,0), (0,2)/(2,0), (1,2)/(2,1).
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
                if (valid && sub == 0) {
                    const BRec<Real> own = bld_rec(sdcur, r);
                    const V3<Real> dn = own.s + own.d * rb;
                    bst4(sdnext + 8 * (size_t)r + 4, dn);
                    bst4(P.q4 + 4 * (size_t)r, acc);
                    dq[0] += dot_acc<Acc>(dn, acc);
                    if (!finite3(acc)) qbad = 1;
                }
            }
            if (!group_exchange<Acc, 1>(slots, stride, members, me, P.sync, ++xgen, dq, qbad, sh_acc, sh_int)) {
                timed_out = true;
                goto finish;
            }
            if (qbad || !acc_finite(dq[0]) || dq[0] <= Acc(0)) {
                fl |= kFlagBreakdown;
                break;
            }
            const Acc alpha = delta / dq[0];
            if (!acc_finite(alpha)) {
                fl |= kFlagBreakdown;
                break;
            }
            // Phase B: x += alpha d; r -= alpha q; s = M^-1 r; partials r.s and r.r
            Acc v[2] = {Acc(0), Acc(0)};
            int sbad = 0;
            for (int r = r0 + tid; r < r1; r += blockDim.x) {
                const V3<Real> dn = bld4(sdnext + 8 * (size_t)r + 4);
                const V3<Real> q = bld4(P.q4 + 4 * (size_t)r);
                const V3<Real> xv = axpy<Real, Acc>(ldplain3(P.x, r), alpha, dn);
                const V3<Real> rv = axpy<Real, Acc>(ldplain3(P.r, r), -alpha, q);
                st3(P.x, r, xv);
                st3(P.r, r, rv);
                const V3<Real> s = mul(ld9(P.minv, (size_t)r), rv);
                if (!finite3(s)) sbad = 1;
                bst4(sdnext + 8 * (size_t)r, s);
                v[0] += dot_acc<Acc>(rv, s);
                v[1] += dot_acc<Acc>(rv, rv);
            }
            if (!group_exchange<Acc, 2>(slots, stride, members, me, P.sync, ++xgen, v, sbad, sh_acc, sh_int)) {
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
    // The body's solve succeeds when its x is present and finite; its integration is
    // all-or-nothing.
    {
        int bad = 0;
        Acc none[1] = {Acc(0)};
        for (int r = r0 + tid; r < r1; r += blockDim.x) {
            const V3<Real> dv = have_x ? ldplain3(P.x, r) : V3<Real>{Real(0), Real(0), Real(0)};
            if (!finite3(dv)) bad |= 1;
            if (P.integrate) {
                const int node = __ldg(P.dyn_to_node + r);
                const V3<Real> xo = ldplain3(P.node_x, node), vo = ldplain3(P.node_v, node);
                const V3<Real> nv = vo + dv;
                const V3<Real> nx = xo + nv * dt;
                if (!finite3(xo) || !finite3(vo) || !finite3(nv) || !finite3(nx)) bad |= 2;
            }
        }
        if (!group_exchange<Acc, 1>(slots, stride, members, me, P.sync, ++xgen, none, bad, sh_acc, sh_int)) {
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
                for (int r = r0 + tid; r < r1; r += blockDim.x) {
                    const int node = __ldg(P.dyn_to_node + r);
                    const V3<Real> dv = ldplain3(P.x, r);
                    const V3<Real> nv = ldplain3(P.node_v, node) + dv;
                    const V3<Real> nx = ldplain3(P.node_x, node) + nv * dt;
                    st3(P.node_v, node, nv);
                    st3(P.node_x, node, nx);
                }
                fl |= kFlagIntegrated;
            }
        }
        if (converged) fl |= kFlagConverged;
    }

finish:
    if (timed_out) fl |= kFlagBarrierTimeout;
    if (me == 0 && tid == 0) {
        bs->iterations = iterations;
        bs->converged = converged ? 1 : 0;
        bs->residual_norm = (double)residual;
        bs->flags = fl;
        // World-wide summary: the largest iteration count, the OR of the failure flags and
        // the AND of the success flags (cleared below by any body that lacks them).
        atomicMax(&P.stats->iterations, iterations);
        if (residual >= Acc(0))  // non-negative doubles order like their bit patterns
            atomicMax(reinterpret_cast<unsigned long long*>(&P.stats->residual_norm),
                      (unsigned long long)__double_as_longlong((double)residual));
        atomicOr(P.flags, fl & ~(kFlagSolved | kFlagIntegrated | kFlagConverged));
        if (!(fl & kFlagSolved)) atomicOr(P.missing, kFlagSolved);
        if (!(fl & kFlagIntegrated)) atomicOr(P.missing, kFlagIntegrated);
        if (!(fl & kFlagConverged)) atomicOr(P.missing, kFlagConverged);
    } else if (timed_out && tid == 0) {
        atomicOr(P.flags, kFlagBarrierTimeout);
    }
}

}  // namespace

// ------------------------------------------------------------------ launchers
template <class Real, class Acc>
int pcg_batch_max_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_batch_kernel<Real, Acc>, kBatchThreads, 0) !=
        cudaSuccess)
        return 0;
    return sms * per_sm;
}

template <class Real, class Acc>
cudaError_t launch_pcg_batch_kernel(const BatchPcgArgs<Real, Acc>& args, int grid, cudaStream_t stream)
{
    BatchPcgArgs<Real, Acc> a = args;
    void* kargs[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)pcg_batch_kernel<Real, Acc>, dim3(grid), dim3(kBatchThreads), kargs,
                                       0, stream);
}

template cudaError_t launch_pcg_batch_kernel<float, float>(const BatchPcgArgs<float, float>&, int, cudaStream_t);
template cudaError_t launch_pcg_batch_kernel<float, double>(const BatchPcgArgs<float, double>&, int, cudaStream_t);
template cudaError_t launch_pcg_batch_kernel<double, double>(const BatchPcgArgs<double, double>&, int, cudaStream_t);
template int pcg_batch_max_grid<float, float>();
template int pcg_batch_max_grid<float, double>();
template int pcg_batch_max_grid<double, double>();

}  // namespace pk
