// pk_kernels.cu -- sm_100a kernels of PhysiK's implicit soft-body step.
//
//   tet_kernel   per tet: F = Ds * DmInv, polar rotation R, corotated stress; stores
//                R and S = R * V * sigma so that node a's elastic force is -S g_a.
//                (FEMModel::ComputeCorotationalElasticForces, FEMModel.cpp:635-679;
//                 ExtractRotationPolar :115-163; ComputeElasticForcesAndStiffness :377-424)
//   row_kernel   per dynamic row: gathers its tets (incidence list, tet order), builds the
//                row's upper blocks dt^2 * sum R Ke_ab R^T (+ m I on the diagonal), the
//                right-hand side dt*(f + m g) - dt^2 * sum K_ab v_b, and the block-Jacobi
//                inverse of its diagonal block.  Deterministic: one thread owns a row and
//                sums in tet order, no atomics.
//                (TetMeshPhysicsComponent::UpdateSystem, TetMeshPhysicsComponent.cpp:293-354;
//                 SolverData::AssembleImplicitMatrixAndRhs, SolverData.cpp:308-465;
//                 SolverData::BuildInversePreconditioner, SolverData.cpp:260-306)
//   spmv_kernel  y = A x for the upper-stored symmetric BSR (SparseBlockMatrix::Multiply,
//                SparseBlockMatrix.cpp:209-268).
// The PCG kernel lives in pk_pcg.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pk_device.cuh"

namespace pk {

namespace {

// ------------------------------------------------------------------ SpMV row
// q_r = sum over the row's upper blocks B x_c plus its transposed lower blocks B^T x_c,
// where x = s + beta*d (d omitted when use_d is false).  W lanes share one row; the
// result is reduced over those lanes (fixed tree) and valid in all of them.
// r < 0 marks an idle row slot that still joins the shuffles.
template <class Real, int W>
__device__ __forceinline__ V3<Real> row_spmv(const BsrView<Real>& A, int r, int hl, const Real* s, const Real* d,
                                             Real beta, bool use_d)
{
    V3<Real> acc{Real(0), Real(0), Real(0)};
    if (r >= 0) {
        const int ks = __ldg(A.row_start + r), ke = __ldg(A.row_start + r + 1);
        const int ls = __ldg(A.lt_start + r), le = __ldg(A.lt_start + r + 1);
        const int nu = ke - ks, tot = nu + (le - ls);
        for (int j = hl; j < tot; j += W) {
            int k, c;
            const bool tr = j >= nu;
            if (!tr) {
                k = ks + j;
                c = __ldg(A.col + k);
            } else {
                const int idx = ls + (j - nu);
                k = __ldg(A.lt_block + idx);
                c = __ldg(A.lt_row + idx);
            }
            const M3<Real> B = ld9(A.values, (size_t)k);
            V3<Real> xc = ldcg3(s, c);
            if (use_d) xc = xc + ldcg3(d, c) * beta;
            acc = acc + (tr ? mul_t(B, xc) : mul(B, xc));
        }
    }
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
    }
    return acc;
}

// ------------------------------------------------------------------ tet records
// A record of kTetRec values moved with 16-byte accesses (it starts on a 16-byte boundary);
// the tet kernel stores its first 18 values (R, S) each step.
__device__ __forceinline__ void st_rec_rs(float* p, const float (&w)[18])
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
        reinterpret_cast<float4*>(p)[i] = make_float4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
    reinterpret_cast<float2*>(p)[8] = make_float2(w[16], w[17]);
}
__device__ __forceinline__ void st_rec_rs(double* p, const double (&w)[18])
{
#pragma unroll
    for (int i = 0; i < 9; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(w[2 * i], w[2 * i + 1]);
}
__device__ __forceinline__ void ld_rec(const float* p, float (&w)[kTetRec])
{
#pragma unroll
    for (int i = 0; i < kTetRec / 4; ++i) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i);
        w[4 * i] = v.x;
        w[4 * i + 1] = v.y;
        w[4 * i + 2] = v.z;
        w[4 * i + 3] = v.w;
    }
}
__device__ __forceinline__ void ld_rec(const double* p, double (&w)[kTetRec])
{
#pragma unroll
    for (int i = 0; i < kTetRec / 2; ++i) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
        w[2 * i] = v.x;
        w[2 * i + 1] = v.y;
    }
}
__device__ __forceinline__ void ld_rec_static(const float* p, float (&w)[12])
{
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(p + 18) + i);
        w[2 * i] = v.x;
        w[2 * i + 1] = v.y;
    }
}
__device__ __forceinline__ void ld_rec_static(const double* p, double (&w)[12])
{
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(p + 18) + i);
        w[2 * i] = v.x;
        w[2 * i + 1] = v.y;
    }
}
template <class Real>
__device__ __forceinline__ M3<Real> rd9(const Real* q)
{
    M3<Real> m;
    m.c[0] = V3<Real>{q[0], q[1], q[2]};
    m.c[1] = V3<Real>{q[3], q[4], q[5]};
    m.c[2] = V3<Real>{q[6], q[7], q[8]};
    return m;
}

// ------------------------------------------------------------------ element stiffness block
// K_ab = V (lambda P_a P_b^T + mu P_b P_a^T + mu (g_a.g_b) R R^T), P = R g, written with
// explicit roundings (products and fused multiply-adds in one fixed order) so that every
// kernel that builds a block produces the same bits, whatever the compiler contracts.
__device__ __forceinline__ float kfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double kfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float kmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double kmul(double a, double b) { return __dmul_rn(a, b); }

__device__ __forceinline__ float kadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double kadd(double a, double b) { return __dadd_rn(a, b); }
template <class Real>
__device__ __forceinline__ V3<Real> kadd3(const V3<Real>& a, const V3<Real>& b)
{
    return V3<Real>{kadd(a.x, b.x), kadd(a.y, b.y), kadd(a.z, b.z)};
}
template <class Real>
__device__ __forceinline__ V3<Real> kscale3(const V3<Real>& a, Real s)
{
    return V3<Real>{kmul(a.x, s), kmul(a.y, s), kmul(a.z, s)};
}
template <class Real>
__device__ __forceinline__ Real kdot(const V3<Real>& a, const V3<Real>& b)
{
    return kfma(a.z, b.z, kfma(a.y, b.y, kmul(a.x, b.x)));
}
// R g for column-major R (R.c[j] is column j).
template <class Real>
__device__ __forceinline__ V3<Real> krot(const M3<Real>& R, const V3<Real>& g)
{
    return V3<Real>{kfma(R.c[2].x, g.z, kfma(R.c[1].x, g.y, kmul(R.c[0].x, g.x))),
                    kfma(R.c[2].y, g.z, kfma(R.c[1].y, g.y, kmul(R.c[0].y, g.x))),
                    kfma(R.c[2].z, g.z, kfma(R.c[1].z, g.y, kmul(R.c[0].z, g.x)))};
}
// R R^T: column j holds the rows' dot products with row j.
template <class Real>
__device__ __forceinline__ M3<Real> krrt(const M3<Real>& R)
{
    const V3<Real> r0{R.c[0].x, R.c[1].x, R.c[2].x}, r1{R.c[0].y, R.c[1].y, R.c[2].y},
        r2{R.c[0].z, R.c[1].z, R.c[2].z};
    M3<Real> m;
    m.c[0] = V3<Real>{kdot(r0, r0), kdot(r1, r0), kdot(r2, r0)};
    m.c[1] = V3<Real>{kdot(r0, r1), kdot(r1, r1), kdot(r2, r1)};
    m.c[2] = V3<Real>{kdot(r0, r2), kdot(r1, r2), kdot(r2, r2)};
    return m;
}
template <class Real>
__device__ __forceinline__ M3<Real> kblock(const V3<Real>& pa, const V3<Real>& pb, const V3<Real>& ga,
                                           const V3<Real>& gb, const M3<Real>& rrt, Real vol, Real lam, Real mu)
{
    const Real l = kmul(vol, lam), m = kmul(vol, mu), md = kmul(m, kdot(ga, gb));
    const Real lp[3] = {kmul(l, pb.x), kmul(l, pb.y), kmul(l, pb.z)};
    const Real mp[3] = {kmul(m, pa.x), kmul(m, pa.y), kmul(m, pa.z)};
    M3<Real> K;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const V3<Real>& rc = rrt.c[j];
        K.c[j] = V3<Real>{kfma(rc.x, md, kfma(pb.x, mp[j], kmul(pa.x, lp[j]))),
                          kfma(rc.y, md, kfma(pb.y, mp[j], kmul(pa.y, lp[j]))),
                          kfma(rc.z, md, kfma(pb.z, mp[j], kmul(pa.z, lp[j])))};
    }
    return K;
}

// ------------------------------------------------------------------ tet kernel
template <class Real, bool kFp64Polar>
__global__ void __launch_bounds__(256) tet_kernel(AssemblyArgs<Real> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.tets.tet_count) return;
    Real* rec = A.tets.rec + kTetRec * (size_t)t;
    // The record's static part: DmInv (values 18..26), volume, lambda, mu (27..29), read
    // with 8-byte loads (value 18 starts on an 8-byte boundary).
    Real st[12];
    ld_rec_static(rec, st);
    const Real vol = st[9];
    const unsigned char en = __ldg(A.tets.enabled + t);
    if (!(en & 1u) || !(vol > Real(0))) {
        rec[0] = qnan<Real>();
        return;
    }
    const bool linear = A.linear || (en & 2u);
    const int4 n = __ldg(A.tets.nodes + t);
    const V3<Real> x0 = ld3(A.x, n.x), x1 = ld3(A.x, n.y), x2 = ld3(A.x, n.z), x3 = ld3(A.x, n.w);
    const M3<Real> ds = mcols(x1 - x0, x2 - x0, x3 - x0);
    const M3<Real> dmi = rd9(st);
    const M3<Real> f = mul(ds, dmi);
    if (!finite9(f)) {
        rec[0] = qnan<Real>();
        return;
    }
    M3<Real> R = mident<Real>();
    if (!linear) {
        int iters = 0;
        bool fallback = false;
        if (kFp64Polar && det(f) <= Real(0.25)) {
            // Near-inverted element: the Newton iteration in double precision.
            R = cast<Real>(polar_rotation<double>(cast<double>(f), &iters, &fallback));
            atomicOr(A.flags, kFlagPolarFp64);
            atomicAdd(&A.stats->polar_fp64_count, 1);
        } else {
            R = polar_rotation<Real>(f, &iters, &fallback);
        }
        if (fallback) {
            atomicOr(A.flags, kFlagPolarIdentity);
            atomicAdd(&A.stats->polar_identity_count, 1);
        }
    }
    const Real lam = st[10], mu = st[11];
    const M3<Real> S = corotated_stress(f, R, linear, vol, lam, mu);
    M3<Real> out = S;
    Real form = Real(0);
    if (A.inc_slot && !A.explicit_mode) {
        // The tet's stiffness times the velocities, folded: with K_ab = R Ke_ab R^T and
        // Ke_ab = V (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I),
        //   sum_b K_ab v_b = Q g_a,  Q = V R (lambda tr(G) I + mu (G + G^T)),
        //   G = R^T sum_b v_b g_b^T = R^T [v1 - v0, v2 - v0, v3 - v0] DmInv,
        // so the row kernel adds T g_a - dt c v_a with T = -(dt S + dt^2 Q) instead of
        // building all 16 blocks.  Used only when every corner force -S g_k - c v_k (the
        // row kernel's force term) and T are finite and no block can overflow; otherwise
        // the row kernel takes the long way with S, which applies the reference's rules
        // for non-finite forces and blocks.
        const V3<Real> vk[4] = {ld3(A.v, n.x), ld3(A.v, n.y), ld3(A.v, n.z), ld3(A.v, n.w)};
        const M3<Real> Q = folded_stiffness(R, dmi, vk, linear, vol, lam, mu);
        const Real dt = A.dt, dt2 = dt * dt;
        M3<Real> T;
#pragma unroll
        for (int j = 0; j < 3; ++j) T.c[j] = -(S.c[j] * dt + Q.c[j] * dt2);
        const Real damp = rec[30];
        V3<Real> gr[4];
        shape_gradients(dmi, gr);
        bool ok = finite9(T);
        Real g2 = Real(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ok = ok && finite3((-mul(S, gr[k])) + vk[k] * (-damp));
            g2 = fmax(g2, dot(gr[k], gr[k]));
        }
        // |K_ab entries| <= V (|lambda| + 2 |mu|) |g_a| |g_b|
        const Real bound = vol * (fabs(lam) + Real(2) * fabs(mu)) * g2;
        ok = ok && bound < Real(sizeof(Real) == 4 ? 1.0e37 : 1.0e306);
        if (ok) {
            out = T;
            form = Real(1);
        }
    }
    Real w[18];
    st9(w, 0, R);
    st9(w + 9, 0, out);
    st_rec_rs(rec, w);
    rec[31] = form;
}

// ------------------------------------------------------------------ row kernel, four lanes per row
// The implicit step with a slot table: four lanes share a row.  Per incidence (tet order)
// each lane loads two of the tet record's eight 16-byte chunks and the lanes exchange
// what they need with shuffles (one 128-byte line per row per incidence, instead of each
// lane reading the whole record); lane b then builds K_ab for the tet's corner b and adds
// it to that column's slot when the row stores it.  The four corners of one tet are four
// different columns, so every slot still receives its terms in tet order and the blocks
// equal the one-thread-per-row kernel's bit for bit.  Lane 0 adds the tet's right-hand-
// side term (T g_a - dt c v_a for a folded tet; for one the tet kernel left unfolded, the
// force -S g_a - c v_a, and the four lanes' K_ab v_b summed in lane order), the point
// connections, the host-emitted blocks and the diagonal's inverse.
template <class Real>
__device__ __forceinline__ Real shfl_row(Real v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}

template <class Real, int MAXU>
__global__ void __launch_bounds__(128) row_lanes_kernel(AssemblyArgs<Real> A)
{
    constexpr int LPR = 4, RPB = 128 / LPR, RS = RPB + 1;  // lanes per row, rows per block, slot stride
    // A row's tet record passes through its warp's staging row: 16 bytes of padding per row
    // put the 8 rows of a warp on different banks for the 16-byte accesses.
    constexpr int kStride = kTetRec + 16 / int(sizeof(Real));
    __shared__ Real acc[MAXU * 9 * RS];
    __shared__ __align__(16) Real stage[128 / 32][32 / LPR][kStride];
    const int tid = threadIdx.x, lane = tid & 31, lb = tid % LPR, rb = tid / LPR;
    const int base = lane - lb;  // lane 0 of this row within the warp
    const int r = blockIdx.x * RPB + rb;
    const bool valid = r < A.a.n;
#define PK_LACC(slot, e) acc[((slot) * 9 + (e)) * RS + rb]
    int node = 0, ks = 0, nu = 0, i0 = 0, i1 = 0;
    if (valid) {
        node = __ldg(A.dyn_to_node + r);
        ks = __ldg(A.a.row_start + r);
        nu = __ldg(A.a.row_start + r + 1) - ks;
        i0 = __ldg(A.inc_start + r);
        i1 = __ldg(A.inc_start + r + 1);
    }
    bool bad = false;
    if (valid && nu > MAXU) {
        if (lb == 0) atomicOr(A.flags, kFlagRowTooLong | kFlagPrecomputeFailed);
        nu = 0;
        i1 = i0;
    }
    for (int j = lb; j < nu; j += LPR)
        for (int e = 0; e < 9; ++e) PK_LACC(j, e) = Real(0);
    const V3<Real> vr = valid ? ld3(A.v, node) : V3<Real>{Real(0), Real(0), Real(0)};
    V3<Real> fsum{Real(0), Real(0), Real(0)}, kv{Real(0), Real(0), Real(0)}, bsum{Real(0), Real(0), Real(0)};
    // every lane of the warp takes part in every step (shuffles, warp barriers)
    int steps = i1 - i0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) steps = max(steps, __shfl_xor_sync(0xffffffffu, steps, off));
    __syncwarp();
    constexpr int kPer = kTetRec / LPR;  // record values each lane loads (two or four 16-byte chunks)
    for (int k = 0; k < steps; ++k) {
        // Every lane runs every step's shuffles and its warp barrier; the work is guarded.
        const bool live = i0 + k < i1;
        int code = 0;
        unsigned slots = 0xffffffffu;
        Real mine[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) mine[q] = Real(0);
        if (live) {
            code = __ldg(A.inc_list + i0 + k);
            slots = __ldg(A.inc_slot + i0 + k);
            const Real* rec = A.tets.rec + kTetRec * (size_t)(code >> 2) + (size_t)lb * kPer;
            if constexpr (sizeof(Real) == 4) {
                const float4 c0 = __ldg(reinterpret_cast<const float4*>(rec));
                const float4 c1 = __ldg(reinterpret_cast<const float4*>(rec) + 1);
                mine[0] = c0.x; mine[1] = c0.y; mine[2] = c0.z; mine[3] = c0.w;
                mine[4] = c1.x; mine[5] = c1.y; mine[6] = c1.z; mine[7] = c1.w;
            } else {
#pragma unroll
                for (int q = 0; q < kPer / 2; ++q) {
                    const double2 c = __ldg(reinterpret_cast<const double2*>(rec) + q);
                    mine[2 * q] = c.x;
                    mine[2 * q + 1] = c.y;
                }
            }
        }
        // record value v: element v % kPer of the row's lane v / kPer, through shared memory
        // (16-byte stores and loads instead of one shuffle per value)
        Real* row_stage = &stage[tid >> 5][lane / LPR][0];
        Real w[kTetRec];
        if constexpr (sizeof(Real) == 4) {
            float4* dst = reinterpret_cast<float4*>(row_stage + lb * kPer);
            dst[0] = make_float4(mine[0], mine[1], mine[2], mine[3]);
            dst[1] = make_float4(mine[4], mine[5], mine[6], mine[7]);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < kTetRec / 4; ++q) {
                const float4 c = reinterpret_cast<const float4*>(row_stage)[q];
                w[4 * q] = c.x;
                w[4 * q + 1] = c.y;
                w[4 * q + 2] = c.z;
                w[4 * q + 3] = c.w;
            }
        } else {
            double2* dst = reinterpret_cast<double2*>(row_stage + lb * kPer);
#pragma unroll
            for (int q = 0; q < kPer / 2; ++q) dst[q] = make_double2(mine[2 * q], mine[2 * q + 1]);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < kTetRec / 2; ++q) {
                const double2 c = reinterpret_cast<const double2*>(row_stage)[q];
                w[2 * q] = c.x;
                w[2 * q + 1] = c.y;
            }
        }
        const M3<Real> R = rd9(w);
        const bool work = live && !isnan(R.c[0].x);  // a skipped tet: no force, no stiffness
        if (work) {
            const bool folded = w[31] != Real(0);
            const M3<Real> SM = rd9(w + 9);  // S, or T in the folded form
            const M3<Real> dmi = rd9(w + 18);
            const Real vol = w[27], lam = w[28], mu = w[29], damp = w[30];
            const int a = code & 3;
            V3<Real> gr[4];
            gr[1] = v3<Real>(dmi.c[0].x, dmi.c[1].x, dmi.c[2].x);
            gr[2] = v3<Real>(dmi.c[0].y, dmi.c[1].y, dmi.c[2].y);
            gr[3] = v3<Real>(dmi.c[0].z, dmi.c[1].z, dmi.c[2].z);
            gr[0] = -((gr[1] + gr[2]) + gr[3]);
            V3<Real> ga = gr[0], gb = gr[0];  // selects: a dynamic index would put gr in local memory
#pragma unroll
            for (int q = 1; q < 4; ++q) {
                if (a == q) ga = gr[q];
                if (lb == q) gb = gr[q];
            }
            if (lb == 0) {
                if (folded) {
                    bsum = kadd3(bsum, kadd3(krot(SM, ga), kscale3(vr, -kmul(A.dt, damp))));
                } else {
                    const V3<Real> fa = kadd3(-krot(SM, ga), kscale3(vr, -damp));
                    if (finite3(fa)) fsum = kadd3(fsum, fa);
                }
            }
            const unsigned sl = (slots >> (8 * lb)) & 255u;
            if (sl == kSlotMissing) bad = true;  // pattern does not hold the block: host/device mismatch
            if (!folded || (int)sl < nu) {
                const M3<Real> K = kblock(krot(R, ga), krot(R, gb), ga, gb, krrt(R), vol, lam, mu);
                bad |= !finite9(K);
                if (!folded) {
                    const int4 tn = __ldg(A.tets.nodes + (code >> 2));
                    int nb = tn.x;
                    if (lb == 1) nb = tn.y;
                    if (lb == 2) nb = tn.z;
                    if (lb == 3) nb = tn.w;
                    const V3<Real> vb = ld3(A.v, nb);
                    bad |= !finite3(vb);
                    kv = kv + mul(K, vb);
                }
                if ((int)sl < nu) {
                    PK_LACC(sl, 0) += K.c[0].x; PK_LACC(sl, 1) += K.c[0].y; PK_LACC(sl, 2) += K.c[0].z;
                    PK_LACC(sl, 3) += K.c[1].x; PK_LACC(sl, 4) += K.c[1].y; PK_LACC(sl, 5) += K.c[1].z;
                    PK_LACC(sl, 6) += K.c[2].x; PK_LACC(sl, 7) += K.c[2].y; PK_LACC(sl, 8) += K.c[2].z;
                } else if (sl != kSlotNone && sl != kSlotMissing) {
                    bad = true;  // a slot beyond the row
                }
            }
        }
        __syncwarp();  // this tet's four blocks land before the next tet's (per-slot tet order)
    }
    __syncwarp();
    // the unfolded tets' K v: lane sums in lane order
    {
        V3<Real> k1{shfl_row(kv.x, base + 1), shfl_row(kv.y, base + 1), shfl_row(kv.z, base + 1)};
        V3<Real> k2{shfl_row(kv.x, base + 2), shfl_row(kv.y, base + 2), shfl_row(kv.z, base + 2)};
        V3<Real> k3{shfl_row(kv.x, base + 3), shfl_row(kv.y, base + 3), shfl_row(kv.z, base + 3)};
        kv = ((kv + k1) + k2) + k3;
    }
    if (valid && lb == 0) {
        // Transient point connections and host-emitted contributions, as the one-thread
        // kernel (slot found by search).
        auto find_slot = [&](int c) {
            int slot = 0;
            while (slot < nu && __ldg(A.a.col + ks + slot) != c) ++slot;
            return slot;
        };
        if (A.conn_inc_start) {
            const int j0 = __ldg(A.conn_inc_start + r), j1 = __ldg(A.conn_inc_start + r + 1);
            for (int i = j0; i < j1; ++i) {
                const int cc = __ldg(A.conn_inc_list + i);
                const int ci = cc >> 2, ca = cc & 3;
                if ((unsigned)ci >= (unsigned)A.conn_count) {
                    bad = true;
                    continue;
                }
                const Real* ev = A.conn_eval + 4 * (size_t)ci;
                if (!(ev[3] != Real(0))) continue;
                const int4 cn = __ldg(A.conn_nodes + ci);
                const int nb[4] = {cn.x, cn.y, cn.z, cn.w};
                const Real* q = A.conn_params + kConnParams * (size_t)ci;
                const Real wq[4] = {__ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3)};
                Real wa = wq[0];
#pragma unroll
                for (int b = 1; b < 4; ++b)
                    if (ca == b) wa = wq[b];
                fsum = fsum + V3<Real>{ev[0], ev[1], ev[2]} * wa;
                const Real kk = __ldg(q + 7);
                if (!(kk > Real(0))) continue;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    if (wq[b] == Real(0)) continue;
                    const Real kab = kk * wa * wq[b];
                    bad |= !isfinite(kab);
                    kv = kv + ld3(A.v, nb[b]) * kab;
                    const int c = __ldg(A.node_to_dyn + nb[b]);
                    if (c >= r) {
                        const int slot = find_slot(c);
                        if (slot < nu) {
                            PK_LACC(slot, 0) += kab;
                            PK_LACC(slot, 4) += kab;
                            PK_LACC(slot, 8) += kab;
                        } else {
                            bad = true;
                        }
                    }
                }
            }
        }
        if (A.ext_rhs_start) {
            const int b0 = __ldg(A.ext_rhs_start + r), b1 = __ldg(A.ext_rhs_start + r + 1);
            for (int i = b0; i < b1; ++i) {
                const int kq = __ldg(A.ext_rhs_list + i);
                const M3<Real> B = ld9(A.ext_blocks, (size_t)kq);
                const int2 nd = __ldg(A.ext_nodes + kq);
                const V3<Real> vb = ld3(A.v, nd.y);
                bad |= !finite3(vb) || !finite9(B);
                kv = kv + mul(B, vb);
            }
            const int m0 = __ldg(A.ext_mat_start + r), m1 = __ldg(A.ext_mat_start + r + 1);
            for (int i = m0; i < m1; ++i) {
                const unsigned cq = (unsigned)__ldg(A.ext_mat_list + i);
                const int kq = (int)(cq & 0x7fffffffu);
                const bool tr = (cq & 0x80000000u) != 0;
                M3<Real> B = ld9(A.ext_blocks, (size_t)kq);
                if (tr) B = transpose(B);
                const int2 nd = __ldg(A.ext_nodes + kq);
                const int c = __ldg(A.node_to_dyn + (tr ? nd.x : nd.y));
                const int slot = find_slot(c);
                if (c < r || slot >= nu) {
                    bad = true;
                    continue;
                }
                PK_LACC(slot, 0) += B.c[0].x; PK_LACC(slot, 1) += B.c[0].y; PK_LACC(slot, 2) += B.c[0].z;
                PK_LACC(slot, 3) += B.c[1].x; PK_LACC(slot, 4) += B.c[1].y; PK_LACC(slot, 5) += B.c[1].z;
                PK_LACC(slot, 6) += B.c[2].x; PK_LACC(slot, 7) += B.c[2].y; PK_LACC(slot, 8) += B.c[2].z;
            }
        }
        if (A.ext_force) fsum = kadd3(fsum, ld3(A.ext_force, r));
    }
    __syncwarp();
    const Real m = valid ? __ldg(A.mass + node) : Real(0);
    const Real dt = A.dt, dt2 = kmul(dt, dt);
    // the row's blocks: lane j writes slots j, j + 4, ...; the diagonal (slot 0) is lane 0's
    M3<Real> diag = mident<Real>();
    for (int j = lb; j < nu; j += LPR) {
        M3<Real> blk;
        blk.c[0] = v3<Real>(PK_LACC(j, 0), PK_LACC(j, 1), PK_LACC(j, 2));
        blk.c[1] = v3<Real>(PK_LACC(j, 3), PK_LACC(j, 4), PK_LACC(j, 5));
        blk.c[2] = v3<Real>(PK_LACC(j, 6), PK_LACC(j, 7), PK_LACC(j, 8));
        bad |= !finite9(blk);
        blk.c[0] = kscale3(blk.c[0], dt2);
        blk.c[1] = kscale3(blk.c[1], dt2);
        blk.c[2] = kscale3(blk.c[2], dt2);
        if (j == 0) {
            blk.c[0].x = kadd(m, blk.c[0].x);
            blk.c[1].y = kadd(m, blk.c[1].y);
            blk.c[2].z = kadd(m, blk.c[2].z);
            diag = blk;
        }
        st9(A.values, (size_t)(ks + j), blk);
    }
#undef PK_LACC
    // the row's four lanes' findings, for lane 0 (the step's flag is global)
    bad = ((__ballot_sync(0xffffffffu, bad) >> base) & 0xFu) != 0u;
    if (!valid || lb != 0) return;
    const V3<Real> grav{A.gravity[0], A.gravity[1], A.gravity[2]};
    fsum = kadd3(fsum, kscale3(grav, m));
    const V3<Real> b = kadd3(bsum, kadd3(kscale3(kv, -dt2), kscale3(fsum, dt)));
    bad |= !finite3(kv) || !finite3(b);
    st3(A.rhs, r, b);
    if (bad) atomicOr(A.flags, kFlagPrecomputeFailed);
    M3<Real> mi = mident<Real>();
    if (A.use_jacobi) {
        const Real d = det(diag);
        if (!finite9(diag) || !isfinite(d) || fabs(d) <= Real(1.0e-8)) {
            atomicOr(A.flags, kFlagSingularDiag);
        } else {
            mi = inverse(diag);
            if (!finite9(mi)) atomicOr(A.flags, kFlagSingularDiag);
        }
    }
    st9(A.minv, (size_t)r, mi);
}

// ------------------------------------------------------------------ sphere contacts
// CollisionSphereComponent::UpdateSystem (CollisionSphereComponent.cpp:112-190): a tet
// whose centroid p = ((x0 w + x1 w) + x2 w) + x3 w (w = 1/4) lies strictly inside the
// sphere, |p - c| < radius, becomes a contact.  The arithmetic rounds each operation once,
// as the reference's Vec3 code does (no contraction into fused multiply-adds).  Only tets
// marked active (flag bit 2) count.  Contacts are appended in any order; the host sorts
// them by tet.
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }

template <class Real>
__global__ void sphere_contact_kernel(const int4* __restrict__ nodes, const unsigned char* __restrict__ flags,
                                      const Real* __restrict__ x, int tet_count, Real cx, Real cy, Real cz,
                                      Real radius, int max_out, int* count, int* out_tet, Real* out_point)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tet_count || !(__ldg(flags + t) & 4u)) return;
    const int4 n = __ldg(nodes + t);
    const int nd[4] = {n.x, n.y, n.z, n.w};
    const Real w = Real(0.25);
    Real p[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Real acc = rn_mul(__ldg(x + 3 * (size_t)nd[0] + a), w);
#pragma unroll
        for (int k = 1; k < 4; ++k) acc = rn_add(acc, rn_mul(__ldg(x + 3 * (size_t)nd[k] + a), w));
        p[a] = acc;
    }
    const Real dx = rn_add(p[0], -cx), dy = rn_add(p[1], -cy), dz = rn_add(p[2], -cz);
    const Real d2 = rn_add(rn_add(rn_mul(dx, dx), rn_mul(dy, dy)), rn_mul(dz, dz));
    if (!(sqrt(d2) < radius)) return;
    const int slot = atomicAdd(count, 1);
    if (slot >= max_out) return;
    out_tet[slot] = t;
    out_point[3 * (size_t)slot] = p[0];
    out_point[3 * (size_t)slot + 1] = p[1];
    out_point[3 * (size_t)slot + 2] = p[2];
}

// ------------------------------------------------------------------ post-step geometry
// Surface triangles (SurfaceVisualComponent::UpdateVisualSurfaceGeometry,
// SurfaceVisualComponent.cpp:150-213): each triangle's three node positions become its three
// visual vertices and its flat normal Cross(p1 - p0, p2 - p0) / length (0, 1, 0 when the
// length is at most 1e-6) their normals.  Embedded vertices (VisualMeshComponent::
// UpdateDeformedVertices, VisualMeshComponent.cpp:257-333): ((x0 w0 + x1 w1) + x2 w2) + x3 w3
// for the vertices marked live, the others keep their last value.  The positions these read
// are the float copies the components hold (a double state is rounded to float first), and
// every operation is a float operation rounded once, as the reference's Vec3 code does.
template <class Real>
__global__ void surface_triangle_kernel(const int* __restrict__ nodes, int count, const Real* __restrict__ x,
                                        float* __restrict__ verts, float* __restrict__ normals)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    float p[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int n = __ldg(nodes + 3 * t + k);
#pragma unroll
        for (int a = 0; a < 3; ++a) p[k][a] = static_cast<float>(__ldg(x + 3 * (size_t)n + a));
    }
    float e1[3], e2[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e1[a] = __fsub_rn(p[1][a], p[0][a]);
        e2[a] = __fsub_rn(p[2][a], p[0][a]);
    }
    const float cx = __fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1]));
    const float cy = __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2]));
    const float cz = __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]));
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz)));
    float nrm[3] = {0.0f, 1.0f, 0.0f};
    if (len > 0.000001f) {
        nrm[0] = __fdiv_rn(cx, len);
        nrm[1] = __fdiv_rn(cy, len);
        nrm[2] = __fdiv_rn(cz, len);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            verts[9 * (size_t)t + 3 * k + a] = p[k][a];
            normals[9 * (size_t)t + 3 * k + a] = nrm[a];
        }
}

template <class Real>
__global__ void embedded_vertex_kernel(const int* __restrict__ nodes, const float* __restrict__ weights,
                                       const unsigned char* __restrict__ live, int count, const Real* __restrict__ x,
                                       float* __restrict__ verts)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= count || !__ldg(live + v)) return;
    int n[4];
    float w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        n[k] = __ldg(nodes + 4 * v + k);
        w[k] = __ldg(weights + 4 * v + k);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float acc = __fmul_rn(static_cast<float>(__ldg(x + 3 * (size_t)n[0] + a)), w[0]);
#pragma unroll
        for (int k = 1; k < 4; ++k)
            acc = __fadd_rn(acc, __fmul_rn(static_cast<float>(__ldg(x + 3 * (size_t)n[k] + a)), w[k]));
        verts[3 * (size_t)v + a] = acc;
    }
}

// Per incidence of row r (tet t, corner a): the row slot of each of the tet's nodes --
// the index of its column among the row's upper blocks, kSlotNone for a column below the
// row or a node without a row, kSlotMissing when the pattern lacks the block.
__global__ void inc_slot_kernel(int n, const int* __restrict__ row_start, const int* __restrict__ col,
                                const int* __restrict__ inc_start, const int* __restrict__ inc_list,
                                const int4* __restrict__ tet_nodes, const int* __restrict__ node_to_dyn,
                                unsigned* __restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int ks = __ldg(row_start + r), ke = __ldg(row_start + r + 1);
    for (int i = __ldg(inc_start + r); i < __ldg(inc_start + r + 1); ++i) {
        const int4 tn = __ldg(tet_nodes + (__ldg(inc_list + i) >> 2));
        const int nb[4] = {tn.x, tn.y, tn.z, tn.w};
        unsigned code = 0u;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int c = __ldg(node_to_dyn + nb[b]);
            unsigned sl = kSlotNone;
            if (c >= r) {
                sl = kSlotMissing;
                for (int k = ks; k < ke; ++k)
                    if (__ldg(col + k) == c) {
                        sl = (unsigned)(k - ks);
                        break;
                    }
            }
            code |= sl << (8 * b);
        }
        out[i] = code;
    }
}

template <class Real>
__global__ void tet_pack_kernel(const Real* __restrict__ dm_inv, const Real* __restrict__ params, Real* rec,
                                int tet_count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tet_count) return;
    Real* q = rec + kTetRec * (size_t)t;
    for (int e = 0; e < 9; ++e) q[18 + e] = dm_inv[9 * (size_t)t + e];
    for (int e = 0; e < 4; ++e) q[27 + e] = params[4 * (size_t)t + e];
    q[31] = Real(0);
}

// ------------------------------------------------------------------ row kernel
// MAXU > 0: accumulate the row's upper blocks in shared memory (MAXU slots per thread);
// MAXU == 0: accumulate in place in the values array (rows of any length).
template <class Real, int MAXU>
__global__ void __launch_bounds__(128) row_kernel(AssemblyArgs<Real> A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* acc = reinterpret_cast<Real*>(smem_raw);
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.a.n) return;
    const int T = blockDim.x, tid = threadIdx.x;
    const int node = __ldg(A.dyn_to_node + r);
    const int ks = __ldg(A.a.row_start + r), ke = __ldg(A.a.row_start + r + 1);
    const int nu = ke - ks;
    if (!A.explicit_mode && MAXU > 0 && nu > MAXU) {
        atomicOr(A.flags, kFlagRowTooLong | kFlagPrecomputeFailed);
        return;
    }
    Real* gacc = A.values + 9 * (size_t)ks;
#define PK_ACC(slot, e) (MAXU > 0 ? acc[((slot) * 9 + (e)) * T + tid] : gacc[(slot) * 9 + (e)])
    if (!A.explicit_mode)
        for (int j = 0; j < nu; ++j)
            for (int e = 0; e < 9; ++e) PK_ACC(j, e) = Real(0);

    // The row's columns in registers (MAXU > 0): the slot search below compares registers.
    int colr[MAXU > 0 ? MAXU : 1];
#pragma unroll
    for (int j = 0; j < (MAXU > 0 ? MAXU : 1); ++j) colr[j] = (MAXU > 0 && j < nu) ? __ldg(A.a.col + ks + j) : -1;
    const V3<Real> vr = ld3(A.v, node);
    V3<Real> fsum{Real(0), Real(0), Real(0)};
    V3<Real> kv{Real(0), Real(0), Real(0)};
    bool bad = false;
    // Right-hand-side terms of the tets in the folded form: sum of T g_a - dt c v_a.
    V3<Real> bsum{Real(0), Real(0), Real(0)};
    const int i0 = __ldg(A.inc_start + r), i1 = __ldg(A.inc_start + r + 1);
    // The next incidence's code and slots are loaded while this one is processed.
    int code_n = 0;
    unsigned slot_n = 0u;
    auto fetch = [&](int i) {
        code_n = __ldg(A.inc_list + i);
        if (A.inc_slot) slot_n = __ldg(A.inc_slot + i);
    };
    if (i0 < i1) fetch(i0);
    for (int i = i0; i < i1; ++i) {
        const int code = code_n;
        const unsigned slots = slot_n;
        const int t = code >> 2, a = code & 3;
        if (i + 1 < i1) fetch(i + 1);
        // The tet's record (the tet kernel's, an earlier launch); R is NaN-marked for a
        // skipped tet.
        Real w[kTetRec];
        ld_rec(A.tets.rec + kTetRec * (size_t)t, w);
        const M3<Real> R = rd9(w);
        if (isnan(R.c[0].x)) continue;  // skipped tet: no force, no stiffness
        const M3<Real> SM = rd9(w + 9);  // S, or T in the folded form
        const bool folded = w[31] != Real(0);
        const M3<Real> dmi = rd9(w + 18);
        const Real vol = w[27], lam = w[28], mu = w[29], damp = w[30];
        // Shape gradients: g1..g3 are the rows of DmInv, g0 = -(g1+g2+g3).
        V3<Real> gr[4];
        gr[1] = v3<Real>(dmi.c[0].x, dmi.c[1].x, dmi.c[2].x);
        gr[2] = v3<Real>(dmi.c[0].y, dmi.c[1].y, dmi.c[2].y);
        gr[3] = v3<Real>(dmi.c[0].z, dmi.c[1].z, dmi.c[2].z);
        gr[0] = -((gr[1] + gr[2]) + gr[3]);
        V3<Real> ga = gr[0];  // selects: a dynamic index would put gr in local memory
#pragma unroll
        for (int k = 1; k < 4; ++k)
            if (a == k) ga = gr[k];
        if (folded) {
            // T g_a - dt c v_a; the upper blocks from the slot table.
            bsum = kadd3(bsum, kadd3(krot(SM, ga), kscale3(vr, -kmul(A.dt, damp))));
        } else {
            // Force on node a from this tet: elastic -S g_a plus damping -c v_a.
            const V3<Real> fa = kadd3(-krot(SM, ga), kscale3(vr, -damp));
            if (finite3(fa)) fsum = kadd3(fsum, fa);
            if (A.explicit_mode) continue;
        }
        const int4 tn = folded ? make_int4(0, 0, 0, 0) : __ldg(A.tets.nodes + t);
        const int nb[4] = {tn.x, tn.y, tn.z, tn.w};
        // K_ab = R Ke_ab R^T with Ke_ab = V (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I)
        //      = V (lambda P_a P_b^T + mu P_b P_a^T + mu (g_a.g_b) R R^T),  P = R g (kblock).
        const V3<Real> pa = krot(R, ga);
        const M3<Real> rrt = krrt(R);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int slot = nu;
            if (folded) {
                // only the blocks this row stores
                const unsigned sl = (slots >> (8 * b)) & 255u;
                if (sl == kSlotNone) continue;
                if (sl == kSlotMissing) {
                    bad = true;  // pattern does not hold the block: host/device mismatch
                    continue;
                }
                slot = (int)sl;
            }
            const V3<Real> gb = gr[b];
            const M3<Real> K = kblock(pa, krot(R, gb), ga, gb, rrt, vol, lam, mu);
            bad |= !finite9(K);
            if (!folded) {
                const V3<Real> vb = ld3(A.v, nb[b]);
                bad |= !finite3(vb);
                kv = kv + mul(K, vb);
                const int c = __ldg(A.node_to_dyn + nb[b]);
                if (c < r) continue;
                if (MAXU > 0) {
#pragma unroll
                    for (int j = (MAXU > 0 ? MAXU : 1) - 1; j >= 0; --j)
                        if (colr[j] == c) slot = j;
                } else {
                    slot = 0;
                    while (slot < nu && __ldg(A.a.col + ks + slot) != c) ++slot;
                }
                if (slot >= nu) {
                    bad = true;  // pattern does not hold the block: host/device mismatch
                    continue;
                }
            }
            PK_ACC(slot, 0) += K.c[0].x; PK_ACC(slot, 1) += K.c[0].y; PK_ACC(slot, 2) += K.c[0].z;
            PK_ACC(slot, 3) += K.c[1].x; PK_ACC(slot, 4) += K.c[1].y; PK_ACC(slot, 5) += K.c[1].z;
            PK_ACC(slot, 6) += K.c[2].x; PK_ACC(slot, 7) += K.c[2].y; PK_ACC(slot, 8) += K.c[2].z;
        }
    }
    // Transient point connections with a corner at this row (PointConnection::UpdateSystem,
    // PointConnection.cpp:55-140): the connection's force times this corner's weight, and
    // for stiffness > 0 the blocks k w_a w_b I to every corner b with a non-zero weight --
    // K v_b into the rhs for every b, and into the matrix where the column is a dynamic row
    // c >= r (the reference emits both orientations and keeps the upper one).
    if (A.conn_inc_start) {
        const int j0 = __ldg(A.conn_inc_start + r), j1 = __ldg(A.conn_inc_start + r + 1);
        for (int i = j0; i < j1; ++i) {
            const int code = __ldg(A.conn_inc_list + i);
            const int ci = code >> 2, a = code & 3;
            if ((unsigned)ci >= (unsigned)A.conn_count) {
                bad = true;
                continue;
            }
            const Real* ev = A.conn_eval + 4 * (size_t)ci;
            if (!(ev[3] != Real(0))) continue;  // point, velocity or target not finite: nothing
            const int4 cn = __ldg(A.conn_nodes + ci);
            const int nb[4] = {cn.x, cn.y, cn.z, cn.w};
            const Real* q = A.conn_params + kConnParams * (size_t)ci;
            const Real w[4] = {__ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3)};
            Real wa = w[0];
#pragma unroll
            for (int b = 1; b < 4; ++b)
                if (a == b) wa = w[b];
            fsum = fsum + V3<Real>{ev[0], ev[1], ev[2]} * wa;
            const Real k = __ldg(q + 7);
            if (A.explicit_mode || !(k > Real(0))) continue;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (w[b] == Real(0)) continue;
                const Real kab = k * wa * w[b];
                bad |= !isfinite(kab);
                const V3<Real> vb = ld3(A.v, nb[b]);
                kv = kv + vb * kab;
                const int c = __ldg(A.node_to_dyn + nb[b]);
                if (c >= r) {
                    int slot = nu;
                    if (MAXU > 0) {
#pragma unroll
                        for (int j = (MAXU > 0 ? MAXU : 1) - 1; j >= 0; --j)
                            if (colr[j] == c) slot = j;
                    } else {
                        slot = 0;
                        while (slot < nu && __ldg(A.a.col + ks + slot) != c) ++slot;
                    }
                    if (slot < nu) {
                        PK_ACC(slot, 0) += kab;
                        PK_ACC(slot, 4) += kab;
                        PK_ACC(slot, 8) += kab;
                    } else {
                        bad = true;  // pattern does not hold the block: host/device mismatch
                    }
                }
            }
        }
    }
    // Host-emitted contributions of custom components (SolverData::AddStiffnessBlock and
    // AddNodeForce, SolverData.cpp:322-365, 407-462): -dt^2 B v_b into the rhs for every
    // block whose row node is this row (column nodes of any kind), the blocks this row
    // holds in its upper row (B, or B^T for a lower block whose upper twin was not
    // emitted), and the summed forces.
    if (A.ext_rhs_start) {
        const int b0 = __ldg(A.ext_rhs_start + r), b1 = __ldg(A.ext_rhs_start + r + 1);
        for (int i = b0; i < b1 && !A.explicit_mode; ++i) {
            const int k = __ldg(A.ext_rhs_list + i);
            const M3<Real> B = ld9(A.ext_blocks, (size_t)k);
            const int2 nd = __ldg(A.ext_nodes + k);
            const V3<Real> vb = ld3(A.v, nd.y);
            bad |= !finite3(vb) || !finite9(B);
            kv = kv + mul(B, vb);
        }
        const int m0 = __ldg(A.ext_mat_start + r), m1 = __ldg(A.ext_mat_start + r + 1);
        for (int i = m0; i < m1 && !A.explicit_mode; ++i) {
            const unsigned code = (unsigned)__ldg(A.ext_mat_list + i);
            const int k = (int)(code & 0x7fffffffu);
            const bool tr = (code & 0x80000000u) != 0;
            M3<Real> B = ld9(A.ext_blocks, (size_t)k);
            if (tr) B = transpose(B);
            const int2 nd = __ldg(A.ext_nodes + k);
            const int c = __ldg(A.node_to_dyn + (tr ? nd.x : nd.y));
            int slot = nu;
            if (MAXU > 0) {
#pragma unroll
                for (int j = (MAXU > 0 ? MAXU : 1) - 1; j >= 0; --j)
                    if (colr[j] == c) slot = j;
            } else {
                slot = 0;
                while (slot < nu && __ldg(A.a.col + ks + slot) != c) ++slot;
            }
            if (c < r || slot >= nu) {
                bad = true;  // pattern does not hold the block: host/device mismatch
                continue;
            }
            PK_ACC(slot, 0) += B.c[0].x; PK_ACC(slot, 1) += B.c[0].y; PK_ACC(slot, 2) += B.c[0].z;
            PK_ACC(slot, 3) += B.c[1].x; PK_ACC(slot, 4) += B.c[1].y; PK_ACC(slot, 5) += B.c[1].z;
            PK_ACC(slot, 6) += B.c[2].x; PK_ACC(slot, 7) += B.c[2].y; PK_ACC(slot, 8) += B.c[2].z;
        }
    }
    if (A.ext_force) fsum = kadd3(fsum, ld3(A.ext_force, r));
    const Real m = __ldg(A.mass + node);
    const V3<Real> grav{A.gravity[0], A.gravity[1], A.gravity[2]};
    fsum = kadd3(fsum, kscale3(grav, m));
    const Real dt = A.dt;

    if (A.explicit_mode) {
        // World::IntegrateExplicitEuler (World.cpp:697-725): a = f/m, v += a dt, x += v dt.
        const V3<Real> acc3{fsum.x / m, fsum.y / m, fsum.z / m};
        const V3<Real> nv = vr + acc3 * dt;
        const V3<Real> nx = ld3(A.x, node) + nv * dt;
        st3(A.v, node, nv);
        st3(A.x_out, node, nx);
        return;
    }

    const Real dt2 = kmul(dt, dt);
    M3<Real> diag;
    for (int j = 0; j < nu; ++j) {
        M3<Real> blk;
        blk.c[0] = v3<Real>(PK_ACC(j, 0), PK_ACC(j, 1), PK_ACC(j, 2));
        blk.c[1] = v3<Real>(PK_ACC(j, 3), PK_ACC(j, 4), PK_ACC(j, 5));
        blk.c[2] = v3<Real>(PK_ACC(j, 6), PK_ACC(j, 7), PK_ACC(j, 8));
        bad |= !finite9(blk);
        blk.c[0] = kscale3(blk.c[0], dt2);
        blk.c[1] = kscale3(blk.c[1], dt2);
        blk.c[2] = kscale3(blk.c[2], dt2);
        if (j == 0) {
            blk.c[0].x = kadd(m, blk.c[0].x);
            blk.c[1].y = kadd(m, blk.c[1].y);
            blk.c[2].z = kadd(m, blk.c[2].z);
            diag = blk;
        }
        st9(A.values, (size_t)(ks + j), blk);
    }
#undef PK_ACC
    const V3<Real> b = kadd3(bsum, kadd3(kscale3(kv, -dt2), kscale3(fsum, dt)));
    bad |= !finite3(kv) || !finite3(b);
    st3(A.rhs, r, b);
    if (bad) atomicOr(A.flags, kFlagPrecomputeFailed);

    // Block-Jacobi inverse of the diagonal block.
    M3<Real> mi = mident<Real>();
    if (A.use_jacobi) {
        const Real d = det(diag);
        if (!finite9(diag) || !isfinite(d) || fabs(d) <= Real(1.0e-8)) {
            atomicOr(A.flags, kFlagSingularDiag);
        } else {
            mi = inverse(diag);
            if (!finite9(mi)) atomicOr(A.flags, kFlagSingularDiag);
        }
    }
    st9(A.minv, (size_t)r, mi);
}

// ------------------------------------------------------------------ point connections
// One thread per connection (PointConnection::UpdateSystem, PointConnection.cpp:55-108):
// the weighted point and velocity of its four nodes, left to right; if they and the
// target are finite, the force k (target - point) - c velocity, else the connection
// contributes nothing this step.  Evaluated before the row kernel, which in explicit mode
// overwrites the nodes' state.
template <class Real>
__global__ void conn_kernel(AssemblyArgs<Real> A)
{
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= A.conn_count) return;
    const int4 cn = __ldg(A.conn_nodes + ci);
    const int nb[4] = {cn.x, cn.y, cn.z, cn.w};
    const Real* q = A.conn_params + kConnParams * (size_t)ci;
    V3<Real> p = ld3(A.x, nb[0]) * __ldg(q);
    V3<Real> u = ld3(A.v, nb[0]) * __ldg(q);
#pragma unroll
    for (int b = 1; b < 4; ++b) {
        p = p + ld3(A.x, nb[b]) * __ldg(q + b);
        u = u + ld3(A.v, nb[b]) * __ldg(q + b);
    }
    const V3<Real> target{__ldg(q + 4), __ldg(q + 5), __ldg(q + 6)};
    Real* ev = A.conn_eval + 4 * (size_t)ci;
    if (!finite3(p) || !finite3(u) || !finite3(target)) {
        ev[0] = ev[1] = ev[2] = Real(0);
        ev[3] = Real(0);
        return;
    }
    const Real k = __ldg(q + 7), damp = __ldg(q + 8);
    const V3<Real> f = (target - p) * k + u * (-damp);
    ev[0] = f.x;
    ev[1] = f.y;
    ev[2] = f.z;
    ev[3] = Real(1);
}

// ------------------------------------------------------------------ SpMV kernel
template <class Real>
__global__ void __launch_bounds__(256) spmv_kernel(BsrView<Real> A, const Real* x, Real* y)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int r = 2 * warp + (lane >> 4);
    const bool valid = r < A.n;
    const V3<Real> q = row_spmv<Real, 16>(A, valid ? r : -1, lane & 15, x, nullptr, Real(0), false);
    if (valid && (lane & 15) == 0) st3(y, r, q);
}

}  // namespace

// ------------------------------------------------------------------ launchers
template <class Real>
cudaError_t launch_tet_kernel(const AssemblyArgs<Real>& args, bool fp64_polar_fallback, cudaStream_t stream)
{
    const int t = args.tets.tet_count;
    if (t <= 0) return cudaSuccess;
    const int threads = 256, blocks = (t + threads - 1) / threads;
    if (fp64_polar_fallback)
        tet_kernel<Real, true><<<blocks, threads, 0, stream>>>(args);
    else
        tet_kernel<Real, false><<<blocks, threads, 0, stream>>>(args);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_tet_pack(const Real* dm_inv, const Real* params, Real* rec, int tet_count, cudaStream_t stream)
{
    if (tet_count <= 0) return cudaSuccess;
    tet_pack_kernel<Real><<<(tet_count + 255) / 256, 256, 0, stream>>>(dm_inv, params, rec, tet_count);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_sphere_contacts(const int* nodes, const unsigned char* flags, const Real* x, int tet_count,
                                   const Real* center, Real radius, int max_out, int* count, int* out_tet,
                                   Real* out_point, cudaStream_t stream)
{
    if (tet_count <= 0) return cudaSuccess;
    sphere_contact_kernel<Real><<<(tet_count + 255) / 256, 256, 0, stream>>>(
        reinterpret_cast<const int4*>(nodes), flags, x, tet_count, center[0], center[1], center[2], radius, max_out,
        count, out_tet, out_point);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_visual_kernel(int kind, const int* nodes, const float* weights, const unsigned char* live, int count,
                                 const Real* x, float* verts, float* normals, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    if (kind == 0)
        surface_triangle_kernel<Real><<<(count + 127) / 128, 128, 0, stream>>>(nodes, count, x, verts, normals);
    else
        embedded_vertex_kernel<Real><<<(count + 127) / 128, 128, 0, stream>>>(nodes, weights, live, count, x, verts);
    return cudaGetLastError();
}

cudaError_t launch_inc_slot_kernel(int n, const int* row_start, const int* col, const int* inc_start,
                                   const int* inc_list, const int4* tet_nodes, const int* node_to_dyn, unsigned* out,
                                   cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    inc_slot_kernel<<<(n + 127) / 128, 128, 0, stream>>>(n, row_start, col, inc_start, inc_list, tet_nodes,
                                                          node_to_dyn, out);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_conn_kernel(const AssemblyArgs<Real>& args, cudaStream_t stream)
{
    if (args.conn_count <= 0) return cudaSuccess;
    conn_kernel<Real><<<(args.conn_count + 127) / 128, 128, 0, stream>>>(args);
    return cudaGetLastError();
}

template <class Real, int MAXU>
static cudaError_t launch_rows(const AssemblyArgs<Real>& args, cudaStream_t stream)
{
    const int n = args.a.n;
    int threads = 128;
    size_t smem = 0;
    if (MAXU > 0) {
        while (threads > 32 && (size_t)MAXU * 9 * sizeof(Real) * threads > 48 * 1024) threads >>= 1;
        smem = (size_t)MAXU * 9 * sizeof(Real) * threads;
    }
    const int blocks = (n + threads - 1) / threads;
    row_kernel<Real, MAXU><<<blocks, threads, smem, stream>>>(args);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_row_kernel(const AssemblyArgs<Real>& args, int max_row_blocks, cudaStream_t stream)
{
    if (args.a.n <= 0) return cudaSuccess;
    if (args.inc_slot && args.row_lanes && !args.explicit_mode && max_row_blocks <= kSlotMaxRow) {
        const int blocks = (args.a.n + 31) / 32;
        if (max_row_blocks <= 8)
            row_lanes_kernel<Real, 8><<<blocks, 128, 0, stream>>>(args);
        else
            row_lanes_kernel<Real, 16><<<blocks, 128, 0, stream>>>(args);
        return cudaGetLastError();
    }
    if (args.explicit_mode || max_row_blocks <= 8) return launch_rows<Real, 8>(args, stream);
    if (max_row_blocks <= 16) return launch_rows<Real, 16>(args, stream);
    return launch_rows<Real, 0>(args, stream);
}

template <class Real>
cudaError_t launch_spmv_kernel(const BsrView<Real>& a, const Real* x, Real* y, cudaStream_t stream)
{
    if (a.n <= 0) return cudaSuccess;
    const int threads = 256;
    const int rows_per_block = threads / 16;
    const int blocks = (a.n + rows_per_block - 1) / rows_per_block;
    spmv_kernel<Real><<<blocks, threads, 0, stream>>>(a, x, y);
    return cudaGetLastError();
}

template cudaError_t launch_tet_kernel<float>(const AssemblyArgs<float>&, bool, cudaStream_t);
template cudaError_t launch_tet_kernel<double>(const AssemblyArgs<double>&, bool, cudaStream_t);
template cudaError_t launch_tet_pack<float>(const float*, const float*, float*, int, cudaStream_t);
template cudaError_t launch_conn_kernel<float>(const AssemblyArgs<float>&, cudaStream_t);
template cudaError_t launch_conn_kernel<double>(const AssemblyArgs<double>&, cudaStream_t);
template cudaError_t launch_tet_pack<double>(const double*, const double*, double*, int, cudaStream_t);
template cudaError_t launch_visual_kernel<float>(int, const int*, const float*, const unsigned char*, int,
                                                 const float*, float*, float*, cudaStream_t);
template cudaError_t launch_visual_kernel<double>(int, const int*, const float*, const unsigned char*, int,
                                                  const double*, float*, float*, cudaStream_t);
template cudaError_t launch_sphere_contacts<float>(const int*, const unsigned char*, const float*, int, const float*,
                                                   float, int, int*, int*, float*, cudaStream_t);
template cudaError_t launch_sphere_contacts<double>(const int*, const unsigned char*, const double*, int,
                                                    const double*, double, int, int*, int*, double*, cudaStream_t);
template cudaError_t launch_row_kernel<float>(const AssemblyArgs<float>&, int, cudaStream_t);
template cudaError_t launch_row_kernel<double>(const AssemblyArgs<double>&, int, cudaStream_t);
template cudaError_t launch_spmv_kernel<float>(const BsrView<float>&, const float*, float*, cudaStream_t);
template cudaError_t launch_spmv_kernel<double>(const BsrView<double>&, const double*, double*, cudaStream_t);

}  // namespace pk
