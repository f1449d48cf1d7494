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
//   pcg_kernel   one cooperative launch per solve: block-Jacobi PCG with the symmetric
//                upper-BSR SpMV fused with d = s + beta d and the d.q partial sums, the
//                x/r/s update fused with r.s, grid-wide reductions in fixed order (the
//                result does not depend on timing), bounded grid barriers, and the
//                all-or-nothing implicit Euler update fused at the end.
//                (SolvePreconditionedConjugateGradient, ConjugateGradientSolver.cpp:114-241;
//                 SparseBlockMatrix::Multiply, SparseBlockMatrix.cpp:209-268;
//                 World::IntegrateImplicitEuler, World.cpp:644-695)
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

// ------------------------------------------------------------------ tet kernel
template <class Real, bool kFp64Polar>
__global__ void __launch_bounds__(256) tet_kernel(AssemblyArgs<Real> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.tets.tet_count) return;
    Real* rot = A.tets.rot + 9 * (size_t)t;
    const Real* prm = A.tets.params + 4 * (size_t)t;
    const Real vol = __ldg(prm + 0);
    const unsigned char en = __ldg(A.tets.enabled + t);
    if (!(en & 1u) || !(vol > Real(0))) {
        rot[0] = qnan<Real>();
        return;
    }
    const bool linear = A.linear || (en & 2u);
    const int4 n = __ldg(A.tets.nodes + t);
    const V3<Real> x0 = ld3(A.x, n.x), x1 = ld3(A.x, n.y), x2 = ld3(A.x, n.z), x3 = ld3(A.x, n.w);
    const M3<Real> ds = mcols(x1 - x0, x2 - x0, x3 - x0);
    const M3<Real> f = mul(ds, ld9(A.tets.dm_inv, (size_t)t));
    if (!finite9(f)) {
        rot[0] = qnan<Real>();
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
    // Displacement gradient in the rotated frame: grad u = R^T F - I (u_0 = 0 by the
    // node-0 anchoring of the corotated displacement), strain = sym(grad u).
    const M3<Real> g = linear ? f : mul(transpose(R), f);
    const Real exx = g.c[0].x - Real(1), eyy = g.c[1].y - Real(1), ezz = g.c[2].z - Real(1);
    const Real exy = Real(0.5) * (g.c[1].x + g.c[0].y);
    const Real eyz = Real(0.5) * (g.c[2].y + g.c[1].z);
    const Real exz = Real(0.5) * (g.c[2].x + g.c[0].z);
    const Real lam = __ldg(prm + 1), mu = __ldg(prm + 2);
    const Real tr = exx + eyy + ezz;
    const Real two_mu = Real(2) * mu;
    // V * sigma, sigma = lambda tr(eps) I + 2 mu eps  (engineering-shear D of BuildElasticityMatrix)
    const Real sxx = vol * (lam * tr + two_mu * exx), syy = vol * (lam * tr + two_mu * eyy),
               szz = vol * (lam * tr + two_mu * ezz);
    const Real sxy = vol * two_mu * exy, syz = vol * two_mu * eyz, sxz = vol * two_mu * exz;
    const M3<Real> sig = mcols(v3<Real>(sxx, sxy, sxz), v3<Real>(sxy, syy, syz), v3<Real>(sxz, syz, szz));
    const M3<Real> S = linear ? sig : mul(R, sig);
    st9(A.tets.rot, (size_t)t, R);
    st9(A.tets.stress, (size_t)t, S);
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

    const V3<Real> vr = ld3(A.v, node);
    V3<Real> fsum{Real(0), Real(0), Real(0)};
    V3<Real> kv{Real(0), Real(0), Real(0)};
    bool bad = false;
    const int i0 = __ldg(A.inc_start + r), i1 = __ldg(A.inc_start + r + 1);
    for (int i = i0; i < i1; ++i) {
        const int code = __ldg(A.inc_list + i);
        const int t = code >> 2, a = code & 3;
        const int4 tn = __ldg(A.tets.nodes + t);
        const int nb[4] = {tn.x, tn.y, tn.z, tn.w};
        V3<Real> vb[4];
        if (!A.explicit_mode) {
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                vb[b] = ld3(A.v, nb[b]);
                bad |= !finite3(vb[b]);
            }
        }
        const Real* rp = A.tets.rot + 9 * (size_t)t;
        if (isnan(__ldcg(rp))) continue;  // skipped tet: no force, no stiffness
        const M3<Real> R = ld9(A.tets.rot, (size_t)t);
        const M3<Real> S = ld9(A.tets.stress, (size_t)t);
        const M3<Real> dmi = ld9(A.tets.dm_inv, (size_t)t);
        const Real* prm = A.tets.params + 4 * (size_t)t;
        const Real vol = __ldg(prm + 0), lam = __ldg(prm + 1), mu = __ldg(prm + 2), damp = __ldg(prm + 3);
        // Shape gradients: g1..g3 are the rows of DmInv, g0 = -(g1+g2+g3).
        V3<Real> gr[4];
        gr[1] = v3<Real>(dmi.c[0].x, dmi.c[1].x, dmi.c[2].x);
        gr[2] = v3<Real>(dmi.c[0].y, dmi.c[1].y, dmi.c[2].y);
        gr[3] = v3<Real>(dmi.c[0].z, dmi.c[1].z, dmi.c[2].z);
        gr[0] = -((gr[1] + gr[2]) + gr[3]);
        const V3<Real> ga = gr[a];
        // Force on node a from this tet: elastic -S g_a plus damping -c v_a.
        const V3<Real> fa = (-mul(S, ga)) + vr * (-damp);
        if (finite3(fa)) fsum = fsum + fa;
        if (A.explicit_mode) continue;
        // K_ab = R Ke_ab R^T with Ke_ab = V (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I)
        //      = V (lambda P_a P_b^T + mu P_b P_a^T + mu (g_a.g_b) R R^T),  P = R g.
        const V3<Real> pa = mul(R, ga);
        const M3<Real> rrt = mul(R, transpose(R));
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const V3<Real> gb = gr[b];
            const V3<Real> pb = mul(R, gb);
            const Real l = vol * lam, m = vol * mu, md = vol * mu * dot(ga, gb);
            M3<Real> K;
            K.c[0] = pa * (l * pb.x) + pb * (m * pa.x) + rrt.c[0] * md;
            K.c[1] = pa * (l * pb.y) + pb * (m * pa.y) + rrt.c[1] * md;
            K.c[2] = pa * (l * pb.z) + pb * (m * pa.z) + rrt.c[2] * md;
            bad |= !finite9(K);
            kv = kv + mul(K, vb[b]);
            const int c = __ldg(A.node_to_dyn + nb[b]);
            if (c >= r) {
                int slot = 0;
                while (slot < nu && __ldg(A.a.col + ks + slot) != c) ++slot;
                if (slot < nu) {
                    PK_ACC(slot, 0) += K.c[0].x; PK_ACC(slot, 1) += K.c[0].y; PK_ACC(slot, 2) += K.c[0].z;
                    PK_ACC(slot, 3) += K.c[1].x; PK_ACC(slot, 4) += K.c[1].y; PK_ACC(slot, 5) += K.c[1].z;
                    PK_ACC(slot, 6) += K.c[2].x; PK_ACC(slot, 7) += K.c[2].y; PK_ACC(slot, 8) += K.c[2].z;
                } else {
                    bad = true;  // pattern does not hold the block: host/device mismatch
                }
            }
        }
    }
    const Real m = __ldg(A.mass + node);
    const V3<Real> grav{A.gravity[0], A.gravity[1], A.gravity[2]};
    fsum = fsum + grav * m;
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

    const Real dt2 = dt * dt;
    M3<Real> diag;
    for (int j = 0; j < nu; ++j) {
        M3<Real> blk;
        blk.c[0] = v3<Real>(PK_ACC(j, 0), PK_ACC(j, 1), PK_ACC(j, 2));
        blk.c[1] = v3<Real>(PK_ACC(j, 3), PK_ACC(j, 4), PK_ACC(j, 5));
        blk.c[2] = v3<Real>(PK_ACC(j, 6), PK_ACC(j, 7), PK_ACC(j, 8));
        bad |= !finite9(blk);
        blk = scale(blk, dt2);
        if (j == 0) {
            blk.c[0].x = m + blk.c[0].x;
            blk.c[1].y = m + blk.c[1].y;
            blk.c[2].z = m + blk.c[2].z;
            diag = blk;
        }
        st9(A.values, (size_t)(ks + j), blk);
    }
#undef PK_ACC
    const V3<Real> b = kv * (-dt2) + fsum * dt;
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

// ------------------------------------------------------------------ PCG kernel
template <class Real, class Acc>
__global__ void __launch_bounds__(kPcgThreads, 2) pcg_kernel(PcgArgs<Real, Acc> P)
{
    __shared__ Acc sh_acc[3 * 32];
    __shared__ int sh_int[32];
    __shared__ int s_flag;
    const int tid = threadIdx.x, T = blockDim.x, blk = blockIdx.x, G = gridDim.x;
    const int n = P.a.n;
    const int per = (n + G - 1) / G;
    const int r0 = min(n, blk * per), r1 = min(n, r0 + per);
    const int lane = tid & 31, warp = tid >> 5, nwarps = T >> 5;
    const int half = lane >> 4, hl = lane & 15;

    unsigned fl = 0;
    int iterations = 0;
    bool converged = false;
    Acc residual = Acc(0);
    bool have_x = true;
    bool timed_out = false;

    const unsigned in_flags = *(volatile unsigned*)P.flags;
    if (P.skip_on_flags && (in_flags & (kFlagPrecomputeFailed | kFlagSingularDiag))) {
        if (blk == 0 && tid == 0) {
            P.stats->iterations = 0;
            P.stats->converged = 0;
            P.stats->residual_norm = 0.0;
        }
        return;
    }

    // x = 0, r = b, s = M^-1 r, d_prev = 0; delta = r.s; also |r|^2 and finiteness.
    {
        Acc loc[2] = {Acc(0), Acc(0)};
        int bad = 0;
        for (int r = r0 + tid; r < r1; r += T) {
            const V3<Real> br = ld3(P.b, r);
            if (!finite3(br)) bad |= 1;
            const V3<Real> z{Real(0), Real(0), Real(0)};
            st3(P.x, r, z);
            st3(P.r, r, br);
            st3(P.d0, r, z);
            const M3<Real> mi = ld9(P.minv, (size_t)r);
            const V3<Real> s = mul(mi, br);
            if (!finite9(mi) || !finite3(s)) bad |= 2;
            st3(P.s, r, s);
            loc[0] += dot_acc<Acc>(br, s);
            loc[1] += dot_acc<Acc>(br, br);
        }
        block_sum<Acc, 2>(loc, sh_acc);
        bad = block_or(bad, sh_int);
        if (tid == 0) {
            P.part_b[2 * blk + 0] = loc[0];
            P.part_b[2 * blk + 1] = loc[1];
            P.part_bad[4 * blk + 1] = bad;
        }
    }
    if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }

    {
        Acc g[2];
        grid_sum<Acc, 2>(P.part_b, 2, g, sh_acc);
        const int bad = grid_or(P.part_bad + 1, 4, sh_int);
        Acc delta = g[0];
        Acc rr = g[1];
        if (bad & 1) {  // non-finite rhs: the reference clears x (solve fails)
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
        const Acc target = P.tolerance * P.tolerance * delta;
        if (!acc_finite(target)) goto final_check;
        if (delta <= target) {
            converged = true;
            residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
            goto final_check;
        }
        Acc beta = Acc(0);
        Real* dcur = P.d0;
        Real* dnext = P.d1;
        for (int it = 0; it < P.max_iterations; ++it) {
            if (delta <= target) {
                converged = true;
                break;
            }
            // Phase A: d_next = s + beta d_cur; q = A d_next; partial d_next . q
            {
                Acc loc[1] = {Acc(0)};
                int qbad = 0;
                for (int base = r0 + 2 * warp; base < r1; base += 2 * nwarps) {
                    const int r = base + half;
                    const bool valid = r < r1;
                    const V3<Real> q = row_spmv<Real, 16>(P.a, valid ? r : -1, hl, P.s, dcur, Real(beta), true);
                    if (valid && hl == 0) {
                        const V3<Real> dn = ldcg3(P.s, r) + ldcg3(dcur, r) * Real(beta);
                        st3(dnext, r, dn);
                        st3(P.q, r, q);
                        loc[0] += dot_acc<Acc>(dn, q);
                        if (!finite3(q)) qbad = 1;
                    }
                }
                block_sum<Acc, 1>(loc, sh_acc);
                qbad = block_or(qbad, sh_int);
                if (tid == 0) {
                    P.part_a[blk] = loc[0];
                    P.part_bad[4 * blk + 0] = qbad;
                }
            }
            if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
            Acc dq;
            {
                Acc g1[1];
                grid_sum<Acc, 1>(P.part_a, 1, g1, sh_acc);
                dq = g1[0];
                if (grid_or(P.part_bad, 4, sh_int)) { fl |= kFlagBreakdown; break; }
            }
            if (!acc_finite(dq) || dq <= Acc(0)) { fl |= kFlagBreakdown; break; }
            const Acc alpha = delta / dq;
            if (!acc_finite(alpha)) { fl |= kFlagBreakdown; break; }
            // Phase B: x += alpha d; r -= alpha q; s = M^-1 r; partial r.s and r.r
            {
                Acc loc[2] = {Acc(0), Acc(0)};
                int sbad = 0;
                for (int r = r0 + tid; r < r1; r += T) {
                    const V3<Real> dn = ldcg3(dnext, r);
                    const V3<Real> q = ldcg3(P.q, r);
                    const V3<Real> xv = axpy<Real, Acc>(ldplain3(P.x, r), alpha, dn);
                    const V3<Real> rv = axpy<Real, Acc>(ldplain3(P.r, r), -alpha, q);
                    st3(P.x, r, xv);
                    st3(P.r, r, rv);
                    const V3<Real> s = mul(ld9(P.minv, (size_t)r), rv);
                    if (!finite3(s)) sbad = 1;
                    st3(P.s, r, s);
                    loc[0] += dot_acc<Acc>(rv, s);
                    loc[1] += dot_acc<Acc>(rv, rv);
                }
                block_sum<Acc, 2>(loc, sh_acc);
                sbad = block_or(sbad, sh_int);
                if (tid == 0) {
                    P.part_b[2 * blk + 0] = loc[0];
                    P.part_b[2 * blk + 1] = loc[1];
                    P.part_bad[4 * blk + 1] = sbad;
                }
            }
            if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
            {
                Acc g2[2];
                grid_sum<Acc, 2>(P.part_b, 2, g2, sh_acc);
                rr = g2[1];
                if (grid_or(P.part_bad + 1, 4, sh_int)) { fl |= kFlagBreakdown; break; }
                const Acc old = delta;
                delta = g2[0];
                if (!acc_finite(delta) || !acc_finite(old) || old <= Acc(0)) { fl |= kFlagBreakdown; break; }
                beta = delta / old;
                if (!acc_finite(beta)) { fl |= kFlagBreakdown; break; }
            }
            Real* t = dcur;
            dcur = dnext;
            dnext = t;
            iterations = it + 1;
        }
        if (delta <= target) converged = true;
        residual = (acc_finite(rr) && rr >= Acc(0)) ? sqrt(rr) : Acc(INFINITY);
    }

final_check:
    // The solve succeeds when x is present and finite; integration is all-or-nothing.
    {
        int bad = 0;
        for (int r = r0 + tid; r < r1; r += T) {
            const V3<Real> dv = have_x ? ldplain3(P.x, r) : V3<Real>{Real(0), Real(0), Real(0)};
            if (!finite3(dv)) bad |= 1;
            if (P.integrate) {
                const int node = __ldg(P.dyn_to_node + r);
                const V3<Real> xo = ldplain3(P.node_x, node), vo = ldplain3(P.node_v, node);
                const V3<Real> nv = vo + dv;
                const V3<Real> nx = xo + nv * P.dt;
                if (!finite3(xo) || !finite3(vo) || !finite3(nv) || !finite3(nx)) bad |= 2;
            }
        }
        bad = block_or(bad, sh_int);
        if (tid == 0) P.part_bad[4 * blk + 2] = bad;
    }
    if (!grid_barrier(P.sync, &s_flag)) { timed_out = true; goto finish; }
    {
        const int bad = grid_or(P.part_bad + 2, 4, sh_int);
        const bool solved = have_x && !(bad & 1);
        if (!have_x) fl |= kFlagInvalidRhs;
        if (have_x && (bad & 1)) fl |= kFlagNonFiniteDv;
        if (solved) fl |= kFlagSolved;
        if (solved && P.integrate) {
            if (bad & 2) {
                fl |= kFlagIntegrateAbort;
            } else {
                for (int r = r0 + tid; r < r1; r += T) {
                    const int node = __ldg(P.dyn_to_node + r);
                    const V3<Real> dv = ldplain3(P.x, r);
                    const V3<Real> nv = ldplain3(P.node_v, node) + dv;
                    const V3<Real> nx = ldplain3(P.node_x, node) + nv * P.dt;
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
    if (blk == 0 && tid == 0) {
        P.stats->iterations = iterations;
        P.stats->converged = converged ? 1 : 0;
        P.stats->residual_norm = (double)residual;
        atomicOr(P.flags, fl);
    } else if (timed_out && tid == 0) {
        atomicOr(P.flags, kFlagBarrierTimeout);
    }
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
    if (args.explicit_mode || max_row_blocks <= 8) return launch_rows<Real, 8>(args, stream);
    if (max_row_blocks <= 16) return launch_rows<Real, 16>(args, stream);
    return launch_rows<Real, 0>(args, stream);
}

template <class Real, class Acc>
int pcg_max_grid(int threads)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<Real, Acc>, threads, 0) != cudaSuccess)
        return 0;
    return sms * per_sm;
}

template <class Real, class Acc>
cudaError_t launch_pcg_kernel(const PcgArgs<Real, Acc>& args, int grid, int threads, cudaStream_t stream)
{
    PcgArgs<Real, Acc> a = args;
    void* kargs[] = {&a};
    return cudaLaunchCooperativeKernel((const void*)pcg_kernel<Real, Acc>, dim3(grid), dim3(threads), kargs, 0,
                                       stream);
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
template cudaError_t launch_row_kernel<float>(const AssemblyArgs<float>&, int, cudaStream_t);
template cudaError_t launch_row_kernel<double>(const AssemblyArgs<double>&, int, cudaStream_t);
template cudaError_t launch_pcg_kernel<float, float>(const PcgArgs<float, float>&, int, int, cudaStream_t);
template cudaError_t launch_pcg_kernel<float, double>(const PcgArgs<float, double>&, int, int, cudaStream_t);
template cudaError_t launch_pcg_kernel<double, double>(const PcgArgs<double, double>&, int, int, cudaStream_t);
template int pcg_max_grid<float, float>(int);
template int pcg_max_grid<float, double>(int);
template int pcg_max_grid<double, double>(int);
template cudaError_t launch_spmv_kernel<float>(const BsrView<float>&, const float*, float*, cudaStream_t);
template cudaError_t launch_spmv_kernel<double>(const BsrView<double>&, const double*, double*, cudaStream_t);

}  // namespace pk
