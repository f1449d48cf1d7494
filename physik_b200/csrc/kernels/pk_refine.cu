// pk_refine.cu -- FP64 outer true-residual refinement of the implicit step's solve.
//
// No counterpart in the reference (PhysiK solves once, in FP32, with
// SolvePreconditionedConjugateGradient, src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:
// 114-241).  With FP32 storage the PCG's recursive residual can claim convergence while the
// true residual of its iterate is larger, and the FP32 blocks and right-hand side carry
// their own rounding; the host loop in pk_system.cu accumulates the solution in FP64,
// recomputes the true residual of the FP64 system -- element by element from the tets in
// FP64 (elem_* kernels) when the world holds only soft bodies, else over the stored blocks
// -- and runs correction solves A e = r within the remaining iteration budget until that
// residual meets the reference's stopping target r^T M^-1 r <= tol^2 b^T M^-1 b.  These
// are its kernels:
//
//   elem_vx_kernel / elem_tet_kernel / elem_row_kernel
//                            the FP64 residual from the tet data (ElemResidualArgs)
//
//   refine_residual_kernel   r = b - A x (x in FP64; NULL: r = b), written rounded to the
//                            storage type as the next correction's right-hand side, and
//                            per-block partials of r^T M^-1 r and r.r (FP64, fixed order)
//   refine_accumulate_kernel x64 (+)= the last solve's delta-v
//   refine_check_kernel /    the all-or-nothing update of World::IntegrateImplicitEuler
//   refine_apply_kernel      (src/Core/World/World.cpp:644-695) from the FP64 delta-v
#include <cuda_runtime.h>
#include <math.h>

#include "pk_device.cuh"

namespace pk {
namespace {

template <class Real>
__global__ void __launch_bounds__(kRefineThreads) refine_residual_kernel(RefineArgs<Real> A)
{
    constexpr int W = 16;  // lanes per row
    const int lane = threadIdx.x & 31;
    const int hl = lane & (W - 1);
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) / W;
    const bool valid = r < A.a.n;
    double ax = 0.0, ay = 0.0, az = 0.0;
    int bad = 0;
    if (valid && A.x64) {
        const int ks = __ldg(A.a.row_start + r), ke = __ldg(A.a.row_start + r + 1);
        const int ls = __ldg(A.a.lt_start + r), le = __ldg(A.a.lt_start + r + 1);
        const int nu = ke - ks, tot = nu + (le - ls);
        for (int j = hl; j < tot; j += W) {
            int k, c;
            const bool tr = j >= nu;
            if (!tr) {
                k = ks + j;
                c = __ldg(A.a.col + k);
            } else {
                const int e = ls + (j - nu);
                k = __ldg(A.a.lt_block + e);
                c = __ldg(A.a.lt_row + e);
            }
            if ((unsigned)c >= (unsigned)A.a.n) {
                bad = 1;
                continue;
            }
            const Real* B = A.a.values + 9 * (size_t)k;
            const double x0 = A.x64[3 * (size_t)c], x1 = A.x64[3 * (size_t)c + 1], x2 = A.x64[3 * (size_t)c + 2];
            // Column-major block: element (i, m) is B[3m + i]; the transposed lower entry
            // uses element (m, i).
            double b[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) b[e] = double(__ldg(B + e));
            if (!tr) {
                ax += b[0] * x0 + b[3] * x1 + b[6] * x2;
                ay += b[1] * x0 + b[4] * x1 + b[7] * x2;
                az += b[2] * x0 + b[5] * x1 + b[8] * x2;
            } else {
                ax += b[0] * x0 + b[1] * x1 + b[2] * x2;
                ay += b[3] * x0 + b[4] * x1 + b[5] * x2;
                az += b[6] * x0 + b[7] * x1 + b[8] * x2;
            }
        }
    }
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, off);
        ay += __shfl_xor_sync(0xffffffffu, ay, off);
        az += __shfl_xor_sync(0xffffffffu, az, off);
    }
    bad = __reduce_or_sync(0xffffffffu, (unsigned)bad);
    double v[2] = {0.0, 0.0};
    if (valid && hl == 0) {
        const Real* bp = A.b + 3 * (size_t)r;
        const double r0 = double(bp[0]) - ax, r1 = double(bp[1]) - ay, r2 = double(bp[2]) - az;
        const Real* m = A.minv + 9 * (size_t)r;
        const double z0 = double(m[0]) * r0 + double(m[3]) * r1 + double(m[6]) * r2;
        const double z1 = double(m[1]) * r0 + double(m[4]) * r1 + double(m[7]) * r2;
        const double z2 = double(m[2]) * r0 + double(m[5]) * r1 + double(m[8]) * r2;
        v[0] = r0 * z0 + r1 * z1 + r2 * z2;
        v[1] = r0 * r0 + r1 * r1 + r2 * r2;
        if (A.rhs_out) {
            Real* o = A.rhs_out + 3 * (size_t)r;
            o[0] = Real(r0);
            o[1] = Real(r1);
            o[2] = Real(r2);
        }
        if (!isfinite(v[0]) || !isfinite(v[1])) bad = 1;
    }
    __shared__ double sh[2 * 32];
    block_sum<double, 2>(v, sh);
    if (threadIdx.x == 0) {
        A.partials[2 * blockIdx.x] = v[0];
        A.partials[2 * blockIdx.x + 1] = v[1];
    }
    if (bad && hl == 0) atomicOr(A.bad, 1);
}

template <class Real>
__global__ void refine_accumulate_kernel(double* x64, const Real* dx, int count, int first)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    x64[i] = (first ? 0.0 : x64[i]) + double(dx[i]);
}

// Pass 1: delta-v in the storage type (also written back as the step's delta-v), and the
// finiteness checks of the update; pass 2 applies it only if nothing failed anywhere.
template <class Real>
__global__ void refine_check_kernel(RefineArgs<Real> A)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.a.n) return;
    const V3<Real> dv{Real(A.x64[3 * (size_t)r]), Real(A.x64[3 * (size_t)r + 1]), Real(A.x64[3 * (size_t)r + 2])};
    st3(A.dx, r, dv);
    int bad = finite3(dv) ? 0 : 1;
    if (A.integrate) {
        const int node = __ldg(A.dyn_to_node + r);
        const V3<Real> xo = ldplain3(A.node_x, node), vo = ldplain3(A.node_v, node);
        const V3<Real> nv = vo + dv;
        const V3<Real> nx = xo + nv * A.dt;
        if (!finite3(xo) || !finite3(vo) || !finite3(nv) || !finite3(nx)) bad |= 2;
    }
    if (bad) atomicOr(A.bad, bad);
}

template <class Real>
__global__ void refine_apply_kernel(RefineArgs<Real> A)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.a.n || *(volatile int*)A.bad) return;
    const int node = __ldg(A.dyn_to_node + r);
    const V3<Real> dv = ldplain3(A.dx, r);
    const V3<Real> nv = ldplain3(A.node_v, node) + dv;
    const V3<Real> nx = ldplain3(A.node_x, node) + nv * A.dt;
    st3(A.node_v, node, nv);
    st3(A.node_x, node, nx);
}

// ---- the FP64 residual from the tet data ----
template <class Real>
__global__ void elem_vx_kernel(ElemResidualArgs<Real> A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.node_count) return;
    const int c = __ldg(A.node_to_dyn + i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double u = double(A.v[3 * (size_t)i + k]);
        if (A.x64 && c >= 0 && c < A.n) u += A.x64[3 * (size_t)c + k];
        A.vx[3 * (size_t)i + k] = u;
    }
}

template <class Real>
__global__ void elem_tet_kernel(ElemResidualArgs<Real> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.tet_count) return;
    double* u = A.u + 9 * (size_t)t;
    const double* p = A.params + 4 * (size_t)t;
    const double vol = p[0], lam = p[1], mu = p[2];
    const unsigned char en = __ldg(A.enabled + t);
    if (!(en & 1u) || !(vol > 0.0)) {
        u[0] = qnan<double>();
        return;
    }
    const bool linear = A.linear || (en & 2u);
    const int4 n = __ldg(A.tet_nodes + t);
    const int nd[4] = {n.x, n.y, n.z, n.w};
    V3<double> xs[4], us[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        xs[k] = V3<double>{double(A.x[3 * (size_t)nd[k]]), double(A.x[3 * (size_t)nd[k] + 1]),
                           double(A.x[3 * (size_t)nd[k] + 2])};
        us[k] = V3<double>{A.vx[3 * (size_t)nd[k]], A.vx[3 * (size_t)nd[k] + 1], A.vx[3 * (size_t)nd[k] + 2]};
    }
    M3<double> dmi;
    for (int e = 0; e < 9; ++e) (&dmi.c[0].x)[e] = A.dm_inv[9 * (size_t)t + e];
    const M3<double> f = mul(mcols(xs[1] - xs[0], xs[2] - xs[0], xs[3] - xs[0]), dmi);
    if (!finite9(f)) {
        u[0] = qnan<double>();
        return;
    }
    M3<double> R = mident<double>();
    if (!linear) {
        int iters = 0;
        bool fallback = false;
        R = polar_rotation<double>(f, &iters, &fallback);
    }
    const M3<double> S = corotated_stress(f, R, linear, vol, lam, mu);
    const M3<double> Q = folded_stiffness(R, dmi, us, linear, vol, lam, mu);
    const double dt = A.dt, dt2 = dt * dt;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const V3<double> c = -(S.c[j] * dt + Q.c[j] * dt2);
        u[3 * j] = c.x;
        u[3 * j + 1] = c.y;
        u[3 * j + 2] = c.z;
    }
}

template <class Real>
__global__ void __launch_bounds__(kRefineThreads) elem_row_kernel(ElemResidualArgs<Real> A)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    int bad = 0;
    if (r < A.n) {
        const int node = __ldg(A.dyn_to_node + r);
        const V3<double> vr{double(A.v[3 * (size_t)node]), double(A.v[3 * (size_t)node + 1]),
                            double(A.v[3 * (size_t)node + 2])};
        V3<double> acc{0.0, 0.0, 0.0};
        for (int i = __ldg(A.inc_start + r); i < __ldg(A.inc_start + r + 1); ++i) {
            const int code = __ldg(A.inc_list + i);
            const int t = code >> 2, a = code & 3;
            const double* u = A.u + 9 * (size_t)t;
            if (isnan(u[0])) continue;  // a skipped tet
            M3<double> dmi, U;
            for (int e = 0; e < 9; ++e) {
                (&dmi.c[0].x)[e] = A.dm_inv[9 * (size_t)t + e];
                (&U.c[0].x)[e] = u[e];
            }
            V3<double> gr[4];
            shape_gradients(dmi, gr);
            V3<double> ga = gr[0];
#pragma unroll
            for (int k = 1; k < 4; ++k)
                if (a == k) ga = gr[k];
            const double damp = A.params[4 * (size_t)t + 3];
            acc = acc + mul(U, ga) + vr * (-(A.dt * damp));
        }
        const double m = A.mass[node];
        V3<double> x{0.0, 0.0, 0.0};
        if (A.x64) x = V3<double>{A.x64[3 * (size_t)r], A.x64[3 * (size_t)r + 1], A.x64[3 * (size_t)r + 2]};
        const V3<double> g{A.gravity[0], A.gravity[1], A.gravity[2]};
        const V3<double> res = acc + g * (A.dt * m) - x * m;
        const Real* mi = A.minv + 9 * (size_t)r;
        const double z0 = double(mi[0]) * res.x + double(mi[3]) * res.y + double(mi[6]) * res.z;
        const double z1 = double(mi[1]) * res.x + double(mi[4]) * res.y + double(mi[7]) * res.z;
        const double z2 = double(mi[2]) * res.x + double(mi[5]) * res.y + double(mi[8]) * res.z;
        v[0] = res.x * z0 + res.y * z1 + res.z * z2;
        v[1] = dot(res, res);
        if (A.rhs_out) {
            Real* o = A.rhs_out + 3 * (size_t)r;
            o[0] = Real(res.x);
            o[1] = Real(res.y);
            o[2] = Real(res.z);
        }
        if (!isfinite(v[0]) || !isfinite(v[1])) bad = 1;
    }
    __shared__ double sh[2 * 32];
    block_sum<double, 2>(v, sh);
    if (threadIdx.x == 0) {
        A.partials[2 * blockIdx.x] = v[0];
        A.partials[2 * blockIdx.x + 1] = v[1];
    }
    if (bad) atomicOr(A.bad, 1);
}

}  // namespace

template <class Real>
int elem_residual_blocks(int n)
{
    return (n + kRefineThreads - 1) / kRefineThreads;
}

template <class Real>
cudaError_t launch_elem_residual(const ElemResidualArgs<Real>& a, cudaStream_t stream)
{
    if (a.n <= 0) return cudaSuccess;
    if (a.node_count > 0) elem_vx_kernel<Real><<<(a.node_count + 255) / 256, 256, 0, stream>>>(a);
    if (a.tet_count > 0) elem_tet_kernel<Real><<<(a.tet_count + 127) / 128, 128, 0, stream>>>(a);
    elem_row_kernel<Real><<<elem_residual_blocks<Real>(a.n), kRefineThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

template <class Real>
int refine_residual_blocks(int n)
{
    const long long threads = 16ll * n;
    return static_cast<int>((threads + kRefineThreads - 1) / kRefineThreads);
}

template <class Real>
cudaError_t launch_refine_residual(const RefineArgs<Real>& args, cudaStream_t stream)
{
    if (args.a.n <= 0) return cudaSuccess;
    refine_residual_kernel<Real><<<refine_residual_blocks<Real>(args.a.n), kRefineThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_refine_accumulate(double* x64, const Real* dx, int count, int first, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    refine_accumulate_kernel<Real><<<(count + 255) / 256, 256, 0, stream>>>(x64, dx, count, first);
    return cudaGetLastError();
}

template <class Real>
cudaError_t launch_refine_update(const RefineArgs<Real>& args, cudaStream_t stream)
{
    if (args.a.n <= 0) return cudaSuccess;
    const int blocks = (args.a.n + 255) / 256;
    refine_check_kernel<Real><<<blocks, 256, 0, stream>>>(args);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !args.integrate) return e;
    refine_apply_kernel<Real><<<blocks, 256, 0, stream>>>(args);
    return cudaGetLastError();
}

template int elem_residual_blocks<float>(int);
template int elem_residual_blocks<double>(int);
template cudaError_t launch_elem_residual<float>(const ElemResidualArgs<float>&, cudaStream_t);
template cudaError_t launch_elem_residual<double>(const ElemResidualArgs<double>&, cudaStream_t);
template int refine_residual_blocks<float>(int);
template int refine_residual_blocks<double>(int);
template cudaError_t launch_refine_residual<float>(const RefineArgs<float>&, cudaStream_t);
template cudaError_t launch_refine_residual<double>(const RefineArgs<double>&, cudaStream_t);
template cudaError_t launch_refine_accumulate<float>(double*, const float*, int, int, cudaStream_t);
template cudaError_t launch_refine_accumulate<double>(double*, const double*, int, int, cudaStream_t);
template cudaError_t launch_refine_update<float>(const RefineArgs<float>&, cudaStream_t);
template cudaError_t launch_refine_update<double>(const RefineArgs<double>&, cudaStream_t);

}  // namespace pk
