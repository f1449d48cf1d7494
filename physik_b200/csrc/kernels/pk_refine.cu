// pk_refine.cu -- FP64 outer true-residual refinement of the implicit step's solve.
//
// No counterpart in the reference (PhysiK solves once, in FP32, with
// SolvePreconditionedConjugateGradient, src/Core/Solvers/Linear/ConjugateGradientSolver.cpp:
// 114-241).  With FP32 storage the PCG's recursive residual can claim convergence while the
// true residual b - A x of its iterate is larger; the host loop in pk_system.cu then
// accumulates the solution in FP64, recomputes the true residual with FP64 arithmetic over
// the assembled (stored) blocks, and runs correction solves A e = r within the remaining
// iteration budget until the true residual meets the reference's stopping target
// r^T M^-1 r <= tol^2 b^T M^-1 b.  These are its kernels:
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

}  // namespace

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

template int refine_residual_blocks<float>(int);
template int refine_residual_blocks<double>(int);
template cudaError_t launch_refine_residual<float>(const RefineArgs<float>&, cudaStream_t);
template cudaError_t launch_refine_residual<double>(const RefineArgs<double>&, cudaStream_t);
template cudaError_t launch_refine_accumulate<float>(double*, const float*, int, int, cudaStream_t);
template cudaError_t launch_refine_accumulate<double>(double*, const double*, int, int, cudaStream_t);
template cudaError_t launch_refine_update<float>(const RefineArgs<float>&, cudaStream_t);
template cudaError_t launch_refine_update<double>(const RefineArgs<double>&, cudaStream_t);

}  // namespace pk
