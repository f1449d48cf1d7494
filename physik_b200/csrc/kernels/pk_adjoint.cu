// pk_adjoint.cu -- backward (adjoint) element kernel of the implicit corotated step.
//
// No counterpart in the reference (PhysiK has no adjoint).  One implicit-Euler step at
// state (x, v) solves A du = b with A = M + dt^2 K(x) and b = dt f(x, v) - dt^2 K(x) v
// (SolverData::AssembleImplicitMatrixAndRhs, src/Core/Solvers/SolverData.cpp:308-465;
// element terms of FEMModel::ComputeCorotationalElasticForces, src/Core/Physics/FEM/
// FEMModel.cpp:635-679), then v' = v + du, x' = x + dt v'.  Given the adjoint solution w
// of A w = g (g = adjoint of v' plus dt times the adjoint of x'), the step's remaining
// sensitivities are those of the scalar
//     J(x, theta) = dt w.f(x) - dt^2 w.K(x) z,      z = v + du (du on dynamic rows),
// with w and z held fixed.  Per tet (nodes a, shape gradients g_a, Wg = sum w_a g_a^T,
// Zg = sum z_a g_a^T, F = Ds DmInv, R = polar(F), sigma = lambda tr(eps) I + 2 mu eps with
// eps = sym(R^T F) - I, elastic force f_a = -V R sigma g_a, block K_ab = V (lambda P_a P_b^T
// + mu P_b P_a^T + mu (g_a.g_b) R R^T), P = R g):
//     T1 = -dt V <R sigma, Wg>
//     T2 = -dt^2 V [lambda <R,Wg> <R,Zg> + mu tr(Aw Az) + mu <Aw, Az>],  Aw = R^T Wg, Az = R^T Zg
// Both are linear in E, so d J / d theta_e (theta = log E) is T1 + T2 of tet e itself.
// The x-gradient goes through F directly (via sigma) and through R: with Sbar = lambda
// tr(Y) I + 2 mu sym(Y), Y = R^T Wg,
//     dJ/dR = -dt V (Wg sigma + F Sbar)
//             - dt^2 V [lambda (<R,Zg> Wg + <R,Wg> Zg) + mu (Wg Az + Zg Aw) + mu (Wg Zg^T + Zg Wg^T) R]
//     dJ/dF = -dt V R Sbar + (dJ/dR pulled back through the forward's polar iteration,
//             reverse mode over its Newton steps; see below), and dJ/dDs = dJ/dF DmInv^T.
// The linear model (R = I) has only the direct term.  Everything is evaluated in double
// from the state in the system's storage precision; R is recomputed by the same Newton
// polar iteration as the forward kernel.
#include <cuda_runtime.h>
#include <math.h>

#include "pk_device.cuh"

namespace pk {
namespace {

__device__ __forceinline__ double frob(const M3<double>& a, const M3<double>& b)
{
    return dot(a.c[0], b.c[0]) + dot(a.c[1], b.c[1]) + dot(a.c[2], b.c[2]);
}
__device__ __forceinline__ M3<double> outer_sum(const V3<double> (&u)[4], const V3<double> (&g)[4])
{
    // sum_a u_a g_a^T (column j = sum_a u_a g_a[j])
    M3<double> m = mzero<double>();
    for (int a = 0; a < 4; ++a) {
        m.c[0] = m.c[0] + u[a] * g[a].x;
        m.c[1] = m.c[1] + u[a] * g[a].y;
        m.c[2] = m.c[2] + u[a] * g[a].z;
    }
    return m;
}
__device__ __forceinline__ M3<double> msym(const M3<double>& m)
{
    return scale(add(m, transpose(m)), 0.5);
}
__device__ __forceinline__ double mtrace(const M3<double>& m) { return m.c[0].x + m.c[1].y + m.c[2].z; }
__device__ __forceinline__ M3<double> diag_add(const M3<double>& m, double s)
{
    M3<double> r = m;
    r.c[0].x += s;
    r.c[1].y += s;
    r.c[2].z += s;
    return r;
}
template <class Real>
__global__ void __launch_bounds__(128) adjoint_tet_kernel(AdjointArgs<Real> A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.tet_count) return;
    double* gx = A.tet_grad + 12 * (size_t)t;
    const Real* prm = A.params + 4 * (size_t)t;
    const double vol = double(__ldg(prm + 0)), lam = double(__ldg(prm + 1)), mu = double(__ldg(prm + 2));
    const unsigned char en = __ldg(A.enabled + t);
    for (int i = 0; i < 12; ++i) gx[i] = 0.0;
    A.tet_theta[t] = 0.0;
    if (!(en & 1u) || !(vol > 0.0)) return;
    const bool linear = A.linear || (en & 2u);
    const int4 tn = __ldg(A.nodes + t);
    const int nd[4] = {tn.x, tn.y, tn.z, tn.w};
    V3<double> x[4], w[4], z[4];
    for (int a = 0; a < 4; ++a) {
        const Real* xp = A.x + 3 * (size_t)nd[a];
        const Real* vp = A.v + 3 * (size_t)nd[a];
        x[a] = v3<double>(double(xp[0]), double(xp[1]), double(xp[2]));
        z[a] = v3<double>(double(vp[0]), double(vp[1]), double(vp[2]));
        w[a] = v3<double>(0.0, 0.0, 0.0);
        const int r = __ldg(A.node_to_dyn + nd[a]);
        if (r >= 0) {
            w[a] = v3<double>(A.w[3 * r], A.w[3 * r + 1], A.w[3 * r + 2]);
            z[a] = z[a] + v3<double>(A.du[3 * r], A.du[3 * r + 1], A.du[3 * r + 2]);
        }
    }
    M3<double> dmi;
    {
        const Real* q = A.dm_inv + 9 * (size_t)t;
        dmi = mcols(v3<double>(q[0], q[1], q[2]), v3<double>(q[3], q[4], q[5]), v3<double>(q[6], q[7], q[8]));
    }
    V3<double> g[4];
    g[1] = v3<double>(dmi.c[0].x, dmi.c[1].x, dmi.c[2].x);
    g[2] = v3<double>(dmi.c[0].y, dmi.c[1].y, dmi.c[2].y);
    g[3] = v3<double>(dmi.c[0].z, dmi.c[1].z, dmi.c[2].z);
    g[0] = -((g[1] + g[2]) + g[3]);
    const M3<double> ds = mcols(x[1] - x[0], x[2] - x[0], x[3] - x[0]);
    const M3<double> F = mul(ds, dmi);
    if (!finite9(F)) return;
    M3<double> R = mident<double>();
    if (!linear) {
        int iters = 0;
        bool fallback = false;
        R = polar_rotation<double>(F, &iters, &fallback);
    }
    const double dt = A.dt, dt2 = A.dt * A.dt;
    const M3<double> Wg = outer_sum(w, g), Zg = outer_sum(z, g);
    const M3<double> Rt = transpose(R);
    const M3<double> eps = diag_add(msym(mul(Rt, F)), -1.0);
    const M3<double> sigma = add(scale(mident<double>(), lam * mtrace(eps)), scale(eps, 2.0 * mu));
    const M3<double> Aw = mul(Rt, Wg), Az = mul(Rt, Zg);
    const double rw = frob(R, Wg), rz = frob(R, Zg);
    const double T1 = -dt * vol * frob(mul(R, sigma), Wg);
    const double T2 = -dt2 * vol * (lam * rw * rz + mu * mtrace(mul(Aw, Az)) + mu * frob(Aw, Az));
    A.tet_theta[t] = T1 + T2;

    const M3<double> Sbar = add(scale(mident<double>(), lam * mtrace(Aw)), scale(msym(Aw), 2.0 * mu));
    M3<double> GF = scale(mul(R, Sbar), -dt * vol);
    if (!linear) {
        M3<double> GR = scale(add(mul(Wg, sigma), mul(F, Sbar)), -dt * vol);
        const M3<double> t2 = add(add(scale(Wg, lam * rz), scale(Zg, lam * rw)),
                                  add(scale(add(mul(Wg, Az), mul(Zg, Aw)), mu),
                                      scale(mul(add(mul(Wg, transpose(Zg)), mul(Zg, transpose(Wg))), R), mu)));
        GR = add(GR, scale(t2, -dt2 * vol));
        // R is the forward's Newton iterate R_n (R_0 = F, R_k+1 = (R_k + R_k^-T) / 2, at most
        // 12 steps, stopped when the squared step <= 1e-10), with column 2 negated when
        // det R_n < 0.  Reverse through exactly those iterations: with G = dJ/dR_k+1,
        // dJ/dR_k = (G - R_k^-T G^T R_k^-T) / 2; dJ/dR_0 is the F-gradient through R.  (The
        // closed-form polar derivative is not exact where the iteration stops short, i.e.
        // for nearly flat elements.)  An identity fallback carries no derivative.
        M3<double> iter[13];
        int n = 0;
        bool fallback = !finite9(F) || fabs(det(F)) <= 1.0e-8;
        if (!fallback) {
            iter[0] = F;
            for (int it = 0; it < 12; ++it) {
                const M3<double> ti = inverse(transpose(iter[it]));
                if (!finite9(ti) || fabs(det(ti)) <= 1.0e-8) {
                    fallback = true;
                    break;
                }
                iter[it + 1] = scale(add(iter[it], ti), 0.5);
                if (!finite9(iter[it + 1])) {
                    fallback = true;
                    break;
                }
                n = it + 1;
                double diff = 0.0;
                for (int col = 0; col < 3; ++col) {
                    const V3<double> d = iter[it + 1].c[col] - iter[it].c[col];
                    diff += dot(d, d);
                }
                if (diff <= 1.0e-10) break;
            }
        }
        if (!fallback) {
            M3<double> G = GR;
            if (det(iter[n]) < 0.0) G.c[2] = G.c[2] * -1.0;
            for (int k = n - 1; k >= 0; --k) {
                // inverse() returns the identity (a constant) when |det| <= 1e-6, as in the forward
                if (fabs(det(iter[k])) <= 1.0e-6) {
                    G = scale(G, 0.5);
                } else {
                    const M3<double> xt = inverse(transpose(iter[k]));
                    G = scale(add(G, scale(mul(mul(xt, transpose(G)), xt), -1.0)), 0.5);
                }
            }
            GF = add(GF, G);
        }
    }
    const M3<double> GDs = mul(GF, transpose(dmi));
    const V3<double> g1 = GDs.c[0], g2 = GDs.c[1], g3 = GDs.c[2];
    const V3<double> g0 = -((g1 + g2) + g3);
    const V3<double> out[4] = {g0, g1, g2, g3};
    for (int a = 0; a < 4; ++a) {
        gx[3 * a] = out[a].x;
        gx[3 * a + 1] = out[a].y;
        gx[3 * a + 2] = out[a].z;
    }
}

}  // namespace

template <class Real>
cudaError_t launch_adjoint_tet_kernel(const AdjointArgs<Real>& args, cudaStream_t stream)
{
    if (args.tet_count <= 0) return cudaSuccess;
    const int threads = 128, blocks = (args.tet_count + threads - 1) / threads;
    adjoint_tet_kernel<Real><<<blocks, threads, 0, stream>>>(args);
    return cudaGetLastError();
}

template cudaError_t launch_adjoint_tet_kernel<float>(const AdjointArgs<float>&, cudaStream_t);
template cudaError_t launch_adjoint_tet_kernel<double>(const AdjointArgs<double>&, cudaStream_t);

}  // namespace pk
