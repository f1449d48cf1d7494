// pk_math.cuh -- 3-vector / 3x3 helpers for the device kernels, templated on the
// scalar type (float for the FP32 and mixed paths, double for the FP64 path).
//
// Conventions follow PhysiK's math (include/PhysiK/Math/Vec3.h, Mat3.h): 3x3 blocks
// are column-major (c[j] is column j), the inverse is the adjugate over the
// determinant and returns the identity when |det| <= 1e-6 (Mat3.h:67-84), and the
// polar rotation is the Newton averaging iteration of FEMModel.cpp:115-163.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace pk {

template <class T>
struct V3 {
    T x, y, z;
};

template <class T>
struct M3 {
    V3<T> c[3];
};

template <class T>
__host__ __device__ __forceinline__ V3<T> v3(T x, T y, T z)
{
    return V3<T>{x, y, z};
}
template <class T>
__host__ __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b)
{
    return V3<T>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b)
{
    return V3<T>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a)
{
    return V3<T>{-a.x, -a.y, -a.z};
}
template <class T>
__host__ __device__ __forceinline__ V3<T> operator*(V3<T> a, T s)
{
    return V3<T>{a.x * s, a.y * s, a.z * s};
}
template <class T>
__host__ __device__ __forceinline__ T dot(V3<T> a, V3<T> b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
__host__ __device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b)
{
    return V3<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
__host__ __device__ __forceinline__ bool finite3(V3<T> a)
{
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}
template <class T>
__host__ __device__ __forceinline__ M3<T> mcols(V3<T> a, V3<T> b, V3<T> c)
{
    M3<T> m;
    m.c[0] = a;
    m.c[1] = b;
    m.c[2] = c;
    return m;
}
template <class T>
__host__ __device__ __forceinline__ M3<T> mident()
{
    return mcols(v3<T>(1, 0, 0), v3<T>(0, 1, 0), v3<T>(0, 0, 1));
}
template <class T>
__host__ __device__ __forceinline__ M3<T> mzero()
{
    return mcols(v3<T>(0, 0, 0), v3<T>(0, 0, 0), v3<T>(0, 0, 0));
}
// M v = c0*x + c1*y + c2*z
template <class T>
__host__ __device__ __forceinline__ V3<T> mul(const M3<T>& m, V3<T> v)
{
    return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z;
}
// M^T v
template <class T>
__host__ __device__ __forceinline__ V3<T> mul_t(const M3<T>& m, V3<T> v)
{
    return V3<T>{dot(m.c[0], v), dot(m.c[1], v), dot(m.c[2], v)};
}
template <class T>
__host__ __device__ __forceinline__ M3<T> mul(const M3<T>& a, const M3<T>& b)
{
    return mcols(mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2]));
}
template <class T>
__host__ __device__ __forceinline__ M3<T> transpose(const M3<T>& m)
{
    return mcols(v3<T>(m.c[0].x, m.c[1].x, m.c[2].x), v3<T>(m.c[0].y, m.c[1].y, m.c[2].y),
                 v3<T>(m.c[0].z, m.c[1].z, m.c[2].z));
}
template <class T>
__host__ __device__ __forceinline__ M3<T> add(const M3<T>& a, const M3<T>& b)
{
    return mcols(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]);
}
template <class T>
__host__ __device__ __forceinline__ M3<T> scale(const M3<T>& a, T s)
{
    return mcols(a.c[0] * s, a.c[1] * s, a.c[2] * s);
}
template <class T>
__host__ __device__ __forceinline__ T det(const M3<T>& m)
{
    return dot(m.c[0], cross(m.c[1], m.c[2]));
}
template <class T>
__host__ __device__ __forceinline__ bool finite9(const M3<T>& m)
{
    return finite3(m.c[0]) && finite3(m.c[1]) && finite3(m.c[2]);
}
// Adjugate inverse; identity when |det| <= 1e-6.
template <class T>
__host__ __device__ __forceinline__ M3<T> inverse(const M3<T>& m)
{
    const V3<T> r0 = cross(m.c[1], m.c[2]);
    const V3<T> r1 = cross(m.c[2], m.c[0]);
    const V3<T> r2 = cross(m.c[0], m.c[1]);
    const T d = dot(m.c[0], r0);
    if (fabs(d) <= T(0.000001)) return mident<T>();
    const T inv = T(1) / d;
    return transpose(mcols(r0 * inv, r1 * inv, r2 * inv));
}
template <class T, class U>
__host__ __device__ __forceinline__ M3<T> cast(const M3<U>& m)
{
    return mcols(v3<T>(T(m.c[0].x), T(m.c[0].y), T(m.c[0].z)), v3<T>(T(m.c[1].x), T(m.c[1].y), T(m.c[1].z)),
                 v3<T>(T(m.c[2].x), T(m.c[2].y), T(m.c[2].z)));
}
template <class T, class U>
__host__ __device__ __forceinline__ V3<T> cast(const V3<U>& a)
{
    return v3<T>(T(a.x), T(a.y), T(a.z));
}

// Polar rotation of F by Newton averaging R <- (R + R^-T)/2: at most 12 iterations,
// stop when ||R_next - R||_F^2 <= 1e-10, identity when F or an iterate is singular
// (|det| <= 1e-8) or non-finite, and negate column 2 if det(R) < 0.
// Returns the iteration count through *iterations; *fallback is set on the identity exits.
template <class T>
__host__ __device__ inline M3<T> polar_rotation(const M3<T>& f, int* iterations, bool* fallback)
{
    const T min_det = T(1.0e-8);
    *iterations = 0;
    *fallback = false;
    if (!finite9(f) || fabs(det(f)) <= min_det) {
        *fallback = true;
        return mident<T>();
    }
    M3<T> r = f;
    for (int it = 0; it < 12; ++it) {
        *iterations = it + 1;
        const M3<T> ti = inverse(transpose(r));
        if (!finite9(ti) || fabs(det(ti)) <= min_det) {
            *fallback = true;
            return mident<T>();
        }
        const M3<T> next = scale(add(r, ti), T(0.5));
        if (!finite9(next)) {
            *fallback = true;
            return mident<T>();
        }
        T diff = T(0);
        for (int col = 0; col < 3; ++col) {
            const V3<T> d = next.c[col] - r.c[col];
            diff += dot(d, d);
        }
        r = next;
        if (diff <= T(1.0e-10)) break;
    }
    if (!finite9(r)) {
        *fallback = true;
        return mident<T>();
    }
    if (det(r) < T(0)) r.c[2] = r.c[2] * T(-1);
    return r;
}

// S = R V sigma of a corotated tet (V sigma for the linear model, R = I), so that corner
// a's elastic force is -S g_a: the displacement gradient in the rotated frame is
// g = R^T F - I (F - I for the linear model; the corotated displacement is anchored at
// node 0), eps = sym(g), V sigma = V (lambda tr(eps) I + 2 mu eps) with the engineering-
// shear D of FEMModel::BuildElasticityMatrix (FEMModel.cpp:174-200, 247-271, 336-424).
template <class T>
__host__ __device__ __forceinline__ M3<T> corotated_stress(const M3<T>& f, const M3<T>& R, bool linear, T vol, T lam,
                                                          T mu)
{
    const M3<T> g = linear ? f : mul(transpose(R), f);
    const T exx = g.c[0].x - T(1), eyy = g.c[1].y - T(1), ezz = g.c[2].z - T(1);
    const T exy = T(0.5) * (g.c[1].x + g.c[0].y);
    const T eyz = T(0.5) * (g.c[2].y + g.c[1].z);
    const T exz = T(0.5) * (g.c[2].x + g.c[0].z);
    const T tr = exx + eyy + ezz;
    const T two_mu = T(2) * mu;
    const T sxx = vol * (lam * tr + two_mu * exx), syy = vol * (lam * tr + two_mu * eyy),
            szz = vol * (lam * tr + two_mu * ezz);
    const T sxy = vol * two_mu * exy, syz = vol * two_mu * eyz, sxz = vol * two_mu * exz;
    const M3<T> sig = mcols(v3<T>(sxx, sxy, sxz), v3<T>(sxy, syy, syz), v3<T>(sxz, syz, szz));
    return linear ? sig : mul(R, sig);
}

// The tet's stiffness applied to per-node vectors u_0..u_3, folded: with
// K_ab = R Ke_ab R^T and Ke_ab = V (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I),
//   sum_b K_ab u_b = Q g_a,  Q = V R (lambda tr(G) I + mu (G + G^T)),
//   G = R^T sum_b u_b g_b^T = R^T [u1 - u0, u2 - u0, u3 - u0] DmInv   (R = I when linear).
template <class T>
__host__ __device__ __forceinline__ M3<T> folded_stiffness(const M3<T>& R, const M3<T>& dmi, const V3<T> (&u)[4],
                                                          bool linear, T vol, T lam, T mu)
{
    const M3<T> fd = mul(mcols(u[1] - u[0], u[2] - u[0], u[3] - u[0]), dmi);
    const M3<T> G = linear ? fd : mul(transpose(R), fd);
    const T ltr = vol * lam * ((G.c[0].x + G.c[1].y) + G.c[2].z);
    const T vm = vol * mu;
    M3<T> P;
    P.c[0] = v3<T>(ltr + vm * (G.c[0].x + G.c[0].x), vm * (G.c[0].y + G.c[1].x), vm * (G.c[0].z + G.c[2].x));
    P.c[1] = v3<T>(vm * (G.c[1].x + G.c[0].y), ltr + vm * (G.c[1].y + G.c[1].y), vm * (G.c[1].z + G.c[2].y));
    P.c[2] = v3<T>(vm * (G.c[2].x + G.c[0].z), vm * (G.c[2].y + G.c[1].z), ltr + vm * (G.c[2].z + G.c[2].z));
    return linear ? P : mul(R, P);
}

// Shape-function gradients: g1..g3 are the rows of DmInv, g0 = -(g1 + g2 + g3).
template <class T>
__host__ __device__ __forceinline__ void shape_gradients(const M3<T>& dmi, V3<T> (&gr)[4])
{
    gr[1] = v3<T>(dmi.c[0].x, dmi.c[1].x, dmi.c[2].x);
    gr[2] = v3<T>(dmi.c[0].y, dmi.c[1].y, dmi.c[2].y);
    gr[3] = v3<T>(dmi.c[0].z, dmi.c[1].z, dmi.c[2].z);
    gr[0] = -((gr[1] + gr[2]) + gr[3]);
}

}  // namespace pk
