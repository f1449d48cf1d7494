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

}  // namespace pk
