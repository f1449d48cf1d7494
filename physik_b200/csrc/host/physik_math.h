// physik_math.h -- host-side Vec3 / Mat3 with PhysiK's layout and semantics
// (include/PhysiK/Math/Vec3.h:7-95, Mat3.h:11-84): FP32 3-vectors, column-major 3x3
// whose default value is the identity, adjugate inverse with an identity result for
// |det| <= 1e-6.  Templated helpers compute the cold-path rest data in the precision
// of the device system (float for the FP32 and mixed paths, double for FP64).
#pragma once

#include <cmath>

namespace PhysiK {

struct Vec3 {
    float x = 0.0f;
    float y = 0.0f;
    float z = 0.0f;
    constexpr Vec3() = default;
    constexpr Vec3(float xv, float yv, float zv) : x(xv), y(yv), z(zv) {}
    constexpr Vec3 operator+(const Vec3& o) const { return Vec3{x + o.x, y + o.y, z + o.z}; }
    constexpr Vec3 operator-(const Vec3& o) const { return Vec3{x - o.x, y - o.y, z - o.z}; }
    constexpr Vec3 operator-() const { return Vec3{-x, -y, -z}; }
    constexpr Vec3 operator*(float s) const { return Vec3{x * s, y * s, z * s}; }
    constexpr Vec3 operator/(float s) const { return Vec3{x / s, y / s, z / s}; }
    Vec3& operator+=(const Vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    Vec3& operator-=(const Vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    Vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    float LengthSquared() const { return x * x + y * y + z * z; }
    float Length() const { return std::sqrt(LengthSquared()); }
};

constexpr Vec3 operator*(float s, const Vec3& v) { return v * s; }

// include/PhysiK/Math/Vec4.h: four floats (barycentric weights of a point connection).
struct Vec4 {
    float x = 0.0f;
    float y = 0.0f;
    float z = 0.0f;
    float w = 0.0f;
};
constexpr float Dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
constexpr Vec3 Cross(const Vec3& a, const Vec3& b)
{
    return Vec3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct Mat3 {
    Vec3 columns[3] = {Vec3{1.0f, 0.0f, 0.0f}, Vec3{0.0f, 1.0f, 0.0f}, Vec3{0.0f, 0.0f, 1.0f}};
    static Mat3 Identity() { return Mat3{}; }
    static Mat3 Zero() { return FromColumns(Vec3{}, Vec3{}, Vec3{}); }
    static Mat3 FromColumns(const Vec3& c0, const Vec3& c1, const Vec3& c2)
    {
        Mat3 m;
        m.columns[0] = c0;
        m.columns[1] = c1;
        m.columns[2] = c2;
        return m;
    }
    Vec3 operator*(const Vec3& v) const { return columns[0] * v.x + columns[1] * v.y + columns[2] * v.z; }
    Mat3 operator-(const Mat3& o) const
    {
        return FromColumns(columns[0] - o.columns[0], columns[1] - o.columns[1], columns[2] - o.columns[2]);
    }
};

inline Mat3 operator*(const Mat3& a, const Mat3& b)
{
    return Mat3::FromColumns(a * b.columns[0], a * b.columns[1], a * b.columns[2]);
}
inline Mat3 Transpose(const Mat3& m)
{
    return Mat3::FromColumns(Vec3{m.columns[0].x, m.columns[1].x, m.columns[2].x},
                             Vec3{m.columns[0].y, m.columns[1].y, m.columns[2].y},
                             Vec3{m.columns[0].z, m.columns[1].z, m.columns[2].z});
}
inline float Determinant(const Mat3& m) { return Dot(m.columns[0], Cross(m.columns[1], m.columns[2])); }
inline Mat3 Inverse(const Mat3& m)
{
    const Vec3 r0 = Cross(m.columns[1], m.columns[2]);
    const Vec3 r1 = Cross(m.columns[2], m.columns[0]);
    const Vec3 r2 = Cross(m.columns[0], m.columns[1]);
    const float d = Dot(m.columns[0], r0);
    if (std::abs(d) <= 0.000001f) return Mat3{};
    const float inv = 1.0f / d;
    return Transpose(Mat3::FromColumns(r0 * inv, r1 * inv, r2 * inv));
}

namespace detail {

// Generic 3-vector / column-major 3x3 in precision T, same operation order as above.
template <class T>
struct V {
    T x, y, z;
};
template <class T>
struct M {
    V<T> c[3];
};
template <class T>
inline V<T> sub(V<T> a, V<T> b) { return V<T>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
inline V<T> add(V<T> a, V<T> b) { return V<T>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
inline V<T> mulv(V<T> a, T s) { return V<T>{a.x * s, a.y * s, a.z * s}; }
template <class T>
inline T dot(V<T> a, V<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
inline V<T> cross(V<T> a, V<T> b)
{
    return V<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
inline T det(const M<T>& m) { return dot(m.c[0], cross(m.c[1], m.c[2])); }
template <class T>
inline M<T> transpose(const M<T>& m)
{
    return M<T>{{V<T>{m.c[0].x, m.c[1].x, m.c[2].x}, V<T>{m.c[0].y, m.c[1].y, m.c[2].y},
                 V<T>{m.c[0].z, m.c[1].z, m.c[2].z}}};
}
template <class T>
inline M<T> inverse(const M<T>& m)
{
    const V<T> r0 = cross(m.c[1], m.c[2]);
    const V<T> r1 = cross(m.c[2], m.c[0]);
    const V<T> r2 = cross(m.c[0], m.c[1]);
    const T d = dot(m.c[0], r0);
    if (std::abs(d) <= T(0.000001)) return M<T>{{V<T>{1, 0, 0}, V<T>{0, 1, 0}, V<T>{0, 0, 1}}};
    const T inv = T(1) / d;
    return transpose(M<T>{{mulv(r0, inv), mulv(r1, inv), mulv(r2, inv)}});
}

}  // namespace detail
}  // namespace PhysiK
