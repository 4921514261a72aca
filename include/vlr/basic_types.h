/* Host math types of the VLR C++ surface (namespace vlr), as libvlr_b200
 * provides them: the value types vlrcpp.h and its callers exchange with the
 * C API (points, vectors, normals, texture coordinates, quaternions, 4x4
 * transforms, the 44-byte vertex) and the usual constructors of transforms.
 * They stand in for libVLR/include/vlr/basic_types.h, whose names and data
 * layouts they keep (Vertex basic_types.h:1496-1501 = VLRVertex; Matrix4x4
 * column-major as vlrStaticTransformCreate takes it); the renderer's own
 * device math lives in the library, not here. */
#pragma once

#include <cmath>
#include <cstdint>

#include "common.h"
#include "public_types.h"

namespace vlr {

struct Vector3D {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    constexpr Vector3D() = default;
    constexpr Vector3D(float vx, float vy, float vz) : x(vx), y(vy), z(vz) {}
    constexpr explicit Vector3D(float v) : x(v), y(v), z(v) {}
    constexpr Vector3D operator-() const { return Vector3D(-x, -y, -z); }
    constexpr Vector3D operator+(const Vector3D &o) const { return Vector3D(x + o.x, y + o.y, z + o.z); }
    constexpr Vector3D operator-(const Vector3D &o) const { return Vector3D(x - o.x, y - o.y, z - o.z); }
    constexpr Vector3D operator*(float s) const { return Vector3D(x * s, y * s, z * s); }
    constexpr Vector3D operator/(float s) const { return Vector3D(x / s, y / s, z / s); }
    float length() const { return std::sqrt(x * x + y * y + z * z); }
    Vector3D normalize() const { return *this / length(); }
};

struct Point3D {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    constexpr Point3D() = default;
    constexpr Point3D(float px, float py, float pz) : x(px), y(py), z(pz) {}
    constexpr explicit Point3D(float v) : x(v), y(v), z(v) {}
    constexpr explicit Point3D(const Vector3D &v) : x(v.x), y(v.y), z(v.z) {}
    constexpr Point3D operator+(const Vector3D &v) const { return Point3D(x + v.x, y + v.y, z + v.z); }
    constexpr Vector3D operator-(const Point3D &o) const { return Vector3D(x - o.x, y - o.y, z - o.z); }
    static constexpr Point3D Zero() { return Point3D(0.0f, 0.0f, 0.0f); }
};

struct Normal3D {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    constexpr Normal3D() = default;
    constexpr Normal3D(float nx, float ny, float nz) : x(nx), y(ny), z(nz) {}
    constexpr explicit Normal3D(const Vector3D &v) : x(v.x), y(v.y), z(v.z) {}
    constexpr Normal3D operator-() const { return Normal3D(-x, -y, -z); }
    float length() const { return std::sqrt(x * x + y * y + z * z); }
    Normal3D normalize() const { const float l = length(); return Normal3D(x / l, y / l, z / l); }
};

inline constexpr Vector3D operator*(float s, const Vector3D &v) { return v * s; }
inline constexpr float dot(const Vector3D &a, const Vector3D &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline constexpr Vector3D cross(const Vector3D &a, const Vector3D &b) {
    return Vector3D(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline Vector3D normalize(const Vector3D &v) { return v.normalize(); }
inline Normal3D normalize(const Normal3D &n) { return n.normalize(); }

struct TexCoord2D {
    float u = 0.0f, v = 0.0f;
    constexpr TexCoord2D() = default;
    constexpr TexCoord2D(float tu, float tv) : u(tu), v(tv) {}
    static constexpr TexCoord2D Zero() { return TexCoord2D(0.0f, 0.0f); }
};

// Rotation quaternion (x, y, z, w), w the real part.
struct Quaternion {
    float x = 0.0f, y = 0.0f, z = 0.0f, w = 1.0f;
    constexpr Quaternion() = default;
    constexpr Quaternion(float qx, float qy, float qz, float qw) : x(qx), y(qy), z(qz), w(qw) {}
    static constexpr Quaternion Identity() { return Quaternion(0.0f, 0.0f, 0.0f, 1.0f); }
    constexpr Quaternion operator*(const Quaternion &q) const {
        return Quaternion(w * q.x + x * q.w + y * q.z - z * q.y, w * q.y - x * q.z + y * q.w + z * q.x,
                          w * q.z + x * q.y - y * q.x + z * q.w, w * q.w - x * q.x - y * q.y - z * q.z);
    }
};

// Rotation by `angle` radians about `axis`.
inline Quaternion qRotate(float angle, const Vector3D &axis) {
    const Vector3D a = axis.normalize();
    const float s = std::sin(0.5f * angle);
    return Quaternion(a.x * s, a.y * s, a.z * s, std::cos(0.5f * angle));
}
inline Quaternion qRotate(float angle, float ax, float ay, float az) { return qRotate(angle, Vector3D(ax, ay, az)); }
inline Quaternion qRotateX(float angle) { return qRotate(angle, Vector3D(1, 0, 0)); }
inline Quaternion qRotateY(float angle) { return qRotate(angle, Vector3D(0, 1, 0)); }
inline Quaternion qRotateZ(float angle) { return qRotate(angle, Vector3D(0, 0, 1)); }

// 4x4 transform, stored column-major (m[4 * column + row]), the order of
// vlrStaticTransformCreate's array.
struct Matrix4x4 {
    float m[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
    constexpr Matrix4x4() = default;
    explicit Matrix4x4(const float array[16]) { for (int i = 0; i < 16; ++i) m[i] = array[i]; }
    static Matrix4x4 Identity() { return Matrix4x4(); }
    float &operator()(int row, int column) { return m[4 * column + row]; }
    float operator()(int row, int column) const { return m[4 * column + row]; }
    void getArray(float array[16]) const { for (int i = 0; i < 16; ++i) array[i] = m[i]; }
    Matrix4x4 operator*(const Matrix4x4 &b) const {
        Matrix4x4 r;
        for (int row = 0; row < 4; ++row)
            for (int col = 0; col < 4; ++col) {
                float s = 0.0f;
                for (int k = 0; k < 4; ++k) s += (*this)(row, k) * b(k, col);
                r(row, col) = s;
            }
        return r;
    }
    Point3D operator*(const Point3D &p) const {
        return Point3D((*this)(0, 0) * p.x + (*this)(0, 1) * p.y + (*this)(0, 2) * p.z + (*this)(0, 3),
                       (*this)(1, 0) * p.x + (*this)(1, 1) * p.y + (*this)(1, 2) * p.z + (*this)(1, 3),
                       (*this)(2, 0) * p.x + (*this)(2, 1) * p.y + (*this)(2, 2) * p.z + (*this)(2, 3));
    }
};

inline Matrix4x4 scale(float sx, float sy, float sz) {
    Matrix4x4 r;
    r(0, 0) = sx; r(1, 1) = sy; r(2, 2) = sz;
    return r;
}
inline Matrix4x4 scale(const Vector3D &s) { return scale(s.x, s.y, s.z); }
inline Matrix4x4 scale(float s) { return scale(s, s, s); }
inline Matrix4x4 translate(float tx, float ty, float tz) {
    Matrix4x4 r;
    r(0, 3) = tx; r(1, 3) = ty; r(2, 3) = tz;
    return r;
}
inline Matrix4x4 translate(const Vector3D &t) { return translate(t.x, t.y, t.z); }
// Rotation by `angle` radians about `axis` (right-handed).
inline Matrix4x4 rotate(float angle, const Vector3D &axis) {
    const Vector3D a = axis.normalize();
    const float c = std::cos(angle), s = std::sin(angle), t = 1.0f - c;
    Matrix4x4 r;
    r(0, 0) = t * a.x * a.x + c;       r(0, 1) = t * a.x * a.y - s * a.z; r(0, 2) = t * a.x * a.z + s * a.y;
    r(1, 0) = t * a.x * a.y + s * a.z; r(1, 1) = t * a.y * a.y + c;       r(1, 2) = t * a.y * a.z - s * a.x;
    r(2, 0) = t * a.x * a.z - s * a.y; r(2, 1) = t * a.y * a.z + s * a.x; r(2, 2) = t * a.z * a.z + c;
    return r;
}
inline Matrix4x4 rotate(float angle, float ax, float ay, float az) { return rotate(angle, Vector3D(ax, ay, az)); }
inline Matrix4x4 rotateX(float angle) { return rotate(angle, Vector3D(1, 0, 0)); }
inline Matrix4x4 rotateY(float angle) { return rotate(angle, Vector3D(0, 1, 0)); }
inline Matrix4x4 rotateZ(float angle) { return rotate(angle, Vector3D(0, 0, 1)); }

// The vertex of a triangle mesh or point node, laid out as VLRVertex.
struct Vertex {
    Point3D position;
    Normal3D normal;
    Vector3D tc0Direction;
    TexCoord2D texCoord;
};
static_assert(sizeof(Vertex) == sizeof(VLRVertex), "vlr::Vertex must match VLRVertex");

} // namespace vlr
