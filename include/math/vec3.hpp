// vec3.hpp -- 3-vector of the drop-in host API (the reference's math::vec3, src/math/vec3.hpp):
// same members (x, y, z and a padding lane, 16-byte aligned so AABB and BVHNode keep the .bvh
// layout) and the same arithmetic: min/max keep the second operand unless the first is
// strictly smaller/larger, dot sums (x*x' + y*y') + (z*z' + w*w').
#pragma once

#include <cmath>

namespace math
{

struct alignas(16) vec3
{
    float x, y, z, _w;

    vec3() : x(0.f), y(0.f), z(0.f), _w(0.f) {}
    vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_), _w(0.f) {}
    vec3(float s) : x(s), y(s), z(s), _w(s) {}

    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : _w)); }
    float  operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : _w)); }

    vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; _w += o._w; return *this; }
    vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; _w -= o._w; return *this; }
    vec3& operator*=(float s) { x *= s; y *= s; z *= s; _w *= s; return *this; }
    vec3& operator/=(float s) { x /= s; y /= s; z /= s; _w /= s; return *this; }
};

inline vec3 lanes(float x, float y, float z, float w) { vec3 r(x, y, z); r._w = w; return r; }
inline vec3 operator+(vec3 a, vec3 b) { return lanes(a.x + b.x, a.y + b.y, a.z + b.z, a._w + b._w); }
inline vec3 operator-(vec3 a, vec3 b) { return lanes(a.x - b.x, a.y - b.y, a.z - b.z, a._w - b._w); }
inline vec3 operator*(vec3 a, vec3 b) { return lanes(a.x * b.x, a.y * b.y, a.z * b.z, a._w * b._w); }
inline vec3 operator/(vec3 a, vec3 b) { return lanes(a.x / b.x, a.y / b.y, a.z / b.z, a._w / b._w); }
inline vec3 operator*(vec3 a, float s) { return lanes(a.x * s, a.y * s, a.z * s, a._w * s); }
inline vec3 operator*(float s, vec3 a) { return lanes(s * a.x, s * a.y, s * a.z, s * a._w); }
inline vec3 operator/(vec3 a, float s) { return lanes(a.x / s, a.y / s, a.z / s, a._w / s); }
inline vec3 operator-(vec3 a) { return lanes(0.f - a.x, 0.f - a.y, 0.f - a.z, 0.f - a._w); }

inline float dot(vec3 a, vec3 b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + a._w * b._w); }
inline vec3 cross(vec3 a, vec3 b)
{
    return lanes(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, a._w * b._w - a._w * b._w);
}
inline float length(vec3 v) { return sqrtf(dot(v, v)); }
inline vec3 normalize(vec3 v)
{
    const float inv = 1.0f / sqrtf(dot(v, v));
    return v * inv;
}
inline vec3 min(vec3 a, vec3 b)
{
    return lanes(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z, a._w < b._w ? a._w : b._w);
}
inline vec3 max(vec3 a, vec3 b)
{
    return lanes(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z, a._w > b._w ? a._w : b._w);
}

} // namespace math
