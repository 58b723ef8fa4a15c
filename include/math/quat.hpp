// quat.hpp -- rotation quaternion of the drop-in host API (the reference's math::quat,
// src/math/quat.hpp): constructed as quat(w, x, y, z); q * v rotates v by
// v + w t + q.xyz x t with t = 2 q.xyz x v.
#pragma once

#include "vec3.hpp"

namespace math
{

struct alignas(16) quat
{
    float x, y, z, w;
    quat() : x(0.f), y(0.f), z(0.f), w(1.f) {}
    quat(float w_, float x_, float y_, float z_) : x(x_), y(y_), z(z_), w(w_) {}
};

inline quat operator*(const quat& a, const quat& b)
{
    return quat(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w);
}

inline vec3 operator*(const quat& q, const vec3& v)
{
    const vec3 qv(q.x, q.y, q.z);
    const vec3 t = cross(qv, v) * 2.0f;
    return v + q.w * t + cross(qv, t);
}

inline quat normalize(const quat& q)
{
    const float inv = 1.0f / sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return quat(q.w * inv, q.x * inv, q.y * inv, q.z * inv);
}

} // namespace math
