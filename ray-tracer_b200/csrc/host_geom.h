// host_geom.h -- host-side scene ingestion: the reference's .scn geometry grammar
// (src/bvh/bvh_IO.cpp:125-234), its sphere and box generators (src/bvh/bvh_geo.cpp), a PLY
// mesh loader standing in for the un-vendored importer, and the camera bases of
// src/main.cpp:43-66. Float expressions keep the reference's operand order; this file is
// compiled without FMA contraction so the generated vertices are bit-identical.
#pragma once

#include <cmath>
#include <string>
#include <vector>

#include "../../include/rt_b200.h"

namespace hg
{

struct V3
{
    float x, y, z;
    V3() : x(0.f), y(0.f), z(0.f) {}
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
};
inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return V3(s * a.x, s * a.y, s * a.z); }
// the reference's dot: (x*x' + y*y') + (z*z' + w*w') with the padding lane w = 0
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + 0.0f); }
inline V3 cross(V3 a, V3 b) { return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V3 normalize(V3 v)
{
    const float inv = 1.0f / sqrtf(dot(v, v));
    return v * inv;
}

struct Q
{
    float x, y, z, w;
    Q() : x(0.f), y(0.f), z(0.f), w(1.f) {}
    Q(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};
// v' = v + w t + q.xyz x t with t = 2 q.xyz x v (src/math/quat.hpp:36-42)
inline V3 rotate(Q q, V3 v)
{
    const V3 qv(q.x, q.y, q.z);
    const V3 t = cross(qv, v) * 2.0f;
    return v + q.w * t + cross(qv, t);
}
inline Q quat_normalize(Q q)
{
    const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    const float inv = 1.0f / len;
    return Q(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
}

struct Camera
{
    V3 pos, fwd, right, up;
    float tan_half_fov_y;
};
Camera camera_lookat(V3 pos, V3 target, float fov_deg);
Camera camera_quat(V3 pos, Q orient, float focal);
void store_camera(const Camera& c, rt_render_cfg* cfg);

void add_sphere(std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, V3 center, float radius, int rings, int sectors);
void add_box(std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, V3 center, V3 he, Q orient);
// Appends the geometry of a .scn file; returns RT_OK or an rt_status with `err` set.
int read_scene(const std::string& path, std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, std::string& err);
// Loads a PLY mesh (ASCII or binary little-endian), fan-triangulating polygons and
// generating area-weighted smooth normals when the file has none, transformed by
// translate * scale * rotate as the reference's mesh line does (bvh_IO.cpp:221-224).
int load_ply(const std::string& path, V3 translate, float scale, Q orient, std::vector<rt_vertex>& v,
             std::vector<rt_triangle>& t, std::string& err);
std::string replace_extension(const std::string& path, const std::string& ext);

// Radiance RGBE (.hdr) images, RGB float in memory, rows in file order (top row first).
int write_hdr(const std::string& path, const float* rgb, uint32_t w, uint32_t h, std::string& err);
int read_hdr(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err);

// The non-geometry lines of a .scn file (parseSceneConfig, src/main.cpp:207-285): screen,
// camera (lookat or focal + quaternion), ambient, ibl. Defaults: 800 x 600, the look-at camera
// from (0, 1, -5) to the origin with 60 degrees.
struct SceneConfig
{
    int         width = 800, height = 600;
    Camera      camera;
    bool        has_camera = false;
    float       ambient[3] = { 0.1f, 0.1f, 0.1f };
    std::string ibl_path;
};
SceneConfig parse_scene_config(const std::string& path);

} // namespace hg
