// ref_harness.cpp -- C entry points around the reference's own bake / load / trace code.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the reference's
// src/bvh/*.cpp sources, read in place (oracle/build_ref.sh), into
// oracle/_ref/<variant>/libref.so. Only tests/, the smoke check and the CPU
// baseline leg of bench.py load that library, and only as the checker.
//
// Geometry is injected bit-exactly by pre-filling bvh::s_vertices / s_triangles and
// baking a scene file with no geometry lines: readScene appends and never clears
// (src/bvh/bvh_IO.cpp:125-234), and initGeos then validates and renormalises
// (src/bvh/bvh_IO.cpp:72-121).

#define BAKING
#include "bvh.hpp"
#include "bvh_bake_state.hpp"
#include "bvh_morton.hpp"
#include "bvh_traverse.hpp"
#include "AABB.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

namespace bvh
{
bool readScene();
bool initGeos();
}

static void fill_geometry(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N)
{
    bvh::s_vertices.resize(V);
    for (uint32_t i = 0; i < V; i++)
    {
        Vertex& v = bvh::s_vertices[i];
        v.x  = verts6[6 * i + 0];
        v.y  = verts6[6 * i + 1];
        v.z  = verts6[6 * i + 2];
        v.nx = verts6[6 * i + 3];
        v.ny = verts6[6 * i + 4];
        v.nz = verts6[6 * i + 5];
    }
    bvh::s_triangles.resize(N);
    for (uint32_t i = 0; i < N; i++)
    {
        bvh::s_triangles[i].v[0] = tris3[3 * i + 0];
        bvh::s_triangles[i].v[1] = tris3[3 * i + 1];
        bvh::s_triangles[i].v[2] = tris3[3 * i + 2];
    }
}

static void clear_state()
{
    bvh::s_vertices.clear();
    bvh::s_triangles.clear();
    bvh::s_nodes.clear();
    bvh::s_mortonData.clear();
    bvh::s_queue.clear();
    bvh::s_sortedTris.clear();
    bvh::s_triIndex.clear();
    bvh::s_centroids.clear();
    bvh::s_triIndexSize   = 0;
    bvh::s_sortedTrisSize = 0;
    bvh::s_totalNodeCount = 0;
    bvh::s_sceneAABB      = AABB();
    bvh::s_scenePath.clear();
}

extern "C" {

// Compile-time constants of this variant (patched copies of src/bvh/bvh_defines.hpp).
void ref_constants(int* out6)
{
    out6[0] = BVH_LBVH_THRESHOLD;
    out6[1] = BVH_MAX_LEAF_SIZE;
    out6[2] = MORTON_UNIT_BIT_SIZE;
    out6[3] = BVH_SAH_BINS_MIN;
    out6[4] = BVH_SAH_BINS_MAX;
    out6[5] = (int)sizeof(BVHNode);
}

// Bake injected geometry: writes an empty scene file at scn_path; the reference then
// writes "<scn_path without extension>.bvh". Returns 1 on success.
int ref_bake_arrays(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N,
                    const char* scn_path)
{
    {
        std::ofstream f(scn_path);
        if (!f.is_open()) { return 0; }
        f << "# geometry injected by the oracle harness\n";
    }
    clear_state();
    fill_geometry(verts6, V, tris3, N);
    bool ok = bvh::bakeBVH(scn_path);
    clear_state();
    return ok ? 1 : 0;
}

// Bake a .scn file as the reference's main() does (src/main.cpp:308).
int ref_bake_scene(const char* scn_path)
{
    clear_state();
    bool ok = bvh::bakeBVH(scn_path);
    clear_state();
    return ok ? 1 : 0;
}

// Geometry that readScene (src/bvh/bvh_IO.cpp:125-234) produces for a .scn file, before
// initGeos. Call with null arrays to get counts2 = {vertices, triangles}, then again.
int ref_scene_geometry(const char* scn_path, float* verts6, uint32_t* tris3, uint32_t* counts2)
{
    clear_state();
    bvh::s_scenePath = scn_path;
    if (!bvh::readScene()) { clear_state(); return 0; }
    counts2[0] = (uint32_t)bvh::s_vertices.size();
    counts2[1] = (uint32_t)bvh::s_triangles.size();
    if (verts6)
    {
        for (size_t i = 0; i < bvh::s_vertices.size(); i++)
        {
            const Vertex& v = bvh::s_vertices[i];
            float* o = verts6 + 6 * i;
            o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.nx; o[4] = v.ny; o[5] = v.nz;
        }
    }
    if (tris3)
    {
        for (size_t i = 0; i < bvh::s_triangles.size(); i++)
        {
            for (int k = 0; k < 3; k++) { tris3[3 * i + k] = bvh::s_triangles[i].v[k]; }
        }
    }
    clear_state();
    return 1;
}

// Morton codes (original triangle order) and the stable radix-sorted permutation
// (src/bvh/bvh_morton.cpp:40-159). scene6 receives the scene AABB min.xyz, max.xyz.
int ref_morton(const float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N,
               uint64_t* codes, uint32_t* sorted, float* scene6)
{
    clear_state();
    fill_geometry(verts6, V, tris3, N);
    if (!bvh::sortTrisByMorton()) { clear_state(); return 0; }
    for (uint32_t i = 0; i < N; i++)
    {
        codes[i]  = bvh::s_mortonData[i].mortonCode;
        sorted[i] = bvh::s_sortedTris[i];
    }
    scene6[0] = bvh::s_sceneAABB.min.x; scene6[1] = bvh::s_sceneAABB.min.y; scene6[2] = bvh::s_sceneAABB.min.z;
    scene6[3] = bvh::s_sceneAABB.max.x; scene6[4] = bvh::s_sceneAABB.max.y; scene6[5] = bvh::s_sceneAABB.max.z;
    clear_state();
    return 1;
}

// Normal renormalisation of initGeos (src/bvh/bvh_IO.cpp:102-118) applied to V vertices in place.
int ref_init_geos(float* verts6, uint32_t V, const uint32_t* tris3, uint32_t N)
{
    clear_state();
    fill_geometry(verts6, V, tris3, N);
    bool ok = bvh::initGeos();
    if (ok)
    {
        for (uint32_t i = 0; i < V; i++)
        {
            verts6[6 * i + 3] = bvh::s_vertices[i].nx;
            verts6[6 * i + 4] = bvh::s_vertices[i].ny;
            verts6[6 * i + 5] = bvh::s_vertices[i].nz;
        }
    }
    clear_state();
    return ok ? 1 : 0;
}

int ref_load(const char* bvh_path)
{
    return bvh::loadBVH(bvh_path) ? 1 : 0;
}

// Trace n rays (o.xyz, tmin, d.xyz, tmax) through the loaded BVH with bvh::trace
// (src/bvh/bvh_traverse.cpp:237-246). trace is read-only after loadBVH, so the rays
// are split over nthreads std::threads. out6 = t, u, v, n.xyz.
void ref_trace(const float* rays8, uint64_t n, float* out6, uint32_t* tri, uint8_t* hit, int nthreads)
{
    if (nthreads < 1) { nthreads = 1; }
    auto work = [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++)
        {
            const float* r = rays8 + 8 * i;
            bvh::Ray ray;
            ray.origin = math::vec3(r[0], r[1], r[2]);
            ray.tmin   = r[3];
            ray.dir    = math::vec3(r[4], r[5], r[6]);
            ray.tmax   = r[7];
            bvh::Hit h = bvh::trace(ray);
            hit[i] = h.hit ? 1 : 0;
            tri[i] = h.triIndex;
            out6[6 * i + 0] = h.t;
            out6[6 * i + 1] = h.u;
            out6[6 * i + 2] = h.v;
            out6[6 * i + 3] = h.normal.x;
            out6[6 * i + 4] = h.normal.y;
            out6[6 * i + 5] = h.normal.z;
        }
    };
    if (nthreads == 1) { work(0, n); return; }
    std::vector<std::thread> th;
    uint64_t chunk = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++)
    {
        uint64_t b = t * chunk, e = b + chunk > n ? n : b + chunk;
        if (b >= e) { break; }
        th.emplace_back(work, b, e);
    }
    for (auto& x : th) { x.join(); }
}

// The transform loadMesh applies to an imported mesh (src/bvh/bvh_IO.cpp:24-70 with the matrix
// readScene builds at bvh_IO.cpp:221-224): positions by translate * scale * toMat4(q),
// normals by transpose(inverse(that)), in the reference's own math library. q_wxyz as the
// .scn line gives it after reordering (w, x, y, z). pos3 / nrm3: n points and normals;
// out6: transformed x, y, z, nx, ny, nz (normals not renormalised, as loadMesh leaves them).
void ref_mesh_transform(const float* t3, float scale, const float* q_wxyz, uint64_t n, const float* pos3,
                        const float* nrm3, float* out6)
{
    math::mat4 transform = math::translate(math::mat4(1.f), math::vec3(t3[0], t3[1], t3[2])) *
                           math::scale(math::mat4(1.f), math::vec3(scale)) *
                           math::toMat4(math::quat(q_wxyz[0], q_wxyz[1], q_wxyz[2], q_wxyz[3]));
    math::mat4 normalTransform = math::transpose(math::inverse(transform));
    for (uint64_t i = 0; i < n; i++)
    {
        math::vec4 tp = transform * math::vec4(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2], 1.0f);
        math::vec4 tn = normalTransform * math::vec4(nrm3[3 * i], nrm3[3 * i + 1], nrm3[3 * i + 2], 0.0f);
        float* o = out6 + 6 * i;
        o[0] = tp.x; o[1] = tp.y; o[2] = tp.z; o[3] = tn.x; o[4] = tn.y; o[5] = tn.z;
    }
}

// clipTriangleToAABB (src/bvh/AABB.cpp:86-171): v9 = three vertices, box6 = min, max.
// out6 = min, max of the clipped polygon (the empty box is +inf / -inf).
void ref_clip_triangle(const float* v9, const float* box6, float* out6)
{
    AABB box;
    box.min = math::vec3(box6[0], box6[1], box6[2]);
    box.max = math::vec3(box6[3], box6[4], box6[5]);
    AABB r = clipTriangleToAABB(math::vec3(v9[0], v9[1], v9[2]), math::vec3(v9[3], v9[4], v9[5]),
                                math::vec3(v9[6], v9[7], v9[8]), box);
    out6[0] = r.min.x; out6[1] = r.min.y; out6[2] = r.min.z;
    out6[3] = r.max.x; out6[4] = r.max.y; out6[5] = r.max.z;
}

} // extern "C"
