// ref_main_harness.cpp -- C entry points around the reference's own path loop (src/main.cpp).
//
// TEST INFRASTRUCTURE ONLY. oracle/build_ref.sh compiles this file, which includes the
// reference's src/main.cpp read in place, into every oracle/_ref/<variant>/libref.so next to
// the reference's BVH sources. Only tests/ and the CPU baseline leg of bench.py load that
// library, and only as the checker.
//
// main.cpp keeps its camera, sampling and path-tracing code in static functions of its own
// translation unit, so this file includes it (its main() renamed to ref_main, never called)
// to reach them: makeCameraQuat / makeCameraLookAt (main.cpp:43-66), primaryRay (69-83),
// IBL::sample (107-117), sampleCosineHemisphere / toWorld (123-141), pathTrace (145-204) and
// parseSceneConfig (218-285). The image libraries it includes are stand-ins (oracle/stubs).
//
// The reference renders every sample of the image from one std::mt19937(42) stream in a
// serial y -> x -> s loop (main.cpp:333-365). ref_path_render keeps its per-sample body --
// two jitter draws, primaryRay, pathTrace with the same generator -- but gives every pixel its
// own std::mt19937 (seeded from (seed, x, y) through std::seed_seq), so rows can run on
// several threads and the estimate of each pixel is independent of the others. It returns
// the per-pixel mean and mean of squares in double precision, for standard-error tests.

#define main ref_main
#include "main.cpp"
#undef main

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace
{

// cam13 = pos.xyz, fwd.xyz, right.xyz, up.xyz, tanHalfFovY
void camera_out(const Camera& c, float* cam13)
{
    const math::vec3* v[4] = { &c.pos, &c.fwd, &c.right, &c.up };
    for (int i = 0; i < 4; i++)
    {
        cam13[3 * i + 0] = v[i]->x;
        cam13[3 * i + 1] = v[i]->y;
        cam13[3 * i + 2] = v[i]->z;
    }
    cam13[12] = c.tanHalfFovY;
}

Camera camera_in(const float* cam13)
{
    Camera c;
    c.pos         = math::vec3(cam13[0], cam13[1], cam13[2]);
    c.fwd         = math::vec3(cam13[3], cam13[4], cam13[5]);
    c.right       = math::vec3(cam13[6], cam13[7], cam13[8]);
    c.up          = math::vec3(cam13[9], cam13[10], cam13[11]);
    c.tanHalfFovY = cam13[12];
    return c;
}

// An IBL whose pixels are a malloc'd copy of map (IBL's destructor frees them through the
// stand-in stbi_image_free).
void ibl_from(IBL& ibl, const float* map, int w, int h)
{
    if (!map || w <= 0 || h <= 0) { return; }
    const size_t n = (size_t)w * (size_t)h * 3;
    ibl.data = static_cast<float*>(std::malloc(n * sizeof(float)));
    std::memcpy(ibl.data, map, n * sizeof(float));
    ibl.w = w;
    ibl.h = h;
}

template <typename F> void parallel_rows(int row0, int nrows, int nthreads, F&& body)
{
    if (nthreads < 1) { nthreads = 1; }
    if (nthreads == 1 || nrows <= 1)
    {
        for (int y = row0; y < row0 + nrows; y++) { body(y); }
        return;
    }
    std::atomic<int> next{ row0 };
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++)
    {
        th.emplace_back([&] {
            for (int y = next++; y < row0 + nrows; y = next++) { body(y); }
        });
    }
    for (auto& x : th) { x.join(); }
}

} // namespace

extern "C" {

// parseSceneConfig (main.cpp:218-285): wh2 = width, height; cam13 as camera_out;
// ambient3 = the ambient line (unused by pathTrace); returns 1 if an ibl line named a map.
int ref_scene_config(const char* scn_path, int* wh2, float* cam13, float* ambient3)
{
    SceneConfig cfg = parseSceneConfig(scn_path);
    wh2[0] = cfg.width;
    wh2[1] = cfg.height;
    camera_out(cfg.camera, cam13);
    ambient3[0] = cfg.ambient.x;
    ambient3[1] = cfg.ambient.y;
    ambient3[2] = cfg.ambient.z;
    return cfg.iblPath.empty() ? 0 : 1;
}

// makeCameraLookAt (main.cpp:55-66) and makeCameraQuat (main.cpp:43-52, with the quaternion
// normalised as parseSceneConfig does at main.cpp:267-269).
void ref_camera_lookat(const float* pos3, const float* target3, float fov_deg, float* cam13)
{
    camera_out(makeCameraLookAt(math::vec3(pos3[0], pos3[1], pos3[2]), math::vec3(target3[0], target3[1], target3[2]),
                                fov_deg),
               cam13);
}
void ref_camera_quat(const float* pos3, const float* q_wxyz, float focal, float* cam13)
{
    camera_out(makeCameraQuat(math::vec3(pos3[0], pos3[1], pos3[2]),
                              math::normalize(math::quat(q_wxyz[0], q_wxyz[1], q_wxyz[2], q_wxyz[3])), focal),
               cam13);
}

// primaryRay (main.cpp:69-83) for n (pixel, jitter) pairs; rays8 = origin.xyz, tmin, dir.xyz, tmax.
void ref_primary_rays(const float* cam13, int W, int H, uint64_t n, const int* px, const int* py, const float* jx,
                      const float* jy, float* rays8)
{
    const Camera cam = camera_in(cam13);
    for (uint64_t i = 0; i < n; i++)
    {
        bvh::Ray r = primaryRay(cam, px[i], py[i], W, H, jx[i], jy[i]);
        float* o = rays8 + 8 * i;
        o[0] = r.origin.x; o[1] = r.origin.y; o[2] = r.origin.z; o[3] = r.tmin;
        o[4] = r.dir.x; o[5] = r.dir.y; o[6] = r.dir.z; o[7] = r.tmax;
    }
}

// toWorld(sampleCosineHemisphere(u1, u2), n) (main.cpp:123-141) for n samples.
void ref_cosine_dirs(uint64_t n, const float* u1, const float* u2, const float* nrm3, float* out3)
{
    for (uint64_t i = 0; i < n; i++)
    {
        math::vec3 w = toWorld(sampleCosineHemisphere(u1[i], u2[i]),
                               math::vec3(nrm3[3 * i], nrm3[3 * i + 1], nrm3[3 * i + 2]));
        out3[3 * i] = w.x; out3[3 * i + 1] = w.y; out3[3 * i + 2] = w.z;
    }
}

// IBL::sample (main.cpp:107-117) of an equirectangular map (h rows of w RGB texels).
void ref_ibl_lookup(const float* map, int w, int h, uint64_t n, const float* dirs3, float* out3)
{
    IBL ibl;
    ibl_from(ibl, map, w, h);
    for (uint64_t i = 0; i < n; i++)
    {
        math::vec3 c = ibl.sample(math::vec3(dirs3[3 * i], dirs3[3 * i + 1], dirs3[3 * i + 2]));
        out3[3 * i] = c.x; out3[3 * i + 1] = c.y; out3[3 * i + 2] = c.z;
    }
}

// The reference's pixel loop (main.cpp:339-365) over rows row0 .. row0+nrows-1 of a W x H image
// (row 0 at the bottom, as the reference's buffer before its flip), spp samples per pixel,
// pathTrace with maxBounce bounces over the BVH that ref_load loaded; the sky when map is
// NULL, else IBL::sample of the map. mean3 / meansq3 (nrows * W * 3, double): per-pixel mean
// of the samples and of their squares. Returns 0 if the camera or sizes are unusable.
int ref_path_render(const float* cam13, int W, int H, int spp, int max_bounce, uint32_t seed, const float* map,
                    int map_w, int map_h, int row0, int nrows, double* mean3, double* meansq3, int nthreads)
{
    if (W <= 0 || H <= 0 || spp <= 0 || row0 < 0 || nrows <= 0 || row0 + nrows > H) { return 0; }
    const Camera cam = camera_in(cam13);
    IBL ibl;
    ibl_from(ibl, map, map_w, map_h);
    const math::vec3 ambient(0.f, 0.f, 0.f);  // pathTrace takes it and never reads it
    parallel_rows(row0, nrows, nthreads, [&](int y) {
        for (int x = 0; x < W; x++)
        {
            std::seed_seq seq{ seed, (uint32_t)x, (uint32_t)y };
            std::mt19937 rng(seq);
            std::uniform_real_distribution<float> jitter(0.f, 1.f);
            double s[3] = { 0, 0, 0 }, s2[3] = { 0, 0, 0 };
            for (int k = 0; k < spp; k++)
            {
                // as main.cpp:353-355: both jitter draws, then pathTrace on the same generator
                bvh::Ray ray = primaryRay(cam, x, y, W, H, jitter(rng), jitter(rng));
                math::vec3 L = pathTrace(ray, ibl, ambient, rng, max_bounce);
                const double c[3] = { L.x, L.y, L.z };
                for (int i = 0; i < 3; i++) { s[i] += c[i]; s2[i] += c[i] * c[i]; }
            }
            const size_t o = ((size_t)(y - row0) * W + x) * 3;
            for (int i = 0; i < 3; i++)
            {
                mean3[o + i] = s[i] / spp;
                meansq3[o + i] = s2[i] / spp;
            }
        }
    });
    return 1;
}

} // extern "C"
