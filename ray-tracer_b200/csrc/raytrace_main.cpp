// raytrace -- the reference's command line renderer (src/main.cpp:297-386) over librt_b200:
//   raytrace [scene.scn] [spp] [--wavefront] [--seed N]
// bakes the .scn into <scene>.bvh (bvh::bakeBVH), loads it back (bvh::loadBVH), renders the
// screen size and camera of the .scn with the reference's shading (albedo 0.8, sky or the
// ibl map, 8 bounces, roulette after bounce 2) on the GPU and writes <scene>.hdr (rows flipped
// so the file is top-down, as the reference writes it). The reference draws its samples from
// one std::mt19937(42) stream in pixel order; here every pixel has its own counter-based
// stream (Philox keyed by the seed), so images agree in distribution, not sample for sample.
#include "../../include/rt_b200.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static std::string replace_extension(const std::string& path, const std::string& ext)
{
    const auto dot = path.rfind('.');
    return (dot != std::string::npos ? path.substr(0, dot) : path) + ext;
}

int main(int argc, char** argv)
{
    std::string scene = "testscene.scn";
    int spp = 4;
    int mode = RT_RENDER_PLAIN;
    uint32_t seed = 42;
    int positional = 0;
    for (int i = 1; i < argc; i++)
    {
        const std::string a = argv[i];
        if (a == "--wavefront") { mode = RT_RENDER_WAVEFRONT; }
        else if (a == "--seed" && i + 1 < argc) { seed = (uint32_t)std::strtoul(argv[++i], nullptr, 10); }
        else if (positional == 0) { scene = a; positional++; }
        else if (positional == 1) { spp = std::atoi(a.c_str()); positional++; }
    }
    if (spp < 1) { std::fprintf(stderr, "Error: spp must be positive\n"); return 1; }
    const std::string bvh_path = replace_extension(scene, ".bvh");
    const std::string hdr_path = replace_extension(scene, ".hdr");

    rt_render_cfg cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    char ibl[4096] = { 0 };
    if (rt_scene_config(scene.c_str(), &cfg, ibl, sizeof(ibl)) != RT_OK)
    {
        std::fprintf(stderr, "Error: %s\n", rt_last_error());
        return 1;
    }
    std::fprintf(stdout, "Baking BVH from %s...\n", scene.c_str());
    if (rt_bake_scene(scene.c_str(), bvh_path.c_str(), nullptr) != RT_OK)
    {
        std::fprintf(stderr, "Error : %s\nError: bakeBVH failed\n", rt_last_error());
        return 1;
    }
    rt_bvh* bvh = nullptr;
    if (rt_load_bvh(bvh_path.c_str(), &bvh) != RT_OK)
    {
        std::fprintf(stderr, "Error : %s\nError: loadBVH failed\n", rt_last_error());
        return 1;
    }

    rt_shading sh;
    std::memset(&sh, 0, sizeof(sh));
    float* d_env = nullptr;
    cfg.env_kind = 0;
    if (ibl[0])
    {
        uint32_t w = 0, h = 0;
        if (rt_read_hdr(ibl, nullptr, &w, &h) != RT_OK)
        {
            std::fprintf(stderr, "Warning: failed to load IBL %s\n", ibl);
        }
        else
        {
            std::vector<float> map((size_t)w * h * 3);
            if (rt_read_hdr(ibl, map.data(), &w, &h) == RT_OK &&
                cudaMalloc(&d_env, map.size() * 4) == cudaSuccess &&
                cudaMemcpy(d_env, map.data(), map.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess)
            {
                sh.env_map = d_env; sh.env_w = w; sh.env_h = h;
                cfg.env_kind = 2;
            }
            else { std::fprintf(stderr, "Warning: failed to load IBL %s\n", ibl); }
        }
    }
    cfg.spp = (uint32_t)spp;
    cfg.max_bounce = 8;
    cfg.rr_after = 2;
    cfg.seed = seed;
    cfg.sample_offset = 0;
    std::fprintf(stdout, "Rendering %ux%u @ %d spp...\n", cfg.width, cfg.height, spp);
    std::vector<float> image((size_t)cfg.width * cfg.height * 3);
    int rc = rt_render_host(bvh, &cfg, &sh, mode, image.data());
    if (rc == RT_OK) { rc = rt_write_hdr(hdr_path.c_str(), image.data(), cfg.width, cfg.height, 1); }
    if (d_env) { cudaFree(d_env); }
    rt_bvh_free(bvh);
    if (rc != RT_OK)
    {
        std::fprintf(stderr, "Error: %s\n", rt_last_error());
        return 1;
    }
    std::fprintf(stdout, "Written: %s\n", hdr_path.c_str());
    return 0;
}
