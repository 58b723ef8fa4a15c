#!/usr/bin/env python3
"""BVH build + traversal microbenchmark on B200 GPUs.

Workload (one "step"): a full bake of the seeded 1,048,576-triangle soup (centroids uniform in
[0,1]^3, vertices at centroid + L*u with L log-uniform in [1e-4, 1e-2]) with the reference's
LBVH semantics (pure Morton split, 63-bit codes, leaf 16), producing the .bvh-layout tree and
the traversal layout, from inputs already resident in HBM. Metric: BVH build throughput in
Mtri/s over all ranks (weak scaling: every rank bakes its own soup; no data-path collective).

Also reported: the same build end to end through the C ABI with host buffers (e2e), the other
build presets, closest-hit / any-hit traversal of 16,777,216 incoherent rays and of 1920x1080
pinhole rays (Mray/s), the roofline of the bake (all its launches as one unit), the
reference's own CPU bake timed on this host, and under "render" the path-loop workloads:
plain path tracing (256x256, 16 spp, depth 4, Cornell box + 20,480-triangle icosphere + two
spheres; plain vs wavefront, and the CPU restatement on all host cores), the batched workload
(64 scenes of 1,000-500,000 triangles built in one launch sequence and rendered at 512x512,
4 spp, depth 5 by the graph-replayed wavefront vs the plain kernel per scene), the adjoint
(512x512, 32 spp, depth 4, Cornell box + 50,000-triangle icosphere: adjoint / forward time)
and the large render (1920x1080, 64 spp, depth 8, roulette after bounce 2, 5,000,000
triangles, binned SAH with spatial splits).

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       torchrun --nproc-per-node N bench.py --gpus N ...   (one process per GPU)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "ray-tracer_b200"))

N_TRIS = 1 << 20
N_RAYS = 1 << 24
METRIC = "BVH Mtri/s"
WORKLOAD = "BVH build microbenchmark: 1,048,576-triangle soup, LBVH 63-bit Morton codes, leaf 16"
# Algorithmic bytes per triangle of a minimal LBVH bake, the roofline's numerator: read the
# triangles and positions once for the Morton codes (12 + 36 in, 8 + 4 out = 60), eight onesweep
# passes over (key, index) pairs plus their histograms (8 x 24 + 8 = 200), the radix-tree
# topology (8 key + 12 links = 20) and the box refit (48 triangle + 2 x 24 child + 24 out = 120):
# 400 for 63-bit codes; with 30-bit codes the Morton step writes 4-byte keys (56) and the sort
# takes four passes over 16-byte pairs (68), with a 16-byte topology: 260.
ROOFLINE_BYTES_PER_TRI = {21: 400, 10: 260}
# What this library's bake moves per triangle by its own count (each array once per read and
# once per write, per kernel; V = 3N vertices): clear 12, vertex renormalisation 144, triangle
# prep 132 (boxes, centroids and the 48-byte triangle records), Morton codes 20, Karras
# topology with leaf boxes, box-hierarchy level 0 and the baked triangles 198, box levels 1,
# boundary 80, slot scan 8 (without SAH subtrees the triangle offsets are the identity), .bvh
# and traversal nodes 45; plus the sort: 44 up to 2^21 keys (top-digit onesweep pass 20 +
# per-bucket pass 24, which also writes the bucket table), else 188 (eight onesweep passes) and
# the bucket-table kernel's 8. It includes the outputs the minimal count leaves out
# (renormalised normals, the .bvh layout, the traversal layout).
BAKE_BYTES_PER_TRI_EXCL_SORT = 12 + 144 + 132 + 20 + 198 + 1 + 80 + 8 + 45


def bake_bytes_per_tri(n: int) -> int:
    return BAKE_BYTES_PER_TRI_EXCL_SORT + (44 if n <= (1 << 21) else 188 + 8)


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n-tris", type=int, default=N_TRIS)
    p.add_argument("--preset", default="lbvh63")
    p.add_argument("--no-extra", action="store_true", help="skip the secondary measurements")
    p.add_argument("--no-render", action="store_true", help="skip the path-loop workloads")
    p.add_argument("--kernels-only", action="store_true",
                   help="time the device bake alone: no end-to-end or CPU legs (for profiling runs)")
    p.add_argument("--only", choices=["trace", "sah5m", "c1", "c3", "c4", "c5"],
                   help="run one secondary workload alone and print its figures (for profiling runs)")
    p.add_argument("--n-rays", type=int, default=N_RAYS, help="incoherent rays of the traversal measurements")
    p.add_argument("--trace-preset", default="lbvh63,hybrid,sah4",
                   help="trees of the traversal measurements (comma-separated presets)")
    return p.parse_args()


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per triangle of one 1M-triangle LBVH bake (all its launches) from the
    committed ncu summary, if present."""
    path = os.path.join(HERE, "profiles", "lbvh_bake_soup1m_traffic.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_tri_per_bake"):
                return float(line.split("=")[1])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------------------------
class quiet_stdout:
    """Sends file descriptor 1 to /dev/null (the reference prints progress lines from C)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        nul = os.open(os.devnull, os.O_WRONLY)
        os.dup2(nul, 1)
        os.close(nul)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def _reference_bake_fn(n_tris: int, seed: int):
    """The reference's own bvh::bakeBVH (oracle/_ref/lbvh63, single-threaded as shipped) on a
    soup sample, ready to call; the C restatement when the reference build is absent."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle as orc
    from rtb200 import scenes
    v, t = scenes.soup(n_tris, seed=seed)
    if orc.Reference.available("lbvh63"):
        ref = orc.Reference("lbvh63")
        return (lambda: ref.bake(v, t)), "reference"
    R = orc.Restatement()
    cfg = orc.make_cfg(**orc.VARIANTS["lbvh63"])
    return (lambda: R.build(v, t, cfg)), "port"


def cpu_reference_bake(n_tris: int, seed: int, reps: int):
    """Rate of the reference's bake on one host core (after one untimed bake)."""
    fn, kind = _reference_bake_fn(n_tris, seed)
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    dt = (time.perf_counter() - t0) / reps
    return n_tris / dt / 1e6, kind, dt


def _ref_process(n, seed, warmup, steps, barrier, queue):
    """One host core's share of the reference arm: set up (soup, library), `warmup` untimed
    bakes, wait for every process to be ready, then time `steps` bakes."""
    with quiet_stdout():
        fn, kind = _reference_bake_fn(n, seed)
        for _ in range(warmup):
            fn()
        barrier.wait(timeout=1800)
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        queue.put((time.perf_counter() - t0, kind))


def run_reference(a):
    """The reference's own bake (bvh::bakeBVH with its LBVH constants, compiled from its sources
    into oracle/_ref/lbvh63) of the same 1,048,576-triangle soup as this arm's N=1 line, on every
    host core: one process per core, since the bake keeps its state in process globals and is
    single-threaded. One step = one bake in every process at once; the wall time of the steps is
    the slowest process's."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import multiprocessing as mp
    from rtb200 import scenes
    cores = os.cpu_count() or 1
    n = a.n_tris
    ctx = mp.get_context("spawn")
    barrier, queue = ctx.Barrier(cores), ctx.Queue()
    procs = [ctx.Process(target=_ref_process, args=(n, scenes.BASE_SEED + 1, a.warmup, a.steps, barrier, queue))
             for _ in range(cores)]
    for p_ in procs:
        p_.start()
    res = [queue.get(timeout=3600) for _ in procs]
    for p_ in procs:
        p_.join()
    wall = max(r[0] for r in res)
    kind = res[0][1]
    value = n * a.steps * cores / wall / 1e6
    out = {"metric": METRIC, "value": round(value, 4), "unit": "Mtri/s", "impl": "reference", "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(wall / a.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded soup)",
           "config": {"workload": WORKLOAD, "n_tris": n, "same_config": True,
                      "preset": "lbvh63 (reference constants patched: BVH_LBVH_THRESHOLD=0)", "processes": cores,
                      "bakes_timed": a.steps * cores,
                      "step": f"one bake of the {n:,}-triangle soup in each of {cores} processes at once"},
           "cpu_baseline": {"value": round(value, 4), "unit": "Mtri/s", "cores": cores, "kind": kind,
                            "sample": f"{cores} processes, each timing {a.steps} bake(s) of the {n:,}-triangle soup "
                                      f"after {a.warmup} untimed one(s) (the reference bake is single-threaded); "
                                      f"wall = the slowest process"},
           "e2e": {"value": round(value, 4), "unit": "Mtri/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------------------------
def run_ours(a):
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    from rtb200.dist import max_over_ranks

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    n = a.n_tris
    if a.only:
        return run_only(a, stream, dev)
    verts, tris = scenes.soup(n, seed=scenes.BASE_SEED + 1 + rank)
    dv = torch.from_numpy(verts).to(dev)
    dt = torch.from_numpy(tris.view(np.int32)).to(dev)
    cfg = rtb200.make_cfg(a.preset)
    bvh = rtb200.Bvh.build(dv, dt, cfg, stream=stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MiB > 126 MB L2
    for _ in range(max(a.warmup, 3)):
        bvh.rebuild(dv, dt, cfg, stream=stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    l0 = rtb200.kernel_launches()
    evs = []
    for _ in range(a.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bvh.rebuild(dv, dt, cfg, stream=stream)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches = rtb200.kernel_launches() - l0
    clocks = clk.stop()
    total_ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in evs), dist, dev)
    ms_step = total_ms / a.steps
    value = world * n / (ms_step * 1e-3) / 1e6
    # stage split from three more bakes with the stage events on (outside the timed region: the
    # event records add host work between the launches)
    bvh.profile(True)
    stages = []
    for _ in range(3):
        flush.zero_()
        bvh.rebuild(dv, dt, cfg, stream=stream)
        stages.append(bvh.stage_ms())
    bvh.profile(False)
    st = {k: statistics.mean(s[k] for s in stages) for k in stages[0]}
    nn, nt, _ = bvh.counts()

    # roofline of the bake as one unit (no single kernel dominates it: the largest takes about
    # 15 % of the step): algorithmic bytes per bake over the device time per bake
    alg_bytes = ROOFLINE_BYTES_PER_TRI.get(int(cfg.morton_bits), 400) * n
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    own_bytes = bake_bytes_per_tri(n) * n
    peak, peak_kind = measured_peak_hbm()
    traffic_per_tri = profiled_traffic() if n == N_TRIS and a.preset == "lbvh63" else None

    # end to end through the C ABI with host buffers: every step uploads its geometry from pinned
    # host memory (rt_rebuild with RT_HOST), bakes it and downloads the baked .bvh arrays into
    # pinned host memory. Three host threads drive three handles on three streams (the library's
    # handles are independent; a bake call returns once its bake has finished), so that one
    # step's upload, another's bake and a third's download (rt_bvh_download_async) overlap; the
    # timed region ends after the last download has landed.
    e2e_value = None
    if not a.kernels_only:
        e2e_value = end_to_end(a, bvh, dv, dt, verts, tris, cfg, nn, nt, dev, dist)
    h2d = verts.nbytes + tris.nbytes
    d2h = nn * 48 + nt * 12 + verts.nbytes

    extra = {}
    if not a.no_extra:
        extra = secondary(a, bvh, dv, dt, verts, stream, dev, flush)
    render = {}
    if not a.no_render and rank == 0:
        render = render_workloads(stream, dev)
    out = None
    if rank == 0:
        cpu_v, cpu_kind = None, None
        if not a.kernels_only:
            with quiet_stdout():
                cpu_v, cpu_kind, cpu_dt = cpu_reference_bake(n, scenes.BASE_SEED + 1, 3)
        out = {"metric": METRIC, "value": round(value, 3), "unit": "Mtri/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded soup, per-rank seed)",
               "config": {"workload": WORKLOAD, "n_tris": n, "preset": a.preset, "nodes": nn, "baked_tris": nt,
                          "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
               "e2e": ({"value": round(e2e_value, 3), "unit": "Mtri/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)} if e2e_value is not None else None),
               "gpu_launches": int(launches),
               "stage_ms": {k: round(v, 4) for k, v in st.items()},
               "roofline": {"bound": "hbm", "kernel": f"LBVH bake, all {launches // a.steps} launches of one rebuild",
                            "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                            "frac": round(achieved / peak, 4),
                            "traffic": (round(traffic_per_tri * n) if traffic_per_tri else None),
                            "algorithmic_bytes_per_launch": int(alg_bytes), "launch_ms": round(ms_step, 5),
                            "builder_bytes_per_launch": int(own_bytes),
                            "builder_frac": round(own_bytes / (ms_step * 1e-3) / 1e9 / peak, 4)},
               "cpu_baseline": None if cpu_v is None else {"value": round(cpu_v, 4), "unit": "Mtri/s", "cores": 1, "kind": cpu_kind,
                                "sample": f"bvh::bakeBVH of the same {n:,}-triangle soup, LBVH constants, 3 timed "
                                          f"repetitions after one untimed, 1 thread (the bake is single-threaded)"},
               "clocks": clocks, "extra": extra, "render": render}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def end_to_end(a, bvh, dv, dt, verts, tris, cfg, nn, nt, dev, dist):
    """The same bake end to end through the C ABI with host buffers (Mtri/s over all ranks)."""
    import numpy as np
    import torch
    import rtb200
    from rtb200.dist import max_over_ranks
    rank, world, _ = env_rank()
    n = dt.shape[0]
    import ctypes as C
    import threading
    hv = torch.from_numpy(verts).pin_memory()
    ht = torch.from_numpy(tris.view(np.int32)).pin_memory()
    L = rtb200.lib()
    depth = 3  # 2 and 4 measured lower
    handles = [bvh] + [rtb200.Bvh.build(dv, dt, cfg) for _ in range(depth - 1)]
    streams = [torch.cuda.Stream(device=dev) for _ in range(depth)]
    outs = [(torch.empty(nn * 48, dtype=torch.uint8).pin_memory(), torch.empty(nt * 12, dtype=torch.uint8).pin_memory(),
             torch.empty(verts.nbytes, dtype=torch.uint8).pin_memory()) for _ in range(depth)]
    hv_np, ht_np = hv.numpy(), ht.numpy().view(np.uint32)

    def e2e_step(j):
        b, s_, (hn, htr, hvo) = handles[j], streams[j], outs[j]
        b.rebuild(hv_np, ht_np, cfg, stream=s_)
        rtb200.api._check(L.rt_bvh_download_async(b.h, C.c_void_p(hn.data_ptr()), C.c_void_p(htr.data_ptr()),
                                                  C.c_void_p(hvo.data_ptr()), C.c_void_p(s_.cuda_stream)))

    def run_e2e(total):
        errs = []

        def worker(j):
            try:
                torch.cuda.set_device(dev)
                for _ in range(j, total, depth):
                    e2e_step(j)
            except Exception as e:  # re-raised on the main thread
                errs.append(e)
        th = [threading.Thread(target=worker, args=(j,)) for j in range(depth)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        torch.cuda.synchronize()
        if errs:
            raise errs[0]
    run_e2e(2 * depth)  # two warm-up bakes per handle: the second captures its launch graph
    k_e2e = max(4 * depth, a.steps)
    t0 = time.perf_counter()
    run_e2e(k_e2e)
    e2e_wall = time.perf_counter() - t0
    for j in range(depth):  # the pipelined copies hold each handle's bake
        assert np.array_equal(outs[j][0].numpy(), handles[j].download()[0].view(np.uint8)), "e2e download mismatch"
    e2e_s = max_over_ranks(e2e_wall / k_e2e, dist, dev)
    return world * n / e2e_s / 1e6


def run_only(a, stream, dev):
    """One secondary workload alone (the command the committed ncu summaries were made with)."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    if a.only in RENDER_WORKLOADS:
        out = render_workloads(stream, dev, a.only)
    elif a.only == "sah5m":
        lsc = scenes.large_scene()
        dvl = torch.from_numpy(lsc.verts).to(dev)
        dtl = torch.from_numpy(lsc.tris.view(np.int32)).to(dev)
        bl = rtb200.Bvh.build(dvl, dtl, "sah4", stream=stream)
        ms = _ev_ms(lambda: bl.rebuild(dvl, dtl, "sah4", stream=stream), stream, 1)
        out = {"sah5m": {"workload": "binned SAH + spatial splits, leaf 4, of the large-render scene (5,000,010 "
                                     "triangles)", "build_ms": round(ms, 1),
                         "build_mtri_s": round(lsc.tris.shape[0] / ms / 1e3, 3)}}
    else:
        verts, tris = scenes.soup(a.n_tris, seed=scenes.BASE_SEED + 1)
        dv = torch.from_numpy(verts).to(dev)
        dt = torch.from_numpy(tris.view(np.int32)).to(dev)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        out = {"trace": secondary(a, None, dv, dt, verts, stream, dev, flush, builds=False)}
    print(json.dumps(out), flush=True)
    return 0


def secondary(a, bvh, dv, dt, verts, stream, dev, flush, builds=True):
    """Other presets' build rates and traversal rates (single measurements after warm-up)."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    n = dt.shape[0]  # triangles (dv holds three vertices per soup triangle)
    res = {}

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    for preset in ("lbvh30", "hybrid", "sah4") if builds else ():
        b = rtb200.Bvh.build(dv, dt, preset, stream=stream)
        ms = timed(lambda: b.rebuild(dv, dt, preset, stream=stream), 3 if preset != "sah4" else 1)
        res[f"build_{preset}_mtri_s"] = round(n / (ms * 1e-3) / 1e6, 3)
        b.free()
    lo, hi = verts[:, :3].min(0), verts[:, :3].max(0)
    n_rays = getattr(a, "n_rays", N_RAYS)
    rays = torch.from_numpy(scenes.incoherent_rays(n_rays, lo, hi, seed=scenes.BASE_SEED + 9)).to(dev)
    prim = torch.from_numpy(scenes.pinhole_rays(1920, 1080, (0.5, 0.5, -1.5), (0.5, 0.5, 0.5), 60.0)).to(dev)
    inc = "incoherent16M" if n_rays == N_RAYS else f"incoherent{n_rays}"
    for preset in getattr(a, "trace_preset", "lbvh63,hybrid,sah4").split(","):
        b = rtb200.Bvh.build(dv, dt, preset, stream=stream)
        for name, r in ((inc, rays), ("primary1080p", prim)):
            for fl, fname in ((rtb200.TRACE_CLOSEST, "closest"), (rtb200.TRACE_ANY_HIT, "anyhit")):
                ms = timed(lambda: b.trace(r, fl, stream=stream), 3)
                res[f"trace_{preset}_{name}_{fname}_mray_s"] = round(r.shape[0] / (ms * 1e-3) / 1e6, 1)
        # the 8-wide layout (opt-in form: same closest distances, ties may name another triangle)
        b.trace_loop(2)
        for name, r in ((inc, rays), ("primary1080p", prim)):
            ms = timed(lambda: b.trace(r, rtb200.TRACE_CLOSEST, stream=stream), 3)
            res[f"trace_{preset}_wide8_{name}_closest_mray_s"] = round(r.shape[0] / (ms * 1e-3) / 1e6, 1)
        b.free()
    return res


def _ev_ms(fn, stream, reps=3):
    """Median CUDA-event time of fn on `stream` after one warm-up call."""
    import torch
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms)


def _orc_cfg(orc, rc):
    o = orc.OrcRenderCfg()
    for name, _ in orc.OrcRenderCfg._fields_:
        val = getattr(rc, name)
        if hasattr(val, "__len__"):
            getattr(o, name)[:] = list(val)
        else:
            setattr(o, name, val)
    return o


def _trace_ceiling(b, verts, stream, dev, n=1 << 22):
    """Closest-hit rate (Mray/s, CUDA events) of n incoherent rays -- origins uniform in the
    scene's box, directions uniform on the sphere -- through the same BVH: the traversal
    ceiling a path loop's segments are measured against."""
    import torch
    from rtb200 import scenes
    lo, hi = verts[:, :3].min(0), verts[:, :3].max(0)
    rays = torch.from_numpy(scenes.incoherent_rays(n, lo, hi, seed=scenes.BASE_SEED + 11, tmin=1e-4)).to(dev)
    ms = _ev_ms(lambda: b.trace(rays, 0, stream=stream), stream)
    return n / (ms * 1e-3) / 1e6


def profiled_render_counters(key):
    """Issue-slot and cache figures of a path-loop kernel from the committed ncu summaries
    (profiles/render_kernels_<workload>.md: lines `key: name=value, ...`), if present."""
    path = os.path.join(HERE, "profiles", f"render_kernels_{key.split('_')[0]}.md")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return {kv.split("=")[0].strip(): float(kv.split("=")[1]) for kv in line.split(":", 1)[1].split(",")}
    except Exception:
        pass
    return None


def _render_roofline(counts, samples_counted, samples, ms, ceiling, kernel, counters_key=None):
    """Traversal roofline of a path-loop workload: segments traced per second against the
    incoherent-ray closest-hit rate on the same BVH; the traversal work per sample (nodes
    popped and triangles tested, 48 bytes each: a node's two child boxes and references, a
    triangle's index and positions) from the oracle's count over the same samples."""
    seg, nodes, tris = (c / samples_counted for c in counts)
    rate = seg * samples / (ms * 1e-3) / 1e6
    out = {"bound": "issue (traversal)", "kernel": kernel, "achieved": round(rate, 1), "peak": round(ceiling, 1),
           "unit": "Mray/s (segments)", "frac": round(rate / ceiling, 4),
           "peak_kind": "closest-hit rate of 4,194,304 incoherent rays on the same BVH (rt_trace, CUDA events)",
           "segments_per_sample": round(seg, 4), "nodes_per_segment": round(nodes / seg, 2),
           "tri_tests_per_segment": round(tris / seg, 2),
           "traversal_bytes_per_sample": round(48 * (nodes + tris), 1),
           "traversal_gbs": round(48 * (nodes + tris) * samples / (ms * 1e-3) / 1e9, 1),
           "counted_samples": int(samples_counted)}
    if counters_key:
        out["ncu"] = profiled_render_counters(counters_key)
    return out


def _mpx(n, ms):
    return round(n / (ms * 1e-3) / 1e6, 1)


def render_c1(stream, dev):
    """Plain path tracing: 256 x 256, 16 spp, depth 4, no roulette; Cornell box + icosphere +
    two spheres; plain vs wavefront; the restated path loop on all host cores as the CPU leg."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    import oracle as orc
    sv, st_ = rtb200.Mesh().add_sphere((0.0, 0.0, 0.0), 0.3).arrays()
    sc = scenes.plain_scene(sphere_tris=(sv, st_))
    b = rtb200.Bvh.build(sc.verts, sc.tris, "lbvh30")
    mot = torch.from_numpy(sc.baked_materials(b.prim_ids()).astype(np.int32)).to(dev)
    mats = torch.from_numpy(rtb200.materials_array(sc.mats)).to(dev)
    rc = rtb200.render_cfg(256, 256, 16, max_bounce=4, rr_after=-1, env_kind=1, seed=7, lookat=sc.lookat)
    n = 256 * 256 * 16
    tp = _ev_ms(lambda: b.render(rc, mats, mot, mode=rtb200.RENDER_PLAIN, stream=stream), stream)
    tw = _ev_ms(lambda: b.render(rc, mats, mot, mode=rtb200.RENDER_WAVEFRONT, stream=stream), stream)
    ip, _ = b.render(rc, mats, mot, mode=rtb200.RENDER_PLAIN)
    iw, _ = b.render(rc, mats, mot, mode=rtb200.RENDER_WAVEFRONT)
    ip64, iw64 = ip.double(), iw.double()
    nodes, tris, vv = b.download()
    R = orc.Restatement()
    ocfg = _orc_cfg(orc, rc)
    cores = os.cpu_count() or 1
    rows = 16
    baked = orc.Baked(nodes, tris, vv)
    bmot = sc.baked_materials(b.prim_ids())
    t0 = time.perf_counter()
    ref, _ = R.render(baked, ocfg, sc.mats, bmot, rows=(120, 120 + rows), threads=cores)
    cpu_s = time.perf_counter() - t0
    _, counts = R.render_stats(baked, ocfg, sc.mats, bmot, rows=(120, 120 + rows), threads=cores)
    ceiling = _trace_ceiling(b, sc.verts, stream, dev)
    sl = ip.cpu().numpy()[120:120 + rows].astype(np.float64)
    out = {
        "workload": "256x256, 16 spp, depth 4, no roulette; Cornell box + 20,480-tri icosphere + 2 spheres (21,462 tris), "
                    "LBVH 30-bit",
        "plain_mpx_spp_s": _mpx(n, tp), "wavefront_mpx_spp_s": _mpx(n, tw), "plain_ms": round(tp, 3),
        "wavefront_ms": round(tw, 3),
        "wavefront_vs_plain_max_rel_diff": float(((iw64 - ip64).abs().max() / ip64.abs().max()).item()),
        "roofline": _render_roofline(counts, 256 * rows * 16, n, min(tp, tw), ceiling,
                                     "wavefront" if tw < tp else "plain", "c1_wavefront_trace"),
        "cpu_baseline": {"value": round(256 * rows * 16 / cpu_s / 1e6, 4), "unit": "Mpx*spp/s", "cores": cores,
                         "kind": "port (the oracle's restated path loop over the reference traversal)",
                         "sample": f"{rows} image rows (of 256) at 16 spp, scaled to the metric"},
        "cpu_rows_match_gpu_rel_mean": float(abs(sl.mean() - ref[120:120 + rows].astype(np.float64).mean()) /
                                             max(ref[120:120 + rows].mean(), 1e-12))}
    b.free()
    return out


def render_c3(stream, dev):
    """Batched: 64 scenes of 1,000-500,000 triangles built in one launch sequence and rendered
    at 512 x 512, 4 spp, depth 5 by the graph-replayed wavefront (autotuned) vs the plain kernel
    per scene; CPU leg: the reference's bake plus the restated path loop per scene, on a subset."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    import oracle as orc
    scs = scenes.batch_scenes(64)
    v, t, vo, to = rtb200.batch_arrays([(s_.verts, s_.tris) for s_ in scs])
    dvb = torch.from_numpy(v).to(dev)
    dtb = torch.from_numpy(t.view(np.int32)).to(dev)
    cfg30 = rtb200.make_cfg("lbvh30")
    bb = rtb200.Bvh.build_batch(dvb, dtb, vo, to, cfg30, stream=stream)
    tbb = _ev_ms(lambda: bb.rebuild_batch(dvb, dtb, vo, to, cfg30, stream=stream), stream)
    singles = [rtb200.Bvh.build(torch.from_numpy(s_.verts).to(dev), torch.from_numpy(s_.tris.view(np.int32)).to(dev), cfg30)
               for s_ in scs]
    sdev = [(torch.from_numpy(s_.verts).to(dev), torch.from_numpy(s_.tris.view(np.int32)).to(dev)) for s_ in scs]

    def rebuild_all():
        for bs, (x, y) in zip(singles, sdev):
            bs.rebuild(x, y, cfg30, stream=stream)
    tbs = _ev_ms(rebuild_all, stream)
    bmats, bmot_in = scenes.batch_shading(scs)
    bmot = torch.from_numpy(bmot_in[bb.prim_ids()].astype(np.int32)).to(dev)
    bmats_d = torch.from_numpy(rtb200.materials_array(bmats)).to(dev)
    rcs = [rtb200.render_cfg(512, 512, 4, max_bounce=5, rr_after=-1, env_kind=1, seed=31 + i, lookat=s_.lookat)
           for i, s_ in enumerate(scs)]
    t0 = time.perf_counter()
    tuned = bb.autotune(rcs, bmats_d, bmot, stream=stream)
    tune_s = time.perf_counter() - t0
    tbr = _ev_ms(lambda: bb.render_batch(rcs, bmats_d, bmot, stream=stream), stream)
    smats = [torch.from_numpy(rtb200.materials_array(s_.mats)).to(dev) for s_ in scs]
    smot = [torch.from_numpy(s_.baked_materials(bs.prim_ids()).astype(np.int32)).to(dev) for s_, bs in zip(scs, singles)]

    def plain_all():
        for i, bs in enumerate(singles):
            bs.render(rcs[i], smats[i], smot[i], mode=rtb200.RENDER_PLAIN, stream=stream)
    tpa = _ev_ms(plain_all, stream, 2)
    nb = 64 * 512 * 512 * 4
    img, _ = bb.render_batch(rcs, bmats_d, bmot)
    diffs = []
    for i in (0, 21, 42, 63):
        r_, _ = singles[i].render(rcs[i], smats[i], smot[i], mode=rtb200.RENDER_PLAIN)
        diffs.append(float(((img[i].double() - r_.double()).abs().max() / max(float(r_.abs().max()), 1e-12))))
    # CPU leg on four scenes of the batch (spread over its size range): the reference's own
    # single-threaded bake of each scene (oracle/_ref lbvh30) plus the restated path loop over
    # 8 of its 512 rows on all host cores, scaled to the full image and to 64 scenes
    cores = os.cpu_count() or 1
    R = orc.Restatement()
    sub = (0, 21, 42, 63)
    bake_s, render_s, counts, ceil = 0.0, 0.0, [0, 0, 0], []
    ref = orc.Reference("lbvh30") if orc.Reference.available("lbvh30") else None
    for i in sub:
        s_ = scs[i]
        if ref is not None:
            with quiet_stdout():
                t0 = time.perf_counter()
                ref.bake(s_.verts, s_.tris)
                bake_s += time.perf_counter() - t0
        nodes, tris, vv = singles[i].download()
        baked = orc.Baked(nodes, tris, vv)
        mot_i = s_.baked_materials(singles[i].prim_ids())
        t0 = time.perf_counter()
        R.render(baked, _orc_cfg(orc, rcs[i]), s_.mats, mot_i, rows=(252, 260), threads=cores)
        render_s += (time.perf_counter() - t0) * 512 / 8
        _, c = R.render_stats(baked, _orc_cfg(orc, rcs[i]), s_.mats, mot_i, rows=(252, 260), threads=cores)
        counts = [a + b_ for a, b_ in zip(counts, c)]
        ceil.append(_trace_ceiling(singles[i], s_.verts, stream, dev, n=1 << 20))
    cpu_total_s = (bake_s + render_s) * 64 / len(sub)
    out = {
        "workload": f"64 scenes, {int(to[-1])} triangles (log-uniform 1,000-500,000 per scene), 512x512, 4 spp, depth 5",
        "build_batched_ms": round(tbb, 3), "build_batched_mtri_s": round(int(to[-1]) / tbb / 1e3, 1),
        "build_64_separate_ms": round(tbs, 3),
        "render_batched_wavefront_mpx_spp_s": _mpx(nb, tbr), "render_plain_per_scene_mpx_spp_s": _mpx(nb, tpa),
        "render_batched_ms": round(tbr, 2), "render_plain_per_scene_ms": round(tpa, 2),
        "autotuned": tuned.as_dict(), "autotune_s": round(tune_s, 2),
        "batched_vs_plain_max_rel_diff": max(diffs),
        "roofline": _render_roofline(counts, len(sub) * 8 * 512 * 4, nb, tbr, statistics.mean(ceil),
                                     "batched wavefront (autotuned)", "c3_wavefront_trace"),
        "cpu_baseline": {"value": round(nb / cpu_total_s / 1e6, 4), "unit": "Mpx*spp/s (bake + render)", "cores": cores,
                         "kind": "reference bake + port (the oracle's restated path loop)",
                         "sample": f"scenes {sub}: the reference's bake of each (1 thread, {bake_s:.2f} s) and the "
                                   f"restated path loop over rows 252-259 of 512 at 4 spp on {cores} threads, the "
                                   f"render scaled by 64 to the full image; the sum scaled by 16 to 64 scenes",
                         "bake_s_subset": round(bake_s, 3), "render_s_subset_scaled": round(render_s, 3)}}
    for bs in singles:
        bs.free()
    bb.free()
    return out


def render_c4(stream, dev):
    """Differentiable rendering: adjoint / forward of the L2 loss against a 1024-spp target
    image rendered from the seeded ground-truth albedos."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    dsc, init, gt = scenes.diff_scene()
    bd = rtb200.Bvh.build(dsc.verts, dsc.tris, "lbvh30")
    prim = bd.prim_ids()
    dmot = torch.from_numpy(dsc.baked_materials(prim).astype(np.int32)).to(dev)
    dmats = torch.from_numpy(rtb200.materials_array(dsc.mats)).to(dev)
    talb = torch.from_numpy(init[prim]).to(dev)
    rct = rtb200.render_cfg(512, 512, 1024, max_bounce=4, rr_after=-1, env_kind=1, seed=77, lookat=dsc.lookat)
    target, _ = bd.render(rct, dmats, dmot, tri_albedo=torch.from_numpy(gt[prim]).to(dev))
    rcd = rtb200.render_cfg(512, 512, 32, max_bounce=4, rr_after=-1, env_kind=1, seed=9, lookat=dsc.lookat)
    fwd = _ev_ms(lambda: bd.render(rcd, dmats, dmot, tri_albedo=talb, stream=stream), stream)
    img, _ = bd.render(rcd, dmats, dmot, tri_albedo=talb)
    loss = float(((img.double() - target.double()) ** 2).sum().item())
    dimg = (2.0 * (img - target)).contiguous()  # dLoss/dimage of the L2 loss
    adj = _ev_ms(lambda: bd.adjoint(rcd, dimg, dmats, dmot, tri_albedo=talb, stream=stream), stream)
    out = {
        "workload": "512x512, 32 spp, depth 4; Cornell box + 50,000-triangle icosphere; L2 loss against a 1024-spp "
                    "target from seeded ground-truth albedos; gradients of per-triangle RGB albedo and material emission",
        "forward_ms": round(fwd, 2), "adjoint_ms": round(adj, 2), "adjoint_over_forward": round(adj / fwd, 3),
        "forward_mpx_spp_s": _mpx(512 * 512 * 32, fwd), "l2_loss": round(loss, 3)}
    bd.free()
    return out


def render_c5(stream, dev):
    """Large render: 1920 x 1080, 64 spp, depth 8, roulette after bounce 2, 5,000,010 triangles,
    binned SAH with spatial splits; plain vs wavefront (defaults and autotuned); CPU leg: the
    restated path loop on a few rows."""
    import numpy as np
    import torch
    import rtb200
    from rtb200 import scenes
    import oracle as orc
    lsc = scenes.large_scene()
    dvl = torch.from_numpy(lsc.verts).to(dev)
    dtl = torch.from_numpy(lsc.tris.view(np.int32)).to(dev)
    bl = rtb200.Bvh.build(dvl, dtl, "sah4", stream=stream)
    tsah = _ev_ms(lambda: bl.rebuild(dvl, dtl, "sah4", stream=stream), stream, 1)
    lmot = torch.from_numpy(lsc.baked_materials(bl.prim_ids()).astype(np.int32)).to(dev)
    lmats = torch.from_numpy(rtb200.materials_array(lsc.mats)).to(dev)
    rcl = rtb200.render_cfg(1920, 1080, 64, max_bounce=8, rr_after=2, env_kind=1, env_color=lsc.env_color, seed=5,
                            lookat=lsc.lookat)
    tlp = _ev_ms(lambda: bl.render(rcl, lmats, lmot, mode=rtb200.RENDER_PLAIN, stream=stream), stream, 1)
    tlw = _ev_ms(lambda: bl.render(rcl, lmats, lmot, mode=rtb200.RENDER_WAVEFRONT, stream=stream), stream, 1)
    tuned = bl.autotune([rcl], lmats, lmot, stream=stream)
    tlt = _ev_ms(lambda: bl.render_batch([rcl], lmats, lmot, stream=stream), stream, 1)
    nl = 1920 * 1080 * 64
    # CPU leg and traversal counts: the restated path loop over 4 of the 1080 rows
    cores = os.cpu_count() or 1
    nodes, tris, vv = bl.download()
    baked = orc.Baked(nodes, tris, vv)
    R = orc.Restatement()
    bmot = lsc.baked_materials(bl.prim_ids())
    rows = (538, 542)
    t0 = time.perf_counter()
    R.render(baked, _orc_cfg(orc, rcl), lsc.mats, bmot, rows=rows, threads=cores)
    cpu_s = time.perf_counter() - t0
    _, counts = R.render_stats(baked, _orc_cfg(orc, rcl), lsc.mats, bmot, rows=rows, threads=cores)
    ceiling = _trace_ceiling(bl, lsc.verts, stream, dev)
    best = min(tlp, tlw, tlt)
    out = {
        "workload": "1920x1080, 64 spp, depth 8, roulette after bounce 2; 400 icospheres x 12,500 triangles + floor + "
                    "4 quad lights (5,000,010 triangles), 80/20 Lambertian/mirror; binned SAH + spatial splits, leaf 4",
        "sah_build_ms": round(tsah, 1), "sah_build_mtri_s": round(lsc.tris.shape[0] / tsah / 1e3, 3),
        "plain_mpx_spp_s": _mpx(nl, tlp), "wavefront_mpx_spp_s": _mpx(nl, tlw),
        "wavefront_tuned_mpx_spp_s": _mpx(nl, tlt), "autotuned": tuned.as_dict(),
        "plain_ms": round(tlp, 1), "wavefront_ms": round(tlw, 1), "wavefront_tuned_ms": round(tlt, 1),
        "roofline": _render_roofline(counts, 1920 * (rows[1] - rows[0]) * 64, nl, best, ceiling,
                                     {tlp: "plain", tlw: "wavefront", tlt: "wavefront (autotuned)"}[best],
                                     "c5_wavefront_trace"),
        "cpu_baseline": {"value": round(1920 * (rows[1] - rows[0]) * 64 / cpu_s / 1e6, 4), "unit": "Mpx*spp/s",
                         "cores": cores, "kind": "port (the oracle's restated path loop over the reference traversal)",
                         "sample": f"rows {rows[0]}-{rows[1] - 1} of 1080 at 64 spp, scaled to the metric"}}
    bl.free()
    return out


RENDER_WORKLOADS = {"c1": render_c1, "c3": render_c3, "c4": render_c4, "c5": render_c5}


def render_workloads(stream, dev, which=None):
    """The path-loop workloads (GPU numbers by CUDA events on torch's stream)."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    names = {"c1": "plain_c1", "c3": "batched_c3", "c4": "adjoint_c4", "c5": "large_c5"}
    return {names[k]: fn(stream, dev) for k, fn in RENDER_WORKLOADS.items() if which is None or k == which}


def main():
    a = parse_args()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
