"""bench.py's reference arm on the host: one JSON line with the metric, unit and direction of
the GPU arm, the CPU baseline it measured (kind, cores, sample) and an end-to-end entry with no
device copies. Runs on the CPU (the reference's bake, or its restatement when the reference
build is absent)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "BVH Mtri/s" and d["unit"] == "Mtri/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Mtri/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_committed_profile_figures_parse():
    """The ncu figures bench.py attaches to its lines come from the committed summaries: the
    bake's DRAM bytes per triangle and the trace kernel's counters of each render workload."""
    sys.path.insert(0, ROOT)
    import bench
    traffic = bench.profiled_traffic()
    assert traffic is not None and 100.0 < traffic < 2000.0
    for key in ("c1_wavefront_trace", "c3_wavefront_trace", "c5_wavefront_trace"):
        c = bench.profiled_render_counters(key)
        assert c is not None, key
        assert set(c) >= {"issue_active_pct", "threads_per_inst", "l1_hit_pct", "l2_hit_pct"}, key
        assert 0.0 < c["issue_active_pct"] <= 100.0 and 0.0 < c["threads_per_inst"] <= 32.0, key
    assert bench.bake_bytes_per_tri(1 << 20) < bench.bake_bytes_per_tri(1 << 24)
