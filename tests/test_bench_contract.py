"""bench.py's contract on the CPU: the reference arm's JSON line (the
reference program's own CPU path, timed on the host cores, on the
single-large workload), rank 0 alone working and printing under torchrun,
and the roofline object of the GPU line computed from known numbers."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref", "mgkde_ref")
CMD = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3", "--scale", "0.1"]
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def run(env=None):
    return subprocess.run(CMD, cwd=REPO, env=env, capture_output=True, text=True, timeout=900)


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference program is not built here")
def test_reference_arm_json_line():
    p = run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "halo points" in cb["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = run(env)
    assert p.returncode == 0, p.stderr[-2000:]
    assert not p.stdout.strip()


def test_density_roofline_fields():
    """The GPU line's roofline object, from known numbers: 4e10 evals in 10 ms
    on 148 SMs at 1965 MHz, 850.6 MB of traffic, 800 MB algorithmic."""
    sys.path.insert(0, REPO)
    import bench

    r = bench.density_roofline(4.0e10, 0.010, 148, 1965.0, "measured", 850_600_000, 800_000_000, 6454.6)
    assert r["bound"] == "fp32" and r["unit"] == "TFLOP/s" and r["kernel"] == "k_density"
    assert abs(r["peak"] - 148 * 128 * 2 * 1965e6 / 1e12) < 1e-9
    assert abs(r["achieved"] - 4.0e10 * 8 / 0.010 / 1e12) < 1e-9
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert r["traffic"] == 850_600_000 and abs(r["kernel_ms"] - 10.0) < 1e-9
    h = r["hbm"]
    assert h["unit"] == "GB/s" and h["peak"] == 6454.6
    assert abs(h["achieved"] - 80.0) < 1e-9 and "traffic_gbs" not in h
    assert abs(h["frac"] - 80.0 / 6454.6) < 1e-12
    # the captured traffic and pipe figures say where they come from
    assert "profiles/k_density_traffic.txt" in r["traffic_note"]
    assert r["pipes_ncu"]["fma_pct"] > 0 and "profiles/" in r["pipes_ncu"]["source"]
    # no measured HBM figure, no traffic capture: the FP32 view alone, no traffic note
    assert "hbm" not in bench.density_roofline(1e9, 0.01, 148, 1965.0, "fallback", None, 1, None)
    assert "traffic_note" not in bench.density_roofline(1e9, 0.01, 148, 1965.0, "measured", None, 8, 6000.0)


def _oracle_study(scale):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np

    import bench
    import oracle_py as o

    c = bench.build_workload("single_large", scale, seed=1)
    eg = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(c["x"], c["y"], eg, o.mark_boundary(eg, c["edge_mask"]))
    ew, eev = o.edge_weights(c["x"], c["y"], c["h"], d2, eg, c["edge_mask"])
    den, dev = o.density(c["x"], c["y"], c["w"], ew, c["h"], o.grid(*c["density_grid"].astuple()),
                         c["density_mask"])
    return bench, np, c, den.astype(np.float32), dev, eev


def test_whole_raster_accuracy_fields():
    """The single-large accuracy leg on a 1/50-scale study: a raster equal to
    the oracle's (rounded to float) passes, one with a cell moved by 1e-5
    relative is reported, and the pair counts are compared."""
    bench, np, c, den, dev, eev = _oracle_study(0.02)
    valid = c["density_mask"] != c["density_grid"].nodata
    bad = den.copy()
    r, k = np.argwhere(valid)[len(np.argwhere(valid)) // 2]
    bad[r, k] *= np.float32(1 + 1e-5)
    a = bench.single_large_accuracy(c, {"step": den, "e2e": bad}, dev, eev + 1)
    assert a["max_rel_err_step"] <= 1e-7 and 0.9e-5 < a["max_rel_err_e2e"] < 1.1e-5
    assert a["max_rel_err"] == a["max_rel_err_e2e"] and a["nodata_cells_equal"]
    assert a["density_evals_equal"] and not a["edge_evals_equal"]
    assert a["cells"] == int(valid.sum()) and a["cells"] + a["nodata_cells"] == valid.size


def test_argmax_check_fields():
    """The bandwidth-selection argmax leg on a 1/20-scale study: given the
    oracle's own logL (slightly perturbed) it finds the same argmax and
    reports the margin to the runner-up."""
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np

    import bench
    import oracle_py as o
    from mgpukde_tiled_b200 import synth

    c = synth.bandwidth_select(scale=0.05, seed=2, nh=8)
    eg = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(c["x"], c["y"], eg, o.mark_boundary(eg, c["edge_mask"]))
    ll = np.array([o.loglik_at(c["x"], c["y"], c["w"], d2, eg, c["edge_mask"], float(h))[0] for h in c["hgrid"]])
    best = int(np.argmax(ll))
    a = bench.loo_argmax_check(c, c["hgrid"], ll * (1 + 1e-12), best)
    assert a["argmax_equal"] and a["argmax_gpu"] == best and best in a["indices_checked"]
    assert a["logl_max_rel_err"] < 1e-11
    assert a["margin_gpu"] > 0 and a["margin_oracle"] > 0 and a["runner_up_gpu"] != best


def test_out_of_core_accuracy_fields():
    """The out-of-core accuracy leg on a 1/100-scale study (400^2 raster) in
    tiles of 128: five tiles, the ragged corner one included."""
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np

    import bench
    import oracle_py as o
    from mgpukde_tiled_b200 import synth

    c = synth.out_of_core(scale=0.01, seed=3)
    dg = c["density_grid"]
    eg = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(c["x"], c["y"], eg, o.mark_boundary(eg, c["edge_mask"]))
    ew, _ = o.edge_weights(c["x"], c["y"], c["h"], d2, eg, c["edge_mask"])
    den, _ = o.density(c["x"], c["y"], c["w"], ew, c["h"], o.grid(*dg.astuple()), None)
    a = bench.out_of_core_accuracy(c, den.astype(np.float32), 128)
    assert len(a["tiles"]) == 5 and a["tiles"][-1]["tile"] == [3, 3] and a["tiles"][-1]["cells"] == 16 * 16
    assert a["max_rel_err"] <= 1e-7
