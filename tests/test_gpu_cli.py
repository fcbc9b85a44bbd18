"""The mgkde_tiled driver (reference command line) on the GPU: the density
GeoTIFF and pntsCUDA.csv agree with the FP64 oracle run of the same case."""
import os
import subprocess

import numpy as np
import pytest

from golden_cases import load, oracle_run
from mgpukde_tiled_b200 import tiff
from test_cli_and_io import CLI, write_case_files

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,hopt", [("redwood_h0", 0), ("redwood_h1", 1), ("loo_h1", 1), ("redwood_h2", 2)])
def test_cli_mode1_matches_oracle(tmp_path, case, hopt):
    g = write_case_files(str(tmp_path), case)
    ref = oracle_run(load(case))
    p = subprocess.run([CLI] + f"1 p.csv e.tif d.tif {hopt} 1 0 1 0 1 1 a.tif b.tif 0 --tile=96".split(),
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:]
    if hopt == 1:
        assert "hopt: %.5f" % float(g["ref_hopt"]) in p.stdout
    den = tiff.read(str(tmp_path / "b.tif")).data
    nd = g["density_mask"] == g["dg"].nodata
    assert np.array_equal(den[nd], g["density_mask"][nd])
    if hopt == 2:
        assert "h0: %.5f alpha0: %.5f" % (ref["h"], ref["alpha"]) in p.stdout
    # adaptive h: the per-point bandwidths carry FP32 pilot densities (one ulp)
    tol = 3e-6 if hopt == 2 else 1e-6
    rel = np.abs(den[~nd] - ref["density"][~nd]) / np.maximum(np.abs(ref["density"][~nd]), 1e-300)
    assert rel.max() <= tol
    pts = np.loadtxt(str(tmp_path / "pntsCUDA.csv"), delimiter=",", skiprows=1, ndmin=2)
    # printed with 6 decimals, input order
    assert np.all(np.abs(pts[:, 3] - ref["ew"]) <= 6e-7 + 3e-6 * np.abs(ref["ew"]))
    if hopt == 2:
        assert np.all(np.abs(pts[:, 2] - ref["hs"]) <= 6e-7 + 4e-7 * np.abs(ref["hs"]))


@pytest.mark.parametrize("case", ["poly_varh", "uniform_c0"])
def test_cli_per_point_bandwidths_match_oracle(tmp_path, case):
    """h_option -1: the bandwidths come from the CSV's h column (the
    reference reads it at kde_cuda_kdtr_tiled.cu:413-421), with sample
    weights and edge correction on.  The density GeoTIFF and pntsCUDA.csv
    (x, y, h, edge weight in input order; written at :1857-1870) agree with
    the FP64 oracle run of the same case."""
    g = write_case_files(str(tmp_path), case, with_h=True)
    ref = oracle_run(g)
    p = subprocess.run([CLI] + "1 p.csv e.tif d.tif -1 1 1 1 0 1 1 a.tif b.tif 0 --tile=64".split(),
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:]
    den = tiff.read(str(tmp_path / "b.tif")).data
    nd = g["density_mask"] == g["dg"].nodata
    assert np.array_equal(den[nd], g["density_mask"][nd])
    rel = np.abs(den[~nd] - ref["density"][~nd]) / np.maximum(np.abs(ref["density"][~nd]), 1e-300)
    assert rel.max() <= 1e-6, rel.max()
    pts = np.loadtxt(str(tmp_path / "pntsCUDA.csv"), delimiter=",", skiprows=1, ndmin=2)
    assert pts.shape == (len(g["x"]), 4)
    # printed with 6 decimals, input order
    assert np.all(np.abs(pts[:, 0] - g["x"]) <= 6e-7 + 1e-7 * np.abs(g["x"]))
    assert np.all(np.abs(pts[:, 1] - g["y"]) <= 6e-7 + 1e-7 * np.abs(g["y"]))
    assert np.all(np.abs(pts[:, 2] - g["h_pp"]) <= 6e-7)
    assert np.all(np.abs(pts[:, 3] - ref["ew"]) <= 6e-7 + 3e-6 * np.abs(ref["ew"]))
    assert np.array_equal(pts[:, 3] == 1.0, ref["ew"] == 1.0)


def test_cli_mode0_runs(tmp_path):
    p = subprocess.run([CLI] + "0 2000 1.0 0.5 0 1 0 1 0 1 1 a.tif b.tif 0".split(), cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:]
    r = tiff.read(str(tmp_path / "b.tif"))
    assert r.data.shape == (200, 200) and np.isfinite(r.data).all() and (r.data > 0).any()


def test_cli_resume_after_a_tile_limit(tmp_path):
    """--max-tiles stops a run after K density tiles (exit code 2, tiles
    logged); --resume computes only the rest; the GeoTIFF equals an
    uninterrupted run's bit for bit."""
    write_case_files(str(tmp_path), "poly_fixed")
    args = "1 p.csv e.tif d.tif 0 1 1 1 0 1 1 a.tif b.tif 0 --tile=32".split()
    full = subprocess.run([CLI] + args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert full.returncode == 0, full.stdout[-2000:]
    ref = tiff.read(str(tmp_path / "b.tif")).data
    os.rename(tmp_path / "b.tif", tmp_path / "full.tif")
    p1 = subprocess.run([CLI] + args + ["--max-tiles=3"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p1.returncode == 2, p1.stdout[-2000:]
    logged = [int(v) for v in open(tmp_path / "b.tif.tiles").read().split()]
    assert logged == [0, 1, 2]
    p2 = subprocess.run([CLI] + args + ["--resume"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p2.returncode == 0, p2.stdout[-2000:]
    wrote = [int(line.split()[2].rstrip(":")) for line in p2.stdout.splitlines() if line.startswith("...wrote tile")]
    assert wrote and not set(wrote) & set(logged)
    assert not os.path.exists(tmp_path / "b.tif.tiles")
    got = tiff.read(str(tmp_path / "b.tif")).data
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_cli_autotune_keeps_parity(tmp_path):
    g = write_case_files(str(tmp_path), "redwood_h0")
    ref = oracle_run(load("redwood_h0"))
    args = "1 p.csv e.tif d.tif 0 1 0 1 0 1 1 a.tif b.tif 0 --autotune=tune.txt".split()
    for k in range(2):
        p = subprocess.run([CLI] + args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:]
        assert "...autotune: bin side" in p.stdout and (("(cached)" in p.stdout) == (k == 1))
        den = tiff.read(str(tmp_path / "b.tif")).data
        nd = g["density_mask"] == g["dg"].nodata
        rel = np.abs(den[~nd] - ref["density"][~nd]) / np.maximum(np.abs(ref["density"][~nd]), 1e-300)
        assert rel.max() <= 1e-6
