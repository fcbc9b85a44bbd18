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


@pytest.mark.parametrize("case,hopt", [("redwood_h0", 0), ("redwood_h1", 1), ("loo_h1", 1)])
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
    rel = np.abs(den[~nd] - ref["density"][~nd]) / np.maximum(np.abs(ref["density"][~nd]), 1e-300)
    assert rel.max() <= 1e-6
    pts = np.loadtxt(str(tmp_path / "pntsCUDA.csv"), delimiter=",", skiprows=1, ndmin=2)
    # printed with 6 decimals, input order
    assert np.all(np.abs(pts[:, 3] - ref["ew"]) <= 6e-7 + 1e-6 * np.abs(ref["ew"]))


def test_cli_mode0_runs(tmp_path):
    p = subprocess.run([CLI] + "0 2000 1.0 0.5 0 1 0 1 0 1 1 a.tif b.tif 0".split(), cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:]
    r = tiff.read(str(tmp_path / "b.tif"))
    assert r.data.shape == (200, 200) and np.isfinite(r.data).all() and (r.data > 0).any()
