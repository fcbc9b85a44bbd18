"""Generates the golden fixtures in tests/golden/ by running the reference.

Runs ONLY in the build container, where the reference sources exist: it builds
the reference program from its unmodified sources (oracle/ref_build.sh), runs
its CPU path (mode 1, skip_gpu_parallel=1) on seeded inputs and on the
reference's own sample data, and stores inputs plus the reference's outputs as
small .npz files.  The tests read only the .npz files.

  python tests/golden/make_golden.py            # all cases
Outputs per case: ref_density (the reference's Float32 density raster),
ref_pnts (its points CSV: x, y, h, edge weight, in its own order), ref_h0 /
ref_hopt (printed bandwidths).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from mgpukde_tiled_b200 import synth, tiff  # noqa: E402

REF_BIN = os.path.join(REPO, "oracle", "_ref", "mgkde_ref")
REF_SAMPLE = "/root/reference/x64/Debug"


def ensure_ref():
    if not os.path.exists(REF_BIN):
        subprocess.run([os.path.join(REPO, "oracle", "ref_build.sh")], check=True)


def write_csv(path, x, y, w, h=None):
    with open(path, "w") as f:
        f.write("x,y,h,w\n" if h is not None else "x,y,w\n")
        for i in range(len(x)):
            if h is not None:
                f.write("%.9g,%.9g,%.9g,%.9g\n" % (x[i], y[i], h[i], w[i]))
            else:
                f.write("%.9g,%.9g,%.9g\n" % (x[i], y[i], w[i]))


def grid_gt(g: synth.Grid):
    return (float(g.xll), float(g.cs), 0.0, float(g.yll) + g.nrows * float(g.cs), 0.0, -float(g.cs))


def run_ref(workdir, csv, edge_tif, dens_tif, hopt, edge, sw, threads=1):
    cmd = [REF_BIN, "1", csv, edge_tif, dens_tif, str(hopt), str(int(edge)), str(int(sw)),
           "0", "1", str(threads), "1", "den_cpu.tif", "den_gpu.tif", "0"]
    p = subprocess.run(cmd, cwd=workdir, capture_output=True, text=True, timeout=3600)
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    out = p.stdout
    den = tiff.read(os.path.join(workdir, "den_cpu.tif")).data
    pnts = np.loadtxt(os.path.join(workdir, "pntsCPU.csv"), delimiter=",", skiprows=1, ndmin=2)
    h0 = float(re.search(r"Rule of thumb bandwidth h0: ([-0-9.eE+]+)", out).group(1))
    m = re.search(r"hopt: ([-0-9.eE+]+)", out)
    hopt_v = float(m.group(1)) if m else float("nan")
    t_den = re.search(r"KernelDesityEstimation took (\d+) ms", out)
    return den, pnts, h0, hopt_v, out, (int(t_den.group(1)) if t_den else -1)


def make_case(name, x, y, w, h_pp, eg, emask, dg, dmask, hoption, edge, sw):
    with tempfile.TemporaryDirectory() as d:
        csv = os.path.join(d, "pts.csv")
        write_csv(csv, x, y, w, h_pp if hoption == -1 else None)
        tiff.write(os.path.join(d, "edge.tif"), tiff.GeoRaster(emask, grid_gt(eg), eg.nodata))
        tiff.write(os.path.join(d, "dens.tif"), tiff.GeoRaster(dmask, grid_gt(dg), dg.nodata))
        den, pnts, h0, hopt, log, _ = run_ref(d, csv, "edge.tif", "dens.tif", hoption, edge, sw)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        x=x, y=y, w=w, h_pp=(h_pp if h_pp is not None else np.zeros(0, np.float32)),
        hoption=hoption, edge=int(edge), sample_weights=int(sw),
        edge_grid=np.array(eg.astuple(), np.float64), edge_mask=emask,
        density_grid=np.array(dg.astuple(), np.float64), density_mask=dmask,
        ref_density=den, ref_pnts=pnts, ref_h0=h0, ref_hopt=hopt)
    print(f"{name}: n={len(x)} h0={h0} hopt={hopt} density {den.shape}")


def main(only=()):
    ensure_ref()

    def want(name):
        return not only or name in only

    # 1-2: the reference's own sample data (62 redwood seedlings, 128x128 mask at 1/128).
    if os.path.isdir(REF_SAMPLE):
        pts = np.loadtxt(os.path.join(REF_SAMPLE, "pntsRedwood.csv"), delimiter=",", skiprows=1)
        x, y, w = (pts[:, 0].astype(np.float32), pts[:, 1].astype(np.float32), pts[:, 2].astype(np.float32))
        r = tiff.read(os.path.join(REF_SAMPLE, "redwood_edgecorrection.tif"))
        g = synth.Grid(r.data.shape[1], r.data.shape[0], np.float32(r.xll), np.float32(r.yll),
                       np.float32(r.cell_size), np.float32(r.nodata))
        if want("redwood_h0"):
            make_case("redwood_h0", x, y, w, None, g, r.data, g, r.data, 0, True, False)
        if want("redwood_h1"):
            make_case("redwood_h1", x, y, w, None, g, r.data, g, r.data, 1, True, False)
    # 3: 10,000 uniform points in 100 x 100, h = 2 (per-point column), all cells valid.
    c = synth.small_uniform(seed=0)
    hpp = np.full(len(c["x"]), 2.0, np.float32)
    if want("uniform_c0"):
        make_case("uniform_c0", c["x"], c["y"], c["w"], hpp, c["edge_grid"], c["edge_mask"],
              c["density_grid"], c["density_mask"], -1, True, True)
    # 4-5: mixture points with lognormal weights under a polygon mask.
    x, y = synth.mixture_points(3000, 6, 100.0, 4.0, 15.0, seed=11)
    w = synth.lognormal_weights(3000, seed=12)
    poly = synth.star_polygon(100.0, seed=13)
    dg = synth.Grid(100, 100, 0.0, 0.0, 1.0)
    eg = synth.Grid(50, 50, 0.0, 0.0, 2.0)
    dm, em = synth.rasterize_polygon(poly, dg), synth.rasterize_polygon(poly, eg)
    if want("poly_fixed"):
        make_case("poly_fixed", x, y, w, np.full(3000, 3.0, np.float32), eg, em, dg, dm, -1, True, True)
    hv = np.random.Generator(np.random.PCG64(14)).uniform(1.5, 5.0, 3000).astype(np.float32)
    if want("poly_varh"):
        make_case("poly_varh", x, y, w, hv, eg, em, dg, dm, -1, True, True)
    # 6: rule-of-thumb bandwidth, edge correction off, offset origin and fractional cells.
    x, y = synth.uniform_points(2000, 10.0, 60.0, seed=21)
    dg = synth.Grid(80, 64, np.float32(5.0), np.float32(7.5), np.float32(0.75))
    dm = synth.all_valid(dg)
    dm[:5, :] = dg.nodata
    dm[:, -3:] = dg.nodata
    if want("uniform_h0_noedge"):
        make_case("uniform_h0_noedge", x, y, np.ones_like(x), None, dg, dm, dg, dm, 0, False, False)
    # 7: golden-section LOO bandwidth search with edge correction.
    x, y = synth.mixture_points(1500, 4, 100.0, 5.0, 12.0, seed=31)
    eg = synth.Grid(50, 50, 0.0, 0.0, 2.0)
    em = synth.rasterize_polygon(synth.star_polygon(100.0, seed=33), eg)
    dg = synth.Grid(25, 25, 0.0, 0.0, 4.0)
    if want("loo_h1"):
        make_case("loo_h1", x, y, np.ones_like(x), None, eg, em, dg, synth.all_valid(dg), 1, True, False)


    # 8-9: adaptive bandwidths (h_option 2): Hooke-Jeeves over (h0, alpha).
    if os.path.isdir(REF_SAMPLE) and want("redwood_h2"):
        pts = np.loadtxt(os.path.join(REF_SAMPLE, "pntsRedwood.csv"), delimiter=",", skiprows=1)
        x, y, w = (pts[:, 0].astype(np.float32), pts[:, 1].astype(np.float32), pts[:, 2].astype(np.float32))
        r = tiff.read(os.path.join(REF_SAMPLE, "redwood_edgecorrection.tif"))
        g = synth.Grid(r.data.shape[1], r.data.shape[0], np.float32(r.xll), np.float32(r.yll),
                       np.float32(r.cell_size), np.float32(r.nodata))
        make_case("redwood_h2", x, y, w, None, g, r.data, g, r.data, 2, True, False)
    if want("poly_h2"):
        x, y = synth.mixture_points(800, 4, 100.0, 4.0, 14.0, seed=41)
        w = synth.lognormal_weights(800, seed=42)
        poly = synth.star_polygon(100.0, seed=43)
        eg = synth.Grid(50, 50, 0.0, 0.0, 2.0)
        dg = synth.Grid(50, 50, 0.0, 0.0, 2.0)
        em = synth.rasterize_polygon(poly, eg)
        make_case("poly_h2", x, y, w, None, eg, em, dg, synth.rasterize_polygon(poly, dg), 2, True, True)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
