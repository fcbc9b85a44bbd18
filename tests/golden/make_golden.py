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
# the reference checkout (read-only); REFERENCE_ROOT overrides the default
# location, as oracle/ref_build.sh reads it
REF_ROOT = os.environ.get("REFERENCE_ROOT", "/root/reference")
REF_SAMPLE = os.path.join(REF_ROOT, "x64", "Debug")


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


    # 10-11: large coordinates (the single-large workload at about 1e4 units,
    # the out-of-core one at about 4e4), where float coordinates have ulps of
    # 2^-10 and 2^-8, with points placed at the 3h cutoff of cell centres.
    if want("c1_crop_h50"):
        large_coordinate_case("c1_crop_h50", xll=9870.0, yll=10050.0, ncols=160, nrows=128, h=50.0,
                              edge_cs=4.0, n=3000, seed=51)
    if want("c3_crop_h30"):
        large_coordinate_case("c3_crop_h30", xll=39620.0, yll=40010.0, ncols=144, nrows=112, h=30.0,
                              edge_cs=5.0, n=2500, seed=61)


def near_cutoff_points(rng, cx, cy, h, k, tol):
    """k float points each within tol (units) of distance 3h from one of the
    given cell centres (exact distance of the float positions)."""
    out = []
    r3 = 3.0 * h
    while len(out) < k:
        i = int(rng.integers(len(cx)))
        t = rng.uniform(0.0, 2.0 * np.pi)
        r = r3 + rng.uniform(-tol, tol)
        px, py = np.float32(cx[i] + r * np.cos(t)), np.float32(cy[i] + r * np.sin(t))
        d = np.hypot(float(px) - float(cx[i]), float(py) - float(cy[i]))
        if abs(d - r3) <= tol:
            out.append((px, py))
    return np.array(out, np.float32).reshape(-1, 2)


def large_coordinate_case(name, xll, yll, ncols, nrows, h, edge_cs, n, seed):
    """Mixture points (three Gaussians over the window and its 3h halo, plus
    a uniform background) with lognormal weights around a density window at
    large coordinates, under a star-polygon mask; edge mask at a coarser cell
    over the window grown by 4h.  Added points: 64 within 1e-5 h of the 3h
    cutoff from valid cell centres, 8 exactly on it (offsets of a 3-4-5
    triangle scaled to 3h) and 8 one float step inside those."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dg = synth.Grid(ncols, nrows, np.float32(xll), np.float32(yll), np.float32(1.0))
    pad = 4.0 * h
    ex0, ey0 = xll - pad, yll - pad
    ecols, erows = int(np.ceil((ncols + 2 * pad) / edge_cs)), int(np.ceil((nrows + 2 * pad) / edge_cs))
    eg = synth.Grid(ecols, erows, np.float32(ex0), np.float32(ey0), np.float32(edge_cs))
    side = max(ecols, erows) * edge_cs
    # centred off the window's centre, so that its edge crosses the window
    poly = synth.star_polygon(side, seed + 1, rmin=0.12, rmax=0.3) + np.array([ex0 + 0.4 * ncols, ey0 - 0.35 * nrows])
    dm, em = synth.rasterize_polygon(poly, dg), synth.rasterize_polygon(poly, eg)
    # three clusters and a uniform background over the window grown by 3h
    lo_x, hi_x, lo_y, hi_y = xll - 3 * h, xll + ncols + 3 * h, yll - 3 * h, yll + nrows + 3 * h
    k = rng.integers(0, 3, n)
    mx = rng.uniform(xll, xll + ncols, 3)
    my = rng.uniform(yll, yll + nrows, 3)
    sg = rng.uniform(0.8 * h, 2.4 * h, 3)
    x = mx[k] + sg[k] * rng.standard_normal(n)
    y = my[k] + sg[k] * rng.standard_normal(n)
    nb = n // 8
    x[:nb] = rng.uniform(lo_x, hi_x, nb)
    y[:nb] = rng.uniform(lo_y, hi_y, nb)
    x, y = x.astype(np.float32), y.astype(np.float32)
    # cell centres as the reference forms them (double, stored to float)
    rows, cols = np.nonzero(dm != dg.nodata)
    ccx = (np.float64(dg.xll) + (cols + 0.5) * np.float64(dg.cs)).astype(np.float32).astype(np.float64)
    ccy = (np.float64(dg.yll) + (dg.nrows - 0.5 - rows) * np.float64(dg.cs)).astype(np.float32).astype(np.float64)
    near = near_cutoff_points(rng, ccx, ccy, h, 64, 1e-5 * h)
    sel = rng.integers(0, len(ccx), 8)
    sx = np.array([1, -1, 1, -1, 1, -1, 1, -1], np.float64)
    sy = np.array([1, 1, -1, -1, 1, 1, -1, -1], np.float64)
    a, b = 0.6 * 3 * h, 0.8 * 3 * h  # 3-4-5: a^2 + b^2 = 9 h^2 exactly
    on_x = (ccx[sel] + sx * np.where(np.arange(8) < 4, a, b)).astype(np.float32)
    on_y = (ccy[sel] + sy * np.where(np.arange(8) < 4, b, a)).astype(np.float32)
    in_x = np.nextafter(on_x, ccx[sel].astype(np.float32))  # one float step towards the centre
    x = np.concatenate([x, near[:, 0], on_x, in_x])
    y = np.concatenate([y, near[:, 1], on_y, on_y])
    w = rng.lognormal(0.0, 0.5, len(x)).astype(np.float32)
    hpp = np.full(len(x), h, np.float32)
    make_case(name, x, y, w, hpp, eg, em, dg, dm, -1, True, True)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
