"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset is involved: every input is generated from numpy's PCG64 with a
fixed seed.  Coordinates are drawn in float64 and rounded once to float32
(the reference reads coordinates as float, kde_cuda_kdtr_tiled.cu:1661-1700),
so every implementation sees the same values.  Mixture draws that fall outside
the domain are redrawn.  The "random polygon" mask is a star-shaped polygon
with 32 vertices (angles sorted uniform, radii uniform in a band around the
domain centre) rasterised by cell centre.

Workloads (sizes as named):
  small_uniform     10,000 uniform points in a 100 x 100 square, h = 2, all
                    cells valid at cell 1.0 (density and edge masks)
  single_large      1e6 points from a 50-component mixture in 1e4 x 1e4,
                    lognormal(0, 0.5) weights, density 1e4^2 at cell 1, edge
                    mask 2500^2 at cell 4, polygon mask, h = 50
  bandwidth_select  2e5 points, 20-component mixture in 5000^2, unit weights,
                    edge mask 1250^2 at cell 4, 64 log-spaced h in [5, 500]
  out_of_core       2e7 points (70 % from 500 components, 30 % uniform) in
                    4e4^2, density 4e4^2 at cell 1 in 4096^2 tiles, edge mask
                    8000^2 at cell 5, h = 30
Each builder takes a `scale` that shrinks the point count and raster sides
together (for tests), keeping densities and h unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

NODATA = -9999.0


@dataclass
class Grid:
    """Raster geometry as the reference's AsciiRaster holds it (float fields)."""

    ncols: int
    nrows: int
    xll: float
    yll: float
    cs: float
    nodata: float = NODATA

    def astuple(self):
        return (self.ncols, self.nrows, self.xll, self.yll, self.cs, self.nodata)


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def uniform_points(n, lo, hi, seed):
    r = _rng(seed)
    x = r.uniform(lo, hi, n).astype(np.float32)
    y = r.uniform(lo, hi, n).astype(np.float32)
    return x, y


def mixture_points(n, k, side, sigma_lo, sigma_hi, seed, background=0.0):
    """n points: (1-background) from k isotropic Gaussians with centres
    uniform in [0, side]^2 and sigma ~ U[sigma_lo, sigma_hi], equal mixture
    weights; the rest uniform.  Draws outside [0, side]^2 are redrawn."""
    r = _rng(seed)
    cx = r.uniform(0, side, k)
    cy = r.uniform(0, side, k)
    sg = r.uniform(sigma_lo, sigma_hi, k)
    n_bg = int(round(n * background))
    n_mix = n - n_bg
    xs = np.empty(n, np.float64)
    ys = np.empty(n, np.float64)
    comp = r.integers(0, k, n_mix)
    xs[:n_mix] = cx[comp] + sg[comp] * r.standard_normal(n_mix)
    ys[:n_mix] = cy[comp] + sg[comp] * r.standard_normal(n_mix)
    bad = np.nonzero((xs[:n_mix] < 0) | (xs[:n_mix] > side) | (ys[:n_mix] < 0) | (ys[:n_mix] > side))[0]
    while bad.size:
        c = comp[bad]
        xs[bad] = cx[c] + sg[c] * r.standard_normal(bad.size)
        ys[bad] = cy[c] + sg[c] * r.standard_normal(bad.size)
        sub = (xs[bad] < 0) | (xs[bad] > side) | (ys[bad] < 0) | (ys[bad] > side)
        bad = bad[sub]
    xs[n_mix:] = r.uniform(0, side, n_bg)
    ys[n_mix:] = r.uniform(0, side, n_bg)
    perm = r.permutation(n)
    return xs[perm].astype(np.float32), ys[perm].astype(np.float32)


def lognormal_weights(n, seed, sigma=0.5):
    return _rng(seed).lognormal(0.0, sigma, n).astype(np.float32)


def star_polygon(side, seed, nverts=32, rmin=0.35, rmax=0.5):
    r = _rng(seed)
    ang = np.sort(r.uniform(0, 2 * np.pi, nverts))
    rad = r.uniform(rmin, rmax, nverts) * side
    c = side / 2.0
    return np.stack([c + rad * np.cos(ang), c + rad * np.sin(ang)], 1)


def rasterize_polygon(verts, g: Grid, inside=1.0):
    """Even-odd fill by cell centre, one scanline per row (row 0 = top)."""
    out = np.full((g.nrows, g.ncols), g.nodata, np.float32)
    vx, vy = verts[:, 0], verts[:, 1]
    wx, wy = np.roll(vx, -1), np.roll(vy, -1)
    rows = np.arange(g.nrows)
    cy = g.yll + (g.nrows - 0.5 - rows) * g.cs
    cols_x = g.xll + (np.arange(g.ncols) + 0.5) * g.cs
    for i, yv in enumerate(cy):
        cross = (vy <= yv) != (wy <= yv)
        if not cross.any():
            continue
        t = (yv - vy[cross]) / (wy[cross] - vy[cross])
        xs = np.sort(vx[cross] + t * (wx[cross] - vx[cross]))
        for a, b in zip(xs[0::2], xs[1::2]):
            lo = np.searchsorted(cols_x, a, "left")
            hi = np.searchsorted(cols_x, b, "left")
            out[i, lo:hi] = inside
    return out


def all_valid(g: Grid, value=1.0):
    return np.full((g.nrows, g.ncols), value, np.float32)


def log_h_grid(lo=5.0, hi=500.0, n=64):
    k = np.arange(n)
    return (lo * (hi / lo) ** (k / (n - 1))).astype(np.float32)


def small_uniform(seed=0):
    x, y = uniform_points(10_000, 0.0, 100.0, seed)
    g = Grid(100, 100, 0.0, 0.0, 1.0)
    return dict(x=x, y=y, w=np.ones_like(x), h=2.0, density_grid=g, density_mask=all_valid(g),
                edge_grid=g, edge_mask=all_valid(g), edge=True)


def single_large(scale=1.0, seed=1):
    side = 10_000.0 * scale
    n = int(round(1_000_000 * scale * scale))
    x, y = mixture_points(n, 50, side, 50.0, 400.0, seed)
    w = lognormal_weights(n, seed + 1000)
    poly = star_polygon(side, seed + 2000)
    dg = Grid(int(round(side)), int(round(side)), 0.0, 0.0, 1.0)
    eg = Grid(int(round(side / 4.0)), int(round(side / 4.0)), 0.0, 0.0, 4.0)
    return dict(x=x, y=y, w=w, h=50.0, density_grid=dg, density_mask=None, polygon=poly,
                edge_grid=eg, edge_mask=rasterize_polygon(poly, eg), edge=True)


def bandwidth_select(scale=1.0, seed=2, nh=64):
    side = 5000.0 * scale
    n = int(round(200_000 * scale * scale))
    x, y = mixture_points(n, 20, side, 50.0, 400.0, seed)
    poly = star_polygon(side, seed + 2000)
    eg = Grid(int(round(side / 4.0)), int(round(side / 4.0)), 0.0, 0.0, 4.0)
    return dict(x=x, y=y, w=np.ones_like(x), hgrid=log_h_grid(5.0, 500.0, nh), polygon=poly,
                edge_grid=eg, edge_mask=rasterize_polygon(poly, eg), edge=True)


def out_of_core(scale=1.0, seed=3):
    side = 40_000.0 * scale
    n = int(round(20_000_000 * scale * scale))
    x, y = mixture_points(n, 500, side, 20.0, 200.0, seed, background=0.3)
    w = lognormal_weights(n, seed + 1000)
    poly = star_polygon(side, seed + 2000)
    dg = Grid(int(round(side)), int(round(side)), 0.0, 0.0, 1.0)
    eg = Grid(int(round(side / 5.0)), int(round(side / 5.0)), 0.0, 0.0, 5.0)
    return dict(x=x, y=y, w=w, h=30.0, density_grid=dg, density_mask=None, polygon=poly,
                edge_grid=eg, edge_mask=rasterize_polygon(poly, eg), edge=True, tile=4096)


def serving_requests(count, seed=4, n_lo=1_000, n_hi=2_000_000, side_lo=256, side_hi=8192):
    """The serving stream's requests: point count lognormal (median 3e4,
    sigma 1.5) clipped to [n_lo, n_hi], Gaussian-mixture points with a
    per-request seed, square raster side uniform in [side_lo, side_hi] at
    cell 1, h uniform in [5, 100] cells, edge correction (polygon mask at
    cell 4) for half of them; lognormal(0, 0.5) weights."""
    r = _rng(seed)
    out = []
    for k in range(count):
        n = int(np.clip(r.lognormal(np.log(3e4), 1.5), n_lo, n_hi))
        side = int(r.integers(side_lo, side_hi + 1))
        h = float(r.uniform(5.0, 100.0))
        edge = bool(r.random() < 0.5)
        x, y = mixture_points(n, 10, float(side), side / 40.0, side / 8.0, seed * 1000 + k)
        w = lognormal_weights(n, seed * 1000 + k + 500)
        g = Grid(side, side, 0.0, 0.0, 1.0)
        q = dict(x=x, y=y, w=w, h=h, grid=g, mask=None, edge_grid=None, edge_mask=None)
        if edge:
            eg = Grid(max(1, side // 4), max(1, side // 4), 0.0, 0.0, 4.0)
            q["edge_grid"] = eg
            q["edge_mask"] = rasterize_polygon(star_polygon(float(side), seed * 1000 + k + 700), eg)
        out.append(q)
    return out


def density_mask_window(poly, g: Grid, r0, c0, nr, nc):
    """Polygon mask for a window of a (possibly huge) density grid."""
    sub = Grid(nc, nr, g.xll + c0 * g.cs, g.yll + (g.nrows - r0 - nr) * g.cs, g.cs, g.nodata)
    return rasterize_polygon(poly, sub)
