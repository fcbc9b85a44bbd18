"""Pins the FP64 oracle to the reference program's own outputs.

The fixtures hold what the reference (built from its sources, CPU path) wrote
for seeded inputs and for its sample data.  The reference accumulates in FP32,
so agreement is at FP32 level; NoData cells, the edge-weight short-circuit
(weight exactly 1.0) and the printed bandwidths must match exactly (to the
printed digits)."""
import numpy as np
import pytest

import oracle_py as o
from golden_cases import CASES, load, match_rows, oracle_run


@pytest.fixture(scope="module")
def runs():
    return {c: (load(c), oracle_run(load(c))) for c in CASES}


def test_cases_present():
    assert {"redwood_h0", "redwood_h1", "uniform_c0", "poly_fixed", "poly_varh",
            "uniform_h0_noedge", "loo_h1", "redwood_h2", "poly_h2", "c1_crop_h50", "c3_crop_h30"} <= set(CASES)


@pytest.mark.parametrize("case", CASES)
def test_rule_of_thumb_matches_printed(runs, case):
    d, r = runs[case]
    assert abs(r["h0"] - float(d["ref_h0"])) <= 5e-6 * max(1.0, abs(r["h0"]))


@pytest.mark.parametrize("case", CASES)
def test_density_matches_reference(runs, case):
    d, r = runs[case]
    ref = d["ref_density"].astype(np.float64)
    nd = d["density_mask"] == d["dg"].nodata
    assert np.array_equal(ref[nd], r["density"][nd])
    v = ~nd
    den = r["density"][v]
    # FP32 accumulation in the reference vs FP64 here; with adaptive bandwidths
    # (h_option 2) the per-point h themselves carry the reference's FP32 pilot
    # density and geometric mean (relative ~1e-6), amplified up to ~7x in K_h
    tol = 3e-5 if int(d["hoption"]) == 2 else 3e-6
    rel = np.abs(den - ref[v]) / np.maximum(np.abs(den), 1e-30)
    assert rel.max() < tol, rel.max()


@pytest.mark.parametrize("case", CASES)
def test_edge_weights_match_reference_csv(runs, case):
    d, r = runs[case]
    P = d["ref_pnts"]
    idx = match_rows(d["x"], d["y"], P)
    ew = r["ew"][idx]
    # the CSV prints 6 decimals; the reference sums up to ~3e4 window cells in FP32
    assert np.all(np.abs(P[:, 3] - ew) <= 6e-7 + 5e-6 * np.abs(ew))
    assert np.array_equal(P[:, 3] == 1.0, ew == 1.0)


def test_golden_section_matches_printed(runs):
    for case in ("redwood_h1", "loo_h1"):
        d, r = runs[case]
        assert abs(r["h"] - float(d["ref_hopt"])) <= 5e-6 * max(1.0, r["h"]) + 5e-6


def test_binned_density_equals_brute_force():
    d = load("poly_varh")
    x, y, w, hs = d["x"], d["y"], d["w"], d["hs"]
    ew = np.linspace(0.9, 1.3, len(x))
    a, ea = o.density(x, y, w, ew, 0.0, d["dg"], d["density_mask"], hs=hs)
    b, eb = o.density(x, y, w, ew, 0.0, d["dg"], d["density_mask"], hs=hs, brute=True)
    assert ea == eb
    np.testing.assert_allclose(a, b, rtol=1e-13, atol=0)


def test_sort_order_is_stable_by_distance():
    d2 = np.array([3.0, 1.0, 3.0, 0.5, 1.0])
    assert list(o.sort_order(d2)) == [3, 1, 4, 0, 2]


def test_adaptive_bandwidths_match_reference_csv(runs):
    """h_option 2: the final per-point bandwidths of the Hooke-Jeeves search
    (pntsCPU.csv column h, printed with 6 decimals) and the resulting
    density raster match the reference."""
    for case in ("redwood_h2", "poly_h2"):
        d, r = runs[case]
        P = d["ref_pnts"]
        idx = match_rows(d["x"], d["y"], P)
        hs = r["hs"][idx].astype(np.float64)
        assert np.all(np.abs(P[:, 2] - hs) <= 6e-7 + 2e-5 * np.abs(hs)), np.abs(P[:, 2] - hs).max()
        assert r["hj_iterations"] >= 1


def test_adaptive_likelihood_is_the_loo_of_the_pilot_bandwidths():
    d = load("poly_h2")
    x, y, w = d["x"], d["y"], d["w"]
    eg, em = d["eg"], d["edge_mask"]
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    h, alpha = 5.0, -0.4
    ll, hs = o.loglik_adaptive(x, y, w, d2, eg, em, h, alpha)
    ew, _ = o.edge_weights(x, y, h, d2, eg, em)
    den0, _ = o.point_density(x, y, w, ew, h, self_term=True)
    gml = np.exp(np.mean(np.log(den0)))
    np.testing.assert_allclose(hs, (h * (den0 / gml) ** alpha).astype(np.float32), rtol=1e-6)
    ew2, _ = o.edge_weights(x, y, 0.0, d2, eg, em, hs=hs)
    den1, _ = o.point_density(x, y, w, ew2, 0.0, hs=hs, self_term=False)
    assert abs(ll - np.sum(np.log(np.maximum(den1, float(np.float32(1e-14)))))) <= 1e-9 * abs(ll)


def cutoff_rule_disagreements(x, y, hs, g, mask):
    """Pairs (point, valid cell of g) that the oracle's cutoff test and the
    reference's classify differently.  The oracle forms dx = x_cell - x_p
    exactly in double; the reference's Distance2 (kde_cuda_kdtr_tiled.cu:50-55)
    subtracts the two floats in float and widens the rounded difference.
    Both then test dx^2 + dy^2 < 9 h^2 in double with h^2 a float product.
    Returns (disagreements, pairs within 3h + one cell of each other, those
    of the pairs whose float dx or dy was rounded)."""
    nd = g.nodata
    diff = 0
    pairs = 0
    rounded = 0
    cs = np.float64(g.cs)
    for px, py, hp in zip(x, y, hs):
        h2 = np.float64(np.float32(hp) * np.float32(hp))
        reach = 3.0 * float(hp) + float(cs)
        c0 = max(0, int(np.floor((float(px) - reach - float(g.xll)) / float(cs))))
        c1 = min(g.ncols - 1, int(np.ceil((float(px) + reach - float(g.xll)) / float(cs))))
        r0 = max(0, int(np.floor(g.nrows - 0.5 - (float(py) + reach - float(g.yll)) / float(cs))))
        r1 = min(g.nrows - 1, int(np.ceil(g.nrows - 0.5 - (float(py) - reach - float(g.yll)) / float(cs))))
        if c0 > c1 or r0 > r1:
            continue
        cols = np.arange(c0, c1 + 1)
        rows = np.arange(r0, r1 + 1)
        cx = (np.float64(g.xll) + (cols + 0.5) * cs).astype(np.float32)
        cy = (np.float64(g.yll) + (g.nrows - 0.5 - rows) * cs).astype(np.float32)
        ok = mask[r0:r1 + 1, c0:c1 + 1] != nd
        dxe = cx.astype(np.float64) - np.float64(px)
        dye = cy.astype(np.float64) - np.float64(py)
        dxr = (cx - np.float32(px)).astype(np.float64)
        dyr = (cy - np.float32(py)).astype(np.float64)
        ine = (dxe[None, :] ** 2 + dye[:, None] ** 2) < 9.0 * h2
        inr = (dxr[None, :] ** 2 + dyr[:, None] ** 2) < 9.0 * h2
        diff += int(np.count_nonzero((ine != inr) & ok))
        pairs += int(np.count_nonzero(ok))
        rounded += int(np.count_nonzero(((dxe != dxr)[None, :] | (dye != dyr)[:, None]) & ok))
    return diff, pairs, rounded


@pytest.mark.parametrize("case", CASES)
def test_cutoff_rules_agree_on_every_fixture(runs, case):
    """The oracle's exact dx and the reference's float-rounded dx classify
    every (point, cell) pair of the fixtures the same way.  Float subtraction
    of two floats within a factor of two of each other is exact (Sterbenz),
    so the rules can differ only for pairs whose difference exceeds one of
    the two coordinates, i.e. near the coordinate origin; the counts here
    cover the density and the edge-mask rasters with each case's bandwidths.
    At the large coordinates of the c1/c3 crops no float difference rounds at
    all (the two rules see the same d^2); near the origin of the small cases
    with cells within 3h of it many do, and none of those flips a cutoff
    decision."""
    d, r = runs[case]
    x, y = d["x"], d["y"]
    hs = r.get("hs") if r.get("hs") is not None else d["hs"]
    if hs is None:
        hs = np.full(len(x), r["h"], np.float32)
    dd, dp, dr = cutoff_rule_disagreements(x, y, hs, d["dg"], d["density_mask"])
    ed, ep, er = cutoff_rule_disagreements(x, y, hs, d["eg"], d["edge_mask"]) if int(d["edge"]) else (0, 0, 0)
    assert dp > 0
    assert dd == 0 and ed == 0, (case, dd, dp, ed, ep)
    if case.startswith(("c1_", "c3_")):
        assert dr == 0 and er == 0, (case, dr, er)
    elif case in ("poly_fixed", "uniform_c0", "redwood_h0"):  # cells within 3h of the origin
        assert dr + er > 0, case
