"""Loads the golden fixtures (reference outputs on seeded and sample inputs)
and rebuilds the oracle's answer for each, exactly as the reference's CPU
path sequences the steps (kde_cuda_kdtr_tiled.cu:484-873)."""
import glob
import os

import numpy as np

import oracle_py as o

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(os.path.splitext(os.path.basename(p))[0]
               for p in glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load(case):
    z = np.load(os.path.join(HERE, "golden", case + ".npz"))
    d = {k: z[k] for k in z.files}
    if not int(d["sample_weights"]):
        d["w"] = np.ones_like(d["x"])
    d["eg"] = o.grid(*d["edge_grid"])
    d["dg"] = o.grid(*d["density_grid"])
    d["hs"] = d["h_pp"] if int(d["hoption"]) == -1 else None
    return d


def oracle_run(d):
    """Oracle pipeline: boundary -> distance -> bandwidth -> edge weights -> density."""
    x, y, w = d["x"], d["y"], d["w"]
    eg, em = d["eg"], d["edge_mask"]
    out = {}
    out["h0"] = o.rule_of_thumb(x, y, w)
    d2 = None
    if int(d["edge"]):
        b = o.mark_boundary(eg, em)
        d2 = o.dist2_boundary(x, y, eg, b)
        out["boundary"], out["dist2"] = b, d2
    h = out["h0"]
    hs = d["hs"]
    if int(d["hoption"]) == 1:
        h, _ = o.mle_fixed_bandwidth(x, y, w, d2, eg, em, out["h0"])
    if int(d["hoption"]) == 2:
        # adaptive bandwidths (Hooke-Jeeves over h0, alpha; main :548-573)
        h, alpha, lmax, hs, it = o.adaptive_search(x, y, w, d2 if int(d["edge"]) else None, eg, em, out["h0"])
        out["alpha"], out["lmax"], out["hj_iterations"], out["hs"] = alpha, lmax, it, hs
    out["h"] = h
    if int(d["edge"]):
        ew, out["edge_evals"] = o.edge_weights(x, y, h, d2, eg, em, hs=hs)
    else:
        ew, out["edge_evals"] = np.ones(len(x)), 0
    out["ew"] = ew
    out["density"], out["density_evals"] = o.density(x, y, w, ew, h, d["dg"], d["density_mask"], hs=hs)
    return out


def match_rows(x, y, pnts):
    """Row i of the reference's points CSV -> input index (by printed x, y)."""
    key = {("%f" % a, "%f" % b): i for i, (a, b) in enumerate(zip(x, y))}
    return np.array([key[("%f" % a, "%f" % b)] for a, b in pnts[:, :2]])
