"""Host-side pieces on CPU: the reference command line of mgkde_tiled
(argument checks, inputs, rule-of-thumb printout) and the TIFF codecs."""
import os
import subprocess

import numpy as np
import pytest

from golden_cases import load
from mgpukde_tiled_b200 import synth, tiff

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "mgpukde_tiled_b200", "_lib", "mgkde_tiled")


def write_case_files(d, case, with_h=False):
    """The case's points CSV (x,y,w; or x,y,h,w with the per-point bandwidth
    column that h_option -1 reads) and its two masks as GeoTIFFs."""
    g = load(case)
    with open(os.path.join(d, "p.csv"), "w") as f:
        if with_h:
            f.write("x,y,h,w\n")
            for a, b, hh, w in zip(g["x"], g["y"], g["h_pp"], g["w"]):
                f.write("%.9g,%.9g,%.9g,%.9g\n" % (a, b, hh, w))
        else:
            f.write("x,y,w\n")
            for a, b, w in zip(g["x"], g["y"], g["w"]):
                f.write("%.9g,%.9g,%.9g\n" % (a, b, w))
    for name, grid, mask in (("e.tif", g["eg"], g["edge_mask"]), ("d.tif", g["dg"], g["density_mask"])):
        gt = (float(grid.xll), float(grid.cs), 0.0, float(grid.yll) + grid.nrows * float(grid.cs), 0.0,
              -float(grid.cs))
        tiff.write(os.path.join(d, name), tiff.GeoRaster(mask, gt, float(grid.nodata)))
    return g


def run_cli(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


def test_cli_rejects_bad_arguments(tmp_path):
    p = run_cli(["0", "100"], tmp_path)
    assert p.returncode == 1 and "Incorrect arguments" in p.stdout
    p = run_cli("0 100 1 1 3 1 0 1 0 1 1 a.tif b.tif 0".split(), tmp_path)
    assert p.returncode == 1 and "unknown h_option 3" in p.stdout
    p = run_cli("0 100 1 1 -1 1 0 1 0 1 1 a.tif b.tif 0".split(), tmp_path)
    assert p.returncode == 1 and "bandwidth option -1 in mode 0" in p.stdout


def test_cli_reads_inputs_like_the_reference(tmp_path):
    g = write_case_files(str(tmp_path), "redwood_h0")
    p = run_cli("1 p.csv e.tif d.tif 0 1 0 1 0 1 1 a.tif b.tif 0".split(), tmp_path)
    assert "Rule of thumb bandwidth h0: %.5f" % float(g["ref_h0"]) in p.stdout
    assert "Number of points: 62" in p.stdout
    assert "Number of cells (density estimation): 16384" in p.stdout


HELPER = r"""
#include "tiff_io.hpp"
#include <cstdio>
int main(int argc, char** argv) {
    mgk_tiff::Raster r; std::string err;
    if (!mgk_tiff::read_tiff(argv[1], r, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 1; }
    FILE* f = std::fopen(argv[2], "wb");
    double hdr[9] = {(double)r.ncols, (double)r.nrows, r.gt[0], r.gt[1], r.gt[3], r.gt[5],
                     r.has_nodata ? 1.0 : 0.0, r.nodata, 0.0};
    std::fwrite(hdr, 8, 9, f);
    std::fwrite(r.data.data(), 4, r.data.size(), f);
    std::fclose(f);
    if (argc > 3) {  // write back through the tiled writer
        if (!mgk_tiff::write_tiff(argv[3], r, 64)) return 2;
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def reader(tmp_path_factory):
    d = tmp_path_factory.mktemp("tiffhelper")
    src = d / "h.cpp"
    src.write_text(HELPER)
    exe = d / "h"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "mgpukde_tiled_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    return str(exe)


def read_with_cpp(reader, path, tmp, back=None):
    out = os.path.join(tmp, "dump.bin")
    args = [reader, path, out] + ([back] if back else [])
    subprocess.run(args, check=True)
    raw = open(out, "rb").read()
    hdr = np.frombuffer(raw[:72], np.float64)
    data = np.frombuffer(raw[72:], np.float32).reshape(int(hdr[1]), int(hdr[0]))
    return hdr, data


def test_tiff_python_writer_cpp_reader_and_back(reader, tmp_path):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((37, 53)).astype(np.float32)
    a[3, 4] = -9999.0
    gt = (100.5, 2.0, 0.0, 900.0, 0.0, -2.0)
    p = str(tmp_path / "a.tif")
    tiff.write(p, tiff.GeoRaster(a, gt, -9999.0))
    back = str(tmp_path / "b.tif")
    hdr, d = read_with_cpp(reader, p, str(tmp_path), back)
    assert np.array_equal(d, a)
    assert tuple(hdr[2:6]) == (gt[0], gt[1], gt[3], gt[5]) and hdr[6] == 1 and hdr[7] == -9999.0
    r = tiff.read(back)  # tiled output of the C++ writer, read by the Python reader
    assert np.array_equal(r.data, a) and r.geotransform == gt and r.nodata == -9999.0


@pytest.mark.parametrize("compression", ["raw", "tiff_lzw"])
def test_tiff_reader_on_third_party_files(reader, tmp_path, compression):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(1)
    for dt in (np.float32, np.uint8, np.int16):
        a = (rng.random((41, 29)) * 100).astype(dt)
        p = str(tmp_path / f"x_{np.dtype(dt).name}_{compression}.tif")
        Image.fromarray(a).save(p, compression=compression)
        _, d = read_with_cpp(reader, p, str(tmp_path))
        assert np.array_equal(d, a.astype(np.float32))


def test_reference_sample_masks_read_identically(reader, tmp_path):
    """The reference's sample GeoTIFF (tiled, GDAL-written), stored in the fixture."""
    g = load("redwood_h0")
    gt = (float(g["eg"].xll), float(g["eg"].cs), 0.0, float(g["eg"].yll) + 128 * float(g["eg"].cs), 0.0,
          -float(g["eg"].cs))
    p = str(tmp_path / "m.tif")
    tiff.write(p, tiff.GeoRaster(g["edge_mask"], gt, float(g["eg"].nodata)))
    _, d = read_with_cpp(reader, p, str(tmp_path))
    assert np.array_equal(d, g["edge_mask"])
