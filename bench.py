"""Benchmark: kernel evaluations/s of the tiled fixed-bandwidth KDE on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mgk|reference]
                  [--workload single_large|bandwidth_select|out_of_core|serving|adaptive] [--scale S]

Workload (default): the single large KDE — 1,000,000 points from a
50-component Gaussian mixture in a 10,000 x 10,000 domain with lognormal(0,
0.5) weights, density raster 10,000 x 10,000 at cell 1 under a random
polygon mask (~80 % valid), edge-correction raster 2,500 x 2,500 at cell 4
with the same polygon, h = 50, FP32-compensated.  Seeded synthetic data.

One step = the whole path over device-resident inputs: boundary marking,
point-to-boundary distances, edge-correction weights, index build, density
over the full raster.  Unit of work = one kernel evaluation, i.e. one
(point, target) pair inside the 3h cutoff, target = valid density cell or
valid edge-mask cell; the count is algorithmic (the kernels count exactly the
oracle's pairs).  value = evals of all ranks / max-over-ranks step time.

Multi-GPU (torchrun): one study is split into contiguous row ranges of
balanced work, one per rank; a rank keeps the points within 3h of its rows
and computes their boundary distances, edge weights, index and density (no
collective touches the data path; strong scaling).  The bandwidth-selection
workload splits its edge weights by points (all-gather) and its
leave-one-out sums by queries (all-reduce of the nh partial sums).

--impl reference times the reference program's own CPU path (built from its
sources into oracle/_ref; the FP64 oracle port if that binary is absent) on
the host cores, on bounded crops of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

from mgpukde_tiled_b200 import synth  # noqa: E402

METRIC = "kernel evals/s (FP32-compensated, rel err <= 1e-6 vs FP64 oracle)"
UNIT = "evals/s"
REF_BIN = os.path.join(REPO, "oracle", "_ref", "mgkde_ref")
FLOP_PER_EVAL = 8.0  # 7 FP32 flops + 1 exp per in-cutoff pair (algorithmic)


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML in a background thread every 10 ms (read-only queries), or
    nvidia-smi -lms 200 when NVML is not importable."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []
        self.stop_flag = False

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.device)
            bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception:
            return self._start_smi()
        import threading

        def run():
            while not self.stop_flag:
                try:
                    sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, mx, [n for n, b in bits.items() if r & b]))
                except Exception:
                    pass
                time.sleep(0.01)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        t0 = time.time()
        while not self.samples and time.time() - t0 < 2.0:
            time.sleep(0.005)

    def _start_smi(self):
        if not shutil.which("nvidia-smi"):
            return
        fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={fields}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(1.0)

    def stop(self):
        if self.thread:
            self.stop_flag = True
            self.thread.join(timeout=2)
            rows = self.samples
            src = "nvml"
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            rows = []
            for line in open(self.path):
                f = [t.strip() for t in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    rows.append((float(f[1]), float(f[2]),
                                 [n for n, v in zip(self.NAMES, f[5:9]) if v.lower() == "active"]))
                except ValueError:
                    continue
            os.unlink(self.path)
            src = "nvidia-smi"
        else:
            return None
        if not rows:
            return None
        reasons = sorted({n for _, _, rs in rows for n in rs})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": float(max(r[1] for r in rows)),
                "reasons": reasons, "samples": len(rows), "source": src}


_ALL_CPUS = None


def bind_local_numa(device):
    """Runs this process on the host cores of the GPU's own NUMA node, so
    that page-locked buffers are allocated in memory next to the GPU's PCIe
    root (read-only sysfs queries; nothing about the GPU changes).  Returns
    the node, or None when the topology is not visible."""
    global _ALL_CPUS
    try:
        import torch
        p = torch.cuda.get_device_properties(device)
        bus = "%04x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        with open(f"/sys/bus/pci/devices/{bus}/numa_node") as f:
            node = int(f.read().strip())
        if node < 0:
            return None
        with open(f"/sys/devices/system/node/node{node}/cpulist") as f:
            cpus = set()
            for part in f.read().strip().split(","):
                a, _, b = part.partition("-")
                cpus.update(range(int(a), int(b or a) + 1))
        _ALL_CPUS = os.sched_getaffinity(0)
        cpus &= _ALL_CPUS
        if not cpus:
            return None
        os.sched_setaffinity(0, cpus)
        return node
    except Exception:
        return None


def unbind_numa():
    """All host cores again (the CPU baselines use every core)."""
    if _ALL_CPUS:
        try:
            os.sched_setaffinity(0, _ALL_CPUS)
        except Exception:
            pass


def build_workload(name, scale, seed):
    if name != "single_large":
        raise SystemExit(f"unknown workload {name}")
    c = synth.single_large(scale=scale, seed=seed)
    dg = c["density_grid"]
    c["density_mask"] = synth.rasterize_polygon(c["polygon"], dg)
    return c


# ------------------------------------------------------------------ CPU legs --
def pick_window(c, side):
    """Of a 5 x 5 grid of candidate windows over the middle of the raster,
    the one whose halo point count is the median: a representative sample."""
    dg = c["density_grid"]
    reach = 3.0 * c["h"]
    x, y = c["x"], c["y"]
    cands = []
    for fr in np.linspace(0.2, 0.8, 5):
        for fc in np.linspace(0.2, 0.8, 5):
            r0 = int(fr * (dg.nrows - side))
            c0 = int(fc * (dg.ncols - side))
            x0 = dg.xll + c0 * dg.cs
            y1 = dg.yll + (dg.nrows - r0) * dg.cs
            n = int(np.count_nonzero((x > x0 - reach) & (x < x0 + side * dg.cs + reach) &
                                     (y > y1 - side * dg.cs - reach) & (y < y1 + reach)))
            cands.append((n, r0, c0))
    cands.sort()
    _, r0, c0 = cands[len(cands) // 2]
    return r0, c0


def crop_inputs(c, side):
    """A side x side window of the density raster, its halo points (within
    3h) and their slice of everything."""
    dg = c["density_grid"]
    side = min(side, dg.nrows, dg.ncols)
    r0, c0 = pick_window(c, side)
    x0 = dg.xll + c0 * dg.cs
    x1 = x0 + side * dg.cs
    y1 = dg.yll + (dg.nrows - r0) * dg.cs
    y0 = y1 - side * dg.cs
    reach = 3.0 * c["h"]
    x, y = c["x"], c["y"]
    keep = (x > x0 - reach) & (x < x1 + reach) & (y > y0 - reach) & (y < y1 + reach)
    g = synth.Grid(side, side, np.float32(x0), np.float32(y0), dg.cs, dg.nodata)
    mask = (np.ones((side, side), np.float32) if c["density_mask"] is None
            else c["density_mask"][r0:r0 + side, c0:c0 + side])
    return dict(x=x[keep], y=y[keep], w=c["w"][keep], grid=g, mask=mask, window=(r0, c0, side, side))


def crop_evals(c, crop):
    import oracle_py as o
    eg = o.grid(*c["edge_grid"].astuple())
    b = o.mark_boundary(eg, c["edge_mask"])
    d2 = o.dist2_boundary(crop["x"], crop["y"], eg, b)
    ew, eev = o.edge_weights(crop["x"], crop["y"], c["h"], d2, eg, c["edge_mask"])
    den, dev = o.density(crop["x"], crop["y"], crop["w"], ew, c["h"], o.grid(*crop["grid"].astuple()), crop["mask"])
    return dev, eev, ew, den


def run_reference_binary(c, crop, threads):
    from mgpukde_tiled_b200 import tiff
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "p.csv"), "w") as f:
            f.write("x,y,h,w\n")
            for a, b, w in zip(crop["x"], crop["y"], crop["w"]):
                f.write("%.9g,%.9g,%.9g,%.9g\n" % (a, b, c["h"], w))
        eg = c["edge_grid"]
        tiff.write(os.path.join(d, "e.tif"), tiff.GeoRaster(c["edge_mask"], (float(eg.xll), float(eg.cs), 0.0,
                   float(eg.yll) + eg.nrows * float(eg.cs), 0.0, -float(eg.cs)), eg.nodata))
        g = crop["grid"]
        tiff.write(os.path.join(d, "d.tif"), tiff.GeoRaster(crop["mask"], (float(g.xll), float(g.cs), 0.0,
                   float(g.yll) + g.nrows * float(g.cs), 0.0, -float(g.cs)), g.nodata))
        p = subprocess.run([REF_BIN, "1", "p.csv", "e.tif", "d.tif", "-1", "1", "1", "0", "1", str(threads), "1",
                            "den_cpu.tif", "den_gpu.tif", "0"], cwd=d, capture_output=True, text=True, timeout=1800)
        if p.returncode != 0:
            raise RuntimeError(p.stdout[-1000:] + p.stderr[-1000:])
        t_den = float(re.search(r"KernelDesityEstimation took (\d+) ms", p.stdout).group(1))
        t_edge = float(re.search(r"EdgeCorrectionWeightsExact took (\d+) ms", p.stdout).group(1))
        return (t_den + t_edge) / 1e3


def run_reference_gpu(c, crop, threads):
    """The reference program's own CUDA path (KernelDesityEstimation_pPoints,
    kde_kernel_kdtr.cu:461-574, after CalcEdgeCorrectionWeights, :192-265) on
    the crop: mode 1, h_option -1, the OpenMP path skipped, one GPU.  Returns
    its printed edge-weight and tile-density times (ms, host clock around its
    launches, copies and halo extraction) and its density raster."""
    from mgpukde_tiled_b200 import tiff
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "p.csv"), "w") as f:
            f.write("x,y,h,w\n")
            for a, b, w in zip(crop["x"], crop["y"], crop["w"]):
                f.write("%.9g,%.9g,%.9g,%.9g\n" % (a, b, c["h"], w))
        eg = c["edge_grid"]
        tiff.write(os.path.join(d, "e.tif"), tiff.GeoRaster(c["edge_mask"], (float(eg.xll), float(eg.cs), 0.0,
                   float(eg.yll) + eg.nrows * float(eg.cs), 0.0, -float(eg.cs)), eg.nodata))
        g = crop["grid"]
        tiff.write(os.path.join(d, "d.tif"), tiff.GeoRaster(crop["mask"], (float(g.xll), float(g.cs), 0.0,
                   float(g.yll) + g.nrows * float(g.cs), 0.0, -float(g.cs)), g.nodata))
        p = subprocess.run([REF_BIN, "1", "p.csv", "e.tif", "d.tif", "-1", "1", "1", "1", "0", str(threads), "1",
                            "den_cpu.tif", "den_gpu.tif", "0"], cwd=d, capture_output=True, text=True, timeout=600)
        if p.returncode != 0:
            raise RuntimeError(p.stdout[-1000:] + p.stderr[-1000:])
        t_edge = float(re.search(r"CalcEdgeCorrectionWeights took (\d+) ms", p.stdout).group(1))
        t_den = sum(float(v) for v in re.findall(r"KernelDesityEstimation on tile \d+ took (\d+) ms", p.stdout))
        den = tiff.read(os.path.join(d, "den_gpu.tif")).data
        return t_edge, t_den, den


def reference_gpu_baseline(c, side=2048):
    """The reference's own CUDA kernels on this GPU, on a side x side crop of
    the workload with its halo points: evals/s of its edge weights plus tile
    density, and its raster's largest relative error against the FP64 oracle
    (its sums are float atomics)."""
    threads = os.cpu_count() or 1
    crop = crop_inputs(c, side)
    dev, eev, ew, den_ref = crop_evals(c, crop)
    t_edge, t_den, den = run_reference_gpu(c, crop, threads)
    valid = crop["mask"] != crop["grid"].nodata
    rel = np.abs(den[valid].astype(np.float64) - den_ref[valid]) / np.maximum(np.abs(den_ref[valid]), 1e-300)
    t = (t_edge + t_den) / 1e3
    return {"value": (dev + eev) / max(t, 1e-9), "unit": UNIT, "edge_ms": t_edge, "density_ms": t_den,
            "density_value": dev / max(t_den / 1e3, 1e-9), "evals": int(dev + eev),
            "max_rel_err": float(rel.max()), "kernels": "CalcEdgeCorrectionWeights + KernelDesityEstimation_pPoints",
            "sample": f"{side}x{side} density window with its {len(crop['x'])} halo points; the reference program "
                      f"(mode 1, h_option -1, OpenMP path skipped, 1 GPU), its printed edge-weight and tile-density "
                      f"times (host clock, ms)"}


def cpu_baseline(c, side=1024):
    """The reference's CPU path (or the FP64 oracle port) on a crop of the
    workload: a side x side density window with its halo points."""
    threads = os.cpu_count() or 1
    crop = crop_inputs(c, side)
    dev, eev, ew, den_ref = crop_evals(c, crop)
    if os.path.exists(REF_BIN):
        t = run_reference_binary(c, crop, threads)
        kind = "reference"
    else:
        import oracle_py as o
        o.set_threads(threads)
        t0 = time.perf_counter()
        o.density(crop["x"], crop["y"], crop["w"], ew, c["h"], o.grid(*crop["grid"].astuple()), crop["mask"])
        t = time.perf_counter() - t0
        kind = "port"
    sample = (f"{side}x{side} density window (median-density of 25 candidate windows) with its {len(crop['x'])} halo points "
              f"(density + edge-correction evals {dev + eev}); reference brute-force CPU path, "
              f"{'mode 1, h_option -1' if kind == 'reference' else 'FP64 oracle'}")
    return {"value": (dev + eev) / max(t, 1e-9), "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
            "seconds": t}


# ------------------------------------------------------------ accuracy legs --
def max_rel_err(got, ref, valid, rows=256):
    """Largest |got - ref| / |ref| over the valid cells, a band of rows at a
    time (bounded temporaries on rasters of 1e8-1e9 cells)."""
    m = 0.0
    for r in range(0, got.shape[0], rows):
        v = valid[r:r + rows]
        if not v.any():
            continue
        g = got[r:r + rows][v].astype(np.float64)
        f = np.asarray(ref[r:r + rows][v], np.float64)
        m = max(m, float(np.max(np.abs(g - f) / np.maximum(np.abs(f), 1e-300))))
    return m


def single_large_accuracy(c, rasters, ev_d, ev_e):
    """The whole study recomputed by the FP64 oracle on all host threads
    (boundary, distances and edge weights of every point, density of every
    cell of the raster), against each GPU raster in `rasters` (name ->
    host array): max relative error over the valid cells, NoData cells equal,
    and the in-cutoff pair counts equal."""
    import oracle_py as o
    threads = os.cpu_count() or 1
    o.set_threads(threads)
    dg, mask = c["density_grid"], c["density_mask"]
    t0 = time.perf_counter()
    eg = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(c["x"], c["y"], eg, o.mark_boundary(eg, c["edge_mask"]))
    ew, eev = o.edge_weights(c["x"], c["y"], c["h"], d2, eg, c["edge_mask"])
    den, dev = o.density(c["x"], c["y"], c["w"], ew, c["h"], o.grid(*dg.astuple()), mask)
    t = time.perf_counter() - t0
    valid = mask != dg.nodata
    out = {"scope": f"every cell of the {dg.nrows}x{dg.ncols} raster", "cells": int(valid.sum()),
           "nodata_cells": int(valid.size - valid.sum())}
    errs, nds = [], []
    for name, r in rasters.items():
        e = max_rel_err(r, den, valid)
        nd = bool(np.array_equal(r[~valid], mask[~valid]))
        out[f"max_rel_err_{name}"] = e
        out[f"nodata_cells_equal_{name}"] = nd
        errs.append(e)
        nds.append(nd)
    out.update({"max_rel_err": max(errs), "nodata_cells_equal": all(nds), "tolerance": 1e-6,
                "density_evals_equal": bool(dev == ev_d), "edge_evals_equal": bool(eev == ev_e),
                "oracle_density_evals": int(dev), "oracle_edge_evals": int(eev),
                "oracle_seconds": t, "oracle_threads": threads,
                "sample": "the FP64 oracle of the whole study against " + " and ".join(
                    {"step": "the last timed step's raster", "e2e": "the last end-to-end call's raster"}.get(k, k)
                    for k in rasters)})
    return out


def density_roofline(evals, kernel_s, nsm, sm_max_mhz, peak_kind, traffic, alg_bytes, hbm_gbs):
    """The roofline object of the density kernel's bench line.  The kernel is
    bound by FP32 issue: `achieved` is its algorithmic FLOP rate (8 flop-
    equivalents per in-cutoff pair) against the nominal FP32 peak (the
    measured peaks hold no FP32 figure).  `hbm` gives the same launch against
    the measured copy bandwidth: its algorithmic bytes (mask read plus
    output write) and its measured DRAM traffic per launch, as GB/s."""
    fp32_peak = nsm * 128 * 2 * sm_max_mhz * 1e6 / 1e12
    achieved = evals * FLOP_PER_EVAL / kernel_s / 1e12
    out = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
           "frac": achieved / fp32_peak, "traffic": traffic, "kernel": "k_density",
           "kernel_ms": kernel_s * 1e3, "flop_per_eval": FLOP_PER_EVAL,
           "peak_note": f"nominal FP32 FMA peak {nsm} SMs x 128 lanes x 2 x {sm_max_mhz:.0f} MHz "
                        f"(MEASURED_PEAKS.json has no FP32 figure; its clocks are {peak_kind})"}
    if traffic is not None:
        out["traffic_note"] = ("dram__bytes_read.sum + dram__bytes_write.sum of one full-size launch, from the ncu "
                               "capture summarised in profiles/k_density_traffic.txt (not measured in this run)")
    # the pipe utilisation behind frac (frac counts 8 flop-equivalents per in-cutoff pair, not issued ops)
    # (fma_pct: FMA-pipe instruction issue; fma_cycles_pct: cycles the FMA pipe is busy, in which a packed
    # f32x2 instruction counts twice)
    out["pipes_ncu"] = {"fma_pct": 30.3, "fma_cycles_pct": 40.7, "alu_pct": 33.8, "xu_pct": 14.0, "lsu_pct": 21.7,
                        "issue_active_pct": 71.2, "thread_inst_per_eval": 4.97,
                        "source": "ncu --set full of one half-scale launch, profiles/k_density_single_large_half.md "
                                  "(not measured in this run)"}
    if hbm_gbs:
        hbm_achieved = alg_bytes / kernel_s / 1e9
        out["hbm"] = {"achieved": hbm_achieved, "peak": hbm_gbs, "unit": "GB/s", "frac": hbm_achieved / hbm_gbs,
                      "algorithmic_bytes": alg_bytes,
                      "peak_note": f"measured copy bandwidth ({peak_kind})"}
    return out


def algo_roofline(evals, seconds, scope, device):
    """Roofline object of a workload whose time is several kernels: its
    algorithmic rate (8 flop-equivalents per in-cutoff pair, as for the
    density kernel) over `seconds` against the nominal FP32 peak.  `scope`
    says which kernels the time covers."""
    import torch

    peaks, peak_kind = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    nsm = torch.cuda.get_device_properties(device).multi_processor_count
    fp32_peak = nsm * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = evals * FLOP_PER_EVAL / seconds / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
            "traffic": None, "flop_per_eval": FLOP_PER_EVAL, "scope": scope,
            "peak_note": f"nominal FP32 FMA peak {nsm} SMs x 128 lanes x 2 x {sm_max:.0f} MHz "
                         f"(MEASURED_PEAKS.json has no FP32 figure; its clocks are {peak_kind})"}


def d2h_link_gbs(nbytes=256 << 20, reps=5):
    """Measured device -> page-locked host copy rate (GB/s): the bound of a
    workload that streams its output to host memory."""
    import torch

    dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    s = torch.cuda.current_stream()
    host.copy_(dev, non_blocking=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        host.copy_(dev, non_blocking=True)
    e1.record(s)
    torch.cuda.synchronize()
    return nbytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9


def run_reference_arm(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    c = build_workload(args.workload, args.scale, seed=1)
    side = 512
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(c, side)
        if k >= args.warmup:
            vals.append(cb)
    v = float(np.mean([b["value"] for b in vals]))
    secs = float(np.mean([b["seconds"] for b in vals]))
    cb = dict(vals[-1])
    cb["value"] = v
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)",
           "config": config_of(args), "cpu_baseline": cb,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def config_of(args):
    split = ("whole raster (one tile)" if args.gpus <= 1 else
             f"one study split into {args.gpus} row ranges of balanced work, one per GPU (no exchange)")
    return {"workload": f"{args.workload}: 1e6 mixture points (50 comps) in 1e4^2, lognormal weights, "
                        f"density 1e4^2 @ cell 1 polygon mask, edge mask 2500^2 @ cell 4, h=50"
                        + ("" if args.scale == 1.0 else f" (scaled x{args.scale})"),
            "scale": args.scale, "tile": split, "parallelism": f"rows x{args.gpus} (no exchange)",
            "l2": "inputs larger than L2 (density mask and output 400 MB each)",
            "host_numa_node": getattr(args, "numa_node", None)}


# ------------------------------------------------------------------ GPU arm --
def run_mgk(args):
    import torch
    import torch.distributed as dist

    import mgpukde_tiled_b200 as mk

    from mgpukde_tiled_b200 import shard

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    # one study; with N ranks each takes a contiguous range of rows of balanced work
    c = build_workload(args.workload, args.scale, seed=1)
    dg, eg = mk.Grid.of(c["density_grid"]), mk.Grid.of(c["edge_grid"])
    h = float(c["h"])
    row0, nrows = 0, dg.nrows
    if world > 1:
        row0, nrows = shard.split_rows(dg.nrows, world, shard.row_costs(c["x"], c["y"], h, c["density_grid"],
                                                                         c["density_mask"]))[rank]
    # the rows' halo: points within 3h of their cell centres (mgk_kde_raster_rows keeps the same)
    reach = 3.0 * h * (1.0 + 1e-6) + 1e-6 * float(dg.cs)
    y_top = float(np.float32(float(dg.yll) + (dg.nrows - 0.5 - row0) * float(dg.cs)))
    y_bot = float(np.float32(float(dg.yll) + (dg.nrows - 0.5 - (row0 + max(nrows, 1) - 1)) * float(dg.cs)))
    stream = torch.cuda.current_stream()
    ctx = mk.Context(local, stream=stream)
    dev = "cuda"
    dx = torch.from_numpy(c["x"]).to(dev)
    dy = torch.from_numpy(c["y"]).to(dev)
    dw = torch.from_numpy(c["w"]).to(dev)
    demask = torch.from_numpy(c["edge_mask"]).to(dev)
    ddmask = torch.from_numpy(c["density_mask"]).to(dev)
    dout = torch.empty((max(nrows, 1), dg.ncols), dtype=torch.float32, device=dev)
    pts = mk.Points.wrap(ctx, dx, dy, dw)
    em = mk.Raster.wrap(ctx, eg, demask)

    def step(count=False):
        mk.mark_boundary(ctx, em)
        p = pts if world == 1 else pts.select(ylo=y_bot - reach, yhi=y_top + reach)
        mk.calc_dist2_boundary(ctx, p, em, reach=reach)  # exact up to 3h: what the edge weights read
        ev_e = mk.edge_correction_weights(ctx, p, em, h, count=count)
        idx = mk.Index(ctx, p, h)
        ev_d = (mk.density_tile(ctx, idx, dg, row0, 0, nrows, dg.ncols, ddmask[row0:row0 + nrows], dout,
                                count=count) if nrows else 0)
        idx.close()
        if p is not pts:
            p.close()
        return ev_e, ev_d

    ev_e, ev_d = step(count=True)
    if world > 1:
        # the study's units: its density pairs (the ranks' rows partition them) and
        # its edge-correction pairs counted once (halo points repeat across ranks)
        mk.calc_dist2_boundary(ctx, pts, em, reach=reach)
        ev_e = mk.edge_correction_weights(ctx, pts, em, h, count=True)
    evals = ev_e + ev_d
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dens_ms = []
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
        dens_ms.append(ctx.last_density_ms)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = (ctx.kernel_launches - l0) / args.steps
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    # the last timed step's raster, for the whole-raster accuracy check
    step_raster = dout.cpu().numpy() if (rank == 0 and world == 1 and not args.no_accuracy) else None
    total_evals = evals
    if world > 1:  # the study's evals: every rank's density pairs plus the edge pairs once
        ev_t = torch.tensor([float(ev_d)], device=dev, dtype=torch.float64)
        dist.all_reduce(ev_t, op=dist.ReduceOp.SUM)
        total_evals = int(ev_t.item()) + ev_e
    value = total_evals / (ms_max / 1e3)

    # end to end: the C ABI from pinned host buffers (inputs H2D and the raster D2H every step)
    hx = torch.from_numpy(c["x"]).pin_memory()
    hy = torch.from_numpy(c["y"]).pin_memory()
    hw = torch.from_numpy(c["w"]).pin_memory()
    hem = torch.from_numpy(c["edge_mask"]).pin_memory()
    hdm = torch.from_numpy(c["density_mask"]).pin_memory()
    hout = torch.empty((max(nrows, 1), dg.ncols), dtype=torch.float32).pin_memory()
    e2e_steps = max(1, min(args.steps, 5))

    def e2e_step():
        if world == 1:
            mk.kde_raster(ctx, hx.numpy(), hy.numpy(), hw.numpy(), h, dg, hdm.numpy(), eg, hem.numpy(),
                          out=hout.numpy())
        elif nrows:
            mk.kde_raster_rows(ctx, hx.numpy(), hy.numpy(), hw.numpy(), h, dg, row0, nrows,
                               hdm.numpy()[row0:row0 + nrows], eg, hem.numpy(), out=hout.numpy())

    e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = torch.tensor([e0.elapsed_time(e1) / e2e_steps], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_val = total_evals / (float(e2e_ms.item()) / 1e3)
    # bytes of the whole job (every rank uploads all points and the edge mask, and its own rows);
    # mgk_kde_raster packs the density mask on the host and sends 1 bit per cell, in rows of
    # whole 16-byte groups (128 cells)
    mask_row_bytes = (dg.ncols + 127) // 128 * 16
    h2d = 4 * world * (3 * len(c["x"]) + c["edge_mask"].size) + mask_row_bytes * dg.nrows
    d2h = 4 * dg.nrows * dg.ncols

    # the plain FP64 GPU form of the density gather on the same raster (one launch, after warm-up)
    fp64_form = None
    if not args.no_fp64_form and world == 1:
        idx = mk.Index(ctx, pts, h)
        mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, ddmask, dout, fp64=True)
        f64_ms = []
        for _ in range(2):
            mk.density_tile(ctx, idx, dg, 0, 0, dg.nrows, dg.ncols, ddmask, dout, fp64=True)
            f64_ms.append(ctx.last_density_ms)
        idx.close()
        f64 = float(np.mean(f64_ms))
        dens_ms_mean = float(np.mean(dens_ms))
        fp64_form = {"value": ev_d / (f64 / 1e3), "unit": UNIT, "kernel": "k_density_fp64", "kernel_ms": f64,
                     "fp32c_kernel_value": ev_d / (dens_ms_mean / 1e3),
                     "fp32c_over_fp64": f64 / dens_ms_mean}

    # roofline of the density kernel (FP32-issue bound; no measured FP32 peak exists, nominal used)
    peaks, peak_kind = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    dens_s = float(np.mean(dens_ms)) / 1e3
    traffic = None
    tp = os.path.join(REPO, "profiles", "k_density_traffic.txt")
    if os.path.exists(tp) and args.scale == 1.0:
        with open(tp) as f:
            for line in f:
                if line.startswith("bytes_per_launch:"):
                    traffic = int(line.split(":", 1)[1].split()[0])
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)", "config": config_of(args),
        "evals_per_step": total_evals, "density_evals": total_evals - ev_e, "edge_evals": ev_e,
        "rows": [int(row0), int(nrows)] if world > 1 else None,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": float(e2e_ms.item()),
                "note": "density mask crosses the link as 1 bit per cell (packed on host threads inside the call)"},
        "gpu_launches": launches,
        "roofline": density_roofline(ev_d, dens_s, nsm, sm_max, peak_kind, traffic,
                                     4 * dg.nrows * dg.ncols * 2, peaks.get("hbm_gbs")),
        "clocks": clocks,
        "fp64_form": fp64_form,
    }
    if rank == 0 and world == 1:
        unbind_numa()
        if not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline(c)
            except Exception as e:  # reported, not fatal
                out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        if not args.no_reference_gpu and os.path.exists(REF_BIN):
            try:
                rg = reference_gpu_baseline(c)
                rg["ratio_step"] = value / rg["value"]
                rg["ratio_density_kernel"] = (ev_d / dens_s) / rg["density_value"]
                out["reference_gpu"] = rg
            except Exception as e:  # reported, not fatal
                out["reference_gpu"] = {"value": None, "error": str(e)[:200]}
        if step_raster is not None:
            out["accuracy"] = single_large_accuracy(c, {"step": step_raster, "e2e": hout.numpy()}, ev_d, ev_e)
    if rank == 0:
        print(json.dumps(out))
    pts.close()
    em.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------- bandwidth selection (C2) --
def loo_cpu_check(c, hgrid, logl, pts, nsmall=16):
    """The FP64 oracle's LogLikelihood (edge weights at h, leave-one-out sum)
    for the nsmall smallest h of the grid, all host threads: the CPU baseline
    (evals/s over those h) and the relative error of the GPU's logL there."""
    import oracle_py as o
    threads = os.cpu_count() or 1
    o.set_threads(threads)
    eg = o.grid(*c["edge_grid"].astuple())
    d2 = o.dist2_boundary(c["x"], c["y"], eg, o.mark_boundary(eg, c["edge_mask"]))
    ks = list(np.argsort(hgrid)[:nsmall])
    t0 = time.perf_counter()
    refs = [o.loglik_at(c["x"], c["y"], c["w"], d2, eg, c["edge_mask"], float(hgrid[k])) for k in ks]
    t = time.perf_counter() - t0
    ev = sum(r[1] for r in refs)
    rel = [abs(float(logl[k]) - r[0]) / abs(r[0]) for k, r in zip(ks, refs)]
    cb = {"value": ev / max(t, 1e-9), "unit": UNIT, "cores": threads, "kind": "port", "seconds": t,
          "sample": f"FP64 oracle LogLikelihood (edge weights + leave-one-out) at the {nsmall} smallest h of the grid "
                    f"({', '.join('%.2f' % hgrid[k] for k in ks)}), all {len(c['x'])} points: {ev} evals"}
    acc = {"logl_max_rel_err": float(max(rel)), "h_checked": [float(hgrid[k]) for k in ks],
           "sample": "GPU logL of the timed batch against the FP64 oracle at those h"}
    return cb, acc


def loo_argmax_check(c, hgrid, logl, best, radius=2):
    """The FP64 oracle's LogLikelihood (its own boundary distances and edge
    weights at each h, then the leave-one-out sum) at the GPU's argmax index
    and its `radius` neighbours on each side: the argmax over that
    neighbourhood must be the same index, and the margin to the runner-up is
    reported next to the largest relative logL error there."""
    import oracle_py as o
    threads = os.cpu_count() or 1
    o.set_threads(threads)
    eg, em = o.grid(*c["edge_grid"].astuple()), c["edge_mask"]
    x, y, w = c["x"], c["y"], c["w"]
    t0 = time.perf_counter()
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    ks = [k for k in range(best - radius, best + radius + 1) if 0 <= k < len(hgrid)]
    refs = [o.loglik_at(x, y, w, d2, eg, em, float(hgrid[k])) for k in ks]
    t = time.perf_counter() - t0
    ref_ll = np.array([r[0] for r in refs])
    gl = np.asarray(logl, np.float64)
    k_or = ks[int(np.argmax(ref_ll))]
    masked = gl.copy()
    masked[best] = -np.inf
    runner = int(np.argmax(masked))
    ib = ks.index(best)
    or_others = np.delete(ref_ll, ib)
    rel = np.abs(gl[ks] - ref_ll) / np.abs(ref_ll)
    return {"argmax_gpu": int(best), "argmax_oracle": int(k_or), "argmax_equal": bool(k_or == best),
            "h_best": float(hgrid[best]), "indices_checked": ks,
            "h_checked": [float(hgrid[k]) for k in ks],
            "logl_oracle": [float(v) for v in ref_ll], "logl_gpu": [float(gl[k]) for k in ks],
            "logl_max_rel_err": float(rel.max()),
            "runner_up_gpu": runner, "margin_gpu": float(gl[best] - gl[runner]),
            "margin_oracle": float(ref_ll[ib] - or_others.max()) if or_others.size else None,
            "margin_rel": float((gl[best] - gl[runner]) / abs(gl[best])),
            "oracle_seconds": t, "oracle_threads": threads,
            "sample": f"FP64 oracle LogLikelihood at the GPU's argmax index and {radius} neighbours on each side, "
                      f"all {len(x)} points"}


def run_bandwidth_select(args):
    """One step = one batched bandwidth selection: point-to-boundary distances,
    then edge weights and the leave-one-out log likelihood for 64 log-spaced
    h in [5, 500] and the argmax, in one graph launch.  Evals = edge-mask
    cells plus point pairs inside the cutoff, summed over the 64 h."""
    import torch
    import torch.distributed as dist

    import mgpukde_tiled_b200 as mk
    from mgpukde_tiled_b200 import shard

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:  # one selection split over the ranks (edge weights by points, queries by groups)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    c = synth.bandwidth_select(scale=args.scale, seed=2, nh=64)
    eg = mk.Grid.of(c["edge_grid"])
    stream = torch.cuda.current_stream()
    ctx = mk.Context(local, stream=stream)
    dx = torch.from_numpy(c["x"]).cuda()
    dy = torch.from_numpy(c["y"]).cuda()
    dw = torch.from_numpy(c["w"]).cuda()
    demask = torch.from_numpy(c["edge_mask"]).cuda()
    pts = mk.Points.wrap(ctx, dx, dy, dw)
    em = mk.Raster.wrap(ctx, eg, demask)
    mk.mark_boundary(ctx, em)
    hgrid = c["hgrid"]
    shared_ev = [0, 0]

    reach = 3.0 * float(np.max(hgrid)) * (1.0 + 1e-6)  # distances exact up to 3 h_max

    def step():
        mk.calc_dist2_boundary(ctx, pts, em, reach=reach)
        if world == 1:
            return mk.log_likelihood_batch(ctx, pts, em, hgrid)
        tot, am, ev = shard.loo_loglik_shared(ctx, pts, em, hgrid, rank, world)
        shared_ev[:] = ev
        return tot, am

    logl, best = step()
    if world == 1:
        ev_edge, ev_loo = ctx.last_loo_evals
    else:  # the shares partition both counts: sum them over ranks
        t = torch.tensor([float(v) for v in shared_ev], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        ev_edge, ev_loo = int(t[0].item()), int(t[1].item())
    evals = ev_edge + ev_loo
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loo_ms, batch_ms = [], []
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
        loo_ms.append(ctx.last_loo_ms)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    launches = (ctx.kernel_launches - l0) / args.steps
    out = {"metric": METRIC, "value": evals / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)",
           "config": {"workload": f"bandwidth_select: {len(c['x'])} mixture points (20 comps) in "
                                  f"{c['edge_grid'].ncols * 4}^2, unit weights, edge mask "
                                  f"{c['edge_grid'].ncols}^2 @ cell 4, 64 log-spaced h in [5, 500]",
                      "scale": args.scale, "l2": "per-h edge weights and point records stay L2-resident",
                      "parallelism": ("one GPU" if world == 1 else
                                      f"one selection over {world} GPUs: edge weights by point share + "
                                      f"all-gather, leave-one-out sums by query share + all-reduce")},
           "evals_per_step": evals, "edge_evals": ev_edge, "loo_evals": ev_loo,
           "batch_ms": float(np.mean(loo_ms)), "argmax": best, "h_best": float(hgrid[best]),
           "gpu_launches": launches, "clocks": clocks,
           "roofline": algo_roofline(evals, float(np.mean(loo_ms)) / 1e3,
                                     "one LOO batch: per-h edge weights, k_loo_multi (about 90 % of it), prep, "
                                     "finish and argmax (the batch's CUDA-event time)", local)}
    if rank == 0:
        if world == 1:
            unbind_numa()
            if not args.no_cpu_baseline:
                out["cpu_baseline"], out["accuracy"] = loo_cpu_check(c, hgrid, logl, pts)
            if not args.no_accuracy:
                out.setdefault("accuracy", {})["argmax"] = loo_argmax_check(c, hgrid, logl, best)
        print(json.dumps(out))
    pts.close()
    em.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------- adaptive bandwidths (h_option 2) --
def adaptive_cpu_baseline(scale, gpu_logl=None):
    """One adaptive likelihood evaluation of the FP64 oracle port, all host
    threads, on the workload's points and mask: edge weights at h, pilot
    density, bandwidths, edge weights at hs, leave-one-out density."""
    import oracle_py as o

    threads = os.cpu_count() or 1
    o.set_threads(threads)
    c = synth.bandwidth_select(scale=scale, seed=5, nh=2)
    x, y, w = c["x"], c["y"], c["w"]
    eg, em = o.grid(*c["edge_grid"].astuple()), c["edge_mask"]
    d2 = o.dist2_boundary(x, y, eg, o.mark_boundary(eg, em))
    h = o.rule_of_thumb(x, y, w)
    t0 = time.perf_counter()
    ew1, e1 = o.edge_weights(x, y, h, d2, eg, em)
    den0, p0 = o.point_density(x, y, w, ew1, h, self_term=True)
    hs = o.adaptive_bandwidths(den0, h, -0.5)
    ew2, e2 = o.edge_weights(x, y, 0.0, d2, eg, em, hs=hs)
    den1, p1 = o.point_density(x, y, w, ew2, 0.0, hs=hs, self_term=False)
    t = time.perf_counter() - t0
    ev = e1 + e2 + p0 + p1
    ref_ll = float(np.sum(np.log(np.maximum(den1, float(np.float32(1e-14))))))
    return {"value": ev / max(t, 1e-9), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one adaptive likelihood evaluation (h = rule of thumb {h:.3f}, alpha = -0.5) of the FP64 "
                      f"oracle on the workload ({len(x)} points, edge mask "
                      f"{c['edge_grid'].ncols}^2): {e1 + e2} edge-mask cells, {p0 + p1} pairs",
            "seconds": t,
            "accuracy": None if gpu_logl is None else
            {"logl_rel_err": abs(gpu_logl - ref_ll) / abs(ref_ll), "h": h, "alpha": -0.5,
             "sample": "the GPU's adaptive LogLikelihood at the rule-of-thumb h and alpha -0.5 against the "
                       "FP64 oracle's"}}


def run_adaptive(args):
    """One step = one adaptive-bandwidth search (h_option 2) on device-resident
    points and edge mask: point-to-boundary distances, the Hooke-Jeeves search
    over (h, alpha) from the rule-of-thumb h0 (each likelihood: edge weights
    at h, pilot density, bandwidths, edge weights at hs, leave-one-out density
    at hs), then the bandwidths of the optimum, copied to the host.
    Evals = edge-mask cells plus point pairs inside the cutoffs, summed over
    every likelihood the search evaluates.  e2e: the same search through the
    public API from host arrays (points and mask uploaded every step)."""
    import torch

    import mgpukde_tiled_b200 as mk

    rank, world, local = env_rank()
    if world > 1:
        raise SystemExit("adaptive runs on one GPU (replicas only)")
    torch.cuda.set_device(local)
    c = synth.bandwidth_select(scale=0.5 * args.scale, seed=5, nh=2)
    eg = mk.Grid.of(c["edge_grid"])
    h0 = mk.rule_of_thumb(c["x"], c["y"], c["w"])
    stream = torch.cuda.current_stream()
    ctx = mk.Context(local, stream=stream)
    dx = torch.from_numpy(c["x"]).cuda()
    dy = torch.from_numpy(c["y"]).cuda()
    dw = torch.from_numpy(c["w"]).cuda()
    demask = torch.from_numpy(c["edge_mask"]).cuda()
    pts = mk.Points.wrap(ctx, dx, dy, dw)
    em = mk.Raster.wrap(ctx, eg, demask)
    mk.mark_boundary(ctx, em)

    def step():
        mk.calc_dist2_boundary(ctx, pts, em)
        return mk.adaptive_bandwidths(ctx, pts, em, h0)

    h, alpha, lmax, iters, _ = step()
    edge_ev, pair_ev = ctx.last_loo_evals
    evals = edge_ev + pair_ev
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (ctx.kernel_launches - l0) / args.steps

    # end to end from host arrays: upload points and mask, boundary, search, hs to host
    hx, hy, hw = (torch.from_numpy(c[k]).pin_memory() for k in ("x", "y", "w"))
    hmask = torch.from_numpy(c["edge_mask"]).pin_memory()

    def e2e_step():
        p = mk.Points.upload(ctx, hx.numpy(), hy.numpy(), hw.numpy())
        r = mk.Raster.upload(ctx, eg, hmask.numpy())
        mk.mark_boundary(ctx, r)
        mk.calc_dist2_boundary(ctx, p, r)
        out = mk.adaptive_bandwidths(ctx, p, r, h0)
        p.close()
        r.close()
        return out

    e2e_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    n = len(c["x"])
    out = {"metric": METRIC, "value": evals / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)",
           "config": {"workload": f"adaptive: {n} mixture points (20 comps) in {eg.ncols * 4}^2, unit weights, "
                                  f"edge mask {eg.ncols}^2 @ cell 4, Hooke-Jeeves over (h, alpha) from the "
                                  f"rule-of-thumb h0 = {h0:.3f}, alpha0 = -0.5",
                      "scale": args.scale, "l2": "point records and edge weights stay L2-resident"},
           "evals_per_step": evals, "edge_evals": edge_ev, "pair_evals": pair_ev,
           "search": {"h": h, "alpha": alpha, "lmax": lmax, "iterations": iters},
           "e2e": {"value": evals / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                   "h2d_bytes_per_step": int(3 * 4 * n + c["edge_mask"].nbytes), "d2h_bytes_per_step": int(4 * n)},
           "gpu_launches": launches, "clocks": clocks,
           "roofline": algo_roofline(evals, ms / 1e3, "one Hooke-Jeeves search: point densities, bandwidths, "
                                                      "edge weights and leave-one-out sums of every step", local)}
    if not args.no_cpu_baseline:
        unbind_numa()
        mk.calc_dist2_boundary(ctx, pts, em)
        gpu_ll = mk.loglik_adaptive(ctx, pts, em, h0, -0.5)
        out["cpu_baseline"] = adaptive_cpu_baseline(0.5 * args.scale, gpu_ll)
        out["accuracy"] = out["cpu_baseline"].pop("accuracy", None)
    print(json.dumps(out))
    pts.close()
    em.close()
    ctx.close()
    return 0


# ---------------------------------------------------------- out of core (C3) --
def run_out_of_core(args):
    """One step = the whole out-of-core job from device-resident points and
    edge mask: boundary, distances, edge weights, index, then the density
    raster in 4096 x 4096 tiles streamed to a host array (the raster never
    exists on the device as a whole: two tile buffers)."""
    import torch

    import mgpukde_tiled_b200 as mk

    import torch.distributed as dist

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:  # one job per rank (seed 3 + rank), no data exchange
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    c = synth.out_of_core(scale=args.scale, seed=3 + rank)
    dg, eg = mk.Grid.of(c["density_grid"]), mk.Grid.of(c["edge_grid"])
    h = float(c["h"])
    tile = int(c["tile"])
    stream = torch.cuda.current_stream()
    ctx = mk.Context(local, stream=stream)
    dx = torch.from_numpy(c["x"]).cuda()
    dy = torch.from_numpy(c["y"]).cuda()
    dw = torch.from_numpy(c["w"]).cuda()
    demask = torch.from_numpy(c["edge_mask"]).cuda()
    pts = mk.Points.wrap(ctx, dx, dy, dw)
    em = mk.Raster.wrap(ctx, eg, demask)
    # tiles land here through the library's copy sink (page-locked: direct 2-D copies)
    host = torch.empty((dg.nrows, dg.ncols), dtype=torch.float32, pin_memory=True).numpy()

    def step(count=False):
        mk.mark_boundary(ctx, em)
        mk.calc_dist2_boundary(ctx, pts, em, reach=3.0 * h * (1.0 + 1e-6))
        ev_e = mk.edge_correction_weights(ctx, pts, em, h, count=count)
        idx = mk.Index(ctx, pts, h)
        ev_d = mk.density_stream(ctx, idx, dg, tile, host, count=count)
        idx.close()
        return ev_e, ev_d

    ev_e, ev_d = step(count=True)
    evals = ev_e + ev_d
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = ctx.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (ctx.kernel_launches - l0) / args.steps
    ntiles = ((dg.nrows + tile - 1) // tile) * ((dg.ncols + tile - 1) // tile)
    total_evals = evals
    if world > 1:  # the slowest rank's time, every rank's evals
        red = torch.tensor([ms, float(evals)], device="cuda", dtype=torch.float64)
        t_max, ev_sum = red[:1].clone(), red[1:].clone()
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.all_reduce(ev_sum, op=dist.ReduceOp.SUM)
        ms, total_evals = float(t_max.item()), int(ev_sum.item())
    out = {"metric": METRIC, "value": total_evals / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)",
           "config": {"workload": f"out_of_core: {len(c['x'])} points (70% from 500 Gaussians, 30% uniform) in "
                                  f"{dg.ncols}^2, density {dg.ncols}^2 @ cell 1 in {ntiles} tiles of {tile}^2 "
                                  f"streamed to host memory, edge mask {eg.ncols}^2 @ cell 5, h={h:g}",
                      "scale": args.scale, "l2": "output streamed through HBM tile buffers to the host"},
           "evals_per_step": evals, "density_evals": ev_d, "edge_evals": ev_e,
           "output_bytes": int(host.nbytes), "output_gb_s": host.nbytes / (ms / 1e3) / 1e9,
           "gpu_launches": launches, "clocks": clocks}
    # the job streams 6.4 GB to page-locked host memory: bound by the copy link
    link = d2h_link_gbs()
    achieved = host.nbytes / (ms / 1e3) / 1e9
    out["roofline"] = {"bound": "d2h link", "achieved": achieved, "peak": link, "unit": "GB/s", "frac": achieved / link,
                       "traffic": None, "algorithmic_bytes": int(host.nbytes),
                       "peak_note": "device -> page-locked host copy rate measured in this run (256 MB, 5 copies)",
                       "fp32_view": algo_roofline(total_evals, ms / 1e3, "the whole job (every kernel and copy)",
                                                  local)}
    if rank == 0 and world == 1:
        unbind_numa()
        if not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline(c, side=512)
            except Exception as e:  # reported, not fatal
                out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        if not args.no_accuracy:
            out["accuracy"] = out_of_core_accuracy(c, host, tile)
    if rank == 0:
        print(json.dumps(out))
    pts.close()
    em.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def out_of_core_accuracy(c, host, tile):
    """Whole output tiles of the streamed raster recomputed by the FP64 oracle
    on all host threads: two corner tiles (the top-left one and the ragged
    bottom-right one), two edge tiles and an interior one.  Each tile's
    oracle sees every point within 3h of it, with its own boundary distances
    and edge weights.  The raster has no density mask (every cell valid)."""
    import oracle_py as o
    threads = os.cpu_count() or 1
    o.set_threads(threads)
    dg = c["density_grid"]
    nt_r, nt_c = (dg.nrows + tile - 1) // tile, (dg.ncols + tile - 1) // tile
    picks = [(0, 0), (0, nt_c // 2), (nt_r // 2, 0), (nt_r // 2, nt_c // 2), (nt_r - 1, nt_c - 1)]
    reach = 3.0 * c["h"]
    t0 = time.perf_counter()
    eg = o.grid(*c["edge_grid"].astuple())
    bnd = o.mark_boundary(eg, c["edge_mask"])
    x, y, w = c["x"], c["y"], c["w"]
    tiles = []
    for tr, tc in picks:
        r0, c0 = tr * tile, tc * tile
        nr, nc = min(tile, dg.nrows - r0), min(tile, dg.ncols - c0)
        x0 = float(dg.xll) + c0 * float(dg.cs)
        x1 = x0 + nc * float(dg.cs)
        y1 = float(dg.yll) + (dg.nrows - r0) * float(dg.cs)
        y0 = y1 - nr * float(dg.cs)
        keep = (x > x0 - reach - 1) & (x < x1 + reach + 1) & (y > y0 - reach - 1) & (y < y1 + reach + 1)
        xs, ys, ws = x[keep], y[keep], w[keep]
        d2 = o.dist2_boundary(xs, ys, eg, bnd)
        ew, _ = o.edge_weights(xs, ys, c["h"], d2, eg, c["edge_mask"])
        den, dev = o.density(xs, ys, ws, ew, c["h"], o.grid(*dg.astuple()), None, window=(r0, c0, nr, nc))
        got = host[r0:r0 + nr, c0:c0 + nc]
        tiles.append({"tile": [int(tr), int(tc)], "cells": int(nr * nc), "points": int(keep.sum()),
                      "evals": int(dev), "max_rel_err": max_rel_err(got, den, np.ones((nr, nc), bool))})
    t = time.perf_counter() - t0
    return {"scope": f"{len(tiles)} whole output tiles of {tile}^2 (ragged at the raster's edge)",
            "tiles": tiles, "max_rel_err": max(tt["max_rel_err"] for tt in tiles), "tolerance": 1e-6,
            "cells": sum(tt["cells"] for tt in tiles), "nodata_cells": 0,
            "oracle_seconds": t, "oracle_threads": threads,
            "sample": "the last timed job's streamed raster against the FP64 oracle, tile by tile"}


# ------------------------------------------------------------ serving (C4) --
def run_serving(args):
    """Poisson arrivals of whole KDE requests into the serving loop, swept
    over arrival rates; per rate: completed requests/s, evals/s and the p50 /
    p99 of submit-to-result latency.  The line's value is the evals/s at the
    highest rate (saturation)."""
    import torch

    import mgpukde_tiled_b200 as mk

    rank, world, local = env_rank()
    if world > 1:
        raise SystemExit("serving runs one server per GPU (replicas only)")
    torch.cuda.set_device(local)
    count = max(4, int(round(args.serve_requests * args.scale)))
    reqs = synth.serving_requests(count, seed=4)
    rates = [8.0, 32.0, 128.0, 512.0, 2048.0]
    rng = np.random.default_rng(7)

    # page-locked result rasters, allocated once outside the arrival process
    outs = [torch.empty((q["grid"].nrows, q["grid"].ncols), dtype=torch.float32, pin_memory=True).numpy()
            for q in reqs]

    def submit(srv, q, k=None):
        return srv.submit(q["x"], q["y"], q["w"], q["h"], mk.Grid.of(q["grid"]), q["mask"],
                          mk.Grid.of(q["edge_grid"]) if q["edge_grid"] is not None else None, q["edge_mask"],
                          out=outs[k] if k is not None else None)

    rows = []
    with mk.Server(local, tile=2048, max_active=8) as srv:
        # warm-up: one untimed pass of the whole request set, so kernels are
        # loaded and the device pool holds blocks of every size the stream needs
        for t in [submit(srv, q, k) for k, q in enumerate(reqs)]:
            srv.wait(t)
        for rate in rates:
            arr = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
            t0 = time.perf_counter()
            tickets = []
            for k, (a, q) in enumerate(zip(arr, reqs)):
                dt = t0 + a - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                tickets.append(submit(srv, q, k))
            res = [srv.wait(t)[1] for t in tickets]
            wall = time.perf_counter() - t0
            lat = np.array([r["total_ms"] for r in res])
            ev = sum(r["evals"] for r in res)
            rows.append({"rate_req_s": rate, "completed_req_s": len(res) / wall, "evals_s": ev / wall,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "mean_queue_ms": float(np.mean([r["queue_ms"] for r in res])), "evals": int(ev)})
        st = srv.stats()
    top = rows[-1]
    out = {"metric": "served evals/s at saturation (mixed-request p50/p99 ms alongside)", "value": top["evals_s"],
           "unit": "evals/s", "n_gpus": 1, "steps": len(rates), "warmup": count, "ms_per_step": None,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded PCG64)",
           "config": {"workload": f"serving: {count} requests per rate, N lognormal [1e3, 2e6], side U[256, 8192], "
                                  f"h U[5, 100], edge correction on half; Poisson arrivals; one untimed "
                                  f"pass of the request set first; largest-first admission, up to 4 tiles per "
                                  f"tick",
                      "output_bytes": int(sum(o.nbytes for o in outs)),
                      "tile": 2048, "max_active": 8, "host_numa_node": getattr(args, "numa_node", None)},
           "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "sweep": rows,
           "server": {k: st[k] for k in ("ticks", "tiles", "max_batch", "completed")}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mgk", choices=["mgk", "reference"])
    ap.add_argument("--workload", default="single_large")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-form", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="serving workload: requests per offered rate (p99 is taken over them)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference program's own CUDA kernels on a crop")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP64 oracle check of the whole output (minutes of host CPU at full scale)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    args.numa_node = bind_local_numa(env_rank()[2])
    if args.workload == "bandwidth_select":
        return run_bandwidth_select(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "out_of_core":
        return run_out_of_core(args)
    if args.workload == "adaptive":
        return run_adaptive(args)
    return run_mgk(args)


if __name__ == "__main__":
    sys.exit(main())
