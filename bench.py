#!/usr/bin/env python
"""Throughput of the GraGLeS_3D level-set timestep on B200.

Workload (default): a 256^3 voxel domain, 20,000 grains from a Voronoi tessellation of
seeded uniform-random points with uniformly random orientations, Read-Shockley
grain-boundary energies (15 degree cutoff), the misorientation mobility model and the
convolution correction on, 10-voxel box border, TimeStepSize 0.2 (the reference's
non-periodic domain with the boundary grain).  ``--workload voronoi-128`` runs the
isotropic 128^3 / 2,000-grain workload instead.  A *step* is one full timestep of the
loop (convolution with its correction, list update, comparison, marching cubes, element
mesh, redistancing, box bookkeeping) over every live grain box.  The unit of work is a
voxel-update: one box voxel carried through one timestep (the sum of n^3 over the boxes
the step convolves).

Headline: the mixed path (FP32 storage, per-axis circulant convolution, FP64
volume tallies).  The FP64 path (bit-exact with the reference) runs beside it
and the maximum per-grain relative volume difference between the two is reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gg|reference]

N > 1 runs one independent replica per GPU (the path shares nothing between
grains of different simulations); launch it with torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-updates/s per timestep, mixed vs FP64 path on 1 B200, at vol err ≤1e-3"
UNIT = "voxel-updates/s"
HULL_CAPACITY = 12000  # triangles per hull for the correction's element build
WORKLOADS = {
    # the configuration the mixed-over-FP64 target is quoted on
    "anisotropic-256": (dict(workload="voronoi-256^3-20000-grains-read-shockley-mobility-correction", domain=256,
                             grains=20000, border=10, time_step=0.2, seed=1003),
                        dict(correction=True, unique_energies=False, mobility_model=True,
                             hull_capacity=HULL_CAPACITY)),
    "voronoi-128": (dict(workload="voronoi-128^3-2000-grains-isotropic", domain=128, grains=2000, border=10,
                         time_step=0.2, seed=1002), {}),
    # the larger configurations: one path at a time (--paths mixed), the pool sized to
    # the initial boxes times pool_factor so that the state fits the 180 GB of HBM
    "stored-energy-384": (dict(workload="voronoi-384^3-100000-grains-lognormal-stored-energy-5pct-nuclei",
                               domain=384, grains=100000, border=10, time_step=0.2, seed=1004, generator="c4",
                               pool_factor=1.3),
                          dict(correction=True, unique_energies=False, mobility_model=True, stored_energy=True,
                               hull_capacity=4000)),
    "laguerre-512": (dict(workload="laguerre-512^3-250000-grains-lognormal-radii-isotropic", domain=512,
                          grains=250000, border=10, time_step=0.2, seed=1005, generator="laguerre",
                          pool_factor=1.03), dict(correction=False)),
}
WORKLOAD = dict(WORKLOADS["anisotropic-256"][0])
PHYSICS = dict(WORKLOADS["anisotropic-256"][1])  # GrainHandler physics keywords of the workload


# ----------------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------------
def microstructure():
    from gragles_3d_b200 import microstructure as msgen

    gen = WORKLOAD.get("generator", "voronoi")
    if gen == "c4":
        ms = msgen.c4(WORKLOAD["domain"], WORKLOAD["grains"], seed=WORKLOAD["seed"])
    elif gen == "laguerre":
        ms = msgen.laguerre(WORKLOAD["domain"], WORKLOAD["grains"], seed=WORKLOAD["seed"])
    else:
        ms = msgen.voronoi(WORKLOAD["domain"], WORKLOAD["grains"], seed=WORKLOAD["seed"])
    ext, counts = ms.grain_extents()
    return ms, ext, counts


def handler(gg, ms, ext, counts, precision, device):
    """A GrainHandler of the workload (its physics and, for the large configurations, a
    pool of pool_factor times the initial boxes' voxels)."""
    from gragles_3d_b200 import microstructure as msgen

    extra = {}
    if "pool_factor" in WORKLOAD:
        e6 = np.asarray(ext).reshape(-1, 6).astype(np.int64)
        side = np.maximum.reduce([e6[:, 1] - e6[:, 0], e6[:, 3] - e6[:, 2], e6[:, 5] - e6[:, 4]]) + 1 \
            + 2 * WORKLOAD["border"]
        need = int(((side ** 3 + 31) // 32 * 32)[np.asarray(counts) > 0].sum())
        extra["pool_voxels"] = int(WORKLOAD["pool_factor"] * need)
    gh = gg.GrainHandler(WORKLOAD["domain"], WORKLOAD["border"], WORKLOAD["time_step"], ms.n_grains,
                         precision=precision, device=device, **PHYSICS, **extra)
    return gh, (lambda: _prepare(gh, ms, msgen))


def _prepare(gh, ms, msgen):
    if PHYSICS.get("correction"):
        gh.set_orientations(ms.euler)
    if PHYSICS.get("stored_energy"):
        gh.set_stored_energy(msgen.stored_energy_of(ms.stored_energy))


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# algorithmic (compulsory) bytes per voxel-update by stage and precision
STAGE_BYTES = {
    "mixed": {"ms_convolution": 8, "ms_comparison": 12, "ms_levelset": 4, "ms_redistancing": 8},
    "fp64": {"ms_convolution": 16, "ms_comparison": 20, "ms_levelset": 8, "ms_redistancing": 16},
}


def source_digest(path: str) -> str:
    import hashlib

    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()[:16]


def measured_traffic(kernel: str, voxels: float):
    """DRAM bytes (read + write) of one launch of `kernel` over `voxels` box voxels,
    scaled from the ncu capture summarised in profiles/dram_traffic.json (bytes per
    voxel-update of the captured launch).  Returns (bytes or None, note): None when no
    capture is recorded, or when the kernel's source has changed since the capture (the
    record keeps a digest of the source it was made from)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(path):
        return None, "no capture recorded"
    with open(path) as f:
        rec = json.load(f).get(kernel)
    if rec is None:
        return None, "no capture recorded"
    src = os.path.join(ROOT, "gragles_3d_b200", "csrc", rec.get("source", ""))
    if not os.path.isfile(src) or source_digest(src) != rec.get("source_sha256"):
        return None, "stale: the kernel source changed after the capture"
    return rec["bytes_per_voxel_update"] * voxels, rec.get("workload", "")


def run_device(gg, precision, ms, ext, counts, steps, warmup, device, dist, keep=False):
    """Device-resident run: state loaded before the timed region."""
    import torch

    gh, prepare = handler(gg, ms, ext, counts, precision, device)
    gh.load(ms.labels, ext, counts)
    gh.default_lists()
    prepare()
    for _ in range(warmup):
        gh.step()
    reps = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        ev0.record()
        for _ in range(steps):
            reps.append(gh.step())
        ev1.record()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms_elapsed = ev0.elapsed_time(ev1)
    st = gh.stats()
    vol = st.volume.copy()
    ex = st.exists.copy()
    if keep:
        return reps, ms_elapsed, clk.summary(), vol, ex, gh
    gh.close()
    return reps, ms_elapsed, clk.summary(), vol, ex


def bench_config(world: int) -> dict:
    """The workload keys both arms report (identical for the GPU and the reference arm)."""
    return dict(WORKLOAD, parallelism=f"replicas{world}",
                l2="inputs larger than L2 (box pool >= 0.3 GB per arena)")


def over_bound_causes(rel, ids, vol_ref, boxes):
    """The grains above 1e-3 relative volume difference, by the cause each falls under:
    a box that reaches a domain-wall plane (where the boundary grain's value is exactly
    0), else a grain of under 50 voxels, else other."""
    N, gb = WORKLOAD["domain"], WORKLOAD["border"]
    lo, hi = gb - 1, N + gb - 1
    out = {"wall": 0, "under_50_voxels": 0, "other": 0}
    for r, g in zip(rel, ids):
        if r <= 1e-3:
            continue
        b = boxes[g]
        if any(b[2 * a] <= lo or b[2 * a + 1] > hi for a in range(3)):
            out["wall"] += 1
        elif vol_ref[g] * N ** 3 < 50:
            out["under_50_voxels"] += 1
        else:
            out["other"] += 1
    return out


def max_sdf_difference(gh_a, gh_b, exists):
    """max |SDF_a - SDF_b| over the current SDF of every grain both runs hold in the same
    box, and how many existing grains hold different boxes."""
    worst, differ = 0.0, 0
    for g in np.nonzero(exists)[0]:
        if g == 0:
            continue
        box_a, a = gh_a.sdf(int(g), 1)
        box_b, b = gh_b.sdf(int(g), 1)
        if box_a != box_b:
            differ += 1
            continue
        if a.size:
            worst = max(worst, float(np.abs(a - b).max()))
    return worst, differ


def run_e2e(gg, precision, ms, ext, counts, steps, warmup, device):
    """Through the public API with host buffers: upload, steps, per-step read-back.
    One untimed pass of `warmup` steps first, then three timed passes of `steps`."""
    import torch

    # the step inputs sit in pinned host memory (the tensor keeps it alive; numpy views it)
    pinned = torch.from_numpy(np.ascontiguousarray(ms.labels)).pin_memory()
    labels = pinned.numpy()

    def one_pass(n, timed):
        gh, prepare = handler(gg, ms, ext, counts, precision, device)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        t0 = time.perf_counter()
        gh.load(labels, ext, counts)
        gh.default_lists()
        prepare()
        t_setup = time.perf_counter() - t0
        vox = 0
        for _ in range(n):
            vox += gh.step()["voxel_updates"]
            gh.stats()
        ev1.record()
        torch.cuda.synchronize()
        gh.close()
        return vox, ev0.elapsed_time(ev1), t_setup * 1e3

    one_pass(max(warmup, 1), False)
    # three timed passes, the median reported: a pass's set-up includes the device
    # allocations of gg_load_state, whose time varies with the driver's memory state
    passes = sorted((one_pass(steps, True) for _ in range(3)), key=lambda r: r[1])
    vox, ms_elapsed, ms_setup = passes[1]
    G1 = ms.n_grains + 1
    h2d = labels.nbytes + ext.astype(np.int32).nbytes + counts.astype(np.int64).nbytes
    if PHYSICS.get("correction"):
        h2d += ms.euler.astype(np.float64).nbytes
    if PHYSICS.get("stored_energy"):
        h2d += ms.n_grains * 8
    d2h = G1 * (1 + 8 + 8 + 24 + 4)
    return {"value": vox / (ms_elapsed / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d // steps),
            "d2h_bytes_per_step": int(d2h), "ms": ms_elapsed, "ms_setup": ms_setup}


# ----------------------------------------------------------------------------------
# reference CPU path (the reference's own solver, compiled from its sources)
# ----------------------------------------------------------------------------------
def run_reference_cpu(ms, steps: int, warmup: int, threads: int):
    """Time `steps` loop iterations after `warmup` of the compiled reference on the
    host cores, on the full workload (loops warmup .. warmup + steps - 1; loop 0 is the
    one without the convolution correction).  Returns (voxel-updates/s, sample
    description, cores, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refdump
    from gragles_3d_b200 import microstructure as msgen

    if os.path.exists(refdump.REF_BINARY):
        with tempfile.TemporaryDirectory() as d:
            msgen.write_mode4(ms, d)
            msgen.write_parameters(os.path.join(d, "parameters.xml"), n_grains=ms.n_grains,
                                   border=WORKLOAD["border"], steps=warmup + steps, threads=threads,
                                   time_step=WORKLOAD["time_step"], correction=bool(PHYSICS.get("correction")),
                                   unique_energies=PHYSICS.get("unique_energies", True),
                                   mobility_factor=bool(PHYSICS.get("mobility_model")))
            # the initial boxes' SDF records are needed only when loop 0 is timed
            res, _ = refdump.run_case(d, threads=threads, timeout=3600, init=warmup == 0)
        lt = res["loop_time"]
        # voxels convolved in loop t: boxes of the grains alive entering loop t
        vox = {}
        if res["init_sdf"]:
            vox[0] = sum(int(np.prod([r.box[1] - r.box[0]] * 3)) for r in res["init_sdf"].values())
        for loop, st in res["stats"].items():
            vox[loop + 1] = sum((b[1] - b[0]) ** 3 for (d_, b) in st.values() if d_[0] == 1.0)
        t = lt[warmup + steps] - lt[warmup]
        v = sum(vox[l] for l in range(warmup, warmup + steps))
        sample = (f"reference solver (g++ -O2, OpenMP, shim DFT) on the full {WORKLOAD['workload']} workload: "
                  f"loops {warmup}..{warmup + steps - 1} of {warmup + steps + 1} timed, {v} voxel-updates "
                  f"in {t:.2f} s")
        return v / t, sample, threads, "reference"
    # the C restatement (single thread) on a smaller slice of the loop
    import pyoracle

    ext, counts = ms.grain_extents()
    sim = pyoracle.OracleSim(ms.n, WORKLOAD["border"], WORKLOAD["time_step"], ms.labels, ext, counts)
    sim.step()
    t0 = time.perf_counter()
    sim.step()
    t = time.perf_counter() - t0
    v = sim.last_voxels()
    return v / t, f"oracle restatement, 1 thread, 1 timestep of the full workload ({v} voxel-updates)", 1, "port"


REF_LOOPS = 2  # loops the host reference times per run (each takes it tens of seconds on 256^3)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ms, _, _ = microstructure()
    threads = os.cpu_count() or 1
    # a bounded sample: loop 0 (no correction) runs untimed, then at most REF_LOOPS loops
    # of the requested steps are timed, so that the run ends within a few minutes
    value, sample, cores, kind = run_reference_cpu(ms, min(args.steps, REF_LOOPS), 1, threads)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": bench_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def aggregate_replicas(elapsed_ms: float, voxels: float, dist, device: str = "cuda"):
    """Whole-job figures over independent replicas: the slowest rank's time and the
    sum of every rank's voxel-updates (every rank takes the same two collectives)."""
    if dist is None:
        return float(elapsed_ms), float(voxels)
    import torch

    t = torch.tensor([float(elapsed_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    v = torch.tensor([float(voxels)], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.SUM)
    return float(t[0]), float(v[0])


# ----------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gg", choices=["gg", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--paths", default="both", choices=["both", "mixed", "fp64"],
                    help="profiling aid: run only one precision path")
    ap.add_argument("--domain", type=int, default=None, help="profiling aid: smaller domain of the same kind")
    ap.add_argument("--grains", type=int, default=None, help="profiling aid: grain count for --domain")
    ap.add_argument("--workload", default="anisotropic-256", choices=sorted(WORKLOADS),
                    help="anisotropic-256 (default): the 256^3 / 20,000-grain anisotropic workload with the "
                         "correction; voronoi-128: the isotropic 128^3 / 2,000-grain workload; "
                         "stored-energy-384 (384^3, 100,000 grains + 5%% nuclei, stored energy) and laguerre-512 "
                         "(512^3, 250,000 Laguerre grains): with --paths mixed")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    WORKLOAD.clear()
    WORKLOAD.update(WORKLOADS[args.workload][0])
    PHYSICS.clear()
    PHYSICS.update(WORKLOADS[args.workload][1])
    if args.domain:
        WORKLOAD.update(workload=f"{args.workload}-at-{args.domain}^3-{args.grains}-grains", domain=args.domain,
                        grains=args.grains)
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import gragles_3d_b200 as gg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
        dist = tdist
    else:
        torch.cuda.set_device(local)
    ms, ext, counts = microstructure()

    if args.paths != "both":  # profiling aid: one path, no comparison, no baselines
        prec = gg.PRECISION_MIXED if args.paths == "mixed" else gg.PRECISION_FP64
        reps, ms_e, clk, _, _ = run_device(gg, prec, ms, ext, counts, args.steps, args.warmup, local, dist)
        if rank == 0:
            vox = sum(r["voxel_updates"] for r in reps)
            keys = ["ms_convolution", "ms_lists", "ms_comparison", "ms_levelset", "ms_redistancing", "ms_total"]
            print(json.dumps({"profile_run": args.paths, "config": dict(WORKLOAD), "value": vox / (ms_e / 1e3),
                              "unit": UNIT, "ms_per_step": ms_e / args.steps, "clocks": clk,
                              "stage_ms": {k: float(np.mean([r[k] for r in reps])) for k in keys},
                              # per timed step: what a captured comparison launch processed
                              "compare_voxels": [int(r["compare_voxels"]) for r in reps],
                              "ms_compare_kernel": [float(r["ms_compare_kernel"]) for r in reps]}))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    reps_m, ms_m, clk_m, vol_m, ex_m, gh_m = run_device(gg, gg.PRECISION_MIXED, ms, ext, counts, args.steps,
                                                        args.warmup, local, dist, keep=True)
    reps_d, ms_d, clk_d, vol_d, ex_d, gh_d = run_device(gg, gg.PRECISION_FP64, ms, ext, counts, args.steps,
                                                        args.warmup, local, dist, keep=True)
    # the SDF error of the mixed path against FP64 after the same loops (host-side, untimed)
    try:
        sdf_err, boxes_differ = max_sdf_difference(gh_m, gh_d, ex_m & ex_d)
    except Exception as exc:  # a report field only: never lose the timed line over it
        print(f"SDF comparison skipped: {exc}", file=sys.stderr)
        sdf_err, boxes_differ = None, None
    boxes_d = gh_d.stats().boxes
    gh_m.close()
    gh_d.close()
    vox_m = sum(r["voxel_updates"] for r in reps_m)
    vox_d = sum(r["voxel_updates"] for r in reps_d)
    elapsed_m, vox_m = aggregate_replicas(ms_m, vox_m, dist)
    elapsed_d, vox_d = aggregate_replicas(ms_d, vox_d, dist)
    value = vox_m / (elapsed_m / 1e3)
    value_fp64 = vox_d / (elapsed_d / 1e3)

    both = ex_m & ex_d
    both[0] = False
    rel = np.abs(vol_m[both] - vol_d[both]) / np.maximum(vol_d[both], 1e-300)
    max_rel = float(rel.max()) if rel.size else None
    # the reference's hull volume jumps when a voxel within ~1e-7 of zero changes sign
    # (its vertex snapping leaves the triangulation open there), so the spread matters too
    rel_spread = ({"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99)),
                   "grains_over_1e-3": int((rel > 1e-3).sum()), "grains": int(rel.size),
                   "over_by_cause": over_bound_causes(rel, np.nonzero(both)[0], vol_d, boxes_d)}
                  if rel.size else None)

    def stage_means(reps):
        keys = ["ms_convolution", "ms_lists", "ms_comparison", "ms_levelset", "ms_redistancing", "ms_total"]
        return {k: float(np.mean([r[k] for r in reps])) for k in keys}

    st_m, st_d = stage_means(reps_m), stage_means(reps_d)
    peak, peak_kind = read_peaks()
    # the dominant kernel (the largest share of the launch list): the comparison,
    # timed alone by the library's events on its stream
    ms_k = float(np.mean([r["ms_compare_kernel"] for r in reps_m]))
    vox_k = float(np.mean([r["compare_voxels"] for r in reps_m]))
    bytes_per = STAGE_BYTES["mixed"]["ms_comparison"]
    achieved = bytes_per * vox_k / (ms_k / 1e3) / 1e9
    traffic, traffic_note = measured_traffic("compare_kernel", vox_k)

    e2e = None
    out = None
    if rank == 0:
        e2e = (run_e2e(gg, gg.PRECISION_MIXED, ms, ext, counts, args.steps, args.warmup, local) if not args.no_e2e else
               {"value": None, "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None})
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cv, sample, cores, kind = run_reference_cpu(ms, 1, 1, os.cpu_count() or 1)
            cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_m / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(world), "path": "mixed",
            "fp64": {"value": value_fp64, "ms_per_step": elapsed_d / args.steps, "dtype": "f64",
                     "stage_ms": st_d, "clocks": clk_d},
            "mixed_over_fp64": value / value_fp64,
            "max_rel_volume_err_mixed_vs_fp64": max_rel,
            "rel_volume_err_spread": rel_spread,
            "max_abs_sdf_err_mixed_vs_fp64": sdf_err,
            "grains_with_different_boxes": boxes_differ,
            "stage_ms": st_m,
            "roofline": {"bound": "hbm", "kernel": "compare_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind, "traffic_source": traffic_note,
                         "bytes_per_voxel_update": bytes_per,
                         "ms_per_launch": ms_k, "voxels_per_launch": vox_k},
            "cpu_baseline": cpu,
            "e2e": {k: e2e.get(k) for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step", "ms",
                                            "ms_setup")},
            "gpu_launches": int(sum(r["kernel_launches"] for r in reps_m)),
            "clocks": clk_m,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
