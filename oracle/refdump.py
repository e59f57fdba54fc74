"""Reader for the binary records that oracle/ref_hooks.cpp makes the compiled
reference write, and a runner for oracle/_ref/ggls_ref (TEST INFRASTRUCTURE).

Only tests/, the golden-fixture script and bench.py's CPU baseline use this.
"""
from __future__ import annotations

import dataclasses
import os
import subprocess
import tempfile
from typing import Iterator, Optional

import numpy as np

KIND = {
    "INIT_SDF": 1, "INIT_LIST": 2, "STATS": 3, "NEIGHBORS": 4, "CONV_IN": 5, "CONV_OUT": 6,
    "LIST": 7, "CMP_OUT": 8, "CMP_ID": 9, "SETCMP_OUT": 10, "REDIST_IN": 11, "REDIST_OUT": 12,
    "MC_ID": 13, "MC_IN": 14, "LOOP_TIME": 15,
}
KIND_NAME = {v: k for k, v in KIND.items()}
HERE = os.path.dirname(os.path.abspath(__file__))
REF_BINARY = os.path.join(HERE, "_ref", "ggls_ref")


@dataclasses.dataclass
class Record:
    kind: str
    loop: int
    grain: int
    box: tuple  # (xmin, xmax, ymin, ymax, zmin, zmax)
    data: np.ndarray

    def cube(self) -> np.ndarray:
        x0, x1, y0, y1, z0, z1 = self.box
        return self.data.reshape(z1 - z0, y1 - y0, x1 - x0)


def read_records(path: str) -> Iterator[Record]:
    raw = np.fromfile(path, dtype=np.uint8)
    off = 0
    n = raw.size
    while off + 52 <= n:
        magic = int(raw[off:off + 4].view("<u4")[0])
        if magic != 0x52444747:
            raise ValueError(f"bad record magic at offset {off}")
        hdr = raw[off + 4:off + 44].view("<i4")
        count = int(raw[off + 44:off + 52].view("<i8")[0])
        off += 52
        dtype = "<f8" if int(hdr[9]) == 0 else "<u4"
        size = 8 if dtype == "<f8" else 4
        data = raw[off:off + count * size].view(dtype).copy()
        off += count * size
        yield Record(KIND_NAME.get(int(hdr[0]), str(int(hdr[0]))), int(hdr[1]), int(hdr[2]),
                     tuple(int(v) for v in hdr[3:9]), data)


def run_reference(workdir: str, params: str = "parameters.xml", *, threads: int = 8,
                  dump: Optional[str] = None, stats: bool = True, grains: Optional[str] = None,
                  loops: Optional[str] = None, timeout: float = 3600.0,
                  binary: str = REF_BINARY, init: bool = True) -> subprocess.CompletedProcess:
    """Run the compiled reference in ``workdir`` (it writes its outputs there)."""
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    env.setdefault("OMP_PLACES", "cores")
    env.setdefault("OMP_PROC_BIND", "close")
    if dump:
        env["GG_REF_DUMP"] = dump
        env["GG_REF_DUMP_STATS"] = "1" if stats else "0"
        if grains:
            env["GG_REF_DUMP_GRAINS"] = grains
        if loops:
            env["GG_REF_DUMP_LOOPS"] = loops
        if not init:
            env["GG_REF_DUMP_INIT"] = "0"
    return subprocess.run([binary, params], cwd=workdir, env=env, capture_output=True,
                          text=True, timeout=timeout)


def parse_timers(stdout: str) -> dict:
    """The reference's own stage timers (grainhdl.cpp:920-933, ggLS.cpp:74)."""
    out = {"coarsening": []}
    keys = {"Convolution time:": "convolution", "Comparison time:": "comparison",
            "Redistancing time:": "redistancing", "Levelset time:": "levelset",
            "GridCoarse/SwitchBuffer/UpNeigh:": "rest", "Sum parallel regions:": "sum",
            "Elapsed seconds for simulation:": "elapsed"}
    for line in stdout.splitlines():
        # gridCoarsement's report (grainhdl.cpp:1454-1455): the loop, then the new size
        if line.startswith("coarsing the current grid in Timestep:"):
            out["coarsening"].append([int(line.split(":")[-1]), 0])
        elif line.startswith("newSize :") and out["coarsening"]:
            out["coarsening"][-1][1] = int(line.split(":")[-1])
        for k, name in keys.items():
            if line.strip().startswith(k):
                try:
                    out[name] = float(line.split(":")[-1])
                except ValueError:
                    pass
    return out


def collect(records) -> dict:
    """Group records: init state, per-loop stats/neighbours/lists, stage buffers."""
    res = {"init_sdf": {}, "init_list": {}, "stats": {}, "neighbors": {}, "lists": {}, "buffers": {},
           "loop_time": {}}
    for r in records:
        if r.kind == "LOOP_TIME":
            res["loop_time"][r.loop] = float(r.data[0])
        elif r.kind == "INIT_SDF":
            res["init_sdf"][r.grain] = r
        elif r.kind == "INIT_LIST":
            res["init_list"][r.grain] = r.data
        elif r.kind == "STATS":
            res["stats"].setdefault(r.loop, {})[r.grain] = (r.data, r.box)
        elif r.kind == "NEIGHBORS":
            res["neighbors"].setdefault(r.loop, {})[r.grain] = r.data
        elif r.kind == "LIST":
            res["lists"].setdefault(r.loop, {})[r.grain] = r.data
        else:
            res["buffers"][(r.kind, r.loop, r.grain)] = r
    return res


def run_case(ms_dir: str, *, threads: int = 8, grains: Optional[str] = None,
             loops: Optional[str] = None, timeout: float = 3600.0, init: bool = True) -> tuple[dict, dict]:
    """Run the reference on a prepared case directory and return (collected dump, timers)."""
    fd, dump = tempfile.mkstemp(suffix=".ggdr", dir=ms_dir)
    os.close(fd)
    proc = run_reference(ms_dir, threads=threads, dump=dump, grains=grains, loops=loops,
                         timeout=timeout, init=init)
    if proc.returncode != 0:
        raise RuntimeError(f"reference failed ({proc.returncode}): {proc.stderr[-2000:]}")
    res = collect(read_records(dump))
    os.unlink(dump)
    return res, parse_timers(proc.stdout)
