"""Offline sweep of the launch-shape table (``csrc/tuning.h``).

    python -m cpsz_b200.autotune [--out cpsz_b200/tuning_b200.json] [--quick]

For each size bucket and each output-invariant launch parameter, the sweep
compresses a seeded synthetic field (2D: the flow density and width of the
8192^2 headline field, scaled to the side) with every candidate value (the other
parameters at their current best), times the stage that the parameter shapes
with the context's CUDA-event stage marks, and keeps the fastest value.  Every
candidate's blob must equal the default's byte for byte, or the sweep stops:
the parameters may change speed, never output.

The table is JSON (format ``cpsz_b200-tuning-1``)::

    {"format": "cpsz_b200-tuning-1", "device": "...", "entries": [
       {"param": "eb2d.tile", "min_points": 0, "value": 0, "ms": {...}}, ...]}

An entry applies to fields of at least ``min_points`` points (the bucket's
lower edge: the geometric mean of neighbouring measured sizes); the library
reads ``param``, ``min_points`` and ``value`` and ignores the rest.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys

import numpy as np

from . import Context, compress_2d_into, compress_3d_into, tuning_clear, tuning_params, tuning_set
from . import workloads

FORMAT = "cpsz_b200-tuning-1"
DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")

# parameter -> (field kind, stage timed, candidate values, smallest field it is swept on)
# A stage "a+b" is the sum of stages a and b: the bound kernel and the
# wavefront run side by side, so either one's shape moves both stages.
SWEEP = {
    "wave2d.overlap": ("2d", "eb2d+wave2d_compress", [0, 1], 0),
    "eb2d.skew": ("2d", "eb2d+wave2d_compress", [0, 1, 2, 4, 8], 0),
    "eb2d.tile": ("2d", "eb2d+wave2d_compress", [0, 1, 2, 3, 4, 5], 0),
    "wave2d.ctas_per_sm": ("2d", "wave2d_compress", [0, 1, 2, 3, 4], 0),
    "h2d.chunks": ("2d_host", "e2e", [1, 2, 4, 8, 16, 24, 32], 1 << 22),
    "eb3d.fill": ("3d", "eb3d", [1, 2, 4, 8, 16], 0),
    "eb3d.min_chunk": ("3d", "eb3d", [4, 8, 16, 32], 0),
}
SIDES_2D = [512, 1024, 2048, 4096, 8192]
SIDES_3D = [64, 128, 256, 384]


def bucket_edges(points: list[int]) -> list[int]:
    """Lower edge of each size's bucket: 0, then geometric means of neighbours."""
    return [0] + [int(math.sqrt(points[k - 1] * points[k])) for k in range(1, len(points))]


class Case:
    """One seeded field, resident on the device (and on the host for e2e timing)."""

    def __init__(self, kind: str, side: int, ctx: Context, seed: int):
        import torch

        self.kind, self.side, self.ctx = kind, side, ctx
        if kind == "2d":
            # the 8192^2 headline field's flow density and width at every side
            n_flows = max(1, round(2000 * (side / 8192) ** 2))
            self.host = workloads.field_2d(seed, side, side, n_flows, 60.0)
            self.shape = (side, side)
            self.eb = 0.1
        else:
            n_flows = max(1, round(500 * (side / 384) ** 3))
            self.host = workloads.field_3d(seed, side, side, side, n_flows, 20.0)
            self.shape = (side, side, side)
            self.eb = 0.05
        self.points = int(np.prod(self.shape))
        self.dev = [torch.from_numpy(a).cuda() for a in self.host]
        cap = 3 * 4 * self.points + (64 << 20)
        self.d_out = torch.empty(cap, dtype=torch.uint8, device="cuda")
        self.h_out = np.empty(cap, np.uint8)

    def run(self, host_input: bool = False) -> int:
        comp = compress_2d_into if self.kind == "2d" else compress_3d_into
        if host_input:
            return comp(*self.host, *self.shape, self.eb, self.h_out, ctx=self.ctx)
        return comp(*self.dev, *self.shape, self.eb, self.d_out, ctx=self.ctx)

    def blob(self, host_input: bool = False) -> bytes:
        n = self.run(host_input)
        if host_input:
            return self.h_out[:n].tobytes()
        return self.d_out[:n].cpu().numpy().tobytes()

    def time(self, stage: str, reps: int) -> float:
        """Median ms of `stage` (or of the whole host-input call for "e2e") over reps runs."""
        import time

        import torch

        host = stage == "e2e"
        for _ in range(2):
            self.run(host)
        torch.cuda.synchronize()
        ts = []
        self.ctx.set_timing(not host)
        try:
            for _ in range(reps):
                if host:
                    t0 = time.perf_counter()
                    self.run(True)
                    ts.append((time.perf_counter() - t0) * 1e3)
                else:
                    self.run(False)
                    st = self.ctx.stage_times()
                    missing = [x for x in stage.split("+") if x not in st]
                    if missing:
                        raise RuntimeError(f"stage {missing[0]!r} not among {sorted(st)}")
                    ts.append(sum(st[x] for x in stage.split("+")))
        finally:
            self.ctx.set_timing(False)
        return statistics.median(ts)


def sweep(quick: bool = False, reps: int = 7, log=print) -> dict:
    import torch

    params = tuning_params()
    tuning_clear()
    ctx = Context(0)
    sides = {"2d": SIDES_2D[:3] if quick else SIDES_2D, "3d": SIDES_3D[:2] if quick else SIDES_3D}
    entries = []
    for kind in ("2d", "3d"):
        names = [p for p, s in SWEEP.items() if s[0].startswith(kind)]
        pts = [s ** (2 if kind == "2d" else 3) for s in sides[kind]]
        edges = bucket_edges(pts)
        for side, lo in zip(sides[kind], edges):
            case = Case(kind, side, ctx, seed=1000 + side)
            ref = {False: case.blob(False)}
            for name in names:
                _, stage, cands, min_pts = SWEEP[name]
                if case.points < min_pts:
                    continue
                host = stage == "e2e"
                if host not in ref:
                    ref[host] = case.blob(host)
                best_v, best_ms, ms = None, math.inf, {}
                for v in cands:
                    if not params[name][1] <= v <= params[name][2]:
                        continue
                    # the value applies to this bucket only while it is measured
                    tuning_set(name, v, lo)
                    if case.blob(host) != ref[host]:
                        raise RuntimeError(f"{name}={v} changed the blob of a {kind} field of side {side}")
                    ms[v] = round(case.time(stage, reps), 4)
                    if ms[v] < best_ms:
                        best_v, best_ms = v, ms[v]
                # keep the default unless another value is clearly faster (2 %)
                d = params[name][0]
                if d in ms and ms[d] <= best_ms * 1.02:
                    best_v = d
                tuning_set(name, best_v, lo)
                entries.append({"param": name, "min_points": lo, "value": best_v, "side": side,
                                "stage": stage, "ms": {str(k): t for k, t in ms.items()}})
                log(f"{kind} side {side:5d} {name:20s} -> {best_v}  {ms}")
            del case
            torch.cuda.empty_cache()
    ctx.close()
    return {"format": FORMAT, "device": torch.cuda.get_device_name(0), "reps": reps, "entries": entries}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--quick", action="store_true", help="small sizes only (a functional check)")
    ap.add_argument("--reps", type=int, default=7)
    a = ap.parse_args(argv)
    table = sweep(a.quick, a.reps, log=lambda s: print(s, file=sys.stderr, flush=True))
    with open(a.out, "w") as f:
        json.dump(table, f, indent=1)
    print(a.out)


if __name__ == "__main__":
    main()
