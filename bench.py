"""Benchmark of the cpSZ offline compressor on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cpsz_b200|reference] [--workload NAME]

One step = one compression of the workload's field(s) (u, v[, w]) through the
library.  Default workload: the 2D 8192x8192 field (2000 Gaussian-windowed
linear flows, sigma 60, relative bound 0.1) -- the largest single-GPU 2D
configuration; its input (537 MB) exceeds L2 (126 MB), so no flush is needed
between steps.

Prints ONE JSON line (rank 0):
  value    compress GB/s of input with the field resident in HBM and the blob
           written to device memory (the host still builds the Huffman trees
           from device histograms inside the call), timed with CUDA events on
           the library's stream, max over ranks;
  e2e      the same through the public API with pinned host input and the blob
           returned to the host (H2D/D2H inside the timed region);
  ratio    raw bytes / ZSTD(level 3)'d blob bytes (the reference's definition),
           plus the pre-ZSTD ratio and decompress GB/s;
  roofline the dominant kernel's algorithmic bytes / its CUDA-event duration
           vs the measured HBM copy bandwidth;
  cpu_baseline the reference's own CPU implementation on a bounded sample.
Multi-GPU: a single field does not shard (its Lorenzo stage is one serial
recurrence), so N GPUs run N independent replicas ("replicas only"); value is
the total input of all ranks / the max per-rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (kind, shape, eb, generator)
    "2d_8192x8192_eb0.1": ("2d", (8192, 8192), 0.1, "cfg1"),
    "2d_8192x8192_eb0.01": ("2d", (8192, 8192), 0.01, "cfg1"),
    "2d_2400x3600_eb0.1": ("2d", (2400, 3600), 0.1, "cfg0"),
    # profiling-size case of the same kernels (cfg0 generator at 4096^2, 134 MB > L2)
    "2d_4096x4096_eb0.1": ("2d", (4096, 4096), 0.1, "cfg0like"),
    "3d_384x384x384_eb0.05": ("3d", (384, 384, 384), 0.05, "cfg2"),
    # profiling-size case of the 3D kernels (cfg2 generator at 256^3, 201 MB > L2)
    "3d_256x256x256_eb0.05": ("3d", (256, 256, 256), 0.05, "cfg2"),
    # 256 fields, sides uniform in [128, 4096], eb in {0.01, 0.05, 0.1}, one flow per 40x40 cells
    "batch_256x2d_cfg3": ("batch", None, None, "cfg3"),
    # the cfg1 field with learned bounds (trained proposer, fallback loop to 0 CP differences)
    "learned_2d_8192x8192_eb0.1": ("learned", (8192, 8192), 0.1, "cfg1"),
}
DEFAULT = "2d_8192x8192_eb0.1"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.th = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.th:
                self.th.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def make_fields(workload: str, seed_offset: int = 0):
    from cpsz_b200 import workloads as W

    kind, shape, eb, gen = WORKLOADS[workload]
    if gen == "cfg1":
        return W.cfg1(1 + seed_offset), eb
    if gen == "cfg0":
        return W.cfg0(0 + seed_offset), eb
    if gen == "cfg0like":
        return W.cfg0_like(5 + seed_offset, *shape), eb
    if gen == "cfg2":
        return W.cfg2(2 + seed_offset, shape[0]), eb
    raise KeyError(workload)


# ---- reference arm ----------------------------------------------------------------------

def _ref_worker(args):
    """One bounded sample of the workload through the reference CPU implementation."""
    kind, arr_paths, eb, use_ref = args
    sys.path.insert(0, ROOT)
    import oracle

    arrs = [np.load(p, mmap_mode="r") for p in arr_paths]
    impl = oracle.Reference() if use_ref else oracle.Oracle()
    arrs = [np.ascontiguousarray(a) for a in arrs]
    t = time.perf_counter()
    if kind == "2d":
        blob = impl.compress_2d(arrs[0], arrs[1], eb)
    else:
        blob = impl.compress_3d(arrs[0], arrs[1], arrs[2], eb)
    return time.perf_counter() - t, len(blob)


def reference_samples(workload: str, fields, eb):
    """Tiles of the workload sized for ~1 s of reference CPU work each."""
    kind = WORKLOADS[workload][0]
    tiles = []
    if kind in ("2d", "learned"):
        U, V = fields
        s = 1024
        for i in range(0, U.shape[0] - s + 1, s):
            for j in range(0, U.shape[1] - s + 1, s):
                tiles.append((U[i:i + s, j:j + s], V[i:i + s, j:j + s]))
    else:
        U, V, Wf = fields
        s = 96
        for i in range(0, U.shape[0] - s + 1, s):
            tiles.append(tuple(a[i:i + s, :s, :s] for a in (U, V, Wf)))
    return tiles


def run_reference(args, rank, world):
    import multiprocessing as mp
    import tempfile

    import oracle

    if rank != 0:
        return None
    kind = WORKLOADS[args.workload][0]
    use_ref = os.path.exists(oracle.REF_SO)
    if kind == "batch":
        # whole fields of the batch (the smaller ones), each with its own bound
        lay = batch_layout()
        order = sorted(range(len(lay)), key=lambda k: lay[k][0] * lay[k][1])
        tiles, tile_ebs = make_batch([k for k in order if lay[k][0] * lay[k][1] <= 1_500_000])
        kind = "2d"
    else:
        fields, eb = make_fields(args.workload)
        tiles = reference_samples(args.workload, fields, eb)
        tile_ebs = [eb] * len(tiles)
        kind = "2d" if kind == "learned" else kind
    cores = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="cpsz_ref_")
    paths = []
    for k, t in enumerate(tiles[:max(cores, 1) * 2]):
        ps = []
        for c, a in enumerate(t):
            p = os.path.join(tmp, f"t{k}_{c}.npy")
            np.save(p, np.ascontiguousarray(a))
            ps.append(p)
        paths.append(ps)
    ctxm = mp.get_context("spawn")
    times = []
    total_bytes = 0
    with ctxm.Pool(cores) as pool:
        jobs = [(kind, p, tile_ebs[k], use_ref) for k, p in enumerate(paths[:cores])]
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, jobs)
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append(dt)
                total_bytes = sum(np.load(p, mmap_mode="r").nbytes for job in jobs for p in job[1])
    per_step = statistics.mean(times)
    gbs = total_bytes / per_step / 1e9
    what = ("whole fields of the batch (up to 1.5M points each)" if WORKLOADS[args.workload][0] == "batch"
            else f"{'1024x1024' if kind == '2d' else '96^3'} tiles of the workload")
    sample = f"{len(jobs)} independent {what}, one per process, compressed concurrently per step"
    line = {
        "impl": "reference", "metric": "compress_GBps", "value": round(gbs, 4), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic", "config": {"workload": args.workload},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": len(jobs),
                         "kind": "reference" if use_ref else "port", "sample": sample},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


# ---- product arm -----------------------------------------------------------------------

def cpu_baseline_single(workload, fields, eb, budget_s=12.0):
    """The reference CPU implementation (1 core, as the reference is single-threaded)
    on 1024x1024 (2D) / 96^3 (3D) tiles of the workload for about budget_s seconds."""
    import oracle

    use_ref = os.path.exists(oracle.REF_SO)
    impl = oracle.Reference() if use_ref else oracle.Oracle()
    tiles = reference_samples(workload, fields, eb)
    kind = WORKLOADS[workload][0]
    t_total, nbytes, n = 0.0, 0, 0
    zt = 0.0
    while t_total < budget_s and n < len(tiles):
        t = [np.ascontiguousarray(a) for a in tiles[n]]
        t0 = time.perf_counter()
        blob = impl.compress_2d(t[0], t[1], eb) if kind == "2d" else impl.compress_3d(t[0], t[1], t[2], eb)
        t_total += time.perf_counter() - t0
        if use_ref:
            t0 = time.perf_counter()
            impl.zstd_compress(blob)
            zt += time.perf_counter() - t0
        nbytes += sum(a.nbytes for a in t)
        n += 1
    return {"value": round(nbytes / t_total / 1e9, 5), "unit": "GB/s", "cores": 1,
            "kind": "reference" if use_ref else "port",
            "sample": f"{n} tiles {'1024x1024' if kind == '2d' else '96^3'} of the workload, 1 thread, "
                      f"{t_total:.1f} s; host ZSTD stage separately {nbytes / max(zt, 1e-9) / 1e9:.3f} GB/s"}


def run_product(args, rank, world, device):
    import torch

    import cpsz_b200

    kind, shape, eb, _ = WORKLOADS[args.workload]
    fields, eb = make_fields(args.workload, seed_offset=rank)
    raw_bytes = sum(a.nbytes for a in fields)
    ctx = cpsz_b200.Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    dev = [torch.from_numpy(a).to(f"cuda:{device}") for a in fields]
    out_cap = raw_bytes * 2 + (64 << 20)
    d_out = torch.empty(out_cap, dtype=torch.uint8, device=f"cuda:{device}")
    comp = (cpsz_b200.compress_2d_into if kind == "2d" else cpsz_b200.compress_3d_into)

    def step_dev():
        return comp(*dev, *shape, eb, d_out, ctx=ctx)

    # the clock sampler runs from the warm-up through the timed region (the
    # timed region alone can be shorter than nvidia-smi's start-up)
    clk = Clocks(device).__enter__()
    for _ in range(args.warmup):
        size = step_dev()
    torch.cuda.synchronize(device)
    lib = cpsz_b200.lib()
    lib.cpsz_b200_ctx_set_timing(ctx.handle, 1)
    stage_acc = {}
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize(device)
    launches0 = ctx.kernel_launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    try:
        ev0.record(stream)
        for _ in range(args.steps):
            size = step_dev()
            for nm, ms in stage_times(ctx).items():
                stage_acc.setdefault(nm, []).append(ms)
        ev1.record(stream)
        torch.cuda.synchronize(device)
    finally:
        clk.__exit__(None, None, None)
    launches = ctx.kernel_launches - launches0
    lib.cpsz_b200_ctx_set_timing(ctx.handle, 0)
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = raw_bytes * world / (ms / 1e3) / 1e9

    # ---- end to end: pinned host fields in, blob written to a pinned host
    # buffer by the public *_into call (host<->device copies inside) ----
    pinned = [torch.from_numpy(a).pin_memory() for a in fields]
    hptr = [p.numpy() for p in pinned]
    h_out = torch.empty(out_cap, dtype=torch.uint8).pin_memory().numpy()
    for _ in range(2):
        e2e_size = comp(*hptr, *shape, eb, h_out, ctx=ctx)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_size = comp(*hptr, *shape, eb, h_out, ctx=ctx)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    blob = h_out[:e2e_size].tobytes()
    # ---- decompression (host blob in, host fields out) ----
    decompress = (cpsz_b200.sz_decompress_cp_preserve_2d_offline if kind == "2d"
                  else cpsz_b200.sz_decompress_cp_preserve_3d_online_log)
    outs = [torch.empty(shape, dtype=torch.float32).pin_memory().numpy() for _ in fields]
    decompress(blob, *shape, *outs, ctx=ctx)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        decompress(blob, *shape, *outs, ctx=ctx)
    dec_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    lossless = cpsz_b200.sz_lossless_compress(blob, 3)

    stages = {k: statistics.mean(v) for k, v in stage_acc.items()}
    n = int(np.prod(shape))
    comps = 2 if kind == "2d" else 3
    # algorithmic bytes per launch of each stage's dominant kernel
    alg = {"eb2d": 4 * comps * n + comps * n,  # read fields, write one id byte per component
           "wave2d_compress": 4 * comps * n + comps * n + 2 * comps * n,  # fields + ids in, u16 codes out
           "eb3d": 4 * 3 * n + n, "wave3d_compress": 0}  # read fields, write one id byte
    # DRAM bytes per point of a launch, read + write, from one ncu capture of the
    # kernel on the 4096^2 case (394.0 MB for 16.8 M vertices), scaled to this
    # launch by its points
    traffic_per_point = {"eb2d": (135.14496e6 + 258.857216e6) / 4096 ** 2}
    dom = max((k for k in stages if k in alg and alg[k]), key=lambda k: stages[k], default=None)
    peak, peak_kind = measured_peaks()
    roof = None
    if dom:
        ach = alg[dom] / (stages[dom] / 1e3) / 1e9
        tr = traffic_per_point.get(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": round(tr * n) if tr else None, "peak_source": peak_kind,
                "algorithmic_bytes": alg[dom]}
    return {
        "value": value, "ms": ms, "e2e_ms": e2e_ms, "dec_ms": dec_ms, "blob": len(blob), "size_dev": size,
        "lossless": len(lossless), "raw": raw_bytes, "stages": stages, "roofline": roof, "launches": launches,
        "clocks": clk.summary(), "fields": fields, "eb": eb,
    }


def run_learned(args, rank, world, device):
    """Learned-bound compression of the cfg1 field: every step runs the MLP over
    all vertices, the fallback loop's reconstruction passes and the final
    compression (fields resident in HBM, blob written to HBM); the plain
    compressor's ratio and the exact CP comparison are reported beside it."""
    import torch

    import cpsz_b200
    from cpsz_b200 import learned

    kind, shape, eb, _ = WORKLOADS[args.workload]
    fields, eb = make_fields("2d_8192x8192_eb0.1", seed_offset=rank)
    raw = sum(a.nbytes for a in fields)
    ctx = cpsz_b200.Context(device)
    mlp = learned.load(ctx)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    dev = [torch.from_numpy(a).to(f"cuda:{device}") for a in fields]
    out = torch.empty(raw + (64 << 20), dtype=torch.uint8, device=f"cuda:{device}")
    clk = Clocks(device).__enter__()
    for _ in range(args.warmup):
        size, st = cpsz_b200.compress_2d_learned(*dev, eb, mlp=mlp, out=out, ctx=ctx)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = ctx.kernel_launches
    try:
        ev0.record(stream)
        for _ in range(args.steps):
            size, st = cpsz_b200.compress_2d_learned(*dev, eb, mlp=mlp, out=out, ctx=ctx)
        ev1.record(stream)
        torch.cuda.synchronize(device)
    finally:
        clk.__exit__(None, None, None)
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = (ctx.kernel_launches - launches0) // max(args.steps, 1)
    blob = out[:size].cpu().numpy().tobytes()
    plain = cpsz_b200.sz_compress_cp_preserve_2d_offline(*fields, max_pwr_eb=eb, ctx=ctx)
    dU, dV = cpsz_b200.sz_decompress_cp_preserve_2d_offline(blob, *shape, ctx=ctx)
    cp = cpsz_b200.cp_check_2d(fields[0], fields[1], dU, dV, ctx=ctx)
    z_learned = len(cpsz_b200.sz_lossless_compress(blob, 3))
    z_plain = len(cpsz_b200.sz_lossless_compress(plain, 3))
    return {
        "metric": "compress_GBps", "value": round(raw * world / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f64+f32", "data": "synthetic",
        "config": {"workload": args.workload, "tuning": _tuning_tag(), "eb": eb, "points": int(raw // 8), "inputs_exceed_l2": True,
                   "parallelism": f"replicas{world}", "value_io": "fields resident in HBM, blob written to HBM"},
        "ratio": round(raw / z_learned, 4), "ratio_pre_zstd": round(raw / size, 4),
        "plain_ratio": round(raw / z_plain, 4), "plain_ratio_pre_zstd": round(raw / len(plain), 4),
        "cp_check": cp, "loop": st, "cpu_baseline": None, "clocks": clk.summary(), "gpu_launches": launches,
    }


def batch_layout():
    """(r1, r2, seed, eb) of the 256 fields of the batched workload."""
    from cpsz_b200 import workloads as W

    return W.batch_layout(3, 256, 128, 4096)


def make_batch(idx=None):
    """Host fields and bounds of the batch's fields `idx` (all when None)."""
    from cpsz_b200 import workloads as W

    lay = batch_layout()
    idx = range(len(lay)) if idx is None else idx
    return [W.cfg3_field(*lay[k][:3]) for k in idx], [lay[k][3] for k in idx]


def run_batch(args, rank, world, device):
    """The batched workload, sharded by field across the ranks (greedy size
    balance, cpsz_b200/shard.py): each step every rank compresses the fields it
    owns with one batched call (fields resident in HBM, blobs written to HBM)
    and the ranks sum-all-reduce the per-field blob sizes, which places every
    blob in the batch's concatenation.  The same fields through one
    single-field call each, and the sharded call end to end from host memory,
    are reported beside it."""
    import torch

    import cpsz_b200
    from cpsz_b200 import shard

    lay = batch_layout()
    n_all = len(lay)
    own = shard.partition([r1 * r2 for r1, r2, _, _ in lay], world)[rank]
    fields, ebs = make_batch(own)
    raw_all = sum(8 * r1 * r2 for r1, r2, _, _ in lay)
    raw = sum(U.nbytes + V.nbytes for U, V in fields)
    ctx = cpsz_b200.Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    dev = [(torch.from_numpy(U).to(f"cuda:{device}"), torch.from_numpy(V).to(f"cuda:{device}")) for U, V in fields]
    out = torch.empty(raw + (256 << 20), dtype=torch.uint8, device=f"cuda:{device}")
    sizes = torch.zeros(n_all, dtype=torch.int64, device=f"cuda:{device}")
    own_t = torch.tensor(own, dtype=torch.int64, device=f"cuda:{device}")
    if world > 1:
        import torch.distributed as dist

    def step():
        offsets = cpsz_b200.compress_2d_batch(dev, ebs, out=out, ctx=ctx)
        if world > 1:
            with torch.cuda.stream(stream):
                sizes.zero_()
                sizes.index_copy_(0, own_t, torch.from_numpy(np.diff(offsets).astype(np.int64)).to(sizes.device))
                dist.all_reduce(sizes)
        return offsets

    clk = Clocks(device).__enter__()
    for _ in range(args.warmup):
        offsets = step()
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    launches0 = ctx.kernel_launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    try:
        ev0.record(stream)
        for _ in range(args.steps):
            offsets = step()
        ev1.record(stream)
        torch.cuda.synchronize(device)
    finally:
        clk.__exit__(None, None, None)
    launches = (ctx.kernel_launches - launches0) // max(args.steps, 1)
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    blob_bytes = int(offsets[-1])
    # one single-field call per field, same device-resident fields
    ev0.record(stream)
    for (u, v), eb in zip(dev, ebs):
        cpsz_b200.compress_2d_into(u, v, u.shape[0], u.shape[1], eb, out, ctx=ctx)
    ev1.record(stream)
    torch.cuda.synchronize(device)
    per_field_ms = ev0.elapsed_time(ev1)
    # end to end through the sharded call: fields in pinned host memory, blobs
    # back into a pinned host buffer (the batched call writes them back to back)
    shapes = [(r1, r2) for r1, r2, _, _ in lay]
    all_ebs = [e for *_, e in lay]
    pos = {k: i for i, k in enumerate(own)}
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    h_fields = [(pin(U), pin(V)) for U, V in fields]
    h_out = torch.empty(raw + (256 << 20), dtype=torch.uint8).pin_memory().numpy()

    def pinned_compress(fs, es):
        offs = cpsz_b200.compress_2d_batch(fs, es, out=h_out, ctx=ctx)
        return [h_out[int(offs[q]):int(offs[q + 1])] for q in range(len(fs))]

    res = shard.compress_2d_batch_sharded(shapes, all_ebs, lambda k: h_fields[pos[k]], ctx=ctx,
                                          compress=pinned_compress)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    res = shard.compress_2d_batch_sharded(shapes, all_ebs, lambda k: h_fields[pos[k]], ctx=ctx,
                                          compress=pinned_compress)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    if world > 1:
        t = torch.tensor([e2e_ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    total_blob = int(res.offsets[-1])
    return {
        "metric": "compress_GBps", "value": round(raw_all / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": args.workload, "tuning": _tuning_tag(), "fields": n_all, "points": int(raw_all // 8),
                   "inputs_exceed_l2": True, "parallelism": f"field-sharded{world}",
                   "value_io": "fields resident in HBM, blobs written to HBM; per-field sizes all-reduced"},
        "ratio_pre_zstd": round(raw_all / total_blob, 4),
        "per_field_calls_GBps": round(raw / (per_field_ms / 1e3) / 1e9, 3),
        "e2e": {"value": round(raw_all / (e2e_ms / 1e3) / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": raw,
                "d2h_bytes_per_step": blob_bytes, "host_input": "pinned host memory"},
        "cpu_baseline": None, "clocks": clk.summary(), "gpu_launches": launches,
    }


def stage_times(ctx):
    return ctx.stage_times()


def _tuning_tag():
    import os

    import cpsz_b200

    src = cpsz_b200.tuning_source()
    return os.path.basename(src) if src else "built-in defaults"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cpsz_b200", choices=["cpsz_b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if rank == 0 and line:
            print(json.dumps(line))
        return

    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if WORKLOADS[args.workload][0] in ("batch", "learned"):
        line = (run_batch if WORKLOADS[args.workload][0] == "batch" else run_learned)(args, rank, world, local)
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line))
        return
    r = run_product(args, rank, world, local)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline_single(args.workload, r["fields"], r["eb"])
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    kind = WORKLOADS[args.workload][0]
    raw = r["raw"]
    line = {
        "metric": "compress_GBps", "value": round(r["value"], 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"], 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": args.workload, "tuning": _tuning_tag(), "eb": r["eb"], "points": int(raw // (4 * (2 if kind == "2d" else 3))),
                   "inputs_exceed_l2": True, "parallelism": f"replicas{world}",
                   "value_io": "fields resident in HBM, blob written to HBM"},
        "ratio": round(raw / r["lossless"], 4), "ratio_pre_zstd": round(raw / r["blob"], 4),
        "decompress_GBps_e2e": round(raw / (r["dec_ms"] / 1e3) / 1e9, 3),
        "e2e": {"value": round(raw / (r["e2e_ms"] / 1e3) / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": raw,
                "d2h_bytes_per_step": r["blob"]},
        "roofline": r["roofline"], "stages_ms": {k: round(v, 4) for k, v in r["stages"].items()},
        "cpu_baseline": cpu, "clocks": r["clocks"], "gpu_launches": r["launches"],
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
