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
           vs the measured HBM copy bandwidth; for the 2D bound kernel, which
           is bound by instruction issue, also its warp instructions a second
           vs 4 a cycle per SM (roofline.issue);
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
    # profiling-size case with the 8192^2 field's flow density and width (cfg1
    # generator at 4096^2: 500 flows, sigma 60; critical points as sparse as there)
    "2d_4096x4096_cfg1like_eb0.1": ("2d", (4096, 4096), 0.1, "cfg1like"),
    "3d_384x384x384_eb0.05": ("3d", (384, 384, 384), 0.05, "cfg2"),
    # profiling-size case of the 3D kernels (cfg2 generator at 256^3, 201 MB > L2)
    "3d_256x256x256_eb0.05": ("3d", (256, 256, 256), 0.05, "cfg2"),
    # 256 fields, sides uniform in [128, 4096], eb in {0.01, 0.05, 0.1}, one flow per 40x40 cells
    "batch_256x2d_cfg3": ("batch", None, None, "cfg3"),
    # the cfg1 field with learned bounds (trained proposer, fallback loop to 0 CP differences)
    "learned_2d_8192x8192_eb0.1": ("learned", (8192, 8192), 0.1, "cfg1"),
    # profiling-size case of the learned path: a held-out field of the proposer's training
    # generator (cfg0 density, sigma 40) at 2048^2 (34 MB of input)
    "learned_2d_2048x2048_eb0.1": ("learned", (2048, 2048), 0.1, "cfg0like_heldout"),
}
DEFAULT = "2d_8192x8192_eb0.1"


def _bf16_peak():
    """Dense BF16 tensor throughput (TFLOP/s) of MEASURED_PEAKS.json (burst), or the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "bf16_tflops" in d:
            return d["bf16_tflops"], "measured"
    return 1590.0, "fallback"


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


def CFG1LIKE_FLOWS(r1: int, r2: int) -> int:
    """Flows of a field with the 8192^2 workload's density (2000 per 8192^2)."""
    return max(1, round(2000 / (8192 * 8192) * r1 * r2))


def make_fields(workload: str, seed_offset: int = 0):
    from cpsz_b200 import workloads as W

    kind, shape, eb, gen = WORKLOADS[workload]
    if gen == "cfg1":
        return W.cfg1(1 + seed_offset), eb
    if gen == "cfg0":
        return W.cfg0(0 + seed_offset), eb
    if gen == "cfg0like":
        return W.cfg0_like(5 + seed_offset, *shape), eb
    if gen == "cfg1like":
        return W.field_2d(1 + seed_offset, *shape, CFG1LIKE_FLOWS(*shape), 60.0), eb
    if gen == "cfg0like_heldout":
        return W.cfg0_like(123457 + seed_offset, *shape), eb
    if gen == "cfg2":
        return W.cfg2(2 + seed_offset, shape[0]), eb
    raise KeyError(workload)


# ---- reference arm ----------------------------------------------------------------------
#
# The reference's own CPU implementation (oracle/_ref: its sources compiled
# here; the C restatement when that is absent) on the same workload, one
# single-threaded process per host core.  The arm never loads the product
# library: inputs come from the oracle's C generator, which builds the
# product's seeded fields bit for bit (tests/test_oracle_gen.py).

def oracle_fields(workload: str, seed_offset: int = 0):
    """The workload's fields from the oracle's generator (no product code)."""
    from oracle import Oracle

    O = Oracle()
    kind, shape, eb, gen = WORKLOADS[workload]
    if gen == "cfg1":
        return O.field_2d(1 + seed_offset, 8192, 8192, 2000, 60.0), eb
    if gen == "cfg1like":
        return O.field_2d(1 + seed_offset, *shape, CFG1LIKE_FLOWS(*shape), 60.0), eb
    if gen == "cfg0":
        return O.field_2d(0 + seed_offset, 2400, 3600, 200, 40.0), eb
    if gen in ("cfg0like", "cfg0like_heldout"):
        r1, r2 = shape
        seed = (5 if gen == "cfg0like" else 123457) + seed_offset
        return O.field_2d(seed, r1, r2, max(1, round(200 / (2400 * 3600) * r1 * r2)), 40.0), eb
    if gen == "cfg2":
        return O.field_3d(2 + seed_offset, *shape, 500, 20.0), eb
    raise KeyError(workload)


def _ref_child(conn, kind, field_src, use_ref):
    """One reference process: loads (or generates) its fields once, then on
    every request compresses all of them and replies with the seconds taken."""
    sys.path.insert(0, ROOT)
    import oracle

    impl = oracle.Reference() if use_ref else oracle.Oracle()
    fields = []
    if field_src[0] == "files":
        for paths, eb in field_src[1]:
            fields.append(([np.ascontiguousarray(np.load(p)) for p in paths], eb))
    else:  # ("batch", [(r1, r2, seed, eb), ...]): this process's fields of the batch
        O = oracle.Oracle()
        for r1, r2, seed, eb in field_src[1]:
            fields.append((list(O.field_2d(seed, r1, r2, max(1, (r1 * r2) // 1600), 40.0)), eb))
    conn.send(sum(a.nbytes for arrs, _ in fields for a in arrs))
    while conn.recv():
        t0 = time.perf_counter()
        for arrs, eb in fields:
            if kind == "3d":
                impl.compress_3d(arrs[0], arrs[1], arrs[2], eb)
            else:
                impl.compress_2d(arrs[0], arrs[1], eb)
        conn.send(time.perf_counter() - t0)
    conn.close()


def _host_procs(per_proc_bytes: float) -> int:
    """Processes to run: one per host core, as many as memory holds."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil

        avail = psutil.virtual_memory().available
        cores = min(cores, max(1, int(avail * 0.7 // per_proc_bytes)))
    except Exception:
        pass
    return max(1, cores)


def run_reference(args, rank, world):
    import multiprocessing as mp
    import tempfile

    import oracle

    if rank != 0:
        return None
    wk = WORKLOADS[args.workload][0]
    use_ref = os.path.exists(oracle.REF_SO)
    tmp = None
    if wk == "batch":
        # the whole batch each step: its fields split over the processes by
        # greedy size balance, each process generating the fields it owns
        lay = oracle.Oracle().batch_layout(3, 256, 128, 4096)
        nproc = _host_procs(2.5e9)
        bins = [[] for _ in range(nproc)]
        load = [0] * nproc
        for k in sorted(range(len(lay)), key=lambda k: -lay[k][0] * lay[k][1]):
            q = load.index(min(load))
            bins[q].append(lay[k])
            load[q] += lay[k][0] * lay[k][1]
        srcs = [("batch", b) for b in bins if b]
        kind = "2d"
        sample = f"the whole 256-field batch per step, split over {len(srcs)} single-threaded processes"
    else:
        fields, eb = oracle_fields(args.workload)
        kind = "3d" if wk == "3d" else "2d"
        if kind == "3d":
            # a 192^3 block of the field per process (the whole 384^3 field takes
            # about 45 s per process, too long for a step)
            fields = tuple(np.ascontiguousarray(a[:192, :192, :192]) for a in fields)
        nbytes = sum(a.nbytes for a in fields)
        nproc = _host_procs(4.0 * nbytes + 0.5e9)
        tmp = tempfile.mkdtemp(prefix="cpsz_ref_")
        paths = []
        for c, a in enumerate(fields):
            p = os.path.join(tmp, f"f{c}.npy")
            np.save(p, a)
            paths.append(p)
        del fields
        srcs = [("files", [(paths, eb)])] * nproc
        what = "192^3 block" if kind == "3d" else f"whole {'x'.join(map(str, WORKLOADS[args.workload][1]))} field"
        sample = f"the {what} per process, {nproc} single-threaded processes compressing concurrently per step"
    ctxm = mp.get_context("spawn")
    procs, conns = [], []
    try:
        for src in srcs:
            a, b = ctxm.Pipe()
            pr = ctxm.Process(target=_ref_child, args=(b, kind, src, use_ref), daemon=True)
            pr.start()
            procs.append(pr)
            conns.append(a)
        step_bytes = sum(c.recv() for c in conns)
        times = []
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            for c in conns:
                c.send(True)
            for c in conns:
                c.recv()
            if step >= args.warmup:
                times.append(time.perf_counter() - t0)
        for c in conns:
            c.send(False)
        for pr in procs:
            pr.join(timeout=60)
    finally:
        for pr in procs:
            if pr.is_alive():
                pr.terminate()
        if tmp:
            import shutil

            shutil.rmtree(tmp, ignore_errors=True)
    per_step = statistics.mean(times)
    gbs = step_bytes / per_step / 1e9
    line = {
        "impl": "reference", "metric": "compress_GBps", "value": round(gbs, 4), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic", "config": {"workload": args.workload},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": len(srcs),
                         "kind": "reference" if use_ref else "port", "sample": sample},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


# ---- product arm -----------------------------------------------------------------------

def _meaninfo_padding_2d(blob: bytes) -> np.ndarray:
    """False at the 3 padding bytes of each field's meanInfo<float> record,
    which the reference writes uninitialised (src/sz_compress_3d.cpp:222)."""
    import struct

    m = np.ones(len(blob), bool)
    eb_size, u_size, _ = struct.unpack_from("<QQQ", blob, 12)
    for off in (36 + eb_size, 36 + eb_size + u_size):
        m[off + 10: off + 13] = False
    return m


def cpu_baseline_single(workload, fields, eb, gpu_blob=None):
    """The reference CPU implementation (1 core: the reference is
    single-threaded), ZSTD timed apart.  2D: the whole field (about 10 s at
    8192^2), whose blob is also compared with the GPU's (`parity`); 3D: the
    first 96^3 blocks of the field for about 12 s."""
    import oracle

    use_ref = os.path.exists(oracle.REF_SO)
    impl = oracle.Reference() if use_ref else oracle.Oracle()
    kind = WORKLOADS[workload][0]
    parity = None
    zt = 0.0
    if kind in ("2d", "learned"):
        U, V = (np.ascontiguousarray(a) for a in fields)
        t0 = time.perf_counter()
        blob = impl.compress_2d(U, V, eb)
        t_total = time.perf_counter() - t0
        t0 = time.perf_counter()
        impl.zstd_compress(blob) if use_ref else None
        zt = time.perf_counter() - t0
        nbytes = U.nbytes + V.nbytes
        sample = f"the whole {U.shape[0]}x{U.shape[1]} field, 1 thread, {t_total:.1f} s"
        if gpu_blob is not None:
            same = len(blob) == len(gpu_blob)
            if same:
                x = np.frombuffer(blob, np.uint8)
                y = np.frombuffer(gpu_blob, np.uint8)
                same = bool(((x == y) | ~_meaninfo_padding_2d(blob)).all())
            parity = {"blob_equal_reference": same, "bytes": len(blob),
                      "compared": "whole blob against the reference's own compressor on the same field "
                                  "(the 6 indeterminate meanInfo padding bytes masked)"}
    else:
        s = 96
        U, V, Wf = fields
        t_total, nbytes, n = 0.0, 0, 0
        for i in range(0, U.shape[0] - s + 1, s):
            t = [np.ascontiguousarray(a[i:i + s, :s, :s]) for a in (U, V, Wf)]
            t0 = time.perf_counter()
            blob = impl.compress_3d(t[0], t[1], t[2], eb)
            t_total += time.perf_counter() - t0
            if use_ref:
                t0 = time.perf_counter()
                impl.zstd_compress(blob)
                zt += time.perf_counter() - t0
            nbytes += sum(a.nbytes for a in t)
            n += 1
            if t_total > 12.0:
                break
        sample = f"{n} blocks 96^3 of the workload, 1 thread, {t_total:.1f} s"
    if use_ref:
        sample += f"; host ZSTD stage separately {nbytes / max(zt, 1e-9) / 1e9:.3f} GB/s"
    return {"value": round(nbytes / t_total / 1e9, 5), "unit": "GB/s", "cores": 1,
            "kind": "reference" if use_ref else "port", "sample": sample}, parity


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
    # ---- end to end with the lossless stage on the GPU: pinned host fields
    # in, the blob built in device memory, a Zstandard frame of it written on
    # the GPU (the reference's sz_lossless_decompress reads it) and read back
    # into pinned host memory ----
    lossless_gpu = None
    if kind == "2d":
        h_frame = torch.empty(e2e_size + e2e_size // 64 + (1 << 20), dtype=torch.uint8).pin_memory().numpy()

        def step_lossless():
            n = comp(*hptr, *shape, eb, d_out, ctx=ctx)
            return cpsz_b200.lossless_compress_gpu(d_out[:n], out=h_frame, ctx=ctx)

        for _ in range(2):
            fsize = step_lossless()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fsize = step_lossless()
        ll_ms = (time.perf_counter() - t0) * 1e3 / args.steps
        frame = h_frame[:fsize].tobytes()
        lossless_gpu = {"e2e": round(raw_bytes / (ll_ms / 1e3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(ll_ms, 4),
                        "frame_bytes": fsize, "ratio": round(raw_bytes / fsize, 4),
                        "frame_decodes_to_blob": cpsz_b200.sz_lossless_decompress(frame, len(blob)) == blob}
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
    # the timed blob's decode against the input: exact critical-point
    # comparison of every cell (lost, spurious or retyped) and the point-wise
    # relative bound |decoded - x| <= max_pwr_eb * |x|
    check = cp_and_bound_check(kind, fields, outs, eb, ctx)

    stages = {k: statistics.mean(v) for k, v in stage_acc.items()}
    n = int(np.prod(shape))
    roof = product_roofline(kind, n, stages, clk.summary().get("sm_mhz"))
    return {
        "value": value, "ms": ms, "e2e_ms": e2e_ms, "dec_ms": dec_ms, "blob": len(blob), "size_dev": size,
        "lossless": len(lossless), "lossless_gpu": lossless_gpu, "raw": raw_bytes, "stages": stages, "roofline": roof,
        "launches": launches,
        "clocks": clk.summary(), "fields": fields, "eb": eb, "blob_bytes": blob, "check": check,
    }


def product_roofline(kind, n, stages, sm_mhz):
    """The roofline of the step's dominant kernel (the stage with the longest
    CUDA-event time among those with algorithmic bytes) for a field of `n`
    points: its algorithmic bytes over the stage time against the measured
    copy bandwidth, its DRAM traffic, and for a kernel bound by instruction
    issue its issue roofline.  None when no such stage was timed."""
    comps = 2 if kind == "2d" else 3
    # algorithmic bytes per launch of each stage's dominant kernel
    alg = {"eb2d": 4 * comps * n + comps * n,  # read fields, write one id byte per component
           "wave2d_compress": 4 * comps * n + comps * n + 2 * comps * n,  # fields + ids in, u16 codes out
           "eb3d": 4 * 3 * n + n, "wave3d_compress": 0}  # read fields, write one id byte
    # DRAM bytes per point of a launch, read + write, from one ncu capture of the
    # kernel on the 4096^2 case (389.4 MB for 16.8 M vertices), scaled to this
    # launch by its points
    traffic_per_point = {"eb2d": (134.725632e6 + 254.642176e6) / 4096 ** 2}
    dom = max((k for k in stages if k in alg and alg[k]), key=lambda k: stages[k], default=None)
    if not dom:
        return None
    peak, peak_kind = measured_peaks()
    ach = alg[dom] / (stages[dom] / 1e3) / 1e9
    tr = traffic_per_point.get(dom)
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4), "traffic": round(tr * n) if tr else None, "peak_source": peak_kind,
            "algorithmic_bytes": alg[dom]}
    issue = issue_roofline(dom, n, stages[dom], sm_mhz)
    if issue:
        roof["issue"] = issue
    return roof


# Warp instructions per point of a kernel that is bound by instruction issue
# rather than by HBM, from one ncu capture of it on the 4096^2 case
# (smsp__inst_executed.sum: 404,377,736 for 16.8 M vertices).
INSTR_PER_POINT = {"eb2d": 404377736 / 4096 ** 2}
B200_SMS = 148
ISSUE_PER_SM_CYCLE = 4  # one warp instruction a cycle on each of an SM's four schedulers


def issue_roofline(kernel, points, ms, sm_mhz):
    """The issue roofline of `kernel` over a launch of `points` points that
    took `ms`: its warp instructions (scaled from the captured case by the
    points) a second against 4 a cycle on each of the 148 SMs at the SM clock
    sampled during the run; None when the kernel has no captured count or no
    clock was sampled."""
    per = INSTR_PER_POINT.get(kernel)
    if per is None or not sm_mhz or not ms or ms <= 0:
        return None
    instr = per * points
    achieved = instr / (ms / 1e3) / 1e9
    peak = B200_SMS * ISSUE_PER_SM_CYCLE * float(sm_mhz) * 1e6 / 1e9
    return {"achieved": round(achieved, 2), "peak": round(peak, 2), "unit": "G warp instructions/s",
            "frac": round(achieved / peak, 4), "instructions": round(instr),
            "min_ms": round(instr / (peak * 1e9) * 1e3, 4)}


def cp_and_bound_check(kind, fields, decoded, eb, ctx):
    """{cp_errors, cps, bound_violations} of a decode: CP cells compared with
    the exact checker on the GPU; the bound checked on the host in double."""
    import cpsz_b200

    if kind == "3d":
        c = cpsz_b200.cp_check_3d(*fields, *decoded, ctx=ctx)
    else:
        c = cpsz_b200.cp_check_2d(*fields, *decoded, ctx=ctx)
    viol = 0
    for x, d in zip(fields, decoded):
        x64 = x.astype(np.float64)
        viol += int(np.count_nonzero(np.abs(d.astype(np.float64) - x64) > eb * np.abs(x64)))
    return {"cp_errors": int(c["lost_or_spurious"] + c["type_changed"]), "cps": int(c["cps_a"]),
            "bound_violations": viol}


def run_learned(args, rank, world, device):
    """Learned-bound compression of the cfg1 field: every step runs the MLP over
    all vertices, the fallback loop's reconstruction passes and the final
    compression (fields resident in HBM, blob written to HBM); the plain
    compressor's ratio and the exact CP comparison are reported beside it."""
    import torch

    import cpsz_b200
    from cpsz_b200 import learned

    kind, shape, eb, _ = WORKLOADS[args.workload]
    fields, eb = make_fields(args.workload, seed_offset=rank)
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
    viol = 0
    for x, d in zip(fields, (dU, dV)):
        x64 = x.astype(np.float64)
        viol += int(np.count_nonzero(np.abs(d.astype(np.float64) - x64) > eb * np.abs(x64)))
    # roofline of the tensor-core part: the fused MLP forward over every vertex
    # (2 * (128*128 + 128*128 + 128) flops a vertex, the 99 inputs padded to 128)
    eb_a, _ = cpsz_b200.debug_eb2d(*fields, eb, ctx=ctx, exact=True)
    d_eb = torch.from_numpy(np.ascontiguousarray(eb_a, np.float64)).to(f"cuda:{device}")
    fwd_ms = mlp.forward_ms(dev[0], dev[1], d_eb, reps=5)
    n = int(np.prod(shape))
    flops = 2.0 * (128 * 128 * 2 + 128) * n
    tf = flops / (fwd_ms / 1e3) / 1e12
    peak = _bf16_peak()
    # DRAM bytes of a launch from one ncu capture on the 2048^2 case (72.5 MB for
    # 4.19 M vertices: fields and exact bounds in, proposals out), scaled by points
    traffic = round((67.25376e6 + 5.274112e6) / 2048 ** 2 * n)
    roofline = {"bound": "tensor", "kernel": "mlp_fwd (features fused)", "achieved": round(tf, 2),
                "peak": peak[0], "unit": "TFLOP/s", "frac": round(tf / peak[0], 4), "traffic": traffic,
                "peak_source": peak[1], "ms_per_launch": round(fwd_ms, 3)}
    # the reference's CPU path on the same field (1 core, the plain method; the
    # reference has no learned form), and its decoder reading the learned blob
    cpu, ref_decodes = None, None
    if rank == 0 and not args.no_cpu_baseline:
        cpu, _ = cpu_baseline_single(args.workload, fields, eb)
        import oracle

        if os.path.exists(oracle.REF_SO):
            ru, rv = oracle.Reference().decompress_2d(blob, *shape)
            ref_decodes = bool(np.array_equal(ru.view(np.uint32), dU.view(np.uint32)) and
                               np.array_equal(rv.view(np.uint32), dV.view(np.uint32)))
    return {
        "metric": "compress_GBps", "value": round(raw * world / (ms / 1e3) / 1e9, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f64+f32", "data": "synthetic",
        "config": {"workload": args.workload, "tuning": _tuning_tag(), "eb": eb, "points": int(raw // 8), "inputs_exceed_l2": True,
                   "parallelism": f"replicas{world}", "value_io": "fields resident in HBM, blob written to HBM"},
        "ratio": round(raw / z_learned, 4), "ratio_pre_zstd": round(raw / size, 4),
        "plain_ratio": round(raw / z_plain, 4), "plain_ratio_pre_zstd": round(raw / len(plain), 4),
        "cp_check": cp, "cp_errors": int(cp["lost_or_spurious"] + cp["type_changed"]), "bound_violations": viol,
        "reference_decoder_reads_blob": ref_decodes, "loop": st, "roofline": roofline, "cpu_baseline": cpu,
        "clocks": clk.summary(), "gpu_launches": launches,
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
    kind = WORKLOADS[args.workload][0]
    r = run_product(args, rank, world, local)
    cpu, parity = None, None
    if rank == 0 and not args.no_cpu_baseline:
        cpu, parity = cpu_baseline_single(args.workload, r["fields"], r["eb"],
                                          r["blob_bytes"] if kind == "2d" else None)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
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
        # the same, with the lossless stage on the GPU (frame read back instead of the blob)
        "e2e_with_lossless_gpu": r["lossless_gpu"],
        "roofline": r["roofline"], "stages_ms": {k: round(v, 4) for k, v in r["stages"].items()},
        "cpu_baseline": cpu, "parity": parity, **r["check"], "clocks": r["clocks"], "gpu_launches": r["launches"],
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
