"""Benchmark of the B200 FastLanes / ALP decoding library on one B200.

Headline (`value`): FFOR decode at scale (the FFOR bit-unpack benchmark
configuration): one uint32 column of 2^28 values for every bit width 0..32
and one uint64 column of 2^27 values for every bit width 0..64, values =
per-vector base + uniform [0, 2^w).  A step decodes every column once into
HBM through the library's C ABI.  The default run then measures the rest of
the benchmark metric in the same invocation, each block with its own clock
samples: the same columns decoded and summed (`ffor_sum`), ALP / ALP-RD /
f32 ALP decode (`alp_decode`), 2 000 uneven columns decoded by the batched
persistent launch against one launch per column plus the pair query
(`batch_decode`), and the learned ALP encoder against the plain search
(`learned_encode`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload ffor|ffor-sum|alp|batch|learned|autotune]
                    [--scale S] [--no-extras] [--no-e2e]

Prints one JSON line (rank 0).  value = (compressed bytes read + decoded
bytes written) / device time, whole job.  Inputs are generated on the
device, as random packed words (every value uniform in [0, 2^w)), and every
column's output (1 GiB) is larger than L2, so no flush is needed between
steps.  Multi-GPU runs are independent replicas (the decode path has no
exchange step): every rank decodes the full column set on its own GPU."""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "msc-thesis-project_b200"))
sys.path.insert(0, str(ROOT / "tests"))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# algorithmic bytes of one headline step (98 FFOR columns, compressed read +
# decoded write), for relating the bounded e2e sample to the headline
HEADLINE_STEP_BYTES = sum(
    (n // 1024) * (w * 128 + b // 8 + 9) + n * b // 8
    for b, n, ws in ((32, 2 ** 28, range(33)), (64, 2 ** 27, range(65))) for w in ws)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler is live
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [x.strip() for x in l.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def profiled_traffic(name: str, alg_bytes_per_launch: float):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of the dominant kernel, from the committed ncu summary `profiles/<name>`,
    scaled to this run's launch size by algorithmic bytes (the capture shows
    traffic proportional to them).  None when the summary is absent."""
    p = Path(__file__).resolve().parent / "profiles" / name
    try:
        txt = p.read_text()
    except OSError:
        return None
    vals = {}
    for line in txt.splitlines():
        k, _, v = line.strip().partition(":")
        if k in ("traffic_bytes_per_launch", "algorithmic_bytes_per_launch"):
            vals[k] = float(v)
    if len(vals) != 2:
        return None
    return round(vals["traffic_bytes_per_launch"] / vals["algorithmic_bytes_per_launch"]
                 * alg_bytes_per_launch)


def dist_init():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The largest of the ranks' values (the slowest replica's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_loop(fn, stream, steps: int, warmup: int, min_seconds: float = 1.5):
    """Mean device time (ms) of fn() over at least `steps` calls and at least
    min_seconds of device time (so that the clock sampler sees the load),
    after `warmup` untimed calls; CUDA events on `stream`.  Returns
    (ms per call, calls timed)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    est = max(e0.elapsed_time(e1), 1e-3)
    n = max(steps, int(min_seconds * 1e3 / est) + 1)
    e0.record(stream)
    for _ in range(n):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / n, n


def job_gbs(bytes_per_replica_step: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job GB/s of `world` replicas each moving bytes_per_replica_step
    per step, timed by the slowest replica."""
    return bytes_per_replica_step * steps * world / (max_ms / 1e3) / 1e9


# ---------------------------------------------------------------------------
# workload: FFOR at scale
# ---------------------------------------------------------------------------
def make_ffor_columns(scale: float, dev, only=None):
    """One u32 column of 2^28 * scale values per width 0..32, one u64 column
    of 2^27 * scale values per width 0..64; random packed words (so every
    value is uniform in [0, 2^w)), random bases.  `only`: a set of
    (bits, width) to build, for profiling one column."""
    import torch
    import flsgpu_b200 as F
    cols = []
    g = torch.Generator(device=dev)
    g.manual_seed(1234)
    for bits, n_values in ((32, int(2 ** 28 * scale)), (64, int(2 ** 27 * scale))):
        n_values -= n_values % 1024
        n_vecs = n_values // 1024
        nl = 1024 // bits
        for w in range(bits + 1):
            if only is not None and (bits, w) not in only:
                continue
            n_words = n_vecs * w * nl
            packed = torch.randint(-2 ** 31, 2 ** 31, (max(n_words, 1) * (bits // 32),),
                                   dtype=torch.int32, device=dev, generator=g)
            packed = packed.view(torch.int64) if bits == 64 else packed
            bw = torch.full((n_vecs,), w, dtype=torch.uint8, device=dev)
            offs = torch.arange(n_vecs, dtype=torch.int64, device=dev) * (w * nl)
            bases = torch.randint(-2 ** 31, 2 ** 31, (n_vecs * (bits // 32),), dtype=torch.int32,
                                  device=dev, generator=g)
            bases = bases.view(torch.int64) if bits == 64 else bases
            bp = F.BPColumnC(n_values, n_vecs, packed.data_ptr(), bw.data_ptr(), offs.data_ptr())
            c = F.DeviceColumn("ffor", f"u{bits}", n_values,
                               F.FFORColumnC(n_values, bp, bases.data_ptr()),
                               {"packed": packed[:n_words * (bits // 32)] if bits == 32 else packed[:n_words],
                                "bit_widths": bw, "vector_offsets": offs, "bases": bases,
                                "_keep": packed}, n_words)
            cols.append((bits, w, c))
    return cols


def col_bytes(c) -> tuple[int, int]:
    """(compressed bytes read, decoded bytes written) by one full decode:
    packed words + base + bit width + vector offset per vector; output."""
    bits = int(c.dtype[1:])
    read = c.n_packed * bits // 8 + c.n_vecs * (bits // 8 + 1 + 8)
    return read, c.n_values * bits // 8


def run_ffor(args, rank, world, dev):
    import torch
    import flsgpu_b200 as F

    only = None
    if args.only:
        only = {(int(t.split(":")[0][1:]), int(t.split(":")[1])) for t in args.only.split(",")}
    cols = make_ffor_columns(args.scale, dev, only)
    cols_n = range(len(cols))
    out = torch.empty(max(c.n_values for _, _, c in cols) * 8 // 4, dtype=torch.int32, device=dev)
    total_read = sum(col_bytes(c)[0] for _, _, c in cols)
    total_write = sum(col_bytes(c)[1] for _, _, c in cols)
    stream = torch.cuda.current_stream()
    fsum = args.workload == "ffor-sum"
    sums = torch.zeros(len(cols), dtype=torch.int64, device=dev)

    def step(events=None):
        for i, (bits, w, c) in enumerate(cols):
            if events is not None:
                events[i][0].record(stream)
            if fsum:
                F.sum_(c, out=sums[i:i + 1], stream=stream)
            else:
                F.decompress(c, out=out.view(torch.int64 if bits == 64 else torch.int32)[:c.n_values],
                             stream=stream)
            if events is not None:
                events[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    events = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in cols] for _ in range(args.steps)]
    launches0 = F.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for s in range(args.steps):
            step(events[s])
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = F.launch_count() - launches0
    ms = t0.elapsed_time(t1)
    ms = max_over_ranks(ms, world)
    per_col_ms = [[events[s][i][0].elapsed_time(events[s][i][1]) for s in range(args.steps)]
                  for i in range(len(cols))]
    read_b = total_read if not fsum else total_read
    write_b = total_write if not fsum else 8 * len(cols)
    bytes_step = read_b + write_b
    gbs = job_gbs(bytes_step, args.steps, world, ms)
    per_width = {"u32": [], "u64": []}
    for (bits, w, c), t in zip(cols, per_col_ms):
        r, wr = col_bytes(c)
        b = r + (wr if not fsum else 8)
        per_width[f"u{bits}"].append(round(b / (statistics.mean(t) / 1e3) / 1e9, 1))
    # dominant kernel: the FFOR decode launches (one per column); algorithmic
    # bytes / mean launch duration, over all columns
    kern_ms = sum(statistics.mean(t) for t in per_col_ms)
    achieved = bytes_step / (kern_ms / 1e3) / 1e9
    fsum_block = run_ffor_sum(args, cols, out, dev) if args.extras and not fsum else None
    del cols, out
    return dict(gbs=gbs, ms=ms, bytes_step=bytes_step, read=read_b, write=write_b,
                per_width=per_width, achieved=achieved, launches=launches, clocks=clk.summary(),
                uncompressed_gbs=total_write * args.steps * world / (ms / 1e3) / 1e9,
                n_columns=len(cols_n), fsum=fsum_block)


def run_ffor_sum(args, cols, out, dev):
    """The FFOR-at-scale columns decoded and summed (the fused-reduction
    kernel, flsgpu_sum_ffor_u32/u64; sums exact mod 2^64), and a full-size
    parity check of the sums of a few columns against a torch sum of the
    same columns' decoded output."""
    import torch
    import flsgpu_b200 as F
    stream = torch.cuda.current_stream()
    sums = torch.zeros(len(cols), dtype=torch.int64, device=dev)

    def step():
        for i, (bits, w, c) in enumerate(cols):
            F.sum_(c, out=sums[i:i + 1], stream=stream)

    launches0 = F.launch_count()
    step()
    torch.cuda.synchronize()
    launches = F.launch_count() - launches0
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms, n = timed_loop(step, stream, args.steps, args.warmup)
    exact = {}
    for i, (bits, w, c) in enumerate(cols):
        if (bits, w) not in ((32, 7), (32, 32), (64, 1), (64, 40), (64, 64)):
            continue
        o = out.view(torch.int64 if bits == 64 else torch.int32)[:c.n_values]
        F.decompress(c, out=o, stream=stream)
        ref = (o.to(torch.int64) & 0xFFFFFFFF).sum() if bits == 32 else o.sum()
        exact[f"u{bits}_w{w}"] = bool(int(ref.item()) == int(sums[i].item()))
    read = sum(col_bytes(c)[0] for _, _, c in cols)
    decoded = sum(col_bytes(c)[1] for _, _, c in cols)
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    gbs = (read + 8 * len(cols)) / (ms / 1e3) / 1e9
    return {"metric": "FFOR decode fused with a sum: GB/s of compressed bytes read + 8 B per column",
            "value": round(gbs, 1), "unit": "GB/s", f"frac_of_{pk_kind}": round(gbs / hbm, 4),
            "decoded_equivalent_gbs": round(decoded / (ms / 1e3) / 1e9, 1),
            "ms_per_step": round(ms, 3), "steps": n, "columns": len(cols),
            "kernel": "k_column<T, FFOR, S_SUM> (flsgpu_sum_ffor_u32/u64)",
            "bound_note": "at low widths a column's compressed reads take a few microseconds; "
                          "the kernel is then bound by each warp's load latency per vector "
                          "(reads only, nothing else in flight), not by HBM",
            "sum_exact_vs_decoded": exact, "gpu_launches_per_step": launches,
            "clocks": clk.summary()}


# ---------------------------------------------------------------------------
# workload: ALP / ALP-RD decode at scale
# ---------------------------------------------------------------------------
def make_alp_columns(scale: float, dev, seed: int = 31):
    """The ALP / ALP-RD decode configuration, generated on the device:
    * f64 ALP, 2^27 values: integers uniform in [-10^6, 10^6] divided by
      10^d (d uniform per vector in 0..4), 1% of positions replaced by random
      non-NaN 64-bit patterns; encoded by the library's GPU encoder (plain
      per-vector search);
    * f64 ALP-RD, 2^27 values uniform in [0, 1) with full mantissa, encoded
      by the library's GPU ALP-RD encoder (cut and dictionary per rowgroup of
      100 vectors);
    * f32 ALP, 2^28 values: integers uniform in [-10^6, 10^6] times the
      float 10^-d (d uniform per vector in 0..3: the values ALP decodes to),
      1% of positions replaced by random non-NaN 32-bit patterns; encoded by
      the library's GPU f32 encoder.
    Returns [(name, column, expected values, read bytes, written bytes)]."""
    import torch
    import flsgpu_b200 as F
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    out = []

    def exc_layout(mask, nv):
        counts = mask.view(nv, 1024).sum(1)
        offs = torch.zeros(nv, dtype=torch.int64, device=dev)
        offs[1:] = torch.cumsum(counts, 0)[:-1]
        flat = torch.nonzero(mask).squeeze(1)
        return counts.to(torch.int16), offs, flat, (flat % 1024).to(torch.int16)

    # f64 ALP, value level, GPU encoder
    n = int(2 ** 27 * scale) // 1024 * 1024
    nv = n // 1024
    ints = torch.randint(-10 ** 6, 10 ** 6 + 1, (n,), dtype=torch.int64, device=dev, generator=g)
    p10 = torch.tensor([1.0, 10.0, 100.0, 1000.0, 10000.0], dtype=torch.float64, device=dev)
    d = torch.randint(0, 5, (nv,), device=dev, generator=g).repeat_interleave(1024)
    vals = ints.double() / p10[d]
    m = torch.rand(n, device=dev, generator=g) < 0.01
    pat = torch.randint(-2 ** 63, 2 ** 63 - 1, (n,), dtype=torch.int64, device=dev, generator=g)
    pat = torch.where(torch.isnan(pat.view(torch.float64)), pat & ~(1 << 62), pat)
    vals.view(torch.int64)[m] = pat[m]
    del ints, d, m, pat
    enc = F.AlpEncoder(seed=1)
    res = enc.encode(vals, 0)
    col = F.encoded_column(res, n, enc)
    col.buffers["_enc"] = enc
    rd_b = int(res.n_packed_words) * 8 + nv * 29 + int(res.n_exceptions) * 10
    out.append(("alp_f64", col, vals, rd_b, n * 8))

    # f64 ALP-RD, encoded by the library's GPU ALP-RD encoder: one cut and
    # dictionary per rowgroup of 100 vectors (rd_encoder::init / encode)
    vals = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
    rres = enc.encode_rd(vals, rowgroup_vecs=100)
    col = F.rd_encoded_column(rres, n, "f64", enc)
    nv = n // 1024
    rd_b = (int(rres.n_right_words) * 8 + int(rres.n_left_words) * 2 + nv * 32
            + int(rres.n_dictionaries) * 16 + int(rres.n_exceptions) * 4)
    out.append(("alprd_f64", col, vals, rd_b, n * 8))

    # f32 ALP, value level: integers times the float 10^-d (the values ALP
    # decodes to), 1% random non-NaN patterns; encoded by the library's GPU
    # f32 encoder (plain per-vector search)
    n = int(2 ** 28 * scale) // 1024 * 1024
    nv = n // 1024
    ints = torch.randint(-10 ** 6, 10 ** 6 + 1, (n,), dtype=torch.int32, device=dev, generator=g)
    frac = torch.tensor([1.0, 0.1, 0.01, 0.001], dtype=torch.float32, device=dev)
    dv = torch.randint(0, 4, (nv,), device=dev, generator=g)
    vals = ints.float() * frac[dv.repeat_interleave(1024)]
    m = torch.rand(n, device=dev, generator=g) < 0.01
    pat = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), dtype=torch.int32, device=dev, generator=g)
    pat = torch.where(torch.isnan(pat.view(torch.float32)), pat & ~(1 << 30), pat)
    vals.view(torch.int32)[m] = pat[m]
    del ints, m, pat, dv
    enc32 = F.AlpEncoder(seed=3)
    res = enc32.encode_f32(vals)
    col = F.encoded_column(res, n, enc32, dtype="f32")
    rd_b = int(res.n_packed_words) * 4 + nv * 25 + int(res.n_exceptions) * 6
    out.append(("alp_f32", col, vals, rd_b, n * 4))
    return out


def cpu_reference_alp(cols, seconds_budget: float = 5.0, sample_vecs: int = 16384):
    """The reference's own CPU ALP decoder (alp::decode: falp + patch
    exceptions, compiled from the reference sources into oracle/_ref) on all
    host threads, over the first sample_vecs vectors of the f64 and f32 ALP
    columns (copied to host memory).  None when oracle/_ref is absent."""
    import flsgpu_b200 as F
    from oracle import binding as B
    r = B.ref()
    if r is None:
        return None
    threads = os.cpu_count() or 1
    work, bytes_one = [], 0
    for name, col, vals, rb, wb in cols:
        if name not in ("alp_f64", "alp_f32"):
            continue
        f64 = name == "alp_f64"
        ut, ft = (np.uint64, np.float64) if f64 else (np.uint32, np.float32)
        nl = 16 if f64 else 32
        c = col.c
        nv = min(sample_vecs, col.n_vecs)
        h = lambda ptr, n, dt: F.device_array(ptr, n, dt).cpu().numpy().view(dt)  # noqa: E731
        bw = h(c.ffor.bp.bit_widths, nv, np.uint8)
        offs = h(c.ffor.bp.vector_offsets, nv, np.uint64)
        counts = h(c.counts, nv, np.uint16)
        eoffs = h(c.exceptions_offsets, nv, np.uint64)
        n_words = int(offs[-1]) + int(bw[-1]) * nl
        n_exc = int(eoffs[-1]) + int(counts[-1])
        arrs = dict(packed=h(c.ffor.bp.packed_array, max(n_words, 1), ut), bw=bw, offs=offs,
                    bases=h(c.ffor.bases, nv, ut), fac=h(c.factor_indices, nv, np.uint8),
                    exp=h(c.fraction_indices, nv, np.uint8), eoffs=eoffs,
                    exc=h(c.exceptions, max(n_exc, 1), ft), pos=h(c.positions, max(n_exc, 1), np.uint16),
                    counts=counts, out=np.zeros(nv * 1024, ft))
        work.append((f64, nv, arrs))
        bytes_one += n_words * (8 if f64 else 4) + nv * (29 if f64 else 25) + n_exc * (10 if f64 else 6) \
            + nv * 1024 * (8 if f64 else 4)

    def run_one(f64, a, v0, v1):
        fn = r.ref_decode_alp_f64 if f64 else r.ref_decode_alp_f32
        fn(B.ptr(a["packed"]), B.ptr(a["bw"]), B.ptr(a["offs"]), B.ptr(a["bases"]), B.ptr(a["fac"]),
           B.ptr(a["exp"]), B.ptr(a["eoffs"]), B.ptr(a["exc"]), B.ptr(a["pos"]), B.ptr(a["counts"]),
           v0, v1, B.ptr(a["out"]))

    def one_pass(pool):
        futs = []
        for f64, nv, a in work:
            chunk = max(1, nv // threads)
            for v0 in range(0, nv, chunk):
                futs.append(pool.submit(run_one, f64, a, v0, min(nv, v0 + chunk)))
        for f in futs:
            f.result()

    with ThreadPoolExecutor(max_workers=threads) as pool:
        one_pass(pool)
        t = time.perf_counter()
        reps = 0
        while time.perf_counter() - t < seconds_budget:
            one_pass(pool)
            reps += 1
        el = time.perf_counter() - t
    return {"value": round(bytes_one * reps / el / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": "reference",
            "sample": f"first {sample_vecs} vectors of the f64 and f32 ALP columns, alp::decode "
                      f"(falp + patch, src/alp/alp-bindings.cu) per thread range, {reps} passes "
                      f"in {el:.1f} s"}


def extended_of(col, dev):
    """The ALP-extended (lane-divided) form of an f64 ALP DeviceColumn, built
    on the device as the reference's host-side conversion does
    (structs.cuh:231-306): a vector's exceptions regrouped by lane
    (position % 16), order kept within a lane, and per vector and lane
    (count << 10) | offset of the lane's first exception in the vector."""
    import torch
    import flsgpu_b200 as F
    c = col.c
    nv = col.n_vecs
    n_exc = int(c.n_exceptions)
    counts = F.device_array(c.counts, nv, np.uint16).to(torch.int64)
    exc = F.device_array(c.exceptions, n_exc, np.float64)
    pos = F.device_array(c.positions, n_exc, np.uint16).to(torch.int64) & 0xFFFF
    vec = torch.repeat_interleave(torch.arange(nv, device=dev), counts)
    key = vec * 16 + pos % 16
    order = torch.argsort(key * 1024 + pos)
    new_exc = exc[order].contiguous()
    new_pos = pos[order].to(torch.int16).contiguous()
    lane_counts = torch.bincount(key, minlength=nv * 16).view(nv, 16)
    lane_offs = torch.cumsum(lane_counts, 1) - lane_counts
    oc = ((lane_counts << 10) | lane_offs).to(torch.int32).to(torch.int16).contiguous()
    cx = F.ALPXColumnC(col.n_values, c.ffor, None, None, c.factor_indices, c.fraction_indices,
                       n_exc, c.exceptions_offsets, new_exc.data_ptr(), new_pos.data_ptr(),
                       oc.data_ptr())
    return F.DeviceColumn("alpx", "f64", col.n_values, cx,
                          {"_exc": new_exc, "_pos": new_pos, "_oc": oc, "_base": col},
                          col.n_packed), n_exc * 10 + nv * 16 * 2


def run_alp(args, rank, world, dev):
    import torch
    import flsgpu_b200 as F
    t0 = time.perf_counter()
    cols = make_alp_columns(args.scale, dev)
    gen_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    outs = [torch.empty_like(v) for _, _, v, _, _ in cols]
    exact = {}
    for (name, c, v, _, _), o in zip(cols, outs):
        F.decompress(c, out=o, stream=stream)
        ib = torch.int64 if v.element_size() == 8 else torch.int32
        exact[name] = bool(torch.equal(o.view(ib), v.view(ib)))

    def step(events=None):
        for i, ((name, c, v, _, _), o) in enumerate(zip(cols, outs)):
            if events is not None:
                events[i][0].record(stream)
            F.decompress(c, out=o, stream=stream)
            if events is not None:
                events[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # enough steps for at least 1.5 s of device time (a step is ~1 ms), so
    # that the clock sampler sees the load
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step()
    e1.record(stream)
    torch.cuda.synchronize()
    steps = max(args.steps, int(1500.0 / max(e0.elapsed_time(e1), 1e-3)) + 1)
    events = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in cols] for _ in range(steps)]
    launches0 = F.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for st in range(steps):
            step(events[st])
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = F.launch_count() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    per = {}
    kern_ms = 0.0
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    for i, (name, c, v, rb, wb) in enumerate(cols):
        t = statistics.mean(events[st][i][0].elapsed_time(events[st][i][1])
                            for st in range(steps))
        kern_ms += t
        gbs = (rb + wb) / (t / 1e3) / 1e9
        per[name] = {"gbs": round(gbs, 1), "ms": round(t, 4), f"frac_of_{pk_kind}": round(gbs / hbm, 4),
                     "read_bytes": rb, "write_bytes": wb, "bit_exact": exact[name],
                     "values": c.n_values}
    bytes_step = sum(rb + wb for _, _, _, rb, wb in cols)
    # the f64 column again in the lane-divided exception layout (the layout
    # the reference's ALP benchmark decodes), reported beside the headline
    xcol, x_extra = extended_of(cols[0][1], dev)
    xo = torch.empty_like(cols[0][2])
    F.decompress(xcol, out=xo, stream=stream)
    x_exact = bool(torch.equal(xo.view(torch.int64), cols[0][2].view(torch.int64)))
    for _ in range(args.warmup):
        F.decompress(xcol, out=xo, stream=stream)
    with ClockSampler(torch.cuda.current_device()) as xclk:
        x_ms, x_n = timed_loop(lambda: F.decompress(xcol, out=xo, stream=stream), stream,
                               args.steps, 0)
    x_bytes = cols[0][3] - cols[0][1].n_vecs * 2 + x_extra + cols[0][4]
    x_gbs = x_bytes / (x_ms / 1e3) / 1e9
    per["alp_f64_extended"] = {"gbs": round(x_gbs, 1), "ms": round(x_ms, 4),
                               f"frac_of_{pk_kind}": round(x_gbs / hbm, 4), "launches_timed": x_n,
                               "bit_exact": x_exact, "in_headline": False, "clocks": xclk.summary()}
    del xcol, xo
    cpu = cpu_reference_alp(cols, args.cpu_seconds / 2) if rank == 0 and world == 1 else None
    return dict(gbs=bytes_step * steps * world / (ms / 1e3) / 1e9, ms=ms, cpu=cpu, steps=steps,
                bytes_step=bytes_step, per=per, achieved=bytes_step / (kern_ms / 1e3) / 1e9,
                launches=launches, clocks=clk.summary(), gen_s=gen_s,
                exact=all(exact.values()) and x_exact)


# ---------------------------------------------------------------------------
# workload: batched uneven decode + fused pair query
# ---------------------------------------------------------------------------
def make_batch_columns(n_cols: int, dev, seed: int = 4):
    """n_cols columns, lengths log-uniform in 2^10..2^24 rounded up to 1024;
    types cycle (f64 ALP, u32 FFOR, f32 ALP); each f64 column and the u32
    column after it share a length and form a query pair (A, B).  Columns
    are generated at the compressed level, as the reference's own test data
    (src/engine/data.cuh:354-477): random packed words at a chosen width,
    FFOR widths uniform 0..32, ALP widths uniform 16..24 (the range that
    integers up to 10^6 scaled by 10^d encode to), ALP factor / exponent
    indices in the lower half of their tables, per-column exception rate
    uniform in [0, 5%] with positions spread over the vector."""
    import torch
    import flsgpu_b200 as F
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    cols, pairs = [], []
    length = 1024

    def rint32(n):
        return torch.randint(-2 ** 31, 2 ** 31, (max(n, 1),), dtype=torch.int32, device=dev,
                             generator=g)

    for i in range(n_cols):
        kind = i % 3
        if kind != 1:
            length = int(2 ** rng.uniform(10, 24))
            length = (length + 1023) // 1024 * 1024
        n_vecs = length // 1024
        if kind == 1:  # u32 FFOR
            w = int(rng.integers(0, 33))
            packed = rint32(n_vecs * w * 32)
            bw = torch.full((n_vecs,), w, dtype=torch.uint8, device=dev)
            offs = torch.arange(n_vecs, dtype=torch.int64, device=dev) * (w * 32)
            bases = rint32(n_vecs)
            bp = F.BPColumnC(length, n_vecs, packed.data_ptr(), bw.data_ptr(), offs.data_ptr())
            c = F.DeviceColumn("ffor", "u32", length, F.FFORColumnC(length, bp, bases.data_ptr()),
                               {"packed": packed[: n_vecs * w * 32], "bit_widths": bw,
                                "vector_offsets": offs, "bases": bases, "_keep": packed},
                               n_vecs * w * 32)
            pairs.append((cols[-1], c))
        else:
            f64 = kind == 0
            words = 2 if f64 else 1
            nl = 16 if f64 else 32
            w = int(rng.integers(16, 25))
            n_words = n_vecs * w * nl
            packed = rint32(n_words * words)
            bw = torch.full((n_vecs,), w, dtype=torch.uint8, device=dev)
            offs = torch.arange(n_vecs, dtype=torch.int64, device=dev) * (w * nl)
            bases = torch.randint(2, 21, (n_vecs,), dtype=torch.int64 if f64 else torch.int32,
                                  device=dev, generator=g)
            fac = torch.randint(0, 9 if f64 else 5, (n_vecs,), dtype=torch.uint8, device=dev,
                                generator=g)
            exp = torch.randint(0, 10 if f64 else 5, (n_vecs,), dtype=torch.uint8, device=dev,
                                generator=g)
            rate = float(rng.uniform(0.0, 0.05))
            cmax = int(round(2 * rate * 1024))
            counts = torch.randint(0, cmax + 1, (n_vecs,), dtype=torch.int32, device=dev,
                                   generator=g)
            eoffs = torch.cumsum(counts.to(torch.int64), 0) - counts.to(torch.int64)
            n_exc = int(counts.sum().item())
            step = 1024 // max(cmax, 1)
            # positions: exception j of vector v at j*step + (v*7 % step), sorted and distinct
            vec_of = torch.repeat_interleave(torch.arange(n_vecs, device=dev), counts.to(torch.int64))
            j = torch.arange(n_exc, device=dev) - eoffs[vec_of] if n_exc else torch.zeros(0, device=dev, dtype=torch.int64)
            pos = (j * step + (vec_of * 7) % step).to(torch.int16) if n_exc else torch.zeros(1, dtype=torch.int16, device=dev)
            exc = rint32(max(n_exc, 1) * words)
            exc = exc.view(torch.float64) if f64 else exc.view(torch.float32)
            fbuf = {"packed": packed[: n_words * words], "bit_widths": bw, "vector_offsets": offs,
                    "bases": bases, "factor_indices": fac, "fraction_indices": exp,
                    "exceptions_offsets": eoffs, "exceptions": exc[:n_exc], "positions": pos[:n_exc],
                    "counts": counts.to(torch.int16), "_keep": (packed, exc, pos)}
            bp = F.BPColumnC(length, n_vecs, packed.data_ptr(), bw.data_ptr(), offs.data_ptr())
            ff = F.FFORColumnC(length, bp, bases.data_ptr())
            ac = F.ALPColumnC(length, ff, None, None, fac.data_ptr(), exp.data_ptr(), n_exc,
                              eoffs.data_ptr(), exc.data_ptr(), pos.data_ptr(),
                              fbuf["counts"].data_ptr())
            c = F.DeviceColumn("alp", "f64" if f64 else "f32", length, ac, fbuf, n_words)
        cols.append(c)
    return cols, pairs


def run_batch(args, dev):
    import torch
    import flsgpu_b200 as F
    t0 = time.perf_counter()
    cols, pairs = make_batch_columns(args.columns, dev)
    outs = [torch.empty(c.n_values, dtype=getattr(torch, F.TORCH_OF_BITS[c.dtype]), device=dev)
            for c in cols]
    gen_s = time.perf_counter() - t0
    b = F.Batch(cols, outs)
    stream = torch.cuda.current_stream()
    read_b = sum(c.compressed_bytes() for c in cols)
    write_b = sum(o.numel() * o.element_size() for o in outs)

    def checksums():
        """Per-column checksum of the decoded bit patterns (wrapping int64
        sum), to compare the batched decode with per-column decodes."""
        return torch.stack([(o.view(torch.int32) if o.element_size() == 4 else o.view(torch.int64))
                            .to(torch.int64).sum() for o in outs])

    b.capture(stream)
    launches0 = F.launch_count()
    b.replay(stream)
    torch.cuda.synchronize()
    launches = F.launch_count() - launches0
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_graph, n_graph = timed_loop(lambda: b.replay(stream), stream, args.steps, args.warmup)
        ms_launch, _ = timed_loop(lambda: b.decompress(stream), stream, args.steps, args.warmup,
                                  min_seconds=0.5)
        ms_each, _ = timed_loop(lambda: b.decompress_each(False, stream), stream,
                                max(2, args.steps // 4), 2, min_seconds=0.5)
    ms_each_sync, _ = timed_loop(lambda: b.decompress_each(True, stream), stream, 2, 1,
                                 min_seconds=0.0)
    # full-size parity: the batched decode equals one flsgpu_decompress_*
    # per column, bit for bit (checksums of every column's output)
    for o in outs:
        o.fill_(0)
    b.replay(stream)
    cs_batch = checksums()
    for o in outs:
        o.fill_(0)
    b.decompress_each(False, stream)
    cs_each = checksums()
    batch_exact = bool(torch.equal(cs_batch, cs_each))
    q = F.PairQuery([p[0] for p in pairs], [p[1] for p in pairs], dev)
    q.capture(stream)
    with ClockSampler(torch.cuda.current_device()) as qclk:
        ms_query, _ = timed_loop(lambda: q.replay(stream), stream, max(3, args.steps // 2), 3,
                                 min_seconds=1.0)
    q_read = sum(a.compressed_bytes() + bb.compressed_bytes() for a, bb in pairs)
    del q, b
    return dict(ms=ms_graph, steps=n_graph, ms_launch=ms_launch, ms_each=ms_each,
                ms_each_sync=ms_each_sync, read=read_b, write=write_b, clocks=clk.summary(),
                launches=launches, n_values=sum(c.n_values for c in cols), gen_s=gen_s,
                ms_query=ms_query, q_read=q_read, n_pairs=len(pairs), q_clocks=qclk.summary(),
                exact_vs_per_column=batch_exact, n_columns=len(cols))


# ---------------------------------------------------------------------------
# workload: learned ALP parameter proposal vs the plain search (GPU encoder)
# ---------------------------------------------------------------------------
def learned_values(seed: int, n_vecs: int):
    """f64 columns of the learned-proposal shape: per vector d in {0..6}
    decimal digits, scale 10^k (k in 0..8), Gaussian or uniform magnitude;
    10% of the vectors are full-mantissa noise.  The same generator as the
    test suite's, so the network trained here sees the tests' distribution."""
    import numpy as np
    rng = np.random.default_rng(seed)
    d = rng.integers(0, 7, n_vecs)
    k = rng.integers(0, 9, n_vecs)
    gauss = rng.random(n_vecs) < 0.5
    noise = rng.random(n_vecs) < 0.1
    m = np.where(np.repeat(gauss, 1024), rng.standard_normal(n_vecs * 1024),
                 rng.uniform(-1.0, 1.0, n_vecs * 1024))
    scale = 10.0 ** np.repeat(k, 1024)
    dd = 10.0 ** np.repeat(d, 1024)
    vals = np.round(m * scale * dd) / dd
    vals = np.where(np.repeat(noise, 1024), m * scale, vals)
    return vals.astype(np.float64)


def run_learned(args, dev):
    """Trains the proposal network on one synthetic column (2^24 values) and
    encodes a second one of 2^26 values (the learned-proposal benchmark
    shape: per vector d in {0..6} decimals, scale 10^k, k in 0..8, Gaussian or
    uniform magnitude, 10% full-mantissa noise vectors) with the plain
    per-vector search and with the network's proposals."""
    import torch
    import flsgpu_b200 as F
    stream = torch.cuda.current_stream()
    n_eval = int(2 ** 26 * args.scale) // 1024 * 1024
    train = torch.from_numpy(learned_values(101, max(1024, int(2 ** 24 * args.scale) // 1024))).to(dev)
    evals = torch.from_numpy(learned_values(202, n_eval // 1024)).to(dev)
    enc = F.AlpEncoder(seed=7)
    t0 = time.perf_counter()
    l0, l1 = enc.train(train, epochs=args.epochs, batch=1024, lr=3e-3)
    train_s = time.perf_counter() - t0

    def ev_time(fn, min_seconds=0.5):
        return timed_loop(fn, stream, 3, 1, min_seconds=min_seconds)[0]

    res = {}
    with ClockSampler(torch.cuda.current_device()) as clk:
        # hybrid columns: vectors that call for ALP-RD are encoded as ALP-RD
        ms_plain = ev_time(lambda: res.__setitem__("plain", enc.encode_hybrid(evals, 0)))
        plain = res["plain"]
        plain_bytes, plain_rd = plain.compressed_bytes, int(plain.n_rd_vectors)
        dec = F.decompress(F.hybrid_column(plain, evals.numel(), enc))
        exact_plain = bool(torch.equal(dec.view(torch.int64), evals.view(torch.int64)))
        ms_learned = ev_time(lambda: res.__setitem__("learned", enc.encode_hybrid(evals, 1)))
        learned = res["learned"]
        hcol = F.hybrid_column(learned, evals.numel(), enc)
        dec = F.decompress(hcol)
        exact = bool(torch.equal(dec.view(torch.int64), evals.view(torch.int64))) and exact_plain
        # decode of the learned hybrid column (before the encoder's next
        # encode reuses its workspace)
        ms_hdec = ev_time(lambda: F.decompress(hcol, out=dec))
        # the same two encoders writing ALP-only columns (ALP-RD vectors kept
        # on their best ALP pair), as the reference's ALPColumn requires
        ms_plain_a = ev_time(lambda: res.__setitem__("plain_a", enc.encode(evals, 0)))
        ms_learned_a = ev_time(lambda: res.__setitem__("learned_a", enc.encode(evals, 1)))
        dec = F.decompress(F.encoded_column(res["learned_a"], evals.numel(), enc))
        exact = exact and bool(torch.equal(dec.view(torch.int64), evals.view(torch.int64)))
    del dec
    ms_search = ev_time(lambda: F.plain_labels(evals))
    ms_propose = ev_time(lambda: enc.propose(evals, 3))
    in_bytes = evals.numel() * 8
    # the reference's CPU encoder (oracle restatement, one thread) on the
    # same column: rowgroup sampling search, one state per rowgroup of 100
    # vectors as upstream ALP; rowgroups it would send to ALP-RD stay on
    # their ALP top-k so that the column is comparable
    from oracle import binding as B
    sample = evals.cpu().numpy()
    t = time.perf_counter()
    ref_col = B.alp_encode(sample, rowgroup_vecs=100, rd_as_alp=True)
    ref_s = time.perf_counter() - t
    alp_only = {"plain_ms": round(ms_plain_a, 3), "learned_ms": round(ms_learned_a, 3),
                "plain_ratio": round(in_bytes / res["plain_a"].compressed_bytes, 4),
                "learned_ratio": round(in_bytes / res["learned_a"].compressed_bytes, 4),
                "speedup": round(ms_plain_a / ms_learned_a, 2),
                "fallback_vectors": int(res["learned_a"].n_fallback)}
    return dict(ms_plain=ms_plain, ms_learned=ms_learned, ms_search=ms_search,
                ms_propose=ms_propose, in_bytes=in_bytes, plain_bytes=plain_bytes,
                learned_bytes=learned.compressed_bytes, fallback=int(learned.n_fallback),
                n_rd=int(learned.n_rd_vectors), plain_rd=plain_rd, alp_only=alp_only,
                n_vecs=evals.numel() // 1024, exact=exact, ms_hdec=ms_hdec,
                loss=(l0, l1), train_s=train_s, clocks=clk.summary(),
                ref_gbs=sample.nbytes / ref_s / 1e9 if ref_col is not None else None,
                ref_ratio=sample.nbytes / ref_col["compressed_bytes"] if ref_col is not None else None)


# ---------------------------------------------------------------------------
# end-to-end through the C ABI with host buffers (bounded sample)
# ---------------------------------------------------------------------------
def run_e2e(args, dev):
    """End to end through the library's host-buffer API (flsgpu_host_*): per
    step every column's packed words and metadata go from pinned host memory
    to the device and the decoded values come back, chunk by chunk on three
    streams (copies in both directions overlap the decode).  Sample: one u32
    column of 2^26 values for w in {1, 7, 16, 32} and one u64 column of 2^25
    values for w in {1, 20, 40, 64}.  Timed on the host clock around whole
    synchronous calls (the pipeline's streams are the library's own)."""
    import torch
    import flsgpu_b200 as F
    rng = np.random.default_rng(7)
    pipe = F.HostPipeline(chunk_values=1 << 22)
    jobs = []
    for bits, n_values, widths in ((32, 2 ** 26, (1, 7, 16, 32)), (64, 2 ** 25, (1, 20, 40, 64))):
        n_vecs = n_values // 1024
        nl = 1024 // bits
        ut = np.uint64 if bits == 64 else np.uint32
        sd = np.int64 if bits == 64 else np.int32
        td = torch.int64 if bits == 64 else torch.int32
        for w in widths:
            packed = torch.from_numpy(rng.integers(0, 2 ** bits, n_vecs * w * nl, dtype=np.uint64)
                                      .astype(ut).view(sd)).pin_memory()
            bw = torch.full((n_vecs,), w, dtype=torch.uint8).pin_memory()
            offs = (torch.arange(n_vecs, dtype=torch.int64) * (w * nl)).pin_memory()
            bases = torch.from_numpy(rng.integers(0, 2 ** 30, n_vecs).astype(sd)).pin_memory()
            desc, kind, dt, keep = F.host_ffor_column(packed, bw, offs, bases, n_values)
            out_h = torch.empty(n_values, dtype=td).pin_memory()
            jobs.append((desc, kind, dt, keep, out_h, n_values, bits, w))

    def step():
        for desc, kind, dt, keep, out_h, *_ in jobs:
            pipe.decompress(desc, kind, dt, out_h, wait=False)
        pipe.sync()

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    h2d = sum(sum(t.numel() * t.element_size() for t in j[3]) for j in jobs)
    d2h = sum(j[4].numel() * j[4].element_size() for j in jobs)
    reads = sum(n * w // 8 + n // 1024 * (bits // 8 + 9) for *_, n, bits, w in jobs)
    writes = sum(n * bits // 8 for *_, n, bits, w in jobs)
    n = 3
    t0 = time.perf_counter()
    for _ in range(n):
        step()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / n
    return {"value": round((reads + writes) / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(ms, 3),
            "share_of_headline": {"columns": "8 of the headline's 98 (u32 w 1, 7, 16, 32; u64 w 1, "
                                             "20, 40, 64), a quarter of their values each",
                                  "bytes_fraction": round((reads + writes) / HEADLINE_STEP_BYTES, 4),
                                  "bound": "PCIe: every step moves the compressed column in and the "
                                           "decoded values out"},
            "sample": "u32 2^26 values x w{1,7,16,32} + u64 2^25 x w{1,20,40,64}, pinned host "
                      "buffers, flsgpu_host_decompress_ffor_*_async for the 8 columns then "
                      "flsgpu_host_pipeline_sync (chunks of 2^22 values, copies overlapping the "
                      "decode and each other), host clock around each step"}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own unffor (oracle/_ref), all host cores
# ---------------------------------------------------------------------------
def cpu_reference_ffor(seconds_budget: float = 10.0, threads: int | None = None):
    from oracle import binding as B
    r = B.ref()
    kind = "reference"
    if r is None:
        r = B.oracle()
        kind = "port"
    threads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(3)
    work = []
    for bits, n_vecs in ((32, 2048), (64, 1024)):
        ut = np.uint64 if bits == 64 else np.uint32
        nl = 1024 // bits
        for w in range(bits + 1):
            packed = rng.integers(0, 2 ** bits, max(n_vecs * w * nl, 1), dtype=np.uint64).astype(ut)
            bw = np.full(n_vecs, w, np.uint8)
            offs = (np.arange(n_vecs, dtype=np.uint64) * (w * nl)).astype(np.uint64)
            bases = rng.integers(0, 2 ** 30, n_vecs).astype(ut)
            out = np.zeros(n_vecs * 1024, ut)
            work.append((bits, w, packed, bw, offs, bases, out, n_vecs))
    bytes_one = sum(n * w * (1024 // b) * b // 8 + n * (b // 8 + 9) + n * 1024 * b // 8
                    for b, w, _, _, _, _, _, n in work)

    def run_one(item, v0, v1):
        bits, w, packed, bw, offs, bases, out, n = item
        if kind == "reference":
            fn = r.ref_decode_ffor_u32 if bits == 32 else r.ref_decode_ffor_u64
            fn(B.ptr(packed), B.ptr(bw), B.ptr(offs), B.ptr(bases), v0, v1, B.ptr(out))
        else:
            fn = r.orc_decode_ffor_u32 if bits == 32 else r.orc_decode_ffor_u64
            fn(B.ptr(packed), B.ptr(bw), B.ptr(offs + 0), B.ptr(bases), v1 - v0, B.ptr(out))

    def one_pass(pool):
        futs = []
        for item in work:
            n = item[7]
            chunk = max(1, n // threads)
            for v0 in range(0, n, chunk):
                futs.append(pool.submit(run_one, item, v0, min(n, v0 + chunk)))
        for f in futs:
            f.result()

    with ThreadPoolExecutor(max_workers=threads) as pool:
        one_pass(pool)
        t = time.perf_counter()
        reps = 0
        while time.perf_counter() - t < seconds_budget:
            one_pass(pool)
            reps += 1
        el = time.perf_counter() - t
    return {"value": round(bytes_one * reps / el / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": kind,
            "sample": f"u32 2048 vectors x w0..32 + u64 1024 vectors x w0..64, {reps} passes in "
                      f"{el:.1f} s, fls::unffor per vector (src/fls/unffor.cpp:22901/:23005)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["ffor", "ffor-sum", "alp", "batch", "learned",
                                           "autotune"], default="ffor")
    ap.add_argument("--tune", action="store_true",
                    help="run the decode autotuner (flsgpu_b200.autotune) before measuring")
    ap.add_argument("--epochs", type=int, default=12, help="learned workload: training epochs")
    ap.add_argument("--columns", type=int, default=2000, help="batch workload: column count")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the benchmark column sizes (1.0 = full)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--variant", type=int, default=0,
                    help="decode kernel variant for the 64-bit-lane columns (0 = tuned default, "
                         "1 register-rich, 2 register-capped, 3 staged)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="ffor workload: only the headline FFOR decode (no fused-sum, ALP, "
                         "batch and learned blocks)")
    ap.add_argument("--only", default="",
                    help="ffor workload: columns to build, e.g. u32:6,u64:20 (profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    config = {"workload": "FFOR bit-unpack at scale: u32 2^28 values x w=0..32 + u64 2^27 "
                          "values x w=0..64, decode to HBM",
              "columns": 98, "values_u32_per_column": int(2 ** 28 * args.scale),
              "values_u64_per_column": int(2 ** 27 * args.scale),
              "l2": "every column's 1 GiB output exceeds L2; no flush",
              "parallelism": f"replicas x{args.gpus}"}
    metric = "FFOR decode GB/s (compressed read + decoded write), 1 B200"
    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload not in ("ffor", "ffor-sum"):
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference arm runs the FFOR workload; the alp and learned "
                              "workloads carry the reference's CPU ALP decoder / rowgroup "
                              "encoder in their cpu_baseline, and the reference has no batched "
                              "decode, pair query or autotuner to run"}))
            return
        res = cpu_reference_ffor(args.cpu_seconds)
        steps_ms = []
        line = {"impl": "reference", "metric": metric, "value": res["value"], "unit": "GB/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u32/u64", "data": "synthetic", "config": config,
                "cpu_baseline": res,
                "e2e": {"value": res["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    rank, world, local = dist_init()
    dev = torch.device("cuda", torch.cuda.current_device())
    if args.variant:
        import flsgpu_b200 as F
        F.tuning_set({"variant": {(t, k): args.variant for t in ("u64", "f64")
                                  for k in (("bp", "ffor") if t == "u64" else ("alp", "alpx"))}})
    if args.tune or args.workload == "autotune":
        import flsgpu_b200 as F
        t0 = time.perf_counter()
        tuned = F.autotune()
        tune_s = time.perf_counter() - t0
        if args.workload == "autotune":
            if rank == 0:
                tab = tuned["table"]
                print(json.dumps({
                    "metric": "decode autotuner: per-width L2 prefetch and kernel variant",
                    "value": round(tune_s, 2), "unit": "s", "n_gpus": world,
                    "higher_is_better": False, "data": "synthetic",
                    "table": {"variant": {f"{k[0]}/{k[1]}": v for k, v in tab["variant"].items()},
                              "prefetch": {str(k): v for k, v in tab["prefetch"].items()}},
                    "report": tuned["report"],
                    "header": F.tuning_header(tab)}))
            return
    if args.workload == "learned":
        if rank == 0:
            print(json.dumps(learned_block(args, dev, world)))
        return
    if args.workload == "alp":
        b = alp_block(args, rank, world, dev)
        if rank == 0:
            print(json.dumps(b))
        return
    if args.workload == "batch":
        b = batch_block(args, dev, world)
        if rank == 0:
            print(json.dumps(b))
        return
    res = run_ffor(args, rank, world, dev)
    torch.cuda.empty_cache()
    e2e = None if args.no_e2e else run_e2e(args, dev)
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    extras = {}
    if args.extras and args.workload == "ffor":
        # the rest of the benchmark metric, each block with its own clocks:
        # fused sum (same columns), ALP / ALP-RD decode, batched decode + pair
        # query, learned vs plain ALP encode
        extras["ffor_sum"] = res["fsum"]
        torch.cuda.empty_cache()
        extras["alp_decode"] = alp_block(args, rank, world, dev)
        torch.cuda.empty_cache()
        extras["batch_decode"] = batch_block(args, dev, world)
        torch.cuda.empty_cache()
        extras["learned_encode"] = learned_block(args, dev, world)
    if rank == 0:
        cpu = None
        if world == 1:
            cpu = cpu_reference_ffor(args.cpu_seconds)
            one = cpu_reference_ffor(args.cpu_seconds / 2, threads=1)
            cpu["nproc"] = os.cpu_count()
            cpu["single_thread"] = {"value": one["value"], "unit": "GB/s", "cores": 1,
                                    "sample": one["sample"]}
        name = "FFOR decode GB/s (compressed read + decoded write), 1 B200"
        if args.workload == "ffor-sum":
            name = "FFOR decode fused with a sum GB/s (compressed read + 8 B per column), 1 B200"
        line = {
            "metric": name, "value": round(res["gbs"], 1), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(res["ms"] / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64", "data": "synthetic",
            "config": config,
            "hbm_fraction": {f"of_{pk_kind}": round(res["gbs"] / world / hbm, 4),
                             "of_spec_8tbs": round(res["gbs"] / world / 8000.0, 4)},
            "uncompressed_gbs": round(res["uncompressed_gbs"], 1),
            "per_width_gbs": res["per_width"],
            "roofline": {"bound": "hbm", "achieved": round(res["achieved"], 1),
                         "peak": hbm, "unit": "GB/s", "frac": round(res["achieved"] / hbm, 4),
                         "peak_kind": pk_kind,
                         "kernel": "k_store<T> (flsgpu_decompress_ffor_u32/u64)",
                         "algorithmic_bytes_per_launch": round(res["bytes_step"] / res["n_columns"]),
                         "traffic": profiled_traffic("k_store_ffor_at_scale.md",
                                                     res["bytes_step"] / res["n_columns"]),
                         "traffic_source": "profiles/k_store_ffor_at_scale.md (ncu, one pass)"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": res["launches"],
            "clocks": res["clocks"],
        }
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def alp_block(args, rank, world, dev) -> dict:
    """The ALP / ALP-RD decode configuration: per column GB/s, fraction of
    the HBM peak and a bit-exact flag, the f64 column again in the extended
    layout, the reference's CPU decoder beside it."""
    r = run_alp(args, rank, world, dev)
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    return {
        "metric": "ALP / ALP-RD decode GB/s (compressed read + decoded write), 1 B200",
        "value": round(r["gbs"], 1), "unit": "GB/s", "n_gpus": world, "steps": r["steps"],
        "warmup": args.warmup, "ms_per_step": round(r["ms"] / r["steps"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64/f32", "data": "synthetic",
        "config": {"workload": "ALP/ALP-RD decode: f64 ALP 2^27 values (d 0..4, 1% "
                               "exceptions), f64 ALP-RD 2^27 uniform [0,1), f32 ALP 2^28 "
                               "values (d 0..3, 1% exceptions)",
                   "scale": args.scale,
                   "l2": "every column's output (1 GiB) exceeds L2; no flush",
                   "parallelism": f"replicas x{world}"},
        "per_column": r["per"], "bit_exact": r["exact"],
        "hbm_fraction": {f"of_{pk_kind}": round(r["gbs"] / world / hbm, 4),
                         "of_spec_8tbs": round(r["gbs"] / world / 8000.0, 4)},
        "roofline": {"bound": "hbm", "achieved": round(r["achieved"], 1), "peak": hbm,
                     "unit": "GB/s", "frac": round(r["achieved"] / hbm, 4),
                     "peak_kind": pk_kind,
                     "kernel": "k_store<f64/f32, ALP> and k_alprd<f64>",
                     "algorithmic_bytes_per_launch": round(r["bytes_step"] / 3),
                     "traffic": profiled_traffic("alp_decode_at_scale.md", r["bytes_step"] / 3),
                     "traffic_source": "profiles/alp_decode_at_scale.md (ncu, one pass)"},
        "cpu_baseline": r["cpu"],
        "gpu_launches": r["launches"], "clocks": r["clocks"],
        "generation_s": round(r["gen_s"], 1)}


def batch_block(args, dev, world) -> dict:
    """Batched uneven decode (graph replay) against one launch per column,
    plus the fused pair query."""
    r = run_batch(args, dev)
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    gbs = (r["read"] + r["write"]) / (r["ms"] / 1e3) / 1e9
    return {
        "metric": "batched uneven decode GB/s (compressed read + decoded write), 1 B200",
        "value": round(gbs, 1), "unit": "GB/s", "n_gpus": world, "steps": r["steps"],
        "warmup": args.warmup, "ms_per_step": round(r["ms"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32/f64", "data": "synthetic",
        "config": {"workload": f"batched uneven decode: {r['n_columns']} columns, lengths "
                               "log-uniform 2^10..2^24 (x1024), types f64 ALP / u32 FFOR / "
                               "f32 ALP, persistent launches replayed from a CUDA graph",
                   "values": r["n_values"], "compressed_bytes": r["read"],
                   "decoded_bytes": r["write"],
                   "l2": "total decoded bytes exceed L2; no flush"},
        "hbm_fraction": {f"of_{pk_kind}": round(gbs / hbm, 4), "of_spec_8tbs": round(gbs / 8000, 4)},
        "bit_exact_vs_per_column": r["exact_vs_per_column"],
        "per_column_launches_ms": round(r["ms_each"], 3),
        "per_column_launches_sync_ms": round(r["ms_each_sync"], 3),
        "eager_batch_launch_ms": round(r["ms_launch"], 3),
        "speedup_vs_per_column": round(r["ms_each"] / r["ms"], 2),
        "speedup_vs_per_column_sync": round(r["ms_each_sync"] / r["ms"], 2),
        "pair_query": {"pairs": r["n_pairs"], "ms": round(r["ms_query"], 3),
                       "compressed_gbs": round(r["q_read"] / (r["ms_query"] / 1e3) / 1e9, 1),
                       "what": "sum(A where B < median(B)) per (f64 ALP, u32 FFOR) pair, "
                               "4 radix passes over packed B + 1 fused decode/sum pass",
                       "clocks": r["q_clocks"]},
        "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(gbs / hbm, 4), "peak_kind": pk_kind,
                     "kernel": "k_batch (flsgpu_batch_replay)",
                     "traffic": profiled_traffic("batch_decode_launches.md", r["read"] + r["write"]),
                     "traffic_source": "profiles/batch_decode_launches.md"},
        "gpu_launches_per_replay": r["launches"], "clocks": r["clocks"],
        "generation_s": round(r["gen_s"], 1)}


def learned_block(args, dev, world) -> dict:
    """Learned ALP parameter proposal against the plain per-vector search:
    end-to-end GPU encode GB/s, compression ratio, fallbacks, selection and
    end-to-end speed-ups, bit-exact decode."""
    r = run_learned(args, dev)
    gbs_l = r["in_bytes"] / (r["ms_learned"] / 1e3) / 1e9
    gbs_p = r["in_bytes"] / (r["ms_plain"] / 1e3) / 1e9
    return {
        "metric": "ALP encode GB/s (input bytes / end-to-end GPU encode), learned vs plain",
        "value": round(gbs_l, 1), "unit": "GB/s", "n_gpus": world,
        "ms_per_step": round(r["ms_learned"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "learned ALP parameter proposal: f64 column of "
                               f"{r['n_vecs'] * 1024} values (d in 0..6, scale 10^0..8, "
                               "Gaussian/uniform, 10% noise vectors); network trained "
                               "on a separate 2^24-value column"},
        "column": "hybrid: ALP vectors + ALP-RD vectors (flsgpu_alp_encode_hybrid_f64)",
        "learned": {"encode_gbs": round(gbs_l, 1), "ms": round(r["ms_learned"], 3),
                    "ratio": round(r["in_bytes"] / r["learned_bytes"], 4),
                    "fallback_vectors": r["fallback"], "rd_vectors": r["n_rd"],
                    "proposal_ms": round(r["ms_propose"], 3),
                    "decode_bit_exact": r["exact"],
                    "decode_gbs": round((r["learned_bytes"] + r["in_bytes"]) / (r["ms_hdec"] / 1e3)
                                        / 1e9, 1),
                    "decode_kernel": "k_hybrid<double> (flsgpu_decompress_alphybrid_f64)"},
        "plain": {"encode_gbs": round(gbs_p, 1), "ms": round(r["ms_plain"], 3),
                  "ratio": round(r["in_bytes"] / r["plain_bytes"], 4),
                  "rd_vectors": r["plain_rd"], "search_ms": round(r["ms_search"], 3)},
        "alp_only_columns": r["alp_only"],
        "speedup_encode_vs_plain": round(r["ms_plain"] / r["ms_learned"], 2),
        "speedup_selection_vs_plain_search": round(r["ms_search"] / r["ms_propose"], 2),
        "ratio_loss_vs_plain": round(1 - r["plain_bytes"] / r["learned_bytes"], 4),
        "training": {"epochs": args.epochs, "seconds": round(r["train_s"], 2),
                     "loss_first_epoch": round(r["loss"][0], 4),
                     "loss_last_epoch": round(r["loss"][1], 4)},
        "clocks": r["clocks"],
        "cpu_baseline": {"value": round(r["ref_gbs"], 3) if r["ref_gbs"] else None,
                         "unit": "GB/s", "cores": 1, "kind": "port",
                         "ratio": round(r["ref_ratio"], 4) if r["ref_ratio"] else None,
                         "sample": "the whole evaluation column, oracle restatement of "
                                   "alp::encode with rowgroup sampling (100 vectors per "
                                   "state, ALP-RD rowgroups kept on ALP)"}}


if __name__ == "__main__":
    main()
