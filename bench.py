"""Channelizer benchmark: MSamples/s of the batched B200 filterbank.

Workload (one "step"): 256 independent cf32 streams, lengths log-uniform in
[2^14, 2^22] samples, nchan from {64, 256, 1024, 4096}, taps/branch from
{8, 12, 16}, 2x oversampled, each stream's next block (3 successive blocks
cycle; filter history carried across steps on the device). Synthetic,
seeded noise + 1-5 tones per stream, generated on the device. Inputs per
step are ~1.5 GB, far larger than L2, so no flush is needed between steps.

Arms printed in ONE JSON line (rank 0):
  value       batched path: one persistent-kernel launch per step for all 256
              streams, replayed from a CUDA graph, inputs resident in HBM
  plain       the same streams, one device-pointer call (launch) per stream
  e2e         the reference-facing C ABI end to end: atkdsp_pfb_process per
              stream with pinned host buffers, from several host threads
              (different handles may run concurrently, as in the reference);
              each call's host->device and device->host copies are inside the
              timed region
  e2e_batch   our batch API with pinned host<->device copies on its stream
  dropin      the same C ABI calls with pageable host buffers
  roofline    dominant kernel (the tile kernel): algorithmic bytes (8 B in +
              8*oversample B out per input sample) / its CUDA-event duration
  cpu_baseline the reference's own C library (built from its sources) on this
              host's cores over a bounded sample of the same workload
  configs     the other configurations, each with its own rate: single
              stream (C ABI, uneven blocks), the unpack front end, the
              coherent array, the overlap-save extractor (64 channels from
              one 61.44 MS/s stream), Undertow's six-scale filterbank bank
              (one launch per chunk), the spectrum reduction, the CFAR
              detector and tracker (W3's gate, Mcells/s), the serving loop

--impl reference runs only the reference's CPU channelizer (all host threads)
on the same workload and prints its line.
Multi-GPU (torchrun): each rank runs its own 256-stream set (weak scaling,
no collective on the data path); timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FS = 2.4e6
WORKLOAD = "uneven_streams_256"
METRIC = "channelized MSamples/s (batched+served vs plain) and p99 block latency, 1 B200"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _specs(rank: int, args=None):
    from atkdsp_b200 import workloads as W
    if args is None:
        return W.uneven_streams(256, seed=4 + 1000 * rank)
    return W.uneven_streams(args.streams, seed=4 + 1000 * rank, min_log2=args.min_log2,
                            max_log2=args.max_log2)


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling (20 ms period) around the timed region; mark() the
    region's start and end, summary() keeps the samples taken inside it (or,
    when the region is shorter than a few periods, the nearest ones)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __enter__(self):
        q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for t, ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 9:
                rows.append((t, f))
        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if self.t0 <= r[0] <= self.t1 + 0.02]
            if len(inside) < 3:           # a short region: the samples nearest to it
                mid = 0.5 * (self.t0 + self.t1)
                inside = sorted(rows, key=lambda r: abs(r[0] - mid))[:3]
            rows = inside
        for t, f in rows:
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "period_ms": 20}


# ------------------------------------------------------------ device inputs
def _device_blocks(specs, torch, device, nblocks=3, seed=0):
    """All streams' blocks as slices of one device tensor per block set."""
    g = torch.Generator(device=device)
    sets = []
    for b in range(nblocks):
        total = sum(s.length for s in specs)
        buf = torch.empty(total, dtype=torch.complex64, device=device)
        views, pos = [], 0
        for i, s in enumerate(specs):
            g.manual_seed(seed * 1_000_003 + i * 7919 + b)
            x = buf[pos:pos + s.length]
            x.copy_(torch.randn(s.length, dtype=torch.complex64, device=device, generator=g))
            rng = np.random.default_rng(s.seed)
            nt = int(rng.integers(1, 6))
            t = torch.arange(b * s.length, (b + 1) * s.length, device=device, dtype=torch.float64)
            for f, ph in zip(rng.uniform(-0.5, 0.5, nt), rng.uniform(0, 2 * math.pi, nt)):
                x += (10.0 * torch.exp(1j * (2 * math.pi * f * t + ph))).to(torch.complex64)
            views.append(x)
            pos += s.length
        sets.append((buf, views))
    return sets


def _out_buffers(specs, torch, device):
    caps = [s.nchan * (s.length // (s.nchan // s.oversample) + 1) for s in specs]
    buf = torch.empty(sum(caps), dtype=torch.complex64, device=device)
    views, pos = [], 0
    for c in caps:
        views.append(buf[pos:pos + c])
        pos += c
    return buf, views


def _alg_bytes(specs, ms):
    return sum(8 * s.length + 8 * s.nchan * m for s, m in zip(specs, ms))


# ------------------------------------------------------------ CPU baseline
def _cpu_reference_rate(specs, budget_s: float = 8.0, threads: int | None = None):
    """The reference library (oracle/_ref) over a bounded sample of the
    workload: streams in order, one block each, until ~budget_s of wall time.
    Returns (MS/s, threads, sample description) or None when not built."""
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        return None
    nth = threads or os.cpu_count() or 1
    ref.lib.atkdsp_set_threads(nth)
    from atkdsp_b200 import workloads as W
    done, t_used, used = 0, 0.0, 0
    for s in specs:
        x = W.stream_samples(s, 0)
        p = ref.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1)
        t0 = time.perf_counter()
        p.process(x)
        t_used += time.perf_counter() - t0
        done += x.size
        used += 1
        if t_used > budget_s:
            break
    return done / t_used / 1e6, nth, f"first {used} of {len(specs)} streams, one block each ({done} samples)"


def run_reference(args, rank, world):
    """The reference's own CPU channelizer (oracle/_ref, built from its
    sources) on this arm's workload: every one of the 256 streams, one block
    each per step through atkdsp_pfb_process_n with its own handle (state
    carried from step to step), all host threads. Rank 0 only."""
    if rank != 0:
        return
    specs = _specs(0, args)
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/_ref)"}))
        return
    from atkdsp_b200 import workloads as W
    nth = os.cpu_count() or 1
    ref.lib.atkdsp_set_threads(nth)
    xs = [W.stream_samples(s, 0) for s in specs]
    tot = sum(x.size for x in xs)
    handles = [ref.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in specs]
    outs = [np.zeros(s.nchan * (s.length // (s.nchan // s.oversample) + 2), np.complex64) for s in specs]
    fn = handles[0]._o._f("pfb_process_n")
    arrs = [(O._pcf * 1)(O._cfp(x)) for x in xs]

    def step():
        for p, a, x, o in zip(handles, arrs, xs, outs):
            if fn(p._p, a, 1, x.size, O._cfp(o), o.size) < 0:
                raise RuntimeError("reference atkdsp_pfb_process_n failed")

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    v = tot * args.steps / dt / 1e6
    desc = f"all {len(specs)} streams, one block each per step ({tot} samples per step)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "MSamples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fold + f64 fft (CPU)",
        "data": "synthetic", "config": _config(args, world),
        "cpu_baseline": {"value": round(v, 3), "unit": "MSamples/s", "cores": nth,
                         "kind": "reference", "sample": desc},
        "e2e": {"value": round(v, 3), "unit": "MSamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "native_so": _native_maps(),
    }))


def _config(args, world):
    """The workload description both arms print."""
    name = WORKLOAD if args.streams == 256 and args.min_log2 == 14 and args.max_log2 == 22 else \
        f"uneven_streams_{args.streams}_2^{args.min_log2:g}-2^{args.max_log2:g}"
    return {"workload": name, "streams": args.streams, "nchan": [64, 256, 1024, 4096],
            "taps_per_branch": [8, 12, 16], "oversample": 2, "blocks": 3,
            "parallelism": f"replicas x{world} (stream-sharded)",
            "l2": "inputs larger than L2 (~1.5 GB per step)"}


# ------------------------------------------- accuracy checks (outside timing)
def _rel_err(y, r):
    """Worst channel's RMS error and largest single error, each divided by
    that channel's RMS (the parity bar's metric)."""
    y = np.asarray(y).reshape(-1, np.asarray(y).shape[-1]).astype(np.complex128)
    r = np.asarray(r).reshape(-1, np.asarray(r).shape[-1]).astype(np.complex128)
    rms = np.sqrt(np.mean(np.abs(r) ** 2, axis=1))
    rms = np.where(rms > 0, rms, 1.0)
    e = np.abs(y - r)
    return float(np.max(np.sqrt(np.mean(e ** 2, axis=1)) / rms)), float(np.max(np.max(e, axis=1) / rms))


def _accuracy(cases, what: str) -> dict:
    """cases: (ours, reference, float64 or None) output triples of the same
    inputs, (..., nchan, m) each (the float64 one may cover fewer hops).
    Returns the worst channel over all cases."""
    vr = vm = v64 = r64 = 0.0
    have64 = False
    for y, r, y64 in cases:
        a, b = _rel_err(y, r)
        vr, vm = max(vr, a), max(vm, b)
        if y64 is not None:
            m = y64.shape[-1]
            have64 = True
            v64 = max(v64, _rel_err(np.asarray(y)[..., :m], y64)[0])
            r64 = max(r64, _rel_err(np.asarray(r)[..., :m], y64)[0])
    out = {"vs_reference_rms": float(f"{vr:.3g}"), "vs_reference_max": float(f"{vm:.3g}"), "checked": what,
           "bar": 1e-5}
    if have64:
        out["vs_fp64_rms"] = float(f"{v64:.3g}")
        out["reference_vs_fp64_rms"] = float(f"{r64:.3g}")
    return out


def _fp64(nchan, os_, taps, atten, xs):
    """The float64 restatement of the filterbank over element arrays xs."""
    from oracle import fp64
    from oracle import oracle as O
    t = fp64.Fp64Pfb(O.oracle().prototype(nchan, taps, atten), nchan, os_, len(xs))
    return t.process_n(xs, len(xs))


def _batched_accuracy(specs, torch, device) -> dict | None:
    """One stream of each (nchan, taps) pair of the workload, through a fresh
    batch of the same kernel and through the reference library, same input
    (the stream's first block, at most 2^18 samples); float64 on 2^15."""
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        return None
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    pick = {}
    for s in specs:
        pick.setdefault((s.nchan, s.taps), s)
    chosen = [pick[k] for k in sorted(pick)]
    xs = [W.stream_samples(s, 0)[: 1 << 18] for s in chosen]
    hs = [ak.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in chosen]
    b = gpu.Batch(hs, use_graph=False)
    din = [torch.from_numpy(x).to(device) for x in xs]
    dout = [torch.empty(max(1, s.nchan * h.out_hops(x.size)), dtype=torch.complex64, device=device)
            for s, h, x in zip(chosen, hs, xs)]
    ms = b.process(din, dout)
    torch.cuda.synchronize()
    cases = []
    for s, x, o, m in zip(chosen, xs, dout, ms):
        y = o[: s.nchan * m].view(s.nchan, m).cpu().numpy()
        r = np.asarray(ref.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1).process(x))
        y64 = _fp64(s.nchan, s.oversample, s.taps, 80.0, [x[: 1 << 15]])[0]
        cases.append((y, r, y64))
    del b, hs
    return _accuracy(cases, f"{len(chosen)} streams, one per (nchan, taps) pair, first block "
                            f"(<= 2^18 samples; float64 on 2^15)")


# -------------------------------------------------------------- our arms
def _timed(stream, torch, fn, steps):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(steps):
        fn(k)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3


def _plain_arm(args, specs, sets, outs, torch, device, barrier, max_over_ranks):
    """One device-pointer call (one launch) per stream, all on one stream."""
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    handles = [ak.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in specs]
    st = torch.cuda.Stream(device=device)

    def step(k):
        for p, x, o in zip(handles, sets[k % 3][1], outs):
            gpu.process_n(p, [x], 1, out=o, stream=st)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    barrier()
    t = max_over_ranks(_timed(st, torch, step, args.steps))
    barrier()
    # where one call per stream loses: one more pass with each call bracketed
    # by events on its stream, grouped by the stream's length (log2 bucket)
    evs = []
    for p, x, o in zip(handles, sets[0][1], outs):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        gpu.process_n(p, [x], 1, out=o, stream=st)
        e1.record(st)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    buckets: dict = {}
    for sp, (e0, e1) in zip(specs, evs):
        b = buckets.setdefault(int(math.log2(sp.length)), [0, 0, 0.0])
        b[0] += 1
        b[1] += sp.length
        b[2] += e0.elapsed_time(e1)
    by_len = [{"log2_length": k, "streams": v[0], "samples": v[1], "ms": round(v[2], 4),
               "msps": round(v[1] / v[2] / 1e3, 1), "us_per_call": round(v[2] / v[0] * 1e3, 1)}
              for k, v in sorted(buckets.items())]
    del handles
    return t, by_len


def _e2e_batch_arm(args, S, sets, obuf, bstream, bstep, torch, barrier, max_over_ranks):
    """Our batch API end to end: pinned host inputs -> device, the batched
    step, outputs -> pinned host, all on the batch's stream."""
    h_in = torch.empty(S, dtype=torch.complex64, pin_memory=True)
    h_in.copy_(sets[0][0].cpu())
    h_out = torch.empty(obuf.numel(), dtype=torch.complex64, pin_memory=True)
    d_in = sets[0][0]

    def step(k):
        with torch.cuda.stream(bstream):
            d_in.copy_(h_in, non_blocking=True)
        bstep(0)
        with torch.cuda.stream(bstream):
            h_out.copy_(obuf, non_blocking=True)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    barrier()
    t = max_over_ranks(_timed(bstream, torch, step, args.steps))
    barrier()
    return t


CABI_THREADS = max(1, min(8, os.cpu_count() or 1))      # --cabi-threads overrides


def _cabi_arm(specs, sets, torch, barrier, max_over_ranks, pinned: bool, steps: int, warmup: int):
    """The reference-facing C ABI with host buffers: atkdsp_pfb_process, one
    handle per stream, called from CABI_THREADS host threads over disjoint
    sets of streams (the reference allows concurrent calls on different
    handles; each handle has its own CUDA stream, so one thread's copies and
    kernels overlap another's). Every call copies its input host->device and
    its output device->host inside the timed region. Returns (seconds for
    `steps` steps, h2d bytes per step, d2h bytes per step)."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    import atkdsp_b200 as ak
    lib = ak.load()
    proc = C.CFUNCTYPE(C.c_ssize_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t)(
        C.cast(lib.atkdsp_pfb_process, C.c_void_p).value)
    handles = [ak.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in specs]
    keep, ins, outs = [], [], []
    for s, v in zip(specs, sets[0][1]):
        hop = s.nchan // s.oversample
        cap = s.nchan * ((hop - 1 + s.length) // hop)
        if pinned:
            x = torch.empty(s.length, dtype=torch.complex64, pin_memory=True)
            x.copy_(v)
            o = torch.empty(max(cap, 1), dtype=torch.complex64, pin_memory=True)
            ins.append(x.data_ptr())
            outs.append((o.data_ptr(), cap))
        else:
            x = v.cpu().numpy().copy()
            o = np.zeros(max(cap, 1), np.complex64)
            ins.append(x.ctypes.data)
            outs.append((o.ctypes.data, cap))
        keep += [x, o]
    order = sorted(range(len(specs)), key=lambda i: -specs[i].length)
    parts = [order[t::CABI_THREADS] for t in range(CABI_THREADS)]
    moved = [0]

    def work(idx):
        d2h = 0
        for i in idx:
            m = proc(handles[i]._p, ins[i], specs[i].length, outs[i][0], outs[i][1])
            if m < 0:
                raise RuntimeError(f"atkdsp_pfb_process returned {m}")
            d2h += 8 * specs[i].nchan * m
        return d2h

    with ThreadPoolExecutor(CABI_THREADS) as ex:
        for _ in range(warmup):
            list(ex.map(work, parts))
        barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            moved[0] = sum(ex.map(work, parts))
        t = max_over_ranks(time.perf_counter() - t0)
    del handles, keep
    return t, 8 * sum(s.length for s in specs), moved[0]


# --------------------------------------------------- the other configurations
def _c1_arm(torch, cpu: bool):
    """Single stream, M=64 critically sampled, 16 taps/branch, beta 8, 2^20 cf32
    samples fed in blocks 1, 999, 4096, 7 (cycling) through the drop-in C ABI
    with host buffers -- each call is synchronous, so this measures per-call
    latency as much as the kernel. The CPU baseline is the reference library
    on one thread over the same calls (its OpenMP start-up makes more threads
    slower on blocks this small)."""
    import atkdsp_b200 as ak
    from atkdsp_b200 import workloads as W
    x = W.single_stream(1 << 20)
    blocks = W.SINGLE_STREAM_BLOCKS
    p = ak.Pfb(FS, 64, 1, 16, W.ATTEN_BETA8, 1)
    p.process(x[:5000])
    p.reset()
    outs = []
    t0 = time.perf_counter()
    pos, i, calls = 0, 0, 0
    while pos < x.size:
        b = blocks[i % len(blocks)]
        outs.append(p.process(x[pos:pos + b]))
        pos += b
        i += 1
        calls += 1
    dt = time.perf_counter() - t0
    res = {"workload": "single_stream_m64_blocks_1_999_4096_7", "value": round(x.size / dt / 1e6, 2),
           "unit": "MSamples/s", "calls": calls, "us_per_call": round(dt / calls * 1e6, 2),
           "path": "atkdsp_pfb_process (host buffers)"}
    if cpu:
        from oracle import oracle as O
        ref = O.reference()
        if ref is not None:
            ref.lib.atkdsp_set_threads(1)
            rp = ref.Pfb(FS, 64, 1, 16, W.ATTEN_BETA8, 1)
            routs = []
            t0 = time.perf_counter()
            pos, i = 0, 0
            while pos < x.size:
                b = blocks[i % len(blocks)]
                routs.append(rp.process(x[pos:pos + b]))
                pos += b
                i += 1
            rdt = time.perf_counter() - t0
            ref.lib.atkdsp_set_threads(os.cpu_count() or 1)
            res["cpu_baseline"] = {"value": round(x.size / rdt / 1e6, 2), "unit": "MSamples/s", "cores": 1,
                                   "kind": "reference", "sample": "the whole workload, same calls"}
            y = np.concatenate([o for o in outs if o.shape[1]], axis=1)
            r = np.concatenate([o for o in routs if np.asarray(o).shape[1]], axis=1)
            y64 = _fp64(64, 1, 16, W.ATTEN_BETA8, [x])[0]
            res["accuracy"] = _accuracy([(y, r, y64)], "the whole stream")
    return res


class _FrontEnd:
    """The front end's per-block calls as the bench issues them. The running
    DC estimate stays on the device: block b's offset is block b-1's mean,
    rounded to float by the kernels (atkdsp_gpu_block_mean_dev and
    atkdsp_gpu_pfb_process_w12_dev). The means run one block ahead on a second
    stream (a block's mean needs only its own samples and the previous mean),
    so they fill the SMs the filterbank's last tiles leave idle. Three mean
    buffers in turn; events order each buffer's writer after the calls that
    read it. Call mean_of(0), then mean_of(b + 1) and filt(b) for b = 0, 1, ..."""

    def __init__(self, torch, device, p, block, **w12):
        import atkdsp_b200 as ak
        from atkdsp_b200 import gpu
        self.gpu, self.p, self.block, self.w12 = gpu, p, block, w12
        self.means = [torch.zeros(2, dtype=torch.float64, device=device) for _ in range(3)]
        self.st = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p.handle), device=device)
        self.sm = torch.cuda.Stream(device=device)
        self.ev_mean = [torch.cuda.Event() for _ in range(3)]   # block b's mean is written
        self.ev_read = [torch.cuda.Event() for _ in range(3)]   # block b's filterbank call is done

    def mean_of(self, b):
        if b >= 2:
            self.sm.wait_event(self.ev_read[(b - 2) % 3])       # the last reader of means[b % 3]
        self.gpu.block_mean(self.block(b), "ci16q11", self.means[(b - 1) % 3], mean=self.means[b % 3],
                            stream=self.sm)
        self.ev_mean[b % 3].record(self.sm)

    def filt(self, b):
        if b >= 1:
            self.st.wait_event(self.ev_mean[(b - 1) % 3])
        y = self.gpu.process_w12(self.p, self.block(b), "ci16q11", self.means[(b - 1) % 3], stream=self.st,
                                 **self.w12)
        self.ev_read[b % 3].record(self.st)
        return y


def _c2_arm(torch, device, steps, cpu: bool):
    """40 MS/s front end: ci16q11 with noise + 8 tones + a constant DC offset,
    2,000,000-sample (50 ms) blocks; per block the running DC estimate (the
    previous block's mean) is the offset, the filterbank (M=1024, 2x, 12 taps)
    reads the raw int16 and converts in its load path, W1 and W2 accumulate in
    one pass. Inputs resident on the device."""
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    blk = 2_000_000
    nblk = (1 << 26) // blk
    g = torch.Generator(device=device)
    g.manual_seed(2)
    n = nblk * blk
    t = torch.arange(n, device=device, dtype=torch.float64)
    sig = torch.randn(n, dtype=torch.complex128, device=device, generator=g) * 64.0
    rng = np.random.default_rng(2)
    for f, ph in zip(rng.uniform(-0.5, 0.5, 8), rng.uniform(0, 2 * math.pi, 8)):
        sig += 202.0 * torch.exp(1j * (2 * math.pi * f * t + ph))
    sig += complex(*W.FRONT_END_DC_LSB)
    raw = torch.stack([sig.real.round(), sig.imag.round()], dim=1).clamp(-2048, 2047).to(torch.int16)
    del sig, t
    p = ak.Pfb(FS, 1024, 2, 12, 80.0, 1)
    m_max = blk // 512 + 1
    out = torch.empty(1024 * m_max, dtype=torch.complex64, device=device)
    R = torch.zeros((1024, 1, 1), dtype=torch.complex64, device=device)
    cnt = torch.zeros(1024, dtype=torch.int32, device=device)
    pwr = torch.zeros((1, 1024), dtype=torch.float32, device=device)
    mp = torch.zeros(1024, dtype=torch.float32, device=device)
    scratch = torch.empty(max(8, ak.load().atkdsp_gpu_pfb_w12_scratch_bytes(p.handle, blk)), dtype=torch.uint8,
                          device=device)
    fe = _FrontEnd(torch, device, p, lambda b: raw[(b % nblk) * blk:(b % nblk + 1) * blk].reshape(-1),
                   out=out, R=R, counts=cnt, pwr=pwr, mean_pwr=mp, scratch=scratch)
    mean_of, filt, st = fe.mean_of, fe.filt, fe.st

    nb = max(steps, 1) * nblk
    mean_of(0)
    for b in range(3):                                   # warm-up blocks
        mean_of(b + 1)
        filt(b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    for b in range(3, 3 + nb):
        mean_of(b + 1)
        filt(b)
    ev1.record(st)
    torch.cuda.synchronize()
    dt = ev0.elapsed_time(ev1) / 1e3
    res = {"workload": "front_end_ci16q11_m1024_os2_k12_blocks_2e6", "value": round(nb * blk / dt / 1e6, 2),
           "unit": "MSamples/s", "x_real_time_at_40msps": round(nb * blk / dt / 40e6, 1),
           "bytes_per_sample": 4 + 4 + 16,
           "path": "block_mean + unpack, filterbank and W1/W2 in one pass (W2 power summed in the "
                   "filterbank's epilogue), per 50 ms block; the DC estimate (the previous block's "
                   "mean) read by the kernels from device memory, no host round trip; block means one "
                   "block ahead on a second stream"}
    if cpu:
        res.update(_c2_check(raw[: 3 * blk].cpu().numpy(), blk, torch, device))
    return res


def _c2_check(raw, blk, torch, device) -> dict:
    """The front end's first three blocks through a fresh handle and through
    the reference library (unpack_dc with the previous block's mean as the
    offset, then the filterbank, then W1 and W2), the same offsets fed to
    both: output and W2 power accuracy, and the reference's rate on all host
    threads for the same work."""
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        return {}
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    nth = os.cpu_count() or 1
    ref.lib.atkdsp_set_threads(nth)
    rp = ref.Pfb(FS, 1024, 2, 12, 80.0, 1)
    R = np.zeros((1024, 1, 1), np.complex64)
    cnt = np.zeros(1024, np.uint32)
    blocks = [raw[b * blk:(b + 1) * blk] for b in range(3)]
    offs, refs, pw_ref = [0j], [], []
    t0 = time.perf_counter()
    for b in range(3):
        x, mean = ref.unpack_dc(blocks[b].tobytes(), "ci16q11", offs[-1])
        y = rp.process_n([x], 1)
        ref.pfb_cov_accumulate(y, 1, 1024, None, R, cnt)
        pw_ref.append(ref.pfb_channel_power(y, 1, 1024)[0])
        refs.append(y)
        offs.append(complex(np.float32(mean.real), np.float32(mean.imag)))
    rdt = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(1)                     # one block again, on one thread
    rp1 = ref.Pfb(FS, 1024, 2, 12, 80.0, 1)
    R1, c1 = np.zeros((1024, 1, 1), np.complex64), np.zeros(1024, np.uint32)
    t0 = time.perf_counter()
    x, _ = ref.unpack_dc(blocks[0].tobytes(), "ci16q11", 0j)
    y1 = rp1.process_n([x], 1)
    ref.pfb_cov_accumulate(y1, 1, 1024, None, R1, c1)
    ref.pfb_channel_power(y1, 1, 1024)
    rdt1 = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(nth)
    # the benchmarked calls, pipelined as the timed loop issues them
    p = ak.Pfb(FS, 1024, 2, 12, 80.0, 1)
    Rg = torch.zeros((1024, 1, 1), dtype=torch.complex64, device=device)
    cg = torch.zeros(1024, dtype=torch.int32, device=device)
    pw = torch.zeros((1, 1024), dtype=torch.float32, device=device)
    mpw = torch.zeros(1024, dtype=torch.float32, device=device)
    dev_blocks = [torch.from_numpy(b.reshape(-1).copy()).to(device) for b in blocks]
    fe = _FrontEnd(torch, device, p, lambda b: dev_blocks[b], R=Rg, counts=cg, pwr=pw, mean_pwr=mpw)
    torch.cuda.synchronize()
    cases, pw_err, off_same = [], 0.0, True
    fe.mean_of(0)
    for b in range(3):
        if b + 1 < 3:
            fe.mean_of(b + 1)
        y = fe.filt(b)
        torch.cuda.synchronize()
        cases.append((y.cpu().numpy(), refs[b], None))
        pv = pw.cpu().numpy().reshape(-1).astype(np.float64)
        pw_err = max(pw_err, float(np.max(np.abs(pv - pw_ref[b].reshape(-1)) / pw_ref[b].reshape(-1))))
        mh = fe.means[b % 3].cpu().numpy()
        off_same &= complex(np.float32(mh[0]), np.float32(mh[1])) == offs[b + 1]
    Rd = Rg.cpu().numpy().reshape(-1)
    acc = _accuracy(cases, "the first three 2,000,000-sample blocks through the benchmarked calls "
                           "(device-held DC estimate, fused W1/W2)")
    acc["w2_power_max_rel"] = float(f"{pw_err:.3g}")
    acc["w1_max_rel"] = float(f"{float(np.max(np.abs(Rd - R.reshape(-1)) / np.abs(R.reshape(-1)))):.3g}")
    # W1 against its exact sum (float64 over the three blocks' outputs): the
    # reference accumulates in float hop by hop, this build in double per block
    r64 = sum(np.sum(np.abs(c[0].astype(np.complex128).reshape(1024, -1)) ** 2, axis=1) for c in cases)
    acc["w1_vs_exact_max_rel"] = float(f"{float(np.max(np.abs(Rd.real - r64) / r64)):.3g}")
    acc["reference_w1_vs_exact_max_rel"] = float(f"{float(np.max(np.abs(R.reshape(-1).real - r64) / r64)):.3g}")
    acc["w1_counts_equal"] = bool(np.array_equal(cg.cpu().numpy().astype(np.uint32), cnt))
    acc["offsets_equal_reference"] = bool(off_same)
    return {"accuracy": acc,
            "cpu_baseline_1thread": {"value": round(blk / rdt1 / 1e6, 2), "unit": "MSamples/s", "cores": 1,
                                     "kind": "reference", "sample": "one 2,000,000-sample block: unpack_dc, "
                                                                    "filterbank, W1, W2"},
            "cpu_baseline": {"value": round(3 * blk / rdt / 1e6, 2), "unit": "MSamples/s", "cores": nth,
                             "kind": "reference", "sample": "three 2,000,000-sample blocks: unpack_dc, "
                                                            "filterbank, W1, W2"}}


def _c3_arm(torch, device, steps, cpu: bool):
    """Coherent array: 8 cf32 element streams, M=2048, 1x, 16 taps, 2^24 samples
    each, 4 common tones with per-element phases + noise at 10 dB; one
    process_n call per step, then W1 (8x8 per channel) and W2 in one pass."""
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    nel, n = 8, 1 << 24
    g = torch.Generator(device=device)
    g.manual_seed(3)
    rng = np.random.default_rng(3)
    freqs = rng.uniform(-0.5, 0.5, 4)
    t = torch.arange(n, device=device, dtype=torch.float64)
    xs = []
    for e in range(nel):
        x = torch.randn(n, dtype=torch.complex64, device=device, generator=g)
        for f, ph in zip(freqs, rng.uniform(0, 2 * math.pi, 4)):
            x += (math.sqrt(10.0) * torch.exp(1j * (2 * math.pi * f * t + ph))).to(torch.complex64)
        xs.append(x)
    del t
    p = ak.Pfb(FS, 2048, 1, 16, W.ATTEN_BETA8, nel)
    m = n // 2048 + 1
    out = torch.empty(nel * 2048 * m, dtype=torch.complex64, device=device)
    R = torch.zeros((2048, nel, nel), dtype=torch.complex64, device=device)
    cnt = torch.zeros(2048, dtype=torch.int32, device=device)
    pwr = torch.zeros((nel, 2048), dtype=torch.float32, device=device)
    mp = torch.zeros(2048, dtype=torch.float32, device=device)
    st = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p.handle), device=device)

    def step():
        y = gpu.process_n(p, xs, nel, out=out, stream=st)
        gpu.accumulate(y, nel, 2048, R, cnt, pwr, mp, stream=st)

    step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    for _ in range(max(steps, 1)):
        step()
    ev1.record(st)
    torch.cuda.synchronize()
    dt = ev0.elapsed_time(ev1) / 1e3
    res = {"workload": "coherent_8el_m2048_os1_k16_2^24", "value": round(nel * n * max(steps, 1) / dt / 1e6, 2),
           "unit": "MSamples/s (aggregate over elements)", "path": "process_n (device) + one-pass W1/W2"}
    if cpu:
        res.update(_c3_check([x[: 1 << 20].cpu().numpy() for x in xs], torch, device))
    return res


def _c3_check(xs, torch, device) -> dict:
    """The coherent array's first 2^20 samples of each element through a
    fresh handle and through the reference library (process_n, W1, W2):
    accuracy of the outputs, W1 and W2, float64 on 2^16, and the reference's
    rate on all host threads for the same work."""
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        return {}
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    nel, M = len(xs), 2048
    nth = os.cpu_count() or 1
    ref.lib.atkdsp_set_threads(nth)
    rp = ref.Pfb(FS, M, 1, 16, W.ATTEN_BETA8, nel)
    R = np.zeros((M, nel, nel), np.complex64)
    cnt = np.zeros(M, np.uint32)
    t0 = time.perf_counter()
    yr = rp.process_n(xs, nel)
    ref.pfb_cov_accumulate(yr, nel, M, None, R, cnt)
    pr, _ = ref.pfb_channel_power(yr, nel, M)
    rdt = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(1)                     # 2^18 samples per element, one thread
    rp1 = ref.Pfb(FS, M, 1, 16, W.ATTEN_BETA8, nel)
    R1, c1 = np.zeros((M, nel, nel), np.complex64), np.zeros(M, np.uint32)
    xs1 = [x[: 1 << 18] for x in xs]
    t0 = time.perf_counter()
    y1 = rp1.process_n(xs1, nel)
    ref.pfb_cov_accumulate(y1, nel, M, None, R1, c1)
    ref.pfb_channel_power(y1, nel, M)
    rdt1 = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(nth)
    p = ak.Pfb(FS, M, 1, 16, W.ATTEN_BETA8, nel)
    st = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p.handle), device=device)
    din = [torch.from_numpy(x).to(device) for x in xs]
    Rd = torch.zeros((M, nel, nel), dtype=torch.complex64, device=device)
    cd = torch.zeros(M, dtype=torch.int32, device=device)
    pd = torch.zeros((nel, M), dtype=torch.float32, device=device)
    md = torch.zeros(M, dtype=torch.float32, device=device)
    torch.cuda.synchronize()
    y = gpu.process_n(p, din, nel, stream=st)
    gpu.accumulate(y, nel, M, Rd, cd, pd, md, stream=st)
    torch.cuda.synchronize()
    y64 = _fp64(M, 1, 16, W.ATTEN_BETA8, [x[: 1 << 16] for x in xs])
    acc = _accuracy([(y.cpu().numpy(), yr, y64)], "2^20 samples of each of the 8 elements (float64 on 2^16)")
    Rg = Rd.cpu().numpy()
    acc["w1_max_rel"] = float(f"{float(np.max(np.abs(Rg - R)) / np.max(np.abs(R))):.3g}")
    acc["w2_power_max_rel"] = float(f"{float(np.max(np.abs(pd.cpu().numpy() - pr) / pr)):.3g}")
    return {"accuracy": acc,
            "cpu_baseline_1thread": {"value": round(nel * (1 << 18) / rdt1 / 1e6, 2),
                                     "unit": "MSamples/s (aggregate over elements)", "cores": 1,
                                     "kind": "reference", "sample": "2^18 samples of each element: process_n, "
                                                                    "W1, W2"},
            "cpu_baseline": {"value": round(nel * xs[0].size / rdt / 1e6, 2),
                             "unit": "MSamples/s (aggregate over elements)", "cores": nth, "kind": "reference",
                             "sample": "2^20 samples of each element: process_n, W1, W2"}}


OSX_N = 1 << 24


def _osx_fold_rate(nch: int, nfft: int, n: int, sec: float) -> dict:
    """What bounds the extractor: its exact fold, not HBM. Every block of
    nfft / 2 new samples folds all nfft spectrum bins into each channel, one
    complex product and add per bin, as 8 separately rounded FP32 operations
    (4 multiplies, 2 adds, 2 accumulating adds: no FMA, for the reference's
    rounding). Against the FP32 pipe's 128 operations per SM per clock (148
    SMs at the 1965 MHz maximum: 37.2 T operations/s)."""
    blocks = n / (nfft // 2)
    ops = nch * nfft * 8 * blocks
    peak = 148 * 128 * 1.965e9
    return {"fp32_ops_per_step": int(ops), "tops": round(ops / sec / 1e12, 2), "peak_tops": round(peak / 1e12, 1),
            "frac": round(ops / sec / peak, 3), "what": "rounded FP32 multiplies and adds of the fold"}


def _osx_arm(torch, device, steps, cpu: bool):
    """The overlap-save extractor: one 61.44 MS/s cf32 stream (noise + tones),
    nfft 4096, 64 channels (workloads.extractor_channels). value: atkdsp_gpu_osx_process_n on
    2^24 samples resident in HBM per step (CUDA events on the handle's stream,
    every kernel of the call inside); e2e: atkdsp_osx_process with pinned
    host buffers (dropin: pageable); cpu: the reference library on 2^20
    samples of the same stream."""
    import ctypes as C
    import atkdsp_b200 as ak
    from atkdsp_b200 import workloads as W
    OSX_FS, OSX_NFFT = W.EXTRACTOR_FS, W.EXTRACTOR_NFFT
    lib = ak.load()
    chans = W.extractor_channels()
    g = torch.Generator(device=device)
    g.manual_seed(9)
    x = torch.randn(OSX_N, dtype=torch.complex64, device=device, generator=g) * 0.5
    t = torch.arange(OSX_N, device=device, dtype=torch.float64)
    for f in (0.013, -0.21, 0.377):
        x += torch.exp(2j * math.pi * f * t).to(torch.complex64)
    del t
    o = ak.Osx(OSX_FS, OSX_NFFT)
    slots = [o.add(*c) for c in chans]
    cap = OSX_N // 64
    ys = [torch.empty(cap, dtype=torch.complex64, device=device) for _ in slots]
    ins = (C.c_void_p * 1)(x.data_ptr())
    outs = (C.c_void_p * len(slots))(*[y.data_ptr() for y in ys])
    counts = (C.c_size_t * len(slots))()
    st = torch.cuda.ExternalStream(lib.atkdsp_gpu_osx_stream(o.handle), device=device)

    def step():
        rc = lib.atkdsp_gpu_osx_process_n(o.handle, ins, 1, OSX_N, outs, counts, cap)
        if rc < 0:
            raise RuntimeError(f"osx: {rc}")

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = max(steps, 1)
    ev0.record(st)
    for _ in range(k):
        step()
    ev1.record(st)
    torch.cuda.synchronize()
    dt = ev0.elapsed_time(ev1) / 1e3
    out_samples = int(sum(counts))
    alg = 8 * OSX_N + 8 * out_samples
    achieved = alg / (dt / k) / 1e9
    peak, peak_kind = _peaks()
    # e2e: the C ABI with host buffers, copies inside the timed region --
    # pinned (as the filterbank's e2e arm) and pageable (the drop-in case)
    oh = ak.Osx(OSX_FS, OSX_NFFT)
    for c in chans:
        oh.add(*c)
    hcnt = (C.c_size_t * len(slots))()
    ke = max(1, min(k, 3))
    te = {}
    for kind in ("pinned", "pageable"):
        if kind == "pinned":
            xt = x.cpu().pin_memory()
            xh = xt.numpy()
            hbt = [torch.zeros(cap, dtype=torch.complex64).pin_memory() for _ in slots]
            hb = [b.numpy() for b in hbt]
        else:
            xh = x.cpu().numpy().copy()
            hb = [np.zeros(cap, np.complex64) for _ in slots]
        hptr = (C.POINTER(ak._Cf32) * len(slots))(*[ak._cfp(b) for b in hb])
        lib.atkdsp_osx_process(oh.handle, ak._cfp(xh), OSX_N, hptr, hcnt, cap)
        t0 = time.perf_counter()
        for _ in range(ke):
            lib.atkdsp_osx_process(oh.handle, ak._cfp(xh), OSX_N, hptr, hcnt, cap)
        te[kind] = (time.perf_counter() - t0) / ke
    res = {"workload": f"extractor_nfft{OSX_NFFT}_64ch_61.44msps_2^24", "value": round(OSX_N * k / dt / 1e6, 2),
           "unit": "MSamples/s", "ms_per_step": round(dt / k * 1e3, 3),
           "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "alg_bytes_per_step": alg, "peak_kind": peak_kind},
           "e2e": {"value": round(OSX_N / te["pinned"] / 1e6, 2), "unit": "MSamples/s",
                   "h2d_bytes_per_step": 8 * OSX_N, "d2h_bytes_per_step": 8 * int(sum(hcnt)),
                   "path": "atkdsp_osx_process, pinned host buffers"},
           "dropin": {"value": round(OSX_N / te["pageable"] / 1e6, 2), "unit": "MSamples/s",
                      "path": "atkdsp_osx_process, pageable host buffers"},
           "fold": _osx_fold_rate(len(slots), OSX_NFFT, OSX_N, dt / k),
           "out_samples_per_step": out_samples,
           "path": "atkdsp_gpu_osx_process_n: fused transform + 64 channel folds/inverses/rolls per block, "
                   "resampler, state carry"}
    if cpu:
        from oracle import oracle as O
        ref = O.reference()
        if ref is not None:
            r = ref.Osx(OSX_FS, OSX_NFFT)
            for c in chans:
                r.add(*c)
            xs = xh[: 1 << 20]
            r.process(xs)
            t0 = time.perf_counter()
            r.process(xs)
            tc = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": round(xs.size / tc / 1e6, 2), "unit": "MSamples/s", "cores": 1,
                                   "kind": "reference", "sample": "2^20 samples of the same stream "
                                   "(atkdsp_osx_process_n is single-threaded)"}
    return res


def _bank_arm(torch, device, steps, cpu: bool):
    """Undertow's per-scale bank (workloads.scale_bank: 8 .. 256 channels, 2x,
    12 taps) on one stream of 65536-sample chunks: every chunk goes through
    all six scales. value: one batch launch per chunk (CUDA graph replay),
    64 chunks per step; plain: one device call per scale per chunk; cpu: the
    reference library's six atkdsp_pfb_process calls per chunk (all host
    threads, the survey's own loop)."""
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    from atkdsp_b200.gpu import Batch
    bank = W.scale_bank(6)
    blk, nchunk = W.SCALE_BANK_BLOCK, 64
    g = torch.Generator(device=device)
    g.manual_seed(11)
    x = torch.randn(blk * nchunk, dtype=torch.complex64, device=device, generator=g)
    chunks = [x[i * blk:(i + 1) * blk] for i in range(nchunk)]
    hs = [ak.Pfb(FS, M, os_, K) for M, os_, K in bank]
    batch = Batch(hs)
    outs = [torch.empty(M * (blk // (M // 2) + 2), dtype=torch.complex64, device=device) for M, _, _ in bank]
    st = torch.cuda.ExternalStream(batch.stream_ptr, device=device)

    def step_batched():
        for c in chunks:
            batch.process([c] * len(bank), outs)

    ps = [ak.Pfb(FS, M, os_, K) for M, os_, K in bank]

    def step_plain():
        for c in chunks:
            for p, o in zip(ps, outs):
                gpu.process_n(p, [c], 1, out=o, stream=st)

    res = {"workload": "scale_bank_6_scales_8-256ch_os2_k12_chunks_65536", "unit": "MSamples/s",
           "path": "atkdsp_gpu_batch_process: one launch per chunk over all six scales"}
    for name, fn in (("value", step_batched), ("plain", step_plain)):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(max(steps, 1)):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        res[name] = round(blk * nchunk * max(steps, 1) / (e0.elapsed_time(e1) / 1e3) / 1e6, 2)
    if cpu:
        from oracle import oracle as O
        ref = O.reference()
        if ref is not None:
            nth = os.cpu_count() or 1
            ref.lib.atkdsp_set_threads(nth)
            rp = [ref.Pfb(FS, M, os_, K) for M, os_, K in bank]
            xh = x[: blk * 8].cpu().numpy()
            t0 = time.perf_counter()
            for i in range(8):
                for p in rp:
                    p.process(xh[i * blk:(i + 1) * blk])
            res["cpu_baseline"] = {"value": round(8 * blk / (time.perf_counter() - t0) / 1e6, 2),
                                   "unit": "MSamples/s", "cores": nth, "kind": "reference",
                                   "sample": "8 chunks through the six scales"}
    return res


def _spectrum_arm(torch, device, steps, cpu: bool):
    """The display reduction on the same kind of device block: 2^24 cf32
    samples, n 4096, hop 2048 (50 % overlap), Hann window; value: the
    average-detector line (atkdsp_gpu_spectrum_reduce); stats: the four
    stats lines in one pass; cpu: the reference's atkdsp_spectrum_reduce on
    2^22 samples with every host thread."""
    from atkdsp_b200.gpu import Spectrum
    n, hop, N = 4096, 2048, 1 << 24
    g = torch.Generator(device=device)
    g.manual_seed(13)
    x = torch.randn(N, dtype=torch.complex64, device=device, generator=g)
    k = np.arange(n)
    w = torch.from_numpy((0.5 - 0.5 * np.cos(2.0 * np.pi * k / (n - 1))).astype(np.float32)).to(device)
    sp = Spectrum(n)
    res = {"workload": "spectrum_n4096_hop2048_hann_2^24", "unit": "MSamples/s",
           "path": "atkdsp_gpu_spectrum_reduce (average detector) / atkdsp_gpu_spectrum_stats"}
    for name, fn in (("value", lambda: sp.reduce(x, hop, w, "avg")), ("stats", lambda: sp.stats(x, hop, w))):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(max(steps, 1)):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = round(N * max(steps, 1) / (e0.elapsed_time(e1) / 1e3) / 1e6, 2)
    res["frames_per_call"] = (N - n) // hop + 1
    if cpu:
        from oracle import oracle as O
        ref = O.reference()
        if ref is not None:
            nth = os.cpu_count() or 1
            ref.lib.atkdsp_set_threads(nth)
            xs = x[: 1 << 22].cpu().numpy()
            wh = w.cpu().numpy()
            ref.spectrum_reduce(xs, n, hop, wh, "avg")
            t0 = time.perf_counter()
            ref.spectrum_reduce(xs, n, hop, wh, "avg")
            res["cpu_baseline"] = {"value": round(xs.size / (time.perf_counter() - t0) / 1e6, 2),
                                   "unit": "MSamples/s", "cores": nth, "kind": "reference",
                                   "sample": "2^22 samples, same n / hop / window"}
    return res


def _cfar_arm(torch, device, steps, cpu: bool):
    """The CFAR detector and tracker over spectrum lines: 4096 bins, 1024
    frames per call (gamma noise floor with a slope, 64 bursts), CA with 16 +
    16 reference cells, 4 guard, k_frames 4, Pfa 1e-6. value: device frames
    (atkdsp_gpu_cfar_process, events to the host); gate: the same with every
    frame's hit mask kept on the device; e2e: host frames through
    atkdsp_cfar_process; cpu: the reference's atkdsp_cfar_process (one
    thread: it has no threading) on 128 frames."""
    import atkdsp_b200 as ak
    from atkdsp_b200.gpu import cfar_process
    from oracle import oracle as O
    nb, nf = 4096, 1024
    rng = np.random.default_rng(21)
    floor = rng.gamma(1.0, 1.0, size=(nf, nb)) * np.linspace(1.0, 2.0, nb)[None, :]
    for _ in range(64):
        lo, f0 = int(rng.integers(0, nb - 8)), int(rng.integers(0, nf - 8))
        floor[f0:f0 + int(rng.integers(4, 200)), lo:lo + int(rng.integers(1, 8))] += 10 ** rng.uniform(1, 3)
    xs = (10.0 * np.log10(floor)).astype(np.float32)
    cfg = dict(k_frames=4)
    d = torch.from_numpy(xs).to(device)
    hits = torch.empty(d.shape, dtype=torch.uint8, device=device)
    res = {"workload": "cfar_ca_4096bins_1024frames_k4", "unit": "Mcells/s",
           "path": "atkdsp_gpu_cfar_process (device frames) / atkdsp_cfar_process (host frames)"}
    for name, fn in (("value", lambda c: cfar_process(c, d, 0.0, 1e-3)),
                     ("gate", lambda c: cfar_process(c, d, 0.0, 1e-3, hits=hits)),
                     ("e2e", lambda c: c.process(xs, 0.0, 1e-3))):
        c = ak.Cfar(nb, **cfg)
        for _ in range(2):
            fn(c)
        n = max(steps, 1)
        t0 = time.perf_counter()
        for _ in range(n):
            ev = fn(c)
        dt = time.perf_counter() - t0
        res[name] = round(nb * nf * n / dt / 1e6, 1)
        res[f"{name}_events_per_call"] = len(ev[0] if isinstance(ev, tuple) else ev)
    res["frames_per_s"] = round(res["value"] * 1e6 / nb, 0)
    if cpu:
        ref = O.reference()
        if ref is not None:
            rc = O.RefCfar(ref, nb, **cfg)
            rc.process(xs[:16], 0.0, 1e-3)
            t0 = time.perf_counter()
            rc.process(xs[16:144], 0.0, 1e-3)
            res["cpu_baseline"] = {"value": round(nb * 128 / (time.perf_counter() - t0) / 1e6, 2),
                                   "unit": "Mcells/s", "cores": 1, "kind": "reference",
                                   "sample": "128 frames of the same workload"}
    return res


def _served_arm(torch, device, duration_s, cpu: bool):
    """Serving: 4096 live streams at {2.4, 10, 40} MS/s delivering 1.6 ms ci16
    blocks with Poisson arrivals, nchan {256, 1024}, 16 taps, 2x, churn 20/s,
    admission by free HBM. Then the largest stream count whose p99 block
    latency stays under 1.6 ms."""
    from atkdsp_b200.serve import Server, simulate
    srv = Server(max_streams=4608, hbm_reserve=16 << 30, use_graph=True)
    raw = torch.randint(-6000, 6000, (2 * (8 << 20),), dtype=torch.int16, device=device)
    out = torch.empty((2 << 30) // 8, dtype=torch.complex64, device=device)
    full = simulate(srv, streams=4096, duration_s=duration_s, warmup_s=0.5, raw_pool=raw, out_pool=out)
    res = {"workload": "served_4096_streams_ci16_m256_1024_k16", "offered_msps": round(full["offered_samples_per_s"] / 1e6, 1),
           "value": round(full["samples_done"] / full["wall_s"] / 1e6, 2), "unit": "MSamples/s",
           "p50_ms": round(full["lat_p50_ms"], 3), "p99_ms": round(full["lat_p99_ms"], 3),
           "blocks_per_round": round(full["blocks_per_round"], 1), "dropped_blocks": int(full["dropped_blocks"]),
           "denied": int(full["denied"]), "churn_events": int(full["churn_events"]),
           "per_round": {"host_launch_ms": round(full["mean_launch_ms"], 3),
                         "gpu_ms": round(full["mean_round_gpu_ms"], 3), "gpu_busy": round(full["gpu_busy"], 3),
                         "capacity_msps": round(full["blocks_per_round"] * (full["samples_done"] / max(1, full["blocks_done"]))
                                                / max(1e-9, full["mean_round_gpu_ms"]) / 1e3, 1)}}
    best = None
    lo, hi = 64, 4096
    if full["lat_p99_ms"] < 1.6:
        best = (4096, full)
    else:
        while hi - lo > 64:
            mid = (lo + hi) // 2
            srv2 = Server(max_streams=mid + 512, hbm_reserve=16 << 30, use_graph=True)
            r = simulate(srv2, streams=mid, duration_s=max(1.0, duration_s / 2), warmup_s=0.3, raw_pool=raw,
                         out_pool=out)
            del srv2
            if r["lat_p99_ms"] < 1.6 and r["dropped_blocks"] == 0:
                lo, best = mid, (mid, r)
            else:
                hi = mid
    if best:
        n, r = best
        res["within_p99_1.6ms"] = {"streams": n, "value": round(r["samples_done"] / r["wall_s"] / 1e6, 2),
                                   "p50_ms": round(r["lat_p50_ms"], 3), "p99_ms": round(r["lat_p99_ms"], 3)}
    if cpu:
        res.update(_served_check(torch, device))
    return res


def _served_check(torch, device) -> dict:
    """Served streams' blocks (ci16, nchan 256 / 1024, 16 taps, 2x): eight
    streams' first four 1.6 ms blocks through the fused int16 device path and
    through the reference library (unpack to cf32, then the filterbank) for
    accuracy; and the reference's rate over one block of each of the first
    512 streams of the trace, one call pair per block, all host threads."""
    from oracle import oracle as O
    ref = O.reference()
    if ref is None:
        return {}
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from atkdsp_b200 import workloads as W
    specs = W.served_streams(4096)
    nth = os.cpu_count() or 1
    ref.lib.atkdsp_set_threads(nth)
    cases = []
    for sp in specs[:8]:
        rp = ref.Pfb(FS, sp.nchan, 2, 16, 80.0, 1)
        p = ak.Pfb(FS, sp.nchan, 2, 16, 80.0, 1)
        st = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p.handle), device=device)
        ys, rs = [], []
        for b in range(4):
            raw = W.ci16_block(sp.block, sp.seed, b)
            x, _ = ref.unpack_dc(raw.tobytes(), "ci16", 0j)
            rs.append(rp.process_n([x], 1))
            d = torch.from_numpy(raw.reshape(-1).copy()).to(device)
            torch.cuda.synchronize()
            ys.append(gpu.process_n_raw(p, [d], 1, "ci16", 0j, stream=st).cpu().numpy())
        cases.append((np.concatenate(ys, axis=-1), np.concatenate(rs, axis=-1), None))
    acc = _accuracy(cases, "eight served streams, four blocks each")
    blocks = [(sp, W.ci16_block(sp.block, sp.seed, 0).tobytes()) for sp in specs[:512]]
    handles = {}
    n = 0
    t0 = time.perf_counter()
    for sp, raw in blocks:
        h = handles.get(sp.nchan) or handles.setdefault(sp.nchan, ref.Pfb(FS, sp.nchan, 2, 16, 80.0, 1))
        x, _ = ref.unpack_dc(raw, "ci16", 0j)
        h.process_n([x], 1)
        n += x.size
    rdt = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(1)                     # the first 64 of those blocks, one thread
    handles1 = {}
    n1 = 0
    t0 = time.perf_counter()
    for sp, raw in blocks[:64]:
        h = handles1.get(sp.nchan) or handles1.setdefault(sp.nchan, ref.Pfb(FS, sp.nchan, 2, 16, 80.0, 1))
        x, _ = ref.unpack_dc(raw, "ci16", 0j)
        h.process_n([x], 1)
        n1 += x.size
    rdt1 = time.perf_counter() - t0
    ref.lib.atkdsp_set_threads(nth)
    return {"accuracy": acc,
            "cpu_baseline_1thread": {"value": round(n1 / rdt1 / 1e6, 2), "unit": "MSamples/s", "cores": 1,
                                     "kind": "reference",
                                     "sample": "one block of each of the first 64 streams of the trace"},
            "cpu_baseline": {"value": round(n / rdt / 1e6, 2), "unit": "MSamples/s", "cores": nth,
                             "kind": "reference",
                             "sample": "one block of each of the first 512 streams of the trace (unpack_dc + "
                                       "filterbank per block)"}}


def run_ours(args, rep):
    import torch

    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu

    rank, world, local_rank = rep.rank, rep.world, rep.local_rank
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    specs = _specs(rank, args)
    S = sum(s.length for s in specs)
    arms = set(args.arms.split(","))
    sets = _device_blocks(specs, torch, device, seed=rank)
    obuf, outs = _out_buffers(specs, torch, device)

    barrier = rep.barrier
    max_over_ranks = rep.max

    # ---- batched path (the headline) ----
    handles = [ak.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in specs]
    batch = gpu.Batch(handles, use_graph=True)
    bstream = torch.cuda.ExternalStream(batch.stream_ptr, device=device)
    ms_list = None

    def bstep(k):
        nonlocal ms_list
        ms_list = batch.process(sets[k % 3][1], outs)

    for k in range(args.warmup):
        bstep(k)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        time.sleep(0.3)                      # let the sampler start
        barrier()
        torch.cuda.synchronize()
        clk.mark_start()
        ev0.record(bstream)
        for k in range(args.steps):
            bstep(args.warmup + k)
        ev1.record(bstream)
        torch.cuda.synchronize()
        clk.mark_end()
        time.sleep(0.05)
    barrier()
    t_batch = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    alg = _alg_bytes(specs, ms_list)
    # the tile kernel alone, per launch (events inside the graph)
    kms = []
    for k in range(max(3, args.steps)):
        bstep(k)
        kms.append(batch.kernel_ms())
    k_ms = float(np.mean(kms))

    t_plain = t_e2e = t_dropin = None
    out_bytes = 8 * sum(s.nchan * m for s, m in zip(specs, ms_list))
    extra = {}
    if "plain" in arms:
        t_plain, plain_by_len = _plain_arm(args, specs, sets, outs, torch, device, barrier, max_over_ranks)
    t_e2e_batch = None
    if "e2e" in arms:
        t_e2e_batch = _e2e_batch_arm(args, S, sets, obuf, bstream, bstep, torch, barrier, max_over_ranks)
        t_e2e = _cabi_arm(specs, sets, torch, barrier, max_over_ranks, True, args.steps, args.warmup)
    if "dropin" in arms:
        t_dropin = _cabi_arm(specs, sets, torch, barrier, max_over_ranks, False, 1, 1)

    del batch, handles, bstream
    torch.cuda.synchronize()
    if rank == 0:
        for name, fn in (("single_stream", lambda: _c1_arm(torch, "cpu" in arms and not args.no_cpu)),
                         ("front_end", lambda: _c2_arm(torch, device, 1, "cpu" in arms and not args.no_cpu)),
                         ("coherent_array", lambda: _c3_arm(torch, device, args.steps, "cpu" in arms and not args.no_cpu)),
                         ("extractor", lambda: _osx_arm(torch, device, args.steps,
                                                        "cpu" in arms and not args.no_cpu)),
                         ("scale_bank", lambda: _bank_arm(torch, device, args.steps,
                                                          "cpu" in arms and not args.no_cpu)),
                         ("spectrum", lambda: _spectrum_arm(torch, device, args.steps,
                                                            "cpu" in arms and not args.no_cpu)),
                         ("cfar", lambda: _cfar_arm(torch, device, args.steps,
                                                    "cpu" in arms and not args.no_cpu)),
                         ("served", lambda: _served_arm(torch, device, 3.0, "cpu" in arms and not args.no_cpu))):
            if name in arms:
                try:
                    extra[name] = fn()
                except Exception as e:                       # report, keep the headline
                    extra[name] = {"error": f"{type(e).__name__}: {e}"}
                torch.cuda.synchronize()
                torch.cuda.empty_cache()
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    achieved = alg / (k_ms / 1e3) / 1e9
    # DRAM traffic per launch: the traffic / algorithmic-bytes ratio of an ncu
    # capture of this kernel on a smaller version of the workload (the full
    # launch is too large for a multi-pass capture), scaled to this launch
    traffic, traffic_src = None, None
    prof = ROOT / "profiles" / "pfb_tiles_uneven256.json"
    if prof.exists():
        pj = json.loads(prof.read_text())
        if pj.get("ratio_traffic_over_algorithmic"):
            traffic = int(round(pj["ratio_traffic_over_algorithmic"] * alg))
            traffic_src = (f"ratio {pj['ratio_traffic_over_algorithmic']} (profiles/pfb_tiles_uneven256.json: "
                           f"{pj.get('captured', 'ncu capture')}) x this launch's algorithmic bytes")
    cpu = _cpu_reference_rate(specs) if "cpu" in arms and not args.no_cpu else None
    cpu1 = _cpu_reference_rate(specs, budget_s=3.0, threads=1) if "cpu" in arms and not args.no_cpu else None
    acc = _batched_accuracy(specs, torch, device) if "cpu" in arms and not args.no_cpu else None
    total = S * world
    value = total * args.steps / t_batch / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "MSamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_batch / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 fold + f64 fft", "data": "synthetic (seeded noise + tones, generated on device)",
        "config": dict(_config(args, world), samples_per_step_per_gpu=S),
        "plain": None if t_plain is None else {
            "value": round(total * args.steps / t_plain / 1e6, 2), "unit": "MSamples/s",
            "what": "one device-pointer call per stream",
            "by_length": plain_by_len},
        "batched_over_plain": None if t_plain is None else round(t_plain / t_batch, 2),
        "e2e": None if t_e2e is None else {
            "value": round(total * args.steps / t_e2e[0] / 1e6, 2), "unit": "MSamples/s",
            "h2d_bytes_per_step": t_e2e[1], "d2h_bytes_per_step": t_e2e[2],
            "path": f"atkdsp_pfb_process (C ABI), pinned host buffers, one handle per stream, "
                    f"{CABI_THREADS} host threads"},
        "e2e_batch": None if t_e2e_batch is None else {
            "value": round(total * args.steps / t_e2e_batch / 1e6, 2), "unit": "MSamples/s",
            "h2d_bytes_per_step": 8 * S, "d2h_bytes_per_step": out_bytes,
            "path": "atkdsp_gpu_batch_process with pinned host<->device copies on its stream"},
        "dropin": None if t_dropin is None else {
            "value": round(total / t_dropin[0] / 1e6, 2), "unit": "MSamples/s",
            "what": f"atkdsp_pfb_process per stream, pageable host buffers, {CABI_THREADS} host threads"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                     "kernel": "pfb_tiles_kernel", "kernel_ms": round(k_ms, 4),
                     "alg_bytes_per_launch": alg, "peak_kind": peak_kind},
        "configs": extra,
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "native_so": _native_maps(),
    }
    if acc:
        line["accuracy"] = acc
    if cpu:
        line["cpu_baseline"] = {"value": round(cpu[0], 2), "unit": "MSamples/s", "cores": cpu[1],
                                "kind": "reference", "sample": cpu[2]}
    if cpu1:
        line["cpu_baseline_1thread"] = {"value": round(cpu1[0], 2), "unit": "MSamples/s", "cores": 1,
                                        "kind": "reference", "sample": cpu1[2]}
    print(json.dumps(line))


def _native_maps() -> list:
    """The shared objects of this repository mapped into this process (read
    from /proc/self/maps): the evidence of which native code ran."""
    seen = []
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                parts = ln.split()
                if len(parts) >= 6 and parts[-1].endswith(".so") and parts[-1].startswith(str(ROOT)):
                    rel = os.path.relpath(parts[-1], ROOT)
                    if rel not in seen:
                        seen.append(rel)
    except OSError:
        pass
    return seen


def _spawn_ranks(n: int) -> int:
    """`--gpus N` without a launcher: start N ranks under torch.distributed.run
    (one process per GPU, rendezvous on 127.0.0.1) and pass their output and
    exit status through."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve())]
    cmd += sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--arms", default="batched,plain,e2e,dropin,cpu,single_stream,front_end,coherent_array,"
                    "extractor,scale_bank,spectrum,cfar,served",
                    help="comma list of arms to run (the batched arm always runs)")
    ap.add_argument("--cabi-threads", type=int, default=0,
                    help="host threads for the C-ABI (e2e, drop-in) arms; 0: min(8, cores)")
    ap.add_argument("--streams", type=int, default=256)
    ap.add_argument("--min-log2", type=float, default=14.0)
    ap.add_argument("--max-log2", type=float, default=22.0)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.cabi_threads > 0:
        global CABI_THREADS
        CABI_THREADS = args.cabi_threads
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(_spawn_ranks(args.gpus))
    from atkdsp_b200.replicas import Replicas

    # one process per GPU; the group exists only for the timing reductions
    rep = Replicas(backend="gloo" if args.impl == "reference" else None, timeout_s=120)
    if rep.world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but the launcher started {rep.world} ranks")
    try:
        if args.impl == "reference":
            run_reference(args, rep.rank, rep.world)
        else:
            run_ours(args, rep)
    finally:
        rep.close()
    sys.stdout.flush()


if __name__ == "__main__":
    main()
