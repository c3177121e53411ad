"""Per-configuration throughput of the tile kernel, one stream at a time.

    python -m atkdsp_b200.microbench --nchan 4096 --taps 16 --oversample 2
    python -m atkdsp_b200.microbench --sweep
    python -m atkdsp_b200.microbench --osx --nfft 4096 --channels 64
    python -m atkdsp_b200.microbench --kernels
    python -m atkdsp_b200.microbench --cfar --nbins 4096 --frames 1024

Each configuration channelizes one device-resident block of 2^log2n cf32
samples (seeded noise, larger than L2 at the default 2^24) through a
one-handle Batch (the same persistent kernel the batched serving path
launches) and reports input samples per second from the kernel's own CUDA
event pair, the median of the timed repetitions after two warm-ups. One JSON
line per configuration: {"nchan", "taps", "oversample", "samples",
"kernel_ms", "gsps", "hbm_gbs"} where hbm_gbs counts the algorithmic bytes
(8 B in + 8*oversample B out per input sample).

--kernels times the other device building blocks once each, on blocks
larger than L2: unpack_dc of 2^25 ci16 samples (conversion + mean),
block_mean alone, the one-pass W1/W2 over an 8-element 2048-channel output
of 2048 hops, and the spectrum reduction / stats of 2^24 samples (n 4096,
hop 2048, Hann). One JSON line per kernel: {"op", "ms", "gbs"} with gbs the
algorithmic bytes (read + written once) per second.

--osx times the overlap-save extractor instead: one device-resident cf32
stream through atkdsp_gpu_osx_process_n with the extractor_channels plan of
workloads.py (CUDA events on the handle's stream around the whole call).

--cfar times the CFAR detector and tracker on device frames (nbins dB lines
of exponential noise with 64 bursts, 16 + 16 cells, 4 guard, k_frames 4;
--mode picks the statistic, CA by default)
through atkdsp_gpu_cfar_process: the whole synchronous call, host clock,
median of the repetitions. {"nbins", "frames", "ms", "mcells_s", "events"}.
"""

from __future__ import annotations

import argparse
import json

import numpy as np


def run_one(nchan: int, taps: int, oversample: int, log2n: int = 24, reps: int = 5, fs: float = 2.4e6):
    import torch

    from . import Pfb
    from .gpu import Batch

    n = 1 << log2n
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(n, dtype=torch.complex64, device="cuda", generator=g)
    p = Pfb(fs, nchan, oversample, taps)
    b = Batch([p], use_graph=False)
    m = p.out_hops(n)
    out = torch.empty(max(1, nchan * m), dtype=torch.complex64, device="cuda")
    ts = []
    for _ in range(2 + reps):
        b.process([x], [out])
        ts.append(b.kernel_ms())
    t = float(np.median(ts[2:]))
    res = {"nchan": nchan, "taps": taps, "oversample": oversample, "samples": n,
           "kernel_ms": round(t, 4), "gsps": round(n / t / 1e6, 2),
           "hbm_gbs": round((8 + 8 * oversample) * n / (t / 1e3) / 1e9, 1)}
    del b, p
    return res


def run_osx(nfft: int = 4096, channels: int = 64, log2n: int = 24, reps: int = 5, nel: int = 1):
    import ctypes as C

    import torch

    from . import Osx, load
    from . import workloads as W

    lib = load()
    n = 1 << log2n
    g = torch.Generator(device="cuda").manual_seed(1)
    xs = [torch.randn(n, dtype=torch.complex64, device="cuda", generator=g) for _ in range(nel)]
    o = Osx(W.EXTRACTOR_FS, nfft, 80.0, nel)
    plan = W.extractor_channels(channels)
    for c in plan:
        o.add(*c)
    cap = n // 16 + 4096
    ys = [torch.empty(cap, dtype=torch.complex64, device="cuda") for _ in range(nel * channels)]
    ins = (C.c_void_p * nel)(*[x.data_ptr() for x in xs])
    outs = (C.c_void_p * len(ys))(*[y.data_ptr() for y in ys])
    counts = (C.c_size_t * channels)()
    st = torch.cuda.ExternalStream(lib.atkdsp_gpu_osx_stream(o.handle))
    ts = []
    for _ in range(2 + reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if lib.atkdsp_gpu_osx_process_n(o.handle, ins, nel, n, outs, counts, cap) < 0:
            raise RuntimeError("osx_process_n failed")
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    t = float(np.median(ts[2:]))
    return {"osx_nfft": nfft, "channels": channels, "elements": nel, "samples": n, "ms": round(t, 3),
            "msps": round(nel * n / t / 1e3, 1), "out_samples": int(sum(counts)) * nel}


def run_cfar(nbins: int = 4096, frames: int = 1024, reps: int = 5, mode: str = "ca") -> dict:
    import time

    import torch

    from . import Cfar
    from .gpu import cfar_process

    g = torch.Generator(device="cuda").manual_seed(21)
    u = torch.rand((frames, nbins), dtype=torch.float64, device="cuda", generator=g)
    p = -torch.log1p(-u) * torch.linspace(1.0, 2.0, nbins, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(21)
    for _ in range(64):
        lo, f0 = int(rng.integers(0, nbins - 8)), int(rng.integers(0, frames - 8))
        p[f0:f0 + int(rng.integers(4, 200)), lo:lo + int(rng.integers(1, 8))] += 10 ** rng.uniform(1, 3)
    x = (10.0 * torch.log10(p)).to(torch.float32).contiguous()
    c = Cfar(nbins, k_frames=4, mode=mode)
    for _ in range(2):
        cfar_process(c, x, 0.0, 1e-3)
    ts, nev = [], 0
    for _ in range(reps):
        t0 = time.perf_counter()
        nev = len(cfar_process(c, x, 0.0, 1e-3)[0])
        ts.append((time.perf_counter() - t0) * 1e3)
    ms = float(np.median(ts))
    return {"nbins": nbins, "frames": frames, "mode": mode, "ms": round(ms, 3),
            "mcells_s": round(nbins * frames / ms / 1e3, 1), "events": nev}


def run_kernels(reps: int = 5) -> list:
    import torch

    from . import gpu

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    g = torch.Generator(device="cuda").manual_seed(5)
    res = []
    n = 1 << 25
    raw = torch.randint(-2048, 2048, (2 * n,), dtype=torch.int16, device="cuda", generator=g)
    out = torch.empty(n, dtype=torch.complex64, device="cuda")
    mean = torch.empty(2, dtype=torch.float64, device="cuda")
    t = timed(lambda: gpu.unpack_dc(raw, "ci16q11", 0.01 - 0.02j, out=out))
    res.append({"op": "unpack_dc ci16q11 2^25", "ms": round(t, 4), "gbs": round(12 * n / t / 1e6, 1)})
    t = timed(lambda: gpu.block_mean(raw, "ci16q11", 0.01 - 0.02j, mean))
    res.append({"op": "block_mean ci16q11 2^25", "ms": round(t, 4), "gbs": round(4 * n / t / 1e6, 1)})
    del raw, out
    nel, M, m = 8, 2048, 2048
    y = torch.randn(nel * M * m, dtype=torch.complex64, device="cuda", generator=g).view(nel, M, m)
    R = torch.zeros((M, nel, nel), dtype=torch.complex64, device="cuda")
    cnt = torch.zeros(M, dtype=torch.int32, device="cuda")
    pwr = torch.zeros((nel, M), dtype=torch.float32, device="cuda")
    mp = torch.zeros(M, dtype=torch.float32, device="cuda")
    t = timed(lambda: gpu.accumulate(y, nel, M, R, cnt, pwr, mp))
    res.append({"op": "W1+W2 one pass, 8 elements x 2048 channels x 2048 hops", "ms": round(t, 4),
                "gbs": round(8 * nel * M * m / t / 1e6, 1)})
    del y
    xs = torch.randn(1 << 24, dtype=torch.complex64, device="cuda", generator=g)
    k = np.arange(4096)
    w = torch.from_numpy((0.5 - 0.5 * np.cos(2 * np.pi * k / 4095)).astype(np.float32)).cuda()
    sp = gpu.Spectrum(4096)
    t = timed(lambda: sp.reduce(xs, 2048, w, "avg"))
    res.append({"op": "spectrum_reduce avg n4096 hop2048 2^24", "ms": round(t, 4),
                "gbs": round(8 * (1 << 24) / t / 1e6, 1)})
    t = timed(lambda: sp.stats(xs, 2048, w))
    res.append({"op": "spectrum_stats n4096 hop2048 2^24", "ms": round(t, 4),
                "gbs": round(8 * (1 << 24) / t / 1e6, 1)})
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--nchan", type=int, default=1024)
    ap.add_argument("--taps", type=int, default=16)
    ap.add_argument("--oversample", type=int, default=2)
    ap.add_argument("--log2n", type=int, default=24)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--sweep", action="store_true",
                    help="nchan 64/256/1024/4096 x taps 8/12/16 x oversample 1/2")
    ap.add_argument("--osx", action="store_true", help="the overlap-save extractor instead")
    ap.add_argument("--kernels", action="store_true", help="unpack, W1/W2 and spectrum kernels")
    ap.add_argument("--nfft", type=int, default=4096)
    ap.add_argument("--channels", type=int, default=64)
    ap.add_argument("--elements", type=int, default=1)
    ap.add_argument("--cfar", action="store_true", help="the CFAR detector and tracker")
    ap.add_argument("--nbins", type=int, default=4096)
    ap.add_argument("--frames", type=int, default=1024)
    ap.add_argument("--mode", default="ca", choices=["ca", "os", "go", "so"], help="the CFAR statistic")
    ap.add_argument("--choice", type=int, default=-1,
                    help="tile shape for the filterbank run (atkdsp_gpu_tune_set: 1 paired, 0 one hop "
                         "per thread, 2 quad; -1 the table's)")
    a = ap.parse_args(argv)
    if a.choice >= 0:
        from . import load
        if load().atkdsp_gpu_tune_set(a.nchan, a.oversample, a.taps, a.choice) != 0:
            raise SystemExit(f"no tile shape {a.choice} for nchan {a.nchan} oversample {a.oversample}")
    if a.cfar:
        print(json.dumps(run_cfar(a.nbins, a.frames, a.reps, a.mode)), flush=True)
    elif a.kernels:
        for r in run_kernels(a.reps):
            print(json.dumps(r), flush=True)
    elif a.osx:
        print(json.dumps(run_osx(a.nfft, a.channels, a.log2n, a.reps, a.elements)), flush=True)
    elif a.sweep:
        for M in (64, 256, 1024, 4096):
            for K in (8, 12, 16):
                for os_ in (1, 2):
                    print(json.dumps(run_one(M, K, os_, a.log2n, a.reps)), flush=True)
    else:
        print(json.dumps(run_one(a.nchan, a.taps, a.oversample, a.log2n, a.reps)), flush=True)


if __name__ == "__main__":
    main()
