"""Per-configuration throughput of the tile kernel, one stream at a time.

    python -m atkdsp_b200.microbench --nchan 4096 --taps 16 --oversample 2
    python -m atkdsp_b200.microbench --sweep
    python -m atkdsp_b200.microbench --osx --nfft 4096 --channels 64

Each configuration channelizes one device-resident block of 2^log2n cf32
samples (seeded noise, larger than L2 at the default 2^24) through a
one-handle Batch (the same persistent kernel the batched serving path
launches) and reports input samples per second from the kernel's own CUDA
event pair, the median of the timed repetitions after two warm-ups. One JSON
line per configuration: {"nchan", "taps", "oversample", "samples",
"kernel_ms", "gsps", "hbm_gbs"} where hbm_gbs counts the algorithmic bytes
(8 B in + 8*oversample B out per input sample).

--osx times the overlap-save extractor instead: one device-resident cf32
stream through atkdsp_gpu_osx_process_n with the extractor_channels plan of
workloads.py (CUDA events on the handle's stream around the whole call).
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
    ap.add_argument("--nfft", type=int, default=4096)
    ap.add_argument("--channels", type=int, default=64)
    ap.add_argument("--elements", type=int, default=1)
    a = ap.parse_args(argv)
    if a.osx:
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
