"""Per-configuration throughput of the tile kernel, one stream at a time.

    python -m atkdsp_b200.microbench --nchan 4096 --taps 16 --oversample 2
    python -m atkdsp_b200.microbench --sweep

Each configuration channelizes one device-resident block of 2^log2n cf32
samples (seeded noise, larger than L2 at the default 2^24) through a
one-handle Batch (the same persistent kernel the batched serving path
launches) and reports input samples per second from the kernel's own CUDA
event pair, the median of the timed repetitions after two warm-ups. One JSON
line per configuration: {"nchan", "taps", "oversample", "samples",
"kernel_ms", "gsps", "hbm_gbs"} where hbm_gbs counts the algorithmic bytes
(8 B in + 8*oversample B out per input sample).
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


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--nchan", type=int, default=1024)
    ap.add_argument("--taps", type=int, default=16)
    ap.add_argument("--oversample", type=int, default=2)
    ap.add_argument("--log2n", type=int, default=24)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--sweep", action="store_true",
                    help="nchan 64/256/1024/4096 x taps 8/12/16 x oversample 1/2")
    a = ap.parse_args(argv)
    if a.sweep:
        for M in (64, 256, 1024, 4096):
            for K in (8, 12, 16):
                for os_ in (1, 2):
                    print(json.dumps(run_one(M, K, os_, a.log2n, a.reps)), flush=True)
    else:
        print(json.dumps(run_one(a.nchan, a.taps, a.oversample, a.log2n, a.reps)), flush=True)


if __name__ == "__main__":
    main()
