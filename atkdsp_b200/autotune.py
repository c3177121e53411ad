"""The tile-shape autotuner.

    python -m atkdsp_b200.autotune            # measure and print
    python -m atkdsp_b200.autotune --write    # ... and rewrite csrc/tune_table.h

For every power-of-two nchan (16..2048), oversample (1, 2, 4) and
taps/branch in the grid, the kernel has two or three tile shapes
(include/atkdsp_gpu.h, atkdsp_gpu_tune_set): the paired fold (two hops per
thread), one hop per thread, and -- at oversample 1 or 2 with nchan <= 1024 --
the quad fold (four hops per thread); at nchan <= 512 the paired and
one-hop shapes also run with the tile window read through L1 instead of
staged in shared memory. Each is timed on one stream of 2^log2n
cf32 samples through the batched kernel (atkdsp_b200.microbench.run_one, the
kernel's own CUDA events, median of the repetitions), and the fastest goes
into the table the library compiles in (the paired fold unless another is
faster by the margin). A shape not in the grid takes the paired fold. Every
shape meets the same parity bar; only speed differs. One JSON line per shape:
{"nchan", "oversample", "taps", "paired_gsps", "single_gsps", "quad_gsps",
"paired_unstaged_gsps", "single_unstaged_gsps", "pair"} ("pair": the chosen code).
"""

from __future__ import annotations

import argparse
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent
TABLE = HERE / "csrc" / "tune_table.h"

NCHANS = (16, 32, 64, 128, 256, 512, 1024, 2048)
OVERSAMPLES = (1, 2, 4)
TAPS = (4, 8, 12, 16, 24)


def tune(nchans=NCHANS, oversamples=OVERSAMPLES, taps=TAPS, log2n: int = 22, reps: int = 5,
         margin: float = 0.01):
    from . import load
    from .microbench import run_one
    lib = load()
    rows = []
    for M in nchans:
        for os_ in oversamples:
            if M % os_:
                continue
            for K in taps:
                r = {}
                for choice in (1, 0, 2, 5, 4):
                    if lib.atkdsp_gpu_tune_set(M, os_, K, choice) != 0:
                        if choice > 1:
                            continue                     # not offered for this shape
                        raise RuntimeError(f"no tile-shape choice for nchan {M} os {os_}")
                    r[choice] = run_one(M, K, os_, log2n, reps)["gsps"]
                lib.atkdsp_gpu_tune_set(M, os_, K, -1)
                # the paired fold stays unless another shape is faster by the margin
                best = max(r, key=lambda c: r[c])
                pair = best if r[best] > r[1] * (1.0 + margin) else 1
                row = {"nchan": M, "oversample": os_, "taps": K, "paired_gsps": r[1],
                       "single_gsps": r[0], "quad_gsps": r.get(2), "paired_unstaged_gsps": r.get(5),
                       "single_unstaged_gsps": r.get(4), "pair": pair}
                print(json.dumps(row), flush=True)
                rows.append(row)
    return rows


def write_table(rows, path: Path = TABLE) -> None:
    lines = ["/* Tile-shape table: 1 = paired fold, 0 = one hop and 8 branches per thread,",
             " * 2 = quad fold (four hops per thread), +4 = tile window read through L1",
             " * rather than staged, per (nchan, oversample, taps/branch). Written by",
             " *   python -m atkdsp_b200.autotune --write",
             " * from device measurements (GS/s paired / one hop per thread / quad /",
             " * paired unstaged / one hop unstaged in each comment); shapes not listed",
             " * take the paired fold. */",
             "static const tune_entry k_tune_table[] = {"]
    for r in rows:
        q = "".join(f" / {r[k]:.2f}" if r.get(k) is not None else " / -"
                    for k in ("quad_gsps", "paired_unstaged_gsps", "single_unstaged_gsps"))
        lines.append(f"    {{{r['nchan']}, {r['oversample']}, {r['taps']}, {r['pair']}}},"
                     f"  /* {r['paired_gsps']:.2f} / {r['single_gsps']:.2f}{q} */")
    lines.append("};")
    path.write_text("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--write", action="store_true", help=f"rewrite {TABLE.name}")
    ap.add_argument("--out", default=None, help="write the table here instead")
    ap.add_argument("--log2n", type=int, default=22)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--nchans", default=None, help="comma list (default: all)")
    ap.add_argument("--oversamples", default=None, help="comma list (default: 1,2,4)")
    ap.add_argument("--taps", default=None, help="comma list (default: all)")
    a = ap.parse_args(argv)

    def lst(v, d):
        return tuple(int(t) for t in v.split(",")) if v else d
    rows = tune(lst(a.nchans, NCHANS), lst(a.oversamples, OVERSAMPLES), lst(a.taps, TAPS),
                log2n=a.log2n, reps=a.reps)
    if a.write or a.out:
        write_table(rows, Path(a.out) if a.out else TABLE)


if __name__ == "__main__":
    main()
