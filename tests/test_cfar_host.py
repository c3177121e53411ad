"""The CFAR's host logic without a GPU (CPU only).

atkdsp_b200/csrc/cfar_host.c (solver, tables, the pass pipeline, the choice
of columns, the tracker) is compiled here against tests/cfar_emu/shim_emu.c,
a plain-C stand-in for the device shim and the four CFAR kernels. The result
runs the golden cases to the reference's events exactly (the stand-in's exp
is glibc's, as the reference's is). A checked build traps any tracker read
outside the pass's columns. Where the reference library is built
(oracle/_ref), random configurations are compared with it over many passes.
"""

from __future__ import annotations

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cfar_cases
from conftest import ROOT
from oracle import oracle as O

SRC = ROOT / "atkdsp_b200" / "csrc" / "cfar_host.c"
EMU = Path(__file__).resolve().parent / "cfar_emu" / "shim_emu.c"
STAT_KEYS = sorted(["frames", "warmup", "cells_tested", "cell_hits", "untestable", "opened", "closed", "updates",
                    "dropped", "resets", "tracks"])

CHECK_PRELUDE = """#include <stdlib.h>
static inline int32_t chk_col(const int32_t *cm, long b) { if (cm[b] < 0) abort(); return cm[b]; }
"""


class _Lib:
    def __init__(self, path):
        self.lib = C.CDLL(str(path))


def _build(tmp: Path, checked: bool) -> _Lib:
    gcc = shutil.which("gcc", path="/usr/bin") or "gcc"
    src = SRC
    if checked:
        text = SRC.read_text()
        text = re.sub(r"cm\[(b|pk)\]", r"chk_col(cm, (long)(\1))", text)
        text = text.replace('#include "host_internal.h"', '#include "host_internal.h"\n' + CHECK_PRELUDE, 1)
        src = tmp / "cfar_host_checked.c"
        src.write_text(text)
    out = tmp / ("libcfar_emu_chk.so" if checked else "libcfar_emu.so")
    subprocess.run([gcc, "-std=c99", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-DATKDSP_BUILD=1",
                    f"-I{ROOT / 'include'}", f"-I{ROOT / 'atkdsp_b200' / 'csrc'}", str(src), str(EMU),
                    "-o", str(out), "-lm", "-lpthread"], check=True)
    return _Lib(out)


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    return _build(tmp_path_factory.mktemp("cfar_emu"), checked=True)


def _arr(events) -> np.ndarray:
    keys = cfar_cases.EVENT_KEYS
    return np.array([[e[k] for k in keys] for e in events], np.float64).reshape(-1, len(keys))


@pytest.mark.parametrize("name", sorted(cfar_cases.CFAR_CASES))
def test_host_logic_reproduces_the_reference_events(emu, golden_cfar, name):
    ev, last, st, desc, al = cfar_cases.run_case(lambda nb, **cfg: O.RefCfar(emu, nb, **cfg), name,
                                                 golden_cfar[f"{name}/in"])
    assert np.array_equal(ev, golden_cfar[f"{name}/events"], equal_nan=True), name
    assert [st[k] for k in STAT_KEYS] == [int(v) for v in golden_cfar[f"{name}/stats"]], name
    assert desc == str(golden_cfar[f"{name}/describe"]), name
    assert al == tuple(golden_cfar[f"{name}/alpha"]), name
    assert np.array_equal(last[2], golden_cfar[f"{name}/last_hits"]), name
    for got, key in ((last[0], "last_avg"), (last[1], "last_thr")):
        assert np.array_equal(got, golden_cfar[f"{name}/{key}"], equal_nan=True), (name, key)


def _frames(rng, nb, nf):
    floor = rng.exponential(1.0, size=(nf, nb)) * np.linspace(1.0, 3.0, nb)[None, :]
    for _ in range(int(rng.integers(1, 60))):
        w = int(rng.integers(1, 40))
        lo, f0 = int(rng.integers(0, nb - w)), int(rng.integers(0, nf))
        dr = int(rng.integers(-2, 3))
        for f in range(f0, min(nf, f0 + int(rng.integers(1, 150)))):
            a = min(max(lo + dr * (f - f0), 0), nb - w)
            floor[f, a:a + w] += 10 ** rng.uniform(0.5, 3)
    return (10.0 * np.log10(floor)).astype(np.float32)


@pytest.mark.skipif(O.reference() is None, reason="reference library not built")
def test_many_passes_and_random_configurations_against_the_reference(emu):
    """Passes of 2^20 cells: 70,000 bins make 14-frame passes, so tracks,
    k-frame windows and the column sets cross many pass boundaries; calls of
    random length split them again."""
    rng = np.random.default_rng(2027)
    done = 0
    while done < 40:
        nb = int(rng.choice([300, 5000, 70000]))
        nf = int(rng.integers(5, 120 if nb < 20000 else 40))
        cfg = dict(mode=int(rng.integers(0, 4)), n_ref=int(rng.integers(1, 24)), n_guard=int(rng.integers(0, 6)),
                   k_frames=int(rng.choice([1, 2, 3, 5, 8])), pfa=float(10 ** rng.uniform(-8, -1.5)),
                   merge_gap=int(rng.integers(0, 12)), min_bins=int(rng.integers(1, 4)),
                   open_n=int(rng.integers(1, 6)), close_k=int(rng.choice([1, 3, 50, 400])),
                   max_tracks=int(rng.choice([4, 64, 256])))
        cfg["open_m"] = int(rng.integers(1, cfg["open_n"] + 1))
        if cfg["mode"] == 1:
            cfg["os_k"] = int(rng.integers(0, 2 * cfg["n_ref"] + 1))
        xs = _frames(rng, nb, nf)
        try:
            a, b = O.RefCfar(emu, nb, **cfg), O.RefCfar(O.reference(), nb, **cfg)
        except ValueError:
            continue
        if rng.uniform() < 0.3:
            mask = (rng.uniform(size=nb) < 0.05).astype(np.uint8)
            a.set_mask(mask)
            b.set_mask(mask)
        pos, ea, eb = 0, [], []
        while pos < nf:
            x = xs[pos:pos + int(rng.integers(1, nf + 1))]
            ea += a.process(x, 1.0 + pos * 0.01, 0.01)
            eb += b.process(x, 1.0 + pos * 0.01, 0.01)
            pos += len(x)
        ea += a.flush()
        eb += b.flush()
        assert np.array_equal(_arr(ea), _arr(eb), equal_nan=True), (nb, nf, cfg)
        assert a.stats() == b.stats(), (nb, nf, cfg)
        la, lb = a.last(), b.last()
        assert (la is None) == (lb is None)
        if la is not None:
            for p, q in zip(la, lb):
                assert np.array_equal(p, q, equal_nan=True), (nb, nf, cfg)
        done += 1
