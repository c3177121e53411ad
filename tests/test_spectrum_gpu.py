"""The device spectrum reduction against the reference (golden fixtures from
its C library, one thread) and the C oracle.

Bars: every line within 1e-4 dB of the reference (kurtosis: 1e-5
relative), frame counts exact. The max and min detectors are order-free
reductions, so their linear powers match wherever the transforms round
alike; the dB values can still differ in the last bit, because the device
log10f is within 2 ulp where glibc's is within 1, so at least half of those
lines' values must be bit-identical. The average detector and the stats'
sums add per CTA and then across CTAs, a different rounding sequence from
one thread's.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import spectrum_case_names
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KINDS = {-1: None, 0: "rect", 1: "hann", 2: "hamming", 3: "blackmanharris"}


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_golden_cases_match_the_reference(golden_spectrum):
    from atkdsp_b200.gpu import Spectrum
    for name in spectrum_case_names(golden_spectrum):
        n, hop, kind, det, frames = (int(v) for v in golden_spectrum[f"{name}/params"])
        x = golden_spectrum[f"{name}/in"]
        w = None if KINDS[kind] is None else O.oracle().window(KINDS[kind], n)
        sp = Spectrum(n)
        line, fr = sp.reduce(_t(x), hop, None if w is None else _t(w), det)
        assert fr == frames, name
        ref = golden_spectrum[f"{name}/line"]
        got = line.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-4, (name, float(np.max(np.abs(got - ref))))
        if det != 2:
            assert np.mean(got == ref) >= 0.5, name
        st = sp.stats(_t(x), hop, None if w is None else _t(w))
        assert st["frames"] == frames
        for q in ("max", "avg", "min"):
            g = st[q].cpu().numpy()
            assert np.max(np.abs(g - golden_spectrum[f"{name}/{q}"])) <= 1e-4, (name, q)
        sk, skr = st["sk"].cpu().numpy(), golden_spectrum[f"{name}/sk"]
        assert np.max(np.abs(sk - skr) / np.abs(skr)) <= 1e-5, name


@pytest.mark.parametrize("n,hop,win,det", [(4096, 2048, "hann", "avg"), (1024, 1000, None, "max"),
                                           (256, 64, "blackmanharris", "min"), (16, 16, "hamming", "avg")])
def test_long_blocks_match_the_oracle(n, hop, win, det):
    """Enough frames that many CTAs each merge a partial line."""
    from atkdsp_b200.gpu import Spectrum
    rng = np.random.default_rng(n + hop)
    N = 1 << 20
    k = np.arange(N)
    x = ((rng.standard_normal(N) + 1j * rng.standard_normal(N)) * 0.1
         + np.exp(2j * np.pi * 0.0731 * k) + 0.01 * np.exp(-2j * np.pi * 0.3 * k)).astype(np.complex64)
    w = None if win is None else O.oracle().window(win, n)
    line, fr = Spectrum(n).reduce(_t(x), hop, None if w is None else _t(w), det)
    ref, frr = O.oracle().spectrum_reduce(x, n, hop, w, det)
    assert fr == frr == (N - n) // hop + 1
    assert np.max(np.abs(line.cpu().numpy() - ref)) <= 1e-4
    st = Spectrum(n).stats(_t(x), hop, None if w is None else _t(w), want=("avg", "sk"))
    so = O.oracle().spectrum_stats(x, n, hop, w)
    assert set(st) == {"avg", "sk", "frames"}
    assert np.max(np.abs(st["avg"].cpu().numpy() - so["avg"])) <= 1e-4
    assert np.max(np.abs(st["sk"].cpu().numpy() - so["sk"]) / so["sk"]) <= 1e-5


def test_argument_rules():
    import torch
    import atkdsp_b200 as ak
    from atkdsp_b200.gpu import Spectrum
    lib = ak.load()
    for n in (8, 100, 8192):
        assert not lib.atkdsp_gpu_spectrum_create(n)
    sp = Spectrum(64)
    x = torch.zeros(200, dtype=torch.complex64, device="cuda")
    assert sp.reduce(x[:63])[1] == 0                       # shorter than one frame
    assert sp.reduce(x, hop=0)[1] == 3                     # hop 0 -> n
    assert sp.reduce(x, hop=1000)[1] == 3                  # hop > n -> n
    assert sp.reduce(x, hop=10)[1] == (200 - 64) // 10 + 1
    line, _ = sp.reduce(x)                                 # silence reads -240 dB
    assert float(torch.max(torch.abs(line + 240.0))) < 1e-3
    with pytest.raises(ak.AtkDspError):
        sp.reduce(x, detector=7)
    with pytest.raises(ak.AtkDspError):
        sp.stats(x, want=())
