"""Pin the CPU oracle before trusting it (CPU only).

The oracle (oracle/pfb_oracle.c, loaded through oracle/oracle.py) is checked
against the golden fixtures, which the reference produced itself
(tests/golden/make_golden.py: the reference's C library built from its own
sources, and its numpy twin). Where the reference library is built here
(oracle/_ref), it is also compared directly on fresh inputs.

Bars: unpack / DC pole / W1 / W2 bit-exact; filterbank outputs bit-exact
except for rare last-bit differences (the reference's FFT is pocketfft, the
oracle's is its own double-precision transform; both round a double result
to float once), which must stay under 1 ulp and a tiny fraction of values.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import pfb_case_names, run_blocks
from oracle import fp64
from oracle import oracle as O

FS = 2.4e6


def _orc():
    return O.oracle()


def _ulp_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ai = a.view(np.float32).view(np.int32).astype(np.int64)
    bi = b.view(np.float32).view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


def test_pfb_oracle_matches_reference_golden(golden_pfb):
    orc = _orc()
    for name in pfb_case_names(golden_pfb):
        M, os_, K, nel, n = (int(v) for v in golden_pfb[f"{name}/params"])
        att = float(golden_pfb[f"{name}/atten"][0])
        p = orc.Pfb(FS, M, os_, K, att, nel)
        if f"{name}/cal" in golden_pfb:
            p.set_cal(golden_pfb[f"{name}/cal"], nel)
        xs = list(golden_pfb[f"{name}/in"])
        y = run_blocks(p, xs, golden_pfb[f"{name}/pattern"])
        ref = golden_pfb[f"{name}/out"]
        assert y.shape == ref.shape, name
        ulps = _ulp_diff(y, ref)
        # a last-bit difference only where the two double FFTs straddle a
        # float rounding boundary (seen with radix-3/5 factors: nchan 24, 60,
        # 192, 200); power-of-two sizes come out bit-identical
        assert ulps.max() <= 1, (name, int(ulps.max()))
        assert np.mean(ulps > 0) < 1e-2, (name, float(np.mean(ulps > 0)))
        if M & (M - 1) == 0:
            assert ulps.max() == 0, name


def test_w12_oracle_bit_exact(golden_w12):
    orc = _orc()
    g = golden_w12
    y = g["y"]
    nel, M = y.shape[0], y.shape[1]
    R, c = g["R0"].copy(), g["c0"].copy()
    orc.pfb_cov_accumulate(y, nel, M, None, R, c)
    assert np.array_equal(R.view(np.uint32), g["R"].view(np.uint32))
    assert np.array_equal(c, g["counts"])
    Rg, cg = g["R0"].copy(), g["c0"].copy()
    orc.pfb_cov_accumulate(y, nel, M, g["gate"], Rg, cg)
    assert np.array_equal(Rg.view(np.uint32), g["Rg"].view(np.uint32))
    assert np.array_equal(cg, g["cg"])
    orc.pfb_cov_reset(Rg, cg, nel, M, g["gate"])
    assert np.array_equal(Rg.view(np.uint32), g["Rr"].view(np.uint32))
    assert np.array_equal(cg, g["cr"])
    pwr, meanp = orc.pfb_channel_power(y, nel, M)
    assert np.array_equal(pwr.view(np.uint32), g["pwr"].view(np.uint32))
    assert np.array_equal(meanp.view(np.uint32), g["meanp"].view(np.uint32))


@pytest.mark.parametrize("fmt", ["cu8", "ci8", "ci16", "ci16q11", "cf32"])
def test_unpack_oracle_bit_exact(golden_unpack, fmt):
    orc = _orc()
    g = golden_unpack
    raw = g[f"{fmt}/raw"].tobytes()
    assert np.array_equal(orc.unpack(raw, fmt).view(np.uint32), g[f"{fmt}/plain"].view(np.uint32))
    for j in range(3):
        off = complex(*g[f"{fmt}/off{j}"].astype(np.float64))
        y, mean = orc.unpack_dc(raw, fmt, off)
        assert np.array_equal(y.view(np.uint32), g[f"{fmt}/dc{j}"].view(np.uint32)), (fmt, j)
        assert mean.real == g[f"{fmt}/mean{j}"][0] and mean.imag == g[f"{fmt}/mean{j}"][1]
    st = np.zeros(1, np.complex64)
    bps = orc.bytes_per_sample(fmt)
    cuts = [0, 40 * bps, 40 * bps + bps, len(raw)]
    ys = [orc.unpack(raw[a:b], fmt, 0.01, st) for a, b in zip(cuts[:-1], cuts[1:])]
    assert np.array_equal(np.concatenate(ys).view(np.uint32), g[f"{fmt}/pole"].view(np.uint32))
    assert np.array_equal(st.view(np.uint32), g[f"{fmt}/pole_state"].view(np.uint32))


def test_prototype_matches_twin(golden_proto):
    orc = _orc()
    i = 0
    while f"h{i}" in golden_proto:
        M, K, att = golden_proto[f"params{i}"]
        h = orc.prototype(int(M), int(K), float(att))
        assert np.array_equal(h, golden_proto[f"h{i}"]), i
        t = golden_proto[f"twin{i}"]
        assert np.max(np.abs(h - t)) / np.max(np.abs(t)) < 1e-13
        assert np.array_equal(h.astype(np.float32), t.astype(np.float32))
        i += 1
    assert i >= 4


def test_fp64_oracle_matches_twin(golden_pfb, golden_twin):
    orc = _orc()
    for key in golden_twin:
        name = key.split("/")[0]
        M, os_, K, nel, n = (int(v) for v in golden_pfb[f"{name}/params"])
        att = float(golden_pfb[f"{name}/atten"][0])
        f = fp64.Fp64Pfb(orc.prototype(M, K, att), M, os_, nel)
        xs = [x.astype(np.complex128) for x in golden_pfb[f"{name}/in"]]
        y = run_blocks(f, xs, golden_pfb[f"{name}/pattern"])
        t = golden_twin[key]
        assert y.shape == t.shape
        err = fp64.channel_rel_error(y, t)
        assert err["max"] < 1e-9, (name, err)


def test_oracle_against_reference_library_directly():
    ref = O.reference()
    if ref is None:
        pytest.skip("reference library not built here (oracle/_ref)")
    orc = _orc()
    rng = np.random.default_rng(99)
    for M, os_, K, nel, blocks in [(256, 2, 8, 1, [3000, 1, 777]), (96, 3, 10, 3, [500]),
                                   (2048, 2, 16, 1, [70000])]:
        n = M * 40 + 13
        xs = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
              for _ in range(nel)]
        a = run_blocks(orc.Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
        b = run_blocks(ref.Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
        u = _ulp_diff(a, b)
        assert u.max() <= 1 and np.mean(u > 0) < 1e-2


# ---- the overlap-save extractor (oracle/osx_oracle.c) ----------------------
def _osx_max_rel(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| over the slot's largest reference magnitude"""
    return float(np.max(np.abs(a - b), initial=0.0) / (np.max(np.abs(b), initial=0.0) + 1e-30))


@pytest.mark.parametrize("name", sorted(__import__("osx_cases").OSX_CASES))
def test_osx_oracle_matches_reference_golden(golden_osx, name):
    """Every slot's output, same length; bit-identical where the two FFTs
    round alike, and within 1e-5 of the slot's peak everywhere."""
    from osx_cases import run_case
    xs = list(golden_osx[f"{name}/in"])
    ys, _ = run_case(lambda fs, nfft, nel: _orc().Osx(fs, nfft, 80.0, nel), name, xs)
    want = sorted(int(k.split("/out")[1]) for k in golden_osx if k.startswith(f"{name}/out"))
    assert sorted(ys) == want
    for ci in want:
        g = golden_osx[f"{name}/out{ci}"]
        assert ys[ci].shape == g.shape
        assert _osx_max_rel(ys[ci], g) < 1e-5, (name, ci)


def test_osx_oracle_bookkeeping_matches_reference_semantics():
    orc = _orc()
    assert orc.lib.orc_osx_create(FS, 100, 80.0, 1) is None       # not a power of two
    assert orc.lib.orc_osx_create(FS, 32, 80.0, 1) is None        # below 64
    assert orc.lib.orc_osx_create(0.0, 4096, 80.0, 1) is None
    o = orc.Osx(FS, 4096)
    assert o.add(300e3, 50e3, 50e3) == 0
    assert o.add(-300e3, 50e3, 75e3) == 1
    assert o.chan_rate(0) == 50e3 and o.chan_rate(1) == 75e3
    assert o.out_max(0, 240000) == 5000 + 64
    o.remove(0)
    assert o.chan_rate(0) == 0.0 and o.channels() == 2
    assert o.add(100e3, 50e3, 50e3) == 0                          # the hole is reused
    with pytest.raises(RuntimeError):
        o.add(0.0, -1.0, 50e3)
    with pytest.raises(RuntimeError):
        o.retune(5, 0.0)
    assert "2 channel(s)" in o.describe()


# ---- the spectrum reduction (oracle/spectrum_oracle.c) -------------------------
def test_spectrum_oracle_matches_reference_golden(golden_spectrum):
    from conftest import spectrum_case_names
    orc = _orc()
    kinds = {-1: None, 0: "rect", 1: "hann", 2: "hamming", 3: "blackmanharris"}
    for name in spectrum_case_names(golden_spectrum):
        n, hop, kind, det, frames = (int(v) for v in golden_spectrum[f"{name}/params"])
        x = golden_spectrum[f"{name}/in"]
        w = None if kinds[kind] is None else orc.window(kinds[kind], n)
        line, fr = orc.spectrum_reduce(x, n, hop, w, det)
        assert fr == frames
        assert np.array_equal(line, golden_spectrum[f"{name}/line"]), name
        st = orc.spectrum_stats(x, n, hop, w)
        for q in ("max", "avg", "min", "sk"):
            assert np.array_equal(st[q], golden_spectrum[f"{name}/{q}"]), (name, q)


# -- CFAR ---------------------------------------------------------------------

def test_cfar_solver_bit_exact_against_the_reference(golden_cfar):
    """The threshold solver is host code of the product (no GPU needed):
    alpha and E[T] over 1200 configurations of (mode, n_ref, pfa, looks, OS
    rank, window correlation) come out as the reference's numbers, bit for
    bit, and the refusals are the reference's."""
    import atkdsp_b200 as ak
    grid, res, rhos = golden_cfar["alpha/grid"], golden_cfar["alpha/res"], golden_cfar["alpha/rho"]
    for (mode, nref, pfa, looks, os_k, ri), (rc, a, et) in zip(grid, res):
        rho = None if ri == 0 else tuple(rhos[int(ri)])
        try:
            got = ak.cfar_alpha(int(mode), int(nref), pfa, looks, int(os_k), rho)
        except ak.AtkDspError:
            assert rc != 0, (mode, nref, pfa, looks, os_k, ri)
            continue
        assert rc == 0 and got == (a, et), (mode, nref, pfa, looks, os_k, ri, got, a, et)


def test_cfar_n_eff_and_window_correlation_bit_exact(golden_cfar):
    import atkdsp_b200 as ak
    rhos = golden_cfar["alpha/rho"]
    for nref, ri, v in golden_cfar["n_eff"]:
        rho = None if ri == 0 else tuple(rhos[int(ri)])
        assert ak.cfar_n_eff(int(nref), rho) == v
    for key in golden_cfar:
        if key.startswith("rho2/"):
            _, kind, n = key.split("/")
            w = O.oracle().window(kind, int(n))
            assert ak.cfar_window_rho2(w) == tuple(golden_cfar[key]), key


def test_cfar_cell_oracle_matches_reference_last_frames(golden_cfar):
    """The numpy restatement of the per-cell test, pinned to the reference's
    last tested frame of every case: averaged power and threshold in dB as
    the reference rounds them to float, and the hit mask."""
    import cfar_cases
    from oracle import cfar_oracle as CO
    for name in cfar_cases.CFAR_CASES:
        xs = golden_cfar[f"{name}/in"]
        a, ac, _et = golden_cfar[f"{name}/alpha"]
        X, thr, hits = CO.cell_test(xs, cfar_cases.cfg_of(name), a, ac, cfar_cases.mask_of(name))
        with np.errstate(divide="ignore", invalid="ignore"):
            avg = (10.0 * np.log10(X[-1])).astype(np.float32)
            tdb = (10.0 * np.log10(thr[-1])).astype(np.float32)
        ref_avg, ref_thr = golden_cfar[f"{name}/last_avg"], golden_cfar[f"{name}/last_thr"]
        assert np.array_equal(hits[-1], golden_cfar[f"{name}/last_hits"]), name
        fin = np.isfinite(ref_avg)
        assert np.array_equal(np.isfinite(avg), fin), name
        assert np.max(np.abs(avg[fin] - ref_avg[fin]), initial=0.0) <= 1e-5, name
        fin = np.isfinite(ref_thr)
        assert np.array_equal(np.isfinite(tdb), fin), name
        assert np.max(np.abs(tdb[fin] - ref_thr[fin]), initial=0.0) <= 1e-5, name
        st = dict(zip(sorted(["frames", "warmup", "cells_tested", "cell_hits", "untestable", "opened", "closed",
                              "updates", "dropped", "resets", "tracks"]), golden_cfar[f"{name}/stats"]))
        assert int(hits.sum()) == int(st["cell_hits"]), name
