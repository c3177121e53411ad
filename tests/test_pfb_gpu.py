"""The filterbank on the GPU against the reference (golden fixtures), the C
oracle and the float64 twin restatement, plus the reference's own channelizer
tests (tests/test_channelizer.py of the reference) restated against this
library.

Parity bar (the tolerance the path states): per-channel error / channel RMS
<= 1e-5 against the reference. In practice the fold is bit-identical and the
double-precision FFT + rotation round to the same float almost everywhere, so
the tests also hold the path to <= 1 ulp and bit-identity for power-of-two
channel counts.
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from conftest import pfb_case_names, run_blocks
from oracle import fp64
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FS = 2.4e6
NCHAN = 192
SP = FS / NCHAN
BLOCKS = [1, 97, 960, 5000, 65537]
TOL = 1e-5


def _tone(fhz, n, seed=0, noise=0.0):
    k = np.arange(n)
    x = np.exp(2j * np.pi * fhz / FS * k)
    if noise:
        rng = np.random.default_rng(seed)
        x = x + noise * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    return x.astype(np.complex64)


def _ulps(a, b):
    ai = np.asarray(a).view(np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b).view(np.float32).view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


# ---- the reference's own outputs (golden fixtures) ---------------------------
def test_golden_cases_match_the_reference(golden_pfb):
    for name in pfb_case_names(golden_pfb):
        M, os_, K, nel, n = (int(v) for v in golden_pfb[f"{name}/params"])
        att = float(golden_pfb[f"{name}/atten"][0])
        p = ak.Pfb(FS, M, os_, K, att, nel)
        if f"{name}/cal" in golden_pfb:
            p.set_cal(golden_pfb[f"{name}/cal"], nel)
        y = run_blocks(p, list(golden_pfb[f"{name}/in"]), golden_pfb[f"{name}/pattern"])
        ref = golden_pfb[f"{name}/out"]
        assert y.shape == ref.shape, name
        err = fp64.channel_rel_error(y, ref)
        assert err["rms"] <= TOL and err["max"] <= TOL, (name, err)
        u = _ulps(y, ref)
        assert u.max() <= 1, (name, int(u.max()))
        assert np.mean(u > 0) < 1e-2, name


def test_golden_against_the_float64_twin(golden_pfb, golden_twin):
    """The error against the all-float64 specification, stated per case."""
    for key in golden_twin:
        name = key.split("/")[0]
        M, os_, K, nel, n = (int(v) for v in golden_pfb[f"{name}/params"])
        att = float(golden_pfb[f"{name}/atten"][0])
        y = run_blocks(ak.Pfb(FS, M, os_, K, att, nel), list(golden_pfb[f"{name}/in"]),
                       golden_pfb[f"{name}/pattern"])
        e_gpu = fp64.channel_rel_error(y, golden_twin[key])
        e_ref = fp64.channel_rel_error(golden_pfb[f"{name}/out"], golden_twin[key])
        # no worse than the reference's own distance from float64
        assert e_gpu["rms"] <= e_ref["rms"] * 1.01 + 1e-12, (name, e_gpu, e_ref)


@pytest.mark.parametrize("M,os_,K,nel,blocks", [
    (64, 1, 16, 1, [1, 999, 4096, 7]),
    (256, 2, 8, 1, [4097, 3, 20000]),
    (1024, 2, 12, 2, [50000, 11]),
    (2048, 1, 16, 3, [70000]),
    (4096, 2, 16, 1, [100000, 5, 33333]),
    (4096, 2, 8, 1, [65536]),
    (512, 4, 10, 1, [12345]),
    (128, 2, 3, 4, [777]),
    (32, 2, 12, 1, [100]),
    (16, 1, 4, 1, [64]),
    (8, 2, 6, 1, [50]),
    (96, 3, 10, 2, [1000, 1]),
    (1000, 2, 12, 1, [30000]),
    (6000, 2, 2, 1, [40000]),
])
def test_matches_the_oracle(M, os_, K, nel, blocks):
    rng = np.random.default_rng(M * 7 + K)
    n = M * 30 + 17
    xs = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
          for _ in range(nel)]
    y = run_blocks(ak.Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
    r = run_blocks(O.oracle().Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
    assert y.shape == r.shape
    err = fp64.channel_rel_error(y, r)
    assert err["rms"] <= TOL and err["max"] <= TOL, err
    u = _ulps(y, r)
    assert u.max() <= 1 and np.mean(u > 0) < 1e-2


# ---- restated from the reference's test_channelizer.py ------------------------
def test_centre_tone_lands_in_its_channel():
    y = ak.Pfb(FS, NCHAN).process(_tone(40 * SP, NCHAN * 120))[:, 40:-5]
    pdb = 10 * np.log10((np.abs(y) ** 2).mean(1) + 1e-20)
    assert np.argmax(pdb) == 40
    assert pdb[40] - np.sort(pdb)[-2] > 80.0


def test_edge_tone_is_not_lost():
    y = ak.Pfb(FS, NCHAN).process(_tone(40.5 * SP, NCHAN * 120))[:, 40:-5]
    pdb = 10 * np.log10((np.abs(y) ** 2).mean(1) + 1e-20)
    peak = pdb.max()
    assert pdb[40] - peak > -7 and pdb[41] - peak > -7
    assert pdb[45] - peak < -60


@pytest.mark.parametrize("blk", BLOCKS)
def test_uneven_blocks_match_the_float64_twin(blk):
    x = _tone(40 * SP, NCHAN * 80, noise=0.02, seed=3)
    orc = O.oracle()
    yt = fp64.Fp64Pfb(orc.prototype(NCHAN, 12, 80.0), NCHAN, 2).process_n([x], 1)[0]
    p = ak.Pfb(FS, NCHAN)
    outs = []
    for i in range(0, x.size, blk):
        o = p.process(x[i:i + blk])
        if o.shape[1]:
            outs.append(o)
    yc = np.concatenate(outs, axis=1)
    m = min(yc.shape[1], yt.shape[1])
    rel = np.max(np.abs(yc[:, :m] - yt[:, :m])) / np.max(np.abs(yt[:, :m]))
    assert rel < 1e-4


def test_chunk_invariance_is_exact():
    x = _tone(40 * SP, NCHAN * 80, noise=0.02, seed=4)
    y1 = ak.Pfb(FS, NCHAN).process(x)
    p = ak.Pfb(FS, NCHAN)
    outs = []
    for seg in (x[:5000], x[5000:5003], x[5003:30000], x[30000:]):
        o = p.process(seg)
        if o.shape[1]:
            outs.append(o)
    y2 = np.concatenate(outs, axis=1)
    m = min(y1.shape[1], y2.shape[1])
    assert np.array_equal(y1[:, :m], y2[:, :m])


def test_streaming_continuity_1_999_4096_7():
    """Blocks of 1, 999, 4096, 7, ... equal one unbroken call (bit for bit)."""
    rng = np.random.default_rng(8)
    x = (rng.standard_normal(200000) + 1j * rng.standard_normal(200000)).astype(np.complex64)
    for M, os_, K in ((64, 1, 16), (1024, 2, 12), (4096, 2, 16)):
        whole = ak.Pfb(FS, M, os_, K).process(x)
        parts = run_blocks(ak.Pfb(FS, M, os_, K), [x], [1, 999, 4096, 7])[0]
        assert np.array_equal(whole, parts), M


def test_elements_are_bit_identical_on_identical_input():
    base = _tone(40 * SP, NCHAN * 80, noise=0.03, seed=5)
    o = ak.Pfb(FS, NCHAN, max_nel=5).process_n([base] * 5, 5)
    assert all(np.array_equal(o[0], o[e]) for e in range(5))


def test_plane_wave_phase_within_tenth_degree():
    phi = np.deg2rad(37.0)
    base = _tone(40 * SP, NCHAN * 200)
    ins = [base * np.exp(1j * e * phi) for e in range(5)]
    o = ak.Pfb(FS, NCHAN, max_nel=5).process_n(ins, 5)[:, 40, 60:-5]
    rel = np.angle(o.mean(1)); rel = rel - rel[0]
    planted = np.array([e * phi for e in range(5)])
    err = np.rad2deg(np.max(np.abs(np.angle(np.exp(1j * (rel - planted))))))
    assert err < 0.1


def test_true_baseband_at_any_oversampling():
    """A tone df above channel k's centre comes out of bin k at +df, at 2x, 3x
    and 4x (reference test_channelizer.py:296-319)."""
    for os_ in (2, 3, 4):
        M = 96
        sp = FS / M
        df = 0.13 * sp
        y = ak.Pfb(FS, M, os_).process(_tone(10 * sp + df, M * 300))[10, 40:]
        rate = os_ * sp
        ph = np.unwrap(np.angle(y))
        f_est = np.polyfit(np.arange(ph.size) / rate, ph, 1)[0] / (2 * np.pi)
        assert abs(f_est - df) < 1e-3 * sp, (os_, f_est, df)


def test_out_rate_and_bookkeeping():
    p = ak.Pfb(FS, NCHAN, oversample=2)
    assert abs(p.out_rate() - 2 * SP) < 1e-6
    assert abs(p.group_delay() - (NCHAN * 12 - 1) / 2.0) < 1e-6
    assert p.block_origin(0) == -(NCHAN * 12 - NCHAN // 2)
    assert "192 chan x2 oversample" in p.describe()


def test_set_cal_applies_once():
    base = _tone(40 * SP, NCHAN * 40, noise=0.02, seed=9)
    y0 = ak.Pfb(FS, NCHAN, max_nel=2).process_n([base, base], 2)
    p1 = ak.Pfb(FS, NCHAN, max_nel=2)
    cal = np.ones((2, NCHAN), np.complex64)
    cal[1, :] = np.exp(1j * np.deg2rad(90.0))
    p1.set_cal(cal, 2)
    y1 = p1.process_n([base, base], 2)
    assert np.allclose(y1[0], y0[0], atol=1e-5)
    assert np.allclose(y1[1], y0[1] * np.exp(1j * np.deg2rad(90.0)), atol=1e-4)
    p1.set_cal(None, 0)
    p1.reset()
    assert np.array_equal(p1.process_n([base, base], 2), y0)


@pytest.mark.parametrize("nchan,os_,nel", [(24, 2, 1), (200, 2, 1), (64, 4, 1), (60, 3, 2), (192, 2, 5)])
def test_identical_at_any_split(nchan, os_, nel):
    rng = np.random.default_rng(nchan + nel)
    n = nchan * 300 + 17
    xs = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64) for _ in range(nel)]
    whole = np.asarray(ak.Pfb(FS, nchan, os_, max_nel=nel).process_n(xs, nel))
    p = ak.Pfb(FS, nchan, os_, max_nel=nel)
    parts, pos = [], 0
    for b in (5, nchan * 7 + 3, 1, n):
        o = np.asarray(p.process_n([x[pos:pos + b] for x in xs], nel))
        if o.shape[-1]:
            parts.append(o)
        pos += b
        if pos >= n:
            break
    split = np.concatenate(parts, axis=-1)
    m = min(whole.shape[-1], split.shape[-1])
    assert np.array_equal(whole[..., :m], split[..., :m])
    f = fp64.Fp64Pfb(O.oracle().prototype(nchan, 12, 80.0), nchan, os_, nel)
    yt = f.process_n(xs, nel)
    m = min(m, yt.shape[-1])
    rel = np.max(np.abs(whole[..., :m] - yt[..., :m])) / np.max(np.abs(yt[..., :m]))
    assert rel < 5e-7, rel


@pytest.mark.parametrize("nchan", [1024, 1026, 2048])
def test_long_transforms_match_the_twin(nchan):
    rng = np.random.default_rng(nchan)
    x = (rng.standard_normal(nchan * 40) + 1j * rng.standard_normal(nchan * 40)).astype(np.complex64)
    yc = ak.Pfb(FS, nchan).process(x)
    yt = fp64.Fp64Pfb(O.oracle().prototype(nchan, 12, 80.0), nchan, 2).process_n([x], 1)[0]
    m = min(yc.shape[1], yt.shape[1])
    assert np.max(np.abs(yc[:, :m] - yt[:, :m])) / np.max(np.abs(yt[:, :m])) < 5e-7


# ---- the drop-in contract's edge cases -----------------------------------------
def test_short_calls_stash_and_return_zero():
    lib = ak.load()
    p = ak.Pfb(FS, 64, 2, 12)
    x = _tone(3 * FS / 64, 200, noise=0.1, seed=1)
    # 31 < hop: m == 0, out may be NULL and is not touched
    got = lib.atkdsp_pfb_process(p.handle, ak._cfp(x[:31]), 31, None, 0)
    assert got == 0
    rest = p.process(x[31:])
    whole = ak.Pfb(FS, 64, 2, 12).process(x)
    assert np.array_equal(rest, whole)


def test_cap_too_small_is_refused_with_state_untouched():
    lib = ak.load()
    p = ak.Pfb(FS, 64, 2, 12)
    x = _tone(3 * FS / 64, 5000, noise=0.1, seed=2)
    m = p.out_hops(x.size)
    out = np.zeros(64 * m, np.complex64)
    assert lib.atkdsp_pfb_process(p.handle, ak._cfp(x), x.size, ak._cfp(out), 64 * m - 1) == -3
    assert lib.atkdsp_pfb_process(p.handle, ak._cfp(x), x.size, None, 64 * m) == -3
    assert np.array_equal(p.process(x), ak.Pfb(FS, 64, 2, 12).process(x))


def test_bad_arguments():
    lib = ak.load()
    p = ak.Pfb(FS, 64, 2, 12, max_nel=2)
    with pytest.raises(ak.AtkDspError):
        p.process_n([np.zeros(100, np.complex64)] * 3, 3)
    assert lib.atkdsp_pfb_process_n(None, None, 1, 0, None, 0) == -1
    assert lib.atkdsp_pfb_set_cal(p.handle, ak._cfp(np.zeros(64 * 3, np.complex64)), 3) == -1
    assert lib.atkdsp_pfb_out_hops(None, 100) == 0 and lib.atkdsp_pfb_nchan(None) == 0


def test_long_input_spans_several_device_chunks():
    """A call longer than the handle's device staging chunk is processed in
    pieces; it must equal the same input fed in short blocks (bit for bit, the
    same kernels) and the oracle's single call (within the parity bar; two
    different double-precision FFTs round a handful of values differently)."""
    rng = np.random.default_rng(77)
    n = 5_000_000
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    y = ak.Pfb(FS, 256, 2, 8).process(x)
    yb = run_blocks(ak.Pfb(FS, 256, 2, 8), [x], [300_001, 17, 1_000_000])[0]
    assert np.array_equal(y, yb)
    r = O.oracle().Pfb(FS, 256, 2, 8).process(x)
    assert y.shape == r.shape
    err = fp64.channel_rel_error(y, r)
    assert err["rms"] <= 1e-7 and err["max"] <= 1e-6, err
    assert np.mean(y != r) < 1e-4
