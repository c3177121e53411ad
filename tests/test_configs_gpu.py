"""Parity at the benchmark's own configurations, against the reference library.

Each test runs one workload configuration at its real shape through this
library and through the reference's C library (oracle/_ref, built from the
reference's sources), on the same seeded inputs, and checks the parity bar:
every channel's RMS error and largest single error within 1e-5 of that
channel's RMS. The float64 restatement of the filterbank (oracle/fp64.py,
after python/atkdsp/reference.py:11481-11581) is run on a prefix of each
input, and the path's distance from it is held to the reference's own
(the FP64 error is stated for every configuration). Model:
tests/test_channelizer.py:74-89, 367-398 of the reference.

  single stream  M=64, 1x, 16 taps, beta 8, 2^20 samples in blocks
                 1, 999, 4096, 7 (the drop-in host API)
  front end      ci16q11 2,000,000-sample blocks, unpack_dc with the running
                 DC estimate, M=1024, 2x, 12 taps, W1 and W2
  coherent       8 elements x 2^18 samples, M=2048, 1x, 16 taps, beta 8,
                 W1 (8x8) and W2
  uneven         the 256-stream workload's streams, one of every (nchan,
                 taps) pair (nchan 4096 with 12 and 16 taps among them), three
                 successive blocks through a graph-replayed batch
  served         served streams' 1.6 ms ci16 blocks at nchan 256 and 1024,
                 16 taps, through the server

plus NaN samples ("unmeasured") through the filterbank and W1/W2: the same
outputs go NaN as in the reference, and the others keep the parity bar.
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from atkdsp_b200 import workloads as W
from conftest import run_blocks
from oracle import fp64
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FS = 2.4e6
TOL = 1e-5


@pytest.fixture(scope="module")
def ref():
    r = O.reference()
    if r is None:
        pytest.skip("the reference library (oracle/_ref) is not built")
    return r


def _parity(y, r, what):
    assert y.shape == r.shape, (what, y.shape, r.shape)
    e = fp64.channel_rel_error(y, r)
    assert e["rms"] <= TOL and e["max"] <= TOL, (what, e)
    return e


def _fp64_holds(y, r, nchan, os_, taps, atten, xs, what, slack=1.1):
    """The float64 filterbank over xs (element arrays, a prefix of the input);
    the path's worst channel is no further from it than the reference's."""
    t = fp64.Fp64Pfb(O.oracle().prototype(nchan, taps, atten), nchan, os_, len(xs))
    y64 = t.process_n(xs, len(xs))
    m = y64.shape[-1]
    ours = fp64.channel_rel_error(np.asarray(y)[..., :m].reshape(y64.shape), y64)
    theirs = fp64.channel_rel_error(np.asarray(r)[..., :m].reshape(y64.shape), y64)
    assert ours["rms"] <= theirs["rms"] * slack + 1e-12, (what, ours, theirs)
    return ours, theirs


def test_single_stream_config(ref):
    x = W.single_stream(1 << 20)
    blocks = list(W.SINGLE_STREAM_BLOCKS)
    y = run_blocks(ak.Pfb(FS, 64, 1, 16, W.ATTEN_BETA8, 1), [x], blocks)
    r = run_blocks(ref.Pfb(FS, 64, 1, 16, W.ATTEN_BETA8, 1), [x], blocks)
    _parity(y, r, "single stream")
    _fp64_holds(y, r, 64, 1, 16, W.ATTEN_BETA8, [x[: 1 << 17]], "single stream")


def test_front_end_config(ref):
    blk = 2_000_000
    raw = W.front_end_raw(3 * blk)
    p = ak.Pfb(FS, 1024, 2, 12, 80.0, 1)
    rp = ref.Pfb(FS, 1024, 2, 12, 80.0, 1)
    R, c = np.zeros((1024, 1, 1), np.complex64), np.zeros(1024, np.uint32)
    Rr, cr = np.zeros((1024, 1, 1), np.complex64), np.zeros(1024, np.uint32)
    from atkdsp_b200 import gpu
    pf = ak.Pfb(FS, 1024, 2, 12, 80.0, 1)
    off = 0j
    ours = []
    for b in range(3):
        rb = raw[b * blk:(b + 1) * blk].tobytes()
        x, mean = ak.unpack_dc(rb, "ci16q11", off)
        xr, mean_r = ref.unpack_dc(rb, "ci16q11", off)
        assert np.array_equal(x.view(np.uint32), xr.view(np.uint32)), b
        assert abs(mean - mean_r) <= 1e-12 * max(1.0, abs(mean_r)), b
        # the fused int16 path on the device equals unpack_dc then the filterbank
        d = torch.from_numpy(raw[b * blk:(b + 1) * blk].reshape(-1).copy()).cuda()
        yf = gpu.process_n_raw(pf, [d], 1, "ci16q11", off)
        torch.cuda.synchronize()
        y = np.asarray(p.process(x))
        r = np.asarray(rp.process(xr))
        assert np.array_equal(yf.cpu().numpy()[0], y), b
        _parity(y, r, f"front end block {b}")
        ours.append(y[None])
        ak.pfb_cov_accumulate(y[None], 1, 1024, None, R, c)
        ref.pfb_cov_accumulate(r[None], 1, 1024, None, Rr, cr)
        pw, mp = ak.pfb_channel_power(y[None], 1, 1024)
        pwr, mpr = ref.pfb_channel_power(r[None], 1, 1024)
        assert np.max(np.abs(pw - pwr) / pwr) <= TOL, b
        assert np.max(np.abs(mp - mpr) / mpr) <= TOL, b
        if b == 0:
            _fp64_holds(y[None], r[None], 1024, 2, 12, 80.0, [x[: 1 << 18]], "front end")
        off = complex(np.float32(mean.real), np.float32(mean.imag))
    exact = _w1_exact(ours)
    assert np.array_equal(c, cr)
    _w1_holds(R, Rr, exact, "front end")


def _w1_exact(ys):
    """W1 of a list of (nel, nchan, m) blocks summed in float64."""
    acc = 0
    for y in ys:
        y = np.asarray(y).astype(np.complex128)
        acc = acc + np.einsum("akm,bkm->kab", y, np.conj(y))
    return acc


def _w1_holds(R, Rr, exact, what):
    """W1 sums in double and rounds once, so it sits within a few float
    roundings of the exact sum of its own outputs; the reference accumulates
    serially in float (src/channelizer.c:430-436), whose error grows with the
    hop count, so the two agree within that (1e-4 of each channel's power)."""
    scale = np.max(np.abs(exact), axis=(1, 2))
    assert np.max(np.max(np.abs(R - exact), axis=(1, 2)) / scale) <= 1e-6, what
    assert np.max(np.max(np.abs(R - Rr), axis=(1, 2)) / scale) <= 1e-4, what


def test_coherent_array_config(ref):
    nel, M = 8, 2048
    xs = W.coherent_array(1 << 18, nel)
    y = ak.Pfb(FS, M, 1, 16, W.ATTEN_BETA8, nel).process_n(xs, nel)
    r = ref.Pfb(FS, M, 1, 16, W.ATTEN_BETA8, nel).process_n(xs, nel)
    _parity(np.asarray(y), np.asarray(r), "coherent array")
    _fp64_holds(y, r, M, 1, 16, W.ATTEN_BETA8, [x[: 1 << 16] for x in xs], "coherent array")
    R, c = np.zeros((M, nel, nel), np.complex64), np.zeros(M, np.uint32)
    Rr, cr = np.zeros((M, nel, nel), np.complex64), np.zeros(M, np.uint32)
    ak.pfb_cov_accumulate(np.asarray(y), nel, M, None, R, c)
    ref.pfb_cov_accumulate(np.asarray(r), nel, M, None, Rr, cr)
    assert np.array_equal(c, cr)
    _w1_holds(R, Rr, _w1_exact([y]), "coherent array")
    pw, mp = ak.pfb_channel_power(np.asarray(y), nel, M)
    pwr, mpr = ref.pfb_channel_power(np.asarray(r), nel, M)
    assert np.max(np.abs(pw - pwr) / pwr) <= TOL and np.max(np.abs(mp - mpr) / mpr) <= TOL


def test_uneven_streams_config(ref):
    from atkdsp_b200 import gpu
    specs = W.uneven_streams(256, seed=4)
    pick = {}
    for s in specs:
        pick.setdefault((s.nchan, s.taps), s)
    chosen = [pick[k] for k in sorted(pick)]
    assert {(4096, 12), (4096, 16)} <= set(pick)
    hs = [ak.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in chosen]
    rs = [ref.Pfb(FS, s.nchan, s.oversample, s.taps, 80.0, 1) for s in chosen]
    b = gpu.Batch(hs, use_graph=True)
    ys = [[] for _ in chosen]
    yr = [[] for _ in chosen]
    for blk in range(3):
        xs = [W.stream_samples(s, blk) for s in chosen]
        din = [torch.from_numpy(x).cuda() for x in xs]
        dout = [torch.empty(max(1, s.nchan * h.out_hops(x.size)), dtype=torch.complex64, device="cuda")
                for s, h, x in zip(chosen, hs, xs)]
        ms = b.process(din, dout)
        torch.cuda.synchronize()
        for i, (s, x) in enumerate(zip(chosen, xs)):
            ys[i].append(dout[i][: s.nchan * ms[i]].view(s.nchan, ms[i]).cpu().numpy())
            yr[i].append(np.asarray(rs[i].process(x)))
    for i, s in enumerate(chosen):
        y, r = np.concatenate(ys[i], axis=1), np.concatenate(yr[i], axis=1)
        _parity(y, r, (s.nchan, s.taps, s.length))
        x0 = W.stream_samples(s, 0)[: 1 << 15]
        _fp64_holds(y[None], r[None], s.nchan, 2, s.taps, 80.0, [x0], (s.nchan, s.taps))


def test_served_config(ref):
    from atkdsp_b200.serve import Server
    specs = W.served_streams(4096)[:12]
    srv = Server(max_streams=16, hbm_reserve=1 << 30)
    ids = [srv.open(FS, sp.nchan, 2, 16, 80.0, "ci16") for sp in specs]
    assert min(ids) >= 0
    rps = [ref.Pfb(FS, sp.nchan, 2, 16, 80.0, 1) for sp in specs]
    got = {i: [] for i in range(len(specs))}
    want = {i: [] for i in range(len(specs))}
    keep, tagmap, tag = [], {}, 0
    for blk in range(4):
        for i, sp in enumerate(specs):
            raw = W.ci16_block(sp.block, sp.seed, blk)
            dev = torch.from_numpy(raw.reshape(-1).copy()).cuda()
            hop = sp.nchan // 2
            out = torch.zeros(sp.nchan * ((hop - 1 + sp.block) // hop) + 1, dtype=torch.complex64, device="cuda")
            keep.append((dev, out))
            assert srv.submit(ids[i], dev, out, tag=tag) == 0
            tagmap[tag] = (i, out)
            x, _ = ref.unpack_dc(raw.tobytes(), "ci16", 0j)
            want[i].append(np.asarray(rps[i].process(x)))
            tag += 1
        srv.launch()
        for _sid, tg, m, _n, _ta, _td in srv.poll():
            i, out = tagmap[tg]
            got[i].append((tg, out[: specs[i].nchan * m].view(specs[i].nchan, m).cpu().numpy()))
    for _sid, tg, m, _n, _ta, _td in srv.drain():
        i, out = tagmap[tg]
        got[i].append((tg, out[: specs[i].nchan * m].view(specs[i].nchan, m).cpu().numpy()))
    for i, sp in enumerate(specs):
        y = np.concatenate([a for _, a in sorted(got[i], key=lambda t: t[0])], axis=1)
        r = np.concatenate(want[i], axis=1)
        _parity(y, r, (sp.nchan, sp.block))


@pytest.mark.parametrize("M,os_,K", [(64, 2, 8), (1024, 2, 12), (2048, 1, 16), (4096, 2, 16), (192, 2, 12)])
def test_nan_samples_keep_their_meaning(ref, M, os_, K):
    """A NaN sample marks a sample as unmeasured: exactly the hops whose
    window holds it come out NaN (every channel, after the transform), as in
    the reference; every other output keeps the parity bar. W1 and W2 then
    carry the NaN into the same channels as the reference's."""
    rng = np.random.default_rng(M + K)
    n = M * 40 + 11
    x = W.tones_noise(n, 2, 20.0, rng)
    bad = rng.choice(n, 3, replace=False)
    x[bad] = np.complex64(complex(np.nan, 0.0))
    x[bad[0] + 1] = np.complex64(complex(0.0, np.nan))
    blocks = [1, 999, 4096, 7]
    y = run_blocks(ak.Pfb(FS, M, os_, K, 80.0, 1), [x], blocks)
    r = run_blocks(ref.Pfb(FS, M, os_, K, 80.0, 1), [x], blocks)
    assert y.shape == r.shape
    ny, nr = np.isnan(y.real) | np.isnan(y.imag), np.isnan(r.real) | np.isnan(r.imag)
    assert ny.any() and np.array_equal(ny, nr)
    keep = ~nr.any(axis=(0, 1))                      # hops with no NaN anywhere
    assert keep.any()
    _parity(y[..., keep], r[..., keep], "finite hops")
    pw, mp = ak.pfb_channel_power(y, 1, M)
    pwr, mpr = ref.pfb_channel_power(r, 1, M)
    assert np.array_equal(np.isnan(pw), np.isnan(pwr)) and np.array_equal(np.isnan(mp), np.isnan(mpr))
    R, c = np.zeros((M, 1, 1), np.complex64), np.zeros(M, np.uint32)
    Rr, cr = np.zeros((M, 1, 1), np.complex64), np.zeros(M, np.uint32)
    ak.pfb_cov_accumulate(y, 1, M, None, R, c)
    ref.pfb_cov_accumulate(r, 1, M, None, Rr, cr)
    assert np.array_equal(np.isnan(R), np.isnan(Rr)) and np.array_equal(c, cr)


@pytest.mark.parametrize("M,os_,K,nel", [(8192, 2, 8, 1), (16384, 1, 4, 1), (6401, 1, 3, 2), (7919, 1, 2, 1),
                                         (12000, 3, 4, 1)])
def test_large_filterbanks_match_the_reference(ref, M, os_, K, nel):
    """nchan beyond one CTA's shared memory (a power of two above 4096, any
    other value above 6400, primes included) runs through the separate fold,
    FFT-pass and epilogue kernels: the reference accepts these, and so does
    this library, with the same parity bar and streaming continuity."""
    rng = np.random.default_rng(M + K)
    n = M * K + 9 * (M // os_) + 17
    xs = [W.tones_noise(n, 2, 20.0, rng) for _ in range(nel)]
    blocks = [n // 3, 1, 999, n]
    y = run_blocks(ak.Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
    r = run_blocks(ref.Pfb(FS, M, os_, K, 80.0, nel), xs, blocks)
    assert y.shape[-1] >= 8
    _parity(y, r, (M, os_, K))


def test_wide_arrays_match_the_reference(ref):
    """More than 32 elements (the reference has no limit): the filterbank and
    W1 / W2 (the wide-array kernel) against the reference."""
    nel, M = 40, 64
    rng = np.random.default_rng(40)
    xs = [W.tones_noise(64 * 50 + 5, 1, 15.0, rng) for _ in range(nel)]
    y = np.asarray(ak.Pfb(FS, M, 2, 8, 80.0, nel).process_n(xs, nel))
    r = np.asarray(ref.Pfb(FS, M, 2, 8, 80.0, nel).process_n(xs, nel))
    _parity(y, r, "wide array")
    R, c = np.zeros((M, nel, nel), np.complex64), np.zeros(M, np.uint32)
    Rr, cr = np.zeros((M, nel, nel), np.complex64), np.zeros(M, np.uint32)
    ak.pfb_cov_accumulate(y, nel, M, None, R, c)
    ref.pfb_cov_accumulate(r, nel, M, None, Rr, cr)
    assert np.array_equal(c, cr)
    _w1_holds(R, Rr, _w1_exact([y]), "wide array")
    pw, mp = ak.pfb_channel_power(y, nel, M)
    pwr, mpr = ref.pfb_channel_power(r, nel, M)
    assert np.max(np.abs(pw - pwr) / pwr) <= TOL and np.max(np.abs(mp - mpr) / mpr) <= TOL


def test_small_calls_then_the_device_api():
    """Blocks that complete no hop wait on the host until the next call that
    produces hops; any other path (the device API here, a batch) first moves
    them into the device state: the result equals one unbroken call."""
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(5)
    x = W.tones_noise(256 * 40 + 3, 2, 20.0, rng)
    whole = np.asarray(ak.Pfb(FS, 256, 2, 12).process(x))
    p = ak.Pfb(FS, 256, 2, 12)
    parts = [np.asarray(p.process(x[:5])), np.asarray(p.process(x[5:40]))]      # no hops yet
    d = torch.from_numpy(x[40:]).cuda()
    torch.cuda.synchronize()
    y = gpu.process_n(p, [d], 1)
    gpu.sync(p)
    parts.append(y[0].cpu().numpy())
    got = np.concatenate([a for a in parts if a.shape[-1]], axis=-1)
    assert np.array_equal(got, whole)
