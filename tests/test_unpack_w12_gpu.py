"""Unpack front end and W1/W2 accumulators on the GPU, against the reference
(golden fixtures, bit-exact) and the reference's own tests
(test_cross_check.py:88-116, 548-587; test_channelizer.py:127-169)."""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FS = 2.4e6
NCHAN = 192
SP = FS / NCHAN


def _bits(a):
    return np.asarray(a).view(np.uint32)


@pytest.mark.parametrize("fmt", ["cu8", "ci8", "ci16", "ci16q11", "cf32"])
def test_unpack_bit_exact_against_golden(golden_unpack, fmt):
    g = golden_unpack
    raw = g[f"{fmt}/raw"].tobytes()
    assert np.array_equal(_bits(ak.unpack(raw, fmt)), _bits(g[f"{fmt}/plain"]))
    for j in range(3):
        off = complex(*g[f"{fmt}/off{j}"].astype(np.float64))
        y, mean = ak.unpack_dc(raw, fmt, off)
        assert np.array_equal(_bits(y), _bits(g[f"{fmt}/dc{j}"])), (fmt, j)
        ref_mean = complex(*g[f"{fmt}/mean{j}"])
        assert abs(mean - ref_mean) <= 1e-12 * max(1.0, abs(ref_mean)), (fmt, j, mean, ref_mean)
    st = np.zeros(1, np.complex64)
    bps = ak.bytes_per_sample(fmt)
    cuts = [0, 40 * bps, 40 * bps + bps, len(raw)]
    ys = [ak.unpack(raw[a:b], fmt, 0.01, st) for a, b in zip(cuts[:-1], cuts[1:])]
    assert np.array_equal(_bits(np.concatenate(ys)), _bits(g[f"{fmt}/pole"]))
    assert np.array_equal(_bits(st), _bits(g[f"{fmt}/pole_state"]))


def test_unpack_large_block_bit_exact_and_mean():
    rng = np.random.default_rng(5)
    raw = rng.integers(-2048, 2048, 2 * 2_000_000, dtype=np.int64).astype("<i2").tobytes()
    orc = O.oracle()
    for off in (0j, 0.0123 - 0.0456j):
        y, mean = ak.unpack_dc(raw, "ci16q11", off)
        r, rmean = orc.unpack_dc(raw, "ci16q11", off)
        assert np.array_equal(_bits(y), _bits(r))
        assert abs(mean - rmean) < 1e-12


def test_unpack_dc_zero_offset_is_unpack_and_torn_tail():
    raw = np.random.default_rng(3).integers(0, 256, 4097, dtype=np.uint8).tobytes()
    for f in ("cu8", "ci16q11", "cf32"):
        a, _ = ak.unpack_dc(raw, f, 0j)
        b = ak.unpack(raw, f)
        assert np.array_equal(_bits(a), _bits(b))
        assert a.size == len(raw) // ak.bytes_per_sample(f)


def test_unpack_dc_mean_is_before_subtraction():
    n = 4096
    off = 0.25 - 0.1j
    rng = np.random.default_rng(11)
    x = (np.full(n, 0.4 + 0.2j) + 0.01 * (rng.standard_normal(n) + 1j * rng.standard_normal(n))).astype(np.complex64)
    y, mean = ak.unpack_dc(x.tobytes(), "cf32", off)
    assert abs(mean - complex(np.mean(x, dtype=np.complex128))) < 1e-5
    assert abs(complex(np.mean(y, dtype=np.complex128)) - (mean - off)) < 1e-5


def test_unpack_empty_and_bad_format():
    y, mean = ak.unpack_dc(b"", "ci16", 0.5 + 0.25j)
    assert y.size == 0 and mean == 0.5 + 0.25j
    lib = ak.load()
    buf = np.zeros(4, np.complex64)
    raw = np.zeros(8, np.uint8)
    assert lib.atkdsp_unpack(raw.ctypes.data, 8, 99, ak._cfp(buf), 4, 0.0, None) == -1
    assert lib.atkdsp_unpack_dc(raw.ctypes.data, 8, 3, None, 4, 0.0, 0.0, None, None) == -1


def test_dc_pole_is_continuous_across_blocks():
    raw = (np.random.default_rng(4).integers(-2048, 2048, 20000, dtype=np.int64) + 300).astype("<i2").tobytes()
    orc = O.oracle()
    sa = np.zeros(1, np.complex64)
    sb = np.zeros(1, np.complex64)
    outs_a, outs_b = [], []
    for chunk in (raw[:4000], raw[4000:4004], raw[4004:]):
        outs_a.append(ak.unpack(chunk, "ci16q11", 0.01, sa))
        outs_b.append(orc.unpack(chunk, "ci16q11", 0.01, sb))
    a, b = np.concatenate(outs_a), np.concatenate(outs_b)
    assert np.array_equal(_bits(a), _bits(b))
    assert abs(a[-2000:].mean()) < 0.05          # the 300-LSB offset (0.146) is gone


# ---- W1 / W2 ------------------------------------------------------------------
def test_w1_w2_against_golden(golden_w12):
    g = golden_w12
    y = g["y"]
    nel, M = y.shape[0], y.shape[1]
    R, c = g["R0"].copy(), g["c0"].copy()
    ak.pfb_cov_accumulate(y, nel, M, None, R, c)
    scale = np.max(np.abs(g["R"]))
    assert np.max(np.abs(R - g["R"])) / scale < 1e-5
    assert np.array_equal(c, g["counts"])
    Rg, cg = g["R0"].copy(), g["c0"].copy()
    ak.pfb_cov_accumulate(y, nel, M, g["gate"], Rg, cg)
    assert np.max(np.abs(Rg - g["Rg"])) / scale < 1e-5
    assert np.array_equal(cg, g["cg"])
    ungated = g["gate"] == 0
    assert np.array_equal(_bits(Rg[ungated]), _bits(g["R0"][ungated]))
    ak.pfb_cov_reset(Rg, cg, nel, M, g["gate"])
    assert np.array_equal(_bits(Rg), _bits(g["Rr"]))
    assert np.array_equal(cg, g["cr"])
    pwr, meanp = ak.pfb_channel_power(y, nel, M)
    assert np.array_equal(_bits(pwr), _bits(g["pwr"]))
    assert np.array_equal(_bits(meanp), _bits(g["meanp"]))


def test_w1_hermitian_and_matches_twin():
    phi = np.deg2rad(37.0)
    rng = np.random.default_rng(6)
    base = (np.exp(2j * np.pi * 40 * SP / FS * np.arange(NCHAN * 80))
            + 0.05 * (rng.standard_normal(NCHAN * 80) + 1j * rng.standard_normal(NCHAN * 80)))
    ins = [(base * np.exp(1j * e * phi)).astype(np.complex64) for e in range(5)]
    oc = ak.Pfb(FS, NCHAN, max_nel=5).process_n(ins, 5)
    R = np.zeros((NCHAN, 5, 5), np.complex64)
    cc = np.zeros(NCHAN, np.uint32)
    ak.pfb_cov_accumulate(oc, 5, NCHAN, None, R, cc)
    y = oc[:, 40, :].astype(np.complex128)
    Rt = y @ y.conj().T
    assert np.max(np.abs(R[40] - Rt)) / np.max(np.abs(Rt)) < 1e-6
    assert np.array_equal(R[40], R[40].conj().T)
    assert cc[40] == oc.shape[2]


@pytest.mark.parametrize("nel,m", [(1, 2048 * 3 + 77), (2, 256 * 5 + 3), (3, 255), (8, 257)])
def test_w12_chunk_edges_against_float64(nel, m):
    """The hops are staged in chunks (2048 for one element, 256 otherwise),
    two buffers in flight: several full chunks plus a ragged tail, and
    blocks just under and over one chunk, against float64 sums."""
    rng = np.random.default_rng(40 + nel)
    M = 24
    y = (rng.standard_normal((nel, M, m)) + 1j * rng.standard_normal((nel, M, m))).astype(np.complex64)
    R = np.zeros((M, nel, nel), np.complex64)
    c = np.zeros(M, np.uint32)
    ak.pfb_cov_accumulate(y, nel, M, None, R, c)
    assert (c == m).all()
    for k in range(M):
        yk = y[:, k, :].astype(np.complex128)
        Rt = yk @ yk.conj().T
        assert np.max(np.abs(R[k] - Rt)) / np.max(np.abs(Rt)) < 1e-6, k
    pwr, meanp = ak.pfb_channel_power(y, nel, M)
    pt = (np.abs(y.astype(np.complex128)) ** 2).mean(axis=2)
    assert np.max(np.abs(pwr - pt) / pt) < 1e-6
    assert np.allclose(meanp, pt.mean(0), rtol=1e-6)


def test_w12_many_elements_and_empty_block():
    rng = np.random.default_rng(12)
    nel, M, m = 32, 16, 300
    y = (rng.standard_normal((nel, M, m)) + 1j * rng.standard_normal((nel, M, m))).astype(np.complex64)
    R = np.zeros((M, nel, nel), np.complex64)
    c = np.zeros(M, np.uint32)
    ak.pfb_cov_accumulate(y, nel, M, None, R, c)
    for k in (0, 7, 15):
        yk = y[:, k, :].astype(np.complex128)
        Rt = yk @ yk.conj().T
        assert np.max(np.abs(R[k] - Rt)) / np.max(np.abs(Rt)) < 1e-6
    pwr, meanp = ak.pfb_channel_power(y, nel, M)
    pt = (np.abs(y.astype(np.complex128)) ** 2).mean(axis=2)
    assert np.max(np.abs(pwr - pt) / pt) < 1e-6
    assert np.allclose(meanp, pt.mean(0), rtol=1e-6)
    empty = np.zeros((nel, M, 0), np.complex64)
    R0 = R.copy()
    ak.pfb_cov_accumulate(empty, nel, M, None, R, c)
    assert np.array_equal(_bits(R), _bits(R0))
    p0, m0 = ak.pfb_channel_power(empty, nel, M)
    assert not p0.any() and not m0.any()


def test_w2_powers_gate_w1_on_the_device():
    """W3's data flow without a host round trip: a block's W2 channel powers,
    a per-channel gate made from them on the device (here a level test
    against the median channel; the reference's CFAR would supply it), and
    W1 accumulated only where the gate is set: the oracle's gated W1 with the
    same gate to W1's bar (1e-5 of the largest entry; the device sums in
    another order), counts exact, ungated channels untouched."""
    torch = pytest.importorskip("torch")
    from atkdsp_b200 import gpu
    from oracle import oracle as O
    M, nel, n = 192, 4, 192 * 40
    rng = np.random.default_rng(91)
    k = np.arange(n)
    base = np.exp(2j * np.pi * (40 * 2.4e6 / M) / 2.4e6 * k)
    xs = [(3.0 * base * np.exp(1j * 0.7 * e) + 0.3 * (rng.standard_normal(n) + 1j * rng.standard_normal(n)))
          .astype(np.complex64) for e in range(nel)]
    p = ak.Pfb(2.4e6, M, 2, 12, 80.0, nel)
    y = gpu.process_n(p, [torch.from_numpy(x).cuda() for x in xs], nel)
    gpu.sync(p)                       # the handle's stream is not the default one
    pwr, meanp = gpu.channel_power(y, nel, M)
    gate = (meanp > 4.0 * torch.median(meanp)).to(torch.uint8)
    assert 0 < int(gate.sum()) < M
    R = torch.zeros((M, nel, nel), dtype=torch.complex64, device="cuda")
    cnt = torch.zeros(M, dtype=torch.int32, device="cuda")
    gpu.cov_accumulate(y, nel, M, gate, R, cnt)
    torch.cuda.synchronize()
    yh, gh = y.cpu().numpy(), gate.cpu().numpy()
    Ro = np.zeros((M, nel, nel), np.complex64)
    co = np.zeros(M, np.uint32)
    O.oracle().pfb_cov_accumulate(yh, nel, M, gh, Ro, co)
    Rd = R.cpu().numpy()
    assert np.max(np.abs(Rd - Ro)) / np.max(np.abs(Ro)) < 1e-5
    assert np.all(Rd[gh == 0] == 0)
    assert np.array_equal(cnt.cpu().numpy().astype(np.uint32), co)
    assert np.all(co[gh == 0] == 0) and np.all(co[gh == 1] == y.shape[-1])


def test_host_w1_w2_and_unpack_from_two_threads_at_once():
    """The host-pointer W1/W2 and unpack calls stage through a per-thread
    device area on their own stream, so calls from different threads run at
    the same time and never share memory: each thread's results equal the
    same calls made one after the other."""
    import threading
    rng = np.random.default_rng(11)
    nel, M, m = 3, 256, 700
    blocks = [(rng.standard_normal((nel, M, m)) + 1j * rng.standard_normal((nel, M, m))).astype(np.complex64)
              for _ in range(2)]
    raws = [rng.integers(-2048, 2048, 2 * 300_001, dtype=np.int64).astype("<i2").tobytes() for _ in range(2)]

    def work(i, res):
        R = np.zeros((M, nel, nel), np.complex64)
        c = np.zeros(M, np.uint32)
        for _ in range(20):
            ak.pfb_cov_accumulate(blocks[i], nel, M, None, R, c)
            pw, mp = ak.pfb_channel_power(blocks[i], nel, M)
            x, mean = ak.unpack_dc(raws[i], "ci16q11", 0.01j)
        res[i] = (R, c, pw, mp, x, mean)

    serial = [None, None]
    for i in range(2):
        work(i, serial)
    par = [None, None]
    ts = [threading.Thread(target=work, args=(i, par)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for i in range(2):
        for a, b in zip(serial[i], par[i]):
            if isinstance(a, np.ndarray):
                assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), i
            else:
                assert a == b, i


@pytest.mark.parametrize("M,os_,K,fmt", [(1024, 2, 12, "cf32"), (1024, 2, 12, "ci16q11"), (256, 2, 16, "ci16"),
                                         (64, 1, 8, "cf32"), (4096, 2, 8, "cf32"), (192, 2, 6, "cf32")])
def test_fused_w12_equals_the_separate_pass(M, os_, K, fmt):
    """atkdsp_gpu_pfb_process_w12 (W2 power sums taken in the filterbank's
    epilogue, tile by tile, then added in tile order) against the filterbank
    followed by the separate W1/W2 pass: the same outputs bit for bit, the
    same counts, and W1 / W2 within a few float roundings (only the order of
    the double additions differs); across three blocks, gated W1. Shapes the
    epilogue does not fuse (nchan 4096, not a power of two) take the separate
    pass inside the same call."""
    import torch
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(M + K)
    p1, p2 = ak.Pfb(2.4e6, M, os_, K), ak.Pfb(2.4e6, M, os_, K)
    s1 = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p1.handle))
    s2 = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p2.handle))
    gate = torch.from_numpy((rng.random(M) < 0.7).astype(np.uint8)).cuda()
    R1 = torch.zeros((M, 1, 1), dtype=torch.complex64, device="cuda"); R2 = R1.clone()
    c1 = torch.zeros(M, dtype=torch.int32, device="cuda"); c2 = c1.clone()
    w1 = torch.zeros((1, M), dtype=torch.float32, device="cuda"); w2 = w1.clone()
    m1 = torch.zeros(M, dtype=torch.float32, device="cuda"); m2 = m1.clone()
    off = 0.0123 - 0.0456j if fmt != "cf32" else 0j
    for b in range(3):
        n = int(rng.integers(M * K, M * K + 50 * M))
        if fmt == "cf32":
            x = torch.from_numpy(((rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 3).astype(np.complex64)).cuda()
        else:
            x = torch.from_numpy(rng.integers(-2000, 2000, 2 * n, dtype=np.int64).astype("<i2")).cuda()
        torch.cuda.synchronize()
        y1 = gpu.process_w12(p1, x, fmt, off, R=R1, counts=c1, pwr=w1, mean_pwr=m1, gate=gate, stream=s1)
        y2 = gpu.process_n(p2, [x], 1, stream=s2) if fmt == "cf32" else \
            gpu.process_n_raw(p2, [x], 1, fmt, off, stream=s2)
        gpu.accumulate(y2, 1, M, R2, c2, w2, m2, gate=gate, stream=s2)
        torch.cuda.synchronize()
        assert np.array_equal(y1.cpu().numpy(), y2.cpu().numpy()), b
        a, r = w1.cpu().numpy(), w2.cpu().numpy()
        assert np.max(np.abs(a - r) / np.maximum(r, 1e-30)) <= 1e-6, b
        assert np.max(np.abs(m1.cpu().numpy() - m2.cpu().numpy()) / np.maximum(m2.cpu().numpy(), 1e-30)) <= 1e-6
    assert np.array_equal(c1.cpu().numpy(), c2.cpu().numpy())
    Ra, Rb = R1.cpu().numpy().reshape(-1), R2.cpu().numpy().reshape(-1)
    assert np.max(np.abs(Ra - Rb) / np.maximum(np.abs(Rb), 1e-30)) <= 1e-6
    assert np.all(Ra[gate.cpu().numpy() == 0] == 0)
