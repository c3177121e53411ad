"""The CFAR detector and burst tracker on the GPU against the reference
(golden fixtures from its C library) and the numpy cell oracle.

Bars:
  - events: type, id, flags, bins, hit counts and times t0 / t1 identical;
    fc_bin within 1e-9 relative; level / noise / SNR / band SNR within
    1e-4 dB. The per-cell sums run in the reference's order; only the device
    exp of the dB conversion may round differently in the last bit;
  - counters, describe() and alpha identical;
  - the last frame's hit mask identical, its averaged power and threshold
    within 1e-5 dB;
  - against the oracle at sizes beyond the fixtures: hits identical except
    where X lies within 1e-12 of the threshold (none expected).
"""

from __future__ import annotations

import numpy as np
import pytest

import cfar_cases
from cfar_cases import CFAR_CASES, EVENT_KEYS, FRAME_DT, FRAME_T0, run_case
from oracle import cfar_oracle as CO

pytestmark = pytest.mark.gpu

STAT_KEYS = sorted(["frames", "warmup", "cells_tested", "cell_hits", "untestable", "opened", "closed", "updates",
                    "dropped", "resets", "tracks"])


def _cfar(nbins, **cfg):
    import atkdsp_b200 as ak
    return ak.Cfar(nbins, **cfg)


def _arr(events) -> np.ndarray:
    return np.array([[e[k] for k in EVENT_KEYS] for e in events], np.float64).reshape(-1, len(EVENT_KEYS))


def _same_events(got: np.ndarray, ref: np.ndarray, what):
    assert got.shape == ref.shape, (what, got.shape, ref.shape)
    if not len(ref):
        return
    ints = [0] + [1 + EVENT_KEYS.index(k) for k in ("type", "id", "flags", "lo", "hi", "n_hits")]
    assert np.array_equal(got[:, ints], ref[:, ints]), what
    for k in ("t0", "t1"):
        c = 1 + EVENT_KEYS.index(k)
        assert np.array_equal(got[:, c], ref[:, c], equal_nan=True), (what, k)
    c = 1 + EVENT_KEYS.index("fc_bin")
    assert np.allclose(got[:, c], ref[:, c], rtol=1e-9, atol=0), what
    for k in ("level_db", "noise_db", "snr_db", "band_snr_db"):
        c = 1 + EVENT_KEYS.index(k)
        g, r = got[:, c], ref[:, c]
        assert np.array_equal(np.isfinite(g), np.isfinite(r)), (what, k)
        f = np.isfinite(r)
        assert np.array_equal(g[~f], r[~f]), (what, k)
        assert np.max(np.abs(g[f] - r[f]), initial=0.0) <= 1e-4, (what, k)


@pytest.mark.parametrize("name", sorted(CFAR_CASES))
def test_golden_cases_match_the_reference(golden_cfar, name):
    xs = golden_cfar[f"{name}/in"]
    ev, last, st, desc, al = run_case(_cfar, name, xs)
    _same_events(ev, golden_cfar[f"{name}/events"], name)
    assert [st[k] for k in STAT_KEYS] == [int(v) for v in golden_cfar[f"{name}/stats"]], (name, st)
    assert desc == str(golden_cfar[f"{name}/describe"]), name
    assert al == tuple(golden_cfar[f"{name}/alpha"]), name
    a, t, h = last
    assert np.array_equal(h, golden_cfar[f"{name}/last_hits"]), name
    for got, key in ((a, "last_avg"), (t, "last_thr")):
        ref = golden_cfar[f"{name}/{key}"]
        f = np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), f), (name, key)
        assert np.max(np.abs(got[f] - ref[f]), initial=0.0) <= 1e-5, (name, key)


@pytest.mark.parametrize("name", ["ca_default", "os_k3_looks4", "go_mask_hann", "ca_k8_long"])
def test_events_do_not_depend_on_how_frames_are_split(golden_cfar, name):
    """One call, one frame per call, and uneven calls give the same events
    (times to the rounding of each call's own start time), counters and last
    frame: the raw ring carries the k - 1 frames before a call."""
    xs = golden_cfar[f"{name}/in"]
    outs = []
    for pattern in ([len(xs)], [1] * len(xs), [5, 1, 2, 17, 1000]):
        c = _cfar(xs.shape[1], **cfar_cases.cfg_of(name))
        m = cfar_cases.mask_of(name)
        if m is not None:
            c.set_mask(m)
        rows, pos = [], 0
        for b in pattern:
            blk = xs[pos:pos + b]
            if not len(blk):
                break
            rows += [[0] + [e[k] for k in EVENT_KEYS] for e in c.process(blk, FRAME_T0 + pos * FRAME_DT, FRAME_DT)]
            pos += len(blk)
        rows += [[0] + [e[k] for k in EVENT_KEYS] for e in c.flush()]
        outs.append((np.array(rows).reshape(-1, 1 + len(EVENT_KEYS)), c.stats(), c.last()))
    times = [1 + EVENT_KEYS.index("t0"), 1 + EVENT_KEYS.index("t1")]
    rest = [c for c in range(1 + len(EVENT_KEYS)) if c not in times]
    for ev, st, last in outs[1:]:
        # a call's frame times start from its own frame_t0 (t0 + pos dt, then
        # + j dt), so they round differently from one call's t0 + (pos + j) dt
        assert ev.shape == outs[0][0].shape, name
        assert np.array_equal(ev[:, rest], outs[0][0][:, rest], equal_nan=True), name
        assert np.allclose(ev[:, times], outs[0][0][:, times], rtol=1e-12, atol=0, equal_nan=True), name
        assert st == outs[0][1], name
        for g, r in zip(last, outs[0][2]):
            assert np.array_equal(g, r, equal_nan=True), name


def test_device_frames_many_passes_against_the_oracle():
    """65536 bins: 16 frames per device pass (2^20 cells), so 150 frames take
    ten passes, with k_frames = 3 windows spanning their boundaries. The device hit masks (every frame's, from
    atkdsp_gpu_cfar_process) against the numpy oracle's, and the events
    against the host entry point's."""
    import torch
    from atkdsp_b200.gpu import cfar_process
    rng = np.random.default_rng(90)
    nb, nf = 65536, 150
    floor = rng.exponential(1.0, size=(nf, nb)) * np.linspace(1.0, 3.0, nb)[None, :]
    for _ in range(40):
        lo = int(rng.integers(0, nb - 16))
        f0 = int(rng.integers(0, nf - 5))
        floor[f0:f0 + int(rng.integers(3, 40)), lo:lo + int(rng.integers(1, 16))] += 10 ** rng.uniform(1, 3)
    xs = (10.0 * np.log10(floor)).astype(np.float32)
    cfg = dict(mode="ca", k_frames=3, n_ref=8, n_guard=2, pfa=1e-7)
    c = _cfar(nb, **cfg)
    ev, hits = cfar_process(c, torch.from_numpy(xs).cuda(), FRAME_T0, FRAME_DT, hits=True)
    X, thr, h_or = CO.cell_test(xs, cfg, c.alpha, c.alpha_ca)
    h_dev = hits.cpu().numpy()
    assert not h_dev[:2].any()                              # warm-up frames
    diff = h_dev[2:] != h_or
    near = np.abs(X - thr) <= 1e-12 * np.abs(thr)
    assert not (diff & ~near).any(), int(diff.sum())
    assert h_or.sum() > 100
    c2 = _cfar(nb, **cfg)
    ev2 = c2.process(xs, FRAME_T0, FRAME_DT)
    assert np.array_equal(_arr(ev), _arr(ev2), equal_nan=True) and len(ev) > 10
    assert c.stats() == c2.stats()


@pytest.mark.parametrize("n_ref,os_k", [(8, 0), (40, 0), (40, 1), (256, 300)])
def test_os_selection_against_the_oracle(n_ref, os_k):
    """The OS statistic gathers a bin's cells into a local array (64 or 512
    entries) and selects the os_k-th smallest: every frame's hits against
    the oracle's sort, for windows of 16 to 512 cells and ranks from the
    smallest to past the middle, with masked bins making some windows
    borrow."""
    import torch
    from atkdsp_b200.gpu import cfar_process
    rng = np.random.default_rng(93 + n_ref)
    nb, nf = 2048, 12
    floor = rng.exponential(1.0, size=(nf, nb)) * np.linspace(1.0, 2.0, nb)[None, :]
    floor[:, 700:702] += 1000.0          # narrower than the guard: the window sees only noise
    floor[3:8, 1500:1503] += 50.0
    xs = (10.0 * np.log10(floor)).astype(np.float32)
    cfg = dict(mode="os", n_ref=n_ref, n_guard=2, pfa=1e-4, os_k=os_k)
    mask = np.zeros(nb, np.uint8)
    mask[100:140] = 1
    c = _cfar(nb, **cfg)
    c.set_mask(mask)
    _ev, hits = cfar_process(c, torch.from_numpy(xs).cuda(), 0.0, 1.0, hits=True)
    X, thr, h_or = CO.cell_test(xs, dict(cfg, os_k=c.cfg["os_k"]), c.alpha, c.alpha_ca, mask)
    diff = hits.cpu().numpy() != h_or
    near = np.abs(X - thr) <= 1e-12 * np.abs(thr)
    assert not (diff & ~near).any(), int(diff.sum())
    assert h_or[:, 700:702].any()         # os_k 1 (the minimum of 80 cells) needs a large alpha


def test_linear_units_take_w2_powers_as_they_come():
    """units="linear": each value is the cell's linear power (clamped below
    at 1e-30); against the oracle fed the same linear values."""
    import torch
    from atkdsp_b200.gpu import cfar_process
    rng = np.random.default_rng(91)
    nb, nf = 1024, 20
    p = (rng.exponential(1.0, size=(nf, nb)) + np.where(np.arange(nb) % 97 == 0, 300.0, 0.0)).astype(np.float32)
    p[3, 10] = 0.0
    cfg = dict(n_ref=8, n_guard=2, pfa=1e-5, k_frames=2)
    c = _cfar(nb, **cfg)
    _ev, hits = cfar_process(c, torch.from_numpy(p).cuda(), 0.0, 1.0, units="linear", hits=True)
    db = 10.0 * np.log10(np.maximum(p.astype(np.float64), 1e-30))
    # the oracle's dB path on the exact dB of the linear values reproduces them to ~1 ulp
    X, thr, h_or = CO.cell_test(db, cfg, c.alpha, c.alpha_ca)
    diff = hits.cpu().numpy()[1:] != h_or
    near = np.abs(X - thr) <= 1e-9 * np.abs(thr)
    assert not (diff & ~near).any()
    assert h_or[:, ::97].all()


def test_w3_cfar_hits_gate_w1_on_the_device():
    """W3 end to end on the device: the filterbank's output, W2's channel
    powers, the CFAR over them (linear units), and that frame's hit mask as
    the gate of W1; R and counts equal the oracle W1 run with the same gate,
    and only the hit channels accumulate."""
    import torch
    import atkdsp_b200 as ak
    from atkdsp_b200 import gpu
    from oracle import oracle as O
    nchan, nel, n = 256, 4, 256 * 64
    rng = np.random.default_rng(92)
    k = np.arange(n)
    xs = []
    for e in range(nel):
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.05
        for f in (0.1003, -0.2501, 0.3302):
            x = x + np.exp(2j * np.pi * f * k + 1j * e)
        xs.append(x.astype(np.complex64))
    p = ak.Pfb(2.4e6, nchan, 2, 12, 80.0, nel)
    y = gpu.process_n(p, [torch.from_numpy(x).cuda() for x in xs], nel)
    gpu.sync(p)                       # the handle's stream is not the default one
    _pwr, meanp = gpu.channel_power(y, nel, nchan)
    c = _cfar(nchan, n_ref=8, n_guard=2, pfa=1e-6)
    _ev, hits = gpu.cfar_process(c, meanp.reshape(1, -1), 0.0, 1.0, units="linear", hits=True)
    gate = hits[0].contiguous()
    assert 3 <= int(gate.sum()) < nchan // 4
    R = torch.zeros((nchan, nel, nel), dtype=torch.complex64, device="cuda")
    cnt = torch.zeros(nchan, dtype=torch.int32, device="cuda")
    gpu.cov_accumulate(y, nel, nchan, gate, R, cnt)
    torch.cuda.synchronize()
    yh, gh = y.cpu().numpy(), gate.cpu().numpy()
    Ro = np.zeros((nchan, nel, nel), np.complex64)
    co = np.zeros(nchan, np.uint32)
    O.oracle().pfb_cov_accumulate(yh, nel, nchan, gh, Ro, co)
    Rd = R.cpu().numpy()
    assert np.max(np.abs(Rd - Ro)) / np.max(np.abs(Ro)) < 1e-5
    assert np.all(Rd[gh == 0] == 0)
    assert np.array_equal(cnt.cpu().numpy().astype(np.uint32), co)
    assert np.all(co[gh == 0] == 0) and np.all(co[gh == 1] == y.shape[-1])
    # the gate is the CFAR's own decision: the same powers through the host API
    db = (10.0 * np.log10(np.maximum(meanp.cpu().numpy().astype(np.float64), 1e-30))).astype(np.float32)
    c2 = _cfar(nchan, n_ref=8, n_guard=2, pfa=1e-6)
    c2.process(db, 0.0, 1.0)
    assert np.array_equal(c2.last()[2], gh)


def test_reset_mask_and_argument_rules():
    import torch
    import atkdsp_b200 as ak
    from atkdsp_b200.gpu import cfar_process
    xs = cfar_cases.frames("ca_default")
    c = _cfar(1024)
    assert c.last() is None
    e1 = c.process(xs, 0.0, 1.0)
    c.reset()
    assert c.last() is None and c.stats()["resets"] == 1
    e2 = c.process(xs, 0.0, 1.0)
    assert len(e1) == len(e2) and e2[0]["id"] > e1[-1]["id"]       # ids keep counting
    keep = [i for i, k in enumerate(EVENT_KEYS) if k != "id"]
    assert np.array_equal(_arr(e1)[:, keep], _arr(e2)[:, keep], equal_nan=True)
    # masking a bin takes it out of the test and out of every window
    c2 = _cfar(1024)
    mask = np.zeros(1024, np.uint8)
    mask[500:540] = 1
    c2.set_mask(mask)
    c2.process(xs[:5], 0.0, 1.0)
    _a, thr, hits = c2.last()
    assert np.isnan(thr[500:540]).all() and not hits[500:540].any()
    assert "40 masked" in c2.describe()
    with pytest.raises(ak.AtkDspError):
        c2.set_mask(np.zeros(10))
    lib = ak.load()
    buf = (ak._CfarEvent * 4)()
    f = np.zeros((2, 1024), np.float32)
    import ctypes as C
    fp = f.ctypes.data_as(C.POINTER(C.c_float))
    assert lib.atkdsp_cfar_process(c2.handle, fp, 2, 0.0, 1.0, buf, 4) == -3      # cap < 2 x 256
    assert lib.atkdsp_cfar_process(c2.handle, None, 2, 0.0, 1.0, buf, 512) == -1
    assert lib.atkdsp_cfar_process(c2.handle, fp, 0, 0.0, 1.0, None, 0) == 0
    assert lib.atkdsp_gpu_cfar_process(c2.handle, None, 0, 2, 0.0, 1.0, buf, 512, None, None) == -1
    d = torch.zeros((2, 1024), dtype=torch.float32, device="cuda")
    assert lib.atkdsp_gpu_cfar_process(c2.handle, C.c_void_p(d.data_ptr()), 2, 2, 0.0, 1.0, buf, 512, None,
                                       None) == -1                                   # units
    with pytest.raises(ak.AtkDspError):
        cfar_process(c2, d[:, :100], 0.0, 1.0)
