"""Device-pointer entry points and batches (include/atkdsp_gpu.h) against the
host-pointer drop-in path: every result must be bit-identical -- the same
kernels compute each hop, only the buffers and the launch grouping differ.
This is also the "same alone and in the mix" check for the batched path."""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from atkdsp_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
FS = 2.4e6


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_device_process_n_equals_host_path():
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(1)
    for M, os_, K, nel in ((64, 1, 16, 1), (1024, 2, 12, 2), (4096, 2, 16, 1), (60, 3, 12, 2)):
        ph, pd = ak.Pfb(FS, M, os_, K, 80.0, nel), ak.Pfb(FS, M, os_, K, 80.0, nel)
        for blk in (M * 5 + 3, 7, M * 40):
            xs = [(rng.standard_normal(blk) + 1j * rng.standard_normal(blk)).astype(np.complex64)
                  for _ in range(nel)]
            yh = ph.process_n(xs, nel)
            yd = gpu.process_n(pd, [_dev(x) for x in xs], nel)
            gpu.sync(pd)
            assert np.array_equal(yh, yd.cpu().numpy()), (M, blk)


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_each_stream_alone(use_graph):
    from atkdsp_b200 import gpu
    specs = W.uneven_streams(24, seed=9, min_log2=10, max_log2=15)
    alone = [ak.Pfb(FS, s.nchan, s.oversample, s.taps) for s in specs]
    mixed = [ak.Pfb(FS, s.nchan, s.oversample, s.taps) for s in specs]
    batch = gpu.Batch(mixed, use_graph=use_graph)
    for blk in range(3):
        xs = [W.stream_samples(s, blk) for s in specs]
        if blk == 1:                                 # an empty block for one stream
            xs[3] = xs[3][:0]
        d_in = [_dev(x) for x in xs]
        ms = batch.out_hops([x.size for x in xs])
        outs = [torch.empty(max(1, s.nchan * m), dtype=torch.complex64, device="cuda")
                for s, m in zip(specs, ms)]
        got = batch.process(d_in, outs)
        assert got == ms
        torch.cuda.synchronize()
        for i, (s, p) in enumerate(zip(specs, alone)):
            y = p.process(xs[i])
            yb = outs[i][: s.nchan * ms[i]].view(s.nchan, ms[i]).cpu().numpy()
            assert np.array_equal(y, yb), (i, blk, s)


def test_device_unpack_and_w12_equal_host_path():
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(2)
    raw = rng.integers(-2048, 2048, 2 * 100_001, dtype=np.int64).astype("<i2")
    for off in (0j, 0.01 - 0.02j):
        yh, mh = ak.unpack_dc(raw.tobytes(), "ci16q11", off)
        yd, md = gpu.unpack_dc(_dev(raw), "ci16q11", off)
        assert np.array_equal(yh.view(np.uint32), yd.cpu().numpy().view(np.uint32))
        assert complex(*md.cpu().numpy()) == mh
    st_h = np.zeros(1, np.complex64)
    st_d = torch.zeros(1, dtype=torch.complex64, device="cuda")
    yh = ak.unpack(raw.tobytes(), "ci16q11", 0.02, st_h)
    yd = gpu.unpack(_dev(raw), "ci16q11", 0.02, st_d)
    assert np.array_equal(yh.view(np.uint32), yd.cpu().numpy().view(np.uint32))
    assert st_h[0] == st_d.cpu().numpy()[0]
    y = (rng.standard_normal((4, 64, 100)) + 1j * rng.standard_normal((4, 64, 100))).astype(np.complex64)
    R = np.zeros((64, 4, 4), np.complex64)
    c = np.zeros(64, np.uint32)
    ak.pfb_cov_accumulate(y, 4, 64, None, R, c)
    Rd = torch.zeros((64, 4, 4), dtype=torch.complex64, device="cuda")
    cd = torch.zeros(64, dtype=torch.int32, device="cuda")
    gpu.cov_accumulate(_dev(y), 4, 64, None, Rd, cd)
    assert np.array_equal(R, Rd.cpu().numpy())
    p1, m1 = ak.pfb_channel_power(y, 4, 64)
    p2, m2 = gpu.channel_power(_dev(y), 4, 64)
    assert np.array_equal(p1, p2.cpu().numpy()) and np.array_equal(m1, m2.cpu().numpy())


def test_fused_front_end_equals_unpack_then_filterbank():
    """atkdsp_gpu_pfb_process_n_raw == atkdsp_unpack_dc then atkdsp_pfb_process,
    bit for bit, across uneven blocks with a changing offset (the running DC
    estimate of the 40 MS/s front end: each block's offset is the previous
    block's mean)."""
    from atkdsp_b200 import gpu
    raw = W.front_end_raw(300_000, seed=7)
    for M, os_, K, fmt in ((1024, 2, 12, "ci16q11"), (256, 2, 16, "ci16"), (64, 1, 16, "ci16q11")):
        ph, pd = ak.Pfb(FS, M, os_, K), ak.Pfb(FS, M, os_, K)
        off, pos = 0j, 0
        for blk in (100_000, 7, 40_001, 159_992):
            chunk = raw[pos:pos + blk]
            x, mean = ak.unpack_dc(chunk.tobytes(), fmt, off)
            yh = ph.process(x)
            yd = gpu.process_n_raw(pd, [_dev(chunk.reshape(-1))], 1, fmt, off)[0]
            gpu.sync(pd)
            assert np.array_equal(yh, yd.cpu().numpy()), (M, blk)
            off = complex(np.float32(mean.real), np.float32(mean.imag))
            pos += blk


def test_batch_raw_equals_each_stream_alone():
    from atkdsp_b200 import gpu
    specs = W.uneven_streams(12, seed=3, min_log2=11, max_log2=15)
    alone = [ak.Pfb(FS, s.nchan, s.oversample, s.taps) for s in specs]
    mixed = [ak.Pfb(FS, s.nchan, s.oversample, s.taps) for s in specs]
    batch = gpu.Batch(mixed, use_graph=True)
    offs = [complex(0.01 * i, -0.02 * i) for i in range(len(specs))]
    for blk in range(3):
        raws = [W.ci16_block(s.length, s.seed, blk) for s in specs]
        ms = batch.out_hops([s.length for s in specs])
        outs = [torch.empty(max(1, s.nchan * m), dtype=torch.complex64, device="cuda")
                for s, m in zip(specs, ms)]
        assert batch.process_raw([_dev(r.reshape(-1)) for r in raws], outs, "ci16", offs) == ms
        torch.cuda.synchronize()
        for i, s in enumerate(specs):
            x, _ = ak.unpack_dc(raws[i].tobytes(), "ci16", offs[i])
            y = alone[i].process(x)
            assert np.array_equal(y, outs[i][: s.nchan * ms[i]].view(s.nchan, ms[i]).cpu().numpy()), i


def test_block_mean_and_one_pass_accumulate():
    from atkdsp_b200 import gpu
    raw = W.front_end_raw(123_457, seed=9)
    for off in (0j, 0.05 - 0.03j):
        _, mh = ak.unpack_dc(raw.tobytes(), "ci16q11", off)
        md = gpu.block_mean(_dev(raw.reshape(-1)), "ci16q11", off).cpu().numpy()
        assert complex(*md) == mh
    rng = np.random.default_rng(4)
    y = (rng.standard_normal((3, 128, 77)) + 1j * rng.standard_normal((3, 128, 77))).astype(np.complex64)
    R = np.zeros((128, 3, 3), np.complex64)
    c = np.zeros(128, np.uint32)
    ak.pfb_cov_accumulate(y, 3, 128, None, R, c)
    p1, m1 = ak.pfb_channel_power(y, 3, 128)
    Rd = torch.zeros((128, 3, 3), dtype=torch.complex64, device="cuda")
    cd = torch.zeros(128, dtype=torch.int32, device="cuda")
    pd = torch.zeros((3, 128), dtype=torch.float32, device="cuda")
    md = torch.zeros(128, dtype=torch.float32, device="cuda")
    gpu.accumulate(_dev(y), 3, 128, Rd, cd, pd, md)
    assert np.array_equal(R, Rd.cpu().numpy()) and np.array_equal(c.astype(np.int32), cd.cpu().numpy())
    assert np.array_equal(p1, pd.cpu().numpy()) and np.array_equal(m1, md.cpu().numpy())
