"""The running DC estimate kept on the device: atkdsp_gpu_block_mean_dev and
atkdsp_gpu_pfb_process_w12_dev read the offset (the previous block's mean,
two doubles) from device memory and round it to float there. They must give
the bits of the host-offset calls made with that mean read back and rounded
on the host -- the reference front end's sequence (unpack_dc with the
previous block's mean as the offset, src/convert.c:122-128, then the
filterbank and W1/W2) -- without the per-block round trip.
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _host_off(mean: torch.Tensor) -> complex:
    mh = mean.cpu().numpy()
    return complex(np.float32(mh[0]), np.float32(mh[1]))


def _raw(fmt, n, rng):
    if fmt == "cf32":
        return torch.from_numpy(((rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.3 + 0.05)
                                .astype(np.complex64)).cuda()
    if fmt == "cu8":
        return torch.from_numpy(rng.integers(0, 256, 2 * n).astype(np.uint8)).cuda()
    if fmt == "ci8":
        return torch.from_numpy(rng.integers(-128, 128, 2 * n).astype(np.int8)).cuda()
    return torch.from_numpy((rng.integers(-1800, 1800, 2 * n) + 150).astype("<i2")).cuda()


@pytest.mark.parametrize("fmt", ["ci16q11", "ci16", "ci8", "cu8", "cf32"])
@pytest.mark.parametrize("n", [1, 5, 4097, 1_000_003])
def test_block_mean_dev_equals_the_host_offset(fmt, n):
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(n + len(fmt))
    prev = torch.tensor([0.01234567891, -0.0456789], dtype=torch.float64, device="cuda")
    raw = _raw(fmt, n, rng)
    a = gpu.block_mean(raw, fmt, _host_off(prev))
    b = gpu.block_mean(raw, fmt, prev)
    c = prev.clone()
    gpu.block_mean(raw, fmt, c, mean=c)                   # in place: offset and mean one buffer
    torch.cuda.synchronize()
    assert np.array_equal(a.cpu().numpy().view(np.uint64), b.cpu().numpy().view(np.uint64))
    assert np.array_equal(a.cpu().numpy().view(np.uint64), c.cpu().numpy().view(np.uint64))


@pytest.mark.parametrize("fmt,M,os_,K", [("ci16q11", 1024, 2, 12), ("ci16", 1024, 2, 12),
                                          ("ci16q11", 192, 2, 6), ("ci16", 8192, 2, 4)])
def test_front_end_with_the_dc_estimate_on_the_device(fmt, M, os_, K):
    """Five blocks: block_mean, then the filterbank with W1/W2, the offset of
    block b the mean of block b-1. The host-offset run reads each mean back;
    the device run never does. Outputs, W1, W2 and the means agree bit for
    bit: with W1/W2 in the epilogue (nchan 1024), as a separate pass (192,
    not a power of two) and through the large-filterbank kernels (8192)."""
    from atkdsp_b200 import gpu
    rng = np.random.default_rng(11)
    blocks = [_raw(fmt, int(rng.integers(40000, 90000)), rng) for _ in range(5)]
    runs = []
    for device_offset in (False, True):
        p = ak.Pfb(2.4e6, M, os_, K)
        st = torch.cuda.ExternalStream(ak.load().atkdsp_gpu_pfb_stream(p.handle))
        R = torch.zeros((M, 1, 1), dtype=torch.complex64, device="cuda")
        cnt = torch.zeros(M, dtype=torch.int32, device="cuda")
        pwr = torch.zeros((1, M), dtype=torch.float32, device="cuda")
        mp = torch.zeros(M, dtype=torch.float32, device="cuda")
        means = [torch.zeros(2, dtype=torch.float64, device="cuda") for _ in range(2)]
        outs, ms = [], []
        for b, raw in enumerate(blocks):
            prev, cur = means[(b + 1) % 2], means[b % 2]
            off = prev if device_offset else _host_off(prev)
            gpu.block_mean(raw, fmt, off, mean=cur, stream=st)
            y = gpu.process_w12(p, raw, fmt, off, R=R, counts=cnt, pwr=pwr, mean_pwr=mp, stream=st)
            torch.cuda.synchronize()
            outs.append(y.cpu().numpy().copy())
            ms.append(cur.cpu().numpy().copy())
        runs.append((outs, ms, R.cpu().numpy(), cnt.cpu().numpy(), pwr.cpu().numpy(), mp.cpu().numpy()))
    (oa, ma, Ra, ca, pa, qa), (ob, mb, Rb, cb, pb, qb) = runs
    for x, y in zip(oa, ob):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    for x, y in zip(ma, mb):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
    assert np.array_equal(Ra.view(np.uint32), Rb.view(np.uint32)) and np.array_equal(ca, cb)
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32)) and np.array_equal(qa.view(np.uint32), qb.view(np.uint32))


def test_device_offset_argument_checks():
    from atkdsp_b200 import gpu
    p = ak.Pfb(2.4e6, 256, 2, 8)
    x = torch.zeros(2 * 4096, dtype=torch.int16, device="cuda")
    with pytest.raises(ak.AtkDspError):
        gpu.process_w12(p, x, "ci16", torch.zeros(2, dtype=torch.float32, device="cuda"))
    lib = ak.load()
    assert lib.atkdsp_gpu_block_mean_dev(x.data_ptr(), 16, 3, None, x.data_ptr(), None) == -1
    y = torch.zeros(4096, dtype=torch.complex64, device="cuda")
    off = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pytest.raises(ak.AtkDspError):
        gpu.process_w12(p, y, "cf32", off)                 # the device offset is for int16 blocks
