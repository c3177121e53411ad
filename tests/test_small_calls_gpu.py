"""Small host calls run one CTA per hop (pfb_hops_kernel); larger calls and
the device API run the tile kernel. The two must give the same bits: the
per-hop kernel folds every branch in the same order and walks the bank's own
FFT plan with the tile kernel's butterfly and twiddle arithmetic.

Checked on every tile shape the autotuner can pick (one hop per thread,
paired, quad, unstaged), oversample 1/2/4, calibration and two elements:
a stream fed in small blocks through ak.Pfb.process_n (host buffers) against
the same stream through gpu.process_n (device buffers, tile kernel), bit for
bit, and both against the oracle within the filterbank bar (reference
tests/test_channelizer.py:74-89 feeds blocks the same way).
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from conftest import run_blocks
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FS = 2.4e6
BLOCKS = [1, 999, 4096, 7, 33, 2500, 64]


def _device_blocks(p, xs, pattern):
    from atkdsp_b200 import gpu
    n = xs[0].size
    dev = [torch.from_numpy(x).cuda() for x in xs]
    outs, pos, bi = [], 0, 0
    while pos < n:
        b = min(pattern[bi % len(pattern)], n - pos)
        y = gpu.process_n(p, [d[pos:pos + b] for d in dev], len(xs))
        gpu.sync(p)
        if y.shape[-1]:
            outs.append(y.cpu().numpy())
        pos += b
        bi += 1
    return np.concatenate(outs, axis=-1)


@pytest.mark.parametrize("M,os_,K,choice", [
    (64, 1, 16, -1), (64, 1, 16, 1), (64, 1, 16, 0), (64, 2, 8, 5), (64, 2, 8, 4),
    (16, 2, 8, -1), (32, 1, 4, -1), (128, 4, 6, -1), (256, 2, 12, 2), (256, 1, 8, 5),
    (512, 2, 12, 1), (1024, 2, 12, -1), (1024, 1, 8, 0), (1024, 2, 16, 2)])
def test_small_host_calls_equal_the_tile_path(M, os_, K, choice):
    lib = ak.load()
    before = lib.atkdsp_gpu_tune_get(M, os_, K)
    if choice >= 0 and lib.atkdsp_gpu_tune_set(M, os_, K, choice) != 0:
        pytest.skip(f"tile shape {choice} does not exist for {M}/{os_}/{K}")
    try:
        rng = np.random.default_rng(M * 31 + K + os_)
        n = 3 * M * K + 20 * M + 17
        x = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / 2).astype(np.complex64)
        y_host = run_blocks(ak.Pfb(FS, M, os_, K), [x], BLOCKS)
        y_dev = _device_blocks(ak.Pfb(FS, M, os_, K), [x], BLOCKS)
    finally:
        lib.atkdsp_gpu_tune_set(M, os_, K, before)
    assert y_host.shape == y_dev.shape
    assert np.array_equal(y_host.view(np.uint32), y_dev.view(np.uint32))
    r = run_blocks(O.oracle().Pfb(FS, M, os_, K), [x], BLOCKS)
    assert r.shape == y_host.shape
    assert np.max(np.abs(y_host - r)) <= 1e-5 * np.max(np.abs(r))


def test_small_calls_two_elements_and_cal():
    M, os_, K = 256, 2, 12
    rng = np.random.default_rng(5)
    n = 6 * M * K
    xs = [((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / 2).astype(np.complex64) for _ in range(2)]
    cal = (rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))).astype(np.complex64)
    p1, p2 = ak.Pfb(FS, M, os_, K, 80.0, 2), ak.Pfb(FS, M, os_, K, 80.0, 2)
    p1.set_cal(cal, 2)
    p2.set_cal(cal, 2)
    y_host = run_blocks(p1, xs, BLOCKS)
    y_dev = _device_blocks(p2, xs, BLOCKS)
    assert np.array_equal(y_host.view(np.uint32), y_dev.view(np.uint32))
    assert ak.load().atkdsp_gpu_pfb_faults(p1.handle) == 0
    ro = O.oracle().Pfb(FS, M, os_, K, 80.0, 2)
    ro.set_cal(cal, 2)
    r = run_blocks(ro, xs, BLOCKS)
    assert np.max(np.abs(y_host - r)) <= 1e-5 * np.max(np.abs(r))


def test_small_calls_then_large_calls_keep_the_state():
    """Small calls (per-hop kernel, carries in its own CTAs) interleaved with
    calls above the small-call limit (tile kernel) on one handle."""
    M, os_, K = 1024, 2, 12
    rng = np.random.default_rng(8)
    n = (1 << 16) + 3 * M * K + 11
    x = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / 2).astype(np.complex64)
    pattern = [700, 40000, 3, 5000, (1 << 15) + 1]
    y = run_blocks(ak.Pfb(FS, M, os_, K), [x], pattern)
    y_dev = _device_blocks(ak.Pfb(FS, M, os_, K), [x], pattern)
    assert np.array_equal(y.view(np.uint32), y_dev.view(np.uint32))
