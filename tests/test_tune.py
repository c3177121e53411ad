"""The tile-shape choice (include/atkdsp_gpu.h atkdsp_gpu_tune_set/get): the
override table on the host (no GPU needed), and on the GPU both tile shapes
against the oracle -- the choice may change speed, never the outputs beyond
the parity bar (<= 1 ulp on < 1 % of values, 1e-5 per-channel RMS). The fold
sums are the same bits in every shape (each branch sums its taps in the same
order); the shapes' FFT plans differ in their first radix, so outputs may
differ from shape to shape by the last bit, as they may from the reference.
Choices: 1 the paired fold, 0 one hop per thread, 2 the quad fold (four hops
per thread; oversample 1 or 2, nchan <= 1024); plus 4 for the fold to read a
small nchan's tile window through L1 instead of staging it in shared memory
(5 paired, 4 one hop per thread; nchan <= 512)."""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from conftest import run_blocks

FS = 2.4e6


def test_override_table_set_get_and_reset():
    lib = ak.load()
    before = lib.atkdsp_gpu_tune_get(256, 2, 12)
    assert before in (0, 1, 2, 4, 5)
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, 0) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == 0
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, 1) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == 1
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, -1) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == before
    # shapes with a single tile shape: nchan 4096, oversample 8, non-powers of two
    assert lib.atkdsp_gpu_tune_set(4096, 2, 12, 1) < 0
    assert lib.atkdsp_gpu_tune_set(256, 8, 12, 0) < 0
    assert lib.atkdsp_gpu_tune_get(192, 2, 12) < 0
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, 2) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == 2
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, -1) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == before
    # the quad fold needs oversample 1 or 2 and nchan <= 1024
    assert lib.atkdsp_gpu_tune_set(256, 4, 12, 2) < 0
    assert lib.atkdsp_gpu_tune_set(2048, 2, 12, 2) < 0
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, 3) < 0 and lib.atkdsp_gpu_tune_set(256, 2, 12, 6) < 0
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, 5) == 0 and lib.atkdsp_gpu_tune_get(256, 2, 12) == 5
    assert lib.atkdsp_gpu_tune_set(256, 2, 12, -1) == 0
    assert lib.atkdsp_gpu_tune_set(1024, 2, 12, 5) < 0          # nothing staged above 512 channels


@pytest.mark.gpu
@pytest.mark.parametrize("M,os_,K", [(64, 2, 8), (512, 2, 16), (256, 1, 12), (1024, 4, 8), (2048, 2, 4),
                                     (16, 2, 2), (16, 1, 3), (32, 1, 2), (1024, 2, 16), (1024, 1, 5),
                                     (128, 2, 7)])
def test_both_tile_shapes_match_the_oracle(M, os_, K):
    from oracle import fp64
    from oracle import oracle as O
    lib = ak.load()
    rng = np.random.default_rng(M + K)
    n = M * 40 + 9
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    blocks = [1, 999, 4096, 7]
    ref = run_blocks(O.oracle().Pfb(FS, M, os_, K, 80.0, 1), [x], blocks)
    # every shape the library offers for this filterbank (tune_set refuses the rest)
    choices = [c for c in (1, 0, 2, 5, 4) if lib.atkdsp_gpu_tune_set(M, os_, K, c) == 0]
    assert choices[:2] == [1, 0] and (2 in choices) == (os_ in (1, 2) and M <= 1024)
    assert (5 in choices) == (M <= 512)
    try:
        ys = []
        for choice in choices:
            assert lib.atkdsp_gpu_tune_set(M, os_, K, choice) == 0
            y = run_blocks(ak.Pfb(FS, M, os_, K, 80.0, 1), [x], blocks)
            assert y.shape == ref.shape
            err = fp64.channel_rel_error(y, ref)
            assert err["rms"] <= 1e-5 and err["max"] <= 1e-5, (choice, err)
            u = np.abs(y.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
            assert u.max() <= 1 and np.mean(u > 0) < 1e-2, choice
            ys.append(y)
        for y in ys[1:]:
            u = np.abs(y.view(np.int32).astype(np.int64) - ys[0].view(np.int32).astype(np.int64))
            assert u.max() <= 1 and np.mean(u > 0) < 1e-2
    finally:
        lib.atkdsp_gpu_tune_set(M, os_, K, -1)
