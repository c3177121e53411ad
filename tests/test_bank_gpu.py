"""Undertow's per-scale filterbank bank as one launch (reference
src/undertow.c:244-257: every scale's atkdsp_pfb_process on the same chunk,
one OpenMP task per scale). Here the scales' handles form one batch and each
chunk is one persistent-kernel launch over all scales; the outputs must be
the per-scale calls' bit for bit, and the oracle's within the path's
tolerance."""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from atkdsp_b200 import workloads as W
from oracle import fp64
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FS = 2.4e6


def test_scale_bank_in_one_launch_matches_per_scale_calls_and_the_oracle():
    torch = pytest.importorskip("torch")
    from atkdsp_b200.gpu import Batch
    bank = W.scale_bank(6)                                 # 8 .. 256 channels
    rng = np.random.default_rng(77)
    chunks = [W.SCALE_BANK_BLOCK, 1000, 3, W.SCALE_BANK_BLOCK - 17, 40000]
    xs = [W.tones_noise(n, 3, 15.0, rng) for n in chunks]
    handles = [ak.Pfb(FS, M, os_, K) for M, os_, K in bank]
    batch = Batch(handles)
    alone = [ak.Pfb(FS, M, os_, K) for M, os_, K in bank]
    orc = [O.oracle().Pfb(FS, M, os_, K) for M, os_, K in bank]
    got = [[] for _ in bank]
    for x in xs:
        d = torch.from_numpy(x).cuda()
        outs = [torch.empty(max(1, M * p.out_hops(x.size)), dtype=torch.complex64, device="cuda")
                for (M, _, _), p in zip(bank, handles)]
        ms = batch.process([d] * len(bank), outs)
        torch.cuda.synchronize()
        for s, ((M, _, _), m) in enumerate(zip(bank, ms)):
            got[s].append(outs[s][: M * m].cpu().numpy().reshape(M, m))
    for s, (M, _, _) in enumerate(bank):
        y = np.concatenate(got[s], axis=1)
        ya = np.concatenate([alone[s].process(x) for x in xs], axis=1)
        yo = np.concatenate([orc[s].process(x) for x in xs], axis=1)
        assert y.shape == ya.shape == yo.shape
        assert np.array_equal(y, ya), f"scale {s}: batched != per-scale call"
        err = fp64.channel_rel_error(y, yo)
        assert err["max"] <= 1e-5, (s, err)
