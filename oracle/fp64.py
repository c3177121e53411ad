"""Float64 numpy restatement of the channelizer -- TEST INFRASTRUCTURE ONLY.

The reference's numpy twin (python/atkdsp/reference.py:11481-11581, class
``Pfb``) is its specification: every step in float64. This module restates
that algorithm, vectorised over hops, so the error of any float32 path can be
stated against an all-float64 computation of the same filterbank:

    hop b's window = s[b*hop, b*hop + L),  s = history ++ input
    fold[q]        = sum_k h[k*nchan + q] * window[k*nchan + q]
    X              = DFT_nchan(fold)
    y[k]           = X[k] * exp(-2 pi i k ((b+1)*hop mod nchan) / nchan)
    out[e][k][b]   (channel-major), times cal[e][k] when a cal table is set

The prototype taps are the double taps of the C prototype
(src/channelizer.c:79-99), taken from the C restatement so that both sides
filter with exactly the same h.
"""

from __future__ import annotations

import numpy as np


class Fp64Pfb:
    def __init__(self, taps: np.ndarray, nchan: int, oversample: int, max_nel: int = 1):
        self.h = np.asarray(taps, np.float64)
        self.nchan = int(nchan)
        self.os = int(oversample)
        self.hop = self.nchan // self.os
        self.L = self.h.size
        self.K = self.L // self.nchan
        self.ov = self.L - self.hop
        self.max_nel = int(max_nel)
        self.cal = None
        self.reset()

    def reset(self):
        self.carry = [np.zeros(self.ov, np.complex128) for _ in range(self.max_nel)]
        self.b = 0

    def set_cal(self, table, nel):
        self.cal = None if table is None else np.asarray(table, np.complex128).reshape(int(nel), self.nchan)

    def process_n(self, ins, nel, chunk_hops: int = 4096):
        nel = int(nel)
        N, hop, L = self.nchan, self.hop, self.L
        xs = [np.asarray(ins[e], np.complex128).ravel() for e in range(nel)]
        s_all = [np.concatenate([self.carry[e], xs[e]]) for e in range(nel)]
        m = (s_all[0].size - self.ov) // hop
        out = np.zeros((nel, N, m), np.complex128)
        k = np.arange(N)
        for e in range(nel):
            s = s_all[e]
            for c0 in range(0, m, chunk_hops):
                c1 = min(m, c0 + chunk_hops)
                idx = np.arange(c0, c1)[:, None] * hop + np.arange(L)[None, :]
                seg = s[idx] * self.h[None, :]
                fold = seg.reshape(c1 - c0, self.K, N).sum(axis=1)
                X = np.fft.fft(fold, axis=1)
                bb = self.b + np.arange(c0, c1)
                shift = ((bb + 1) * hop) % N
                rot = np.exp(-2j * np.pi * ((k[None, :] * shift[:, None]) % N) / N)
                out[e, :, c0:c1] = (X * rot).T
            if self.cal is not None and e < self.cal.shape[0]:
                out[e] *= self.cal[e][:, None]
            self.carry[e] = s[m * hop:]
        self.b += m
        return out


def channel_rel_error(y: np.ndarray, yref: np.ndarray) -> dict:
    """Per-channel error divided by that channel's RMS, worst channel.

    y, yref: (..., nchan, m). Returns the worst channel's RMS error / RMS and
    its max-sample error / RMS, over every element and channel."""
    y = np.asarray(y).reshape(-1, y.shape[-1]).astype(np.complex128)
    r = np.asarray(yref).reshape(-1, yref.shape[-1]).astype(np.complex128)
    rms = np.sqrt(np.mean(np.abs(r) ** 2, axis=1))
    rms = np.where(rms > 0, rms, 1.0)
    err = np.abs(y - r)
    return {"rms": float(np.max(np.sqrt(np.mean(err ** 2, axis=1)) / rms)),
            "max": float(np.max(np.max(err, axis=1) / rms))}
