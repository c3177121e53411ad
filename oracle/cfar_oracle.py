"""CPU restatement of the CFAR detector's per-cell test -- TEST INFRASTRUCTURE ONLY.

Nothing in the product imports this. It restates, in numpy, the first half of
the reference's one_frame (src/cfar.c:524-592) and its table walk
(src/cfar.c:344-372):
  - each frame in dB becomes linear power exp(v ln10 / 10), v clamped at
    -300 (src/cfar.c:531-535);
  - the tested frame's X is the mean of the last k_frames raw frames, summed
    oldest first (src/cfar.c:544-548);
  - each bin's reference cells: the nearest unmasked cells beyond the guard
    on the left, then on the right, then what a short side borrows beyond
    the other side's far end; a bin without N cells is untestable;
  - T is CA's mean, OS's os_k-th smallest, GO / SO's greater / smaller side
    mean (CA with CA's alpha where the window borrowed); a NaN cell makes T
    NaN; a bin hits when X > alpha T (src/cfar.c:550-592).
Sums run in the reference's order, so the outputs match it wherever numpy's
exp rounds as glibc's does. Pinned by tests/test_oracle_pinned.py against the
last-frame lines of tests/golden/cfar.npz (the reference's own outputs).
"""

from __future__ import annotations

import numpy as np

LN10_OVER_10 = 0.23025850929940458


def tables(nbins: int, n_ref: int, n_guard: int, mask=None):
    """(idx (nbins, N) int64, ok bool, sided bool) with the reference's walk."""
    m = np.zeros(nbins, bool) if mask is None else np.asarray(mask).astype(bool)
    N = 2 * n_ref
    idx = np.zeros((nbins, N), np.int64)
    ok = np.zeros(nbins, bool)
    sided = np.zeros(nbins, bool)
    for i in range(nbins):
        if m[i]:
            continue
        left, right, ext = [], [], []
        j = i - n_guard - 1
        while j >= 0 and len(left) < n_ref:
            if not m[j]:
                left.append(j)
            j -= 1
        jl = j
        j = i + n_guard + 1
        while j < nbins and len(right) < n_ref:
            if not m[j]:
                right.append(j)
            j += 1
        jr = j
        short_l, short_r = n_ref - len(left), n_ref - len(right)
        j = jr
        while short_l > 0 and j < nbins:
            if not m[j]:
                ext.append(j)
                short_l -= 1
            j += 1
        j = jl
        while short_r > 0 and j >= 0:
            if not m[j]:
                ext.append(j)
                short_r -= 1
            j -= 1
        cells = left + right + ext
        if len(cells) < N:
            continue
        idx[i] = cells
        ok[i] = True
        sided[i] = not ext
    return idx, ok, sided


def raw_power(frames_db: np.ndarray) -> np.ndarray:
    v = np.asarray(frames_db, np.float32).astype(np.float64)
    v = np.where(v < -300.0, -300.0, v)
    return np.exp(v * LN10_OVER_10)


def cell_test(frames_db, cfg: dict, alpha: float, alpha_ca: float, mask=None):
    """Every tested frame of a run from reset: returns (X, thr, hits), one row
    per tested frame (frames k-1 .. end), thr NaN where untestable."""
    nbins = frames_db.shape[1]
    mode = cfg.get("mode", 0)
    mode = {"ca": 0, "os": 1, "go": 2, "so": 3}[mode] if isinstance(mode, str) else int(mode)
    k, n_ref = int(cfg.get("k_frames", 1)), int(cfg.get("n_ref", 16))
    N = 2 * n_ref
    os_k = int(cfg.get("os_k", 0)) or (3 * N + 3) // 4
    idx, ok, sided = tables(nbins, n_ref, int(cfg.get("n_guard", 4)), mask)
    raw = raw_power(frames_db)
    Xs, thrs, hitss = [], [], []
    for f in range(k - 1, raw.shape[0]):
        s = np.zeros(nbins)
        for r in range(k):
            s = s + raw[f - k + 1 + r]
        X = s / k
        cells = X[idx]                                   # (nbins, N), table order
        if mode == 1:
            Z = np.sort(cells, axis=1)[:, os_k - 1]
            Z = np.where(np.isnan(cells).any(axis=1), np.nan, Z)
            a = np.full(nbins, alpha)
        else:
            tot = np.zeros(nbins)
            for q in range(N):
                tot = tot + cells[:, q]
            Z = tot / N
            a = np.full(nbins, alpha)
            if mode in (2, 3):
                L = np.zeros(nbins)
                R = np.zeros(nbins)
                for q in range(n_ref):
                    L = L + cells[:, q]
                for q in range(n_ref, N):
                    R = R + cells[:, q]
                L, R = L / n_ref, R / n_ref
                side = np.maximum(L, R) if mode == 2 else np.minimum(L, R)
                Z = np.where(sided, side, Z)
                a = np.where(sided, alpha, alpha_ca)
        with np.errstate(invalid="ignore"):
            thr = np.where(ok, a * Z, np.nan)
            hits = ok & (X > thr)
        Xs.append(X)
        thrs.append(thr)
        hitss.append(hits.astype(np.uint8))
    return np.array(Xs), np.array(thrs), np.array(hitss)
