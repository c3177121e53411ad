"""Seeded CFAR workloads shared by the fixture generator and the tests.

Each case is a configuration, a frame count and the block pattern the frames
are fed in. The frames are spectrum lines in dB: a unit-mean gamma noise
floor of `looks` looks with a gentle slope, plus bursts (a band of bins that
switches on for a run of frames, some drifting by a bin per frame). Some
cases blank bins to NaN or carry a mask.
"""

from __future__ import annotations

import numpy as np

# name: (nbins, nframes, block pattern, config, mask spans, nan bins, seed)
CFAR_CASES = {
    "ca_default": (1024, 60, [1, 7, 30, 1000], {}, [], [], 71),
    "os_k3_looks4": (512, 80, [80], dict(mode="os", k_frames=3, looks=4.0, n_ref=8, n_guard=2, pfa=1e-4,
                                          merge_gap=2, min_bins=2), [], [], 72),
    "go_mask_hann": (2048, 40, [3, 3, 34], dict(mode="go", k_frames=2, n_ref=12,
                                                 rho2=(4 / 9, 1 / 36, 0.0, 0.0)),
                     [(0, 40), (900, 960), (2000, 2048)], [], 73),
    "so_tracks_capped": (256, 100, [50, 50], dict(mode="so", n_ref=32, n_guard=0, open_m=1, open_n=1,
                                                   close_k=1, max_tracks=4, pfa=2e-2), [], [], 74),
    "os_rho_k4": (1024, 50, [10, 40], dict(mode="os", os_k=20, k_frames=4, looks=2.0,
                                           rho2=(0.3, 0.05, 0.01, 0.0), open_m=3, open_n=5), [], [], 75),
    "ca_nan_bins": (768, 45, [45], dict(n_ref=6, n_guard=1, pfa=1e-5, close_k=2), [(100, 104)],
                    [5, 300, 301, 555], 76),
    "ca_mostly_masked": (200, 40, [40], dict(n_ref=16, n_guard=4, pfa=1e-2), [(15, 120), (125, 180)], [], 78),
    "ca_k8_long": (4096, 30, [2, 28], dict(k_frames=8, looks=1.0, n_ref=24, n_guard=3, merge_gap=3), [], [], 77),
}


def cfg_of(name: str) -> dict:
    return dict(CFAR_CASES[name][3])


def frames(name: str) -> np.ndarray:
    """(nframes, nbins) float32 dB frames of a case."""
    nbins, nframes, _pattern, cfg, _mask, nan_bins, seed = CFAR_CASES[name]
    rng = np.random.default_rng(seed)
    looks = float(cfg.get("looks", 1.0))
    floor = rng.gamma(looks, 1.0 / looks, size=(nframes, nbins))
    floor *= np.linspace(1.0, 2.0, nbins)[None, :]
    sig = np.zeros((nframes, nbins))
    for _ in range(max(3, nbins // 128)):
        width = int(rng.integers(1, 9))
        lo = int(rng.integers(0, nbins - width))
        f0 = int(rng.integers(0, nframes - 3))
        f1 = int(min(nframes, f0 + rng.integers(3, 25)))
        level = 10 ** (rng.uniform(0.8, 3.0))
        drift = int(rng.integers(-1, 2)) if rng.uniform() < 0.3 else 0
        for f in range(f0, f1):
            a = min(max(lo + drift * (f - f0), 0), nbins - width)
            sig[f, a:a + width] += level * rng.uniform(0.5, 1.5, size=width)
    x = 10.0 * np.log10(floor + sig)
    x[:, nan_bins] = np.nan
    return x.astype(np.float32)


def mask_of(name: str) -> np.ndarray | None:
    nbins, _nf, _p, _cfg, spans, _nan, _seed = CFAR_CASES[name]
    if not spans:
        return None
    m = np.zeros(nbins, np.uint8)
    for a, b in spans:
        m[a:b] = 1
    return m


EVENT_KEYS = ("type", "id", "flags", "lo", "hi", "n_hits", "t0", "t1", "fc_bin", "level_db", "noise_db",
              "snr_db", "band_snr_db")

FRAME_T0, FRAME_DT = 12.5, 0.001


def run_case(factory, name: str, xs: np.ndarray | None = None):
    """Feed a case through a Cfar made by factory(nbins, **cfg) in its block
    pattern, then flush. Returns (events array (call, *EVENT_KEYS), last
    (avg, thr, hits) or None, stats dict, describe string, (alpha, alpha_ca,
    et))."""
    nbins, nframes, pattern, _cfg, _m, _n, _s = CFAR_CASES[name]
    xs = frames(name) if xs is None else xs
    c = factory(nbins, **cfg_of(name))
    m = mask_of(name)
    if m is not None:
        c.set_mask(m)
    rows = []
    pos, call = 0, 0
    for b in pattern:
        if pos >= nframes:
            break
        blk = xs[pos:pos + b]
        for e in c.process(blk, FRAME_T0 + pos * FRAME_DT, FRAME_DT):
            rows.append([call] + [e[k] for k in EVENT_KEYS])
        pos += blk.shape[0]
        call += 1
    for e in c.flush():
        rows.append([call] + [e[k] for k in EVENT_KEYS])
    ev = np.array(rows, np.float64).reshape(-1, 1 + len(EVENT_KEYS))
    return ev, c.last(), c.stats(), c.describe(), (c.alpha, c.alpha_ca, c.et)
