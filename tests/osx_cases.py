"""Overlap-save extractor cases shared by the golden-fixture generator and the
tests: the same seeded inputs, channel plans and block schedules replayed
against any object with the binding's ``Osx`` surface (the reference build,
the C oracle, or the B200 library)."""

from __future__ import annotations

import numpy as np

FS = 2.4e6

# name -> (nfft, nel, channels [(offset_hz, bw_hz, out_rate)], nsamples,
#          block pattern, seed, events {block index: op})
# ops: ("remove", slot) / ("retune", slot, offset_hz) / ("add", offset, bw, rate)
OSX_CASES = {
    # the reference tests' channel (50 kHz at 300 kHz, resampled 75 -> 50 kHz)
    # and its hard offsets: an odd bin, a fractional and a negative fractional
    "n4096_hard_offsets": (4096, 1, [(300e3, 50e3, 50e3), (513 * FS / 4096, 50e3, 50e3),
                                     (300200.0, 50e3, 50e3), (-411737.3, 50e3, 50e3)],
                           4096 * 12 + 77, [1, 999, 4096, 7, 20000], 51, {}),
    # channels landed without resampling, a wide one (decimation 4), a
    # narrow one (decimation 128, resampled)
    "n4096_mixed": (4096, 1, [(-500e3, 50e3, 75e3), (0.0, 400e3, 600e3), (1e6, 10e3, 12.5e3)],
                    4096 * 10 + 5, [5000, 3, 12288], 52, {}),
    # three elements, add / remove / retune between blocks
    "n1024_nel3_events": (1024, 3, [(200e3, 50e3, 37.5e3), (-123456.7, 25e3, 20e3)],
                          1024 * 24 + 11, [700, 1, 2500, 1024], 53,
                          {2: ("add", 650e3, 100e3, 150e3), 4: ("remove", 0),
                           6: ("retune", 1, 333333.3), 8: ("add", -90e3, 30e3, 37.5e3)}),
    # the smallest transform, decimation 2 and 1
    "n64_small": (64, 2, [(100e3, 200e3, 300e3), (-300e3, 300e3, 1.2e6)],
                  64 * 100 + 3, [1, 63, 64, 65, 500], 54, {}),
    # transforms larger than one CTA's shared memory
    "n16384": (16384, 1, [(300e3, 50e3, 50e3), (717e3, 5e3, 4e3), (-1e6, 600e3, 800e3)],
               16384 * 4 + 9, [10000, 30000], 55, {}),
}


def signal(n: int, nel: int, seed: int) -> list[np.ndarray]:
    """Unit-power complex noise plus three tones per element (seeded)."""
    rng = np.random.default_rng(seed)
    k = np.arange(n)
    out = []
    for _ in range(nel):
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * np.sqrt(0.5)
        for _ in range(3):
            f = rng.uniform(-0.45, 0.45)
            x = x + 3.0 * np.exp(2j * np.pi * (f * k + rng.uniform()))
        out.append(x.astype(np.complex64))
    return out


def run_case(osx_factory, name: str, xs=None):
    """Replay case `name`; returns (per-slot outputs [nel][n] or None, counts
    per slot, slot list). `osx_factory(fs, nfft, max_nel)` makes the object."""
    nfft, nel, chans, n, pattern, seed, events = OSX_CASES[name]
    if xs is None:
        xs = signal(n, nel, seed)
    o = osx_factory(FS, nfft, nel)
    for c in chans:
        o.add(*c)
    acc: dict[int, list] = {}
    pos, bi = 0, 0
    while pos < n:
        ev = events.get(bi)
        if ev is not None:
            if ev[0] == "remove":
                o.remove(ev[1])
            elif ev[0] == "retune":
                o.retune(ev[1], ev[2])
            else:
                o.add(*ev[1:])
        b = min(pattern[bi % len(pattern)], n - pos)
        bi += 1
        y, cnt = o.process_n([x[pos:pos + b] for x in xs], nel, cap=b + nfft)
        for ci, yc in enumerate(y):
            if yc is not None and cnt[ci]:
                acc.setdefault(ci, []).append(np.asarray(yc))
        pos += b
    slots = sorted(acc)
    return {ci: np.concatenate(acc[ci], axis=-1) for ci in slots}, xs
