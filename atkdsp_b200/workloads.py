"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is involved anywhere: every workload is generated here from
a fixed seed, so the bench, the tests and the golden-fixture script all see
the same samples for the same arguments.

Shapes (one function each):
  * ``single_stream``   -- M=64 critically sampled, 16 taps/branch, beta=8,
                           2^20 cf32 of unit-variance complex noise plus three
                           tones at 20 dB SNR, fed in blocks 1, 999, 4096, 7.
  * ``front_end_raw``   -- 40 MS/s front end: ci16q11 (12-bit values in int16
                           containers, /2048) carrying noise, eight tones and a
                           constant complex DC offset, clipped to [-2048, 2047];
                           2,000,000-sample (50 ms) blocks into an M=1024, 2x
                           oversampled, 12 taps/branch filterbank.
  * ``coherent_array``  -- 8 element streams sharing M=2048, 16 taps/branch:
                           four common tones with seeded per-element phases
                           and independent noise at 10 dB SNR.
  * ``uneven_streams``  -- 256 independent streams, lengths log-uniform in
                           [2^14, 2^22], M from {64, 256, 1024, 4096}, taps
                           per branch from {8, 12, 16}, 2x oversampled, each
                           noise plus 1-5 tones, fed as 3 successive blocks.
  * ``served_streams``  -- 4096 live streams at {2.4, 10, 40} MS/s delivering
                           1.6 ms ci16 blocks, M from {256, 1024}, 16 taps.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

#: Kaiser beta = 8 expressed as the stopband the prototype design takes
#: (beta = 0.1102 (A - 8.7) above 50 dB).
ATTEN_BETA8 = 8.0 / 0.1102 + 8.7


def tones_noise(n: int, ntones: int, snr_db: float, rng: np.random.Generator,
                noise_power: float = 1.0, t0: int = 0) -> np.ndarray:
    """Complex white Gaussian noise of the given power plus ``ntones`` complex
    tones at uniform random frequencies in [-0.5, 0.5) cycles/sample, each at
    ``snr_db`` above the noise power."""
    sd = math.sqrt(noise_power / 2.0)
    x = (rng.standard_normal(n) * sd + 1j * rng.standard_normal(n) * sd)
    amp = math.sqrt(noise_power * 10.0 ** (snr_db / 10.0))
    t = np.arange(t0, t0 + n, dtype=np.float64)
    for _ in range(ntones):
        f = rng.uniform(-0.5, 0.5)
        ph = rng.uniform(0.0, 2.0 * math.pi)
        x = x + amp * np.exp(1j * (2.0 * math.pi * f * t + ph))
    return x.astype(np.complex64)


def single_stream(n: int = 1 << 20, seed: int = 1) -> np.ndarray:
    return tones_noise(n, 3, 20.0, np.random.default_rng(seed))


SINGLE_STREAM_BLOCKS = (1, 999, 4096, 7)

#: the DC offset carried by the front-end samples, in LSB of the 12-bit scale
FRONT_END_DC_LSB = (120.0, -80.0)


def front_end_raw(n: int, seed: int = 2) -> np.ndarray:
    """ci16q11 samples as an (n, 2) int16 array (I, Q interleaved)."""
    rng = np.random.default_rng(seed)
    sig = tones_noise(n, 8, 10.0, rng, noise_power=2.0 * 64.0 ** 2).astype(np.complex128)
    sig += FRONT_END_DC_LSB[0] + 1j * FRONT_END_DC_LSB[1]
    iq = np.empty((n, 2), np.float64)
    iq[:, 0] = np.rint(sig.real)
    iq[:, 1] = np.rint(sig.imag)
    return np.clip(iq, -2048, 2047).astype("<i2")


def coherent_array(n: int, nel: int = 8, seed: int = 3) -> list:
    rng = np.random.default_rng(seed)
    freqs = rng.uniform(-0.5, 0.5, 4)
    t = np.arange(n, dtype=np.float64)
    amp = math.sqrt(10.0)                                  # 10 dB over unit noise
    outs = []
    for _ in range(nel):
        phase = rng.uniform(0.0, 2.0 * math.pi, 4)
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / math.sqrt(2.0)
        for f, ph in zip(freqs, phase):
            x = x + amp * np.exp(1j * (2.0 * math.pi * f * t + ph))
        outs.append(x.astype(np.complex64))
    return outs


@dataclass
class StreamSpec:
    nchan: int
    taps: int
    oversample: int
    length: int            # samples per block
    seed: int


def uneven_streams(count: int = 256, seed: int = 4, min_log2: float = 14.0,
                   max_log2: float = 22.0) -> list:
    rng = np.random.default_rng(seed)
    specs = []
    for s in range(count):
        length = int(2.0 ** rng.uniform(min_log2, max_log2))
        specs.append(StreamSpec(nchan=int(rng.choice([64, 256, 1024, 4096])),
                                taps=int(rng.choice([8, 12, 16])), oversample=2,
                                length=length, seed=int(rng.integers(1 << 30))))
    return specs


def stream_samples(spec: StreamSpec, block: int) -> np.ndarray:
    """Block ``block`` (0, 1, 2, ...) of a stream: noise plus 1-5 tones, with
    the tone phases continuous across blocks."""
    rng = np.random.default_rng(spec.seed)
    ntones = int(rng.integers(1, 6))
    freqs = rng.uniform(-0.5, 0.5, ntones)
    phases = rng.uniform(0, 2 * math.pi, ntones)
    nrng = np.random.default_rng([spec.seed, block])
    n = spec.length
    x = (nrng.standard_normal(n) + 1j * nrng.standard_normal(n)) / math.sqrt(2.0)
    t = np.arange(block * n, (block + 1) * n, dtype=np.float64)
    for f, ph in zip(freqs, phases):
        x = x + 10.0 * np.exp(1j * (2 * math.pi * f * t + ph))
    return x.astype(np.complex64)


@dataclass
class ServedSpec:
    rate: float            # samples/s
    nchan: int
    block: int             # samples per 1.6 ms block
    seed: int


SERVED_RATES = (2.4e6, 10e6, 40e6)
SERVED_BLOCK_S = 1.6e-3


def served_streams(count: int = 4096, seed: int = 5) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        rate = float(rng.choice(SERVED_RATES))
        out.append(ServedSpec(rate=rate, nchan=int(rng.choice([256, 1024])),
                              block=int(round(rate * SERVED_BLOCK_S)),
                              seed=int(rng.integers(1 << 30))))
    return out


def ci16_block(n: int, seed: int, block: int) -> np.ndarray:
    """A ci16 block (n, 2) int16: noise plus two tones, full-scale 32768."""
    rng = np.random.default_rng([seed, block])
    x = tones_noise(n, 2, 15.0, rng, noise_power=2.0 * 600.0 ** 2, t0=block * n)
    iq = np.stack([np.rint(x.real), np.rint(x.imag)], axis=1)
    return np.clip(iq, -32768, 32767).astype("<i2")


# ---- the overlap-save extractor ---------------------------------------------
EXTRACTOR_FS = 61.44e6
EXTRACTOR_NFFT = 4096


def extractor_channels(nch: int = 64, fs: float = EXTRACTOR_FS, seed: int = 9) -> list:
    """A many-channel extractor plan: nch channels at seeded offsets across
    +-0.45 fs, bandwidths cycling 12.5 / 25 / 50 / 200 kHz; odd channels land
    at 1.25 x bw (their decimated rate: no resampling), even ones at 1.0 x bw
    (through the arbitrary resampler). Returns (offset_hz, bw_hz, out_rate)."""
    rng = np.random.default_rng(seed)
    bws = (12.5e3, 25e3, 50e3, 200e3)
    return [(float(rng.uniform(-0.45, 0.45) * fs), bws[i % 4], bws[i % 4] * (1.25 if i % 2 else 1.0))
            for i in range(nch)]


# ---- Undertow's per-scale filterbank bank -----------------------------------
def scale_bank(nscales: int = 6, nchan0: int = 8, taps: int = 12) -> list:
    """The dyadic bank Undertow runs on every input chunk (reference
    src/undertow.c:87-95, :112-143): scale s has nchan0 << s channels, 2x
    oversampled, taps per branch as configured (12 by default), 80 dB.
    Returns (nchan, oversample, taps) per scale."""
    return [(nchan0 << s, 2, taps) for s in range(nscales)]


SCALE_BANK_BLOCK = 65536      # Undertow's max_block: samples per chunk (src/undertow.c:95)
