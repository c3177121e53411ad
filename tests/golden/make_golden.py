"""Generate the committed golden fixtures from the reference itself.

Run in a container that has the reference sources (it reads them; nothing on
the GPU machine does):

    make -C oracle REF=<reference tree>     # builds oracle/_ref/libatkdsp_ref.so
    python tests/golden/make_golden.py [REF_ROOT] [--only NAME ...]

REF_ROOT defaults to the ATKDSP_REFERENCE environment variable.

Every output here is produced by the REFERENCE: its C library (compiled from
its own sources by oracle/Makefile) for float32 results, and its numpy twin
(python/atkdsp/reference.py, imported from REF_ROOT) for the float64
specification values. The inputs are seeded and stored beside the outputs, so
the tests never regenerate them.

Fixture files (tests/golden/*.npz):
  pfb_cases.npz     filterbank outputs at several (nchan, oversample, taps,
                    elements, block pattern) shapes, with cal tables
  pfb_twin.npz      the twin's float64 outputs for three of those cases
  w12.npz           W1 (gated and ungated) and W2 on an element-array output
  unpack.npz        unpack / unpack_dc / DC pole on all five formats
  proto.npz         prototype taps: the twin's (numpy), the C restatement's,
                    and hashes of the C restatement's for long prototypes
  osx.npz           overlap-save extractor outputs per channel slot for the
                    cases of tests/osx_cases.py (reference C library)
  spectrum.npz      spectrum reduction lines (max / min / avg detector) and
                    per-bin stats (max, avg, min dB, spectral kurtosis) from
                    the reference C library run with one thread
  cfar.npz          the CFAR solver over a grid of (mode, n_ref, pfa, looks,
                    os_k, rho2), n_eff and window correlations, and the
                    detector's events, counters and last-frame lines for the
                    cases of tests/cfar_cases.py (reference C library)
"""

from __future__ import annotations

import hashlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from oracle import oracle as O                 # noqa: E402
from atkdsp_b200 import workloads as W         # noqa: E402

sys.path.insert(0, str(HERE.parent))
from osx_cases import OSX_CASES, run_case      # noqa: E402
import cfar_cases                              # noqa: E402

_ARGS = [a for a in sys.argv[1:] if not a.startswith("--")]
ONLY = sys.argv[sys.argv.index("--only") + 1:] if "--only" in sys.argv else None
REF_ROOT = Path(_ARGS[0]) if _ARGS and (ONLY is None or sys.argv.index(_ARGS[0]) < sys.argv.index("--only")) \
    else Path(os.environ["ATKDSP_REFERENCE"])
sys.path.insert(0, str(REF_ROOT / "python"))
from atkdsp import reference as twin           # noqa: E402

FS = 2.4e6

# (name, nchan, oversample, taps, atten, nel, nsamples, block pattern, seed, cal)
PFB_CASES = [
    ("single_stream_m64", 64, 1, 16, W.ATTEN_BETA8, 1, 16384, [1, 999, 4096, 7], 11, False),
    ("m192_os2_uneven", 192, 2, 12, 80.0, 1, 192 * 60, [1, 97, 960, 5000, 65537], 12, False),
    ("m24_os2", 24, 2, 12, 80.0, 1, 24 * 200 + 17, [5, 24 * 7 + 3, 1, 100000], 13, False),
    ("m60_os3_nel2", 60, 3, 12, 80.0, 2, 60 * 100 + 17, [5, 60 * 7 + 3, 1, 100000], 14, False),
    ("m64_os4", 64, 4, 12, 80.0, 1, 64 * 80 + 17, [333], 15, False),
    ("m1026_os2", 1026, 2, 12, 80.0, 1, 1026 * 14, [100000], 16, False),
    ("m1024_os2_k12", 1024, 2, 12, 80.0, 1, 1024 * 16, [5000, 7, 3000], 17, False),
    ("m2048_os1_nel8", 2048, 1, 16, W.ATTEN_BETA8, 8, 2048 * 3 + 5, [2048 * 3 + 5], 18, False),
    ("m4096_os2_k8", 4096, 2, 8, 80.0, 1, 4096 * 5, [9000, 1, 40000], 19, False),
    ("m192_nel5_cal", 192, 2, 12, 80.0, 5, 192 * 25, [2000, 3, 100000], 20, True),
    ("m200_os2_k5_att30", 200, 2, 5, 30.0, 1, 200 * 50, [777], 21, False),
    ("m2_os2_k2", 2, 2, 2, 10.0, 1, 999, [3, 1, 50], 22, False),
]
TWIN_CASES = ("single_stream_m64", "m192_os2_uneven", "m1024_os2_k12")


def _signal(n, nel, seed):
    rng = np.random.default_rng(seed)
    return [W.tones_noise(n, 3, 20.0, rng) for _ in range(nel)]


def _run_blocks(p, xs, pattern):
    n = xs[0].size
    nel = len(xs)
    outs, pos, bi = [], 0, 0
    while pos < n:
        b = min(pattern[bi % len(pattern)], n - pos)
        bi += 1
        o = np.asarray(p.process_n([x[pos:pos + b] for x in xs], nel))
        if o.shape[-1]:
            outs.append(o)
        pos += b
    return np.concatenate(outs, axis=-1)


def make_pfb(ref):
    data, tw = {}, {}
    for name, M, os_, K, att, nel, n, pattern, seed, cal in PFB_CASES:
        xs = _signal(n, nel, seed)
        p = ref.Pfb(FS, M, os_, K, att, nel)
        table = None
        if cal:
            rng = np.random.default_rng(seed + 1000)
            table = (rng.standard_normal((nel, M)) + 1j * rng.standard_normal((nel, M))).astype(np.complex64)
            p.set_cal(table, nel)
        y = _run_blocks(p, xs, pattern)
        data[f"{name}/in"] = np.stack(xs)
        data[f"{name}/out"] = y.astype(np.complex64)
        data[f"{name}/params"] = np.array([M, os_, K, nel, n], np.int64)
        data[f"{name}/atten"] = np.array([att], np.float64)
        data[f"{name}/pattern"] = np.array(pattern, np.int64)
        if cal:
            data[f"{name}/cal"] = table
        if name in TWIN_CASES:
            t = twin.Pfb(FS, M, os_, K, att, nel)
            yt = _run_blocks(t, [x.astype(np.complex128) for x in xs], pattern)
            tw[f"{name}/out"] = yt
        print(f"{name}: out {y.shape}")
    return data, tw


def make_w12(ref):
    M, nel = 192, 5
    rng = np.random.default_rng(31)
    base = W.tones_noise(192 * 30, 2, 15.0, rng)
    phi = np.deg2rad(37.0)
    ins = [(base * np.exp(1j * e * phi)).astype(np.complex64) for e in range(nel)]
    y = ref.Pfb(FS, M, 2, 12, 80.0, nel).process_n(ins, nel)
    R = (rng.standard_normal((M, nel, nel)) + 1j * rng.standard_normal((M, nel, nel))).astype(np.complex64)
    counts = rng.integers(0, 1000, M).astype(np.uint32)
    R0, c0 = R.copy(), counts.copy()
    ref.pfb_cov_accumulate(y, nel, M, None, R, counts)
    gate = (rng.random(M) < 0.3).astype(np.uint8)
    Rg, cg = R0.copy(), c0.copy()
    ref.pfb_cov_accumulate(y, nel, M, gate, Rg, cg)
    Rr, cr = Rg.copy(), cg.copy()
    ref.pfb_cov_reset(Rr, cr, nel, M, gate)
    pwr, meanp = ref.pfb_channel_power(y, nel, M)
    return {"y": y, "R0": R0, "c0": c0, "R": R, "counts": counts, "gate": gate,
            "Rg": Rg, "cg": cg, "Rr": Rr, "cr": cr, "pwr": pwr, "meanp": meanp}


def make_unpack(ref):
    rng = np.random.default_rng(41)
    out = {}
    for f in ("cu8", "ci8", "ci16", "ci16q11", "cf32"):
        if f == "cu8":
            raw = rng.integers(0, 256, 8001, dtype=np.uint8).tobytes()
        elif f == "ci8":
            raw = rng.integers(-128, 128, 8001, dtype=np.int8).tobytes()
        elif f == "cf32":
            raw = rng.standard_normal(4001).astype("<f4").tobytes()[:-1]
        else:
            raw = rng.integers(-2048, 2048, 4001, dtype="<i2").tobytes()[:-1]
        out[f"{f}/raw"] = np.frombuffer(raw, np.uint8).copy()
        out[f"{f}/plain"] = ref.unpack(raw, f)
        for j, off in enumerate((0j, 0.123 - 0.045j, -0.031 + 0.017j)):
            y, mean = ref.unpack_dc(raw, f, off)
            out[f"{f}/dc{j}"] = y
            out[f"{f}/mean{j}"] = np.array([mean.real, mean.imag])
            out[f"{f}/off{j}"] = np.array([off.real, off.imag], np.float32)
        st = np.zeros(1, np.complex64)
        ys = []
        bps = ref.bytes_per_sample(f)
        cuts = [0, 40 * bps, 40 * bps + bps, len(raw)]
        for a, b in zip(cuts[:-1], cuts[1:]):
            ys.append(ref.unpack(raw[a:b], f, 0.01, st))
        out[f"{f}/pole"] = np.concatenate(ys)
        out[f"{f}/pole_state"] = st.copy()
    return out


def make_proto():
    orc = O.oracle()
    out = {}
    for i, (M, K, att) in enumerate(((64, 16, W.ATTEN_BETA8), (192, 12, 80.0), (256, 8, 80.0),
                                     (24, 12, 10.0))):
        out[f"params{i}"] = np.array([M, K, att], np.float64)
        out[f"h{i}"] = orc.prototype(M, K, att)
        out[f"twin{i}"] = twin.pfb_prototype(M, K, att)
    for i, (M, K, att) in enumerate(((1024, 12, 80.0), (2048, 16, W.ATTEN_BETA8), (4096, 16, 80.0))):
        h = orc.prototype(M, K, att)
        out[f"shaparams{i}"] = np.array([M, K, att], np.float64)
        out[f"sha{i}"] = np.frombuffer(hashlib.sha256(h.astype("<f8").tobytes()).digest(), np.uint8).copy()
    return out


def make_osx(ref):
    out = {}
    for name in OSX_CASES:
        ys, xs = run_case(lambda fs, nfft, nel: ref.Osx(fs, nfft, 80.0, nel), name)
        out[f"{name}/in"] = np.stack(xs)
        for ci, y in ys.items():
            out[f"{name}/out{ci}"] = y.astype(np.complex64)
        print(f"{name}: " + ", ".join(f"slot {ci}: {y.shape}" for ci, y in ys.items()))
    return out


# (name, n, hop, window kind or None, detector, samples, seed)
SPECTRUM_CASES = [
    ("n64_rect_avg", 64, 0, None, "avg", 5000, 61),
    ("n1024_hann_max_hop512", 1024, 512, "hann", "max", 40000, 62),
    ("n4096_bh_min_hop1000", 4096, 1000, "blackmanharris", "min", 70000, 63),
    ("n256_hamming_avg_hop100", 256, 100, "hamming", "avg", 30000, 64),
    ("n16_rect_max_hop3", 16, 3, None, "max", 100, 65),
    ("n2048_hann_avg_one_frame", 2048, 2048, "hann", "avg", 3000, 66),
]


def make_spectrum(ref):
    ref.lib.atkdsp_set_threads(1)      # frames in order: the sums have one rounding sequence
    out = {}
    kinds = {"rect": 0, "hann": 1, "hamming": 2, "blackmanharris": 3}
    for name, n, hop, win, det, N, seed in SPECTRUM_CASES:
        rng = np.random.default_rng(seed)
        k = np.arange(N)
        x = ((rng.standard_normal(N) + 1j * rng.standard_normal(N)) * 0.3
             + np.exp(2j * np.pi * rng.uniform(-0.5, 0.5) * k)).astype(np.complex64)
        w = None if win is None else ref.window(win, n)
        line, frames = ref.spectrum_reduce(x, n, hop, w, det)
        st = ref.spectrum_stats(x, n, hop, w)
        out[f"{name}/in"] = x
        out[f"{name}/params"] = np.array([n, hop, -1 if win is None else kinds[win],
                                          {"max": 0, "min": 1, "avg": 2}[det], frames], np.int64)
        out[f"{name}/line"] = line
        for q in ("max", "avg", "min", "sk"):
            out[f"{name}/{q}"] = st[q]
        print(f"{name}: {frames} frames")
    ref.lib.atkdsp_set_threads(0)
    return out


# the solver grid: (mode, n_ref, pfa, looks, os_k, rho2 or None)
CFAR_RHO = {"none": None, "hann": (4 / 9, 1 / 36, 0.0, 0.0), "mild": (0.3, 0.05, 0.01, 0.0)}
CFAR_ALPHA_GRID = [(mode, nref, pfa, looks, os_k, rho)
                   for mode in range(4) for nref in (1, 3, 16, 64, 256) for pfa in (0.5, 1e-3, 1e-6, 1e-15)
                   for looks in (0.25, 1.0, 7.5, 400.0) for os_k in (0, 1) for rho in CFAR_RHO
                   if not (os_k and mode != 1)]


def make_cfar(ref):
    import ctypes as C
    L = ref.lib
    L.atkdsp_cfar_alpha.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.atkdsp_cfar_alpha.restype = C.c_int
    L.atkdsp_cfar_n_eff.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.atkdsp_cfar_n_eff.restype = C.c_double
    L.atkdsp_cfar_window_rho2.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_double)]
    L.atkdsp_cfar_window_rho2.restype = C.c_int
    out = {}
    grid, res = [], []
    for mode, nref, pfa, looks, os_k, rho in CFAR_ALPHA_GRID:
        r = None if CFAR_RHO[rho] is None else (C.c_double * 4)(*CFAR_RHO[rho])
        a, e = C.c_double(), C.c_double()
        rc = L.atkdsp_cfar_alpha(mode, nref, pfa, looks, os_k, r, C.byref(a), C.byref(e))
        grid.append([mode, nref, pfa, looks, os_k, list(CFAR_RHO).index(rho)])
        res.append([rc, a.value if rc == 0 else np.nan, e.value if rc == 0 else np.nan])
    out["alpha/grid"] = np.array(grid, np.float64)
    out["alpha/res"] = np.array(res, np.float64)
    out["alpha/rho"] = np.array([v or (0.0,) * 4 for v in CFAR_RHO.values()], np.float64)
    neff = []
    for nref in range(0, 12):
        for rho in CFAR_RHO.values():
            r = None if rho is None else (C.c_double * 4)(*rho)
            neff.append([nref, 0 if rho is None else 1 + list(CFAR_RHO.values()).index(rho) - 1,
                         L.atkdsp_cfar_n_eff(nref, r)])
    out["n_eff"] = np.array(neff, np.float64)
    for kind in ("rect", "hann", "hamming", "blackmanharris"):
        for n in (16, 1000, 4096):
            w = ref.window(kind, n)
            r = (C.c_double * 4)()
            assert L.atkdsp_cfar_window_rho2(w.ctypes.data_as(C.POINTER(C.c_float)), n, r) == 0
            out[f"rho2/{kind}/{n}"] = np.array(list(r))
    print(f"alpha grid: {len(grid)} points, {sum(1 for v in res if v[0] == 0)} solved")
    for name in cfar_cases.CFAR_CASES:
        xs = cfar_cases.frames(name)
        ev, last, st, desc, al = cfar_cases.run_case(lambda nb, **cfg: O.RefCfar(ref, nb, **cfg), name, xs)
        out[f"{name}/in"] = xs
        out[f"{name}/events"] = ev
        out[f"{name}/stats"] = np.array([st[k] for k in sorted(st)], np.uint64)
        out[f"{name}/describe"] = np.array(desc)
        out[f"{name}/alpha"] = np.array(al)
        if last is not None:
            out[f"{name}/last_avg"], out[f"{name}/last_thr"], out[f"{name}/last_hits"] = last
        print(f"{name}: {len(ev)} events, stats {st}")
    return out


def main():
    ref = O.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libatkdsp_ref.so is not built: run make -C oracle")
    want = (lambda k: ONLY is None or k in ONLY)
    if want("pfb"):
        data, tw = make_pfb(ref)
        np.savez_compressed(HERE / "pfb_cases.npz", **data)
        np.savez_compressed(HERE / "pfb_twin.npz", **tw)
    if want("w12"):
        np.savez_compressed(HERE / "w12.npz", **make_w12(ref))
    if want("unpack"):
        np.savez_compressed(HERE / "unpack.npz", **make_unpack(ref))
    if want("proto"):
        np.savez_compressed(HERE / "proto.npz", **make_proto())
    if want("osx"):
        np.savez_compressed(HERE / "osx.npz", **make_osx(ref))
    if want("spectrum"):
        np.savez_compressed(HERE / "spectrum.npz", **make_spectrum(ref))
    if want("cfar"):
        np.savez_compressed(HERE / "cfar.npz", **make_cfar(ref))
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
