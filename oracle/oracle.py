"""ctypes front end for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Two libraries share one Python interface here:

* ``liboracle.so`` -- this repository's C restatement of the reference's
  channelizer / unpack algorithm (``oracle/pfb_oracle.c``);
* ``_ref/libatkdsp_ref.so`` -- the reference library itself, compiled from its
  own sources by ``oracle/Makefile`` (present only where it was built).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module. The product (``atkdsp_b200``) never imports it.

The Python surface mirrors the reference binding (python/atkdsp/__init__.py:
``Pfb`` at :4159-4219, ``unpack``/``unpack_dc`` at :337-385, W1/W2 at
:4222-4266) so a parity test reads the same against either side.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libatkdsp_ref.so"

FMT = {"cu8": 0, "ci8": 1, "ci16": 2, "ci16q11": 3, "cf32": 4}


class _Cf32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


_P = C.POINTER
_pcf = _P(_Cf32)


def _cfp(a: np.ndarray):
    return a.ctypes.data_as(_pcf)


def _fmt(f) -> int:
    return FMT[f] if isinstance(f, str) else int(f)


class CpuLib:
    """One of the two CPU libraries, behind the reference binding's surface."""

    def __init__(self, path: Path, prefix: str):
        self.path = Path(path)
        if not self.path.exists():
            raise FileNotFoundError(f"{self.path} is not built (make -C oracle)")
        self.lib = C.CDLL(str(self.path))
        self.prefix = prefix
        self._bind()

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def _bind(self):
        vp, sz, u, d, i64 = C.c_void_p, C.c_size_t, C.c_uint, C.c_double, C.c_int64
        f = self._f
        f("pfb_create").argtypes = [d, u, u, u, d, u]
        f("pfb_create").restype = vp
        f("pfb_destroy").argtypes = [vp]
        f("pfb_destroy").restype = None
        f("pfb_reset").argtypes = [vp]
        f("pfb_reset").restype = None
        f("pfb_out_hops").argtypes = [vp, sz]
        f("pfb_out_hops").restype = sz
        f("pfb_process_n").argtypes = [vp, _P(_pcf), u, sz, _pcf, sz]
        f("pfb_process_n").restype = C.c_ssize_t
        f("pfb_set_cal").argtypes = [vp, _pcf, u]
        f("pfb_set_cal").restype = C.c_int
        f("pfb_cov_accumulate" if self.prefix == "atkdsp_" else "cov_accumulate").argtypes = \
            [_pcf, u, u, sz, _P(C.c_uint8), _pcf, _P(C.c_uint32)]
        f("pfb_cov_reset" if self.prefix == "atkdsp_" else "cov_reset").argtypes = \
            [_pcf, _P(C.c_uint32), u, u, _P(C.c_uint8)]
        f("pfb_channel_power" if self.prefix == "atkdsp_" else "channel_power").argtypes = \
            [_pcf, u, u, sz, _P(C.c_float), _P(C.c_float)]
        f("unpack").argtypes = [C.c_void_p, sz, C.c_int, _pcf, sz, C.c_float, _pcf]
        f("unpack").restype = C.c_ssize_t
        f("unpack_dc").argtypes = [C.c_void_p, sz, C.c_int, _pcf, sz, C.c_float, C.c_float,
                                   _P(C.c_double), _P(C.c_double)]
        f("unpack_dc").restype = C.c_ssize_t
        f("bytes_per_sample").argtypes = [C.c_int]
        f("bytes_per_sample").restype = C.c_int
        f("osx_create").argtypes = [d, sz, d, u]
        f("osx_create").restype = vp
        f("osx_destroy").argtypes = [vp]
        f("osx_destroy").restype = None
        f("osx_reset").argtypes = [vp]
        f("osx_reset").restype = None
        f("osx_add").argtypes = [vp, d, d, d]
        f("osx_add").restype = C.c_int
        f("osx_retune").argtypes = [vp, C.c_int, d]
        f("osx_retune").restype = C.c_int
        f("osx_remove").argtypes = [vp, C.c_int]
        f("osx_remove").restype = C.c_int
        f("osx_channels").argtypes = [vp]
        f("osx_channels").restype = C.c_int
        f("osx_chan_rate").argtypes = [vp, C.c_int]
        f("osx_chan_rate").restype = d
        f("osx_out_max").argtypes = [vp, C.c_int, sz]
        f("osx_out_max").restype = sz
        f("osx_process_n").argtypes = [vp, _P(_pcf), u, sz, _P(_pcf), _P(sz), sz]
        f("osx_process_n").restype = C.c_ssize_t
        f("osx_describe").argtypes = [vp, C.c_char_p, sz]
        f("osx_describe").restype = C.c_int
        if self.prefix == "orc_":
            self.lib.orc_window.argtypes = [C.c_int, sz, _P(C.c_float)]
            self.lib.orc_window.restype = C.c_int
            self.lib.orc_spectrum_reduce.argtypes = [sz, _pcf, sz, sz, _P(C.c_float), C.c_int, _P(C.c_float)]
            self.lib.orc_spectrum_reduce.restype = C.c_longlong
            self.lib.orc_spectrum_stats.argtypes = [sz, _pcf, sz, sz, _P(C.c_float)] + [_P(C.c_float)] * 4
            self.lib.orc_spectrum_stats.restype = C.c_longlong
        else:
            self.lib.atkdsp_window.argtypes = [C.c_int, sz, _P(C.c_float)]
            self.lib.atkdsp_window.restype = C.c_int
            self.lib.atkdsp_fft_create.argtypes = [sz]
            self.lib.atkdsp_fft_create.restype = vp
            self.lib.atkdsp_fft_destroy.argtypes = [vp]
            self.lib.atkdsp_fft_destroy.restype = None
            self.lib.atkdsp_spectrum_reduce.argtypes = [vp, _pcf, sz, sz, _P(C.c_float), C.c_int, _P(C.c_float)]
            self.lib.atkdsp_spectrum_reduce.restype = C.c_ssize_t
            self.lib.atkdsp_spectrum_stats.argtypes = [vp, _pcf, sz, sz, _P(C.c_float)] + [_P(C.c_float)] * 4
            self.lib.atkdsp_spectrum_stats.restype = C.c_ssize_t
        if self.prefix == "orc_":
            self.lib.orc_pfb_prototype.argtypes = [u, u, d, _P(C.c_double)]
            self.lib.orc_pfb_prototype.restype = None
        else:
            self.lib.atkdsp_set_threads.argtypes = [C.c_int]
            self.lib.atkdsp_set_threads.restype = C.c_int
            self.lib.atkdsp_get_threads.restype = C.c_int

    # -- the filterbank -------------------------------------------------------
    def Pfb(self, fs, nchan, oversample=2, taps_per_poly=12, atten_db=80.0, max_nel=1):
        return _CpuPfb(self, fs, nchan, oversample, taps_per_poly, atten_db, max_nel)

    def prototype(self, nchan, taps_per_poly, atten_db):
        h = np.zeros(int(nchan) * int(taps_per_poly), np.float64)
        self.lib.orc_pfb_prototype(int(nchan), int(taps_per_poly), float(atten_db),
                                   h.ctypes.data_as(_P(C.c_double)))
        return h

    # -- the spectrum reduction (python/atkdsp/__init__.py:566-600) -------------
    def window(self, kind, n):
        kinds = {"rect": 0, "hann": 1, "hamming": 2, "blackmanharris": 3}
        out = np.empty(int(n), np.float32)
        f = self.lib.orc_window if self.prefix == "orc_" else self.lib.atkdsp_window
        if f(kinds[kind] if isinstance(kind, str) else int(kind), int(n), out.ctypes.data_as(_P(C.c_float))):
            raise RuntimeError("window")
        return out

    def _spec(self, name, n, x, hop, win, *rest):
        x = np.ascontiguousarray(x, np.complex64)
        wp = None if win is None else np.ascontiguousarray(win, np.float32).ctypes.data_as(_P(C.c_float))
        if self.prefix == "orc_":
            return getattr(self.lib, "orc_" + name)(int(n), _cfp(x), x.size, int(hop or n), wp, *rest)
        h = self.lib.atkdsp_fft_create(int(n))
        try:
            return getattr(self.lib, "atkdsp_" + name)(h, _cfp(x), x.size, int(hop or n), wp, *rest)
        finally:
            self.lib.atkdsp_fft_destroy(h)

    def spectrum_reduce(self, x, n, hop=None, win=None, detector="max"):
        det = {"max": 0, "min": 1, "avg": 2}[detector] if isinstance(detector, str) else int(detector)
        out = np.empty(int(n), np.float32)
        fr = self._spec("spectrum_reduce", n, x, hop, win, det, out.ctypes.data_as(_P(C.c_float)))
        if fr < 0:
            raise RuntimeError(f"spectrum_reduce: {fr}")
        return out, int(fr)

    def spectrum_stats(self, x, n, hop=None, win=None):
        outs = {k: np.empty(int(n), np.float32) for k in ("max", "avg", "min", "sk")}
        fr = self._spec("spectrum_stats", n, x, hop, win,
                        *[outs[k].ctypes.data_as(_P(C.c_float)) for k in ("max", "avg", "min", "sk")])
        if fr < 0:
            raise RuntimeError(f"spectrum_stats: {fr}")
        outs["frames"] = int(fr)
        return outs

    # -- the overlap-save extractor ----------------------------------------------
    def Osx(self, fs, nfft=4096, atten_db=80.0, max_nel=1):
        return _CpuOsx(self, fs, nfft, atten_db, max_nel)

    # -- W1 / W2 ---------------------------------------------------------------
    def _w(self, name):
        return self._f(("pfb_" if self.prefix == "atkdsp_" else "") + name)

    def pfb_cov_accumulate(self, out, nel, nchan, gate, R, counts):
        o = np.ascontiguousarray(out, np.complex64)
        m = o.shape[2] if o.ndim == 3 else 0
        gp = None
        if gate is not None:
            g = np.ascontiguousarray(gate, np.uint8)
            gp = g.ctypes.data_as(_P(C.c_uint8))
        self._w("cov_accumulate")(_cfp(o.reshape(-1)), int(nel), int(nchan), m, gp,
                                  _cfp(R.reshape(-1)), counts.ctypes.data_as(_P(C.c_uint32)))

    def pfb_cov_reset(self, R, counts, nel, nchan, gate=None):
        gp = None
        if gate is not None:
            g = np.ascontiguousarray(gate, np.uint8)
            gp = g.ctypes.data_as(_P(C.c_uint8))
        self._w("cov_reset")(_cfp(R.reshape(-1)), counts.ctypes.data_as(_P(C.c_uint32)),
                             int(nel), int(nchan), gp)

    def pfb_channel_power(self, out, nel, nchan):
        o = np.ascontiguousarray(out, np.complex64)
        m = o.shape[2] if o.ndim == 3 else 0
        pwr = np.zeros(int(nel) * int(nchan), np.float32)
        meanp = np.zeros(int(nchan), np.float32)
        self._w("channel_power")(_cfp(o.reshape(-1)), int(nel), int(nchan), m,
                                 pwr.ctypes.data_as(_P(C.c_float)),
                                 meanp.ctypes.data_as(_P(C.c_float)))
        return pwr.reshape(int(nel), int(nchan)), meanp

    # -- unpack ----------------------------------------------------------------
    def bytes_per_sample(self, fmt) -> int:
        return int(self._f("bytes_per_sample")(_fmt(fmt)))

    def unpack(self, raw, fmt, dc_alpha=0.0, dc_state=None):
        src = np.frombuffer(raw, np.uint8) if not isinstance(raw, np.ndarray) \
            else np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
        bps = self.bytes_per_sample(fmt)
        out = np.empty(src.size // bps, np.complex64)
        st = _cfp(dc_state) if (dc_alpha > 0 and dc_state is not None) else None
        got = self._f("unpack")(src.ctypes.data, src.size, _fmt(fmt), _cfp(out), out.size,
                                float(dc_alpha), st)
        if got < 0:
            raise RuntimeError(f"unpack: {got}")
        return out[:got]

    def unpack_dc(self, raw, fmt, offset=0j, want_mean=True):
        src = np.frombuffer(raw, np.uint8) if not isinstance(raw, np.ndarray) \
            else np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
        bps = self.bytes_per_sample(fmt)
        out = np.empty(src.size // bps, np.complex64)
        mr, mi = C.c_double(0.0), C.c_double(0.0)
        got = self._f("unpack_dc")(src.ctypes.data, src.size, _fmt(fmt), _cfp(out), out.size,
                                   float(np.float32(offset.real)), float(np.float32(offset.imag)),
                                   C.byref(mr) if want_mean else None,
                                   C.byref(mi) if want_mean else None)
        if got < 0:
            raise RuntimeError(f"unpack_dc: {got}")
        return out[:got], complex(mr.value, mi.value)


class _CpuPfb:
    def __init__(self, owner: CpuLib, fs, nchan, os_, K, atten, max_nel):
        self._o = owner
        self._p = owner._f("pfb_create")(float(fs), int(nchan), int(os_), int(K), float(atten),
                                         int(max_nel))
        if not self._p:
            raise ValueError("pfb_create rejected its arguments")
        self.nchan = int(nchan)
        self.max_nel = int(max_nel)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            self._o._f("pfb_destroy")(p)
            self._p = None

    def reset(self):
        self._o._f("pfb_reset")(self._p)

    def out_hops(self, n):
        return int(self._o._f("pfb_out_hops")(self._p, int(n)))

    def set_cal(self, table, nel):
        if table is None:
            return self._o._f("pfb_set_cal")(self._p, None, 0)
        t = np.ascontiguousarray(np.asarray(table, np.complex64)).reshape(int(nel), self.nchan)
        return self._o._f("pfb_set_cal")(self._p, _cfp(t), int(nel))

    def process_n(self, ins, nel):
        nel = int(nel)
        arrs = [np.ascontiguousarray(np.asarray(ins[e]).ravel(), np.complex64) for e in range(nel)]
        n = arrs[0].size
        m = self.out_hops(n)
        out = np.zeros(max(nel * self.nchan * m, 1), np.complex64)
        arr = (_pcf * nel)(*[_cfp(a) for a in arrs])
        got = self._o._f("pfb_process_n")(self._p, arr, nel, n, _cfp(out), nel * self.nchan * m)
        if got < 0:
            raise RuntimeError(f"pfb_process_n: {got}")
        return out[: nel * self.nchan * got].reshape(nel, self.nchan, got)

    def process(self, x):
        return self.process_n([x], 1)[0]


class _CpuOsx:
    """The binding's ``Osx`` (python/atkdsp/__init__.py:4269-4342) over a CPU library."""

    def __init__(self, owner: CpuLib, fs, nfft, atten, max_nel):
        self._o = owner
        self._p = owner._f("osx_create")(float(fs), int(nfft), float(atten), int(max_nel))
        if not self._p:
            raise ValueError("osx_create rejected its arguments")
        self.max_nel = int(max_nel)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            self._o._f("osx_destroy")(p)
            self._p = None

    def reset(self):
        self._o._f("osx_reset")(self._p)

    def add(self, offset_hz, bw_hz, out_rate):
        ch = self._o._f("osx_add")(self._p, float(offset_hz), float(bw_hz), float(out_rate))
        if ch < 0:
            raise RuntimeError(f"osx_add: {ch}")
        return ch

    def retune(self, ch, offset_hz):
        rc = self._o._f("osx_retune")(self._p, int(ch), float(offset_hz))
        if rc < 0:
            raise RuntimeError(f"osx_retune: {rc}")

    def remove(self, ch):
        rc = self._o._f("osx_remove")(self._p, int(ch))
        if rc < 0:
            raise RuntimeError(f"osx_remove: {rc}")

    def channels(self):
        return int(self._o._f("osx_channels")(self._p))

    def chan_rate(self, ch):
        return float(self._o._f("osx_chan_rate")(self._p, int(ch)))

    def out_max(self, ch, n):
        return int(self._o._f("osx_out_max")(self._p, int(ch), int(n)))

    def describe(self):
        buf = C.create_string_buffer(256)
        n = self._o._f("osx_describe")(self._p, buf, 256)
        return buf.value.decode() if n > 0 else ""

    def process_n(self, ins, nel, cap=None):
        """cap: the per-channel capacity passed as cap_each (default the
        binding's, the largest out_max; a larger one admits calls whose
        carried samples complete more hops than out_max allows for)."""
        nel = int(nel)
        arrs = [np.ascontiguousarray(np.asarray(ins[e]).ravel(), np.complex64) for e in range(nel)]
        n = arrs[0].size
        ns = self.channels()
        active = [self.chan_rate(ci) > 0 for ci in range(ns)]
        if cap is None:
            cap = max([self.out_max(ci, n) for ci in range(ns) if active[ci]], default=0)
        bufs = [[np.zeros(cap, np.complex64) if active[ci] else None for ci in range(ns)]
                for _ in range(nel)]
        ptrs = (_pcf * max(nel * ns, 1))()
        for e in range(nel):
            for ci in range(ns):
                ptrs[e * ns + ci] = _cfp(bufs[e][ci]) if active[ci] else None
        counts = (C.c_size_t * max(ns, 1))()
        inarr = (_pcf * nel)(*[_cfp(a) for a in arrs])
        got = self._o._f("osx_process_n")(self._p, inarr, nel, n, ptrs, counts, cap)
        if got < 0:
            raise RuntimeError(f"osx_process_n: {got}")
        cnts = [int(counts[ci]) for ci in range(ns)]
        outs = [None] * ns
        for ci in range(ns):
            if active[ci]:
                outs[ci] = np.array([bufs[e][ci][:cnts[ci]] for e in range(nel)], np.complex64) \
                    if cnts[ci] else np.zeros((nel, 0), np.complex64)
        return outs, cnts

    def process(self, x, cap=None):
        outs, cnts = self.process_n([x], 1, cap)
        return [o[0] if o is not None else None for o in outs], cnts


_cache: dict = {}


def oracle() -> CpuLib:
    """The C restatement (always built by ``make -C oracle``)."""
    if "orc" not in _cache:
        _cache["orc"] = CpuLib(ORACLE_SO, "orc_")
    return _cache["orc"]


def reference() -> CpuLib | None:
    """The reference library built from its own sources, or None if absent."""
    if "ref" not in _cache:
        _cache["ref"] = CpuLib(REF_SO, "atkdsp_") if REF_SO.exists() else None
    return _cache["ref"]


# -- the reference's CFAR (its C library only: the product's is the thing tested)
class _CfarConfig(C.Structure):
    _fields_ = [("mode", C.c_int32), ("n_ref", C.c_int32), ("n_guard", C.c_int32),
                ("k_frames", C.c_int32), ("pfa", C.c_double), ("looks", C.c_double),
                ("os_k", C.c_int32), ("open_m", C.c_int32), ("open_n", C.c_int32),
                ("close_k", C.c_int32), ("merge_gap", C.c_int32), ("min_bins", C.c_int32),
                ("max_tracks", C.c_int32), ("reserved", C.c_int32), ("rho2", C.c_double * 4)]


class _CfarEvent(C.Structure):
    _fields_ = [("t0", C.c_double), ("t1", C.c_double), ("fc_bin", C.c_double),
                ("type", C.c_int32), ("id", C.c_uint32), ("flags", C.c_uint32),
                ("lo_bin", C.c_int32), ("hi_bin", C.c_int32), ("n_hits", C.c_int32),
                ("level_db", C.c_float), ("noise_db", C.c_float), ("snr_db", C.c_float),
                ("band_snr_db", C.c_float)]


class _CfarCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in
                ("frames", "warmup", "cells_tested", "cell_hits", "untestable",
                 "opened", "closed", "updates", "dropped", "resets", "tracks")]


_CFAR_MODES = {"ca": 0, "os": 1, "go": 2, "so": 3}


def _ev_dict(e) -> dict:
    return {"type": int(e.type), "id": int(e.id), "flags": int(e.flags), "lo": int(e.lo_bin),
            "hi": int(e.hi_bin), "n_hits": int(e.n_hits), "t0": float(e.t0), "t1": float(e.t1),
            "fc_bin": float(e.fc_bin), "level_db": float(e.level_db), "noise_db": float(e.noise_db),
            "snr_db": float(e.snr_db), "band_snr_db": float(e.band_snr_db)}


class RefCfar:
    """atkdsp_cfar_* of the reference library, with the surface of the
    reference binding's Cfar (python/atkdsp/__init__.py:2431-2541)."""

    def __init__(self, lib: CpuLib, nbins: int, **cfg):
        L = self._L = lib.lib
        vp, sz, d = C.c_void_p, C.c_size_t, C.c_double
        for name, args, res in (
                ("atkdsp_cfar_defaults", [_P(_CfarConfig)], None),
                ("atkdsp_cfar_create", [sz, _P(_CfarConfig)], vp),
                ("atkdsp_cfar_destroy", [vp], None),
                ("atkdsp_cfar_set_mask", [vp, _P(C.c_uint8)], C.c_int),
                ("atkdsp_cfar_process", [vp, _P(C.c_float), sz, d, d, _P(_CfarEvent), sz], C.c_ssize_t),
                ("atkdsp_cfar_flush", [vp, _P(_CfarEvent), sz], C.c_ssize_t),
                ("atkdsp_cfar_last", [vp, _P(C.c_float), _P(C.c_float), _P(C.c_uint8)], C.c_int),
                ("atkdsp_cfar_info", [vp, _P(d), _P(d), _P(d), _P(_CfarConfig)], C.c_int),
                ("atkdsp_cfar_describe", [vp, C.c_char_p, sz], C.c_int),
                ("atkdsp_cfar_stats", [vp, _P(_CfarCounters)], C.c_int),
                ("atkdsp_cfar_reset", [vp], None)):
            getattr(L, name).argtypes = args
            getattr(L, name).restype = res
        k = _CfarConfig()
        L.atkdsp_cfar_defaults(C.byref(k))
        for key, v in cfg.items():
            if key == "mode" and isinstance(v, str):
                v = _CFAR_MODES[v]
            if key == "rho2":
                k.rho2 = (C.c_double * 4)(*[float(x) for x in v])
            else:
                setattr(k, key, float(v) if key in ("pfa", "looks") else int(v))
        self.nbins = int(nbins)
        self.max_tracks = k.max_tracks
        self._h = L.atkdsp_cfar_create(self.nbins, C.byref(k))
        if not self._h:
            raise ValueError(f"reference cfar_create refused {cfg}")
        a, ac, et = C.c_double(), C.c_double(), C.c_double()
        L.atkdsp_cfar_info(self._h, C.byref(a), C.byref(ac), C.byref(et), None)
        self.alpha, self.alpha_ca, self.et = a.value, ac.value, et.value

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._L.atkdsp_cfar_destroy(h)

    def set_mask(self, mask):
        m = None if mask is None else np.ascontiguousarray(np.asarray(mask) != 0, np.uint8)
        self._L.atkdsp_cfar_set_mask(self._h, None if m is None else m.ctypes.data_as(_P(C.c_uint8)))

    def reset(self):
        self._L.atkdsp_cfar_reset(self._h)

    def process(self, frames_db, frame_t0, frame_dt):
        f = np.ascontiguousarray(frames_db, np.float32).reshape(-1, self.nbins)
        cap = max(1, f.shape[0] * self.max_tracks)
        buf = (_CfarEvent * cap)()
        n = self._L.atkdsp_cfar_process(self._h, f.ctypes.data_as(_P(C.c_float)), f.shape[0],
                                        float(frame_t0), float(frame_dt), buf, cap)
        if n < 0:
            raise ValueError(f"reference cfar_process: {n}")
        return [_ev_dict(buf[j]) for j in range(n)]

    def flush(self):
        buf = (_CfarEvent * self.max_tracks)()
        n = self._L.atkdsp_cfar_flush(self._h, buf, self.max_tracks)
        return [_ev_dict(buf[j]) for j in range(n)]

    def last(self):
        a = np.empty(self.nbins, np.float32)
        t = np.empty(self.nbins, np.float32)
        h = np.empty(self.nbins, np.uint8)
        rc = self._L.atkdsp_cfar_last(self._h, a.ctypes.data_as(_P(C.c_float)),
                                      t.ctypes.data_as(_P(C.c_float)), h.ctypes.data_as(_P(C.c_uint8)))
        return None if rc else (a, t, h)

    def stats(self):
        s = _CfarCounters()
        self._L.atkdsp_cfar_stats(self._h, C.byref(s))
        return {n: int(getattr(s, n)) for n, _t in s._fields_}

    def describe(self):
        buf = C.create_string_buffer(1024)
        self._L.atkdsp_cfar_describe(self._h, buf, 1024)
        return buf.value.decode()
