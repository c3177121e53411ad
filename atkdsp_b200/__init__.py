"""atkdsp_b200 -- the atkdsp channelizer path on B200, with atkdsp's Python surface.

This package loads ``lib/libatkdsp_b200.so`` (built in-tree by ``make -C
atkdsp_b200``), a C-ABI library that exports the reference's
``atkdsp_pfb_*`` / ``atkdsp_unpack*`` entry points and runs them on the GPU.
The Python names, arguments, return shapes and errors below mirror the
reference binding's (python/atkdsp/__init__.py: ``Pfb`` at :4159-4219,
``unpack`` / ``unpack_dc`` at :337-385, W1/W2 at :4222-4266, ``Osx`` at
:4269-4342, ``Cfar`` / ``cfar_alpha`` / ``cfar_n_eff`` / ``cfar_window_rho2``
at :2315-2541, identity at :285-313), so code and tests written against ``atkdsp`` read the same here.

There is no CPU fallback: if the library is missing or no GPU is usable,
``load()`` / ``Pfb(...)`` raise ``AtkDspError``.

Every call releases the GIL (ctypes foreign calls) and is synchronous on
return, like the reference's.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = ["ABI_VERSION", "AtkDspError", "load", "available", "lib_path", "version",
           "build_info", "set_threads", "get_threads", "FMT", "bytes_per_sample",
           "unpack", "unpack_dc", "Pfb", "pfb_cov_accumulate", "pfb_cov_reset",
           "pfb_channel_power", "Osx", "Cfar", "cfar_defaults", "cfar_alpha", "cfar_n_eff",
           "cfar_window_rho2", "CFAR_MODES", "CFAR_OPEN", "CFAR_UPDATE", "CFAR_CLOSE",
           "CFAR_T0_COARSE", "CFAR_T1_COARSE", "CFAR_EDGE", "CFAR_MASK_ADJ", "CFAR_FLUSHED",
           "E_EMPTY"]

#: the ABI the library reports (the reference's, include/atkdsp.h:63)
ABI_VERSION = 26

FMT = {"cu8": 0, "ci8": 1, "ci16": 2, "ci16_le": 2, "cs16": 2,
       "ci16q11": 3, "cf32": 4, "cf32_le": 4}

_ERRORS = {-1: "bad argument", -2: "out of memory", -3: "output buffer too small",
           -4: "FFT backend failure", -7: "nothing to return"}
E_EMPTY = -7

HERE = Path(__file__).resolve().parent
LIB_FILE = HERE / "lib" / "libatkdsp_b200.so"

_lib = None
_lib_path: Path | None = None


class AtkDspError(RuntimeError):
    pass


class _Cf32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class _CfarConfig(C.Structure):
    """atkdsp_cfar_config (96 bytes)"""
    _fields_ = [("mode", C.c_int32), ("n_ref", C.c_int32), ("n_guard", C.c_int32),
                ("k_frames", C.c_int32), ("pfa", C.c_double), ("looks", C.c_double),
                ("os_k", C.c_int32), ("open_m", C.c_int32), ("open_n", C.c_int32),
                ("close_k", C.c_int32), ("merge_gap", C.c_int32), ("min_bins", C.c_int32),
                ("max_tracks", C.c_int32), ("reserved", C.c_int32), ("rho2", C.c_double * 4)]


class _CfarEvent(C.Structure):
    """atkdsp_cfar_event (64 bytes)"""
    _fields_ = [("t0", C.c_double), ("t1", C.c_double), ("fc_bin", C.c_double),
                ("type", C.c_int32), ("id", C.c_uint32), ("flags", C.c_uint32),
                ("lo_bin", C.c_int32), ("hi_bin", C.c_int32), ("n_hits", C.c_int32),
                ("level_db", C.c_float), ("noise_db", C.c_float), ("snr_db", C.c_float),
                ("band_snr_db", C.c_float)]


class _CfarCounters(C.Structure):
    """atkdsp_cfar_counters (88 bytes)"""
    _fields_ = [(n, C.c_uint64) for n in
                ("frames", "warmup", "cells_tested", "cell_hits", "untestable",
                 "opened", "closed", "updates", "dropped", "resets", "tracks")]


def _check(rc: int, what: str) -> int:
    if rc < 0:
        raise AtkDspError(f"{what}: {_ERRORS.get(rc, f'error {rc}')}")
    return rc


def _bind(lib) -> None:
    P = C.POINTER
    vp, sz, u, d, i64, ssz = C.c_void_p, C.c_size_t, C.c_uint, C.c_double, C.c_int64, C.c_ssize_t
    pcf, ppcf = P(_Cf32), P(P(_Cf32))
    sigs = {
        "atkdsp_abi_version": ([], C.c_int),
        "atkdsp_version_string": ([], C.c_char_p),
        "atkdsp_build_info": ([], C.c_char_p),
        "atkdsp_bytes_per_sample": ([C.c_int], C.c_int),
        "atkdsp_set_threads": ([C.c_int], C.c_int),
        "atkdsp_get_threads": ([], C.c_int),
        "atkdsp_unpack": ([vp, sz, C.c_int, pcf, sz, C.c_float, pcf], ssz),
        "atkdsp_unpack_dc": ([vp, sz, C.c_int, pcf, sz, C.c_float, C.c_float, P(d), P(d)], ssz),
        "atkdsp_pfb_create": ([d, u, u, u, d, u], vp),
        "atkdsp_pfb_destroy": ([vp], None),
        "atkdsp_pfb_reset": ([vp], None),
        "atkdsp_pfb_nchan": ([vp], u),
        "atkdsp_pfb_out_rate": ([vp], d),
        "atkdsp_pfb_out_hops": ([vp, sz], sz),
        "atkdsp_pfb_process": ([vp, pcf, sz, pcf, sz], ssz),
        "atkdsp_pfb_process_n": ([vp, ppcf, u, sz, pcf, sz], ssz),
        "atkdsp_pfb_block_origin": ([vp, i64], i64),
        "atkdsp_pfb_group_delay": ([vp], d),
        "atkdsp_pfb_set_cal": ([vp, pcf, u], C.c_int),
        "atkdsp_pfb_describe": ([vp, C.c_char_p, sz], C.c_int),
        "atkdsp_pfb_cov_accumulate": ([pcf, u, u, sz, P(C.c_uint8), pcf, P(C.c_uint32)], None),
        "atkdsp_pfb_cov_reset": ([pcf, P(C.c_uint32), u, u, P(C.c_uint8)], None),
        "atkdsp_pfb_channel_power": ([pcf, u, u, sz, P(C.c_float), P(C.c_float)], None),
        # device-pointer entry points (include/atkdsp_gpu.h)
        "atkdsp_gpu_pfb_stream": ([vp], vp),
        "atkdsp_gpu_pfb_sync": ([vp], C.c_int),
        "atkdsp_gpu_pfb_process_n": ([vp, P(vp), u, sz, vp, sz, vp], ssz),
        "atkdsp_gpu_pfb_process_n_raw": ([vp, P(vp), u, sz, C.c_int, C.c_float, C.c_float, vp, sz, vp], ssz),
        "atkdsp_gpu_pfb_w12_scratch_bytes": ([vp, sz], sz),
        "atkdsp_gpu_pfb_process_w12": ([vp, vp, sz, C.c_int, C.c_float, C.c_float, vp, sz, vp, vp, vp, vp, vp,
                                        vp, sz, vp], ssz),
        "atkdsp_gpu_batch_process_raw": ([vp, P(vp), P(sz), C.c_int, P(C.c_float), P(vp), P(ssz), vp], ssz),
        "atkdsp_gpu_unpack_dc_noalloc": ([vp, sz, C.c_int, vp, sz, C.c_float, C.c_float, vp, vp], ssz),
        "atkdsp_gpu_unpack_dc": ([vp, sz, C.c_int, vp, sz, C.c_float, C.c_float, vp, vp], ssz),
        "atkdsp_gpu_unpack": ([vp, sz, C.c_int, vp, sz, C.c_float, vp, vp], ssz),
        "atkdsp_gpu_block_mean": ([vp, sz, C.c_int, C.c_float, C.c_float, vp, vp], ssz),
        "atkdsp_gpu_block_mean_dev": ([vp, sz, C.c_int, vp, vp, vp], ssz),
        "atkdsp_gpu_pfb_process_w12_dev": ([vp, vp, sz, C.c_int, vp, vp, sz, vp, vp, vp, vp, vp, vp, sz, vp], ssz),
        "atkdsp_gpu_pfb_accumulate": ([vp, u, u, sz, vp, vp, vp, vp, vp, vp], C.c_int),
        "atkdsp_gpu_pfb_cov_accumulate": ([vp, u, u, sz, vp, vp, vp, vp], C.c_int),
        "atkdsp_gpu_pfb_cov_reset": ([vp, vp, u, u, vp, vp], C.c_int),
        "atkdsp_gpu_pfb_channel_power": ([vp, u, u, sz, vp, vp, vp], C.c_int),
        "atkdsp_gpu_batch_create": ([P(vp), u, C.c_int], vp),
        "atkdsp_gpu_batch_destroy": ([vp], None),
        "atkdsp_gpu_batch_process": ([vp, P(vp), P(sz), P(vp), P(ssz), vp], ssz),
        "atkdsp_gpu_batch_stream": ([vp], vp),
        "atkdsp_gpu_batch_kernel_ms": ([vp], C.c_float),
        "atkdsp_osx_create": ([d, sz, d, u], vp),
        "atkdsp_osx_destroy": ([vp], None),
        "atkdsp_osx_reset": ([vp], None),
        "atkdsp_osx_add": ([vp, d, d, d], C.c_int),
        "atkdsp_osx_retune": ([vp, C.c_int, d], C.c_int),
        "atkdsp_osx_remove": ([vp, C.c_int], C.c_int),
        "atkdsp_osx_channels": ([vp], C.c_int),
        "atkdsp_osx_chan_rate": ([vp, C.c_int], d),
        "atkdsp_osx_out_max": ([vp, C.c_int, sz], sz),
        "atkdsp_osx_process": ([vp, pcf, sz, ppcf, P(sz), sz], ssz),
        "atkdsp_osx_process_n": ([vp, ppcf, u, sz, ppcf, P(sz), sz], ssz),
        "atkdsp_osx_describe": ([vp, C.c_char_p, sz], C.c_int),
        "atkdsp_gpu_osx_process_n": ([vp, P(vp), u, sz, P(vp), P(sz), sz], ssz),
        "atkdsp_gpu_osx_stream": ([vp], vp),
        "atkdsp_gpu_osx_sync": ([vp], C.c_int),
        "atkdsp_gpu_spectrum_create": ([sz], vp),
        "atkdsp_gpu_spectrum_destroy": ([vp], None),
        "atkdsp_gpu_spectrum_reduce": ([vp, vp, sz, sz, vp, C.c_int, vp, vp], ssz),
        "atkdsp_gpu_spectrum_stats": ([vp, vp, sz, sz, vp, vp, vp, vp, vp, vp], ssz),
        "atkdsp_cfar_defaults": ([P(_CfarConfig)], None),
        "atkdsp_cfar_alpha": ([C.c_int, C.c_int, d, d, C.c_int, P(d), P(d), P(d)], C.c_int),
        "atkdsp_cfar_n_eff": ([C.c_int, P(d)], d),
        "atkdsp_cfar_window_rho2": ([P(C.c_float), sz, P(d)], C.c_int),
        "atkdsp_cfar_create": ([sz, P(_CfarConfig)], vp),
        "atkdsp_cfar_destroy": ([vp], None),
        "atkdsp_cfar_reset": ([vp], None),
        "atkdsp_cfar_set_mask": ([vp, P(C.c_uint8)], C.c_int),
        "atkdsp_cfar_events_max": ([vp, sz], sz),
        "atkdsp_cfar_process": ([vp, P(C.c_float), sz, d, d, P(_CfarEvent), sz], ssz),
        "atkdsp_cfar_flush": ([vp, P(_CfarEvent), sz], ssz),
        "atkdsp_cfar_last": ([vp, P(C.c_float), P(C.c_float), P(C.c_uint8)], C.c_int),
        "atkdsp_cfar_info": ([vp, P(d), P(d), P(d), P(_CfarConfig)], C.c_int),
        "atkdsp_cfar_describe": ([vp, C.c_char_p, sz], C.c_int),
        "atkdsp_cfar_stats": ([vp, P(_CfarCounters)], C.c_int),
        "atkdsp_gpu_cfar_process": ([vp, vp, C.c_int, sz, d, d, P(_CfarEvent), sz, vp, vp], ssz),
        "atkdsp_gpu_tune_set": ([u, u, u, C.c_int], C.c_int),
        "atkdsp_gpu_fail_alloc_after": ([C.c_longlong], None),
        "atkdsp_gpu_pfb_faults": ([vp], C.c_int),
        "atkdsp_gpu_batch_faults": ([vp], C.c_int),
        "atkdsp_gpu_debug_build": ([], C.c_int),
        "atkdsp_gpu_inject_short_window": ([C.c_longlong], None),
        "atkdsp_gpu_tune_get": ([u, u, u], C.c_int),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    # second function objects for the per-block calls, taking addresses as
    # ints: numpy's ctypes.data_as costs more than the call itself
    for attr, name, args, res in (("_lean_pfb_process", "atkdsp_pfb_process", [vp, vp, sz, vp, sz], ssz),
                                  ("_lean_pfb_process_n", "atkdsp_pfb_process_n", [vp, vp, u, sz, vp, sz], ssz)):
        f = lib._FuncPtr((name, lib))
        f.argtypes = args
        f.restype = res
        setattr(lib, attr, f)


def load(path: str | os.PathLike | None = None):
    """Load the library (once). Raises AtkDspError when it is missing."""
    global _lib, _lib_path
    if _lib is not None and path is None:
        return _lib
    cand = Path(path) if path else Path(os.environ.get("ATKDSP_B200_LIB", str(LIB_FILE)))
    if not cand.exists():
        raise AtkDspError(f"could not load {cand}: not built (make -C atkdsp_b200)")
    try:
        lib = C.CDLL(str(cand))
    except OSError as e:
        raise AtkDspError(f"could not load {cand}: {e}") from None
    lib.atkdsp_abi_version.restype = C.c_int
    abi = int(lib.atkdsp_abi_version())
    if abi != ABI_VERSION:
        raise AtkDspError(f"{cand}: ABI {abi}, this binding needs {ABI_VERSION}")
    _bind(lib)
    _lib, _lib_path = lib, cand
    return lib


def available() -> bool:
    try:
        load()
        return True
    except AtkDspError:
        return False


def lib_path() -> Path | None:
    return _lib_path


def version() -> str:
    return load().atkdsp_version_string().decode()


def build_info() -> str:
    return load().atkdsp_build_info().decode()


def set_threads(n: int) -> int:
    return int(load().atkdsp_set_threads(int(n)))


def get_threads() -> int:
    return int(load().atkdsp_get_threads())


def _fmt(fmt) -> int:
    if isinstance(fmt, str):
        try:
            return FMT[fmt]
        except KeyError:
            raise AtkDspError(f"unknown sample format {fmt!r}") from None
    return int(fmt)


def bytes_per_sample(fmt) -> int:
    return int(load().atkdsp_bytes_per_sample(_fmt(fmt)))


def _cfp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(_Cf32))


def _raw_u8(raw) -> np.ndarray:
    return np.frombuffer(raw, dtype=np.uint8) if not isinstance(raw, np.ndarray) \
        else np.ascontiguousarray(raw).view(np.uint8).reshape(-1)


# -- unpack (reference binding :337-385) -------------------------------------
def unpack(raw, fmt, dc_alpha: float = 0.0, dc_state: np.ndarray | None = None,
           out: np.ndarray | None = None) -> np.ndarray:
    """Raw bytes -> complex64, optional one-pole DC block (state in dc_state)."""
    lib = load()
    src = _raw_u8(raw)
    n = src.size // bytes_per_sample(fmt)
    if out is None:
        out = np.empty(n, dtype=np.complex64)
    elif out.dtype != np.complex64 or not out.flags.c_contiguous:
        raise AtkDspError("out must be a contiguous complex64 array")
    st = None
    if dc_alpha > 0:
        if dc_state is None or dc_state.dtype != np.complex64 or dc_state.size != 1:
            raise AtkDspError("dc_state must be a 1-element complex64 array")
        st = _cfp(dc_state)
    got = _check(lib.atkdsp_unpack(src.ctypes.data, src.size, _fmt(fmt), _cfp(out), out.size,
                                   float(dc_alpha), st), "unpack")
    return out[:got]


def unpack_dc(raw, fmt, offset: complex = 0j, out: np.ndarray | None = None,
              want_mean: bool = True):
    """Raw bytes -> complex64 with ``offset`` removed; returns ``(x, mean)``,
    the mean taken BEFORE the offset came out."""
    lib = load()
    src = _raw_u8(raw)
    n = src.size // bytes_per_sample(fmt)
    if out is None:
        out = np.empty(n, dtype=np.complex64)
    elif out.dtype != np.complex64 or not out.flags.c_contiguous:
        raise AtkDspError("out must be a contiguous complex64 array")
    mr, mi = C.c_double(0.0), C.c_double(0.0)
    got = _check(lib.atkdsp_unpack_dc(src.ctypes.data, src.size, _fmt(fmt), _cfp(out), out.size,
                                      float(offset.real), float(offset.imag),
                                      C.byref(mr) if want_mean else None,
                                      C.byref(mi) if want_mean else None), "unpack_dc")
    return out[:got], complex(mr.value, mi.value)


# -- the channelizer (reference binding :4159-4219) ----------------------------
class Pfb:
    """Oversampled polyphase filterbank on the GPU (atkdsp_pfb). nchan channels
    on a uniform grid spaced fs/nchan, ``oversample``x. process_n runs N
    element streams on one block clock."""

    def __init__(self, fs, nchan, oversample=2, taps_per_poly=12, atten_db=80.0, max_nel=1):
        self._lib = load()
        self._p = self._lib.atkdsp_pfb_create(float(fs), int(nchan), int(oversample),
                                              int(taps_per_poly), float(atten_db), int(max_nel))
        if not self._p:
            raise AtkDspError("pfb_create: check fs>0, nchan>=2, nchan%oversample==0, "
                              "a usable GPU and free device memory")
        self.nchan = int(nchan)
        self.max_nel = int(max_nel)
        self.oversample = int(oversample)
        self.taps_per_poly = int(taps_per_poly)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            self._lib.atkdsp_pfb_destroy(p)
            self._p = None

    @property
    def handle(self):
        return self._p

    def reset(self):
        self._lib.atkdsp_pfb_reset(self._p)

    def out_rate(self):
        return self._lib.atkdsp_pfb_out_rate(self._p)

    def out_hops(self, n):
        return int(self._lib.atkdsp_pfb_out_hops(self._p, int(n)))

    def group_delay(self):
        return self._lib.atkdsp_pfb_group_delay(self._p)

    def block_origin(self, hop_index):
        return int(self._lib.atkdsp_pfb_block_origin(self._p, int(hop_index)))

    def set_cal(self, table, nel):
        if table is None:
            _check(self._lib.atkdsp_pfb_set_cal(self._p, None, 0), "pfb_set_cal")
            return
        t = np.ascontiguousarray(np.asarray(table, np.complex64)).reshape(int(nel), self.nchan)
        _check(self._lib.atkdsp_pfb_set_cal(self._p, _cfp(t), int(nel)), "pfb_set_cal")

    def describe(self):
        buf = C.create_string_buffer(256)
        n = self._lib.atkdsp_pfb_describe(self._p, buf, 256)
        return buf.value.decode() if n > 0 else ""

    def process_n(self, ins, nel):
        nel = int(nel)
        arrs = [np.ascontiguousarray(np.asarray(ins[e]).ravel(), np.complex64) for e in range(nel)]
        n = arrs[0].size
        for a in arrs:
            if a.size != n:
                raise AtkDspError("pfb: elements must be equal length")
        lib = self._lib
        m = lib.atkdsp_pfb_out_hops(self._p, n)
        out = np.empty(nel * self.nchan * m, np.complex64)     # every entry is written
        if nel == 1:
            got = lib._lean_pfb_process(self._p, arrs[0].ctypes.data, n, out.ctypes.data, out.size)
        else:
            inarr = (C.c_void_p * nel)(*[a.ctypes.data for a in arrs])
            got = lib._lean_pfb_process_n(self._p, inarr, nel, n, out.ctypes.data, out.size)
        _check(int(got), "pfb_process_n")
        return out[: nel * self.nchan * got].reshape(nel, self.nchan, got)

    def process(self, x):
        return self.process_n([x], 1)[0]


class Osx:
    """Overlap-save extractor on the GPU (atkdsp_osx): arbitrary channels at
    arbitrary centres from one forward FFT per block, each landed on its own
    out_rate. add/retune/remove between calls without disturbing the others;
    process_n runs N elements phase-coherently."""

    def __init__(self, fs, nfft=4096, atten_db=80.0, max_nel=1):
        self._lib = load()
        self._p = self._lib.atkdsp_osx_create(float(fs), int(nfft), float(atten_db), int(max_nel))
        if not self._p:
            raise AtkDspError("osx_create: check fs>0, nfft a power of two >= 64, "
                              "a usable GPU and free device memory")
        self.max_nel = int(max_nel)
        self.nfft = int(nfft)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            self._lib.atkdsp_osx_destroy(p)
            self._p = None

    @property
    def handle(self):
        return self._p

    def reset(self):
        self._lib.atkdsp_osx_reset(self._p)

    def add(self, offset_hz, bw_hz, out_rate):
        ch = self._lib.atkdsp_osx_add(self._p, float(offset_hz), float(bw_hz), float(out_rate))
        return _check(int(ch), "osx_add")

    def retune(self, ch, offset_hz):
        _check(self._lib.atkdsp_osx_retune(self._p, int(ch), float(offset_hz)), "osx_retune")

    def remove(self, ch):
        _check(self._lib.atkdsp_osx_remove(self._p, int(ch)), "osx_remove")

    def channels(self):
        return int(self._lib.atkdsp_osx_channels(self._p))

    def chan_rate(self, ch):
        return float(self._lib.atkdsp_osx_chan_rate(self._p, int(ch)))

    def out_max(self, ch, n):
        return int(self._lib.atkdsp_osx_out_max(self._p, int(ch), int(n)))

    def describe(self):
        buf = C.create_string_buffer(256)
        n = self._lib.atkdsp_osx_describe(self._p, buf, 256)
        return buf.value.decode() if n > 0 else ""

    def process_n(self, ins, nel, cap=None):
        """(outs, counts): outs[slot] is an (nel, count) array or None for a
        free slot. cap: cap_each (default the binding's, the largest
        out_max over the active slots)."""
        nel = int(nel)
        arrs = [np.ascontiguousarray(np.asarray(ins[e]).ravel(), np.complex64) for e in range(nel)]
        n = arrs[0].size
        for a in arrs:
            if a.size != n:
                raise AtkDspError("osx: elements must be equal length")
        ns = self.channels()
        active = [self.chan_rate(ci) > 0 for ci in range(ns)]
        if cap is None:
            cap = max([self.out_max(ci, n) for ci in range(ns) if active[ci]], default=0)
        bufs = [[np.zeros(cap, np.complex64) if active[ci] else None for ci in range(ns)]
                for _ in range(nel)]
        ptrs = (C.POINTER(_Cf32) * max(nel * ns, 1))()
        for e in range(nel):
            for ci in range(ns):
                ptrs[e * ns + ci] = _cfp(bufs[e][ci]) if active[ci] else None
        counts = (C.c_size_t * max(ns, 1))()
        inarr = (C.POINTER(_Cf32) * nel)(*[_cfp(a) for a in arrs])
        got = self._lib.atkdsp_osx_process_n(self._p, inarr, nel, n, ptrs, counts, int(cap))
        _check(int(got), "osx_process_n")
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


def pfb_cov_accumulate(out, nel, nchan, gate, R, counts):
    """W1: R[k] += sum_i y_k y_k^H over gated channels; counts[k] += m.
    out (nel, nchan, m) complex64; R (nchan, nel, nel) complex64 and counts
    (nchan,) uint32 are updated in place."""
    lib = load()
    o = np.ascontiguousarray(out, np.complex64)
    nel = int(nel); nchan = int(nchan); m = o.shape[2] if o.ndim == 3 else 0
    if not (R.flags["C_CONTIGUOUS"] and R.dtype == np.complex64):
        raise AtkDspError("pfb_cov_accumulate: R must be contiguous complex64")
    if not (counts.flags["C_CONTIGUOUS"] and counts.dtype == np.uint32):
        raise AtkDspError("pfb_cov_accumulate: counts must be contiguous uint32")
    gp = None
    if gate is not None:
        g = np.ascontiguousarray(gate, np.uint8)
        gp = g.ctypes.data_as(C.POINTER(C.c_uint8))
    lib.atkdsp_pfb_cov_accumulate(_cfp(o.reshape(-1)), nel, nchan, m, gp,
                                  _cfp(R.reshape(-1)), counts.ctypes.data_as(C.POINTER(C.c_uint32)))


def pfb_cov_reset(R, counts, nel, nchan, gate=None):
    lib = load()
    gp = None
    if gate is not None:
        g = np.ascontiguousarray(gate, np.uint8)
        gp = g.ctypes.data_as(C.POINTER(C.c_uint8))
    lib.atkdsp_pfb_cov_reset(_cfp(R.reshape(-1)), counts.ctypes.data_as(C.POINTER(C.c_uint32)),
                             int(nel), int(nchan), gp)


def pfb_channel_power(out, nel, nchan):
    """W2: returns (pwr[nel, nchan], mean_pwr[nchan]) float32."""
    lib = load()
    o = np.ascontiguousarray(out, np.complex64)
    nel = int(nel); nchan = int(nchan); m = o.shape[2] if o.ndim == 3 else 0
    pwr = np.zeros(nel * nchan, np.float32)
    meanp = np.zeros(nchan, np.float32)
    lib.atkdsp_pfb_channel_power(_cfp(o.reshape(-1)), nel, nchan, m,
                                 pwr.ctypes.data_as(C.POINTER(C.c_float)),
                                 meanp.ctypes.data_as(C.POINTER(C.c_float)))
    return pwr.reshape(nel, nchan), meanp


# ---- CFAR across frequency and the burst tracker ---------------------------

CFAR_MODES = {"ca": 0, "os": 1, "go": 2, "so": 3}
CFAR_OPEN, CFAR_UPDATE, CFAR_CLOSE = 1, 2, 3
CFAR_T0_COARSE, CFAR_T1_COARSE, CFAR_EDGE, CFAR_MASK_ADJ, CFAR_FLUSHED = 1, 2, 4, 8, 16


def cfar_defaults() -> dict:
    """The default atkdsp_cfar_config as a dict (rho2 a 4-tuple)."""
    k = _CfarConfig()
    load().atkdsp_cfar_defaults(C.byref(k))
    d = {n: getattr(k, n) for n, _t in _CfarConfig._fields_ if n != "reserved"}
    d["rho2"] = tuple(float(v) for v in k.rho2)
    return d


def _rho2_arg(rho2):
    if rho2 is None:
        return None
    v = [float(x) for x in rho2]
    if len(v) != 4:
        raise AtkDspError(f"rho2 needs 4 values, got {len(v)}")
    return (C.c_double * 4)(*v)


def cfar_alpha(mode, n_ref: int, pfa: float, looks: float = 1.0, os_k: int = 0, rho2=None) -> tuple:
    """(alpha, E[T]): the CFAR threshold multiplier solved for `pfa` per cell."""
    m = CFAR_MODES.get(mode, mode) if isinstance(mode, str) else int(mode)
    a, et = C.c_double(), C.c_double()
    _check(load().atkdsp_cfar_alpha(int(m), int(n_ref), float(pfa), float(looks), int(os_k),
                                    _rho2_arg(rho2), C.byref(a), C.byref(et)), "cfar_alpha")
    return a.value, et.value


def cfar_n_eff(n_ref: int, rho2=None) -> float:
    """Equivalent independent cells among 2 n_ref correlated ones."""
    return float(load().atkdsp_cfar_n_eff(int(n_ref), _rho2_arg(rho2)))


def cfar_window_rho2(window) -> tuple:
    """The power correlation of bins 1..4 apart through `window`."""
    w = np.ascontiguousarray(window, np.float32)
    out = (C.c_double * 4)()
    _check(load().atkdsp_cfar_window_rho2(w.ctypes.data_as(C.POINTER(C.c_float)), w.size, out),
           "cfar_window_rho2")
    return tuple(float(v) for v in out)


def _cfar_event_dict(e) -> dict:
    return {"type": int(e.type), "id": int(e.id), "flags": int(e.flags), "lo": int(e.lo_bin),
            "hi": int(e.hi_bin), "n_hits": int(e.n_hits), "t0": float(e.t0),
            "t1": float(e.t1), "fc_bin": float(e.fc_bin), "level_db": float(e.level_db),
            "noise_db": float(e.noise_db), "snr_db": float(e.snr_db),
            "band_snr_db": float(e.band_snr_db)}


class Cfar:
    """CFAR across frequency and the burst tracker. Options are the
    atkdsp_cfar_config fields as keywords (mode may be 'ca' / 'os' / 'go' /
    'so'). process() returns the OPEN / UPDATE / CLOSE events as dicts. The
    per-cell work of each call runs on the GPU; the tracker on the host."""

    def __init__(self, nbins: int, **cfg):
        self._lib = load()
        c = cfar_defaults()
        for key, v in cfg.items():
            if key not in c:
                raise AtkDspError(f"unknown CFAR option {key!r}; known: {sorted(c)}")
            c[key] = CFAR_MODES.get(v, v) if key == "mode" and isinstance(v, str) else v
        k = _CfarConfig()
        for key, v in c.items():
            if key == "rho2":
                k.rho2 = (C.c_double * 4)(*[float(x) for x in v])
            else:
                setattr(k, key, float(v) if key in ("pfa", "looks") else int(v))
        self.nbins = int(nbins)
        self._h = self._lib.atkdsp_cfar_create(self.nbins, C.byref(k))
        if not self._h:
            raise AtkDspError(f"cfar_create({nbins} bins, {c}) refused: a configuration outside the "
                              "ranges, a threshold that could not be solved, or no GPU memory")
        self._buf = None
        a, ac, et, rc = C.c_double(), C.c_double(), C.c_double(), _CfarConfig()
        self._lib.atkdsp_cfar_info(self._h, C.byref(a), C.byref(ac), C.byref(et), C.byref(rc))
        self.alpha, self.alpha_ca, self.et = a.value, ac.value, et.value
        self.cfg = {n: getattr(rc, n) for n, _t in _CfarConfig._fields_ if n != "reserved"}
        self.cfg["rho2"] = tuple(float(v) for v in rc.rho2)
        self.n_eff = cfar_n_eff(self.cfg["n_ref"], self.cfg["rho2"])

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.atkdsp_cfar_destroy(h)

    @property
    def handle(self):
        return self._h

    def describe(self) -> str:
        buf = C.create_string_buffer(1024)
        self._lib.atkdsp_cfar_describe(self._h, buf, 1024)
        return buf.value.decode()

    def stats(self) -> dict:
        s = _CfarCounters()
        self._lib.atkdsp_cfar_stats(self._h, C.byref(s))
        return {n: int(getattr(s, n)) for n, _t in s._fields_}

    def reset(self) -> None:
        self._lib.atkdsp_cfar_reset(self._h)

    def set_mask(self, mask) -> None:
        if mask is None:
            self._lib.atkdsp_cfar_set_mask(self._h, None)
            return
        m = np.ascontiguousarray(np.asarray(mask).ravel() != 0, dtype=np.uint8)
        if m.size != self.nbins:
            raise AtkDspError(f"mask has {m.size} entries; the CFAR has {self.nbins} bins")
        _check(self._lib.atkdsp_cfar_set_mask(self._h, m.ctypes.data_as(C.POINTER(C.c_uint8))),
               "cfar_set_mask")

    def events_max(self, nframes: int) -> int:
        return int(self._lib.atkdsp_cfar_events_max(self._h, int(nframes)))

    def _events(self, nf):
        cap = self.events_max(nf)
        if self._buf is None or len(self._buf) < cap:
            self._buf = (_CfarEvent * max(cap, 1))()
        return cap

    def process(self, frames_db, frame_t0: float, frame_dt: float) -> list:
        f = np.ascontiguousarray(frames_db, dtype=np.float32)
        if f.ndim == 1:
            f = f.reshape(1, -1)
        if f.ndim != 2 or f.shape[1] != self.nbins:
            raise AtkDspError(f"frames must be (nframes, {self.nbins}); got {f.shape}")
        nf = f.shape[0]
        cap = self._events(nf)
        n = _check(self._lib.atkdsp_cfar_process(self._h, f.ctypes.data_as(C.POINTER(C.c_float)), nf,
                                                 float(frame_t0), float(frame_dt), self._buf, cap),
                   "cfar_process")
        return [_cfar_event_dict(self._buf[j]) for j in range(n)]

    def flush(self) -> list:
        cap = int(self.cfg["max_tracks"])
        buf = (_CfarEvent * cap)()
        n = _check(self._lib.atkdsp_cfar_flush(self._h, buf, cap), "cfar_flush")
        return [_cfar_event_dict(buf[j]) for j in range(n)]

    def last(self):
        """(averaged power dB, threshold dB (NaN untested), hits) of the last
        tested frame, or None before one."""
        a = np.empty(self.nbins, np.float32)
        t = np.empty(self.nbins, np.float32)
        h = np.empty(self.nbins, np.uint8)
        P = C.POINTER
        rc = self._lib.atkdsp_cfar_last(self._h, a.ctypes.data_as(P(C.c_float)),
                                        t.ctypes.data_as(P(C.c_float)), h.ctypes.data_as(P(C.c_uint8)))
        if rc == E_EMPTY:
            return None
        _check(rc, "cfar_last")
        return a, t, h
