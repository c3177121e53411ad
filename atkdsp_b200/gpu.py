"""Device-pointer front end (include/atkdsp_gpu.h) for torch tensors.

torch is used here only as the owner of device memory and streams: every
computation runs in the library's own CUDA kernels. Tensors must be
contiguous and on the handle's device; complex samples are ``torch.complex64``
(the cf32 layout), raw front-end samples ``torch.uint8`` / ``int8`` /
``int16`` byte buffers.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import AtkDspError, Cfar, Pfb, _cfar_event_dict, _check, _fmt, bytes_per_sample, load

__all__ = ["Spectrum", "cfar_process", "process_n", "process_n_raw", "process_w12", "unpack_dc", "unpack", "block_mean", "accumulate",
           "cov_accumulate", "channel_power", "Batch", "sync"]


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise AtkDspError("device tensors must be contiguous CUDA tensors")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def sync(p: Pfb) -> None:
    _check(load().atkdsp_gpu_pfb_sync(p.handle), "gpu_pfb_sync")


def process_n(p: Pfb, ins, nel: int, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """atkdsp_gpu_pfb_process_n: ins are nel complex64 CUDA tensors of equal
    length; returns (nel, nchan, m) complex64 on the device. Asynchronous on
    ``stream`` (default: the handle's stream)."""
    lib = load()
    nel = int(nel)
    n = int(ins[0].numel())
    for t in ins[:nel]:
        if t.numel() != n or t.dtype != torch.complex64:
            raise AtkDspError("gpu process_n: inputs must be complex64 of equal length")
    m = p.out_hops(n)
    if out is None:
        out = torch.empty(nel * p.nchan * max(m, 1), dtype=torch.complex64, device=ins[0].device)
    arr = (C.c_void_p * nel)(*[t.data_ptr() for t in ins[:nel]])
    got = lib.atkdsp_gpu_pfb_process_n(p.handle, arr, nel, n, _ptr(out), out.numel(), _stream(stream))
    _check(int(got), "gpu_pfb_process_n")
    return out[: nel * p.nchan * got].view(nel, p.nchan, got)


def process_n_raw(p: Pfb, raws, nel: int, fmt, offset: complex = 0j,
                  out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """atkdsp_gpu_pfb_process_n_raw: unpack_dc(raw, fmt, offset) fused into the
    filterbank. raws are nel int16 CUDA tensors of 2n values (I, Q pairs)."""
    lib = load()
    nel = int(nel)
    n = int(raws[0].numel()) // 2
    for t in raws[:nel]:
        if t.numel() != 2 * n or t.dtype != torch.int16:
            raise AtkDspError("gpu process_n_raw: inputs must be int16 I/Q of equal length")
    m = p.out_hops(n)
    if out is None:
        out = torch.empty(nel * p.nchan * max(m, 1), dtype=torch.complex64, device=raws[0].device)
    arr = (C.c_void_p * nel)(*[t.data_ptr() for t in raws[:nel]])
    got = lib.atkdsp_gpu_pfb_process_n_raw(p.handle, arr, nel, n, _fmt(fmt), float(offset.real),
                                           float(offset.imag), _ptr(out), out.numel(), _stream(stream))
    _check(int(got), "gpu_pfb_process_n_raw")
    return out[: nel * p.nchan * got].view(nel, p.nchan, got)


def process_w12(p: Pfb, x: torch.Tensor, fmt="cf32", offset: complex = 0j, out: torch.Tensor | None = None,
                R: torch.Tensor | None = None, counts: torch.Tensor | None = None,
                pwr: torch.Tensor | None = None, mean_pwr: torch.Tensor | None = None,
                gate: torch.Tensor | None = None, scratch: torch.Tensor | None = None,
                stream=None) -> torch.Tensor:
    """atkdsp_gpu_pfb_process_w12: one element's block through the filterbank
    with W1 / W2 fused into its epilogue. x: complex64 samples (fmt "cf32") or
    int16 I/Q pairs (fmt "ci16" / "ci16q11"). offset: a complex, or a (2,)
    float64 CUDA tensor holding it on the device (a block_mean output: the
    _dev entry point, no host round trip). Returns (1, nchan, m)."""
    lib = load()
    n = int(x.numel()) if x.dtype == torch.complex64 else int(x.numel()) // 2
    m = p.out_hops(n)
    if out is None:
        out = torch.empty(p.nchan * max(m, 1), dtype=torch.complex64, device=x.device)
    need = int(lib.atkdsp_gpu_pfb_w12_scratch_bytes(p.handle, n))
    if scratch is None or scratch.numel() * scratch.element_size() < need:
        scratch = torch.empty(max(need, 8), dtype=torch.uint8, device=x.device)
    if isinstance(offset, torch.Tensor):
        _check_offset(offset)
        got = lib.atkdsp_gpu_pfb_process_w12_dev(p.handle, _ptr(x), n, _fmt(fmt), _ptr(offset), _ptr(out),
                                                 out.numel(), _ptr(gate), _ptr(R), _ptr(counts), _ptr(pwr),
                                                 _ptr(mean_pwr), _ptr(scratch),
                                                 scratch.numel() * scratch.element_size(), _stream(stream))
    else:
        got = lib.atkdsp_gpu_pfb_process_w12(p.handle, _ptr(x), n, _fmt(fmt), float(offset.real),
                                             float(offset.imag), _ptr(out), out.numel(), _ptr(gate), _ptr(R),
                                             _ptr(counts), _ptr(pwr), _ptr(mean_pwr), _ptr(scratch),
                                             scratch.numel() * scratch.element_size(), _stream(stream))
    _check(int(got), "gpu_pfb_process_w12")
    return out[: p.nchan * got].view(1, p.nchan, got)


def unpack_dc(raw: torch.Tensor, fmt, offset: complex = 0j, out: torch.Tensor | None = None,
              want_mean: bool = True, stream=None):
    """atkdsp_gpu_unpack_dc: returns (samples, mean) with mean a (2,) float64
    CUDA tensor (re, im) or None."""
    lib = load()
    nbytes = raw.numel() * raw.element_size()
    n = nbytes // bytes_per_sample(fmt)
    if out is None:
        out = torch.empty(max(n, 1), dtype=torch.complex64, device=raw.device)
    mean = torch.empty(2, dtype=torch.float64, device=raw.device) if want_mean else None
    got = lib.atkdsp_gpu_unpack_dc(_ptr(raw), nbytes, _fmt(fmt), _ptr(out), out.numel(),
                                   float(offset.real), float(offset.imag), _ptr(mean),
                                   _stream(stream))
    _check(int(got), "gpu_unpack_dc")
    return out[:got], mean


def unpack(raw: torch.Tensor, fmt, dc_alpha: float = 0.0, dc_state: torch.Tensor | None = None,
           out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    lib = load()
    nbytes = raw.numel() * raw.element_size()
    n = nbytes // bytes_per_sample(fmt)
    if out is None:
        out = torch.empty(max(n, 1), dtype=torch.complex64, device=raw.device)
    got = lib.atkdsp_gpu_unpack(_ptr(raw), nbytes, _fmt(fmt), _ptr(out), out.numel(),
                                float(dc_alpha), _ptr(dc_state), _stream(stream))
    _check(int(got), "gpu_unpack")
    return out[:got]


def block_mean(raw: torch.Tensor, fmt, offset: complex = 0j, mean: torch.Tensor | None = None,
               stream=None) -> torch.Tensor:
    """atkdsp_gpu_block_mean: the unpack_dc mean of a raw block, (2,) float64.
    offset: a complex, or a (2,) float64 CUDA tensor (atkdsp_gpu_block_mean_dev;
    it may be ``mean`` itself)."""
    if mean is None:
        mean = torch.empty(2, dtype=torch.float64, device=raw.device)
    if isinstance(offset, torch.Tensor):
        _check_offset(offset)
        got = load().atkdsp_gpu_block_mean_dev(_ptr(raw), raw.numel() * raw.element_size(), _fmt(fmt),
                                               _ptr(offset), _ptr(mean), _stream(stream))
    else:
        got = load().atkdsp_gpu_block_mean(_ptr(raw), raw.numel() * raw.element_size(), _fmt(fmt),
                                           float(offset.real), float(offset.imag), _ptr(mean), _stream(stream))
    _check(int(got), "gpu_block_mean")
    return mean


def _check_offset(offset: torch.Tensor) -> None:
    if offset.dtype != torch.float64 or offset.numel() != 2 or not offset.is_cuda or not offset.is_contiguous():
        raise AtkDspError("a device offset is a contiguous (2,) float64 CUDA tensor (re, im)")


def accumulate(out: torch.Tensor, nel: int, nchan: int, R: torch.Tensor | None,
               counts: torch.Tensor | None, pwr: torch.Tensor | None = None,
               mean_pwr: torch.Tensor | None = None, gate: torch.Tensor | None = None,
               stream=None) -> None:
    """atkdsp_gpu_pfb_accumulate: W1 and W2 in one pass over a device block."""
    m = out.shape[-1] if out.dim() == 3 else 0
    _check(load().atkdsp_gpu_pfb_accumulate(_ptr(out), int(nel), int(nchan), m, _ptr(gate), _ptr(R),
                                            _ptr(counts), _ptr(pwr), _ptr(mean_pwr), _stream(stream)),
           "gpu_pfb_accumulate")


def cov_accumulate(out: torch.Tensor, nel: int, nchan: int, gate: torch.Tensor | None,
                   R: torch.Tensor, counts: torch.Tensor, stream=None) -> None:
    m = out.shape[-1] if out.dim() == 3 else 0
    _check(load().atkdsp_gpu_pfb_cov_accumulate(_ptr(out), int(nel), int(nchan), m, _ptr(gate),
                                                _ptr(R), _ptr(counts), _stream(stream)),
           "gpu_cov_accumulate")


def channel_power(out: torch.Tensor, nel: int, nchan: int, stream=None):
    m = out.shape[-1] if out.dim() == 3 else 0
    pwr = torch.zeros(int(nel) * int(nchan), dtype=torch.float32, device=out.device)
    meanp = torch.zeros(int(nchan), dtype=torch.float32, device=out.device)
    _check(load().atkdsp_gpu_pfb_channel_power(_ptr(out), int(nel), int(nchan), m, _ptr(pwr),
                                               _ptr(meanp), _stream(stream)), "gpu_channel_power")
    return pwr.view(int(nel), int(nchan)), meanp


class Batch:
    """atkdsp_gpu_batch: many single-element handles, one launch per block set."""

    def __init__(self, pfbs, use_graph: bool = True):
        self._lib = load()
        self.pfbs = list(pfbs)
        arr = (C.c_void_p * len(self.pfbs))(*[p.handle for p in self.pfbs])
        self._b = self._lib.atkdsp_gpu_batch_create(arr, len(self.pfbs), 1 if use_graph else 0)
        if not self._b:
            raise AtkDspError("gpu_batch_create failed")
        n = len(self.pfbs)
        self._ins = (C.c_void_p * n)()
        self._outs = (C.c_void_p * n)()
        self._ns = (C.c_size_t * n)()
        self._ms = (C.c_ssize_t * n)()

    def __del__(self):
        b = getattr(self, "_b", None)
        if b:
            self._lib.atkdsp_gpu_batch_destroy(b)
            self._b = None

    @property
    def stream_ptr(self) -> int:
        return int(self._lib.atkdsp_gpu_batch_stream(self._b) or 0)

    def kernel_ms(self) -> float:
        """Device time of the last call's filterbank kernel (waits for it)."""
        return float(self._lib.atkdsp_gpu_batch_kernel_ms(self._b))

    def out_hops(self, ns) -> list:
        return [p.out_hops(int(n)) for p, n in zip(self.pfbs, ns)]

    def process(self, ins, outs, stream=None) -> list:
        """ins[i]: complex64 CUDA tensor (new block of handle i; may be empty);
        outs[i]: complex64 CUDA tensor of >= nchan_i * out_hops_i samples.
        Returns the per-handle hop counts. Asynchronous."""
        for i, (x, o) in enumerate(zip(ins, outs)):
            self._ins[i] = x.data_ptr() if x.numel() else None
            self._outs[i] = o.data_ptr() if o is not None and o.numel() else None
            self._ns[i] = x.numel()
        got = self._lib.atkdsp_gpu_batch_process(self._b, self._ins, self._ns, self._outs, self._ms,
                                                 _stream(stream))
        _check(int(got), "gpu_batch_process")
        return [int(self._ms[i]) for i in range(len(self.pfbs))]

    def process_raw(self, raws, outs, fmt, offs=None, stream=None) -> list:
        """The same with int16 I/Q blocks (2 values per sample) converted in the
        filterbank's load path; offs: per-handle complex offsets or None."""
        n = len(self.pfbs)
        for i, (x, o) in enumerate(zip(raws, outs)):
            self._ins[i] = x.data_ptr() if x.numel() else None
            self._outs[i] = o.data_ptr() if o is not None and o.numel() else None
            self._ns[i] = x.numel() // 2
        po = None
        if offs is not None:
            fo = (C.c_float * (2 * n))()
            for i, z in enumerate(offs):
                fo[2 * i], fo[2 * i + 1] = float(complex(z).real), float(complex(z).imag)
            po = fo
        got = self._lib.atkdsp_gpu_batch_process_raw(self._b, self._ins, self._ns, _fmt(fmt), po,
                                                     self._outs, self._ms, _stream(stream))
        _check(int(got), "gpu_batch_process_raw")
        return [int(self._ms[i]) for i in range(n)]


DET = {"max": 0, "min": 1, "avg": 2}


class Spectrum:
    """atkdsp_gpu_spectrum: the display reduction of the binding's
    ``Fft.spectrum_reduce`` / ``Fft.spectrum_stats`` (python/atkdsp/__init__.py:
    566-600) on device tensors, for power-of-two n from 16 to 4096."""

    def __init__(self, n: int):
        self._lib = load()
        self.n = int(n)
        self._p = self._lib.atkdsp_gpu_spectrum_create(self.n)
        if not self._p:
            raise AtkDspError(f"gpu_spectrum_create({n}): n must be a power of two in 16..4096")

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            self._lib.atkdsp_gpu_spectrum_destroy(p)
            self._p = None

    def reduce(self, x: torch.Tensor, hop: int | None = None, win: torch.Tensor | None = None,
               detector="max", out: torch.Tensor | None = None, stream=None):
        """Every frame of x reduced to one fftshifted dB line: (line, frames)."""
        if out is None:
            out = torch.empty(self.n, dtype=torch.float32, device=x.device)
        det = DET[detector] if isinstance(detector, str) else int(detector)
        fr = self._lib.atkdsp_gpu_spectrum_reduce(self._p, _ptr(x), x.numel(), int(hop or self.n), _ptr(win),
                                                  det, _ptr(out), _stream(stream))
        _check(int(fr), "gpu_spectrum_reduce")
        return out, int(fr)

    def stats(self, x: torch.Tensor, hop: int | None = None, win: torch.Tensor | None = None,
              want=("max", "avg", "min", "sk"), stream=None) -> dict:
        """Per-bin peak / mean / floor (dB) and spectral kurtosis in one pass."""
        want = set(want)
        outs = {k: (torch.empty(self.n, dtype=torch.float32, device=x.device) if k in want else None)
                for k in ("max", "avg", "min", "sk")}
        fr = self._lib.atkdsp_gpu_spectrum_stats(self._p, _ptr(x), x.numel(), int(hop or self.n), _ptr(win),
                                                 *[_ptr(outs[k]) for k in ("max", "avg", "min", "sk")],
                                                 _stream(stream))
        _check(int(fr), "gpu_spectrum_stats")
        res = {k: v for k, v in outs.items() if v is not None}
        res["frames"] = int(fr)
        return res


def cfar_process(c: Cfar, frames: torch.Tensor, frame_t0: float, frame_dt: float, units: str = "db",
                 hits: bool | torch.Tensor = False, stream=None):
    """atkdsp_gpu_cfar_process: the CFAR and tracker over device frames
    (nframes, nbins) float32, in dB (units "db", as atkdsp_cfar_process takes
    them) or linear power ("linear": W2's channel powers as they come).
    Returns (events, hit masks): with hits=True (or a uint8 device tensor of
    the frames' shape) every frame's hit mask stays on the device, ready as
    the W1 gate of that frame; otherwise None. `stream`: the frames'
    producer, waited for on the device (None: the legacy default stream)."""
    f = frames if frames.dim() == 2 else frames.reshape(1, -1)
    if f.dtype != torch.float32 or f.shape[1] != c.nbins:
        raise AtkDspError(f"frames must be float32 (nframes, {c.nbins}); got {f.dtype} {tuple(f.shape)}")
    if units not in ("db", "linear"):
        raise AtkDspError(f"units must be 'db' or 'linear', not {units!r}")
    h = None
    if isinstance(hits, torch.Tensor):
        h = hits
        if h.dtype != torch.uint8 or h.shape != f.shape:
            raise AtkDspError("hits must be a uint8 tensor of the frames' shape")
    elif hits:
        h = torch.empty(f.shape, dtype=torch.uint8, device=f.device)
    nf = f.shape[0]
    cap = c._events(nf)
    n = _check(load().atkdsp_gpu_cfar_process(c.handle, _ptr(f), 0 if units == "db" else 1, nf,
                                              float(frame_t0), float(frame_dt), c._buf, cap, _ptr(h),
                                              _stream(stream)), "gpu_cfar_process")
    return [_cfar_event_dict(c._buf[j]) for j in range(n)], h
