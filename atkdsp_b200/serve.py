"""The serving loop (include/atkdsp_serve.h) from Python.

``Server`` keeps many live channelizer streams on one GPU and channelizes
every stream's pending block in one launch per round (continuous batching);
``simulate`` runs the native open-loop load generator (Poisson block arrivals
per stream, stream churn, admission by free HBM) and returns throughput and
block-latency percentiles. Device buffers are torch tensors.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import AtkDspError, FMT, _check, load

__all__ = ["Server", "SimResult", "simulate"]


class Done(C.Structure):
    _fields_ = [("id", C.c_int), ("tag", C.c_uint64), ("m", C.c_ssize_t), ("n", C.c_size_t),
                ("t_arrival", C.c_double), ("t_done", C.c_double)]


class Stats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("admitted", "denied", "closed", "rounds",
                                          "blocks_launched", "samples_launched", "blocks_done")]


class SimConfig(C.Structure):
    _fields_ = [("streams", C.c_uint), ("rates", C.POINTER(C.c_double)), ("nrates", C.c_uint),
                ("nchans", C.POINTER(C.c_uint)), ("nnchan", C.c_uint), ("oversample", C.c_uint),
                ("taps", C.c_uint), ("atten_db", C.c_double), ("fmt", C.c_int),
                ("block_s", C.c_double), ("churn_per_s", C.c_double), ("duration_s", C.c_double),
                ("warmup_s", C.c_double), ("d_raw_pool", C.c_void_p), ("raw_pool_bytes", C.c_size_t),
                ("d_out_pool", C.c_void_p), ("out_pool_bytes", C.c_size_t), ("seed", C.c_uint64)]


class SimResult(C.Structure):
    _fields_ = [("offered_samples_per_s", C.c_double), ("offered_blocks", C.c_uint64),
                ("dropped_blocks", C.c_uint64), ("blocks_done", C.c_uint64),
                ("samples_done", C.c_uint64), ("churn_events", C.c_uint64), ("admitted", C.c_uint64),
                ("denied", C.c_uint64), ("rounds", C.c_uint64), ("blocks_per_round", C.c_double),
                ("wall_s", C.c_double), ("lat_p50_ms", C.c_double), ("lat_p90_ms", C.c_double),
                ("lat_p99_ms", C.c_double), ("lat_max_ms", C.c_double), ("max_open_ms", C.c_double),
                ("max_close_ms", C.c_double), ("max_launch_ms", C.c_double), ("max_poll_ms", C.c_double),
                ("max_loop_ms", C.c_double), ("mean_launch_ms", C.c_double), ("mean_round_gpu_ms", C.c_double),
                ("gpu_busy", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def _bind(lib):
    if getattr(lib, "_serve_bound", False):
        return lib
    vp, u, sz, d, i = C.c_void_p, C.c_uint, C.c_size_t, C.c_double, C.c_int
    sigs = {
        "atkdsp_server_create": ([u, sz, i], vp),
        "atkdsp_server_destroy": ([vp], None),
        "atkdsp_server_open": ([vp, d, u, u, u, d, i], i),
        "atkdsp_server_close": ([vp, i], i),
        "atkdsp_server_submit": ([vp, i, vp, sz, vp, sz, C.c_uint64, d], i),
        "atkdsp_server_launch": ([vp], i),
        "atkdsp_server_poll": ([vp, C.POINTER(Done), i, i], i),
        "atkdsp_server_pending": ([vp], i),
        "atkdsp_server_inflight": ([vp], i),
        "atkdsp_server_get_stats": ([vp, C.POINTER(Stats)], None),
        "atkdsp_server_now": ([], d),
        "atkdsp_server_simulate": ([vp, C.POINTER(SimConfig), C.POINTER(SimResult)], i),
    }
    for name, (args, res) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    lib._serve_bound = True
    return lib


class Server:
    def __init__(self, max_streams: int = 4096, hbm_reserve: int = 8 << 30, use_graph: bool = True):
        self._lib = _bind(load())
        self._s = self._lib.atkdsp_server_create(int(max_streams), int(hbm_reserve), int(bool(use_graph)))
        if not self._s:
            raise AtkDspError("server_create failed (no GPU or no memory)")
        self.max_streams = int(max_streams)
        self._done = (Done * (4 * self.max_streams))()

    def __del__(self):
        s = getattr(self, "_s", None)
        if s:
            self._lib.atkdsp_server_destroy(s)
            self._s = None

    def open(self, fs, nchan, oversample=2, taps_per_poly=12, atten_db=80.0, fmt="cf32") -> int:
        """Returns the stream id, or a negative ATKDSP_E_* (-2: not admitted)."""
        return int(self._lib.atkdsp_server_open(self._s, float(fs), int(nchan), int(oversample),
                                                int(taps_per_poly), float(atten_db), FMT[fmt]))

    def close(self, sid: int) -> int:
        return int(self._lib.atkdsp_server_close(self._s, int(sid)))

    def submit(self, sid: int, block: torch.Tensor, out: torch.Tensor, tag: int = 0,
               t_arrival: float = 0.0) -> int:
        """block: complex64 (cf32 stream) or int16 I/Q pairs (ci16 streams)."""
        n = block.numel() if block.dtype == torch.complex64 else block.numel() // 2
        return int(self._lib.atkdsp_server_submit(self._s, int(sid), C.c_void_p(block.data_ptr()), n,
                                                  C.c_void_p(out.data_ptr()), out.numel(),
                                                  int(tag), float(t_arrival)))

    def launch(self) -> int:
        return _check(int(self._lib.atkdsp_server_launch(self._s)), "server_launch")

    def poll(self, wait: bool = False) -> list:
        got = _check(int(self._lib.atkdsp_server_poll(self._s, self._done, len(self._done),
                                                      int(bool(wait)))), "server_poll")
        return [(self._done[k].id, self._done[k].tag, self._done[k].m, self._done[k].n,
                 self._done[k].t_arrival, self._done[k].t_done) for k in range(got)]

    def pending(self) -> int:
        return int(self._lib.atkdsp_server_pending(self._s))

    def inflight(self) -> int:
        return int(self._lib.atkdsp_server_inflight(self._s))

    def stats(self) -> dict:
        st = Stats()
        self._lib.atkdsp_server_get_stats(self._s, C.byref(st))
        return {k: int(getattr(st, k)) for k, _ in st._fields_}

    def drain(self) -> list:
        """Launch and complete everything pending."""
        out = []
        while self.pending() or self.inflight():
            self.launch()
            out += self.poll(wait=True)
        return out


def simulate(server: Server, *, streams: int, rates=(2.4e6, 10e6, 40e6), nchans=(256, 1024),
             oversample: int = 2, taps: int = 16, atten_db: float = 80.0, fmt: str = "ci16",
             block_s: float = 1.6e-3, churn_per_s: float = 20.0, duration_s: float = 3.0,
             warmup_s: float = 0.5, raw_pool: torch.Tensor, out_pool: torch.Tensor,
             seed: int = 5) -> dict:
    lib = server._lib
    r = (C.c_double * len(rates))(*rates)
    nc = (C.c_uint * len(nchans))(*nchans)
    cfg = SimConfig(int(streams), r, len(rates), nc, len(nchans), int(oversample), int(taps),
                    float(atten_db), FMT[fmt], float(block_s), float(churn_per_s), float(duration_s),
                    float(warmup_s), C.c_void_p(raw_pool.data_ptr()),
                    raw_pool.numel() * raw_pool.element_size(), C.c_void_p(out_pool.data_ptr()),
                    out_pool.numel() * out_pool.element_size(), int(seed))
    res = SimResult()
    _check(int(lib.atkdsp_server_simulate(server._s, C.byref(cfg), C.byref(res))), "server_simulate")
    return res.as_dict()
