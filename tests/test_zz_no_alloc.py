"""The allocation-free unpack_dc entry point (atkdsp_gpu_unpack_dc_noalloc).

It exists for callers that cannot allocate GPU memory when they call in --
an application that gives all device memory to its own pool, a real-time
thread that must not block in the CUDA allocator, a plugin handed buffers
but no allocator. Its scratch (the mean's partial sums) is a static device
array, so every call shares it and keeps the previous call's contents.

Checked here through the C ABI, against the allocating entry point
(atkdsp_gpu_unpack_dc) on the same device buffers: two calls in a row of
different sizes and formats must give the same samples and the same means
(tolerance 1e-12 on the means, as the other unpack tests use; in practice
identical bits), and a call beyond the array's limit must be refused.
This file is collected last so that a run stopping at the first failure has
already run everything else; it also passes on its own in a fresh process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import atkdsp_b200 as ak

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_SAMPLES = 2048 * 2048          # the static array covers 2048 blocks of 2048 samples


def _entry(lib, name):
    f = getattr(lib, name)
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t, C.c_float,
                  C.c_float, C.c_void_p, C.c_void_p]
    f.restype = C.c_ssize_t
    return f


def _call(f, raw, fmt, n, out, off, mean):
    return f(C.c_void_p(raw.data_ptr()), raw.numel() * raw.element_size(), ak.FMT[fmt],
             C.c_void_p(out.data_ptr()), n, float(off.real), float(off.imag),
             C.c_void_p(mean.data_ptr()), None)


def test_no_alloc_unpack_dc_matches_the_allocating_entry_point():
    lib = ak.load()
    noalloc = _entry(lib, "atkdsp_gpu_unpack_dc_noalloc")
    alloc = _entry(lib, "atkdsp_gpu_unpack_dc")
    rng = np.random.default_rng(2027)
    cases = [  # two calls in a row: a large block, then a smaller one in another format
        ("ci16q11", rng.integers(-2048, 2048, 2 * 3_000_001, dtype=np.int64).astype("<i2"), 0.0123 - 0.0456j),
        ("cu8", rng.integers(0, 256, 2 * 100_003, dtype=np.uint8), -0.25 + 0.125j),
    ]
    for fmt, raw_np, off in cases:
        raw = torch.from_numpy(raw_np).cuda()
        n = raw_np.nbytes // ak.bytes_per_sample(fmt)
        out_a = torch.empty(n, dtype=torch.complex64, device="cuda")
        out_b = torch.empty(n, dtype=torch.complex64, device="cuda")
        mean_a = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        mean_b = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        assert _call(noalloc, raw, fmt, n, out_a, off, mean_a) == n
        assert _call(alloc, raw, fmt, n, out_b, off, mean_b) == n
        torch.cuda.synchronize()
        a = out_a.cpu().numpy()
        b = out_b.cpu().numpy()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), fmt
        ma, mb = mean_a.cpu().numpy(), mean_b.cpu().numpy()
        assert np.all(np.abs(ma - mb) <= 1e-12 * np.maximum(1.0, np.abs(mb))), (fmt, ma, mb)


def test_no_alloc_unpack_dc_refuses_calls_beyond_its_scratch():
    lib = ak.load()
    noalloc = _entry(lib, "atkdsp_gpu_unpack_dc_noalloc")
    n = MAX_SAMPLES + 1
    raw = torch.zeros(2 * n, dtype=torch.int16, device="cuda")
    out = torch.zeros(n, dtype=torch.complex64, device="cuda")
    mean = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _call(noalloc, raw, "ci16", n, out, 0.5 + 0.5j, mean) == -1
    torch.cuda.synchronize()
    assert not out.any().item() and not mean.any().item()      # nothing written
    # the limit itself is accepted
    assert _call(noalloc, raw, "ci16", MAX_SAMPLES, out, 0.5 + 0.5j, mean) == MAX_SAMPLES
    torch.cuda.synchronize()
    m = mean.cpu().numpy()                     # raw zeros: the mean before the offset is 0
    assert abs(m[0]) < 1e-12 and abs(m[1]) < 1e-12
    assert torch.all(out[:MAX_SAMPLES] == complex(-0.5, -0.5)).item()
