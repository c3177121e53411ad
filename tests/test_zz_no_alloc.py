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


def _call_ptr(f, ptr, nbytes, fmt, out, n, off, mean):
    return f(C.c_void_p(ptr), nbytes, ak.FMT[fmt], C.c_void_p(out.data_ptr()), n, float(off.real),
             float(off.imag), None if mean is None else C.c_void_p(mean.data_ptr()), None)


@pytest.mark.parametrize("case", ["empty", "unaligned_ci16", "cf32_copy_no_mean"])
def test_no_alloc_unpack_dc_edge_paths(case):
    """The paths where the entry point's code differs from the allocating
    one's: an empty block (the mean is the offset), a raw pointer 4 bytes
    past a 16-byte boundary (the scalar conversion kernel), and cf32 with a
    zero offset and no mean (a plain copy). Each is run twice in a row, and
    must give the allocating entry point's samples and mean."""
    lib = ak.load()
    noalloc = _entry(lib, "atkdsp_gpu_unpack_dc_noalloc")
    alloc = _entry(lib, "atkdsp_gpu_unpack_dc")
    rng = np.random.default_rng(7)
    if case == "empty":
        fmt, off, n = "ci16q11", 0.25 - 0.5j, 0
        buf = torch.zeros(16, dtype=torch.int16, device="cuda")
        ptr, nbytes = buf.data_ptr(), 0
    elif case == "unaligned_ci16":
        fmt, off, n = "ci16", -0.125 + 0.0625j, 50_001
        buf = torch.from_numpy(rng.integers(-32768, 32768, 2 * n + 2, dtype=np.int64).astype("<i2")).cuda()
        ptr, nbytes = buf.data_ptr() + 4, 4 * n
        assert ptr % 16 == 4
    else:
        fmt, off, n = "cf32", 0j, 70_003
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
        buf = torch.from_numpy(x).cuda()
        ptr, nbytes = buf.data_ptr(), 8 * n
    want_mean = case != "cf32_copy_no_mean"
    for _ in range(2):
        out_a = torch.full((max(n, 1),), complex(7.0, 7.0), dtype=torch.complex64, device="cuda")
        out_b = out_a.clone()
        mean_a = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda") if want_mean else None
        mean_b = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda") if want_mean else None
        assert _call_ptr(noalloc, ptr, nbytes, fmt, out_a, n, off, mean_a) == n
        assert _call_ptr(alloc, ptr, nbytes, fmt, out_b, n, off, mean_b) == n
        torch.cuda.synchronize()
        assert np.array_equal(out_a.cpu().numpy().view(np.uint32), out_b.cpu().numpy().view(np.uint32)), case
        if want_mean:
            ma, mb = mean_a.cpu().numpy(), mean_b.cpu().numpy()
            assert np.all(np.abs(ma - mb) <= 1e-12 * np.maximum(1.0, np.abs(mb))), (case, ma, mb)
            if n == 0:
                assert np.allclose(ma, [np.float32(off.real), np.float32(off.imag)], rtol=0, atol=0)
