"""Host-side fault injection: out-of-memory at every allocation of create, and
the rule that a process call allocates nothing.

atkdsp_gpu_fail_alloc_after(n) makes the n-th device / pool / pinned
allocation fail as cudaMalloc would on an exhausted device (the reference's
ATKDSP_E_NOMEM path, include/atkdsp.h:202-209); no kernel is involved and no
GPU fault is raised. Checked here:

* create returns NULL (AtkDspError in Python) whichever allocation fails,
  frees what it had taken, and the next create works and computes the
  reference's outputs;
* process / process_n, small and chunked, allocate nothing (the reference's
  rule 2, include/atkdsp.h:10-14): the armed hook survives them and fires at
  the next create instead;
* the server's open reports E_NOMEM and admits nothing;
* a host W1 call whose staging cannot be allocated leaves R and counts as
  they were.
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from conftest import run_blocks
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FS = 2.4e6


def _arm(n):
    ak.load().atkdsp_gpu_fail_alloc_after(n)


def test_create_fails_cleanly_at_every_allocation():
    x = (np.random.default_rng(1).standard_normal(20000) * (1 + 1j)).astype(np.complex64)
    free0 = torch.cuda.mem_get_info()[0]
    failed = 0
    try:
        for k in range(1, 40):
            _arm(k)
            try:
                p = ak.Pfb(FS, 1024, 2, 12, 80.0, 2)
            except ak.AtkDspError:
                failed += 1
                continue
            _arm(0)                           # create made fewer than k allocations
            del p
            break
    finally:
        _arm(0)
    assert failed >= 5                         # create allocates state, staging, tables, ...
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] < (64 << 20)    # nothing of note left behind
    y = run_blocks(ak.Pfb(FS, 1024, 2, 12, 80.0, 1), [x], [5000, 3, 20000])
    r = run_blocks(O.oracle().Pfb(FS, 1024, 2, 12, 80.0, 1), [x], [5000, 3, 20000])
    assert y.shape == r.shape and np.max(np.abs(y - r)) <= 1e-5 * np.max(np.abs(r))


def test_process_calls_allocate_nothing():
    rng = np.random.default_rng(2)
    p = ak.Pfb(FS, 256, 2, 16, 80.0, 2)
    xs = [(rng.standard_normal(1 << 22) + 1j * rng.standard_normal(1 << 22)).astype(np.complex64)
          for _ in range(2)]
    p.process_n([x[:10] for x in xs], 2)        # first calls: nothing to warm up either way
    _arm(1)
    try:
        for n in (1, 7, 999, 4096, 33333, 1 << 22):       # small calls and a multi-chunk one
            p.process_n([x[:n] for x in xs], 2)
        with pytest.raises(ak.AtkDspError):
            ak.Pfb(FS, 256, 2, 16, 80.0, 1)               # the hook was still armed
    finally:
        _arm(0)


def test_server_open_reports_out_of_memory():
    from atkdsp_b200.serve import Server
    srv = Server(max_streams=8, hbm_reserve=1 << 30)
    before = srv.stats()
    _arm(1)
    try:
        sid = srv.open(FS, 512, 2, 16, 80.0, "ci16")
    finally:
        _arm(0)
    assert sid == -2                                   # ATKDSP_E_NOMEM
    after = srv.stats()
    assert after["admitted"] == before["admitted"]
    assert srv.open(FS, 512, 2, 16, 80.0, "ci16") >= 0


def test_host_w1_leaves_outputs_when_staging_fails():
    import threading
    rng = np.random.default_rng(3)
    y = (rng.standard_normal((2, 64, 50)) + 1j * rng.standard_normal((2, 64, 50))).astype(np.complex64)
    R = np.full((64, 2, 2), 1 + 2j, np.complex64)
    c = np.full(64, 7, np.uint32)

    def call():                    # a fresh thread: its first call allocates its staging
        _arm(1)
        try:
            ak.pfb_cov_accumulate(y, 2, 64, None, R, c)
        finally:
            _arm(0)

    t = threading.Thread(target=call)
    t.start()
    t.join()
    assert np.all(R == 1 + 2j) and np.all(c == 7)


def test_bounds_checks_report_and_skip_without_touching_memory():
    """The tile kernel's window check: a step whose jobs claim fewer samples
    than their windows need (a host-side injection; the buffers hold every
    sample) has its last tiles and its carry skipped and reported, and the
    handle works again after a reset. Normal work reports nothing."""
    from atkdsp_b200 import gpu
    lib = ak.load()
    rng = np.random.default_rng(9)
    x = torch.from_numpy(W_noise(rng, 1024 * 40)).cuda()
    p = ak.Pfb(FS, 1024, 2, 12)
    y = gpu.process_n(p, [x], 1)
    assert lib.atkdsp_gpu_pfb_faults(p.handle) == 0
    out = torch.full((1024 * 80,), complex(7.0, 7.0), dtype=torch.complex64, device="cuda")
    lib.atkdsp_gpu_inject_short_window(100)
    m = y.shape[-1]
    gpu.process_n(p, [x], 1, out=out)
    f = lib.atkdsp_gpu_pfb_faults(p.handle)
    assert f > 0 and (f & 1) and (f & 4), f                  # last windows, and the carry
    o = out[: 1024 * m].view(1024, m).cpu().numpy()
    assert np.all(o[:, -1] == complex(7.0, 7.0))             # the last tile was not written
    assert lib.atkdsp_gpu_pfb_faults(p.handle) == 0           # cleared by the query
    p.reset()
    gpu.process_n(p, [x], 1, out=out)
    gpu.sync(p)
    assert np.array_equal(out[: 1024 * m].view(1024, m).cpu().numpy(), y[0].cpu().numpy())
    assert lib.atkdsp_gpu_pfb_faults(p.handle) == 0


def W_noise(rng, n):
    return ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)).astype(np.complex64)


def test_index_checked_build_runs_clean():
    """The library built with every kernel's per-thread index checks runs the
    filterbank shapes (staged, paired, quad, one hop per thread, nchan 4096,
    the generic and the large path) and W1/W2 with no index flagged, and
    matches the oracle. Run in a child process: it loads the other library."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    dbg = root / "atkdsp_b200" / "lib" / "libatkdsp_b200_debug.so"
    if not dbg.exists():
        pytest.skip("the index-checked library is not built (make -C atkdsp_b200 debug)")
    code = r"""
import numpy as np, atkdsp_b200 as ak
from conftest import run_blocks
from oracle import oracle as O
lib = ak.load()
assert lib.atkdsp_gpu_debug_build() == 1
rng = np.random.default_rng(3)
for M, os_, K, choice in ((64, 2, 8, 1), (256, 2, 12, 2), (1024, 2, 16, 1), (1024, 1, 8, 0), (4096, 2, 8, -1),
                          (192, 2, 6, -1), (8192, 2, 4, -1)):
    if choice >= 0:
        assert lib.atkdsp_gpu_tune_set(M, os_, K, choice) == 0
    n = M * K + 40 * (M // os_) + 5
    x = ((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / 2).astype(np.complex64)
    p = ak.Pfb(2.4e6, M, os_, K)
    y = run_blocks(p, [x], [1, 999, 4096, 7, n])
    r = run_blocks(O.oracle().Pfb(2.4e6, M, os_, K), [x], [1, 999, 4096, 7, n])
    assert y.shape == r.shape and np.max(np.abs(y - r)) <= 1e-5 * np.max(np.abs(r)), M
    assert lib.atkdsp_gpu_pfb_faults(p.handle) == 0, M
print("clean")
"""
    env = dict(os.environ, ATKDSP_B200_LIB=str(dbg), PYTHONPATH=f"{root}:{root / 'tests'}")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and "clean" in res.stdout, res.stdout + res.stderr
