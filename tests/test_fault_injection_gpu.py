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
