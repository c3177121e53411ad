"""The serving loop: continuous batching gives each stream exactly what it
gets alone; admission by free HBM; close/reopen; the load generator runs.

"Same alone and in the mix": several streams of different nchan / taps /
formats, blocks submitted unevenly (some streams several blocks ahead, some
idle in a round), rounds launched while others are still on the GPU -- every
stream's output must equal a standalone handle fed the same blocks through
the drop-in API, bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

import atkdsp_b200 as ak
from atkdsp_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
FS = 2.4e6


def test_each_stream_same_alone_and_in_the_mix():
    from atkdsp_b200.serve import Server
    srv = Server(max_streams=32, hbm_reserve=1 << 30)
    specs = [(64, 2, 16, "ci16"), (256, 2, 16, "ci16"), (1024, 2, 16, "ci16"), (1024, 2, 12, "cf32"),
             (4096, 2, 8, "cf32"), (256, 4, 8, "ci16q11"), (128, 1, 12, "cf32")]
    ids, alone = [], []
    for M, os_, K, fmt in specs:
        sid = srv.open(FS, M, os_, K, 80.0, fmt)
        assert sid >= 0
        ids.append(sid)
        alone.append(ak.Pfb(FS, M, os_, K))
    rng = np.random.default_rng(3)
    outs_mix = {i: [] for i in range(len(specs))}
    outs_alone = {i: [] for i in range(len(specs))}
    keep = []
    tagmap = {}
    tag = 0
    for rnd in range(6):
        for i, (M, os_, K, fmt) in enumerate(specs):
            nblk = int(rng.integers(0, 3))           # 0, 1 or 2 blocks this round
            for _ in range(nblk):
                n = int(rng.integers(1, 9000))
                if fmt == "cf32":
                    x = W.tones_noise(n, 2, 15.0, rng)
                    dev = torch.from_numpy(x).cuda()
                    ref_in = x
                else:
                    raw = np.clip(rng.normal(0, 900, (n, 2)), -2048, 2047).astype("<i2")
                    dev = torch.from_numpy(raw.reshape(-1)).cuda()
                    ref_in, _ = ak.unpack_dc(raw.tobytes(), fmt, 0j)
                hop = M // os_
                cap = M * ((hop - 1 + n) // hop)
                out = torch.zeros(max(cap, 1), dtype=torch.complex64, device="cuda")
                keep.append((dev, out))
                assert srv.submit(ids[i], dev, out, tag=tag) == 0
                tagmap[tag] = (i, out)
                outs_alone[i].append(alone[i].process(ref_in))
                tag += 1
        srv.launch()
        for sid, tg, m, n, ta, td in srv.poll():
            i, out = tagmap[tg]
            M = specs[i][0]
            outs_mix[i].append((tg, out[: M * m].view(M, m).cpu().numpy()))
    for sid, tg, m, n, ta, td in srv.drain():
        i, out = tagmap[tg]
        M = specs[i][0]
        outs_mix[i].append((tg, out[: M * m].view(M, m).cpu().numpy()))
    for i in range(len(specs)):
        mix = [y for _, y in sorted(outs_mix[i], key=lambda t: t[0])]
        assert len(mix) == len(outs_alone[i]), i
        for a, b in zip(outs_alone[i], mix):
            assert a.shape == b.shape and np.array_equal(a, b), (i, specs[i])
    st = srv.stats()
    assert st["blocks_done"] == tag and st["admitted"] == len(specs)


def test_admission_by_free_hbm_and_close_reopen():
    from atkdsp_b200.serve import Server
    greedy = Server(max_streams=4, hbm_reserve=1 << 50)       # more than any GPU has
    assert greedy.open(FS, 256, 2, 16) == -2                  # ATKDSP_E_NOMEM: not admitted
    assert greedy.stats()["denied"] == 1
    srv = Server(max_streams=2, hbm_reserve=1 << 30)
    a, b = srv.open(FS, 256, 2, 16), srv.open(FS, 256, 2, 16)
    assert a >= 0 and b >= 0 and srv.open(FS, 256, 2, 16) == -3  # full
    x = torch.zeros(4096, dtype=torch.complex64, device="cuda")
    out = torch.zeros(256 * 32, dtype=torch.complex64, device="cuda")
    assert srv.submit(a, x, out) == 0
    assert srv.close(a) == 0                                    # queued block dropped
    assert srv.pending() == 0
    c = srv.open(FS, 1024, 2, 12)
    assert c == a                                                # the slot is reused
    assert srv.submit(c, x, torch.zeros(1024 * 8, dtype=torch.complex64, device="cuda")) == 0
    done = srv.drain()
    assert len(done) == 1 and done[0][0] == c and done[0][2] == 8


def test_load_generator_runs():
    from atkdsp_b200.serve import Server, simulate
    srv = Server(max_streams=128, hbm_reserve=1 << 30)
    raw = torch.randint(-3000, 3000, (2 * (1 << 20),), dtype=torch.int16, device="cuda")
    out = torch.empty(64 << 20, dtype=torch.complex64, device="cuda")
    r = simulate(srv, streams=64, duration_s=0.6, warmup_s=0.1, raw_pool=raw, out_pool=out)
    assert r["blocks_done"] > 0 and r["admitted"] >= 64
    assert 0 < r["lat_p50_ms"] <= r["lat_p99_ms"] <= r["lat_max_ms"]
    assert r["blocks_per_round"] >= 1.0


def test_reopened_stream_reuses_a_parked_handle_with_clean_state():
    """A closed stream's handle is parked and handed to the next open of the
    same filter -- here while the closed stream's last round may still be on
    the GPU. The new stream must behave exactly like a fresh handle: its
    state cleared, its hop counter at zero."""
    from atkdsp_b200.serve import Server
    srv = Server(max_streams=4, hbm_reserve=1 << 30)
    rng = np.random.default_rng(11)
    M, os_, K = 256, 2, 16
    a = srv.open(FS, M, os_, K)
    keep = []
    for _ in range(3):                                   # give stream a some history
        x = torch.from_numpy(W.tones_noise(5000, 3, 15.0, rng)).cuda()
        out = torch.zeros(M * 40, dtype=torch.complex64, device="cuda")
        keep.append((x, out))
        assert srv.submit(a, x, out) == 0
    srv.launch()                                         # in flight when closed
    assert srv.close(a) == 0
    b = srv.open(FS, M, os_, K)                          # takes the parked handle
    assert b >= 0
    fresh = ak.Pfb(FS, M, os_, K)
    got, want = [], []
    for blk in (3000, 7, 12000):
        x = W.tones_noise(blk, 2, 15.0, rng)
        d = torch.from_numpy(x).cuda()
        hop = M // os_
        out = torch.zeros(M * ((hop - 1 + blk) // hop) + M, dtype=torch.complex64, device="cuda")
        keep.append((d, out))
        assert srv.submit(b, d, out, tag=blk) == 0
        want.append(fresh.process(x))
    done = srv.drain()
    for sid, tag, m, n, ta, td in done:
        if sid == b:
            out = [o for (d, o) in keep if d.numel() == n][-1]
            got.append((tag, out[: M * m].view(M, m).cpu().numpy()))
    got = [y for _, y in sorted(got, key=lambda t: [3000, 7, 12000].index(t[0]))]
    assert len(got) == 3
    for y, r in zip(got, want):
        assert y.shape == r.shape and np.array_equal(y, r)
