"""Multi-GPU host logic on CPU: stream partition, and a world-size-2 gloo run
in which each rank channelizes its own shard (through the oracle, since there
is no GPU here) and the ranks agree on ownership and the reductions that
bench.py reports (max of the timed regions, sum of the work)."""

from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from atkdsp_b200.replicas import Replicas, partition

FS = 2.4e6


def _streams(n=12, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        M = int(rng.choice([16, 64, 256]))
        out.append({"id": i, "nchan": M, "os": int(rng.choice([1, 2])), "taps": int(rng.choice([4, 8])),
                    "length": int(rng.integers(1, 6000)), "seed": 100 + i})
    return out


def _channelize(s) -> str:
    """Two blocks of the stream through the oracle; digest of the outputs."""
    from oracle.oracle import oracle
    rng = np.random.default_rng(s["seed"])
    p = oracle().Pfb(FS, s["nchan"], s["os"], s["taps"])
    h = hashlib.sha256()
    for _ in range(2):
        x = (rng.standard_normal(s["length"]) + 1j * rng.standard_normal(s["length"])).astype(np.complex64)
        h.update(np.ascontiguousarray(p.process(x)).tobytes())
    return h.hexdigest()


def test_partition_is_disjoint_complete_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    w = list(rng.choice([2.4e6, 10e6, 40e6], 4096) * 4)
    for world in (1, 2, 3, 8):
        parts = partition(w, world)
        assert parts == partition(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - sum(w) / world <= max(w) + 1e-6
    assert partition([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    rep = Replicas(backend="gloo", timeout_s=60)
    try:
        streams = _streams()
        mine = rep.my_streams([8.0 * s["length"] for s in streams])
        digests = {s["id"]: _channelize(s) for s in streams if s["id"] in mine}
        gathered = rep.gather(digests)
        t_max = rep.max(1.5 + rank)
        work = rep.sum(sum(streams[i]["length"] for i in mine))
        rep.barrier()
        if rank == 0:
            with open(os.path.join(out_dir, "result.json"), "w") as f:
                json.dump({"gathered": gathered, "t_max": t_max, "work": work}, f)
    finally:
        rep.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_streams_and_reduce(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
        assert p.exitcode == 0
    res = json.loads((tmp_path / "result.json").read_text())
    streams = _streams()
    owned = [set(map(int, d)) for d in res["gathered"]]
    assert owned[0].isdisjoint(owned[1]) and owned[0] | owned[1] == set(range(len(streams)))
    assert all(owned)                                  # both ranks got work
    alone = {s["id"]: _channelize(s) for s in streams}
    for d in res["gathered"]:
        for k, v in d.items():
            assert alone[int(k)] == v                  # a shard's output is the stream's output
    assert res["t_max"] == 2.5
    assert res["work"] == sum(s["length"] for s in streams)
