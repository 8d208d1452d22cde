"""The multi-GPU form is replicas: each rank scores its own source, nothing crosses ranks on the data path, and a
segment's accumulators from several ranks meet with es_accum_merge (src/stats.hpp:50-64). Its host side runs here on
CPU ranks (gloo, world size 2): the accumulators gathered and merged on rank 0 equal the oracle's merge, and bench.py's
reference arm, launched as a multi-GPU run is launched, prints one JSON line from rank 0 only."""

import ctypes
import datetime
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import es_b200
import oracle
from test_abi_cpu import make_accum

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 2


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_accum(rank):
    """Rank r's segment accumulator (and the oracle's), from its own seeded figures."""
    return make_accum(np.random.default_rng(100 + rank), 10 + rank, 120 + 10 * rank)


def _merge_worker(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, _ = rank_accum(rank)
        raw = torch.frombuffer(bytearray(ctypes.string_at(ctypes.addressof(a), ctypes.sizeof(a))), dtype=torch.uint8)
        parts = [torch.empty_like(raw) for _ in range(world)]
        dist.all_gather(parts, raw)
        if rank == 0:
            total = es_b200.new_accum()
            for p in parts:  # in rank order
                part = es_b200.Accum.from_buffer_copy(p.numpy().tobytes())
                es_b200.lib().es_accum_merge(ctypes.byref(total), ctypes.byref(part))
            with open(out_path, "w") as f:
                json.dump({"frames": total.frames, "lasting_n": total.lasting.n, "amount1": list(total.amount[1].bins),
                           "matching0": list(total.matching[0].bins), "all_r": list(total.all_r), "own": total.own,
                           "score": es_b200.accum_score(total).score}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_segment_accumulators_merge_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as tmp

    out = str(tmp_path / "merged.json")
    tmp.spawn(_merge_worker, args=(WORLD, free_port(), out), nprocs=WORLD, join=True)
    got = json.load(open(out))
    want = oracle.Accum()
    for r in range(WORLD):
        want.merge(rank_accum(r)[1])
    assert got["frames"] == want.frames == 10 + 11
    assert got["lasting_n"] == want.lasting.n
    assert np.array_equal(np.array(got["amount1"]), want.amount[1].bins)
    assert np.array_equal(np.array(got["matching0"]), want.matching[0].bins)
    assert np.allclose(got["all_r"], want.all_r, rtol=1e-15, atol=0)
    assert got["own"] == want.own
    assert got["score"] == pytest.approx(want.score()["score"], rel=1e-14)


def test_reference_arm_prints_one_line_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={WORLD}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", "bench.py", "--impl", "reference",
           "--gpus", str(WORLD), "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == WORLD and line["steps"] == 1
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
