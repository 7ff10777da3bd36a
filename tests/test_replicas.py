"""Replica bookkeeping across ranks (replicas.py) with the gloo backend: two CPU processes.

Each rank draws exact samples for its own block of sample indices (the oracle stands in for the GPU engine), the
ranks' results gathered in rank order equal one process drawing the union, and the job time is the slowest rank's.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import case_plan_text

FIRST, COUNT, SEED = 40, 3, 123


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, plan_path, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import replicas
    from oracle import Oracle
    r, w, _ = replicas.init(backend="gloo", timeout_s=60)
    assert (r, w) == (rank, world)
    start, count = replicas.item_range(FIRST, COUNT, r)
    o = Oracle(plan_path)
    mine = [o.sample(0, SEED, i) for i in range(start, start + count)]
    allres = replicas.gather([(start, mine)], w)
    slowest = replicas.max_over_ranks(0.25 + r, w)
    replicas.barrier(w)
    if r == 0:
        np.save(os.path.join(out_dir, "gathered.npy"), np.array(
            [(s + i, ''.join(map(str, b)), lp) for part in allres for s, res in part for i, (b, lp) in enumerate(res)],
            dtype=object), allow_pickle=True)
        np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
    replicas.finish(w)


def test_two_gloo_replicas_cover_disjoint_samples(planner_cases, tmp_path):
    from oracle import Oracle
    case = [c for c in planner_cases["cases"] if c["n"] >= 8][0]
    path = str(tmp_path / "plan.txt")
    with open(path, "w") as f:
        f.write(case_plan_text(case)[0])
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), path, str(tmp_path)), nprocs=world, join=True)
    got = np.load(tmp_path / "gathered.npy", allow_pickle=True)
    o = Oracle(path)
    want = [(i,) + o.sample(0, SEED, i) for i in range(FIRST, FIRST + world * COUNT)]
    assert [int(g[0]) for g in got] == [w[0] for w in want]
    for g, (i, bits, lp) in zip(got, want):
        assert g[1] == ''.join(map(str, bits)) and abs(float(g[2]) - lp) <= 1e-12 * abs(lp)   # OpenMP sum order
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 1.25
