"""Patch-parallel path across ranks (gloo, world size 2, CPU).

The oracle stands in for the GPU runner so the host logic (LPT assignment,
per-rank execution, gathering in input order) runs without a device.
"""
import os
import socket

import numpy as np
import pytest

from pystamps_b200 import batch


def test_lpt_assign_balances_and_covers():
    costs = [10, 9, 8, 7, 6, 5, 4, 3, 2, 1]
    parts = batch.lpt_assign(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(10))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert batch.lpt_assign([5.0], 4) == [[0], [], [], []]
    with pytest.raises(ValueError):
        batch.lpt_assign([1.0], 0)


def test_patch_cost_orders_work():
    small = batch.patch_cost(5_000, 30, 161, 24, 24)
    big = batch.patch_cost(400_000, 120, 161, 200, 200)
    assert big > 100 * small


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _tiny_patches():
    from pystamps_b200 import synth

    out = []
    for k, (n, m, cells) in enumerate([(800, 6, 24), (300, 5, 18), (1200, 8, 26), (500, 4, 24), (900, 7, 25)]):
        p = synth.make_patch(n, m, cells, 21, seed=900 + k, n_rand=400, gamma_max_iterations=3)
        p.pop("truth")
        out.append(p)
    return out


def _oracle_runner(patches):
    from oracle import oracle as O

    res = []
    for p in patches:
        r = O.stage2_run(p, threads=1)
        res.append({"coh_ps": r["coh_ps"], "K_ps": r["K_ps"], "i_loop": r["i_loop"]})
    return res


def _costs(patches):
    return [batch.patch_cost(p["ph"].shape[0], p["ph"].shape[1] - 1, 21, 20, 20) for p in patches]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        patches = _tiny_patches()
        out = batch.run_distributed(patches, costs=_costs(patches), runner=_oracle_runner)
        if rank == 0:
            q.put([(r["i_loop"], r["coh_ps"].tolist(), r["K_ps"].tolist()) for r in out])
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_every_patch_in_order():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    patches = _tiny_patches()
    ref = _oracle_runner(patches)
    assert len(got) == len(ref)
    for (il, coh, k), r in zip(got, ref):
        assert il == r["i_loop"]
        np.testing.assert_array_equal(np.array(coh), r["coh_ps"])
        np.testing.assert_array_equal(np.array(k), r["K_ps"])
    # both ranks had work
    parts = batch.lpt_assign(_costs(patches), 2)
    assert all(parts)
