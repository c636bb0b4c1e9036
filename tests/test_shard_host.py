"""One patch over several ranks: the cell split and the iteration loop.

The split and sub-patch logic run on numpy. The loop (two all-reduces per
iteration, the stop rule taken from the summed statistics) runs as two gloo
ranks on CPU with a host stand-in for the GPU shard: each stand-in writes its
own cells of the grid, checks that it receives the whole grid back, reports
statistics from its rows and stops on the summed statistics, as
ps2_shard_finalize does.
"""
import os
import socket

import numpy as np
import pytest

from pystamps_b200 import shard
from pystamps_b200.stage2 import PreparedPatch


def _fake_prepared(n=600, m=5, n_i=12, n_j=10, seed=0, row_invariant=False):
    rng = np.random.default_rng(seed)
    gl = np.sort(rng.integers(0, n_i * n_j, n))
    rng.shuffle(gl)  # rows in any order
    return PreparedPatch(
        n_ps=n, n_ifg=m, ph_nm=rng.standard_normal((n, m)).astype(np.complex64),
        amp=np.ones((n, m), np.float32),
        bperp=(rng.standard_normal(m) if row_invariant else rng.standard_normal((n, m))).astype(np.float32),
        row_invariant=row_invariant, bperp_nm=rng.standard_normal(m),
        grid_ij=np.stack([gl // n_j + 1, gl % n_j + 1], axis=1).astype(np.float32), grid_lin=gl.astype(np.int64),
        n_i=n_i, n_j=n_j, weight0=rng.random(n), low_pass=np.ones((32, 32)), n_trial_wraps=5.0,
        nr=np.ones(100), nr_max_nz_ix=100.0, low_coh_thresh=31, psquare=True, gamma_change_convergence=0.005,
        gamma_max_iterations=6, clap_window=32, clap_alpha=1.0, clap_beta=0.3, grid_size=50.0)


@pytest.mark.parametrize("n_shards", [1, 2, 3, 7])
def test_split_cells_contiguous_and_balanced(n_shards):
    p = _fake_prepared()
    ranges = shard.split_cells(p.grid_lin, p.n_i * p.n_j, n_shards)
    assert ranges[0][0] == 0 and ranges[-1][1] == p.n_i * p.n_j
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    counts = np.bincount(p.grid_lin, minlength=p.n_i * p.n_j)
    sizes = [int(counts[lo:hi].sum()) for lo, hi in ranges]
    assert sum(sizes) == p.n_ps and min(sizes) > 0
    assert max(sizes) - p.n_ps / n_shards <= counts.max()


def test_split_cells_rejects_bad_requests():
    gl = np.array([0, 0, 0, 5])
    with pytest.raises(ValueError):
        shard.split_cells(gl, 6, 0)
    with pytest.raises(ValueError):
        shard.split_cells(gl, 6, 5)  # more shards than PS
    with pytest.raises(ValueError):
        shard.split_cells(np.array([0, 9]), 6, 1)  # cell outside the grid
    with pytest.raises(ValueError):
        shard.split_cells(np.zeros(10, np.int64), 6, 2)  # one cell cannot be split


@pytest.mark.parametrize("row_invariant", [False, True])
def test_shard_patch_keeps_rows_in_order(row_invariant):
    p = _fake_prepared(row_invariant=row_invariant)
    ranges = shard.split_cells(p.grid_lin, p.n_i * p.n_j, 3)
    seen = []
    for lo, hi in ranges:
        sub, rows = shard.shard_patch(p, lo, hi)
        assert np.all(np.diff(rows) > 0)
        assert sub.n_ps == rows.size
        assert np.all((sub.grid_lin >= lo) & (sub.grid_lin < hi))
        np.testing.assert_array_equal(sub.ph_nm, p.ph_nm[rows])
        np.testing.assert_array_equal(sub.weight0, p.weight0[rows])
        if row_invariant:
            assert sub.bperp is p.bperp
        else:
            np.testing.assert_array_equal(sub.bperp, p.bperp[rows])
        assert (sub.n_i, sub.n_j, sub.n_trial_wraps) == (p.n_i, p.n_j, p.n_trial_wraps)
        seen.append(rows)
    np.testing.assert_array_equal(np.sort(np.concatenate(seen)), np.arange(p.n_ps))


EXCHANGE = "halo"


class HostShard:
    """Stand-in for ShardRank on CPU: the grid holds, per cell, the sum of its
    rows' weight0 plus the iteration; statistics are the rows' counts per
    coherence bin and a sum that shrinks with the iteration."""

    def __init__(self, p, lo, hi):
        import torch

        self.p, self.lo, self.hi = p, lo, hi
        self.sub, self.rows = shard.shard_patch(p, lo, hi)
        self.grid = torch.zeros(p.n_i * p.n_j, dtype=torch.float64)
        self.it = 0
        self.grids_ok = []

    def bin(self):
        import torch

        g = np.zeros(self.p.n_i * self.p.n_j)
        np.add.at(g, self.sub.grid_lin, self.sub.weight0)
        g[self.lo:self.hi] += self.it
        self.grid.copy_(torch.from_numpy(g))
        return self.grid

    def filter(self, grid):
        whole = np.zeros(self.p.n_i * self.p.n_j)
        np.add.at(whole, self.p.grid_lin, self.p.weight0)
        whole += self.it
        c0, c1 = shard.needed_cells(self.lo, self.hi, self.p.n_i, self.p.n_j, self.p.clap_window)
        if EXCHANGE == "allreduce":
            c0, c1 = 0, whole.size
        self.grids_ok.append(bool(np.allclose(grid.numpy()[c0:c1], whole[c0:c1], rtol=0, atol=1e-12)))

    def fit(self):
        st = np.zeros(shard.SHARD_STATS)
        st[: 100] = np.bincount(self.rows % 100, minlength=100)
        st[100] = float(self.rows.size) / (self.it + 1)
        st[101] = float(self.lo)
        return st

    def finalize(self, stats, n_total):
        assert stats[:100].sum() == n_total
        self.it += 1
        rms = stats[100] / n_total
        return {"i_loop": self.it, "stop": int(rms < 0.3), "gamma_change_rms": rms}

    def download(self, keys=None):
        return {"K_ps": self.sub.weight0 * 2.0, "grids_ok": self.grids_ok}

    def close(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q, exchange="halo", n_i=12):
    import torch.distributed as dist

    global EXCHANGE
    EXCHANGE = exchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _fake_prepared(seed=3, n_i=n_i)
        out = shard.run_sharded(p, rank_factory=lambda pp, lo, hi: HostShard(pp, lo, hi), exchange=exchange)
        q.put((rank, out["rows"].tolist(), out["K_ps"].tolist(), out["grids_ok"], out["stats"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange,world,n_i", [("halo", 2, 12), ("allreduce", 2, 12), ("halo", 3, 80)])
def test_gloo_ranks_exchange_grid_and_statistics(exchange, world, n_i):
    """Two or three gloo ranks: every rank receives the patch grid on every
    cell its CLAP reads (the halo) or the whole summed grid, and all stop on
    the summed statistics. With 80 rows of cells and a 32-cell window the
    halo of a middle rank reaches both neighbours."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, exchange, n_i)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = sorted([q.get(timeout=300) for _ in range(world)])
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    p = _fake_prepared(seed=3, n_i=n_i)
    rows = np.concatenate([np.array(g[1]) for g in got])
    np.testing.assert_array_equal(np.sort(rows), np.arange(p.n_ps))
    for _, r, k, ok, _st in got:
        np.testing.assert_array_equal(np.array(k), p.weight0[np.array(r)] * 2.0)
        assert ok and all(ok)  # every rank received the whole grid every iteration
    # the stop rule came from the summed statistics: sum(rows)/(it+1)/n < 0.3 first at it = 3
    assert all(g[4] == got[0][4] for g in got)
    assert got[0][4]["i_loop"] == 4 and got[0][4]["stop"] == 1
    assert len(got[0][3]) == 4


def test_halo_plan_covers_every_window():
    """Each rank's needed rows contain every CLAP window that meets its rows
    (windows at stride n_win/4 with the reference's shifted edge windows,
    native_stage2.rs:957-995), and the plan delivers exactly the needed cells
    owned by other ranks."""
    n_i, n_j, nw = 70, 9, 24
    rng = np.random.default_rng(1)
    gl = rng.integers(0, n_i * n_j, 5000)
    ranges = shard.split_cells(gl, n_i * n_j, 5)
    inc = nw // 4
    wins = []
    for ix in range((n_i + inc - 1) // inc - 3):
        i1 = ix * inc
        wins.append(min(i1, n_i - nw))
    plan = shard.halo_plan(ranges, n_i, n_j, nw)
    for r, (lo, hi) in enumerate(ranges):
        c0, c1 = shard.needed_cells(lo, hi, n_i, n_j, nw)
        a, b = lo // n_j, (hi - 1) // n_j
        for i1 in wins:
            if i1 <= b and i1 + nw - 1 >= a:  # the window meets the rank's rows
                assert c0 <= i1 * n_j and (i1 + nw) * n_j <= c1
        got = np.zeros(n_i * n_j, bool)
        got[lo:hi] = True
        for q, dst, s0, s1 in plan:
            if dst == r:
                assert not got[s0:s1].any()
                got[s0:s1] = True
        assert got[c0:c1].all()
