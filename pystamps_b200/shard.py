"""One patch over several GPUs: the rows split into contiguous cell ranges.

The reference iterates one patch on one host (native_stage2.rs:261-406). Here a
patch too large or too slow for one GPU is split by rows: rank r owns the PS of
grid cells [lo_r, hi_r) (cells in grid_lin order, ranges balanced by PS count)
and holds a Stage2Context loaded with those rows only, in their original
relative order, so each cell's rows are binned in the reference's order. One
gamma iteration is

    ps2_shard_bin      the rank's rows into its copy of the grid
    halo exchange      each rank receives, from the ranks owning them, the
                       cells its CLAP windows read (cells are disjoint, so a
                       copy is the patch grid exactly)
    ps2_shard_filter   CLAP of the windows that meet the rank's rows of cells,
                       overlap-add of its own cells
    ps2_shard_fit      topofit of the rank's rows -> histogram, sum of squared
                       coherence changes, invalid count
    sum over ranks
    ps2_shard_finalize stop rule and P-square update from the sums (identical
                       on every rank, so every rank stops at the same iteration)

Per-PS results are those of one context over the whole patch; the convergence
RMS adds rank totals and can differ from it in the last bits.

run_sharded(prep, group) runs one rank under torch.distributed (NCCL for CUDA
tensors; per iteration a halo exchange of the grid cells each rank's CLAP
reads, point to point, and one all-reduce of 102 doubles). run_sharded_local(prep, n) runs n ranks as n contexts of one
process, the sums taken in rank order, the same arithmetic without a process
group.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Callable, Sequence

import numpy as np

from . import _lib
from ._lib import check, ptr
from .stage2 import PRECISION_FP64, PreparedPatch, Stage2Context

SHARD_STATS = 102  # PS2_SHARD_STATS: histogram [100], sum of squared changes, invalid rows


def split_cells(grid_lin: np.ndarray, n_cells: int, n_shards: int) -> list[tuple[int, int]]:
    """Contiguous cell ranges [lo, hi) covering 0..n_cells, one per shard, with
    about the same number of PS in each (a cell is never split)."""
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    gl = np.asarray(grid_lin, dtype=np.int64).reshape(-1)
    if gl.size and (gl.min() < 0 or gl.max() >= n_cells):
        raise ValueError("grid_lin outside 0..n_cells-1")
    if gl.size < n_shards:
        raise ValueError(f"{gl.size} PS cannot fill {n_shards} shards")
    counts = np.bincount(gl, minlength=n_cells)
    cum = np.cumsum(counts)
    bounds = [0]
    for k in range(1, n_shards):
        target = gl.size * k / n_shards
        c = int(np.searchsorted(cum, target, side="left")) + 1  # first cell after the crossing
        c = max(c, bounds[-1] + 1)
        bounds.append(min(c, n_cells))
    bounds.append(n_cells)
    ranges = [(bounds[k], bounds[k + 1]) for k in range(n_shards)]
    for lo, hi in ranges:
        if hi <= lo or cum[hi - 1] - (cum[lo - 1] if lo > 0 else 0) == 0:
            raise ValueError(f"shard cells [{lo}, {hi}) hold no PS; use fewer shards")
    return ranges


def shard_patch(p: PreparedPatch, lo: int, hi: int) -> tuple[PreparedPatch, np.ndarray]:
    """The sub-patch of the PS in cells [lo, hi) (rows kept in their relative
    order) and their row indices in the whole patch."""
    gl = np.asarray(p.grid_lin, dtype=np.int64)
    rows = np.nonzero((gl >= lo) & (gl < hi))[0]
    sub = dataclasses.replace(
        p, n_ps=int(rows.size), ph_nm=np.ascontiguousarray(p.ph_nm[rows]), amp=np.ascontiguousarray(p.amp[rows]),
        bperp=p.bperp if p.row_invariant else np.ascontiguousarray(p.bperp[rows]),
        grid_ij=np.ascontiguousarray(p.grid_ij[rows]), grid_lin=np.ascontiguousarray(gl[rows]),
        weight0=np.ascontiguousarray(p.weight0[rows]))
    return sub, rows


def needed_cells(lo: int, hi: int, n_i: int, n_j: int, n_win: int) -> tuple[int, int]:
    """Cells [c0, c1) whose binned values the CLAP of a rank owning cells
    [lo, hi) reads: every window that meets the rank's rows of cells spans
    n_win rows, so the rows from n_win - 1 above its first row to n_win - 1
    below its last (clipped to the grid) cover them all."""
    a, b = lo // n_j, (hi - 1) // n_j
    r0, r1 = max(0, a - n_win + 1), min(n_i - 1, b + n_win - 1)
    return r0 * n_j, (r1 + 1) * n_j


def halo_plan(ranges: Sequence[tuple[int, int]], n_i: int, n_j: int, n_win: int) -> list[tuple[int, int, int, int]]:
    """(src, dst, c0, c1) for every ordered pair of ranks: the cells of src's
    range that dst reads. Cells are disjoint between ranks, so dst's grid
    after receiving these slices holds the patch grid on every cell it reads."""
    need = [needed_cells(lo, hi, n_i, n_j, n_win) for lo, hi in ranges]
    plan = []
    for q, (lo, hi) in enumerate(ranges):
        for r, (n0, n1) in enumerate(need):
            c0, c1 = max(lo, n0), min(hi, n1)
            if q != r and c0 < c1:
                plan.append((q, r, c0, c1))
    return plan


def halo_exchange(grid, plan, rank: int, n_cells: int, group=None) -> None:
    """This rank's part of one halo exchange under torch.distributed: send
    the planned slices of its own cells, receive the slices it reads, in place
    in the flat grid buffer (n_cells rows of equal width)."""
    import torch.distributed as dist

    g = grid.view(-1, grid.numel() // n_cells)
    peer = (lambda r: r) if group is None else (lambda r: dist.get_global_rank(group, r))
    ops = []
    for q, dst, c0, c1 in plan:
        if q == rank:
            ops.append(dist.P2POp(dist.isend, g[c0:c1], peer(dst), group))
        elif dst == rank:
            ops.append(dist.P2POp(dist.irecv, g[c0:c1], peer(q), group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class ShardRank:
    """One rank's rows of a patch on one GPU, with the four shard calls."""

    def __init__(self, p: PreparedPatch, lo: int, hi: int, *, device: int = 0, precision: str = "fp32",
                 shapes=None):
        import torch

        self.lo, self.hi = int(lo), int(hi)
        self.sub, self.rows = shard_patch(p, lo, hi)
        self.ctx = Stage2Context(device)
        self.ctx.load(self.sub, precision)
        if shapes is not None:  # launch shapes pinned (Stage2Context.launch_shapes)
            self.ctx.launch_shapes(shapes)
        fp64 = self.ctx.precision == PRECISION_FP64
        mp = (p.n_ifg + 3) // 4 * 4
        self.grid = torch.zeros(p.n_i * p.n_j * mp * 2, dtype=torch.float64 if fp64 else torch.float32,
                                device=torch.device("cuda", device))
        self._lib = _lib.lib()

    def bin(self):
        check(self._lib.ps2_shard_bin(self.ctx._ctx, ctypes.c_void_p(self.grid.data_ptr())))
        return self.grid

    def filter(self, grid) -> None:
        import torch

        # the summed grid comes from torch's stream (collective or local sum);
        # the library reads it on its own stream
        torch.cuda.current_stream(grid.device).synchronize()
        check(self._lib.ps2_shard_filter(self.ctx._ctx, ctypes.c_void_p(grid.data_ptr()), ctypes.c_int64(self.lo),
                                         ctypes.c_int64(self.hi)))

    def fit(self) -> np.ndarray:
        st = np.zeros(SHARD_STATS, dtype=np.float64)
        check(self._lib.ps2_shard_fit(self.ctx._ctx, ctypes.c_void_p(ptr(st))))
        return st

    def finalize(self, stats: np.ndarray, n_total: int) -> dict:
        s = np.ascontiguousarray(stats, dtype=np.float64)
        it = _lib.IterStats()
        check(self._lib.ps2_shard_finalize(self.ctx._ctx, ctypes.c_void_p(ptr(s)), ctypes.c_int64(int(n_total)),
                                           ctypes.byref(it)))
        return it.as_dict()

    def download(self, keys=None) -> dict:
        return self.ctx.download(keys)

    def close(self) -> None:
        self.ctx.close()


def iterate_shards(ranks: Sequence, sum_grids: Callable, sum_stats: Callable, n_total: int,
                   max_iterations: int) -> dict:
    """The gamma loop over the ranks this process holds (one under a process
    group, all of them for the local form). sum_grids / sum_stats return the
    sum over every rank of the patch. Stops when finalize raises the stop flag
    (the same on every rank) or after max(max_iterations, 1) + 1 iterations,
    the bound of ps2_run_to_convergence."""
    last = None
    for _ in range(max(int(max_iterations), 1) + 1):
        grids = sum_grids([r.bin() for r in ranks])
        for r, g in zip(ranks, grids):
            r.filter(g)
        stats = sum_stats([r.fit() for r in ranks])
        its = [r.finalize(stats, n_total) for r in ranks]
        last = its[0]
        if any(it["stop"] != last["stop"] or it["i_loop"] != last["i_loop"] for it in its):
            raise RuntimeError("ranks disagree on the stop rule")
        if last["stop"]:
            break
    return last


def run_sharded_local(p: PreparedPatch, n_shards: int, *, device: int = 0, precision: str = "fp32",
                      keys=("K_ps", "C_ps", "coh_ps", "N_opt"), exchange: str = "halo", shapes=None) -> dict:
    """All shards of a patch as contexts of this process on one GPU (ranks
    emulated: the halo slices copied between the ranks' grids, or the grids
    summed in rank order). Returns the per-PS keys in the whole patch's row
    order, ph_grid if asked, and the last statistics."""
    import torch

    ranges = split_cells(p.grid_lin, p.n_i * p.n_j, n_shards)
    ranks = [ShardRank(p, lo, hi, device=device, precision=precision, shapes=shapes) for lo, hi in ranges]
    plan = halo_plan(ranges, p.n_i, p.n_j, p.clap_window)
    try:
        def sum_grids(gs):
            if exchange == "halo":
                w = gs[0].numel() // (p.n_i * p.n_j)
                views = [g.view(-1, w) for g in gs]
                for q, r, c0, c1 in plan:
                    views[r][c0:c1].copy_(views[q][c0:c1])
                return gs
            acc = torch.zeros_like(gs[0])
            for g in gs:
                acc += g
            return [acc] * len(gs)

        def sum_stats(ss):
            acc = np.zeros(SHARD_STATS)
            for s in ss:
                acc = acc + s
            return acc

        last = iterate_shards(ranks, sum_grids, sum_stats, p.n_ps, p.gamma_max_iterations)
        return _merge(p, ranks, keys, last)
    finally:
        for r in ranks:
            r.close()


def run_sharded(p: PreparedPatch, *, group=None, device: int | None = None, precision: str = "fp32",
                keys=("K_ps", "C_ps", "coh_ps", "N_opt"), rank_factory: Callable | None = None,
                exchange: str = "halo") -> dict:
    """This process's shard of a patch under torch.distributed (one rank per
    GPU; every rank passes the whole PreparedPatch and takes shard `rank` of
    `world`). Returns this rank's rows ("rows": their indices in the patch),
    its per-PS keys and the last statistics (the same on every rank).
    exchange "halo": each rank sends the other ranks only the cells of its
    range their CLAP windows read (halo_plan; point-to-point, at the
    full-scale shape about 23 of 256 cell rows per neighbour instead of the
    whole 78.6 MB grid); "allreduce": the grid summed over all ranks.
    rank_factory(p, lo, hi) replaces the GPU shard (host tests of the loop)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    ranges = split_cells(p.grid_lin, p.n_i * p.n_j, world)
    lo, hi = ranges[rank]
    plan = halo_plan(ranges, p.n_i, p.n_j, p.clap_window)

    if rank_factory is None:
        dev = torch.cuda.current_device() if device is None else int(device)
        r = ShardRank(p, lo, hi, device=dev, precision=precision)
    else:
        r = rank_factory(p, lo, hi)
    try:
        def sum_grids(gs):
            if exchange != "halo":
                dist.all_reduce(gs[0], op=dist.ReduceOp.SUM, group=group)
                return gs
            halo_exchange(gs[0], plan, rank, p.n_i * p.n_j, group)
            return gs

        def sum_stats(ss):
            t = torch.from_numpy(np.ascontiguousarray(ss[0], dtype=np.float64)).to(r.grid.device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            return t.cpu().numpy()

        # every rank joins one collective first (the communicator then exists
        # before the first point-to-point batch)
        dist.barrier(group=group)
        last = iterate_shards([r], sum_grids, sum_stats, p.n_ps, p.gamma_max_iterations)
        out = r.download(keys)
        out["rows"] = r.rows
        out["stats"] = last
        return out
    finally:
        r.close()


def _merge(p: PreparedPatch, ranks: Sequence[ShardRank], keys, last: dict) -> dict:
    out: dict = {"stats": last}
    per_ps = [k for k in keys if k in ("K_ps", "C_ps", "coh_ps", "N_opt", "coh_ps_save", "ph_res", "ph_patch",
                                       "ph_weight")]
    parts = [(r.rows, r.download(per_ps + (["ph_grid"] if "ph_grid" in keys and r is ranks[0] else [])))
             for r in ranks]
    for k in per_ps:
        first = parts[0][1][k]
        full = np.zeros((p.n_ps,) + first.shape[1:], dtype=first.dtype)
        for rows, d in parts:
            full[rows] = d[k]
        out[k] = full
    if "ph_grid" in keys:
        out["ph_grid"] = parts[0][1]["ph_grid"]
    out["i_loop"] = int(last["i_loop"])
    return out
