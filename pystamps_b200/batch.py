"""Many stage-2 patches on one GPU and across GPUs.

`run_batched` loads every patch into its own context and runs them together
with ps2_batch_run: each gamma iteration is one launch per step over all
still-iterating patches (one persistent topofit launch per lane-width class).
`run_patches` is the stream-per-patch alternative (a context per worker
thread). Across GPUs, patches are spread by longest-processing-time (LPT)
assignment.

Patches are independent (the reference runs them one after another,
pystamps/pipeline/stages.py:184-221), so the multi-GPU split is by patch:
rank r runs the patches LPT gives it and only a small per-patch summary is
gathered to rank 0 at the end; no collective touches the data path.
"""
from __future__ import annotations

import ctypes
import math
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Sequence

from . import _lib
from ._lib import check
from .stage2 import PreparedPatch, Stage2Context

SUMMARY_KEYS = ("K_ps", "C_ps", "coh_ps", "N_opt")


def patch_cost(n_ps: int, n_ifg: int, n_trials: int, n_i: int, n_j: int) -> float:
    """Work estimate of one gamma iteration: the topofit sweep, (8T+32) flop
    per PS x ifg, plus CLAP, about 1.4e5 flop per window x ifg."""
    w = max(0, math.ceil(n_i / 6) - 3) * max(0, math.ceil(n_j / 6) - 3)
    return float(n_ps) * n_ifg * (8 * n_trials + 32) + w * n_ifg * 1.4e5


def prepared_cost(p: PreparedPatch) -> float:
    return patch_cost(p.n_ps, p.n_ifg, 2 * math.ceil(8 * p.n_trial_wraps) + 1, p.n_i, p.n_j)


def lpt_assign(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Longest processing time first: each patch, largest first, goes to the
    least loaded rank (ties: lower rank, lower index)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * n_ranks
    out: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += costs[i]
    return out


class Batch:
    """Loaded contexts of many patches, run together by ps2_batch_run."""

    def __init__(self, patches: Sequence[PreparedPatch], device: int = 0, load_threads: int = 8):
        self.device = device
        self.load_threads = load_threads
        self.patches: list[PreparedPatch] = []
        self.ctxs: list[Stage2Context] = []
        try:
            self.load(patches)
        except Exception:
            self.close()
            raise

    def load(self, patches: Sequence[PreparedPatch]) -> None:
        """(Re)load the patches, one context each; contexts and their device
        buffers are kept from the previous load where the counts allow. Loads
        run on `load_threads` host threads (the library releases the GIL; each
        context has its own stream)."""
        patches = list(patches)
        while len(self.ctxs) < len(patches):
            self.ctxs.append(Stage2Context(self.device))
        while len(self.ctxs) > len(patches):
            self.ctxs.pop().close()
        self.patches = patches
        if len(patches) > 1 and self.load_threads > 1:
            with ThreadPoolExecutor(max_workers=min(self.load_threads, len(patches))) as ex:
                list(ex.map(lambda cp: cp[0].load(cp[1], "fp32"), zip(self.ctxs, patches)))
        else:
            for c, p in zip(self.ctxs, patches):
                c.load(p, "fp32")

    def run(self) -> list[dict]:
        """All patches to convergence; per-patch last-iteration statistics."""
        n = len(self.ctxs)
        arr = (ctypes.c_void_p * n)(*[c._ctx.value for c in self.ctxs])
        st = (_lib.IterStats * n)()
        check(_lib.lib().ps2_batch_run(arr, ctypes.c_int64(n), st))
        return [s.as_dict() for s in st]

    def reset(self) -> None:
        for c in self.ctxs:
            c.reset()

    def timing_ms(self) -> float:
        return self.ctxs[0].timing()[0]

    def launch_count(self) -> int:
        return self.ctxs[0].launch_count()

    def download(self, keys=SUMMARY_KEYS) -> list[dict]:
        if len(self.ctxs) > 1 and self.load_threads > 1:
            with ThreadPoolExecutor(max_workers=min(self.load_threads, len(self.ctxs))) as ex:
                return list(ex.map(lambda c: c.download(keys), self.ctxs))
        return [c.download(keys) for c in self.ctxs]

    def close(self) -> None:
        for c in self.ctxs:
            c.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_batched(patches: Sequence[PreparedPatch], *, device: int = 0, keys=SUMMARY_KEYS) -> list[dict]:
    """Load, run together to convergence and download every patch."""
    with Batch(patches, device) as b:
        stats = b.run()
        res = b.download(keys)
        for r, st in zip(res, stats):
            r["stats"] = st
        return res


def run_patches(patches: Sequence[PreparedPatch], *, device: int = 0, streams: int = 4, precision: str = "fp32",
                keys=SUMMARY_KEYS, autotune: bool = False) -> list[dict]:
    """Run every patch to convergence on one GPU, `streams` at a time.

    Each worker thread owns a Stage2Context (its own CUDA stream and buffers);
    the library releases the GIL inside every call, so patches overlap on the
    GPU. Results come back in input order."""
    n = len(patches)
    results: list[dict | None] = [None] * n
    local = threading.local()
    ctxs: list[Stage2Context] = []
    lock = threading.Lock()

    def work(i: int) -> None:
        ctx = getattr(local, "ctx", None)
        if ctx is None:
            ctx = Stage2Context(device)
            local.ctx = ctx
            with lock:
                ctxs.append(ctx)
        ctx.load(patches[i], precision)
        if autotune:
            ctx.autotune()
        st = ctx.run()
        res = ctx.download(keys)
        res["stats"] = st
        res["ms"] = ctx.timing()[0]
        results[i] = res

    try:
        with ThreadPoolExecutor(max_workers=max(1, min(streams, n or 1))) as ex:
            list(ex.map(work, range(n)))
    finally:
        for c in ctxs:
            c.close()
    return results  # type: ignore[return-value]


def run_distributed(patches: Sequence, *, costs: Sequence[float] | None = None,
                    runner: Callable[[Sequence], list] | None = None, group=None) -> list | None:
    """Run `patches` across the ranks of the default process group.

    Every rank passes the same patch list (or lightweight descriptors that
    `runner` turns into work); rank r runs LPT's share with `runner` (default:
    run_patches on its GPU) and rank 0 returns all results in input order."""
    import torch.distributed as dist

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if costs is None:
        costs = [prepared_cost(p) for p in patches]
    share = lpt_assign(costs, world)[rank]
    run = runner or (lambda ps: run_patches(ps))
    mine = run([patches[i] for i in share])
    local = list(zip(share, mine))
    if world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    if rank != 0:
        return None
    out: list = [None] * len(patches)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
