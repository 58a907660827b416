"""Batched independent clouds: many small clouds, each with its own tree.

The clouds share nothing, so the ranks of a multi-GPU job share them out and
never exchange data: each cloud goes, in order of decreasing cost
N log N (the tree build and the walks grow as N log N), to the rank with the
least cost so far (longest-processing-time assignment, ties to the lower
rank).  Every rank computes the same assignment from the cloud sizes alone.
On its GPU a rank keeps one device-resident context per cloud, each with its
own CUDA stream, so a force evaluation of the batch is a set of device-resident
force steps that host threads issue side by side (the library's calls release
the interpreter lock); small clouds then share the GPU instead of queueing.
"""
from __future__ import annotations

import heapq
import math
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Sequence

from .cabi import Params


def cloud_cost(n: int) -> float:
    """Work model of one force evaluation of an N-particle cloud."""
    return float(n) * math.log(max(int(n), 2))


def lpt_partition(ns: Sequence[int], nparts: int) -> List[List[int]]:
    """Cloud indices per rank: longest processing time first, each cloud to the
    least-loaded rank (ties to the lower rank); indices ascending per rank."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(ns)), key=lambda i: (-cloud_cost(ns[i]), i))
    heap = [(0.0, r) for r in range(nparts)]
    parts: List[List[int]] = [[] for _ in range(nparts)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + cloud_cost(ns[i]), r))
    return [sorted(p) for p in parts]


def part_loads(ns: Sequence[int], parts: List[List[int]]) -> List[float]:
    return [sum(cloud_cost(ns[i]) for i in p) for p in parts]


def params_for(ic: Dict, precision: int) -> Params:
    return Params.make(h_fac=ic["h_fac"], thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"],
                       precision=precision)


class CloudBatch:
    """Device-resident contexts for one rank's clouds (seren_b200.gpu.GpuHotPath
    each, created on the current CUDA device)."""

    def __init__(self, clouds: Sequence[Dict], precision: int = 1, threads: int = 8):
        from .gpu import GpuHotPath
        self.threads = max(1, int(threads))
        self.ctx = []
        for ic in clouds:
            g = GpuHotPath(ic["parray"].shape[0], params_for(ic, precision))
            g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
            self.ctx.append(g)
        self.n = sum(ic["parray"].shape[0] for ic in clouds)

    def step(self, first_call: bool = False, dt: float = 0.0) -> int:
        """One force evaluation of every cloud (after a drift by dt when dt != 0);
        returns the number of kernels launched."""
        def one(g):
            n = 0
            if dt != 0.0:
                g.drift(dt)
                n += 1
            g.force_step(first_call=first_call)
            return n + g.last_step_stats()[1]

        if self.threads == 1 or len(self.ctx) < 2:
            return sum(one(g) for g in self.ctx)
        # largest clouds first, so the tail of the batch is short
        order = sorted(self.ctx, key=lambda g: -g.ptot)
        with ThreadPoolExecutor(max_workers=min(self.threads, len(order))) as ex:
            return sum(ex.map(one, order))

    def download(self) -> List[Dict]:
        return [g.download() for g in self.ctx]

    def close(self):
        for g in self.ctx:
            g.close()
        self.ctx = []
