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


class CloudForest:
    """One device-resident context holding one rank's clouds as a forest
    (seren_gpu_set_clouds): every force evaluation builds all the clouds'
    trees with one sort and one level-by-level split, and runs each stage
    (grad-h walk and passes, neighbour lists, hydro, gravity) as one launch
    over every cloud.  The clouds must share h_fac, theta and alpha (their
    sound speeds differ freely)."""

    def __init__(self, clouds: Sequence[Dict], precision: int = 1):
        import numpy as np

        from .gpu import GpuHotPath
        ic0 = clouds[0]
        for ic in clouds:
            if (ic["h_fac"], ic["thetamaxsqd"], ic["alpha"]) != \
                    (ic0["h_fac"], ic0["thetamaxsqd"], ic0["alpha"]):
                raise ValueError("the clouds of a forest share h_fac, theta and alpha")
        self.ns = [int(ic["parray"].shape[0]) for ic in clouds]
        self.offsets = [0]
        for n in self.ns[:-1]:
            self.offsets.append(self.offsets[-1] + n)
        self.n = sum(self.ns)
        self.g = GpuHotPath(self.n, params_for(ic0, precision))
        self.g.upload(np.vstack([ic["parray"] for ic in clouds]),
                      np.vstack([ic["v"] for ic in clouds]),
                      np.concatenate([np.asarray(ic["sound"]) ** 2 for ic in clouds]))
        self.g.set_clouds(self.ns)

    def step(self, first_call: bool = False, dt: float = 0.0) -> int:
        """One force evaluation of every cloud (after a drift by dt when
        dt != 0); returns the number of kernels launched."""
        n = 0
        if dt != 0.0:
            self.g.drift(dt)
            n += 1
        self.g.force_step(first_call=first_call)
        return n + self.g.last_step_stats()[1]

    def download(self) -> List[Dict]:
        """Per-cloud results in each cloud's tree order (perm: the cloud's own
        upload indices), as CloudBatch.download gives them."""
        st = self.g.download()
        out = []
        for off, n in zip(self.offsets, self.ns):
            rows = slice(off, off + n)
            d = {k: v[rows] for k, v in st.items()}
            d["perm"] = d["perm"] - off
            out.append(d)
        return out

    def close(self):
        self.g.close()
