"""Batched independent clouds: the rank assignment, a two-rank gloo run that
shares the clouds out with no exchange, and the GPU batch against single-cloud
runs and the oracle."""
import os
import socket
import tempfile

import numpy as np
import pytest

from seren_b200 import ics
from seren_b200.batch import cloud_cost, lpt_partition, part_loads
from tests.helpers import params, rel_rows, run_pipeline


def test_lpt_partition_covers_every_cloud_once():
    ns = [int(x) for x in np.random.default_rng(3).integers(8192, 262144, 256)]
    for nparts in (1, 2, 3, 8, 300):
        parts = lpt_partition(ns, nparts)
        assert len(parts) == nparts
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(ns)))
        assert all(p == sorted(p) for p in parts)
        assert parts == lpt_partition(ns, nparts)          # same on every rank


def test_lpt_partition_is_balanced():
    ns = [int(x) for x in np.rint(np.exp(np.random.default_rng(1000).uniform(
        np.log(8192), np.log(262144), 256)))]
    for nparts in (2, 4, 8):
        loads = part_loads(ns, lpt_partition(ns, nparts))
        lower = max(sum(cloud_cost(n) for n in ns) / nparts, max(cloud_cost(n) for n in ns))
        # Graham's bound for longest-processing-time assignment
        assert max(loads) <= (4.0 / 3.0 - 1.0 / (3.0 * nparts)) * lower + 1e-6


def test_lpt_partition_rejects_no_ranks():
    with pytest.raises(ValueError):
        lpt_partition([10, 20], 0)


def _clouds():
    return ics.batched_clouds(ncloud=6, nmin=120, nmax=360, seed0=77)


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist

    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    clouds = _clouds()
    mine = lpt_partition([c["parray"].shape[0] for c in clouds], world)[rank]
    out = {}
    for i in mine:
        ic = clouds[i]
        r = run_pipeline(Oracle(ic["parray"].shape[0], params(ic)), ic)
        out[i] = (r["perm"], r["a"], r["gpot"])
    gathered = [None] * world
    dist.all_gather_object(gathered, sorted(out))          # bookkeeping only, no particle data
    if rank == 0:
        np.save(os.path.join(outdir, "owners.npy"), np.array(
            [[i, r] for r, ids in enumerate(gathered) for i in ids], dtype=np.int64))
    np.savez(os.path.join(outdir, f"rank{rank}.npz"),
             **{f"{k}_{i}": v for i, t in out.items() for k, v in zip(("perm", "a", "gpot"), t)})
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_ranks_share_the_clouds_without_exchange():
    import torch.multiprocessing as mp

    from oracle.oracle import Oracle
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank_main, args=(2, _free_port(), d), nprocs=2, join=True)
        owners = np.load(os.path.join(d, "owners.npy"))
        clouds = _clouds()
        assert sorted(owners[:, 0].tolist()) == list(range(len(clouds)))
        parts = lpt_partition([c["parray"].shape[0] for c in clouds], 2)
        for i, r in owners:
            assert i in parts[r]
        per_rank = [np.load(os.path.join(d, f"rank{r}.npz")) for r in range(2)]
        for i, ic in enumerate(clouds):
            ref = run_pipeline(Oracle(ic["parray"].shape[0], params(ic)), ic)
            z = per_rank[int(owners[owners[:, 0] == i][0, 1])]
            assert np.array_equal(z[f"perm_{i}"], ref["perm"])
            assert np.array_equal(z[f"a_{i}"], ref["a"])
            assert np.array_equal(z[f"gpot_{i}"], ref["gpot"])


@pytest.mark.gpu
def test_gpu_batch_equals_single_cloud_runs_and_oracle():
    from oracle.oracle import Oracle
    from seren_b200.batch import CloudBatch
    from seren_b200.gpu import GpuHotPath
    clouds = ics.batched_clouds(ncloud=4, nmin=1500, nmax=6000, seed0=1000)
    b = CloudBatch(clouds, precision=0)
    b.step(first_call=True)
    got = b.download()
    for ic, st in zip(clouds, got):
        n = ic["parray"].shape[0]
        g = GpuHotPath(n, params(ic))
        g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
        g.force_step(first_call=True)
        one = g.download()
        assert np.array_equal(st["perm"], one["perm"])
        assert np.array_equal(st["a"], one["a"])
        r = run_pipeline(Oracle(n, params(ic)), ic)
        assert np.array_equal(st["perm"], r["perm"])
        assert rel_rows(st["a"], r["a"]).max() < 1e-11
    b.close()


def _forest_clouds():
    """Uneven clouds, all in the same unit sphere (their trees overlap in
    space), sizes from just above pp_gather to tens of thousands, ragged."""
    sizes = [100, 777, 4096, 20000, 333, 2500, 9001]
    out = []
    for k, n in enumerate(sizes):
        ic = ics.uniform_sphere(n=n, seed=500 + k, sound=0.05 + 0.03 * k)
        ic["v"] = np.random.Generator(np.random.PCG64(600 + k)).normal(0.0, 0.1, (n, 3))
        out.append(ic)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_forest_equals_single_cloud_runs(precision):
    """seren_gpu_set_clouds: every cloud of a forest, built and walked in single
    launches over all clouds, equals a context holding that cloud alone bit for
    bit (order, h, rho, omega, a, gpot) through a first call, a drift and a
    second force step."""
    from seren_b200.gpu import GpuHotPath
    clouds = _forest_clouds()
    ns = [c["parray"].shape[0] for c in clouds]
    g = GpuHotPath(sum(ns), params(clouds[0], precision=precision))
    g.upload(np.vstack([c["parray"] for c in clouds]), np.vstack([c["v"] for c in clouds]),
             np.concatenate([c["sound"] ** 2 for c in clouds]))
    g.set_clouds(ns)
    g.force_step(first_call=True)
    g.drift(1.0e-3)
    g.force_step()
    st = g.download()
    g.close()
    off = 0
    for ic, n in zip(clouds, ns):
        one = GpuHotPath(n, params(ic, precision=precision))
        one.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
        one.force_step(first_call=True)
        one.drift(1.0e-3)
        one.force_step()
        d = one.download()
        one.close()
        rows = slice(off, off + n)
        assert np.array_equal(st["perm"][rows], d["perm"] + off)
        for k in ("parray", "rho", "omega", "a", "gpot"):
            assert np.array_equal(st[k][rows], d[k]), k
        off += n


@pytest.mark.gpu
def test_forest_whole_gpu_gradh_path():
    """With a tiny redo scratch (redo_cap = 8) the grad-h walks of many particles
    of every cloud go to the whole-GPU path, whose walks and passes run over a
    cover of the whole forest restricted to the particle's own cloud.  Its
    partial sums are grouped by slices and tiles of the whole forest, so the
    results equal single-cloud runs to the FP64 rounding of that grouping
    (1e-12), not bit for bit; the tree order is the same."""
    from seren_b200.gpu import GpuHotPath
    clouds = _forest_clouds()
    ns = [c["parray"].shape[0] for c in clouds]
    g = GpuHotPath(sum(ns), params(clouds[0], redo_cap=8))
    g.upload(np.vstack([c["parray"] for c in clouds]), np.vstack([c["v"] for c in clouds]),
             np.concatenate([c["sound"] ** 2 for c in clouds]))
    g.set_clouds(ns)
    g.force_step(first_call=True)
    assert g.last_step_stats()[2][8] > 0            # particles on the whole-GPU path
    st = g.download()
    g.close()
    off = 0
    for ic, n in zip(clouds, ns):
        one = GpuHotPath(n, params(ic, redo_cap=8))
        one.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
        one.force_step(first_call=True)
        d = one.download()
        one.close()
        rows = slice(off, off + n)
        assert np.array_equal(st["perm"][rows], d["perm"] + off)
        assert rel_rows(st["parray"][rows, 4], d["parray"][:, 4]).max() < 1e-12
        for k in ("rho", "omega"):
            assert rel_rows(st[k][rows], d[k]).max() < 1e-12, k
        assert rel_rows(st["a"][rows], d["a"]).max() < 1e-11
        off += n


@pytest.mark.gpu
def test_forest_refuses_what_it_does_not_support():
    from seren_b200.cabi import SerenError
    from seren_b200.gpu import GpuHotPath
    clouds = _forest_clouds()[:3]
    ns = [c["parray"].shape[0] for c in clouds]
    g = GpuHotPath(sum(ns), params(clouds[0]))
    g.upload(np.vstack([c["parray"] for c in clouds]), np.vstack([c["v"] for c in clouds]),
             np.concatenate([c["sound"] ** 2 for c in clouds]))
    with pytest.raises(SerenError):
        g.set_clouds([ns[0], ns[1]])                       # counts must add up to ptot
    g.set_clouds(ns)
    with pytest.raises(SerenError):
        g.set_sinks(np.array([[0.0, 0.0, 0.0, 1.0, 0.05]]))
    g.force_step(first_call=True)
    with pytest.raises(SerenError):
        g.block_start()
    g.close()


@pytest.mark.gpu
def test_cloud_forest_equals_cloud_batch():
    """seren_b200.batch.CloudForest (one forest context) gives every cloud the
    results of CloudBatch (one context per cloud), bit for bit, after two
    steps with a drift."""
    from seren_b200.batch import CloudBatch, CloudForest
    clouds = ics.batched_clouds(ncloud=5, nmin=800, nmax=5000, seed0=1000)
    got = []
    for cls in (CloudForest, CloudBatch):
        b = cls(clouds, precision=1)
        b.step(first_call=True)
        b.step(dt=1.0e-3)
        got.append(b.download())
        b.close()
    for f, one in zip(*got):
        for k in ("perm", "parray", "v", "rho", "omega", "a", "gpot"):
            assert np.array_equal(f[k], one[k]), k
