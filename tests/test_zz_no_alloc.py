"""seren_gpu_hydro_forces_noalloc: hydro accelerations for callers that cannot
allocate device memory.

Such a caller (an application whose GPU memory belongs to its own pool
allocator, or that runs under a fixed memory budget) cannot create a context,
so it hands the entry point device buffers it already owns; the kernel's
scratch lives in a fixed array inside the library.  Here torch owns the
buffers, standing in for the caller's allocator.  The results must equal those
of the context entry point seren_gpu_hydro_forces on the same state, on two
calls in a row with different particle sets (the second call runs on a
smaller set over what the first left in the shared scratch array).

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import case, params, rel_rows

pytestmark = pytest.mark.gpu

NOALLOC_PMAX = 32768


def _fn():
    from seren_b200.gpu import library
    f = library().seren_gpu_hydro_forces_noalloc
    f.restype = C.c_int
    f.argtypes = ([C.c_int32] + [C.c_void_p] * 8 + [C.c_int32] * 3 +
                  [C.c_double, C.c_void_p, C.c_void_p])
    return f


def _context_state(name, precision):
    """Particle state, neighbour lists and hydro accelerations from the
    context entry points (tree order, 0-based ids)."""
    from seren_b200.gpu import GpuHotPath
    ic = case(name)
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params(ic, precision=precision))
    try:
        p, perm = g.tree_update(ic["parray"])
        v = ic["v"][perm]
        s = g.sph_update(p, v, first_call=True)
        sound = ic["sound"][perm]
        press = sound * sound * s["rho"]
        a_ref = g.hydro_forces(press, sound)
        return dict(n=n, parray=s["parray"], v=v, rho=s["rho"], omega=s["omega"], press=press,
                    sound=sound, pptot=s["pptot"], pplist=s["pplist"],
                    L=g.params.pp_limit, kernel=g.params.kernel, alpha=g.params.alpha,
                    a_ref=a_ref)
    finally:
        g.close()


def _noalloc(st, precision, expect=0):
    import torch
    dev = torch.device("cuda:0")
    t = {k: torch.as_tensor(np.ascontiguousarray(st[k]), device=dev)
         for k in ("parray", "v", "rho", "omega", "press", "sound", "pptot", "pplist")}
    a = torch.full((st["n"], 3), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = _fn()(st["n"], *(t[k].data_ptr() for k in ("parray", "v", "rho", "omega", "press",
                                                    "sound", "pptot", "pplist")),
               st["L"], st["kernel"], precision, st["alpha"], a.data_ptr(), None)
    assert rc == expect, rc
    return a.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_hydro_equals_context_entry_point(precision):
    states = [_context_state("sphere4k", precision), _context_state("ragged777", precision)]
    for st in states:
        assert st["pptot"].max() <= st["L"]        # every row holds its whole list
    for st in states:                               # two calls in a row
        a = _noalloc(st, precision)
        assert np.all(np.isfinite(a))
        assert rel_rows(a, st["a_ref"]).max() <= 1e-12


def test_noalloc_rejects_sizes_beyond_its_scratch():
    # refused on the host before anything touches the GPU
    assert _fn()(NOALLOC_PMAX + 1, *([None] * 8), 114, 0, 0, 1.0, None, None) == 2
    assert _fn()(16, *([None] * 8), 114, 0, 0, 1.0, None, None) == 1


def test_noalloc_refuses_rows_it_cannot_evaluate_then_recovers():
    """The list checks made on the device: a row longer than pp_limit (the
    context entry point would walk the tree for it; there is no tree here)
    gives SEREN_GPU_ERR_CAPACITY, a listed id outside 0..n-1 gives
    SEREN_GPU_ERR_ARG.  The check only reads inside each row, and a refused
    call leaves nothing behind that changes the next call's results."""
    st = _context_state("ragged777", 0)
    L = st["L"]
    long_row = dict(st, pptot=st["pptot"].copy())
    long_row["pptot"][5] = L + 1
    _noalloc(long_row, 0, expect=2)
    bad_id = dict(st, pplist=st["pplist"].copy())
    bad_id["pplist"][7, 0] = st["n"]
    _noalloc(bad_id, 0, expect=1)
    a = _noalloc(st, 0)
    assert rel_rows(a, st["a_ref"]).max() <= 1e-12
