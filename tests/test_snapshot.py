"""SEREN binary snapshots (io/write_data_seren_unform.F90 layout): round trips,
record framing checked with an independent Fortran-record reader, subrecords."""
import io
import struct

import numpy as np
import pytest

from seren_b200 import snapshot as snap


def _sample(n=257, seed=0):
    rng = np.random.default_rng(seed)
    return dict(r=rng.normal(size=(n, 3)), m=np.full(n, 1.0 / n), h=rng.uniform(0.01, 0.1, n),
                v=rng.normal(size=(n, 3)), rho=rng.uniform(0.5, 2.0, n),
                temp=np.full(n, 10.0))


@pytest.mark.parametrize("pr", [8, 4])
def test_round_trip(tmp_path, pr):
    d = _sample()
    sinks = [dict(r=np.array([0.1, 0.2, 0.3]), v=np.array([1.0, 0.0, 0.0]), m=1.0, h=0.05,
                  radius=0.1, id=7, ncreate=3, accrete=True, static=False, tcreate=0.5)]
    p = tmp_path / f"s{pr}.bin"
    snap.write_seren_unform(str(p), pr=pr, sinks=sinks, time=1.25, snapshot=4, nsteps=99,
                            h_fac=1.2, dmdt_range=2, **d)
    s = snap.read_seren_unform(str(p))
    tol = 0 if pr == 8 else 1e-6
    assert s["PR"] == pr and s["NDIM"] == 3 and s["VDIM"] == 3 and s["BDIM"] == 3
    assert s["ptot"] == 257 and s["pgas"] == 257 and s["stot"] == 1
    assert s["data_id"] == ["porig", "r", "m", "h", "v", "rho", "temp", "sink_v1"]
    assert s["typedata"][1].tolist() == [3, 1, 257, 4, 1]
    assert np.array_equal(s["porig"], np.arange(1, 258))
    for k in ("r", "m", "h", "v", "rho", "temp"):
        assert np.allclose(s[k], d[k], rtol=tol, atol=0), k
    assert s["time"] == 1.25 and s["snapshot"] == 4 and s["nsteps"] == 99
    assert abs(s["h_fac"] - 1.2) <= tol * 2
    (sk,) = s["sinks"]
    assert sk["id"] == 7 and sk["ncreate"] == 3 and sk["accrete"] and not sk["static"]
    assert np.allclose(sk["r"], [0.1, 0.2, 0.3], rtol=tol) and abs(sk["m"] - 1.0) <= tol
    assert sk["macc"].shape == (2,)
    parray, v, sinks_rmh = snap.to_hot_path(s)
    assert parray.shape == (257, 6) and np.allclose(parray[:, 4], d["h"], rtol=tol)
    assert sinks_rmh.shape == (1, 5)


def test_records_read_by_an_independent_fortran_reader(tmp_path):
    """scipy's FortranFile (4-byte markers) reads the same records in the
    order write_data_seren_unform.F90:134-147 writes them."""
    from scipy.io import FortranFile
    d = _sample(n=33)
    p = tmp_path / "f.bin"
    snap.write_seren_unform(str(p), **d)
    with FortranFile(str(p), "r") as f:
        assert f.read_record(dtype="S20")[0].decode().rstrip() == "SERENBINARYDUMPV2"
        assert [int(f.read_ints(np.int32)[0]) for _ in range(4)] == [8, 3, 3, 3]
        idata = f.read_ints(np.int32)
        assert idata.size == 50 and idata[0] == 33 and idata[4] == 33 and idata[20] == 7
        assert f.read_ints(np.int64).size == 50
        assert f.read_reals(np.float64).size == 50                       # rdata, PR = 8
        dp = f.read_reals(np.float64)
        assert dp.size == 50 and abs(dp[2] - d["m"].sum()) < 1e-15       # mgas_orig
        ids = f.read_record(dtype="S20")
        assert [x.decode().rstrip() for x in ids] == ["porig", "r", "m", "h", "v", "rho", "temp"]
        td = f.read_ints(np.int32).reshape(7, 5)
        assert td[4].tolist() == [3, 1, 33, 4, 4]
        assert np.array_equal(f.read_ints(np.int32), np.arange(1, 34))
        assert np.array_equal(f.read_reals(np.float64).reshape(33, 3), d["r"])


def test_subrecords(monkeypatch):
    """Records longer than the subrecord limit split as gfortran splits them:
    leading marker negative while more follow, trailing marker negative on
    every continuation."""
    monkeypatch.setattr(snap, "_MAXREC", 10)
    buf = io.BytesIO()
    payload = bytes(range(25))
    snap._write_record(buf, payload)
    raw = buf.getvalue()
    marks = [struct.unpack("<i", raw[o:o + 4])[0] for o in (0, 14, 18, 32, 36, 45)]
    assert marks == [-10, 10, -10, -10, 5, -5]
    buf.seek(0)
    assert snap._read_record(buf) == payload


def test_not_a_snapshot(tmp_path):
    p = tmp_path / "x.bin"
    with open(p, "wb") as f:
        snap._write_record(f, b"SOMETHINGELSE".ljust(20))
    with pytest.raises(ValueError):
        snap.read_seren_unform(str(p))
