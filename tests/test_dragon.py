"""DRAGON snapshots (io/read_data_dragon_unform.F90, io/read_data_dragon_form.F90 and
their writers): files built here record by record, independently of the writers, then
read; the type sort, sink defaults, refusals, the binary writer's density-temperature
cut and round trips through both formats."""
import struct

import numpy as np
import pytest

from seren_b200 import snapshot as snap

# entry types in file order: gas, boundary, sink, intercloud, accreted, gas, boundary
TYPES = [1, 6, -1, 9, 0, 1, 6]


def _rec(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def _entries(n=len(TYPES)):
    k = np.arange(n, dtype=np.float64)
    return dict(pos=np.stack([k + 0.1, k + 0.2, k + 0.3], 1), vel=np.stack([-k, 2 * k, 3 * k], 1),
                temp=10.0 + k, h=0.01 * (k + 1), rho=1.0 + k, m=0.5 + k)


def _binary(path, types, pr=4, ids=None):
    e = _entries(len(types))
    real = "<f4" if pr == 4 else "<f8"
    idata = np.zeros(20, "<i4")
    idata[0], idata[1], idata[3], idata[19] = len(types), 12, 3, 99
    rdata = np.zeros(50, real)
    rdata[0], rdata[1], rdata[49] = 1.5, 1.25, 2.0
    body = _rec(idata.tobytes()) + _rec(rdata.tobytes())
    for k in ("pos", "vel", "temp", "h", "rho", "m"):
        body += _rec(np.asarray(e[k], real).tobytes())
    body += _rec(np.asarray(types, "<i4").tobytes())
    if ids is not None:
        body += _rec(np.asarray(ids, "<i4").tobytes())
    path.write_bytes(body)
    return e


@pytest.mark.parametrize("pr", [4, 8])
def test_binary_reader_sorts_types(tmp_path, pr):
    p = tmp_path / "a.du"
    e = _binary(p, TYPES, pr=pr)
    s = snap.read_dragon_unform(str(p))
    # boundary (file entries 2 and 7), intercloud (4), gas (1 and 6), 1-based
    order = [1, 6, 3, 0, 5]
    assert s["ptot"] == 5 and s["stot"] == 1 and s["pdead"] == 1
    assert (s["pboundary"], s["picm"], s["pgas"]) == (2, 1, 2)
    assert s["porig"].tolist() == [i + 1 for i in order]
    assert s["ptype"].tolist() == [6, 6, 9, 1, 1]
    real = np.float32 if pr == 4 else np.float64
    for k, key in (("pos", "r"), ("vel", "v"), ("temp", "temp"), ("h", "h"), ("rho", "rho"),
                   ("m", "m")):
        assert np.array_equal(s[key], np.asarray(e[k], real)[order].astype(np.float64)), key
    (sk,) = s["sinks"]
    assert np.array_equal(sk["r"], np.asarray(e["pos"][2], real).astype(np.float64))
    assert sk["m"] == np.float64(real(e["m"][2])) and sk["accrete"] and not sk["static"]
    assert sk["radius"] == 2.0 * sk["h"]
    assert s["nsteps"] == 12 and s["snapshot"] == 3 and s["pgas_orig"] == 99
    assert s["time"] == 1.5 and s["lastsnap"] == 1.25 and s["mgas_orig"] == 2.0


def test_binary_reader_ids_and_refusals(tmp_path):
    p = tmp_path / "a.du"
    _binary(p, TYPES, ids=[11, 12, 0, 14, 15, 16, 17])
    s = snap.read_dragon_unform(str(p), ids=True)
    assert s["porig"].tolist() == [12, 17, 14, 11, 16]
    _binary(p, [1, 4, 1])
    with pytest.raises(ValueError, match="splitting"):
        snap.read_dragon_unform(str(p))
    _binary(p, [1, 10, 1])                      # the binary reader counts no dark matter
    with pytest.raises(ValueError, match="add up"):
        snap.read_dragon_unform(str(p))
    p.write_bytes(_rec(b"\0" * 16))
    with pytest.raises(ValueError, match="not a DRAGON"):
        snap.read_dragon_unform(str(p))


def _ascii(path, types, ids=None):
    e = _entries(len(types))
    lines = [str(len(types)), "12", "0", "3"] + ["0"] * 15 + ["99"]
    # header reals, one read statement each: a D exponent; a repeat count on a
    # line gives one value, the rest of the line is dropped
    lines += ["1.5D0", "1.25"] + ["47*0.0"] * 47 + ["2.0"]
    for row in e["pos"]:
        lines.append(f"{float(row[0])!r}, {float(row[1])!r}")   # one vector over two lines
        lines.append(f"{float(row[2])!r}   trailing words are skipped")
    lines.append("3*0.0")                              # velocity of the first entry
    for row in e["vel"][1:]:
        lines.append(" ".join(repr(float(x)) for x in row))
    for k in ("temp", "h", "rho", "m"):
        lines += [repr(float(x)) for x in e[k]]
    lines += [f"{t}.0" for t in types]                 # types are read as reals
    if ids is not None:
        lines += [str(i) for i in ids]
    path.write_text("\n".join(lines) + "\n")
    return e


def test_ascii_reader_rounds_to_single_and_takes_dark_matter(tmp_path):
    p = tmp_path / "a.df"
    types = TYPES + [10]
    e = _ascii(p, types, ids=list(range(101, 109)))
    s = snap.read_dragon_form(str(p), ids=True)
    order = [1, 6, 3, 0, 5, 7]                        # dark matter after the gas
    assert s["ptot"] == 6 and s["pcdm"] == 1 and s["stot"] == 1
    assert s["porig"].tolist() == [101 + i for i in order]
    for k, key in (("pos", "r"), ("vel", "v"), ("h", "h"), ("m", "m")):
        want = np.asarray(e[k], np.float64)[order].astype(np.float32).astype(np.float64)
        assert np.array_equal(s[key], want), key
    assert s["r"][3, 0] != e["pos"][0, 0]             # 0.1 does not survive float32
    assert s["time"] == 1.5 and s["mgas_orig"] == 2.0
    assert s["sinks"][0]["radius"] == 2.0 * s["sinks"][0]["h"]


def test_binary_writer_cut_and_round_trip(tmp_path):
    n = 6
    rng = np.random.default_rng(3)
    r, v = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    m, h = np.full(n, 0.25), rng.uniform(0.01, 0.1, n)
    rho = np.array([1e-14, 1e-12, 1e-14, 1.0, 1e-15, 1e-10])
    temp = np.array([2000.0, 2000.0, 10.0, 10.0, 5000.0, 10.0])
    sinks = [dict(r=[0.5, 0.5, 0.5], v=[0.0, 1.0, 0.0], m=2.0, h=0.2)]
    p = tmp_path / "w.du"
    kept = snap.write_dragon_unform(str(p), r, m, h, v, rho, temp, sinks=sinks, pr=8, ids=True,
                                    time=3.0, snapshot=5, nsteps=40, rhosink=7.0)
    keep = [1, 2, 3, 5]                               # rho > 1e-13 or temp < 1000
    assert kept == 4
    s = snap.read_dragon_unform(str(p), ids=True)
    assert s["idata"][0] == 5 and s["idata"][2] == 4 and s["ptot"] == 4 and s["stot"] == 1
    assert np.array_equal(s["r"], r[keep]) and np.array_equal(s["rho"], rho[keep])
    assert s["porig"].tolist() == [k + 1 for k in keep]
    assert s["sinks"][0]["m"] == 2.0 and s["sinks"][0]["radius"] == 0.4
    assert s["time"] == 3.0 and s["snapshot"] == 5 and s["nsteps"] == 40
    parray, vv, sk = snap.to_hot_path(s)
    assert parray.shape == (4, 6) and np.array_equal(parray[:, 4], h[keep])
    assert sk.shape == (1, 5) and np.array_equal(vv, v[keep])


@pytest.mark.parametrize("pr", [8, 4])
def test_ascii_writer_round_trip(tmp_path, pr):
    n = 9
    rng = np.random.default_rng(4)
    r, v = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    m, h, rho = rng.uniform(0.1, 1, n), rng.uniform(0.01, 0.1, n), rng.uniform(0.5, 2, n)
    types = [6, 9, 1, 1, 1, 1, 1, 1, 1]
    p = tmp_path / "w.df"
    snap.write_dragon_form(str(p), r, m, h, v, rho, ptype=types, pr=pr, ids=True,
                           sinks=[dict(r=[0, 0, 1], m=1.0, h=0.3)], time=0.75)
    s = snap.read_dragon_form(str(p), ids=True)
    sp = lambda a: np.asarray(a, np.float64).astype(np.float32).astype(np.float64)  # noqa: E731
    assert s["ptot"] == n and s["stot"] == 1 and (s["pboundary"], s["picm"]) == (1, 1)
    assert np.array_equal(s["r"], sp(r)) and np.array_equal(s["m"], sp(m))
    assert s["porig"].tolist() == list(range(1, n + 1)) and s["time"] == 0.75
    assert s["sinks"][0]["h"] == sp(0.3)
