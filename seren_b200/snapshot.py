"""SEREN binary snapshots (format id SERENBINARYDUMPV2) read and written in
the layout of io/write_data_seren_unform.F90 and io/read_data_seren_unform.F90,
so that snapshots of the Fortran code can feed the GPU path and its results
can be read back by the Fortran tools.

The files are Fortran unformatted sequential files: every record is framed by
a 4-byte length before and after it; a record longer than 2**31 - 9 bytes is
split into subrecords whose leading length is negative while more follow
(gfortran's convention).  Records, in order (write_data_seren_unform.F90:134-147):

  format_id (character*20) | PR | NDIM | VDIM | BDIM (int32 each) |
  idata(50) int32 | ilpdata(50) int64 | rdata(50) real(PR) | dpdata(50) float64 |
  unit_data(nunit) character*20 (when nunit > 0) |
  data_id(ndata) character*20 | typedata(5, ndata) int32 (when ndata > 0) |
  one record per data block in data_id order (arrays of particles stored
  column-major: the components of one particle together) | sink records.

typedata(1:5, i) = (components, first, last, type, unit) with type 1 logical,
2 int32, 3 int64, 4 real(PR), 5 float64, 7 sinks (read_data_seren_unform.F90:
215-262).  Values are in the snapshot's units: the Fortran writer multiplies
by its unit scales, and a dimensionless run writes no unit records.
"""
from __future__ import annotations

import struct
from typing import Dict, List, Optional

import numpy as np

FORMAT_ID = "SERENBINARYDUMPV2"
_MAXREC = 2147483639          # longest subrecord gfortran writes
_TYPES = {1: np.dtype("<i4"), 2: np.dtype("<i4"), 3: np.dtype("<i8"), 5: np.dtype("<f8")}

# idata slots (write_data_seren_unform.F90:110-123)
_IDATA = {"ptot": 0, "stot": 1, "pboundary": 2, "picm": 3, "pgas": 4, "pcdm": 5, "pdust": 6,
          "pion": 7, "nunit": 19, "ndata": 20, "dmdt_range": 29, "pgas_orig": 30,
          "pp_gather": 31}


# ---------------------------------------------------------------------------
# record framing
def _read_record(f) -> bytes:
    parts = []
    while True:
        head = f.read(4)
        if len(head) < 4:
            raise EOFError("end of file inside a record")
        n = struct.unpack("<i", head)[0]
        size = -n if n < 0 else n
        parts.append(f.read(size))
        tail = struct.unpack("<i", f.read(4))[0]
        if abs(tail) != size:
            raise ValueError("Fortran record markers do not match")
        if n >= 0:
            return b"".join(parts)


def _write_record(f, payload: bytes) -> None:
    n = len(payload)
    if n == 0:
        f.write(struct.pack("<ii", 0, 0))
        return
    pos = 0
    while pos < n:
        size = min(_MAXREC, n - pos)
        more = pos + size < n
        # gfortran: leading marker negative while subrecords follow, trailing
        # marker negative on every subrecord after the first
        lead = -size if more else size
        trail = -size if pos > 0 else size
        f.write(struct.pack("<i", lead))
        f.write(payload[pos:pos + size])
        f.write(struct.pack("<i", trail))
        pos += size


def _chars(b: bytes, n: int) -> List[str]:
    return [b[20 * k:20 * (k + 1)].decode("ascii", "replace").rstrip() for k in range(n)]


def _pad(s: str) -> bytes:
    b = s.encode("ascii")
    if len(b) > 20:
        raise ValueError(f"identifier longer than 20 characters: {s!r}")
    return b.ljust(20, b" ")


# ---------------------------------------------------------------------------
def read_seren_unform(path: str) -> Dict:
    """A SEREN binary snapshot as a dict: header arrays (idata, ilpdata, rdata,
    dpdata), counts (ptot, stot, pgas, ...), units, data_id, typedata, the
    particle blocks by id (r [ptot, NDIM], m, h, v [ptot, VDIM], rho, temp, u, B,
    porig; any other id by its own name) and sinks (a list of dicts)."""
    out: Dict = {}
    with open(path, "rb") as f:
        fid = _read_record(f).decode("ascii", "replace").rstrip()
        if fid != FORMAT_ID:
            raise ValueError(f"not a SEREN binary snapshot (format id {fid!r})")
        pr = struct.unpack("<i", _read_record(f))[0]
        if pr not in (4, 8):
            raise ValueError(f"unknown real kind PR = {pr}")
        ndim = struct.unpack("<i", _read_record(f))[0]
        vdim = struct.unpack("<i", _read_record(f))[0]
        bdim = struct.unpack("<i", _read_record(f))[0]
        real = np.dtype("<f4") if pr == 4 else np.dtype("<f8")
        idata = np.frombuffer(_read_record(f), "<i4").copy()
        ilpdata = np.frombuffer(_read_record(f), "<i8").copy()
        rdata = np.frombuffer(_read_record(f), real).copy()
        dpdata = np.frombuffer(_read_record(f), "<f8").copy()
        out.update(format_id=fid, PR=pr, NDIM=ndim, VDIM=vdim, BDIM=bdim, idata=idata,
                   ilpdata=ilpdata, rdata=rdata, dpdata=dpdata)
        for k, i in _IDATA.items():
            out[k] = int(idata[i])
        nunit, ndata = out["nunit"], out["ndata"]
        if out["ptot"] != (out["pgas"] + out["picm"] + out["pboundary"] + out["pcdm"] +
                           out["pdust"] + out["pion"]):
            raise ValueError("particle counts do not add up (read_data_seren_unform.F90:100-101)")
        out["units"] = _chars(_read_record(f), nunit) if nunit > 0 else []
        data_id = _chars(_read_record(f), ndata) if ndata > 0 else []
        typedata = (np.frombuffer(_read_record(f), "<i4").reshape(ndata, 5).copy()
                    if ndata > 0 else np.zeros((0, 5), np.int32))
        out["data_id"], out["typedata"] = data_id, typedata
        out["time"], out["lastsnap"], out["mgas_orig"] = (float(dpdata[0]), float(dpdata[1]),
                                                          float(dpdata[2]))
        out["snapshot"], out["nsteps"] = int(ilpdata[0]), int(ilpdata[1])
        out["h_fac"], out["gamma"], out["mu_bar"] = (float(rdata[0]), float(rdata[1]),
                                                     float(rdata[2]))
        out["sinks"] = []
        for name, td in zip(data_id, typedata):
            comp, first, last, kind = int(td[0]), int(td[1]), int(td[2]), int(td[3])
            count = last - first + 1
            if name == "sink_v1" or kind == 7:
                out["sinks"] = _read_sinks(f, count, ndim, vdim, real, out["dmdt_range"])
                continue
            dt = real if kind == 4 else _TYPES.get(kind)
            if dt is None:
                raise ValueError(f"data block {name!r} has unknown type {kind}")
            a = np.frombuffer(_read_record(f), dt).copy()
            if kind == 1:
                a = a != 0
            if comp > 1:
                a = a.reshape(count, comp)
            out[name] = a
    return out


def _read_sinks(f, stot, ndim, vdim, real, dmdt_range) -> List[Dict]:
    # read_data_seren_unform.F90:178-213
    _read_record(f)                                   # nl, ni, nli, npr, ndp, nchar
    length = 11 + ndim + vdim + 2 * dmdt_range
    sinks = []
    for _ in range(stot):
        ld = np.frombuffer(_read_record(f), "<i4")
        ii = np.frombuffer(_read_record(f), "<i4")
        raux = np.frombuffer(_read_record(f), real).astype(np.float64)
        if raux.size != length:
            raise ValueError("sink record length differs from 11 + NDIM + VDIM + 2 DMDT_RANGE")
        b = ndim + vdim
        s = dict(accrete=bool(ld[0]), static=bool(ld[1]), id=int(ii[0]), ncreate=int(ii[1]),
                 tcreate=raux[0], r=raux[1:ndim + 1], v=raux[ndim + 1:b + 1], m=raux[b + 1],
                 h=raux[b + 2], radius=raux[b + 3], angmom=raux[b + 4:b + 7], dmdt=raux[b + 7],
                 star_radius=raux[b + 8], luminosity=raux[b + 9], temperature=raux[b + 10])
        if dmdt_range > 0:
            s["macc"] = raux[b + 11:b + 11 + dmdt_range]
            s["tacc"] = raux[b + 11 + dmdt_range:b + 11 + 2 * dmdt_range]
        sinks.append(s)
    return sinks


# ---------------------------------------------------------------------------
def write_seren_unform(path: str, r, m, h, v, rho, temp=None, u=None, porig=None,
                       sinks: Optional[List[Dict]] = None, pr: int = 8, time: float = 0.0,
                       lastsnap: float = 0.0, snapshot: int = 0, nsteps: int = 0,
                       h_fac: float = 1.2, gamma: float = 1.0, mu_bar: float = 2.35,
                       pp_gather: int = 0, units: Optional[List[str]] = None,
                       dmdt_range: int = 0) -> None:
    """Write gas particles (r [N, 3], m, h, v [N, 3], rho; temp and u when
    given) and sinks in the layout of write_data_seren_unform.F90 (all
    particles counted as gas; porig defaults to 1..N; pr = 8 or 4 sets the
    real kind; units, when given, are the 21 unit names of a run with units)."""
    if pr not in (4, 8):
        raise ValueError("pr must be 4 or 8")
    real = np.dtype("<f4") if pr == 4 else np.dtype("<f8")
    r = np.asarray(r, np.float64).reshape(-1, 3)
    n = r.shape[0]
    v = np.asarray(v, np.float64).reshape(n, 3)
    cols = {"m": m, "h": h, "rho": rho}
    for k in list(cols):
        cols[k] = np.asarray(cols[k], np.float64).reshape(n)
    porig = np.arange(1, n + 1, dtype=np.int32) if porig is None else \
        np.asarray(porig, np.int32).reshape(n)
    sinks = sinks or []
    stot = len(sinks)
    units = units or []
    blocks = []                                        # (id, typedata row, payload)
    if n > 0:
        blocks += [("porig", (1, 1, n, 2, 0), porig.astype("<i4").tobytes()),
                   ("r", (3, 1, n, 4, 1), r.astype(real).tobytes()),
                   ("m", (1, 1, n, 4, 2), cols["m"].astype(real).tobytes()),
                   ("h", (1, 1, n, 4, 1), cols["h"].astype(real).tobytes()),
                   ("v", (3, 1, n, 4, 4), v.astype(real).tobytes()),
                   ("rho", (1, 1, n, 4, 6), cols["rho"].astype(real).tobytes())]
        if temp is not None:
            blocks.append(("temp", (1, 1, n, 4, 21),
                           np.asarray(temp, np.float64).reshape(n).astype(real).tobytes()))
        if u is not None:
            blocks.append(("u", (1, 1, n, 4, 20),
                           np.asarray(u, np.float64).reshape(n).astype(real).tobytes()))
    if stot > 0:
        blocks.append(("sink_v1", (0, 1, stot, 7, 0), None))
    idata = np.zeros(50, np.int32)
    idata[_IDATA["ptot"]] = n
    idata[_IDATA["stot"]] = stot
    idata[_IDATA["pgas"]] = n
    idata[_IDATA["nunit"]] = len(units)
    idata[_IDATA["ndata"]] = len(blocks)
    idata[_IDATA["dmdt_range"]] = dmdt_range
    idata[_IDATA["pgas_orig"]] = n
    idata[_IDATA["pp_gather"]] = pp_gather
    ilpdata = np.zeros(50, np.int64)
    ilpdata[0], ilpdata[1] = snapshot, nsteps
    rdata = np.zeros(50, real)
    rdata[0], rdata[1], rdata[2] = h_fac, gamma, mu_bar
    dpdata = np.zeros(50, np.float64)
    dpdata[0], dpdata[1] = time, lastsnap
    dpdata[2] = float(np.sum(cols["m"])) if n > 0 else 0.0
    with open(path, "wb") as f:
        _write_record(f, _pad(FORMAT_ID))
        for x in (pr, 3, 3, 3):                         # PR, NDIM, VDIM, BDIM
            _write_record(f, struct.pack("<i", x))
        _write_record(f, idata.astype("<i4").tobytes())
        _write_record(f, ilpdata.astype("<i8").tobytes())
        _write_record(f, rdata.astype(real).tobytes())
        _write_record(f, dpdata.astype("<f8").tobytes())
        if units:
            _write_record(f, b"".join(_pad(x) for x in units))
        if blocks:
            _write_record(f, b"".join(_pad(b[0]) for b in blocks))
            _write_record(f, np.array([b[1] for b in blocks], "<i4").tobytes())
        for name, _, payload in blocks:
            if payload is not None:
                _write_record(f, payload)
        if stot > 0:                                    # write_data_seren_unform.F90:246-276
            length = 11 + 3 + 3 + 2 * dmdt_range
            _write_record(f, struct.pack("<6i", 2, 2, 0, length, 0, 0))
            for s in sinks:
                raux = np.zeros(length)
                raux[0] = s.get("tcreate", 0.0)
                raux[1:4] = s["r"]
                raux[4:7] = s.get("v", (0.0, 0.0, 0.0))
                raux[7] = s["m"]
                raux[8] = s["h"]
                raux[9] = s.get("radius", 0.0)
                raux[10:13] = s.get("angmom", (0.0, 0.0, 0.0))
                raux[13] = s.get("dmdt", 0.0)
                raux[14] = s.get("star_radius", 0.0)
                raux[15] = s.get("luminosity", 0.0)
                raux[16] = s.get("temperature", 0.0)
                if dmdt_range > 0:
                    raux[17:17 + dmdt_range] = s.get("macc", np.zeros(dmdt_range))
                    raux[17 + dmdt_range:17 + 2 * dmdt_range] = s.get("tacc", np.zeros(dmdt_range))
                _write_record(f, struct.pack("<2i", int(s.get("accrete", False)),
                                             int(s.get("static", False))))
                _write_record(f, struct.pack("<2i", int(s.get("id", 0)),
                                             int(s.get("ncreate", 0))))
                _write_record(f, raux.astype(real).tobytes())


# ---------------------------------------------------------------------------
def to_hot_path(snap: Dict):
    """(parray [N, 6] = x, y, z, m, h, 0 in float64, v [N, 3], sinks [S, 5] =
    x, y, z, m, h or None) from a snapshot, for the GPU path's calls."""
    n = snap["ptot"]
    parray = np.zeros((n, 6))
    parray[:, 0:3] = snap["r"].reshape(n, -1)[:, 0:3]
    parray[:, 3] = snap["m"]
    parray[:, 4] = snap["h"]
    v = np.asarray(snap["v"], np.float64).reshape(n, -1)[:, 0:3].copy()
    sinks = None
    if snap.get("sinks"):
        sinks = np.array([[*s["r"][0:3], s["m"], s["h"]] for s in snap["sinks"]])
    return parray, v, sinks
