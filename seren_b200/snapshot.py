"""SEREN binary snapshots (format id SERENBINARYDUMPV2) read and written in
the layout of io/write_data_seren_unform.F90 and io/read_data_seren_unform.F90,
and DRAGON snapshots (binary and ASCII, io/read_data_dragon_unform.F90,
io/read_data_dragon_form.F90 and their writers), so that snapshots of the
Fortran code can feed the GPU path and its results can be read back by the
Fortran tools.

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


# ---------------------------------------------------------------------------
# DRAGON snapshots
#
# Layout (write_data_dragon_unform.F90:44-271, write_data_dragon_form.F90:34-171):
#   idata(20) int | rdata(50) real | positions (NDIM per particle) |
#   velocities (VDIM per particle) | temperatures | h | rho | m | types (int) |
#   particle ids (int, PARTICLE_ID builds only)
# with ptot + stot entries in every per-particle block, the sinks last.  In the
# binary file each block is one Fortran record (reals of kind PR); in the ASCII
# file every value or particle vector is one list-directed record (line).
# idata(1) = entries, idata(2) = nsteps, idata(3) = gas entries, idata(4) =
# snapshot, idata(20) = pgas_orig; rdata(1) = time, rdata(2) = lastsnap,
# rdata(50) = mgas_orig.  Types: 1 gas, 6 boundary, 9 intercloud, 10 dark
# matter (ASCII reader only), -1 sink, 0 accreted (dropped), 4 split (refused).

DRAGON_GAS, DRAGON_BOUNDARY, DRAGON_ICM, DRAGON_CDM = 1, 6, 9, 10
DRAGON_SINK, DRAGON_DEAD, DRAGON_SPLIT = -1, 0, 4
_KERNRANGE = 2.0                 # sink radius = KERNRANGE * h for DRAGON sinks
_DRAGON_TRESTR = 1000.0          # write_data_dragon_unform.F90:31-32 (cgs)
_DRAGON_RHORESTR = 1.0e-13


def _dragon_assemble(idata, rdata, pos, vel, temp, h, rho, m, ptype, ids, with_cdm: bool,
                     rounding=None) -> Dict:
    """Sort DRAGON entries into SEREN's particle order: boundary, intercloud,
    gas (and dark matter for the ASCII reader), each in file order; sinks
    apart; accreted entries dropped (read_data_dragon_unform.F90:91-116 and
    135-343, read_data_dragon_form.F90:81-113 and 143-371).  Without ids, a
    particle's porig is its 1-based position in the file, as the reference
    sets it when no restart log exists."""
    ntot = int(idata[0])
    ptype = np.asarray(ptype).astype(np.int64)
    counts = {t: int(np.count_nonzero(ptype == t)) for t in
              (DRAGON_SINK, DRAGON_DEAD, DRAGON_GAS, DRAGON_SPLIT, DRAGON_BOUNDARY, DRAGON_ICM,
               DRAGON_CDM)}
    stot, pdead = counts[DRAGON_SINK], counts[DRAGON_DEAD]
    ptot = ntot - (stot + pdead)
    if counts[DRAGON_SPLIT] != 0:
        raise ValueError("particle splitting not supported (DRAGON type 4)")
    kinds = [DRAGON_BOUNDARY, DRAGON_ICM, DRAGON_GAS] + ([DRAGON_CDM] if with_cdm else [])
    if ptot != sum(counts[t] for t in kinds):
        raise ValueError("particles do not add up (types other than "
                         + ", ".join(str(t) for t in kinds) + ", -1 and 0 present)")
    order = np.concatenate([np.flatnonzero(ptype == t) for t in kinds]) if ptot else \
        np.zeros(0, np.int64)
    sk = np.flatnonzero(ptype == DRAGON_SINK)
    rnd = (lambda a: a) if rounding is None else rounding
    out: Dict = dict(format_id="DRAGON", idata=np.asarray(idata), rdata=np.asarray(rdata),
                     ptot=ptot, stot=stot, pdead=pdead, pboundary=counts[DRAGON_BOUNDARY],
                     picm=counts[DRAGON_ICM], pgas=counts[DRAGON_GAS],
                     pcdm=counts[DRAGON_CDM] if with_cdm else 0,
                     nsteps=int(idata[1]), snapshot=int(idata[3]), pgas_orig=int(idata[19]),
                     time=float(rnd(rdata[0])), lastsnap=float(rnd(rdata[1])),
                     mgas_orig=float(rnd(rdata[49])))
    out["r"] = pos[order].astype(np.float64)
    out["v"] = vel[order].astype(np.float64)
    out["temp"] = temp[order].astype(np.float64)
    out["h"] = h[order].astype(np.float64)
    out["rho"] = rho[order].astype(np.float64)
    out["m"] = m[order].astype(np.float64)
    out["ptype"] = ptype[order].astype(np.int32)
    out["porig"] = (np.asarray(ids)[order].astype(np.int32) if ids is not None
                    else (order + 1).astype(np.int32))
    # sink fields the DRAGON format does not hold take the reader's defaults
    # (read_data_dragon_unform.F90:341-349)
    out["sinks"] = [dict(r=pos[s].astype(np.float64), v=vel[s].astype(np.float64),
                         m=float(m[s]), h=float(h[s]), radius=_KERNRANGE * float(h[s]),
                         accrete=True, static=False) for s in sk]
    return out


def read_dragon_unform(path: str, ids: bool = False, ndim: int = 3) -> Dict:
    """A binary DRAGON snapshot (read_data_dragon_unform.F90:9-364) as a dict
    with the keys of read_seren_unform's particle blocks (r, v, temp, h, rho,
    m, porig, ptype), the counts and the sinks.  The real kind (4 or 8 bytes)
    is taken from the length of the rdata record.  ids=True reads porig from
    the id record (a PARTICLE_ID build restarting a run); otherwise porig is
    the file position.  Dark-matter entries (type 10) are refused, as this
    reader of the reference counts no dark matter."""
    with open(path, "rb") as f:
        rec = _read_record(f)
        if len(rec) != 80:
            raise ValueError(f"not a DRAGON snapshot (idata record of {len(rec)} bytes)")
        idata = np.frombuffer(rec, "<i4").copy()
        rec = _read_record(f)
        if len(rec) not in (200, 400):
            raise ValueError(f"not a DRAGON snapshot (rdata record of {len(rec)} bytes)")
        real = np.dtype("<f4") if len(rec) == 200 else np.dtype("<f8")
        rdata = np.frombuffer(rec, real).copy()
        n = int(idata[0])
        if n < 0:
            raise ValueError("negative particle count in a DRAGON header")

        def block(dt, comp):
            a = np.frombuffer(_read_record(f), dt)
            if a.size != n * comp:
                raise ValueError(f"DRAGON block holds {a.size} values, expected {n * comp}")
            return a.reshape(n, comp) if comp > 1 else a.copy()

        pos = block(real, ndim)
        vel = block(real, ndim)
        temp, h, rho, m = (block(real, 1) for _ in range(4))
        ptype = block("<i4", 1)
        idv = block("<i4", 1) if ids else None
    return _dragon_assemble(idata, rdata, pos, vel, temp, h, rho, m, ptype, idv,
                            with_cdm=False)


class _ListDirected:
    """Fortran list-directed input over a text file: every read statement
    starts on a new record (line), takes values from as many lines as it
    needs and drops the rest of its last line; values are separated by
    blanks or commas; r*c repeats c r times; D exponents are accepted."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.i = 0

    def read(self, n: int) -> List[str]:
        vals: List[str] = []
        while len(vals) < n:
            if self.i >= len(self.lines):
                raise EOFError("end of file in a list-directed read")
            line = self.lines[self.i]
            self.i += 1
            for tok in line.replace(",", " ").split():
                if "*" in tok:
                    k, _, v = tok.partition("*")
                    vals.extend([v] * int(k))
                else:
                    vals.append(tok)
        return vals[:n]

    def reals(self, n: int) -> List[float]:
        return [float(t.replace("D", "E").replace("d", "e")) for t in self.read(n)]


def read_dragon_form(path: str, ids: bool = False, ndim: int = 3) -> Dict:
    """An ASCII DRAGON snapshot (read_data_dragon_form.F90:9-396) as a dict
    like read_dragon_unform's.  The reference reads every real value of this
    format into a single-precision variable, so positions, velocities, h, rho,
    m, temperatures and the header times come back rounded to float32 and
    widened again, as in the reference; types are read as reals and
    truncated.  Dark matter (type 10) is accepted and placed after the gas."""
    with open(path, "r") as f:
        rd = _ListDirected(f.read())
    idata = np.array([int(rd.read(1)[0]) for _ in range(20)], np.int64)
    rdata = np.array([rd.reals(1)[0] for _ in range(50)], np.float64).astype(np.float32)
    n = int(idata[0])
    if n < 0:
        raise ValueError("negative particle count in a DRAGON header")
    sp = np.float32
    pos = np.array([rd.reals(ndim) for _ in range(n)], np.float64).reshape(n, ndim).astype(sp)
    vel = np.array([rd.reals(ndim) for _ in range(n)], np.float64).reshape(n, ndim).astype(sp)
    temp, h, rho, m = (np.array([rd.reals(1)[0] for _ in range(n)], np.float64).astype(sp)
                       for _ in range(4))
    ptype = np.trunc(np.array([rd.reals(1)[0] for _ in range(n)], np.float64).astype(sp))
    idv = None
    if ids:
        idv = np.array([int(rd.read(1)[0]) for _ in range(n)], np.int64)
    return _dragon_assemble(idata, rdata.astype(np.float64), pos, vel, temp, h, rho, m,
                            ptype.astype(np.int64), idv, with_cdm=True)


def _dragon_columns(r, m, h, v, rho, temp, ptype, porig, sinks, scales):
    r = np.asarray(r, np.float64).reshape(-1, 3)
    n = r.shape[0]
    v = np.asarray(v, np.float64).reshape(n, 3)
    m, h, rho = (np.asarray(x, np.float64).reshape(n) for x in (m, h, rho))
    temp = np.zeros(n) if temp is None else np.asarray(temp, np.float64).reshape(n)
    ptype = np.full(n, DRAGON_GAS, np.int32) if ptype is None else \
        np.asarray(ptype, np.int32).reshape(n)
    porig = np.arange(1, n + 1, dtype=np.int32) if porig is None else \
        np.asarray(porig, np.int32).reshape(n)
    sinks = sinks or []
    rs, vs, ms, rhos = scales["rscale"], scales["vscale"], scales["mscale"], scales["rhoscale"]
    cols = dict(r=r * rs, v=v * vs, temp=temp, h=h * rs, rho=rho * rhos, m=m * ms, ptype=ptype,
                porig=porig)
    if sinks:
        cols["r"] = np.vstack([cols["r"], [np.asarray(s["r"], np.float64) * rs for s in sinks]])
        cols["v"] = np.vstack([cols["v"], [np.asarray(s.get("v", (0.0, 0.0, 0.0)), np.float64)
                                           * vs for s in sinks]])
        cols["temp"] = np.concatenate([cols["temp"], np.zeros(len(sinks))])
        cols["h"] = np.concatenate([cols["h"], [s["h"] * rs for s in sinks]])
        cols["rho"] = np.concatenate([cols["rho"], np.full(len(sinks),
                                                           scales["rhosink"] * rhos)])
        cols["m"] = np.concatenate([cols["m"], [s["m"] * ms for s in sinks]])
        cols["ptype"] = np.concatenate([cols["ptype"], np.full(len(sinks), DRAGON_SINK,
                                                               np.int32)])
        cols["porig"] = np.concatenate([cols["porig"], np.zeros(len(sinks), np.int32)])
    return n, len(sinks), cols


def _dragon_header(entries, gas_entries, nsteps, snapshot, pgas_orig, time, lastsnap,
                   mgas_orig, tscale, mscale):
    idata = np.zeros(20, np.int64)
    idata[0], idata[1], idata[2], idata[3], idata[19] = (entries, nsteps, gas_entries, snapshot,
                                                         pgas_orig)
    rdata = np.zeros(50, np.float64)
    rdata[0], rdata[1], rdata[49] = time * tscale, lastsnap * tscale, mgas_orig * mscale
    return idata, rdata


def write_dragon_unform(path: str, r, m, h, v, rho, temp=None, ptype=None, porig=None,
                        sinks: Optional[List[Dict]] = None, pr: int = 4, ids: bool = False,
                        time: float = 0.0, lastsnap: float = 0.0, snapshot: int = 0,
                        nsteps: int = 0, pgas_orig: Optional[int] = None,
                        mgas_orig: Optional[float] = None, rhosink: float = 0.0,
                        rscale: float = 1.0, vscale: float = 1.0, mscale: float = 1.0,
                        rhoscale: float = 1.0, tscale: float = 1.0) -> int:
    """Write a binary DRAGON snapshot as write_data_dragon_unform.F90 does,
    including its density-temperature cut: only particles with
    rho * rhoscale > 1e-13 or temp < 1000 are written (:57-67), then the sinks
    (type -1, temperature 0, density rhosink).  Particles must come in SEREN's
    order (boundary, intercloud, gas); their types are written for the kept
    particles in that order (the reference offsets the intercloud and gas types
    by the uncut boundary and intercloud counts, which is the same whenever
    the cut keeps every boundary and intercloud particle).  ids=True adds the
    id record of a PARTICLE_ID build.  Returns the number of particles kept."""
    if pr not in (4, 8):
        raise ValueError("pr must be 4 or 8")
    real = np.dtype("<f4") if pr == 4 else np.dtype("<f8")
    sc = dict(rscale=rscale, vscale=vscale, mscale=mscale, rhoscale=rhoscale, rhosink=rhosink)
    n, stot, c = _dragon_columns(r, m, h, v, rho, temp, ptype, porig, sinks, sc)
    keep = np.concatenate([(c["rho"][:n] > _DRAGON_RHORESTR) | (c["temp"][:n] < _DRAGON_TRESTR),
                           np.ones(stot, bool)])
    kept = int(np.count_nonzero(keep[:n]))
    mg = float(np.sum(np.asarray(m, np.float64))) if mgas_orig is None else mgas_orig
    idata, rdata = _dragon_header(kept + stot, kept, nsteps, snapshot,
                                  n if pgas_orig is None else pgas_orig, time, lastsnap, mg,
                                  tscale, mscale)
    with open(path, "wb") as f:
        _write_record(f, idata.astype("<i4").tobytes())
        _write_record(f, rdata.astype(real).tobytes())
        for k in ("r", "v", "temp", "h", "rho", "m"):
            _write_record(f, c[k][keep].astype(real).tobytes())
        _write_record(f, c["ptype"][keep].astype("<i4").tobytes())
        if ids:
            _write_record(f, c["porig"][keep].astype("<i4").tobytes())
    return kept


def _fort_real(x: float, pr: int) -> str:
    return f"{x: .9E}" if pr == 4 else f"{x: .17E}"


def write_dragon_form(path: str, r, m, h, v, rho, temp=None, ptype=None, porig=None,
                      sinks: Optional[List[Dict]] = None, pr: int = 8, ids: bool = False,
                      time: float = 0.0, lastsnap: float = 0.0, snapshot: int = 0,
                      nsteps: int = 0, pgas_orig: Optional[int] = None,
                      mgas_orig: Optional[float] = None, rhosink: float = 0.0,
                      rscale: float = 1.0, vscale: float = 1.0, mscale: float = 1.0,
                      rhoscale: float = 1.0, tscale: float = 1.0) -> None:
    """Write an ASCII DRAGON snapshot as write_data_dragon_form.F90 does
    (every particle, no density-temperature cut; one value or one particle
    vector per line; sinks last).  Reals are printed with enough digits to
    read back exactly at real kind pr."""
    if pr not in (4, 8):
        raise ValueError("pr must be 4 or 8")
    sc = dict(rscale=rscale, vscale=vscale, mscale=mscale, rhoscale=rhoscale, rhosink=rhosink)
    n, stot, c = _dragon_columns(r, m, h, v, rho, temp, ptype, porig, sinks, sc)
    mg = float(np.sum(np.asarray(m, np.float64))) if mgas_orig is None else mgas_orig
    idata, rdata = _dragon_header(n + stot, n, nsteps, snapshot, n if pgas_orig is None
                                  else pgas_orig, time, lastsnap, mg, tscale, mscale)
    cast = (lambda a: np.asarray(a, np.float64).astype(np.float32)) if pr == 4 else \
        (lambda a: np.asarray(a, np.float64))
    out: List[str] = [f"{int(x):12d}" for x in idata]
    out += [_fort_real(float(x), pr) for x in cast(rdata)]
    for k in ("r", "v"):
        out += [" ".join(_fort_real(float(x), pr) for x in row) for row in cast(c[k])]
    for k in ("temp", "h", "rho", "m"):
        out += [_fort_real(float(x), pr) for x in cast(c[k])]
    out += [f"{int(x):12d}" for x in c["ptype"]]
    if ids:
        out += [f"{int(x):12d}" for x in c["porig"]]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
