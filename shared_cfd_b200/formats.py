"""Reference file formats and the block-connectivity generator.

* plot3d ASCII grids (store/dim/2d/geometry.f90:27-78 reads them),
* control.inp (store/core/read_control.f90:1-32 and the keyed lines of
  store/high_order/muscl/muscl.f90:76-116, NR/q2d/sch_NR.raw.f90:239-275),
* big-endian Fortran sequential-unformatted restart.bin / result files
  (store/core/inout.f90:1-142, written with ifort -convert big_endian),
* cut_copro000.inp generation (store/cond/core/*.py), which finds block
  interfaces by exact equality of boundary node coordinates.
"""
import struct

import numpy as np


# ----------------------------------------------------------------------------
# plot3d
# ----------------------------------------------------------------------------
def read_plot3d(path):
    """Return [(xh, rh)] per plane; xh, rh have shape (ni+1, nj+1) (node index
    order of the reference, xh[i, j] = xh(i,j)).  Values are parsed exactly as
    the text gives them."""
    with open(path) as f:
        toks = f.read().split()
    pos = 0
    nplane = int(float(toks[pos])); pos += 1
    dims = []
    for _ in range(nplane):
        a, b, c = (int(float(t)) for t in toks[pos:pos + 3]); pos += 3
        if c != 1:
            raise ValueError("3-D grids are not supported (checkout_flow.py:56-60)")
        dims.append((a, b))
    planes = []
    for (a, b) in dims:
        ng = a * b
        xs = np.array([float(t) for t in toks[pos:pos + ng]]); pos += ng
        rs = np.array([float(t) for t in toks[pos:pos + ng]]); pos += ng
        pos += ng  # z, discarded (geometry.f90:66-70)
        planes.append((xs.reshape(b, a).T.copy(), rs.reshape(b, a).T.copy()))
    return planes


def format_plot3d(planes):
    """Text of a plot3d grid: 4 values per line like the sample grids, with 17
    significant digits so that the text reads back bit-identically."""
    out = ["%8d" % len(planes)]
    for xh, _ in planes:
        out.append("%8d %8d %8d" % (xh.shape[0], xh.shape[1], 1))
    for xh, rh in planes:
        for arr in (xh, rh, np.zeros_like(xh)):
            flat = arr.T.reshape(-1)
            for k in range(0, flat.size, 4):
                out.append(" ".join("%24.16e" % v for v in flat[k:k + 4]))
    return "\n".join(out) + "\n"


def roundtrip_plot3d_values(planes):
    """The node coordinates a reader of format_plot3d(planes) gets back."""
    return [(np.array([float("%24.16e" % v) for v in xh.reshape(-1)]).reshape(xh.shape),
             np.array([float("%24.16e" % v) for v in rh.reshape(-1)]).reshape(rh.shape))
            for xh, rh in planes]


# ----------------------------------------------------------------------------
# control.inp
# ----------------------------------------------------------------------------
def read_control(path):
    """Parse control.inp: the four fixed-column lines after the comment line
    (read_control.f90:9-13, format (25x,es15.7) / (25x,i10)) and every
    'key (25 chars) : value' line."""
    with open(path) as f:
        lines = f.read().splitlines()
    out = {}
    fixed = ["max_step", "min_rms", "cfl", "out_period"]
    for k, name in enumerate(fixed):
        s = lines[1 + k][25:]
        out[name] = int(s.split()[0]) if name == "out_period" else float(s[:15].split()[0])
    keyed = {}
    for ln in lines:
        if len(ln) > 25 and ln[24] == ":":
            keyed[ln[:25]] = ln[25:].split("#")[0].strip()
    out["keyed"] = keyed
    return out


def control_value(ctrl, key, default=None, cast=float):
    """A keyed control.inp value; key is the 25-character prefix."""
    v = ctrl["keyed"].get(key)
    if v is None:
        return default
    if cast is bool:
        return v.strip().lower().strip(".") in ("true", "t")
    return cast(float(v)) if cast is int else cast(v)


# ----------------------------------------------------------------------------
# Fortran sequential unformatted, big endian
# ----------------------------------------------------------------------------
def _read_records(buf):
    recs = []
    pos = 0
    while pos < len(buf):
        if pos + 4 > len(buf):
            raise ValueError("truncated record marker")
        (n,) = struct.unpack(">i", buf[pos:pos + 4])
        if n < 0 or pos + 8 + n > len(buf):
            raise ValueError("truncated or corrupt record")
        payload = buf[pos + 4:pos + 4 + n]
        (n2,) = struct.unpack(">i", buf[pos + 4 + n:pos + 8 + n])
        if n2 != n:
            raise ValueError("record markers disagree")
        recs.append(payload)
        pos += 8 + n
    return recs


def _record(payload):
    n = len(payload)
    return struct.pack(">i", n) + payload + struct.pack(">i", n)


def read_restart(path, dimq, planes_ij):
    """restart.bin / result*.bin (inout.f90:77-100).  Returns (step, tt, cells)
    where cells[p] has shape (nj+2, ni+2, dimq+3): q(1:dimq), R, gamma, p for
    i = 0..ni+1 (fast), j = 0..nj+1."""
    with open(path, "rb") as f:
        buf = f.read()
    recs = _read_records(buf)
    if len(recs) != 3:
        raise ValueError("restart file must hold 3 records, found %d" % len(recs))
    if len(recs[0]) != 4 or len(recs[1]) != 8:
        raise ValueError("bad step / time record")
    (step,) = struct.unpack(">i", recs[0])
    (tt,) = struct.unpack(">d", recs[1])
    need = sum((ni + 2) * (nj + 2) for ni, nj in planes_ij) * (dimq + 3) * 8
    if len(recs[2]) != need:
        raise ValueError("field record has %d bytes, expected %d" % (len(recs[2]), need))
    arr = np.frombuffer(recs[2], dtype=">f8").astype(np.float64)
    cells = []
    pos = 0
    for ni, nj in planes_ij:
        n = (ni + 2) * (nj + 2) * (dimq + 3)
        cells.append(arr[pos:pos + n].reshape(nj + 2, ni + 2, dimq + 3).copy())
        pos += n
    return step, tt, cells


def restart_bytes(step, tt, cells):
    """Bytes of restart.bin / result*.bin for the given cells (inverse of
    read_restart; out_bin, inout.f90:44-56)."""
    field = b"".join(np.ascontiguousarray(c, dtype=">f8").tobytes() for c in cells)
    return _record(struct.pack(">i", step)) + _record(struct.pack(">d", tt)) + _record(field)


def read_geometry_bin(path):
    """geometry.bin of out_geo_bin (store/dim/2d/geometry.f90:182-193): a list
    of (xh, rh) node arrays of shape (ni+1, nj+1)."""
    with open(path, "rb") as f:
        recs = _read_records(f.read())
    if len(recs) % 3:
        raise ValueError("geometry.bin holds %d records, not three per plane" % len(recs))
    planes = []
    for k in range(0, len(recs), 3):
        (ni,) = struct.unpack(">i", recs[k])
        (nj,) = struct.unpack(">i", recs[k + 1])
        arr = np.frombuffer(recs[k + 2], dtype=">f8").astype(np.float64)
        if arr.size != 2 * (ni + 1) * (nj + 1):
            raise ValueError("plane %d: node record size" % (k // 3 + 1))
        xr = arr.reshape(nj + 1, ni + 1, 2)
        planes.append((xr[..., 0].T.copy(), xr[..., 1].T.copy()))
    return planes


def write_restart(path, step, tt, cells):
    with open(path, "wb") as f:
        f.write(restart_bytes(step, tt, cells))


# ----------------------------------------------------------------------------
# block connectivity: store/cond/core/{read_plot3d,set_cond_var,mod_cond,fetchMPI,out_cond}.py
# ----------------------------------------------------------------------------
class _BD:
    __slots__ = ("grid", "plane", "cind", "lu", "index")

    def __init__(self, grid, plane, cind, lu, index):
        self.grid, self.plane, self.cind, self.lu, self.index = grid, plane, cind, lu, index

    def same_line(self, o):  # mod_cond.py:206-209
        return self.plane == o.plane and self.cind == o.cind and self.lu == o.lu


def _boundary_nodes(planes):
    """Boundary node list in the generator's order (read_plot3d.py:77-90)."""
    bd = []
    for p, (xh, rh) in enumerate(planes):
        a, b = xh.shape
        for j in range(b):
            bd.append(_BD((xh[0, j], rh[0, j]), p, 0, 0, j))
        for j in range(b):
            bd.append(_BD((xh[a - 1, j], rh[a - 1, j]), p, 0, 1, j))
        for i in range(a):
            bd.append(_BD((xh[i, 0], rh[i, 0]), p, 1, 0, i))
        for i in range(a):
            bd.append(_BD((xh[i, b - 1], rh[i, b - 1]), p, 1, 1, i))
    return bd


def _touches(bd):
    """set_touch (set_cond_var.py:5-42), including its Python quirks: the j
    loop continues after a match with the updated BDI, and j+width*pm may go
    negative, which indexes from the end of the list."""
    touch = []
    i = 0
    n = len(bd)
    while i < n - 1:
        BDi = bd[i]
        BDI = bd[i + 1]
        if not BDi.same_line(BDI):
            i += 1
            continue
        for j in range(i + 1, n):
            BDj = bd[j]
            if BDi.grid == BDj.grid:
                pm = 0
                if j + 1 < n and BDj.same_line(bd[j + 1]) and BDI.grid == bd[j + 1].grid:
                    pm = +1
                elif BDj.same_line(bd[j - 1]) and BDI.grid == bd[j - 1].grid:
                    pm = -1
                if pm != 0:
                    t = {
                        "geo": BDi.cind * 2 + BDj.cind + 1, "order": pm,
                        "p1": BDi.plane, "p2": BDj.plane, "cind1": BDi.cind, "cind2": BDj.cind,
                        "lu1": BDi.lu, "lu2": BDj.lu, "s1": BDi.index + 1,
                        "s2": BDj.index + 1 if pm > 0 else BDj.index,
                        "pm1": -1 + 2 * BDi.lu, "pm2": -1 + 2 * BDj.lu,
                    }
                    width = 1
                    while True:
                        if j + width * pm >= n or i + width >= n:
                            break
                        BDI = bd[i + width]
                        BDJ = bd[j + width * pm]
                        if BDi.same_line(BDI) and BDj.same_line(BDJ) and BDI.grid == BDJ.grid:
                            width += 1
                        else:
                            break
                    t["width"] = width - 1
                    i += width - 2
                    touch.append(t)
        i += 1
    return touch


def connectivity(planes):
    """Block-interface records of cut_copro000.inp for a single-process run
    (fetchMPI.py:177-197 gives every boundary to rank 0, so modify_touch keeps
    the touches unsplit).  Returns (records, to_set_manually) where records is
    a list of 11-int lists and to_set_manually[p][cind][lu] the ranges the user
    boundary conditions must cover (set_cond_var.py:44-91)."""
    nijk = [xh.shape for xh, _ in planes]
    touch = _touches(_boundary_nodes(planes))
    recs = []
    for t in touch:
        c1 = 1 if t["pm1"] < 0 else nijk[t["p1"]][t["cind1"]] - 1  # fetchc12, mod_cond.py:247-257
        c2 = 1 if t["pm2"] < 0 else nijk[t["p2"]][t["cind2"]] - 1
        recs.append([t["geo"], t["width"], t["order"], t["p1"] + 1, c1, t["s1"], t["pm1"],
                     t["p2"] + 1, c2, t["s2"], t["pm2"]])
    tsm = []
    for p in range(len(planes)):
        tsm.append([])
        for cind in range(2):
            n = nijk[p][1] - 1 if cind == 0 else nijk[p][0] - 1
            tsm[p].append([[[1, n]], [[1, n]]])
    for t in touch:
        for side in range(2):
            if side == 0:
                rem = [t["s1"], t["s1"] + t["width"] - 1]
                p, cind, lu = t["p1"], t["cind1"], t["lu1"]
            else:
                rem = sorted([t["s2"], t["s2"] + t["order"] * (t["width"] - 1)])
                p, cind, lu = t["p2"], t["cind2"], t["lu2"]
            work = tsm[p][cind][lu]
            for k, elm in enumerate(work):
                if elm[0] <= rem[0] and rem[1] <= elm[1]:
                    rep = []
                    if elm[0] < rem[0]:
                        rep.append([elm[0], rem[0] - 1])
                    if elm[1] > rem[1]:
                        rep.append([rem[1] + 1, elm[1]])
                    work[k:k + 1] = rep
                    rem = None
                    break
            if rem is not None:
                raise ValueError("Unexpected Situation Occured! (set_cond_var.py:178-181)")
    return recs, tsm


def format_cut_copro(recs, myid=0):
    """Text of cut_copro%03i.inp (out_cond.py:143-155)."""
    s = "# myid = %03i\n" % myid
    s += "%i\n" % len(recs)
    s += "# geo width order    p1    c1    s1   pm1    p2    c2    s2   pm2\n"
    for r in recs:
        s += " ".join(["%5i"] * 11) % tuple(r) + "\n"
    return s


def read_cut_copro(path):
    """set_cut_copro (PC/mod_mpi_dummy.f90:59-79): comment, count, comment, records."""
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[1].split()[0])
    recs = []
    for ln in lines[3:3 + n]:
        # format (11i6): six-character fields
        recs.append([int(ln[6 * k:6 * k + 6].strip() or "0") for k in range(11)])
    return recs
