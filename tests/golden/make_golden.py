"""Generate the committed golden fixtures from a checkout of the reference
(read-only).  Run from the repository root:

    python tests/golden/make_golden.py /path/to/shared_cfd

forward_step_bd.npz / forward_step_expected.json
    Boundary node coordinates of the four forward-step samples
    (sample/no06..no09/forward_step.x) and, as the expected answer, the user
    boundary ranges that the reference's own generator wrote into those
    samples' condition.f90 (lines `do j=max(  lo,nys(plane)),min(nye(plane), hi)`
    under the `!i=1/2`, `!i=ni+1/2`, `!j=1/2`, `!j=nj+1/2` markers).
no27_cells.npz / no27_mech.json
    A seeded sample of cells of sample/no27.chemkin_reaction/restart.bin: q
    and the R, gamma, p the reference computed for them, and the mechanism
    parsed from that sample's chem.inp with the reference's MW.inp/trans.inp.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from shared_cfd_b200 import chem as CH  # noqa: E402
from shared_cfd_b200 import formats as F  # noqa: E402

CASES = ["no06.step_flow", "no07.step_flow2", "no08.step_flow3", "no09.step_flow4"]
MARK = {"!i=1/2": (0, 0), "!i=ni+1/2": (0, 1), "!j=1/2": (1, 0), "!j=nj+1/2": (1, 1)}


def condition_ranges(path):
    """{plane: {(cind, lu): [[lo, hi], ...]}} from a generated condition.f90."""
    out = {}
    plane = None
    side = None
    phase = 0  # 0: before the i loops, 1: i-direction block, 2: j-direction block
    for ln in open(path).read().splitlines():
        s = ln.strip()
        if "!boundary right and left" in s:
            phase = 1
        if "!boundary upper and lower" in s:
            phase = 2
        if "call MPI_COMMUNICATIONS_J_DIRECTION" in s:
            phase = 3
        if phase not in (1, 2):
            continue
        m = re.match(r"case\(\s*(\d+)\)", s)
        if m:
            plane = int(m.group(1))
            continue
        if s in MARK:
            side = MARK[s]
            continue
        m = re.match(r"do [ij]=max\(\s*(\d+),n[xy]s\(plane\)\),min\(n[xy]e\(plane\),\s*(\d+)\)", s)
        if m and plane is not None and side is not None:
            out.setdefault(str(plane), {}).setdefault("%d%d" % side, []).append([int(m.group(1)), int(m.group(2))])
    return out


def main(ref):
    bd = {}
    expected = {}
    for c in CASES:
        d = os.path.join(ref, "sample", c)
        planes = F.read_plot3d(os.path.join(d, "forward_step.x"))
        for p, (xh, rh) in enumerate(planes):
            for nm, arr in (("x", xh), ("r", rh)):
                bd["%s/%d/%s/ilo" % (c, p, nm)] = arr[0, :]
                bd["%s/%d/%s/ihi" % (c, p, nm)] = arr[-1, :]
                bd["%s/%d/%s/jlo" % (c, p, nm)] = arr[:, 0]
                bd["%s/%d/%s/jhi" % (c, p, nm)] = arr[:, -1]
        expected[c] = {"shapes": [list(xh.shape) for xh, _ in planes],
                       "ranges": condition_ranges(os.path.join(d, "condition.f90"))}
    np.savez_compressed(os.path.join(HERE, "forward_step_bd.npz"), **bd)
    with open(os.path.join(HERE, "forward_step_expected.json"), "w") as f:
        json.dump(expected, f, indent=1, sort_keys=True)

    core = os.path.join(ref, "store/therm_lib/chemkin/core")
    s27 = os.path.join(ref, "sample/no27.chemkin_reaction")
    m = CH.parse_chem(open(os.path.join(s27, "chem.inp")).read(), open(os.path.join(core, "MW.inp")).read())
    CH.parse_trans(open(os.path.join(core, "trans.inp")).read(), m)
    comp = CH.parse_control_chem(open(os.path.join(s27, "control_chem.inp")).read(), m)
    fo = CH.fuel_oxidizer(m, comp, len(m.species))
    mech = {"species": m.species, "mws": m.mws, "tthre": m.tthre, "coeff": m.coeff,
            "reactions": m.reactions, "trans": m.trans, "rtol": m.rtol, "atol": m.atol,
            "wo": list(fo["o"]["w"]), "wf": list(fo["f"]["w"])}
    with open(os.path.join(HERE, "no27_mech.json"), "w") as f:
        json.dump(mech, f)
    planes = F.read_plot3d(os.path.join(s27, "ideal_bl.x"))
    ni, nj = planes[0][0].shape[0] - 1, planes[0][0].shape[1] - 1
    D = len(m.species) + 3
    step, tt, cells = F.read_restart(os.path.join(s27, "restart.bin"), D, [(ni, nj)])
    rng = np.random.default_rng(27)
    jj = rng.integers(0, nj + 2, size=600)
    ii = rng.integers(0, ni + 2, size=600)
    vals = cells[0][jj, ii]
    np.savez_compressed(os.path.join(HERE, "no27_cells.npz"), i=ii, j=jj, vals=vals, step=step, tt=tt,
                        ni=ni, nj=nj, dimq=D)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: %s" % "python tests/golden/make_golden.py /path/to/shared_cfd")
    main(sys.argv[1])
