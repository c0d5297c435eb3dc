"""Reference file formats and the block-connectivity generator (CPU)."""
import json
import os

import numpy as np
import pytest

from shared_cfd_b200 import formats as F

from conftest import REFERENCE

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["no06.step_flow", "no07.step_flow2", "no08.step_flow3", "no09.step_flow4"]
# geo width order p1 c1 s1 pm1 p2 c2 s2 pm2, derived by hand from the sample
# layouts (manual.tex:2423-2442: the same two-block step in four orientations)
EXPECTED_RECORDS = {
    "no06.step_flow": [[1, 80, 1, 1, 60, 21, 1, 2, 1, 1, -1]],
    "no07.step_flow2": [[4, 60, 1, 1, 1, 1, -1, 2, 20, 1, 1]],
    "no08.step_flow3": [[3, 60, 1, 1, 20, 1, 1, 2, 80, 1, 1]],
    "no09.step_flow4": [[2, 60, -1, 1, 20, 1, 1, 2, 1, 60, -1]],
}


def _planes_from_boundaries(case):
    bd = np.load(os.path.join(GOLD, "forward_step_bd.npz"))
    shapes = json.load(open(os.path.join(GOLD, "forward_step_expected.json")))[case]["shapes"]
    planes = []
    for p, (a, b) in enumerate(shapes):
        arrs = []
        for nm in ("x", "r"):
            z = np.full((a, b), np.nan)
            z[0, :] = bd["%s/%d/%s/ilo" % (case, p, nm)]
            z[-1, :] = bd["%s/%d/%s/ihi" % (case, p, nm)]
            z[:, 0] = bd["%s/%d/%s/jlo" % (case, p, nm)]
            z[:, -1] = bd["%s/%d/%s/jhi" % (case, p, nm)]
            arrs.append(z)
        planes.append(tuple(arrs))
    return planes


@pytest.mark.parametrize("case", CASES)
def test_connectivity_matches_reference_generated_boundaries(case):
    """The user-boundary ranges left after removing the detected interfaces
    equal the ranges the reference generator wrote into the sample's
    condition.f90, and the interface record equals the hand-derived one."""
    planes = _planes_from_boundaries(case)
    recs, tsm = F.connectivity(planes)
    assert recs == EXPECTED_RECORDS[case]
    exp = json.load(open(os.path.join(GOLD, "forward_step_expected.json")))[case]["ranges"]
    for p in range(len(planes)):
        for cind in range(2):
            for lu in range(2):
                got = tsm[p][cind][lu]
                want = exp.get(str(p + 1), {}).get("%d%d" % (cind, lu), [])
                assert got == want, (case, p, cind, lu)


def test_cut_copro_text_round_trip():
    recs = [[1, 80, 1, 1, 60, 21, 1, 2, 1, 1, -1], [2, 60, -1, 1, 20, 1, 1, 2, 1, 60, -1]]
    txt = F.format_cut_copro(recs)
    lines = txt.splitlines()
    assert lines[0] == "# myid = 000" and lines[1] == "2"
    # (11i6) fields: every record line is 11 six-character fields wide (last one 5)
    assert all(len(ln) == 65 for ln in lines[3:])
    p = os.path.join(GOLD, "..", "_tmp_cut.inp")
    with open(p, "w") as f:
        f.write(txt)
    try:
        assert F.read_cut_copro(p) == recs
    finally:
        os.unlink(p)


def test_restart_round_trip_synthetic(tmp_path):
    rng = np.random.default_rng(0)
    planes_ij = [(5, 3), (4, 6)]
    cells = [rng.standard_normal((nj + 2, ni + 2, 7)) for ni, nj in planes_ij]
    path = tmp_path / "restart.bin"
    F.write_restart(str(path), 1234, 5.5e-3, cells)
    step, tt, back = F.read_restart(str(path), 4, planes_ij)
    assert step == 1234 and tt == 5.5e-3
    for a, b in zip(cells, back):
        assert np.array_equal(a, b)
    raw = path.read_bytes()
    assert raw[:4] == (4).to_bytes(4, "big")   # record marker of the step record


def test_restart_truncated_is_rejected(tmp_path):
    cells = [np.zeros((4, 5, 7))]
    path = tmp_path / "restart.bin"
    F.write_restart(str(path), 1, 0.0, cells)
    raw = path.read_bytes()
    (tmp_path / "cut.bin").write_bytes(raw[:-6])
    with pytest.raises(ValueError):
        F.read_restart(str(tmp_path / "cut.bin"), 4, [(3, 2)])


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE),
                    reason="SCFD_REFERENCE does not name a reference checkout")
def test_no27_restart_bin_bytes_round_trip():
    p = os.path.join(REFERENCE, "sample/no27.chemkin_reaction/restart.bin")
    step, tt, cells = F.read_restart(p, 11, [(223, 99)])
    assert step == 40000 and tt == 0.0
    assert F.restart_bytes(step, tt, cells) == open(p, "rb").read()


def test_plot3d_round_trip():
    xs = np.linspace(0.0, 1.0, 7)
    rs = np.linspace(0.1, 0.5, 4)
    xh = np.repeat(xs[:, None], 4, axis=1)
    rh = np.repeat(rs[None, :], 7, axis=0)
    txt = F.format_plot3d([(xh, rh)])
    p = os.path.join(GOLD, "..", "_tmp.x")
    with open(p, "w") as f:
        f.write(txt)
    try:
        back = F.read_plot3d(p)
    finally:
        os.unlink(p)
    assert np.array_equal(back[0][0], xh) and np.array_equal(back[0][1], rh)


def test_control_inp(tmp_path):
    txt = ("#FOR GENERAL PARAMETERS\n"
           "Max Step Number         : 1.e7\n"
           "convergent RMS          : 1.e-14\n"
           "CFL Number              : .5\n"
           "File Output Period      : 500\n\n"
           "MUSCL ON(1)/OFF(0)      : 1\n"
           "MUSCL Precision Order   : 3\n"
           "InternalLoop Max Number : 21\n")
    p = tmp_path / "control.inp"
    p.write_text(txt)
    c = F.read_control(str(p))
    assert c["cfl"] == 0.5 and c["out_period"] == 500 and c["max_step"] == 1e7
    assert F.control_value(c, "MUSCL Precision Order   :", cast=int) == 3
    assert F.control_value(c, "InternalLoop Max Number :", cast=int) == 21
