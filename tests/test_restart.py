"""restart.bin / result files written and read through the C ABI
(scfd_write_restart / scfd_read_restart, out_bin and restart_bin of
store/core/inout.f90), on the CPU restatement: the record layout read back by
formats.read_restart (whose bytes are pinned to the reference's own
sample/no27.chemkin_reaction/restart.bin in test_formats.py), set_bc_q on the
first ghost layer, the read-back state, and the error paths."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200 import formats as F
from shared_cfd_b200.solver import Solver, SolverError


def expected_cells(case, q, w):
    """The field record of out_bin from reference-layout q and w, with
    set_bc_q (inout.f90:144-200) applied to the first ghost layer."""
    nY, D = case.nY, case.D
    iht, iR, ig = D + 2, D + 3, D + 1
    out = []
    for p in range(len(case.planes)):
        ni, nj = case.ni[p], case.nj[p]
        qq = q[p, 1:nj + 3, 1:ni + 3].copy()     # j = 0..nj+1, i = 0..ni+1
        ww = w[p, 1:nj + 3, 1:ni + 3]
        ring = np.zeros((nj + 2, ni + 2), dtype=bool)
        ring[1:nj + 1, 0] = ring[1:nj + 1, ni + 1] = True
        ring[0, :] = ring[nj + 1, :] = True
        rho = ww[..., 0]
        fromw = np.concatenate([rho[..., None] * ww[..., 4:4 + nY], (rho * ww[..., 1])[..., None],
                                (rho * ww[..., 2])[..., None], (rho * ww[..., iht] - ww[..., 3])[..., None]], axis=-1)
        qq[ring] = fromw[ring]
        out.append(np.concatenate([qq, ww[..., iR:iR + 1], ww[..., ig:ig + 1], ww[..., 3:4]], axis=-1))
    return out


@pytest.fixture
def stepped(orc):
    case = cases.perturb(cases.forward_step(2, n=8, scheme=abi.SCHEME_LUSGS, viscous=1), seed=7)
    s = Solver(case, lib=orc)
    s.upload(tt=0.25)
    s.prepare(1)
    s.run(1, 3)
    yield case, s
    s.close()


def test_write_restart_layout_and_set_bc_q(stepped, tmp_path):
    case, s = stepped
    path = tmp_path / "restart.bin"
    s.write_restart(str(path), 1234)
    q, w, _, tt = s.download()
    step, tt_file, cells = F.read_restart(str(path), case.D, list(zip(case.ni, case.nj)))
    assert step == 1234 and tt_file == tt
    for a, b in zip(cells, expected_cells(case, q, w)):
        assert np.array_equal(a, b)


def test_read_restart_restores_the_written_state(stepped, orc, tmp_path):
    case, s = stepped
    path = tmp_path / "restart.bin"
    s.write_restart(str(path), 77)
    written = F.read_restart(str(path), case.D, list(zip(case.ni, case.nj)))[2]
    fresh = Solver(case, lib=orc)
    try:
        step, tt = fresh.read_restart(str(path))
        assert step == 77 and tt == s.download()[3]
        q, w, _, tt2 = fresh.download()
        assert tt2 == tt
        D = case.D
        for p, cells in enumerate(written):
            ni, nj = case.ni[p], case.nj[p]
            assert np.array_equal(q[p, 1:nj + 3, 1:ni + 3], cells[..., :D])
            assert np.array_equal(w[p, 1:nj + 3, 1:ni + 3, D + 3], cells[..., D])
            assert np.array_equal(w[p, 1:nj + 3, 1:ni + 3, D + 1], cells[..., D + 1])
            assert np.array_equal(w[p, 1:nj + 3, 1:ni + 3, 3], cells[..., D + 2])
        # a restarted context steps on from the file's state
        fresh.prepare(1)
        assert fresh.run(1, 1).status == 0
    finally:
        fresh.close()


def test_restart_errors(stepped, orc, tmp_path):
    case, s = stepped
    with pytest.raises(SolverError) as e:
        s.read_restart(str(tmp_path / "missing.bin"))
    assert e.value.code == abi.E_IO
    path = tmp_path / "restart.bin"
    s.write_restart(str(path), 1)
    raw = path.read_bytes()
    (tmp_path / "cut.bin").write_bytes(raw[:-5])
    with pytest.raises(SolverError) as e:
        s.read_restart(str(tmp_path / "cut.bin"))
    assert e.value.code == abi.E_IO
    other = cases.forward_step(2, n=6)
    o = Solver(other, lib=orc)
    try:
        with pytest.raises(SolverError) as e:
            o.read_restart(str(path))
        assert e.value.code == abi.E_IO
    finally:
        o.close()
    with pytest.raises(SolverError) as e:
        s.write_restart(str(tmp_path / "no" / "such" / "dir.bin"), 1)
    assert e.value.code == abi.E_IO
    assert s.lib.read_restart(s.ctx, b"x", None, None) == abi.E_ARG


def test_write_geometry_bin(orc, tmp_path):
    case = cases.reacting_step(scale=0.03)
    s = Solver(case, lib=orc)
    try:
        s.write_geometry(str(tmp_path / "geometry.bin"))
    finally:
        s.close()
    back = F.read_geometry_bin(str(tmp_path / "geometry.bin"))
    assert len(back) == 4
    for (xh, rh), (x2, r2) in zip(case.planes, back):
        assert np.array_equal(xh, x2) and np.array_equal(rh, r2)
    raw = (tmp_path / "geometry.bin").read_bytes()
    assert raw[:12] == (4).to_bytes(4, "big") + case.ni[0].to_bytes(4, "big") + (4).to_bytes(4, "big")
