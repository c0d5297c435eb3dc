"""scfd_write_restart / scfd_read_restart of the CUDA library: the bytes of
the CPU restatement for the same state, the out_bin layout after GPU steps,
and the read-back state."""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200 import formats as F
from shared_cfd_b200.solver import Solver

from test_restart import expected_cells

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: cases.perturb(cases.forward_step(3, n=16), seed=2),
                                  lambda: cases.reacting_step(scale=0.0625, inner=2)])
def test_restart_bytes_equal_restatement(gpu, orc, tmp_path, make):
    case = make()
    paths = []
    for lib, tag in ((gpu, "gpu"), (orc, "orc")):
        s = Solver(case, lib=lib)
        try:
            s.upload(tt=1.5e-4)
            paths.append(tmp_path / ("%s.bin" % tag))
            s.write_restart(str(paths[-1]), 42)
        finally:
            s.close()
    assert paths[0].read_bytes() == paths[1].read_bytes()


def test_restart_after_gpu_steps(gpu, tmp_path):
    case = cases.reacting_step(scale=0.0625, inner=2)
    s = Solver(case, lib=gpu)
    try:
        s.upload()
        s.prepare(1)
        s.run(1, 2)
        path = tmp_path / "restart.bin"
        s.write_restart(str(path), 2)
        q, w, _, tt = s.download()
        step, tt_file, cells = F.read_restart(str(path), case.D, list(zip(case.ni, case.nj)))
        assert step == 2 and tt_file == tt
        for a, b in zip(cells, expected_cells(case, q, w)):
            assert np.array_equal(a, b)
        t = Solver(case, lib=gpu)
        try:
            assert t.read_restart(str(path)) == (2, tt)
            q2, w2, _, _ = t.download()
            D = case.D
            for p, c in enumerate(cells):
                ni, nj = case.ni[p], case.nj[p]
                assert np.array_equal(q2[p, 1:nj + 3, 1:ni + 3], c[..., :D])
                assert np.array_equal(w2[p, 1:nj + 3, 1:ni + 3, 3], c[..., D + 2])
            t.prepare(1)
            assert t.run(1, 1).status == 0
        finally:
            t.close()
    finally:
        s.close()


def test_geometry_bin_equals_restatement(gpu, orc, tmp_path):
    case = cases.reacting_step(scale=0.0625)
    for lib, tag in ((gpu, "gpu"), (orc, "orc")):
        s = Solver(case, lib=lib)
        try:
            s.write_geometry(str(tmp_path / ("%s.bin" % tag)))
        finally:
            s.close()
    assert (tmp_path / "gpu.bin").read_bytes() == (tmp_path / "orc.bin").read_bytes()
