"""The autotuner of the CUDA library: it reports a choice among timed
candidates, and the tuned launch shapes give the same bits as the default
ones (every candidate computes each face and cell alike)."""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _run(case, lib, nsteps):
    s = Solver(case, lib=lib)
    try:
        s.upload()
        s.prepare(1)
        s.run(1, nsteps)
        return s.download()[0], s.tuning()
    finally:
        s.close()


@pytest.mark.parametrize("make", [lambda: cases.reacting_step(scale=0.125, inner=3, precision=abi.PREC_MIXED),
                                  lambda: cases.reacting_step(scale=0.125, inner=3),
                                  lambda: cases.sod(200, 4)])
def test_tuned_shapes_give_the_default_bits(gpu, monkeypatch, make):
    case = make()
    q_tuned, rep = _run(case, gpu, 3)
    assert rep["enabled"] is True
    assert rep["thermo_block"] in (64, 128, 256)
    assert set(rep["thermo_ms"]) == {"64", "128", "256"}
    assert rep["residual_tile"] in rep["residual_ms"]
    assert min(rep["residual_ms"].values()) == rep["residual_ms"][rep["residual_tile"]]
    monkeypatch.setenv("SCFD_AUTOTUNE", "0")
    q_default, rep0 = _run(case, gpu, 3)
    assert rep0["enabled"] is False
    assert np.array_equal(q_tuned, q_default)
