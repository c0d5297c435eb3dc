"""The DVODE restatement of the CPU checker (oracle/dvode.h, the
reference's dvode.f on its MF = 21 path), checked against problems with
known solutions: stiff linear systems against the matrix exponential, and
Robertson's stiff kinetics against published reference values."""
import ctypes as C

import numpy as np
import pytest


def _run(orc, problem, y0, t0, tout, rtol, atol, A=None):
    f = orc.orc_dvode_test
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.POINTER(C.c_int64)]
    y = np.ascontiguousarray(y0, dtype=np.float64).copy()
    Aa = None if A is None else np.ascontiguousarray(A, dtype=np.float64)
    nst = C.c_int64()
    st = f(problem, len(y), None if Aa is None else Aa.ctypes.data, y.ctypes.data, t0, tout, rtol, atol,
           C.byref(nst))
    return st, y, nst.value


@pytest.fixture(scope="module")
def orc_raw():
    from conftest import build_oracle
    return C.CDLL(build_oracle())


def test_stiff_diagonal_system(orc_raw):
    lam = np.array([-1.0, -10.0, -1000.0, -1e5])
    y0 = np.array([1.0, 2.0, -1.0, 0.5])
    for tout in (0.01, 0.3, 2.0):
        st, y, nst = _run(orc_raw, 0, y0, 0.0, tout, 1e-9, 1e-14, np.diag(lam))
        assert st == 2
        exact = y0 * np.exp(lam * tout)
        # components that decayed below the absolute tolerance are held to it
        err = np.abs(y - exact) / (np.abs(exact) + 1e-12)
        assert err.max() < 1e-5, (tout, err)


def test_stiff_coupled_system_against_expm(orc_raw):
    from scipy.linalg import expm
    rng = np.random.default_rng(5)
    n = 6
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(-np.logspace(0, 4, n)) @ Q.T
    y0 = rng.standard_normal(n)
    st, y, nst = _run(orc_raw, 0, y0, 0.0, 0.5, 1e-10, 1e-14, A)
    assert st == 2 and nst > 10
    exact = expm(A * 0.5) @ y0
    assert np.linalg.norm(y - exact) / np.linalg.norm(exact) < 1e-6


def test_robertson_reference_values(orc_raw):
    """Robertson's problem at t = 40 (E. Hairer, G. Wanner, Solving ODEs II,
    reference solution): y1 = 0.7158270687..., y2 = 9.185534765e-6,
    y3 = 0.2841637457..."""
    st, y, nst = _run(orc_raw, 1, [1.0, 0.0, 0.0], 0.0, 40.0, 1e-8, 1e-14)
    assert st == 2
    ref = np.array([0.7158270687193e0, 0.9185534764557e-5, 0.2841637457395e0])
    assert np.max(np.abs(y - ref) / ref) < 1e-5
    assert abs(y.sum() - 1.0) < 1e-10   # the kinetics conserve y1 + y2 + y3


def test_excess_work_restarts_continue_the_integration(orc_raw):
    """Over 1e5 time units Robertson needs more than MXSTEP = 500 steps per
    call: the reference's loop restarts DVODE from where it stopped
    (ISTATE = -1) and reaches tout."""
    st, y, nst = _run(orc_raw, 1, [1.0, 0.0, 0.0], 0.0, 4.0e5, 1e-8, 1e-14)
    assert st == 2 and nst > 500
    assert abs(y.sum() - 1.0) < 1e-8 and y[0] < 0.01


def test_reactor_flags_under_one_ulp():
    """The envelope the GPU reactor test allows: the oracle's own reactors,
    with T0 moved by one ulp, keep their ignited / failed flags and ignition
    delays (to 1e-4) but flip the DVODE flag of a few tenths of a percent
    (whether an interval uses up its 10 CHEMEQ2 attempts turns on rounding)."""
    import ctypes as C

    from conftest import build_oracle
    from shared_cfd_b200 import abi, cases
    from shared_cfd_b200.reactors import Reactors

    orc = abi.Bound(C.CDLL(build_oracle()), "orc_")
    n = 2048
    _, ch, T0, v, _ = cases.reactor_batch(n)
    with Reactors(ch, n, lib=orc) as r:
        a = r.run(T0, v, 2e-3)
        b = r.run(np.nextafter(T0, np.inf), v, 2e-3)
    hard = abi.REACTOR_IGNITED | abi.REACTOR_FAILED
    assert np.array_equal(a["flags"] & hard, b["flags"] & hard)
    flips = np.count_nonzero((a["flags"] ^ b["flags"]) & abi.REACTOR_FELL_BACK)
    assert 0 < flips <= 0.005 * n, flips
    ign = (a["flags"] & abi.REACTOR_IGNITED) > 0
    assert np.allclose(a["t_ign"][ign], b["t_ign"][ign], rtol=1e-4, atol=0.0)
