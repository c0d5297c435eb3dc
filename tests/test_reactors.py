"""Batched 0-D reactors on the CPU restatement: inputs, conservation, the
ignition bookkeeping of reaction_one_steps (sub_chem.f90:1467-1472), the
reaction_chemeq2 call loop, and argument checking of the C ABI (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200 import chem as CH
from shared_cfd_b200.reactors import Reactors


@pytest.fixture(scope="module")
def hot_batch():
    # hot, stoichiometric-to-rich mixtures: most of these ignite within 2 ms
    return cases.reactor_batch(12, seed=7, T_range=(1540.0, 1600.0), phi_range=(0.8, 1.5))


def test_reactor_inputs_follow_the_draws():
    m, ch, T0, vrho, (T, p, phi) = cases.reactor_batch(16, seed=3)
    mw = np.asarray(m.mws)
    idx = {s.strip().upper(): k for k, s in enumerate(m.species)}
    n = vrho / mw  # mol / m^3 * 1e-3 scale: ratios only
    assert np.allclose(n[:, idx["H2"]] / n[:, idx["O2"]], 2.0 * phi, rtol=1e-12)
    assert np.allclose(n[:, idx["N2"]] / n[:, idx["O2"]], 3.76, rtol=1e-12)
    # ideal-gas pressure of the partial densities (n in mol/cm^3 -> Pa)
    ncgs = vrho / mw * 1e-3
    p_back = ncgs.sum(axis=1) * CH.RU_CGS * T0 / 1e1
    assert np.allclose(p_back, p, rtol=1e-12)
    assert (T0 >= 900.0).all() and (T0 <= 1600.0).all()


def test_oracle_reactors_conserve_mass_and_flag_ignition(orc, hot_batch):
    m, ch, T0, vrho, _ = hot_batch
    with Reactors(ch, len(T0), lib=orc) as r:
        out = r.run(T0, vrho, 2e-3)
    assert out["status"] == 0
    assert not (out["flags"] & abi.REACTOR_FAILED).any()
    assert np.isfinite(out["T_end"]).all()
    # CHEMEQ2's alpha-QSS update is not conservative (each species is advanced on
    # its own); over 2000 calls the total mass drifts at the integrator tolerance
    m0, m1 = vrho.sum(axis=1), out["vrho_end"].sum(axis=1)
    assert np.allclose(m1, m0, rtol=1e-3)
    ign = (out["flags"] & abi.REACTOR_IGNITED) > 0
    assert ign.sum() >= 3
    assert (out["t_ign"][ign] > 0.0).all() and (out["t_ign"][ign] < 2e-3).all()
    assert (out["t_ign"][~ign] == -1.0).all()
    assert (out["T_end"][ign] >= T0[ign] + 400.0).all()
    assert (out["evals"] >= 2 * 2000).all()   # at least one CHEMEQ2 attempt per 1 us call


def test_ignition_delay_is_insensitive_to_the_call_interval(orc, hot_batch):
    m, ch, T0, vrho, _ = hot_batch
    res = {}
    for dtc in (1e-6, 5e-7):
        with Reactors(ch, len(T0), lib=orc) as r:
            res[dtc] = r.run(T0, vrho, 2e-3, dt_call=dtc)
    a, b = res[1e-6], res[5e-7]
    both = ((a["flags"] & b["flags"]) & abi.REACTOR_IGNITED) > 0
    assert both.sum() >= 3
    assert np.allclose(a["t_ign"][both], b["t_ign"][both], rtol=0.05)


def test_single_call_equals_chemeq2(orc, orc_raw):
    """With dt_call = t_end a reactor is one reaction_chemeq2 call."""
    m, ch, T0, vrho, _ = cases.reactor_batch(4, seed=11)
    t_end = 1e-7
    with Reactors(ch, 4, lib=orc) as r:
        out = r.run(T0, vrho, t_end, dt_call=0.0)
    ns = ch.ns
    f = orc_raw.orc_chemeq2
    f.argtypes = [C.POINTER(abi.Chem), C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    inv = 1.0 / np.asarray(m.mws)
    for k in range(4):
        y = np.zeros(ns + 1)
        y[:ns] = np.maximum(vrho[k] * inv * 1e-3, 1e-40)
        y[ns] = T0[k]
        a, fb = C.c_int64(), C.c_int()
        assert f(C.byref(ch), y.ctypes.data_as(C.POINTER(C.c_double)), t_end, C.byref(a), C.byref(fb)) == 0
        assert out["T_end"][k] == y[ns]
        vr = np.maximum(np.maximum(y[:ns], 1e-40) * np.asarray(m.mws) * 1e3 * inv * 1e-3, 1e-40) * \
            np.asarray(m.mws) * 1e3
        assert np.array_equal(out["vrho_end"][k], vr)


def test_reactor_api_rejects_bad_arguments_without_gpu():
    from shared_cfd_b200 import build
    build.build()
    lib = abi.Bound(C.CDLL(build.OUT), "scfd_")
    m, ch, _, _, _ = cases.reactor_batch(2)
    h = C.c_void_p()
    assert lib.reactors_create(C.byref(ch), 0, C.byref(h)) == abi.E_ARG
    bad = abi.Chem()
    C.memmove(C.byref(bad), C.byref(ch), C.sizeof(abi.Chem))
    bad.ns = 0
    assert lib.reactors_create(C.byref(bad), 8, C.byref(h)) == abi.E_ARG
    assert lib.reactors_launch(None, None) == abi.E_ARG
    assert lib.reactors_download(None, None, None, None, None, None) == abi.E_ARG
