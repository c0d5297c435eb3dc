"""CEA equilibrium (store/therm_lib/NASA/core/sub_chem.f90:1320-1651) on the
CPU: the NASA-9 / trans.inp readers, the restatement's stream states, and the
restatement pinned against an independent solution of the same equilibrium.

The independent solution: at fixed T the equilibrium moles of the
element-potential method are n_j = p0 / (rho Ru T) exp(-g_j/RT + sum_i a_ij pi_i)
(the stationarity condition of the Helmholtz energy at fixed density); the
element balance A n = b0 is solved for pi with scipy, and T with a bracketing
root finder on the internal energy.  g_j/RT = h_j/RT - s_j/R is written from
the NASA-9 polynomial forms, not from the restatement's vector of T-powers.
The restatement stops at its own 1e-9 tests (sub_chem.f90:1575-1583), so the
two agree to about 1e-7 in T and in the major species."""
import ctypes as C

import numpy as np
import pytest
from scipy import optimize

from shared_cfd_b200 import abi, cea

RU = 8.3144621
PST = 1e5


@pytest.fixture(scope="module")
def data():
    return cea.h2_air_data()


@pytest.fixture(scope="module")
def model(orc, data):
    with cea.Cea(data, lib=orc) as m:
        yield m


def test_tables_follow_the_reference_readers(data):
    assert (data.ns, data.ne, data.nt) == (9, 3, 7)
    # thermo.inp H2: 3 sections, MW 2.0158800, H 2.00
    assert list(data.nsec)[:9] == [3, 3, 2, 3, 3, 3, 2, 2, 3]
    assert data.mw[0] == pytest.approx(2.01588, abs=1e-12)
    ac = np.frombuffer(data.ac, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_ELEMENTS)
    assert list(ac[2, :3]) == [2.0, 1.0, 0.0]        # H2O
    assert list(ac[8, :3]) == [0.0, 0.0, 2.0]        # N2
    co = np.frombuffer(data.co, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_SECTIONS, 9)
    assert co[0, 0, 0] == pytest.approx(4.078323210e4)
    assert co[0, 0, 8] == pytest.approx(-3.043788844e1)
    # trans.inp order H, H2, H2O, N2, O, OH, O2 ('E 00' exponents read as E+00)
    assert list(data.tr2th)[:7] == [3, 0, 2, 8, 4, 5, 1]
    tr = np.frombuffer(data.trans, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_TSECTIONS, 4)
    assert tr[1, 0, 0] == pytest.approx(0.74553182)
    assert tr[1, 0, 1] == pytest.approx(43.555109)
    assert list(data.mwe)[:3] == [1.00797, 15.9994, 14.0067]


def test_generic_set_reads(orc):
    d = cea.hon17_data()
    assert d.ns == 17 and d.nt >= 10
    with cea.Cea(d, lib=orc) as m:
        assert m.info().fuel.T == pytest.approx(300.0, rel=1e-9)


def test_stream_states(model, data):
    inf = model.info()
    mwf = data.mw[0]
    mwo = (data.mw[1] + 3.76 * data.mw[8]) / 4.76
    assert inf.fuel.mw == pytest.approx(mwf, rel=1e-9)
    assert inf.oxidizer.mw == pytest.approx(mwo, rel=1e-9)
    assert inf.fuel.p == pytest.approx(1e5, rel=1e-9) and inf.oxidizer.p == pytest.approx(1e5, rel=1e-9)
    assert inf.fuel.T == pytest.approx(300.0, rel=1e-9) and inf.oxidizer.T == pytest.approx(300.0, rel=1e-9)
    assert inf.of == pytest.approx((data.mw[1] + 3.76 * data.mw[8]) / data.mw[0])
    assert inf.fuel.kappa == pytest.approx(1.405, abs=5e-3)
    assert inf.oxidizer.kappa == pytest.approx(1.40, abs=5e-3)
    # pure streams keep only their own elements (masks of initialize_cea):
    # the others sit at the floor tinytinyn = 1e-14 sum(n) of the entry state
    sf, so = sum(inf.fuel.n[:9]), sum(inf.oxidizer.n[:9])
    assert max(inf.fuel.n[j] for j in (1, 2, 4, 5, 6, 7, 8)) <= 1e-14 * sf * (1 + 1e-6)
    assert max(inf.oxidizer.n[j] for j in (0, 3, 5, 6, 7)) <= 1e-14 * so * (1 + 1e-6)
    assert inf.n_init == pytest.approx((sum(inf.fuel.n[:9]) + sum(inf.oxidizer.n[:9])) / 9)


def _g_rt(co, tr, nsec, T):
    """g/RT = h/RT - s/R of the NASA-9 forms (a1..a7, b1, b2)."""
    s = 0
    if tr[0][0] <= T:
        s = nsec - 1
        for l in range(nsec):
            if tr[l][1] > T:
                s = l
                break
    a = co[s]
    lt = np.log(T)
    h = (-a[0] / T**2 + a[1] * lt / T + a[2] + a[3] * T / 2 + a[4] * T**2 / 3 + a[5] * T**3 / 4
         + a[6] * T**4 / 5 + a[7] / T)
    sr = (-a[0] / (2 * T**2) - a[1] / T + a[2] * lt + a[3] * T + a[4] * T**2 / 2 + a[5] * T**3 / 3
          + a[6] * T**4 / 4 + a[8])
    return h - sr, h


def independent_equilibrium(data, b0, rho, E, species_mask, T_bracket=(250.0, 5000.0)):
    ns, ne = data.ns, data.ne
    co = np.frombuffer(data.co, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_SECTIONS, 9)
    tr = np.frombuffer(data.trange, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_SECTIONS, 2)
    A = np.frombuffer(data.ac, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_ELEMENTS)[:ns, :ne].T
    keep = b0 > 0
    sp = species_mask.copy()
    for i in range(ne):
        if not keep[i]:
            sp &= A[i] == 0
    Ak = A[keep][:, sp]
    bk = b0[keep]

    @np.errstate(over="ignore", invalid="ignore")
    def comp(T):
        g = np.array([_g_rt(co[j], tr[j], data.nsec[j], T)[0] for j in range(ns)])[sp]
        c = np.log(PST / (rho * RU * T))

        def resid(pi):
            n = np.exp(c - g + Ak.T @ pi)
            return (Ak @ n - bk) / bk

        pi0 = np.linalg.lstsq(Ak.T, g - c + np.log(np.maximum(Ak.T @ (bk / Ak.sum(axis=1)) / 2, 1e-3)),
                              rcond=None)[0]
        sol = optimize.root(resid, pi0, method="hybr", options={"xtol": 1e-14})
        n = np.zeros(ns)
        n[sp] = np.exp(c - g + Ak.T @ sol.x)
        return n

    def energy(T):
        n = comp(T)
        h = np.array([_g_rt(co[j], tr[j], data.nsec[j], T)[1] for j in range(ns)])
        return np.sum(n * (h - 1.0)) * RU * T - E

    T = optimize.brentq(energy, *T_bracket, xtol=1e-12, rtol=1e-14)
    return T, comp(T)


@pytest.mark.parametrize("yf,rho,de", [(0.0283, 1.0, 1.5e6), (0.01, 0.3, 2.5e6), (0.1, 0.5, 1.0e6),
                                       (0.5, 0.1, 4.0e6), (1.0, 0.08, 2e6), (0.0, 1.2, 3e6)])
def test_restatement_matches_independent_equilibrium(model, data, yf, rho, de):
    inf = model.info()
    Y = np.array([[yf], [1.0 - yf]])
    E = yf * inf.fuel.e + (1 - yf) * inf.oxidizer.e + de
    b0 = yf * np.array(inf.fuel.b0[:3]) + (1 - yf) * np.array(inf.oxidizer.b0[:3])
    out = model.solve(np.array([rho]), Y, np.array([E]), np.array([1500.0]), model.initial_n(1))
    assert out["not_converged"] == 0 and out["iters"][0] > 0
    T_ref, n_ref = independent_equilibrium(data, b0, rho, E, np.ones(9, dtype=bool))
    T, n = out["T"][0], out["n"][:, 0]
    assert abs(T - T_ref) / T_ref < 1e-7
    sn = n.sum()
    major = n_ref > 1e-6 * sn
    np.testing.assert_allclose(n[major], n_ref[major], rtol=1e-6)
    np.testing.assert_allclose(n[~major], n_ref[~major], atol=1e-6 * sn)
    assert out["MWave"][0] == pytest.approx(1e3 / sn, rel=1e-15)


def test_restatement_conserves_elements_and_energy(model, data):
    inf = model.info()
    rho, Y, e, T = cea.random_states(inf, 500, seed=11)
    out = model.solve(rho, Y, e, T, model.initial_n(500))
    assert out["not_converged"] == 0
    A = np.frombuffer(data.ac, dtype=np.float64).reshape(abi.CEA_MAX_SPECIES, abi.CEA_MAX_ELEMENTS)[:9, :3].T
    b0 = np.array(inf.fuel.b0[:3])[:, None] * Y[0] + np.array(inf.oxidizer.b0[:3])[:, None] * Y[1]
    # a stream below Y_eps = 1e-6 loses the elements only it carries (sub_chem.f90:1362-1378)
    b0[0, Y[0] < 1e-6] = 0.0
    b0[1:, Y[1] < 1e-6] = 0.0
    assert (Y[0] < 1e-6).any()
    bal = np.abs(A @ out["n"] - b0).max(axis=0) / b0.max(axis=0)
    assert bal.max() < 1e-8
    # relative to |e| + R T sum(n): the mixed-stream energy can pass through zero
    scale = np.abs(e) + 8.3144621 * out["T"] * out["n"].sum(axis=0)
    assert np.max(np.abs(cea.energy(data, out["T"], out["n"]) - e) / scale) < 1e-8
    # Yv sums to one; vhi is h_j per kg of species j
    # (less the dropped stream's mass, below 1e-6, in one-stream cells)
    mixed = (Y[0] >= 1e-6) & (Y[1] >= 1e-6)
    np.testing.assert_allclose(out["Yv"].sum(axis=0)[mixed], 1.0, rtol=1e-8)
    np.testing.assert_allclose(out["Yv"].sum(axis=0), 1.0, rtol=1e-6)


def test_warm_restart_is_idempotent(model):
    inf = model.info()
    rho, Y, e, T = cea.random_states(inf, 200, seed=5)
    a = model.solve(rho, Y, e, T, model.initial_n(200))
    b = model.solve(rho, Y, e, a["T"], a["n"])
    assert b["iters"].max() <= 2
    np.testing.assert_allclose(b["T"], a["T"], rtol=1e-8)


def test_one_stream_cells_drop_the_other_streams_elements(model):
    inf = model.info()
    rho = np.array([0.08, 1.2, 0.5, 0.5])
    Y = np.array([[1.0, 0.0, 1.0 - 1e-7, 1e-7], [0.0, 1.0, 1e-7, 1.0 - 1e-7]])
    e = np.array([inf.fuel.e + 1e6, inf.oxidizer.e + 2e6, inf.fuel.e + 1e6, inf.oxidizer.e + 2e6])
    out = model.solve(rho, Y, e, np.full(4, 1000.0), model.initial_n(4))
    n = out["n"]
    for c, absent in ((0, (1, 2, 4, 5, 6, 7, 8)), (1, (0, 2, 3, 5, 6, 7)), (2, (1, 2, 4, 5, 6, 7, 8)),
                      (3, (0, 2, 3, 5, 6, 7))):
        assert n[list(absent), c].max() <= 1e-13 * n[:, c].sum()


def test_empty_batch_and_bad_arguments(model, orc, data):
    z = np.zeros(0)
    out = model.solve(z, np.zeros((2, 0)), z, z, np.zeros((9, 0)))
    assert out["T"].size == 0
    assert orc.cea_solve(model.h, -1, None, None, None, None, None, None, None, None, None, None, None, None,
                         None) == abi.E_ARG
    assert orc.cea_solve(model.h, 4, None, None, None, None, None, None, None, None, None, None, None, None,
                         None) == abi.E_ARG
    bad = abi.CeaData.from_buffer_copy(data)
    bad.ns = 40
    h = C.c_void_p()
    assert orc.cea_create(C.byref(bad), C.byref(h)) == abi.E_ARG
    bad = abi.CeaData.from_buffer_copy(data)
    bad.abi_version = 99
    assert orc.cea_create(C.byref(bad), C.byref(h)) == abi.E_ARG
    bad = abi.CeaData.from_buffer_copy(data)
    for j in range(9):
        bad.nf[j] = 0.0
    assert orc.cea_create(C.byref(bad), C.byref(h)) == abi.E_ARG


def uv_states(model, m=300, seed=13):
    """Equilibrium states from cea (uv): rho, Y, e, T, n, p, h."""
    inf = model.info()
    rho, Y, e, T = cea.random_states(inf, m, seed=seed)
    out = model.solve(rho, Y, e, T, model.initial_n(m))
    p = rho * RU * 1e3 / out["MWave"] * out["T"]
    return rho, Y, e, out, p, e + p / rho


def test_hp_recovers_the_uv_equilibrium(model):
    """cea_hp at the p and h of a cea (uv) equilibrium, from a different start,
    returns the same T and composition (sub_chem.f90:1652-1962)."""
    rho, Y, e, uv, p, h = uv_states(model)
    mixed = (Y[0] >= 1e-6) & (Y[1] >= 1e-6)
    out = model.solve_hp(p[mixed], Y[:, mixed], h[mixed], np.full(mixed.sum(), 1200.0),
                         model.initial_n(int(mixed.sum())))
    assert out["not_converged"] == 0
    np.testing.assert_allclose(out["T"], uv["T"][mixed], rtol=1e-7)
    sn = uv["n"][:, mixed].sum(axis=0)
    assert np.max(np.abs(out["n"] - uv["n"][:, mixed]) / sn) < 1e-7
    np.testing.assert_allclose(out["kappa"], uv["kappa"][mixed], rtol=1e-6)
    np.testing.assert_allclose(out["mu"], uv["mu"][mixed], rtol=1e-6)


def test_tp_recovers_the_uv_equilibrium_and_its_enthalpy(model):
    """cea_tp at the p and T of a cea (uv) equilibrium returns its composition
    and h = e + p/rho (sub_chem.f90:1963-2248)."""
    rho, Y, e, uv, p, h = uv_states(model, seed=14)
    mixed = (Y[0] >= 1e-6) & (Y[1] >= 1e-6)
    out = model.solve_tp(p[mixed], Y[:, mixed], uv["T"][mixed], model.initial_n(int(mixed.sum())))
    assert out["not_converged"] == 0
    sn = uv["n"][:, mixed].sum(axis=0)
    assert np.max(np.abs(out["n"] - uv["n"][:, mixed]) / sn) < 1e-7
    scale = np.abs(h[mixed]) + RU * uv["T"][mixed] * sn
    assert np.max(np.abs(out["h"] - h[mixed]) / scale) < 1e-7


def test_hp_stream_states(orc):
    """initialize_cea('hp'): the streams at their own p and h stay at 300 K,
    1e5 Pa and reproduce the 'uv' states."""
    with cea.Cea(cea.h2_air_data(init_hp=True), lib=orc) as a, cea.Cea(cea.h2_air_data(), lib=orc) as b:
        x, y = a.info(), b.info()
        for s in ("fuel", "oxidizer"):
            u, v = getattr(x, s), getattr(y, s)
            assert u.p == pytest.approx(1e5, rel=1e-12)
            assert u.T == pytest.approx(v.T, rel=1e-8)
            for k in ("rho", "e", "h", "mw", "kappa", "mu"):
                assert getattr(u, k) == pytest.approx(getattr(v, k), rel=1e-7), (s, k)
