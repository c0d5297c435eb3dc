"""Chemkin set-up and thermodynamics against the reference's own data (CPU).

sample/no27.chemkin_reaction/restart.bin stores, per cell, q together with the
gas constant R, gamma and pressure p that the reference computed with calc_T
(store/core/inout.f90:51-56).  Recomputing R, gamma, p from q with the parsed
mechanism must reproduce them."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from shared_cfd_b200 import chem as CH

from conftest import REFERENCE

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_mech():
    d = json.load(open(os.path.join(GOLD, "no27_mech.json")))
    m = CH.Mechanism()
    m.species, m.mws, m.tthre, m.coeff = d["species"], d["mws"], d["tthre"], d["coeff"]
    m.reactions, m.trans, m.rtol, m.atol = d["reactions"], d["trans"], d["rtol"], d["atol"]
    return m, d


def _cells():
    z = np.load(os.path.join(GOLD, "no27_cells.npz"))
    return z["vals"], int(z["dimq"])


def _recompute(calc, m, vals, D):
    nY = D - 3
    out = []
    for v in vals:
        q, R, g, p = v[:D], v[D], v[D + 1], v[D + 2]
        rho = q[:nY].sum()
        u, vv = q[nY] / rho, q[nY + 1] / rho
        ei = q[nY + 2] / rho - 0.5 * (u * u + vv * vv)
        T, kap, MW = calc(q[:nY], rho, ei, p / (rho * R))
        R2 = CH.R_UNI / MW
        out.append((abs(R2 / R - 1), abs(kap / g - 1), abs(rho * R2 * T / p - 1)))
    return np.array(out)


def test_no27_state_known_answer_python():
    m, _ = load_mech()
    vals, D = _cells()

    def calc(vrho, rho, E, T):
        T2, kap, MW, _, _, _ = CH.calc_T(m, list(vrho), rho, E, T)
        return T2, kap, MW
    e = _recompute(calc, m, vals, D)
    # The stored R, gamma, p lag q by one update wherever the flow changed in
    # the last step; about 70% of the sampled cells are converged to rounding.
    assert np.median(e, axis=0).max() < 1e-13
    assert (e.max(axis=1) < 1e-11).mean() > 0.65
    assert e.max() < 1e-3


def test_no27_state_known_answer_oracle(orc_raw):
    m, _ = load_mech()
    ch = CH.to_struct(m)
    vals, D = _cells()
    nY = D - 3
    f = orc_raw.orc_calc_T
    f.restype = C.c_int
    dp = C.POINTER(C.c_double)
    f.argtypes = [C.c_void_p, dp, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp]

    def calc(vrho, rho, E, T):
        v = np.ascontiguousarray(vrho, dtype=np.float64)
        Tt, k, mw, mu = C.c_double(T), C.c_double(), C.c_double(), C.c_double()
        dh = np.zeros(nY)
        vh = np.zeros(nY)
        st = f(C.byref(ch), v.ctypes.data_as(dp), rho, E, C.byref(Tt), C.byref(k), C.byref(mw),
               dh.ctypes.data_as(dp), vh.ctypes.data_as(dp), C.byref(mu))
        assert st == 0
        return Tt.value, k.value, mw.value
    e = _recompute(calc, m, vals, D)
    assert np.median(e, axis=0).max() < 1e-13
    assert (e.max(axis=1) < 1e-11).mean() > 0.65


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE),
                    reason="SCFD_REFERENCE does not name a reference checkout")
def test_parser_reproduces_frozen_mechanism():
    core = os.path.join(REFERENCE, "store/therm_lib/chemkin/core")
    s27 = os.path.join(REFERENCE, "sample/no27.chemkin_reaction")
    m = CH.parse_chem(open(os.path.join(s27, "chem.inp")).read(), open(os.path.join(core, "MW.inp")).read())
    CH.parse_trans(open(os.path.join(core, "trans.inp")).read(), m)
    comp = CH.parse_control_chem(open(os.path.join(s27, "control_chem.inp")).read(), m)
    fo = CH.fuel_oxidizer(m, comp, len(m.species))
    _, d = load_mech()
    assert m.species == d["species"] and m.mws == d["mws"] and m.coeff == d["coeff"]
    assert json.loads(json.dumps(m.reactions)) == d["reactions"]
    assert list(fo["o"]["w"]) == d["wo"] and list(fo["f"]["w"]) == d["wf"]


def test_species_reordering_puts_reactants_first():
    from shared_cfd_b200 import cases
    m, fo = cases.h2air_mechanism()
    assert m.species[:3] == ["H2", "O2", "N2"]
    # oxidiser: only O2 and N2; fuel: only H2
    assert fo["o"]["q"][0] == 0.0 and fo["o"]["q"][1] > 0 and fo["o"]["q"][2] > 0
    assert fo["f"]["q"][0] > 0 and fo["f"]["q"][1] == 0.0


def test_mechanism_parse_details():
    from shared_cfd_b200 import cases
    m, _ = cases.h2air_mechanism()
    assert len(m.reactions) == 19
    # +M reactions carry Rstate(,2) = 4 and no species named M
    tb = [r for r in m.reactions if r["exist_m"]]
    assert len(tb) == 6 and all(r["rstate"][1] == 4 for r in tb)
    for r in m.reactions:
        assert -1 not in r["reac"] and -1 not in r["prod"]
    # element balance of every reaction
    comp = {"H2": (2, 0, 0), "O2": (0, 2, 0), "H2O": (2, 1, 0), "H": (1, 0, 0), "O": (0, 1, 0),
            "OH": (1, 1, 0), "HO2": (1, 2, 0), "H2O2": (2, 2, 0), "N2": (0, 0, 2)}
    for r in m.reactions:
        a = np.sum([comp[m.species[k - 1]] for k in r["reac"]], axis=0)
        b = np.sum([comp[m.species[k - 1]] for k in r["prod"]], axis=0)
        assert np.array_equal(a, b), r["text"]
