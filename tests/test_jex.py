"""Jex, the exact Jacobian of the constant-volume source terms
(store/therm_lib/chemkin/uvhp/uv/FJ.f90:454-709), in the CPU restatement:
against central differences of Fex (FJ.f90:152-300), and its dndt against
Fex's.  The mechanism variants switch some reactions of the seeded H2/air
mechanism to the other rate forms of the reference (REV, fall-off LOW and
TROE, REV with +M, irreversible), so that every branch of Jex is exercised."""
import ctypes as C

import numpy as np
import pytest

from shared_cfd_b200 import abi, cases


def mechanism_variants():
    """(name, scfd_chem, checkable by differences) for the seeded mechanism and
    variants with the other rate forms.  The last variant flags a third-body
    table on a reaction whose rate has no third-body term; the reference's
    Jex then adds a third-body derivative with the dlnkdlnM of an earlier
    reaction, which differences of Fex cannot confirm (compared only between
    the device and the restatement)."""
    _, ch, _, _, _ = cases.reactor_batch(4)
    out = [("seeded", ch, True)]
    third = [i for i in range(ch.nr) if ch.exist_m[i]]
    plain = [i for i in range(ch.nr) if not ch.exist_m[i] and ch.rstate[i][1] == 0]
    v = abi.Chem.from_buffer_copy(ch)
    a, b, c = third[0], third[1], third[2]
    for i, kind in ((a, 2), (b, 3)):         # fall-off: LOW, TROE
        v.rstate[i][1] = kind
        v.cabe[i][0] = v.abe[i][0] + 3.0
        v.cabe[i][1] = v.abe[i][1] - 0.5
        v.cabe[i][2] = v.abe[i][2] * 0.8
    v.troe[b][0], v.troe[b][1], v.troe[b][2], v.troe[b][3] = 0.6, 1.0 / 120.0, 1.0 / 1500.0, 4000.0
    v.rstate[c][1] = 5                       # REV with +M
    v.cabe[c][0], v.cabe[c][1], v.cabe[c][2] = v.abe[c][0] - 1.0, v.abe[c][1], v.abe[c][2] + 3000.0
    v.rstate[plain[0]][1] = 1                # REV
    v.cabe[plain[0]][0] = v.abe[plain[0]][0] - 2.0
    v.cabe[plain[0]][1] = v.abe[plain[0]][1] + 0.3
    v.cabe[plain[0]][2] = v.abe[plain[0]][2] + 1000.0
    v.rstate[plain[1]][0] = 1                # irreversible
    out.append(("rate forms", v, True))
    q = abi.Chem.from_buffer_copy(v)
    q.rstate[third[3]][1] = 0                # third-body table, no third-body rate
    out.append(("stale dlnkdlnM", q, False))
    return out


def states(ch, m=12, seed=3):
    """Moles (mol/cm^3) and T: the benchmark's initial mixtures (floored at
    n_eps = 1e-40 as every call of the reference floors them), and partly
    burnt ones with radicals from 1e-12 to 1e-2 of the total."""
    _, _, T0, vrho, _ = cases.reactor_batch(m, seed=seed)
    mw = np.array([ch.mws[j] for j in range(ch.ns)])
    n = np.maximum(vrho / mw * 1e-3, 1e-40)
    rng = np.random.default_rng(seed)
    burnt = n * rng.uniform(0.2, 1.0, n.shape) + n.sum(axis=1, keepdims=True) * 10.0 ** rng.uniform(-12, -2, n.shape)
    T = np.concatenate([T0, rng.uniform(1100.0, 2800.0, m)])
    y = np.concatenate([np.concatenate([n, burnt]), T[:, None]], axis=1)
    # stay clear of the NASA-7 section switch at 1000 K
    y[:, -1] = np.where(np.abs(y[:, -1] - 1000.0) < 5.0, 1010.0, y[:, -1])
    return np.ascontiguousarray(y)


def rates(lib, ch, y, jac=True):
    n, N = y.shape
    f = np.zeros((n, N))
    J = np.zeros((n, N, N)) if jac else None
    code = lib.chem_rates(C.byref(ch), n, abi.dptr(y), abi.dptr(f), abi.dptr(J) if jac else None)
    assert code == 0
    return f, J


@pytest.mark.parametrize("k", range(3))
def test_jex_dndt_is_fex(orc, k):
    name, ch, _ = mechanism_variants()[k]
    y = states(ch)
    f, _ = rates(orc, ch, y, jac=False)
    g, _ = rates(orc, ch, y, jac=True)
    np.testing.assert_array_equal(f, g)


@pytest.mark.parametrize("k", range(2))
def test_jex_matches_central_differences_of_fex(orc, k):
    name, ch, _ = mechanism_variants()[k]
    y = states(ch)
    n, N = y.shape
    _, J = rates(orc, ch, y)
    fd = np.zeros_like(J)
    for j in range(N):
        h = 1e-6 * np.abs(y[:, j])
        yp, ym = y.copy(), y.copy()
        yp[:, j] += h
        ym[:, j] -= h
        fp, _ = rates(orc, ch, yp, jac=False)
        fm, _ = rates(orc, ch, ym, jac=False)
        fd[:, :, j] = (fp - fm) / (2.0 * h[:, None])
    # entries relative to the row's largest |J_ij y_j| / y_j scale
    scale = np.max(np.abs(J) * np.abs(y)[:, None, :], axis=2, keepdims=True) / np.abs(y)[:, None, :]
    err = np.abs(fd - J) / (scale + 1e-300)
    assert err.max() < 1e-5, (name, err.max())


def test_bad_arguments(orc):
    _, ch, _ = mechanism_variants()[0]
    assert orc.chem_rates(C.byref(ch), -1, None, None, None) == abi.E_ARG
    assert orc.chem_rates(C.byref(ch), 2, None, None, None) == abi.E_ARG
    assert orc.chem_rates(C.byref(ch), 0, None, None, None) == 0
