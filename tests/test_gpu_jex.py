"""Fex and Jex on the GPU (scfd_chem_rates, the per-thread form the flow
chemistry's fallback uses) against the CPU restatement, through the C ABI, for
the seeded mechanism and the rate-form variants of tests/test_jex.py.  The
device contracts multiply-adds and evaluates exp / log with its own library:
entries agree to 1e-11 of their row's scale."""
import numpy as np
import pytest

from test_jex import mechanism_variants, rates, states

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", range(3))
def test_gpu_fex_jex_match_restatement(gpu, orc, k):
    name, ch, _ = mechanism_variants()[k]
    y = states(ch, m=64, seed=11)
    f, J = rates(gpu, ch, y)
    g, K = rates(orc, ch, y)
    fs = np.abs(g).max(axis=1, keepdims=True)
    assert (np.abs(f - g) <= 1e-11 * fs).all(), (name, np.max(np.abs(f - g) / fs))
    Js = np.max(np.abs(K) * np.abs(y)[:, None, :], axis=2, keepdims=True) / np.abs(y)[:, None, :]
    assert (np.abs(J - K) <= 1e-11 * Js + 1e-300).all(), (name, np.max(np.abs(J - K) / (Js + 1e-300)))
    f2, _ = rates(gpu, ch, y, jac=False)
    np.testing.assert_allclose(f2, f, rtol=0, atol=0)
