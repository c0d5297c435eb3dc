"""Batched 0-D reactors on the GPU (scfd_reactors_*) against the CPU
restatement, through the C ABI.

Tolerances.  The device and the host evaluate exp / log with different
libraries; the adaptive substep sequence of a reactor can then branch
differently (CHEMEQ2 and the Rosenbrock fallback choose their steps from error
ratios), so results are compared reactor by reactor with tolerances at the
integration error, not bit by bit: the flags must agree, the ignition delays
to 1e-3, most final temperatures exactly and all to 1e-2.  Runs of the same
batch on the GPU (graph replay, one launch per reactor) must agree bit by bit.
"""
import numpy as np
import pytest

from shared_cfd_b200 import abi, cases
from shared_cfd_b200.reactors import Reactors

pytestmark = pytest.mark.gpu

KEYS = ("T_end", "vrho_end", "t_ign", "evals", "flags")


@pytest.fixture(scope="module")
def batch():
    # 192 reactors of the benchmark distribution and 32 hot ones that ignite
    _, ch, T0, v, _ = cases.reactor_batch(192)
    _, _, T1, v1, _ = cases.reactor_batch(32, seed=7, T_range=(1540.0, 1600.0), phi_range=(0.8, 1.5))
    return ch, np.concatenate([T0, T1]), np.concatenate([v, v1])


@pytest.fixture(scope="module")
def reference(batch, orc):
    ch, T0, v = batch
    with Reactors(ch, len(T0), lib=orc) as r:
        return r.run(T0, v, 2e-3)


def test_reactors_match_restatement(gpu, batch, reference):
    ch, T0, v = batch
    with Reactors(ch, len(T0)) as r:
        out = r.run(T0, v, 2e-3)
    ref = reference
    assert out["status"] == 0
    assert np.array_equal(out["flags"], ref["flags"])
    ign = (ref["flags"] & abi.REACTOR_IGNITED) > 0
    assert ign.sum() >= 5
    assert np.allclose(out["t_ign"][ign], ref["t_ign"][ign], rtol=1e-3, atol=0.0)
    assert (out["t_ign"][~ign] == -1.0).all()
    rel = np.abs(out["T_end"] - ref["T_end"]) / ref["T_end"]
    assert (rel <= 1e-2).all(), rel.max()
    assert np.mean(rel == 0.0) >= 0.5
    mass = out["vrho_end"].sum(axis=1) / ref["vrho_end"].sum(axis=1)
    assert np.allclose(mass, 1.0, rtol=1e-3)


def test_graph_replay_and_per_launch_are_bit_identical(gpu, batch):
    ch, T0, v = batch
    with Reactors(ch, len(T0)) as r:
        a = r.run(T0, v, 2e-3)           # captures the CUDA graph
        b = r.run(T0, v, 2e-3)           # replays it
        assert r.launch_count() == 1
        for k in KEYS:
            assert np.array_equal(a[k], b[k]), k
        n = 24
        c = r.run(T0[:n], v[:n], 2e-3, mode=abi.REACTOR_PER_LAUNCH)
        assert r.launch_count() == n
        d = r.run(T0[:n], v[:n], 2e-3)
        for k in KEYS:
            assert np.array_equal(c[k], d[k]), k
