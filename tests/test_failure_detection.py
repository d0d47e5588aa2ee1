"""Failure detection of the BP loops, with faults made on the host.

The reference handles one failure: the iteration cap of its BP loop ends
with a ``log.warning`` (bp_quantum_emulator.py:254-261, 284-291). Its NaN
handling is implicit: ``while vidal_dist > accuracy`` is false for NaN, so
the loop stops and the NaN state flows on silently. This package keeps the
warning, records DQZ_ERR_NOT_CONVERGED, and raises NonFiniteError
(DQZ_ERR_NONFINITE) on a NaN / Inf distance.

CPU tests drive the shared stopping rule (``engine.converge``) with fake
sweeps and distances; GPU tests load NaN / Inf node tensors and all-zero
messages from the host and run a loop that cannot converge within a cap of 5.
No test faults, traps or hangs a GPU: the bad values are ordinary data.
"""

import logging
import math

import numpy as np
import pytest

from dequantizer_b200 import _lib
from dequantizer_b200.engine import converge


class FakeLoop:
    def __init__(self, distances):
        self.distances = list(distances)
        self.steps = 0

    def step(self):
        self.steps += 1

    def distance(self):
        return self.distances[self.steps - 1]


def test_converge_stops_at_the_tolerance():
    f = FakeLoop([1.0, 0.1, 1e-7, 1e-9])
    assert converge(f.step, f.distance, 1e-6, 100) == (3, _lib.DQZ_OK)


def test_converge_reports_the_cap_with_the_reference_warning(caplog):
    f = FakeLoop([1.0, -1.0] * 10)  # an oscillating loop never meets tol = 0
    with caplog.at_level(logging.WARNING):
        done, status = converge(f.step, lambda: abs(f.distance()), 0.0, 5)
    assert (done, status) == (5, _lib.DQZ_ERR_NOT_CONVERGED)
    assert "maximal number of iterations" in caplog.text


@pytest.mark.parametrize("bad", [math.nan, math.inf])
def test_converge_raises_on_a_non_finite_distance(bad):
    f = FakeLoop([1.0, bad, 0.0])
    with pytest.raises(_lib.NonFiniteError) as ei:
        converge(f.step, f.distance, 1e-6, 100)
    assert ei.value.status == _lib.DQZ_ERR_NONFINITE
    assert f.steps == 2


def test_converge_counts_blocks_of_sweeps():
    f = FakeLoop([1.0, 1.0, 1e-9])
    assert converge(f.step, f.distance, 1e-6, 100, sweeps_per_step=8, first=2) == (26, _lib.DQZ_OK)


# ----------------------------------------------------------------- GPU
def _engine(chi=4, seed=3):
    from dequantizer_b200.engine import BPEngine
    from dequantizer_b200.graph import get_random_regular_graph
    from tests.helpers import random_messages, random_tensors

    g = get_random_regular_graph(10, 3, 2, chi, seed)
    eng = BPEngine(g, schedule="sync")
    ts = random_tensors(g, seed)
    ms = random_messages(g, seed + 1)
    from dequantizer_b200.graph import MessageID

    eng.load_tensors([ts[n.id] for n in eng.topo.nodes])
    eng.load_messages([ms[MessageID(nd.id, e.id)] for nd, e in eng.topo.half_ids()],
                      [ms[MessageID(e.id, nd.id)] for nd, e in eng.topo.half_ids()])
    return eng


@pytest.mark.gpu
def test_count_nonfinite_counts_exactly():
    import torch

    x = torch.zeros(1000, dtype=torch.complex128, device="cuda")
    x[3] = complex(math.nan, 0.0)
    x[500] = complex(0.0, math.inf)
    x[999] = complex(-math.inf, math.nan)
    assert _lib.count_nonfinite(x) == 4
    assert _lib.count_nonfinite(x.to(torch.complex64)) == 4
    assert _lib.count_nonfinite(torch.ones(7, device="cuda", dtype=torch.float64)) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [math.nan, math.inf])
def test_bp_run_reports_non_finite_node_tensors(bad):
    eng = _engine()
    eng.check_finite()
    eng.T[17] = complex(bad, 0.0)
    with pytest.raises(_lib.NonFiniteError):
        eng.check_finite()
    with pytest.raises(_lib.NonFiniteError) as ei:
        eng.run(1e-8, max_sweeps=50)
    assert ei.value.status == _lib.DQZ_ERR_NONFINITE


@pytest.mark.gpu
@pytest.mark.parametrize("graphed", [False, True])
def test_bp_run_reports_zero_messages(graphed):
    """All-zero incoming messages give a zero trace: the normalised update is
    NaN (as in the reference, tensor_ops.py:58), and the loop reports it."""
    eng = _engine()
    eng.e2n.zero_()
    eng.n2e.zero_()
    with pytest.raises(_lib.NonFiniteError):
        if graphed:
            eng.run_graphed(1e-8, max_sweeps=50)
        else:
            eng.run(1e-8, max_sweeps=50)


@pytest.mark.gpu
def test_bp_run_reports_the_cap(caplog):
    eng = _engine()
    with caplog.at_level(logging.WARNING):
        done = eng.run(0.0, max_sweeps=5)
    assert done == 5 and eng.status == _lib.DQZ_ERR_NOT_CONVERGED
    assert "maximal number of iterations" in caplog.text
    eng2 = _engine()
    eng2.run(1e-8, max_sweeps=500)
    assert eng2.status == _lib.DQZ_OK


@pytest.mark.gpu
def test_emulator_reports_a_non_finite_regauge():
    """A NaN entry in the emulator's state: the regauge loop raises instead of
    carrying the NaN on (the reference's loop would stop silently)."""
    import torch

    from dequantizer_b200.emulator import BPQuantumEmulator
    from dequantizer_b200.graph import get_nd_lattice

    lat = get_nd_lattice([2, 3], 2, 1, True)
    em = BPQuantumEmulator(lat, 1, 4, lat.edges_number, 1e-6, 50)
    bad = np.eye(2, dtype=complex)
    bad[0, 0] = math.nan
    em.apply_q1(bad, (0, 0))
    for e in lat.edges:
        em.apply_q2(np.eye(4, dtype=complex).reshape(2, 2, 2, 2), *e)
    with pytest.raises(_lib.NonFiniteError):
        em.dens_q1((0, 0))
        torch.cuda.synchronize()
