"""FP64 numpy restatement of the emulators and of the annealing / kicked-Ising
drivers.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

* ``BPQuantumEmulator``    -- quantum_emulator/bp_quantum_emulator.py:32-300
* ``ExactQuantumEmulator`` -- quantum_emulator/exact_quantum_emulator.py:11-147
* annealing gates / loop   -- examples/quantum_annealing/quantum_annealing/src/
                              quantum_annealer.py:44-152, scheduler.py:7-14
"""

import logging
from typing import Dict, List, Optional

import numpy as np

from dequantizer_b200.graph import Edge, Node, TensorGraph
from dequantizer_b200.initializers import (
    get_message_random_nonnegative_initializer,
    get_tensor_std_state_initializer,
)
from . import maps

log = logging.getLogger(__name__)

EMULATOR_EPS = 1e-10  # bp_quantum_emulator.py:84-86, 161


class BPQuantumEmulator:
    """Vidal-form emulator with a BP regauging loop.

    ``key`` is an integer seed; each Vidal canonicalisation draws a fresh
    message-initializer seed from a numpy generator seeded with it, standing in
    for the reference's ``split(self.prng_key)`` (bp_quantum_emulator.py:247)."""

    def __init__(
        self,
        tensor_graph: TensorGraph,
        key: int,
        max_chi: int,
        gates_number_per_regauging: int,
        belief_propagation_accuracy: float = 1e-5,
        max_belief_propagation_iterations: Optional[int] = 100,
        synchronous_update: bool = False,
        traversal_type: str = "dfs",
    ):
        self.tensor_graph = tensor_graph
        self._rng = np.random.default_rng(key)
        self.max_chi = max_chi
        self.max_iters = max_belief_propagation_iterations
        self.per_regauging = gates_number_per_regauging
        self.accuracy = belief_propagation_accuracy
        self.passed = 0
        self.traverser = list(tensor_graph.get_traversal_iterator(ordering=traversal_type))
        self.bp_map = maps.get_belief_propagation_map(self.traverser, synchronous_update)
        self.vg_map = maps.get_vidal_gauge_fixing_map(self.traverser, EMULATOR_EPS)
        self.vd_map = maps.get_vidal_gauge_distance_map(self.traverser, EMULATOR_EPS)
        self.sg_map = maps.get_symmetric_gauge_fixing_map(self.traverser, EMULATOR_EPS)
        self.tensors = maps.init_tensors(tensor_graph, get_tensor_std_state_initializer())
        self.lambdas = None
        self.after_regauging_vidal_distances: List[float] = []
        self.truncated_affected_vidal_distances: List[float] = []
        self.truncation_errors: List[float] = []
        self.entropies: List[float] = []
        self.bp_iterations: List[int] = []
        self._set_to_vidal_canonical()

    def _next_seed(self) -> int:
        return int(self._rng.integers(0, 2**31 - 1))

    def _init_messages(self):
        return self.tensor_graph.init_messages(get_message_random_nonnegative_initializer(self._next_seed()))

    def set_to_product_state(self, state: Dict):
        """bp_quantum_emulator.py:110-130."""
        self.tensor_graph.to_product()

        def init(node: Node):
            t = np.zeros((node.dimension,), dtype=np.complex128)
            t[state[node.id]] = 1.0
            return t.reshape(node.bond_shape + (node.dimension,))

        self.tensors = maps.init_tensors(self.tensor_graph, init)
        self._set_to_vidal_canonical()
        self.passed = 0

    def apply_q2(self, gate, id1, id2):
        """bp_quantum_emulator.py:144-167."""
        if self.passed >= self.per_regauging:
            self._vidal_regauging()
            self.passed = 0
        _, _, err, entropy = maps.apply2_to_vidal_canonical(
            self.tensor_graph, id1, id2, self.tensors, self.lambdas, np.asarray(gate),
            EMULATOR_EPS, None, self.max_chi,
        )
        self.truncation_errors.append(err)
        self.entropies.append(entropy)
        self.passed += 1

    def apply_q1(self, gate, node_id):
        """bp_quantum_emulator.py:175-180."""
        self.tensors = maps.apply1(self.tensor_graph, node_id, self.tensors, np.asarray(gate))

    def dens_q1(self, node_id) -> np.ndarray:
        """bp_quantum_emulator.py:188-207."""
        if self.passed != 0:
            self._vidal_regauging()
            self.passed = 0
        tensors = self.sg_map(self.tensors, self.lambdas)
        messages = maps.lambdas2messages(self.lambdas)
        node = self.tensor_graph.get_node(node_id)
        dens = maps.get_one_side_density_matrix(node, tensors, messages)
        assert np.isclose(np.trace(dens), 1.0, 1e-8)
        return dens

    def measure(self, node_id, sample: float) -> int:
        """bp_quantum_emulator.py:215-233, with the uniform sample passed in."""
        dens = self.dens_q1(node_id)
        result = 0 if dens[0, 0].real > sample else 1
        proj = np.zeros((2, 2))
        proj[result, result] = 1.0
        self.apply_q1(proj, node_id)
        self.tensors = self.sg_map(self.tensors, self.lambdas)
        self._set_to_vidal_canonical()
        self.passed = 0
        return result

    def _bp_loop(self, tensors, messages, start_dist):
        vidal_dist = start_dist
        iters = 0
        canonical, lambdas = None, None
        while vidal_dist > self.accuracy:
            if self.max_iters is not None and self.max_iters <= iters:
                log.warning("Belief propagation reached the maximal number of iterations.")
                break
            messages = self.bp_map(tensors, messages)
            canonical, lambdas = self.vg_map(tensors, messages)
            vidal_dist = self.vd_map(canonical, lambdas)
            iters += 1
        self.bp_iterations.append(iters)
        return canonical, lambdas, vidal_dist

    def _set_to_vidal_canonical(self):
        """bp_quantum_emulator.py:245-270."""
        messages = self._init_messages()
        canonical, lambdas, vd = self._bp_loop(self.tensors, messages, np.finfo(np.float64).max)
        self.after_regauging_vidal_distances.append(vd)
        self.lambdas = lambdas
        self.tensors = canonical

    def _vidal_regauging(self):
        """bp_quantum_emulator.py:272-300."""
        tensors = self.sg_map(self.tensors, self.lambdas)
        messages = maps.lambdas2messages(self.lambdas)
        canonical, lambdas = self.vg_map(tensors, messages)
        vd = self.vd_map(canonical, lambdas)
        self.truncated_affected_vidal_distances.append(vd)
        c2, l2, vd2 = self._bp_loop(tensors, messages, vd)
        if c2 is not None:
            canonical, lambdas, vd = c2, l2, vd2
        self.after_regauging_vidal_distances.append(vd)
        self.lambdas = lambdas
        self.tensors = canonical


class ExactQuantumEmulator:
    """Dense state-vector emulator (exact_quantum_emulator.py:11-147); qubit
    order = BFS order of nodes."""

    def __init__(self, tensor_graph: TensorGraph):
        self.n = tensor_graph.nodes_number
        self.node2pos = {}
        pos = 0
        for element in tensor_graph.get_traversal_iterator():
            if isinstance(element, Node):
                self.node2pos[element.id] = pos
                pos += 1
        self.state = np.zeros((2**self.n,), dtype=np.complex128)
        self.state[0] = 1.0

    def set_to_product_state(self, state: Dict):
        shift = 0
        for node_id, pos in self.node2pos.items():
            if state[node_id] == 1:
                shift += 2 ** (self.n - pos - 1)
        self.state = np.zeros((2**self.n,), dtype=np.complex128)
        self.state[shift] = 1.0

    def apply_q2(self, gate, id1, id2):
        p1, p2 = self.node2pos[id1], self.node2pos[id2]
        back = list(range(self.n - 2))
        if p1 < p2:
            back.insert(p1, self.n - 2)
            back.insert(p2, self.n - 1)
        else:
            back.insert(p2, self.n - 1)
            back.insert(p1, self.n - 2)
        st = np.tensordot(self.state.reshape(self.n * (2,)), np.asarray(gate), axes=[[p1, p2], [2, 3]])
        self.state = np.transpose(st, back).reshape((-1,))

    def apply_q1(self, gate, node_id):
        pos = self.node2pos[node_id]
        back = list(range(pos)) + [self.n - 1] + list(range(pos, self.n - 1))
        st = np.tensordot(self.state.reshape(self.n * (2,)), np.asarray(gate), axes=[[pos], [1]])
        self.state = np.transpose(st, back).reshape((-1,))

    def dens_q1(self, node_id) -> np.ndarray:
        pos = self.node2pos[node_id]
        st = self.state.reshape(self.n * (2,))
        st = np.swapaxes(st, 0, pos).reshape((2, -1))
        return st @ st.T.conj()

    def measure(self, node_id, sample: float) -> int:
        dens = self.dens_q1(node_id)
        p = dens[0, 0].real
        result, norm = (0, p) if p > sample else (1, 1 - p)
        proj = np.zeros((2, 2))
        proj[result, result] = 1.0
        self.apply_q1(proj, node_id)
        self.state = self.state / np.sqrt(norm)
        return result


# ---------------------------------------------------------------------------
# Annealing / kicked-Ising gate construction
# ---------------------------------------------------------------------------

HADAMARD = np.sqrt(0.5) * np.array([[1, 1], [1, -1]], dtype=np.complex128)


def q2_annealing_gate(coupling: float, h1_over_deg: float, h2_over_deg: float, tau: float) -> np.ndarray:
    """exp(-i tau (J ZZ + h1/deg1 Z1 + h2/deg2 Z2)) as a (2,2,2,2) diagonal gate
    (quantum_annealer.py:59-68)."""
    ham = (
        coupling * np.array([1, -1, -1, 1], dtype=np.complex128)
        + h1_over_deg * np.array([1, 1, -1, -1], dtype=np.complex128)
        + h2_over_deg * np.array([1, -1, 1, -1], dtype=np.complex128)
    )
    return np.diag(np.exp(-1j * tau * ham)).reshape((2, 2, 2, 2))


def q1_mixing_gate(tau: float) -> np.ndarray:
    """exp(-i tau X) (quantum_annealer.py:72-84)."""
    return np.array([[np.cos(tau), -1j * np.sin(tau)], [-1j * np.sin(tau), np.cos(tau)]], dtype=np.complex128)


def scheduler(total_time_step_size: float, schedule, steps_number: int):
    """scheduler.py:7-14: yields (mixing_time, coupling_time)."""
    for i in range(steps_number):
        f = schedule(i / (steps_number - 1))
        yield total_time_step_size * f, total_time_step_size * (1 - f)


def eval_energy(pairs: np.ndarray, couplings: np.ndarray, fields: np.ndarray, config: np.ndarray) -> float:
    """energy_evaluation.py:8-16: E(s) = -sum h s - sum J s_i s_j."""
    return float(-(fields @ config) - (config[pairs[:, 0]] * config[pairs[:, 1]]) @ couplings)


def kicked_ising_gates(theta: float):
    """RZZ(-pi/2) and RX(theta) of examples/ibm_eagle_processor.py:97-118."""
    rzz = np.diag(np.exp(np.array([1j, -1j, -1j, 1j]) * np.pi / 4)).reshape((2, 2, 2, 2))
    rx = np.array(
        [[np.cos(theta / 2), -1j * np.sin(theta / 2)], [-1j * np.sin(theta / 2), np.cos(theta / 2)]],
        dtype=np.complex128,
    )
    return rzz, rx
