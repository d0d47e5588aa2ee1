"""B200-native graph-tensor-network hot path: belief propagation, Vidal
canonicalisation and simple-update gate application, behind the public API of
LuchnikovI/dequantizer (dequantizer/__init__.py:5-29).

All numerics run in libdqz.so (hand-written sm_100a CUDA kernels behind a C
ABI, include/dqz.h); PyTorch provides device memory and the current stream.
"""

from .graph import (
    Edge,
    EdgeID,
    Element,
    MessageID,
    Node,
    NodeID,
    TensorGraph,
    get_heavy_hex_ibm_eagle_lattice,
    get_heavy_hex_ibm_eagle_lattice_infinite,
    get_nd_lattice,
    get_random_regular_graph,
    get_random_tree_tensor_graph,
    greedy_edge_coloring,
)
from .initializers import (
    get_message_random_nonnegative_initializer,
    get_potts_initializer,
    get_tensor_bloated_ghz_initializer,
    get_tensor_random_normal_initializer,
    get_tensor_std_state_initializer,
)
from .maps import (
    get_belief_propagation_map,
    get_one_side_density_matrix,
    get_symmetric_gauge_fixing_map,
    get_vidal_gauge_distance_map,
    get_vidal_gauge_fixing_map,
    lambdas2messages,
    messages_frob_distance,
)
from . import tensor_graph_ops as _tgo

_tgo.install()

from .emulator import BPQuantumEmulator  # noqa: E402

__all__ = [
    "TensorGraph", "NodeID", "EdgeID", "Node", "Edge", "Element", "MessageID",
    "get_nd_lattice", "get_random_tree_tensor_graph", "get_tensor_std_state_initializer",
    "get_potts_initializer", "get_message_random_nonnegative_initializer",
    "get_heavy_hex_ibm_eagle_lattice", "get_heavy_hex_ibm_eagle_lattice_infinite",
    "get_belief_propagation_map", "get_vidal_gauge_fixing_map", "get_vidal_gauge_distance_map",
    "get_symmetric_gauge_fixing_map", "lambdas2messages", "messages_frob_distance",
    "get_one_side_density_matrix", "BPQuantumEmulator",
    "get_tensor_bloated_ghz_initializer", "get_tensor_random_normal_initializer",
    "get_random_regular_graph", "greedy_edge_coloring",
]
