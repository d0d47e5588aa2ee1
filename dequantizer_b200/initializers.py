"""Host-side initializers for node tensors and messages.

They return numpy complex128 arrays; ``TensorGraph.init_tensors`` /
``init_messages`` move them to the GPU. Randomness uses numpy's PCG64 seeded
by an integer ``key`` (JAX's threefry stream cannot be reproduced without
JAX). As in the reference, a random initializer re-seeds on every call, so all
tensors (messages) of the same shape come out identical
(graph/tensor_initializers.py:28, graph/message_initializer.py:22).

Reference counterparts:
* get_tensor_random_normal_initializer  -- graph/tensor_initializers.py:25-32
* get_tensor_std_state_initializer      -- graph/tensor_initializers.py:43-49
* get_tensor_bloated_ghz_initializer    -- graph/tensor_initializers.py:61-79
* get_potts_initializer                 -- graph/tensor_initializers.py:93-138
* get_message_random_nonnegative_initializer -- graph/message_initializer.py:14-26
"""

from typing import Callable

import numpy as np

from .graph import Edge, MessageDir, Node


def _gen_ghz_core(phys_dimension: int, modes_number: int) -> np.ndarray:
    """GHZ tensor: ones on the main diagonal of a ``modes_number``-way cube."""
    if phys_dimension == 1:
        return np.ones(modes_number * (1,), dtype=np.complex128)
    core = np.zeros(modes_number * (phys_dimension,), dtype=np.complex128)
    for i in range(phys_dimension):
        core[modes_number * (i,)] = 1.0
    return core


def _complex_normal(key: int, shape) -> np.ndarray:
    z = np.random.default_rng(key).standard_normal(tuple(shape) + (2,))
    return z[..., 0] + 1j * z[..., 1]


def get_tensor_random_normal_initializer(key: int) -> Callable[[Node], np.ndarray]:
    def initializer(node: Node) -> np.ndarray:
        return _complex_normal(key, (*node.bond_shape, node.dimension))

    return initializer


def get_tensor_std_state_initializer() -> Callable[[Node], np.ndarray]:
    """Product state |0...0> with all bonds of dimension 1."""

    def initializer(node: Node) -> np.ndarray:
        t = np.zeros(node.degree * (1,) + (node.dimension,), dtype=np.complex128)
        t[..., 0] = 1.0
        return t

    return initializer


def get_tensor_bloated_ghz_initializer(key: int) -> Callable[[Node], np.ndarray]:
    """GHZ cores whose bonds are isometrically embedded into larger bond
    dimensions; the isometry for a given (bond, phys) shape is fixed by ``key``."""

    def initializer(node: Node) -> np.ndarray:
        core = _gen_ghz_core(node.dimension, node.degree + 1)
        for bond_dim in reversed(node.bond_shape):
            if bond_dim < node.dimension:
                raise ValueError(
                    "For GHZ initializer all bond indices must be >= the physical index, "
                    f"got one of the bond dimensions {bond_dim} and physical dimension {node.dimension}."
                )
            bloater = np.random.default_rng(key).standard_normal((bond_dim, node.dimension)).astype(np.complex128)
            bloater, _ = np.linalg.qr(bloater)
            core = np.tensordot(bloater, core, axes=[1, -1])
        return core

    return initializer


def get_potts_initializer(two_spin_factor, single_spin_factor) -> Callable[[Node], np.ndarray]:
    """Square-root Potts/Ising tensors: contracting the network with itself
    gives the partition function. With W = sqrt(two_spin_factor) = S^T S,
    T[a_1..a_k, s] = sqrt(h[s]) prod_e S[a_e, s]."""
    two = np.asarray(two_spin_factor)
    one = np.asarray(single_spin_factor)
    if one.ndim != 1:
        raise ValueError("A single spin factor must be a tensor of rank 1.")
    if two.ndim != 2:
        raise ValueError("A two spin factor must be a tensor of rank 2.")
    if two.shape[0] != two.shape[1]:
        raise ValueError("A two spin facto must have the same dimension per index.")
    if two.shape[0] != one.shape[0]:
        raise ValueError("Index dimension of a single spin factor must match the dimension of two factor indices.")
    phys_dim = one.shape[0]
    one_sqrt = np.sqrt(one).astype(np.complex128)
    two_sqrt = np.sqrt(two)
    lmbd, u = np.linalg.eigh(two_sqrt)
    s_mat = (u * np.sqrt(lmbd.astype(np.complex128))[None]).T
    assert np.linalg.norm(np.tensordot(s_mat, s_mat, axes=[0, 0]) - two_sqrt) < 1e-5

    def initializer(node: Node) -> np.ndarray:
        if node.dimension != phys_dim:
            raise ValueError("Node dimension must match with the factor index dimension.")
        t = one_sqrt
        for nb in node.neighbors:
            if nb.dimension != phys_dim:
                raise ValueError("Bond dimensions of the node must match dimension of the factor indices.")
            t = t[..., None, :] * s_mat
        return t

    return initializer


def get_message_random_nonnegative_initializer(key: int) -> Callable[[MessageDir], np.ndarray]:
    """Random PSD messages A A^dagger with A complex standard normal."""

    def initializer(direction: MessageDir) -> np.ndarray:
        d = direction[0].dimension if isinstance(direction[0], Edge) else direction[1].dimension
        a = _complex_normal(key, (d, d))
        return a @ a.conj().T

    return initializer
