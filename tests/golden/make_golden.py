"""Generates tests/golden/tensor_ops_golden.npz and tests/golden/maps_golden.npz:
inputs and outputs of the reference's own hot-path functions
(dequantizer/src/tensor_ops.py of LuchnikovI/dequantizer) and of its maps
(dequantizer/src/mappings) on deterministic graphs, for pinning the oracle.

JAX is not installed where this runs and cannot be, so the reference module
is imported under a minimal stand-in package named ``jax``: ``jax.numpy``
forwards to numpy, ``jax.scipy.special.entr`` is scipy's and ``jax.Array`` is
a type name only. Every call the module makes (tensordot, transpose,
linalg.eigh / svd / qr, norm, trace, sqrt, cumsum, finfo, newaxis, entr)
exists with the same meaning in numpy / scipy. JAX arrays are immutable:
``x *= y`` rebinds ``x`` to a new array. numpy would write into the array
instead, and the reference relies on the JAX meaning (``up_part = tensor;
up_part *= ...`` in vidal_dist must leave ``tensor`` alone), so every array
the stand-in hands out is an ndarray subclass whose in-place operators
return new arrays (and whose ``x.at[i].set(v)`` returns an updated copy, as
in JAX). The module is the reference's source as it is.

Usage: python tests/golden/make_golden.py <path to the reference checkout>
"""

import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


JNP_SHIM = """
import types as _types
import numpy as _np


class JArray(_np.ndarray):
    # in-place operators rebind, as for immutable JAX arrays
    def __iadd__(self, o):
        return _np.add(self, o)

    def __isub__(self, o):
        return _np.subtract(self, o)

    def __imul__(self, o):
        return _np.multiply(self, o)

    def __itruediv__(self, o):
        return _np.true_divide(self, o)

    def __ipow__(self, o):
        return _np.power(self, o)

    def swapaxes(self, *args, axis1=None, axis2=None):
        # JAX's method also takes its axes by keyword
        if args:
            return _np.ndarray.swapaxes(self, *args)
        return _np.ndarray.swapaxes(self, axis1, axis2)

    @property
    def at(self):
        # x.at[idx].set(v): a copy of x with x[idx] = v (JAX's functional update)
        return _At(self)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self._arr, idx)


class _AtIndex:
    def __init__(self, arr, idx):
        self._arr, self._idx = arr, idx

    def set(self, value):
        new = _np.array(self._arr, copy=True).view(JArray)
        new[self._idx] = value
        return new


def wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    if isinstance(x, tuple):
        return tuple(wrap(y) for y in x)
    if isinstance(x, list):
        return [wrap(y) for y in x]
    return x


def _wrapped(fn):
    def call(*a, **k):
        return wrap(fn(*a, **k))
    return call


class _Module:
    def __init__(self, mod):
        self._mod = mod

    def __getattr__(self, name):
        obj = getattr(self._mod, name)
        if isinstance(obj, _types.ModuleType):
            return _Module(obj)
        if callable(obj) and not isinstance(obj, type):  # functions, ufuncs, array-function dispatchers
            return _wrapped(obj)
        return obj


linalg = _Module(_np.linalg)
newaxis = None
complex_ = _np.complex128  # JAX's aliases under 64-bit mode
float_ = _np.float64


def __getattr__(name):
    return getattr(_Module(_np), name)
"""


# The package imports jit (maps are plain functions here), jax.config, the
# PRNG (never called: every input below is given explicitly) and
# lax.dynamic_slice (TensorGraph.truncate).
JAX_SHIM = """
Array = object


def jit(f, *args, **kwargs):
    return f


class _Config:
    def update(self, *args, **kwargs):
        pass


config = _Config()
"""

# The PRNG stand-in reproduces the draws of this package's oracle emulator:
# a key holds numpy's default_rng(seed); split() returns the key and its next
# 31-bit integer (one per Vidal canonicalisation); normal(subkey, shape) is
# default_rng(subkey).standard_normal(shape), uniform(subkey, shape) is
# default_rng(subkey).uniform(size=shape). The JAX PRNG stream itself is
# not reproduced (nothing here depends on it but the choice of start).
RANDOM_SHIM = """
import numpy as _np


class _Key:
    def __init__(self, seed):
        self.rng = _np.random.default_rng(int(seed))


def PRNGKey(seed):
    return _Key(seed)


def split(key, num=2):
    if not isinstance(key, _Key) or num != 2:
        raise RuntimeError("split(key) of a PRNGKey only")
    return key, int(key.rng.integers(0, 2**31 - 1))


def normal(key, shape):
    from jax.numpy import wrap

    if isinstance(key, _Key):
        raise RuntimeError("normal() of a split subkey only")
    return wrap(_np.random.default_rng(int(key)).standard_normal(shape))


def uniform(key, shape):
    from jax.numpy import wrap

    if isinstance(key, _Key):
        raise RuntimeError("uniform() of a split subkey only")
    return wrap(_np.random.default_rng(int(key)).uniform(size=shape))


def _unavailable(*args, **kwargs):
    raise RuntimeError("not available under the stand-in")


randint = _unavailable
"""

LAX_SHIM = """
def dynamic_slice(operand, start_indices, slice_sizes):
    return operand[tuple(slice(int(s), int(s) + int(n)) for s, n in zip(start_indices, slice_sizes))]
"""


def load_reference(ref_root):
    shim = tempfile.mkdtemp()
    os.makedirs(os.path.join(shim, "jax", "numpy"))
    os.makedirs(os.path.join(shim, "jax", "scipy"))
    with open(os.path.join(shim, "jax", "__init__.py"), "w") as f:
        f.write(JAX_SHIM)
    with open(os.path.join(shim, "jax", "random.py"), "w") as f:
        f.write(RANDOM_SHIM)
    with open(os.path.join(shim, "jax", "lax.py"), "w") as f:
        f.write(LAX_SHIM)
    with open(os.path.join(shim, "jax", "numpy", "__init__.py"), "w") as f:
        f.write(JNP_SHIM)
    with open(os.path.join(shim, "jax", "scipy", "__init__.py"), "w") as f:
        f.write("")
    with open(os.path.join(shim, "jax", "scipy", "special.py"), "w") as f:
        f.write("from scipy.special import entr\n")
    sys.path.insert(0, shim)
    path = os.path.join(ref_root, "dequantizer", "src", "tensor_ops.py")
    spec = importlib.util.spec_from_file_location("reference_tensor_ops", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def crandn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def psd(rng, n, rank=None):
    a = crandn(rng, n, rank or n)
    m = a @ a.conj().T
    return m / np.trace(m).real


def unitary(rng, n):
    q, r = np.linalg.qr(crandn(rng, n, n))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def cp(x):
    """Inputs for a reference call: copies, as the stand-in's immutable-semantics arrays."""
    import jax.numpy as jnp_shim

    return jnp_shim.wrap([np.array(y, copy=True) for y in x] if isinstance(x, list) else np.array(x, copy=True))


def main(ref_root):
    R = load_reference(ref_root)
    rng = np.random.default_rng(20261203)
    out = {}

    import jax.numpy as jnp_shim

    def put(case, name, v):
        if isinstance(v, (list, tuple)):
            for i, x in enumerate(v):
                out[f"{case}/{name}{i}"] = np.array(np.asarray(x))
            out[f"{case}/{name}_n"] = np.array(len(v))
        else:
            out[f"{case}/{name}"] = np.array(np.asarray(v))

    # pass_through_node (tensor_ops.py:36-60)
    for case, shape in [("ptn_k2", (3, 4, 2)), ("ptn_k3", (2, 3, 4, 2)), ("ptn_k4", (2, 3, 2, 2, 2)),
                        ("ptn_k3_d3", (2, 2, 3, 3))]:
        t = crandn(rng, *shape)
        msgs = [psd(rng, d) for d in shape[:-1]]
        put(case, "tensor", t)
        put(case, "msg", msgs)
        put(case, "out", R.pass_through_node(cp(t), cp(msgs)))
    # edge_svd (tensor_ops.py:108-130), full rank and rank deficient
    for case, ranks in [("esvd_full", (None, None)), ("esvd_def", (2, 3))]:
        ms = [psd(rng, 4, ranks[0]), psd(rng, 4, ranks[1])]
        orth, lam = R.edge_svd(cp(ms), 1e-10)
        put(case, "msg", ms)
        put(case, "orth", orth)
        put(case, "lam", lam)
    # absorb_by_node (tensor_ops.py:88-93)
    t = crandn(rng, 2, 3, 4, 2)
    mats = [crandn(rng, d, d) for d in (2, 3, 4)]
    put("abs_k3", "tensor", t)
    put("abs_k3", "mat", mats)
    put("abs_k3", "out", R.absorb_by_node(cp(t), cp(mats)))
    # vidal_dist (tensor_ops.py:143-175) and canonicalize (tensor_ops.py:189-199)
    t = crandn(rng, 2, 3, 4, 2)
    lams = [np.array([0.8, 0.6]), np.array([0.9, 0.4, 1e-12]), np.abs(rng.standard_normal(4)) + 0.1]
    put("vd_k3", "tensor", t)
    put("vd_k3", "lam", lams)
    put("vd_k3", "out", R.vidal_dist(cp(t), cp(lams), 1e-10))
    put("can_k3", "out", R.canonicalize(cp(t), cp(lams), 1e-10))
    # _decompose_gate (tensor_ops.py:202-218)
    cnot = np.eye(4, dtype=complex)[[0, 1, 3, 2]].reshape(2, 2, 2, 2)
    zz = np.diag(np.exp(1j * np.array([0.3, -0.3, -0.3, 0.3]))).reshape(2, 2, 2, 2)
    rnd = unitary(rng, 4).reshape(2, 2, 2, 2)
    for case, gate in [("dg_cnot", cnot), ("dg_zz", zz), ("dg_rand", rnd)]:
        h1, h2 = R._decompose_gate(cp(gate), 1e-10)
        put(case, "gate", gate)
        put(case, "half", [h1, h2])
    h1, h2 = R._decompose_gate(cp(rnd), 1e-10)
    # _apply_half_gate (tensor_ops.py:221-237)
    t = crandn(rng, 2, 3, 2)
    put("ahg", "tensor", t)
    put("ahg", "out", R._apply_half_gate(cp(t), cp(h1), 1))
    # simple_update (tensor_ops.py:318-389): bond 4 between t1's bond 2 and t2's bond 0
    t1, t2 = crandn(rng, 2, 3, 4, 2), crandn(rng, 4, 3, 2)
    shared = np.sort(np.abs(rng.standard_normal(4)))[::-1] + 0.05
    lam1 = [np.abs(rng.standard_normal(2)) + 0.1, np.abs(rng.standard_normal(3)) + 0.1, shared]
    lam2 = [shared, np.abs(rng.standard_normal(3)) + 0.1]
    # the production shapes: a degree-3 node with bonds of dimension 16 (the
    # mixed-precision benchmark) and a simple update between degree-3 nodes
    # with bonds of dimension 8 under a rank cap of 8 (batched annealing)
    rng16 = np.random.default_rng(16)
    t = crandn(rng16, 16, 16, 16, 2) / 64
    msgs = [psd(rng16, 16) for _ in range(3)]
    put("ptn_k3_chi16", "tensor", t)
    put("ptn_k3_chi16", "msg", msgs)
    put("ptn_k3_chi16", "out", R.pass_through_node(cp(t), cp(msgs)))
    t8a, t8b = crandn(rng16, 8, 8, 8, 2), crandn(rng16, 8, 8, 8, 2)
    sh8 = np.sort(np.abs(rng16.standard_normal(8)))[::-1] + 0.01
    l8a = [np.abs(rng16.standard_normal(8)) + 0.01, np.abs(rng16.standard_normal(8)) + 0.01, sh8]
    l8b = [sh8, np.abs(rng16.standard_normal(8)) + 0.01, np.abs(rng16.standard_normal(8)) + 0.01]
    res = R.simple_update(cp(t8a), cp(t8b), cp(l8a), cp(l8b), cp(h1), cp(h2), 2, 0, 1e-10, None, 8)
    put("su_chi8", "t", [t8a, t8b])
    put("su_chi8", "lam1", l8a)
    put("su_chi8", "lam2", l8b)
    put("su_chi8", "half", [h1, h2])
    put("su_chi8", "out", [res[0], res[1], res[2], np.array(res[3]), np.array(res[4])])
    for case, acc, rank in [("su_acc", 1e-2, None), ("su_rank", None, 3)]:
        res = R.simple_update(cp(t1), cp(t2), cp(lam1), cp(lam2), cp(h1), cp(h2), 2, 0, 1e-10, acc, rank)
        put(case, "t", [t1, t2])
        put(case, "lam1", lam1)
        put(case, "lam2", lam2)
        put(case, "half", [h1, h2])
        put(case, "out", [res[0], res[1], res[2], np.array(res[3]), np.array(res[4])])
    np.savez_compressed(os.path.join(HERE, "tensor_ops_golden.npz"), **out)
    print(f"{len(out)} arrays written")
    maps_golden(ref_root)


MAP_GRAPHS = {  # name -> (constructor name, arguments): the same constructors exist in dequantizer_b200.graph
    "lat232": ("get_nd_lattice", ([2, 3, 2], 2, 2, True)),
    "lat222_chi3": ("get_nd_lattice", ([2, 2, 2], 2, 3, True)),
    "hexinf": ("get_heavy_hex_ibm_eagle_lattice_infinite", ()),
}


def maps_golden(ref_root):
    """Inputs and outputs of the reference's maps (dequantizer/src/mappings)
    on deterministic graphs, keyed by graph, quantity and repr of the element
    or message ID."""
    sys.path.insert(0, ref_root)
    import jax.numpy as jnp_shim

    import dequantizer as D

    rng = np.random.default_rng(7)
    out = {}
    for gname, (ctor, args) in MAP_GRAPHS.items():
        graph = getattr(D, ctor)(*args)
        for ordering in ("dfs", "bfs"):
            trav = list(graph.get_traversal_iterator(ordering=ordering))
            out[f"{gname}/traversal_{ordering}"] = np.array([repr(el.id) for el in trav])
        trav = list(graph.get_traversal_iterator())

        def tensor_init(node):
            return jnp_shim.wrap(crandn(rng, *node.bond_shape, node.dimension))

        def message_init(md):
            d = md[0].dimension if isinstance(md[0], D.Edge) else md[1].dimension
            return jnp_shim.wrap(psd(rng, d))

        tensors = graph.init_tensors(tensor_init)
        messages = graph.init_messages(message_init)

        def put(what, d):
            """One dict as three arrays: repr keys, the shapes, the flat values.
            Every array the reference returned must carry the stand-in's
            immutable semantics (a plain ndarray would mean an in-place operator
            could have written into an input)."""
            assert all(isinstance(v, jnp_shim.JArray) for v in d.values()), what
            arrs = [np.array(np.asarray(v)) for v in d.values()]
            out[f"{gname}/{what}/keys"] = np.array([repr(k) for k in d])
            out[f"{gname}/{what}/ndim"] = np.array([a.ndim for a in arrs])
            out[f"{gname}/{what}/dims"] = np.array([n for a in arrs for n in a.shape], dtype=np.int64)
            out[f"{gname}/{what}/data"] = np.concatenate([a.ravel().astype(np.complex128) for a in arrs])

        put("tensors", tensors)
        put("messages", messages)
        for ordering in ("dfs", "bfs"):
            t_ord = list(graph.get_traversal_iterator(ordering=ordering))
            for sync in (False, True):
                bp = D.get_belief_propagation_map(t_ord, sync)
                m = messages
                for _ in range(2):
                    m = bp(tensors, m)
                put(f"bp2_{ordering}_{'sync' if sync else 'async'}", m)
        bp = D.get_belief_propagation_map(trav)
        m = messages
        for _ in range(30):
            m = bp(tensors, m)
        put("messages_30", m)
        m_next = bp(tensors, m)
        out[f"{gname}/frob_30_31"] = np.array(float(D.messages_frob_distance(m, m_next)))
        g_t, lam = D.get_vidal_gauge_fixing_map(trav, 1e-10)(tensors, m)
        put("vidal_tensors", g_t)
        put("vidal_lambdas", lam)
        out[f"{gname}/vidal_distance"] = np.array(float(D.get_vidal_gauge_distance_map(trav, 1e-10)(g_t, lam)))
        put("symmetric_tensors", D.get_symmetric_gauge_fixing_map(trav, 1e-10)(g_t, lam))
        put("lambda_messages", D.lambdas2messages(lam))
        rho = {el.id: D.get_one_side_density_matrix(el, tensors, m) for el in trav if isinstance(el, D.Node)}
        put("density", rho)
        if gname == "lat232":
            graph_ops(D, graph, out, put, g_t, lam, rng)
    emulator(D, out)
    exact_emulator(D, out)
    annealer(ref_root, out)
    np.savez_compressed(os.path.join(HERE, "maps_golden.npz"), **out)
    print(f"{len(out)} map arrays written")


def annealer(ref_root, out):
    """run_quantum_annealer of the reference's annealing example
    (examples/quantum_annealing/quantum_annealing/src/quantum_annealer.py:90-152,
    first-order Trotter steps from get_scheduler, scheduler.py:7-14) on a
    10-spin random 3-regular instance with J = +-1 and random fields: key 7,
    bond <= 4, a regauge per layer of couplings, BP accuracy 1e-7, six steps of
    size 0.2 with f(t) = 1 - t. Recorded: the instance, every step's density
    matrices, truncation errors, entropies and Vidal distances."""
    from jax.random import PRNGKey

    sys.path.insert(0, os.path.join(ref_root, "examples", "quantum_annealing"))
    from quantum_annealing.src.energy_function import EnergyFunction
    from quantum_annealing.src.quantum_annealer import run_quantum_annealer
    from quantum_annealing.src.scheduler import get_scheduler

    rng = np.random.default_rng(11)
    n = 10
    while True:  # pairing-model 3-regular graph without loops or repeated edges
        stubs = rng.permutation(np.repeat(np.arange(n), 3))
        pairs = np.sort(stubs.reshape(-1, 2), axis=1)
        if np.all(pairs[:, 0] != pairs[:, 1]) and len({tuple(p) for p in pairs}) == len(pairs):
            break
    amps = rng.choice([-1.0, 1.0], size=len(pairs))
    fields = 0.5 * rng.standard_normal(n)
    out["anneal/pairs"], out["anneal/amps"], out["anneal/fields"] = pairs, amps, fields
    energy = EnergyFunction(amps, pairs, fields)
    res = run_quantum_annealer(energy, get_scheduler(0.2, lambda t: 1 - t, 6), PRNGKey(7), 4, len(pairs), 1e-7,
                               100, False, "dfs", False, True)
    out["anneal/rho_history"] = np.stack([np.asarray(r) for r in res.density_matrices_history])
    out["anneal/rho"] = np.asarray(res.density_matrices)
    out["anneal/truncation_errors"] = np.asarray(res.truncation_errors, dtype=float)
    out["anneal/entropies"] = np.asarray(res.entropies, dtype=float)
    out["anneal/after_regauging"] = np.array([float(x) for x in np.asarray(res.vidal_distances_after_regauging)])


def exact_emulator(D, out):
    """ExactQuantumEmulator (quantum_emulator/exact_quantum_emulator.py:11-147)
    on a 2x3 lattice (6 qubits): a product state, two layers of seeded random
    one-qubit unitaries on every qubit and two-qubit unitaries on every edge,
    then measurements of two qubits with key 5. Recorded: the gates, every
    qubit's density matrix after each layer, the state before the
    measurements, the outcomes and the state after them."""
    import jax.numpy as jnp_shim
    from jax.random import PRNGKey

    from dequantizer.src.quantum_emulator.exact_quantum_emulator import ExactQuantumEmulator

    rng = np.random.default_rng(21)
    lat = D.get_nd_lattice([2, 3], 2, 2, True)
    trav = list(lat.get_traversal_iterator())
    nodes = [el.id for el in trav if isinstance(el, D.Node)]
    edges = [el.id for el in trav if isinstance(el, D.Edge)]
    em = ExactQuantumEmulator(lat, PRNGKey(5))
    bits = {n: int(i % 2) for i, n in enumerate(nodes)}
    em.set_to_product_state(bits)
    out["exact/nodes"] = np.array([repr(n) for n in nodes])
    out["exact/bits"] = np.array([bits[n] for n in nodes])
    for layer in range(2):
        g1 = [unitary(rng, 2) for _ in nodes]
        g2 = [unitary(rng, 4).reshape(2, 2, 2, 2) for _ in edges]
        out[f"exact/g1_{layer}"], out[f"exact/g2_{layer}"] = np.stack(g1), np.stack(g2)
        for n, g in zip(nodes, g1):
            em.apply_q1(jnp_shim.wrap(g), n)
        for e, g in zip(edges, g2):
            em.apply_q2(jnp_shim.wrap(g), e[0], e[1])
        out[f"exact/rho_{layer}"] = np.stack([np.asarray(em.dens_q1(n)) for n in nodes])
    out["exact/measured"] = np.array([0, 3])
    out["exact/outcomes"] = np.array([int(em.measure(nodes[i])) for i in (0, 3)])
    out["exact/rho_after"] = np.stack([np.asarray(em.dens_q1(n)) for n in nodes])


def emulator(D, out):
    """BPQuantumEmulator (bp_quantum_emulator.py:50-300) on the infinite
    heavy-hex cell: key 42, bond dimension <= 4, regauge after every layer of
    two-site gates (BP accuracy 1e-7, at most 100 iterations), three layers
    of RX(0.8) on every qubit and RZZ(-pi/2) on every edge in traversal order.
    Then two measurements (samples from the stand-in PRNG, re-canonicalisation
    after each). Recorded: every qubit's density matrix after each layer and
    after the measurements, the outcomes, and the emulator's truncation
    errors, entropies and Vidal distances."""
    import jax.numpy as jnp_shim
    from jax.random import PRNGKey

    lat = D.get_heavy_hex_ibm_eagle_lattice_infinite()
    trav = list(lat.get_traversal_iterator())
    em = D.BPQuantumEmulator(lat, PRNGKey(42), 4, lat.edges_number, 1e-7, 100)
    rzz = jnp_shim.wrap(np.diag(np.exp(np.array([1j, -1j, -1j, 1j]) * np.pi / 4)).reshape(2, 2, 2, 2))
    rx = jnp_shim.wrap(np.array([[np.cos(0.4), -1j * np.sin(0.4)], [-1j * np.sin(0.4), np.cos(0.4)]]))
    nodes = [el.id for el in trav if isinstance(el, D.Node)]
    out["emu/nodes"] = np.array([repr(n) for n in nodes])
    for layer in range(3):
        for n in nodes:
            em.apply_q1(rx, n)
        for el in trav:
            if isinstance(el, D.Edge):
                em.apply_q2(rzz, *el.id)
        out[f"emu/rho_{layer}"] = np.stack([np.asarray(em.dens_q1(n)) for n in nodes])
    out["emu/measured"] = np.array([0, 2])
    out["emu/outcomes"] = np.array([int(em.measure(nodes[i])) for i in (0, 2)])
    out["emu/rho_after_measure"] = np.stack([np.asarray(em.dens_q1(n)) for n in nodes])
    out["emu/truncation_errors"] = np.array([float(x) for x in em.truncation_errors])
    out["emu/entropies"] = np.array([float(x) for x in em.entropies])
    out["emu/after_regauging"] = np.array([float(x) for x in np.asarray(em.after_regauging_vidal_distances)])
    out["emu/truncated_affected"] = np.array([float(x) for x in np.asarray(em.truncated_affected_vidal_distances)])


def graph_ops(D, graph, out, put, tensors, lambdas, rng):
    """TensorGraph.apply1 / apply2_to_vidal_canonical / truncate / apply2
    (tensor_graph.py:235-446) from the lattice's Vidal form; the gate
    methods also change the graph's bond dimensions, recorded after each step."""
    import jax.numpy as jnp_shim

    edges = [el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, D.Edge)]
    rx = jnp_shim.wrap(np.array([[np.cos(0.3), -1j * np.sin(0.3)], [-1j * np.sin(0.3), np.cos(0.3)]]))
    cnot = jnp_shim.wrap(np.eye(4, dtype=complex)[[0, 1, 3, 2]].reshape(2, 2, 2, 2))
    zz = jnp_shim.wrap(np.diag(np.exp(1j * np.array([0.3, -0.3, -0.3, 0.3]))).reshape(2, 2, 2, 2))
    rnd = jnp_shim.wrap(unitary(rng, 4).reshape(2, 2, 2, 2))
    out["ops/gate_rnd"] = np.array(np.asarray(rnd))
    tensors, lambdas = dict(tensors), dict(lambdas)
    first = next(el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, D.Node))
    tensors = graph.apply1(first.id, tensors, rx)
    put("ops/after_apply1", tensors)
    steps = [(cnot, edges[0], None, 3), (rnd, edges[1], 1e-3, None), (zz, edges[2], None, None)]
    for i, (gate, edge, acc, rank) in enumerate(steps):
        a, b = edge.id
        tensors, lambdas, err, ent = graph.apply2_to_vidal_canonical(a, b, tensors, lambdas, gate, 1e-10, acc, rank)
        put(f"ops/step{i}_tensors", tensors)
        put(f"ops/step{i}_lambdas", lambdas)
        out[f"ops/step{i}_err"] = np.array(float(err))
        out[f"ops/step{i}_entropy"] = np.array(float(ent))
        out[f"ops/step{i}_edge_dims"] = np.array([e.dimension for e in edges])
    tensors, lambdas = graph.truncate(tensors, lambdas, 1e-2)
    put("ops/truncated_tensors", tensors)
    put("ops/truncated_lambdas", lambdas)
    out["ops/truncated_edge_dims"] = np.array([e.dimension for e in edges])
    a, b = edges[3].id
    tensors = graph.apply2(a, b, tensors, rnd, 1e-10)
    put("ops/apply2_tensors", tensors)
    out["ops/apply2_edge_dims"] = np.array([e.dimension for e in edges])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to a checkout of LuchnikovI/dequantizer>")
    main(sys.argv[1])
