"""libdqz entry points as PyTorch operators, ``torch.ops.dqz.*``.

Importing this module registers one custom operator per hot-path entry point
of the C ABI (include/dqz.h). They are for code that composes the kernels
with other torch operators (``torch.library`` custom ops are opaque to
``torch.compile`` and carry their mutation annotations); the package itself
calls the library through ctypes (``dequantizer_b200._lib``) and needs no
registration.

Conventions:
* ``graph`` is the integer handle of a packed graph, ``GraphLayout.handle``
  (the address of its host-side table descriptor); the layout object must
  outlive the calls.
* Arenas are the layout's flat device tensors (complex128 or complex64 node
  tensors and messages, float64 lambdas, int32 index lists, uint8 source
  selectors); outputs are written in place and every operator returns None.
* Work runs on the current CUDA stream of the tensors' device. Scratch memory,
  where the kernel needs some, is allocated by the operator.
* The operators are registered for CUDA only: a call with CPU tensors raises,
  there is no CPU implementation. Each has a fake implementation, so tracing
  works.

Arguments are passed to the C functions by parameter name; ``PARAMS`` lists
each function's parameters in declaration order, and a CPU test checks it
against the header.
"""

import ctypes
from typing import Dict, List, Optional

import torch
from torch import Tensor

from . import _lib

# C parameter names per entry point, in declaration order (include/dqz.h)
PARAMS: Dict[str, List[str]] = {
    "dqz_bp_node_update": ["g", "tensors", "n2e_old", "e2n_old", "n2e_new", "src_sel", "halves", "n_halves",
                           "max_slice", "max_chi", "scratch", "stream"],
    "dqz_bp_node_update_k3": ["g", "chi", "precision", "tensors", "n2e_old", "e2n_old", "n2e_new", "src_sel",
                              "halves", "n_halves", "error_flag", "stream"],
    "dqz_bp_node_update_k3_umma": ["g", "tensors_bf16", "n2e_old", "e2n_old", "n2e_new", "src_sel", "nodes",
                                   "n_nodes", "error_flag", "stream"],
    "dqz_pack_bf16_umma": ["g", "tensors_c64", "tensors_bf16", "stream"],
    "dqz_bp_edge_pass": ["g", "n2e_old", "n2e_new", "edge_new", "e2n_new", "max_chi", "stream"],
    "dqz_bp_edge_pass_c64": ["g", "n2e_old", "n2e_new", "edge_new", "e2n_new", "stream"],
    "dqz_messages_distance": ["g", "n2e_a", "n2e_b", "e2n_a", "e2n_b", "partial", "out", "max_chi", "stream"],
    "dqz_vidal_edges": ["g", "n2e", "eps", "orth", "lambdas", "max_chi", "edges", "n_sel", "scratch", "stream"],
    "dqz_absorb": ["g", "tensors_in", "orth", "tensors_out", "max_size", "nodes", "n_sel", "scratch", "stream"],
    "dqz_vidal_distance": ["g", "tensors", "lambdas", "eps", "partial", "out", "max_chi", "max_slice", "halves",
                           "n_sel", "stream"],
    "dqz_symmetric_gauge": ["g", "tensors_in", "lambdas", "eps", "tensors_out", "stream"],
    "dqz_lambdas_to_messages": ["g", "lambdas", "n2e", "e2n", "max_chi", "stream"],
    "dqz_density_matrices": ["g", "tensors", "e2n", "nodes", "n_nodes", "rho", "max_size", "scratch", "stream"],
    "dqz_apply1": ["g", "tensors", "nodes", "gates", "n", "stream"],
    "dqz_simple_update": ["g", "tensors", "lambdas", "edges", "ctrl_is_first", "halves", "ranks", "n", "eps",
                          "max_rank", "max_rows", "max_cols", "err", "entropy", "scratch", "stream"],
    "dqz_bp_node_vjp": ["g", "tensors", "e2n", "n2e_cot", "e2n_cot", "t_cot", "nodes", "n_nodes", "max_size",
                        "max_chi", "scratch", "stream"],
}


# ------------------------------------------------------------------ plumbing
def _check(*tensors: Optional[Tensor]) -> None:
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise RuntimeError("torch.ops.dqz operators take CUDA tensors only")
        if t is not None and not t.is_contiguous():
            raise RuntimeError("torch.ops.dqz operators take contiguous tensors only")


def _stream(t: Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _scratch(nbytes: int, like: Tensor) -> Optional[Tensor]:
    return torch.empty(int(nbytes), dtype=torch.uint8, device=like.device) if nbytes else None


def _call(func: str, *args) -> None:
    _lib.call(func, *args)


def _run(func: str, named: Dict) -> None:
    """Calls ``func`` with ``named`` ordered by its parameter list; tensors
    become device pointers, None a null pointer, ``g`` the graph handle."""
    names = PARAMS[func]
    if set(named) != set(names):
        raise TypeError(f"{func}: arguments {sorted(named)} do not match parameters {names}")
    args = []
    for n in names:
        v = named[n]
        if n == "g":
            v = ctypes.cast(ctypes.c_void_p(int(v)), ctypes.POINTER(_lib.GraphDesc))
        elif isinstance(v, Tensor):
            v = v.data_ptr()
        args.append(v)
    _call(func, *args)


def _lib_size(func: str, *args) -> int:
    return int(getattr(_lib.lib(), func)(*args))


# ---------------------------------------------------------------- operators
IMPL: Dict = {}  # operator name -> the Python function registered as its CUDA implementation


def _op(name: str, mutates):
    def deco(fn):
        IMPL[name] = fn
        return torch.library.custom_op(f"dqz::{name}", mutates_args=mutates, device_types="cuda")(fn)

    return deco


@_op("bp_node_update", ("n2e_new",))
def bp_node_update(graph: int, tensors: Tensor, n2e_old: Tensor, e2n_old: Tensor, n2e_new: Tensor, src_sel: Tensor,
                   halves: Tensor, max_slice: int, max_chi: int) -> None:
    """tensor_ops.py:36-60 for the listed half-edges (any degree, complex128)."""
    _check(tensors, n2e_old, e2n_old, n2e_new, src_sel, halves)
    n = halves.numel()
    scratch = _scratch(_lib_size("dqz_bp_node_scratch_bytes", n, max_slice, max_chi), tensors)
    _run("dqz_bp_node_update", dict(g=graph, tensors=tensors, n2e_old=n2e_old, e2n_old=e2n_old, n2e_new=n2e_new,
                                    src_sel=src_sel, halves=halves, n_halves=n, max_slice=max_slice,
                                    max_chi=max_chi, scratch=scratch, stream=_stream(tensors)))


@_op("bp_node_update_k3", ("n2e_new", "error_flag"))
def bp_node_update_k3(graph: int, chi: int, tensors: Tensor, n2e_old: Tensor, e2n_old: Tensor, n2e_new: Tensor,
                      src_sel: Tensor, halves: Tensor, error_flag: Tensor) -> None:
    """tensor_ops.py:36-60, degree-3 nodes, bonds of dimension 8 or 16; FP64
    for complex128 arenas, FP32 for complex64."""
    _check(tensors, n2e_old, e2n_old, n2e_new, src_sel, halves, error_flag)
    precision = 64 if tensors.dtype == torch.complex128 else 32
    _run("dqz_bp_node_update_k3", dict(g=graph, chi=chi, precision=precision, tensors=tensors, n2e_old=n2e_old,
                                       e2n_old=e2n_old, n2e_new=n2e_new, src_sel=src_sel, halves=halves,
                                       n_halves=halves.numel(), error_flag=error_flag, stream=_stream(tensors)))


@_op("bp_node_update_k3_umma", ("n2e_new", "error_flag"))
def bp_node_update_k3_umma(graph: int, tensors_bf16: Tensor, n2e_old: Tensor, e2n_old: Tensor, n2e_new: Tensor,
                           src_sel: Tensor, nodes: Tensor, error_flag: Tensor) -> None:
    """tensor_ops.py:36-60, mixed precision on tcgen05 (degree 3, bond 16);
    ``tensors_bf16`` from pack_bf16_umma, messages complex64."""
    _check(tensors_bf16, n2e_old, e2n_old, n2e_new, src_sel, nodes, error_flag)
    _run("dqz_bp_node_update_k3_umma", dict(g=graph, tensors_bf16=tensors_bf16, n2e_old=n2e_old, e2n_old=e2n_old,
                                            n2e_new=n2e_new, src_sel=src_sel, nodes=nodes, n_nodes=nodes.numel(),
                                            error_flag=error_flag, stream=_stream(n2e_new)))


@_op("pack_bf16_umma", ("tensors_bf16",))
def pack_bf16_umma(graph: int, tensors_c64: Tensor, tensors_bf16: Tensor) -> None:
    """complex64 node tensors -> the BF16 core layouts of bp_node_update_k3_umma."""
    _check(tensors_c64, tensors_bf16)
    _run("dqz_pack_bf16_umma", dict(g=graph, tensors_c64=tensors_c64, tensors_bf16=tensors_bf16,
                                    stream=_stream(tensors_c64)))


@_op("bp_edge_pass", ("e2n_new",))
def bp_edge_pass(graph: int, n2e_old: Tensor, n2e_new: Tensor, edge_new: Tensor, e2n_new: Tensor,
                 max_chi: int) -> None:
    """tensor_ops.py:70-76: e2n_new[h] = (edge_new[h] ? n2e_new : n2e_old)[twin(h)]."""
    _check(n2e_old, n2e_new, edge_new, e2n_new)
    if e2n_new.dtype == torch.complex64:
        _run("dqz_bp_edge_pass_c64", dict(g=graph, n2e_old=n2e_old, n2e_new=n2e_new, edge_new=edge_new,
                                          e2n_new=e2n_new, stream=_stream(e2n_new)))
    else:
        _run("dqz_bp_edge_pass", dict(g=graph, n2e_old=n2e_old, n2e_new=n2e_new, edge_new=edge_new,
                                      e2n_new=e2n_new, max_chi=max_chi, stream=_stream(e2n_new)))


@_op("messages_distance", ("partial", "out"))
def messages_distance(graph: int, n2e_a: Tensor, n2e_b: Tensor, e2n_a: Tensor, e2n_b: Tensor, partial: Tensor,
                      out: Tensor, max_chi: int) -> None:
    """mappings/messages_distance.py:14-22 (``partial`` holds 2 x n_halves float64)."""
    _check(n2e_a, n2e_b, e2n_a, e2n_b, partial, out)
    _run("dqz_messages_distance", dict(g=graph, n2e_a=n2e_a, n2e_b=n2e_b, e2n_a=e2n_a, e2n_b=e2n_b,
                                       partial=partial, out=out, max_chi=max_chi, stream=_stream(out)))


@_op("vidal_edges", ("orth", "lambdas"))
def vidal_edges(graph: int, n2e: Tensor, eps: float, orth: Tensor, lambdas: Tensor, max_chi: int, n_edges: int,
                edges: Optional[Tensor] = None) -> None:
    """tensor_ops.py:108-130 (edge_svd) for every edge, or for ``edges``."""
    _check(n2e, orth, lambdas, edges)
    n = n_edges if edges is None else edges.numel()
    scratch = _scratch(_lib_size("dqz_vidal_edges_scratch_bytes", n, max_chi), n2e)
    _run("dqz_vidal_edges", dict(g=graph, n2e=n2e, eps=float(eps), orth=orth, lambdas=lambdas, max_chi=max_chi,
                                 edges=edges, n_sel=0 if edges is None else n, scratch=scratch,
                                 stream=_stream(n2e)))


@_op("absorb", ("tensors_out",))
def absorb(graph: int, tensors_in: Tensor, orth: Tensor, tensors_out: Tensor, max_size: int, n_nodes: int,
           nodes: Optional[Tensor] = None) -> None:
    """tensor_ops.py:88-93 (absorb_by_node) for every node, or for ``nodes``."""
    _check(tensors_in, orth, tensors_out, nodes)
    n = n_nodes if nodes is None else nodes.numel()
    scratch = _scratch(_lib_size("dqz_absorb_scratch_bytes", n, max_size), tensors_in)
    _run("dqz_absorb", dict(g=graph, tensors_in=tensors_in, orth=orth, tensors_out=tensors_out, max_size=max_size,
                            nodes=nodes, n_sel=0 if nodes is None else n, scratch=scratch,
                            stream=_stream(tensors_in)))


@_op("vidal_distance", ("partial", "out"))
def vidal_distance(graph: int, tensors: Tensor, lambdas: Tensor, eps: float, partial: Tensor, out: Tensor,
                   max_chi: int, max_slice: int, halves: Optional[Tensor] = None) -> None:
    """tensor_ops.py:143-175 per half-edge into ``partial``; ``out`` = their mean."""
    _check(tensors, lambdas, partial, out, halves)
    _run("dqz_vidal_distance", dict(g=graph, tensors=tensors, lambdas=lambdas, eps=float(eps), partial=partial,
                                    out=out, max_chi=max_chi, max_slice=max_slice, halves=halves,
                                    n_sel=0 if halves is None else halves.numel(), stream=_stream(tensors)))


@_op("symmetric_gauge", ("tensors_out",))
def symmetric_gauge(graph: int, tensors_in: Tensor, lambdas: Tensor, eps: float, tensors_out: Tensor) -> None:
    """tensor_ops.py:189-199 (canonicalize) for every node."""
    _check(tensors_in, lambdas, tensors_out)
    _run("dqz_symmetric_gauge", dict(g=graph, tensors_in=tensors_in, lambdas=lambdas, eps=float(eps),
                                     tensors_out=tensors_out, stream=_stream(tensors_in)))


@_op("lambdas_to_messages", ("n2e", "e2n"))
def lambdas_to_messages(graph: int, lambdas: Tensor, n2e: Tensor, e2n: Tensor, max_chi: int) -> None:
    """mappings/symmetric_gauge.py:50-61: diag(lambda) in both directions."""
    _check(lambdas, n2e, e2n)
    _run("dqz_lambdas_to_messages", dict(g=graph, lambdas=lambdas, n2e=n2e, e2n=e2n, max_chi=max_chi,
                                         stream=_stream(n2e)))


@_op("density_matrices", ("rho",))
def density_matrices(graph: int, tensors: Tensor, e2n: Tensor, nodes: Tensor, rho: Tensor, max_size: int) -> None:
    """mappings/density_matrix.py:16-37 for the listed nodes."""
    _check(tensors, e2n, nodes, rho)
    n = nodes.numel()
    scratch = _scratch(_lib_size("dqz_density_scratch_bytes", n, max_size), tensors)
    _run("dqz_density_matrices", dict(g=graph, tensors=tensors, e2n=e2n, nodes=nodes, n_nodes=n, rho=rho,
                                      max_size=max_size, scratch=scratch, stream=_stream(tensors)))


@_op("apply1", ("tensors",))
def apply1(graph: int, tensors: Tensor, nodes: Tensor, gates: Tensor) -> None:
    """graph/tensor_graph.py:268-275 for the listed nodes (gates d x d, padded)."""
    _check(tensors, nodes, gates)
    _run("dqz_apply1", dict(g=graph, tensors=tensors, nodes=nodes, gates=gates, n=nodes.numel(),
                            stream=_stream(tensors)))


@_op("simple_update", ("tensors", "lambdas", "err", "entropy"))
def simple_update(graph: int, tensors: Tensor, lambdas: Tensor, edges: Tensor, ctrl_is_first: Tensor,
                  halves: Tensor, ranks: Tensor, eps: float, max_rank: int, max_rows: int, max_cols: int,
                  err: Tensor, entropy: Tensor) -> None:
    """tensor_ops.py:265-389 (simple_update) for a node-disjoint batch of gates."""
    _check(tensors, lambdas, edges, ctrl_is_first, halves, ranks, err, entropy)
    n = edges.numel()
    scratch = _scratch(_lib_size("dqz_simple_update_scratch_bytes", n, max_rows, max_cols), tensors)
    _run("dqz_simple_update", dict(g=graph, tensors=tensors, lambdas=lambdas, edges=edges,
                                   ctrl_is_first=ctrl_is_first, halves=halves, ranks=ranks, n=n, eps=float(eps),
                                   max_rank=max_rank, max_rows=max_rows, max_cols=max_cols, err=err,
                                   entropy=entropy, scratch=scratch, stream=_stream(tensors)))


@_op("bp_node_vjp", ("e2n_cot", "t_cot"))
def bp_node_vjp(graph: int, tensors: Tensor, e2n: Tensor, n2e_cot: Tensor, e2n_cot: Tensor, t_cot: Tensor,
                nodes: Tensor, max_size: int, max_chi: int) -> None:
    """Reverse of tensor_ops.py:36-60 for the listed nodes (cotangents of the
    incoming messages and of the node tensors); no reference counterpart."""
    _check(tensors, e2n, n2e_cot, e2n_cot, t_cot, nodes)
    n = nodes.numel()
    scratch = _scratch(_lib_size("dqz_bp_node_vjp_scratch_bytes", n, max_size), tensors)
    _run("dqz_bp_node_vjp", dict(g=graph, tensors=tensors, e2n=e2n, n2e_cot=n2e_cot, e2n_cot=e2n_cot, t_cot=t_cot,
                                 nodes=nodes, n_nodes=n, max_size=max_size, max_chi=max_chi, scratch=scratch,
                                 stream=_stream(tensors)))


OPS = list(IMPL)


def _register_fakes() -> None:
    """Every operator writes only into its arguments: the fake implementation
    does nothing (shape propagation under tracing)."""
    for name in OPS:
        op = globals()[name]

        def fake(*args, **kwargs):
            return None

        op.register_fake(fake)


_register_fakes()
