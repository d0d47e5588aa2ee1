"""torch.ops.dqz registration and argument plumbing, on the CPU.

* every operator is registered, with its outputs annotated as mutated;
* each operator's C parameter list (PARAMS) is the one declared in include/dqz.h;
* with the library call recorded instead of made, every operator passes each
  tensor's pointer, the derived counts and the graph handle in the parameter
  of that name;
* CPU tensors are rejected (the operators have no CPU implementation).
The GPU tests exercise the same entry points through the package's own calls.
"""

import ctypes
import os
import re

import pytest
import torch

import dequantizer_b200.torch_ops as T
from dequantizer_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_params():
    h = open(os.path.join(ROOT, "include", "dqz.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|size_t|int32_t)\s+(dqz_\w+)\s*\(([^;]*?)\)\s*;", h, flags=re.S):
        names = [re.findall(r"(\w+)\s*$", p.strip())[0] for p in m.group(2).split(",") if p.strip()]
        out[m.group(1)] = names
    return out


def test_operators_registered_with_mutations():
    for name in T.OPS:
        schema = str(getattr(torch.ops.dqz, name).default._schema)
        assert schema.startswith(f"dqz::{name}(")
        assert "!)" in schema  # every operator writes into at least one argument


def test_parameter_lists_match_header():
    hp = header_params()
    for func, names in T.PARAMS.items():
        assert hp[func] == names, func


def _fake_tensors():
    """Distinct CPU tensors: their data pointers identify them in the recorded call."""
    f = {}
    for name in ["tensors", "tensors_bf16", "tensors_c64", "tensors_in", "tensors_out", "n2e_old", "e2n_old",
                 "n2e_new", "e2n_new", "n2e", "e2n", "n2e_a", "n2e_b", "e2n_a", "e2n_b", "orth", "rho", "gates",
                 "n2e_cot", "e2n_cot", "t_cot"]:
        f[name] = torch.zeros(8, dtype=torch.complex128)
    for name in ["lambdas", "partial", "out", "err", "entropy"]:
        f[name] = torch.zeros(8, dtype=torch.float64)
    for name, n in [("halves", 5), ("nodes", 3), ("edges", 4), ("ranks", 4)]:
        f[name] = torch.zeros(n, dtype=torch.int32)
    for name in ["src_sel", "edge_new", "ctrl_is_first", "error_flag"]:
        f[name] = torch.zeros(8, dtype=torch.int32)
    f["halves_gates"] = torch.zeros(8, dtype=torch.complex128)
    return f


CALLS = {  # operator -> keyword arguments (tensors by name from _fake_tensors, plus scalars)
    "bp_node_update": dict(max_slice=32, max_chi=4),
    "bp_node_update_k3": dict(chi=16),
    "bp_node_update_k3_umma": dict(),
    "pack_bf16_umma": dict(),
    "bp_edge_pass": dict(max_chi=4),
    "messages_distance": dict(max_chi=4),
    "vidal_edges": dict(eps=1e-10, max_chi=4, n_edges=7),
    "absorb": dict(max_size=64, n_nodes=6),
    "vidal_distance": dict(eps=1e-10, max_chi=4, max_slice=32),
    "symmetric_gauge": dict(eps=1e-10),
    "lambdas_to_messages": dict(max_chi=4),
    "density_matrices": dict(max_size=64),
    "apply1": dict(),
    "simple_update": dict(eps=1e-10, max_rank=8, max_rows=64, max_cols=16),
    "bp_node_vjp": dict(max_size=64, max_chi=4),
}
OPTIONAL = {"vidal_edges": "edges", "absorb": "nodes", "vidal_distance": "halves"}


@pytest.mark.parametrize("op,without_selection", [(o, False) for o in T.OPS] + [(o, True) for o in OPTIONAL])
def test_arguments_reach_the_named_parameters(op, without_selection, monkeypatch):
    f = _fake_tensors()
    recorded = []
    monkeypatch.setattr(T, "_check", lambda *a: None)
    monkeypatch.setattr(T, "_stream", lambda t: 12345)
    monkeypatch.setattr(T, "_lib_size", lambda func, *a: 0)
    monkeypatch.setattr(T, "_call", lambda func, *args: recorded.append((func, args)))
    fn = T.IMPL[op]
    code = fn.__code__
    params = code.co_varnames[:code.co_argcount]
    kwargs = dict(CALLS[op])
    desc = _lib.GraphDesc()
    handle = ctypes.addressof(desc)
    for p in params:
        if p == "graph":
            kwargs[p] = handle
        elif p not in kwargs and p in f:
            kwargs[p] = f["halves_gates"] if (op == "simple_update" and p == "halves") else f[p]
    if without_selection:
        kwargs.pop(OPTIONAL[op])
    fn(**kwargs)
    assert len(recorded) == 1
    func, args = recorded[0]
    names = T.PARAMS[func]
    got = dict(zip(names, args))
    assert ctypes.cast(got["g"], ctypes.c_void_p).value == handle
    assert got["stream"] == 12345
    for n in names:
        if n in kwargs and isinstance(kwargs[n], torch.Tensor):
            assert got[n] == kwargs[n].data_ptr(), (func, n)
        elif n in kwargs and n != "graph":
            assert got[n] == kwargs[n], (func, n)
    if "n_halves" in got:
        assert got["n_halves"] == kwargs["halves"].numel()
    if "n_nodes" in got:
        assert got["n_nodes"] == kwargs["nodes"].numel()
    if func in ("dqz_apply1",):
        assert got["n"] == kwargs["nodes"].numel()
    if func == "dqz_simple_update":
        assert got["n"] == kwargs["edges"].numel()
    if "n_sel" in got:
        sel = {"dqz_vidal_edges": "edges", "dqz_absorb": "nodes", "dqz_vidal_distance": "halves"}[func]
        assert got["n_sel"] == (0 if kwargs.get(sel) is None else kwargs[sel].numel())
        assert got[sel] is None or got[sel] == kwargs[sel].data_ptr()
    if func == "dqz_bp_node_update_k3":
        assert got["precision"] == 64


def test_cpu_tensors_are_rejected():
    x = torch.zeros(4, dtype=torch.complex128)
    with pytest.raises((NotImplementedError, RuntimeError)):
        torch.ops.dqz.apply1(0, x, torch.zeros(1, dtype=torch.int32), x)
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        T.IMPL["apply1"](0, x, torch.zeros(1, dtype=torch.int32), x)


def test_every_operator_traces_with_fake_tensors():
    """Under FakeTensorMode (what torch.compile and export trace with) every
    operator accepts fake CUDA tensors and runs its fake implementation;
    nothing executes and no GPU is needed."""
    from torch._subclasses.fake_tensor import FakeTensorMode

    real = _fake_tensors()
    with FakeTensorMode():
        fakes = {k: torch.empty(v.shape, dtype=v.dtype, device="cuda") for k, v in real.items()}
        for op in T.OPS:
            fn = T.IMPL[op]
            code = fn.__code__
            kwargs = dict(CALLS[op])
            for p in code.co_varnames[:code.co_argcount]:
                if p == "graph":
                    kwargs[p] = 0
                elif p not in kwargs and p in fakes:
                    kwargs[p] = fakes["halves_gates"] if (op == "simple_update" and p == "halves") else fakes[p]
            assert getattr(torch.ops.dqz, op)(**kwargs) is None
