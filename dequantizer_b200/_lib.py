"""ctypes binding of libdqz.so (the C ABI declared in include/dqz.h).

The product has no CPU path: every numerical entry point needs CUDA tensors
and the compiled library. ``lib()`` raises ``RuntimeError`` when the library
is missing and ``require_cuda`` raises when a tensor is not on a CUDA device.
"""

import ctypes
import os
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdqz.so")

DQZ_OK = 0
DQZ_ERR_ARG = 1
DQZ_ERR_UNSUPPORTED = 2
DQZ_ERR_CUDA = 3
DQZ_ERR_NOT_CONVERGED = 4
DQZ_ERR_NONFINITE = 5

MAX_DEGREE = 8
MAX_CHI = 64
MAX_PHYS = 8

SRC_E2N_OLD = 0
SRC_N2E_OLD = 1
SRC_N2E_NEW = 2
PLAN_WORDS = 5 + MAX_DEGREE + MAX_DEGREE - 1  # DQZ_PLAN_WORDS
TUNE_SWEEP_ONECTA = 5  # DQZ_TUNE_SWEEP_ONECTA


class DqzError(RuntimeError):
    """A libdqz entry point returned a non-zero status."""

    def __init__(self, func: str, status: int):
        names = {
            DQZ_ERR_ARG: "bad argument",
            DQZ_ERR_UNSUPPORTED: "shape outside the supported range",
            DQZ_ERR_CUDA: "CUDA launch/runtime error",
            DQZ_ERR_NOT_CONVERGED: "not converged",
            DQZ_ERR_NONFINITE: "non-finite value",
        }
        super().__init__(f"{func} failed: status {status} ({names.get(status, 'unknown')})")
        self.status = status


class GraphDesc(ctypes.Structure):
    """Mirror of dqz_graph_t."""

    _fields_ = [
        ("n_nodes", ctypes.c_int32),
        ("n_edges", ctypes.c_int32),
        ("n_halves", ctypes.c_int32),
        ("node_degree", ctypes.c_void_p),
        ("node_phys", ctypes.c_void_p),
        ("node_half", ctypes.c_void_p),
        ("node_off", ctypes.c_void_p),
        ("half_node", ctypes.c_void_p),
        ("half_edge", ctypes.c_void_p),
        ("half_twin", ctypes.c_void_p),
        ("half_msg_off", ctypes.c_void_p),
        ("edge_half", ctypes.c_void_p),
        ("edge_lam_off", ctypes.c_void_p),
        ("edge_chi", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int32
_D = ctypes.c_double
_S = ctypes.c_size_t
_G = ctypes.POINTER(GraphDesc)

# name -> (restype, argtypes)
_SIGNATURES = {
    "dqz_version": (ctypes.c_int, []),
    "dqz_device_supported": (ctypes.c_int, [ctypes.c_int]),
    "dqz_bp_node_update": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P]),
    "dqz_bp_node_scratch_bytes": (_S, [_I, _I, _I]),
    "dqz_bp_edge_pass": (ctypes.c_int, [_G, _P, _P, _P, _P, _I, _P]),
    "dqz_bp_sweep_levels": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P]),
    "dqz_bp_sweep_planned": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P]),
    "dqz_bp_sweep_sliced": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P,
                                           _P]),
    "dqz_bp_node_update_k3": (ctypes.c_int, [_G, _I, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P]),
    "dqz_bp_edge_pass_c64": (ctypes.c_int, [_G, _P, _P, _P, _P, _P]),
    "dqz_bp_node_update_k3_tc": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _P, _P]),
    "dqz_bp_node_update_k3_umma": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _P, _P]),
    "dqz_bf16_umma_elems_per_node": (_S, []),
    "dqz_pack_bf16_umma": (ctypes.c_int, [_G, _P, _P, _P]),
    "dqz_pack_bf16_umma_nodes": (ctypes.c_int, [_G, _P, _P, _I, _I, _P]),
    "dqz_pack_bf16_planes": (ctypes.c_int, [_G, _P, _P, _P]),
    "dqz_messages_distance": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _P]),
    "dqz_reduce_sum": (ctypes.c_int, [_P, _I, _D, _P, _P]),
    "dqz_message_changes_c64": (ctypes.c_int, [_G, _P, _P, _P, _P]),
    "dqz_segment_distance": (ctypes.c_int, [_P, _P, _P, _I, _P, _P, _P]),
    "dqz_bp_node_vjp": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _P]),
    "dqz_qr_batched": (ctypes.c_int, [_P, ctypes.c_int64, _I, _I, _P, _P, _P, _P]),
    "dqz_set_tuning": (ctypes.c_int, [_I, _I]),
    "dqz_sv_set_basis": (ctypes.c_int, [_P, _I, ctypes.c_int64, _P]),
    "dqz_sv_apply1": (ctypes.c_int, [_P, _I, _I, _P, _P]),
    "dqz_sv_apply2": (ctypes.c_int, [_P, _I, _I, _I, _P, _P]),
    "dqz_sv_density1": (ctypes.c_int, [_P, _I, _I, _P, _P, _P]),
    "dqz_sv_density_scratch_bytes": (_S, [_I]),
    "dqz_sv_project": (ctypes.c_int, [_P, _I, _I, _I, _D, _P]),
    "dqz_get_tuning": (ctypes.c_int32, [_I]),
    "dqz_qr_batched_scratch_bytes": (_S, [ctypes.c_int64, _I, _I]),
    "dqz_bp_node_vjp_scratch_bytes": (_S, [_I, _I]),
    "dqz_vidal_edges": (ctypes.c_int, [_G, _P, _D, _P, _P, _I, _P, _I, _P, _P]),
    "dqz_vidal_edges_scratch_bytes": (_S, [_I, _I]),
    "dqz_absorb": (ctypes.c_int, [_G, _P, _P, _P, _I, _P, _I, _P, _P]),
    "dqz_absorb_split": (ctypes.c_int, [_G, _P, _P, _P, ctypes.c_int64, _P, _I, _P, _P]),
    "dqz_absorb_split_scratch_bytes": (_S, [_I]),
    "dqz_absorb_scratch_bytes": (_S, [_I, _I]),
    "dqz_absorb_k3": (ctypes.c_int, [_G, _I, _P, _P, _P, _P, _I, _P, _P]),
    "dqz_vidal_distance": (ctypes.c_int, [_G, _P, _P, _D, _P, _P, _I, _I, _P, _I, _P]),
    "dqz_symmetric_gauge": (ctypes.c_int, [_G, _P, _P, _D, _P, _P]),
    "dqz_lambdas_to_messages": (ctypes.c_int, [_G, _P, _P, _P, _I, _P]),
    "dqz_density_matrices": (ctypes.c_int, [_G, _P, _P, _P, _I, _P, _I, _P, _P]),
    "dqz_density_scratch_bytes": (_S, [_I, _I]),
    "dqz_apply1": (ctypes.c_int, [_G, _P, _P, _P, _I, _P]),
    "dqz_apply_half_gates": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I, _P]),
    "dqz_simple_update": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _D, _I, _I, _I, _P, _P, _P, _P]),
    "dqz_simple_update_scratch_bytes": (_S, [_I, _I, _I]),
    "dqz_simple_update_noalloc": (ctypes.c_int, [_G, _P, _P, _P, _P, _P, _P, _I, _D, _I, _I, _I, _P, _P, _P]),
    "dqz_repack": (ctypes.c_int, [_P, _P, _P, _P, _P, _I, _I, _P]),
    "dqz_count_nonfinite": (ctypes.c_int, [_P, ctypes.c_int64, _I, _P, _P]),
}

_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """Loads libdqz.so once; raises RuntimeError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libdqz.so not found at {LIB_PATH}; build it with `python -m dequantizer_b200.build`"
            )
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(func: str, status: int):
    if status != DQZ_OK:
        raise DqzError(func, status)


def call(func: str, *args):
    """Calls a status-returning entry point and raises DqzError on failure."""
    check(func, getattr(lib(), func)(*args))


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def require_cuda(*tensors: torch.Tensor):
    for t in tensors:
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise RuntimeError(
                "dequantizer_b200 runs on the GPU only: expected CUDA tensors "
                f"(got {type(t).__name__} on {getattr(t, 'device', 'host')})"
            )


class NonFiniteError(DqzError):
    """NaN or Inf met in the state of a BP loop (status DQZ_ERR_NONFINITE)."""

    def __init__(self, where: str):
        super().__init__(where, DQZ_ERR_NONFINITE)


def count_nonfinite(t: torch.Tensor) -> int:
    """Number of NaN / Inf real words in a CUDA tensor (complex entries count
    their real and imaginary parts); synchronises with the stream."""
    require_cuda(t)
    t = t.contiguous()
    real = torch.view_as_real(t) if t.is_complex() else t
    if real.dtype not in (torch.float64, torch.float32):
        raise TypeError(f"count_nonfinite takes float32/64 or complex64/128 tensors, not {t.dtype}")
    cnt = torch.zeros(1, dtype=torch.int32, device=t.device)
    call("dqz_count_nonfinite", real.data_ptr(), real.numel(), real.element_size(), cnt.data_ptr(), stream_handle())
    return int(cnt.item())


def device() -> torch.device:
    """The device new tensors are created on (cuda:0 when available)."""
    return torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
