"""ctypes binding of the C ABI in include/btorch_b200.h.

The shared library is built in-tree (btorch_b200/_lib/libbtorch_b200.so, see
btorch_b200/csrc/build.py).  There is no fallback: if the library is missing
or no CUDA device is present, every compute entry point raises.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libbtorch_b200.so"

BT_OK, BT_ERR_INVALID, BT_ERR_CUDA, BT_ERR_TIMEOUT, BT_ERR_UNSUPPORTED, BT_ERR_LAYOUT = range(6)
BT_NEURON_LIF, BT_NEURON_ALIF = 0, 1
BT_MODE_SCATTER, BT_MODE_GATHER, BT_MODE_PULL, BT_MODE_TILE, BT_MODE_CLUSTER = 0, 1, 2, 3, 4
BT_BIN_SHIFT = 25
BT_MAX_BINS = 128

_vp = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32


ABI_VERSION = 11  # BT_ABI_VERSION of include/btorch_b200.h the structures below mirror


class BtParam(C.Structure):
    _fields_ = [("ptr", _vp), ("stride", _i64)]


class BtNeuronDesc(C.Structure):
    _fields_ = [
        ("kind", _i32), ("hard_reset", _i32), ("use_refractory", _i32), ("spiking", _i32),
        ("dt", C.c_float), ("sg_alpha", C.c_float), ("sg_damping", C.c_float), ("pad_", C.c_float),
        ("v_threshold", BtParam), ("v_reset", BtParam), ("c_m", BtParam), ("tau", BtParam),
        ("tau_ref", BtParam), ("g_leak", BtParam), ("E_leak", BtParam), ("E_k", BtParam),
        ("dg_k", BtParam), ("tau_adapt", BtParam), ("coef_gk", BtParam),
        ("uniform", _i32), ("sv", C.c_float * 11), ("fast_div", _i32), ("rcp", C.c_float * 4),
    ]


class BtEngineDesc(C.Structure):
    _fields_ = [
        ("n", _i64), ("batch", _i64), ("n_bins", _i32), ("mode", _i32), ("t0", _i64), ("n_steps", _i64),
        ("bin_lo", _i32), ("bin_hi", _i32), ("hist_len", _i32), ("scatter_lanes", _i32),
        ("neuron", BtNeuronDesc), ("psc_coef", BtParam), ("psc_tau", BtParam),
        ("csr_ptr", _vp), ("csr_dst", _vp), ("csr_w", _vp),
        ("csc_ptr", _vp), ("csc_src", _vp), ("csc_w", _vp),
        ("v", _vp), ("refractory", _vp), ("g_k", _vp), ("psc", _vp), ("ring", _vp), ("hist", _vp),
        ("x", _vp), ("sample_len", _vp),
        ("raster", _vp), ("spikes", _vp), ("v_trace", _vp), ("psc_trace", _vp), ("ref_trace", _vp),
        ("gk_trace", _vp),
        ("sl_ptr", _vp), ("sl_src", _vp), ("sl_w", _vp), ("masks", _vp), ("outdeg", _vp),
        ("pull_words_per_warp", _i32), ("neuron_spt", _i32),
        ("work", _vp), ("stats", _vp), ("dense_rows", _i64),
        ("psc_uniform", _i32), ("psc_coef_s", C.c_float), ("psc_tau_s", C.c_float), ("psc_fast_div", _i32),
        ("psc_rcp", C.c_float), ("n_rec", _i32), ("csr_edges", _vp),
        ("tile_posts", _i32), ("n_tiles", _i32), ("tile_off", _vp), ("tile_work", _vp), ("spin_limit", _i32),
        ("tile_rows", _i64), ("cl_w", _vp), ("cl_src", _vp), ("cl_gptr", _vp),
    ]


_PROTOS = {
    "bt_last_error": (C.c_char_p, []),
    "bt_abi_version": (C.c_int, []),
    "bt_layout_build": (C.c_int, [_i64, _vp, _vp, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _vp]),
    "bt_layout_slices": (C.c_int, [_i64, _vp, _vp, C.c_uint32, _vp, _vp, _vp, _i64, _vp]),
    "bt_spmv_gather": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_spmv_scatter": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_spmv_gather_noalloc": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_spmv_grad_input": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_spmv_grad_input_t": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_spmv_grad_weight": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_check_neuron_desc": (C.c_int, [C.POINTER(BtNeuronDesc)]),
    "bt_fast_div_check": (C.c_int, [C.c_float, C.c_float, _vp, _vp]),
    "bt_neuron_step": (C.c_int, [C.POINTER(BtNeuronDesc), _i64, _i64] + [_vp] * 11 + [_vp]),
    "bt_neuron_step_backward": (C.c_int, [C.POINTER(BtNeuronDesc), _i64, _i64] + [_vp] * 13 + [_i32, _vp]),
    "bt_psc_step": (C.c_int, [_i64, _i64, BtParam, BtParam, _vp, _vp, _vp, _vp]),
    "bt_engine_run": (C.c_int, [C.POINTER(BtEngineDesc), _vp]),
    "bt_engine_prime": (C.c_int, [C.POINTER(BtEngineDesc), _vp]),
    "bt_input_project": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_input_project_live": (C.c_int, [_i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_bits_to_float": (C.c_int, [_i64, _i64, _vp, _vp, _vp]),
    "bt_float_to_bits": (C.c_int, [_i64, _i64, _vp, _vp, _vp]),
    "bt_raster_count": (C.c_int, [_i64, _i64, _vp, _vp, _vp]),
    "bt_raster_coords": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_float_to_masks": (C.c_int, [_i64, _i64, _vp, _vp, _vp]),
    "bt_mask_stride": (C.c_int, [_i64]),
    "bt_engine_work_words": (C.c_int64, [_i64, _i64, _i32]),
    "bt_masks_to_float": (C.c_int, [_i64, _i64, _vp, _vp, _vp]),
    "bt_tile_work_words": (C.c_int64, [_i64, _i32, _i32]),
    "bt_tile_smem_bytes": (C.c_int64, [_i64, _i32, _i32]),
    "bt_cluster_smem_bytes": (C.c_int64, [_i64, _i64, _i32, _i64, _i32]),
    "bt_tile_offsets": (C.c_int, [_i64, _vp, _vp, _i32, _i32, _vp, _vp]),
    "bt_input_grad_weight": (C.c_int, [_i64, _i64, _i64, _vp, _vp, _vp, _i32, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def lib():
    """Load the shared library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"btorch_b200 CUDA library not found at {LIB_PATH}; build it with "
                    "`python -m btorch_b200.csrc.build` (there is no CPU fallback)."
                )
            h = C.CDLL(str(LIB_PATH))
            for name, (res, args) in _PROTOS.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            if h.bt_abi_version() != ABI_VERSION:
                raise RuntimeError(f"{LIB_PATH} has ABI {h.bt_abi_version()}, this package needs {ABI_VERSION}; "
                                   "rebuild it with `python -m btorch_b200.csrc.build`.")
            _lib = h
    return _lib


def check(status: int, what: str = "") -> None:
    if status == BT_OK:
        return
    msg = lib().bt_last_error().decode(errors="replace")
    text = f"{what}: {msg}" if what else msg
    if status in (BT_ERR_INVALID, BT_ERR_LAYOUT):
        raise ValueError(text)
    if status == BT_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    raise RuntimeError(text)


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_of(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(*tensors: torch.Tensor, what: str = "btorch_b200") -> torch.device:
    """All tensors must be CUDA fp32; returns their device."""
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise RuntimeError(f"{what} requires CUDA tensors (there is no CPU path); got {t.device}.")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise RuntimeError(f"{what}: tensors on different devices ({dev} vs {t.device}).")
    if dev is None:
        raise RuntimeError(f"{what}: no tensor given")
    lib()
    return dev


def param(t: torch.Tensor) -> BtParam:
    """Scalar (numel 1) or per-neuron contiguous fp32 tensor -> bt_param."""
    return BtParam(t.data_ptr(), 0 if t.numel() == 1 else 1)
