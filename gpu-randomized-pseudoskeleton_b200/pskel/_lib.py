"""ctypes binding of libpskel_b200.so (the C ABI declared in include/pskel.h).

The library is loaded from this package's parent directory; there is no CPU fallback: if the
shared library is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libpskel_b200.so")
HEADER = os.path.join(ROOT, "include", "pskel.h")

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int)
I64 = ctypes.POINTER(ctypes.c_int64)
VP = ctypes.c_void_p
ci = ctypes.c_int
cd = ctypes.c_double

PSKEL_OK = 0
STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_NOCONV", -4: "ERR_NEAR",
          -5: "ERR_OOM", -6: "ERR_RANGE", -7: "ERR_UNSUPPORTED", -8: "ERR_STATE"}


class PskelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class EM(ctypes.Structure):
    _fields_ = [("k", cd), ("eta", cd), ("q_test", ci), ("q_src", ci)]


class Opts(ctypes.Structure):
    _fields_ = [("tol", cd), ("tau", cd), ("tau_relative", ci), ("precision", ci),
                ("start", ci), ("oversample", ci), ("extra_rows", ci), ("extra_cols", ci),
                ("max_rounds", ci), ("recompress", ci), ("seed", ctypes.c_uint64),
                ("recompress_tol", cd), ("est_safety", cd), ("use_graph", ci),
                ("per_block", ci), ("est_verify", cd), ("full_tau", cd)]


class BlockStat(ctypes.Structure):
    _fields_ = [("m", ci), ("n", ci), ("r", ci), ("rank", ci), ("rank_recompressed", ci),
                ("rounds", ci), ("status", ci), ("est", cd)]


# argument tails shared by the reference fill signatures
_MESH = [D] * 8  # vertex topol trian edges un ds ln cent
_SIZES = [ci] * 18  # N n_r1 n_r2 rows/cols ... cols_cent
_LAUNCH = [ci] * 6  # blocks_x blocks_y threads_x threads_y limx limy
_EM = [ci, cd, cd, cd, cd, cd, ci, ci]  # field k eta Rinteg_s Ranal_s Rinteg_f cor_solid flag

SIGNATURES = {
    "pskel_last_error": (ci, [ctypes.POINTER(ctypes.c_char_p)]),
    "impedance_matrix_cuda_elbyel4": (cd, [VP] + _EM + [D, D] + _MESH + _SIZES + _LAUNCH),
    "impedance_matrix_cuda_elbyel3": (ci, [VP] + _EM + [D, D] + _MESH + _SIZES + _LAUNCH),
    "impedance_matrix_cuda_elbyel2": (ci, [D, D] + _EM + [D, D] + _MESH + _SIZES + _LAUNCH),
    "cuda_cur_pure": (ci, [D, D] + _EM + [D, D] + _MESH + [D] * 6 + _SIZES + _LAUNCH + [cd]),
    "cuda_complete_compression": (cd, [VP, VP, VP, ci, D, cd, VP, VP, VP, D, D] + [ci] * 12 +
                                  [VP] + _EM + [D, D] + _MESH + _SIZES + _LAUNCH),
    "compute_error_compression": (cd, [VP] * 6 + [ci] * 3),
    "aux_pinv_compression": (ci, [VP] * 4 + [I64, I64, ci, ci, ci, cd]),
    "cuda_pinv": (ci, [VP, VP, D, VP, VP, ci, ci, cd]),
    "cuda_svd": (ci, [VP, D, VP, VP, ci, ci]),
    "cuda_svd2": (ci, [VP, D, VP, VP, ci, ci]),
    "cuda_filter": (ci, [D, cd, ci]),
    "pskel_create": (ci, [ctypes.POINTER(VP), ci]),
    "pskel_destroy": (ci, [VP]),
    "pskel_upload_mesh": (ci, [VP, D, ci, D, ci, D, ci, D, D, ctypes.POINTER(EM)]),
    "pskel_fill_device": (ci, [VP, VP, ci, VP, ci, VP, ci, ci]),
    "pskel_set_blocks": (ci, [VP, I32, I32, ci, I32, I32, ci]),
    "pskel_compress_blocks": (ci, [VP, ctypes.POINTER(Opts), I32, ctypes.POINTER(BlockStat)]),
    "pskel_last_timing": (ci, [VP, D, ci]),
    "pskel_get_block": (ci, [VP, ci, VP, VP, VP, I32, I32]),
    "pskel_true_errors": (ci, [VP, D]),
    "pskel_true_errors_blocks": (ci, [VP, I32, ci, D]),
    "pskel_dense_far_matvec": (ci, [VP, VP, ci, VP, ci, ci]),
    "pskel_set_fill_split": (ci, [VP, ci, ci]),
    "pskel_set_tri_cols": (ci, [VP, ci]),
    "pskel_set_pipeline": (ci, [VP, ci]),
    "pskel_set_round_growth": (ci, [VP, cd]),
    "pskel_set_fill_geometry": (ci, [VP, ci]),
    "pskel_set_symmetric": (ci, [VP, ci]),
    "pskel_fill_near_device": (ci, [VP, VP, ci, VP, ci, VP, ci, cd, cd, cd, ci]),
    "pskel_store_save": (ci, [VP, ctypes.c_char_p, cd]),
    "pskel_store_load": (ci, [VP, ctypes.c_char_p, I32]),
    "pskel_aca_compress": (ci, [VP, cd, ci, I32, I32]),
    "pskel_aca_get_block": (ci, [VP, ci, VP, VP, I32, I32]),
    "pskel_aca_true_errors": (ci, [VP, D]),
    "pskel_near_build": (ci, [VP, I32, I32, ci, cd, cd, cd, ci, ctypes.POINTER(ctypes.c_longlong)]),
    "pskel_near_matvec": (ci, [VP, VP, ci, VP, ci, ci, ci, VP]),
    "pskel_plane_wave": (ci, [VP, cd, cd, cd, VP, VP]),
    "pskel_octree_build": (ci, [VP, cd, D, cd, ci, ci, I32, ctypes.POINTER(ctypes.c_longlong)]),
    "pskel_octree_get": (ci, [VP, I32, I32, D, D, I32, I32]),
    "pskel_matvec": (ci, [VP, VP, ci, VP, ci, ci, ci, VP]),
    "pskel_recompress": (ci, [VP, cd, I32]),
    "pskel_set_recompress_path": (ci, [VP, ci]),
    "pskel_recompress_split_blocks": (ci, [VP, I32]),
    "pskel_get_recompressed": (ci, [VP, ci, VP, D, VP]),
    "pskel_store_build": (ci, [VP, ctypes.POINTER(ctypes.c_longlong)]),
    "pskel_store_build_mode": (ci, [VP, ci, ctypes.POINTER(ctypes.c_longlong)]),
    "pskel_store_matvec": (ci, [VP, VP, ci, VP, ci, ci, VP]),
    "pskel_store_matvec_strided": (ci, [VP, VP, ctypes.c_longlong, ctypes.c_longlong, VP,
                                        ctypes.c_longlong, ctypes.c_longlong, ci, VP]),
    "pskel_store_status": (ci, [VP, I32]),
    "pskel_mlp_num_params": (ci, []),
    "pskel_mlp_forward": (ci, [VP, VP, ci, VP, VP]),
    "pskel_mlp_grad": (ci, [VP, VP, VP, ci, VP, VP, VP]),
    "pskel_mlp_adam": (ci, [VP, VP, VP, VP, ci, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                            ctypes.c_float, VP]),
    "pskel_kernel_launches": (ctypes.c_longlong, []),
    "pskel_fma_peak": (ci, [D, D]),
    "pskel_pinv_noalloc": (ci, [VP, ci, ci, cd, ci, VP, VP, VP, VP]),
    "pskel_diag_sincos": (ci, [VP, ci, VP]),
}

_LIB = None


def header_symbols() -> list[str]:
    """Function names declared in include/pskel.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][A-Za-z0-9_]*\s+\**)+([a-z_][a-z0-9_]*)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def lib() -> ctypes.CDLL:
    """Load libpskel_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run gpu-randomized-pseudoskeleton_b200/build.py")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _LIB = h
    return _LIB


def last_error() -> tuple[int, str]:
    msg = ctypes.c_char_p()
    code = lib().pskel_last_error(ctypes.byref(msg))
    return code, (msg.value or b"").decode()


def check(code: int):
    if code != PSKEL_OK:
        c, m = last_error()
        raise PskelError(code, m)
