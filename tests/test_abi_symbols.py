"""The C ABI library loads and exports every function include/pskel.h declares (no compute)."""
import ctypes

from pskel import _lib


def test_library_exports_header_symbols():
    names = _lib.header_symbols()
    assert "impedance_matrix_cuda_elbyel4" in names and "cuda_complete_compression" in names
    h = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(h, n)]
    assert not missing, missing


def test_reference_symbols_declared():
    names = set(_lib.header_symbols())
    for n in ("impedance_matrix_cuda_elbyel4", "impedance_matrix_cuda_elbyel3",
              "impedance_matrix_cuda_elbyel2", "cuda_cur_pure", "cuda_complete_compression",
              "compute_error_compression", "aux_pinv_compression", "cuda_pinv", "cuda_svd",
              "cuda_svd2", "cuda_filter"):
        assert n in names, n


def test_signature_table_covers_header():
    names = set(_lib.header_symbols())
    assert names <= set(_lib.SIGNATURES), names - set(_lib.SIGNATURES)
