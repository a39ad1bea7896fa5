"""CPU-only checks of the C ABI boundary: the library loads without a GPU and
exports every entry point that include/hsb200.h declares; the Python host
mirror keeps the reference's argument validation."""
import ctypes
import os
import re

import pytest

import hsb200
from hsb200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hsb200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("hs_l1gs_create", "hs_l1gs_apply", "hs_l1gs_apply_host", "hs_l1gs_get_packed",
                 "hs_cheb_create", "hs_cheb_smooth", "hs_matrix_spmv", "hs_pcg_solve", "hs_gmres_solve"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.PROTOTYPES)


def test_version_and_counters_without_gpu():
    L = hsb200.lib()
    assert L.hs_version().startswith(b"hsb200")
    assert hsb200.kernel_launches() >= 0


def test_gpuconfig_validation():
    """GPUConfig/CPUConfig raise like src/l1_gauss_seidel.jl:201, :217-218."""
    with pytest.raises(ValueError, match="threads"):
        hsb200.GPUConfig(0, 4)
    with pytest.raises(ValueError, match="blocks"):
        hsb200.GPUConfig(4, 0)
    with pytest.raises(ValueError, match="chunks"):
        hsb200.CPUConfig(0)


def test_cpu_backend_is_refused():
    from hsb200 import workloads as W
    b = hsb200.L1GSPrecBuilder(hsb200.CPU(), chunks=4)
    with pytest.raises(NotImplementedError):
        b(W.poisson_test_matrix(9), 2)


def test_default_partsize_is_blocks():
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=7)
    assert b._default_partsize() == 7


def test_symmetric_wrapper_materializes():
    import scipy.sparse as sp
    from hsb200 import workloads as W
    A = W.poisson2d_matrix(6, 0.5)
    for uplo, tri in (("U", sp.triu(A)), ("L", sp.tril(A))):
        full = hsb200.Symmetric(tri.tocsc(), uplo).materialize()
        assert abs(full - A).max() == 0
