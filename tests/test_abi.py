"""The C-ABI library loads and exports every entry point include/bpf.h declares (no GPU)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "bpf.h")).read()
    return sorted(set(re.findall(r"BPF_API\s+[^;()]*?\b(bpf_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "bpf_block_gmres" in syms and "bpf_rf_analyze" in syms and "bpf_ilu0_create" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    import ctypes

    from blockpowerflow_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libbpf.so not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert not [s for s in declared_symbols() if s not in _lib.SIGNATURES]


def test_solve_status_strings_match_reference():
    """src/block_gmres.jl:397-399 status strings, returned by the library itself."""
    from blockpowerflow_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libbpf.so not built")
    lib = _lib.load()
    assert lib.bpf_solve_status_string(1).decode() == "solution good enough given atol and rtol"
    assert lib.bpf_solve_status_string(2).decode() == "maximum number of iterations exceeded"
    assert lib.bpf_solve_status_string(3).decode() == "time limit exceeded"
    assert lib.bpf_solve_status_string(0).decode() == "unknown"


def test_product_path_has_no_cpu_fallback():
    """The solvers refuse to run without a CUDA device instead of falling back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    import blockpowerflow_b200 as bpf

    with pytest.raises(RuntimeError):
        bpf._lib.context()
