"""CPU checks of the C ABI library: it loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            syms += re.findall(r"\b(cq_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(syms))


def test_headers_declare_entry_points():
    s = declared_symbols()
    for name in ("cq_system_create", "cq_mat_mult", "cq_m_kern_max", "cq_m_kern_min"):
        assert name in s


def test_library_exports_every_declared_symbol():
    from cq_b200 import LIB_PATH
    if not os.path.exists(LIB_PATH):
        pytest.fail("libcqb200.so is not built")
    L = ctypes.CDLL(LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_errors_without_device_are_reported_not_crashing():
    import cq_b200
    L = cq_b200.lib()
    assert L.cq_version().decode().startswith("cqb200")
    # a null system is rejected with CQ_ERR_ARG before any CUDA call
    n = ctypes.c_int64()
    assert L.cq_range_length(None, 0, ctypes.byref(n), ctypes.byref(n)) == cq_b200.CQ_ERR_ARG


def test_lnv_parameter_defaults_and_names():
    """cq_lnv_params_default (a host call): the reference's fdf defaults and the precision form's
    defaults (three-part split to the final tolerance, FP64 on the tensor cores); the Python mirror
    rejects unknown field names instead of setting a stray attribute."""
    import cq_b200
    p = cq_b200.lnv_params()
    assert (p.n_L_iterations, p.tolerance, p.maxpulay, p.exact) == (50, 1e-7, 5, 1)
    assert (p.mixed, p.split_parts, p.fp64_tensor, p.mixed_tolerance, p.mixed_max_outer) == (0, 3, 1, 0.0, 0)
    p = cq_b200.lnv_params(split_parts=2, mixed=1)
    assert (p.split_parts, p.mixed) == (2, 1)
    with pytest.raises(TypeError):
        cq_b200.lnv_params(split_part=3)


def test_precision_constants_match_header():
    import cq_b200
    txt = open(os.path.join(ROOT, "include", "cq_b200.h")).read()
    for name in ("FP64_FMA", "FP64", "BF16X3", "BF16X6", "FP64_TC"):
        m = re.search(r"#define CQ_PREC_%s (\d+)" % name, txt)
        assert m and int(m.group(1)) == getattr(cq_b200, "PREC_" + name)
