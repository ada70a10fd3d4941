"""The C-ABI library: it builds for sm_100a, loads, and exports every entry
point include/eqd.h declares (no GPU needed; no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, load_package

HEADER = os.path.join(ROOT, "include", "eqd.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(eqd_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def built():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "eqd_build", os.path.join(ROOT, "earthquakediffinitive.jl_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.build()


def test_header_declares_the_abi():
    names = declared_functions()
    for must in ("eqd_grid_create", "eqd_stiffness_exact", "eqd_stiffness_toeplitz", "eqd_cg_solve",
                 "eqd_kmat_gemv", "eqd_apply", "eqd_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(built)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True).stdout
    for n in declared_functions():
        assert re.search(rf"\bT {n}\b", out), n


def test_binding_lists_match_header(built):
    eqd = load_package()
    assert sorted(eqd._abi.EXPORTS) == declared_functions()


def test_build_targets_sm100a():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "eqd_build2", os.path.join(ROOT, "earthquakediffinitive.jl_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    assert "arch=compute_100a,code=sm_100a" in m.NVCC_FLAGS


def test_struct_layouts(built):
    eqd = load_package()
    # Layouts follow the C header field by field (natural alignment).
    assert C.sizeof(eqd._abi.GridDesc) == 88
    assert C.sizeof(eqd._abi.SolveOpts) == 64
    assert C.sizeof(eqd._abi.Stats) == 72
    assert C.sizeof(eqd._abi.RequestInfo) == 48
    from eqd_b200.timeloop import RhsParams
    assert C.sizeof(RhsParams) == 176


def test_defaults_match_reference_cgsolver(built):
    eqd = load_package()
    o = eqd._abi.default_opts()
    assert o.rtol == 1e-10 and o.atol == 0.0 and o.itmax == 0   # src/ElasticitySplitNode.jl:365
    assert o.precond == eqd._abi.EQD_PRECOND_NONE


def test_bad_arguments_rejected_without_gpu(built):
    eqd = load_package()
    with pytest.raises(ValueError):
        eqd.CGSolver(precond="nonsense")
    with pytest.raises(ValueError):
        eqd.build_model(dz=100.0, L_fault=800.0, L_normal=400.0)   # n1 = 5 < 9 (src/BP8.jl:198-204)
    with pytest.raises(ValueError):
        eqd.build_model(dz=30.0)   # does not divide l_f


def test_flag_constants_match_header():
    """The Python and Julia bindings' opts.flags bits are the header's."""
    txt = open(HEADER).read()
    hdr = {k: int(v) for k, v in re.findall(r"#define (EQD_FLAG_[A-Z_]+) (\d+)u", txt)}
    assert set(hdr) == {"EQD_FLAG_STRICT", "EQD_FLAG_NO_SPLIT", "EQD_FLAG_FUSE"}
    eqd = load_package()
    for k, v in hdr.items():
        assert getattr(eqd._abi, k) == v
    jl = open(os.path.join(ROOT, "earthquakediffinitive.jl_b200", "julia", "EqdB200.jl")).read()
    for k, v in hdr.items():
        assert re.search(rf"const {k} = UInt32\({v}\)", jl), k
