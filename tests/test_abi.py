"""The C ABI library loads and exports every entry point include/b2s.h
declares (no GPU needed: no compute call is made)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))
LIB = ROOT / "tnl-dev_b200" / "libb2sparse.so"


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(b2s_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["b2s_matrix_create", "b2s_spmv", "b2s_solve", "b2s_solver_create", "b2s_matrix_export",
                 "b2s_dot", "b2s_scan_i32"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    assert LIB.exists(), "libb2sparse.so not built"
    lib = C.CDLL(str(LIB))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_abi_host_only_calls():
    import b2s
    lib = b2s.lib
    assert lib.b2s_abi_version() == 2
    assert lib.b2s_status_string(b2s.OK) == b"ok"
    assert b"32-bit" in lib.b2s_status_string(b2s.INDEX_OVERFLOW)
    # argument checks happen before any device call
    h = C.c_void_p()
    st = lib.b2s_matrix_create(7, 0, 4, 4, 0, None, None, None, 0, 0, None, None, C.byref(h))
    assert st == b2s.INVALID_ARG
    assert b"format" in lib.b2s_last_error()
    st = lib.b2s_matrix_create(0, 0, -1, 4, 0, None, None, None, 0, 0, None, None, C.byref(h))
    assert st == b2s.INVALID_ARG


def test_solve_opts_defaults_follow_tnl():
    import b2s
    from b2s import _abi
    o = _abi.SolveOpts()
    b2s.lib.b2s_solve_opts_default(C.byref(o))
    # IterativeSolver.h:226-235 and GMRES.h:220-237 / GMRES.hpp configSetup
    assert o.convergence_residue == 1e-6
    assert o.max_iterations == 1000000000
    assert o.min_iterations == 0
    assert o.gmres_restarting_min == 10 and o.gmres_restarting_max == 10
    assert o.gmres_restarting_step_min == 3 and o.gmres_restarting_step_max == 3
    assert o.gmres_variant == _abi.GMRES_MGSR
    # Jacobi.h:126-128, SOR.h:125-127 (and their configSetup)
    assert o.omega == 1.0 and o.residue_period == 4
    assert C.sizeof(_abi.SolveOpts) == 128


@pytest.mark.parametrize("name", ["CG", "BICGStab", "GMRES"])
def test_tnl_shaped_solver_api(name):
    import b2s
    s = getattr(b2s, name)()
    s.setConvergenceResidue(1e-10)
    s.setMaxIterations(500)
    assert s.setup({"gmres-variant": "CGSR", "gmres-restarting-min": 30, "gmres-restarting-max": 30})
    assert not s.setup({"gmres-variant": "CWYX"})
    assert s.opts.gmres_restarting_max == 30 and s.opts.gmres_variant == 1
    with pytest.raises(RuntimeError):
        s.solve(None, None)
