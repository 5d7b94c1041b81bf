"""CPU checks of the C-ABI library: it loads without a GPU and exports every function
that include/*.h declares; the Python mirror keeps the reference's names."""
import ctypes
import glob
import os

from hsps_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    headers = glob.glob(os.path.join(ROOT, "include", "*.h"))
    assert headers
    missing = []
    for h in headers:
        for name in _abi.declared_symbols(h):
            if not hasattr(L, name):
                missing.append(name)
    assert not missing, missing


def test_struct_layouts_match_header():
    # sizes computed by the C compiler from include/hamlss.h
    import subprocess, tempfile
    src = (
        '#include <stdio.h>\n#include "hamlss.h"\n'
        'int main(){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(hamlss_params), sizeof(hamlss_stats),'
        ' sizeof(hamlss_escalation), sizeof(hamlss_server_config), sizeof(hamlss_server_report),'
        ' sizeof(hamlss_batch_result));return 0;}\n')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert [int(x) for x in out] == [ctypes.sizeof(_abi.Params), ctypes.sizeof(_abi.Stats),
                                     ctypes.sizeof(_abi.Escalation), ctypes.sizeof(_abi.ServerConfig),
                                     ctypes.sizeof(_abi.ServerReport), ctypes.sizeof(_abi.BatchResult)]


def test_server_config_defaults():
    c = _abi.ServerConfig()
    _abi.lib().hamlss_server_config_default(ctypes.byref(c))
    assert (c.device, c.slots, c.hbm_budget_bytes, c.batch_max_rows, c.batch_max_count, c.order) == \
           (0, 4, 150 * 10**9, 16384, 2048, 0)


def test_solver_classes_mirror_reference():
    # PipelinedFGMRESSolver has no SolverType and reports FGMRES; SStepCGSolver(k = 4)
    # (sstep_cg_solver.hpp:57-60) is made by the factory with params.sstep_k
    import hsps_b200 as H
    assert H.PipelinedFGMRESSolver.solver_type == _abi.SOLVER_PIPELINED_FGMRES == 5
    assert H.SStepCGSolver().k == 4
    s = H.SolverFactory.make_solver(H.SolverFactory.parse_solver("s-step"), _abi.default_params(sstep_k=6))
    assert isinstance(s, H.SStepCGSolver) and s.k == 6 and s.type() == _abi.SOLVER_SSTEP_CG
    import pytest
    with pytest.raises(ValueError):
        H.SolverFactory.make_solver(H.SolverFactory.parse_solver("async"), _abi.default_params())


def test_params_default_matches_reference_defaults():
    p = _abi.Params()
    _abi.lib().hamlss_params_default(ctypes.byref(p))
    q = _abi.default_params()
    for name, _ in _abi.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name
    # SolverParams defaults (include/core/types.hpp:119-143)
    assert (p.tol, p.max_iter, p.restart_size, p.drop_tol, p.amg_levels) == (1e-8, 2000, 50, 1e-4, 10)
    assert (p.amg_strong, p.amg_smooth_pre, p.amg_smooth_post, p.stall_window) == (0.25, 2, 2, 15)


def test_version_and_no_device_error():
    L = _abi.lib()
    assert b"sm_100a" in L.hamlss_version()
    import torch
    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        rc = L.hamlss_ctx_create(0, ctypes.byref(h))
        assert rc < 0 and L.hamlss_last_error()


def test_factory_parse_names():
    import hsps_b200 as H
    import pytest
    assert H.SolverFactory.parse_solver("cg") == 0
    assert H.SolverFactory.parse_solver("FGMRES") == 1
    assert H.SolverFactory.parse_precond("ilu0") == 2
    assert H.SolverFactory.parse_precond("diag") == 1
    with pytest.raises(ValueError):
        H.SolverFactory.parse_solver("gmres2")
    with pytest.raises(ValueError):
        H.SolverFactory.parse_precond("sor")
