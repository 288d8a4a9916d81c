"""CPU-side checks of the drop-in boundary: the C-ABI library loads and exports every symbol
that include/exa_aderdg.h declares (no device calls)."""
import ctypes
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, "include", "exa_aderdg.h")
LIB = os.path.join(REPO, "exahype-engine_b200", "libexa_aderdg.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(exa_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("exa_solver_create", "exa_fused_predictor_volume_integral", "exa_riemann_solver_nonlinear",
                 "exa_surface_integral_and_update", "exa_stable_time_step_size", "exa_patch_step",
                 "exa_spaceTimePredictorNonlinear"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        import __graft_entry__
        __graft_entry__.build()
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls():
    import exa_aderdg
    lib = exa_aderdg.load_library()
    assert lib.exa_version().startswith(b"exa_aderdg")
    # invalid configurations are rejected before touching a device
    cfg = exa_aderdg._Config(4, 5, 0, 0, 0.9, 0.0, 0, 0)
    h = ctypes.c_void_p()
    assert lib.exa_solver_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert b"dim" in lib.exa_last_error()
    cfg = exa_aderdg._Config(3, 8, 0, 0, 0.9, 0.0, 0, 0)
    assert lib.exa_solver_create(ctypes.byref(cfg), ctypes.byref(h)) == 2  # not instantiated
    assert lib.exa_solver_create(None, ctypes.byref(h)) == 1


def test_missing_library_fails_loudly(tmp_path):
    """Without the compiled library the binding raises; there is no CPU fallback to run instead."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import exa_aderdg\n"
            "try:\n"
            "    exa_aderdg.load_library(%r)\n"
            "except exa_aderdg.ExaError as e:\n"
            "    print('raised:', e)\n"
            "    sys.exit(0)\n"
            "sys.exit(1)\n") % (os.path.join(REPO, "exahype-engine_b200"), str(tmp_path / "libexa_aderdg.so"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "missing" in r.stdout
