"""The C-ABI library builds, loads and exports every entry point declared in
include/*.h (no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+[\s\*]+(gem_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from gemini_unified_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("gem_ctx_create", "gem_fk_run", "gem_fk_run_device", "gem_synth_run", "gem_last_error"):
        assert n in names, n


def test_library_exports_all_declared_symbols(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctx_create_fails_cleanly_without_gpu(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = ctypes.c_void_p()
    lib.gem_ctx_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    assert lib.gem_ctx_create(0, 1, ctypes.byref(h)) == 2
    assert not h.value


def test_product_never_imports_oracle():
    """The CUDA product path must not route through the CPU oracle."""
    for f in glob.glob(os.path.join(ROOT, "gemini_unified_b200", "**", "*"), recursive=True):
        if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
            txt = open(f).read()
            assert "oracle" not in re.sub(r"(#|//).*", "", txt).lower(), f


def test_new_entry_points_reject_a_null_context(lib):
    """The ASKI and coupling entry points return the error level 2 for a null
    context before touching the GPU; gem_fk_aski_nsp gives the spectra per node."""
    vp, i = ctypes.c_void_p, ctypes.c_int
    lib.gem_fk_run_dsv.argtypes = [vp, vp, i, i, vp, vp, vp, vp]
    lib.gem_fk_run_aski.argtypes = [vp, vp, i, vp, i, i, vp, vp, vp, vp]
    lib.gem_coupling_run.argtypes = [vp, vp, vp, vp, vp, vp, vp, i, vp, vp, vp, vp, vp]
    lib.gem_fk_aski_nsp.argtypes = [i]
    assert lib.gem_fk_run_dsv(None, None, 2, 3, None, None, None, None) == 2
    assert lib.gem_fk_run_aski(None, None, 1, None, 2, 3, None, None, None, None) == 2
    assert lib.gem_coupling_run(None, None, None, None, None, None, None, 1, None, None, None, None, None) == 2
    assert lib.gem_fk_aski_nsp(1) == 20 and lib.gem_fk_aski_nsp(0) == 10


def test_tuning_calls_reject_a_null_context(lib):
    """The schedule, deferral and queue-granularity calls return the error
    level 2 for a null context or a null array, before touching the GPU."""
    vp = ctypes.c_void_p
    three = (ctypes.c_int * 3)(0, 0, 0)
    for name in ("gem_fk_schedule_set", "gem_fk_schedule_get", "gem_fk_defer_set", "gem_fk_defer_get",
                 "gem_fk_queue_set", "gem_fk_queue_get"):
        f = getattr(lib, name)
        f.argtypes = [vp, vp]
        assert f(None, three) == 2, name
        assert f(None, None) == 2, name
