"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        names += re.findall(r"PULSE_API\s+[\w\s\*]+?\b(pulse_\w+)\s*\(", h.read_text())
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from pulse_b200 import build, _ffi
    build.build()
    return _ffi.load()


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("pulse_render_forward", "pulse_build_blas", "pulse_build_tlas", "pulse_scene_set_buffers",
              "pulse_instances_set", "pulse_mesh_upload", "pulse_trace"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_ffi_binds_every_declared_symbol():
    from pulse_b200 import _ffi
    assert sorted(_ffi.SIGNATURES) == declared_symbols()


def test_default_params_are_reference_constants(lib):
    from pulse_b200 import _ffi
    p = _ffi.RenderParams()
    lib.pulse_default_params(C.byref(p))
    assert (p.max_depth, p.spp, p.nee_mode, p.quirks, p.stack_depth, p.iter_cap) == (5, 1, 0, 1, 32, 100000)
    assert p.eps_origin == C.c_float(0.001).value and p.eps_par == C.c_float(1e-4).value
    assert p.eps_shadow == C.c_float(0.005).value


def test_no_device_is_reported(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = C.c_void_p()
    assert lib.pulse_ctx_create(0, C.byref(h)) == -8
