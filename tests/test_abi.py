"""The C ABI library without a GPU: it loads, exports every entry point that
include/vvm_gpu.h declares, and its host-only helpers work."""
import ctypes
import re

import pytest

from conftest import REPO

HEADER = REPO / "include" / "vvm_gpu.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vvm_gpu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from vvm_b200 import build, gpu
    build.build()
    return gpu.load_library()


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("vvm_gpu_create", "vvm_gpu_destroy", "vvm_gpu_upload_state",
                 "vvm_gpu_download_state", "vvm_gpu_step", "vvm_gpu_poisson_solve",
                 "vvm_gpu_last_error", "vvm_gpu_cal_w", "vvm_gpu_kessler", "vvm_gpu_turbulence"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header(lib):
    from vvm_b200 import gpu
    assert set(gpu.EXPORTS) == set(declared_functions())


def test_desc_default_has_reference_constants(lib):
    from vvm_b200.gpu import Desc
    d = Desc()
    lib.vvm_gpu_desc_default(ctypes.byref(d), 128, 64, 200.0, 200.0, 1.0)
    # src/main.cpp:68-72
    assert (d.gravity, d.cp, d.cv, d.rd, d.lv, d.p0, d.psurf) == \
        (9.80665, 1003.5, 716.5, 287.0, 2.5e6, 1e5, 96500.0)
    assert (d.NX, d.NZ, d.dx, d.dz, d.dt) == (128, 64, 200.0, 200.0, 1.0)
    assert d.poisson_tol == 1e-10 and d.case_id == 1


def test_invalid_descriptor_is_rejected_before_any_device_call(lib):
    from vvm_b200.gpu import Desc
    d = Desc()
    lib.vvm_gpu_desc_default(ctypes.byref(d), 2, 64, 200.0, 200.0, 1.0)   # NX < 4
    h = ctypes.c_void_p()
    assert lib.vvm_gpu_create(ctypes.byref(d), 0, ctypes.byref(h)) == 1     # VVM_GPU_EINVAL
    buf = ctypes.create_string_buffer(256)
    lib.vvm_gpu_last_error(None, buf, 256)
    assert b"NX and NZ" in buf.value
    d.NX, d.precision = 64, 7
    assert lib.vvm_gpu_create(ctypes.byref(d), 0, ctypes.byref(h)) == 1
    d.precision, d.flags = 0, 4                                             # no such flag
    assert lib.vvm_gpu_create(ctypes.byref(d), 0, ctypes.byref(h)) == 1
    lib.vvm_gpu_last_error(None, buf, 256)
    assert b"flags" in buf.value


def test_null_context_is_an_error(lib):
    assert lib.vvm_gpu_step(None, 1) == 1
    assert lib.vvm_gpu_cal_w(None) == 1
