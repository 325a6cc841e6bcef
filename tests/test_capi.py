"""The C-ABI library loads, exports every entry point include/luvas3d.h declares, and rejects bad
arguments before touching a device (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from luvas3d import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "luvas3d.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(l3d_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for needed in ("l3d_stereo_create", "l3d_stereo_set_image", "l3d_stereo_solve",
                   "l3d_stereo_solve_all", "l3d_stereo_filter", "l3d_stereo_read_filtered",
                   "l3d_stereo_read_depth", "l3d_stereo_read_hyp", "l3d_stereo_destroy",
                   "l3d_tsdf_create", "l3d_tsdf_integrate", "l3d_tsdf_integrate_many",
                   "l3d_tsdf_read", "l3d_tsdf_destroy", "l3d_last_error"):
        assert needed in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_struct_layouts_match_the_c_abi():
    # sizes under the x86-64 System V ABI
    assert C.sizeof(_lib.View) == 16 * 8
    assert C.sizeof(_lib.StereoOpts) == 8 + 5 * 4 + 4 + 8 + 4 + 4
    assert C.sizeof(_lib.SolveOpts) == 8 + 8 + 16 + 8 + 16
    assert C.sizeof(_lib.IntegrationView) == 16 * 8 + 8 + 8 + 8
    assert C.sizeof(_lib.TsdfDesc) == 7 * 8 + 4 * 4 + 8 + 4 * 4 + 8


def _views(n=2):
    arr = (_lib.View * n)()
    for i in range(n):
        arr[i].intrinsics = _lib.Intrinsics(100, 100, 50, 50)
        arr[i].pose.R[:] = [1, 0, 0, 0, 1, 0, 0, 0, 1]
    return arr


def test_bad_arguments_are_rejected_with_a_message():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.l3d_stereo_create(0, 10, 2, _views(), None, C.byref(h)) == _lib.L3D_EINVAL
    assert "positive" in _lib.last_error()
    assert lib.l3d_stereo_create(10, 10, 0, _views(), None, C.byref(h)) == _lib.L3D_EINVAL
    opts = _lib.StereoOpts()
    lib.l3d_stereo_opts_default(C.byref(opts))
    assert (opts.depth_maps, opts.storage, opts.form, opts.window, opts.dilation) == (1, 1, 0, 6, 2)
    opts.window = 7
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    assert "window" in _lib.last_error()
    lib.l3d_stereo_opts_default(C.byref(opts))
    opts.storage = _lib.DTYPE_F16
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    opts.form = _lib.FORM_EXACT  # the exact form keeps FP32 texels
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    assert "exact form" in _lib.last_error()
    lib.l3d_stereo_opts_default(C.byref(opts))
    opts.compensated = 1  # the plain form is the oracle's uncompensated order
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    assert "compensated" in _lib.last_error()
    lib.l3d_stereo_opts_default(C.byref(opts))
    opts.form = _lib.FORM_EXACT
    opts.window, opts.dilation = 11, 1
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    lib.l3d_stereo_opts_default(C.byref(opts))
    opts.form = 3
    assert lib.l3d_stereo_create(10, 10, 2, _views(), C.byref(opts), C.byref(h)) == _lib.L3D_EINVAL
    bad = _views()
    bad[1].intrinsics.fx = 0
    assert lib.l3d_stereo_create(10, 10, 2, bad, None, C.byref(h)) == _lib.L3D_EINVAL
    assert h.value is None
    d = _lib.TsdfDesc()
    assert lib.l3d_tsdf_create(C.byref(d), C.byref(h)) == _lib.L3D_EINVAL
    # NULL handles
    assert lib.l3d_stereo_synchronize(None) == _lib.L3D_EINVAL
    assert lib.l3d_tsdf_read(None, None, None) == _lib.L3D_EINVAL
    lib.l3d_stereo_destroy(None)
    lib.l3d_tsdf_destroy(None)
    buf = (C.c_float * 4)()
    assert lib.l3d_tsdf_integrate_many_read(None, None, None, None, 1, None, None, None) == _lib.L3D_EINVAL
    assert "no output" in _lib.last_error()
    assert lib.l3d_tsdf_integrate_many_read(None, None, None, None, 1, None, buf, None) == _lib.L3D_EINVAL
    assert "NULL handle" in _lib.last_error()
    assert lib.l3d_tsdf_integrate_many_read_async(None, None, None, None, 1, None, None, None) == _lib.L3D_EINVAL
    assert "no output" in _lib.last_error()
    assert lib.l3d_tsdf_wait_read(None) == _lib.L3D_EINVAL
    rate = C.c_double(-1.0)
    assert lib.l3d_measure_texture_rate(_lib.DTYPE_BF16, 1, C.byref(rate)) == _lib.L3D_EINVAL
    assert "dtype" in _lib.last_error()
    assert lib.l3d_measure_texture_rate(_lib.DTYPE_F16, 1, None) == _lib.L3D_EINVAL
    assert lib.l3d_memory_trim(-1) == _lib.L3D_EINVAL
    assert "keep_bytes" in _lib.last_error()
    assert lib.l3d_memory_reserved(None, None) == _lib.L3D_EINVAL


def test_python_layer_raises_typed_errors():
    with pytest.raises(_lib.L3dError) as e:
        _lib.check(_lib.L3D_EINVAL)
    assert e.value.status == _lib.L3D_EINVAL
    from luvas3d import trim_memory
    with pytest.raises(_lib.L3dError, match="keep_bytes") as e:
        trim_memory(-1)
    assert e.value.status == _lib.L3D_EINVAL
