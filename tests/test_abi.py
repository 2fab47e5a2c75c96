"""The C-ABI library builds, loads without a GPU and exports exactly what
include/srf_b200.h declares (no compute calls: this runs on CPU-only machines)."""

import ctypes
import os
import re

from srf_b200 import _lib, build

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "srf_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(srf_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("srf_tor_projection", "srf_tor_backprojection", "srf_tor_maplors",
              "srf_siddon_projection", "srf_siddon_backprojection", "srf_siddon_maplors",
              "srf_recon_process", "srf_map_process"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    assert os.path.exists(build.LIBPATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_lib.exported_symbols())


def test_status_strings_without_gpu():
    lib = _lib.load()
    assert lib.srf_status_string(0) == b"ok"
    assert lib.srf_status_string(1) == b"invalid argument"
    assert lib.srf_version() >= 1


def test_invalid_arguments_rejected_before_any_launch():
    """Argument validation happens on the host and returns a status; nothing is
    launched, so this is safe without a GPU."""
    lib = _lib.load()
    g = (ctypes.c_int * 3)(0, 4, 4)  # grid[0] = 0 is invalid
    c = (ctypes.c_float * 3)(0, 0, 0)
    s = (ctypes.c_float * 3)(1, 1, 1)
    st = lib.srf_tor_projection(*([None] * 10), 0, None, g, c, s, 1.0, 1.0, 1.0, None, 0, 1,
                                None)
    assert st == 1
    g2 = (ctypes.c_int * 3)(4, 4, 4)
    st = lib.srf_siddon_projection(*([None] * 7), None, g2, c, s, 1.0, 1.0, None, -1, 1, None)
    assert st == 1
    assert lib.srf_preprocess_workspace_size(-1) == -1
    assert lib.srf_preprocess_workspace_size(10) > 0


def test_new_entry_points_validate_before_any_launch():
    """The fused PSF, the generated-LOR map and the Siddon family switch reject bad
    arguments on the host (status 1 invalid argument, 3 unsupported) without a GPU."""
    lib = _lib.load()
    unsupported = 3
    # PSF: nz above the shared-memory limit, a bad orientation flag, a negative size
    assert lib.srf_psf_apply(None, None, None, 4, 4, None, 300, None, 0, None, 0, None) \
        == unsupported
    assert lib.srf_psf_apply(None, None, None, 4, 4, None, 8, None, 2, None, 0, None) == 1
    assert lib.srf_psf_apply(None, None, None, -1, 4, None, 8, None, 0, None, 0, None) == 1
    # generated map LORs: unknown kind, bad axis, a ring scanner given blocks, a block-pair
    # range past the enumeration's end
    g = (ctypes.c_int * 3)(4, 4, 4)
    c = (ctypes.c_float * 3)(0, 0, 0)
    s = (ctypes.c_float * 3)(1, 1, 1)
    f = lib.srf_tor_maplors_generated
    assert f(2, None, 1, 1, 8, 0, 0, 10, 0, 0, g, c, s, 1.0, None, 0, None) == 1
    assert f(0, None, 1, 1, 8, 0, 0, 10, 3, 0, g, c, s, 1.0, None, 0, None) == 1
    assert f(0, None, 2, 3, 8, 0, 0, 10, 0, 0, g, c, s, 1.0, None, 0, None) == 1
    # 2 rings x 2 blocks x 1 crystal: 2 * (1 * 2 + 1) = 6 pairs
    assert f(1, None, 2, 2, 1, 0, 5, 2, 0, 0, g, c, s, 1.0, None, 0, None) == 1
    assert lib.srf_siddon_set_tuning(2) == 1
    assert lib.srf_siddon_set_tuning(0) == 0


def test_strided_batched_call_validates_strides():
    """The strided batched call rejects missing, non-positive and frame-overrunning image
    strides on the host (status 1), before any launch."""
    lib = _lib.load()
    g = (ctypes.c_int * 3)(4, 5, 6)
    c = (ctypes.c_float * 3)(0, 0, 0)
    s = (ctypes.c_float * 3)(1, 1, 1)
    f = lib.srf_tor_projection_backprojection_batched_strided

    def call(strides, frame_stride=120):
        st = None if strides is None else (ctypes.c_int64 * 3)(*strides)
        # 0 events: no LOR columns needed; images / back_images distinct dummy addresses
        return f(*([None] * 10), 0, None, 2, frame_stride, None, g, c, s, 1.0, 1.0, 1.0,
                 ctypes.c_void_p(4096), ctypes.c_void_p(8192), st, 0, 1, 1, None)

    assert call(None) == 1
    assert call((0, 4, 20)) == 1
    assert call((1, -4, 20)) == 1
    # the frame's last voxel (3 + 4 * 4 + 5 * 30 = 169) must lie below frame_stride
    assert call((1, 4, 30), frame_stride=160) == 1
    # a frame_stride below the grid's voxel count is rejected as for the batched calls
    assert call((1, 4, 20), frame_stride=100) == 1
