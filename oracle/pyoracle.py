"""ctypes bindings to the oracle (``_build/liboracle.so``) and to the reference's own
projectors built by ``oracle/Makefile`` (``_ref/libref_*``).

TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline. The shipped package never
imports this module.

All LOR arrays are the reference's SoA layout, float32, shape ``[ncols, N]``
(TOR ``[10,N]``: x1,y1,z1,x2,y2,z2,xc,yc,zc,sigma2_factor; TOR map ``[7,N]``:
x1..z2,sigma2_factor; Siddon ``[7,N]``: x1..z2,tof). Images are float32 in the
kernel's layout ``[g_slow, g_mid, g_fast]`` with ``grid = (g_fast, g_mid, g_slow)``,
exactly what the reference op sees (``src/python/srf/physics/split_lors.py:79-89``).
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# the SRF checkout: $SRF_REFERENCE, else its location in the build container
DEFAULT_REFERENCE = os.environ.get("SRF_REFERENCE", "/root/reference")

_f = C.c_float
_i64 = C.c_int64
_int = C.c_int
_p = C.c_void_p


def build_oracle():
    """Compile liboracle.so (g++ only; needs no reference checkout)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def build_reference(gpu=True, reference=DEFAULT_REFERENCE):
    """Compile the reference's own sources (host shim, and sm_100a if ``gpu``).

    Only possible where the reference checkout exists; returns False otherwise."""
    if not os.path.isdir(os.path.join(reference, "src", "cpp", "tf_custom_ops")):
        return False
    targets = ["ref-host"] + (["ref-gpu"] if gpu else [])
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + reference] + targets, check=True)
    return True


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        geo = [_p, _p, _p]
        L.oracle_tor_projection_f32.argtypes = [_p, _i64] + geo + [_f, _int, _f, _f, _p, _int, _p]
        L.oracle_tor_projection_f64.argtypes = [_p, _i64] + geo + [_f, _int, _f, _f, _p, _p]
        L.oracle_tor_backprojection_f32.argtypes = [_p, _p, _i64] + geo + [_f, _int, _f, _f, _int, _p]
        L.oracle_tor_backprojection_f64.argtypes = [_p, _p, _i64] + geo + [_f, _int, _f, _f, _p]
        L.oracle_tor_maplors_f32.argtypes = [_p, _p, _i64] + geo + [_f, _int, _int, _p]
        L.oracle_tor_maplors_f64.argtypes = [_p, _p, _i64] + geo + [_f, _int, _p]
        L.oracle_tor_counts.argtypes = [_p, _i64, _int] + geo + [_f, _int, _p, _p, _p]
        L.oracle_siddon_projection_f32.argtypes = [_p, _i64] + geo + [_f, _f, _p, _int, _p]
        L.oracle_siddon_projection_f64.argtypes = [_p, _i64] + geo + [_f, _f, _p, _p]
        L.oracle_siddon_backprojection_f32.argtypes = [_p, _p, _i64] + geo + [_f, _f, _int, _p]
        L.oracle_siddon_backprojection_f64.argtypes = [_p, _p, _i64] + geo + [_f, _f, _p]
        L.oracle_siddon_maplors_f32.argtypes = [_p, _p, _i64] + geo + [_int, _p]
        L.oracle_siddon_maplors_f64.argtypes = [_p, _p, _i64] + geo + [_p]
        L.oracle_siddon_counts.argtypes = [_p, _i64] + geo + [_p]
        for name in ("oracle_siddon_projection_f32", "oracle_siddon_projection_f64",
                     "oracle_siddon_backprojection_f32", "oracle_siddon_backprojection_f64",
                     "oracle_siddon_maplors_f32", "oracle_siddon_maplors_f64",
                     "oracle_siddon_counts"):
            getattr(L, name).restype = _i64
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(_p)


def _soa(lors, ncols):
    a = np.ascontiguousarray(lors, dtype=np.float32)
    assert a.ndim == 2 and a.shape[0] == ncols, a.shape
    return a


def _geom(grid, center, size):
    g = np.ascontiguousarray(grid, dtype=np.int32)
    c = np.ascontiguousarray(center, dtype=np.float32)
    s = np.ascontiguousarray(size, dtype=np.float32)
    return g, c, s


def _nvox(grid):
    return int(grid[0]) * int(grid[1]) * int(grid[2])


def _image_shape(grid):
    return (int(grid[2]), int(grid[1]), int(grid[0]))


# ----------------------------------------------------------------------------- TOR


def tor_projection(lors, image, grid, center, size, kernel_width, geo_sigma2_flag, tof_bin,
                   tof_sigma2, mode="f32", contract=True):
    lors = _soa(lors, 10)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    img = np.ascontiguousarray(image, dtype=np.float32)
    assert img.size == _nvox(g)
    if mode == "f32":
        out = np.zeros(n, np.float32)
        lib().oracle_tor_projection_f32(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s), kernel_width,
                                        int(geo_sigma2_flag), tof_bin, tof_sigma2, _ptr(img),
                                        int(contract), _ptr(out))
    else:
        out = np.zeros(n, np.float64)
        lib().oracle_tor_projection_f64(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s), kernel_width,
                                        int(geo_sigma2_flag), tof_bin, tof_sigma2, _ptr(img),
                                        _ptr(out))
    return out


def tor_backprojection(lors, lors_value, grid, center, size, kernel_width, geo_sigma2_flag,
                       tof_bin, tof_sigma2, mode="f32", contract=True):
    lors = _soa(lors, 10)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    v = np.ascontiguousarray(lors_value, dtype=np.float32)
    assert v.size == n
    if mode == "f32":
        out = np.zeros(_image_shape(g), np.float32)
        lib().oracle_tor_backprojection_f32(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                            kernel_width, int(geo_sigma2_flag), tof_bin,
                                            tof_sigma2, int(contract), _ptr(out))
    else:
        out = np.zeros(_image_shape(g), np.float64)
        lib().oracle_tor_backprojection_f64(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                            kernel_width, int(geo_sigma2_flag), tof_bin,
                                            tof_sigma2, _ptr(out))
    return out


def tor_maplors(lors, lors_value, grid, center, size, kernel_width, geo_sigma2_flag, mode="f32",
                contract=True):
    lors = _soa(lors, 7)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    v = np.ascontiguousarray(lors_value, dtype=np.float32)
    if mode == "f32":
        out = np.zeros(_image_shape(g), np.float32)
        lib().oracle_tor_maplors_f32(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                     kernel_width, int(geo_sigma2_flag), int(contract), _ptr(out))
    else:
        out = np.zeros(_image_shape(g), np.float64)
        lib().oracle_tor_maplors_f64(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                     kernel_width, int(geo_sigma2_flag), _ptr(out))
    return out


def tor_counts(lors, grid, center, size, kernel_width, geo_sigma2_flag=False):
    """Per-LOR (slots, useful, slices): patch voxels visited by the reference, those
    with non-zero weight, and slices crossed."""
    lors = np.ascontiguousarray(lors, dtype=np.float32)
    ncols, n = lors.shape
    g, c, s = _geom(grid, center, size)
    slots = np.zeros(n, np.int64)
    useful = np.zeros(n, np.int64)
    slices = np.zeros(n, np.int64)
    lib().oracle_tor_counts(_ptr(lors), n, ncols, _ptr(g), _ptr(c), _ptr(s), kernel_width,
                            int(geo_sigma2_flag), _ptr(slots), _ptr(useful), _ptr(slices))
    return slots, useful, slices


# -------------------------------------------------------------------------- Siddon


def siddon_projection(lors, image, grid, center, size, tof_bin, tof_sigma2, mode="f32",
                      contract=True, return_bad=False):
    lors = _soa(lors, 7)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    img = np.ascontiguousarray(image, dtype=np.float32)
    if mode == "f32":
        out = np.zeros(n, np.float32)
        bad = lib().oracle_siddon_projection_f32(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s),
                                                 tof_bin, tof_sigma2, _ptr(img), int(contract),
                                                 _ptr(out))
    else:
        out = np.zeros(n, np.float64)
        bad = lib().oracle_siddon_projection_f64(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s),
                                                 tof_bin, tof_sigma2, _ptr(img), _ptr(out))
    return (out, bad) if return_bad else out


def siddon_backprojection(lors, lors_value, grid, center, size, tof_bin, tof_sigma2, mode="f32",
                          contract=True):
    lors = _soa(lors, 7)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    v = np.ascontiguousarray(lors_value, dtype=np.float32)
    if mode == "f32":
        out = np.zeros(_image_shape(g), np.float32)
        lib().oracle_siddon_backprojection_f32(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                               tof_bin, tof_sigma2, int(contract), _ptr(out))
    else:
        out = np.zeros(_image_shape(g), np.float64)
        lib().oracle_siddon_backprojection_f64(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                               tof_bin, tof_sigma2, _ptr(out))
    return out


def siddon_maplors(lors, lors_value, grid, center, size, mode="f32", contract=True):
    lors = np.ascontiguousarray(lors, dtype=np.float32)
    assert lors.shape[0] >= 6
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    v = np.ascontiguousarray(lors_value, dtype=np.float32)
    if mode == "f32":
        out = np.zeros(_image_shape(g), np.float32)
        lib().oracle_siddon_maplors_f32(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                        int(contract), _ptr(out))
    else:
        out = np.zeros(_image_shape(g), np.float64)
        lib().oracle_siddon_maplors_f64(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                        _ptr(out))
    return out


def siddon_counts(lors, grid, center, size):
    """Per-LOR voxel visits and the number of rays whose start voxel is off-grid."""
    lors = np.ascontiguousarray(lors, dtype=np.float32)
    n = lors.shape[1]
    g, c, s = _geom(grid, center, size)
    visits = np.zeros(n, np.int64)
    bad = lib().oracle_siddon_counts(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s), _ptr(visits))
    return visits, bad


# ------------------------------------------------- the reference's own compiled code


class ReferenceHost:
    """The reference's projector sources compiled for the CPU (oracle/_ref)."""

    def __init__(self):
        tor = os.path.join(REF_DIR, "libref_tor_host.so")
        sid = os.path.join(REF_DIR, "libref_siddon_host.so")
        if not (os.path.exists(tor) and os.path.exists(sid)):
            raise FileNotFoundError("reference host build missing (make -C oracle ref-host)")
        self.tor = C.CDLL(tor)
        self.sid = C.CDLL(sid)
        geo = [_p, _p, _p]
        self.tor.ref_tor_projection.argtypes = [_p, _i64] + geo + [_f, _int, _f, _f, _p, _p, _int]
        self.tor.ref_tor_backprojection.argtypes = [_p, _p, _i64] + geo + [_f, _int, _f, _f, _p, _int]
        self.tor.ref_tor_maplors.argtypes = [_p, _p, _i64] + geo + [_f, _int, _p, _int]
        self.sid.ref_siddon_projection.argtypes = [_p, _i64] + geo + [_f, _f, _p, _p, _int]
        self.sid.ref_siddon_backprojection.argtypes = [_p, _p, _i64] + geo + [_f, _f, _p, _int]
        self.sid.ref_siddon_maplors.argtypes = [_p, _p, _i64] + geo + [_p, _int]

    @staticmethod
    def available():
        return all(os.path.exists(os.path.join(REF_DIR, f))
                   for f in ("libref_tor_host.so", "libref_siddon_host.so"))

    def tor_projection(self, lors, image, grid, center, size, kernel_width, geo_sigma2_flag,
                       tof_bin, tof_sigma2, nthreads=1):
        lors = _soa(lors, 10)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        img = np.ascontiguousarray(image, dtype=np.float32)
        out = np.zeros(n, np.float32)
        self.tor.ref_tor_projection(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s), kernel_width,
                                    int(geo_sigma2_flag), tof_bin, tof_sigma2, _ptr(img),
                                    _ptr(out), nthreads)
        return out

    def tor_backprojection(self, lors, lors_value, grid, center, size, kernel_width,
                           geo_sigma2_flag, tof_bin, tof_sigma2, nthreads=1):
        lors = _soa(lors, 10)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        v = np.ascontiguousarray(lors_value, dtype=np.float32)
        out = np.zeros(_image_shape(g), np.float32)
        self.tor.ref_tor_backprojection(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                        kernel_width, int(geo_sigma2_flag), tof_bin, tof_sigma2,
                                        _ptr(out), nthreads)
        return out

    def tor_maplors(self, lors, lors_value, grid, center, size, kernel_width, geo_sigma2_flag,
                    nthreads=1):
        lors = _soa(lors, 7)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        v = np.ascontiguousarray(lors_value, dtype=np.float32)
        out = np.zeros(_image_shape(g), np.float32)
        self.tor.ref_tor_maplors(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s), kernel_width,
                                 int(geo_sigma2_flag), _ptr(out), nthreads)
        return out

    def siddon_projection(self, lors, image, grid, center, size, tof_bin, tof_sigma2,
                          nthreads=1):
        lors = _soa(lors, 7)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        img = np.ascontiguousarray(image, dtype=np.float32)
        out = np.zeros(n, np.float32)
        self.sid.ref_siddon_projection(_ptr(lors), n, _ptr(g), _ptr(c), _ptr(s), tof_bin,
                                       tof_sigma2, _ptr(img), _ptr(out), nthreads)
        return out

    def siddon_backprojection(self, lors, lors_value, grid, center, size, tof_bin, tof_sigma2,
                              nthreads=1):
        lors = _soa(lors, 7)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        v = np.ascontiguousarray(lors_value, dtype=np.float32)
        out = np.zeros(_image_shape(g), np.float32)
        self.sid.ref_siddon_backprojection(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                           tof_bin, tof_sigma2, _ptr(out), nthreads)
        return out

    def siddon_maplors(self, lors, lors_value, grid, center, size, nthreads=1):
        lors = _soa(lors, 7)
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        v = np.ascontiguousarray(lors_value, dtype=np.float32)
        out = np.zeros(_image_shape(g), np.float32)
        self.sid.ref_siddon_maplors(_ptr(lors), _ptr(v), n, _ptr(g), _ptr(c), _ptr(s),
                                    _ptr(out), nthreads)
        return out


class ReferenceGPU:
    """The reference's own CUDA kernels built for sm_100a (oracle/_ref/libref_*_gpu.so).

    Takes torch CUDA tensors (data pointers are passed through). The reference
    launchers synchronise the device; each call returns after its kernels finished.
    Only run on inputs the oracle has checked (``siddon_counts`` reports rays whose
    first voxel would fall off the grid, which the reference would read out of bounds)."""

    def __init__(self):
        tor = os.path.join(REF_DIR, "libref_tor_gpu.so")
        sid = os.path.join(REF_DIR, "libref_siddon_gpu.so")
        if not (os.path.exists(tor) and os.path.exists(sid)):
            raise FileNotFoundError("reference GPU build missing (make -C oracle ref-gpu)")
        self.tor = C.CDLL(tor)
        self.sid = C.CDLL(sid)
        geo = [_p, _p, _p]
        self.tor.refgpu_tor_projection.argtypes = [_p, _i64] + geo + [_f, _int, _f, _f, _p, _p]
        self.tor.refgpu_tor_backprojection.argtypes = [_p, _p, _i64] + geo + [_f, _int, _f, _f, _p]
        self.tor.refgpu_tor_maplors.argtypes = [_p, _p, _i64] + geo + [_f, _int, _p]
        self.sid.refgpu_siddon_projection.argtypes = [_p, _i64] + geo + [_f, _f, _p, _p]
        self.sid.refgpu_siddon_backprojection.argtypes = [_p, _p, _i64] + geo + [_f, _f, _p]
        self.sid.refgpu_siddon_maplors.argtypes = [_p, _p, _i64] + geo + [_p]

    @staticmethod
    def available():
        return all(os.path.exists(os.path.join(REF_DIR, f))
                   for f in ("libref_tor_gpu.so", "libref_siddon_gpu.so"))

    @staticmethod
    def _check(rc, what):
        if rc != 0:
            raise RuntimeError(f"reference GPU {what} failed with CUDA error {rc}")

    def tor_projection(self, lors, image, grid, center, size, kw, geo, tof_bin, tof_sigma2):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(n, dtype=torch.float32, device=lors.device)
        self._check(self.tor.refgpu_tor_projection(lors.data_ptr(), n, _ptr(g), _ptr(c), _ptr(s),
                                                   kw, int(geo), tof_bin, tof_sigma2,
                                                   image.data_ptr(), out.data_ptr()), "proj")
        return out

    def tor_backprojection(self, lors, values, grid, center, size, kw, geo, tof_bin,
                           tof_sigma2):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(_image_shape(g), dtype=torch.float32, device=lors.device)
        self._check(self.tor.refgpu_tor_backprojection(lors.data_ptr(), values.data_ptr(), n,
                                                       _ptr(g), _ptr(c), _ptr(s), kw, int(geo),
                                                       tof_bin, tof_sigma2, out.data_ptr()),
                    "bproj")
        return out

    def tor_maplors(self, lors, values, grid, center, size, kw, geo):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(_image_shape(g), dtype=torch.float32, device=lors.device)
        self._check(self.tor.refgpu_tor_maplors(lors.data_ptr(), values.data_ptr(), n, _ptr(g),
                                                _ptr(c), _ptr(s), kw, int(geo), out.data_ptr()),
                    "map")
        return out

    def siddon_projection(self, lors, image, grid, center, size, tof_bin, tof_sigma2):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(n, dtype=torch.float32, device=lors.device)
        self._check(self.sid.refgpu_siddon_projection(lors.data_ptr(), n, _ptr(g), _ptr(c),
                                                      _ptr(s), tof_bin, tof_sigma2,
                                                      image.data_ptr(), out.data_ptr()), "proj")
        return out

    def siddon_backprojection(self, lors, values, grid, center, size, tof_bin, tof_sigma2):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(_image_shape(g), dtype=torch.float32, device=lors.device)
        self._check(self.sid.refgpu_siddon_backprojection(lors.data_ptr(), values.data_ptr(), n,
                                                          _ptr(g), _ptr(c), _ptr(s), tof_bin,
                                                          tof_sigma2, out.data_ptr()), "bproj")
        return out

    def siddon_maplors(self, lors, values, grid, center, size):
        import torch
        n = lors.shape[1]
        g, c, s = _geom(grid, center, size)
        out = torch.empty(_image_shape(g), dtype=torch.float32, device=lors.device)
        self._check(self.sid.refgpu_siddon_maplors(lors.data_ptr(), values.data_ptr(), n,
                                                   _ptr(g), _ptr(c), _ptr(s), out.data_ptr()),
                    "map")
        return out
