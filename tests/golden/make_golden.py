"""Generate tests/golden/reference_outputs.npz from the reference itself.

Run in a container that has the SRF checkout (``--reference``, else $SRF_REFERENCE, else
/root/reference):

    python tests/golden/make_golden.py [--reference PATH]

* LOR preprocessing: the reference's own ``on_tor_lors.py``
  (src/python/srf/preprocess/function/on_tor_lors.py) is imported by path. Its only
  dependency, the authors' ``doufo`` helper package (doufo==0.0.4, not installed here),
  supplies function-composition wrappers (``WrappedFunction``, ``func``, ``>>``) and
  ``abs_``; a minimal stand-in with that behaviour is installed in ``sys.modules`` for
  the import. All numpy arithmetic is the reference's.
* Projectors: the reference's own ``tor.cu.cc`` / ``siddon.cu.cc`` compiled for the
  host by ``oracle/Makefile`` (target ref-host).

The fixture holds only seeded synthetic inputs and these outputs.
"""

import argparse
import dataclasses
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "reference_outputs.npz")


def _install_doufo_standin():
    class _Composable:
        def __rshift__(self, other):
            first = self
            return _Fn(lambda *a: other(first(*a)))

    class _Fn(_Composable):
        def __init__(self, f):
            self.f = f

        def __call__(self, *a):
            return self.f(*a)

    class WrappedFunction(_Composable):
        def __call__(self, *a):
            return self.f(*a)

    def func(nargs=None, nouts=None):
        return lambda f: _Fn(f)

    doufo = types.ModuleType("doufo")
    doufo.WrappedFunction = WrappedFunction
    doufo.Function = _Fn
    doufo.func = func
    doufo.dataclass = dataclasses.dataclass
    tensor = types.ModuleType("doufo.tensor")
    tensor.abs_ = np.abs
    tensor.norm = np.linalg.norm
    doufo.tensor = tensor
    sys.modules["doufo"] = doufo
    sys.modules["doufo.tensor"] = tensor


def load_reference_preprocessing(reference):
    _install_doufo_standin()
    path = os.path.join(reference, "src", "python", "srf", "preprocess", "function",
                        "on_tor_lors.py")
    spec = importlib.util.spec_from_file_location("srf_ref_on_tor_lors", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference",
                    default=os.environ.get("SRF_REFERENCE", "/root/reference"))
    a = ap.parse_args(argv)

    from oracle import pyoracle as O
    from tests import _cases as K

    ref_pre = load_reference_preprocessing(a.reference)
    if not O.ReferenceHost.available():
        O.build_reference(gpu=False, reference=a.reference)
    R = O.ReferenceHost()

    out = {}
    # ---- TOR: events (ring scanner + box events), preprocessing, projectors
    tof_res = 530.0
    ev = np.vstack([K.events(700, 101, tof_res), K.box_events(300, 102)]).astype(np.float32)
    groups = ref_pre.recon_process(ev.copy(), tof_res)
    grid, voxel = (32, 32, 16), 12.8
    size = [g * voxel for g in grid]
    center = [0.0, 0.0, 0.0]
    image = K.phantom_image(grid, voxel, seed=9)
    b, s2 = K.tof_params(tof_res)
    kw = float(np.float32(K.KW_CONFIG))
    out.update(tor_events=ev, tor_image=image, grid=np.array(grid, np.int32),
               center=np.array(center, np.float32), size=np.array(size, np.float32),
               tor_params=np.array([kw, b, s2, tof_res], np.float64))
    for ax, key in zip("xyz", (ref_pre.Axis.x, ref_pre.Axis.y, ref_pre.Axis.z)):
        g = np.asarray(groups[key], np.float32)
        out[f"pre_{ax}"] = g
        img, kg, kc, ks = K.P.axis_view(image, center, size, ax)
        lors = np.ascontiguousarray(g.T)
        pv = R.tor_projection(lors, img, kg, kc, ks, kw, False, b, s2)
        out[f"tor_proj_{ax}"] = pv
        pv_in = pv.copy()
        pv_in[::5] = 0.0
        out[f"tor_bproj_in_{ax}"] = pv_in
        out[f"tor_bproj_{ax}"] = R.tor_backprojection(lors, pv_in, kg, kc, ks, kw, False, b, s2)
        out[f"tor_proj_geo_{ax}"] = R.tor_projection(lors, img, kg, kc, ks, kw, True, b, s2)

    # ---- TOR map: random crystal pairs through the reference's map_process
    mlors = K.random_lors(1000, K.SCANNER, 103).numpy()
    mlors = np.vstack([mlors, K.box_events(200, 104)[:, :6]]).astype(np.float32)
    mgroups = ref_pre.map_process(mlors.copy())
    out["map_lors"] = mlors
    for ax, key in zip("xyz", (ref_pre.Axis.x, ref_pre.Axis.y, ref_pre.Axis.z)):
        g = np.asarray(mgroups[key], np.float32)
        out[f"map_pre_{ax}"] = g
        _, kg, kc, ks = K.P.axis_view(image, center, size, ax)
        ones = np.ones(g.shape[0], np.float32)
        out[f"tor_map_{ax}"] = R.tor_maplors(np.ascontiguousarray(g.T), ones, kg, kc, ks, kw,
                                             False)

    # ---- Siddon: complete LORs, kernel-layout image [nz,ny,nx]
    sg, sv = (32, 32, 16), 6.8
    ssize = [g * sv for g in sg]
    simg = np.ascontiguousarray(np.transpose(K.phantom_image(sg, sv, seed=10), (2, 1, 0)))
    sev = np.vstack([K.events(800, 105, tof_res), K.box_events(200, 106)]).astype(np.float32)
    slors = np.ascontiguousarray(sev.T)
    out.update(sid_lors=slors, sid_image=simg, sid_grid=np.array(sg, np.int32),
               sid_size=np.array(ssize, np.float32))
    for tag, s2x in (("tof", s2), ("notof", 1.0e6)):
        pv = R.siddon_projection(slors, simg, sg, center, ssize, b, s2x)
        out[f"sid_proj_{tag}"] = pv
        out[f"sid_bproj_{tag}"] = R.siddon_backprojection(slors, pv, sg, center, ssize, b, s2x)
    out["sid_map"] = R.siddon_maplors(slors, np.ones(slors.shape[1], np.float32), sg, center,
                                      ssize)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
