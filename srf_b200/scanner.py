"""Scanner geometry, TOF constants and task-config parsing.

* ``tof_info`` — ``SRFApp._get_tof_info`` (src/python/srf/api/app/srfapp_new.py:244-251).
* ``CylindricalPET`` — the ring scanner of src/python/srf/scanner/pet/pet.py:55-177 with
  crystal centres from ``RingBlock.get_meshes`` (src/python/srf/scanner/pet/block.py:73-109)
  and the ring/block expansion of ``modified_ring_scanner``
  (src/python/srf/function/scanner.py:22-26).
* ``RingScanner`` — the simplified crystal ring used by the synthetic workloads:
  ``n_crystals`` crystals per ring at radius R, ``n_rings`` rings at a fixed pitch.
* ``load_task_config`` — accepts the ``srfapp_new`` schema (``scanner.petscanner.*``)
  and the older resource schema (``scanner.ring`` ...; resource/recon_task.json).
"""

import json
import math
from dataclasses import dataclass

import numpy as np

GAUSSIAN_FACTOR = 2.35482005
TOF_OFF = (1.0e4, 1.0e4)  # PETScanner default TOF(res, bin) in ps (scanner/pet/pet.py:25-26)


def tof_info(tof_res_ps, tof_bin_ps):
    """(tof_bin [mm], tof_sigma2 [mm^2]) from resolution and bin in ps."""
    limit = tof_res_ps * 0.15 / GAUSSIAN_FACTOR * 3
    return tof_bin_ps * 0.15, (limit ** 2) / 9


@dataclass
class RingScanner:
    radius: float
    n_crystals: int
    n_rings: int
    pitch: float

    @property
    def axial_length(self):
        return self.n_rings * self.pitch

    @property
    def inner_radius(self):
        return self.radius

    def crystal_positions(self):
        """[n_rings * n_crystals, 3] float32: ring-major crystal centres."""
        k = np.arange(self.n_crystals)
        phi = 2 * np.pi * k / self.n_crystals
        z = (np.arange(self.n_rings) - (self.n_rings - 1) / 2) * self.pitch
        x = np.tile(self.radius * np.cos(phi), self.n_rings)
        y = np.tile(self.radius * np.sin(phi), self.n_rings)
        zz = np.repeat(z, self.n_crystals)
        return np.stack([x, y, zz], 1).astype(np.float32)


class CylindricalPET:
    """Ring-of-blocks scanner (scanner/pet/pet.py:55-177)."""

    def __init__(self, inner_radius, outer_radius, axial_length, nb_rings, nb_blocks_per_ring,
                 gap, block_grid, block_size, tof_res=TOF_OFF[0], tof_bin=TOF_OFF[1],
                 name="default"):
        self.inner_radius = float(inner_radius)
        self.outer_radius = float(outer_radius)
        self.axial_length = float(axial_length)
        self.nb_rings = int(nb_rings)
        self.nb_blocks_per_ring = int(nb_blocks_per_ring)
        self.gap = float(gap)
        self.block_grid = [int(g) for g in block_grid]
        self.block_size = [float(s) for s in block_size]
        self.tof_res = tof_res
        self.tof_bin = tof_bin
        self.name = name

    @classmethod
    def from_config(cls, petscanner):
        """``make_scanner`` + ``modified_ring_scanner`` (function/scanner.py:5-26)."""
        ring, block = dict(petscanner["ring"]), dict(petscanner["block"])
        grid = list(block["grid"])
        size = list(block["size"])
        nb_rings = ring["nb_rings"] * grid[2]
        size[2] = size[2] / grid[2]
        grid[2] = 1
        tof = petscanner.get("tof")
        res, bin_ = (tof["resolution"], tof["bin"]) if tof else TOF_OFF
        return cls(ring["inner_radius"], ring["outer_radius"], ring["axial_length"], nb_rings,
                   ring["nb_blocks_per_ring"], ring["gap"], grid, size, res, bin_,
                   petscanner.get("name", "default"))

    def ring_z(self, ir):
        bz = self.block_size[2]
        bottom = -(bz + self.gap) * (self.nb_rings - 1) / 2
        return bottom + ir * (bz + self.gap)

    def block_meshes(self, ir, ib):
        """Crystal centres of block ``ib`` of ring ``ir`` ([n, 3]), in the enumeration
        order of ``RingBlock.get_meshes`` (np.meshgrid 'xy': y-major, then x, then z)."""
        size = np.array(self.block_size)
        grid = np.array(self.block_grid)
        center = np.array([(self.inner_radius + self.outer_radius) / 2, 0.0, self.ring_z(ir)])
        interval = size / grid
        p0 = center - (size - interval) / 2
        p1 = center + (size - interval) / 2
        r = [np.linspace(p0[i], p1[i], grid[i]) for i in range(3)]
        m = np.array(np.meshgrid(r[0], r[1], r[2])).reshape((3, -1))
        a = ib * 2 * np.pi / self.nb_blocks_per_ring
        rot = np.array([[math.cos(a), -math.sin(a), 0.0], [math.sin(a), math.cos(a), 0.0],
                        [0.0, 0.0, 1.0]])
        return (rot @ m).T

    def crystal_table(self):
        """[nb_rings * nb_blocks_per_ring * crystals per block, 3] float32 crystal centres,
        ring major, then block, then the block's mesh order (``block_meshes``): the table
        the generated block-pair LORs index (``synthetic.GeneratedPairs.block_pairs``)."""
        return np.vstack([self.block_meshes(ir, ib) for ir in range(self.nb_rings)
                          for ib in range(self.nb_blocks_per_ring)]).astype(np.float32)

    @staticmethod
    def block_pairs(n_blocks, same_ring):
        """Block index pairs of ``make_block_pairs`` (scanner/pet/pet.py:149-168)."""
        if same_ring:
            return [(i, j) for i in range(n_blocks) for j in range(n_blocks) if i < j]
        return [(i, j) for i in range(n_blocks) for j in range(n_blocks) if i != j]

    def make_ring_pairs_lors(self, ir1, ir2):
        """[N, 6] LORs of every crystal pair between the blocks of two rings
        (``make_ring_pairs_lors``, scanner/pet/pet.py:170-177)."""
        out = []
        for i, j in self.block_pairs(self.nb_blocks_per_ring, ir1 == ir2):
            m0 = self.block_meshes(ir1, i)
            m1 = self.block_meshes(ir2, j)
            a = np.repeat(m0, len(m1), 0)
            b = np.tile(m1, (len(m0), 1))
            out.append(np.hstack([a, b]))
        return np.vstack(out) if out else np.zeros((0, 6))


def load_task_config(path_or_dict):
    """Parse a recon/map task JSON, normalising the older resource schema
    (``scanner.ring``) to the ``srfapp_new`` one (``scanner.petscanner.ring``)."""
    cfg = path_or_dict
    if not isinstance(cfg, dict):
        with open(cfg) as f:
            cfg = json.load(f)
    cfg = json.loads(json.dumps(cfg))
    sc = cfg.get("scanner", {})
    if "petscanner" not in sc and "ring" in sc:
        cfg["scanner"] = {"petscanner": sc}
    alg = cfg.setdefault("algorithm", {})
    pm = alg.setdefault("projection_model", {})
    if "tor" in pm:
        pm["tor"].setdefault("geometry_sigma2_correction", False)
    out = cfg.setdefault("output", {})
    img = out.setdefault("image", {})
    if "path_file" in out and "path_dataset_prefix" not in img:
        img["path_dataset_prefix"] = out["path_file"].rsplit(".", 1)[0]
    return cfg
