"""Seeded synthetic list-mode workloads (the shapes of the benchmark configurations).

No public dataset is involved: every event list is generated here from a fixed seed.

Event model. Emission points are drawn with density proportional to the phantom's
activity (rejection sampling in its bounding box), each with an isotropic direction.
The line is intersected with the detector cylinder r = R; events whose two ends fall
outside the axial extent are dropped; each end is snapped to the nearest crystal centre
(crystals at r = R, phi_k = 2 pi k / n_c, z_j = (j - (n_r - 1)/2) pitch). The TOF column
follows the reference's convention (CutLoRs, on_tor_lors.py:210-215, and siddon.cu.cc:460):
for an emission at distance d from the first endpoint along a LOR of length L,
t = L/2 - d + eps, eps ~ N(0, sigma_TOF).

Random LORs for the efficiency map are uniform crystal pairs with different crystals.

All generation runs in torch on the requested device (CUDA for the large workloads).
"""

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from .scanner import RingScanner


@dataclass
class Sphere:
    center: tuple
    radius: float
    activity: float


@dataclass
class Cylinder:
    """A cylinder parallel to z: axis at (x, y), radius, axial range [z_lo, z_hi]."""

    xy: tuple
    radius: float
    z_lo: float
    z_hi: float
    activity: float


@dataclass
class Phantom:
    """A uniform cylinder (axis z) plus inner cylinders, then spheres. Each later shape's
    activity replaces what lies under it (inner cylinders in list order, then spheres)."""

    radius: float = 100.0
    half_length: float = 51.2
    activity: float = 1.0
    spheres: list = field(default_factory=list)
    cylinders: list = field(default_factory=list)

    @property
    def max_activity(self):
        return max([self.activity] + [s.activity for s in self.spheres]
                   + [c.activity for c in self.cylinders])

    def activity_at(self, p):
        """Activity at points p [N,3] (torch)."""
        r2 = p[:, 0] ** 2 + p[:, 1] ** 2
        a = torch.where((r2 <= self.radius ** 2) & (p[:, 2].abs() <= self.half_length),
                        torch.full_like(r2, self.activity), torch.zeros_like(r2))
        for c in self.cylinders:
            inside = (((p[:, 0] - c.xy[0]) ** 2 + (p[:, 1] - c.xy[1]) ** 2 <= c.radius ** 2)
                      & (p[:, 2] >= c.z_lo) & (p[:, 2] <= c.z_hi))
            a = torch.where(inside, torch.full_like(a, c.activity), a)
        for s in self.spheres:
            c = torch.tensor(s.center, dtype=p.dtype, device=p.device)
            inside = ((p - c) ** 2).sum(1) <= s.radius ** 2
            a = torch.where(inside, torch.full_like(a, s.activity), a)
        return a

    def voxelize(self, grid, center, size, oversample=2):
        """Mean activity per voxel on an [nx,ny,nz] grid (numpy float32)."""
        grid = [int(g) for g in grid]
        axes = []
        for k in range(3):
            v = size[k] / grid[k]
            sub = (np.arange(grid[k] * oversample) + 0.5) * v / oversample
            axes.append(torch.tensor(center[k] - size[k] / 2 + sub, dtype=torch.float64))
        X, Y, Z = torch.meshgrid(*axes, indexing="ij")
        a = self.activity_at(torch.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1))
        a = a.reshape(grid[0], oversample, grid[1], oversample, grid[2], oversample)
        return a.mean(dim=(1, 3, 5)).numpy().astype(np.float32)


def standard_phantom(half_length=51.2, radius=100.0):
    """Cylinder r = 100 mm, activity 1, with four r = 5 mm hot spheres at 4:1."""
    z = min(20.0, half_length * 0.5)
    return Phantom(radius=radius, half_length=half_length, activity=1.0, spheres=[
        Sphere((50.0, 0.0, 0.0), 5.0, 4.0), Sphere((-50.0, 0.0, 0.0), 5.0, 4.0),
        Sphere((0.0, 50.0, z), 5.0, 4.0), Sphere((0.0, -50.0, -z), 5.0, 4.0)])


def large_fov_phantom(half_length=500.0, radius=200.0):
    """Large axial FOV multi-cylinder phantom: a body cylinder r = 200 mm (activity 1)
    over the whole axial length; an off-centre cylinder r = 60 mm at 2:1 over the
    central 60 % of it and a cold (activity 0.25) centred cylinder r = 40 mm over the
    outer axial thirds; and eight cylindrical inserts of 80 mm length along the axis,
    alternating around it at 120 mm from the centre, four hot (4:1, r = 20 mm) and four
    cold (activity 0, r = 25 mm)."""
    cyl = [Cylinder((-70.0, 40.0), 60.0, -0.6 * half_length, 0.6 * half_length, 2.0),
           Cylinder((0.0, 0.0), 40.0, -half_length, -half_length / 3.0, 0.25),
           Cylinder((0.0, 0.0), 40.0, half_length / 3.0, half_length, 0.25)]
    for k in range(8):
        z = (k - 3.5) / 4.0 * half_length * 0.9
        ph = k * math.pi / 4.0
        hot = k % 2 == 0
        cyl.append(Cylinder((120.0 * math.cos(ph), 120.0 * math.sin(ph)),
                            20.0 if hot else 25.0, z - 40.0, z + 40.0, 4.0 if hot else 0.0))
    return Phantom(radius=radius, half_length=half_length, activity=1.0, cylinders=cyl)


def random_phantom(seed, half_length, r_lo=60.0, r_hi=150.0):
    """Per-frame phantom of the batched workload: radius U(r_lo, r_hi), four spheres
    at seeded positions inside it."""
    g = np.random.default_rng(seed)
    r = float(g.uniform(r_lo, r_hi))
    spheres = []
    for _ in range(4):
        rr = g.uniform(0.2, 0.7) * r
        ph = g.uniform(0, 2 * np.pi)
        z = g.uniform(-0.6, 0.6) * half_length
        spheres.append(Sphere((rr * math.cos(ph), rr * math.sin(ph), z), 5.0, 4.0))
    return Phantom(radius=r, half_length=half_length, activity=1.0, spheres=spheres)


def _snap(p, sc):
    """Nearest crystal centre of points on the cylinder; returns [N,3] float32 and a
    validity mask (inside the axial extent)."""
    phi = torch.atan2(p[:, 1], p[:, 0])
    dphi = 2 * math.pi / sc.n_crystals
    k = torch.round(phi / dphi).remainder(sc.n_crystals)
    zj = p[:, 2] / sc.pitch + (sc.n_rings - 1) / 2
    j = torch.round(zj)
    ok = (j >= 0) & (j <= sc.n_rings - 1)
    ang = k * dphi
    out = torch.stack([sc.radius * torch.cos(ang), sc.radius * torch.sin(ang),
                       (j - (sc.n_rings - 1) / 2) * sc.pitch], 1)
    return out.to(torch.float32), ok, (k + j * sc.n_crystals).long()


def generate_events(n_events, scanner, phantom, seed, tof_sigma_mm=None, device="cpu",
                    batch=1 << 22):
    """[n_events, 7] float32 (x1,y1,z1,x2,y2,z2,tof) on ``device``."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    out = []
    have = 0
    R = scanner.radius
    half = scanner.axial_length / 2
    hl = min(phantom.half_length, half)
    box = torch.tensor([phantom.radius, phantom.radius, hl], dtype=torch.float64, device=dev)
    amax = phantom.max_activity
    while have < n_events:
        p = (torch.rand(batch, 3, generator=g, device=dev, dtype=torch.float64) * 2 - 1) * box
        keep = torch.rand(batch, generator=g, device=dev, dtype=torch.float64) * amax < \
            phantom.activity_at(p)
        p = p[keep]
        m = p.shape[0]
        if m == 0:
            continue
        u = torch.randn(m, 3, generator=g, device=dev, dtype=torch.float64)
        u = u / u.norm(dim=1, keepdim=True)
        # |p_xy + t u_xy| = R
        a = u[:, 0] ** 2 + u[:, 1] ** 2
        b = 2 * (p[:, 0] * u[:, 0] + p[:, 1] * u[:, 1])
        c = p[:, 0] ** 2 + p[:, 1] ** 2 - R * R
        disc = torch.clamp(b * b - 4 * a * c, min=0)
        sq = torch.sqrt(disc)
        a = torch.clamp(a, min=1e-12)
        t1 = (-b - sq) / (2 * a)
        t2 = (-b + sq) / (2 * a)
        e1 = p + t1[:, None] * u
        e2 = p + t2[:, None] * u
        ok = (e1[:, 2].abs() <= half) & (e2[:, 2].abs() <= half)
        c1, ok1, id1 = _snap(e1, scanner)
        c2, ok2, id2 = _snap(e2, scanner)
        ok = ok & ok1 & ok2 & (id1 != id2)
        c1, c2, p = c1[ok], c2[ok], p[ok]
        if c1.shape[0] == 0:
            continue
        d = (c2 - c1).double()
        L = d.norm(dim=1)
        dist = ((p - c1.double()) * d).sum(1) / L
        t = L / 2 - dist
        if tof_sigma_mm is not None and tof_sigma_mm > 0:
            t = t + tof_sigma_mm * torch.randn(t.shape[0], generator=g, device=dev,
                                               dtype=torch.float64)
        ev = torch.cat([c1, c2, t.to(torch.float32)[:, None]], 1)
        out.append(ev)
        have += ev.shape[0]
    return torch.cat(out, 0)[:n_events].contiguous()


def random_lors(n, scanner, seed, device="cpu"):
    """[n, 6] float32 LORs between uniformly random distinct crystals."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    ncry = scanner.n_crystals * scanner.n_rings
    pos = torch.as_tensor(scanner.crystal_positions(), device=dev)
    i = torch.randint(0, ncry, (n,), generator=g, device=dev)
    j = torch.randint(0, ncry - 1, (n,), generator=g, device=dev)
    j = j + (j >= i).long()
    return torch.cat([pos[i], pos[j]], 1).contiguous()


_GAMMA = 0x9E3779B97F4A7C15
_MASK64 = (1 << 64) - 1


def splitmix64(seed, k):
    """SplitMix64 output number ``k`` (numpy uint64 array) of the stream seeded ``seed``
    (Steele, Lea and Flood, OOPSLA 2014): the finaliser of seed + (k + 1) * gamma. The
    host mirror of the generator in the TOR map kernels (``srf_tor_maplors_generated``)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & _MASK64) + (np.asarray(k, np.uint64) + np.uint64(1)) * np.uint64(_GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


CHORD_GROUP = 256


def random_pair_indices(n_rings, n_per_ring, seed, first, count):
    """Crystal indices (a, b) of generated random chords first .. first+count-1 of a ring
    scanner (crystal k of ring r at index r * n_per_ring + k): the host mirror of kind 0
    of ``srf_tor_maplors_generated``. Groups of ``CHORD_GROUP`` consecutive numbers share
    the chord class s = (k_a + k_b) mod n (the transverse direction) and the ring offset
    d = r_b - r_a; within a group r_a is drawn per LOR and k_a stratified (LOR i of a
    group in the i-th of CHORD_GROUP equal parts of the ring), so neighbouring LORs are
    near-identical chords. Every ordered crystal pair is equally likely; a pair of one
    crystal with itself (a == b) maps nothing."""
    n, nr = np.uint64(n_per_ring), np.uint64(n_rings)
    g = np.arange(first, first + count, dtype=np.uint64)
    grp = g // np.uint64(CHORD_GROUP)
    hg = splitmix64(seed, np.uint64(4) * grp)
    hg2 = splitmix64(seed, np.uint64(4) * grp + np.uint64(2))
    hi, lo = np.uint64(32), np.uint64(0xFFFFFFFF)

    def scale(u, m):
        return ((u * m) >> hi).astype(np.int64)

    s = scale(hg >> hi, n)
    d = scale(hg2 >> hi, nr) - scale(hg & lo, nr)
    h = splitmix64(seed, np.uint64(2) * g + np.uint64(1))
    i = g % np.uint64(CHORD_GROUP)  # stratified: LOR i of a group in the i-th part of the ring
    a_pos = ((((i << hi) | (h >> hi)) * n) >> np.uint64(40)).astype(np.int64)
    b_pos = (s + int(n) - a_pos) % int(n)
    r_a = np.maximum(0, -d) + scale(h & lo, (np.int64(n_rings) - np.abs(d)).astype(np.uint64))
    return r_a * int(n) + a_pos, (r_a + d) * int(n) + b_pos


class GeneratedPairs:
    """Detector-pair LORs that the TOR map kernels make on the fly from their number, so
    that no LOR array exists at any point (``srf_tor_maplors_generated``):

    * ``GeneratedPairs.random(scanner, n, seed)``: n uniform crystal pairs of a ring
      scanner, drawn in groups that share a direction (SplitMix64, see
      ``random_pair_indices``);
    * ``GeneratedPairs.block_pairs(cylindrical_pet)``: every crystal pair of the scanner's
      block pairs over all ring pairs, in the reference's effmap order
      (srfapp_new.py:153-157, scanner/pet/pet.py:149-177).

    ``crystals`` (float32 [n, 3]) is uploaded once; ``host_lors(first, count)`` returns the
    same LORs as a numpy [count, 6] array (for checks and for models without the fused
    path)."""

    def __init__(self, kind, crystals, n, seed=0, n_rings=1, n_blocks=1, n_per_block=None,
                 chunk=1 << 26, device="cuda"):
        self.kind = int(kind)
        self.host_crystals = np.ascontiguousarray(crystals, np.float32)
        self.n = int(n)
        self.seed = int(seed)
        self.n_rings, self.n_blocks = int(n_rings), int(n_blocks)
        self.n_per_block = int(n_per_block if n_per_block is not None
                               else len(self.host_crystals) // (self.n_rings * self.n_blocks))
        self.chunk = int(chunk)
        self.device = torch.device(device)
        self.crystals = torch.as_tensor(self.host_crystals, device=self.device)

    @classmethod
    def random(cls, scanner, n, seed, chunk=1 << 26, device="cuda"):
        """n random chords of a ``RingScanner`` (``random_pair_indices``)."""
        pos = scanner.crystal_positions()
        return cls(0, pos, n, seed, scanner.n_rings, 1, scanner.n_crystals, chunk, device)

    @classmethod
    def block_pairs(cls, pet, chunk=1 << 26, device="cuda"):
        table = pet.crystal_table()
        nr, nb = pet.nb_rings, pet.nb_blocks_per_ring
        ncb = len(table) // (nr * nb)
        cb = ncb * ncb
        n = nr * ((nr - 1) * nb * (nb - 1) * cb + nb * (nb - 1) // 2 * cb)
        return cls(1, table, n, 0, nr, nb, ncb, chunk, device)

    def __len__(self):
        return self.n

    def pair_indices(self, first, count):
        """(a, b) crystal indices of LORs first .. first+count-1 (host)."""
        if self.kind == 0:
            return random_pair_indices(self.n_rings, self.n_per_block, self.seed, first, count)
        nr, nb, ncb = self.n_rings, self.n_blocks, self.n_per_block
        a_all, b_all = [], []
        for ir1 in range(nr):
            for ir2 in range(nr):
                for i1 in range(nb):
                    for i2 in range(nb):
                        if (ir1 == ir2 and i1 < i2) or (ir1 != ir2 and i1 != i2):
                            c1 = (ir1 * nb + i1) * ncb + np.repeat(np.arange(ncb), ncb)
                            c2 = (ir2 * nb + i2) * ncb + np.tile(np.arange(ncb), ncb)
                            a_all.append(c1)
                            b_all.append(c2)
        a, b = np.concatenate(a_all), np.concatenate(b_all)
        return a[first:first + count], b[first:first + count]

    def host_lors(self, first, count):
        """The same LORs as the kernels make, [count, 6] (a pair of one crystal with itself,
        which the kernels skip, comes out with both ends equal)."""
        a, b = self.pair_indices(first, count)
        return np.hstack([self.host_crystals[a], self.host_crystals[b]])

    def __call__(self, start, count):
        """[count, 6] LORs on the device (materialised: models without the fused path)."""
        return torch.as_tensor(self.host_lors(start, count), device=self.device)


class RandomLorSource:
    """Random detector-pair LORs generated on the device chunk by chunk: chunk k of
    ``chunk`` LORs is ``random_lors(count, scanner, seed * 1000003 + k)``, so any chunk
    can be regenerated on its own and a pass over n LORs never holds more than one chunk.
    Call as ``source(start, count)`` with ``start`` a multiple of ``chunk``."""

    def __init__(self, n, scanner, seed, chunk=16_000_000, device="cuda"):
        self.n, self.scanner, self.seed, self.chunk = int(n), scanner, int(seed), int(chunk)
        self.device = torch.device(device)

    def __len__(self):
        return self.n

    def __call__(self, start, count):
        if start % self.chunk or count > self.chunk:
            raise ValueError("chunks start at multiples of the chunk size")
        return random_lors(count, self.scanner, self.seed * 1000003 + start // self.chunk,
                           self.device)


# --------------------------------------------------------------- named workloads


@dataclass
class Workload:
    name: str
    scanner: RingScanner
    grid: tuple
    voxel: float
    n_events: int
    tof_res_ps: float
    tof_bin_ps: float
    kernel_width: float
    n_effmap: int
    iterations: int
    subsets: int
    seed: int

    @property
    def size(self):
        return [g * self.voxel for g in self.grid]

    @property
    def center(self):
        return [0.0, 0.0, 0.0]


def siddon_64():
    """Plain non-TOF Siddon OSEM: R 400 mm, 400 x 32 crystals, pitch 3.2 mm; image
    64x64x32 at 3.4 mm; 1M events; effmap from 10M random pairs; 3 it x 4 subsets."""
    return Workload("siddon_64x64x32_1M", RingScanner(400.0, 400, 32, 3.2), (64, 64, 32), 3.4,
                    1_000_000, 1.0e4, 1.0e4, 0.0, 10_000_000, 3, 4, 1)


def tor_128():
    """TOF TOR at 128x128x64, 3.2 mm voxels, same scanner; 10M events, 530 ps FWHM,
    40 ps bin (6 mm); TOR FWHM 4 mm -> kernel_width = 6 sigma = 10.19 mm; effmap from 50M
    random LORs; OSEM 3 it x 10 subsets."""
    kw = 6 * 4.0 / GAUSSIAN_FWHM
    return Workload("tor_tof_128x128x64_10M", RingScanner(400.0, 400, 32, 3.2), (128, 128, 64),
                    3.2, 10_000_000, 530.0, 40.0, kw, 50_000_000, 3, 10, 2)


def batched_96(frame):
    """One frame of the batched TOF OSEM workload (96x96x48, 3.2 mm)."""
    g = np.random.default_rng(1000 + frame)
    n = int(round(math.exp(g.uniform(math.log(2e5), math.log(5e6)))))
    kw = 6 * 4.0 / GAUSSIAN_FWHM
    return Workload(f"batched_96x96x48_frame{frame}", RingScanner(400.0, 400, 32, 3.2),
                    (96, 96, 48), 3.2, n, 530.0, 40.0, kw, 0, 3, 10, 1000 + frame)


def large_256():
    """Large axial FOV: R 390 mm, 600 x 320 crystals over 1 m; 256x256x128 at 2.5 mm;
    200M events at 400 ps; OSEM 2 x 20; effmap from 500M random LORs."""
    kw = 6 * 4.0 / GAUSSIAN_FWHM
    return Workload("large_256x256x128_200M", RingScanner(390.0, 600, 320, 3.125),
                    (256, 256, 128), 2.5, 200_000_000, 400.0, 40.0, kw, 500_000_000, 2, 20, 5)


GAUSSIAN_FWHM = 2.35482005
