"""Seeded synthetic axon lattices.

The reference builds its lattices from EM segmentations in MATLAB
(part1_demo2_artificial_shape_generation.m, analysis/visualizeaxon.m:28-67:
caliber variation and undulation of a segmented axon).  Those segmentations
are not part of the checkout, so this module draws the same two kinds of
variation from an explicit law instead:

    radius   r(z) = r0 * (1 + 0.2 * sum_{k=1..4} a_k sin(2 pi z / lam_k + phi_k))
             a_k ~ U(0, 0.5), lam_k ~ U(2, 20) um, phi_k ~ U(0, 2 pi)
    centre   c(z) = c_box + A (cos(2 pi z / lam_u + psi), sin(2 pi z / lam_u + psi))
             A = 0.5 um, lam_u = 15 um, psi ~ U(0, 2 pi)

A voxel is intra-axonal (label 1) when its centre lies within r(z) of c(z);
every other voxel gets ``exterior`` (0 = null compartment, 2 = extra-axonal).
Lattice index order is (i, j, k) = (x, y, z), k fastest, as the simulator
reads fiber.txt (hpc_code/lib/main.cu:461-466).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class AxonShape:
    r0: float
    a: np.ndarray
    lam: np.ndarray
    phi: np.ndarray
    und_amp: float
    und_lam: float
    psi: float

    def radius(self, z: np.ndarray) -> np.ndarray:
        s = np.zeros_like(z, dtype=np.float64)
        for ak, lk, pk in zip(self.a, self.lam, self.phi):
            s += ak * np.sin(2.0 * np.pi * z / lk + pk)
        return self.r0 * (1.0 + 0.2 * s)


def draw_shape(rng: np.random.Generator, r0: float = 1.0, und_amp: float = 0.5,
               und_lam: float = 15.0) -> AxonShape:
    a = rng.uniform(0.0, 0.5, 4)
    lam = rng.uniform(2.0, 20.0, 4)
    phi = rng.uniform(0.0, 2.0 * np.pi, 4)
    psi = float(rng.uniform(0.0, 2.0 * np.pi))
    return AxonShape(r0, a, lam, phi, und_amp, und_lam, psi)


def axon_slices(n1: int, n2: int, n3: int, res: float = 0.1, seed: int = 0, r0: float = 1.0,
                shape: AxonShape | None = None):
    """Per-slice (radius^2, centre x, centre y), um, of the axon along z: the
    tables both the host builder below and the GPU builder
    (Sim.set_tube_lattice, rms_sim_set_tube_lattice) fill voxels from."""
    if shape is None:
        shape = draw_shape(np.random.default_rng(seed), r0=r0)
    z = (np.arange(n3) + 0.5) * res
    r = shape.radius(z)
    ang = 2.0 * np.pi * z / shape.und_lam + shape.psi
    cx = 0.5 * n1 * res + shape.und_amp * np.cos(ang)
    cy = 0.5 * n2 * res + shape.und_amp * np.sin(ang)
    return r ** 2, cx, cy


def axon_lattice(n1: int, n2: int, n3: int, res: float = 0.1, seed: int = 0,
                 exterior: int = 0, r0: float = 1.0, shape: AxonShape | None = None
                 ) -> np.ndarray:
    """uint8 lattice (n1, n2, n3) of one undulating, caliber-varying axon
    along z, centred in the x-y box (built on the host; Sim.set_tube_lattice
    builds the same lattice on the GPU)."""
    r2, cx, cy = axon_slices(n1, n2, n3, res, seed, r0, shape)
    x = (np.arange(n1) + 0.5) * res
    y = (np.arange(n2) + 0.5) * res
    out = np.full((n1, n2, n3), exterior, dtype=np.uint8)
    # slab by slab over z keeps peak memory at one x-y plane of floats
    for k in range(n3):
        dx = x[:, None] - cx[k]
        dy = y[None, :] - cy[k]
        d2 = dx * dx + dy * dy
        out[:, :, k][d2 < r2[k]] = 1
    return out


def config_axon(kind: str = "single", seed: int = 0) -> np.ndarray:
    """Named synthetic lattices used by the tests and the benchmark.

    single      64 x 64 x 512, labels {0, 1}          (one axon, null outside)
    two_comp    64 x 64 x 512, labels {1, 2}          (same axon, extra-axonal outside)
    production  256 x 256 x 2048, labels {1, 2}
    """
    if kind == "single":
        return axon_lattice(64, 64, 512, 0.1, seed, exterior=0)
    if kind == "two_comp":
        return axon_lattice(64, 64, 512, 0.1, seed, exterior=2)
    if kind == "production":
        return axon_lattice(256, 256, 2048, 0.1, seed, exterior=2)
    raise ValueError(kind)


def batch_sizes(n_axons: int = 64, seed: int = 0, lo=(64, 64, 256), hi=(256, 256, 2048)):
    """Lattice shapes with log-uniform voxel counts between ``lo`` and ``hi``:
    one shared scale s in [0, 1] per axon, each side = lo * (hi/lo)^s rounded
    to a multiple of 8."""
    rng = np.random.default_rng(seed)
    s = rng.uniform(0.0, 1.0, n_axons)
    shapes = []
    for si in s:
        dims = []
        for a, b in zip(lo, hi):
            v = a * (b / a) ** si
            dims.append(int(max(a, min(b, 8 * round(v / 8)))))
        shapes.append(tuple(dims))
    return shapes
