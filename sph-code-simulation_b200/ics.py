"""Initial conditions of the benchmark workloads in numpy, without the device
library (so the CPU reference arm of bench.py and the GPU arm start from the
same arrays while the reference arm maps no product library).

They restate the C generators of host/samples.cpp (sphgpu_sample_*), which
follow the reference's sample set-ups:
  evrard       Solver::make_evrard (src/sample/evrard.cpp:13-87)
  shear_layer  Solver::make_khi (src/sample/khi.cpp:12-73) extruded to 3-D
  shock_tube   a 3-D two-state tube along x
  blast_field  many Sedov-like point blasts in a periodic cube (rho = 1, a
               low background pressure, blast particles at 1e2 .. 1e4 times
               it), a stress case for the exact Riemann solver
numpy's vectorised pow / sin / exp may round differently from the C
library's in the last bit, so a position can differ from the C generator's
by an ulp (tests/test_ics.py bounds the difference); both arms of the bench
use these arrays.
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np

from sphparams import FIELDS


def _empty(n: int) -> Dict[str, np.ndarray]:
    return {f: np.zeros(n) for f in FIELDS}


def evrard(N: int, G: float = 1.0, gamma: float = 5.0 / 3.0) -> Dict[str, np.ndarray]:
    """Evrard sphere: an N^3 lattice in [-1, 1]^3 cut to the unit sphere, each
    radius remapped r -> r^1.5, equal masses 1/Np, rho = 1/(2 pi r),
    u = 0.05 G, v = 0 (lattice order i, j, k as the reference's loops)."""
    dx = 2.0 / N
    g = (np.arange(N) + 0.5) * dx - 1.0
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    r0 = np.sqrt((x * x + y * y) + z * z)
    keep = r0 <= 1.0
    x, y, z, r0 = x[keep], y[keep], z[keep], r0[keep]
    s = np.ones_like(r0)
    nz = r0 > 0.0
    s[nz] = np.power(r0[nz], 1.5) / r0[nz]
    x, y, z = x * s, y * s, z * s
    n = x.size
    out = _empty(n)
    out["pos_x"], out["pos_y"], out["pos_z"] = x, y, z
    out["mass"][:] = 1.0 / n
    r = np.sqrt((x * x + y * y) + z * z)
    dens = 1.0 / (2.0 * math.pi * r)
    u = 0.05 * G
    out["dens"] = dens
    out["ene"][:] = u
    out["pres"] = (gamma - 1.0) * dens * u
    return out


def _lattice(nx: int, ny: int, nz: int, hx: float, hy: float, hz: float, x0: float, y0: float):
    a, b, c = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return (x0 + (a.ravel() + 0.5) * hx, y0 + (b.ravel() + 0.5) * hy, (c.ravel() + 0.5) * hz)


def shear_layer(dx: float, lz: float = 0.125, gamma: float = 5.0 / 3.0) -> Dict[str, np.ndarray]:
    """Periodic 3-D shear layer in [0,1] x [0,1] x [0,lz]: the band
    0.25 < y < 0.75 holds rho = 2, vx = -0.5 on a lattice of spacing
    dx 2^(-1/3), the rest rho = 1, vx = +0.5 at spacing dx; P = 2.5;
    vy = 0.025 sin(4 pi x) [exp(-(y-.25)^2/(2 s^2)) + exp(-(y-.75)^2/(2 s^2))],
    s = 0.05; equal masses."""
    dx2 = dx * 2.0 ** (-1.0 / 3.0)
    lats = [(round(1.0 / dx), round(0.25 / dx), round(lz / dx), 0.0, 0.25, 1.0, 0.5),
            (round(1.0 / dx2), round(0.5 / dx2), round(lz / dx2), 0.25, 0.5, 2.0, -0.5),
            (round(1.0 / dx), round(0.25 / dx), round(lz / dx), 0.75, 0.25, 1.0, 0.5)]
    parts = []
    for nx, ny, nz, y0, ly, rho, vx in lats:
        x, y, z = _lattice(nx, ny, nz, 1.0 / nx, ly / ny, lz / nz, 0.0, y0)
        parts.append((x, y, z, rho, vx))
    n = sum(p[0].size for p in parts)
    out = _empty(n)
    mass = (1.0 * 0.5 * lz + 2.0 * 0.5 * lz) / n
    s2 = 0.05 * 0.05
    k = 0
    for x, y, z, rho, vx in parts:
        sl = slice(k, k + x.size)
        out["pos_x"][sl], out["pos_y"][sl], out["pos_z"][sl] = x, y, z
        out["vel_x"][sl] = vx
        out["vel_y"][sl] = 0.025 * np.sin(4.0 * math.pi * x) * (
            np.exp(-(y - 0.25) * (y - 0.25) / (2 * s2)) + np.exp(-(y - 0.75) * (y - 0.75) / (2 * s2)))
        out["dens"][sl] = rho
        out["ene"][sl] = 2.5 / ((gamma - 1.0) * rho)
        k += x.size
    out["mass"][:] = mass
    out["pres"][:] = 2.5
    return out


def shock_tube(dx: float, ly: float = 0.05, p_left: float = 1000.0, p_right: float = 0.01,
               gamma: float = 1.4) -> Dict[str, np.ndarray]:
    """Tube x in [-0.5, 0.5], y, z in [0, ly] on one lattice; rho = 1,
    p = p_left for x < 0 and p_right otherwise."""
    nx, ny = round(1.0 / dx), round(ly / dx)
    x, y, z = _lattice(nx, ny, ny, 1.0 / nx, ly / ny, ly / ny, -0.5, 0.0)
    n = x.size
    out = _empty(n)
    out["pos_x"], out["pos_y"], out["pos_z"] = x, y, z
    out["mass"][:] = 1.0 * ly * ly / n
    out["dens"][:] = 1.0
    p = np.where(x < 0.0, p_left, p_right)
    out["pres"] = p
    out["ene"] = p / ((gamma - 1.0) * 1.0)
    return out


def blast_field(dx: float, frac: float = 0.25, p_bg: float = 1e-4, p_lo: float = 1e-2, p_hi: float = 1.0,
                gamma: float = 1.4, seed: int = 12345) -> Dict[str, np.ndarray]:
    """Periodic cube [-0.5, 0.5]^3 on one lattice of spacing dx; rho = 1,
    v = 0, a low background pressure p_bg (the Sedov set-up of
    src/sample/sedov.cpp has 1e-6) except on a random fraction `frac` of the
    particles (numpy Philox stream `seed`), which hold a pressure drawn
    log-uniform in [p_lo, p_hi]: many point blasts, so nearly half of the
    particle pairs pose a Riemann problem with a pressure jump of 1e2 .. 1e4
    (the range the learned guess is trained on)."""
    n1 = round(1.0 / dx)
    h = 1.0 / n1
    x, y, z = _lattice(n1, n1, n1, h, h, h, -0.5, -0.5)
    z = z - 0.5
    n = x.size
    rng = np.random.Generator(np.random.Philox(seed))
    blast = rng.random(n) < frac
    p = np.full(n, p_bg)
    p[blast] = np.exp(rng.uniform(np.log(p_lo), np.log(p_hi), int(blast.sum())))
    out = _empty(n)
    out["pos_x"], out["pos_y"], out["pos_z"] = x, y, z
    out["mass"][:] = 1.0 / n
    out["dens"][:] = 1.0
    out["pres"] = p
    out["ene"] = p / ((gamma - 1.0) * 1.0)
    return out
