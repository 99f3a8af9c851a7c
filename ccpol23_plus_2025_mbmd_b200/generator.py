"""Seeded synthetic water boxes (the inputs of every benchmark and parity case).

Centres of mass on a jittered simple-cubic lattice (n^3 lattice points with n = floor(N^1/3),
the remaining N - n^3 molecules on randomly chosen cube centres; an extra molecule that
cannot be placed after 20 draws moves to another cube centre; when N - n^3 > n^3, a random
subset of an (n+1)^3 lattice), uniform jitter of
+-0.3 A per component, uniformly random orientations (Shoemake's unit quaternions), and no
oxygen-oxygen distance below 2.5 A under the minimum image (offending molecules are
redrawn).  COM velocities are Maxwell-Boltzmann at the target temperature with the drift
removed; body-frame angular momenta are Gaussian with variance k_B T I_a.  COMs are wrapped
into [-L/2, L/2) as the reference does when it reads a REVCON (initialization.f90:71-75).

The module imports nothing from the package at load time: ``water_box`` needs from its
``model`` only ``pcoord``, ``pmi``, ``get_double("totm")`` and ``sites(q, ld)``, which the
library's Model and the oracle's SiteFrame both provide, so the CPU reference timing builds
the same box without loading the library.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BOLTZ = 0.831451115  # (10 J/mol)/K, common_arrays.f90:29

# The box sizes and seeds of the benchmark configurations (densities ~1 g/cm^3).
CONFIGS = {
    "c1_128": dict(nm=128, box=15.64, variant="fs3", seed=1001),
    "c2_512": dict(nm=512, box=24.84, variant="fs2fs3", seed=2002),
    "c3_512": dict(nm=512, box=24.84, variant="fs2fs3", seed=3003),
    "c4_256": dict(nm=256, box=19.71, variant="fs3", seed=4004),
    "c5_2048": dict(nm=2048, box=39.40, variant="fs2fs3", seed=5005),
}


@dataclass
class Box:
    nm: int
    box: float
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    q: np.ndarray      # (nm, 4) unit quaternions q0..q3
    xs: np.ndarray     # (nm, ld) site offsets
    ys: np.ndarray
    zs: np.ndarray
    v: np.ndarray      # (nm, 3) COM velocities (A/ps)
    jb: np.ndarray     # (nm, 3) body-frame angular momenta


def random_quaternions(rng, n):
    """Shoemake's uniform random unit quaternions."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    return np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                     b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)


def _wrap(v, box):
    return v - box * np.round(v / box)


def water_box(model, nm: int, box: float, seed: int, *, ld: int | None = None,
              jitter: float = 0.3, min_oo: float = 2.5, temperature: float = 298.0,
              o_site: int = 0, max_tries: int = 200) -> Box:
    rng = np.random.default_rng(seed)
    n = int(np.floor(nm ** (1.0 / 3.0) + 1e-9))
    if n ** 3 > nm:
        n -= 1
    subset = nm - n ** 3 > n ** 3  # too few cube centres: use a random subset of (n+1)^3
    if subset:
        n += 1
    a = box / n
    g = (np.arange(n) + 0.5) * a - 0.5 * box
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    centres = list(_wrap(lattice + 0.5 * a, box)[rng.permutation(n ** 3)])
    if subset:
        lattice = lattice[np.sort(rng.permutation(n ** 3)[:nm])]
        n_lat = nm
    else:
        n_lat = n ** 3
    base = _wrap(lattice, box)
    pcoord = model.pcoord
    o_off = pcoord[o_site]
    com = np.empty((nm, 3))
    q = np.empty((nm, 4))
    oxy = np.empty((nm, 3))

    def rot(qq):
        q0, q1, q2, q3 = qq
        return np.array([
            [q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
            [2 * (q1 * q2 + q0 * q3), q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * (q2 * q3 - q0 * q1)],
            [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]])

    for m in range(nm):
        for attempt in range(max_tries):
            if m < n_lat:
                site = base[m]
            else:  # extra molecules take a cube centre; move to another one if crowded
                if attempt % 20 == 0:
                    site = centres.pop()
            c = _wrap(site + rng.uniform(-jitter, jitter, 3), box)
            qq = random_quaternions(rng, 1)[0]
            o = c + rot(qq) @ o_off
            if m:
                d = _wrap(oxy[:m] - o, box)
                if np.min(np.einsum("ij,ij->i", d, d)) < min_oo * min_oo:
                    continue
            com[m], q[m], oxy[m] = c, qq, o
            break
        else:
            raise RuntimeError("could not place molecule %d" % m)
    xs, ys, zs = model.sites(q, ld)
    mass = model.get_double("totm")
    sig = np.sqrt(BOLTZ * temperature / mass)
    v = rng.normal(0.0, sig, (nm, 3))
    v -= v.mean(axis=0)
    pmi = model.pmi
    jb = rng.normal(0.0, 1.0, (nm, 3)) * np.sqrt(BOLTZ * temperature * pmi)
    return Box(nm, box, com[:, 0].copy(), com[:, 1].copy(), com[:, 2].copy(), q, xs, ys, zs, v, jb)


def config_box(name: str, model=None, ld: int | None = None) -> Box:
    from .api import Model, data_dir
    cfg = CONFIGS[name]
    model = model or Model(data_dir(cfg["variant"]))
    return water_box(model, cfg["nm"], cfg["box"], cfg["seed"], ld=ld)
