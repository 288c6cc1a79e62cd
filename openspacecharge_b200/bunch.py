"""Seeded synthetic bunches with the shapes of the reference's test generator.

``gendist`` (code/test_mod.f90:19-93) draws Box-Muller Gaussians rejected outside a radius
of ``gaussiancutoff`` in sigma units (or points uniform in the unit ball), optionally
rejects points outside 90% of a rectangular pipe's half-apertures, scales by the sigmas,
subtracts the sample centroid and zeroes the first particle.  Its numbers come from the
gfortran PRNG and cannot be reproduced here, so this module draws the same distributions
from numpy's PCG64 with an explicit seed; the same arrays feed the oracle and the GPU.
"""
from __future__ import annotations

import numpy as np


def gendist(n: int, sigma=(1e-3, 1e-3, 1e-3), cutoff: float = 4.0, disttype: int = 1, seed: int = 1,
            pipe: tuple | None = None, centroid=(0.0, 0.0, 0.0), zero_first: bool = True):
    """Return x, y, z (float64, length n).

    disttype 1: Gaussian truncated at radius ``cutoff`` (sigma units, all three axes);
    disttype 0: uniform in the unit ball scaled by sigma.  ``pipe=(apipe, bpipe)`` rejects
    points with (x/(a/2))^2 + (y/(b/2))^2 > 0.9^2 (code/test_mod.f90:49-62)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sig = np.asarray(sigma, dtype=np.float64)
    out = np.empty((0, 3))
    need = n
    while need > 0:
        m = int(need * 1.3) + 1024
        if disttype == 1:
            r = rng.standard_normal((m, 3))
            keep = (r * r).sum(1) <= cutoff * cutoff
        else:
            r = rng.uniform(-1.0, 1.0, (m, 3))
            keep = (r * r).sum(1) <= 1.0
        if pipe is not None:
            a, b = pipe
            keep &= (r[:, 0] ** 2 * sig[0] ** 2 / (0.5 * a) ** 2 + r[:, 1] ** 2 * sig[1] ** 2 / (0.5 * b) ** 2) <= 0.81
        r = r[keep][:need]
        out = np.concatenate([out, r])
        need = n - len(out)
    pts = out * sig
    pts -= pts.mean(axis=0)
    if zero_first and n > 0:
        pts[0] = 0.0
    pts += np.asarray(centroid, dtype=np.float64)
    return (np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1]),
            np.ascontiguousarray(pts[:, 2]))


def gamma_of(e_tot: float, mc2: float = 0.510998910e6) -> float:
    """gamma = E_tot/mc^2 as in the reference driver (code/test_opensc.f90:102)."""
    return e_tot / mc2
