"""Photon batches (structure of arrays) and the seeded photon sources of the
benchmark configurations.

A batch is a dict of numpy (or torch) arrays with the keys support_x,
support_y, support_z, direction_x, direction_y, direction_z, wavelength and
id -- the fields of merlict::Photon (merlict/Photon.h, RayForPropagation.h)
that a propagation reads.
"""
from __future__ import annotations

import numpy as np

PLANES = ("support_x", "support_y", "support_z",
          "direction_x", "direction_y", "direction_z", "wavelength")


def make_batch(support, direction, wavelength, ids=None) -> dict:
    """Photons from (n,3) supports, (n,3) directions and (n,) wavelengths.

    Like the merlict::Photon constructor (Photon.cpp:20-28) a wavelength
    must be positive; invalid photons raise ValueError.
    """
    support = np.asarray(support, dtype=np.float64).reshape(-1, 3)
    direction = np.asarray(direction, dtype=np.float64).reshape(-1, 3)
    wavelength = np.asarray(wavelength, dtype=np.float64).reshape(-1)
    n = wavelength.shape[0]
    if support.shape[0] != n or direction.shape[0] != n:
        raise ValueError("support, direction and wavelength differ in length")
    if np.any(~(wavelength > 0.0)):
        raise ValueError("Expected photon wavelength lambda > 0.0nm")
    b = {
        "support_x": support[:, 0].copy(), "support_y": support[:, 1].copy(),
        "support_z": support[:, 2].copy(),
        "direction_x": direction[:, 0].copy(), "direction_y": direction[:, 1].copy(),
        "direction_z": direction[:, 2].copy(),
        "wavelength": wavelength.copy(),
        "id": (np.arange(n, dtype=np.int32) if ids is None
               else np.asarray(ids, dtype=np.int32).reshape(-1)),
    }
    return b


def num_photons(batch: dict) -> int:
    return int(len(batch["wavelength"]))


def slice_batch(batch: dict, start: int, stop: int) -> dict:
    return {k: v[start:stop] for k, v in batch.items()}


def downward_disc_source(n: int, seed: int, disc_radius: float, height: float,
                         max_zenith_deg: float, lambda_min: float = 300e-9,
                         lambda_max: float = 700e-9, center=(0.0, 0.0)) -> dict:
    """Supports uniform on a horizontal disc at `height`, directions
    downwards, uniform in solid angle within `max_zenith_deg` of -z,
    wavelengths uniform in [lambda_min, lambda_max)."""
    rng = np.random.default_rng(seed)
    r = disc_radius * np.sqrt(rng.random(n))
    phi = 2.0 * np.pi * rng.random(n)
    cos_max = np.cos(np.deg2rad(max_zenith_deg))
    cos_t = 1.0 - rng.random(n) * (1.0 - cos_max)
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    az = 2.0 * np.pi * rng.random(n)
    lam = lambda_min + (lambda_max - lambda_min) * rng.random(n)
    sup = np.stack([center[0] + r * np.cos(phi), center[1] + r * np.sin(phi),
                    np.full(n, float(height))], axis=1)
    d = np.stack([sin_t * np.cos(az), sin_t * np.sin(az), -cos_t], axis=1)
    return make_batch(sup, d, lam)


def isotropic_shell_source(n: int, seed: int, radius: float, aim_radius: float,
                           lambda_min: float = 250e-9, lambda_max: float = 750e-9) -> dict:
    """Supports on a sphere of `radius` around the origin, each aimed at a
    random point within `aim_radius` of the origin (test scenes)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    sup = v * radius
    t = rng.normal(size=(n, 3))
    t /= np.linalg.norm(t, axis=1)[:, None]
    aim = t * (aim_radius * rng.random(n) ** (1.0 / 3.0))[:, None]
    d = aim - sup
    lam = lambda_min + (lambda_max - lambda_min) * rng.random(n)
    return make_batch(sup, d, lam)
