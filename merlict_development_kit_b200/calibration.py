"""Plenoscope calibration on the GPU: plenoscope::calibration::Calibrator
(merlict_portal_plenoscope/calibration/Calibrator.cpp:38-168).

Photons start 10 km up the back-running ray of a point uniform on the
aperture disc (1.05 x the imaging system's aperture radius) and a direction
uniform in solid angle within 1.2 x the field of view's radius, at 433 nm;
they are propagated by the exact tracer, and every lixel gets merlict's
LixelStatistic: efficiency and its error, mean and spread of the incident
direction (cx, cy), of the support on the aperture (x, y) and of the time
delay (time of flight minus the 10 km to the aperture).  The statistics are
computed on the device by mlgpu_lixel_statistics, bit for bit as
LixelStatisticsFiller computes them from the same photons.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import engine
from ._native import check, lib

WAVELENGTH = 433e-9                   # Calibrator.h:30
DISTANCE_TO_APERTURE_PLANE = 1e4      # Calibrator.h:31
APERTURE_RADIUS_OVERHEAD = 1.05       # night_sky_background/NightSkyBackground.h:11
FOV_RADIUS_OVERHEAD = 1.20            # NightSkyBackground.h:12
SPEED_OF_LIGHT = 299792458.0
FIELDS = ("efficiency", "efficiency_std", "cx_mean", "cx_std", "cy_mean", "cy_std",
          "x_mean", "x_std", "y_mean", "y_std", "time_delay_mean", "time_delay_std")


def calibration_photons(n: int, seed: int, aperture_radius: float, max_fov_radius: float,
                        device="cuda"):
    """(photon planes, per-photon cx, cy, x, y) of Calibrator::one_photon
    (Calibrator.cpp:49-100) with torch's generator."""
    g = torch.Generator(device=device).manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    u = torch.rand((4, n), generator=g, device=device, dtype=torch.float64)
    r_max = APERTURE_RADIUS_OVERHEAD * aperture_radius
    r = r_max * torch.sqrt(u[0])
    phi = 2.0 * math.pi * u[1]
    sx, sy = r * torch.cos(phi), r * torch.sin(phi)
    # ZenithDistancePicker(0, max): z uniform in [(cos max + 1)/2, 1], zd = acos(2z - 1)
    z_min = (math.cos(0.0) + 1.0) / 2.0
    z_range = (math.cos(FOV_RADIUS_OVERHEAD * max_fov_radius) + 1.0) / 2.0 - z_min
    zd = torch.acos(2.0 * (z_range * u[2] + z_min) - 1.0)
    az = 2.0 * math.pi * u[3]
    ix, iy, iz = torch.sin(zd) * torch.cos(az), torch.sin(zd) * torch.sin(az), torch.cos(zd)
    d = DISTANCE_TO_APERTURE_PLANE
    planes = {"support_x": sx + ix * d, "support_y": sy + iy * d, "support_z": iz * d,
              "direction_x": -ix, "direction_y": -iy, "direction_z": -iz,
              "wavelength": torch.full_like(sx, WAVELENGTH)}
    return planes, (ix.float(), iy.float(), sx.float(), sy.float())


def lixel_statistics(scene: engine.Scene, sensor: torch.Tensor, cx, cy, x, y, time_delay,
                     photons_emitted_per_lixel: float, stream=None) -> dict:
    """merlict's LixelStatistic of every sensor from per-photon results
    (mlgpu_lixel_statistics); returns {field: numpy array [num_sensors]}."""
    n = int(sensor.shape[0])
    arrays = [sensor.to(torch.int32).contiguous()] + [
        a.to(torch.float32).contiguous() for a in (cx, cy, x, y, time_delay)]
    out = torch.empty((scene.num_sensors, 12), dtype=torch.float32, device=sensor.device)
    check(lib().mlgpu_lixel_statistics(scene.handle, *[C.c_void_p(a.data_ptr()) for a in arrays],
                                       n, float(photons_emitted_per_lixel),
                                       C.c_void_p(out.data_ptr()),
                                       C.c_void_p(engine._stream_handle(stream))))
    o = out.cpu().numpy()
    return {f: o[:, k] for k, f in enumerate(FIELDS)}


def calibrate(scene: engine.Scene, aperture_radius: float, max_fov_radius: float,
              num_photons: int = 8_000_000, seed: int = 0, max_interactions: int = 5,
              chunk: int = 1 << 24) -> dict:
    """Calibrator::run_calibration (Calibrator.cpp:145-168) on the GPU:
    propagates num_photons calibration photons and returns every lixel's
    statistics (the default PropagationConfig of Calibrator's environment
    allows 5 interactions)."""
    sensors, vals = [], [[], [], [], [], []]
    for a in range(0, num_photons, chunk):
        m = min(chunk, num_photons - a)
        ph, (cx, cy, x, y) = calibration_photons(m, seed * 1000003 + a, aperture_radius,
                                                 max_fov_radius, device="cuda")
        out = scene.propagate(ph, engine.PropagationConfig(max_interactions),
                              engine.Philox(seed, photon_offset=a), outputs=("sensor", "time"))
        delay = (out["time"] - DISTANCE_TO_APERTURE_PLANE / SPEED_OF_LIGHT).float()
        sensors.append(out["sensor"])
        for v, t in zip(vals, (cx, cy, x, y, delay)):
            v.append(t)
        del ph, out
    cat = lambda xs: torch.cat(xs) if len(xs) > 1 else xs[0]
    return lixel_statistics(scene, cat(sensors), *[cat(v) for v in vals],
                            num_photons / scene.num_sensors)


# ---- the lixel statistics file, LixelStatistics.cpp:19-83 -------------------------------
# A file of LixelStatistic records, twelve float32 each (FIELDS order),
# written back to back; a trailing partial record is ignored.

def write(statistics: dict, path: str) -> None:
    """calibration::write: `statistics` as lixel_statistics returns it."""
    rows = np.stack([np.asarray(statistics[f], dtype="<f4") for f in FIELDS], axis=1)
    try:
        with open(path, "wb") as f:
            f.write(np.ascontiguousarray(rows).tobytes())
    except OSError:
        raise RuntimeError(f"LixelStatistics: Unable to write file: '{path}'") from None


def read(path: str) -> dict:
    """calibration::read."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError:
        raise RuntimeError(f"LixelStatistics: Unable to read file: '{path}'") from None
    n = len(data) // (4 * len(FIELDS))
    rows = np.frombuffer(data, dtype="<f4", count=n * len(FIELDS)).reshape(n, len(FIELDS))
    return {f: rows[:, k].copy() for k, f in enumerate(FIELDS)}


def read_efficiencies(path: str) -> np.ndarray:
    """calibration::read_efficiencies: the efficiency of every lixel, the
    per-lixel input of the night-sky background injection."""
    return read(path)["efficiency"].astype(np.float32)
