"""Precision study of the single-precision tracer forms against the FP64
tracer (which reproduces merlict bit for bit).

The forms trace the same photons with the same Philox streams, so every
photon makes the same random choices in each form until the forms disagree
on a surface; the study reports, per form:

* the sensor disagreement rate (photons ending on another sensor, or on a
  sensor in one form and none in the other);
* for photons on the same sensor: the error distribution of the hit
  position in the sensor frame (x, y), of the incident direction (theta_x,
  theta_y) and of the arrival time;
* the Jensen-Shannon divergence of the per-sensor count histograms.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine

OUTPUTS = ("sensor", "x", "y", "time", "theta_x", "theta_y")
QUANTILES = (0.5, 0.99, 0.999, 1.0)


def js_divergence(a: np.ndarray, b: np.ndarray) -> float:
    """Jensen-Shannon divergence (natural log) of two count histograms."""
    p = a / max(a.sum(), 1)
    q = b / max(b.sum(), 1)
    m = 0.5 * (p + q)

    def kl(x, y):
        k = x > 0
        return float(np.sum(x[k] * np.log(x[k] / y[k])))
    return 0.5 * kl(p, m) + 0.5 * kl(q, m)


def _quantiles(x: np.ndarray) -> dict:
    if x.size == 0:
        return {f"q{q:g}": None for q in QUANTILES}
    return {f"q{q:g}": float(np.quantile(x, q)) for q in QUANTILES}


def _trace(scene, part: dict, tracer: str, seed: int, offset: int, max_interactions: int):
    dtype = torch.float32 if tracer.startswith("fp32") else torch.float64
    ph = {k: v.to(dtype).contiguous() for k, v in part.items()}
    return scene.propagate(ph, engine.PropagationConfig(max_interactions),
                           engine.Philox(seed, photon_offset=offset), tracer=tracer,
                           outputs=OUTPUTS, out_dtype=torch.float64)


def study(flat, photons: dict, seed: int = 1, max_interactions: int = 5,
          forms=("fp32", "fp32_pure"), chunk: int = 1 << 24) -> dict:
    """Traces `photons` (device planes, rounded to float32 first so that every
    form reads the same photons) with the FP64 tracer and with each form in
    `forms`, chunk by chunk with the same Philox streams, and compares them
    photon by photon."""
    scene = engine.Scene(flat)
    n = int(photons["wavelength"].shape[0])
    acc = {f: {"same": 0, "on": 0, "pos": [], "dir": [], "time": [],
               "h_ref": np.zeros(flat.num_sensors), "h": np.zeros(flat.num_sensors)}
           for f in forms}
    try:
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            part = {k: v[a:b].to(torch.float32) for k, v in photons.items()}
            ref = _trace(scene, part, "fp64", seed, a, max_interactions)
            rs = ref["sensor"]
            h_ref = torch.bincount(rs[rs >= 0].long(), minlength=flat.num_sensors).cpu().numpy()
            for f in forms:
                got = _trace(scene, part, f, seed, a, max_interactions)
                gs = got["sensor"]
                both = (rs == gs) & (rs >= 0)
                A = acc[f]
                A["same"] += int((rs == gs).sum())
                A["on"] += int((rs >= 0).sum())
                A["pos"].append(torch.hypot(ref["x"][both] - got["x"][both],
                                            ref["y"][both] - got["y"][both]).float().cpu().numpy())
                A["dir"].append(torch.hypot(ref["theta_x"][both] - got["theta_x"][both],
                                            ref["theta_y"][both] - got["theta_y"][both]
                                            ).float().cpu().numpy())
                A["time"].append((ref["time"][both] - got["time"][both]).abs().float().cpu().numpy())
                A["h_ref"] += h_ref
                A["h"] += torch.bincount(gs[gs >= 0].long(),
                                         minlength=flat.num_sensors).cpu().numpy()
                del got, gs, both
            del part, ref, rs
    finally:
        scene.close()
    out = {}
    for f, A in acc.items():
        out[f] = {
            "photons": n,
            "on_sensors": A["on"],
            "sensor_disagreement": 1.0 - A["same"] / n,
            "position_error_m": _quantiles(np.concatenate(A["pos"])),
            "direction_error_rad": _quantiles(np.concatenate(A["dir"])),
            "time_error_s": _quantiles(np.concatenate(A["time"])),
            "histogram_js": js_divergence(A["h_ref"], A["h"]),
        }
    return out
