"""Comparison helpers shared by the parity tests."""
import numpy as np

PER_PHOTON = ("sensor", "final_leaf", "x", "y", "theta_x", "theta_y",
              "final_position", "final_direction")
HISTORY_FIELDS = ("position", "normal", "distance", "leaf", "interaction",
                  "from_outside_to_inside")


def same(a, b):
    """Elementwise equality that treats NaN == NaN (bit-exact otherwise)."""
    a = np.asarray(a)
    b = np.asarray(b)
    eq = a == b
    if a.dtype.kind == "f":
        eq |= np.isnan(a) & np.isnan(b)
    return eq


def mismatches(ref: dict, got: dict, keys=PER_PHOTON, info_mask=0xFFFFFF) -> dict:
    bad = {}
    for k in keys:
        if k not in got:
            continue
        eq = same(ref[k], got[k])
        if eq.ndim > 1:
            eq = eq.all(axis=tuple(range(1, eq.ndim)))
        if not eq.all():
            bad[k] = int((~eq).sum())
    if "info" in got:
        eq = (np.asarray(ref["info"]) & info_mask) == (np.asarray(got["info"]).astype(np.uint32) & info_mask)
        if not eq.all():
            bad["info"] = int((~eq).sum())
    s = np.asarray(ref["sensor"]) >= 0
    if "time" in got:
        eq = same(np.asarray(ref["time"])[s], np.asarray(got["time"])[s])
        if not eq.all():
            bad["time"] = int((~eq).sum())
    return bad


def history_mismatches(ref_hist, got_hist) -> dict:
    bad = {}
    n = min(len(ref_hist), len(got_hist))
    for f in HISTORY_FIELDS:
        eq = same(ref_hist[f][:n], got_hist[f][:n])
        if eq.ndim > 2:
            eq = eq.all(axis=2)
        if not eq.all():
            bad[f] = int((~eq).sum())
    return bad
