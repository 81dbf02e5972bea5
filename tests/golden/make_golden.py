"""Generates the golden fixtures in tests/golden/*.npz from the reference.

Each fixture holds a scene built by the reference library's own classes and
factories and flattened by the product's shim, a seeded photon batch, and
the results of the reference's own Propagator on it: merlict's propagation
driven photon by photon with a random::Generator that replays the engine's
Philox stream (or, for *_replay fixtures, an explicit uniform stream), then
Sensors::assign_photons.  Per-photon outputs are stored for every photon and
complete histories for the first HISTORY photons.

    python tests/golden/make_golden.py        # needs oracle/_ref (make -C oracle ref)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from merlict_development_kit_b200 import photons as P  # noqa: E402
from oracle.oracle import REPLAY_PHILOX, REPLAY_UNIFORMS, RefScene  # noqa: E402

HISTORY = 256
SEED = 20241203

# the config-0 reflector camera: f=4.9 m Davies-Cotton dish of 30 facets,
# 1440 hexagonal pixels of 9.5 mm, shield disc
REFLECTOR_CAMERA = (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2)
# the light-field sensor of config 1 with a 1 degree field of view
LIGHT_FIELD_SMALL = (10.7, 5.35, 1.0, 0.186, 9, 1.1, 0.9)


def sources():
    n = 2000
    return [
        # name, scene kind, params, photons, max interactions, rng
        ("two_mirrors", "two_mirrors", (),
         P.make_batch(np.tile([0.0, 0.0, 0.5], (16, 1)), np.tile([0.0, 0.0, 1.0], (16, 1)),
                      np.full(16, 433e-9)), 42, "philox"),
        ("mirror_absorber", "mirror_absorber", (),
         P.make_batch(np.tile([-2.0, 0.0, 0.0], (n, 1)), np.tile([1.0, 0.0, 0.0], (n, 1)),
                      np.arange(1, n + 1) / n * 100e-9 + 250e-9), 5, "philox"),
        ("water_box", "water_box", (),
         P.make_batch(np.zeros((n, 3)), np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 433e-9)),
         5, "philox"),
        ("absorbing_box", "absorbing_box", (),
         P.make_batch(np.zeros((n, 3)), np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 433e-9)),
         5, "philox"),
        ("biconvex_lens", "biconvex_lens", (), P.downward_disc_source(n, 3, 0.125, 1.0, 0.5), 5,
         "philox"),
        ("sphere", "sphere", (), P.isotropic_shell_source(500, 4, 4.0, 1.5), 5, "philox"),
        ("primitive_zoo", "primitive_zoo", (), P.isotropic_shell_source(4000, 5, 4.0, 2.5), 10,
         "philox"),
        ("reflector_camera", "reflector_camera", REFLECTOR_CAMERA,
         P.downward_disc_source(4000, 6, 2.0, 10.0, 1.5), 5, "philox"),
        ("reflector_camera_replay", "reflector_camera", REFLECTOR_CAMERA,
         P.downward_disc_source(1000, 7, 2.0, 10.0, 1.5), 5, "uniforms"),
        ("light_field_small", "light_field_sensor", LIGHT_FIELD_SMALL,
         P.downward_disc_source(4000, 8, 5.55, 21.4, 0.5), 10, "philox"),
    ]


def main(out_dir: str = HERE) -> None:
    for name, kind, params, ph, max_int, rng in sources():
        scene = RefScene(kind, params)
        flat = scene.flat()
        flat.validate()
        uniforms = None
        if rng == "uniforms":
            g = np.random.default_rng(SEED)
            uniforms = g.random((len(ph["wavelength"]), 3 * max_int))
            status, res, _ = scene.propagate(ph, max_int, REPLAY_UNIFORMS, uniforms=uniforms,
                                             history=True)
        else:
            status, res, _ = scene.propagate(ph, max_int, REPLAY_PHILOX, seed=SEED, history=True)
        if status != 0:
            raise RuntimeError(f"{name}: reference status {status}")
        d = flat.to_npz_dict()
        d.update({f"photon_{k}": v for k, v in ph.items()})
        d["max_interactions"] = np.int32(max_int)
        d["seed"] = np.uint64(SEED)
        if uniforms is not None:
            d["uniforms"] = uniforms
        for k in ("sensor", "final_leaf", "x", "y", "time", "theta_x", "theta_y",
                  "final_position", "final_direction"):
            d[f"ref_{k}"] = res[k]
        d["ref_info"] = res["info"] & np.uint32(0xFFFFFF)
        d["ref_history"] = res["history"][:HISTORY]
        path = os.path.join(out_dir, f"{name}.npz")
        np.savez_compressed(path, **d)
        hit = float((res["sensor"] >= 0).mean())
        print(f"{name}: {len(ph['wavelength'])} photons, {flat.num_leaves} leaves, "
              f"{hit:.3f} on sensors, {os.path.getsize(path) / 1e3:.0f} kB")


if __name__ == "__main__":
    main()
