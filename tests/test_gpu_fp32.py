"""The batched FP32 tracer against the FP64 tracer (which is bit-identical
to the reference): same uniforms photon by photon, and per-sensor
histograms."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def js_divergence(a, b):
    """Jensen-Shannon divergence (natural log) of two count histograms."""
    p = a / a.sum()
    q = b / b.sum()
    m = 0.5 * (p + q)
    def kl(x, y):
        k = x > 0
        return float(np.sum(x[k] * np.log(x[k] / y[k])))
    return 0.5 * kl(p, m) + 0.5 * kl(q, m)


def trace(eng, flat, ph, tracer, seed, max_int, outputs=("sensor", "x", "y", "time")):
    import torch
    scene = eng.Scene(flat)
    dtype = torch.float32 if tracer.startswith("fp32") else torch.float64
    out = scene.propagate(eng.photons_to_device(ph, dtype=dtype), eng.PropagationConfig(max_int),
                          eng.Philox(seed), tracer=tracer, outputs=outputs,
                          out_dtype=dtype)
    got = {k: v.cpu().numpy() for k, v in out.items()}
    scene.close()
    return got


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available()
    from merlict_development_kit_b200 import engine
    return engine


def rounded_to_f32(ph):
    """The photon batch with every plane rounded to float32: the FP32 tracer
    reads exactly these values, and the FP64 tracer gets them widened."""
    return {k: v.astype(np.float32).astype(np.float64) for k, v in ph.items()}


@pytest.mark.parametrize("name,source,n", [
    ("reflector_camera", (2.0, 10.0, 1.5), 400_000),
    ("light_field_small", (5.55, 21.4, 0.5), 400_000),
])
def test_fp32_replay_agreement_with_fp64(eng, name, source, n):
    """Same photons, same Philox stream: at least 99.99 % of the photons end
    on the same sensor, and those agree on the hit position within 1e-6 m
    (99.9th percentile) and on the arrival time within 1e-14 s."""
    from merlict_development_kit_b200 import photons as P
    flat, _, _, meta = load_golden(name)
    ph = rounded_to_f32(P.downward_disc_source(n, 77, *source))
    a = trace(eng, flat, ph, "fp64", 5, meta["max_interactions"])
    b = trace(eng, flat, ph, "fp32", 5, meta["max_interactions"])
    agree = float(np.mean(a["sensor"] == b["sensor"]))
    assert agree >= 0.9999, agree
    both = (a["sensor"] >= 0) & (a["sensor"] == b["sensor"])
    dx = np.hypot(a["x"][both] - b["x"][both], a["y"][both] - b["y"][both])
    assert np.quantile(dx, 0.999) < 1e-6, np.quantile(dx, 0.999)
    assert np.max(np.abs(a["time"][both] - b["time"][both])) < 1e-14


def test_fp32_histograms_match_fp64_within_js(eng):
    from merlict_development_kit_b200 import photons as P
    flat, _, _, meta = load_golden("light_field_small")
    ph = P.downward_disc_source(1_000_000, 78, 5.55, 21.4, 0.5)
    a = trace(eng, flat, ph, "fp64", 11, 10, outputs=("sensor",))
    b = trace(eng, flat, ph, "fp32", 12, 10, outputs=("sensor",))
    ha = np.bincount(a["sensor"][a["sensor"] >= 0], minlength=flat.num_sensors)
    hb = np.bincount(b["sensor"][b["sensor"] >= 0], minlength=flat.num_sensors)
    assert js_divergence(ha.astype(float), hb.astype(float)) < 1e-3


def test_fp32_primitive_zoo_statistics(eng):
    """Every primitive kind.  A ray that leaves a sphere or cylinder has a
    root within rounding of zero, and merlict takes the surface's far side
    or nothing on the sign of that rounding (Sphere.cpp:96-103,
    ZaxisCylinderRayIntersectionEquation.cpp:54-60); no other arithmetic can
    repeat that coin flip photon by photon, so photons that met a sphere or
    cylinder are compared by their histograms only."""
    import torch
    from merlict_development_kit_b200 import abi, photons as P
    flat, _, _, meta = load_golden("primitive_zoo")
    ph = rounded_to_f32(P.isotropic_shell_source(400_000, 79, 4.0, 2.5))
    out = {}
    for tracer in ("fp64", "fp32"):
        scene = eng.Scene(flat)
        dtype = torch.float32 if tracer == "fp32" else torch.float64
        o = scene.propagate(eng.photons_to_device(ph, dtype=dtype), eng.PropagationConfig(10),
                            eng.Philox(13), tracer=tracer, outputs=("sensor",), history=True)
        out[tracer] = (o["sensor"].cpu().numpy(), eng.history_to_numpy(o["history"])["leaf"])
        scene.close()
    prim = np.asarray(flat.leaf_primitive)
    coin = np.isin(prim, [abi.PRIM_SPHERE, abi.PRIM_CYLINDER])
    def touched(leaves):
        return (coin[np.clip(leaves, 0, None)] & (leaves >= 0)).any(axis=1)
    (sa, la), (sb, lb) = out["fp64"], out["fp32"]
    plain = ~touched(la) & ~touched(lb)
    assert plain.mean() > 0.8
    assert float(np.mean(sa[plain] == sb[plain])) >= 0.9999
    ha = np.bincount(sa[sa >= 0], minlength=flat.num_sensors)
    hb = np.bincount(sb[sb >= 0], minlength=flat.num_sensors)
    assert js_divergence(ha.astype(float), hb.astype(float)) < 1e-3


def test_fp32_out_of_range_wavelength_raises(eng):
    flat, photons, _, _ = load_golden("mirror_absorber")
    ph = {k: v.copy() for k, v in photons.items()}
    ph["wavelength"][:] = 1500e-9
    with pytest.raises(IndexError):
        trace(eng, flat, ph, "fp32", 1, 5)


def test_fp32_pure_is_no_better_than_fp32(eng):
    """The textbook single-precision form (no rebasing, no Newton step) is
    the precision study's lower bound: it agrees with FP64 less often than
    the FP32 form, but still traces the scene."""
    from merlict_development_kit_b200 import photons as P
    flat, _, _, meta = load_golden("reflector_camera")
    ph = rounded_to_f32(P.downward_disc_source(200_000, 80, 2.0, 10.0, 1.5))
    a = trace(eng, flat, ph, "fp64", 5, 5)
    b = trace(eng, flat, ph, "fp32", 5, 5)
    c = trace(eng, flat, ph, "fp32_pure", 5, 5)
    agree_fp32 = float(np.mean(a["sensor"] == b["sensor"]))
    agree_pure = float(np.mean(a["sensor"] == c["sensor"]))
    assert agree_fp32 >= agree_pure
    assert agree_pure > 0.5


def test_precision_study_on_the_large_reflector(eng):
    """The precision study of the large reflector (curvature radius 213 m,
    8,443 pixels at 106.5 m): FP32 with the FP64 Newton step keeps >= 99.99 %
    of the photons on the FP64 tracer's pixel; the textbook single-precision
    cap quadratic (no correction) is no more accurate."""
    from merlict_development_kit_b200 import factories as F, photons as P, precision
    flat = F.large_reflector_camera().flatten()
    ph = P.downward_disc_source_device(1_000_000, 31, 40.0, 110.0, 3.5)
    r = precision.study(flat, ph, seed=3, max_interactions=5)
    fp32, pure = r["fp32"], r["fp32_pure"]
    assert fp32["on_sensors"] > 100_000
    assert fp32["sensor_disagreement"] <= 1e-4, fp32
    assert fp32["histogram_js"] < 1e-3
    assert fp32["position_error_m"]["q0.999"] < 1e-4, fp32
    assert pure["position_error_m"]["q0.99"] >= fp32["position_error_m"]["q0.99"], (pure, fp32)
