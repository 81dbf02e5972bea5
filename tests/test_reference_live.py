"""Oracle against the live reference library (built here from the reference
sources) on larger samples than the fixtures hold, including the full
config-1 light-field telescope."""
import numpy as np
import pytest

from merlict_development_kit_b200 import photons as P
from oracle import oracle as O
from parity import mismatches

pytestmark = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")


@pytest.mark.parametrize("kind,params,source,n,max_int", [
    ("light_field_sensor", (10.7, 5.35, 6.5, 0.186, 9, 1.1, 0.9), (5.55, 21.4, 1.5), 20000, 10),
    ("reflector_camera", (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2), (2.0, 10.0, 1.5), 50000, 5),
    ("primitive_zoo", (), None, 50000, 10),
])
def test_oracle_matches_live_reference(oracle, kind, params, source, n, max_int):
    scene = O.RefScene(kind, params)
    flat = scene.flat()
    ph = (P.isotropic_shell_source(n, 31, 4.0, 2.5) if source is None
          else P.downward_disc_source(n, 31, *source))
    status, ref, _ = scene.propagate(ph, max_int, O.REPLAY_PHILOX, seed=4242, threads=8)
    assert status == 0
    st, got, _ = oracle.propagate(flat, ph, max_int, seed=4242)
    assert st == 0
    assert mismatches(ref, got) == {}


def test_reference_production_mode_statistics_agree_with_philox(oracle):
    """Production RNG: merlict's Mt19937 path and the Philox stream give the
    same per-pixel statistics (chi-squared on the config-0 camera)."""
    params = (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2)
    scene = O.RefScene("reflector_camera", params)
    flat = scene.flat()
    ph = P.downward_disc_source(200000, 5, 2.0, 10.0, 1.5)
    _, ref, _ = scene.propagate(ph, 5, O.REFERENCE_SINGLE_THREAD, seed=1)
    _, got, _ = oracle.propagate(flat, ph, 5, seed=99)
    a = np.bincount(ref["sensor"][ref["sensor"] >= 0], minlength=flat.num_sensors)
    b = np.bincount(got["sensor"][got["sensor"] >= 0], minlength=flat.num_sensors)
    m = (a + b) > 0
    chi2 = (((a - b) ** 2)[m] / (a + b)[m]).sum()
    dof = int(m.sum())
    assert chi2 < dof + 5 * np.sqrt(2 * dof)
