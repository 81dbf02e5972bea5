"""The CPU oracle reproduces the reference library bit for bit on the golden
fixtures (which hold the reference's own outputs, see golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from parity import history_mismatches, mismatches


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_golden(oracle, name):
    flat, photons, ref, meta = load_golden(name)
    flat.validate()
    status, got, counters = oracle.propagate(
        flat, photons, meta["max_interactions"], seed=meta["seed"],
        uniforms=meta["uniforms"], history=True)
    assert status == 0
    assert mismatches(ref, got) == {}
    assert history_mismatches(ref["history"], got["history"]) == {}
    assert counters["steps"] > 0


def test_known_answer_two_mirrors(oracle):
    """PhotonTest.cpp:27-82: 42 bounces between two mirrors 1 m apart."""
    flat, photons, ref, meta = load_golden("two_mirrors")
    status, got, _ = oracle.propagate(flat, photons, 42, seed=1, history=True)
    n_int = (got["info"] >> 8) & 0xFF
    assert np.all(n_int == 43)
    dist = got["history"]["distance"].sum(axis=1)
    assert np.all(dist == 42 * 1.0 - 0.5)


def test_wavelength_out_of_table_range_is_an_error(oracle):
    """Func1::evaluate throws std::out_of_range outside [x_first, x_last)
    (Limits.cpp:37-46); the oracle reports MLGPU_ERR_OUT_OF_RANGE."""
    flat, photons, ref, meta = load_golden("mirror_absorber")
    ph = {k: v.copy() for k, v in photons.items()}
    ph["wavelength"][:] = 1500e-9
    status, got, _ = oracle.propagate(flat, ph, 5, seed=1)
    assert status == 2
    assert np.all(((got["info"] >> 24) & 0xFF)[got["final_leaf"] >= 0] == 2)
