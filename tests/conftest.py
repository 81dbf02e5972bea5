import glob
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    from merlict_development_kit_b200 import abi
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    flat = abi.FlatScene.from_npz(z)
    photons = {k[len("photon_"):]: z[k] for k in z.files if k.startswith("photon_")}
    ref = {k[len("ref_"):]: z[k] for k in z.files if k.startswith("ref_")}
    meta = {"max_interactions": int(z["max_interactions"]), "seed": int(z["seed"]),
            "uniforms": z["uniforms"] if "uniforms" in z.files else None}
    return flat, photons, ref, meta


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()
