"""The BVH the tracers walk, checked on the host: the builder
(csrc/bvh_build.cu) is compiled with the host compiler together with
tests/bvh_invariants.cpp, which checks that every child box contains the
bounding spheres of all leaves beneath it, that every leaf with geometry
is in exactly one leaf range, and that each level is the index range the
level kernels walk.  The candidates the BVH proposes are then put through
merlict's own sphere test, so these properties are what keeps the tracers'
hits merlict's."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden_names, load_golden

CSRC = os.path.join(REPO, "merlict_development_kit_b200", "csrc")
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INCLUDE, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    out = str(tmp_path_factory.mktemp("bvh") / "bvh_invariants.so")
    cmd = ["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", CSRC, "-I", os.path.join(REPO, "include"),
           "-I", CUDA_INCLUDE, "-x", "c++", os.path.join(REPO, "tests", "bvh_invariants.cpp"),
           "-x", "c++", os.path.join(CSRC, "bvh_build.cu"), "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = C.CDLL(out)
    lib.bvh_invariants.restype = C.c_int64
    lib.bvh_invariants.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    return lib


def check(lib, flat):
    s = flat.as_struct()
    info = (C.c_int64 * 4)()
    bad = lib.bvh_invariants(C.addressof(s), info)
    return bad, {"nodes": info[0], "levels": info[1], "width": info[2], "leaves": info[3]}


@pytest.mark.parametrize("name", golden_names())
def test_bvh_of_every_golden_scene(checker, name):
    flat, *_ = load_golden(name)
    bad, info = check(checker, flat)
    assert bad == 0, info
    with_geometry = int(np.count_nonzero(np.asarray(flat.leaf_primitive) != 0))
    assert info["leaves"] == with_geometry


def test_bvh_of_the_light_field_telescope(checker):
    """78,378 leaves; eight children per node give a tree of 8 levels."""
    from merlict_development_kit_b200 import factories as F
    flat = F.light_field_telescope().flatten()
    bad, info = check(checker, flat)
    assert bad == 0, info
    assert info["width"] == 8 and info["leaves"] == 78378
    assert info["levels"] == 8


def test_bvh_of_the_large_reflector(checker):
    from merlict_development_kit_b200 import factories as F
    flat = F.large_reflector_camera().flatten()
    bad, info = check(checker, flat)
    assert bad == 0, info
