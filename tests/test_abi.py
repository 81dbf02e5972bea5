"""The C ABI: the shared library exports every symbol the headers in include/
declare, and the ctypes mirror matches the C struct layouts."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import REPO
from merlict_development_kit_b200 import abi

HEADERS = [os.path.join(REPO, "include", h) for h in ("merlict_b200.h", "merlict_b200_surrogate.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|uint64_t|size_t)\s+(mlgpu_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from merlict_development_kit_b200 import _native
    lib = _native.lib()
    names = declared_functions()
    assert set(names) == set(_native.EXPORTED)
    for name in names:
        assert hasattr(lib, name), name
    assert lib.mlgpu_abi_version() == abi.ABI_VERSION


def test_struct_layouts_match_header(tmp_path):
    from merlict_development_kit_b200 import _native
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "merlict_b200.h"\n'
        '#include "merlict_b200_surrogate.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\","
        "sizeof(mlgpu_flat_scene), sizeof(mlgpu_photons), sizeof(mlgpu_history_entry),"
        "sizeof(mlgpu_results), sizeof(mlgpu_rng), sizeof(mlgpu_settings),"
        "offsetof(mlgpu_flat_scene, hex_unit_u), offsetof(mlgpu_flat_scene, num_sensors),"
        "sizeof(mlgpu_sg_sensor_grid), offsetof(mlgpu_sg_sensor_grid, hex_u),"
        "sizeof(mlgpu_signal_chain_config), offsetof(mlgpu_signal_chain_config, num_lixel),"
        "sizeof(mlgpu_photon_stream), offsetof(mlgpu_photon_stream, nsb_exposure_start_time));"
        "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I" + os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    expected = [C.sizeof(abi.mlgpu_flat_scene), C.sizeof(abi.mlgpu_photons),
                C.sizeof(abi.mlgpu_history_entry), C.sizeof(abi.mlgpu_results),
                C.sizeof(abi.mlgpu_rng), C.sizeof(abi.mlgpu_settings),
                abi.mlgpu_flat_scene.hex_unit_u.offset, abi.mlgpu_flat_scene.num_sensors.offset,
                C.sizeof(_native.mlgpu_sg_sensor_grid), _native.mlgpu_sg_sensor_grid.hex_u.offset,
                C.sizeof(abi.mlgpu_signal_chain_config), abi.mlgpu_signal_chain_config.num_lixel.offset,
                C.sizeof(abi.mlgpu_photon_stream),
                abi.mlgpu_photon_stream.nsb_exposure_start_time.offset]
    assert [int(x) for x in out] == expected


def test_scene_create_without_device_fails_cleanly():
    """No CPU fallback: without a GPU the engine refuses (here) or creates."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from merlict_development_kit_b200 import _native
    from conftest import load_golden
    flat, *_ = load_golden("sphere")
    s = flat.as_struct()
    h = C.c_void_p()
    status = _native.lib().mlgpu_scene_create(C.byref(s), C.byref(h))
    assert status == abi.ERR_NO_DEVICE
    assert "device" in _native.last_error()


def test_invalid_scene_is_rejected_before_any_device_work():
    from merlict_development_kit_b200 import _native
    from conftest import load_golden
    flat, *_ = load_golden("water_box")
    flat.node_skip[0] = 3   # root no longer covers the tree
    s = flat.as_struct()
    h = C.c_void_p()
    status = _native.lib().mlgpu_scene_create(C.byref(s), C.byref(h))
    assert status == abi.ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError):
        flat.validate()
