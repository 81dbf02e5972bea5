"""Allocation-free arrival binning, mlgpu_bin_arrivals_noalloc.

Some callers of this library cannot allocate device memory once they are
running: an application whose GPU memory is handed out by its own pool or
caching allocator, or an event loop with real-time deadlines, where
cudaMalloc/cudaFree may synchronise the device.  The binning kernels need
no scratch (they accumulate in the caller's outputs), so both binning entry
points allocate nothing; mlgpu_bin_arrivals_noalloc also checks that the
scene's device is current.  This file checks, through the C ABI, that it
gives exactly the counts and time histograms of mlgpu_bin_arrivals on two
calls in a row (integer counts: the tolerance is zero) without changing the
device's free memory, that the allocating entry point does not change it
either, and that a histogram of more keys than a scratch-based design
could hold is binned exactly.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def call_noalloc(scene, sensor, time, counts, hist, bins, t0, t1):
    import torch
    from merlict_development_kit_b200 import _native
    stream = torch.cuda.current_stream().cuda_stream
    status = _native.lib().mlgpu_bin_arrivals_noalloc(
        scene.handle, C.c_void_p(sensor.data_ptr()),
        C.c_void_p(time.data_ptr() if time is not None else None), int(sensor.shape[0]),
        C.c_void_p(counts.data_ptr()), C.c_void_p(hist.data_ptr() if hist is not None else None),
        int(bins), float(t0), float(t1), C.c_void_p(stream))
    return status


def test_noalloc_binning_matches_the_allocating_entry_point_on_two_calls():
    import torch
    from merlict_development_kit_b200 import _native, engine, photons as P
    flat, _, _, _ = load_golden("light_field_small")
    scene = engine.Scene(flat)
    ph = P.downward_disc_source(200_000, 21, 5.55, 21.4, 0.5)
    out = scene.propagate(engine.photons_to_device(ph), engine.PropagationConfig(10),
                          engine.Philox(8), outputs=("sensor", "time"))
    sensor, time = out["sensor"], out["time"]
    t = time[sensor >= 0]
    t0, t1 = float(t.min()) - 1e-12, float(t.max()) + 1e-12
    n_s = flat.num_sensors
    half = sensor[: sensor.shape[0] // 2].contiguous()
    counts = torch.full((n_s,), -1, dtype=torch.int32, device="cuda")
    hist = torch.full((n_s, 16), -1, dtype=torch.int32, device="cuda")
    counts2 = torch.full((n_s,), -1, dtype=torch.int32, device="cuda")
    launches0 = scene.kernel_launches()

    # A first call may load the library's device code into the context;
    # after it, calls must not change the device's free memory.
    _native.check(call_noalloc(scene, half, None, counts2, None, 0, 0.0, 1.0))
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]

    # first call: counts and a 16-bin time histogram of all photons
    _native.check(call_noalloc(scene, sensor, time, counts, hist, 16, t0, t1))
    torch.cuda.synchronize()
    # second call, right after: counts only, of a different (half) batch, so
    # anything left over from the first call in the outputs would show
    counts2.fill_(-1)
    _native.check(call_noalloc(scene, half, None, counts2, None, 0, 0.0, 1.0))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert scene.kernel_launches() - launches0 == 6

    # the allocating entry point on the same inputs
    ref_counts, ref_hist = scene.bin_arrivals(sensor, time, 16, t0, t1)
    ref_counts2, _ = scene.bin_arrivals(half)
    torch.cuda.synchronize()
    assert torch.equal(counts, ref_counts)
    assert torch.equal(hist, ref_hist)
    assert torch.equal(counts2, ref_counts2)
    assert int(counts2.sum()) == int((half >= 0).sum())
    assert not torch.equal(counts2, counts)
    scene.close()


def test_binning_allocates_nothing_and_takes_large_histograms():
    import torch
    from merlict_development_kit_b200 import engine
    flat, _, _, _ = load_golden("light_field_small")
    scene = engine.Scene(flat)
    n_s = flat.num_sensors
    bins = (4 * 1024 * 1024) // n_s + 1            # sensors x (bins + 1) > 4 Mi keys
    g = torch.Generator(device="cpu").manual_seed(3)
    n = 3_000_000
    sensor = torch.randint(-1, n_s + 2, (n,), generator=g, dtype=torch.int32)
    sensor[: n // 3] = 7                            # one sensor takes a third of the arrivals
    time = torch.rand(n, generator=g, dtype=torch.float64) * 1.2 - 0.1
    s_d, t_d = sensor.cuda(), time.cuda()
    counts = torch.full((n_s,), -1, dtype=torch.int32, device="cuda")
    hist = torch.full((n_s, bins), -1, dtype=torch.int32, device="cuda")
    # warm-up, then neither entry point may change the free device memory
    _native_check(call_noalloc(scene, s_d, t_d, counts, hist, bins, 0.0, 1.0))
    scene.bin_arrivals(s_d, t_d, bins, 0.0, 1.0)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    counts.fill_(-1)
    hist.fill_(-1)
    _native_check(call_noalloc(scene, s_d, t_d, counts, hist, bins, 0.0, 1.0))
    ref_counts, ref_hist = scene.bin_arrivals(s_d, t_d, bins, 0.0, 1.0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    # numpy: sensors in [0, n_s) counted; times in [0, 1) binned
    s_np, t_np = sensor.numpy(), time.numpy()
    ok = (s_np >= 0) & (s_np < n_s)
    want_counts = np.bincount(s_np[ok], minlength=n_s)
    f = t_np[ok] * bins
    inb = (f >= 0) & (f < bins)
    keys = s_np[ok][inb].astype(np.int64) * bins + f[inb].astype(np.int64)
    want_hist = np.bincount(keys, minlength=n_s * bins).reshape(n_s, bins)
    assert np.array_equal(counts.cpu().numpy(), want_counts)
    assert np.array_equal(hist.cpu().numpy(), want_hist)
    assert torch.equal(ref_counts, counts) and torch.equal(ref_hist, hist)
    scene.close()


def _native_check(status):
    from merlict_development_kit_b200 import _native
    _native.check(status)
