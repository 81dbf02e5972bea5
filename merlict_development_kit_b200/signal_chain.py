"""The signal chain after binning, on the device: from the photons that
reached the lixels of a light-field sensor to the extracted single pulses
of every lixel, and the photon-stream files merlict writes them to.

The steps and their merlict counterparts, as plenoscope_propagation.cpp:
201-247 chains them for one event:

* photon pipelines: each lixel's arrivals by arrival time
  (merlict_signal_processing/PipelinePhoton.cpp:25-65);
* night-sky background: an exposure window centred on the mode of the
  Cherenkov arrival times, Poisson background photons per lixel with
  wavelengths from the background spectrum, and all times relative to the
  window's start (merlict_portal_plenoscope/night_sky_background/
  Injector.cpp:8-98, Light.cpp:8-24);
* photo-electric conversion: quantum efficiency, crosstalk, dark pulses
  (merlict_signal_processing/PhotoElectricConverter.cpp:31-90);
* single-pulse extraction into 100 time slices
  (merlict_signal_processing/pulse_extraction.cpp:9-52);
* the photon stream and its simulation truth
  (merlict_signal_processing/PhotonStream.cpp:15-196).

`run` does the first four for one event in csrc/signal_chain.cu (one
thread per lixel, counter-based draws, two passes: count, then write);
the file formats are host code here.

Random draws.  merlict threads one generator through all lixels, which
would serialise the device.  Here stage s (1 background, 2 conversion,
3 extraction) of lixel i draws uniforms k = 0, 1, ... of the Philox stream
((0xF0 | s) << 56) | (offset + i) in the order merlict's code asks for
them, and a normal deviate (merlict's Generator::normal) is
mean + std sqrt(-2 ln(1 - u1)) cos(2 pi u2) of two uniforms.  With those
draws replayed into merlict's own code the outputs agree; with merlict's
own Mt19937 they agree in distribution.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass

import numpy as np

from . import abi
from .scenery import Func1, function_integral, function_inverse

NUMBER_TIME_SLICES = 100                       # pulse_extraction.h:13
NEXT_CHANNEL_MARKER = 255                      # PhotonStream.h:14
DEFAULT_SIMULATION_TRUTH = -1                  # simulation_truth.h:14-17
NIGHT_SKY_BACKGROUND = -100
PHOTO_ELECTRIC_CONVERTER_ACCIDENTAL = -201
PHOTO_ELECTRIC_CONVERTER_CROSSTALK = -202
APERTURE_RADIUS_OVERHEAD = 1.05                # NightSkyBackground.h:9-10
FOV_RADIUS_OVERHEAD = 1.20

ZERO_EFFICIENCY = Func1([[200e-9, 0.0], [1200e-9, 0.0]])   # PhotoElectricConverter.h:22-27


@dataclass
class PhotoElectricConverterConfig:
    """PhotoElectricConverter::Config (PhotoElectricConverter.cpp:10-14)."""
    quantum_efficiency_vs_wavelength: Func1 = ZERO_EFFICIENCY
    dark_rate: float = 0.0
    probability_for_second_puls: float = 0.0

    def check(self):
        """Converter::Converter (PhotoElectricConverter.cpp:16-27)."""
        if not self.probability_for_second_puls < 1.0:
            raise ValueError("Expected config->probability_for_second_puls < 1.0, but actual "
                             f"it is: {self.probability_for_second_puls}")


class SamplesFromDistribution:
    """random::SamplesFromDistribution (SamplesFromDistribution.cpp:7-28):
    draws by inverting the integral of a distribution."""

    def __init__(self, distribution: Func1):
        self.distribution = distribution
        integral = function_integral(distribution)
        self.total_integral_of_distribution = integral.max()
        self.cumulative_distribution_function = function_inverse(integral)

    def draw(self, uniform_0_to_1: float) -> float:
        return self.cumulative_distribution_function.evaluate(
            uniform_0_to_1 * self.total_integral_of_distribution)


def solid_angle_for_opening_angle(theta: float) -> float:
    """merlict/tools.cpp:25-48."""
    return 2.0 * math.pi * (1.0 - math.cos(theta))


class NightSkyBackgroundLight:
    """night_sky_background::Light (Light.cpp:8-24): the background's rate
    into the light-field sensor and its wavelength distribution.
    `sensor_geometry` is a factories.LightFieldSensorGeometry."""

    def __init__(self, sensor_geometry, flux_vs_wavelength: Func1):
        self.sensor_geometry = sensor_geometry
        self.flux_vs_wavelength = flux_vs_wavelength
        self.wavelength_probability = SamplesFromDistribution(flux_vs_wavelength)
        cfg = sensor_geometry.cfg
        self.fov_radius = FOV_RADIUS_OVERHEAD * (cfg.max_FoV_diameter / 2.0)
        self.fov_solid_angle = solid_angle_for_opening_angle(self.fov_radius)
        self.aperture_radius = (APERTURE_RADIUS_OVERHEAD *
                                cfg.expected_imaging_system_max_aperture_radius)
        self.aperture_area = math.pi * self.aperture_radius * self.aperture_radius
        self.rate = (self.wavelength_probability.total_integral_of_distribution *
                     self.aperture_area * self.fov_solid_angle)

    @property
    def num_lixel(self) -> int:
        return self.sensor_geometry.num_lixels


@dataclass
class SignalChainConfig:
    """Everything the chain needs besides the photons: the converter, the
    background light and the photon-stream settings of the plenoscope
    programs' configuration (plenoscope_propagation.cpp:138-175)."""
    converter: PhotoElectricConverterConfig
    light: NightSkyBackgroundLight
    nsb_exposure_time: float
    time_slice_duration: float
    single_photon_arrival_time_resolution: float


@dataclass
class PhotonStream:
    """The extracted pulses of one event: channel c holds
    arrival_time_slice[channel_offset[c]:channel_offset[c + 1]] and the same
    slice of simulation_truth_id (merlict's PhotonStream::Stream)."""
    channel_offset: np.ndarray
    arrival_time_slice: np.ndarray
    simulation_truth_id: np.ndarray
    time_slice_duration: float
    nsb_exposure_start_time: float = 0.0
    nsb_count: np.ndarray | None = None

    @property
    def num_channels(self) -> int:
        return len(self.channel_offset) - 1

    def channel(self, c: int):
        a, b = int(self.channel_offset[c]), int(self.channel_offset[c + 1])
        return self.arrival_time_slice[a:b], self.simulation_truth_id[a:b]

    @staticmethod
    def from_channels(channels, time_slice_duration: float) -> "PhotonStream":
        """From a list of [(slice, truth id)] per channel."""
        off = np.zeros(len(channels) + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(c) for c in channels])
        sl = np.array([p[0] for c in channels for p in c], dtype=np.uint8)
        tr = np.array([p[1] for c in channels for p in c], dtype=np.int32)
        return PhotonStream(off, sl, tr, float(time_slice_duration))


# ---- the photon-stream files, PhotonStream.cpp -------------------------------------------

def num_symbols_to_represent(stream: PhotonStream) -> int:
    """PhotonStream.cpp:183-194: one symbol per pulse plus one marker
    between channels."""
    n = int(stream.channel_offset[-1]) + stream.num_channels
    return n - 1 if n > 0 else 0


def write(stream: PhotonStream, path: str):
    """PhotonStream::write (PhotonStream.cpp:15-57): a 16-byte header
    (float32 time slice duration, uint32 channels, uint32 time slices,
    uint32 symbols), then each channel's slices with a 255 between
    channels."""
    if np.any(stream.arrival_time_slice == NEXT_CHANNEL_MARKER):
        raise RuntimeError(f"PhotonStream::write({path}) Expected arrival slice of photon != "
                           "NEXT_CHANNEL_MARKER")
    n = stream.num_channels
    body = bytearray()
    for c in range(n):
        sl, _ = stream.channel(c)
        body += sl.astype(np.uint8).tobytes()
        if c < n - 1:
            body.append(NEXT_CHANNEL_MARKER)
    try:
        with open(path, "wb") as f:
            f.write(struct.pack("<fIII", stream.time_slice_duration, n, NUMBER_TIME_SLICES,
                                num_symbols_to_represent(stream)))
            f.write(bytes(body))
    except OSError:
        raise RuntimeError(f"Can not write file '{path}'.") from None


def write_simulation_truth(stream: PhotonStream, path: str):
    """PhotonStream::write_simulation_truth (PhotonStream.cpp:59-78): the
    int32 truth id of every pulse, channel after channel."""
    try:
        with open(path, "wb") as f:
            f.write(np.asarray(stream.simulation_truth_id, dtype="<i4").tobytes())
    except OSError:
        raise RuntimeError(f"Can not write file '{path}'.") from None


def read(path: str) -> PhotonStream:
    """PhotonStream::read (PhotonStream.cpp:80-121)."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError:
        raise RuntimeError(f"PhotonStream: Unable to open file: '{path}'") from None
    duration, _, slices, symbols = struct.unpack_from("<fIII", data, 0)
    if slices != NUMBER_TIME_SLICES:
        raise RuntimeError(f"PhotonStream::read({path}) Expected num_time_slices == "
                           f"{NUMBER_TIME_SLICES}, but actual it is {slices}")
    sym = np.frombuffer(data, dtype=np.uint8, count=symbols, offset=16)
    marks = np.flatnonzero(sym == NEXT_CHANNEL_MARKER)
    num_channels = len(marks) + 1 if symbols > 0 else 0
    pulses = sym[sym != NEXT_CHANNEL_MARKER]
    off = np.zeros(num_channels + 1, dtype=np.uint64)
    if num_channels:
        # pulses before the k-th marker belong to channels < k+1
        before = marks - np.arange(len(marks))
        off[1:num_channels] = before
        off[num_channels] = len(pulses)
    return PhotonStream(off, pulses.copy(), np.full(len(pulses), DEFAULT_SIMULATION_TRUTH,
                                                    dtype=np.int32), float(duration))


def read_with_simulation_truth(path: str, truth_path: str) -> PhotonStream:
    """PhotonStream::read_with_simulation_truth (PhotonStream.cpp:123-154)."""
    s = read(path)
    try:
        with open(truth_path, "rb") as f:
            data = f.read()
    except OSError:
        raise RuntimeError(f"PhotonStream: Unable to open file: '{truth_path}'") from None
    n = int(s.channel_offset[-1]) if s.num_channels else 0
    s.simulation_truth_id = np.frombuffer(data, dtype="<i4", count=n).astype(np.int32)
    return s


# ---- one event on the device ---------------------------------------------------------

def _points(f: Func1) -> np.ndarray:
    return np.ascontiguousarray(np.array(f.points, dtype=np.float64).reshape(-1, 3))


def device_config(cfg: SignalChainConfig):
    """The mlgpu_signal_chain_config of `cfg` and the arrays it points to
    (built once per configuration object and kept on it)."""
    cached = getattr(cfg, "_device_config", None)
    if cached is not None and cached[0] == _config_key(cfg):
        return cached[1], cached[2]
    cfg.converter.check()
    qe = _points(cfg.converter.quantum_efficiency_vs_wavelength)
    cdf = _points(cfg.light.wavelength_probability.cumulative_distribution_function)
    c = abi.mlgpu_signal_chain_config()
    c.quantum_efficiency = qe.ctypes.data
    c.num_quantum_efficiency = qe.shape[0]
    c.dark_rate = cfg.converter.dark_rate
    c.probability_for_second_puls = cfg.converter.probability_for_second_puls
    c.nsb_wavelength_cdf = cdf.ctypes.data
    c.num_nsb_wavelength_cdf = cdf.shape[0]
    c.nsb_total_integral = cfg.light.wavelength_probability.total_integral_of_distribution
    c.nsb_rate = cfg.light.rate
    c.num_lixel = cfg.light.num_lixel
    c.nsb_exposure_time = cfg.nsb_exposure_time
    c.time_slice_duration = cfg.time_slice_duration
    c.arrival_time_std = cfg.single_photon_arrival_time_resolution
    cfg._device_config = (_config_key(cfg), c, [qe, cdf])
    return c, [qe, cdf]


def _config_key(cfg: SignalChainConfig):
    conv = cfg.converter
    return (id(conv.quantum_efficiency_vs_wavelength), conv.dark_rate,
            conv.probability_for_second_puls, id(cfg.light), cfg.light.rate,
            cfg.nsb_exposure_time, cfg.time_slice_duration,
            cfg.single_photon_arrival_time_resolution)


def run(scene, cfg: SignalChainConfig, sensor, arrival_time, wavelength, truth_id,
        lixel_efficiency, rng, capacity: int | None = None, stream=None) -> PhotonStream:
    """The signal chain for one event on the device (mlgpu_signal_chain).
    `sensor`, `arrival_time`, `wavelength` and `truth_id` are per-photon
    CUDA tensors (int32, float64, float64, int32; sensor < 0: none), e.g. a
    propagation's outputs with its input wavelengths and ids;
    `lixel_efficiency` a float32 CUDA tensor, one efficiency per sensor (the
    calibration's, see calibration.read_efficiencies); `rng` an
    engine.Philox.  Returns the PhotonStream with its arrays on the device
    (torch tensors)."""
    import ctypes as C

    import torch

    from . import _native
    from .engine import _stream_handle
    dev = sensor.device
    n = int(sensor.numel())
    num_sensors = int(lixel_efficiency.numel())
    c, keep = device_config(cfg)
    r, rkeep = rng._struct(n)
    cap = int(capacity) if capacity is not None else max(1024, 2 * n + 8 * num_sensors)
    args = [sensor.contiguous(), arrival_time.contiguous().to(torch.float64),
            wavelength.contiguous().to(torch.float64), truth_id.contiguous().to(torch.int32),
            lixel_efficiency.contiguous().to(torch.float32)]
    sh = C.c_void_p(_stream_handle(stream))
    for _ in range(2):
        off = torch.empty(num_sensors + 1, dtype=torch.int64, device=dev)
        sl = torch.empty(max(cap, 1), dtype=torch.uint8, device=dev)
        tr = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
        nsb = torch.empty(max(num_sensors, 1), dtype=torch.int32, device=dev)
        out = abi.mlgpu_photon_stream()
        out.channel_offset = off.data_ptr()
        out.arrival_time_slice = sl.data_ptr()
        out.simulation_truth_id = tr.data_ptr()
        out.nsb_count = nsb.data_ptr()
        out.capacity = cap
        rc = _native.lib().mlgpu_signal_chain(
            scene.handle, C.byref(c), *[C.c_void_p(a.data_ptr()) for a in args[:4]], n,
            C.c_void_p(args[4].data_ptr()), num_sensors, C.byref(r), C.byref(out), sh)
        if rc == abi.ERR_INVALID_ARGUMENT and out.num_pulses > cap:
            cap = int(out.num_pulses)
            continue
        _native.check(rc)
        m = int(out.num_pulses)
        del keep, rkeep
        return PhotonStream(off, sl[:m], tr[:m], cfg.time_slice_duration,
                            float(out.nsb_exposure_start_time), nsb[:num_sensors])
    raise RuntimeError("the photon stream did not fit its buffers twice")


__all__ = [
    "NUMBER_TIME_SLICES", "NEXT_CHANNEL_MARKER", "NIGHT_SKY_BACKGROUND",
    "PHOTO_ELECTRIC_CONVERTER_ACCIDENTAL", "PHOTO_ELECTRIC_CONVERTER_CROSSTALK",
    "PhotoElectricConverterConfig", "SamplesFromDistribution", "NightSkyBackgroundLight",
    "SignalChainConfig", "PhotonStream", "write", "write_simulation_truth", "read",
    "read_with_simulation_truth", "num_symbols_to_represent", "run",
]
