"""TEST INFRASTRUCTURE -- a plain-Python restatement of merlict's signal
chain after binning, the checker of csrc/signal_chain.cu.

For one event, with the random draws taken from per-lixel Philox streams
(the engine's draw schedule, below):

1. photon pipelines: each sensor's arrivals sorted by arrival time
   (merlict_signal_processing/PipelinePhoton.cpp:25-65);
2. night-sky background: the exposure window centred on the mode of the
   Cherenkov arrival times, a Poisson stream of background photons per
   lixel, everything shifted to the window's start
   (merlict_portal_plenoscope/night_sky_background/Injector.cpp:8-98);
3. photo-electric conversion: quantum efficiency, crosstalk, dark pulses
   (merlict_signal_processing/PhotoElectricConverter.cpp:31-90);
4. single-pulse extraction into time slices
   (merlict_signal_processing/pulse_extraction.cpp:9-35).

Draw schedule: stage s (1 background, 2 conversion, 3 extraction) of lixel
i draws uniforms k = 0, 1, 2, ... of Philox stream
((0xF0 | s) << 56) | (offset + i), in the order merlict's code asks for
them; a normal deviate takes two uniforms u1, u2 and is
mean + std sqrt(-2 ln(1 - u1)) cos(2 pi u2).

Only tests/ import this module.
"""
from __future__ import annotations

import math

import numpy as np

from merlict_development_kit_b200.scenery import Func1

STAGE_NSB, STAGE_PEC, STAGE_EXTRACT = 1, 2, 3
NUMBER_TIME_SLICES = 100
NIGHT_SKY_BACKGROUND = -100
PHOTO_ELECTRIC_CONVERTER_ACCIDENTAL = -201
PHOTO_ELECTRIC_CONVERTER_CROSSTALK = -202
DBL_MAX = np.finfo(np.float64).max
DBL_MIN = np.finfo(np.float64).tiny

_M0, _M1, _W0, _W1, _TAG = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85, 0x6d6c6374
_U32 = 0xFFFFFFFF


def philox_bits(seed: int, stream: int, k: int) -> int:
    """mlgpu_philox_bits of include/merlict_b200_philox.h."""
    c0, c1, c2, c3 = k & _U32, stream & _U32, (stream >> 32) & _U32, _TAG
    k0, k1 = seed & _U32, (seed >> 32) & _U32
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & _U32, p1 & _U32, ((p0 >> 32) ^ c3 ^ k1) & _U32, p0 & _U32
        k0 = (k0 + _W0) & _U32
        k1 = (k1 + _W1) & _U32
    return (c0 << 32) | c1


def philox_uniform(seed: int, stream: int, k: int) -> float:
    return float(philox_bits(seed, stream, k) >> 11) * (1.0 / 9007199254740992.0)


def signal_stream(stage: int, offset: int, lixel: int) -> int:
    return ((0xF0 | stage) << 56) | ((offset + lixel) & ((1 << 56) - 1))


class Draws:
    """One lixel's stream of one stage."""

    def __init__(self, seed, stage, offset, lixel):
        self.seed = seed
        self.stream = signal_stream(stage, offset, lixel)
        self.k = 0

    def uniform(self) -> float:
        u = philox_uniform(self.seed, self.stream, self.k)
        self.k += 1
        return u

    def expovariate(self, rate: float) -> float:
        """Generator::expovariate (merlict/random/Generator.cpp:36-39)."""
        u = self.uniform()
        with np.errstate(divide="ignore"):
            return float(np.float64(-math.log(u) if u > 0.0 else math.inf) / np.float64(rate))

    def normal(self, mean: float, std: float) -> float:
        u1 = self.uniform()
        u2 = self.uniform()
        return mean + std * (math.sqrt(-2.0 * math.log(1.0 - u1)) * math.cos(2.0 * math.pi * u2))


def photon_pipelines(sensor, time, wavelength, truth, num_sensors):
    """get_photon_pipelines: per sensor [(time, wavelength, truth)] by time
    (ties in input order)."""
    pipes = [[] for _ in range(num_sensors)]
    for i in range(len(sensor)):
        s = int(sensor[i])
        if s >= 0:
            pipes[s].append((float(time[i]), float(wavelength[i]), int(truth[i])))
    for p in pipes:
        p.sort(key=lambda r: r[0])
    return pipes


def nsb_exposure_start_time(pipes, exposure_time: float) -> float:
    """Injector.cpp:20-59: the mode of the Cherenkov arrival times on
    2 + sqrt(n) linearly spaced bin edges, minus half the exposure."""
    n = 0
    lo, hi = DBL_MAX, DBL_MIN
    times = []
    for p in pipes:
        if p:
            if p[0][0] < lo:
                lo = p[0][0]
            if p[-1][0] > hi:
                hi = p[-1][0]
            n += len(p)
        times.extend(r[0] for r in p)
    if n == 0:
        mode = 0.0
    else:
        count = int(2.0 + math.sqrt(float(n)))
        step = (hi - lo) / float(count - 1)
        edges = [lo + step * float(i) for i in range(count)]
        edges.sort()
        bins = [0] * (count - 1)
        import bisect
        for t in times:
            j = bisect.bisect_right(edges, t)
            if j == 0 or j == len(edges):
                continue
            bins[j - 1] += 1
        arg, best = 0, 0
        for j, c in enumerate(bins):
            if c > best:
                arg, best = j, c
        mode = 0.5 * (edges[arg + 1] + edges[arg])
    return mode - 0.5 * exposure_time


def inject_nsb(pipes, exposure_time, lixel_efficiency, nsb_rate, num_lixel, cdf: Func1,
               total_integral, seed, offset):
    """Injector.cpp:8-98 with per-lixel streams.  Returns the new pipelines
    (times shifted by the window start), the start, and the background
    photons per lixel."""
    if len(pipes) == 0:
        return pipes, 0.0, []
    S = nsb_exposure_start_time(pipes, exposure_time)
    out, counts = [], []
    for i, p in enumerate(pipes):
        q, k = inject_nsb_lixel(p, S, exposure_time, lixel_efficiency[i], nsb_rate, num_lixel,
                                cdf, total_integral, Draws(seed, STAGE_NSB, offset, i))
        out.append(q)
        counts.append(k)
    return out, S, counts


def inject_nsb_lixel(p, S, exposure_time, efficiency, nsb_rate, num_lixel, cdf: Func1,
                     total_integral, d: Draws):
    """One lixel of Injector.cpp:60-97 for a window starting at S."""
    rate = nsb_rate * float(np.float32(efficiency)) / float(num_lixel)
    times = []
    s = d.expovariate(rate)
    while s < exposure_time:
        nxt = d.expovariate(rate)
        times.append(S + s)
        s = s + nxt
    q = list(p)
    for t in times:
        q.append((t, cdf.evaluate(d.uniform() * total_integral), NIGHT_SKY_BACKGROUND))
    q.sort(key=lambda r: r[0])
    return [(t - S, w, tr) for (t, w, tr) in q], len(times)


def photo_electric(pipe, qe: Func1, dark_rate, p_second, exposure_time, d: Draws):
    """Converter::get_pulse_pipeline_for_photon_pipeline and add_pulse."""
    pulses = []

    def add(t, truth):
        pulses.append((t, truth))
        if p_second >= d.uniform():
            add(t, PHOTO_ELECTRIC_CONVERTER_CROSSTALK)

    for (t, w, truth) in pipe:
        if qe.evaluate(w) >= d.uniform():
            add(t, truth)
    s = d.expovariate(dark_rate)
    while s < exposure_time:
        nxt = d.expovariate(dark_rate)
        add(s, PHOTO_ELECTRIC_CONVERTER_ACCIDENTAL)
        s = s + nxt
    return pulses


def c_round(x: float) -> int:
    """C's round(): to the nearest integer, halves away from zero."""
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1
    return int(r) if x >= 0 else -int(r)


def extract(pulses, time_slice_duration, arrival_time_std, d: Draws):
    """pulse_extraction.cpp:9-35."""
    out = []
    for (t, truth) in pulses:
        reco = t + d.normal(0.0, arrival_time_std)
        x = reco / time_slice_duration if time_slice_duration != 0.0 else math.nan
        if not (-2147483648.0 <= x <= 2147483647.0):
            continue
        sl = c_round(x)
        if 0 <= sl < NUMBER_TIME_SLICES:
            out.append((sl, truth))
    return out


def signal_chain(sensor, time, wavelength, truth, num_sensors, lixel_efficiency, *,
                 qe: Func1, dark_rate, probability_for_second_puls, nsb_cdf: Func1,
                 nsb_total_integral, nsb_rate, num_lixel, nsb_exposure_time,
                 time_slice_duration, arrival_time_std, seed, offset=0):
    """The whole chain for one event; returns a dict of the channels (list
    of [(slice, truth)]), the background window start, the background
    counts and the intermediate photon and pulse pipelines."""
    pipes = photon_pipelines(sensor, time, wavelength, truth, num_sensors)
    pipes, S, counts = inject_nsb(pipes, nsb_exposure_time, lixel_efficiency, nsb_rate, num_lixel,
                                  nsb_cdf, nsb_total_integral, seed, offset)
    electric = [photo_electric(p, qe, dark_rate, probability_for_second_puls, nsb_exposure_time,
                               Draws(seed, STAGE_PEC, offset, i)) for i, p in enumerate(pipes)]
    channels = [extract(e, time_slice_duration, arrival_time_std,
                        Draws(seed, STAGE_EXTRACT, offset, i)) for i, e in enumerate(electric)]
    return {"channels": channels, "nsb_exposure_start_time": S, "nsb_count": counts,
            "photon_pipelines": pipes, "electric_pipelines": electric}
