"""Photon batches (structure of arrays) and the seeded photon sources of the
benchmark configurations.

A batch is a dict of numpy (or torch) arrays with the keys support_x,
support_y, support_z, direction_x, direction_y, direction_z, wavelength and
id -- the fields of merlict::Photon (merlict/Photon.h, RayForPropagation.h)
that a propagation reads.
"""
from __future__ import annotations

import numpy as np

PLANES = ("support_x", "support_y", "support_z",
          "direction_x", "direction_y", "direction_z", "wavelength")


def make_batch(support, direction, wavelength, ids=None) -> dict:
    """Photons from (n,3) supports, (n,3) directions and (n,) wavelengths.

    Like the merlict::Photon constructor (Photon.cpp:20-28) a wavelength
    must be positive; invalid photons raise ValueError.
    """
    support = np.asarray(support, dtype=np.float64).reshape(-1, 3)
    direction = np.asarray(direction, dtype=np.float64).reshape(-1, 3)
    wavelength = np.asarray(wavelength, dtype=np.float64).reshape(-1)
    n = wavelength.shape[0]
    if support.shape[0] != n or direction.shape[0] != n:
        raise ValueError("support, direction and wavelength differ in length")
    if np.any(~(wavelength > 0.0)):
        raise ValueError("Expected photon wavelength lambda > 0.0nm")
    b = {
        "support_x": support[:, 0].copy(), "support_y": support[:, 1].copy(),
        "support_z": support[:, 2].copy(),
        "direction_x": direction[:, 0].copy(), "direction_y": direction[:, 1].copy(),
        "direction_z": direction[:, 2].copy(),
        "wavelength": wavelength.copy(),
        "id": (np.arange(n, dtype=np.int32) if ids is None
               else np.asarray(ids, dtype=np.int32).reshape(-1)),
    }
    return b


def num_photons(batch: dict) -> int:
    return int(len(batch["wavelength"]))


def slice_batch(batch: dict, start: int, stop: int) -> dict:
    return {k: v[start:stop] for k, v in batch.items()}


def downward_disc_source(n: int, seed: int, disc_radius: float, height: float,
                         max_zenith_deg: float, lambda_min: float = 300e-9,
                         lambda_max: float = 700e-9, center=(0.0, 0.0)) -> dict:
    """Supports uniform on a horizontal disc at `height`, directions
    downwards, uniform in solid angle within `max_zenith_deg` of -z,
    wavelengths uniform in [lambda_min, lambda_max)."""
    rng = np.random.default_rng(seed)
    r = disc_radius * np.sqrt(rng.random(n))
    phi = 2.0 * np.pi * rng.random(n)
    cos_max = np.cos(np.deg2rad(max_zenith_deg))
    cos_t = 1.0 - rng.random(n) * (1.0 - cos_max)
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    az = 2.0 * np.pi * rng.random(n)
    lam = lambda_min + (lambda_max - lambda_min) * rng.random(n)
    sup = np.stack([center[0] + r * np.cos(phi), center[1] + r * np.sin(phi),
                    np.full(n, float(height))], axis=1)
    d = np.stack([sin_t * np.cos(az), sin_t * np.sin(az), -cos_t], axis=1)
    return make_batch(sup, d, lam)


def isotropic_shell_source(n: int, seed: int, radius: float, aim_radius: float,
                           lambda_min: float = 250e-9, lambda_max: float = 750e-9) -> dict:
    """Supports on a sphere of `radius` around the origin, each aimed at a
    random point within `aim_radius` of the origin (test scenes)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    sup = v * radius
    t = rng.normal(size=(n, 3))
    t /= np.linalg.norm(t, axis=1)[:, None]
    aim = t * (aim_radius * rng.random(n) ** (1.0 / 3.0))[:, None]
    d = aim - sup
    lam = lambda_min + (lambda_max - lambda_min) * rng.random(n)
    return make_batch(sup, d, lam)


# ---- merlict's own photon sources and photon tables -------------------------
#
# merlict::photon_source (merlict/Photons.cpp:83-127) and the raw photon
# table (Photons.cpp:24-81, tsvio.cpp:80-132).  A merlict::Photon stores its
# direction normalised (Ray.cpp:16-20); these sources store it the same way,
# and the engine's own normalisation at intake then finds a unit vector.

def _normalized(d: np.ndarray) -> np.ndarray:
    """Vec3::normalize (Vec3.cpp:20-26): each component / sqrt(x x + y y + z z)."""
    n = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    return d / n[:, None]


def point_like_towards_z_opening_angle_num_photons(opening_angle: float, num_photons: int,
                                                   prng) -> dict:
    """Photons from the origin into a cone of half angle `opening_angle`
    around +z, uniform in solid angle, 433 nm, id = index (Photons.cpp:85-106,
    SpherePointPicker.cpp:8-44).  Each photon draws the azimuth first, then
    the zenith distance, from `prng` (a prng.Mt19937)."""
    import math
    n = int(num_photons)
    u = prng.uniforms(2 * n).reshape(n, 2) if n else np.zeros((0, 2))
    z_min = (math.cos(0.0) + 1.0) / 2.0
    z_range = (math.cos(float(opening_angle)) + 1.0) / 2.0 - z_min
    d = np.empty((n, 3))
    two_pi = 2 * math.pi
    for i in range(n):
        az = two_pi * float(u[i, 0]) + 0.0
        zd = math.acos(2.0 * (z_range * float(u[i, 1]) + z_min) - 1.0)
        sin_zd = math.sin(zd)
        d[i] = (sin_zd * math.cos(az), sin_zd * math.sin(az), math.cos(zd))
    return make_batch(np.zeros((n, 3)), _normalized(d), np.full(n, 433e-9))


def parallel_towards_z_from_xy_disc(disc_radius: float, num_photons: int, prng) -> dict:
    """Photons along +z from points uniform on the xy disc of `disc_radius`,
    433 nm, id = index (Photons.cpp:108-125).  Points come from rejection
    sampling of pairs of draws (Generator.cpp:22-34)."""
    n = int(num_photons)
    r = float(disc_radius)
    r_sq = r * r
    xs, ys = [], []
    have = 0
    while have < n:
        pairs = max(64, int((n - have) * 1.3) + 16)
        saved = prng.getstate()
        u = prng.uniforms(2 * pairs).reshape(pairs, 2)
        x = r * (u[:, 0] * 2.0 - 1.0)
        y = r * (u[:, 1] * 2.0 - 1.0)
        ok = ~(x * x + y * y > r_sq)
        idx = np.flatnonzero(ok)
        if have + len(idx) > n:
            # consume only the pairs up to the last photon's, as merlict does
            idx = idx[:n - have]
            prng.setstate(saved)
            prng.uniforms(2 * (int(idx[-1]) + 1))
        xs.append(x[idx])
        ys.append(y[idx])
        have += len(idx)
    sx = np.concatenate(xs) if xs else np.zeros(0)
    sy = np.concatenate(ys) if ys else np.zeros(0)
    sup = np.stack([sx, sy, np.zeros(n)], axis=1)
    d = np.zeros((n, 3))
    d[:, 2] = 1.0
    return make_batch(sup, _normalized(d), np.full(n, 433e-9))


def transform_photons(batch: dict, T) -> dict:
    """Ray::transform (Ray.cpp:40-43) with the 3x4 transformation T of
    HomTra3::set_transformation: supports by HomTra3::position, directions
    by HomTra3::orientation (HomTra3.cpp:154-200), in merlict's order of
    operations."""
    sx, sy, sz = batch["support_x"], batch["support_y"], batch["support_z"]
    dx, dy, dz = batch["direction_x"], batch["direction_y"], batch["direction_z"]
    out = dict(batch)
    out["support_x"] = sx * T[0][0] + sy * T[0][1] + sz * T[0][2] + T[0][3]
    out["support_y"] = sx * T[1][0] + sy * T[1][1] + sz * T[1][2] + T[1][3]
    out["support_z"] = sx * T[2][0] + sy * T[2][1] + sz * T[2][2] + T[2][3]
    out["direction_x"] = dx * T[0][0] + dy * T[0][1] + dz * T[0][2]
    out["direction_y"] = dx * T[1][0] + dy * T[1][1] + dz * T[1][2]
    out["direction_z"] = dx * T[2][0] + dy * T[2][1] + dz * T[2][2]
    return out


def raw_matrix2photons(rows) -> dict:
    """Rows of [id, support x y z, direction x y z, wavelength] to photons
    (Photons.cpp:24-81).  A row that does not have exactly 8 columns, or a
    wavelength <= 0, raises ValueError.  The id column is a double in
    merlict; here it is kept as int32 after a check that it is integral."""
    m = [list(r) for r in rows]
    for r in m:
        if len(r) != 8:
            raise ValueError("PhotonBunch, raw row of doubles to photon. Expected row to "
                             f"have exactly 8 columns, but actual it has {len(r)} columns.")
    a = np.asarray(m, dtype=np.float64).reshape(-1, 8)
    ids = a[:, 0]
    if np.any(ids != np.floor(ids)) or np.any(np.abs(ids) > 2**31 - 1):
        raise ValueError("photon ids must be integers that fit in 32 bits")
    return make_batch(a[:, 1:4], _normalized(a[:, 4:7]) if len(a) else a[:, 4:7], a[:, 7],
                      ids.astype(np.int32))


def photons2raw_matrix(batch: dict) -> np.ndarray:
    """Photons to rows of [id, support, direction, wavelength] (Photons.cpp:33-59)."""
    return np.stack([np.asarray(batch["id"], dtype=np.float64)] +
                    [np.asarray(batch[k], dtype=np.float64) for k in PLANES], axis=1)


def _to_double(token: str) -> float:
    """txt::to_double (txt.cpp:108-125): the whole token must parse as a
    number (strtod's syntax: decimal, hexadecimal, inf, nan)."""
    t = token
    low = t.lower().lstrip("+-")
    try:
        if "_" in t or not t:
            raise ValueError
        if low.startswith("0x"):
            return float.fromhex(t)
        return float(t)
    except ValueError:
        raise ValueError(f"txt::to_double: Can not parse '{token}' to double.") from None


def gen_table_from_string(text: str) -> list:
    """tsvio::TableReader (tsvio.cpp:80-132): one row per line, tokens split
    at tabs and spaces, blank lines and lines starting with '#' skipped."""
    table = []
    for row_number, line in enumerate(text.split("\n"), start=1):
        row = line.strip()
        if not row or row[0] == "#":
            continue
        tokens = [t for t in row.replace("\t", " ").split(" ") if t]
        numeric = []
        for col, tok in enumerate(tokens, start=1):
            try:
                numeric.append(_to_double(tok))
            except ValueError as e:
                raise ValueError(f"TableReader: Can not convert item '{tok}' into a floating "
                                 f"point number in row {row_number} and column {col}. {e}") from None
        table.append(numeric)
    return table


def gen_table_from_file(path: str) -> list:
    """tsvio::gen_table_from_file (tsvio.cpp:13-36)."""
    try:
        with open(path, "r") as f:
            text = f.read()
    except OSError:
        raise RuntimeError(f"tsvio::gen_table_from_file Can not open file '{path}'.") from None
    return gen_table_from_string(text)


def load_photon_table(path: str) -> dict:
    """A photon file of merlict's propagation program: raw_matrix2photons of
    the table at `path` (merlict_tests/apps/propagate.cpp:63-64)."""
    return raw_matrix2photons(gen_table_from_file(path))


SPEED_OF_LIGHT = 299792458.0             # merlict/PhysicalConstants.h:7
PRODUCTION_DISTANCE_OFFSET = 1e3         # merlict_corsika/PhotonFactory.cpp:51-57


def cherenkov_event_sizes(num_events: int, seed: int, min_photons: int = 100,
                          max_photons: int = 10**6) -> np.ndarray:
    """Photons per event, log-uniform in [min_photons, max_photons]."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(float(min_photons)), np.log(float(max_photons))
    return np.rint(np.exp(lo + (hi - lo) * rng.random(num_events))).astype(np.int64)


def cherenkov_events(sizes, seed: int, device="cpu", dtype=None, core_radius: float = 150.0,
                     clip_radius: float = 40.0, max_axis_zenith_deg: float = 3.0,
                     cone_deg: float = 1.0, cone_spread_deg: float = 0.2,
                     time_sigma: float = 5e-9, lambda_min: float = 300e-9,
                     lambda_max: float = 700e-9, chunk: int = 1 << 25):
    """Air-shower-like photon events, concatenated, as torch planes on
    `device` (returns (batch, offsets); event e is photons
    [offsets[e], offsets[e + 1])).

    Per event: a shower axis uniform in solid angle within
    `max_axis_zenith_deg` of the zenith, a core uniform within `core_radius`
    of the telescope and a Cherenkov angle uniform in cone_deg +-
    cone_spread_deg.  Per photon: a ground point uniform within
    `clip_radius` of the telescope, a direction on the event's cone about
    its axis at the azimuth of the ground point seen from the core, an
    arrival time ~ N(0, time_sigma) and a wavelength from the 1/lambda^2
    Cherenkov spectrum.  The support is placed like merlict's CORSIKA
    photon factory places it (merlict_corsika/PhotonFactory.cpp:31-62): up
    the ray from the ground point by c*t plus a 1 km offset, so that the
    arrival time is part of the time of flight.
    """
    import torch
    dtype = dtype or torch.float64
    sizes = np.asarray(sizes, dtype=np.int64)
    offsets = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    total = int(offsets[-1])
    rng = np.random.default_rng(seed)
    e = len(sizes)
    cos_max = np.cos(np.deg2rad(max_axis_zenith_deg))
    cz = 1.0 - rng.random(e) * (1.0 - cos_max)
    sz = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
    pa = 2.0 * np.pi * rng.random(e)
    axis = np.stack([sz * np.cos(pa), sz * np.sin(pa), -cz], axis=1)
    rc = core_radius * np.sqrt(rng.random(e))
    pc = 2.0 * np.pi * rng.random(e)
    core = np.stack([rc * np.cos(pc), rc * np.sin(pc)], axis=1)
    cone = np.deg2rad(cone_deg + cone_spread_deg * (2.0 * rng.random(e) - 1.0))
    # orthonormal basis (e1, e2) perpendicular to each axis
    ref = np.where(np.abs(axis[:, 2:3]) < 0.9, [[0.0, 0.0, 1.0]], [[1.0, 0.0, 0.0]])
    e1 = np.cross(axis, ref)
    e1 /= np.linalg.norm(e1, axis=1)[:, None]
    e2 = np.cross(axis, e1)
    out = {k: torch.empty(total, dtype=dtype, device=device) for k in PLANES}
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    ev_of = torch.repeat_interleave(torch.arange(e, device=device),
                                    torch.as_tensor(sizes, device=device))
    t_axis = torch.as_tensor(axis, device=device)
    t_core = torch.as_tensor(core, device=device)
    t_cone = torch.as_tensor(cone, device=device)
    t_e1 = torch.as_tensor(e1, device=device)
    t_e2 = torch.as_tensor(e2, device=device)
    inv_lo, inv_hi = 1.0 / lambda_min, 1.0 / lambda_max
    f64 = torch.float64
    for a in range(0, total, chunk):
        b = min(total, a + chunk)
        m = b - a
        ev = ev_of[a:b]
        u = torch.rand((5, m), generator=gen, device=device, dtype=f64)
        r = clip_radius * torch.sqrt(u[0])
        phi = 2.0 * np.pi * u[1]
        gx, gy = r * torch.cos(phi), r * torch.sin(phi)
        psi = torch.atan2(gy - t_core[ev, 1], gx - t_core[ev, 0])
        ca, sa = torch.cos(t_cone[ev]), torch.sin(t_cone[ev])
        rad = (torch.cos(psi)[:, None] * t_e1[ev] + torch.sin(psi)[:, None] * t_e2[ev])
        d = ca[:, None] * t_axis[ev] + sa[:, None] * rad
        d = d / torch.linalg.norm(d, dim=1, keepdim=True)
        t = time_sigma * torch.randn(m, generator=gen, device=device, dtype=f64)
        back = t * SPEED_OF_LIGHT + PRODUCTION_DISTANCE_OFFSET
        lam = 1.0 / (inv_lo - u[2] * (inv_lo - inv_hi))
        planes = (gx - d[:, 0] * back, gy - d[:, 1] * back, -d[:, 2] * back,
                  d[:, 0], d[:, 1], d[:, 2], lam)
        for k, v in zip(PLANES, planes):
            out[k][a:b] = v.to(dtype)
        del u, r, phi, gx, gy, psi, ca, sa, rad, d, t, back, lam, planes
    return out, offsets


def downward_disc_source_device(n: int, seed: int, disc_radius: float, height: float,
                                max_zenith_deg: float, device="cuda", lambda_min: float = 300e-9,
                                lambda_max: float = 700e-9, dtype=None) -> dict:
    """downward_disc_source's law, drawn with torch on `device` (for batches
    too large to make on the host)."""
    import torch
    dtype = dtype or torch.float64
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    u = torch.rand((5, n), generator=g, device=device, dtype=torch.float64)
    r = disc_radius * torch.sqrt(u[0])
    phi = 2.0 * np.pi * u[1]
    cos_max = float(np.cos(np.deg2rad(max_zenith_deg)))
    cos_t = 1.0 - u[2] * (1.0 - cos_max)
    sin_t = torch.sqrt(torch.clamp(1.0 - cos_t * cos_t, min=0.0))
    az = 2.0 * np.pi * u[3]
    planes = (r * torch.cos(phi), r * torch.sin(phi), torch.full_like(r, float(height)),
              sin_t * torch.cos(az), sin_t * torch.sin(az), -cos_t,
              lambda_min + (lambda_max - lambda_min) * u[4])
    return {k: v.to(dtype).contiguous() for k, v in zip(PLANES, planes)}
