"""The learned surrogate of the photon propagation (tensor-core MLP).

A BF16 MLP (5 inputs, sin/cos-encoded -> 4 x 256, SiLU -> 73) maps a
photon's entrance state --
support x, y on the entrance plane of the source, direction x, y and
wavelength -- to the probability that the photon reaches a sensor and to an
8-component Gaussian mixture over where it ends on the sensor plane (x, y)
and its direction there (x, y).  Sampling the mixture and looking the sample
up in the exact hexagonal sensor grid gives the photon's sensor without
tracing it.  Photons outside the training domain, or whose sampled component
is too wide to pin down a sensor, are traced exactly instead.

The mixture models the residual of a linear fit (targets = A x + b +
scale * t), so the network only learns what a linear optical map misses.

Training data come from the exact tracer (`training_data`); the network is
trained by the library's own tensor-core kernels (mlgpu_sg_train_step).
The C ABI is include/merlict_b200_surrogate.h; merlict has no counterpart.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import abi, engine
from ._native import check, lib, mlgpu_sg_sensor_grid

IN_LD = 8            # floats per input row
OUT_LD = 80          # floats per output row
COMPONENTS = 8
TILE = 128


def image_offsets(rows: int, k: int) -> np.ndarray:
    """Byte offsets of every element of a rows x k tile image
    (mlgpu_sg_image_offset)."""
    r = np.arange(rows, dtype=np.int64)[:, None]
    c = np.arange(k, dtype=np.int64)[None, :]
    return (((c >> 6) * (rows >> 3) + (r >> 3)) * 1024 + (r & 7) * 128 +
            ((((c & 63) >> 3) ^ (r & 7)) << 4) + ((c & 7) << 1))


def to_image(mat: torch.Tensor) -> torch.Tensor:
    """The tile image (uint8) of a rows x k matrix (rounded to BF16)."""
    rows, k = mat.shape
    assert rows % 8 == 0 and k % 64 == 0
    off = torch.as_tensor(image_offsets(rows, k) // 2, device=mat.device)
    out = torch.zeros(rows * k, dtype=torch.bfloat16, device=mat.device)
    out[off.reshape(-1)] = mat.to(torch.bfloat16).reshape(-1)
    return out.view(torch.uint8)


def from_image(img: torch.Tensor, rows: int, k: int) -> torch.Tensor:
    off = torch.as_tensor(image_offsets(rows, k) // 2, device=img.device)
    return img.view(torch.bfloat16)[off.reshape(-1)].reshape(rows, k)


def gemm(a_img, a_rows, b_img, b_rows, m, n, k_chunks, bias=None, stream=None) -> torch.Tensor:
    """C = A B^T on the tensor cores (mlgpu_sg_gemm_f32)."""
    c = torch.empty((m, n), dtype=torch.float32, device=a_img.device)
    check(lib().mlgpu_sg_gemm_f32(a_img.data_ptr(), a_rows, b_img.data_ptr(), b_rows, m, n,
                                  k_chunks, bias.data_ptr() if bias is not None else None,
                                  c.data_ptr(), engine._stream_handle(stream)))
    return c


def sync_errors(stream=None) -> None:
    check(lib().mlgpu_sg_sync_errors(engine._stream_handle(stream)))


# ---- parameters ---------------------------------------------------------------

ENCODED = 128        # encoded input width (mlgpu_sg: 5 inputs, sin/cos of 12 octaves)
LAYERS = ((ENCODED, 256), (256, 256), (256, 256), (256, 256), (256, 73))


def param_slices() -> list:
    """(W slice, shape, b slice) of each layer in the flat parameter vector."""
    out, o = [], 0
    for fin, fout in LAYERS:
        w = slice(o, o + fin * fout)
        o += fin * fout
        b = slice(o, o + fout)
        o += fout
        out.append((w, (fout, fin), b))
    assert o == int(lib().mlgpu_sg_param_count())
    return out


def init_params(seed: int, device="cuda") -> torch.Tensor:
    g = torch.Generator(device="cpu").manual_seed(seed)
    p = torch.zeros(int(lib().mlgpu_sg_param_count()), dtype=torch.float32)
    for i, (w, shape, b) in enumerate(param_slices()):
        fout, fin = shape
        bound = math.sqrt(6.0 / fin) if i < len(LAYERS) - 1 else 0.1 / math.sqrt(fin)
        p[w] = (torch.rand(fout * fin, generator=g) * 2.0 - 1.0) * bound
    return p.to(device)


# ---- the sensor grid ------------------------------------------------------------

class SensorGrid:
    """The hexagonal sensors of a flat scene that lie on one plane normal to
    z, bucketed in a uniform grid for the exact lookup of mlgpu_sg_sample."""

    def __init__(self, flat: abi.FlatScene, device="cuda"):
        leaves = np.flatnonzero((flat.leaf_sensor >= 0) &
                                (flat.leaf_primitive == abi.PRIM_HEX_PLANE))
        if leaves.size == 0:
            raise ValueError("the scene has no hexagonal sensors")
        T = flat.leaf_frame2world[leaves]
        if not (np.allclose(T[:, 8:11], [0.0, 0.0, 1.0]) and np.ptp(T[:, 11]) < 1e-9):
            raise ValueError("the hexagonal sensors do not share one plane normal to z")
        self.z = float(T[0, 11])
        center = T[:, [3, 7]].astype(np.float64)
        rot = np.stack([T[:, 0], T[:, 4]], axis=1)          # cos, sin of the z rotation
        inner = flat.leaf_params[leaves, 0]
        outer = inner * 2.0 / math.sqrt(3.0)
        self.cell = float(2.0 * outer.max())
        lo = center.min(axis=0) - outer.max()
        hi = center.max(axis=0) + outer.max()
        nx = int(np.ceil((hi[0] - lo[0]) / self.cell)) + 1
        ny = int(np.ceil((hi[1] - lo[1]) / self.cell)) + 1
        cells = [[] for _ in range(nx * ny)]
        for i in range(leaves.size):
            x0 = int(np.floor((center[i, 0] - outer[i] - lo[0]) / self.cell))
            x1 = int(np.floor((center[i, 0] + outer[i] - lo[0]) / self.cell))
            y0 = int(np.floor((center[i, 1] - outer[i] - lo[1]) / self.cell))
            y1 = int(np.floor((center[i, 1] + outer[i] - lo[1]) / self.cell))
            for cy in range(max(y0, 0), min(y1, ny - 1) + 1):
                for cx in range(max(x0, 0), min(x1, nx - 1) + 1):
                    cells[cy * nx + cx].append(i)
        start = np.zeros(nx * ny + 1, np.uint32)
        start[1:] = np.cumsum([len(c) for c in cells])
        items = np.fromiter((i for c in cells for i in c), dtype=np.uint32, count=int(start[-1]))
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device=device)
        self.t_center = t(center, np.float32)
        self.t_rot = t(rot, np.float32)
        self.t_inner = t(inner, np.float32)
        self.t_sensor = t(flat.leaf_sensor[leaves], np.int32)
        # uint32 on the device; every index is far below 2^31
        self.t_start = t(start, np.int32)
        self.t_items = t(items, np.int32)
        self.inner_min = float(inner.min())
        s = mlgpu_sg_sensor_grid()
        s.num_sensors = int(leaves.size)
        s.center, s.rotation = self.t_center.data_ptr(), self.t_rot.data_ptr()
        s.inner, s.sensor_id = self.t_inner.data_ptr(), self.t_sensor.data_ptr()
        s.x0, s.y0, s.cell = float(lo[0]), float(lo[1]), self.cell
        s.nx, s.ny = nx, ny
        s.cell_start, s.cell_items = self.t_start.data_ptr(), self.t_items.data_ptr()
        for k in range(2):
            s.hex_u[k] = flat.hex_unit_u[k]
            s.hex_v[k] = flat.hex_unit_v[k]
            s.hex_w[k] = flat.hex_unit_w[k]
        self.struct = s


# ---- data -----------------------------------------------------------------------

@dataclass
class Source:
    """The entrance plane and input ranges the surrogate is trained on: the
    downward disc source of the benchmark (photons.downward_disc_source)."""
    disc_radius: float = 5.55
    height: float = 21.4
    max_zenith_deg: float = 1.5
    lambda_min: float = 300e-9
    lambda_max: float = 700e-9

    def inputs(self, ph: dict) -> torch.Tensor:
        """[n][8] normalised inputs; photons not on the entrance plane get an
        out-of-domain input."""
        n = ph["wavelength"].shape[0]
        dev = ph["wavelength"].device
        x = torch.zeros((n, IN_LD), dtype=torch.float32, device=dev)
        s = math.sin(math.radians(self.max_zenith_deg))
        lc = 0.5 * (self.lambda_min + self.lambda_max)
        lh = 0.5 * (self.lambda_max - self.lambda_min)
        x[:, 0] = (ph["support_x"] / self.disc_radius).float()
        x[:, 1] = (ph["support_y"] / self.disc_radius).float()
        x[:, 2] = (ph["direction_x"] / s).float()
        x[:, 3] = (ph["direction_y"] / s).float()
        x[:, 4] = ((ph["wavelength"] - lc) / lh).float()
        off = (ph["support_z"] - self.height).abs() > 1e-6 * max(1.0, abs(self.height))
        x[off, 0] = 1e3
        return x

    def photons(self, n: int, seed: int, device="cuda") -> dict:
        from .photons import downward_disc_source_device
        return downward_disc_source_device(n, seed, self.disc_radius, self.height,
                                           self.max_zenith_deg, device=device,
                                           lambda_min=self.lambda_min, lambda_max=self.lambda_max)


def training_data_plane(scene: engine.Scene, source: Source, n: int, seed: int, plane_z: float,
                        chunk: int = 1 << 24) -> dict:
    """Photons of `source` traced exactly (FP64) through their first
    interaction: a photon "reaches" if it was reflected upwards below the
    plane z = plane_z; its targets are where it crosses that plane and its
    direction (x, y) there."""
    xs, ts, rs = [], [], []
    for a in range(0, n, chunk):
        m = min(chunk, n - a)
        ph = source.photons(m, seed * 1000003 + a)
        out = scene.propagate(ph, engine.PropagationConfig(1), engine.Philox(seed, photon_offset=a),
                              outputs=("sensor", "info", "final_position", "final_direction"))
        p, d = out["final_position"], out["final_direction"]
        kind = out["info"] & 0xFF
        ok = (kind == abi.REFLECTION_ON_SURFACE) & (d[:, 2] > 0.0) & (p[:, 2] < plane_z)
        t = torch.where(ok, (plane_z - p[:, 2]) / d[:, 2].clamp_min(1e-12), torch.zeros_like(p[:, 2]))
        xs.append(source.inputs(ph))
        ts.append(torch.stack([p[:, 0] + d[:, 0] * t, p[:, 1] + d[:, 1] * t, d[:, 0], d[:, 1]],
                              dim=1).float())
        rs.append(ok.to(torch.uint8))
        del ph, out
    return {"inputs": torch.cat(xs), "targets": torch.cat(ts), "reached": torch.cat(rs)}


def training_data(scene: engine.Scene, source: Source, n: int, seed: int,
                  max_interactions: int = 10, chunk: int = 1 << 24) -> dict:
    """Photons of `source` traced exactly (FP64): inputs, the final position
    and direction (x, y) of photons that reached a sensor, and the flag."""
    xs, ts, rs = [], [], []
    for a in range(0, n, chunk):
        m = min(chunk, n - a)
        ph = source.photons(m, seed * 1000003 + a)
        out = scene.propagate(ph, engine.PropagationConfig(max_interactions),
                              engine.Philox(seed, photon_offset=a),
                              outputs=("sensor", "final_position", "final_direction"))
        xs.append(source.inputs(ph))
        t = torch.stack([out["final_position"][:, 0], out["final_position"][:, 1],
                         out["final_direction"][:, 0], out["final_direction"][:, 1]], dim=1)
        ts.append(t.float())
        rs.append((out["sensor"] >= 0).to(torch.uint8))
        del ph, out
    return {"inputs": torch.cat(xs), "targets": torch.cat(ts), "reached": torch.cat(rs)}


# ---- the model ------------------------------------------------------------------

class Surrogate:
    """Parameters, Adam state and normalisation of one trained network."""

    def __init__(self, flat: abi.FlatScene, source: Source | None = None, seed: int = 0,
                 device="cuda", plane_z: float | None = None):
        """With plane_z the network models the photon where it crosses the
        plane z = plane_z on its way to the sensors (hit point and
        direction), and the exact tracer carries each sampled photon on from
        there ("plane" mode, for sensors with optics of their own such as a
        light-field sensor); without, it models the final hit on a plane of
        hexagonal sensors looked up exactly ("lookup" mode)."""
        self.device = torch.device(device)
        self.source = source or Source()
        self.plane_z = plane_z
        self.grid = SensorGrid(flat, device=device) if plane_z is None else None
        self.params = init_params(seed, device)
        self.images = torch.zeros(int(lib().mlgpu_sg_image_bytes()), dtype=torch.uint8,
                                  device=device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.linear = torch.zeros((4, 6), dtype=torch.float32, device=device)
        self.scale = torch.ones(4, dtype=torch.float32, device=device)
        self.reach_rate = 0.5
        self._ws = None
        self._ws_key = None
        self.pack()

    def pack(self) -> None:
        check(lib().mlgpu_sg_pack_weights(self.params.data_ptr(), self.images.data_ptr(), None))

    def _workspace(self, batch: int, training: bool) -> torch.Tensor:
        key = (batch, training)
        if self._ws_key != key:
            nbytes = int(lib().mlgpu_sg_workspace_bytes(batch, int(training)))
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws_key = key
        return self._ws

    # the linear part of the map
    def fit_baseline(self, data: dict, rows: int = 1 << 22) -> None:
        """Least-squares linear map of the targets of photons that reached a
        sensor (on at most `rows` of them) and the spread of its residual."""
        r = data["reached"][:4 * rows].bool()
        x = data["inputs"][:4 * rows][r][:rows, :5].double()
        t = data["targets"][:4 * rows][r][:rows].double()
        X = torch.cat([x, torch.ones((x.shape[0], 1), dtype=x.dtype, device=x.device)], dim=1)
        sol = torch.linalg.lstsq(X.cpu(), t.cpu()).solution          # [6][4]
        self.linear = sol.T.contiguous().float().to(self.device)
        res = t - X @ sol.to(t.device)
        self.scale = res.std(dim=0).clamp_min(1e-9).float().to(self.device)
        self.reach_rate = float(r.float().mean())

    def normalised_targets(self, data: dict) -> torch.Tensor:
        x = data["inputs"][:, :5]
        base = x @ self.linear[:, :5].T + self.linear[:, 5]
        return ((data["targets"] - base) / self.scale).contiguous()

    def train_step(self, x: torch.Tensor, t: torch.Tensor, r: torch.Tensor, lr: float,
                   loss: torch.Tensor | None = None, grads: torch.Tensor | None = None) -> None:
        batch = x.shape[0]
        self.step += 1
        check(lib().mlgpu_sg_train_step(
            self.params.data_ptr(), self.images.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
            x.data_ptr(), t.data_ptr(), r.data_ptr(), batch, self.step, float(lr),
            loss.data_ptr() if loss is not None else None,
            grads.data_ptr() if grads is not None else None,
            self._workspace(batch, True).data_ptr(), None))

    def train(self, data: dict, epochs: int = 4, batch: int = 65536, lr: float = 2e-3,
              lr_min: float = 2e-5, seed: int = 0, log=None) -> list:
        """Adam over shuffled batches with a cosine learning-rate decay;
        returns the mean loss of each epoch."""
        if self.step == 0:
            self.fit_baseline(data)
        t_all = self.normalised_targets(data)
        x_all, r_all = data["inputs"], data["reached"]
        n = x_all.shape[0] // batch * batch
        steps = epochs * (n // batch)
        g = torch.Generator(device=self.device).manual_seed(seed)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        history, k = [], 0
        for ep in range(epochs):
            perm = torch.randperm(x_all.shape[0], generator=g, device=self.device)[:n]
            acc = torch.zeros((), dtype=torch.float64, device=self.device)
            for b in range(n // batch):
                idx = perm[b * batch:(b + 1) * batch]
                lr_k = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * k / max(1, steps)))
                self.train_step(x_all[idx].contiguous(), t_all[idx].contiguous(),
                                r_all[idx].contiguous(), lr_k, loss=loss)
                acc += loss[0].double()
                k += 1
            sync_errors()
            history.append(float(acc) / max(1, n // batch))
            if log:
                log(f"epoch {ep}: loss {history[-1]:.4f}")
        return history

    def forward(self, x: torch.Tensor, layered: bool = False) -> torch.Tensor:
        """The network's outputs [n][80] for inputs [n][8]: one fused launch
        (mlgpu_sg_forward), or with `layered` one launch per layer with the
        activations in device memory (mlgpu_sg_forward_layered, the training
        step's form; the same bits)."""
        n = x.shape[0]
        pad = (-n) % TILE
        if pad:
            x = torch.cat([x, torch.zeros((pad, IN_LD), dtype=x.dtype, device=x.device)])
        y = torch.empty((n + pad, OUT_LD), dtype=torch.float32, device=self.device)
        if layered:
            check(lib().mlgpu_sg_forward_layered(self.params.data_ptr(), self.images.data_ptr(),
                                                 x.data_ptr(), n + pad, y.data_ptr(),
                                                 self._workspace(n + pad, False).data_ptr(), None))
        else:
            check(lib().mlgpu_sg_forward(self.params.data_ptr(), self.images.data_ptr(),
                                         x.data_ptr(), n + pad, y.data_ptr(), None, None))
        return y[:n]

    def sample(self, y: torch.Tensor, x: torch.Tensor, seed: int, photon_offset: int = 0,
               sigma_limit: float | None = None, in_limit: float = 1.0001) -> dict:
        n = x.shape[0]
        if sigma_limit is None:
            sigma_limit = self.grid.inner_min if self.grid is not None else 2e-3
        sl = sigma_limit
        out = {"sensor": torch.empty(n, dtype=torch.int32, device=self.device),
               "x": torch.empty(n, dtype=torch.float32, device=self.device),
               "y": torch.empty(n, dtype=torch.float32, device=self.device),
               "cx": torch.empty(n, dtype=torch.float32, device=self.device),
               "cy": torch.empty(n, dtype=torch.float32, device=self.device),
               "fallback": torch.empty(n, dtype=torch.uint8, device=self.device)}
        check(lib().mlgpu_sg_sample(
            y.contiguous().data_ptr(), x.contiguous().data_ptr(), n, self.linear.data_ptr(),
            self.scale.data_ptr(), float(in_limit), float(sl), seed & 0xFFFFFFFFFFFFFFFF,
            photon_offset, C.byref(self.grid.struct) if self.grid is not None else None,
            out["sensor"].data_ptr(),
            out["x"].data_ptr(), out["y"].data_ptr(), out["cx"].data_ptr(), out["cy"].data_ptr(),
            out["fallback"].data_ptr(), None))
        return out

    def null_outputs(self, n: int) -> torch.Tensor:
        """The outputs of 'no network': the linear map with one Gaussian of
        the residual's spread and the mean reach rate (the ablation)."""
        y = torch.zeros((n, OUT_LD), dtype=torch.float32, device=self.device)
        p = min(max(self.reach_rate, 1e-6), 1 - 1e-6)
        y[:, 0] = math.log(p / (1 - p))
        for k in range(1, COMPONENTS):
            y[:, 1 + 9 * k] = -30.0
        return y

    def propagate(self, photons: dict, seed: int, scene: engine.Scene | None = None,
                  max_interactions: int = 10, chunk: int = 1 << 23, use_network: bool = True,
                  sigma_limit: float | None = None, tuning: dict | None = None) -> dict:
        """Sensor of every photon: sampled from the network (in plane mode
        carried on from the plane by `scene`'s exact tracer, in one call for
        the whole batch), with the photons it flags traced exactly by
        `scene` (if given).  `tuning` goes to those tracer calls."""
        n = int(photons["wavelength"].shape[0])
        sensor = torch.empty(n, dtype=torch.int32, device=self.device)
        fallback = torch.empty(n, dtype=torch.uint8, device=self.device)
        plane = self.plane_z is not None and scene is not None
        if plane:
            pxy = torch.empty((n, 4), dtype=torch.float32, device=self.device)
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            part = {k: v[a:b] for k, v in photons.items()}
            x = self.source.inputs(part)
            y = self.forward(x) if use_network else self.null_outputs(b - a)
            s = self.sample(y, x, seed, a, sigma_limit=sigma_limit)
            sensor[a:b] = s["sensor"]
            fallback[a:b] = s["fallback"]
            if plane:
                pxy[a:b] = torch.stack([s["x"], s["y"], s["cx"], s["cy"]], dim=1)
            del x, y, s
        if plane:
            # every sampled photon, carried on from the plane by the exact tracer
            idx = torch.nonzero(sensor == -2, as_tuple=False).flatten()
            if idx.numel():
                q = pxy[idx].double()
                cz = torch.sqrt(torch.clamp(1.0 - q[:, 2] * q[:, 2] - q[:, 3] * q[:, 3], min=0.0))
                sub = {"support_x": q[:, 0].contiguous(), "support_y": q[:, 1].contiguous(),
                       "support_z": torch.full_like(cz, self.plane_z),
                       "direction_x": q[:, 2].contiguous(), "direction_y": q[:, 3].contiguous(),
                       "direction_z": cz,
                       "wavelength": photons["wavelength"][idx].double().contiguous()}
                del q
                r = scene.propagate(sub, engine.PropagationConfig(max(1, max_interactions - 1)),
                                    engine.Philox(seed ^ 0x2545F491), outputs=("sensor",),
                                    tuning=tuning)
                sensor[idx] = r["sensor"]
                del sub, r
            sensor[sensor == -2] = -1
            del pxy
        if scene is not None:
            idx = torch.nonzero(fallback, as_tuple=False).flatten()
            if idx.numel():
                sub = {k: v[idx].contiguous() for k, v in photons.items()}
                r = scene.propagate(sub, engine.PropagationConfig(max_interactions),
                                    engine.Philox(seed ^ 0x5DEECE66D), outputs=("sensor",),
                                    tuning=tuning)
                sensor[idx] = r["sensor"]
        sync_errors()
        return {"sensor": sensor, "fallback": fallback}


def _forward_probe(n: int, repeats: int = 3) -> None:
    """Times the forward pass of an untrained network on the light-field
    telescope on n random inputs (the tensor-core layers' throughput), fused
    and layer by layer, and checks that both give the same bits."""
    from . import factories
    model = Surrogate(factories.light_field_telescope().flatten(), seed=1)
    x = torch.rand((n, IN_LD), device=model.device) * 2.0 - 1.0
    flops = 2.0 * sum(fin * (80 if fout == 73 else fout) for fin, fout in LAYERS) * n
    out = {}
    for layered in (False, True):
        out[layered] = model.forward(x, layered=layered).clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            model.forward(x, layered=layered)
        e1.record()
        torch.cuda.synchronize()
        sync_errors()
        ms = e0.elapsed_time(e1) / repeats
        print(f"{'layered' if layered else 'fused'} forward of {n} photons: {ms:.3f} ms, "
              f"{flops / ms / 1e9:.1f} TFLOP/s on the tensor-core layers, "
              f"{n / ms / 1e3:.1f} M photons/s")
    same = torch.equal(out[False][:, :73], out[True][:, :73])
    print(f"fused == layered bit for bit: {same}")
    if not same:
        raise SystemExit(1)


if __name__ == "__main__":
    import sys
    if len(sys.argv) >= 3 and sys.argv[1] == "forward":
        _forward_probe(int(sys.argv[2]))
    else:
        print("usage: python -m merlict_development_kit_b200.surrogate forward N")
