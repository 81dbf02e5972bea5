"""ctypes mirror of include/merlict_b200.h.

The structures here are byte-for-byte the C structs of the engine's C ABI;
`FlatScene` is the host-side image of an `mlgpu_flat_scene` held in numpy
arrays (the layout merlict's frame tree is flattened into).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

ABI_VERSION = 8

# status codes
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_RUNTIME = 3
ERR_CUDA = 4
ERR_NO_DEVICE = 5

# interactions, numbered as merlict/RayForPropagation.h:14-28
PRODUCTION = 0
ABSORPTION_IN_VOID = 1
ABSORPTION_IN_MEDIUM = 2
ABSORPTION_ON_SURFACE = 3
FRESNEL_REFLECTION_ON_SURFACE = 4
REFLECTION_ON_SURFACE = 5
REFRACTION_TO_OUTSIDE = 6
REFRACTION_TO_INSIDE = 7

INTERACTION_NAMES = {
    PRODUCTION: "production",
    ABSORPTION_IN_VOID: "absorption_in_void",
    ABSORPTION_IN_MEDIUM: "absorption_in_medium",
    ABSORPTION_ON_SURFACE: "absorption_on_surface",
    FRESNEL_REFLECTION_ON_SURFACE: "fresnel_reflection_on_surface",
    REFLECTION_ON_SURFACE: "reflection_on_surface",
    REFRACTION_TO_OUTSIDE: "refraction_to_outside",
    REFRACTION_TO_INSIDE: "refraction_to_inside",
}

# leaf primitives
PRIM_NONE = 0
PRIM_SPHERE_CAP_HEX = 1
PRIM_SPHERE_CAP_CYL = 2
PRIM_SPHERE_CAP_RECT = 3
PRIM_ELLIPTIC_CAP_HEX = 4
PRIM_DISC = 5
PRIM_HEX_PLANE = 6
PRIM_PLANE = 7
PRIM_ANNULUS = 8
PRIM_PLANE_DUAL_SPHERE = 9
PRIM_TRIANGLE = 10
PRIM_CYLINDER = 11
PRIM_SPHERE = 12
PRIM_COUNT = 13
LEAF_PARAMS = 8

SURF_OUTER_REFLECTION = 0
SURF_INNER_REFLECTION = 1
SURF_OUTER_REFRACTION = 2
SURF_INNER_REFRACTION = 3
SURF_OUTER_ABSORPTION = 4
SURF_INNER_ABSORPTION = 5
SURF_ALLOWED_NODE = 6
SURF_FLAGS = 7
SURF_COLUMNS = 8

FLAG_TRANSPARENT = 1
FLAG_INNER_REFRACTION_DEFAULT = 2
FLAG_OUTER_REFRACTION_DEFAULT = 4

LEAF_VOID = -1
LEAF_PHOTON_SOURCE = -2

F64 = 0
F32 = 1

RNG_PHILOX = 0
RNG_REPLAY = 1

TRACER_FP64 = 0
TRACER_FP32 = 1
TRACER_FP32_PURE = 2
TRACER_FP64_PLAIN = 3
TRACER_FP64_QUEUE = 4

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class mlgpu_flat_scene(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_int32),
        ("node_sphere", _dp),
        ("node_skip", _ip),
        ("node_leaf", _ip),
        ("num_leaves", C.c_int32),
        ("leaf_node", _ip),
        ("leaf_frame2world", _dp),
        ("leaf_primitive", _ip),
        ("leaf_params", _dp),
        ("leaf_surface", _ip),
        ("leaf_sensor", _ip),
        ("num_functions", C.c_int32),
        ("function_offset", _ip),
        ("function_points", _dp),
        ("default_refraction", C.c_int32),
        ("hex_unit_u", C.c_double * 3),
        ("hex_unit_v", C.c_double * 3),
        ("hex_unit_w", C.c_double * 3),
        ("num_sensors", C.c_int32),
    ]


class mlgpu_photons(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32),
        ("support_x", C.c_void_p),
        ("support_y", C.c_void_p),
        ("support_z", C.c_void_p),
        ("direction_x", C.c_void_p),
        ("direction_y", C.c_void_p),
        ("direction_z", C.c_void_p),
        ("wavelength", C.c_void_p),
        ("simulation_truth_id", C.c_void_p),
    ]


class mlgpu_history_entry(C.Structure):
    _fields_ = [
        ("position", C.c_double * 3),
        ("normal", C.c_double * 3),
        ("distance", C.c_double),
        ("leaf", C.c_int32),
        ("interaction", C.c_uint8),
        ("from_outside_to_inside", C.c_uint8),
        ("pad", C.c_uint8 * 2),
    ]


HISTORY_DTYPE = np.dtype([
    ("position", "<f8", (3,)),
    ("normal", "<f8", (3,)),
    ("distance", "<f8"),
    ("leaf", "<i4"),
    ("interaction", "u1"),
    ("from_outside_to_inside", "u1"),
    ("pad", "u1", (2,)),
])
assert HISTORY_DTYPE.itemsize == C.sizeof(mlgpu_history_entry) == 64


class mlgpu_results(C.Structure):
    _fields_ = [
        ("dtype", C.c_int32),
        ("sensor", C.c_void_p),
        ("x", C.c_void_p),
        ("y", C.c_void_p),
        ("time", C.c_void_p),
        ("theta_x", C.c_void_p),
        ("theta_y", C.c_void_p),
        ("final_leaf", C.c_void_p),
        ("info", C.c_void_p),
        ("final_position", C.c_void_p),
        ("final_direction", C.c_void_p),
        ("history", C.c_void_p),
    ]


class mlgpu_rng(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("stride", C.c_uint32),
        ("seed", C.c_uint64),
        ("photon_offset", C.c_uint64),
        ("uniforms", C.c_void_p),
    ]


class mlgpu_photon_buffers(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in (
        "support_x", "support_y", "support_z", "direction_x", "direction_y", "direction_z",
        "wavelength", "simulation_truth_id")] + [("capacity", C.c_uint64)]


class mlgpu_signal_chain_config(C.Structure):
    _fields_ = [
        ("quantum_efficiency", C.c_void_p),
        ("num_quantum_efficiency", C.c_uint32),
        ("num_nsb_wavelength_cdf", C.c_uint32),
        ("nsb_wavelength_cdf", C.c_void_p),
        ("nsb_total_integral", C.c_double),
        ("nsb_rate", C.c_double),
        ("dark_rate", C.c_double),
        ("probability_for_second_puls", C.c_double),
        ("nsb_exposure_time", C.c_double),
        ("time_slice_duration", C.c_double),
        ("arrival_time_std", C.c_double),
        ("num_lixel", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class mlgpu_photon_stream(C.Structure):
    _fields_ = [
        ("channel_offset", C.c_void_p),
        ("arrival_time_slice", C.c_void_p),
        ("simulation_truth_id", C.c_void_p),
        ("nsb_count", C.c_void_p),
        ("capacity", C.c_uint64),
        ("num_pulses", C.c_uint64),
        ("nsb_exposure_start_time", C.c_double),
    ]


TRAVERSAL_BVH = 0
TRAVERSAL_FRAME_TREE = 1

ORDER_DEFAULT = 0
ORDER_INPUT = 1
ORDER_COHERENT = 2

WALK_DEFAULT = 0
WALK_LEVELS = 1
WALK_STACK = 2



class mlgpu_settings(C.Structure):
    _fields_ = [
        ("max_num_interactions_per_photon", C.c_uint32),
        ("start_node", C.c_int32),
        ("tracer", C.c_int32),
        ("block_size", C.c_int32),
        ("traversal", C.c_int32),
        ("pool_size", C.c_uint32),
        ("check_period", C.c_int32),
        ("use_graph", C.c_int32),
        ("grid_blocks", C.c_int32),
        ("staged_levels", C.c_int32),
        ("photon_order", C.c_int32),
        ("walk", C.c_int32),
        ("queue_capacity", C.c_uint32),
    ]

    TUNING = ("pool_size", "check_period", "use_graph", "grid_blocks", "staged_levels",
              "photon_order", "walk", "queue_capacity")

    def tuning(self) -> dict:
        return {k: int(getattr(self, k)) for k in self.TUNING}


class mlgpu_wavefront_stats(C.Structure):
    _fields_ = [("calls", C.c_uint64), ("iterations", C.c_uint64), ("overflow_rays", C.c_uint64)]


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class FlatScene:
    """Host image of an mlgpu_flat_scene (see include/merlict_b200.h)."""
    node_sphere: np.ndarray          # float64 [num_nodes, 4]
    node_skip: np.ndarray            # int32 [num_nodes]
    node_leaf: np.ndarray            # int32 [num_nodes]
    leaf_node: np.ndarray            # int32 [num_leaves]
    leaf_frame2world: np.ndarray     # float64 [num_leaves, 12]
    leaf_primitive: np.ndarray       # int32 [num_leaves]
    leaf_params: np.ndarray          # float64 [num_leaves, 8]
    leaf_surface: np.ndarray         # int32 [num_leaves, 8]
    leaf_sensor: np.ndarray          # int32 [num_leaves]
    function_offset: np.ndarray      # int32 [num_functions + 1]
    function_points: np.ndarray      # float64 [points, 3]
    default_refraction: int
    hex_unit_u: np.ndarray           # float64 [3]
    hex_unit_v: np.ndarray
    hex_unit_w: np.ndarray
    num_sensors: int
    sensor_ids: np.ndarray | None = None   # user ids of the sensors, by index
    leaf_names: list | None = field(default=None, repr=False)

    ARRAYS = ("node_sphere", "node_skip", "node_leaf", "leaf_node",
              "leaf_frame2world", "leaf_primitive", "leaf_params",
              "leaf_surface", "leaf_sensor", "function_offset",
              "function_points", "hex_unit_u", "hex_unit_v", "hex_unit_w")

    def __post_init__(self):
        f64 = ("node_sphere", "leaf_frame2world", "leaf_params",
               "function_points", "hex_unit_u", "hex_unit_v", "hex_unit_w")
        for name in self.ARRAYS:
            dt = np.float64 if name in f64 else np.int32
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=dt))
        self.node_sphere = self.node_sphere.reshape(-1, 4)
        self.leaf_frame2world = self.leaf_frame2world.reshape(-1, 12)
        self.leaf_params = self.leaf_params.reshape(-1, LEAF_PARAMS)
        self.leaf_surface = self.leaf_surface.reshape(-1, SURF_COLUMNS)
        self.function_points = self.function_points.reshape(-1, 3)
        self.default_refraction = int(self.default_refraction)
        self.num_sensors = int(self.num_sensors)

    @property
    def num_nodes(self) -> int:
        return int(self.node_skip.shape[0])

    @property
    def num_leaves(self) -> int:
        return int(self.leaf_node.shape[0])

    @property
    def num_functions(self) -> int:
        return int(self.function_offset.shape[0]) - 1

    def as_struct(self) -> mlgpu_flat_scene:
        s = mlgpu_flat_scene()
        s.num_nodes = self.num_nodes
        s.node_sphere = _ptr(self.node_sphere, C.c_double)
        s.node_skip = _ptr(self.node_skip, C.c_int32)
        s.node_leaf = _ptr(self.node_leaf, C.c_int32)
        s.num_leaves = self.num_leaves
        s.leaf_node = _ptr(self.leaf_node, C.c_int32)
        s.leaf_frame2world = _ptr(self.leaf_frame2world, C.c_double)
        s.leaf_primitive = _ptr(self.leaf_primitive, C.c_int32)
        s.leaf_params = _ptr(self.leaf_params, C.c_double)
        s.leaf_surface = _ptr(self.leaf_surface, C.c_int32)
        s.leaf_sensor = _ptr(self.leaf_sensor, C.c_int32)
        s.num_functions = self.num_functions
        s.function_offset = _ptr(self.function_offset, C.c_int32)
        s.function_points = _ptr(self.function_points, C.c_double)
        s.default_refraction = self.default_refraction
        for k in range(3):
            s.hex_unit_u[k] = float(self.hex_unit_u[k])
            s.hex_unit_v[k] = float(self.hex_unit_v[k])
            s.hex_unit_w[k] = float(self.hex_unit_w[k])
        s.num_sensors = self.num_sensors
        return s

    @classmethod
    def from_struct(cls, s: mlgpu_flat_scene) -> "FlatScene":
        """Copies the arrays a C producer handed out (e.g. the shim)."""
        def arr(ptr, n, dtype):
            if n == 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
        nn, nl, nf = s.num_nodes, s.num_leaves, s.num_functions
        off = arr(s.function_offset, nf + 1, np.int32)
        return cls(
            node_sphere=arr(s.node_sphere, 4 * nn, np.float64),
            node_skip=arr(s.node_skip, nn, np.int32),
            node_leaf=arr(s.node_leaf, nn, np.int32),
            leaf_node=arr(s.leaf_node, nl, np.int32),
            leaf_frame2world=arr(s.leaf_frame2world, 12 * nl, np.float64),
            leaf_primitive=arr(s.leaf_primitive, nl, np.int32),
            leaf_params=arr(s.leaf_params, LEAF_PARAMS * nl, np.float64),
            leaf_surface=arr(s.leaf_surface, SURF_COLUMNS * nl, np.int32),
            leaf_sensor=arr(s.leaf_sensor, nl, np.int32),
            function_offset=off,
            function_points=arr(s.function_points, 3 * int(off[-1]), np.float64),
            default_refraction=s.default_refraction,
            hex_unit_u=np.array(list(s.hex_unit_u)),
            hex_unit_v=np.array(list(s.hex_unit_v)),
            hex_unit_w=np.array(list(s.hex_unit_w)),
            num_sensors=s.num_sensors,
        )

    def to_npz_dict(self, prefix: str = "scene_") -> dict:
        d = {prefix + k: getattr(self, k) for k in self.ARRAYS}
        d[prefix + "default_refraction"] = np.int32(self.default_refraction)
        d[prefix + "num_sensors"] = np.int32(self.num_sensors)
        return d

    @classmethod
    def from_npz(cls, z, prefix: str = "scene_") -> "FlatScene":
        kw = {k: z[prefix + k] for k in cls.ARRAYS}
        kw["default_refraction"] = int(z[prefix + "default_refraction"])
        kw["num_sensors"] = int(z[prefix + "num_sensors"])
        return cls(**kw)

    def validate(self) -> None:
        """Host-side bounds checks of every index the kernels follow."""
        nn, nl, nf = self.num_nodes, self.num_leaves, self.num_functions
        if nn < 1:
            raise ValueError("scene has no nodes")
        idx = np.arange(nn)
        if np.any(self.node_skip <= idx) or np.any(self.node_skip > nn):
            raise ValueError("node_skip out of range")
        if self.node_skip[0] != nn:
            raise ValueError("node 0 must be the root of the whole tree")
        leaf = self.node_leaf
        if np.any((leaf < -1) | (leaf >= nl)):
            raise ValueError("node_leaf out of range")
        is_leaf = leaf >= 0
        if np.any(self.node_skip[is_leaf] != idx[is_leaf] + 1):
            raise ValueError("a leaf node must have an empty subtree")
        if np.any(self.node_skip[~is_leaf] == idx[~is_leaf] + 1):
            raise ValueError("a frame with children has an empty subtree")
        if nl and np.any(self.leaf_node[leaf[is_leaf]] != idx[is_leaf]):
            raise ValueError("leaf_node and node_leaf disagree")
        if np.any((self.leaf_primitive < 0) | (self.leaf_primitive >= PRIM_COUNT)):
            raise ValueError("unknown primitive")
        f = self.leaf_surface[:, :6]
        if np.any((f < 0) | (f >= nf)):
            raise ValueError("property table id out of range")
        allowed = self.leaf_surface[:, SURF_ALLOWED_NODE]
        if np.any((allowed < -1) | (allowed >= nn)):
            raise ValueError("allowed node out of range")
        if np.any((self.leaf_sensor < -1) | (self.leaf_sensor >= self.num_sensors)):
            raise ValueError("sensor index out of range")
        sensed = self.leaf_sensor[self.leaf_sensor >= 0]
        if len(np.unique(sensed)) != len(sensed):
            # one sensor per frame and no two sensors on one frame
            # (Sensors::assert_no_two_sensors_have_same_frame)
            raise ValueError("a sensor index is on two leaves")
        off = self.function_offset
        if off[0] != 0 or np.any(np.diff(off) < 1) or off[-1] != self.function_points.shape[0]:
            raise ValueError("function offsets malformed")
        for k in range(nf):
            x = self.function_points[off[k]:off[k + 1], 0]
            if np.any(np.diff(x) <= 0):
                raise ValueError(f"function {k} arguments not strictly increasing")
        if not (0 <= self.default_refraction < nf):
            raise ValueError("default refraction id out of range")
