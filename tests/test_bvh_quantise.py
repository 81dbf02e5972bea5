"""The quantised BVH node (QNode) bounds the float node it stands for.

The level kernels test 96-byte nodes whose child bounds are 8-bit steps of
a power-of-two grid from a per-axis origin.  A child box that came out
smaller than the float box would drop candidates, so every decoded bound
must lie outside the float bound, exactly (checked here in rational
arithmetic), and no more than one step beyond the tightest grid bound.
The quantiser is the library's own C++ function, called through its
exported (mangled) symbol; it needs no GPU.
"""
import ctypes
from fractions import Fraction

import numpy as np
import pytest

from merlict_development_kit_b200 import _native

EMPTY = 0x7FFFFFFF
WIDTH = 8
SYMBOL = "_ZN5mlgpu17quantise_bvh_nodeERKNS_7BvhNodeEPNS_5QNodeE"


class BvhNode(ctypes.Structure):
    _fields_ = [("lo", (ctypes.c_float * WIDTH) * 3), ("hi", (ctypes.c_float * WIDTH) * 3),
                ("child", ctypes.c_int32 * WIDTH), ("pad", ctypes.c_int32 * WIDTH)]


class QNode(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_float * 3), ("exps", ctypes.c_uint32),
                ("child", ctypes.c_int32 * WIDTH),
                ("qlo", (ctypes.c_uint32 * 2) * 3), ("qhi", (ctypes.c_uint32 * 2) * 3)]


assert ctypes.sizeof(BvhNode) == 256 and ctypes.sizeof(QNode) == 96


def _quantiser():
    lib = _native.lib()
    try:
        f = getattr(lib, SYMBOL)
    except AttributeError:
        pytest.skip("quantiser symbol not exported by this build")
    f.argtypes = [ctypes.POINTER(BvhNode), ctypes.POINTER(QNode)]
    f.restype = None
    return f


def _node(rng, centre, size, empty):
    n = BvhNode()
    for k in range(WIDTH):
        n.child[k] = EMPTY if k in empty else k + 1
        for a in range(3):
            c = centre[a] + rng.uniform(-1, 1) * size
            h = abs(rng.normal()) * size * rng.choice([1e-4, 1e-2, 0.3])
            lo, hi = np.float32(c - h), np.float32(c + h)
            n.lo[a][k], n.hi[a][k] = (1.0, -1.0) if k in empty else (lo, hi)
    return n


def _check(n, q):
    for a in range(3):
        e = ((q.exps >> (8 * a)) & 0xFF) - 127
        step = Fraction(2) ** e
        origin = Fraction(float(q.origin[a]))
        live = [k for k in range(WIDTH) if n.child[k] != EMPTY]
        assert live
        assert float(q.origin[a]) == min(float(n.lo[a][k]) for k in live)
        top = max(Fraction(float(n.hi[a][k])) for k in live)
        # the smallest power-of-two step whose 255 steps reach the top
        assert 255 * step >= top - origin
        assert e == -126 or 255 * step / 2 < top - origin
        for k in range(WIDTH):
            ql = (q.qlo[a][k >> 2] >> (8 * (k & 3))) & 0xFF
            qh = (q.qhi[a][k >> 2] >> (8 * (k & 3))) & 0xFF
            assert q.child[k] == n.child[k]
            if n.child[k] == EMPTY:
                continue
            lo, hi = Fraction(float(n.lo[a][k])), Fraction(float(n.hi[a][k]))
            assert origin + ql * step <= lo, (a, k)
            assert origin + qh * step >= hi, (a, k)
            assert origin + (ql + 1) * step > lo or ql == 255
            assert origin + (qh - 1) * step < hi or qh == 0


def test_quantised_nodes_bound_their_float_boxes():
    f = _quantiser()
    rng = np.random.default_rng(5)
    for t in range(400):
        centre = rng.normal(size=3) * rng.choice([1e-3, 1.0, 30.0, 2e3])
        size = float(rng.choice([1e-5, 1e-3, 0.1, 5.0, 200.0]))
        empty = set(rng.choice(WIDTH, size=int(rng.integers(0, WIDTH)), replace=False).tolist())
        n = _node(rng, centre, size, empty)
        q = QNode()
        f(ctypes.byref(n), ctypes.byref(q))
        _check(n, q)


def test_degenerate_boxes_quantise_to_the_smallest_step():
    f = _quantiser()
    n = BvhNode()
    for k in range(WIDTH):
        n.child[k] = k + 1
        for a in range(3):
            n.lo[a][k] = n.hi[a][k] = 1.25   # a point: zero extent on every axis
    q = QNode()
    f(ctypes.byref(n), ctypes.byref(q))
    _check(n, q)
    assert q.exps == (1 | (1 << 8) | (1 << 16))
