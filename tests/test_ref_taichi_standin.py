"""The serial Taichi stand-in that runs the reference for the golden fixtures
(tests/golden/ref_taichi): the Taichi semantics it claims, one by one."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

_spec = importlib.util.spec_from_file_location(
    "ref_taichi_standin", Path(__file__).resolve().parent / "golden" / "ref_taichi" / "taichi" / "__init__.py")
ti = importlib.util.module_from_spec(_spec)
sys.modules[_spec.name] = ti  # not as "taichi": nothing else sees the stand-in
_spec.loader.exec_module(ti)


@ti.func
def _add_to(ret: ti.template(), v):
    ret += v


@ti.func
def _add_item(ret: ti.template(), k, v):
    ret[k] += v


@ti.kernel
def _typing(out: ti.template()):
    d = 2 * (3 + 2)          # a Python int folded by Python, then an i32 local
    out[0] = d * 0.001       # i32 promoted: f32(10) * f32(0.001)
    out[1] = 0.01 * 0.04 ** 2  # Python values only: folded in float64, stored as f32
    h = 25.0
    out[2] = h ** 3          # f32 ** int: repeated squaring in f32
    s = 0.0
    _add_to(s, 0.1)          # a template argument is the caller's variable
    _add_to(s, 0.2)
    out[3] = s
    vec = ti.Vector([0.0, 0.0, 0.0])
    _add_item(vec, 1, 0.5)
    out[4] = vec[1]
    out[5] = 7 / 2           # Python: true division
    k = 7
    out[6] = k / 2           # i32 / Python int: true division in f32


@ti.kernel
def _atomics(out: ti.template()):
    idx = 0
    for i in range(5):
        old = ti.atomic_add(idx, 2)
        out[i] = old
    out[5] = idx


@ti.kernel
def _values(f: ti.template()):
    a = f[0]
    a[0] = 5.0               # a local copy: the field keeps its value
    f[1][0] = 7.0            # an element of a field element: written through
    f[2] += ti.Vector([1.0, 1.0])


def test_typing_and_folding():
    out = ti.field(float, shape=8)
    _typing(out)
    assert out.arr[0] == np.float32(10) * np.float32(0.001)
    assert out.arr[0] != np.float32(0.01)  # the f32 product differs from the folded constant
    assert out.arr[1] == np.float32(0.01 * 0.04 ** 2)
    assert out.arr[2] == np.float32(15625.0)
    assert out.arr[3] == np.float32(np.float32(0.1) + np.float32(0.2))
    assert out.arr[4] == np.float32(0.5)
    assert out.arr[5] == np.float32(3.5) and out.arr[6] == np.float32(3.5)


def test_atomic_add_returns_the_old_value():
    out = ti.field(int, shape=6)
    _atomics(out)
    assert out.arr.tolist() == [0, 2, 4, 6, 8, 10]


def test_element_reads_are_values_and_component_writes_reach_the_field():
    f = ti.Vector.field(2, dtype=float, shape=3)
    f.from_numpy(np.array([[1, 2], [3, 4], [5, 6]], dtype=np.float32))
    _values(f)
    assert f.arr.tolist() == [[1, 2], [7, 4], [6, 7]]


def test_python_scope_scalar_reads_are_python_numbers():
    dt = ti.field(float, shape=())
    dt[None] = 4e-4
    v = dt[None]
    assert type(v) is float and v == float(np.float32(4e-4))


def test_vector_reductions_left_to_right():
    a = ti.Vector([1e8, 1.0, -1e8])
    # (1e8 + 1) + (-1e8) in f32 is 0; a pairwise or reordered sum could give 1
    assert a.sum() == np.float32(0.0)
    assert a.dot(ti.Vector([1.0, 1.0, 1.0])) == np.float32(0.0)
    c = ti.Vector([1.0, 0.0, 0.0]).cross(ti.Vector([0.0, 1.0, 0.0]))
    assert c.a.tolist() == [0.0, 0.0, 1.0]


def test_prefix_sum_is_inclusive():
    f = ti.field(int, shape=5)
    f.from_numpy(np.array([1, 0, 2, 3, 0]))
    ti.algorithms.PrefixSumExecutor(5).run(f)
    assert f.arr.tolist() == [1, 1, 3, 6, 6]
