"""Serial stand-in for the part of Taichi that DIMCV-SPH's hot path uses.

TEST INFRASTRUCTURE ONLY.  Taichi cannot be installed here, so this module
lets the reference's own, unmodified ``particle_system.py``, ``sph_base.py``,
``dimcv_sph.py`` and ``karman_vortex.py`` run on the CPU, one particle after
another, to produce golden fixtures (``tests/golden/make_reference_fixtures.py``).
Nothing in the product imports it.

What it reproduces of Taichi's semantics (Taichi 1.x, default_fp = f32):

* ``@ti.kernel`` / ``@ti.func`` bodies are rewritten with ``ast`` before they
  run:
  - every binary operator and comparison follows Taichi's typing: an
    expression made only of Python values is folded by Python (Taichi's
    frontend does the same at compile time); otherwise floats are f32 and
    integers i32, with an integer operand promoted to f32 when the other is
    a float, ``/`` always true division in f32, and ``x ** n`` with an
    integer ``n`` by repeated squaring in f32;
  - ``name = value`` makes a typed local (a Python float becomes f32, an int
    i32) holding a *copy* of a vector, as Taichi variables do;
  - parameters annotated ``ti.template()`` are passed by reference: a task's
    ``ret += ...`` reaches the caller's variable;
  - ``ti.atomic_add`` / ``ti.atomic_sub`` update their target and return the
    old value.
* Fields are numpy arrays (f32 / i32), zero-initialised.  Reading an element
  inside a kernel gives a value (a vector copy that still writes through on
  ``field[i][d] = ...``); reading ``field[None]`` from Python scope gives a
  Python number, as Taichi's host accessors do.
* Parallel ``for`` loops run serially in index order, so atomics and the
  counting sort are deterministic (slot order).
* Vector ``sum`` / ``dot`` / ``norm_sqr`` add their terms left to right, as
  ``Matrix.sum`` does; ``cross`` uses Taichi's component formula.
* ``ti.pow(x, 3.0)`` (float exponent) is ``powf`` (numpy's float32 power);
  ``ti.exp`` / ``ti.sqrt`` are numpy's float32 functions.  Taichi's fast-math
  code generation may contract or reassociate; that is not modelled.
* ``ti.random`` calls a hook that the fixture script installs.
"""
from __future__ import annotations

import ast
import builtins
import functools
import inspect
import operator
import sys
import textwrap

import numpy as np

__version__ = (0, 0, 0)  # a stand-in, not Taichi

f32 = np.float32
i32 = np.int32
u1 = np.int32
f64 = np.float64
i64 = np.int64
cpu = "cpu"
cuda = "cuda"
gpu = "gpu"

_depth = 0  # > 0 while a kernel runs (Taichi scope)
_random_hook = None


def init(*args, **kwargs):
    return None


def set_random_hook(fn):
    """fn(caller_locals) -> float in [0, 1)."""
    global _random_hook
    _random_hook = fn


def _np_dtype(dt):
    if dt is float or dt is np.float32 or dt is f32:
        return np.float32
    if dt is int or dt is np.int32 or dt is i32:
        return np.int32
    if dt is bool:
        return np.int32
    if dt is np.float64:
        return np.float64
    if dt is np.int64:
        return np.int64
    raise TypeError(f"unsupported dtype {dt!r}")


_TI_SCALARS = (np.float32, np.int32, np.bool_)


def _is_np(x):
    """A Taichi value: an f32 / i32 scalar.  numpy float64 / int64 scalars
    come from Python-scope data and fold like Python numbers."""
    return isinstance(x, _TI_SCALARS)


def _is_float(x):
    return isinstance(x, (float, np.floating))


def _to_f32(x):
    return np.float32(x)


def _to_i32(x):
    return np.int32(x)


# ---------------------------------------------------------------- vectors
class Matrix:
    """A Taichi vector (1-D) or matrix (2-D) value of f32 or i32 entries."""

    __slots__ = ("a", "owner")

    def __init__(self, data, dt=None, owner=None):
        if isinstance(data, Matrix):
            arr = data.a.copy()
        elif isinstance(data, np.ndarray):
            arr = data.copy()
        else:
            flat = _flatten(data)
            if dt is None:
                dt = np.float32 if any(_is_float(v) for v in flat) else np.int32
            arr = np.array(data, dtype=dt)
        if dt is not None and arr.dtype != dt:
            arr = arr.astype(dt)
        elif arr.dtype == np.float64:
            arr = arr.astype(np.float32)
        elif arr.dtype == np.int64 or arr.dtype == np.bool_:
            arr = arr.astype(np.int32)
        self.a = arr
        self.owner = owner

    # --- construction helpers used as ti.Vector.zero / ti.Matrix.identity
    @staticmethod
    def zero(dt, n, m=None):
        shape = (n,) if m is None else (n, m)
        return Matrix(np.zeros(shape, dtype=_np_dtype(dt)))

    @staticmethod
    def identity(dt, n):
        return Matrix(np.eye(n, dtype=_np_dtype(dt)))

    @staticmethod
    def field(n, m, dtype=float, shape=(), **kwargs):
        return Field(dtype, shape, (n, m))

    # --- element access
    @property
    def n(self):
        return self.a.shape[0]

    @property
    def m(self):
        return 1 if self.a.ndim == 1 else self.a.shape[1]

    def __len__(self):
        return self.a.shape[0]

    def __iter__(self):
        return iter(self.a[k] for k in range(self.a.shape[0]))

    def __getitem__(self, k):
        k = _key(k)
        return self.a[k]

    def __setitem__(self, k, v):
        k = _key(k)
        self.a[k] = v
        if self.owner is not None:
            fld, idx = self.owner
            fld.arr[idx][k] = v

    def fill(self, v):
        self.a[...] = v
        if self.owner is not None:
            fld, idx = self.owner
            fld.arr[idx][...] = v

    def copy(self):
        return _wrap(self.a.copy())

    def to_numpy(self):
        return self.a.copy()

    def cast(self, dt):
        return _wrap(self.a.astype(_np_dtype(dt)))

    # --- reductions in Taichi's order (entries left to right, row-major)
    def sum(self):
        flat = self.a.reshape(-1)
        s = flat[0]
        for k in range(1, flat.shape[0]):
            s = s + flat[k]
        return s

    def dot(self, other):
        return _mat_bin(operator.mul, self, other).sum()

    def norm_sqr(self):
        return _wrap(self.a * self.a).sum()

    def norm(self, eps=0):
        s = self.norm_sqr()
        if eps:
            s = s + np.float32(eps)
        return np.sqrt(np.float32(s) if s.dtype != np.float32 else s)

    def cross(self, other):
        a, b = _common(self, other)
        if a.shape[0] == 3:
            return _wrap(np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                                   a[0] * b[1] - a[1] * b[0]], dtype=a.dtype))
        return a[0] * b[1] - a[1] * b[0]

    def outer_product(self, other):
        a, b = _common(self, other)
        return _wrap(np.array([[a[i] * b[j] for j in range(b.shape[0])] for i in range(a.shape[0])],
                              dtype=a.dtype))

    def transpose(self):
        a = self.a if self.a.ndim == 2 else self.a.reshape(-1, 1)
        return _wrap(a.T.copy())

    @property
    def T(self):
        return self.transpose()

    def __matmul__(self, other):
        a, b = _common(self, other)
        a = a if a.ndim == 2 else a.reshape(-1, 1)
        vec = b.ndim == 1
        if vec:
            b = b.reshape(-1, 1)
        dt = np.result_type(a, b)
        out = np.zeros((a.shape[0], b.shape[1]), dtype=dt)
        for i in range(a.shape[0]):
            for j in range(b.shape[1]):
                s = a[i, 0] * b[0, j]
                for k in range(1, a.shape[1]):
                    s = s + a[i, k] * b[k, j]
                out[i, j] = s
        return _wrap(out.reshape(-1) if vec else out)

    def __neg__(self):
        return _wrap(-self.a)

    def __abs__(self):
        return _wrap(np.abs(self.a))

    def __repr__(self):
        return f"ti.Matrix({self.a.tolist()})"


def _flatten(x):
    if isinstance(x, (list, tuple)):
        out = []
        for v in x:
            out.extend(_flatten(v))
        return out
    return [x]


def _wrap(arr, owner=None):
    """A Matrix around a fresh array (no conversion, no copy)."""
    m = object.__new__(Matrix)
    m.a = arr
    m.owner = owner
    return m


def _common(x, y):
    """Both operands' arrays in one type: f32 if either is a float, else i32."""
    a = x.a if isinstance(x, Matrix) else np.asarray(x)
    b = y.a if isinstance(y, Matrix) else np.asarray(y)
    dt = np.float32 if (a.dtype.kind == "f" or b.dtype.kind == "f") else np.int32
    return (a if a.dtype == dt else a.astype(dt)), (b if b.dtype == dt else b.astype(dt))


def _key(k):
    if isinstance(k, Matrix):
        t = tuple(int(v) for v in k.a.reshape(-1))
        return t[0] if len(t) == 1 else t
    if isinstance(k, tuple):
        return tuple(int(v) for v in k)
    return int(k)


class Vector(Matrix):
    """ti.Vector: a 1-D Matrix."""

    __slots__ = ()

    @staticmethod
    def field(n, dtype=float, shape=(), **kwargs):
        return Field(dtype, shape, (n,))


def _mat_bin(op, a, b):
    am, bm = isinstance(a, Matrix), isinstance(b, Matrix)
    if op is operator.truediv:
        fl = True
    else:
        fl = any((m and x.a.dtype.kind == "f") or (not m and _is_float(x)) for m, x in ((am, a), (bm, b)))
    dt = np.float32 if fl else np.int32

    def conv(m, x):
        if m:
            return x.a if x.a.dtype == dt else x.a.astype(dt)
        return dt(x)

    r = op(conv(am, a), conv(bm, b))
    if r.dtype == np.bool_:
        r = r.astype(np.int32)
    return _wrap(r)


def _pow_int(x, n):
    # Taichi lowers x ** n (n an integer) to binary exponentiation
    if n == 0:
        return type(x)(1)
    neg = n < 0
    n = builtins.abs(int(n))
    result = None
    base = x
    while n:
        if n & 1:
            result = base if result is None else result * base
        n >>= 1
        if n:
            base = base * base
    if neg:
        result = np.float32(1.0) / np.float32(result)
    return result


def _bin(op, a, b):
    """One binary operator with Taichi's typing (see the module docstring)."""
    if isinstance(a, Matrix) or isinstance(b, Matrix):
        if op is operator.pow:
            if isinstance(b, (int, np.integer)):
                return Matrix(_pow_int(a.a if a.a.dtype == np.float32 else a.a.astype(np.float32), b)
                              if a.a.dtype.kind == "f" else _pow_int(a.a, b))
            return Matrix(np.power(a.a.astype(np.float32), np.float32(b)))
        if op is operator.matmul:
            return a @ b
        return _mat_bin(op, a, b)
    if not (_is_np(a) or _is_np(b)):
        return op(a, b)  # folded by Python, as Taichi's frontend folds Python values
    if op is operator.pow:
        if isinstance(b, (int, np.integer)) and not isinstance(b, bool):
            if _is_float(a):
                return _pow_int(np.float32(a), b)
            return _pow_int(np.int32(a), b)
        return np.power(np.float32(a), np.float32(b))
    if op is operator.truediv:
        return np.float32(a) / np.float32(b)
    if _is_float(a) or _is_float(b):
        return op(np.float32(a), np.float32(b))
    return op(np.int32(a), np.int32(b))


def _cmp(op, a, b):
    if isinstance(a, Matrix) or isinstance(b, Matrix):
        return _mat_bin(op, a, b)
    if not (_is_np(a) or _is_np(b)):
        return op(a, b)
    if _is_float(a) or _is_float(b):
        return bool(op(np.float32(a), np.float32(b)))
    return bool(op(int(a), int(b)))


def _var(v):
    """A new Taichi local: typed, and a copy of a vector."""
    if isinstance(v, bool):
        return v
    if isinstance(v, float):
        return np.float32(v)
    if isinstance(v, int):
        return np.int32(v)
    if isinstance(v, Matrix):
        return Matrix(v.a.copy())
    if isinstance(v, Struct):
        return Struct(**{k: _var(x) for k, x in v.__dict__.items()})
    return v


class _Box:
    """A ti.template() argument: the caller's variable, by reference."""

    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v


def _box(v):
    return v if isinstance(v, _Box) else _Box(v)


def _template_positions(f):
    fn = getattr(f, "__func__", f)
    return getattr(fn, "_ti_template_pos", ())


def _call_wb(f, args, is_name):
    """Calls a ti.func; returns the final values of the bare-name arguments
    (changed only where the callee's parameter is ti.template())."""
    tpos = _template_positions(f)
    boxes = {}
    call_args = list(args)
    for k in tpos:
        if k < len(args) and is_name[k]:
            boxes[k] = _Box(args[k])
            call_args[k] = boxes[k]
    f(*call_args)
    return tuple(boxes[k].v if k in boxes else args[k] for k in range(len(args)) if is_name[k])


def _aug_item(container, key, op, value):
    container[key] = _bin(op, container[key], value)


def _atomic_item(container, key, op, value):
    old = container[key]
    container[key] = _bin(op, old, value)
    return old


def _atomic_attr(obj, name, op, value):
    old = getattr(obj, name)
    setattr(obj, name, _bin(op, old, value))
    return old


# ------------------------------------------------------------------ fields
class Field:
    def __init__(self, dtype, shape, comp=()):
        self.dtype = _np_dtype(dtype)
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        self.shape = tuple(int(s) for s in shape)
        self.comp = tuple(comp)
        self.arr = np.zeros(self.shape + self.comp, dtype=self.dtype)

    def _idx(self, key):
        if key is None:
            return ()
        return _key(key)

    def __getitem__(self, key):
        idx = self._idx(key)
        if self.comp:
            return _wrap(self.arr[idx].copy(), owner=(self, idx))
        v = self.arr[idx]
        if _depth == 0:
            return v.item()
        return v

    def __setitem__(self, key, value):
        idx = self._idx(key)
        if self.comp:
            val = value.a if isinstance(value, Matrix) else np.asarray(value)
            if _depth == 0 and val.shape[0] > self.comp[0]:
                val = val[: self.comp[0]]  # host accessors write the field's own components
            self.arr[idx] = val
        else:
            self.arr[idx] = value

    def fill(self, v):
        self.arr[...] = v

    def from_numpy(self, a):
        self.arr[...] = np.asarray(a).reshape(self.arr.shape).astype(self.dtype)

    def to_numpy(self):
        return self.arr.copy()

    def __iter__(self):
        raise TypeError("iterate a field with ti.grouped(field)")


def field(dtype, shape=(), **kwargs):
    return Field(dtype, shape)



class Struct:
    def __init__(self, **kwargs):
        for k, v in kwargs.items():
            setattr(self, k, _var(v))


# ------------------------------------------------------------ loops, math
class _NDRange:
    def __init__(self, *ranges):
        self.ranges = [(r, ) if isinstance(r, int) else tuple(r) for r in ranges]

    def __iter__(self):
        import itertools
        rs = [range(0, r[0]) if len(r) == 1 else range(r[0], r[1]) for r in self.ranges]
        for t in itertools.product(*rs):
            yield t


def ndrange(*ranges):
    return _NDRange(*ranges)


def grouped(x):
    if isinstance(x, _NDRange):
        return (_wrap(np.array(t, dtype=np.int32)) for t in x)
    if isinstance(x, Field):
        import itertools
        return (_wrap(np.array(t, dtype=np.int32)) for t in itertools.product(*[range(s) for s in x.shape]))
    raise TypeError(x)


def static(x, *rest):
    return x


def template():
    return _TEMPLATE


_TEMPLATE = object()


class _Types:
    @staticmethod
    def ndarray(*a, **k):
        return "ndarray"

    @staticmethod
    def vector(n, dt):
        return ("vector", n, dt)

    @staticmethod
    def matrix(n, m, dt):
        return ("matrix", n, m, dt)


types = _Types()


def cast(x, dt):
    if isinstance(x, Matrix):
        return x.cast(dt)
    return _np_dtype(dt)(x)


def exp(x):
    if isinstance(x, Matrix):
        return Matrix(np.exp(x.a.astype(np.float32)))
    return np.exp(np.float32(x))


def sqrt(x):
    if isinstance(x, Matrix):
        return Matrix(np.sqrt(x.a.astype(np.float32)))
    return np.sqrt(np.float32(x))


def pow(x, y):  # noqa: A001 - Taichi's name
    return _bin(operator.pow, x, y)


def abs(x):  # noqa: A001
    if isinstance(x, Matrix):
        return Matrix(np.abs(x.a))
    if _is_np(x):
        return np.abs(x)
    return np.abs(np.float32(x)) if isinstance(x, float) else np.abs(np.int32(x))


def max(a, b):  # noqa: A001
    if _is_float(a) or _is_float(b):
        return np.fmax(np.float32(a), np.float32(b))
    return np.maximum(np.int32(a), np.int32(b))


def min(a, b):  # noqa: A001
    if _is_float(a) or _is_float(b):
        return np.fmin(np.float32(a), np.float32(b))
    return np.minimum(np.int32(a), np.int32(b))


def random(dtype=float):
    if _random_hook is None:
        raise RuntimeError("ti.random: no random hook installed")
    return np.float32(_random_hook(sys._getframe(1).f_locals))


def atomic_add(x, v):
    raise RuntimeError("ti.atomic_add outside a rewritten kernel")


def atomic_sub(x, v):
    raise RuntimeError("ti.atomic_sub outside a rewritten kernel")


def polar_decompose(A):
    raise NotImplementedError("polar_decompose: not on the DIMCV hot path")


class _MathNS:
    @staticmethod
    def cross(a, b):
        return a.cross(b)

    @staticmethod
    def clamp(x, lo, hi):
        return min(max(x, lo), hi)


math = _MathNS()


class PrefixSumExecutor:
    """ti.algorithms.PrefixSumExecutor: in-place inclusive scan."""

    def __init__(self, length):
        self.length = int(length)

    def run(self, fld):
        a = fld.arr
        a[: self.length] = np.cumsum(a[: self.length], dtype=np.int64).astype(a.dtype)


class _AlgoNS:
    PrefixSumExecutor = PrefixSumExecutor


algorithms = _AlgoNS()


def data_oriented(cls):
    return cls


# ------------------------------------------------------------- rewriting
_OPS = {ast.Add: "add", ast.Sub: "sub", ast.Mult: "mul", ast.Div: "truediv", ast.FloorDiv: "floordiv",
        ast.Mod: "mod", ast.Pow: "pow", ast.MatMult: "matmul", ast.BitAnd: "and_", ast.BitOr: "or_",
        ast.BitXor: "xor", ast.LShift: "lshift", ast.RShift: "rshift"}
_CMPS = {ast.Lt: "lt", ast.LtE: "le", ast.Gt: "gt", ast.GtE: "ge", ast.Eq: "eq", ast.NotEq: "ne"}


def _rt(name):
    return ast.Attribute(value=ast.Name(id="_ti_rt", ctx=ast.Load()), attr=name, ctx=ast.Load())


def _op(name):
    return ast.Attribute(value=ast.Name(id="_ti_op", ctx=ast.Load()), attr=name, ctx=ast.Load())


def _is_ti_call(node, names):
    f = node.func
    return (isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name) and f.value.id == "ti"
            and f.attr in names)


class _Rewriter(ast.NodeTransformer):
    def __init__(self, templates):
        self.templates = set(templates)

    # template parameters live in boxes
    def visit_Name(self, node):
        if node.id in self.templates:
            return ast.copy_location(ast.Attribute(value=ast.Name(id=node.id, ctx=ast.Load()), attr="v",
                                                   ctx=node.ctx), node)
        return node

    def visit_BinOp(self, node):
        self.generic_visit(node)
        name = _OPS[type(node.op)]
        return ast.copy_location(ast.Call(func=_rt("_bin"), args=[_op(name), node.left, node.right],
                                          keywords=[]), node)

    def visit_Compare(self, node):
        self.generic_visit(node)
        if len(node.ops) != 1 or type(node.ops[0]) not in _CMPS:
            return node
        return ast.copy_location(ast.Call(func=_rt("_cmp"), args=[_op(_CMPS[type(node.ops[0])]), node.left,
                                                                  node.comparators[0]], keywords=[]), node)

    def visit_Call(self, node):
        if _is_ti_call(node, ("atomic_add", "atomic_sub")):
            opname = "add" if node.func.attr == "atomic_add" else "sub"
            tgt = node.args[0]
            val = self.visit(node.args[1])
            if isinstance(tgt, ast.Name) and tgt.id not in self.templates:
                # (old := x, x := old op v)[0]
                old = ast.NamedExpr(target=ast.Name(id="_ti_old", ctx=ast.Store()),
                                    value=ast.Name(id=tgt.id, ctx=ast.Load()))
                new = ast.NamedExpr(target=ast.Name(id=tgt.id, ctx=ast.Store()),
                                    value=ast.Call(func=_rt("_bin"), args=[_op(opname),
                                                                           ast.Name(id="_ti_old", ctx=ast.Load()),
                                                                           val], keywords=[]))
                return ast.copy_location(ast.Subscript(value=ast.Tuple(elts=[old, new], ctx=ast.Load()),
                                                       slice=ast.Constant(0), ctx=ast.Load()), node)
            if isinstance(tgt, ast.Name):  # a template parameter: its box
                return ast.copy_location(ast.Call(func=_rt("_atomic_attr"), args=[
                    ast.Name(id=tgt.id, ctx=ast.Load()), ast.Constant("v"), _op(opname), val], keywords=[]), node)
            if isinstance(tgt, ast.Subscript):
                return ast.copy_location(ast.Call(func=_rt("_atomic_item"), args=[
                    self.visit(tgt.value), self.visit(tgt.slice), _op(opname), val], keywords=[]), node)
            if isinstance(tgt, ast.Attribute):
                return ast.copy_location(ast.Call(func=_rt("_atomic_attr"), args=[
                    self.visit(tgt.value), ast.Constant(tgt.attr), _op(opname), val], keywords=[]), node)
            raise SyntaxError("unsupported atomic target")
        self.generic_visit(node)
        return node

    def visit_Assign(self, node):
        self.generic_visit(node)
        if len(node.targets) == 1 and isinstance(node.targets[0], (ast.Name, ast.Attribute)):
            node.value = ast.Call(func=_rt("_var"), args=[node.value], keywords=[])
        return node

    def visit_AugAssign(self, node):
        target = node.target
        value = self.visit(node.value)
        opname = _OPS[type(node.op)]
        if isinstance(target, ast.Subscript):
            call = ast.Call(func=_rt("_aug_item"), args=[self.visit(target.value), self.visit(target.slice),
                                                         _op(opname), value], keywords=[])
            return ast.copy_location(ast.Expr(value=call), node)
        if isinstance(target, ast.Name):
            load = self.visit(ast.Name(id=target.id, ctx=ast.Load()))
            store = self.visit(ast.Name(id=target.id, ctx=ast.Store()))
        elif isinstance(target, ast.Attribute):
            base = self.visit(target.value)
            load = ast.Attribute(value=base, attr=target.attr, ctx=ast.Load())
            store = ast.Attribute(value=base, attr=target.attr, ctx=ast.Store())
        else:
            raise SyntaxError("unsupported augmented assignment")
        new = ast.Assign(targets=[store], value=ast.Call(func=_rt("_bin"), args=[_op(opname), load, value],
                                                         keywords=[]))
        return ast.copy_location(new, node)

    def visit_Expr(self, node):
        # a bare call statement: template arguments written back to the caller
        if isinstance(node.value, ast.Call) and not _is_ti_call(node.value, ("atomic_add", "atomic_sub")):
            call = node.value
            name_args = [isinstance(a, ast.Name) for a in call.args]
            if any(name_args) and not call.keywords and not any(isinstance(a, ast.Starred) for a in call.args):
                targets = [self.visit(ast.Name(id=a.id, ctx=ast.Store())) for a, is_n in zip(call.args, name_args)
                           if is_n]
                func = self.visit(call.func)
                args = [self.visit(a) for a in call.args]
                wb = ast.Call(func=_rt("_call_wb"), args=[func, ast.Tuple(elts=args, ctx=ast.Load()),
                                                          ast.Constant(tuple(name_args))], keywords=[])
                new = ast.Assign(targets=[ast.Tuple(elts=targets, ctx=ast.Store())], value=wb)
                return ast.copy_location(new, node)
        self.generic_visit(node)
        return node


def _rewrite(fn, kind):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    assert isinstance(fdef, ast.FunctionDef)
    fdef.decorator_list = []
    params = [a.arg for a in fdef.args.args]
    templates = []
    for a in fdef.args.args:
        ann = a.annotation
        if (kind == "func" and isinstance(ann, ast.Call) and isinstance(ann.func, ast.Attribute)
                and ann.func.attr == "template"):
            templates.append(a.arg)
        a.annotation = None
    fdef.returns = None
    fdef = _Rewriter(templates).visit(fdef)
    # box the template parameters on entry (a non-variable argument gets a fresh box)
    entry = [ast.Assign(targets=[ast.Name(id=t, ctx=ast.Store())],
                        value=ast.Call(func=_rt("_box"), args=[ast.Name(id=t, ctx=ast.Load())], keywords=[]))
             for t in templates]
    fdef.body = entry + fdef.body
    ast.fix_missing_locations(tree)
    lineno = inspect.getsourcelines(fn)[1]
    ast.increment_lineno(tree, lineno - 1)
    g = dict(fn.__globals__)
    g["_ti_rt"] = sys.modules[__name__]
    g["_ti_op"] = operator
    code = compile(tree, inspect.getsourcefile(fn), "exec")
    ns = {}
    exec(code, g, ns)
    new = ns[fdef.name]
    offset = 1 if params and params[0] == "self" else 0
    new._ti_template_pos = tuple(params.index(t) - offset for t in templates)
    return new, params


def func(fn):
    new, _ = _rewrite(fn, "func")
    return new


def kernel(fn):
    new, params = _rewrite(fn, "kernel")
    sig = inspect.signature(fn)
    anns = [sig.parameters[p].annotation for p in params]
    ret_ann = sig.return_annotation

    @functools.wraps(fn)
    def run(*args):
        global _depth
        conv = list(args)
        off = 1 if params and params[0] == "self" else 0
        for k in range(off, len(params)):
            ann = anns[k]
            if ann is float:
                conv[k] = np.float32(conv[k])
            elif ann is int:
                conv[k] = np.int32(conv[k])
        _depth += 1
        try:
            r = new(*conv)
        finally:
            _depth -= 1
        if ret_ann is float:
            return float(r)
        if ret_ann is int:
            return int(r)
        return r

    return run


class kernel_scope:
    """Context manager: run stand-in ti.func code from Python as a kernel would."""

    def __enter__(self):
        global _depth
        _depth += 1

    def __exit__(self, *exc):
        global _depth
        _depth -= 1
        return False
