"""Serial stand-in for the slice of the Taichi API used by the reference's
jfa.py, grid.py and dynamics.py.

TEST INFRASTRUCTURE ONLY.  Taichi cannot be installed here or on the GPU
hosts, so this package lets the UNMODIFIED reference modules execute on the
CPU, one loop iteration after another, and the fixture generator
(tests/golden/make_golden.py) records what the reference's own code computes
on small inputs.  Nothing in the product imports it.

A decorated kernel or function is not run as written by Python: its source is
parsed and every arithmetic operator, comparison, local assignment and atomic
is routed through this module, which applies Taichi's rules:

- every top-level loop runs serially in index order (``ti.ndrange`` /
  ``ti.grouped`` row-major, last index fastest): the serial semantics;
- typed arithmetic on f32/i32 (numpy scalars).  A Python int or float meeting
  a typed value becomes an i32 or f32 constant; int with float promotes to
  the float type; ``/`` of two ints divides in f32; ``//`` floors; ``%`` takes
  the divisor's sign; integer arithmetic wraps;
- an expression of Python values only is evaluated by Python (in double) and
  rounded to f32 once where it meets a typed value: Taichi folds such
  expressions at compile time the same way;
- a local variable takes the type of its first assignment (a Python float
  literal declares an f32, an int an i32); later assignments are cast to it;
- ``ti.func`` arguments are passed by value (vectors are copied), annotated
  scalars and vectors are cast, and results are cast to the return
  annotation; kernel scalar arguments are cast to their annotation;
- ``int(x)`` / ``float(x)`` inside a kernel are casts to i32 / f32;
- atomics read, modify and write the lvalue and return the old value;
- ``x ** n`` with an integer ``n`` is square-and-multiply in x's type (Taichi
  demotes integer powers to multiplications); with a float exponent it is
  libm ``powf``, which Taichi's CPU backend calls;
- ``ti.round`` rounds halfway cases away from zero;
- ``ti.random()`` returns the next value of a queue that the caller fills
  (``set_random_source``), so both sides of a comparison see the same draws.

Not modelled: Taichi's default ``fast_math`` (LLVM may contract a*b+c into an
FMA or reassociate sums on hosts that allow it).  Each operation here is one
IEEE-754 f32 operation rounded to nearest, in the order the source writes it.
Python globals are read when a kernel runs; Taichi bakes them at the kernel's
first compilation, which is the same value for a process that sets them
before the first call (the fixture generator loads the modules fresh for each
case).
"""
from __future__ import annotations

import ast
import builtins
import ctypes
import ctypes.util
import inspect
import itertools
import operator
import math as _pymath
import sys
import textwrap

import numpy as np

# ------------------------------------------------------------------ types
_NP = {"i8": np.int8, "i16": np.int16, "i32": np.int32, "i64": np.int64,
       "u8": np.uint8, "u16": np.uint16, "u32": np.uint32, "u64": np.uint64,
       "f16": np.float16, "f32": np.float32, "f64": np.float64, "u1": np.int32}


class DataType:
    """A scalar type token (ti.i32, ti.f32, ...); calling it casts."""

    def __init__(self, name):
        self.name = name
        self.np = np.dtype(_NP[name])

    def __call__(self, x):
        return cast(x, self)

    def __repr__(self):
        return f"ti.{self.name}"


i8, i16, i32, i64 = (DataType(n) for n in ("i8", "i16", "i32", "i64"))
u8, u16, u32, u64 = (DataType(n) for n in ("u8", "u16", "u32", "u64"))
f16, f32, f64 = (DataType(n) for n in ("f16", "f32", "f64"))
u1 = DataType("u1")
int8, int16, int32, int64 = i8, i16, i32, i64
uint8, uint16, uint32, uint64 = u8, u16, u32, u64
float16, float32, float64 = f16, f32, f64

_F32 = np.dtype(np.float32)
_I32 = np.dtype(np.int32)
_F32T = np.float32
_I32T = np.int32

cpu = "cpu"
gpu = "gpu"
cuda = "cuda"
vulkan = "vulkan"
metal = "metal"
opengl = "opengl"
x64 = "x64"


def _dt(d) -> np.dtype:
    if isinstance(d, DataType):
        return d.np
    if d is builtins.int:
        return _I32
    if d is builtins.float:
        return _F32
    if isinstance(d, np.dtype):
        return d
    return np.dtype(d)


class _Template:
    def __repr__(self):
        return "ti.template()"


def template():
    return _Template()


class VectorType:
    """ti.math.vec3, ti.types.vector(n, dtype): annotation and constructor."""

    def __init__(self, n, dtype):
        self.n = n
        self.dtype = _dt(dtype)

    def __call__(self, *args):
        if len(args) == 1 and isinstance(args[0], (list, tuple, Vector, np.ndarray)):
            vals = list(args[0])
        elif len(args) == 1:
            vals = [args[0]] * self.n
        else:
            vals = list(args)
        if len(vals) != self.n:
            raise ValueError(f"vector of {self.n} built from {len(vals)} values")
        return Vector(vals, dt=self.dtype)


class _Types:
    @staticmethod
    def vector(n, dtype):
        return VectorType(n, dtype)

    @staticmethod
    def matrix(n, m, dtype):
        raise NotImplementedError("matrix types are not used on the hot path")


types = _Types()


def _typeof(x):
    """numpy dtype of a typed value, or None for a Python constant."""
    if isinstance(x, (bool, np.bool_)):
        return _I32 if isinstance(x, np.bool_) else None
    if isinstance(x, np.generic):
        return x.dtype
    return None


def _const_type(x) -> np.dtype:
    if isinstance(x, (bool, int, np.integer, np.bool_)):
        return _I32
    return _F32


def _promote(a: np.dtype, b: np.dtype) -> np.dtype:
    fa, fb = a.kind == "f", b.kind == "f"
    if fa and fb:
        return a if a.itemsize >= b.itemsize else b
    if fa:
        return a
    if fb:
        return b
    if a.itemsize != b.itemsize:
        return a if a.itemsize > b.itemsize else b
    if a.kind == "u" or b.kind == "u":
        return np.dtype(f"u{a.itemsize}")
    return a


def _scalar(v, dt: np.dtype):
    """Cast one scalar to dtype: float -> int truncates, ints wrap."""
    tv = type(v)
    if dt is _F32 and (tv is _F32T or tv is float or tv is _I32T or tv is int):
        return _F32T(v)
    if dt is _I32 and tv is _I32T:
        return v
    if isinstance(v, Vector):
        raise TypeError("vector where a scalar was expected")
    if dt.kind == "f":
        return dt.type(v)
    if isinstance(v, (float, np.floating)):
        v = _pymath.trunc(float(v))
    v = int(v)
    bits = dt.itemsize * 8
    v &= (1 << bits) - 1
    if dt.kind == "i" and v >= 1 << (bits - 1):
        v -= 1 << bits
    return dt.type(v)


def cast(x, dtype):
    dt = _dt(dtype)
    if isinstance(x, Vector):
        return Vector([_scalar(v, dt) for v in x.a], dt=dt)
    return _scalar(x, dt)


# ------------------------------------------------------------ arithmetic
_PY = {
    "add": lambda a, b: a + b, "sub": lambda a, b: a - b, "mul": lambda a, b: a * b,
    "truediv": lambda a, b: a / b, "floordiv": lambda a, b: a // b,
    "mod": lambda a, b: a % b, "pow": lambda a, b: a ** b,
    "lshift": lambda a, b: a << b, "rshift": lambda a, b: a >> b,
    "bitand": lambda a, b: a & b, "bitor": lambda a, b: a | b, "bitxor": lambda a, b: a ^ b,
    "matmul": lambda a, b: a @ b,
}

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.powf.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.pow.restype = ctypes.c_double
_libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
for _fn in ("expf", "logf", "sinf", "cosf", "tanf", "tanhf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]
_libm.atan2f.restype = ctypes.c_float
_libm.atan2f.argtypes = [ctypes.c_float, ctypes.c_float]


def _pow(a, b, ta, tb):
    if tb.kind in "iu":
        n = int(b)
        base = ta.type(a)
        res = ta.type(1)
        e = abs(n)
        while e:
            if e & 1:
                res = ta.type(res * base)
            base = ta.type(base * base)
            e >>= 1
        if n < 0:
            if ta.kind != "f":
                raise ValueError("negative integer power of an integer")
            res = ta.type(ta.type(1) / res)
        return res
    rt = _promote(ta, tb)
    if rt.kind != "f":
        rt = _F32
    if rt == _F32:
        return np.float32(_libm.powf(float(np.float32(a)), float(np.float32(b))))
    return rt.type(_libm.pow(float(a), float(b)))


def _f32_floordiv(x, y):
    return np.floor(x / y)


def _f32_mod(x, y):
    return x - y * np.floor(x / y)


def _i32_truediv(x, y):
    return _F32T(x) / _F32T(y)


def _f32_pow(x, y):
    return _pow(x, y, _F32, _typeof(y) or _const_type(y))


def _i32_pow(x, y):
    return _pow(x, y, _I32, _typeof(y) or _const_type(y))


_F32OP = {"add": operator.add, "sub": operator.sub, "mul": operator.mul,
          "truediv": operator.truediv, "floordiv": _f32_floordiv, "mod": _f32_mod}
_I32OP = {"add": operator.add, "sub": operator.sub, "mul": operator.mul,
          "truediv": _i32_truediv, "floordiv": operator.floordiv, "mod": operator.mod,
          "lshift": operator.lshift, "rshift": operator.rshift, "bitand": operator.and_,
          "bitor": operator.or_, "bitxor": operator.xor}
_I32_MIN, _I32_MAX = -(1 << 31), (1 << 31) - 1


def bin(op, a, b):
    """One binary operator under Taichi's typing rules."""
    ta, tb = type(a), type(b)
    # fast paths: f32/i32 values and Python constants (same rules as below)
    if op != "pow":
        if ta is _F32T:
            if tb is _F32T:
                return _F32OP[op](a, b)
            if tb is float or tb is int or tb is _I32T:
                return _F32OP[op](a, _F32T(b))
        elif ta is _I32T:
            if tb is _I32T:
                return _I32OP[op](a, b)
            if tb is int and _I32_MIN <= b <= _I32_MAX:
                return _I32OP[op](a, _I32T(b))
            if tb is _F32T or tb is float:
                return _F32OP[op](_F32T(a), _F32T(b))
        elif ta is float or ta is int:
            if tb is float or tb is int:
                return _PY[op](a, b)
            if tb is _F32T:
                return _F32OP[op](_F32T(a), b)
            if tb is _I32T:
                if ta is int and _I32_MIN <= a <= _I32_MAX:
                    return _I32OP[op](_I32T(a), b)
                return _F32OP[op](_F32T(a), _F32T(b))
    return _bin_general(op, a, b)


def _bin_general(op, a, b):
    if isinstance(a, Vector) or isinstance(b, Vector):
        return _vbin(op, a, b)
    ta, tb = _typeof(a), _typeof(b)
    if ta is None and tb is None:
        return _PY[op](a, b)
    if ta is None:
        ta = _const_type(a)
    if tb is None:
        tb = _const_type(b)
    if op == "pow":
        return _pow(a, b, ta, tb)
    rt = _promote(ta, tb)
    if op == "truediv" and rt.kind != "f":
        rt = _F32
    x, y = _scalar(a, rt), _scalar(b, rt)
    if True:
        if op == "add":
            r = x + y
        elif op == "sub":
            r = x - y
        elif op == "mul":
            r = x * y
        elif op == "truediv":
            r = x / y
        elif op == "floordiv":
            r = x // y if rt.kind != "f" else np.floor(x / y)
        elif op == "mod":
            r = x % y if rt.kind != "f" else x - y * np.floor(x / y)
        elif op in ("lshift", "rshift", "bitand", "bitor", "bitxor"):
            r = _PY[op](x, y)
        else:
            raise NotImplementedError(op)
    return rt.type(r)


def _vbin(op, a, b):
    if isinstance(a, Vector) and isinstance(b, Vector):
        if a.n != b.n:
            raise ValueError("vector sizes differ")
        vals = [bin(op, a.a[k], b.a[k]) for k in range(a.n)]
    elif isinstance(a, Vector):
        vals = [bin(op, a.a[k], b) for k in range(a.n)]
    else:
        vals = [bin(op, a, b.a[k]) for k in range(b.n)]
    return Vector(vals)


def un(op, x):
    if isinstance(x, Vector):
        return Vector([un(op, v) for v in x.a])
    t = _typeof(x)
    if t is None:
        return {"neg": lambda v: -v, "pos": lambda v: +v, "invert": lambda v: ~v}[op](x)
    if op == "neg":
        return t.type(-x)
    if op == "pos":
        return x
    return t.type(~x)


_CMP = {"lt": lambda a, b: a < b, "le": lambda a, b: a <= b, "gt": lambda a, b: a > b,
        "ge": lambda a, b: a >= b, "eq": lambda a, b: a == b, "ne": lambda a, b: a != b}


def cmp(op, a, b):
    ta, tb = type(a), type(b)
    if (ta is tb and (ta is _F32T or ta is _I32T or ta is int)) or \
            (ta is _F32T and tb is float) or (ta is _I32T and tb is int):
        if ta is _F32T and tb is float:
            b = _F32T(b)
        return bool(_CMP[op](a, b))
    if isinstance(a, Vector) or isinstance(b, Vector):
        raise NotImplementedError("vector comparison")
    ta, tb = _typeof(a), _typeof(b)
    if ta is None and tb is None:
        return _CMP[op](a, b)
    if ta is None:
        ta = _const_type(a)
    if tb is None:
        tb = _const_type(b)
    rt = _promote(ta, tb)
    return bool(_CMP[op](_scalar(a, rt), _scalar(b, rt)))


# ------------------------------------------------------------ variables
class _Unbound:
    def __repr__(self):
        return "<unbound>"


UNBOUND = _Unbound()


def _declare(v):
    if isinstance(v, (bool, np.bool_)):
        return v
    if isinstance(v, int):
        return _scalar(v, _I32)
    if isinstance(v, float):
        return np.float32(v)
    if isinstance(v, Vector):
        return v.copy()
    return v


def assign(old, v):
    """``x = v``: declare on first assignment, else cast to x's type."""
    if old is UNBOUND:
        return _declare(v)
    if isinstance(old, Vector):
        if not isinstance(v, Vector):
            raise TypeError("scalar assigned to a vector variable")
        return Vector([_scalar(x, old.dtype) for x in v.a], dt=old.dtype)
    if isinstance(old, (bool, np.bool_)):
        return v
    t = _typeof(old)
    if t is None or isinstance(v, Vector) or not isinstance(v, (int, float, np.generic)):
        return _declare(v)
    return _scalar(v, t)


def augitem(container, idx, op, v):
    """``container[idx] op= v`` (Taichi makes it atomic; serial here)."""
    container[idx] = bin(op, container[idx], v)


def atomic(op, container, idx, v):
    old = container[idx]
    if op in ("add", "sub", "bitand", "bitor", "bitxor"):
        new = bin(op, old, v)
    elif op == "max":
        new = max(old, v)
    elif op == "min":
        new = min(old, v)
    else:
        raise NotImplementedError(op)
    container[idx] = new
    return old


# -------------------------------------------------------------- vectors
class Vector:
    """A small vector over a 1-D numpy array (its own, or a view of a field)."""

    __slots__ = ("a",)

    def __init__(self, data, dt=None):
        if isinstance(data, np.ndarray) and dt is None:
            self.a = data
            return
        if type(data) is list and data:
            t0 = type(data[0])
            if t0 is _F32T or t0 is _I32T:
                same = all(type(v) is t0 for v in data)
                if same and (dt is None or _dt(dt) is (_F32 if t0 is _F32T else _I32)):
                    self.a = np.array(data, dtype=t0)
                    return
        vals = list(data.a if isinstance(data, Vector) else data)
        if dt is None:
            t = None
            for v in vals:
                vt = _typeof(v) or _const_type(v)
                t = vt if t is None else _promote(t, vt)
            dt = t or _I32
        dt = _dt(dt)
        self.a = np.array([_scalar(v, dt) for v in vals], dtype=dt)

    @classmethod
    def field(cls, n, dtype, shape):
        return Field(dtype, shape, n)

    @property
    def n(self):
        return self.a.shape[0]

    @property
    def dtype(self):
        return self.a.dtype

    def copy(self):
        return Vector(self.a.copy())

    def __getitem__(self, k):
        return self.a[int(k)]

    def __setitem__(self, k, v):
        self.a[int(k)] = _scalar(v, self.a.dtype)

    def __len__(self):
        return self.n

    def __iter__(self):
        return iter(list(self.a))

    def dot(self, o):
        acc = None
        for k in range(self.n):
            p = bin("mul", self.a[k], o.a[k])
            acc = p if acc is None else bin("add", acc, p)
        return acc

    def norm_sqr(self):
        return self.dot(self)

    def norm(self, eps=0):
        return sqrt(bin("add", self.norm_sqr(), eps))

    def normalized(self, eps=0):
        inv = bin("truediv", 1, bin("add", self.norm(), eps))
        return bin("mul", inv, self)

    def sum(self):
        acc = self.a[0]
        for k in range(1, self.n):
            acc = bin("add", acc, self.a[k])
        return acc

    def to_numpy(self):
        return self.a.copy()

    # Python-scope arithmetic (kernel code goes through bin() already)
    def __add__(self, o): return bin("add", self, o)
    def __radd__(self, o): return bin("add", o, self)
    def __sub__(self, o): return bin("sub", self, o)
    def __rsub__(self, o): return bin("sub", o, self)
    def __mul__(self, o): return bin("mul", self, o)
    def __rmul__(self, o): return bin("mul", o, self)
    def __truediv__(self, o): return bin("truediv", self, o)
    def __neg__(self): return un("neg", self)

    def __repr__(self):
        return f"Vector({self.a.tolist()}, {self.a.dtype})"


Matrix = Vector


# --------------------------------------------------------------- fields
_KERNEL_DEPTH = [0]


class Field:
    """ti.field / ti.Vector.field over a numpy array."""

    def __init__(self, dtype, shape, n=None):
        if isinstance(shape, (int, np.integer)):
            shape = (int(shape),)
        self.shape = tuple(int(s) for s in shape)
        self.n = n
        self.dtype = _dt(dtype)
        self.a = np.zeros(self.shape + ((n,) if n else ()), self.dtype)

    def _key(self, key):
        if key is None:
            key = ()
        elif isinstance(key, Vector):
            key = tuple(int(v) for v in key.a)
        elif isinstance(key, tuple):
            flat = []
            for k in key:
                if isinstance(k, Vector):
                    flat.extend(int(v) for v in k.a)
                else:
                    flat.append(int(k))
            key = tuple(flat)
        else:
            key = (int(key),)
        if len(key) != len(self.shape):
            raise IndexError(f"{len(key)} indices for a field of shape {self.shape}")
        for k, s in zip(key, self.shape):
            if not 0 <= k < s:
                raise IndexError(f"index {key} out of range for a field of shape {self.shape}")
        return key

    def __getitem__(self, key):
        k = self._key(key)
        if self.n:
            return Vector(self.a[k])
        v = self.a[k]
        return v if _KERNEL_DEPTH[0] else v.item()

    def __setitem__(self, key, v):
        k = self._key(key)
        if self.n:
            vals = v.a if isinstance(v, Vector) else list(v)
            self.a[k] = [_scalar(x, self.dtype) for x in vals]
        else:
            self.a[k] = _scalar(v, self.dtype)

    def to_numpy(self):
        return self.a.copy()

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if arr.shape != self.a.shape:
            raise ValueError(f"from_numpy shape {arr.shape} != field {self.a.shape}")
        self.a[...] = arr.astype(self.dtype)

    def fill(self, v):
        self.a[...] = _scalar(v, self.dtype)


def field(dtype, shape=(), **kw):
    return Field(dtype, shape)


# ---------------------------------------------------------------- loops
class ndrange:
    def __init__(self, *dims):
        self.ranges = []
        for d in dims:
            if isinstance(d, (tuple, list)):
                self.ranges.append(range(int(d[0]), int(d[1])))
            else:
                self.ranges.append(range(int(d)))

    def __iter__(self):
        for t in itertools.product(*self.ranges):
            yield t if len(t) > 1 else t[0]


class grouped:
    def __init__(self, x):
        if isinstance(x, Field):
            self.it = ndrange(*x.shape)
        elif isinstance(x, ndrange):
            self.it = x
        else:
            raise TypeError("ti.grouped over an unsupported object")

    def __iter__(self):
        for t in self.it:
            t = t if isinstance(t, tuple) else (t,)
            yield Vector(np.array(t, np.int32))


def static(x, *rest):
    return (x, *rest) if rest else x


def loop_config(**kw):
    return None


def init(*a, **kw):
    return None


def sync():
    return None


# ----------------------------------------------------------- functions
_PYMATH = {}


def _float_unary(fn, x):
    if isinstance(x, Vector):
        return Vector([_float_unary(fn, v) for v in x.a])
    if type(x) in (int, float):
        # a Python constant: Taichi applies Python's own math to it (in double)
        return _PYMATH[fn](x)
    t = _typeof(x) or _const_type(x)
    if t.kind != "f":
        t = _F32
    return t.type(fn(t.type(x)))


def floor(x, dtype=None):
    r = _float_unary(np.floor, x)
    return cast(r, dtype) if dtype is not None else r


def ceil(x, dtype=None):
    r = _float_unary(np.ceil, x)
    return cast(r, dtype) if dtype is not None else r


def _round_away(v):
    f = float(v)
    r = _pymath.floor(abs(f) + 0.5)
    return _pymath.copysign(r, f)


def round(x, dtype=None):  # noqa: A001 - Taichi's name
    r = _float_unary(_round_away, x)
    return cast(r, dtype) if dtype is not None else r


def sqrt(x):
    return _float_unary(np.sqrt, x)


def exp(x):
    if type(x) in (int, float):
        return _pymath.exp(x)
    return _float_unary(lambda v: _libm.expf(float(v)) if v.dtype == _F32 else np.exp(v), x)


def log(x):
    if type(x) in (int, float):
        return _pymath.log(x)
    return _float_unary(lambda v: _libm.logf(float(v)) if v.dtype == _F32 else np.log(v), x)


def sin(x):
    if type(x) in (int, float):
        return _pymath.sin(x)
    return _float_unary(lambda v: _libm.sinf(float(v)) if v.dtype == _F32 else np.sin(v), x)


def cos(x):
    if type(x) in (int, float):
        return _pymath.cos(x)
    return _float_unary(lambda v: _libm.cosf(float(v)) if v.dtype == _F32 else np.cos(v), x)


def abs(x):  # noqa: A001
    if isinstance(x, Vector):
        return Vector([abs(v) for v in x.a])
    t = _typeof(x)
    if t is None:
        return builtins.abs(x)
    with np.errstate(all="ignore"):
        return t.type(np.abs(x))


def _minmax(pick, a, b):
    if isinstance(a, Vector) or isinstance(b, Vector):
        n = a.n if isinstance(a, Vector) else b.n
        ga = (lambda k: a.a[k]) if isinstance(a, Vector) else (lambda k: a)
        gb = (lambda k: b.a[k]) if isinstance(b, Vector) else (lambda k: b)
        return Vector([_minmax(pick, ga(k), gb(k)) for k in range(n)])
    ta, tb = _typeof(a), _typeof(b)
    if ta is None and tb is None:
        return pick(a, b)
    rt = _promote(ta or _const_type(a), tb or _const_type(b))
    return pick(_scalar(a, rt), _scalar(b, rt))


def max(a, b, *more):  # noqa: A001
    r = _minmax(lambda x, y: x if x >= y else y, a, b)
    for m in more:
        r = max(r, m)
    return r


def min(a, b, *more):  # noqa: A001
    r = _minmax(lambda x, y: x if x <= y else y, a, b)
    for m in more:
        r = min(r, m)
    return r


def select(c, a, b):
    return a if c else b


_RANDOM = [None]


def set_random_source(fn):
    """fn(dtype) -> next draw; the fixture generator supplies Philox draws."""
    _RANDOM[0] = fn


def random(dtype=None):
    if _RANDOM[0] is None:
        raise RuntimeError("ti.random() has no source: call set_random_source first")
    return _RANDOM[0](_dt(dtype) if dtype is not None else _F32)


def atomic_add(x, v):
    raise RuntimeError("atomics are rewritten inside kernels and are not callable directly")


atomic_sub = atomic_max = atomic_min = atomic_or = atomic_and = atomic_xor = atomic_add


# ------------------------------------------------- kernel / func rewrite
_BINOPS = {ast.Add: "add", ast.Sub: "sub", ast.Mult: "mul", ast.Div: "truediv",
           ast.FloorDiv: "floordiv", ast.Mod: "mod", ast.Pow: "pow", ast.LShift: "lshift",
           ast.RShift: "rshift", ast.BitAnd: "bitand", ast.BitOr: "bitor",
           ast.BitXor: "bitxor", ast.MatMult: "matmul"}
_CMPOPS = {ast.Lt: "lt", ast.LtE: "le", ast.Gt: "gt", ast.GtE: "ge", ast.Eq: "eq",
           ast.NotEq: "ne"}
_ATOMICS = {"atomic_add": "add", "atomic_sub": "sub", "atomic_max": "max",
            "atomic_min": "min", "atomic_or": "bitor", "atomic_and": "bitand",
            "atomic_xor": "bitxor"}
_RT = "_taichi_standin_rt_"


def _rt(attr):
    return ast.Attribute(value=ast.Name(id=_RT, ctx=ast.Load()), attr=attr, ctx=ast.Load())


def _call(attr, *args):
    return ast.Call(func=_rt(attr), args=list(args), keywords=[])


def _locals_get(name):
    get = ast.Attribute(value=ast.Call(func=ast.Name(id="locals", ctx=ast.Load()), args=[],
                                       keywords=[]), attr="get", ctx=ast.Load())
    return ast.Call(func=get, args=[ast.Constant(name), _rt("UNBOUND")], keywords=[])


class _Rewriter(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        return _call("bin", ast.Constant(_BINOPS[type(node.op)]), node.left, node.right)

    def visit_UnaryOp(self, node):
        self.generic_visit(node)
        op = {ast.USub: "neg", ast.UAdd: "pos", ast.Invert: "invert"}.get(type(node.op))
        return node if op is None else _call("un", ast.Constant(op), node.operand)

    def visit_Compare(self, node):
        self.generic_visit(node)
        parts, left = [], node.left
        for op, right in zip(node.ops, node.comparators):
            if type(op) not in _CMPOPS:
                parts.append(ast.Compare(left=left, ops=[op], comparators=[right]))
            else:
                parts.append(_call("cmp", ast.Constant(_CMPOPS[type(op)]), left, right))
            left = right
        return parts[0] if len(parts) == 1 else ast.BoolOp(op=ast.And(), values=parts)

    def visit_Assign(self, node):
        self.generic_visit(node)
        if len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            node.value = _call("assign", _locals_get(node.targets[0].id), node.value)
        return node

    def visit_AnnAssign(self, node):
        self.generic_visit(node)
        if node.value is not None and isinstance(node.target, ast.Name):
            node.value = _call("cast", node.value, node.annotation)
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        op = ast.Constant(_BINOPS[type(node.op)])
        t = node.target
        if isinstance(t, ast.Name):
            val = _call("bin", op, ast.Name(id=t.id, ctx=ast.Load()), node.value)
            return ast.Assign(targets=[ast.Name(id=t.id, ctx=ast.Store())],
                              value=_call("assign", _locals_get(t.id), val))
        if isinstance(t, ast.Subscript):
            return ast.Expr(value=_call("augitem", _load(t.value), _load(t.slice), op,
                                        node.value))
        raise NotImplementedError("augmented assignment to an attribute")

    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if (isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name)
                and f.value.id == "ti" and f.attr in _ATOMICS):
            tgt = node.args[0]
            if not isinstance(tgt, ast.Subscript):
                raise NotImplementedError("atomic on a non-subscript target")
            return _call("atomic", ast.Constant(_ATOMICS[f.attr]), _load(tgt.value),
                         _load(tgt.slice), node.args[1])
        if isinstance(f, ast.Name) and f.id in ("int", "float") and len(node.args) == 1:
            return _call("cast", node.args[0], _rt("i32" if f.id == "int" else "f32"))
        return node


def _load(node):
    for n in ast.walk(node):
        if hasattr(n, "ctx"):
            n.ctx = ast.Load()
    return node


def _rewrite(fn):
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    tree = ast.fix_missing_locations(_Rewriter().visit(tree))
    ast.increment_lineno(tree, fn.__code__.co_firstlineno - 1)
    code = compile(tree, fn.__code__.co_filename, "exec")
    g = fn.__globals__
    g[_RT] = sys.modules[__name__]
    ns: dict = {}
    exec(code, g, ns)
    return ns[fdef.name]


def _cast_to(v, ann):
    if ann is f32 and type(v) is _F32T:
        return v
    if ann is i32 and type(v) is _I32T:
        return v
    if isinstance(ann, DataType):
        return _scalar(v, ann.np) if not isinstance(v, Vector) else cast(v, ann)
    if isinstance(ann, VectorType):
        if v.a.dtype is ann.dtype:
            return v
        return Vector([_scalar(x, ann.dtype) for x in v.a], dt=ann.dtype)
    return v


def _python_value(v):
    if isinstance(v, Vector):
        return v.a.copy()
    if isinstance(v, np.generic):
        return v.item()
    return v


def kernel(fn):
    impl = _rewrite(fn)
    sig = inspect.signature(fn)
    ret = sig.return_annotation

    def wrapper(*args, **kw):
        b = sig.bind(*args, **kw)
        for name, val in list(b.arguments.items()):
            b.arguments[name] = _cast_to(val, sig.parameters[name].annotation)
        _KERNEL_DEPTH[0] += 1
        try:
            with np.errstate(all="ignore"):
                r = impl(*b.args, **b.kwargs)
        finally:
            _KERNEL_DEPTH[0] -= 1
        if r is None:
            return None
        if isinstance(ret, tuple):
            return tuple(_python_value(_cast_to(v, a)) for v, a in zip(r, ret))
        return _python_value(_cast_to(r, ret))

    wrapper.__name__ = fn.__name__
    wrapper.__wrapped_reference__ = fn
    return wrapper


def func(fn):
    impl = _rewrite(fn)
    sig = inspect.signature(fn)
    ret = sig.return_annotation
    params = list(sig.parameters.values())

    def wrapper(*args):
        conv = []
        for p, a in zip(params, args):
            if isinstance(a, Vector):
                a = a.copy()
            conv.append(_cast_to(a, p.annotation))
        r = impl(*conv)
        if isinstance(ret, tuple):
            return tuple(_cast_to(v, a) for v, a in zip(r, ret))
        return _cast_to(r, ret)

    wrapper.__name__ = fn.__name__
    return wrapper


_PYMATH.update({np.floor: _pymath.floor, np.ceil: _pymath.ceil, np.sqrt: _pymath.sqrt,
                _round_away: _round_away})


def data_oriented(cls):
    return cls


from . import math  # noqa: E402,F401  (ti.math.vec3 and friends)
