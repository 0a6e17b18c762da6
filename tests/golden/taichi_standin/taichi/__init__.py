"""A numpy stand-in for the Taichi runtime, used only to generate golden fixtures.

Taichi (taichi==1.7.4) is not installed in this environment, so the reference's
own mpm_sim.py cannot run under its real runtime here.  This module provides the
small part of the Taichi API that mpm_sim.py touches, so that the reference
module imports and its @ti.kernel functions execute as plain Python:

* ``@ti.kernel`` / ``@ti.func`` are identity decorators; kernels run serially
  in struct-for order (the reference's kernels have no intra-offload races
  apart from atomic adds, whose order this fixes).
* fields are numpy arrays; element access returns numpy views, so in-place
  updates (``v[m, p][1] -= ...``) write through as in Taichi.
* arithmetic follows Taichi's default_fp=f32: field values, vectors and
  matrices are float32 or int32; Python scalar constants are folded in double
  by Python and rounded to f32 when they meet a field value (numpy 2's
  promotion rules do exactly that); struct-for indices are i32 whose products
  with float constants are f32 (``_I32``); float ``%`` is ``a - b*floor(a/b)``;
  ``@`` accumulates left to right with separate roundings.
* ``ti.svd`` restates taichi 1.7.4 python/taichi/_funcs.py ``_svd2d``: polar
  decomposition A = R S with R = [[c,-s],[s,c]] from (A00+A11, A10-A01), then
  one Jacobi rotation of S (skipped when |S01| < 1e-5), singular values sorted
  descending with the matching V, U = R V.
* ``ti.cos``, ``ti.tanh`` and ``ti.atan2`` are evaluated in double and
  rounded to f32 once; ``float(i)`` of a loop index is a Python float (the
  renderer's pixel mappings stay exact in both, since their operands are small
  integers over powers of two).

Nothing here is used by the product; it exists so that tests/golden/
make_golden.py can record the reference's outputs.
"""
from __future__ import annotations

import itertools
import math as _pymath
import operator

import numpy as np

f32 = np.float32
i32 = np.int32
f64 = np.float64
i64 = np.int64
ERROR = "error"
WARN = "warn"
INFO = "info"
cuda = "cuda"
cpu = "cpu"
gpu = "gpu"
vulkan = "vulkan"


def set_logging_level(*_a, **_k):
    return None


def init(*_a, **_k):
    return None


def sync():
    return None


def _np_dtype(dtype):
    if dtype is float or dtype is f32:
        return np.float32
    if dtype is int or dtype is i32:
        return np.int32
    return np.dtype(dtype).type


class _I32:
    """A struct-for / ndrange index: an i32 whose arithmetic with floats is f32.

    Not an ``int`` subclass on purpose: ``0.05 * i`` must reach ``__rmul__``
    (a Python float would otherwise multiply an int subclass in double).
    """
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = int(v)

    def __index__(self):
        return self.v

    def __int__(self):
        return self.v

    def __float__(self):
        return float(self.v)

    def __hash__(self):
        return hash(self.v)

    def __repr__(self):
        return f"i32({self.v})"

    def __neg__(self):
        return _I32(-self.v)

    @staticmethod
    def _wrap(op, rev=False):
        def f(self, other):
            if isinstance(other, _I32):
                other = other.v
            a, b = (other, self.v) if rev else (self.v, other)
            if isinstance(other, (float, np.floating)):
                return op(np.float32(a), np.float32(b))
            if isinstance(other, (int, np.integer)):
                if op is operator.truediv:
                    return np.float32(int(a)) / np.float32(int(b))
                return _I32(op(int(a), int(b)))
            return NotImplemented
        return f

    @staticmethod
    def _cmp(op):
        def f(self, other):
            if isinstance(other, _I32):
                other = other.v
            return op(self.v, other)
        return f


for _name, _op in [("add", operator.add), ("sub", operator.sub), ("mul", operator.mul),
                   ("truediv", operator.truediv), ("floordiv", operator.floordiv),
                   ("mod", operator.mod)]:
    setattr(_I32, f"__{_name}__", _I32._wrap(_op))
    setattr(_I32, f"__r{_name}__", _I32._wrap(_op, rev=True))
for _name, _op in [("eq", operator.eq), ("ne", operator.ne), ("lt", operator.lt),
                   ("le", operator.le), ("gt", operator.gt), ("ge", operator.ge)]:
    setattr(_I32, f"__{_name}__", _I32._cmp(_op))


class TiArray(np.ndarray):
    """float32 / int32 vector or matrix value with Taichi's element methods."""

    def cast(self, dtype):
        return np.asarray(self).astype(_np_dtype(dtype)).view(TiArray)

    def outer_product(self, other):
        a = np.asarray(self)
        b = np.asarray(other)
        out = np.empty((a.shape[0], b.shape[0]), dtype=np.result_type(a, b))
        for i in range(a.shape[0]):
            for j in range(b.shape[0]):
                out[i, j] = a[i] * b[j]
        return out.view(TiArray)

    def transpose(self, *axes):
        return np.asarray(self).T.copy().view(TiArray)

    def __matmul__(self, other):
        a = np.asarray(self)
        b = np.asarray(other)
        if b.ndim == 1:
            out = np.empty((a.shape[0],), dtype=np.result_type(a, b))
            for i in range(a.shape[0]):
                acc = a[i, 0] * b[0]
                for k in range(1, a.shape[1]):
                    acc = acc + a[i, k] * b[k]
                out[i] = acc
            return out.view(TiArray)
        out = np.empty((a.shape[0], b.shape[1]), dtype=np.result_type(a, b))
        for i in range(a.shape[0]):
            for j in range(b.shape[1]):
                acc = a[i, 0] * b[0, j]
                for k in range(1, a.shape[1]):
                    acc = acc + a[i, k] * b[k, j]
                out[i, j] = acc
        return out.view(TiArray)

    def __mod__(self, other):
        a = np.asarray(self)
        if np.issubdtype(a.dtype, np.floating):
            q = np.floor(a / other)
            return (a - other * q).view(TiArray) if np.ndim(a) else np.float32(a - other * q)
        return np.asarray(a % other).view(TiArray)

    def norm(self):
        a = np.asarray(self)
        return np.sqrt(np.sum(a * a))


def _unwrap(values):
    if isinstance(values, _I32):
        return values.v
    if isinstance(values, (list, tuple)):
        return [_unwrap(v) for v in values]
    return values


def _to_tiarray(values, dtype=None):
    arr = np.asarray(_unwrap(values))
    if dtype is not None:
        arr = arr.astype(_np_dtype(dtype))
    elif np.issubdtype(arr.dtype, np.integer):
        arr = arr.astype(np.int32)
    else:
        arr = arr.astype(np.float32)
    return arr.view(TiArray)


class Field:
    def __init__(self, shape, elem_shape, dtype):
        if isinstance(shape, int):
            shape = (shape,)
        self.shape = tuple(shape)
        self.elem_shape = tuple(elem_shape)
        self.dtype = _np_dtype(dtype)
        self.data = np.zeros(self.shape + self.elem_shape, dtype=self.dtype).view(TiArray)

    def _key(self, key):
        if key is None:
            return ()
        if not isinstance(key, tuple):
            key = (key,)
        flat = []
        for k in key:
            if isinstance(k, np.ndarray) and k.ndim == 1:
                flat.extend(int(v) for v in k)
            else:
                flat.append(int(k))
        return tuple(flat)

    def __getitem__(self, key):
        idx = self._key(key)
        return self.data[idx + (Ellipsis,)]

    def __setitem__(self, key, value):
        idx = self._key(key)
        self.data[idx + (Ellipsis,)] = np.asarray(value, dtype=self.dtype)

    def __iter__(self):
        for idx in np.ndindex(*self.shape):
            t = tuple(_I32(i) for i in idx)
            yield t if len(t) > 1 else t[0]

    def to_numpy(self):
        return np.array(self.data, dtype=self.dtype)

    def from_numpy(self, arr):
        self.data[...] = np.asarray(arr, dtype=self.dtype)

    def fill(self, val):
        self.data[...] = val


def field(dtype, shape=()):
    return Field(shape, (), dtype)


class _VectorNS:
    def __call__(self, values, dt=None):
        return _to_tiarray(values, dt)

    def field(self, n, dtype, shape):
        return Field(shape, (n,), dtype)

    def zero(self, dtype, n):
        return np.zeros((n,), dtype=_np_dtype(dtype)).view(TiArray)


class _MatrixNS:
    def __call__(self, rows, dt=None):
        return _to_tiarray(rows, dt)

    def field(self, n, m, dtype, shape):
        return Field(shape, (n, m), dtype)

    def identity(self, dtype, n):
        return np.eye(n, dtype=_np_dtype(dtype)).view(TiArray)

    def zero(self, dtype, n, m):
        return np.zeros((n, m), dtype=_np_dtype(dtype)).view(TiArray)


Vector = _VectorNS()
Matrix = _MatrixNS()


class _Types:
    @staticmethod
    def ndarray(*_a, **_k):
        return None

    @staticmethod
    def vector(*_a, **_k):
        return None

    @staticmethod
    def matrix(*_a, **_k):
        return None


types = _Types()


def kernel(fn):
    return fn


def func(fn):
    return fn


def static(x, *_a):
    return x


def ndrange(*dims):
    for idx in itertools.product(*[range(d) for d in dims]):
        yield tuple(_I32(i) for i in idx)


def max(a, b):  # noqa: A001 - mirrors ti.max
    return np.maximum(a, b)


def min(a, b):  # noqa: A001 - mirrors ti.min
    return np.minimum(a, b)


def abs(a):  # noqa: A001 - mirrors ti.abs
    return np.abs(a)


def sqrt(a):
    return np.sqrt(a)


def cos(a):
    return np.float32(_pymath.cos(float(a)))


def sin(a):
    return np.float32(_pymath.sin(float(a)))


def tanh(a):
    return np.float32(_pymath.tanh(float(a)))


def atan(a):
    return np.float32(_pymath.atan(float(a)))


def atan2(y, x):
    return np.float32(_pymath.atan2(float(y), float(x)))


def pow(a, b):  # noqa: A001 - mirrors ti.pow
    return np.power(a, b)


def atomic_add(ref, val):
    ref[...] += val
    return ref


class _MathNS:
    @staticmethod
    def sign(a):
        return np.sign(a)


math = _MathNS()


def svd(A, dt=None):
    """taichi 1.7.4 _svd2d restated (see module docstring)."""
    A = np.asarray(A).astype(np.float32).view(TiArray)
    x = A[0, 0] + A[1, 1]
    y = A[1, 0] - A[0, 1]
    scale = np.float32(1.0) / np.sqrt(x * x + y * y)
    c = x * scale
    s = y * scale
    R = Matrix([[c, -s], [s, c]])
    S = R.transpose() @ A
    if np.abs(S[0, 1]) < np.float32(1e-5):
        cc, ss = np.float32(1), np.float32(0)
        s1, s2 = S[0, 0], S[1, 1]
    else:
        tao = np.float32(0.5) * (S[0, 0] - S[1, 1])
        w = np.sqrt(tao * tao + S[0, 1] * S[0, 1])
        if tao > 0:
            t = S[0, 1] / (tao + w)
        else:
            t = S[0, 1] / (tao - w)
        cc = np.float32(1) / np.sqrt(t * t + np.float32(1))
        ss = -t * cc
        s1 = cc * cc * S[0, 0] - np.float32(2) * cc * ss * S[0, 1] + ss * ss * S[1, 1]
        s2 = ss * ss * S[0, 0] + np.float32(2) * cc * ss * S[0, 1] + cc * cc * S[1, 1]
    if s1 < s2:
        s1, s2 = s2, s1
        V = Matrix([[-ss, cc], [-cc, -ss]])
    else:
        V = Matrix([[cc, ss], [-ss, cc]])
    U = R @ V
    return U, Matrix([[s1, 0.0], [0.0, s2]]), V
