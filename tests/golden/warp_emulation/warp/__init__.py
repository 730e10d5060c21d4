"""CPU emulation of the subset of NVIDIA Warp's kernel language that the reference's rigid-contact
path is written in -- TEST INFRASTRUCTURE ONLY.

It lets the reference's own kernel source (``newton/_src/geometry/*.py``, ``sim/collide.py``,
``solvers/xpbd/*.py``, ``solvers/solver.py``, ``math/*.py``) run unmodified as plain Python, so the
golden vectors in ``tests/golden/`` come from the reference code itself rather than from a
restatement of it.  ``tests/golden/make_golden.py`` puts this directory first on ``sys.path``;
nothing in the package or in ``bench.py`` imports it.

Semantics (Warp's documented kernel semantics, restated):

* fp32 arithmetic: every value of a ``float`` / ``wp.float32`` type is a ``numpy.float32`` scalar,
  and NumPy scalar arithmetic rounds every operation to float32 (no fused multiply-add), in the
  order the source writes it; Python float literals adopt float32 when they meet a float32
  (NumPy's scalar promotion rules).  Struct fields convert on assignment to their declared type.
* vectors, quaternions (x, y, z, w), transforms (p, q), spatial vectors (top, bottom) and
  row-major matrices are value types; ``quat_rotate``, ``transform_*``, ``normalize`` and the
  other builtins follow Warp's definitions (same operation order as Warp's C++ builtins).
* ``wp.launch`` runs a kernel's threads one after another in thread-index order, so atomic sums
  accumulate in that order (Warp's device order is unspecified).
* ``wp.func`` / ``wp.kernel`` / ``wp.struct`` bodies are ordinary Python functions and classes;
  ``wp.static`` and ``wp.constant`` return their argument.
"""

from __future__ import annotations

import builtins
import contextlib
import math as _math
import types as _pytypes

import numpy as np

np.seterr(all="ignore")

__version__ = "emulated"

# ----------------------------------------------------------------------------- scalar types
float16 = np.float16
float32 = np.float32
float64 = np.float64
int8, uint8, int16, uint16 = np.int8, np.uint8, np.int16, np.uint16
int32, uint32, int64, uint64 = np.int32, np.uint32, np.int64, np.uint64
bool = builtins.bool  # noqa: A001
Any = object

_FLOAT_TYPES = (np.float16, np.float32, np.float64)
_INT_TYPES = (np.int8, np.uint8, np.int16, np.uint16, np.int32, np.uint32, np.int64, np.uint64)

pi = np.float32(_math.pi)
tau = np.float32(2.0 * _math.pi)
e = np.float32(_math.e)
inf = np.float32(np.inf)
nan = np.float32(np.nan)
INF = inf


class DeviceLike:  # annotation only
    pass


Device = DeviceLike


class Float32Cast:
    """Stand-in for the builtin ``float`` inside emulated modules: a kernel's ``float(x)`` is an
    fp32 conversion, and ``float`` as an annotation means fp32."""

    def __new__(cls, x=0.0):
        return np.float32(x)


def _is_scalar(x):
    return isinstance(x, (builtins.int, builtins.float, builtins.bool, np.integer, np.floating, np.bool_))


def _conv(dtype, x):
    if dtype is np.float32:
        return np.float32(x)
    if dtype in _INT_TYPES:
        return dtype(builtins.int(x))
    return dtype(x)


# ----------------------------------------------------------------------------- vectors
class _VecBase:
    _n = 0
    _dtype = np.float32
    __slots__ = ("c",)
    __array_ufunc__ = None  # numpy scalars defer to the value type's reflected operators

    def __init__(self, *args, **kw):
        n, dt = self._n, self._dtype
        if kw:
            # vector(length=..., dtype=...) style construction is not used inside kernels
            raise TypeError("keyword construction of a vector value is not supported")
        flat = []
        for a in args:
            if isinstance(a, (_VecBase, list, tuple, np.ndarray)):
                flat.extend(list(a))
            elif isinstance(a, Transform):
                flat.extend(a.components())
            else:
                flat.append(a)
        if not flat:
            c = [_conv(dt, 0)] * n
        elif len(flat) == 1 and n != 1:
            c = [_conv(dt, flat[0])] * n
        elif len(flat) == n:
            c = [_conv(dt, x) for x in flat]
        else:
            raise TypeError(f"{type(self).__name__} takes {n} components, got {len(flat)}")
        self.c = c

    @classmethod
    def _make(cls, comps):
        v = cls.__new__(cls)
        v.c = list(comps)
        return v

    # sequence protocol
    def __len__(self):
        return self._n

    def __iter__(self):
        return iter(self.c)

    def __getitem__(self, i):
        if isinstance(i, slice):
            comps = self.c[i]
            return vector(len(comps), self._dtype)._make(comps)
        return self.c[builtins.int(i)]

    def __setitem__(self, i, v):
        self.c[builtins.int(i)] = _conv(self._dtype, v)

    def _get(self, k):
        return self.c[k]

    x = property(lambda s: s.c[0], lambda s, v: s.__setitem__(0, v))
    y = property(lambda s: s.c[1], lambda s, v: s.__setitem__(1, v))
    z = property(lambda s: s.c[2], lambda s, v: s.__setitem__(2, v))
    w = property(lambda s: s.c[3], lambda s, v: s.__setitem__(3, v))

    def __repr__(self):
        return f"{type(self).__name__}({', '.join(repr(builtins.float(x)) for x in self.c)})"

    def __array__(self, dtype=None, copy=None):
        return np.array(self.c, dtype=dtype or self._dtype)

    # arithmetic (component-wise, in component order)
    def _bin(self, o, f):
        if isinstance(o, _VecBase):
            if o._n != self._n:
                raise TypeError("vector length mismatch")
            return type(self)._make([f(a, b) for a, b in zip(self.c, o.c)])
        return NotImplemented

    def __add__(self, o):
        return self._bin(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._bin(o, lambda a, b: a - b)

    def __neg__(self):
        return type(self)._make([-a for a in self.c])

    def __pos__(self):
        return type(self)._make(list(self.c))

    def __mul__(self, o):
        if _is_scalar(o):
            s = _conv(self._dtype, o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([a * s for a in self.c])
        if isinstance(o, Mat):
            return _vec_mat(self, o)
        return NotImplemented

    def __rmul__(self, o):
        if _is_scalar(o):
            s = _conv(self._dtype, o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([s * a for a in self.c])
        return NotImplemented

    def __truediv__(self, o):
        if _is_scalar(o):
            s = _conv(self._dtype, o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([a / s for a in self.c])
        return NotImplemented

    def __rtruediv__(self, o):
        if _is_scalar(o):
            s = _conv(self._dtype, o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([s / a for a in self.c])
        return NotImplemented

    def __matmul__(self, o):
        if isinstance(o, Mat):
            return _vec_mat(self, o)
        return NotImplemented

    def __eq__(self, o):
        if isinstance(o, _VecBase):
            return builtins.all(a == b for a, b in zip(self.c, o.c))
        return NotImplemented

    def __ne__(self, o):
        r = self.__eq__(o)
        return r if r is NotImplemented else not r

    __hash__ = None


_vector_cache: dict = {}


def vector(length=None, dtype=np.float32, **kw):
    """wp.types.vector(length, dtype): a vector value class."""
    if length is None:
        length = kw.get("length")
    dtype = kw.get("dtype", dtype)
    if dtype in (builtins.float, Float32Cast):
        dtype = np.float32
    if dtype is builtins.int:
        dtype = np.int32
    key = (builtins.int(length), dtype)
    if key not in _vector_cache:
        name = f"vec{length}{'i' if dtype in _INT_TYPES else ''}"
        _vector_cache[key] = type(name, (_VecBase,), {"_n": builtins.int(length), "_dtype": dtype,
                                                       "__slots__": ()})
    return _vector_cache[key]


vec2 = vector(2, np.float32)
vec3 = vector(3, np.float32)
vec4 = vector(4, np.float32)
vec2i = vector(2, np.int32)
vec3i = vector(3, np.int32)
vec4i = vector(4, np.int32)
vec2f, vec3f, vec4f = vec2, vec3, vec4
vec2d = vector(2, np.float64)
vec3d = vector(3, np.float64)
spatial_vector = vector(6, np.float32)
spatial_vectorf = spatial_vector


class quat(_VecBase):
    """Quaternion (x, y, z, w); the default value is the identity."""

    _n = 4
    _dtype = np.float32
    __slots__ = ()

    def __init__(self, *args):
        if not args:
            self.c = [np.float32(0), np.float32(0), np.float32(0), np.float32(1)]
            return
        super().__init__(*args)

    def __mul__(self, o):
        if isinstance(o, quat):
            return _qmul(self, o)
        return super().__mul__(o)


quatf = quat


def _qmul(a, b):
    ax, ay, az, aw = a.c
    bx, by, bz, bw = b.c
    return quat._make([aw * bx + bw * ax + ay * bz - by * az,
                       aw * by + bw * ay + az * bx - bz * ax,
                       aw * bz + bw * az + ax * by - bx * ay,
                       aw * bw - ax * bx - ay * by - az * bz])


# ----------------------------------------------------------------------------- matrices
class Mat:
    _rows = 0
    _cols = 0
    _dtype = np.float32
    __slots__ = ("m",)
    __array_ufunc__ = None

    def __init__(self, *args):
        R, C = self._rows, self._cols
        flat = []
        for a in args:
            if isinstance(a, Mat):
                flat.extend([x for row in a.m for x in row])
            elif isinstance(a, (_VecBase, list, tuple, np.ndarray)):
                flat.extend(list(np.asarray(a, dtype=np.float64).reshape(-1)) if isinstance(a, np.ndarray)
                            else list(a))
            else:
                flat.append(a)
        if not flat:
            self.m = [[np.float32(0)] * C for _ in range(R)]
        elif len(flat) == 1:
            self.m = [[_conv(self._dtype, flat[0])] * C for _ in range(R)]
        elif len(flat) == R * C:
            self.m = [[_conv(self._dtype, flat[i * C + j]) for j in range(C)] for i in range(R)]
        else:
            raise TypeError(f"{type(self).__name__} takes {R * C} values, got {len(flat)}")

    @classmethod
    def _make(cls, rows):
        v = cls.__new__(cls)
        v.m = [list(r) for r in rows]
        return v

    def __getitem__(self, i):
        if isinstance(i, tuple):
            return self.m[builtins.int(i[0])][builtins.int(i[1])]
        return vector(self._cols, self._dtype)._make(self.m[builtins.int(i)])

    def __setitem__(self, i, v):
        if isinstance(i, tuple):
            self.m[builtins.int(i[0])][builtins.int(i[1])] = _conv(self._dtype, v)
        else:
            self.m[builtins.int(i)] = [_conv(self._dtype, x) for x in v]

    def __len__(self):
        return self._rows

    def __iter__(self):
        return (self[i] for i in range(self._rows))

    def __array__(self, dtype=None, copy=None):
        return np.array(self.m, dtype=dtype or self._dtype)

    def __repr__(self):
        return f"{type(self).__name__}({self.m})"

    def _ew(self, o, f):
        if isinstance(o, Mat):
            return type(self)._make([[f(a, b) for a, b in zip(ra, rb)] for ra, rb in zip(self.m, o.m)])
        return NotImplemented

    def __add__(self, o):
        return self._ew(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._ew(o, lambda a, b: a - b)

    def __neg__(self):
        return type(self)._make([[-a for a in r] for r in self.m])

    def __mul__(self, o):
        if _is_scalar(o):
            s = np.float32(o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([[a * s for a in r] for r in self.m])
        return self.__matmul__(o)

    def __rmul__(self, o):
        if _is_scalar(o):
            s = np.float32(o) if isinstance(o, (builtins.float, builtins.int)) else o
            return type(self)._make([[s * a for a in r] for r in self.m])
        return NotImplemented

    def __truediv__(self, o):
        s = np.float32(o) if isinstance(o, (builtins.float, builtins.int)) else o
        return type(self)._make([[a / s for a in r] for r in self.m])

    def __matmul__(self, o):
        if isinstance(o, _VecBase):
            return _mat_vec(self, o)
        if isinstance(o, Mat):
            return _mat_mat(self, o)
        return NotImplemented

    __hash__ = None


def _mat_vec(a, v):
    # Warp: r = col0 * v0; r += col_i * v_i -> per row a left-to-right sum
    out = []
    for row in a.m:
        s = row[0] * v.c[0]
        for j in range(1, a._cols):
            s = s + row[j] * v.c[j]
        out.append(s)
    return vector(a._rows, a._dtype)._make(out)


def _vec_mat(v, a):
    out = []
    for j in range(a._cols):
        s = v.c[0] * a.m[0][j]
        for i in range(1, a._rows):
            s = s + v.c[i] * a.m[i][j]
        out.append(s)
    return vector(a._cols, a._dtype)._make(out)


def _mat_mat(a, b):
    R, K, C = a._rows, a._cols, b._cols
    rows = []
    for i in range(R):
        row = []
        for j in range(C):
            s = np.float32(0.0)
            for k in range(K):
                s = s + a.m[i][k] * b.m[k][j]
            row.append(s)
        rows.append(row)
    return matrix((R, C), a._dtype)._make(rows)


_matrix_cache: dict = {}


def matrix(shape=None, dtype=np.float32, **kw):
    if shape is None:
        shape = kw.get("shape")
    dtype = kw.get("dtype", dtype)
    if dtype in (builtins.float, Float32Cast):
        dtype = np.float32
    key = (builtins.int(shape[0]), builtins.int(shape[1]), dtype)
    if key not in _matrix_cache:
        _matrix_cache[key] = type(f"mat{shape[0]}{shape[1]}", (Mat,),
                                  {"_rows": key[0], "_cols": key[1], "_dtype": dtype, "__slots__": ()})
    return _matrix_cache[key]


mat22 = matrix((2, 2))
mat33 = matrix((3, 3))
mat44 = matrix((4, 4))
mat33f = mat33
spatial_matrix = matrix((6, 6))


# ----------------------------------------------------------------------------- transforms
class Transform:
    """wp.transform: translation p (vec3) and rotation q (quat)."""

    __slots__ = ("p", "q")
    __array_ufunc__ = None

    def __init__(self, *args, p=None, q=None):
        if p is not None or q is not None:
            self.p = vec3(p) if p is not None else vec3()
            self.q = quat(q) if q is not None else quat()
            return
        if not args:
            self.p, self.q = vec3(), quat()
        elif len(args) == 2 and not _is_scalar(args[0]):
            self.p, self.q = vec3(args[0]), quat(args[1])
        elif len(args) == 1 and isinstance(args[0], Transform):
            self.p, self.q = vec3(args[0].p), quat(args[0].q)
        else:
            flat = []
            for a in args:
                flat.extend(list(a) if not _is_scalar(a) else [a])
            if len(flat) != 7:
                raise TypeError("transform takes 7 components")
            self.p, self.q = vec3(*flat[:3]), quat(*flat[3:])

    def components(self):
        return list(self.p.c) + list(self.q.c)

    def __getitem__(self, i):
        return self.components()[builtins.int(i)]

    def __setitem__(self, i, v):
        i = builtins.int(i)
        if i < 3:
            self.p[i] = v
        else:
            self.q[i - 3] = v

    def __len__(self):
        return 7

    def __iter__(self):
        return iter(self.components())

    def __mul__(self, o):
        if isinstance(o, Transform):
            return transform_multiply(self, o)
        return NotImplemented

    def __array__(self, dtype=None, copy=None):
        return np.array(self.components(), dtype=dtype or np.float32)

    def __repr__(self):
        return f"transform({self.components()})"


transform = Transform
transformf = Transform


# ----------------------------------------------------------------------------- structs
def struct(cls):
    """wp.struct: a value class whose fields start at the zero value of their declared type and
    convert on assignment."""
    ann = {}
    for klass in reversed(cls.__mro__):
        ann.update(getattr(klass, "__annotations__", {}))
    # string annotations (modules with `from __future__ import annotations`) are evaluated in the
    # defining module's namespace
    import sys as _sys

    g = vars(_sys.modules[cls.__module__]) if cls.__module__ in _sys.modules else {}
    fields = {}
    for k, t in ann.items():
        if isinstance(t, str):
            try:
                t = eval(t, dict(g))  # noqa: S307 - annotations of the reference's own source
            except Exception:
                pass
        fields[k] = t

    def _zero(t):
        t = _resolve(t)
        if t in (np.float32, np.float64, np.float16, Float32Cast, builtins.float):
            return np.float32(0) if t is not np.float64 else np.float64(0)
        if t in _INT_TYPES or t is builtins.int:
            return 0
        if t is builtins.bool:
            return False
        if isinstance(t, type) and issubclass(t, (_VecBase, Mat, Transform)):
            return t()
        if getattr(t, "_wp_struct", False):
            return t()
        if t is array:
            return array(None, shape=(0,))
        return None

    def _cast(t, v):
        t = _resolve(t)
        if v is None and t is not array:
            return None
        if t in (np.float32, Float32Cast, builtins.float):
            return np.float32(v)
        if t is np.float64:
            return np.float64(v)
        if t in _INT_TYPES:
            return t(builtins.int(v))
        if t is builtins.int:
            return builtins.int(v)
        if t is builtins.bool:
            return builtins.bool(v)
        if isinstance(t, type) and issubclass(t, (_VecBase, Mat)):
            return t(v)
        if t is Transform:
            return Transform(v)
        if t is array and v is None:
            return array(None, shape=(0,))  # a struct's unset array field is an empty array
        return v

    def __init__(self, **kw):
        for k, t in fields.items():
            object.__setattr__(self, k, _zero(t))
        for k, v in kw.items():
            setattr(self, k, v)

    def __setattr__(self, k, v):
        t = fields.get(k)
        object.__setattr__(self, k, _cast(t, v) if t is not None else v)

    ns = {"__init__": __init__, "__setattr__": __setattr__, "_wp_struct": True, "_fields": fields,
          "__doc__": cls.__doc__, "__module__": cls.__module__, "__qualname__": cls.__qualname__}
    for k, v in cls.__dict__.items():
        if k not in ("__dict__", "__weakref__", "__annotations__") and k not in ns:
            if not (k in fields and not callable(v)):
                ns[k] = v
    return type(cls.__name__, (), ns)


def _resolve(t):
    if isinstance(t, str):
        return {"float": np.float32, "int": builtins.int, "bool": builtins.bool}.get(t, t)
    if t is Float32Cast:
        return np.float32
    return t


# ----------------------------------------------------------------------------- arrays
class array:
    """Host array of Warp values.  Vector/matrix/transform elements are stored as trailing numpy
    dimensions of float32 (or int32) components; element reads return value copies."""

    def __class_getitem__(cls, item):
        return cls

    def __init__(self, data=None, dtype=np.float32, shape=None, device=None, requires_grad=False, copy=True,
                 ndim=None, ptr=None, **kw):
        dtype = _norm_dtype(dtype)
        self.dtype = dtype
        self.device = device
        self.requires_grad = requires_grad
        self.grad = None
        comp = _comp_shape(dtype)
        base = _base_dtype(dtype)
        if ptr is not None:
            # an array over existing memory (the reference aliases part of a local buffer this way)
            if isinstance(shape, (builtins.int, np.integer)):
                shape = (builtins.int(shape),)
            owner = ptr.owner.data
            item = np.dtype(base).itemsize * builtins.int(np.prod(comp)) if comp else np.dtype(base).itemsize
            if owner.dtype != np.dtype(base) or ptr.offset % item:
                raise NotImplementedError("pointer alias with a different element layout")
            flat = owner.reshape((-1,) + comp)
            start = ptr.offset // item
            n = builtins.int(np.prod(shape))
            self.data = flat[start:start + n].reshape(tuple(shape) + comp)
            return
        if data is None:
            if shape is None:
                shape = (0,)
            if isinstance(shape, (builtins.int, np.integer)):
                shape = (builtins.int(shape),)
            self.data = np.zeros(tuple(shape) + comp, dtype=base)
        else:
            if isinstance(data, array):
                data = data.data
            if isinstance(data, (list, tuple)) and data and isinstance(data[0], (Transform, _VecBase, Mat)):
                data = np.stack([np.asarray(x, dtype=base) for x in data])
            arr = np.array(data, dtype=base, copy=True)
            if comp and arr.shape[-len(comp):] != comp:
                arr = arr.reshape(arr.shape[:-1] + comp) if arr.ndim else arr
            self.data = arr
        self.grad = None

    @property
    def ptr(self):
        return _Ptr(self, 0)

    @property
    def shape(self):
        comp = _comp_shape(self.dtype)
        return self.data.shape[: self.data.ndim - len(comp)] if comp else self.data.shape

    @property
    def ndim(self):
        return len(self.shape)

    @property
    def size(self):
        return builtins.int(np.prod(self.shape))

    def __len__(self):
        return self.shape[0]

    def __bool__(self):
        # a null / empty array is falsy (Warp kernels test `if arr:` for a null array)
        return self.data.size > 0

    def _wrap(self, raw):
        dt = self.dtype
        if isinstance(dt, type) and issubclass(dt, Transform):
            return Transform(*[np.float32(x) for x in raw])
        if isinstance(dt, type) and issubclass(dt, _VecBase):
            return dt._make([dt._dtype(x) for x in raw])
        if isinstance(dt, type) and issubclass(dt, Mat):
            return dt._make([[np.float32(x) for x in r] for r in raw])
        return raw[()] if isinstance(raw, np.ndarray) else raw

    def _index(self, i):
        if isinstance(i, tuple):
            return tuple(builtins.int(k) for k in i)
        return builtins.int(i)

    def _view(self, data):
        v = array.__new__(array)
        v.dtype, v.device, v.requires_grad, v.grad = self.dtype, self.device, self.requires_grad, None
        v.data = data
        return v

    def __getitem__(self, i):
        if isinstance(i, slice):
            return self._view(self.data[i])  # a view: shares the elements, like a Warp array slice
        idx = self._index(i)
        nd = len(idx) if isinstance(idx, tuple) else 1
        if nd < self.ndim:
            return self._view(self.data[idx])
        return self._wrap(self.data[idx])

    def __setitem__(self, i, v):
        idx = self._index(i)
        base = self.data.dtype.type
        if isinstance(v, (Transform, _VecBase, Mat)):
            self.data[idx] = np.asarray(v, dtype=base)
        else:
            self.data[idx] = base(v)

    def numpy(self):
        return self.data

    def zero_(self):
        self.data[...] = 0

    def fill_(self, v):
        self.data[...] = np.asarray(v, dtype=self.data.dtype)

    def assign(self, src):
        self.data[...] = src.data if isinstance(src, array) else np.asarray(src, dtype=self.data.dtype)

    def flatten(self):
        return self

    def __repr__(self):
        return f"array(shape={self.shape}, dtype={getattr(self.dtype, '__name__', self.dtype)})"


array1d = array2d = array3d = array4d = indexedarray = array


class _Ptr:
    """Address of an emulated array's first element plus a byte offset (``arr.ptr + k``)."""

    def __init__(self, owner, offset):
        self.owner, self.offset = owner, builtins.int(offset)

    def __add__(self, k):
        return _Ptr(self.owner, self.offset + builtins.int(k))

    __radd__ = __add__


def _norm_dtype(dt):
    if dt in (builtins.float, Float32Cast):
        return np.float32
    if dt is builtins.int:
        return np.int32
    if dt is builtins.bool:
        return np.bool_
    return dt


def _comp_shape(dt):
    if isinstance(dt, type):
        if issubclass(dt, Transform):
            return (7,)
        if issubclass(dt, _VecBase):
            return (dt._n,)
        if issubclass(dt, Mat):
            return (dt._rows, dt._cols)
    return ()


def _base_dtype(dt):
    if isinstance(dt, type):
        if issubclass(dt, Transform) or issubclass(dt, Mat):
            return np.float32
        if issubclass(dt, _VecBase):
            return dt._dtype
    return dt


def zeros(shape, dtype=np.float32, device=None, requires_grad=False, **kw):
    return array(None, dtype=dtype, shape=shape, device=device, requires_grad=requires_grad)


def empty(shape, dtype=np.float32, device=None, requires_grad=False, **kw):
    return zeros(shape, dtype=dtype)


def full(shape, value, dtype=np.float32, device=None, **kw):
    a = zeros(shape, dtype=dtype)
    a.fill_(value)
    return a


def zeros_like(a, **kw):
    return zeros(a.shape, dtype=a.dtype)


def empty_like(a, **kw):
    return zeros(a.shape, dtype=a.dtype)


def clone(a, **kw):
    return array(a.data.copy(), dtype=a.dtype)


def copy(dest, src, **kw):
    dest.data[...] = src.data


def from_numpy(arr, dtype=np.float32, **kw):
    return array(arr, dtype=dtype)


# ----------------------------------------------------------------------------- kernels
_tid_stack: list = []


def tid():
    return _tid_stack[-1]


class Kernel:
    def __init__(self, func, **options):
        self.func = func
        self.key = func.__name__
        self.options = options

    def __call__(self, *a, **k):
        return self.func(*a, **k)


def kernel(f=None, **options):
    if f is None:
        return lambda g: Kernel(g, **options)
    return Kernel(f)


def func(f=None, **options):
    if f is None:
        return lambda g: g
    return f


def func_native(*a, **k):
    raise NotImplementedError("native functions are not emulated")


def overload(kernel, *a, **k):
    return kernel


# Thread order of emulated launches: None runs threads in index order; a callable n -> permutation
# of range(n) runs a 1-D launch's threads in that order instead (a device leaves the order of its
# threads, and so of their atomic updates, unspecified).
launch_order = None


def launch(kernel, dim, inputs=(), outputs=(), device=None, stream=None, record_tape=True, block_dim=None,
           max_blocks=None, **kw):
    args = list(inputs) + list(outputs)
    if isinstance(dim, (tuple, list)) and len(dim) == 1:
        dim = dim[0]
    if isinstance(dim, (tuple, list)):
        dims = [builtins.int(d) for d in dim]
        ranges = np.ndindex(*dims)
    else:
        n = builtins.int(dim)
        ranges = range(n) if launch_order is None else [builtins.int(t) for t in launch_order(n)]
    f = kernel.func if isinstance(kernel, Kernel) else kernel
    for t in ranges:
        _tid_stack.append(t if isinstance(t, builtins.int) else tuple(builtins.int(x) for x in t))
        try:
            f(*args)
        finally:
            _tid_stack.pop()


def static(x):
    # a float evaluated at code-generation time becomes an fp32 constant of the kernel
    return np.float32(x) if isinstance(x, builtins.float) else x


def constant(x):
    return x


def synchronize(*a, **k):
    pass


def synchronize_device(*a, **k):
    pass


class _CpuDevice:
    is_cpu = True
    is_cuda = False
    alias = "cpu"
    ordinal = -1

    def __str__(self):
        return "cpu"

    def __eq__(self, o):
        return str(o) == "cpu"

    def __hash__(self):
        return hash("cpu")


_CPU = _CpuDevice()


def get_device(*a, **k):
    return _CPU


def get_preferred_device():
    return _CPU


def get_cuda_device_count():
    return 0


def is_cuda_available():
    return False


class ScopedDevice(contextlib.nullcontext):
    def __init__(self, *a, **k):
        super().__init__()


class ScopedTimer(contextlib.nullcontext):
    def __init__(self, *a, **k):
        super().__init__()


class ScopedStream(contextlib.nullcontext):
    def __init__(self, *a, **k):
        super().__init__()


def set_module_options(*a, **k):
    pass


def printf(*a, **k):
    pass


def expect_eq(a, b):
    assert a == b


# ----------------------------------------------------------------------------- atomics
def _atomic(arr, idx, val, op):
    old = arr[idx]
    arr[idx] = op(old, val)
    return old


def atomic_add(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    return _atomic(arr, idx, val, lambda a, b: a + b)


def atomic_sub(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    return _atomic(arr, idx, val, lambda a, b: a - b)


def atomic_min(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    return _atomic(arr, idx, val, lambda a, b: min(a, b))


def atomic_max(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    return _atomic(arr, idx, val, lambda a, b: max(a, b))


def atomic_cas(arr, *args):
    *idx, compare, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    old = arr[idx]
    if old == compare:
        arr[idx] = val
    return old


def atomic_exch(arr, *args):
    *idx, val = args
    idx = tuple(idx) if len(idx) > 1 else idx[0]
    old = arr[idx]
    arr[idx] = val
    return old


# ----------------------------------------------------------------------------- builtins
def _f32(x):
    """Python float -> float32 (a float literal in a kernel is fp32); integers stay integers."""
    return np.float32(x) if isinstance(x, builtins.float) else x


def _map(f, *xs):
    v = next((x for x in xs if isinstance(x, (_VecBase, Mat))), None)
    if v is None:
        return f(*xs)
    if isinstance(v, Mat):
        return type(v)._make([[f(*[x.m[i][j] if isinstance(x, Mat) else x for x in xs])
                               for j in range(v._cols)] for i in range(v._rows)])
    return type(v)._make([f(*[x.c[i] if isinstance(x, _VecBase) else x for x in xs]) for i in range(v._n)])


def dot(a, b):
    if isinstance(a, _VecBase):
        s = a.c[0] * b.c[0]
        for i in range(1, a._n):
            s = s + a.c[i] * b.c[i]
        return s
    return a * b


def cross(a, b):
    ax, ay, az = a.c
    bx, by, bz = b.c
    return type(a)._make([ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx])


def length_sq(a):
    return dot(a, a)


def length(a):
    return np.sqrt(dot(a, a))


def normalize(a):
    if isinstance(a, quat):
        l_ = np.sqrt(dot(a, a))
        if l_ > np.float32(0.0):
            return quat._make([c / l_ for c in a.c])
        return quat()
    l_ = length(a)
    if l_ > np.float32(0.0):
        return type(a)._make([c / l_ for c in a.c])
    return type(a)()


def cw_mul(a, b):
    return _map(lambda x, y: x * y, a, b)


def cw_div(a, b):
    return _map(lambda x, y: x / y, a, b)


def _min2(a, b):
    return a if a < b else b


def _max2(a, b):
    return a if a > b else b


def min(a, b=None):  # noqa: A001
    # Warp: a < b ? a : b
    if b is None:
        return builtins.min(a.c)
    return _map(lambda x, y: _f32(x) if x < y else _f32(y), a, b)


def max(a, b=None):  # noqa: A001
    # Warp: a > b ? a : b
    if b is None:
        return builtins.max(a.c)
    return _map(lambda x, y: _f32(x) if x > y else _f32(y), a, b)


def abs(a):  # noqa: A001
    return _map(lambda x: builtins.abs(_f32(x)), a)


def sign(a):
    return _map(lambda x: np.float32(-1.0) if x < 0 else np.float32(1.0), a)


def clamp(x, lo, hi):
    # Warp: min(max(a, lo), hi)
    return _map(lambda v, a, b: _f32(min(max(v, a), b)), x, lo, hi)


def where(cond, a, b):
    return a if cond else b


def select(cond, value_if_false, value_if_true):
    return value_if_true if cond else value_if_false


def sqrt(x):
    return np.sqrt(_f32(x))


def sin(x):
    return np.sin(_f32(x))


def cos(x):
    return np.cos(_f32(x))


def tan(x):
    return np.tan(_f32(x))


def asin(x):
    return np.arcsin(_f32(x))


def acos(x):
    return np.arccos(_f32(x))


def atan(x):
    return np.arctan(_f32(x))


def atan2(y, x):
    return np.arctan2(_f32(y), _f32(x))


def exp(x):
    return np.exp(_f32(x))


def log(x):
    return np.log(_f32(x))


def pow(x, y):  # noqa: A001
    return np.power(_f32(x), _f32(y))


def floor(x):
    return np.floor(_f32(x))


def ceil(x):
    return np.ceil(_f32(x))


def round(x):  # noqa: A001
    return np.round(_f32(x))


def mod(a, b):
    return np.fmod(a, b)


def isnan(x):
    return builtins.bool(np.isnan(x))


def isinf(x):
    return builtins.bool(np.isinf(x))


def isfinite(x):
    if isinstance(x, (_VecBase,)):
        return builtins.all(np.isfinite(c) for c in x.c)
    return builtins.bool(np.isfinite(x))


def step(x):
    return np.float32(0.0) if x >= 0 else np.float32(1.0)


def nonzero(x):
    return np.float32(1.0) if x != 0 else np.float32(0.0)


def degrees(x):
    return _f32(x) * np.float32(180.0 / _math.pi)


def radians(x):
    return _f32(x) * np.float32(_math.pi / 180.0)


def lerp(a, b, t):
    return a * (np.float32(1.0) - t) + b * t


def outer(a, b):
    return matrix((a._n, b._n))._make([[x * y for y in b.c] for x in a.c])


def transpose(m):
    return matrix((m._cols, m._rows), m._dtype)._make([[m.m[i][j] for i in range(m._rows)] for j in range(m._cols)])


def determinant(m):
    a = m.m
    if m._rows == 2:
        return a[0][0] * a[1][1] - a[0][1] * a[1][0]
    return (a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2])
            - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
            + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]))


def inverse(m):
    inv = np.linalg.inv(np.asarray(m, dtype=np.float64)).astype(np.float32)
    return type(m)._make(inv.tolist())


def diag(v):
    n = v._n
    return matrix((n, n))._make([[v.c[i] if i == j else np.float32(0) for j in range(n)] for i in range(n)])


def identity(n=3, dtype=np.float32):
    return matrix((n, n))._make([[np.float32(1 if i == j else 0) for j in range(n)] for i in range(n)])


def skew(v):
    x, y, z = v.c
    z0 = np.float32(0)
    return mat33._make([[z0, -z, y], [z, z0, -x], [-y, x, z0]])


def trace(m):
    s = m.m[0][0]
    for i in range(1, m._rows):
        s = s + m.m[i][i]
    return s


def matrix_from_rows(*rows):
    return matrix((len(rows), rows[0]._n))._make([list(r.c) for r in rows])


def matrix_from_cols(*cols):
    R = cols[0]._n
    return matrix((R, len(cols)))._make([[c.c[i] for c in cols] for i in range(R)])


def mul(a, b):
    if _is_scalar(a) or _is_scalar(b):
        return a * b
    if isinstance(a, quat) and isinstance(b, quat):
        return _qmul(a, b)
    if isinstance(a, Transform) and isinstance(b, Transform):
        return transform_multiply(a, b)
    return a @ b


def add(a, b):
    return a + b


def sub(a, b):
    return a - b


def div(a, b):
    return a / b


def neg(a):
    return -a


# quaternions ---------------------------------------------------------------
def quat_identity(dtype=None):
    return quat()


def quat_inverse(q):
    return quat._make([-q.c[0], -q.c[1], -q.c[2], q.c[3]])


def quat_rotate(q, x):
    qx, qy, qz, qw = q.c
    vx, vy, vz = x.c
    two = np.float32(2.0)
    c = two * qw * qw - np.float32(1.0)
    d = two * (qx * vx + qy * vy + qz * vz)
    return vec3._make([vx * c + qx * d + (qy * vz - qz * vy) * qw * two,
                       vy * c + qy * d + (qz * vx - qx * vz) * qw * two,
                       vz * c + qz * d + (qx * vy - qy * vx) * qw * two])


def quat_rotate_inv(q, x):
    qx, qy, qz, qw = q.c
    vx, vy, vz = x.c
    two = np.float32(2.0)
    c = two * qw * qw - np.float32(1.0)
    d = two * (qx * vx + qy * vy + qz * vz)
    return vec3._make([vx * c + qx * d - (qy * vz - qz * vy) * qw * two,
                       vy * c + qy * d - (qz * vx - qx * vz) * qw * two,
                       vz * c + qz * d - (qx * vy - qy * vx) * qw * two])


def quat_to_matrix(q):
    c0 = quat_rotate(q, vec3(1.0, 0.0, 0.0))
    c1 = quat_rotate(q, vec3(0.0, 1.0, 0.0))
    c2 = quat_rotate(q, vec3(0.0, 0.0, 1.0))
    return matrix_from_cols(c0, c1, c2)


def quat_from_axis_angle(axis, angle):
    half = _f32(angle) * np.float32(0.5)
    w = np.cos(half)
    s = np.sin(half)
    return quat._make([axis.c[0] * s, axis.c[1] * s, axis.c[2] * s, w])


def quat_to_axis_angle(q):
    raise NotImplementedError


def quat_between_vectors(a, b):
    raise NotImplementedError


def quat_from_matrix(m):
    raise NotImplementedError


# transforms ------------------------------------------------------------------
def transform_identity(dtype=None):
    return Transform()


def transform_get_translation(t):
    return vec3(t.p)


def transform_get_rotation(t):
    return quat(t.q)


def transform_point(t, x):
    if isinstance(t, Mat):
        raise NotImplementedError
    return quat_rotate(t.q, x) + t.p


def transform_vector(t, x):
    return quat_rotate(t.q, x)


def transform_multiply(a, b):
    return Transform(quat_rotate(a.q, b.p) + a.p, _qmul(a.q, b.q))


def transform_inverse(t):
    qi = quat_inverse(t.q)
    return Transform(-quat_rotate(qi, t.p), qi)


# spatial vectors ----------------------------------------------------------------
def spatial_top(a):
    return vec3._make(a.c[0:3])


def spatial_bottom(a):
    return vec3._make(a.c[3:6])


def spatial_cross(a, b):
    raise NotImplementedError


def spatial_dot(a, b):
    return dot(a, b)


def velocity_at_point(qd, r):
    return cross(spatial_bottom(qd), r) + spatial_top(qd)


# ----------------------------------------------------------------------------- the `types` namespace
types = _pytypes.SimpleNamespace(
    vector=vector, matrix=matrix, float32=np.float32, float64=np.float64, int32=np.int32, int64=np.int64,
    uint32=np.uint32, uint64=np.uint64, int8=np.int8, uint8=np.uint8, int16=np.int16, uint16=np.uint16,
    array=array, transform=Transform, quaternion=lambda dtype=np.float32: quat,
    type_is_vector=lambda t: isinstance(t, type) and issubclass(t, _VecBase),
    type_is_matrix=lambda t: isinstance(t, type) and issubclass(t, Mat),
    type_is_transformation=lambda t: t is Transform,
    type_is_quaternion=lambda t: t is quat,
    types_equal=lambda a, b, **k: a is b,
    float_types=(np.float16, np.float32, np.float64),
    int_types=_INT_TYPES,
    scalar_types=(np.float16, np.float32, np.float64) + _INT_TYPES,
    Array=array,
    Any=object,
)
transformation = lambda *a, **k: Transform  # noqa: E731
config = _pytypes.SimpleNamespace(mode="release", verify_cuda=False, verbose=False, quiet=True,
                                  enable_backward=False)
context = _pytypes.SimpleNamespace()


class Tape:  # not emulated (the reference's gradients are not part of these fixtures)
    def __init__(self, *a, **k):
        raise NotImplementedError("wp.Tape is not emulated")


def __getattr__(name):
    """Any other Warp attribute a reference module touches at import time (for code outside the
    emulated path) resolves to a placeholder that fails if it is ever called."""

    def _missing(*a, **k):
        raise NotImplementedError(f"warp.{name} is not emulated")

    _missing.__name__ = name
    return _missing
