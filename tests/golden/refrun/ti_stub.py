"""A plain-Python stand-in for the part of Taichi that the reference's SPH/main.py uses,
so that the reference's own kernels can run (slowly, on the CPU, one particle at a
time) where Taichi is not installed. TEST INFRASTRUCTURE: only the
scripts tests/golden/make_reference_*.py load it, to generate golden fixtures.

Semantics kept from Taichi where the reference depends on them:
  - fields are arrays of their dtype (float: f32, int: i32); reading an element gives
    a value (a copy), writing stores it; `for i in field` and ti.grouped(field) visit
    every index; under a pointer or dynamic SNode a field is stored per leaf block,
    which its first write activates, and struct-fors visit the active blocks (bitmasked
    SNodes are dense: the reference only reads their written elements);
  - vectors and matrices are value types (`Vec`, a numpy array with Taichi's methods);
    with numpy's promotion rules, f32 values combined with Python floats stay f32;
  - ti.func calls are inlined in Taichi, so a `ti.template()` argument is passed by
    reference; make_reference_run.py rewrites the reference's source for the cases
    that depend on it (neighbour tasks, writes into field elements, atomics).
"""
from __future__ import annotations

import builtins
import itertools
import types as _types

import numpy as np

f32, f64, i32, i64, u8 = np.float32, np.float64, np.int32, np.int64, np.uint8
cpu = gpu = cuda = vulkan = "arch"
ijk, ij, i, j, k, l = "ijk", "ij", "i", "j", "k", "l"


def _dt(dtype):
    if dtype is None or dtype is float:
        return np.float32
    if dtype is int:
        return np.int32
    return np.dtype(dtype).type


def init(*a, **kw):
    pass


def kernel(f):
    return f


def func(f):
    return f


def data_oriented(c):
    return c


def template():
    return None


def static(x):
    return x


class Vec(np.ndarray):
    """Taichi vector / matrix value."""

    def norm(self):
        return np.sqrt(np.sum(self * self))

    def norm_sqr(self):
        return np.sum(self * self)

    def dot(self, o):
        return np.sum(self * o)

    def outer_product(self, o):
        return np.outer(self, o).view(Vec)

    def cross(self, o):
        return np.cross(self, o).view(Vec)

    def determinant(self):
        return self.dtype.type(np.linalg.det(np.asarray(self, np.float64)))

    def inverse(self):
        return np.linalg.inv(np.asarray(self, np.float64)).astype(self.dtype).view(Vec)

    def transpose(self):
        return np.ascontiguousarray(np.asarray(self).T).view(Vec)

    def trace(self):
        return np.trace(np.asarray(self))

    def normalized(self):
        return self / self.norm()

    def cast(self, dtype):
        return np.asarray(self).astype(_dt(dtype)).view(Vec)

    def sum(self, *a, **kw):
        return np.sum(np.asarray(self), *a, **kw)

    def max(self, *a, **kw):
        return np.max(np.asarray(self), *a, **kw)

    def min(self, *a, **kw):
        return np.min(np.asarray(self), *a, **kw)

    def to_numpy(self):
        return np.asarray(self).copy()


def _vec(vals, dt=None):
    a = np.asarray(vals)
    if dt is None:
        dt = np.float32 if a.dtype.kind == "f" else np.int32 if a.dtype.kind in "iub" else a.dtype.type
    return np.array(a, dtype=_dt(dt)).view(Vec)


def _index(key):
    """Field index: ints, numpy ints, Vec indices and tuples of those, flattened."""
    if key is None:
        return ()
    if not isinstance(key, tuple):
        key = (key,)
    out = []
    for kk in key:
        if isinstance(kk, np.ndarray):
            out.extend(int(v) for v in np.asarray(kk).reshape(-1))
        else:
            out.append(int(kk))
    return tuple(out)


class Field:
    """A Taichi field. Placed under a pointer or dynamic SNode it is sparse: storage per
    leaf block (the dense levels below the last pointer), created by the first write into
    it (`+= 0` included); reads elsewhere give 0; `for I in field` visits every cell of
    the active blocks. Otherwise it is one dense array."""

    def __init__(self, dtype, shape=None, elem=()):
        self.dtype = _dt(dtype)
        self.elem = tuple(elem)
        self.data = None
        self.sparse = False
        self.snode = None
        if shape is not None:
            self._alloc(shape)

    def _alloc(self, shape):
        shape = (shape,) if np.isscalar(shape) else tuple(int(s) for s in shape)
        self.shape = shape
        self.data = np.zeros(shape + self.elem, self.dtype)

    def _bind_sparse(self, shape, block):
        self.shape, self.block, self.sparse = tuple(shape), tuple(block), True
        self.blocks = {}

    def parent(self):
        return self.snode

    def _where(self, idx):
        return (tuple(v // b for v, b in zip(idx, self.block)), tuple(v % b for v, b in zip(idx, self.block)))

    def __getitem__(self, key):
        idx = _index(key)
        if self.sparse:
            bk, loc = self._where(idx)
            blk = self.blocks.get(bk)
            v = np.zeros(self.elem, self.dtype) if blk is None else blk[loc]
        else:
            v = self.data[idx]
        if self.elem:
            return np.array(v).view(Vec)
        return self.dtype(v)

    def __setitem__(self, key, val):
        idx = _index(key)
        if self.sparse:
            bk, loc = self._where(idx)
            blk = self.blocks.get(bk)
            if blk is None:
                blk = self.blocks[bk] = np.zeros(self.block + self.elem, self.dtype)
            blk[loc] = np.asarray(val)
        else:
            self.data[idx] = np.asarray(val)

    def __iter__(self):
        if self.sparse:
            def cells():
                for bk in sorted(self.blocks):
                    base = [b * e for b, e in zip(bk, self.block)]
                    for loc in itertools.product(*[range(e) for e in self.block]):
                        yield tuple(b + l_ for b, l_ in zip(base, loc))
            return cells()
        if len(self.shape) == 1:
            return iter(range(self.shape[0]))
        return itertools.product(*[range(s) for s in self.shape])

    def _clear(self):
        if self.sparse:
            self.blocks = {}
            self.lengths = {}
        else:
            self.data[...] = 0

    def fill(self, v):
        if self.sparse:
            for blk in self.blocks.values():
                blk[...] = np.asarray(v)
        else:
            self.data[...] = np.asarray(v)

    def to_numpy(self):
        return self.data.copy()

    def from_numpy(self, a):
        self.data[...] = np.asarray(a).astype(self.dtype)

    def copy_from(self, other):
        self.data[...] = other.data


def field(dtype=float, shape=None, **kw):
    return Field(dtype, shape)


class _VectorType:
    def __call__(self, vals, dt=None):
        return _vec(vals, dt)

    def field(self, n, dtype=float, shape=None, **kw):
        return Field(dtype, shape, (n,))


class _MatrixType:
    def __call__(self, vals, dt=None):
        return _vec(vals, dt)

    def field(self, n, m, dtype=float, shape=None, **kw):
        return Field(dtype, shape, (n, m))

    def identity(self, dt, n):
        return np.eye(n, dtype=_dt(dt)).view(Vec)

    def zero(self, dt, n, m):
        return np.zeros((n, m), _dt(dt)).view(Vec)


Vector = _VectorType()
Matrix = _MatrixType()


def _vector_of(n, dt=float):
    def make(*vals):
        if len(vals) == 1 and np.isscalar(vals[0]):
            return np.full(n, vals[0], _dt(dt)).view(Vec)
        flat = np.concatenate([np.atleast_1d(np.asarray(v)) for v in vals])
        return flat.astype(_dt(dt)).view(Vec)
    return make


def _matrix_of(n, m, dt=float):
    def make(*vals):
        if len(vals) == 1 and np.isscalar(vals[0]):
            return np.full((n, m), vals[0], _dt(dt)).view(Vec)
        return np.asarray(vals if len(vals) > 1 else vals[0], _dt(dt)).reshape(n, m).view(Vec)
    return make


math = _types.SimpleNamespace(
    vec2=_vector_of(2), vec3=_vector_of(3), vec4=_vector_of(4), ivec3=_vector_of(3, int),
    mat2=_matrix_of(2, 2), mat3=_matrix_of(3, 3),
    eye=lambda n: np.eye(n, dtype=np.float32).view(Vec), pi=np.pi)
types = _types.SimpleNamespace(vector=lambda n, dt=float: _vector_of(n, dt),
                               matrix=lambda n, m, dt=float: _matrix_of(n, m, dt), ndarray=lambda *a, **kw: None)


def Struct(**kw):
    return _types.SimpleNamespace(**kw)


def ndrange(*args):
    rs = [range(a[0], a[1]) if isinstance(a, tuple) else range(a) for a in args]
    return list(itertools.product(*rs))


def grouped(x):
    if isinstance(x, Field):
        if len(x.shape) == 1:
            return range(x.shape[0])
        return (_vec(t, int) for t in itertools.product(*[range(s) for s in x.shape]))
    return (_vec(t, int) for t in x)


def cast(x, dt):
    if isinstance(x, np.ndarray):
        return np.asarray(x).astype(_dt(dt)).view(Vec)
    return _dt(dt)(x)


def pow(a, b):  # noqa: A001 - Taichi's name
    return np.power(a, b)


sqrt, abs, exp, log, floor, sin, cos = np.sqrt, np.abs, np.exp, np.log, np.floor, np.sin, np.cos


def max(*a):  # noqa: A001
    return np.maximum.reduce([np.asarray(v) for v in a]) if len(a) > 1 else np.max(a[0])


def min(*a):  # noqa: A001
    return np.minimum.reduce([np.asarray(v) for v in a]) if len(a) > 1 else np.min(a[0])


def polar_decompose(F, dt=None):
    """F = R S with R a rotation (det +1) and S symmetric, through the SVD."""
    A = np.asarray(F, np.float64)
    U, s, Vt = np.linalg.svd(A)
    if np.linalg.det(U) < 0:
        U[:, -1] *= -1
        s[-1] *= -1
    if np.linalg.det(Vt) < 0:
        Vt[-1] *= -1
        s[-1] *= -1
    R = U @ Vt
    S = Vt.T @ np.diag(s) @ Vt
    t = np.asarray(F).dtype
    return R.astype(t).view(Vec), S.astype(t).view(Vec)


def is_active(*a):
    return True


class SNode:
    """A level of an SNode tree: `kind` (root, dense, pointer, bitmasked, dynamic) over
    `axes` ("ijk" or one letter) with `dims` cells per axis."""

    def __init__(self, kind="root", axes="", dims=(), parent=None):
        self.kind, self.axes, self.parent_node = kind, axes, parent
        dims = [dims] * len(axes) if np.isscalar(dims) else [int(d) for d in np.asarray(dims).reshape(-1)]
        self.dims = dims
        self.children, self.fields = [], []

    def _child(self, kind, axes, dims, *a, **kw):
        c = SNode(kind, axes, dims, self)
        self.children.append(c)
        return c

    def dense(self, axes, dims):
        return self._child("dense", axes, dims)

    def pointer(self, axes, dims):
        return self._child("pointer", axes, dims)

    def bitmasked(self, axes, dims):
        return self._child("bitmasked", axes, dims)

    def dynamic(self, axes, n, chunk_size=None):
        return self._child("dynamic", axes, n)

    def _chain(self):
        c, n = [], self
        while n is not None and n.kind != "root":
            c.append(n)
            n = n.parent_node
        return c[::-1]

    def place(self, *fs):
        chain = self._chain()
        order = []
        for lv in chain:
            for ax in lv.axes:
                if ax not in order:
                    order.append(ax)
        shape = {ax: 1 for ax in order}
        block = {ax: 1 for ax in order}
        last_ptr = builtins.max([n for n, lv in enumerate(chain) if lv.kind in ("pointer", "dynamic")], default=-1)
        for n, lv in enumerate(chain):
            for ax, d in zip(lv.axes, lv.dims):
                shape[ax] *= d
                if n > last_ptr or lv.kind == "dynamic":
                    block[ax] *= d
        for f in fs:
            f.snode = self
            if last_ptr >= 0:
                f._bind_sparse([shape[a] for a in order], [block[a] for a in order])
            else:
                f._alloc([shape[a] for a in order])
            self.fields.append(f)
        return self

    def deactivate_all(self):
        for f in self.fields:
            f._clear()
        for c in self.children:
            c.deactivate_all()


root = SNode()


class _Linalg:
    def LinearOperator(self, *a, **kw):
        raise NotImplementedError("ti.linalg is not part of this stand-in")

    MatrixFreeCG = LinearOperator


linalg = _Linalg()
ui = _types.SimpleNamespace()


# helpers the source rewrite calls -------------------------------------------------------
def _atomic(fld, key, v, op):
    old = fld[key]
    fld[key] = old + v if op == "add" else np.maximum(old, v) if op == "max" else np.minimum(old, v)
    return old


def _setcomp(obj, key, comp, v):
    """obj[key][comp] = v, through to the field when obj is one."""
    if isinstance(obj, Field):
        e = obj[key]
        e[comp] = v
        obj[key] = e
    else:
        obj[key][comp] = v


def _fill_elem(obj, key, v):
    if isinstance(obj, Field):
        e = obj[key]
        e[...] = v
        obj[key] = e
    else:
        obj[key].fill(v)


def _copy(v):
    return v.copy() if isinstance(v, np.ndarray) else v


def _all(x):
    return bool(np.all(np.asarray(x)))


def _any(x):
    return bool(np.any(np.asarray(x)))


def append(node, idx, v):
    """ti.append on a dynamic SNode: the next slot of the list at cell `idx`."""
    f = node.fields[0]
    key = _index(idx)
    lens = f.__dict__.setdefault("lengths", {})
    n = lens.get(key, 0)
    f[key + (n,)] = v
    lens[key] = n + 1
    return n


def length(node, idx):
    return node.fields[0].__dict__.get("lengths", {}).get(_index(idx), 0)


def svd(A, dt=None):
    """A = U diag(s) V^T, singular values in descending order, as Taichi's 3x3 SVD."""
    U, sv, Vt = np.linalg.svd(np.asarray(A, np.float64))
    t = np.asarray(A).dtype
    return U.astype(t).view(Vec), np.diag(sv).astype(t).view(Vec), Vt.T.astype(t).view(Vec)


_np_ceil = np.ceil


def ceil(x, dtype=None):
    return _np_ceil(x) if dtype is None else _dt(dtype)(_np_ceil(x))


def loop_config(*a, **kw):
    pass


tools = _types.SimpleNamespace(PLYWriter=None)
