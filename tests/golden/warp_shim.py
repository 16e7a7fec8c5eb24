"""A minimal numpy stand-in for the Warp builtins used by the reference VBD kernels.

Test infrastructure only. It lets ``make_golden.py`` execute the reference's own
``@wp.func`` / ``@wp.kernel`` bodies (from ``newton/_src/solvers/vbd/particle_vbd_kernels.py``
and ``rigid_vbd_kernels.py``) in plain Python, in float64, so that golden vectors come
from the reference's code rather than from a restatement of it. Warp itself
(``warp-lang==1.14.0rc2``, ``uv.lock:6813-6815`` of the reference) is not installed here.

Only the subset of Warp semantics that those kernels touch is provided:

* ``vec3`` / ``mat22`` / ``mat33`` values with Warp operator meaning (``mat * vec`` is a
  matrix-vector product, ``mat * mat`` a matrix product, ``vec * scalar`` scaling);
* builtins ``dot cross length normalize outer skew transpose determinant inverse identity
  atan2 sqrt max min abs sign`` with Warp's definitions (``sign(0) == 1``, ``normalize(0) == 0``);
* rigid transforms as ``(p, q)`` with ``q = (x, y, z, w)``;
* arrays indexed by ``a[i]`` / ``a[i, j]`` and truthy when non-empty (Warp tests the pointer);
* ``tid()`` driven by the launcher below, ``atomic_add`` / ``atomic_min`` as plain read-modify-writes;
* ``closest_point_edge_edge``: Warp implements it natively (not in the reference tree). Here it is
  restated from the published segment-segment closest-point method (C. Ericson, *Real-Time Collision
  Detection*, 2005, sec. 5.1.9) with ``epsilon`` as the degenerate-segment threshold on squared lengths;
* ``bvh_query_aabb``: a brute-force query that yields every primitive whose box overlaps the query box,
  in index order (the set a BVH returns; Warp's traversal order is not reproduced). ``make_golden.py``
  rewrites ``while wp.bvh_query_next(query, i):`` loops into ``for i in query:``.
"""

from __future__ import annotations

import math

import numpy as np

DTYPE = np.float64

inf = math.inf
float32 = float
int32 = int
bool = bool  # noqa: A001 - ``wp.bool``


class Vec:
    __slots__ = ("a",)

    def __init__(self, a):
        self.a = np.asarray(a, dtype=DTYPE).copy()

    def __add__(self, o):
        return Vec(self.a + o.a)

    def __sub__(self, o):
        return Vec(self.a - o.a)

    def __neg__(self):
        return Vec(-self.a)

    def __mul__(self, s):
        if isinstance(s, (Vec, Mat)):
            raise TypeError("vec * vec/mat is not a Warp operation")
        return Vec(self.a * s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return Vec(self.a / s)

    def __getitem__(self, i):
        return float(self.a[i])

    def __setitem__(self, i, x):
        self.a[i] = x

    def __len__(self):
        return len(self.a)

    def __array__(self, dtype=None, copy=None):
        return self.a if dtype is None else self.a.astype(dtype)

    def __repr__(self):
        return f"Vec({self.a.tolist()})"


class Mat:
    __slots__ = ("a",)

    def __init__(self, a):
        self.a = np.asarray(a, dtype=DTYPE).copy()

    def __add__(self, o):
        return Mat(self.a + o.a)

    def __sub__(self, o):
        return Mat(self.a - o.a)

    def __neg__(self):
        return Mat(-self.a)

    def __mul__(self, o):
        if isinstance(o, Mat):
            return Mat(self.a @ o.a)
        if isinstance(o, Vec):
            return Vec(self.a @ o.a)
        return Mat(self.a * o)

    def __rmul__(self, s):
        if isinstance(s, (Vec, Mat)):
            raise TypeError("unsupported")
        return Mat(self.a * s)

    def __truediv__(self, s):
        return Mat(self.a / s)

    def __getitem__(self, ij):
        return float(self.a[ij])

    def __setitem__(self, ij, x):
        self.a[ij] = x

    def __array__(self, dtype=None, copy=None):
        return self.a if dtype is None else self.a.astype(dtype)

    def __repr__(self):
        return f"Mat({self.a.tolist()})"


def _vec_ctor(n):
    def ctor(*args):
        if len(args) == 0:
            return Vec(np.zeros(n))
        if len(args) == 1:
            x = args[0]
            if isinstance(x, Vec):
                return Vec(x.a)
            if np.isscalar(x):
                return Vec(np.full(n, float(x)))
            return Vec(np.asarray(x, dtype=DTYPE).reshape(n))
        assert len(args) == n
        return Vec(np.array([float(x) for x in args]))

    return ctor


def _mat_ctor(r, c):
    def ctor(*args):
        if len(args) == 0:
            return Mat(np.zeros((r, c)))
        if len(args) == 1:
            x = args[0]
            if isinstance(x, Mat):
                return Mat(x.a)
            if np.isscalar(x):
                return Mat(np.full((r, c), float(x)))
            return Mat(np.asarray(x, dtype=DTYPE).reshape(r, c))
        assert len(args) == r * c, "only the scalar-list matrix constructor is supported"
        return Mat(np.array([float(x) for x in args]).reshape(r, c))

    return ctor


vec3 = _vec_ctor(3)
vec2 = _vec_ctor(2)
vec4 = _vec_ctor(4)
mat22 = _mat_ctor(2, 2)
mat33 = _mat_ctor(3, 3)
mat32 = _mat_ctor(3, 2)
uint64 = int


def vector(*args, length=None, dtype=None):
    """``wp.vector(..., length=n, dtype=wp.bool)``: a plain list of the values."""
    return list(args)


def spatial_vector(*args):
    return _vec_ctor(6)(*args)


def spatial_top(v):
    return Vec(v.a[:3])


def spatial_bottom(v):
    return Vec(v.a[3:])


def matrix_from_cols(*cols):
    return Mat(np.stack([c.a for c in cols], axis=1))


def dot(a, b):
    return float(np.dot(a.a, b.a))


def cross(a, b):
    return Vec(np.cross(a.a, b.a))


def length(a):
    return float(np.sqrt(np.dot(a.a, a.a)))


def length_sq(a):
    return float(np.dot(a.a, a.a))


def normalize(a):
    n = length(a)
    return Vec(a.a / n) if n > 0.0 else Vec(np.zeros_like(a.a))


def outer(a, b):
    return Mat(np.outer(a.a, b.a))


def skew(a):
    x, y, z = a.a
    return Mat(np.array([[0.0, -z, y], [z, 0.0, -x], [-y, x, 0.0]]))


def transpose(m):
    return Mat(m.a.T)


def determinant(m):
    return float(np.linalg.det(m.a))


def inverse(m):
    return Mat(np.linalg.inv(m.a))


def identity(n=3, dtype=float):
    return Mat(np.eye(n))


def atan2(y, x):
    return math.atan2(y, x)


def sqrt(x):
    return math.sqrt(x)


def max(a, b=None):  # noqa: A001
    if b is None:  # reduction over the components of a vector
        return float(a.a.max())
    if isinstance(a, Vec):
        return Vec(np.maximum(a.a, b.a))
    return a if a > b else b


def min(a, b=None):  # noqa: A001
    if b is None:
        return float(a.a.min())
    if isinstance(a, Vec):
        return Vec(np.minimum(a.a, b.a))
    return a if a < b else b


def clamp(x, lo, hi):
    return lo if x < lo else (hi if x > hi else x)


def abs(x):  # noqa: A001
    return -x if x < 0 else x


def sign(x):
    return -1.0 if x < 0.0 else 1.0


def static(x):
    return x


def constant(x):
    return x


def printf(*args):
    pass


# ---------------------------------------------------------------- transforms (p, q=(x,y,z,w))
def _quat_rotate(q, v):
    x, y, z, w = q
    u = np.array([x, y, z])
    return v * (2.0 * w * w - 1.0) + np.cross(u, v) * 2.0 * w + u * 2.0 * np.dot(u, v)


def quat_from_axis_angle(axis, angle):
    ax = np.asarray(axis.a if isinstance(axis, Vec) else axis, dtype=DTYPE)
    ax = ax / np.linalg.norm(ax)
    s = math.sin(angle * 0.5)
    return np.array([ax[0] * s, ax[1] * s, ax[2] * s, math.cos(angle * 0.5)])


def quat_identity():
    return np.array([0.0, 0.0, 0.0, 1.0])


def quat_to_matrix(q):
    e = np.eye(3)
    return Mat(np.stack([_quat_rotate(q, e[i]) for i in range(3)], axis=1))


def transform_identity():
    return (np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))


def quat_rotate(q, v):
    return Vec(_quat_rotate(np.asarray(q, dtype=DTYPE), np.asarray(v.a if isinstance(v, Vec) else v, dtype=DTYPE)))


def transform_point(X, p):
    return Vec(_quat_rotate(X[1], p.a) + X[0])


def transform_vector(X, v):
    return Vec(_quat_rotate(X[1], v.a))


def transform_inverse(X):
    p, q = X
    qi = np.array([-q[0], -q[1], -q[2], q[3]])
    return (-_quat_rotate(qi, np.asarray(p, dtype=DTYPE)), qi)


def _quat_mul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz])  # fmt: skip


def transform_multiply(A, B):
    return (_quat_rotate(A[1], np.asarray(B[0], dtype=DTYPE)) + A[0], _quat_mul(A[1], B[1]))


def cw_mul(a, b):
    return Vec(a.a * b.a)


def cw_div(a, b):
    return Vec(a.a / b.a)


# ---------------------------------------------------------------- arrays and launches
class Array:
    """A host array of scalars, Vec or Mat values; truthy when non-empty, like a Warp array."""

    def __init__(self, items):
        self.items = list(items)

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            return self.items[idx[0]][idx[1]]
        return self.items[idx]

    def __setitem__(self, idx, value):
        if isinstance(idx, tuple):
            row = self.items[idx[0]]
            row[idx[1]] = value
        else:
            self.items[idx] = value

    def __bool__(self):
        return len(self.items) > 0

    def __len__(self):
        return len(self.items)

    @property
    def shape(self):
        return (len(self.items),)


_TID = [0]


def tid():
    return _TID[0]


def atomic_add(arr, idx, value):
    old = arr[idx]
    arr[idx] = old + value
    return old


def atomic_min(arr, idx, value):
    old = arr[idx]
    if value < old:
        arr[idx] = value
    return old


def closest_point_edge_edge(p1, q1, p2, q2, epsilon):
    """Closest points of segments p1-q1 and p2-q2: returns vec3(s, t, distance) (Ericson, sec. 5.1.9)."""
    d1, d2 = q1.a - p1.a, q2.a - p2.a
    r = p1.a - p2.a
    a, e, f = float(np.dot(d1, d1)), float(np.dot(d2, d2)), float(np.dot(d2, r))
    if a <= epsilon and e <= epsilon:
        s = t = 0.0
    elif a <= epsilon:
        s, t = 0.0, clamp(f / e, 0.0, 1.0)
    else:
        c = float(np.dot(d1, r))
        if e <= epsilon:
            s, t = clamp(-c / a, 0.0, 1.0), 0.0
        else:
            b = float(np.dot(d1, d2))
            denom = a * e - b * b
            s = clamp((b * f - c * e) / denom, 0.0, 1.0) if denom != 0.0 else 0.0
            t = (b * s + f) / e
            if t < 0.0:
                t, s = 0.0, clamp(-c / a, 0.0, 1.0)
            elif t > 1.0:
                t, s = 1.0, clamp((b - c) / a, 0.0, 1.0)
    c1, c2 = p1.a + d1 * s, p2.a + d2 * t
    return Vec([s, t, float(np.sqrt(np.dot(c1 - c2, c1 - c2)))])


class Bvh:
    """Primitive boxes; ``bvh_query_aabb`` tests them all."""

    def __init__(self, lowers, uppers):
        self.lo = np.asarray(lowers, dtype=DTYPE).reshape(-1, 3)
        self.hi = np.asarray(uppers, dtype=DTYPE).reshape(-1, 3)


def bvh_query_aabb(bvh, lower, upper):
    hit = np.all(bvh.lo <= upper.a, axis=1) & np.all(bvh.hi >= lower.a, axis=1)
    return [int(i) for i in np.nonzero(hit)[0]]


def launch(kernel, dim, *args):
    for i in range(dim):
        _TID[0] = i
        kernel(*args)


def vec_array(a):
    return Array([Vec(r) for r in np.asarray(a, dtype=DTYPE).reshape(-1, 3)])


def mat33_array(a):
    return Array([Mat(r) for r in np.asarray(a, dtype=DTYPE).reshape(-1, 3, 3)])


def mat22_array(a):
    return Array([Mat(r) for r in np.asarray(a, dtype=DTYPE).reshape(-1, 2, 2)])


def scalar_array(a, kind=float):
    return Array([kind(x) for x in np.asarray(a).reshape(-1)])


def array2d(a, kind=float):
    return Array([[kind(x) for x in r] for r in np.asarray(a)])


def to_numpy(arr):
    out = []
    for x in arr.items:
        out.append(x.a if isinstance(x, (Vec, Mat)) else x)
    return np.array(out, dtype=DTYPE)


class types:  # noqa: N801 - mirrors ``wp.types``
    @staticmethod
    def matrix(shape, dtype):
        return object

    @staticmethod
    def vector(length, dtype):
        return object
