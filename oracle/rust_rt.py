"""Runtime for Rust code translated to Python by oracle/rust2py.py.

TEST INFRASTRUCTURE ONLY (part of the oracle).  It gives the translated
reference functions the semantics of the Rust standard library they call:

  * f32 values are numpy.float32 scalars, so every +, -, *, / is one
    correctly rounded binary32 operation (Rust never contracts a*b+c);
    sqrt is correctly rounded, acos/cos/... call the C library's binary32
    functions (what Rust's f32 methods call on Linux), round() is
    half-away-from-zero, powi(2) is x*x, min/max return the non-NaN operand;
  * integers are Python ints; `as` casts truncate floats toward zero with
    saturation (NaN -> 0) and wrap integers to the target width, so a
    negative i32 cast to usize becomes a huge index, as in Rust;
  * integer / and % truncate toward zero;
  * Option<T> is T or None; Result<T, E> is T, and Err(e) raises RustError;
  * Vec / slices / arrays are lists, HashMap dict, HashSet set, VecDeque
    collections.deque; Iterator adaptors are lazy (It);
  * `&mut` places that a callee writes through (`*p = ...`) are passed as
    Cell / AttrRef objects.

Third-party crates the reference calls are shims restating their published
behaviour:
  * kd-tree 0.5.1 (KdIndexTree::build_by_ordered_float, within_by_cmp,
    item): within_by_cmp returns every item for which the comparison is
    Equal in every dimension.  The crate returns them in the order of its
    tree walk; the shim returns them in index order (the order only decides
    exact score ties in the subnet search);
  * ndarray (ArrayView::from_shape, get, 2-D indexing) over numpy arrays;
  * bitflags (LinkingWarning) as integers.
"""
import collections
import copy as _copy
import ctypes
import functools
import math
import sys

import numpy as np

F32 = np.float32
_libm = ctypes.CDLL("libm.so.6")
for _n in ("acosf", "cosf", "sinf", "atan2f", "expf", "logf", "log10f", "powf", "asinf", "atanf", "tanf"):
    getattr(_libm, _n).restype = ctypes.c_float
    getattr(_libm, _n).argtypes = [ctypes.c_float] * (2 if _n in ("atan2f", "powf") else 1)

np.seterr(all="ignore")
sys.setrecursionlimit(100000)


class RustError(Exception):
    """An Err(...) value or a panic of the translated code."""

    def __init__(self, kind, detail=None):
        super().__init__(kind)
        self.kind = kind
        self.detail = detail


def err(e):
    raise RustError(e.tag if isinstance(e, REnum) else e, e)


def panic(msg="panic"):
    raise RustError("panic", msg)


class REnum:
    """A value of a Rust enum: variant name plus tuple or named fields."""
    __slots__ = ("tag", "vals", "named")

    def __init__(self, tag, vals=(), named=None):
        self.tag = tag
        self.vals = list(vals)
        self.named = named or {}

    def __eq__(self, other):
        return isinstance(other, REnum) and other.tag == self.tag and other.vals == self.vals

    def __hash__(self):
        return hash(self.tag)

    def __repr__(self):
        return "REnum(%s, %r, %r)" % (self.tag, self.vals, self.named)

    def __getattr__(self, k):
        named = object.__getattribute__(self, "named")
        if k in named:
            return named[k]
        raise AttributeError(k)


class _Ordering:
    Less = REnum("Less")
    Equal = REnum("Equal")
    Greater = REnum("Greater")
    # std::sync::atomic::Ordering shares the name in the reference's imports
    Relaxed = REnum("Relaxed")
    SeqCst = REnum("SeqCst")
    Acquire = REnum("Acquire")
    Release = REnum("Release")


Ordering = _Ordering


def Error(kind, **named):
    return REnum(kind, (), named)


def tag_is(x, name):
    """Whether x is the enum variant called name (the last path segment)."""
    return isinstance(x, REnum) and x.tag == name


class Struct:
    """Base of translated structs: keyword construction with derived defaults."""
    _fields = ()

    def __init__(self, **kw):
        for name, default in self._fields:
            if name in kw:
                v = kw.pop(name)
            else:
                v = default() if callable(default) else default
            object.__setattr__(self, name, v)
        if kw:
            raise TypeError("unknown fields %s for %s" % (list(kw), type(self).__name__))

    def __repr__(self):
        return "%s(%s)" % (type(self).__name__, ", ".join("%s=%r" % (n, getattr(self, n)) for n, _ in self._fields))


def default_struct(cls):
    return cls()


def struct_update(cls, base, **kw):
    d = {n: _copy.copy(getattr(base, n)) for n, _ in cls._fields}
    d.update(kw)
    return cls(**d)


def assign_self(obj, new):
    obj.__dict__.clear()
    obj.__dict__.update(new.__dict__)


# --------------------------------------------------------------- references
class Cell:
    """A `&mut` to a temporary (let x = &mut 0.0)."""
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v


class AttrRef:
    """A `&mut obj.field` passed to a callee that writes through it."""
    __slots__ = ("_o", "_n")

    def __init__(self, o, n):
        self._o = o
        self._n = n

    @property
    def v(self):
        return getattr(self._o, self._n)

    @v.setter
    def v(self, x):
        setattr(self._o, self._n, x)


class IndexRef:
    __slots__ = ("_o", "_i")

    def __init__(self, o, i):
        self._o = o
        self._i = i

    @property
    def v(self):
        return self._o[self._i]

    @v.setter
    def v(self, x):
        self._o[self._i] = x


# --------------------------------------------------------------- numerics
_INT_BITS = {"u8": (8, False), "u16": (16, False), "u32": (32, False), "u64": (64, False), "usize": (64, False),
             "i8": (8, True), "i16": (16, True), "i32": (32, True), "i64": (64, True), "isize": (64, True)}


def cast(x, ty):
    if ty in ("f32",):
        if isinstance(x, (bool, np.bool_)):
            return F32(1.0 if x else 0.0)
        return F32(x)
    if ty == "f64":
        return float(x)
    if ty == "bool":
        return bool(x)
    bits, signed = _INT_BITS[ty]
    if isinstance(x, (float, np.floating)):
        xf = float(x)
        if math.isnan(xf):
            return 0
        lo = -(1 << (bits - 1)) if signed else 0
        hi = (1 << (bits - 1)) - 1 if signed else (1 << bits) - 1
        if xf <= lo:
            return lo
        if xf >= hi:
            return hi
        return int(xf)  # truncation toward zero
    x = int(x)
    x &= (1 << bits) - 1
    if signed and x >= (1 << (bits - 1)):
        x -= 1 << bits
    return x


def div(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)) and not isinstance(a, bool):
        a, b = int(a), int(b)
        if b == 0:
            panic("attempt to divide by zero")
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q
    return F32(a) / F32(b) if not isinstance(a, float) else a / b


def rem(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
        a, b = int(a), int(b)
        if b == 0:
            panic("attempt to calculate the remainder with a divisor of zero")
        return a - b * div(a, b)
    return F32(math.fmod(float(a), float(b)))


def _isf(x):
    return isinstance(x, (np.floating, float))


def f_round(x):
    xf = float(x)
    if math.isnan(xf) or math.isinf(xf):
        return F32(xf)
    return F32(math.copysign(math.floor(abs(xf) + 0.5), xf))


def f_min(a, b):
    if _isf(a):
        if math.isnan(a):
            return b
        if math.isnan(b):
            return a
        return a if a <= b else b
    return a if a <= b else b


def f_max(a, b):
    if _isf(a):
        if math.isnan(a):
            return b
        if math.isnan(b):
            return a
        return a if a >= b else b
    return a if a >= b else b


def powi(x, n):
    if _isf(x):
        x = F32(x)
        if n == 0:
            return F32(1.0)
        r = x
        for _ in range(abs(int(n)) - 1):
            r = F32(r * x)
        return F32(1.0) / r if n < 0 else r
    return int(x) ** int(n)


def partial_cmp(a, b):
    if _isf(a) or _isf(b):
        if math.isnan(float(a)) or math.isnan(float(b)):
            return None
    if a < b:
        return Ordering.Less
    if a > b:
        return Ordering.Greater
    return Ordering.Equal


def max_by(a, b, cmp):
    """std::cmp::max_by: the second argument when they compare equal."""
    return a if cmp(a, b) is Ordering.Greater else b


def min_by(a, b, cmp):
    return b if cmp(a, b) is Ordering.Greater else a


def _ord_int(o):
    return {"Less": -1, "Equal": 0, "Greater": 1}[o.tag]


# --------------------------------------------------------------- iterators
class It:
    """A lazy Rust iterator."""
    __slots__ = ("_g",)

    def __init__(self, g):
        self._g = iter(g)

    def __iter__(self):
        return self._g

    def __next__(self):
        return next(self._g)

    def next(self):
        return next(self._g, None)

    def map(self, f):
        return It(f(x) for x in self._g)

    def filter(self, f):
        return It(x for x in self._g if f(x))

    def filter_map(self, f):
        return It(y for y in (f(x) for x in self._g) if y is not None)

    def enumerate(self):
        return It(enumerate(self._g))

    def zip(self, other):
        return It(zip(self._g, iterate(other)))

    def chain(self, other):
        def g():
            yield from self._g
            yield from iterate(other)
        return It(g())

    def take(self, n):
        def g():
            if n <= 0:
                return
            for i, x in enumerate(self._g):
                yield x
                if i + 1 >= n:
                    return
        return It(g())

    def skip(self, n):
        def g():
            for i, x in enumerate(self._g):
                if i >= n:
                    yield x
        return It(g())

    def flatten(self):
        def g():
            for x in self._g:
                if x is None:
                    continue
                if isinstance(x, (list, collections.deque, It, range)):
                    yield from x
                else:
                    yield x
        return It(g())

    def cloned(self):
        return It(_copy.copy(x) for x in self._g)

    copied = cloned

    def collect(self):
        return list(self._g)

    def sum(self):
        """Iterator::sum: a fold from zero of the element type (0.0 for f32)."""
        acc = None
        for x in self._g:
            if acc is None:
                acc = F32(0.0) if _isf(x) else 0
            acc = acc + x
        if acc is None:
            return F32(0.0)
        return acc

    def count(self):
        return sum(1 for _ in self._g)

    def all(self, f):
        return all(f(x) for x in self._g)

    def any(self, f):
        return any(f(x) for x in self._g)

    def for_each(self, f):
        for x in self._g:
            f(x)

    def rev(self):
        return It(reversed(list(self._g)))

    def last(self):
        r = None
        for x in self._g:
            r = x
        return r

    def fold(self, init, f):
        acc = init
        for x in self._g:
            acc = f(acc, x)
        return acc

    def cycle(self):
        items = list(self._g)

        def g():
            while items:
                yield from items
        return It(g())

    def max_by(self, f):
        best = None
        for x in self._g:
            if best is None or f(x, best) is not Ordering.Less:
                best = x
        return best

    def min_by(self, f):
        best = None
        for x in self._g:
            if best is None or f(x, best) is Ordering.Less:
                best = x
        return best

    def position(self, f):
        for i, x in enumerate(self._g):
            if f(x):
                return i
        return None

    def into_iter(self):
        return self

    iter = into_iter


def from_next(obj):
    """Iterator over a translated struct that implements Iterator::next."""
    def g():
        while True:
            x = obj.next()
            if x is None:
                return
            yield x
    return It(g())


def iterate(x):
    if isinstance(x, It):
        return x
    if isinstance(x, dict):
        return It(x.items())
    if hasattr(x, "next") and not isinstance(x, (list, tuple, collections.deque, set, range, np.ndarray)):
        return from_next(x)
    return It(x)


def once(x):
    return It([x])


class _Entry:
    def __init__(self, d, k):
        self.d, self.k = d, k

    def or_insert(self, v):
        if self.k not in self.d:
            self.d[self.k] = v
        return self.d[self.k]


def vec_rep(v, n):
    return [_copy.deepcopy(v) for _ in range(int(n))]


# --------------------------------------------------------------- method dispatch
_ITER_METHODS = set(k for k in It.__dict__ if not k.startswith("_"))


def _sort_by(lst, f):
    lst.sort(key=functools.cmp_to_key(lambda a, b: _ord_int(f(a, b))))


def _get(x, i):
    if isinstance(x, np.ndarray):
        idx = tuple(int(v) for v in i) if isinstance(i, (list, tuple)) else (int(i),)
        if len(idx) != x.ndim or any(v < 0 or v >= s for v, s in zip(idx, x.shape)):
            return None
        return x[idx]
    if isinstance(x, dict):
        return x.get(i)
    i = int(i)
    return x[i] if 0 <= i < len(x) else None


def _f32_method(x, m, a):
    if m == "sqrt":
        return F32(np.sqrt(F32(x)))
    if m == "abs":
        return F32(abs(F32(x)))
    if m == "round":
        return f_round(x)
    if m == "ceil":
        return F32(math.ceil(float(x))) if math.isfinite(float(x)) else F32(x)
    if m == "floor":
        return F32(math.floor(float(x))) if math.isfinite(float(x)) else F32(x)
    if m in ("powi", "pow"):
        if _isf(a[0]):
            return F32(_libm.powf(float(x), float(a[0])))
        return powi(x, a[0])
    if m == "powf":
        return F32(_libm.powf(float(x), float(a[0])))
    if m in ("acos", "cos", "sin", "exp", "asin", "atan", "tan"):
        return F32(getattr(_libm, m + "f")(float(x)))
    if m == "ln":
        return F32(_libm.logf(float(x)))
    if m == "log10":
        return F32(_libm.log10f(float(x)))
    if m == "atan2":
        return F32(_libm.atan2f(float(x), float(a[0])))
    if m == "min":
        return f_min(F32(x), F32(a[0]))
    if m == "max":
        return f_max(F32(x), F32(a[0]))
    if m == "clamp":
        v = F32(x)
        if v < a[0]:
            v = F32(a[0])
        if v > a[1]:
            v = F32(a[1])
        return v
    if m == "to_bits":
        return int(np.array(F32(x)).view(np.uint32))
    if m == "is_nan":
        return math.isnan(float(x))
    if m == "is_finite":
        return math.isfinite(float(x))
    if m == "signum":
        return F32(math.copysign(1.0, float(x))) if not math.isnan(float(x)) else F32(x)
    raise AttributeError("f32 method %s" % m)


def call(x, m, *a):
    """x.m(a...) with Rust semantics for the standard types."""
    if isinstance(x, (Struct, REnum)) and hasattr(type(x), m):
        return getattr(x, m)(*a)
    if hasattr(x, "__rust_methods__") and m in x.__rust_methods__:
        return getattr(x, m)(*a)
    # methods every type shares
    if m in ("clone", "to_owned", "to_vec", "into_owned"):
        if isinstance(x, list):
            return list(x)
        if isinstance(x, (dict, set, collections.deque)):
            return type(x)(x)
        return _copy.copy(x)
    if m in ("as_ref", "as_mut", "borrow", "borrow_mut", "into", "as_slice", "as_mut_slice", "deref",
             "into_slice"):
        return x
    if m == "partial_cmp" or m == "cmp":
        return partial_cmp(x, a[0])
    # Option / Result
    if x is None:
        if m in ("map", "and_then", "as_deref", "copied", "cloned", "filter"):
            return None
        if m == "unwrap_or":
            return a[0]
        if m == "unwrap_or_else":
            return a[0]()
        if m == "unwrap_or_default":
            return F32(0.0)
        if m == "is_some":
            return False
        if m == "is_none":
            return True
        if m in ("unwrap", "expect"):
            panic("called `Option::unwrap()` on a `None` value")
        if m == "ok_or":
            err(a[0])
        raise AttributeError("None.%s" % m)
    if isinstance(x, It) or isinstance(x, range):
        if isinstance(x, range):
            x = It(x)
        return getattr(x, m)(*a)
    if m in ("unwrap", "expect", "unwrap_or", "unwrap_or_else", "unwrap_or_default", "ok", "map_err"):
        return x
    if m == "is_some":
        return True
    if m == "is_none":
        return False
    if m == "and_then":
        return a[0](x)
    # Option::map (Vec, HashMap, ... have no `map`: any other receiver is an Option's value)
    if m == "map" and not hasattr(x, "next"):
        return a[0](x)
    # numbers
    if isinstance(x, (np.floating, float)):
        return _f32_method(x, m, a)
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        if m in ("pow", "powi"):
            return int(x) ** int(a[0])
        if m == "abs":
            return abs(int(x))
        if m == "min":
            return min(int(x), int(a[0]))
        if m == "max":
            return max(int(x), int(a[0]))
        if m == "saturating_sub":
            return max(0, int(x) - int(a[0]))
        raise AttributeError("int method %s" % m)
    # collections
    if isinstance(x, list) or isinstance(x, np.ndarray):
        if m == "len":
            return len(x)
        if m == "push":
            x.append(a[0])
            return None
        if m == "pop":
            return x.pop() if x else None
        if m in ("iter", "iter_mut", "into_iter"):
            return It(x)
        if m == "clear":
            del x[:]
            return None
        if m in ("get", "get_mut"):
            return _get(x, a[0])
        if m == "sort_by":
            _sort_by(x, a[0])
            return None
        if m in ("extend", "extend_from_slice", "append"):
            x.extend(list(iterate(a[0])))
            return None
        if m == "contains":
            return a[0] in x
        if m == "is_empty":
            return len(x) == 0
        if m == "first":
            return x[0] if len(x) else None
        if m == "last":
            return x[-1] if len(x) else None
        if m == "chunks_exact":
            n = int(a[0])
            return It(x[i:i + n] for i in range(0, len(x) - len(x) % n, n))
        if m == "swap":
            x[a[0]], x[a[1]] = x[a[1]], x[a[0]]
            return None
        if m == "insert":
            x.insert(a[0], a[1])
            return None
        if m == "remove":
            return x.pop(a[0])
        if m == "truncate":
            del x[a[0]:]
            return None
        if m == "reverse":
            x.reverse()
            return None
        if m == "shape":
            return list(x.shape)
        if m == "rows":
            return It(list(x))
        if m == "at":
            return x[a[0]]
        if m in _ITER_METHODS:
            return getattr(It(x), m)(*a)
        raise AttributeError("list method %s" % m)
    if isinstance(x, tuple):
        if m == "at":  # kd-tree: a (point, data) tuple is its point
            return call(x[0], "at", *a)
        if m == "len":
            return len(x)
        raise AttributeError("tuple method %s" % m)
    if isinstance(x, dict):
        if m == "contains_key":
            return a[0] in x
        if m == "insert":
            old = x.get(a[0])
            x[a[0]] = a[1]
            return old
        if m == "remove":
            return x.pop(a[0], None)
        if m in ("get", "get_mut"):
            return x.get(a[0])
        if m in ("iter", "iter_mut", "into_iter"):
            return It(list(x.items()))
        if m == "keys":
            return It(list(x.keys()))
        if m == "values":
            return It(list(x.values()))
        if m == "len":
            return len(x)
        if m == "clear":
            x.clear()
            return None
        if m == "entry":
            return _Entry(x, a[0])
        if m == "is_empty":
            return not x
        raise AttributeError("dict method %s" % m)
    if isinstance(x, set):
        if m == "contains":
            return a[0] in x
        if m == "insert":
            new = a[0] not in x
            x.add(a[0])
            return new
        if m == "remove":
            present = a[0] in x
            x.discard(a[0])
            return present
        if m == "len":
            return len(x)
        if m in ("iter", "into_iter"):
            return It(list(x))
        if m == "clear":
            x.clear()
            return None
        if m == "is_empty":
            return not x
        raise AttributeError("set method %s" % m)
    if isinstance(x, collections.deque):
        if m == "push_back":
            x.append(a[0])
            return None
        if m == "push_front":
            x.appendleft(a[0])
            return None
        if m == "pop_front":
            return x.popleft() if x else None
        if m == "pop_back":
            return x.pop() if x else None
        if m == "len":
            return len(x)
        if m in ("iter", "iter_mut", "into_iter"):
            return It(list(x))
        if m == "front":
            return x[0] if x else None
        if m == "back":
            return x[-1] if x else None
        if m == "clear":
            x.clear()
            return None
        if m == "is_empty":
            return not x
        raise AttributeError("deque method %s" % m)
    if hasattr(x, "next") and m in _ITER_METHODS:
        return getattr(from_next(x), m)(*a)
    if m == "map":
        return a[0](x)
    if hasattr(x, m):
        return getattr(x, m)(*a)
    raise AttributeError("%s has no method %s" % (type(x).__name__, m))


def at(x, k):
    return call(x, "at", k)


def length(x):
    return len(x)


# --------------------------------------------------------------- shims of crates
class KdIndexTree:
    """kd-tree 0.5.1 KdIndexTree: queries answer with indices into the points."""
    __rust_methods__ = ("within_by_cmp", "item", "within_radius_rd2")

    def __init__(self, points):
        self.points = points

    @staticmethod
    def build_by_ordered_float(points):
        return KdIndexTree(points)

    def item(self, i):
        return self.points[i]

    def within_by_cmp(self, cmp):
        out = []
        for i, p in enumerate(self.points):
            if all(cmp(p, k) is Ordering.Equal for k in range(2)):
                out.append(i)
        return out


class LinkingWarning:
    """bitflags! LinkingWarning (src/linking.rs): flags as integer bits."""
    SUBNET_FRACTION_TOO_HIGH = 1
    COMPUTATION_TOO_HEAVY = 2

    @staticmethod
    def empty():
        return 0


class ArrayView:
    """ndarray's ArrayView::from_shape over a flat numpy buffer."""

    @staticmethod
    def from_shape(dims, data):
        return np.asarray(data).reshape(tuple(int(d) for d in dims))


def Ix2(a, b):
    return (a, b)


class AtomicBool:
    __rust_methods__ = ("load", "store")

    def __init__(self, v=False):
        self.v = bool(v)

    def load(self, _order):
        return self.v

    def store(self, v, _order):
        self.v = bool(v)


PI = F32(math.pi)
INFINITY = F32(np.inf)
NEG_INFINITY = F32(-np.inf)
NAN = F32(np.nan)
