"""A serial, FP64 stand-in for the part of Taichi 1.7.4 that the reference's
solver path uses -- test infrastructure for generating golden vectors only.

Taichi is absent from this image (and the reference pins cp313 wheels while
the interpreter is 3.12), so the reference's `@ti.kernel` functions cannot run
as published. This module lets them run unmodified, on the CPU, in this
container: it is installed as `sys.modules['taichi']` before the reference
package is imported.

Semantics implemented (Taichi 1.7.4 language reference, restated):
  * `ti.field(dtype, shape)`: dense 0-D/1-D/2-D arrays; `for i in field`
    iterates indices; `fill`, `from_numpy`, `to_numpy`, `field[None]`.
  * `@ti.kernel`: top-level for-loops run serially in program order (one
    valid schedule of Taichi's parallel loops); `x += v` into a kernel-local
    scalar is a reduction, here a serial sum; `ti.atomic_add(a[i], v)` adds in
    place; `ti.atomic_max(x, v)` on a local takes the max.
  * `ti.static(range(n))` is `range(n)`; `ti.Matrix.zero(dt, r, c)` is an r x c
    array; `ti.pow/sqrt/max/min/abs/cast` are the scalar maths.
  * Precision: every field and every scalar is an IEEE double, whatever
    dtype the caller declared -- this executes the reference's algorithm
    in FP64. `promote_reference_numpy()` additionally makes the reference's
    own host-side `np.float32` casts (Ke, Ke_inv, the load vector, filter
    weights) FP64, so no value is rounded to single precision anywhere.

Kernel bodies are rewritten once at decoration time (an AST pass) so that
subscripts address Python lists directly; that makes the pure-Python
execution fast enough for the small meshes the golden vectors use.
"""

from __future__ import annotations

import ast
import inspect
import math
import sys
import textwrap
import types

import numpy as np

f32, f64, i32, i64, u8 = "f32", "f64", "i32", "i64", "u8"
cpu, cuda, metal, vulkan = "cpu", "cuda", "metal", "vulkan"
_INT_TYPES = (i32, i64, u8)


def init(arch=None, default_fp=None, default_ip=None, **kwargs):
    return None


def template():
    return None


def sync():
    return None


def static(x):
    return x


pow = lambda a, b: float(a) ** float(b)  # noqa: E731  (Taichi's ti.pow)
sqrt = math.sqrt
abs = lambda x: x if x >= 0 else -x      # noqa: E731
max = lambda a, b: a if a >= b else b    # noqa: E731  (Taichi's ti.max)
min = lambda a, b: a if a <= b else b    # noqa: E731


def cast(x, dtype):
    return int(x) if dtype in _INT_TYPES else float(x)


class Field:
    """Dense field; `_d` is a flat list (0-D/1-D) or list of rows (2-D)."""

    def __init__(self, dtype, shape):
        self.dtype = dtype
        self.shape = () if shape == () else (tuple(shape) if isinstance(shape, (tuple, list))
                                             else (int(shape),))
        zero = 0 if dtype in _INT_TYPES else 0.0
        if len(self.shape) <= 1:
            self._d = [zero] * (self.shape[0] if self.shape else 1)
        elif len(self.shape) == 2:
            self._d = [[zero] * self.shape[1] for _ in range(self.shape[0])]
        else:
            raise NotImplementedError("fields of rank > 2 are not needed")

    def _conv(self, v):
        return int(v) if self.dtype in _INT_TYPES else float(v)

    def __iter__(self):
        return iter(range(self.shape[0] if self.shape else 1))

    def __getitem__(self, k):
        if k is None:
            return self._d[0]
        if isinstance(k, tuple):
            return self._d[k[0]][k[1]]
        return self._d[k]

    def __setitem__(self, k, v):
        if k is None:
            self._d[0] = self._conv(v)
        elif isinstance(k, tuple):
            self._d[k[0]][k[1]] = self._conv(v)
        else:
            self._d[k] = self._conv(v)

    def fill(self, v):
        v = self._conv(v)
        if len(self.shape) == 2:
            self._d = [[v] * self.shape[1] for _ in range(self.shape[0])]
        else:
            self._d = [v] * len(self._d)

    def from_numpy(self, arr):
        arr = np.asarray(arr)
        if len(self.shape) == 2:
            self._d = [[self._conv(x) for x in row] for row in arr.tolist()]
        else:
            self._d = [self._conv(x) for x in arr.reshape(-1).tolist()]

    def to_numpy(self):
        dt = np.int32 if self.dtype in _INT_TYPES else np.float64
        if not self.shape:
            return np.array(self._d[0], dtype=dt)
        return np.array(self._d, dtype=dt).reshape(self.shape)


def field(dtype, shape=()):
    return Field(dtype, shape)


class _Mat:
    """`ti.Matrix` value: list of rows."""

    def __init__(self, r, c):
        self._d = [[0.0] * c for _ in range(r)]


class Matrix:
    @staticmethod
    def zero(dtype, r, c=1):
        return _Mat(r, c)


class _Rewrite(ast.NodeTransformer):
    """Kernel-body rewrite: direct list subscripts and in-place atomics."""

    @staticmethod
    def _data(node):
        return ast.Attribute(value=node, attr="_d", ctx=ast.Load())

    def visit_Subscript(self, node):
        self.generic_visit(node)
        sl = node.slice
        if isinstance(sl, ast.Constant) and sl.value is None:          # f[None]
            return ast.Subscript(value=self._data(node.value),
                                 slice=ast.Constant(0), ctx=node.ctx)
        if isinstance(sl, ast.Tuple) and len(sl.elts) == 2:           # f[i, j]
            row = ast.Subscript(value=self._data(node.value), slice=sl.elts[0],
                                ctx=ast.Load())
            return ast.Subscript(value=row, slice=sl.elts[1], ctx=node.ctx)
        return ast.Subscript(value=self._data(node.value), slice=sl, ctx=node.ctx)

    def visit_Expr(self, node):
        call = node.value
        if (isinstance(call, ast.Call) and isinstance(call.func, ast.Attribute)
                and isinstance(call.func.value, ast.Name) and call.func.value.id == "ti"
                and call.func.attr in ("atomic_add", "atomic_max")):
            target, val = call.args
            target = self.visit(target)
            val = self.visit(val)
            if call.func.attr == "atomic_add":
                tgt = _store(target)
                return ast.copy_location(ast.AugAssign(target=tgt, op=ast.Add(), value=val),
                                         node)
            cur = _load(target)
            new = ast.Call(func=ast.Attribute(value=ast.Name("ti", ast.Load()), attr="max",
                                              ctx=ast.Load()),
                           args=[cur, val], keywords=[])
            return ast.copy_location(ast.Assign(targets=[_store(target)], value=new), node)
        return self.generic_visit(node)


def _store(node):
    node = _copy(node)
    node.ctx = ast.Store()
    return node


def _load(node):
    node = _copy(node)
    node.ctx = ast.Load()
    return node


def _copy(node):
    return ast.parse(ast.unparse(node), mode="eval").body


def kernel(fn):
    """Compile `fn` with list-level subscripts; run it serially."""
    src = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(src)
    fdef = tree.body[0]
    fdef.decorator_list = []
    fdef.returns = None
    for a in fdef.args.args:
        a.annotation = None
    fdef.body = [_Rewrite().visit(s) for s in fdef.body]
    tree = ast.fix_missing_locations(tree)
    code = compile(tree, filename=f"<taichi-shim:{fn.__module__}.{fn.__name__}>",
                   mode="exec")
    ns: dict = {}
    exec(code, fn.__globals__, ns)
    compiled = ns[fn.__name__]
    compiled.__wrapped__ = fn
    return compiled


def func(fn):
    return kernel(fn)


class _NumpyFP64(types.ModuleType):
    """numpy, except that `float32` names the double type."""

    def __getattr__(self, name):
        if name == "float32":
            return np.float64
        return getattr(np, name)


def install():
    """Register this module as `taichi` (call before importing the reference)."""
    sys.modules["taichi"] = sys.modules[__name__]


def promote_reference_numpy():
    """Make the reference's host-side `np.float32` casts FP64 (see header)."""
    shim_np = _NumpyFP64("numpy")
    for mod in ("toptimization.fem.fields", "toptimization.optimizer.filter"):
        m = __import__(mod, fromlist=["_"])
        m.np = shim_np
