"""A numpy stand-in for the few JAX primitives that mitgcm_jax's CG2D path uses, so that the reference's OWN
cg2d_fortran (mitgcm_jax/core/cg2d.py:205-269) and Exchanger (mitgcm_jax/parallel/exchange.py:146-183) can run in a
container without JAX and produce golden outputs (make_golden.py). Test infrastructure only.

Every primitive is the plain IEEE float64 operation: elementwise +, -, *, / and sqrt, `where`, `max`, gathers and
slice updates; `lax.while_loop` and `lax.scan` become Python loops (the "fortran" tile sum stays strictly
sequential, as the reference's scan is). That is the arithmetic the reference gets from XLA on CPU with the
determinism flags of its test suite (no FMA, no algebraic simplification), so outputs are bitwise what the
reference computes on the same inputs. The "tile" sum order (an XLA tree reduction) is NOT reproduced.
"""

import sys
import types

import numpy as np


class Arr(np.ndarray):
    """ndarray with JAX's functional `.at[idx].set(v)` / `.add(v)`."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, a):
        self.a = a

    def __getitem__(self, idx):
        return _AtIdx(self.a, idx)


class _AtIdx:
    def __init__(self, a, idx):
        self.a, self.idx = a, idx

    def set(self, v):
        out = np.array(self.a, copy=True).view(Arr)
        out[self.idx] = v
        return out

    def add(self, v):
        out = np.array(self.a, copy=True).view(Arr)
        out[self.idx] += v
        return out


def _w(x):
    if isinstance(x, np.ndarray):
        return x.view(Arr)
    if isinstance(x, (np.generic, float, int, bool)):
        return np.asarray(x).view(Arr)
    return x


def _wrap(fn):
    def f(*a, **k):
        return _w(fn(*a, **k))
    return f


def install():
    """Insert `jax`, `jax.numpy`, `jax.lax`, ... into sys.modules (idempotent)."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "__standin__", False):
        return
    jax = types.ModuleType("jax")
    jax.__standin__ = True
    jnp = types.ModuleType("jax.numpy")
    lax = types.ModuleType("jax.lax")
    adc = types.ModuleType("jax.ad_checkpoint")
    tu = types.ModuleType("jax.tree_util")
    tree = types.ModuleType("jax.tree")
    dtypes = types.ModuleType("jax.dtypes")

    for name in ("zeros", "ones", "zeros_like", "ones_like", "where", "sum", "max", "min", "abs", "sqrt", "maximum",
                 "minimum", "moveaxis", "logical_not", "logical_and", "vdot", "stack", "concatenate", "full",
                 "arange", "isfinite", "all", "any", "argmax"):
        setattr(jnp, name, _wrap(getattr(np, name)))
    jnp.asarray = _wrap(lambda a, dtype=None: np.array(a, dtype=dtype, copy=True))
    jnp.array = jnp.asarray
    for name in ("float64", "float32", "int32", "int64", "int8", "bool_", "floating", "integer", "issubdtype",
                 "result_type", "shape", "ndarray"):
        setattr(jnp, name, getattr(np, name))

    def while_loop(cond, body, init):
        st = init
        while bool(cond(st)):
            st = body(st)
        return st

    def scan(f, init, xs, length=None, reverse=False, unroll=1):
        # xs: an array, or a tuple / list of arrays sliced together along their first axis (a pytree of arrays)
        carry = init
        ys = []
        multi = isinstance(xs, (tuple, list))
        n = (len(xs[0]) if multi else len(xs)) if xs is not None else length
        order = range(n - 1, -1, -1) if reverse else range(n)

        def item(i):
            if xs is None:
                return None
            return type(xs)(_w(a[i]) for a in xs) if multi else _w(xs[i])

        for i in order:
            carry, y = f(carry, item(i))
            ys.append(y)
        if all(y is None for y in ys):
            return carry, None
        if reverse:
            ys = ys[::-1]
        return carry, _w(np.stack(ys))

    lax.while_loop = while_loop
    lax.scan = scan
    lax.stop_gradient = lambda x: x

    def _unsupported(*a, **k):
        raise NotImplementedError("not available in the numpy stand-in")

    lax.custom_linear_solve = _unsupported
    lax.psum = _unsupported
    adc.checkpoint_name = lambda x, name: x

    def jit(fun=None, **kw):
        if fun is None:
            return lambda f: f
        return fun

    class custom_jvp:
        def __init__(self, fun, nondiff_argnums=()):
            self.fun = fun

        def defjvp(self, jvp):
            self.jvp = jvp
            return jvp

        def __call__(self, *a, **k):
            return self.fun(*a, **k)

    tu.register_pytree_node_class = lambda cls: cls
    tu.register_dataclass = lambda cls, data_fields=None, meta_fields=None: cls
    tree.map = lambda f, t: {k: f(v) for k, v in t.items()} if isinstance(t, dict) else f(t)

    # pytrees of tuples, lists and dicts (keys in sorted order); anything else is a leaf
    def flatten(t):
        if isinstance(t, (tuple, list)):
            parts = [flatten(x) for x in t]
            return [leaf for ls, _ in parts for leaf in ls], (type(t), None, [d for _, d in parts])
        if isinstance(t, dict):
            keys = sorted(t)
            parts = [flatten(t[k]) for k in keys]
            return [leaf for ls, _ in parts for leaf in ls], (dict, keys, [d for _, d in parts])
        return [t], None

    def unflatten(treedef, leaves):
        it = iter(leaves)

        def build(d):
            if d is None:
                return next(it)
            typ, keys, subs = d
            if typ is dict:
                return {k: build(s) for k, s in zip(keys, subs)}
            return typ(build(s) for s in subs)

        return build(treedef)

    tree.flatten = flatten
    tree.unflatten = unflatten
    dtypes.float0 = np.dtype([])

    class _Config:
        def update(self, *a, **k):
            pass

    jax.numpy, jax.lax, jax.ad_checkpoint, jax.tree_util, jax.tree, jax.dtypes = jnp, lax, adc, tu, tree, dtypes
    jax.jit = jit
    jax.custom_jvp = custom_jvp
    jax.config = _Config()
    jax.Array = np.ndarray
    jax.grad = _unsupported
    jax.vjp = _unsupported
    for name, mod in (("jax", jax), ("jax.numpy", jnp), ("jax.lax", lax), ("jax.ad_checkpoint", adc),
                      ("jax.tree_util", tu), ("jax.tree", tree), ("jax.dtypes", dtypes)):
        sys.modules[name] = mod
