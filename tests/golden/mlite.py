"""TEST INFRASTRUCTURE: a small interpreter for the MATLAB subset the
reference's layer solve is written in, so that tests/golden/make_golden.py can
execute the reference's own functions (xpbdLayer3D.layerSolve and what it
calls) on small inputs where MATLAB itself is not installed.

Values are numpy arrays with MATLAB semantics: at least two dimensions,
column-major linear indexing, implicit expansion aligned from the first
dimension, 1-based indices, `end` inside subscripts.  Supported: functions
(with local functions and `end`-terminated bodies), static methods of
classdef files (extracted by name), if/elseif/else, for, while, break,
continue, return, multiple assignment with `~`, indexed and logical
assignment, matrix literals with `,`/`;`, strings, the operators of the
language, and the builtins listed in BUILTINS.  Anything else raises.
"""
from __future__ import annotations

import math
import re
import time
from pathlib import Path

import numpy as np

# ---------------------------------------------------------------------------
# values


def M(x):
    """Python value -> MATLAB-like array (>= 2 dims)."""
    if isinstance(x, str):
        return x
    a = np.asarray(x)
    if a.dtype == np.float32 or a.dtype == np.int64 and not isinstance(x, np.ndarray):
        a = a.astype(np.float64)
    if a.dtype.kind in "iu" and a.dtype != np.int32:
        a = a.astype(np.float64)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(1, -1)
    return _squeeze_trailing(a)


def _squeeze_trailing(a):
    while a.ndim > 2 and a.shape[-1] == 1:
        a = a.reshape(a.shape[:-1])
    return a


def _pad(a, nd):
    if a.ndim < nd:
        a = a.reshape(a.shape + (1,) * (nd - a.ndim))
    return a


def scalar(a):
    a = np.asarray(a)
    assert a.size == 1, f"expected a scalar, got shape {a.shape}"
    v = a.reshape(-1)[0]
    return v.item() if hasattr(v, "item") else v


def is_vector(a):
    return a.ndim == 2 and (a.shape[0] == 1 or a.shape[1] == 1) and a.size != 1


def truthy(a):
    if isinstance(a, str):
        return len(a) > 0
    a = np.asarray(a)
    return a.size > 0 and bool(np.all(a != 0))


def colmajor(a):
    return np.asarray(a).reshape(-1, order="F")


def _result_type(a, b):
    if a.dtype == np.int32 or b.dtype == np.int32:
        return np.int32
    return None


def _to_int32(x):
    r = np.where(x >= 0, np.floor(x + 0.5), np.ceil(x - 0.5))
    return np.clip(r, -2 ** 31, 2 ** 31 - 1).astype(np.int32)


def elementwise(fn, a, b):
    a = M(a)
    b = M(b)
    nd = max(a.ndim, b.ndim)
    x = _pad(a, nd)
    y = _pad(b, nd)
    xf = x.astype(np.float64) if x.dtype != np.bool_ else x
    yf = y.astype(np.float64) if y.dtype != np.bool_ else y
    with np.errstate(divide="ignore", invalid="ignore"):
        r = fn(xf.astype(np.float64), yf.astype(np.float64))
    rt = _result_type(a, b)
    if rt is np.int32 and r.dtype != np.bool_:
        r = _to_int32(r)
    return _squeeze_trailing(np.asarray(r))


def mtimes(a, b):
    a = M(a)
    b = M(b)
    if a.size == 1 or b.size == 1:
        return elementwise(np.multiply, a, b)
    assert a.ndim == 2 and b.ndim == 2, "matrix product of N-D arrays"
    return M(a.astype(np.float64) @ b.astype(np.float64))


def mrdivide(a, b):
    a = M(a)
    b = M(b)
    if b.size == 1:
        return elementwise(np.divide, a, b)
    raise NotImplementedError("matrix right division")


def mldivide(a, b):
    a = M(a)
    b = M(b)
    if a.size == 1:
        return elementwise(np.divide, b, a)
    return M(np.linalg.solve(a.astype(np.float64), b.astype(np.float64)))


def mpower(a, b):
    a = M(a)
    b = M(b)
    if a.size == 1 and b.size == 1:
        return elementwise(np.power, a, b)
    raise NotImplementedError("matrix power")


def transpose(a):
    a = M(a)
    if isinstance(a, str):
        return a
    assert a.ndim == 2, "transpose of an N-D array"
    return a.T.copy()


# ---------------------------------------------------------------------------
# indexing

class End:
    pass


def _subscript_to_index(s, extent):
    """One subscript -> 0-based integer array (1-D)."""
    if isinstance(s, slice):
        return np.arange(extent)
    s = np.asarray(s)
    if s.dtype == np.bool_:
        return np.nonzero(colmajor(s))[0]
    idx = colmajor(s).astype(np.int64) - 1
    if idx.size and idx.min() < 0:
        raise IndexError("index must be a positive integer")
    return idx


def index(a, subs):
    if isinstance(a, str):
        raise TypeError("indexing a string")
    a = M(a)
    if len(subs) == 1:
        s = subs[0]
        flat = colmajor(a)
        if isinstance(s, slice):
            return flat.reshape(-1, 1).copy()
        s = M(s)
        if s.dtype == np.bool_:
            if s.size > flat.size:
                raise IndexError("logical index too long")
            idx = np.nonzero(colmajor(s))[0]
            is_row = (s.ndim == 2 and s.shape[0] == 1 and s.size != 1) or (a.ndim == 2 and a.shape[0] == 1)
            out = flat[idx]
            return out.reshape(1, -1) if is_row and (is_vector(a) or a.size == 1) and a.shape[0] == 1 else out.reshape(-1, 1)
        idx = _subscript_to_index(s, flat.size)
        if idx.size and idx.max() >= flat.size:
            raise IndexError(f"index {idx.max() + 1} exceeds {flat.size} elements")
        out = flat[idx]
        if is_vector(a) and is_vector(s):
            return out.reshape(a.shape[0] if a.shape[1] == 1 else 1, -1) if a.shape[0] == 1 else out.reshape(-1, 1)
        return out.reshape(s.shape, order="F")
    nd = len(subs)
    shape = list(a.shape) + [1] * max(0, nd - a.ndim)
    if nd < a.ndim:  # fold trailing dimensions into the last subscript
        shape = list(a.shape[:nd - 1]) + [int(np.prod(a.shape[nd - 1:]))]
    b = a.reshape(shape, order="F")
    idxs = [_subscript_to_index(s, shape[k]) for k, s in enumerate(subs)]
    for k, ix in enumerate(idxs):
        if ix.size and ix.max() >= shape[k]:
            raise IndexError(f"index exceeds dimension {k + 1} ({shape[k]})")
    out = b[np.ix_(*idxs)]
    return _squeeze_trailing(out.reshape(out.shape) if out.ndim >= 2 else M(out))


def assign_index(a, subs, v):
    """a(subs) = v; returns the new array (grows with zeros when needed)."""
    v = M(v)
    if a is None:
        a = np.zeros((0, 0))
    a = M(a)
    if v.dtype == np.bool_ and a.dtype != np.bool_:
        v = v.astype(a.dtype)
    if a.dtype == np.bool_ and v.dtype != np.bool_:
        a = a.astype(np.float64)
    if a.dtype == np.int32 and v.dtype != np.int32:
        v = _to_int32(v.astype(np.float64))
    if v.dtype == np.int32 and a.dtype == np.float64:
        v = v.astype(np.float64)
    if len(subs) == 1:
        s = subs[0]
        flat = colmajor(a).copy()
        if isinstance(s, slice):
            idx = np.arange(flat.size)
        else:
            s = M(s)
            idx = np.nonzero(colmajor(s))[0] if s.dtype == np.bool_ else _subscript_to_index(s, flat.size)
        if idx.size and idx.max() >= flat.size:
            if a.size == 0 or is_vector(a) or a.size == 1:
                n = idx.max() + 1
                grown = np.zeros(n, dtype=flat.dtype)
                grown[:flat.size] = flat
                flat = grown
                row = a.size == 0 or a.shape[0] == 1
                a = flat.reshape(1, -1) if row else flat.reshape(-1, 1)
            else:
                raise IndexError("linear-index growth of a matrix")
        vals = colmajor(v)
        if vals.size == 1:
            flat[idx] = vals[0]
        else:
            if vals.size != idx.size:
                raise ValueError(f"assignment of {vals.size} values to {idx.size} elements")
            flat[idx] = vals
        return flat.reshape(a.shape, order="F")
    nd = len(subs)
    shape = list(a.shape) + [1] * max(0, nd - a.ndim)
    if nd < a.ndim:
        shape = list(a.shape[:nd - 1]) + [int(np.prod(a.shape[nd - 1:]))]
        folded = True
    else:
        folded = False
    b = a.reshape(shape, order="F").copy()
    idxs = []
    for k, s in enumerate(subs):
        ix = _subscript_to_index(s, shape[k])
        idxs.append(ix)
    need = [max(shape[k], (ix.max() + 1) if ix.size else 0) for k, ix in enumerate(idxs)]
    if need != shape:
        if folded:
            raise IndexError("growth of a folded array")
        nb = np.zeros(need, dtype=b.dtype)
        nb[tuple(slice(0, n) for n in shape)] = b
        b = nb
    target_shape = tuple(ix.size for ix in idxs)
    vals = colmajor(v)
    if vals.size == 1:
        b[np.ix_(*idxs)] = vals[0]
    else:
        if vals.size != int(np.prod(target_shape)):
            raise ValueError(f"assignment of {vals.size} values into {target_shape}")
        b[np.ix_(*idxs)] = vals.reshape(target_shape, order="F")
    if folded:
        return b.reshape(a.shape, order="F")
    return _squeeze_trailing(b)


# ---------------------------------------------------------------------------
# builtins

def _dims_args(args):
    dims = []
    for x in args:
        if isinstance(x, str):
            continue
        x = M(x)
        dims += [int(v) for v in colmajor(x)]
    if len(dims) == 1:
        dims = [dims[0], dims[0]]
    return dims


def b_zeros(*args):
    cls = [x for x in args if isinstance(x, str)]
    d = _dims_args(args) if any(not isinstance(x, str) for x in args) else [1, 1]
    return _squeeze_trailing(np.zeros(d, dtype=np.int32 if "int32" in cls else np.float64))


def b_ones(*args):
    d = _dims_args(args) if args else [1, 1]
    return _squeeze_trailing(np.ones(d))


def b_false(*args):
    d = _dims_args(args) if args else [1, 1]
    return _squeeze_trailing(np.zeros(d, dtype=np.bool_))


def b_true(*args):
    d = _dims_args(args) if args else [1, 1]
    return _squeeze_trailing(np.ones(d, dtype=np.bool_))


def b_eye(*args):
    d = _dims_args(args) if args else [1, 1]
    return np.eye(d[0], d[1])


def b_size(a, dim=None):
    a = M(a)
    if dim is None:
        return M(np.array([a.shape], dtype=np.float64))
    d = int(scalar(dim))
    return M(float(a.shape[d - 1]) if d <= a.ndim else 1.0)


def b_numel(a):
    return M(float(np.asarray(a).size))


def b_reshape(a, *dims):
    a = M(a)
    if len(dims) == 1:
        ds = [int(v) for v in colmajor(M(dims[0]))]
    else:
        ds = []
        for d in dims:
            d = M(d)
            ds.append(None if d.size == 0 else int(scalar(d)))
    if None in ds:
        known = int(np.prod([d for d in ds if d is not None]))
        ds[ds.index(None)] = a.size // known if known else 0
    return _squeeze_trailing(colmajor(a).reshape(ds, order="F"))


def b_permute(a, order):
    a = M(a)
    o = [int(v) - 1 for v in colmajor(M(order))]
    a = _pad(a, len(o))
    return _squeeze_trailing(np.transpose(a, o))


def b_repmat(a, *reps):
    a = M(a)
    r = _dims_args(reps) if len(reps) > 1 or M(reps[0]).size > 1 else [int(scalar(reps[0]))] * 2
    nd = max(a.ndim, len(r))
    return _squeeze_trailing(np.tile(_pad(a, nd), r + [1] * (nd - len(r))))


def b_cat(dim, *arrs):
    d = int(scalar(dim))
    arrs = [M(x) for x in arrs if not (M(x).size == 0 and M(x).ndim == 2 and M(x).shape == (0, 0))]
    if not arrs:
        return np.zeros((0, 0))
    nd = max(d, max(x.ndim for x in arrs))
    arrs = [_pad(x, nd) for x in arrs]
    dt = np.result_type(*[x.dtype for x in arrs])
    return _squeeze_trailing(np.concatenate([x.astype(dt) for x in arrs], axis=d - 1))


def b_find(a):
    a = M(a)
    idx = np.nonzero(colmajor(a))[0].astype(np.float64) + 1
    if a.ndim == 2 and a.shape[0] == 1 and a.shape[1] != 1:
        return idx.reshape(1, -1)
    return idx.reshape(-1, 1)


def _pages(a):
    a = M(a).astype(np.float64)
    nd = max(a.ndim, 3)
    a = _pad(a, nd)
    return a


def b_pagemtimes(*args):
    if len(args) == 2:
        A, B, ta, tb = args[0], args[1], "none", "none"
    else:
        A, ta, B, tb = args
    A = _pages(A)
    B = _pages(B)
    nd = max(A.ndim, B.ndim)
    A = _pad(A, nd)
    B = _pad(B, nd)
    if ta == "transpose":
        A = np.swapaxes(A, 0, 1)
    if tb == "transpose":
        B = np.swapaxes(B, 0, 1)
    Am = np.moveaxis(A, (0, 1), (-2, -1))
    Bm = np.moveaxis(B, (0, 1), (-2, -1))
    R = np.matmul(Am, Bm)
    return _squeeze_trailing(np.moveaxis(R, (-2, -1), (0, 1)))


def b_pagetranspose(A):
    A = _pages(A)
    return _squeeze_trailing(np.swapaxes(A, 0, 1).copy())


def b_pagemldivide(A, B):
    A = _pages(A)
    B = _pages(B)
    nd = max(A.ndim, B.ndim)
    A = _pad(A, nd)
    B = _pad(B, nd)
    Am = np.moveaxis(A, (0, 1), (-2, -1))
    Bm = np.moveaxis(B, (0, 1), (-2, -1))
    shape = np.broadcast_shapes(Am.shape[:-2], Bm.shape[:-2])
    Am = np.broadcast_to(Am, shape + Am.shape[-2:])
    Bm = np.broadcast_to(Bm, shape + Bm.shape[-2:])
    if int(np.prod(shape)) == 0:
        R = np.zeros(shape + (Am.shape[-1], Bm.shape[-1]))
    else:
        R = np.linalg.solve(Am, Bm)
    return _squeeze_trailing(np.moveaxis(R, (-2, -1), (0, 1)))


def b_pageinv(A):
    A = _pages(A)
    Am = np.moveaxis(A, (0, 1), (-2, -1))
    return _squeeze_trailing(np.moveaxis(np.linalg.inv(Am), (-2, -1), (0, 1)))


def b_accumarray(subs, vals, sz=None):
    s = colmajor(M(subs)).astype(np.int64) - 1
    v = colmajor(M(vals)).astype(np.float64)
    n = int(s.max() + 1) if s.size else 0
    if sz is not None:
        n = max(n, int(colmajor(M(sz))[0]))
    out = np.zeros(n)
    for i, k in enumerate(s):  # MATLAB sums in index order
        out[k] += v[i] if v.size > 1 else v[0]
    return out.reshape(-1, 1)


def _dim_arg(a, dim):
    if dim is None:
        sh = M(a).shape
        return next((k for k, n in enumerate(sh) if n != 1), 0)
    return int(scalar(dim)) - 1


def b_vecnorm(a, p=2, dim=None):
    a = M(a).astype(np.float64)
    k = _dim_arg(a, dim)
    a = _pad(a, k + 1)
    return _squeeze_trailing(np.sqrt(np.sum(a * a, axis=k, keepdims=True)))


def b_norm(a, p=2):
    a = M(a).astype(np.float64)
    assert is_vector(a) or a.size <= 1, "matrix norm"
    return M(float(np.sqrt(np.sum(a * a))))


def b_cross(a, b, dim=None):
    a = M(a).astype(np.float64)
    b = M(b).astype(np.float64)
    nd = max(a.ndim, b.ndim)
    a = _pad(a, nd)
    b = _pad(b, nd)
    k = int(scalar(dim)) - 1 if dim is not None else next(i for i, n in enumerate(a.shape) if n == 3)
    a, b = np.broadcast_arrays(a, b)
    a0, a1, a2 = [np.take(a, i, axis=k) for i in range(3)]
    b0, b1, b2 = [np.take(b, i, axis=k) for i in range(3)]
    r = np.stack([a1 * b2 - a2 * b1, a2 * b0 - a0 * b2, a0 * b1 - a1 * b0], axis=k)
    return _squeeze_trailing(r)


def b_dot(a, b, dim=None):
    a = M(a).astype(np.float64)
    b = M(b).astype(np.float64)
    nd = max(a.ndim, b.ndim)
    a = _pad(a, nd)
    b = _pad(b, nd)
    k = _dim_arg(a, dim)
    return _squeeze_trailing(np.sum(a * b, axis=k, keepdims=True))


def b_min(a, b=None, dim=None):
    if b is not None and not (isinstance(b, np.ndarray) and b.size == 0 and dim is not None):
        return elementwise(np.minimum, a, b)
    a = M(a)
    return _squeeze_trailing(np.min(a, axis=_dim_arg(a, dim), keepdims=True))


def b_max(a, b=None, dim=None):
    if b is not None and not (isinstance(b, np.ndarray) and b.size == 0 and dim is not None):
        return elementwise(np.maximum, a, b)
    a = M(a)
    return _squeeze_trailing(np.max(a, axis=_dim_arg(a, dim), keepdims=True))


def b_sum(a, dim=None):
    a = M(a).astype(np.float64)
    return _squeeze_trailing(np.sum(a, axis=_dim_arg(a, dim), keepdims=True))


def b_any(a):
    return M(bool(np.any(M(a) != 0)))


def b_all(a):
    return M(bool(np.all(M(a) != 0)))


def b_unary(fn):
    return lambda a: _squeeze_trailing(fn(M(a).astype(np.float64)))


def b_isnan(a):
    return _squeeze_trailing(np.isnan(M(a).astype(np.float64)))


def b_assert(cond, *msg):
    if not truthy(cond):
        raise AssertionError("assert failed in reference code")
    return None


def b_disp(x):
    print("[mlite disp]", x if isinstance(x, str) else np.asarray(x).ravel()[:8])
    return None


_T0 = time.perf_counter()


def b_tic():
    return M(time.perf_counter())


def b_toc(t=None):
    return M(time.perf_counter() - (scalar(t) if t is not None else _T0))


def b_int32(a):
    return _to_int32(M(a).astype(np.float64))


def b_double(a):
    return M(a).astype(np.float64)


def b_logical(a):
    return M(a) != 0


def b_isempty(a):
    return M(np.asarray(a).size == 0)


def b_floor(a):
    return _squeeze_trailing(np.floor(M(a).astype(np.float64)))


BUILTINS = {
    "zeros": b_zeros, "ones": b_ones, "eye": b_eye, "false": b_false, "true": b_true, "size": b_size,
    "numel": b_numel, "reshape": b_reshape, "permute": b_permute, "repmat": b_repmat, "cat": b_cat,
    "find": b_find, "pagemtimes": b_pagemtimes, "pagetranspose": b_pagetranspose,
    "pagemldivide": b_pagemldivide, "pageinv": b_pageinv, "accumarray": b_accumarray, "vecnorm": b_vecnorm,
    "norm": b_norm, "cross": b_cross, "dot": b_dot, "min": b_min, "max": b_max, "sum": b_sum, "any": b_any,
    "all": b_all, "abs": b_unary(np.abs), "sqrt": b_unary(np.sqrt), "sin": b_unary(np.sin),
    "cos": b_unary(np.cos), "isnan": b_isnan, "assert": b_assert, "disp": b_disp, "tic": b_tic, "toc": b_toc,
    "int32": b_int32, "double": b_double, "logical": b_logical, "isempty": b_isempty, "floor": b_floor,
}

# ---------------------------------------------------------------------------
# lexer

TOKEN_RE = re.compile(r"""
    (?P<cont>\.\.\.[^\n]*\n)
  | (?P<comment>%[^\n]*)
  | (?P<nl>\n)
  | (?P<ws>[ \t\r]+)
  | (?P<num>(?:\d+(?:\.(?![*/\\^'])\d*)?|\.\d+)(?:[eE][+-]?\d+)?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<str>"[^"\n]*")
  | (?P<op>\.\*|\./|\.\\|\.\^|\.'|==|~=|<=|>=|&&|\|\||[-+*/\\^'<>=&|~!:,;()\[\]{}.@])
""", re.X)

KEYWORDS = {"function", "end", "if", "elseif", "else", "for", "while", "break", "continue", "return",
            "classdef", "methods", "properties", "switch", "case", "otherwise", "try", "catch", "parfor"}


def tokenize(src):
    """Tokens (kind, text, followed_by_space).  Newlines inside [] become row
    separators and are dropped inside () and {}; a quote after a value is a
    transpose, elsewhere it opens a char array."""
    toks = []
    stack = []
    pos = 0
    while pos < len(src):
        if src[pos] == "'":
            prev = toks[-1] if toks else None
            value_like = prev is not None and (
                prev[0] in ("num", "str") or (prev[0] == "id" and (prev[1] not in KEYWORDS or prev[1] == "end"))
                or prev[1] in (")", "]", "}", "'", ".'"))
            if not value_like or (prev[2] and stack and stack[-1] == "["):
                j = pos + 1
                s = ""
                while True:
                    k = src.index("'", j)
                    s += src[j:k]
                    if k + 1 < len(src) and src[k + 1] == "'":
                        s += "'"
                        j = k + 2
                        continue
                    pos = k + 1
                    break
                toks.append(("str", s, False))
                continue
        m = TOKEN_RE.match(src, pos)
        if not m:
            raise SyntaxError(f"cannot tokenize at {src[pos:pos + 30]!r}")
        kind = m.lastgroup
        text = m.group(kind)
        pos = m.end()
        if kind in ("cont", "comment"):
            continue
        if kind == "ws":
            if toks:
                toks[-1] = (toks[-1][0], toks[-1][1], True)
            continue
        if kind == "str":
            toks.append(("str", text[1:-1], False))
            continue
        if kind == "nl":
            if not stack:
                toks.append(("nl", "\n", False))
            elif stack[-1] == "[":
                toks.append(("op", ";", False))
            continue
        if kind == "op":
            if text in ("(", "[", "{"):
                stack.append(text)
            elif text in (")", "]", "}"):
                stack.pop()
        toks.append((kind, text, False))
    toks.append(("nl", "\n", False))
    toks.append(("eof", "", False))
    return toks


# ---------------------------------------------------------------------------
# parser (AST as tuples)


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0
        self.in_index = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def accept(self, text):
        if self.peek()[1] == text and self.peek()[0] != "str":
            self.i += 1
            return True
        return False

    def expect(self, text):
        tok = self.next()
        if tok[1] != text:
            raise SyntaxError(f"expected {text!r}, got {tok[1]!r} near token {self.i}")
        return tok

    def skip_nl(self):
        while self.peek()[0] == "nl" or self.peek()[1] in (";", ","):
            self.i += 1

    # ---- statements
    def block(self, terminators):
        body = []
        while True:
            self.skip_nl()
            tok = self.peek()
            if tok[0] == "eof" or (tok[0] == "id" and tok[1] in terminators):
                return body
            body.append(self.statement())

    def statement(self):
        tok = self.peek()
        kw = tok[1] if tok[0] == "id" else None
        if kw == "if":
            self.next()
            clauses = []
            cond = self.expr()
            body = self.block({"elseif", "else", "end"})
            clauses.append((cond, body))
            orelse = []
            while True:
                t = self.next()[1]
                if t == "elseif":
                    cond = self.expr()
                    clauses.append((cond, self.block({"elseif", "else", "end"})))
                elif t == "else":
                    orelse = self.block({"end"})
                elif t == "end":
                    break
            return ("if", clauses, orelse)
        if kw in ("for", "parfor"):
            self.next()
            paren = self.accept("(")
            var = self.next()[1]
            self.expect("=")
            rng = self.expr()
            if paren:
                self.expect(")")
            body = self.block({"end"})
            self.expect("end")
            return ("for", var, rng, body)
        if kw == "while":
            self.next()
            cond = self.expr()
            body = self.block({"end"})
            self.expect("end")
            return ("while", cond, body)
        if kw in ("break", "continue", "return"):
            self.next()
            return (kw,)
        # assignment or expression
        start = self.i
        if tok[1] == "[":
            # try multiple assignment [a, ~, b] = ...
            j = self.i
            depth = 0
            while True:
                tt = self.t[j]
                if tt[1] in ("[", "(", "{"):
                    depth += 1
                elif tt[1] in ("]", ")", "}"):
                    depth -= 1
                    if depth == 0:
                        break
                j += 1
            if self.t[j + 1][1] == "=" and self.t[j + 2][1] != "=":
                self.next()
                targets = []
                while not self.accept("]"):
                    if self.accept(","):
                        continue
                    if self.accept("~"):
                        targets.append(None)
                    else:
                        targets.append(self.postfix())
                self.expect("=")
                rhs = self.expr()
                return ("massign", targets, rhs)
        lhs = self.expr()
        if self.peek()[1] == "=" and self.peek()[0] == "op":
            self.next()
            rhs = self.expr()
            return ("assign", lhs, rhs)
        return ("expr", lhs)

    # ---- expressions (precedence climbing)
    def expr(self):
        return self.oror()

    def oror(self):
        a = self.andand()
        while self.peek()[1] == "||":
            self.next()
            a = ("bin", "||", a, self.andand())
        return a

    def andand(self):
        a = self.orop()
        while self.peek()[1] == "&&":
            self.next()
            a = ("bin", "&&", a, self.orop())
        return a

    def orop(self):
        a = self.andop()
        while self.peek()[1] == "|":
            self.next()
            a = ("bin", "|", a, self.andop())
        return a

    def andop(self):
        a = self.cmp()
        while self.peek()[1] == "&":
            self.next()
            a = ("bin", "&", a, self.cmp())
        return a

    def cmp(self):
        a = self.rng()
        while self.peek()[1] in ("==", "~=", "<", "<=", ">", ">=") and self.peek()[0] == "op":
            op = self.next()[1]
            a = ("bin", op, a, self.rng())
        return a

    def rng(self):
        if self.in_index and self.peek()[1] == ":" and self.peek(1)[1] in (",", ")"):
            self.next()
            return ("colon_all",)
        a = self.add()
        if self.peek()[1] == ":" and self.peek()[0] == "op":
            self.next()
            b = self.add()
            if self.peek()[1] == ":" and self.peek()[0] == "op":
                self.next()
                c = self.add()
                return ("range", a, b, c)
            return ("range", a, None, b)
        return a

    def add(self):
        a = self.mul()
        while self.peek()[1] in ("+", "-") and self.peek()[0] == "op":
            if self.in_matrix and self.t[self.i - 1][2] and not self.peek()[2]:
                break  # "[a -b]": a new element
            op = self.next()[1]
            a = ("bin", op, a, self.mul())
        return a

    in_matrix = 0

    def mul(self):
        a = self.unary()
        while self.peek()[1] in ("*", "/", "\\", ".*", "./", ".\\") and self.peek()[0] == "op":
            op = self.next()[1]
            a = ("bin", op, a, self.unary())
        return a

    def unary(self):
        if self.peek()[1] in ("-", "+", "~", "!") and self.peek()[0] == "op":
            op = self.next()[1]
            return ("un", op, self.unary())
        return self.power()

    def power(self):
        a = self.postfix()
        while self.peek()[1] in ("^", ".^") and self.peek()[0] == "op":
            op = self.next()[1]
            if self.peek()[1] in ("-", "+") and self.peek()[0] == "op":
                sign = self.next()[1]
                b = ("un", sign, self.postfix())
            else:
                b = self.postfix()
            a = ("bin", op, a, b)
        return a

    def postfix(self):
        a = self.primary()
        while True:
            tok = self.peek()
            if tok[1] == "(" and tok[0] == "op" and not (self.in_matrix and self.t[self.i - 1][2]):
                self.next()
                args = self.args(")")
                a = ("call", a, args)
            elif tok[1] == "." and tok[0] == "op" and self.peek(1)[0] == "id":
                self.next()
                name = self.next()[1]
                a = ("field", a, name)
            elif tok[1] in ("'", ".'") and tok[0] == "op":
                self.next()
                a = ("transpose", a)
            else:
                return a

    def args(self, close):
        args = []
        self.in_index += 1
        saved = self.in_matrix
        self.in_matrix = 0
        while not self.accept(close):
            if self.accept(","):
                continue
            args.append(self.expr())
        self.in_index -= 1
        self.in_matrix = saved
        return args

    def primary(self):
        tok = self.next()
        if tok[0] == "num":
            return ("num", float(tok[1]))
        if tok[0] == "str":
            return ("str", tok[1])
        if tok[0] == "id":
            if tok[1] == "end" and self.in_index:
                return ("end",)
            return ("id", tok[1])
        if tok[1] == "(":
            saved = self.in_matrix
            self.in_matrix = 0
            saved_idx = self.in_index
            self.in_index = 0
            e = self.expr()
            self.in_index = saved_idx
            self.in_matrix = saved
            self.expect(")")
            return ("paren", e)
        if tok[1] == "[":
            rows = [[]]
            saved_idx = self.in_index
            self.in_index = 0
            self.in_matrix += 1
            while True:
                t = self.peek()
                if t[1] == "]":
                    self.next()
                    break
                if t[1] == ";" or t[0] == "nl":
                    self.next()
                    rows.append([])
                    continue
                if t[1] == ",":
                    self.next()
                    continue
                rows[-1].append(self.expr())
            self.in_matrix -= 1
            self.in_index = saved_idx
            return ("matrix", [r for r in rows if r])
        raise SyntaxError(f"unexpected token {tok[1]!r}")


# ---------------------------------------------------------------------------
# function extraction from files


def _find_function(src, name):
    toks = tokenize(src)
    for i, t in enumerate(toks):
        if t[0] == "id" and t[1] == "function":
            # function [outs] = name(args) | function out = name(args) | function name(args)
            j = i + 1
            k = j
            while toks[k][0] != "nl" and not (toks[k][0] == "id" and toks[k][1] == name and toks[k + 1][1] in ("(", "\n")):
                k += 1
            if toks[k][0] == "id" and toks[k][1] == name:
                return toks, i
    raise KeyError(f"function {name} not found")


def parse_function(src, name):
    toks, i = _find_function(src, name)
    p = Parser(toks)
    p.i = i + 1
    outs = []
    if p.peek()[1] == "[":
        p.next()
        while not p.accept("]"):
            if p.accept(","):
                continue
            outs.append(p.next()[1])
        p.expect("=")
    elif p.peek(1)[1] == "=":
        outs.append(p.next()[1])
        p.expect("=")
    fname = p.next()[1]
    assert fname == name
    args = []
    if p.accept("("):
        while not p.accept(")"):
            if p.accept(","):
                continue
            args.append(p.next()[1])
    body = p.block({"end", "function"})
    return {"name": name, "outs": outs, "args": args, "body": body}


# ---------------------------------------------------------------------------
# interpreter

class _Return(Exception):
    pass


class _Break(Exception):
    pass


class _Continue(Exception):
    pass


class Interpreter:
    """Runs functions of a MATLAB source tree.  `table` maps a callable name
    ("xpbdLayer3D.projectGS" or "expRodrigues") to (file, function name)."""

    def __init__(self, root, table):
        self.root = Path(root)
        self.table = table
        self.cache = {}
        self.calls = 0

    def function(self, qualname):
        if qualname not in self.cache:
            file, fname = self.table[qualname]
            self.cache[qualname] = parse_function((self.root / file).read_text(), fname)
        return self.cache[qualname]

    def call(self, qualname, args, nargout=1):
        self.calls += 1
        if qualname in BUILTINS:
            r = BUILTINS[qualname](*args)
            return [r] if nargout <= 1 else list(r)
        f = self.function(qualname)
        env = {}
        if len(args) > len(f["args"]):
            raise TypeError(f"{qualname}: too many arguments")
        for n, v in zip(f["args"], args):
            env[n] = v
        env["__nargin__"] = len(args)
        try:
            self.run(f["body"], env)
        except _Return:
            pass
        outs = []
        for k in range(max(nargout, 1) if f["outs"] else 0):
            if k >= len(f["outs"]):
                raise TypeError(f"{qualname}: too many outputs requested")
            n = f["outs"][k]
            if n not in env:
                if k < nargout:
                    raise NameError(f"{qualname}: output {n} not set")
                outs.append(None)
            else:
                outs.append(env[n])
        return outs

    def callable_name(self, node, env):
        if node[0] == "id" and node[1] not in env:
            return node[1]
        if node[0] == "field" and node[1][0] == "id" and node[1][1] not in env:
            return f"{node[1][1]}.{node[2]}"
        if node[0] == "field" and node[1][0] == "field":
            inner = self.callable_name(node[1], env)
            return f"{inner}.{node[2]}" if inner else None
        return None

    # ---- statements
    def run(self, body, env):
        for st in body:
            self.stmt(st, env)

    def stmt(self, st, env):
        k = st[0]
        if k == "expr":
            e = st[1]
            fn = e[1] if e[0] == "call" else e
            name = self.callable_name(fn, env) if fn[0] in ("id", "field") else None
            if name and name.startswith("coder."):
                return
            if name and (name in self.table or name in BUILTINS):
                args = [self.eval(a, env) for a in e[2]] if e[0] == "call" else []
                if name in BUILTINS:
                    BUILTINS[name](*args)
                else:
                    self.call(name, args, nargout=0)
                return
            self.eval(e, env)
        elif k == "assign":
            self.assign(st[1], self.eval(st[2], env, nargout=1), env)
        elif k == "massign":
            targets, rhs = st[1], st[2]
            vals = self.eval(rhs, env, nargout=len(targets))
            if not isinstance(vals, list):
                vals = [vals]
            for tgt, v in zip(targets, vals):
                if tgt is not None:
                    self.assign(tgt, v, env)
        elif k == "if":
            for cond, body in st[1]:
                if truthy(self.eval(cond, env)):
                    self.run(body, env)
                    return
            self.run(st[2], env)
        elif k == "for":
            rng = M(self.eval(st[2], env))
            cols = rng.reshape(rng.shape[0], -1, order="F") if rng.size else np.zeros((1, 0))
            for j in range(cols.shape[1]):
                env[st[1]] = M(cols[:, j].reshape(-1, 1)) if cols.shape[0] > 1 else M(cols[0, j])
                try:
                    self.run(st[3], env)
                except _Break:
                    break
                except _Continue:
                    continue
        elif k == "while":
            while truthy(self.eval(st[1], env)):
                try:
                    self.run(st[2], env)
                except _Break:
                    break
                except _Continue:
                    continue
        elif k == "break":
            raise _Break()
        elif k == "continue":
            raise _Continue()
        elif k == "return":
            raise _Return()
        else:
            raise NotImplementedError(k)

    def assign(self, tgt, v, env):
        if tgt[0] == "id":
            env[tgt[1]] = v
        elif tgt[0] == "call" and tgt[1][0] == "id":
            name = tgt[1][1]
            cur = env.get(name)
            subs = [self.eval_sub(s, cur, k, len(tgt[2]), env) for k, s in enumerate(tgt[2])]
            env[name] = assign_index(cur, subs, v)
        else:
            raise NotImplementedError(f"assignment target {tgt[0]}")

    # ---- expressions
    def eval_sub(self, node, arr, k, n, env):
        if node[0] == "colon_all":
            return slice(None)
        saved = getattr(self, "_end_ctx", None)
        self._end_ctx = (arr, k, n)
        try:
            return self.eval(node, env)
        finally:
            self._end_ctx = saved

    def eval(self, node, env, nargout=1):
        k = node[0]
        if k == "num":
            return M(node[1])
        if k == "str":
            return node[1]
        if k == "paren":
            return self.eval(node[1], env)
        if k == "id":
            name = node[1]
            if name in env:
                return env[name]
            if name in ("pi",):
                return M(math.pi)
            if name in ("Inf", "inf"):
                return M(np.inf)
            if name in ("NaN", "nan"):
                return M(np.nan)
            r = self.call(name, [], nargout=max(nargout, 1))
            return r if nargout > 1 else r[0]
        if k == "end":
            arr, pos, n = self._end_ctx
            a = M(arr)
            if n == 1:
                return M(float(a.size))
            shape = list(a.shape) + [1] * max(0, n - a.ndim)
            if pos == n - 1 and n < a.ndim:
                return M(float(np.prod(a.shape[n - 1:])))
            return M(float(shape[pos]))
        if k == "matrix":
            rows = []
            for r in node[1]:
                vals = [self.eval(e, env) for e in r]
                vals = [v for v in vals if not (isinstance(v, np.ndarray) and v.shape == (0, 0))]
                rows.append(b_cat(2, *vals) if vals else np.zeros((0, 0)))
            rows = [r for r in rows if not (isinstance(r, np.ndarray) and r.shape == (0, 0))]
            return b_cat(1, *rows) if rows else np.zeros((0, 0))
        if k == "range":
            a = scalar(self.eval(node[1], env))
            step = scalar(self.eval(node[2], env)) if node[2] is not None else 1.0
            b = scalar(self.eval(node[3], env))
            n = int(math.floor((b - a) / step + 1e-10)) + 1 if step != 0 else 0
            return M(np.array([a + i * step for i in range(max(n, 0))], dtype=np.float64).reshape(1, -1))
        if k == "transpose":
            return transpose(self.eval(node[1], env))
        if k == "un":
            v = self.eval(node[2], env)
            if node[1] == "-":
                return elementwise(lambda x, y: -x, v, 0.0) if M(v).dtype != np.int32 else -M(v)
            if node[1] == "+":
                return v
            return _squeeze_trailing(M(v) == 0)
        if k == "bin":
            op = node[1]
            if op == "||":
                return M(truthy(self.eval(node[2], env)) or truthy(self.eval(node[3], env)))
            if op == "&&":
                return M(truthy(self.eval(node[2], env)) and truthy(self.eval(node[3], env)))
            a = self.eval(node[2], env)
            b = self.eval(node[3], env)
            return BINOPS[op](a, b)
        if k == "field":
            name = self.callable_name(node, env)
            if name is None:
                raise NotImplementedError("struct field access")
            if name.startswith("coder."):
                return None
            r = self.call(name, [], nargout=max(nargout, 1))
            return r if nargout > 1 else r[0]
        if k == "call":
            fn = node[1]
            if fn[0] == "id" and fn[1] in env:
                arr = env[fn[1]]
                subs = [self.eval_sub(s, arr, i, len(node[2]), env) for i, s in enumerate(node[2])]
                return index(arr, subs)
            name = self.callable_name(fn, env)
            if name is None:
                base = self.eval(fn, env)
                subs = [self.eval_sub(s, base, i, len(node[2]), env) for i, s in enumerate(node[2])]
                return index(base, subs)
            if name.startswith("coder."):
                return None
            args = [self.eval(a, env) for a in node[2]]
            r = self.call(name, args, nargout=max(nargout, 1))
            return r if nargout > 1 else r[0]
        raise NotImplementedError(k)


BINOPS = {
    "+": lambda a, b: elementwise(np.add, a, b),
    "-": lambda a, b: elementwise(np.subtract, a, b),
    ".*": lambda a, b: elementwise(np.multiply, a, b),
    "./": lambda a, b: elementwise(np.divide, a, b),
    ".\\": lambda a, b: elementwise(lambda x, y: y / x, a, b),
    ".^": lambda a, b: elementwise(np.power, a, b),
    "*": mtimes,
    "/": mrdivide,
    "\\": mldivide,
    "^": mpower,
    "==": lambda a, b: elementwise(np.equal, a, b),
    "~=": lambda a, b: elementwise(np.not_equal, a, b),
    "<": lambda a, b: elementwise(np.less, a, b),
    "<=": lambda a, b: elementwise(np.less_equal, a, b),
    ">": lambda a, b: elementwise(np.greater, a, b),
    ">=": lambda a, b: elementwise(np.greater_equal, a, b),
    "&": lambda a, b: elementwise(lambda x, y: (x != 0) & (y != 0), a, b),
    "|": lambda a, b: elementwise(lambda x, y: (x != 0) | (y != 0), a, b),
}


# The reference functions the layer solve reaches (file, function name).
LAYER_SOLVE_TABLE = {
    **{f"xpbdLayer3D.{n}": ("3d/integrator/xpbdLayer3D.m", n) for n in (
        "layerSolve", "projectGS", "stvkVoigtConstraints", "rigidElasticBoundaryAccumulationConstraints",
        "contactConstraints", "rotateAllVerts", "rotateResidual", "simpleMonitorError",
        "simpleEvaluateAllConstraintResiduals")},
    "matStvkVoigtConstraint3D": ("3d/constraints/matStvkVoigtConstraint3D.m", "matStvkVoigtConstraint3D"),
    "decomposeSolve": ("3d/constraints/matStvkVoigtConstraint3D.m", "decomposeSolve"),
    "StVKconstraintGrad3D": ("3d/constraints/StVKconstraintGrad3D.m", "StVKconstraintGrad3D"),
    "rigidBoundaryConstraint.project": ("3d/constraints/rigidBoundaryConstraint.m", "project"),
    "penaltyConstraint.projectElastic": ("3d/constraints/penaltyConstraint.m", "projectElastic"),
    "penaltyConstraint.projectRigid": ("3d/constraints/penaltyConstraint.m", "projectRigid"),
    "rigidGeneralizedInverseMass": ("3d/constraints/rigidGeneralizedInverseMass.m", "rigidGeneralizedInverseMass"),
    "AdaptiveMesh3D.makeRigidsFromConnectivity": ("3d/@AdaptiveMesh3D/AdaptiveMesh3D.m",
                                                  "makeRigidsFromConnectivity"),
    **{f"RigidBody3D.{n}": ("3d/@RigidBody3D/RigidBody3D.m", n) for n in (
        "rigidSymplecticImperativeStep", "pageRelativeVertexPosition", "matComputeRigidBodyProperties3D",
        "buildInertiaTensor")},
    "RigidBody.pageRelativeVertexPosition": ("2d/@RigidBody/RigidBody.m", "pageRelativeVertexPosition"),
    "expRodrigues": ("3d/tools/math/expRodrigues.m", "expRodrigues"),
    "crossProductMatrix": ("3d/tools/math/crossProductMatrix.m", "crossProductMatrix"),
    "formatPositions3D": ("3d/tools/functionalities/formatPositions3D.m", "formatPositions3D"),
    "pagePositions3D": ("3d/tools/functionalities/pagePositions3D.m", "pagePositions3D"),
    "BDF.BDF1": ("2d/tools/math/BDF.m", "BDF1"),
}
