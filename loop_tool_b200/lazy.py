"""Lazy tensors with symbolic shapes -- the host-side mirror of loop_tool's
lazy frontend (include/loop_tool/lazy.h, src/frontends/lazy.cpp) and of its
Python binding (src/frontends/python.cpp:338-560): lt.Symbol, lt.Expr,
lt.Size, lt.SymbolGenerator, lt.Tensor with to / [] / pad / | / transpose /
flatten / sum / max_reduce and the elementwise ops.

A tensor lowers to the reference's serialized IR (serialization.cpp:175-237)
with the reference's default schedule (lazy.cpp:90-126: every compute node
loops over its vars sorted by VarRef at full size) and runs on the B200
backend.  Compiled loop trees are cached by their IR text, which names vars
canonically, so structurally identical programs of equal sizes share one
compiled object (the role of TensorImpl::hash, lazy.h:82-115).

Views are lowered with explicit read-direction constraints: for every var of
a view's input the IR carries `input_var = f(output vars)` (solved here from
the user's constraints), which is the form Compiler::gen_index_equations
reads (compile.cpp:653-660), so the reference's CPU backends run the same
IR text with the same meaning.
"""
import itertools
import threading
from collections import OrderedDict

import numpy as np

from .backend import Compiled

_ids = itertools.count()

# symbolic::Op codes (symbolic.h:38-50)
E_NEG, E_RECIP, E_SIZE, E_MAX, E_ADD, E_MUL, E_DIV, E_MOD = 1, 2, 3, 4, 5, 6, 7, 8
# Operation codes (ir.h:21-39)
OPS = {n: i for i, n in enumerate(
    ["constant", "write", "read", "view", "copy", "add", "subtract", "multiply", "divide",
     "min", "max", "log", "exp", "sqrt", "abs", "negate", "reciprocal", "name"])}


class Symbol:
    """A named dimension (lazy::Symbol, symbolic.h:54-75)."""

    def __init__(self, name="X"):
        self.name = name
        self.id = next(_ids)

    def __repr__(self):
        return self.name

    def __hash__(self):
        return hash(self.id)

    def __eq__(self, other):
        return isinstance(other, Symbol) and other.id == self.id

    def _e(self):
        return Expr(("sym", self))

    def __add__(self, o):
        return self._e() + o

    __radd__ = __add__

    def __mul__(self, o):
        return self._e() * o

    __rmul__ = __mul__

    def __sub__(self, o):
        return self._e() - o


class Expr:
    """Index expression (symbolic::Expr): values, symbols, Size(symbol), + * / %."""

    def __init__(self, x):
        if isinstance(x, Expr):
            x = x.t
        elif isinstance(x, Symbol):
            x = ("sym", x)
        elif isinstance(x, (int, np.integer)):
            x = ("val", int(x))
        self.t = x

    @staticmethod
    def of(x):
        return x if isinstance(x, Expr) else Expr(x)

    def _bin(self, op, o):
        return Expr(("fn", op, self.t, Expr.of(o).t))

    def __add__(self, o):
        return self._bin(E_ADD, o)

    __radd__ = __add__

    def __mul__(self, o):
        return self._bin(E_MUL, o)

    __rmul__ = __mul__

    def __sub__(self, o):
        return self + Expr(("fn", E_NEG, Expr.of(o).t))

    def __floordiv__(self, o):
        return self._bin(E_DIV, o)

    def __mod__(self, o):
        return self._bin(E_MOD, o)

    def __repr__(self):
        return _dump(self.t)


def Size(sym):
    """lt.Size(sym) (python.cpp:366)."""
    return Expr(("size", sym))


class SymbolGenerator:
    """`with lt.SymbolGenerator() as s: s.N ...` (python.cpp:35-47)."""

    def __init__(self):
        self._syms = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if name not in self._syms:
            self._syms[name] = Symbol(name)
        return self._syms[name]


def _dump(t):
    k = t[0]
    if k == "val":
        return str(t[1])
    if k == "sym":
        return t[1].name
    if k == "size":
        return f"|{t[1].name}|"
    op = t[1]
    if op == E_NEG:
        return f"-({_dump(t[2])})"
    s = {E_ADD: "+", E_MUL: "*", E_DIV: "/", E_MOD: "%", E_MAX: " max "}.get(op, "?")
    return f"({_dump(t[2])}{s}{_dump(t[3])})"


# ------------------------------------------------------------- symbolic
def _syms(t, out):
    if t[0] in ("sym", "size"):
        if t[1] not in out:
            out.append(t[1])
    elif t[0] == "fn":
        for a in t[2:]:
            _syms(a, out)
    return out


def _eval(t, env):
    """Integer value with every symbol (and size) bound, else None."""
    k = t[0]
    if k == "val":
        return t[1]
    if k == "sym":
        return env.get(("v", t[1]))
    if k == "size":
        return env.get(("s", t[1]))
    args = [_eval(a, env) for a in t[2:]]
    if any(a is None for a in args):
        return None
    op = t[1]
    if op == E_ADD:
        return args[0] + args[1]
    if op == E_MUL:
        return args[0] * args[1]
    if op == E_NEG:
        return -args[0]
    if op == E_DIV:
        return int(args[0] / args[1]) if args[1] else None
    if op == E_MOD:
        return args[0] - int(args[0] / args[1]) * args[1] if args[1] else None
    if op == E_MAX:
        return max(args)
    return None


def _affine(t, sizes):
    """t as (coef by symbol, const), sizes substituted; None if not affine."""
    k = t[0]
    if k == "val":
        return {}, t[1]
    if k == "sym":
        return {t[1]: 1}, 0
    if k == "size":
        return ({}, sizes[t[1]]) if t[1] in sizes else None
    op = t[1]
    if op in (E_ADD, E_NEG, E_MUL):
        parts = [_affine(a, sizes) for a in t[2:]]
        if any(p is None for p in parts):
            return None
        if op == E_NEG:
            c, k0 = parts[0]
            return {s: -v for s, v in c.items()}, -k0
        if op == E_ADD:
            c = dict(parts[0][0])
            for s, v in parts[1][0].items():
                c[s] = c.get(s, 0) + v
            return c, parts[0][1] + parts[1][1]
        (ca, ka), (cb, kb) = parts
        if not ca:
            return {s: v * ka for s, v in cb.items()}, ka * kb
        if not cb:
            return {s: v * kb for s, v in ca.items()}, ka * kb
    return None


def _lin(coefs, const):
    """Expression tree of sum(coef * sym) + const."""
    t = ("val", const)
    for s, c in coefs.items():
        if c == 0:
            continue
        term = ("sym", s) if c == 1 else ("fn", E_MUL, ("val", c), ("sym", s))
        t = term if t == ("val", 0) else ("fn", E_ADD, t, term)
    return t


# ---------------------------------------------------------------- tensor
class Tensor:
    """lazy::Tensor (lazy.h:347-688) / lt.Tensor (python.cpp:376-560)."""

    def __init__(self, *args, data=None):
        self.op = "constant"
        self.deps = []
        self.constraints = []  # (lhs tree, rhs tree): lhs a symbol or size()
        self.data = None
        if len(args) == 1 and isinstance(args[0], np.ndarray):
            data = args[0]
            args = data.shape
        if args and all(isinstance(a, Symbol) for a in args):
            self.shape = list(args)
        else:
            self.shape = [Symbol() for _ in args]
            for s, n in zip(self.shape, args):
                self.constraints.append((("size", s), ("val", int(n))))
        if data is not None:
            self.set(data)

    @classmethod
    def _make(cls, op, shape, deps, constraints=()):
        t = cls.__new__(cls)
        t.op, t.shape, t.deps = op, list(shape), list(deps)
        t.constraints = list(constraints)
        t.data = None
        return t

    # data binding (python.cpp:538-547)
    def set(self, array):
        assert not self.deps, "cannot set data to a computed tensor"
        a = np.ascontiguousarray(np.asarray(array, dtype=np.float32))
        if len(a.shape) != len(self.shape):
            a = a.reshape([-1] * 0 + list(a.shape))
        known = {c[0][1]: c[1][1] for c in self.constraints if c[0][0] == "size"}
        for s, n in zip(self.shape, a.shape):
            if s in known:
                assert known[s] == n, f"already bound {s.name} to {known[s]}, got {n}"
            else:
                self.constraints.append((("size", s), ("val", int(n))))
        self.data = a
        return self

    # -- elementwise (broadcast by symbol identity, lazy.h:361-376)
    def _bshape(self, o):
        out = list(self.shape)
        for s in o.shape:
            if s not in out:
                out.append(s)
        return out

    def _bin(self, op, o):
        return Tensor._make(op, self._bshape(o), [self, o])

    def __add__(self, o):
        return self._bin("add", o)

    def __sub__(self, o):
        return self._bin("subtract", o)

    def __mul__(self, o):
        return self._bin("multiply", o)

    def __truediv__(self, o):
        return self._bin("divide", o)

    def max(self, o):
        return self._bin("max", o)

    def min(self, o):
        return self._bin("min", o)

    def _un(self, op):
        return Tensor._make(op, self.shape, [self])

    def exp(self):
        return self._un("exp")

    def log(self):
        return self._un("log")

    def sqrt(self):
        return self._un("sqrt")

    def abs(self):
        return self._un("abs")

    def reciprocal(self):
        return self._un("reciprocal")

    def __neg__(self):
        return self._un("negate")

    # -- reductions (lazy.h:561-601)
    def _reduce(self, op, syms):
        assert syms, "reduction variables required (got none)"
        shape = [s for s in self.shape if s not in syms]
        assert len(shape) != len(self.shape), "reduction variables not over any input"
        return Tensor._make(op, shape, [self])

    def sum(self, *syms):
        return self._reduce("add", list(syms))

    def max_reduce(self, *syms):
        return self._reduce("max", list(syms))

    def min_reduce(self, *syms):
        return self._reduce("min", list(syms))

    def prod(self, *syms):
        return self._reduce("multiply", list(syms))

    # -- views (lazy.h:627-641, python.cpp:454-517)
    def to(self, *shape, constraints=None):
        if not constraints:
            return self.as_(*shape)
        cs = []
        for lhs, rhs in constraints:
            lt_ = ("sym", lhs) if isinstance(lhs, Symbol) else Expr.of(lhs).t
            cs.append((lt_, Expr.of(rhs).t))
        return Tensor._make("view", shape, [self], cs)

    def as_(self, *shape):
        """Rename (Tensor::as, lazy.h:619-624): a view with no constraints
        whose vars match the input positionally."""
        assert len(shape) == len(self.shape), "rename must keep the rank"
        t = Tensor._make("name", shape, [self])
        return t

    def __getitem__(self, idx):
        if not isinstance(idx, tuple):
            idx = (idx,)
        if len(idx) != len(self.shape):
            raise IndexError(f"Expected shape of size {len(self.shape)} got {len(idx)}")
        out, cs = [], []
        for s, e in zip(self.shape, idx):
            e = Expr.of(e)
            for x in _syms(e.t, []):
                if x not in out:
                    out.append(x)
            cs.append((("sym", s), e.t))
        return Tensor._make("view", out, [self], cs)

    def pad(self, sym, pre, post=None):
        """Tensor::pad (lazy.h:481-502)."""
        post = pre if post is None else post
        assert pre >= 0 and post >= 0 and (pre or post)
        new = Symbol(f"{sym.name}_p_{pre}_{post}")
        shape = [new if s == sym else s for s in self.shape]
        return self.to(*shape, constraints=[(new, Expr(sym) + pre),
                                            (Size(new), Size(sym) + (pre + post))])

    def __or__(self, o):
        """Concatenation (lazy.h:460-479)."""
        assert len(self.shape) == len(o.shape)
        out, cs = [], []
        for a, b in zip(self.shape, o.shape):
            if a == b:
                out.append(a)
            else:
                n = Symbol(a.name + b.name)
                out.append(n)
                cs += [(n, Expr(a)), (n, Expr(b) + Size(a)), (Size(n), Size(a) + Size(b))]
        return self.to(*out, constraints=cs) + o.to(*out, constraints=cs)

    def transpose(self, *shape):
        assert sorted(s.id for s in shape) == sorted(s.id for s in self.shape)
        t = Tensor._make(self.op, shape, self.deps, self.constraints)
        t.data = self.data
        return t

    def flatten(self, *syms, new=None):
        """Tensor::flatten (lazy.h:517-559)."""
        new = new or Symbol("X")
        keep = [s for s in self.shape if s not in syms]
        e, run = Expr(0), Expr(1)
        for s in reversed(syms):
            e = Expr(s) * run + e
            run = Size(s) * run
        return self.to(*(keep + [new]), constraints=[(new, e)])

    # ------------------------------------------------------------ lowering
    def _collect(self):
        nodes, seen = [], set()

        def visit(t):
            if id(t) in seen:
                return
            seen.add(id(t))
            for d in t.deps:
                visit(d)
            nodes.append(t)
        visit(self)
        return nodes

    def _unify(self):
        """Symbol renames (as) and sizes from every constraint (the role of
        TensorImpl::unify, lazy.cpp:402-412)."""
        nodes = self._collect()
        parent = {}

        def find(s):
            while parent.get(s, s) != s:
                s = parent[s]
            return s
        for t in nodes:
            if t.op == "name":
                for a, b in zip(t.deps[0].shape, t.shape):
                    ra, rb = find(a), find(b)
                    if ra != rb:
                        parent[ra] = rb

        def canon_t(tr):
            if tr[0] in ("sym", "size"):
                return (tr[0], find(tr[1]))
            if tr[0] == "fn":
                return (tr[0], tr[1]) + tuple(canon_t(a) for a in tr[2:])
            return tr
        cons = []
        for t in nodes:
            for l, r in t.constraints:
                cons.append((canon_t(l), canon_t(r)))
        sizes = {}
        for _ in range(256):
            changed = False
            # explicit size constraints win over sizes implied by indexing
            for l, r in cons:
                env = {("s", s): n for s, n in sizes.items()}
                if l[0] == "size":
                    v = _eval(r, env)
                    if v is not None and l[1] not in sizes:
                        sizes[l[1]] = v
                        changed = True
            if changed:
                continue
            for l, r in cons:
                if changed:
                    break
                if l[0] == "sym":
                    aff = _affine(r, sizes)
                    if aff is None:
                        continue
                    coefs, c0 = aff
                    unknown = [s for s in coefs if s not in sizes]
                    if l[1] not in sizes and not unknown:
                        hi = c0 + sum(c * (sizes[s] - 1) for s, c in coefs.items() if c > 0)
                        sizes[l[1]] = hi + 1
                        changed = True
                    elif l[1] in sizes and len(unknown) == 1:
                        x = unknown[0]
                        cx = coefs[x]
                        rest = c0 + sum(c * (sizes[s] - 1) for s, c in coefs.items()
                                        if s != x and c > 0)
                        if cx > 0:
                            sizes[x] = (sizes[l[1]] - 1 - rest) // cx + 1
                            changed = True
            if not changed:
                break
        return nodes, find, canon_t, cons, sizes

    def _lower(self):
        nodes, find, canon_t, cons, sizes = self._unify()
        var_of, var_names = {}, []
        lines, node_of, inputs, leaves = [], {}, [], []

        def var(s):
            s = find(s)
            if s not in var_of:
                assert s in sizes, f"size for {s.name} could not be deduced"
                var_of[s] = len(var_names)
                var_names.append(f"{s.name}_{len(var_names)}")
            return var_of[s]

        node_rows = []  # (op code, inputs, vars, constraint text, symmap, order)

        def add_node(op, ins, vs, ctext="", smap="", order=None):
            node_rows.append((OPS[op], ins, vs, ctext, smap, order))
            return len(node_rows) - 1

        def resolve(t):
            if id(t) in node_of:
                return node_of[id(t)]
            if t.op == "name":
                nr = resolve(t.deps[0])
                node_of[id(t)] = nr
                return nr
            deps = [resolve(d) for d in t.deps]
            vs = [var(s) for s in t.shape]
            if t.op == "constant":
                nr = add_node("read", [], vs)
                inputs.append(nr)
                leaves.append(t)
            elif t.op == "view":
                nr = add_node("view", deps, vs, *self._view_constraints(t, find, canon_t, sizes, var))
            else:
                nr = add_node(t.op, deps, vs)
            node_of[id(t)] = nr
            return nr

        root = resolve(self)
        out = add_node("write", [root], [var(s) for s in self.shape])
        # default schedule (lazy.cpp:90-126): loop vars sorted, full sizes
        rows = []
        for i, (op, ins, vs, ctext, smap, _) in enumerate(node_rows):
            order = ""
            if op not in (OPS["read"], OPS["view"]):
                loop_vars = sorted(set(vs) | {v for x in ins for v in node_rows[x][2]})
                size_of = {var_of[s]: n for s, n in sizes.items() if s in var_of}
                order = "".join(f"{v};{size_of[v]};0," for v in loop_vars)
                annots = "," * len(loop_vars)
            else:
                annots = ""
            rows.append(f"n:{op}:{''.join(f'{x},' for x in ins)}:{''.join(f'{v},' for v in vs)}"
                        f":{ctext}:{smap}:0:{order}::{annots}::")
        text = "".join(f"v:{n}\n" for n in var_names) + "\n".join(rows) + "\n"
        text += "i:" + "".join(f"{x}," for x in inputs) + "\n"
        text += f"o:{out},\n"
        shape_sizes = [sizes[find(s)] for s in self.shape]
        return text, leaves, shape_sizes

    @staticmethod
    def _view_constraints(t, find, canon_t, sizes, var):
        """Read-direction constraints of a view: each input var as a function
        of the view's output vars, plus the sizes of all of them."""
        outs = [find(s) for s in t.shape]
        ins = [find(s) for s in t.deps[0].shape]
        eqs = []
        for l, r in t.constraints:
            l, r = canon_t(l), canon_t(r)
            if l[0] == "sym":
                eqs.append((l[1], r))
        exprs = {}
        for v in ins:
            if v in outs:
                continue  # same var on both sides: identity
            e = None
            for lhs, rhs in eqs:  # v = f(outputs)
                if lhs == v and all(s in outs for s in _vsyms(rhs)):
                    e = _resolve_sizes(rhs, sizes)
                    break
            if e is None:
                for lhs, rhs in eqs:  # out = a*v + g(outputs): v = (out - g) / a
                    if lhs not in outs:
                        continue
                    aff = _affine(rhs, sizes)
                    if aff is None or v not in aff[0]:
                        continue
                    coefs, c0 = aff
                    others = {s: c for s, c in coefs.items() if s != v}
                    if all(s in outs for s in others):
                        a = coefs[v]
                        num = ("fn", E_ADD, ("sym", lhs),
                               ("fn", E_NEG, _lin(others, c0)))
                        e = num if a == 1 else ("fn", E_DIV, num, ("val", a))
                        break
                    # flatten: out = sum c_i * in_i (all inputs): mixed radix
                    if all(s in ins for s in coefs) and len(coefs) > 1:
                        base = ("fn", E_ADD, ("sym", lhs), ("val", -c0)) if c0 else ("sym", lhs)
                        e = ("fn", E_DIV, base, ("val", coefs[v]))
                        if coefs[v] != max(coefs.values()):
                            e = ("fn", E_MOD, e, ("val", sizes[v]))
                        break
            if e is not None:
                exprs[v] = e
        # serialize: one constraint per mapped input var, then sizes
        body, sym_idx, idx = [], {}, [0]

        def ser(tr):
            toks = []

            def emit(x):
                if x[0] == "val":
                    toks.append(f"0|v|{x[1]}|")
                    idx[0] += 1
                    return idx[0] - 1
                if x[0] == "sym":
                    s = x[1]
                    if s in sym_idx:
                        toks.append(f"0|r|{sym_idx[s]}|")
                        idx[0] += 1
                        return sym_idx[s]
                    sym_idx[s] = idx[0]
                    toks.append(f"0|s|{s.name}|")
                    idx[0] += 1
                    return sym_idx[s]
                if x[0] == "size":
                    a = emit(("sym", x[1]))
                    toks.append(f"{E_SIZE}|f|{a},|")
                    idx[0] += 1
                    return idx[0] - 1
                args = [emit(a) for a in x[2:]]
                toks.append(f"{x[1]}|f|{''.join(f'{a},' for a in args)}|")
                idx[0] += 1
                return idx[0] - 1
            emit(tr)
            return "".join(f"{t_};" for t_ in toks)

        for v, e in exprs.items():
            body.append(ser(("sym", v)) + "=" + ser(e))
        for s in outs + [x for x in ins if x not in outs]:
            body.append(ser(("size", s)) + "=" + ser(("val", sizes[s])))
        smap = "".join(f"{i}={var(s)}," for s, i in sym_idx.items())
        return "".join(f"{b}/" for b in body), smap

    # ------------------------------------------------------------- running
    def compile(self, **opts):
        text, _, _ = self._lower()
        return compiled(text, **opts)

    @property
    def ir(self):
        return self._lower()[0]

    loop_tree = ir  # the serialized IR is the loop tree (ir.cpp:531)

    @property
    def code(self):
        return self.compile().code

    @property
    def symbolic_shape(self):
        return list(self.shape)

    @property
    def shape_sizes(self):
        return self._lower()[2]

    def numpy(self, **opts):
        """Tensor.numpy (python.cpp:548-560): compile (cached) and run."""
        if self.op == "constant" and self.data is not None:
            return self.data
        text, leaves, out_sizes = self._lower()
        c = compiled(text, **opts)
        for lf in leaves:
            assert lf.data is not None, "an input tensor has no data bound"
        out = np.empty(out_sizes, np.float32)
        c([lf.data for lf in leaves] + [out])
        return out

    def resolve(self, **opts):
        self.numpy(**opts)


def _vsyms(t, out=None):
    """Symbols used as values (not only inside size())."""
    out = [] if out is None else out
    if t[0] == "sym":
        if t[1] not in out:
            out.append(t[1])
    elif t[0] == "fn":
        for a in t[2:]:
            _vsyms(a, out)
    return out


def _resolve_sizes(t, sizes):
    if t[0] == "size":
        return ("val", sizes[t[1]])
    if t[0] == "fn":
        return (t[0], t[1]) + tuple(_resolve_sizes(a, sizes) for a in t[2:])
    return t


# ------------------------------------------------------------ kernel cache
_CACHE = OrderedDict()
_CACHE_MAX = 4096
_CACHE_LOCK = threading.Lock()  # serving threads share the cache


def compiled(ir_text, **opts):
    """Compiled loop tree for an IR text, reused across calls (the
    compilation cache of lazy.cpp:12-21, keyed by IR text + options).
    Thread-safe: concurrent callers of one key get one compiled object."""
    key = (ir_text, tuple(sorted(opts.items())))
    with _CACHE_LOCK:
        c = _CACHE.get(key)
        if c is not None:
            _CACHE.move_to_end(key)
            return c
        c = Compiled(ir_text, **opts)
        _CACHE[key] = c
        if len(_CACHE) > _CACHE_MAX:
            _CACHE.popitem(last=False)
        return c


def cache_info():
    with _CACHE_LOCK:
        return {"entries": len(_CACHE), "max": _CACHE_MAX}


def set_cache_limit(n):
    """Most compiled loop trees kept (least recently used evicted first)."""
    global _CACHE_MAX
    with _CACHE_LOCK:
        _CACHE_MAX = max(1, int(n))
        while len(_CACHE) > _CACHE_MAX:
            _CACHE.popitem(last=False)


def clear_cache():
    with _CACHE_LOCK:
        _CACHE.clear()
