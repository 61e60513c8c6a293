"""CPU oracle: a numpy restatement of the reference loop_tool semantics.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py may import this module, and only as the
checker: the loop_tool_b200 package never calls it (there is no CPU
fallback).

It evaluates a serialized loop tree (the text serialize() writes,
serialization.cpp:175-237) on the CPU:
  * index equations of views follow Compiler::gen_index_equations
    (compile.cpp:611-756) with get_expr's rules (compile.cpp:634-692);
  * out-of-bounds reads through a view produce 0 (cpp.cpp:103-106) and the
    bounds are checked per base-buffer dim (compile.cpp:464-480);
  * element values follow the default "cpp" backend (cpp.cpp:172-270):
    n-ary ops fold left, min/max are the ternaries a<b?a:b / a>b?a:b,
    exp/log/sqrt are the C double functions rounded to float; abs is the
    float abs of the interpreter (compile.cpp:1066) -- the C path's
    integer abs() truncates and is not followed;
  * reductions fold sequentially in loop order from the reset values of
    gen_reset (compile.cpp:217-271: add 0, mul 1, max -FLT_MAX, min FLT_MAX).

Symbols are bound to IR variables at parse time, like the lazy frontend's
in-memory loop tree (a serialize/deserialize round trip in the reference
re-creates symbols per node, which it does not do here).

Pinned against the golden vectors the reference itself produced
(tests/golden/, tests/test_cpu_oracle.py).
"""
import numpy as np

FLT_MAX = np.float32(3.4028234663852886e38)

# ---------------------------------------------------------------- parsing
# serialization.cpp:239-332 (deserialize); expression tokens "op|type|arg|"
# with symbolic::Op codes (symbolic.h:38-50).
E_NEG, E_RECIP, E_SIZE, E_MAX, E_ADD, E_MUL, E_DIV, E_MOD = 1, 2, 3, 4, 5, 6, 7, 8
OPS = ["constant", "write", "read", "view", "copy", "add", "subtract", "multiply",
       "divide", "min", "max", "log", "exp", "sqrt", "abs", "negate", "reciprocal", "name"]


def _split(s, d):
    """std::getline semantics: no trailing empty field."""
    if s == "":
        return []
    parts = s.split(d)
    if parts and parts[-1] == "":
        parts.pop()
    return parts


def _parse_expr(s, sym_idx, counter):
    idx_map = {}
    for tok in _split(s, ";"):
        f = tok.split("|")
        op, ty = int(f[0]), f[1]
        i = counter[0]
        if ty == "s":
            sym_idx.add(i)
            idx_map[i] = ("sym", i)
        elif ty == "r":
            ref = int(f[2])
            sym_idx.add(i)
            idx_map[i] = ("sym", ref)
        elif ty == "v":
            idx_map[i] = ("val", int(f[2]))
        elif ty == "f":
            args = []
            for a in _split(f[2], ","):
                a = int(a)
                args.append(idx_map[a] if a in idx_map else ("sym", a))
            if len(args) == 1 and op == E_SIZE:
                idx_map[i] = ("size", args[0][1])
            else:
                idx_map[i] = ("fn", op, *args)
        counter[0] += 1
    return idx_map[counter[0] - 1]


def _remap(e, m):
    if e[0] == "sym":
        return ("var", m[e[1]])
    if e[0] == "size":
        return ("size", m[e[1]])
    if e[0] == "val":
        return e
    return (e[0], e[1]) + tuple(_remap(a, m) for a in e[2:])


def parse(text):
    g = {"vars": [], "nodes": [], "inputs": [], "outputs": []}
    for line in text.splitlines():
        if not line:
            continue
        ch = line.split(":")
        if ch[0] == "v":
            g["vars"].append(ch[1])
        elif ch[0] == "n":
            ch = ch + [""] * (12 - len(ch))
            node = {"op": OPS[int(ch[1])],
                    "inputs": [int(x) for x in _split(ch[2], ",")],
                    "vars": [int(x) for x in _split(ch[3], ",")],
                    "order": [tuple(int(t) for t in o.split(";")) for o in _split(ch[7], ",")]}
            sym_idx, counter, raw = set(), [0], []
            for cs in _split(ch[4], "/"):
                l, r = cs.split("=", 1)
                raw.append((_parse_expr(l, sym_idx, counter), _parse_expr(r, sym_idx, counter)))
            m = {}
            for kv in _split(ch[5], ","):
                k, v = kv.split("=")
                m[int(k)] = int(v)
            node["constraints"] = [(_remap(l, m), _remap(r, m)) for l, r in raw]
            g["nodes"].append(node)
        elif ch[0] == "i":
            g["inputs"] = [int(x) for x in _split(ch[1], ",")]
        elif ch[0] == "o":
            g["outputs"] = [int(x) for x in _split(ch[1], ",")]
    for i, n in enumerate(g["nodes"]):
        # one entry per input slot (a node may read the same input twice)
        n["consumers"] = [j for j, m in enumerate(g["nodes"]) for x in m["inputs"] if x == i]
    g["sizes"] = var_sizes(g)
    return g


# ------------------------------------------------------------- symbolic
def e_vars(e, out, include_sized=False):
    if e[0] == "var" or (include_sized and e[0] == "size"):
        if e[1] not in out:
            out.append(e[1])
    elif e[0] == "fn":
        for a in e[2:]:
            e_vars(a, out, include_sized)
    return out


def e_contains(e, v):
    if e[0] in ("var", "size"):
        return e[1] == v
    if e[0] == "fn":
        return any(e_contains(a, v) for a in e[2:])
    return False


def e_replace(e, v, w):
    if e[0] == "var":
        return w if e[1] == v else e
    if e[0] == "fn":
        return (e[0], e[1]) + tuple(e_replace(a, v, w) for a in e[2:])
    return e


def e_reify(e, sizes):
    if e[0] == "size":
        return ("val", sizes[e[1]]) if e[1] in sizes else e
    if e[0] == "fn":
        return (e[0], e[1]) + tuple(e_reify(a, sizes) for a in e[2:])
    return e


def _tdiv(a, b):  # C truncating division on int64 arrays / scalars
    q = np.abs(a) // np.abs(b)
    return np.where((np.asarray(a) < 0) ^ (np.asarray(b) < 0), -q, q)


def _tmod(a, b):
    return a - _tdiv(a, b) * b


def e_eval(e, env):
    """Evaluate with C int64 semantics; env maps var -> int or int array."""
    k = e[0]
    if k == "val":
        return e[1]
    if k in ("var", "size"):
        return env[e[1]] if k == "var" else env[("size", e[1])]
    op, args = e[1], [e_eval(a, env) for a in e[2:]]
    if op == E_ADD:
        return args[0] + args[1]
    if op == E_MUL:
        return args[0] * args[1]
    if op == E_DIV:
        return _tdiv(args[0], args[1])
    if op == E_MOD:
        return _tmod(args[0], args[1])
    if op == E_MAX:
        return np.maximum(args[0], args[1])
    if op == E_NEG:
        return -args[0]
    if op == E_RECIP:
        return _tdiv(1, args[0])
    raise ValueError(op)


def e_eval_float(e):
    """symbolic.cpp:305-353: float evaluation of a constant expression."""
    k = e[0]
    if k == "val":
        return float(np.float32(e[1]))
    if k != "fn":
        return None
    args = [e_eval_float(a) for a in e[2:]]
    if any(a is None for a in args):
        return None
    op = e[1]
    f = np.float32
    if op == E_ADD:
        return float(f(args[0]) + f(args[1]))
    if op == E_MUL:
        return float(f(args[0]) * f(args[1]))
    if op == E_DIV:
        return float(f(args[0]) / f(args[1]))
    if op == E_NEG:
        return -args[0]
    if op == E_MAX:
        return max(args)
    if op == E_MOD:
        return float(int(args[0]) % int(args[1]))
    return None


def e_diff(e, v):
    """symbolic.cpp:907-962."""
    if not e_contains(e, v):
        return ("val", 0)
    if e[0] == "var":
        return ("val", 1)
    if e[0] == "size":
        return ("val", 0)
    op, args = e[1], e[2:]
    if op == E_ADD:
        a, b = args
        if not e_contains(b, v):
            return e_diff(a, v)
        if not e_contains(a, v):
            return e_diff(b, v)
        return ("fn", E_ADD, e_diff(a, v), e_diff(b, v))
    if op == E_MUL:
        a, b = args
        if not e_contains(b, v):
            return ("fn", E_MUL, e_diff(a, v), b)
        if not e_contains(a, v):
            return ("fn", E_MUL, e_diff(b, v), a)
        return ("fn", E_ADD, ("fn", E_MUL, e_diff(a, v), b), ("fn", E_MUL, e_diff(b, v), a))
    if op == E_DIV:
        a, b = args
        if not e_contains(b, v):
            return ("fn", E_DIV, e_diff(a, v), b)
        num = ("fn", E_ADD, ("fn", E_MUL, e_diff(a, v), b),
               ("fn", E_NEG, ("fn", E_MUL, a, e_diff(b, v))))
        return ("fn", E_DIV, num, ("fn", E_MUL, b, b))
    if op == E_NEG:
        return ("fn", E_NEG, e_diff(args[0], v))
    if op == E_RECIP:
        a = args[0]
        return ("fn", E_DIV, e_diff(a, v), ("fn", E_MUL, a, a))
    raise ValueError(f"cannot differentiate op {op}")


def e_simplify_const(e):
    """Fold fully constant subtrees (integer semantics)."""
    if e[0] != "fn":
        return e
    args = [e_simplify_const(a) for a in e[2:]]
    if all(a[0] == "val" for a in args):
        return ("val", int(e_eval((e[0], e[1]) + tuple(args), {})))
    return (e[0], e[1]) + tuple(args)


# ------------------------------------------------------------ analysis
def var_sizes(g):
    """compile.cpp:62-120: size() constraints, then loop orders."""
    sizes = {}
    for n in g["nodes"]:
        for l, r in n["constraints"]:
            if l[0] == "size":
                r2 = e_simplify_const(r)
                if r2[0] == "val":
                    sizes[l[1]] = r2[1]
        tmp = {}
        for v, s, t in reversed(n["order"]):
            tmp[v] = tmp.get(v, 1) * s + t
        for v, s in tmp.items():
            sizes[v] = max(sizes.get(v, s), s)
    for _ in range(8):
        for n in g["nodes"]:
            for l, r in n["constraints"]:
                if l[0] == "size" and l[1] not in sizes:
                    try:
                        sizes[l[1]] = int(e_eval(e_reify(r, sizes), {}))
                    except KeyError:
                        pass
    return sizes


def all_vars(g, n):
    """ir.cpp:223-239: node vars plus its inputs' vars, sorted."""
    out = list(g["nodes"][n]["vars"])
    for i in g["nodes"][n]["inputs"]:
        for v in g["nodes"][i]["vars"]:
            if v not in out:
                out.append(v)
    return sorted(out)


def reduction_vars(g, n):
    """ir.cpp:206-221."""
    node = g["nodes"][n]
    out = []
    for i in node["inputs"]:
        for v in g["nodes"][i]["vars"]:
            if v not in node["vars"] and v not in out:
                out.append(v)
    return out


def view_is_many_to_one(g, n):
    """ir.cpp:146-204 (IR::view_reduction_vars), as a yes/no."""
    node = g["nodes"][n]
    outv = node["vars"]
    rhs = []
    for l, r in node["constraints"]:
        if l[0] == "var" and l[1] in outv:
            for s in e_vars(r, [], True):
                if s not in outv and s not in rhs:
                    rhs.append(s)
    for l, r in node["constraints"]:
        if not (l[0] == "var" and l[1] in outv):
            continue
        strides = {s: e_diff(r, s) for s in rhs}
        for s in rhs:
            contiguous = [k for k, d in strides.items()
                          if e_eval_float(d) is not None and e_eval_float(d) <= 1]
            for k in contiguous:
                del strides[k]
            for k in list(strides):
                if e_contains(strides[k], s):
                    strides[k] = ("fn", E_DIV, strides[k], ("size", s))
            if len(contiguous) > 1:
                return True
        if len(strides) > 1:
            return True
    return False


def view_expr(g, view, var):
    """get_expr (compile.cpp:634-692), read direction."""
    node = g["nodes"][view]
    outv = node["vars"]
    for l, r in node["constraints"]:
        if not (l[0] == "var" and l[1] == var):
            continue
        syms = e_vars(r, [])
        if all(s in outv for s in syms):
            return r
        if not view_is_many_to_one(g, view):
            e = r
            for s in syms:
                if s in outv:
                    continue
                mod = ("fn", E_NEG, e_diff(e, s))
                e = e_replace(e, s, ("val", 0))
                mf = e_eval_float(mod)
                if mf is not None and mf > 1:
                    e = ("fn", E_MOD, e, e_simplify_const(mod))
            if all(s in outv for s in e_vars(e, [])):
                return e
    return ("var", var)


def derive_access(g, consumer, inp):
    """collect_fw of gen_index_equations (compile.cpp:694-740)."""
    chain = []
    x = inp
    while g["nodes"][x]["op"] == "view":
        chain.append(x)
        x = g["nodes"][x]["inputs"][0]
    idx = [("var", v) for v in g["nodes"][x]["vars"]]
    avail = all_vars(g, consumer)
    for nr in reversed(chain):
        src = g["nodes"][nr]["inputs"][0]
        for v in g["nodes"][src]["vars"]:
            if v in avail:
                continue
            ne = view_expr(g, nr, v)
            idx = [e_reify(e_replace(e, v, ne), {v: g["sizes"][v]}) for e in idx]
    idx = [e_reify(e, g["sizes"]) for e in idx]
    return x, idx


# ----------------------------------------------------------- evaluation
_DT = [np.float32]  # evaluation precision: float32 (reference) or float64


def _f32(x):
    return np.asarray(x, dtype=_DT[0])


def _unary(op, a):
    if op == "exp":
        with np.errstate(over="ignore"):
            return _f32(np.exp(a.astype(np.float64)))
    if op == "log":
        with np.errstate(divide="ignore", invalid="ignore"):
            return _f32(np.log(a.astype(np.float64)))
    if op == "sqrt":
        with np.errstate(invalid="ignore"):
            return _f32(np.sqrt(a.astype(np.float64)))
    if op == "abs":
        return np.abs(a)
    if op == "negate":
        return -a
    if op == "reciprocal":
        with np.errstate(divide="ignore"):
            return _f32(_DT[0](1) / a)
    raise ValueError(op)


def _binary(op, a, b):
    with np.errstate(all="ignore"):
        if op == "add":
            return _f32(a + b)
        if op == "subtract":
            return _f32(a - b)
        if op == "multiply":
            return _f32(a * b)
        if op == "divide":
            return _f32(a / b)
        if op == "min":
            return np.where(a < b, a, b).astype(_DT[0])
        if op == "max":
            return np.where(a > b, a, b).astype(_DT[0])
    raise ValueError(op)


RESET = {"add": np.float32(0), "subtract": np.float32(0), "multiply": np.float32(1),
         "divide": np.float32(1), "min": FLT_MAX, "max": -FLT_MAX}


def _gather(g, vals, base, idx, loop_vars):
    """Values of `base` at index expressions over the loop-var grid, 0 where
    a base dim's index leaves [0, size)."""
    sizes = g["sizes"]
    shape = [sizes[v] for v in loop_vars]
    env = {}
    for k, v in enumerate(loop_vars):
        sh = [1] * len(loop_vars)
        sh[k] = shape[k]
        env[v] = np.arange(shape[k], dtype=np.int64).reshape(sh)
    src = vals[base]
    bvars = g["nodes"][base]["vars"]
    valid = np.ones([1] * len(loop_vars), dtype=bool)
    flat = np.zeros([1] * len(loop_vars), dtype=np.int64)
    for d, e in enumerate(idx):
        # vars not iterated here read index 0 (scoped exprs, compile.cpp:858-872)
        for v in e_vars(e, []):
            if v not in env:
                e = e_replace(e, v, ("val", 0))
        iv = np.asarray(e_eval(e, env), dtype=np.int64)
        n = sizes[bvars[d]]
        valid = valid & (iv >= 0) & (iv < n)
        flat = flat * n + np.clip(iv, 0, n - 1)
    flat = np.broadcast_to(flat, shape)
    valid = np.broadcast_to(valid, shape)
    out = src.reshape(-1)[flat]
    return np.where(valid, out, 0).astype(_DT[0])


def evaluate(ir_text, inputs, dtype=np.float32):
    """Run a serialized loop tree on numpy inputs; returns the outputs.

    dtype=np.float32 restates the reference's FP32 arithmetic; np.float64
    is the high-precision oracle that FP32 results are measured against."""
    _DT[0] = dtype
    try:
        return _evaluate(ir_text, inputs)
    finally:
        _DT[0] = np.float32


def _evaluate(ir_text, inputs):
    g = parse(ir_text) if isinstance(ir_text, str) else ir_text
    sizes = g["sizes"]
    vals = {}
    for i, n in enumerate(g["inputs"]):
        shape = [sizes[v] for v in g["nodes"][n]["vars"]]
        vals[n] = _f32(inputs[i]).reshape(shape)
    order = _topo(g)
    for n in order:
        node = g["nodes"][n]
        op = node["op"]
        if op in ("read", "view"):
            continue
        loop_vars = all_vars(g, n)
        red = [v for v in loop_vars if v not in node["vars"]]
        # reductions fold in loop order: the order of the node's loops
        order_vars = [v for v, _, _ in node["order"]]
        red.sort(key=lambda v: order_vars.index(v) if v in order_vars else 1 << 20)
        loop_vars = [v for v in loop_vars if v not in red] + red
        terms = []
        for x in node["inputs"]:
            base, idx = derive_access(g, n, x)
            terms.append(_gather(g, vals, base, idx, loop_vars))
        nout = len(loop_vars) - len(red)
        if op == "write":
            val = terms[0]
        elif op in ("exp", "log", "sqrt", "abs", "negate", "reciprocal"):
            val = _unary(op, terms[0])
        elif op == "copy":
            val = terms[0]
        elif red:
            R = int(np.prod([sizes[v] for v in red]))
            out_shape = [sizes[v] for v in loop_vars[:nout]]
            ts = [t.reshape(out_shape + [R]) for t in terms]
            acc = np.full(out_shape, RESET[op], dtype=_DT[0])
            for r in range(R):
                for t in ts:
                    acc = _binary(op, acc, t[..., r])
            val = acc
        else:
            val = terms[0]
            for t in terms[1:]:
                val = _binary(op, val, t)
        # permute from loop order to the node's own var order
        perm = [loop_vars[:nout].index(v) for v in node["vars"]]
        vals[n] = np.ascontiguousarray(np.transpose(val, perm)) if perm else val
    return [vals[o].reshape(-1) for o in g["outputs"]]


def _topo(g):
    n = len(g["nodes"])
    indeg = [len(g["nodes"][i]["inputs"]) for i in range(n)]
    ready = sorted(i for i in range(n) if indeg[i] == 0)
    out = []
    while ready:
        i = ready.pop(0)
        out.append(i)
        for c in g["nodes"][i]["consumers"]:
            indeg[c] -= 1
            if indeg[c] == 0:
                ready.append(c)
                ready.sort()
    return out
