"""The golden programs written with this package's lazy frontend
(loop_tool_b200.lazy), parameterised like oracle/ref_harness.cpp builds them
with the reference's lazy frontend."""
import loop_tool_b200.lazy as lt
import loop_tool_b200.nn as nn


def _bin(op):
    def build(n):
        A, B = lt.Tensor(n), lt.Tensor(n)
        N = lt.Symbol("N")
        a, b = A.to(N), B.to(N)
        out = {"add": lambda: a + b, "sub": lambda: a - b, "mul": lambda: a * b,
               "div": lambda: a / b, "min": lambda: a.min(b), "max": lambda: a.max(b)}[op]()
        return out, [A, B]
    return build


def _un(op):
    def build(n):
        A = lt.Tensor(n)
        a = A.to(lt.Symbol("N"))
        return {"exp": a.exp, "sqrt": a.sqrt, "neg": a.__neg__, "recip": a.reciprocal,
                "abs": a.abs}[op](), [A]
    return build


def chain(n):
    A, B, C = lt.Tensor(n), lt.Tensor(n), lt.Tensor(n)
    N = lt.Symbol("N")
    a, b, c = A.to(N), B.to(N), C.to(N)
    t = a * b + c
    return ((t * t).sqrt() / (-a)).max(c) - b.reciprocal(), [A, B, C]


def mm(M, K, N):
    A, B = lt.Tensor(M, K), lt.Tensor(K, N)
    m, k, n = lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
    return (A.to(m, k) * B.to(k, n)).sum(k), [A, B]


def bmm(Bn, M, K, N):
    A, B = lt.Tensor(Bn, M, K), lt.Tensor(Bn, K, N)
    b, m, k, n = lt.Symbol("b"), lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
    return (A.to(b, m, k) * B.to(b, k, n)).sum(k), [A, B]


def softmax(R, C):
    X = lt.Tensor(R, C)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    x = X.to(r, n)
    e = (x - x.max_reduce(n)).exp()
    return e / e.sum(n), [X]


def _rows(kind):
    def build(R, C):
        X = lt.Tensor(R, C)
        r, n = lt.Symbol("r"), lt.Symbol("n")
        x = X.to(r, n)
        return {"rowsum": lambda: x.sum(n), "rowmax": lambda: x.max_reduce(n),
                "rowmin": lambda: x.min_reduce(n), "colsum": lambda: x.sum(r),
                "colmax": lambda: x.max_reduce(r), "fullsum": lambda: x.sum(r, n)}[kind](), [X]
    return build


def maxpool(N, C, H, W, k, s):
    X = lt.Tensor(N, C, H, W)
    n, c, h, w = (lt.Symbol(x) for x in "nchw")
    return nn.maxpool(X.to(n, c, h, w), [h, w], k, s), [X]


def conv(N, C, H, W, CO, K, pad, stride):
    X, Wt = lt.Tensor(N, C, H, W), lt.Tensor(CO, C, K, K)
    n, c, h, w, co, kh, kw = (lt.Symbol(x) for x in ["n", "c", "h", "w", "co", "kh", "kw"])
    x, sp = X.to(n, c, h, w), [h, w]
    if pad:
        x = x.pad(h, pad)
        x = x.pad(x.shape[3], pad)
        sp = [x.shape[2], x.shape[3]]
    return nn.conv(x, Wt.to(co, c, kh, kw), sp, [kh, kw], stride), [X, Wt]


def conv1d(n, k):
    A, Wt = lt.Tensor(n), lt.Tensor(k)
    N, No, K = lt.Symbol("N"), lt.Symbol("No"), lt.Symbol("K")
    X = A.to(N).to(No, K, constraints=[(N, lt.Expr(No) + K)])
    return (X * Wt.to(K)).sum(K), [A, Wt]


def padconv1d(n, k, p):
    A, Wt = lt.Tensor(n), lt.Tensor(k)
    N, No, K = lt.Symbol("n"), lt.Symbol("no"), lt.Symbol("k")
    xp = A.to(N).pad(N, p)
    Np = xp.shape[0]
    return (xp.to(No, K, constraints=[(Np, lt.Expr(No) + K)]) * Wt.to(K)).sum(K), [A, Wt]


def pad1d(n, pre, post):
    X = lt.Tensor(n)
    N = lt.Symbol("N")
    return X.to(N).pad(N, pre, post), [X]


def pad2d(m, n, p):
    X = lt.Tensor(m, n)
    M, N = lt.Symbol("m"), lt.Symbol("n")
    return X.to(M, N).pad(N, p), [X]


def concat1d(a, b):
    A, B = lt.Tensor(a), lt.Tensor(b)
    return A.to(lt.Symbol("N")) | B.to(lt.Symbol("M")), [A, B]


def concat2d(bb, m0, m1):
    A, B = lt.Tensor(bb, m0), lt.Tensor(bb, m1)
    N = lt.Symbol("N")
    return A.to(N, lt.Symbol("M0")) | B.to(N, lt.Symbol("M1")), [A, B]


def transpose_flatten(m, n):
    A = lt.Tensor(m, n)
    M, N, K = lt.Symbol("M"), lt.Symbol("N"), lt.Symbol("K")
    return A.to(M, N).to(K, constraints=[(K, lt.Expr(N) * lt.Size(M) + M)]), [A]


def flatten(m, n):
    A = lt.Tensor(m, n)
    M, N = lt.Symbol("M"), lt.Symbol("N")
    return A.to(M, N).flatten(M, N), [A]


def transpose(m, n):
    """B[n, m] = A[m, n] as an explicit view (the C++ A.to({N, M}))."""
    A = lt.Tensor(m, n)
    M, N, Mt, Nt = lt.Symbol("M"), lt.Symbol("N"), lt.Symbol("Mt"), lt.Symbol("Nt")
    return A.to(M, N).to(Nt, Mt, constraints=[(M, lt.Expr(Mt)), (N, lt.Expr(Nt))]), [A]


def scale(n):
    B, S = lt.Tensor(n), lt.Tensor(1)
    return B.to(lt.Symbol("N")) * S.to(lt.Symbol("O")), [B, S]


def bcast_add(R, C):
    X, Bv = lt.Tensor(R, C), lt.Tensor(C)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    return X.to(r, n) + Bv.to(n), [X, Bv]


def mean_rows(R, C):
    X, One = lt.Tensor(R, C), lt.Tensor(C)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    return X.to(r, n).sum(n) / One.to(n).sum(n), [X, One]


def layernorm(R, C):
    X, Cnt, Eps = lt.Tensor(R, C), lt.Tensor(1), lt.Tensor(1)
    r, n, e = lt.Symbol("r"), lt.Symbol("n"), lt.Symbol("e")
    x = X.to(r, n)
    mean = x.sum(n) / Cnt.to(e)
    d = x - mean
    var = (d * d).sum(n) / Cnt.to(e)
    return d / (var + Eps.to(e)).sqrt(), [X, Cnt, Eps]


BUILDERS = {
    "add": _bin("add"), "sub": _bin("sub"), "mul": _bin("mul"), "div": _bin("div"),
    "min": _bin("min"), "max": _bin("max"), "exp": _un("exp"), "sqrt": _un("sqrt"),
    "neg": _un("neg"), "recip": _un("recip"), "abs": _un("abs"), "chain": chain, "mm": mm,
    "bmm": bmm, "softmax": softmax, "rowsum": _rows("rowsum"), "rowmax": _rows("rowmax"),
    "rowmin": _rows("rowmin"), "colsum": _rows("colsum"), "colmax": _rows("colmax"),
    "fullsum": _rows("fullsum"), "maxpool": maxpool, "conv": conv, "conv1d": conv1d,
    "padconv1d": padconv1d, "pad1d": pad1d, "pad2d": pad2d, "concat1d": concat1d,
    "concat2d": concat2d, "transpose_flatten": transpose_flatten, "flatten": flatten,
    "transpose": transpose,
    "scale": scale, "bcast_add": bcast_add, "mean_rows": mean_rows, "layernorm": layernorm,
}


def build(case):
    """(tensor, leaves) of a golden case, leaves bound to the case's inputs."""
    T, leaves = BUILDERS[case["program"]](*[int(p) for p in case["params"]])
    for lf, a in zip(leaves, case["inputs"]):
        lf.set(a.reshape([int(x) for x in _leaf_sizes(lf)]))
    return T, leaves


def _leaf_sizes(t):
    return [c[1][1] for c in t.constraints if c[0][0] == "size"]
