"""nn helpers over lazy tensors, after the reference's python/nn.py and
src/frontends/nn.cpp: pad, conv (python/nn.py:96-109, keeping every
non-spatial dim of X), maxpool (nn.cpp:48-76), linear, mean, relu."""
from .lazy import Expr, Size, Symbol, Tensor


def pad(X, *args):
    """pad(X, (s.h, 1), (s.w, (0, 1))) -- python/nn.py:87-93."""
    for d, p in args:
        X = X.pad(d, *p) if isinstance(p, tuple) else X.pad(d, p)
    return X


def conv(X, W, spatial, window, stride=1, channel_reduce=True):
    """X viewed with sp = stride * sp_o + k, then (X * W).sum(channels shared
    with W, window dims) -- python/nn.py:96-109."""
    assert len(spatial) == len(window)
    new_spatial = [Symbol(x.name + "o") for x in spatial]
    outer = [d for d in X.shape if d not in spatial]
    exprs = [Expr(stride) * x + k for x, k in zip(new_spatial, window)]
    X = X.to(*outer, *new_spatial, *window, constraints=list(zip(spatial, exprs)))
    if channel_reduce:
        red = [d for d in X.shape if d in W.shape or d in window]
    else:
        red = list(window)
    return (X * W).sum(*red)


def maxpool(X, spatial, k, stride=1):
    """nn.cpp:48-76: view h = stride * h_p + h_k (|h_k| = k), max over the
    window dims."""
    new_sp, new_win, cs = [], [], []
    for s in spatial:
        p, w = Symbol(s.name + "_p"), Symbol(s.name + "_k")
        new_sp.append(p)
        new_win.append(w)
        cs += [(s, Expr(stride) * p + w), (Size(w), Expr(k))]
    batch = [d for d in X.shape if d not in spatial]
    X = X.to(*batch, *new_sp, *new_win, constraints=cs)
    return X.max_reduce(*new_win)


def linear(X, W, bias=None):
    red = [d for d in X.shape if d in W.shape]
    Y = (X * W).sum(*red)
    return Y + bias if bias is not None else Y


def relu(T, zero):
    return T.max(zero)
