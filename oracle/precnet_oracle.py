"""TEST INFRASTRUCTURE ONLY -- numpy restatement (float64) of the learned
preconditioner network of bamrex_b200/csrc/precnet.cu: the same layer
sequence and parameter layout, forward with BF16-rounded weights, and the
analytic backward pass, for checking the device forward and gradients.
Only tests/ import this module."""
from __future__ import annotations

import numpy as np

C = 16


def layer_plan():
    """(kind, in, in2, out, cin, cout, relu) in execution order; activation 0
    is the input; the last activation is the output."""
    plan, acts = [], [(2, 0)]

    def act(c, lev):
        acts.append((c, lev))
        return len(acts) - 1

    def conv(i, cin, cout, relu, lev):
        o = act(cout, lev)
        plan.append(("conv", i, None, o, cin, cout, relu))
        return o

    def pool(i, lev):
        o = act(C, lev + 1)
        plan.append(("pool", i, None, o, C, C, 0))
        return o

    def upadd(a, s, lev):
        o = act(C, lev)
        plan.append(("upadd", a, s, o, C, C, 0))
        return o

    h0 = conv(conv(0, 2, C, 1, 0), C, C, 1, 0)
    h1 = conv(conv(pool(h0, 0), C, C, 1, 1), C, C, 1, 1)
    h2 = conv(conv(pool(h1, 1), C, C, 1, 2), C, C, 1, 2)
    h3 = conv(conv(pool(h2, 2), C, C, 1, 3), C, C, 1, 3)
    g2 = conv(upadd(h3, h2, 2), C, C, 1, 2)
    g1 = conv(upadd(g2, h1, 1), C, C, 1, 1)
    g0 = conv(upadd(g1, h0, 0), C, C, 1, 0)
    conv(g0, C, 1, 0, 0)
    return plan, acts


def param_slices():
    plan, _ = layer_plan()
    out, p = [], 0
    for L in plan:
        if L[0] != "conv":
            out.append(None)
            continue
        cin, cout = L[4], L[5]
        out.append((p, p + cout * cin * 9, p + cout * cin * 9 + cout))
        p += cout * cin * 9 + cout
    return out, p


def bf16(w):
    """Round float32 values to the nearest bfloat16 (ties to even)."""
    u = np.asarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _shift(x, dj, di):
    # value at (j + dj, i + di), periodic
    return np.roll(x, (-dj, -di), axis=(-2, -1))


def _conv(x, w, b):
    # x: (B, cin, H, W); w: (cout, cin, 9); b: (cout,)
    y = np.zeros((x.shape[0], w.shape[0]) + x.shape[2:])
    for tap in range(9):
        xs = _shift(x, tap // 3 - 1, tap % 3 - 1)
        y += np.einsum("oc,bchw->bohw", w[:, :, tap], xs)
    return y + b[None, :, None, None]


def forward(params, inp, round_weights=True):
    """Activations list (float64) of the network on inp (B, 2, H, W)."""
    plan, acts = layer_plan()
    sl, _ = param_slices()
    wq = (bf16(params) if round_weights else np.asarray(params)).astype(np.float64)
    A = [None] * len(acts)
    A[0] = np.asarray(inp, dtype=np.float64)
    for L, s in zip(plan, sl):
        kind, i, i2, o, cin, cout, relu = L
        if kind == "conv":
            w = wq[s[0]:s[1]].reshape(cout, cin, 9)
            y = _conv(A[i], w, wq[s[1]:s[2]])
            A[o] = np.maximum(y, 0.0) if relu else y
        elif kind == "pool":
            x = A[i]
            A[o] = 0.25 * (x[..., 0::2, 0::2] + x[..., 0::2, 1::2] + x[..., 1::2, 0::2] + x[..., 1::2, 1::2])
        else:
            A[o] = np.repeat(np.repeat(A[i], 2, axis=-2), 2, axis=-1) + A[i2]
    return A


def backward(params, A, dout, round_weights=True):
    """Parameter gradient of sum(out * dout) (at the BF16-rounded weights)."""
    plan, acts = layer_plan()
    sl, P = param_slices()
    wq = (bf16(params) if round_weights else np.asarray(params)).astype(np.float64)
    G = [np.zeros_like(a) for a in A]
    G[-1] = np.asarray(dout, dtype=np.float64).reshape(A[-1].shape)
    grad = np.zeros(P)
    for L, s in reversed(list(zip(plan, sl))):
        kind, i, i2, o, cin, cout, relu = L
        if kind == "conv":
            g = G[o] * (A[o] > 0) if relu else G[o]
            w = wq[s[0]:s[1]].reshape(cout, cin, 9)
            dw = np.zeros((cout, cin, 9))
            for tap in range(9):
                xs = _shift(A[i], tap // 3 - 1, tap % 3 - 1)
                dw[:, :, tap] = np.einsum("bohw,bchw->oc", g, xs)
                G[i] += _shift(np.einsum("oc,bohw->bchw", w[:, :, tap], g), -(tap // 3 - 1), -(tap % 3 - 1))
            grad[s[0]:s[1]] = dw.ravel()
            grad[s[1]:s[2]] = g.sum(axis=(0, 2, 3))
        elif kind == "pool":
            G[i] += 0.25 * np.repeat(np.repeat(G[o], 2, axis=-2), 2, axis=-1)
        else:
            d = G[o]
            G[i] += d[..., 0::2, 0::2] + d[..., 0::2, 1::2] + d[..., 1::2, 0::2] + d[..., 1::2, 1::2]
            G[i2] += d
    return grad
