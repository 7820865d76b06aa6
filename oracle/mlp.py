"""fp64 restatement of the learned table selector -- TEST INFRASTRUCTURE ONLY.

The checker for bzip2gpu_b200/csrc/mlp.cu (the selector has no counterpart in
the reference; its definition is include/bz2g.h, "learned table selector").
Only tests/ import it.

Parameters are the flat fp32 array of include/bz2g.h: W1 [256 x 272], b1,
W2 [256 x 256], b2, W3 [16 x 256], b3 [16].  A group's features are its
symbol counts c (258 bins) and n = its symbol count:

    Z1 = (c . W1^T) / n + b1    H1 = relu(Z1)
    Z2 = H1 . W2^T + b2         H2 = relu(Z2)
    Z3 = H2 . W3^T + b3         logits = Z3[:, :6]

Loss: mean softmax cross-entropy over the batch.  With emulate=True the
values the kernels hold in bf16 are rounded to bf16 at the same points
(weights, H1, H2, dZ3, dZ2, dZ1 and dZ1/n staged for dW1); everything else is
fp64.  With emulate=False the computation is exact fp64 over the fp32
parameters.
"""
from __future__ import annotations

import numpy as np

IN, IN_PAD, HID, OUT, OUT_PAD = 258, 272, 256, 6, 16
W1_, B1_ = 0, HID * IN_PAD
W2_ = B1_ + HID
B2_ = W2_ + HID * HID
W3_ = B2_ + HID
B3_ = W3_ + OUT_PAD * HID
PARAMS = B3_ + OUT_PAD
PAD_SYM = 0xFFFF


def bf16(x) -> np.ndarray:
    """Round to bf16 (nearest, ties to even) and return as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def views(P):
    P = np.asarray(P, np.float64)
    return (P[W1_:B1_].reshape(HID, IN_PAD), P[B1_:W2_], P[W2_:B2_].reshape(HID, HID),
            P[B2_:W3_], P[W3_:B3_].reshape(OUT_PAD, HID), P[B3_:B3_ + OUT_PAD])


def features(gsyms):
    """Group symbols [G, 50] (PAD_SYM past the end) -> counts [G, 272], n [G]."""
    g = np.asarray(gsyms).astype(np.int64) & 0xFFFF
    G = g.shape[0]
    c = np.zeros((G, IN_PAD), np.float64)
    valid = g != PAD_SYM
    rows = np.repeat(np.arange(G), g.shape[1]).reshape(g.shape)
    np.add.at(c, (rows[valid], g[valid]), 1.0)
    n = valid.sum(1).astype(np.float64)
    return c, n


def groups_of_stream(syms):
    """A block's symbol stream -> group symbols [ceil(s/50), 50] with padding."""
    s = np.asarray(syms).astype(np.int64)
    G = (s.size + 49) // 50
    out = np.full((G, 50), PAD_SYM, np.int64)
    out.reshape(-1)[: s.size] = s
    return out


def forward(P, c, n, emulate: bool = True):
    W1, b1, W2, b2, W3, b3 = views(P)
    r = bf16 if emulate else (lambda x: np.asarray(x, np.float64))
    inv = np.where(n > 0, 1.0 / np.maximum(n, 1), 0.0)
    Z1 = (c @ r(W1).T) * inv[:, None] + b1
    H1 = r(np.maximum(Z1, 0))
    Z2 = H1 @ r(W2).T + b2
    H2 = r(np.maximum(Z2, 0))
    Z3 = H2 @ r(W3).T + b3
    return {"inv": inv, "Z1": Z1, "H1": H1, "Z2": Z2, "H2": H2, "Z3": Z3}


def logits(P, c, n, emulate: bool = True) -> np.ndarray:
    return forward(P, c, n, emulate)["Z3"][:, :OUT]


def loss_grads(P, c, n, labels, emulate: bool = True):
    """(summed loss, correct count, gradient [PARAMS]) of the mean CE."""
    W1, b1, W2, b2, W3, b3 = views(P)
    r = bf16 if emulate else (lambda x: np.asarray(x, np.float64))
    f = forward(P, c, n, emulate)
    B = c.shape[0]
    z = f["Z3"][:, :OUT]
    mx = z.max(1, keepdims=True)
    e = np.exp(z - mx)
    p = e / e.sum(1, keepdims=True)
    y = np.asarray(labels, np.int64)
    loss = -(z[np.arange(B), y] - mx[:, 0] - np.log(e.sum(1)))
    correct = (z.argmax(1) == y).sum()
    dZ3 = np.zeros((B, OUT_PAD))
    dZ3[:, :OUT] = p
    dZ3[np.arange(B), y] -= 1.0
    dZ3 = r(dZ3 / B)
    g = np.zeros(PARAMS)
    gW1, gb1, gW2, gb2, gW3, gb3 = (g[W1_:B1_].reshape(HID, IN_PAD), g[B1_:W2_],
                                    g[W2_:B2_].reshape(HID, HID), g[B2_:W3_],
                                    g[W3_:B3_].reshape(OUT_PAD, HID), g[B3_:B3_ + OUT_PAD])
    gW3[:] = dZ3.T @ f["H2"]
    gb3[:] = dZ3.sum(0)
    dZ2 = r((dZ3 @ r(W3)) * (f["H2"] > 0))
    gW2[:] = dZ2.T @ f["H1"]
    gb2[:] = dZ2.sum(0)
    dZ1 = r((dZ2 @ r(W2)) * (f["H1"] > 0))
    gW1[:] = r(dZ1 * f["inv"][:, None]).T @ c
    gb1[:] = dZ1.sum(0)
    return float(loss.sum()), int(correct), g
