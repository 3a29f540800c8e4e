"""CPU oracle of the learned CG preconditioner's network (numpy, FP64 sums).

TEST INFRASTRUCTURE ONLY: tests compare the CUDA forward/backward kernels of
peridigm_b200/csrc/k_mpnn.cu against this restatement. The network has no
counterpart in the reference; this file restates the network the CUDA code
defines (hidden 64, 3 mean-aggregation message-passing layers with residual
connections, BF16 weights and BF16 stored activations):

  f   = (a / s_a, r / s_r)                     s = rms over all 3n entries
  h0  = bf16(relu(W0 f + b0))
  h_l = bf16(h_{l-1} + relu(Ws_l h_{l-1} + Wn_l m_l + b_l)),  m_l = mean_{j in N(i)} h_{l-1, j}
  out = Wd h3 + bd,   z = a + s_a out

Two training losses are restated: the error-space L = |z - e|^2 / |e|^2
(loss_grad) and the residual-space L = |K z - r|^2 / |r|^2 with prescribed
dofs zeroed (loss_grad_residual), the one the CUDA trainer minimises.
Gradients treat the BF16 roundings as identity (straight-through), as the
kernels do.
"""
from __future__ import annotations

import numpy as np

H, F, NL = 64, 6, 3
OFF_W0, OFF_B0 = 0, H * F
OFF_L = OFF_B0 + H
LSZ = 2 * H * H + H
OFF_WD = OFF_L + NL * LSZ
OFF_BD = OFF_WD + 3 * H
NPARAM = OFF_BD + 3


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    b = (b + 0x7FFF + lsb) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    W0 = w[OFF_W0:OFF_B0].reshape(H, F)
    b0 = w[OFF_B0:OFF_L]
    layers = []
    for l in range(NL):
        o = OFF_L + l * LSZ
        layers.append((w[o:o + H * H].reshape(H, H), w[o + H * H:o + 2 * H * H].reshape(H, H),
                       w[o + 2 * H * H:o + LSZ]))
    Wd = w[OFF_WD:OFF_BD].reshape(3, H)
    bd = w[OFF_BD:OFF_BD + 3]
    return W0, b0, layers, Wd, bd


def loss_grad(w, a, r, e, mrow, mcol, round_bf16=True):
    """Loss and gradient (length NPARAM) of one pair; a, r, e are [3n] float32."""
    rnd = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float32))
    wb = rnd(np.asarray(w, np.float32)).astype(np.float64)
    W0, b0, layers, Wd, bd = unpack(wb)
    n = len(mrow) - 1
    a = np.asarray(a, np.float32).reshape(n, 3)
    r = np.asarray(r, np.float32).reshape(n, 3)
    e = np.asarray(e, np.float32).reshape(n, 3).astype(np.float64)
    sa = np.sqrt(np.sum(a.astype(np.float64) ** 2) / (3 * n))
    sr = np.sqrt(np.sum(r.astype(np.float64) ** 2) / (3 * n))
    ia, ir = np.float32(1.0 / sa), np.float32(1.0 / sr)
    f = np.concatenate([a * ia, r * ir], axis=1).astype(np.float64)
    deg = np.diff(mrow).astype(np.float64)
    owner = np.repeat(np.arange(n), np.diff(mrow))

    def mean_agg(h):
        m = np.zeros_like(h)
        np.add.at(m, owner, h[mcol])
        return m / np.maximum(deg, 1.0)[:, None]

    pre0 = f @ W0.T + b0
    hs = [rnd(np.maximum(pre0, 0.0)).astype(np.float64)]
    pres, ms = [], []
    for (Ws, Wn, b) in layers:
        h = hs[-1]
        m = mean_agg(h)
        pre = h @ Ws.T + m @ Wn.T + b
        pres.append(pre)
        ms.append(m)
        hs.append(rnd(h + np.maximum(pre, 0.0)).astype(np.float64))
    out = hs[-1] @ Wd.T + bd
    z = a.astype(np.float64) + sa * out
    e2 = np.sum(e * e)
    L = float(np.sum((z - e) ** 2) / e2)
    # backward
    g = np.zeros(NPARAM)
    gout = 2.0 * sa * (z - e) / e2
    g[OFF_WD:OFF_BD] = (gout.T @ hs[-1]).ravel()
    g[OFF_BD:OFF_BD + 3] = gout.sum(0)
    dh = gout @ Wd
    for l in range(NL - 1, -1, -1):
        Ws, Wn, b = layers[l]
        dpre = dh * (pres[l] > 0)
        o = OFF_L + l * LSZ
        g[o:o + H * H] = (dpre.T @ hs[l]).ravel()
        g[o + H * H:o + 2 * H * H] = (dpre.T @ ms[l]).ravel()
        g[o + 2 * H * H:o + LSZ] = dpre.sum(0)
        dm = (dpre @ Wn) / np.maximum(deg, 1.0)[:, None]
        dprev = dh + dpre @ Ws
        np.add.at(dprev, mcol, dm[owner])
        dh = dprev
    dpre0 = dh * (pre0 > 0)
    g[OFF_W0:OFF_B0] = (dpre0.T @ f).ravel()
    g[OFF_B0:OFF_L] = dpre0.sum(0)
    return L, g


def loss_grad_residual(w, a, r, K, fixed_dofs, mrow, mcol, round_bf16=True):
    """Residual-space loss L = |K z - r|^2 / |r|^2 (z = a + s_a out, prescribed
    dofs of z and r zero) and its gradient; K is a dense tangent [3n, 3n]."""
    wb = (bf16 if round_bf16 else (lambda v: np.asarray(v, np.float32)))(np.asarray(w, np.float32))
    n = len(mrow) - 1
    a32 = np.asarray(a, np.float32)
    r32 = np.asarray(r, np.float32)
    fixed = np.zeros(3 * n, bool)
    fixed[list(fixed_dofs)] = True
    # forward through the shared network body, with a target-free pass
    L0, _, aux = _forward(wb, a32, r32, mrow, mcol, round_bf16)
    z = a32.astype(np.float64) + aux["sa"] * aux["out"].ravel()
    z[fixed] = 0.0
    rr = r32.astype(np.float64).copy()
    rr[fixed] = 0.0
    res = K @ z - rr
    res[fixed] = 0.0
    r2 = float(rr @ rr)
    L = float(res @ res) / r2
    dz = 2.0 * (K.T @ res) / r2
    dz[fixed] = 0.0
    gout = (aux["sa"] * dz).reshape(n, 3)
    return L, _backward(wb, gout, aux, mrow, mcol)


def _forward(wb, a, r, mrow, mcol, round_bf16):
    rnd = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float32))
    W0, b0, layers, Wd, bd = unpack(np.asarray(wb, np.float64))
    n = len(mrow) - 1
    a = a.reshape(n, 3)
    r = r.reshape(n, 3)
    sa = np.sqrt(np.sum(a.astype(np.float64) ** 2) / (3 * n))
    sr = np.sqrt(np.sum(r.astype(np.float64) ** 2) / (3 * n))
    ia, ir = np.float32(1.0 / sa), np.float32(1.0 / sr)
    f = np.concatenate([a * ia, r * ir], axis=1).astype(np.float64)
    deg = np.diff(mrow).astype(np.float64)
    owner = np.repeat(np.arange(n), np.diff(mrow))

    def mean_agg(h):
        m = np.zeros_like(h)
        np.add.at(m, owner, h[mcol])
        return m / np.maximum(deg, 1.0)[:, None]

    pre0 = f @ W0.T + b0
    hs = [rnd(np.maximum(pre0, 0.0)).astype(np.float64)]
    pres, ms = [], []
    for (Ws, Wn, b) in layers:
        h = hs[-1]
        m = mean_agg(h)
        pre = h @ Ws.T + m @ Wn.T + b
        pres.append(pre)
        ms.append(m)
        hs.append(rnd(h + np.maximum(pre, 0.0)).astype(np.float64))
    out = hs[-1] @ Wd.T + bd
    aux = dict(sa=sa, f=f, pre0=pre0, hs=hs, pres=pres, ms=ms, out=out, deg=deg, owner=owner)
    return 0.0, None, aux


def _backward(wb, gout, aux, mrow, mcol):
    W0, b0, layers, Wd, bd = unpack(np.asarray(wb, np.float64))
    hs, pres, ms, deg, owner = aux["hs"], aux["pres"], aux["ms"], aux["deg"], aux["owner"]
    g = np.zeros(NPARAM)
    g[OFF_WD:OFF_BD] = (gout.T @ hs[-1]).ravel()
    g[OFF_BD:OFF_BD + 3] = gout.sum(0)
    dh = gout @ Wd
    for l in range(NL - 1, -1, -1):
        Ws, Wn, b = layers[l]
        dpre = dh * (pres[l] > 0)
        o = OFF_L + l * LSZ
        g[o:o + H * H] = (dpre.T @ hs[l]).ravel()
        g[o + H * H:o + 2 * H * H] = (dpre.T @ ms[l]).ravel()
        g[o + 2 * H * H:o + LSZ] = dpre.sum(0)
        dm = (dpre @ Wn) / np.maximum(deg, 1.0)[:, None]
        dprev = dh + dpre @ Ws
        np.add.at(dprev, mcol, dm[owner])
        dh = dprev
    dpre0 = dh * (aux["pre0"] > 0)
    g[OFF_W0:OFF_B0] = (dpre0.T @ aux["f"]).ravel()
    g[OFF_B0:OFF_L] = dpre0.sum(0)
    return g


def subgraph(x, row, col, radius, bond_damage=None):
    """Bonds shorter than radius, in bond-family order (the kernel's subgraph)."""
    P = np.asarray(x, float).reshape(-1, 3)
    n = len(P)
    owner = np.repeat(np.arange(n), np.diff(row))
    d = P[col] - P[owner]
    keep = np.einsum("ij,ij->i", d, d) <= radius * radius
    if bond_damage is not None:
        keep &= np.asarray(bond_damage) == 0
    mrow = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(owner[keep], minlength=n), out=mrow[1:])
    return mrow, np.asarray(col)[keep].astype(np.int64)
