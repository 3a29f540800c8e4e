"""CPU oracle of the learned middle level of the QS CG preconditioner (numpy).

TEST INFRASTRUCTURE ONLY: tests compare the CUDA kernels of
peridigm_b200/csrc/k_mpnn.cu against this restatement. The preconditioner has
no counterpart in the reference; this file restates the one the CUDA code
defines:

  z = a + z0 + Q S G^T G S Q^T r        a = P_bj r, z0 = the coarse correction

  patches: the non-empty cells (cell order, x fastest) of a grid of side
           `side` from the coordinate minimum, dims = floor(extent / side) + 1;
           neighbors of a patch: the non-empty cells of its 3x3x3
           neighborhood (itself excluded), z then y then x ascending
  Q:       piecewise constant from patches to the free dofs of their points
  S:       s_I = sqrt(sum_{i in I} sum_{c free} (D_i^-1)_cc / 3) / |I|
  G:       h0 = W0 v,  h_l = h_{l-1} + Ws_l h_{l-1} + Wn_l mean_{J in N(I)} h_{l-1,J}

with BF16 weights (activations and sums in FP64 here, FP32 on the device).
Loss (pairs r = K e): the energy-norm error left by one optimally scaled
step, L = 1 - (r.z)^2 / ((z.K z)(e.r)), prescribed dofs of z, r and e zeroed;
the gradient of <g_c, G^T G v> is the sum of two backward passes of G.
"""
from __future__ import annotations

import numpy as np

H, NL = 64, 3
OFF_W0 = 0
OFF_L = 3 * H
LSZ = 2 * H * H
NPARAM = OFF_L + NL * LSZ


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    b = (b + 0x7FFF + lsb) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    W0 = w[OFF_W0:OFF_L].reshape(H, 3)
    layers = []
    for l in range(NL):
        o = OFF_L + l * LSZ
        layers.append((w[o:o + H * H].reshape(H, H), w[o + H * H:o + 2 * H * H].reshape(H, H)))
    return W0, layers


def patches(x, side):
    """(patch of each point, neighbor lists) of the patch graph."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    lo, hi = x.min(0), x.max(0)
    dims = np.floor((hi - lo) / side).astype(np.int64) + 1
    c = np.clip(np.floor((x - lo) / side).astype(np.int64), 0, dims - 1)
    cid = (c[:, 2] * dims[1] + c[:, 1]) * dims[0] + c[:, 0]
    cells = np.unique(cid)
    pid = np.searchsorted(cells, cid)
    where = {int(q): k for k, q in enumerate(cells)}
    nbrs = []
    for q in cells:
        cx, cy, cz = q % dims[0], (q // dims[0]) % dims[1], q // (dims[0] * dims[1])
        out = []
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if dx == 0 and dy == 0 and dz == 0:
                        continue
                    X, Y, Z = cx + dx, cy + dy, cz + dz
                    if X < 0 or Y < 0 or Z < 0 or X >= dims[0] or Y >= dims[1] or Z >= dims[2]:
                        continue
                    k = where.get(int((Z * dims[1] + Y) * dims[0] + X))
                    if k is not None:
                        out.append(k)
        nbrs.append(out)
    return pid, nbrs


def scales(dinv_blocks, pid, fixed_dofs=()):
    """s_I from the block-Jacobi inverse blocks [n, 3, 3], prescribed dofs left
    out (rounded to float32)."""
    npatch = int(pid.max()) + 1
    dg = np.einsum("nii->ni", np.asarray(dinv_blocks, np.float64)).copy()
    dg.ravel()[list(fixed_dofs)] = 0.0
    tr = dg.sum(1) / 3.0
    s = np.bincount(pid, tr, npatch)
    cnt = np.bincount(pid, minlength=npatch)
    return (np.sqrt(s) / cnt).astype(np.float32).astype(np.float64)


def _mean_matrix(nbrs):
    n = len(nbrs)
    A = np.zeros((n, n))
    for i, js in enumerate(nbrs):
        for j in js:
            A[i, j] += 1.0 / len(js)
    return A


def _q(pid, fixed, npatch):
    n = pid.size
    Q = np.zeros((3 * n, 3 * npatch))
    for i in range(n):
        for c in range(3):
            if not fixed[3 * i + c]:
                Q[3 * i + c, 3 * pid[i] + c] = 1.0
    return Q


def forward(wb, v, Am):
    """G v for v [np, 3]; returns the output and the saved (h_{l-1}, mean) pairs."""
    W0, layers = unpack(wb)
    h = v @ W0.T
    saved = []
    for Ws, Wn in layers:
        m = Am @ h
        saved.append((h, m))
        h = h + h @ Ws.T + m @ Wn.T
    return h, saved


def transpose(wb, y, Am):
    """G^T y for y [np, 64]; returns [np, 3]."""
    W0, layers = unpack(wb)
    x = y
    for Ws, Wn in reversed(layers):
        x = x + x @ Ws + Am.T @ (x @ Wn)
    return x @ W0


def backward(wb, v, saved, U, Am):
    """Gradient of <U, G v> with respect to the weights (length NPARAM)."""
    W0, layers = unpack(wb)
    g = np.zeros(NPARAM)
    cur = U
    for l in range(NL - 1, -1, -1):
        Ws, Wn = layers[l]
        h, m = saved[l]
        o = OFF_L + l * LSZ
        g[o:o + H * H] += (cur.T @ h).ravel()
        g[o + H * H:o + 2 * H * H] += (cur.T @ m).ravel()
        cur = cur + cur @ Ws + Am.T @ (cur @ Wn)
    g[OFF_W0:OFF_L] += (cur.T @ v).ravel()
    return g


def loss_grad(w, a, r, e, K, fixed_dofs, pid, nbrs, scale, z0=None, round_bf16=True):
    """L = 1 - (r.z)^2 / ((z.K z)(e.r)), z = a + z0 + Q S G^T G S Q^T r, and dL/dw."""
    wb = (bf16(np.asarray(w, np.float32)) if round_bf16 else np.asarray(w, np.float32)).astype(np.float64)
    n = pid.size
    npatch = int(pid.max()) + 1
    fixed = np.zeros(3 * n, bool)
    fixed[list(fixed_dofs)] = True
    Am = _mean_matrix(nbrs)
    Q = _q(pid, fixed, npatch)
    S = np.repeat(np.asarray(scale, np.float64), 3)
    rr = np.asarray(r, np.float32).astype(np.float64)
    rr[fixed] = 0.0
    ee = np.asarray(e, np.float32).astype(np.float64)
    ee[fixed] = 0.0
    v0 = (S * (Q.T @ rr)).reshape(npatch, 3)
    y0, sv0 = forward(wb, v0, Am)
    z = np.asarray(a, np.float32).astype(np.float64) + Q @ (S * transpose(wb, y0, Am).ravel())
    if z0 is not None:
        z = z + np.asarray(z0, np.float64)
    z[fixed] = 0.0
    kz = K @ z
    A, B, E = float(rr @ z), float(z @ kz), float(ee @ rr)
    L = 1.0 - A * A / (B * E)
    gz = -2.0 * A / (B * E) * rr + 2.0 * A * A / (B * B * E) * kz
    gz[fixed] = 0.0
    v1 = (S * (Q.T @ gz)).reshape(npatch, 3)
    y1, sv1 = forward(wb, v1, Am)
    g = backward(wb, v0, sv0, y1, Am) + backward(wb, v1, sv1, y0, Am)
    return L, g


def loss_grad_steps(w, r, e, K, Mfix, fixed_dofs, pid, nbrs, scale, ksteps, round_bf16=True):
    """Loss after `ksteps` steps of preconditioned steepest descent and dL/dw.

    From x0 = 0 on K x = r (r = K e): z_t = M r_t with M = Mfix + Q S G^T G S Q^T
    (Mfix: block Jacobi and coarse correction, a dense symmetric matrix here),
    q_t = K z_t, alpha_t = (r_t.z_t)/(z_t.q_t), e_{t+1} = e_t - alpha_t z_t,
    r_{t+1} = r_t - alpha_t q_t; L = (e_k.r_k)/(e_0.r_0), the energy-norm error
    left after k steps (1 step: the single-step loss above). The exact step
    makes L invariant to the scale of M; the error after several steps is
    made of the slow modes of M K, which set CG's iteration count. The
    gradient runs the recurrence backwards (M and K symmetric):
        abar = -(z_t.ebar) - (q_t.rbar)
        zbar = -alpha ebar + abar (r_t/b - a q_t/b^2),  qbar = -alpha rbar - abar a z_t/b^2
        zbar += K qbar;  rbar += abar z_t/b + M zbar;  dL/dw += d<zbar, N r_t>/dw
    with a = r_t.z_t, b = z_t.q_t, ebar and rbar starting at r_k/E0 and e_k/E0."""
    wb = (bf16(np.asarray(w, np.float32)) if round_bf16 else np.asarray(w, np.float32)).astype(np.float64)
    n = pid.size
    npatch = int(pid.max()) + 1
    fixed = np.zeros(3 * n, bool)
    fixed[list(fixed_dofs)] = True
    Am = _mean_matrix(nbrs)
    Q = _q(pid, fixed, npatch)
    S = np.repeat(np.asarray(scale, np.float64), 3)
    free = ~fixed

    def net(x):
        v = (S * (Q.T @ x)).reshape(npatch, 3)
        y, sv = forward(wb, v, Am)
        out = Q @ (S * transpose(wb, y, Am).ravel())
        out[fixed] = 0.0
        return out, v, y, sv

    def M(x):
        out = Mfix @ x + net(x)[0]
        out[fixed] = 0.0
        return out

    rt = np.asarray(r, np.float64).copy()
    et = np.asarray(e, np.float64).copy()
    rt[fixed] = 0.0
    et[fixed] = 0.0
    E0 = float(et @ rt)
    hist = []
    for _ in range(ksteps):
        z = M(rt)
        q = K @ z
        q[fixed] = 0.0
        a, b = float(rt @ z), float(z @ q)
        if not b > 0.0:  # converged exactly: the remaining steps change nothing
            break
        al = a / b
        hist.append((rt.copy(), z, q, a, b, al))
        et = et - al * z
        rt = rt - al * q
    L = float(et @ rt) / E0
    ebar = rt / E0
    rbar = et / E0
    g = np.zeros(NPARAM)
    for rt_, z, q, a, b, al in reversed(hist):
        abar = -float(z @ ebar) - float(q @ rbar)
        zbar = -al * ebar + abar * (rt_ / b - a * q / (b * b))
        qbar = -al * rbar - abar * a * z / (b * b)
        zbar = zbar + K @ qbar
        zbar[~free] = 0.0
        _, v0, y0, sv0 = net(rt_)
        Mz, v1, y1, sv1 = net(zbar)
        g += backward(wb, v0, sv0, y1, Am) + backward(wb, v1, sv1, y0, Am)
        rbar = rbar + abar * z / b + Mfix @ zbar + Mz
        rbar[fixed] = 0.0
    return L, g
