"""numpy restatement of the SHIFTED storage form (TEST INFRASTRUCTURE ONLY).

The two-component Shan-Chen step of the reference (src/lbm.cpp:144-435,
src/fluid.cpp:175-278) rewritten for populations stored as deviations
d_i = f_i - w_i*rho_ref, with the storage rounded to float32 or float16 and
the arithmetic in float32 -- the same algebra as the GPU kernel's shifted
path:

    drho   = sum_i d_i,            rho = rho_ref + drho
    j      = sum_i c_i d_i         (sum_i w_i c_i = 0)
    sum over fluid neighbours of w c psi = sum w c drho_nbr - rho_ref * S,
        S = sum over solid neighbours of w c (the solid-force sums)
    d_eq_i = w_i (drho + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2))
    d*_i   = d_i + omega (d_eq_i - d_i) [+ F_i]     (i = 1..8, rounded to storage)
    d*_0   = d_0 + sum_{i>=1} (d_i - d*_i) [+ sum_i F_i]   (the rest population
             closes the node's mass, as the kernel does: equal to the BGK
             value in exact arithmetic)

followed by push streaming with half-way bounce-back.  The tests use it as
the checker of the GPU float path (same rounding regime, so agreement is
tight over a few steps) and to size the tolerances of the shifted forms
against the FP64 oracle.  Not fused-multiply-add exact; never bit-exact.
"""
from __future__ import annotations

import numpy as np

CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
OPP = [0, 3, 4, 1, 2, 7, 8, 5, 6]
WSC = np.array([0, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36])
WEQ = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def _shift(a, i, back=False):
    s = -1 if back else 1
    return np.roll(np.roll(a, s * -CY[i], 0), s * -CX[i], 1)


def step(d, mask, p, store=np.float32, compute=np.float32):
    """One step; d: [2][9][ny][nx] deviations (storage dtype), mask [ny][nx] bool."""
    T = compute
    x = d.astype(T)
    drho = [np.where(mask, x[k].sum(0, dtype=T), T(0)) for k in range(2)]
    A = np.zeros((2, 2) + mask.shape, T)
    S = np.zeros((2,) + mask.shape, T)
    for i in range(1, 9):
        nf = _shift(mask, i)
        for k in range(2):
            nb = _shift(drho[1 - k], i)
            A[k, 0] += np.where(nf, T(WSC[i] * CX[i]) * nb, T(0))
            A[k, 1] += np.where(nf, T(WSC[i] * CY[i]) * nb, T(0))
        S[0] += np.where(nf, T(0), T(WSC[i] * CX[i]))
        S[1] += np.where(nf, T(0), T(WSC[i] * CY[i]))
    rr = [T(p["rho_ref"][k]) for k in range(2)]
    r = [rr[k] + drho[k] for k in range(2)]
    F = [[T(-p["G"][k]) * r[k] * (A[k, a] - rr[1 - k] * S[a]) for a in range(2)] for k in range(2)]
    j = [[sum(T(c[i]) * x[k][i] for i in range(9)) for c in (CX, CY)] for k in range(2)]
    om = [T(1.0 / p["tau"][k]) for k in range(2)]
    den = r[0] * om[0] + r[1] * om[1]
    uc = [(j[0][a] * om[0] + j[1][a] * om[1]) / den for a in range(2)]
    out = np.zeros_like(x)
    for k in range(2):
        io = T(1) / om[k]
        u = [uc[a] + F[k][a] * (io / r[k]) + T(-p["Gs"][k]) * S[a] * io for a in range(2)]
        usq = T(1.5) * (u[0] * u[0] + u[1] * u[1])
        rest = x[k][0] + (sum(T(p["force"][k][i]) for i in range(9))
                          if p["force"][k] is not None else T(0))
        for i in range(1, 9):
            cu = T(CX[i]) * u[0] + T(CY[i]) * u[1]
            fe = T(WEQ[i]) * (r[k] * (cu * (T(4.5) * cu + T(3)) - usq) + drho[k])
            v = x[k][i] + om[k] * (fe - x[k][i])
            if p["force"][k] is not None:
                v = v + T(p["force"][k][i])
            v = np.where(mask, v, T(0)).astype(store).astype(T)
            out[k][i] = v
            rest = rest + (x[k][i] - v)
        out[k][0] = np.where(mask, rest, T(0))
    out = out.astype(store)
    new = np.zeros_like(out)
    for k in range(2):
        new[k][0] = out[k][0]
        for i in range(1, 9):
            up_fluid = _shift(mask, i, back=True)
            pulled = _shift(out[k][i], i, back=True)
            new[k][i] = np.where(mask & up_fluid, pulled, np.where(mask, out[k][OPP[i]], 0))
    return new


def run(case, f1, f2, steps, rho_ref, store=np.float32, compute=np.float32):
    """Advance a two-component case from FP64 populations; returns the FP64
    densities of both components (reference layout)."""
    nx, ny = case["nx"], case["ny"]
    mask = np.asarray(case["_mask"], bool).reshape(ny, nx)
    d = np.zeros((2, 9, ny, nx), store)
    for k, f in enumerate((f1, f2)):
        d[k] = np.where(mask, f.reshape(9, ny, nx) - WEQ[:, None, None] * rho_ref[k], 0)
    t1, G1, gs1 = case["fluid1"]
    t2, G2, gs2 = case["fluid2"]
    fmode, fv = case.get("force", (0, [0.0] * 9))
    p = dict(rho_ref=rho_ref, G=(G1, G2), tau=(t1, t2), Gs=(gs1, gs2),
             force=(fv if fmode in (1, 3) else None, fv if fmode in (2, 3) else None))
    for _ in range(steps):
        d = step(d, mask, p, store, compute)
    rho = []
    for k in range(2):
        x = d[k].astype(np.float64) + WEQ[:, None, None] * rho_ref[k]
        rho.append(np.where(mask, x.sum(0), 0.0).ravel())
    return rho
