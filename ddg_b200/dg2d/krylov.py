"""Restarted GMRES on the device SIPG operator (``IterativeConfig(method=
"gmres")``; an extension: the reference's sipg solves accept only "cg",
``src/ddg/dg2d/sipg.py:603-611``, and its GMRES lives in the coupled NS
solver, ``src/ddg/dg2d/coupled_ns.py:605-624``).

Right-preconditioned GMRES(m) with modified Gram-Schmidt.  Basis vectors,
the operator and every dot/axpy run as library kernels on the device; only
the (m+1) x m Hessenberg least-squares problem lives on the host.  Stops when
``||b - A x|| <= max(tol ||b||, atol)``.
"""

from __future__ import annotations

import numpy as np

from .operator import axpby, dot


def gmres(op, b, x, *, alpha=0.0, shift=0.0, tol=1e-9, atol=0.0, maxiter=1000, restart=30, M=None):
    import torch
    from .sipg import SolveInfo

    def A(v):
        y = op.apply(v, alpha=alpha)
        if shift != 0.0:
            axpby(shift, v, 1.0, y)
        return y

    def Minv(v):
        if M is None:
            return v
        return torch.as_tensor(M(v), dtype=torch.float64, device=v.device).contiguous()

    bn = float(np.sqrt(dot(b, b)))
    target = max(tol * bn, atol)
    total = 0
    beta = float("inf")
    while True:
        r = b.clone()
        axpby(-1.0, A(x), 1.0, r)
        beta = float(np.sqrt(dot(r, r)))
        if beta <= target or total >= maxiter:
            break
        m = min(restart, maxiter - total)
        V = [r / beta]
        Z = []
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        g[0] = beta
        cs, sn = np.zeros(m), np.zeros(m)
        j_end = 0
        for j in range(m):
            z = Minv(V[j])
            Z.append(z)
            w = A(z)
            for i in range(j + 1):
                H[i, j] = dot(w, V[i])
                axpby(-H[i, j], V[i], 1.0, w)
            hn = float(np.sqrt(dot(w, w)))
            H[j + 1, j] = hn
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = np.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if den == 0.0 else (H[j, j] / den, H[j + 1, j] / den)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            total += 1
            j_end = j + 1
            if abs(g[j + 1]) <= target or H[j, j] == 0.0:
                break
            V.append(w / hn)
        y = np.linalg.solve(np.triu(H[:j_end, :j_end]), g[:j_end])
        for i in range(j_end):
            axpby(float(y[i]), Z[i], 1.0, x)
    status = "converged" if beta <= target else "maxiter"
    return SolveInfo(status, total, beta, bn)
