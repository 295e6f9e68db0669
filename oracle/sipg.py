"""Oracle: SIPG operator, loads, CG, block-Jacobi and the Poisson/Helmholtz
solves, float64.

Test infrastructure only (see ``oracle/__init__.py``).

Restates ``src/ddg/dg2d/sipg.py`` (all of :53-918) and, for the Krylov loop,
the published algorithm of ``jax.scipy.sparse.linalg.cg`` (a third-party
function, not under the reference tree; ``pyproject.toml:30-33`` pins no
JAX version).  Its semantics, as used at ``sipg.py:604,910``: x0 defaults to
0, r0 = b - A x0, stop when r.r <= max(tol^2 b.b, atol^2) or k == maxiter,
checked before every iteration; the preconditioner is applied as z = M(r).

Two restatements of the operator are kept:
  * :func:`bilinear_form_torch` / :func:`apply_autograd` -- the literal
    scalar form ``sipg_bilinear_form`` (:142-301) differentiated with
    ``torch.autograd.grad`` in place of ``jax.grad`` (:331-337);
  * :func:`apply` -- the same derivative written out explicitly as the
    scatter-add transpose AD produces (numpy, batched over trailing columns).
The tests require them to agree to 1e-13.
"""

from __future__ import annotations

import numpy as np

BC_INTERIOR = 0
BC_DIRICHLET = 1
BC_NEUMANN = 2


class IterativeConfig:
    """``src/ddg/dg2d/sipg.py:59-71``."""

    def __init__(self, method="cg", tol=1e-9, atol=0.0, maxiter=1000):
        self.method, self.tol, self.atol, self.maxiter = method, tol, atol, maxiter


# ------------------------------------------------------------ helpers -----

def bc_face_arrays(mesh, bc_types):
    """``sipg.py:117-139``: per-face-node flags (F order), per-face tags
    (Nfaces, K) and weights (0.5 interior, 1 Dirichlet, 0 Neumann)."""
    bcf = np.asarray(bc_types).T.astype(np.int32)                    # (3, K)
    bcn = np.broadcast_to(bcf[None], (mesh.Nfp, 3, mesh.K)).reshape(-1, order="F")
    w = np.where(bcf == BC_DIRICHLET, 1.0, np.where(bcf == BC_NEUMANN, 0.0, 0.5))
    return bcn, bcf, w


def _flat(u):
    """(Np, K[, B]) -> element-major flat (K*Np, B)."""
    if u.ndim == 2:
        u = u[:, :, None]
    Np, K, B = u.shape
    return u.transpose(1, 0, 2).reshape(K * Np, B)


def _unflat(f, Np, K):
    B = f.shape[1]
    return f.reshape(K, Np, B).transpose(1, 0, 2)


def _face(mesh, a):
    """flat (3 Nfp K[, B]) -> (Nfp, 3, K[, B]) (the reference's order='F')."""
    if a.ndim == 1:
        return a.reshape((mesh.Nfp, 3, mesh.K), order="F")
    B = a.shape[1]
    return a.reshape(mesh.K, 3, mesh.Nfp, B).transpose(2, 1, 0, 3)


def _unface(mesh, a):
    """(Nfp, 3, K, B) -> flat (3 Nfp K, B)."""
    B = a.shape[3]
    return a.transpose(2, 1, 0, 3).reshape(-1, B)


# ----------------------------------------------------- the operator -------

def apply(mesh, u, *, bc_types, u_dir=None, tau_scale=200.0, kappa=None, cub=None):
    """Explicit ``sipg_apply_2d`` (``sipg.py:304-337``): d a(u, v) / d v at
    v = 0, including the affine Dirichlet offset when ``u_dir`` is given.

    ``u`` is (Np, K) or (Np, K, B); the result has the same shape.

    ``cub`` (an ``oracle.cubature.MeshCubature``) selects the curved-element
    branch (``sipg.py:190-201`` volume, ``sipg.py:281-299`` faces): the
    volume integral at the cubature points with their geometric factors, the
    face integrals at the 1D face points with the surface Jacobian there
    (normals, tau and the traces stay nodal).

    ``kappa`` (K,) is the per-element diffusivity extension (no reference
    counterpart): volume kappa_k grad u . grad v, face averages
    {kappa grad u . n} = (kappa_M Dn_M + kappa_P Dn_P)/2, penalty weighted by
    kappa_F = (kappa_M + kappa_P)/2 (kappa_M on boundary faces).  kappa = 1
    is the reference operator.
    """
    squeeze = u.ndim == 2
    ref = mesh.ref
    Np, K, Nfp = mesh.Np, mesh.K, mesh.Nfp
    U = u[:, :, None] if squeeze else u
    B = U.shape[2]
    M, m1d = ref.M, ref.m1d
    Dr, Ds = ref.Dr, ref.Ds
    rx, sx, ry, sy, J = (a[:, :, None] for a in (mesh.rx, mesh.sx, mesh.ry, mesh.sy, mesh.J))
    kap = np.ones(K) if kappa is None else np.asarray(kappa, dtype=np.float64)
    kvol = kap[None, :, None]

    ur = np.einsum("ij,jkb->ikb", Dr, U)
    us = np.einsum("ij,jkb->ikb", Ds, U)
    ux = rx * ur + sx * us
    uy = ry * ur + sy * us

    if cub is None:
        # volume term sum J*(ux*(M vx) + uy*(M vy))  (sipg.py:189)
        cx = np.einsum("ji,jkb->ikb", M, kvol * J * ux)     # M^T (kappa J ux)
        cy = np.einsum("ji,jkb->ikb", M, kvol * J * uy)
        gx = cx.copy()                                       # dL/dvx (per node)
        gy = cy.copy()
        yvol = 0.0
    else:
        if kappa is not None:
            raise ValueError("kappa is not defined for the cubature branch")
        # sum_q w J (ux_q vx_q + uy_q vy_q)  (sipg.py:191-201)
        urq = np.einsum("qi,ikb->qkb", cub.Drq, U)
        usq = np.einsum("qi,ikb->qkb", cub.Dsq, U)
        crx, csx, cry, csy = (a[:, :, None] for a in (cub.rx, cub.sx, cub.ry, cub.sy))
        wJ = (cub.w[:, None] * cub.J)[:, :, None]
        uxq = crx * urq + csx * usq
        uyq = cry * urq + csy * usq
        yvol = (np.einsum("qi,qkb->ikb", cub.Drq, wJ * (crx * uxq + cry * uyq))
                + np.einsum("qi,qkb->ikb", cub.Dsq, wJ * (csx * uxq + csy * uyq)))
        gx = np.zeros_like(U)
        gy = np.zeros_like(U)

    # traces (sipg.py:204-249)
    uf, uxf, uyf = _flat(U), _flat(ux), _flat(uy)
    vM, vP = mesh.vmapM, mesh.vmapP
    nxf = mesh.nx.reshape(-1, order="F")[:, None]
    nyf = mesh.ny.reshape(-1, order="F")[:, None]
    uM, uPraw = uf[vM], uf[vP]
    DnM = nxf * uxf[vM] + nyf * uyf[vM]
    DnPraw = nxf * uxf[vP] + nyf * uyf[vP]
    bcn, bcf, w = bc_face_arrays(mesh, bc_types)
    isd = (bcn == BC_DIRICHLET)[:, None]
    isn = (bcn == BC_NEUMANN)[:, None]
    isb = isd | isn
    uPd = np.zeros_like(uM) if u_dir is None else _flat(np.asarray(u_dir, dtype=np.float64))[vM]
    if uPd.shape[1] != B:
        uPd = np.broadcast_to(uPd, uM.shape)
    uPeff = np.where(isd, uPd, np.where(isn, uM, uPraw))
    DnPeff = np.where(isb, DnM, DnPraw)
    kM = kap[vM // Np][:, None]
    kP = np.where(isb, kM, kap[vP // Np][:, None])
    avg = 0.5 * (kM * DnM + kP * DnPeff)
    jmp = uM - uPeff
    kF = _face(mesh, (0.5 * (kM + kP))[:, 0])                         # (Nfp,3,K)

    sJ1 = _face(mesh, mesh.sJ.reshape(-1, order="F"))[0]             # (3, K)
    Fs1 = _face(mesh, mesh.Fscale.reshape(-1, order="F"))[0]
    tau = tau_scale * (mesh.N + 1) * (mesh.N + 1) * Fs1
    avgF, jmpF = _face(mesh, avg), _face(mesh, jmp)                   # (Nfp,3,K,B)
    if cub is None:
        wsJ = (w * sJ1)[None, :, :, None]
        wtsJ = (w * tau * sJ1)[None, :, :, None] * kF[0][None, :, :, None]
        # d/d(jmp_v): -w sJ m1d^T avg + w tau kappa_F sJ m1d^T jmp   (sipg.py:270-279)
        dj = (-wsJ * np.einsum("fpq,pfkb->qfkb", m1d, avgF)
              + wtsJ * np.einsum("fpq,pfkb->qfkb", m1d, jmpF))
        # d/d(avg_v): -w sJ m1d^T jmp_u
        da = -wsJ * np.einsum("fpq,pfkb->qfkb", m1d, jmpF)
    else:
        # face cubature (sipg.py:284-299): traces interpolated by face_L1d,
        # weights face_w * face_sJ * w at the face points
        L1 = cub.face_L1d                                              # (3, Nq, Nfp)
        Wq = (cub.face_w[:, None, None] * np.transpose(cub.face_sJ, (1, 0, 2))
              * w[None, :, :])[:, :, :, None]                          # (Nq, 3, K, 1)
        avq = np.einsum("fqp,pfkb->qfkb", L1, avgF)
        jmq = np.einsum("fqp,pfkb->qfkb", L1, jmpF)
        tq = tau[None, :, :, None]
        dj = np.einsum("fqp,qfkb->pfkb", L1, Wq * (-avq + tq * jmq))
        da = -np.einsum("fqp,qfkb->pfkb", L1, Wq * jmq)
    dj, da = _unface(mesh, dj), _unface(mesh, da)

    yf = np.zeros((K * Np, B))
    gxf = np.zeros((K * Np, B))
    gyf = np.zeros((K * Np, B))
    # jmp_v = v_M - v_Peff: Neumann faces cancel, interior faces scatter to P
    isi = (bcn == BC_INTERIOR)
    np.add.at(yf, vM, np.where(isn, 0.0, dj))
    np.add.at(yf, vP[isi], -dj[isi])
    # avg_v = 0.5 (Dn_vM + Dn_vPeff), Dn_vPeff = Dn_vM on boundary faces
    cM = np.where(isb, 1.0, 0.5) * kM
    np.add.at(gxf, vM, cM * nxf * da)
    np.add.at(gyf, vM, cM * nyf * da)
    np.add.at(gxf, vP[isi], 0.5 * kP[isi] * nxf[isi] * da[isi])
    np.add.at(gyf, vP[isi], 0.5 * kP[isi] * nyf[isi] * da[isi])

    gx = gx + _unflat(gxf, Np, K)
    gy = gy + _unflat(gyf, Np, K)
    y = _unflat(yf, Np, K) + yvol
    y = y + np.einsum("ji,jkb->ikb", Dr, rx * gx + ry * gy) \
          + np.einsum("ji,jkb->ikb", Ds, sx * gx + sy * gy)
    return y[:, :, 0] if squeeze else y


def bilinear_form_torch(mesh, u, v, *, bc_types, u_dir=None, tau_scale=200.0, kappa=None, cub=None):
    """Literal restatement of ``sipg_bilinear_form`` (``sipg.py:142-301``,
    both the nodal ``cub=None`` branch and the cubature branch) on torch
    float64 tensors; ``kappa`` (a (K,) tensor, may require grad) adds the
    diffusivity extension described in :func:`apply` (kappa = 1 is the
    reference form; nodal branch only)."""
    import torch
    ref = mesh.ref
    T = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64)  # noqa: E731
    Np, K, Nfp = mesh.Np, mesh.K, mesh.Nfp
    M, Dr, Ds, m1d = T(ref.M), T(ref.Dr), T(ref.Ds), T(ref.m1d)
    rx, sx, ry, sy, J = T(mesh.rx), T(mesh.sx), T(mesh.ry), T(mesh.sy), T(mesh.J)
    ux = rx * (Dr @ u) + sx * (Ds @ u)
    uy = ry * (Dr @ u) + sy * (Ds @ u)
    vx = rx * (Dr @ v) + sx * (Ds @ v)
    vy = ry * (Dr @ v) + sy * (Ds @ v)
    kap = torch.ones(K, dtype=torch.float64) if kappa is None else kappa
    if cub is None:
        vol = torch.sum(kap[None, :] * J * (ux * (M @ vx) + uy * (M @ vy)))
    else:
        Drq, Dsq = T(cub.Drq), T(cub.Dsq)
        crx, csx, cry, csy = T(cub.rx), T(cub.sx), T(cub.ry), T(cub.sy)
        uxq = crx * (Drq @ u) + csx * (Dsq @ u)
        uyq = cry * (Drq @ u) + csy * (Dsq @ u)
        vxq = crx * (Drq @ v) + csx * (Dsq @ v)
        vyq = cry * (Drq @ v) + csy * (Dsq @ v)
        vol = torch.sum(T(cub.w)[:, None] * T(cub.J) * (uxq * vxq + uyq * vyq))
    fl = lambda a: a.T.reshape(-1)  # noqa: E731
    vM, vP = torch.as_tensor(mesh.vmapM), torch.as_tensor(mesh.vmapP)
    nx = T(mesh.nx.reshape(-1, order="F"))
    ny = T(mesh.ny.reshape(-1, order="F"))
    u_M, u_P = fl(u)[vM], fl(u)[vP]
    v_M, v_P = fl(v)[vM], fl(v)[vP]
    DuM = nx * fl(ux)[vM] + ny * fl(uy)[vM]
    DuP = nx * fl(ux)[vP] + ny * fl(uy)[vP]
    DvM = nx * fl(vx)[vM] + ny * fl(vy)[vM]
    DvP = nx * fl(vx)[vP] + ny * fl(vy)[vP]
    bcn, bcf, w = bc_face_arrays(mesh, bc_types)
    isd = torch.as_tensor(bcn == BC_DIRICHLET)
    isn = torch.as_tensor(bcn == BC_NEUMANN)
    isb = isd | isn
    tf = lambda a: a.reshape(K, 3, Nfp).permute(2, 1, 0)  # noqa: E731  (Nfp,3,K)
    uPd = torch.zeros_like(u_M) if u_dir is None else fl(T(u_dir))[vM]
    vPd = torch.zeros_like(v_M)
    uPe = torch.where(isd, uPd, torch.where(isn, u_M, u_P))
    vPe = torch.where(isd, vPd, torch.where(isn, v_M, v_P))
    kM = kap[vM // Np]
    kP = torch.where(isb, kM, kap[vP // Np])
    aDu = 0.5 * (kM * DuM + kP * torch.where(isb, DuM, DuP))
    aDv = 0.5 * (kM * DvM + kP * torch.where(isb, DvM, DvP))
    kF = tf(0.5 * (kM + kP))[0]                                       # (3, K)
    ju, jv = u_M - uPe, v_M - vPe
    sJ1 = T(mesh.sJ.reshape((Nfp, 3, K), order="F")[0])
    Fs1 = T(mesh.Fscale.reshape((Nfp, 3, K), order="F")[0])
    tau = tau_scale * (mesh.N + 1) * (mesh.N + 1) * Fs1
    wt = T(w)
    if cub is not None:
        L1 = T(cub.face_L1d)
        q = lambda a: torch.einsum("fqp,pfk->qfk", L1, tf(a))  # noqa: E731
        W = T(cub.face_w)[:, None, None] * T(np.transpose(cub.face_sJ, (1, 0, 2))) * wt[None]
        cons = -torch.sum(W * q(aDu) * q(jv))
        adj = -torch.sum(W * q(ju) * q(aDv))
        pen = torch.sum(W * tau[None] * q(ju) * q(jv))
        return vol + cons + adj + pen
    wsJ = wt * sJ1
    cons = -torch.einsum("fk,pfk,fpq,qfk->", wsJ, tf(aDu), m1d, tf(jv))
    adj = -torch.einsum("fk,pfk,fpq,qfk->", wsJ, tf(ju), m1d, tf(aDv))
    pen = torch.einsum("fk,pfk,fpq,qfk->", wt * tau * sJ1 * kF, tf(ju), m1d, tf(jv))
    return vol + cons + adj + pen


def apply_autograd(mesh, u, *, bc_types, u_dir=None, tau_scale=200.0, kappa=None, cub=None):
    """``sipg_apply_2d`` exactly as the reference computes it: the gradient
    of the scalar form w.r.t. v at v = 0 (``sipg.py:329-337``)."""
    import torch
    ut = torch.as_tensor(np.asarray(u), dtype=torch.float64)
    v = torch.zeros_like(ut, requires_grad=True)
    kt = None if kappa is None else torch.as_tensor(np.asarray(kappa), dtype=torch.float64)
    a = bilinear_form_torch(mesh, ut, v, bc_types=bc_types, u_dir=u_dir, tau_scale=tau_scale, kappa=kt,
                            cub=cub)
    (g,) = torch.autograd.grad(a, v)
    return g.numpy()


def grad_kappa(mesh, u, lam, *, bc_types, tau_scale=200.0, kappa=None):
    """d a(u, lam; kappa) / d kappa_k per element, by torch autograd of the
    literal form (a is linear in kappa, so this is exact).  With u the
    solution of A(kappa) u = b and lam the adjoint A lam = dL/du, the loss
    gradient is dL/dkappa = -grad_kappa(u, lam)."""
    import torch
    K = mesh.K
    kt = torch.as_tensor(np.ones(K) if kappa is None else np.asarray(kappa), dtype=torch.float64)
    kt.requires_grad_(True)
    a = bilinear_form_torch(mesh, torch.as_tensor(np.asarray(u), dtype=torch.float64),
                            torch.as_tensor(np.asarray(lam), dtype=torch.float64),
                            bc_types=bc_types, tau_scale=tau_scale, kappa=kt)
    (g,) = torch.autograd.grad(a, kt)
    return g.numpy()


def mass_apply(mesh, u, cub=None):
    """J * (M_ref u), ``sipg.py:565,597,853``; with ``cub`` the cubature
    mass ``cubature_mass_apply`` (``cubature.py:243-254``)."""
    if cub is not None:
        from .cubature import cubature_mass_apply
        return cubature_mass_apply(cub, u)
    if u.ndim == 3:
        return mesh.J[:, :, None] * np.einsum("ij,jkb->ikb", mesh.ref.M, u)
    return mesh.J * (mesh.ref.M @ u)


def flat_op(mesh, *, bc_types, tau_scale=200.0, alpha=0.0, kappa=None, cub=None):
    """Matvec on the element-major flat vector; ``alpha M + A`` (alpha=0:
    ``sipg.py:876-883``; alpha>0: ``sipg.py:589-601`` and
    ``multigrid.py:53-74``).  Accepts (n,) or (n, B)."""
    Np, K = mesh.Np, mesh.K

    def op(x):
        X = x[:, None] if x.ndim == 1 else x
        U = _unflat(X, Np, K)
        Y = apply(mesh, U, bc_types=bc_types, tau_scale=tau_scale, kappa=kappa, cub=cub)
        if alpha != 0.0:
            Y = Y + alpha * mass_apply(mesh, U, cub)
        out = _flat(Y)
        return out[:, 0] if x.ndim == 1 else out
    return op


def dense_matrix(mesh, *, bc_types, tau_scale=200.0, alpha=0.0, chunk=512, kappa=None, cub=None):
    """``sipg_matrix_2d`` (``sipg.py:344-364``) / ``sipg_helmholtz_matrix_2d``
    (``:460-496``; ``nu`` unused there too): columns of the apply."""
    n = mesh.Np * mesh.K
    op = flat_op(mesh, bc_types=bc_types, tau_scale=tau_scale, alpha=alpha, kappa=kappa, cub=cub)
    A = np.zeros((n, n))
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        E = np.zeros((n, c1 - c0))
        E[np.arange(c0, c1), np.arange(c1 - c0)] = 1.0
        A[:, c0:c1] = op(E)
    return A


# ------------------------------------------------------------- loads ------

def dirichlet_load(mesh, u_dir, *, bc_types, tau_scale=200.0):
    """``sipg.py:398-417``: apply(0; u_dir)."""
    return apply(mesh, np.zeros_like(u_dir), bc_types=bc_types, u_dir=u_dir, tau_scale=tau_scale)


def neumann_load(mesh, q_neu, *, bc_types):
    """``sipg.py:420-453``: sJ m1d q on Neumann faces, scattered to Fmask."""
    Nfp, K = mesh.Nfp, mesh.K
    _, bcf, _ = bc_face_arrays(mesh, bc_types)
    isnf = (bcf == BC_NEUMANN).astype(np.float64)
    qf = np.asarray(q_neu).reshape((Nfp, 3, K), order="F")
    sJ1 = mesh.sJ.reshape((Nfp, 3, K), order="F")[0]
    c = np.einsum("fpq,qfk->pfk", mesh.ref.m1d, qf) * (sJ1 * isnf)[None]
    out = np.zeros((mesh.Np, K))
    for f in range(3):
        np.add.at(out, mesh.ref.Fmask[:, f], c[:, f, :])
    return out


# ---------------------------------------------------------------- CG ------

def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """Restatement of the published ``jax.scipy.sparse.linalg.cg`` loop.
    Returns ``(x, iterations)``."""
    if maxiter is None:
        maxiter = 10 * b.shape[0]
    Mf = (lambda v: v) if M is None else M
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    atol2 = max(tol * tol * float(b @ b), atol * atol)
    r = b - A(x)
    z = Mf(r)
    p = z.copy()
    gamma = float(r @ z)
    k = 0
    while True:
        rs = gamma if M is None else float(r @ r)
        if not (rs > atol2 and k < maxiter):
            break
        Ap = A(p)
        alpha = gamma / float(p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = Mf(r)
        g2 = float(r @ z)
        p = z + (g2 / gamma) * p
        gamma = g2
        k += 1
    return x, k


# ------------------------------------------------------- block Jacobi -----

def color_elements(mesh):
    """``sipg.py:651-668``: greedy colouring in element order."""
    K = mesh.K
    col = -np.ones(K, dtype=np.int64)
    for k in range(K):
        used = {int(col[nb]) for nb in mesh.EToE[k] if nb != k and col[nb] >= 0}
        c = 0
        while c in used:
            c += 1
        col[k] = c
    return col, int(col.max()) + 1


def extract_block_diag_matfree(apply_flat, mesh):
    """``sipg.py:671-704``: coloured probing, ncolours*Np applies."""
    Np, K = mesh.Np, mesh.K
    col, nc = color_elements(mesh)
    blocks = np.zeros((K, Np, Np))
    for c in range(nc):
        mask = (col == c).astype(np.float64)
        for j in range(Np):
            probe = np.zeros((K, Np))
            probe[:, j] = mask
            r = apply_flat(probe.reshape(-1)).reshape(K, Np)
            blocks[:, :, j] += np.where(mask[:, None] > 0, r, 0.0)
    return blocks


def extract_block_diag_dense(A, Np, K):
    """``sipg.py:636-648``."""
    rows = np.arange(K)[:, None] * Np + np.arange(Np)[None, :]
    return A[rows[:, :, None], rows[:, None, :]]


def block_jacobi_from_blocks(blocks):
    """``sipg.py:707-715``: explicit inverses, batched GEMV."""
    Binv = np.linalg.inv(blocks)
    K, Np, _ = blocks.shape

    def Minv(v):
        return np.einsum("kij,kj->ki", Binv, v.reshape(K, Np)).reshape(-1)
    Minv.Binv = Binv
    return Minv


def make_block_jacobi(mesh, *, bc_types, tau_scale=200.0, alpha=0.0, matfree=True):
    """``make_sipg_block_jacobi_preconditioner`` (``sipg.py:718-761``) and
    its Helmholtz twin (``:764-805``) in one (alpha = 0 is the SIPG one)."""
    if matfree:
        blocks = extract_block_diag_matfree(
            flat_op(mesh, bc_types=bc_types, tau_scale=tau_scale, alpha=alpha), mesh)
    else:
        A = dense_matrix(mesh, bc_types=bc_types, tau_scale=tau_scale, alpha=alpha)
        blocks = extract_block_diag_dense(A, mesh.Np, mesh.K)
    return block_jacobi_from_blocks(blocks)


# ------------------------------------------------------------ solves ------

def _rhs(mesh, source, bc_types, u_dir, q_neu, tau_scale, cub=None):
    # the mass of the source uses the cubature; the Dirichlet load does not
    # (sipg.py:852-864, :404-417)
    rhs = mass_apply(mesh, np.asarray(source, dtype=np.float64), cub)
    if u_dir is not None:
        rhs = rhs - dirichlet_load(mesh, np.asarray(u_dir, dtype=np.float64),
                                   bc_types=bc_types, tau_scale=tau_scale)
    if q_neu is not None:
        rhs = rhs + neumann_load(mesh, q_neu, bc_types=bc_types)
    return rhs.T.reshape(-1)


def solve_poisson(mesh, source, *, bc_types, u_dir=None, q_neu=None, tau_scale=200.0,
                  iterative=None, x0=None, preconditioner=None, return_info=False, cub=None):
    """``solve_sipg_poisson_2d`` (``sipg.py:812-918``)."""
    import scipy.linalg as sla
    Np, K = mesh.Np, mesh.K
    b = _rhs(mesh, source, bc_types, u_dir, q_neu, tau_scale, cub)
    if iterative is None:
        A = dense_matrix(mesh, bc_types=bc_types, tau_scale=tau_scale, cub=cub)
        x = sla.lu_solve(sla.lu_factor(A), b)
        return x.reshape(K, Np).T
    raw = flat_op(mesh, bc_types=bc_types, tau_scale=tau_scale, cub=cub)
    singular = not bool(np.any(np.asarray(bc_types) == BC_DIRICHLET))
    if singular:                                                     # :891-906
        probe = np.sin(np.arange(Np * K, dtype=np.float64))
        probe = probe - probe.mean()
        shift = 1.0e-6 * np.linalg.norm(raw(probe)) / np.linalg.norm(probe)
        op = lambda v: raw(v) + shift * v  # noqa: E731
        b = b - b.mean()
    else:
        op = raw
    if iterative.method != "cg":
        raise ValueError(f"iterative method {iterative.method!r} not supported for SPD")
    xf = None if x0 is None else np.asarray(x0).T.reshape(-1)
    x, it = cg(op, b, xf, tol=iterative.tol, atol=iterative.atol,
               maxiter=iterative.maxiter, M=preconditioner)
    u = x.reshape(K, Np).T
    return (u, it) if return_info else u


def solve_helmholtz(mesh, rhs_field, *, alpha, nu=1.0, bc_types, u_dir=None, q_neu=None,
                    tau_scale=200.0, iterative=None, x0=None, preconditioner=None,
                    return_info=False, cub=None):
    """``solve_sipg_helmholtz_2d`` (``sipg.py:536-612``); ``nu`` is unused,
    as in the reference."""
    import scipy.linalg as sla
    Np, K = mesh.Np, mesh.K
    b = _rhs(mesh, rhs_field, bc_types, u_dir, q_neu, tau_scale, cub)
    if iterative is None:
        A = dense_matrix(mesh, bc_types=bc_types, tau_scale=tau_scale, alpha=alpha, cub=cub)
        return sla.lu_solve(sla.lu_factor(A), b).reshape(K, Np).T
    if iterative.method != "cg":
        raise ValueError(f"iterative method {iterative.method!r} not supported for SPD")
    op = flat_op(mesh, bc_types=bc_types, tau_scale=tau_scale, alpha=alpha, cub=cub)
    xf = None if x0 is None else np.asarray(x0).T.reshape(-1)
    x, it = cg(op, b, xf, tol=iterative.tol, atol=iterative.atol,
               maxiter=iterative.maxiter, M=preconditioner)
    u = x.reshape(K, Np).T
    return (u, it) if return_info else u


def boundary_bc(mesh, code=BC_DIRICHLET):
    """Tag every self-pointing face with ``code`` (the tests' helper,
    ``test/test_block_jacobi_preconditioner.py:29-41``)."""
    isb = mesh.EToE == np.arange(mesh.K)[:, None]
    return np.where(isb, code, BC_INTERIOR).astype(np.int32)
