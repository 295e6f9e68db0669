"""Device-resident curved-element SIPG operator: the owner of one
``ddg_curved_op`` handle (``libddg_sipg.so``).

Built from a ``Mesh2D`` whose geometric factors vary node by node and,
optionally, its ``MeshCubature``.  Every operation takes the quadrature to
use: ``"nodal"`` (the reference's ``cub=None`` on such a mesh) or
``"cubature"`` (its ``cub=...`` branch).  Vectors are element-major flat
float64 torch CUDA tensors used as device buffers; all arithmetic runs in the
library.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib

_QUAD = {"nodal": _lib.DDG_QUAD_NODAL, "cubature": _lib.DDG_QUAD_CUBATURE}


class CurvedOperator:
    def __init__(self, mesh, bc_types: np.ndarray, *, tau_scale: float = 200.0, cub=None, device: int = 0):
        import torch
        if not torch.cuda.is_available():
            raise _lib.DdgError(-1, "CurvedOperator", "no CUDA device: the SIPG kernels need a B200 GPU")
        if mesh.N > _lib.DDG_MAX_DEGREE:
            raise _lib.DdgError(3, "CurvedOperator", f"degree {mesh.N} > {_lib.DDG_MAX_DEGREE} not built")
        L = _lib.lib()
        ref = mesh.ref
        self.mesh = mesh
        self.cub = cub
        self.N, self.Np, self.K = mesh.N, mesh.Np, mesh.K
        self.n = mesh.Np * mesh.K
        self.tau_scale = float(tau_scale)
        self.device = device
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)    # noqa: E731
        keep = dict(Dr=f64(ref.Dr), Ds=f64(ref.Ds), M=f64(ref.M), m1d=f64(ref.m1d), Fmask=i64(ref.Fmask),
                    rx=f64(mesh.rx), sx=f64(mesh.sx), ry=f64(mesh.ry), sy=f64(mesh.sy), J=f64(mesh.J),
                    nx=f64(mesh.nx), ny=f64(mesh.ny), sJ=f64(mesh.sJ), Fscale=f64(mesh.Fscale),
                    EToE=i64(mesh.EToE), EToF=i64(mesh.EToF), vmapM=i64(mesh.vmapM), vmapP=i64(mesh.vmapP),
                    bc=np.ascontiguousarray(bc_types, dtype=np.int32))
        Ncub = Nfq = 0
        if cub is not None:
            Ncub, Nfq = int(cub.w.shape[0]), int(cub.face_w.shape[0])
            keep.update(cw=f64(cub.w), Drq=f64(cub.Drq), Dsq=f64(cub.Dsq), Lq=f64(cub.Lq), cJ=f64(cub.J),
                        crx=f64(cub.rx), csx=f64(cub.sx), cry=f64(cub.ry), csy=f64(cub.sy),
                        face_w=f64(cub.face_w), face_L1d=f64(cub.face_L1d), face_sJ=f64(cub.face_sJ))
        dp = lambda k: keep[k].ctypes.data_as(C.POINTER(C.c_double)) if k in keep else None  # noqa: E731
        ip = lambda k: keep[k].ctypes.data_as(C.POINTER(C.c_int64))                          # noqa: E731
        d = _lib.CurvedDesc(N=mesh.N, K=mesh.K, device=device, Ncub=Ncub, Nfq=Nfq, reserved=0,
                            tau_scale=self.tau_scale, Dr=dp("Dr"), Ds=dp("Ds"), M=dp("M"), m1d=dp("m1d"),
                            Fmask=ip("Fmask"), rx=dp("rx"), sx=dp("sx"), ry=dp("ry"), sy=dp("sy"), J=dp("J"),
                            nx=dp("nx"), ny=dp("ny"), sJ=dp("sJ"), Fscale=dp("Fscale"),
                            EToE=ip("EToE"), EToF=ip("EToF"), vmapM=ip("vmapM"), vmapP=ip("vmapP"),
                            bc_types=keep["bc"].ctypes.data_as(C.POINTER(C.c_int32)),
                            cw=dp("cw"), Drq=dp("Drq"), Dsq=dp("Dsq"), Lq=dp("Lq"), cJ=dp("cJ"), crx=dp("crx"),
                            csx=dp("csx"), cry=dp("cry"), csy=dp("csy"), face_w=dp("face_w"),
                            face_L1d=dp("face_L1d"), face_sJ=dp("face_sJ"))
        h = C.c_void_p()
        _lib.check(L.ddg_curved_create(C.byref(d), C.byref(h)), "ddg_curved_create")
        self._h = h
        self.bc = keep["bc"].copy()
        self.pc_alpha = None
        self.pc_quad = None
        # the operator's own quadrature: the cubature rule when one is attached
        self.quad = "cubature" if cub is not None else "nodal"

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().ddg_curved_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bc(self, bc_types):
        bc = np.ascontiguousarray(bc_types, dtype=np.int32)
        if np.array_equal(bc, self.bc):
            return
        _lib.check(_lib.lib().ddg_curved_set_bc(self._h, bc.ctypes.data_as(C.POINTER(C.c_int32))),
                   "ddg_curved_set_bc")
        self.bc = bc.copy()
        self.pc_alpha = self.pc_quad = None

    # -- helpers ---------------------------------------------------------------
    def _dev(self):
        import torch
        return torch.device("cuda", self.device)

    def _q(self, quad):
        q = self.quad if quad is None else quad
        if q not in _QUAD:
            raise ValueError(f"quad must be 'nodal' or 'cubature', got {q!r}")
        return _QUAD[q]

    def _vec(self, v):
        import torch
        t = torch.as_tensor(v, device=self._dev())
        if t.dtype != torch.float64:
            t = t.to(torch.float64)
        t = t.contiguous()
        if t.numel() != self.n:
            raise ValueError(f"vector has {t.numel()} entries, expected K*Np = {self.n}")
        return t

    # -- operator --------------------------------------------------------------
    def apply(self, u, *, alpha: float = 0.0, out=None, quad=None, stream=None):
        """y = A u + alpha M u (float64 flat device vectors)."""
        import torch
        u = self._vec(u)
        y = torch.empty_like(u) if out is None else out
        _lib.check(_lib.lib().ddg_curved_apply(self._h, self._q(quad), float(alpha), u.data_ptr(), y.data_ptr(),
                                               _lib.stream_handle(stream)), "ddg_curved_apply")
        return y

    def apply_dir(self, u, u_dir, *, out=None, quad=None, stream=None):
        """A u plus the Dirichlet load of the ghost ``u_dir`` (``u`` None: the
        load alone), both by ``quad``."""
        import torch
        u = None if u is None else self._vec(u)
        u_dir = self._vec(u_dir)
        y = torch.empty_like(u_dir) if out is None else out
        _lib.check(_lib.lib().ddg_curved_apply_dir(self._h, self._q(quad), _lib.ptr(u), u_dir.data_ptr(),
                                                   y.data_ptr(), _lib.stream_handle(stream)), "ddg_curved_apply_dir")
        return y

    def mass(self, f, *, out=None, quad=None, stream=None):
        import torch
        f = self._vec(f)
        y = torch.empty_like(f) if out is None else out
        _lib.check(_lib.lib().ddg_curved_mass(self._h, self._q(quad), f.data_ptr(), y.data_ptr(),
                                              _lib.stream_handle(stream)), "ddg_curved_mass")
        return y

    def rhs(self, f=None, u_dir=None, q_neu=None, *, quad=None, stream=None):
        """M f - L_D(u_dir) + L_N(q_neu): the mass by ``quad``, the loads by
        the nodal face rule (as the reference's load functions)."""
        import torch
        out = torch.empty(self.n, dtype=torch.float64, device=self._dev())
        f = None if f is None else self._vec(f)
        u_dir = None if u_dir is None else self._vec(u_dir)
        if q_neu is not None:
            q_neu = torch.as_tensor(q_neu, dtype=torch.float64, device=self._dev()).contiguous()
        _lib.check(_lib.lib().ddg_curved_rhs(self._h, self._q(quad), _lib.ptr(f), _lib.ptr(u_dir), _lib.ptr(q_neu),
                                             out.data_ptr(), _lib.stream_handle(stream)), "ddg_curved_rhs")
        return out

    # -- block Jacobi ------------------------------------------------------------
    def pc_build(self, alpha: float = 0.0, quad=None, stream=None):
        _lib.check(_lib.lib().ddg_curved_pc_build(self._h, self._q(quad), float(alpha), _lib.stream_handle(stream)),
                   "ddg_curved_pc_build")
        self.pc_alpha = float(alpha)
        self.pc_quad = self.quad if quad is None else quad

    def pc_apply(self, r, out=None, stream=None):
        import torch
        r = self._vec(r)
        z = torch.empty_like(r) if out is None else out
        _lib.check(_lib.lib().ddg_curved_pc_apply(self._h, r.data_ptr(), z.data_ptr(), _lib.stream_handle(stream)),
                   "ddg_curved_pc_apply")
        return z

    def pc_blocks(self):
        import torch
        b = torch.empty((self.K, self.Np, self.Np), dtype=torch.float64, device=self._dev())
        _lib.check(_lib.lib().ddg_curved_pc_blocks(self._h, b.data_ptr(), _lib.stream_handle(None)),
                   "ddg_curved_pc_blocks")
        return b

    # -- Krylov ----------------------------------------------------------------
    def cg(self, b, x, *, tol=1e-9, atol=0.0, maxiter=1000, pc=False, alpha=0.0, shift=0.0, quad=None,
           precision="fp64", stream=None):
        """Device CG (graph loop) on (alpha M + A + shift I) x = b; ``x`` holds
        x0 and is overwritten.  Returns (status, iterations, r.r, b.b)."""
        if precision != "fp64":
            raise ValueError("the curved-element operator solves in float64")
        info = _lib.SolveInfo()
        cfg = _lib.CgConfig(tol=float(tol), atol=float(atol), maxiter=int(maxiter),
                            pc=_lib.DDG_PC_JACOBI if pc else _lib.DDG_PC_NONE,
                            alpha=float(alpha), shift=float(shift), precision=_lib.DDG_FP64, reserved=0)
        _lib.check(_lib.lib().ddg_curved_cg(self._h, self._q(quad), C.byref(cfg), b.data_ptr(), x.data_ptr(),
                                            _lib.stream_handle(stream), C.byref(info)), "ddg_curved_cg")
        return _lib.SOLVE_STATUS.get(info.status, str(info.status)), info.iterations, info.res_norm2, info.b_norm2
