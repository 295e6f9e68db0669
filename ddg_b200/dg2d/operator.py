"""Device-resident SIPG operator: a thin owner of one ``ddg_sipg_op`` handle.

All vectors are torch CUDA tensors used purely as device buffers; every
arithmetic operation runs in ``libddg_sipg.so``.  Vectors are element-major
flat (``u.T.reshape(-1)`` of an ``(Np, K)`` field, ``sipg.py:204``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib


class SipgOperator:
    def __init__(self, mesh, bc_types: np.ndarray, *, tau_scale: float = 200.0, device: int = 0):
        import torch
        if not torch.cuda.is_available():
            raise _lib.DdgError(-1, "SipgOperator", "no CUDA device: the SIPG kernels need a B200 GPU")
        if mesh.N > _lib.DDG_MAX_DEGREE:
            raise _lib.DdgError(3, "SipgOperator", f"degree {mesh.N} > {_lib.DDG_MAX_DEGREE} not built")
        L = _lib.lib()
        ref = mesh.ref
        self.mesh = mesh
        self.N, self.Np, self.K = mesh.N, mesh.Np, mesh.K
        self.n = mesh.Np * mesh.K
        self.tau_scale = float(tau_scale)
        self.device = device
        keep = dict(
            Dr=np.ascontiguousarray(ref.Dr), Ds=np.ascontiguousarray(ref.Ds),
            M=np.ascontiguousarray(ref.M), m1d=np.ascontiguousarray(ref.m1d),
            Fmask=np.ascontiguousarray(ref.Fmask, dtype=np.int64),
            rot=np.ascontiguousarray(ref.rot_perm, dtype=np.int64),
            geo=np.ascontiguousarray(mesh.element_geometry()),
            EToE=np.ascontiguousarray(mesh.EToE, dtype=np.int64),
            EToF=np.ascontiguousarray(mesh.EToF, dtype=np.int64),
            vmapM=np.ascontiguousarray(mesh.vmapM, dtype=np.int64),
            vmapP=np.ascontiguousarray(mesh.vmapP, dtype=np.int64),
            bc=np.ascontiguousarray(bc_types, dtype=np.int32))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))   # noqa: E731
        d = _lib.MeshDesc(N=mesh.N, K=mesh.K, device=device, reserved=0, tau_scale=self.tau_scale,
                          Dr=dp(keep["Dr"]), Ds=dp(keep["Ds"]), M=dp(keep["M"]), m1d=dp(keep["m1d"]),
                          Fmask=ip(keep["Fmask"]), rot_perm=ip(keep["rot"]), geo=dp(keep["geo"]),
                          EToE=ip(keep["EToE"]), EToF=ip(keep["EToF"]),
                          vmapM=ip(keep["vmapM"]), vmapP=ip(keep["vmapP"]),
                          bc_types=keep["bc"].ctypes.data_as(C.POINTER(C.c_int32)))
        h = C.c_void_p()
        _lib.check(L.ddg_sipg_create(C.byref(d), C.byref(h)), "ddg_sipg_create")
        self._h = h
        self.bc = keep["bc"].copy()
        self.pc_alpha = None

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().ddg_sipg_destroy(self._h)
            self._h = None
        self._kappa_state = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bc(self, bc_types):
        bc = np.ascontiguousarray(bc_types, dtype=np.int32)
        if np.array_equal(bc, self.bc):
            return
        _lib.check(_lib.lib().ddg_sipg_set_bc(self._h, bc.ctypes.data_as(C.POINTER(C.c_int32))),
                   "ddg_sipg_set_bc")
        self.bc = bc.copy()
        self.pc_alpha = None

    # -- helpers ---------------------------------------------------------------
    def _dev(self):
        import torch
        return torch.device("cuda", self.device)

    def _vec(self, v, dtype):
        import torch
        t = torch.as_tensor(v, device=self._dev())
        if t.dtype != dtype:
            t = t.to(dtype)
        t = t.contiguous()
        if t.numel() != self.n:
            raise ValueError(f"vector has {t.numel()} entries, expected K*Np = {self.n}")
        return t

    @staticmethod
    def _prec(dtype):
        import torch
        if dtype == torch.float64:
            return _lib.DDG_FP64
        if dtype == torch.float32:
            return _lib.DDG_FP32
        raise TypeError("vectors must be float64 or float32")

    # -- operator --------------------------------------------------------------
    def apply(self, u, *, alpha: float = 0.0, out=None, stream=None):
        """y = A u + alpha J M u on a flat device vector (float64 or float32)."""
        import torch
        u = self._vec(u, u.dtype if isinstance(u, torch.Tensor) and u.dtype in (torch.float32, torch.float64)
                      else torch.float64)
        y = torch.empty_like(u) if out is None else out
        _lib.check(_lib.lib().ddg_sipg_apply(self._h, self._prec(u.dtype), float(alpha), u.data_ptr(),
                                             y.data_ptr(), _lib.stream_handle(stream)), "ddg_sipg_apply")
        return y

    def apply_host(self, u, *, alpha: float = 0.0, out=None, stream=None):
        """y = A u + alpha J M u for a float64 HOST field of shape (Np, K)
        (the reference's own field layout).  Copies, kernels and the copy
        back overlap chunk by chunk inside the library; pinned arrays (see
        :func:`ddg_b200.pinned_empty`) move at full copy-engine speed,
        pageable ones are staged.  Returns ``out`` (allocated if None)."""
        u = np.asarray(u)
        if u.dtype != np.float64 or not u.flags.c_contiguous:
            u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (self.Np, self.K):
            raise ValueError(f"u has shape {u.shape}, expected (Np, K) = {(self.Np, self.K)}")
        y = np.empty((self.Np, self.K), dtype=np.float64) if out is None else out
        if y.shape != (self.Np, self.K) or y.dtype != np.float64 or not y.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 (Np, K) array")
        _lib.check(_lib.lib().ddg_sipg_apply_host(self._h, float(alpha), u.ctypes.data, y.ctypes.data,
                                                  _lib.stream_handle(stream)), "ddg_sipg_apply_host")
        return y

    def set_engine(self, engine: str):
        """Apply engine: "tensor" (float32 on tcgen05 with 3xTF32 splitting,
        degrees 1..4; float64 on the FP64 tensor cores, mma.sync f64, degrees
        1..5) or "cuda" (plain FMA on the CUDA cores).  Default: tensor cores
        for every apply (float64, float32, and the float32 CG iterations)."""
        code = {"tensor": _lib.DDG_ENGINE_TENSOR_CORES, "cuda": _lib.DDG_ENGINE_CUDA_CORES}[engine]
        _lib.check(_lib.lib().ddg_sipg_set_engine(self._h, code), "ddg_sipg_set_engine")

    def rhs(self, f=None, u_dir=None, q_neu=None, stream=None):
        """J M f - L_D(u_dir) + L_N(q_neu), float64 flat vectors (q_neu: face flat)."""
        import torch
        dev = self._dev()
        conv = lambda a: None if a is None else torch.as_tensor(a, dtype=torch.float64, device=dev).contiguous()  # noqa: E731
        f, u_dir, q_neu = conv(f), conv(u_dir), conv(q_neu)
        out = torch.empty(self.n, dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().ddg_sipg_rhs(self._h, _lib.ptr(f), _lib.ptr(u_dir), _lib.ptr(q_neu),
                                           out.data_ptr(), _lib.stream_handle(stream)), "ddg_sipg_rhs")
        return out

    # -- per-element diffusivity (extension) ------------------------------------
    def set_kappa(self, kappa):
        """Set (K positive values) or clear (None) the per-element diffusivity;
        the block-Jacobi preconditioner must be rebuilt afterwards."""
        if kappa is None:
            _lib.check(_lib.lib().ddg_sipg_set_kappa(self._h, None), "ddg_sipg_set_kappa")
        else:
            k = np.ascontiguousarray(np.asarray(kappa, dtype=np.float64).reshape(-1))
            if k.size != self.K:
                raise ValueError(f"kappa needs {self.K} entries")
            _lib.check(_lib.lib().ddg_sipg_set_kappa(self._h, k.ctypes.data), "ddg_sipg_set_kappa")
        self.pc_alpha = None

    def grad_kappa(self, u, lam, stream=None):
        """g_k = d a(u, lam; kappa) / d kappa_k (float64 device vectors)."""
        import torch
        g = torch.empty(self.K, dtype=torch.float64, device=self._dev())
        _lib.check(_lib.lib().ddg_sipg_grad_kappa(self._h, u.data_ptr(), lam.data_ptr(), g.data_ptr(),
                                                  _lib.stream_handle(stream)), "ddg_sipg_grad_kappa")
        return g

    # -- block Jacobi ----------------------------------------------------------
    def pc_build(self, alpha: float = 0.0, stream=None):
        _lib.check(_lib.lib().ddg_sipg_pc_build(self._h, float(alpha), _lib.stream_handle(stream)),
                   "ddg_sipg_pc_build")
        self.pc_alpha = float(alpha)

    def pc_apply(self, r, out=None, stream=None):
        import torch
        r = self._vec(r, r.dtype if isinstance(r, torch.Tensor) else torch.float64)
        z = torch.empty_like(r) if out is None else out
        _lib.check(_lib.lib().ddg_sipg_pc_apply(self._h, self._prec(r.dtype), r.data_ptr(), z.data_ptr(),
                                                _lib.stream_handle(stream)), "ddg_sipg_pc_apply")
        return z

    def pc_blocks(self):
        import torch
        b = torch.empty((self.K, self.Np, self.Np), dtype=torch.float64, device=self._dev())
        _lib.check(_lib.lib().ddg_sipg_pc_blocks(self._h, b.data_ptr(), _lib.stream_handle(None)),
                   "ddg_sipg_pc_blocks")
        return b

    # -- Krylov ----------------------------------------------------------------
    def cg(self, b, x, *, tol=1e-9, atol=0.0, maxiter=1000, pc=False, alpha=0.0, shift=0.0,
           precision="fp64", stream=None):
        """Device CG (graph loop); ``x`` holds x0 and is overwritten in place.
        Returns (status, iterations, r.r, b.b)."""
        info = _lib.SolveInfo()
        cfg = _lib.CgConfig(tol=float(tol), atol=float(atol), maxiter=int(maxiter),
                            pc=_lib.DDG_PC_JACOBI if pc else _lib.DDG_PC_NONE,
                            alpha=float(alpha), shift=float(shift),
                            precision=_lib.DDG_FP64 if precision == "fp64" else _lib.DDG_FP32, reserved=0)
        _lib.check(_lib.lib().ddg_sipg_cg(self._h, C.byref(cfg), b.data_ptr(), x.data_ptr(),
                                          _lib.stream_handle(stream), C.byref(info)), "ddg_sipg_cg")
        return _lib.SOLVE_STATUS.get(info.status, str(info.status)), info.iterations, info.res_norm2, info.b_norm2


    def cg_mixed(self, b, x, *, tol=1e-9, atol=0.0, maxiter=1000, pc=False, alpha=0.0, shift=0.0,
                 delta=0.1, stream=None):
        """Mixed-precision CG with float64 reliable updates (float64 b, x;
        x holds x0 and is overwritten).  Returns (status, float32 iterations,
        float64 r.r, b.b, reliable updates)."""
        info = _lib.SolveInfo()
        cfg = _lib.CgConfig(tol=float(tol), atol=float(atol), maxiter=int(maxiter),
                            pc=_lib.DDG_PC_JACOBI if pc else _lib.DDG_PC_NONE,
                            alpha=float(alpha), shift=float(shift), precision=_lib.DDG_FP32, reserved=0)
        _lib.check(_lib.lib().ddg_sipg_cg_mixed(self._h, C.byref(cfg), float(delta), b.data_ptr(), x.data_ptr(),
                                                _lib.stream_handle(stream), C.byref(info)), "ddg_sipg_cg_mixed")
        return (_lib.SOLVE_STATUS.get(info.status, str(info.status)), info.iterations, info.res_norm2,
                info.b_norm2, info.updates)


    def cg_mg(self, mg, b, x, *, tol=1e-9, atol=0.0, maxiter=1000, alpha=0.0, shift=0.0, stream=None):
        """float64 CG preconditioned by the device V-cycle ``mg`` (float64 b,
        x; x holds x0, overwritten).  Returns (status, iterations, r.r, b.b)."""
        info = _lib.SolveInfo()
        cfg = _lib.CgConfig(tol=float(tol), atol=float(atol), maxiter=int(maxiter), pc=0,
                            alpha=float(alpha), shift=float(shift), precision=_lib.DDG_FP64, reserved=0)
        _lib.check(_lib.lib().ddg_sipg_cg_mg(self._h, C.byref(cfg), mg._h, b.data_ptr(), x.data_ptr(),
                                             _lib.stream_handle(stream), C.byref(info)), "ddg_sipg_cg_mg")
        return _lib.SOLVE_STATUS.get(info.status, str(info.status)), info.iterations, info.res_norm2, info.b_norm2


def dot(x, y, stream=None) -> float:
    """x . y with float64 accumulation (device kernel), returned to the host."""
    import torch
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    prec = _lib.DDG_FP64 if x.dtype == torch.float64 else _lib.DDG_FP32
    _lib.check(_lib.lib().ddg_dot(x.numel(), prec, x.data_ptr(), y.data_ptr(), out.data_ptr(),
                                  _lib.stream_handle(stream)), "ddg_dot")
    return float(out.item())


def axpby(a: float, x, b: float, y, stream=None):
    """y <- a x + b y (float64, device kernel)."""
    _lib.check(_lib.lib().ddg_axpby(x.numel(), float(a), x.data_ptr(), float(b), y.data_ptr(),
                                    _lib.stream_handle(stream)), "ddg_axpby")
    return y


def cast(x, dtype, stream=None):
    import torch
    out = torch.empty(x.shape, dtype=dtype, device=x.device)
    to = _lib.DDG_FP32 if dtype == torch.float32 else _lib.DDG_FP64
    _lib.check(_lib.lib().ddg_cast(x.numel(), to, x.data_ptr(), out.data_ptr(), _lib.stream_handle(stream)),
               "ddg_cast")
    return out
