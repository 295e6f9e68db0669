"""Benchmark of the B200 SIPG solve path.

Workload (the metric's configuration): SIPG Helmholtz (alpha = k^2 = 5) on a
256 x 256 quad grid of [0,1]^2 split into 131072 triangles, N = 4 (Np = 15,
1,966,080 DOFs), Dirichlet on x = 0, 1 and Neumann on y = 0, 1, penalty
tau = (N+1)^2 / h (tau_scale = 0.5), RHS = sum of 8 seeded Fourier modes
(integer wavenumbers 1..6, N(0,1) amplitudes, seed 0).

One step = one float64 operator apply (y = (alpha M + A) u) over the whole
mesh, inputs resident in HBM; L2 is flushed (256 MB write) between timed
steps and only the apply itself is timed (CUDA events on the launching
stream).  value = DOFs / apply time (GDOF/s).  The JSON line also reports
the float32 apply, the mixed-precision vs float64 block-Jacobi PCG solves
(solves/s, latency, relative error), the roofline of the dominant kernel,
the end-to-end rate through the public API with host buffers, and the CPU
baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SIPG matvec GDOF/s; solves/s + p99 latency at 1e-8 err, mixed vs FP64 on GPU"
KX = KY = 256
NDEG = 4
ALPHA = 5.0
TAU_SCALE = 0.5


def workload_arrays(build_mesh, uniform_mesh, kx=KX, ky=KY):
    VX, VY, E = uniform_mesh(0.0, 1.0, 0.0, 1.0, kx, ky)
    m = build_mesh(VX, VY, E, NDEG)
    isb = m.EToE == np.arange(m.K)[:, None]
    nxf = m.nx.reshape((m.Nfp, 3, m.K), order="F")[0].T
    bc = np.where(isb, np.where(np.abs(nxf) > 0.5, 1, 2), 0).astype(np.int32)
    rng = np.random.default_rng(0)
    wx = rng.integers(1, 7, size=8)
    wy = rng.integers(1, 7, size=8)
    amp = rng.standard_normal(8)
    f = sum(a * np.sin(np.pi * i * m.x) * np.cos(np.pi * j * m.y) for a, i, j in zip(amp, wx, wy))
    return m, bc, f


def algorithmic_bytes(K, Np, sv, sg):
    """B_apply = K [2 Np s_v + 14 s_g + 12]: u read, y written, 14 geometry
    scalars per element, 3 packed int32 neighbour words."""
    return K * (2 * Np * sv + 14 * sg + 12)


# side of the reduced precision workload whose solves are graded against the
# oracle's float64 solution (the full size takes minutes on the host cores)
SMALL = 64
SMALL_SOLVES: dict = {}
CURVED_SAMPLE: dict = {}

# DRAM bytes of one float64 tensor-core apply launch on this workload, from
# an ncu capture (56.16 MB read + 1.23 MB written; y stays in L2)
DM_TRAFFIC_BYTES = 57_386_752


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, dev):
        self.dev, self.samples, self.proc = dev, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 9
                          for i in range(4) if s[5 + i].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------------- our arm

def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    m, bc, f = workload_arrays(pm.build_mesh_2d, pm.uniform_rectangle_mesh_2d)
    op = m.device_operator(bc, TAU_SCALE)
    n = op.n
    g = torch.Generator(device=dev).manual_seed(1 + rank)
    u64 = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    y64 = torch.empty_like(u64)
    u32 = u64.float()
    y32 = torch.empty_like(u32)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2
    stream = torch.cuda.current_stream()

    def timed_applies(u, y, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            op.apply(u, alpha=ALPHA, out=y)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) * 1e-3 for a, b in ev]

    for _ in range(args.warmup):
        op.apply(u64, alpha=ALPHA, out=y64)
        op.apply(u32, alpha=ALPHA, out=y32)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        t64 = timed_applies(u64, y64, args.steps)
        t32 = timed_applies(u32, y32, args.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    tot64 = sum(t64)
    if world > 1:
        tt = torch.tensor([tot64], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot64 = float(tt.item())
    ms_step = tot64 / args.steps * 1e3
    value = world * n * args.steps / tot64 / 1e9
    a64 = float(np.mean(t64))
    a32 = float(np.mean(t32))
    hbm, peak_kind = peaks()
    B64 = algorithmic_bytes(m.K, m.Np, 8, 8)
    B32 = algorithmic_bytes(m.K, m.Np, 4, 4)

    # ---- end to end through the public API with host buffers: the (Np, K)
    # float64 field in pinned host memory -> SipgOperator.apply_host (copy in,
    # apply, copy out, overlapped chunk by chunk) -> (Np, K) result in pinned
    # host memory; every byte of u and y crosses PCIe inside the timed region
    import ddg_b200
    u_host = ddg_b200.pinned_empty((m.Np, m.K))
    u_host[...] = np.random.default_rng(2).standard_normal((m.Np, m.K))
    y_host = ddg_b200.pinned_empty((m.Np, m.K))
    e2e_steps = max(5, args.steps)
    for _ in range(3):
        op.apply_host(u_host, alpha=ALPHA, out=y_host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        op.apply_host(u_host, alpha=ALPHA, out=y_host)
    te2e = (time.perf_counter() - t0) / e2e_steps
    # the same through the reference-named function with pageable numpy arrays
    u_np = np.array(u_host)
    for _ in range(2):
        ps.sipg_apply_2d(m, u_np, bc_types=bc, tau_scale=TAU_SCALE)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ps.sipg_apply_2d(m, u_np, bc_types=bc, tau_scale=TAU_SCALE)
    tpage = (time.perf_counter() - t0) / e2e_steps
    e2e = {"value": world * n / te2e / 1e9, "unit": "GDOF/s", "h2d_bytes_per_step": int(u_host.nbytes),
           "d2h_bytes_per_step": int(y_host.nbytes), "ms_per_step": te2e * 1e3,
           "note": "SipgOperator.apply_host(pinned (Np,K) float64 u -> pinned y), alpha=5, host wall clock "
                   "per synchronous call; copies overlap the per-chunk applies",
           "pageable_sipg_apply_2d": {"value": world * n / tpage / 1e9, "ms_per_step": tpage * 1e3,
                                      "note": "sipg_apply_2d(mesh, numpy u) with pageable arrays, alpha=0"}}

    # ---- solves: float64 PCG vs mixed-precision refinement (rel err 1e-8 target)
    solves = None
    if not args.skip_solves:
        pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=ALPHA, nu=1.0, bc_types=bc,
                                                           tau_scale=TAU_SCALE)
        ref_u = ps.solve_sipg_helmholtz_2d(m, f, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE,
                                           preconditioner=pc,
                                           iterative=ps.IterativeConfig(tol=1e-13, maxiter=20000))
        out = {}
        for name, cfg in (("fp64", ps.IterativeConfig(tol=args.solve_tol, maxiter=20000)),
                          ("mixed", ps.IterativeConfig(tol=args.solve_tol, maxiter=20000, precision="mixed",
                                                       inner_tol=args.inner_tol))):
            lat, info, u = [], None, None
            for _ in range(args.solve_reps + 1):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                u, info = ps.solve_sipg_helmholtz_2d(m, f, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE,
                                                     preconditioner=pc, iterative=cfg, return_info=True)
                lat.append(time.perf_counter() - t0)
            lat = lat[1:]
            out[name] = {"solves_per_s": 1.0 / float(np.mean(lat)), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                         "p99_ms": float(np.percentile(lat, 99) * 1e3), "iterations": info.iterations,
                         "refinements": info.refinements, "status": info.status,
                         "rel_err_vs_fp64_tol1e-13": float(np.linalg.norm(u - ref_u) / np.linalg.norm(ref_u))}
        out["speedup_mixed_vs_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
        # the same two solves on the 64 x 64 version of the workload, graded in
        # the CPU leg against the oracle's float64 block-Jacobi PCG solution
        ms, bcs, fs = workload_arrays(pm.build_mesh_2d, pm.uniform_rectangle_mesh_2d, SMALL, SMALL)
        pcs = ps.make_helmholtz_block_jacobi_preconditioner(ms, alpha=ALPHA, nu=1.0, bc_types=bcs,
                                                            tau_scale=TAU_SCALE)
        SMALL_SOLVES.clear()
        for name, prec in (("fp64", "fp64"), ("mixed", "mixed")):
            cfg = ps.IterativeConfig(tol=args.solve_tol, maxiter=20000, precision=prec, inner_tol=args.inner_tol)
            SMALL_SOLVES[name] = ps.solve_sipg_helmholtz_2d(ms, fs, alpha=ALPHA, nu=1.0, bc_types=bcs,
                                                            tau_scale=TAU_SCALE, preconditioner=pcs, iterative=cfg)
        out["note"] = ("block-Jacobi PCG, tol %.0e; latency = host wall clock of the public API call "
                       "(numpy in/out); reference solution = float64 device PCG at tol 1e-13" % args.solve_tol)
        solves = out

    line = {
        "metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "precision: Helmholtz k^2=5, 256x256 quads -> 131072 triangles, N=4, "
                               "1,966,080 DOFs, Dirichlet x / Neumann y, tau_scale=0.5",
                   "step": "one float64 operator apply (alpha M + A) u",
                   "l2": "flushed (256 MB write) between timed steps", "parallelism": "replicas"},
        "apply_fp32": {"gdofs": n / a32 / 1e9, "us": a32 * 1e6},
        "roofline": {"bound": "hbm", "achieved": B64 / a64 / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": B64 / a64 / 1e9 / hbm, "traffic": DM_TRAFFIC_BYTES, "peak_kind": peak_kind,
                     "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum per launch, one ncu capture of "
                                     "this kernel on this workload (profiles/); reads the per-element coefficient "
                                     "table (296 B per element) instead of the 112 B of geometry",
                     "kernel": "k_apply_dm<4,APPLY> (FP64 tensor cores, mma.sync m16n8k8 f64)",
                     "algorithmic_bytes": B64},
        "roofline_fp32": {"bound": "hbm", "achieved": B32 / a32 / 1e9, "peak": hbm, "unit": "GB/s",
                          "frac": B32 / a32 / 1e9 / hbm,
                          "kernel": "k_apply_tc<4,APPLY> (tcgen05 kind::tf32, 3xTF32 split)",
                          "algorithmic_bytes": B32},
        "e2e": e2e,
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
        "solves": solves,
    }
    if not args.skip_workloads:
        line["curved"] = curved_leg(args.steps, hbm)
        line["plain"] = plain_leg()
        line["hpmg_pressure_poisson"] = hpmg_leg()
        line["serving"] = serving_leg(args.serving_requests)
        line["adjoint"] = adjoint_leg()
    if rank == 0 and not args.skip_cpu:
        line["cpu_baseline"] = cpu_baseline(budget_s=args.cpu_seconds)
    return line


def hpmg_leg():
    """Pressure-Poisson workload: pure Neumann on [0,1] x [0,2], 128 x 256
    quads -> 65,536 triangles, N = 3 (655,360 DOFs), seeded smooth mean-free
    source; hp-multigrid (p 3 -> 2 -> 1, then 3 h-levels down to 16 x 32 quads)
    preconditioned CG to 1e-8 with float64 vs float32 smoothing/transfers."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import multigrid as pmg
    from ddg_b200.dg2d import sipg as ps
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 16, 32)
    base = pm.build_mesh_2d(VX, VY, E, 3)

    def nbc(m):
        return np.where(m.EToE == np.arange(m.K)[:, None], ps.BC_NEUMANN, 0).astype(np.int32)
    out, sol = {}, {}
    for prec in ("fp64", "fp32"):
        t0 = time.perf_counter()
        mg, fin = pmg.make_sipg_hpmg_preconditioner(base, 3, bc_fn=nbc, regularize=True, tau_scale=TAU_SCALE,
                                                    precision=prec)
        setup = time.perf_counter() - t0
        rng = np.random.default_rng(0)
        kx, ky, a = rng.integers(1, 5, 6), rng.integers(1, 5, 6), rng.standard_normal(6)
        src = sum(ai * np.cos(np.pi * i * fin.x) * np.cos(np.pi * j * fin.y / 2) for ai, i, j in zip(a, kx, ky))
        src = src - src.mean()
        lat = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            u, info = ps.solve_sipg_poisson_2d(fin, src, bc_types=nbc(fin), tau_scale=TAU_SCALE, preconditioner=mg,
                                               iterative=ps.IterativeConfig(tol=1e-8, maxiter=2000),
                                               return_info=True)
            torch.cuda.synchronize()
            lat.append(time.perf_counter() - t0)
        sol[prec] = u
        out["vcycle_" + prec] = {"iterations": info.iterations, "status": info.status,
                                 "solve_ms": 1e3 * float(np.median(lat)), "setup_s": setup}
        if prec == "fp64":
            # the exact mean-free solution (no shift; RHS projected onto
            # range(A)) against which the reference's epsilon-shift mode is graded
            up, infop = ps.solve_sipg_poisson_2d(fin, src, bc_types=nbc(fin), tau_scale=TAU_SCALE,
                                                 preconditioner=mg, return_info=True,
                                                 iterative=ps.IterativeConfig(tol=1e-10, maxiter=2000,
                                                                              nullspace="project"))
            sol["projected"] = up
            out["projected_fp64"] = {"iterations": infop.iterations, "status": infop.status, "tol": 1e-10}
        mg.close()
    # the plain float64 path on the same system: block-Jacobi PCG
    pcb = ps.make_sipg_block_jacobi_preconditioner(fin, bc_types=nbc(fin), tau_scale=TAU_SCALE)
    lat = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ub, info = ps.solve_sipg_poisson_2d(fin, src, bc_types=nbc(fin), tau_scale=TAU_SCALE, preconditioner=pcb,
                                            iterative=ps.IterativeConfig(tol=1e-8, maxiter=50000), return_info=True)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t0)
    out["block_jacobi_fp64"] = {"iterations": info.iterations, "status": info.status,
                                "solve_ms": 1e3 * float(np.min(lat)),
                                "rel_diff_vs_vcycle_fp64": float(np.linalg.norm(ub - sol["fp64"]) /
                                                                 np.linalg.norm(sol["fp64"]))}
    up = sol["projected"]
    out["rel_diff_shift_vs_projected"] = {
        name: float(np.linalg.norm(sol[name] - up) / np.linalg.norm(up)) for name in ("fp64", "fp32")}
    out["rel_diff_shift_vs_projected"]["block_jacobi_fp64"] = float(np.linalg.norm(ub - up) / np.linalg.norm(up))
    out["dofs"] = int(fin.K * fin.Np)
    out["rel_diff_fp32_vs_fp64"] = float(np.linalg.norm(sol["fp32"] - sol["fp64"]) / np.linalg.norm(sol["fp64"]))
    out["note"] = "latency = host wall clock of solve_sipg_poisson_2d (numpy in/out); set-up (host meshes) apart"
    return out


def plain_leg():
    """Plain workload exactly as specified: 12 x 12 quads -> 288 triangles,
    N = 4 (4,320 DOFs), Dirichlet from u = sin(pi x) sin(pi y), f = 2 pi^2 u,
    tau_scale = 0.5, unpreconditioned CG to tol 1e-9, through
    solve_sipg_poisson_2d.  Matvec, iteration count and L2 error are compared
    with the numbers the reference's own code produced for this workload
    (tests/golden, generated from the unmodified reference)."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    gold = os.path.join(ROOT, "tests", "golden")
    ga, gs = np.load(os.path.join(gold, "applies.npz")), np.load(os.path.join(gold, "solves.npz"))
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 12, 12)
    m = pm.build_mesh_2d(VX, VY, E, 4)
    bc = np.where(m.EToE == np.arange(m.K)[:, None], ps.BC_DIRICHLET, 0).astype(np.int32)
    case = "plain12_N4/dirichlet/tau0.5"
    Au = ps.sipg_apply_2d(m, ga[case + "/u"], bc_types=ga[case + "/bc"], tau_scale=0.5)
    mv = float(np.max(np.abs(Au - ga[case + "/Au"])) / np.max(np.abs(ga[case + "/Au"])))
    ue = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    cfg = ps.IterativeConfig(tol=1e-9)
    lat = []
    for _ in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u, info = ps.solve_sipg_poisson_2d(m, 2 * np.pi ** 2 * ue, bc_types=bc, u_dir=ue, tau_scale=0.5,
                                           iterative=cfg, return_info=True)
        lat.append(time.perf_counter() - t0)

    def l2(d):
        return float(np.sqrt(np.sum(m.J * d * (m.ref.M @ d))))
    return {"workload": "12x12 quads -> 288 triangles, N=4, 4320 DOFs, Dirichlet sin(pi x) sin(pi y), "
                        "tau_scale=0.5, CG tol 1e-9, no preconditioner",
            "matvec_rel_err_vs_reference": mv, "cg_iterations": info.iterations,
            "reference_cg_iterations": int(gs["plain/cg_iterations"]), "status": info.status,
            "l2_err_vs_exact": l2(u - ue), "reference_l2_err_vs_exact": l2(gs["plain/u_cg"] - ue),
            "rel_err_vs_reference_solution": float(np.linalg.norm(u - gs["plain/u_cg"]) /
                                                   np.linalg.norm(gs["plain/u_cg"])),
            "solve_ms": 1e3 * float(np.median(lat[1:]))}


def curved_workload(build_mesh, channel, bend, attach):
    """Cylinder in a channel: [0,32]^2 split into 256 x 256 cells minus the
    grid-aligned box of half-side 2 around (16, 16), plus an O-grid of 8
    layers (growth 1.2) down to a cylinder of radius 1 whose faces are bent
    onto the circle -> 131,072 triangles, N = 4 (1,966,080 DOFs, the size of
    the precision workload), all boundaries Dirichlet, with its cubature."""
    VX, VY, E = channel(0.0, 32.0, 0.0, 32.0, 256, 256, cx=16.0, cy=16.0, radius=1.0, R_outer=2.0,
                        n_radial=8, radial_growth=1.2)
    m = bend(build_mesh(VX, VY, E, NDEG), cx=16.0, cy=16.0, radius=1.0)
    bc = np.where(np.asarray(m.EToE) == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    return m, bc, attach(m)


def curved_bytes(N, Ncub, quad):
    """Algorithmic bytes per element of one curved-element apply: every array
    each of the three passes reads or writes, counted once per pass (float64
    values, int32 tags and slot maps)."""
    Np, Nfp = (N + 1) * (N + 2) // 2, N + 1
    Ns, nq = 3 * Nfp, Nfp * (Nfp + 1) // 2
    p1 = 8 * (Np + 4 * 3 * N + 2 * Ns)
    p2 = 4 * 3 + 8 * 2 * Ns + 8 * 3 * N + 4 * 2 * Ns + 8 * 2 * Ns + 8 * 3 * Ns
    p2 += 8 * 3 * (1 + nq) if quad == "cubature" else 8 * 2 * 3
    p3 = 8 * Np + 4 * 3 + 4 * Ns + 8 * 3 * Ns + 8 * 4 * Np + 8 * Np
    p3 += 8 * 4 * Ncub if quad == "cubature" else 8 * Np
    return p1 + p2 + p3


def curved_leg(steps, hbm):
    """The curved-element branch (cub=...) on the cylinder workload: the
    nodal and cubature applies (device-timed, L2 flushed), the cubature
    Helmholtz solve with block-Jacobi PCG, and the matvec against the
    reference's own cubature apply (tests/golden/curved.npz)."""
    import torch
    from ddg_b200.dg2d import cubature as pcub
    from ddg_b200.dg2d import curved as pcur
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    m, bc, cub = curved_workload(pm.build_mesh_2d, pm.channel_with_circle_mesh_2d, pcur.apply_circular_hole_2d,
                                 pcub.attach_cubature)
    op = m.curved_operator(bc, TAU_SCALE, cub)
    n = op.n
    u = torch.randn(n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    y = torch.empty_like(u)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {"workload": f"cylinder in a channel (O-grid, faces bent onto the circle): {m.K} triangles, N={NDEG}, "
                       f"{n} DOFs, {cub.w.shape[0]}-point volume cubature, Dirichlet, alpha={ALPHA:g}, "
                       f"tau_scale={TAU_SCALE}"}
    for quad in ("nodal", "cubature"):
        for _ in range(3):
            op.apply(u, alpha=ALPHA, out=y, quad=quad)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record()
            op.apply(u, alpha=ALPHA, out=y, quad=quad)
            ev[i][1].record()
        torch.cuda.synchronize()
        t = float(np.mean([a.elapsed_time(b) * 1e-3 for a, b in ev]))
        B = curved_bytes(NDEG, int(cub.w.shape[0]), quad) * m.K
        out[quad] = {"gdofs": n / t / 1e9, "us": t * 1e6, "launches": 3,
                     "roofline": {"bound": "hbm", "achieved": B / t / 1e9, "peak": hbm, "unit": "GB/s",
                                  "frac": B / t / 1e9 / hbm, "algorithmic_bytes": B,
                                  "kernels": "k_cv_trace, k_cv_dual, k_cv_gather (one apply)"}}
    # end to end through the reference-named function with (Np, K) host
    # arrays: sipg_apply_2d(mesh, u, cub=cub), both PCIe directions inside
    u_np = np.random.default_rng(5).standard_normal((m.Np, m.K))
    for _ in range(2):
        ps.sipg_apply_2d(m, u_np, bc_types=bc, tau_scale=TAU_SCALE, cub=cub)
    reps = max(5, steps)
    t0 = time.perf_counter()
    for _ in range(reps):
        ps.sipg_apply_2d(m, u_np, bc_types=bc, tau_scale=TAU_SCALE, cub=cub)
    te = (time.perf_counter() - t0) / reps
    out["e2e"] = {"value": n / te / 1e9, "unit": "GDOF/s", "h2d_bytes_per_step": int(u_np.nbytes),
                  "d2h_bytes_per_step": int(u_np.nbytes), "ms_per_step": te * 1e3,
                  "note": "sipg_apply_2d(mesh, numpy u, cub=cub): pageable host arrays in and out, host wall clock"}
    f = np.cos(0.3 * m.x) * np.sin(0.2 * m.y) + 0.1
    pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE,
                                                       cub=cub)
    cfg = ps.IterativeConfig(tol=1e-8, maxiter=20000)
    lat = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, info = ps.solve_sipg_helmholtz_2d(m, f, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE, cub=cub,
                                             preconditioner=pc, iterative=cfg, return_info=True)
        lat.append(time.perf_counter() - t0)
    out["solve"] = {"iterations": info.iterations, "status": info.status, "tol": 1e-8,
                    "solves_per_s": 1.0 / float(np.median(lat[1:])), "ms_per_iteration":
                    1e3 * float(np.median(lat[1:])) / max(info.iterations, 1),
                    "note": "solve_sipg_helmholtz_2d(cub=...) with the cubature block-Jacobi; host wall clock"}
    gold = np.load(os.path.join(ROOT, "tests", "golden", "curved.npz"))
    gm = pm.build_mesh_2d(gold["annulus8_N3/VX"], gold["annulus8_N3/VY"], gold["annulus8_N3/EToV"], 3)
    gm = pcur.apply_circular_hole_2d(gm, cx=0.0, cy=0.0, radius=0.5, detection_tol=0.5)
    k = "annulus8_N3/apply/random/tau0.5"
    Au = ps.sipg_apply_2d(gm, gold[k + "/u"], bc_types=gold[k + "/bc"], tau_scale=0.5, cub=pcub.attach_cubature(gm))
    out["matvec_rel_err_vs_reference"] = float(np.max(np.abs(Au - gold[k + "/Au_cub"])) /
                                               np.max(np.abs(gold[k + "/Au_cub"])))
    CURVED_SAMPLE["gdofs_cubature"] = out["cubature"]["gdofs"]
    return out


def serving_leg(count=4096, loads=(0.5, 0.8)):
    """Serving workload: the seeded stream of `count` requests (n ~ U{8..96}
    quads per side, N ~ U{2,3,4}, k^2 ~ U[0,10], Dirichlet, 8-mode source,
    tol 1e-6 -- run in the float32 pools -- or 1e-9), admitted against a
    120 GB HBM budget with the tile autotuner on: first all at once
    (saturation throughput; the autotuner settles its tiles here), then with
    Poisson arrivals at each fraction of that throughput in `loads`
    (latency); one-at-a-time float64 solves of the first 24 requests as the
    baseline."""
    from ddg_b200 import serving
    eng = serving.ServingEngine(degrees=(2, 3, 4), hbm_budget_bytes=120e9, capacity=4_000_000, max_requests=1024,
                                pairs=4)
    done = eng.run(serving.make_requests(count=count, seed=0), realtime=False)
    burst = serving.summarize(done, eng.elapsed)
    out = {"requests": count, "saturation": burst, "load_sweep": []}
    for frac in loads:
        rate = frac * burst["solves_per_s"]
        done = eng.run(serving.make_requests(count=count, seed=1, rate=rate), realtime=True)
        out["load_sweep"].append({"load_fraction": frac, "arrival_rate_per_s": rate,
                                  **serving.summarize(done, eng.elapsed)})
    out["autotuner_tiles"] = eng.tuner.table()
    eng.close()
    _, tb = serving.solve_one_at_a_time(serving.make_requests(count=24, seed=0))
    out["one_at_a_time_fp64_solves_per_s"] = 24.0 / tb
    out["note"] = ("the full 4096-request stream; tol 1e-6 requests iterate in float32 pools, 1e-9 in float64; "
                   "120 GB admission budget; latency = arrival to retirement on the host clock")
    return out


def adjoint_leg(batch=64, fd_dirs=32):
    """Differentiation workload: 64 x 64 quads -> 8192 triangles, N = 4,
    kappa = exp(g), g ~ N(0, 0.5^2) per element; gradient of
    1/2 ||u - u_obs||_M^2 for a batch of `batch` kappas via the adjoint
    (forward + adjoint block-Jacobi PCG + contraction kernel), checked against
    centred differences (h = 1e-6) on `fd_dirs` random directions."""
    import torch
    from ddg_b200 import adjoint
    from ddg_b200.dg2d import mesh as pm
    VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 64, 64)
    m = pm.build_mesh_2d(VX, VY, E, 4)
    bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    op = m.device_operator(bc, TAU_SCALE)
    f = torch.as_tensor((np.sin(np.pi * m.x) * np.sin(np.pi * m.y) + 0.5).T.reshape(-1).copy(), device="cuda")
    g_obs = torch.as_tensor(0.5 * np.random.default_rng(1).standard_normal(m.K), device="cuda")
    adjoint._state(op).use(op, torch.exp(g_obs).cpu().numpy())
    uo, _ = adjoint._cg(op, adjoint.mass_apply(op, f), 1e-12, 40000)
    G = torch.as_tensor(0.5 * np.random.default_rng(2).standard_normal((batch, m.K)), device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L, grads, its = adjoint.loss_and_grad(op, G, f, uo, tol=1e-12, maxiter=40000)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(fd_dirs):
        d = torch.as_tensor(rng.standard_normal(m.K), device="cuda")
        lp = adjoint.loss_only(op, G[0] + 1e-6 * d, f, uo)
        lm = adjoint.loss_only(op, G[0] - 1e-6 * d, f, uo)
        fd = (float(lp) - float(lm)) / 2e-6
        ad = float((grads[0] * d).sum())
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-300))
    return {"batch": batch, "gradients_per_s": batch / dt, "cg_iterations": int(its),
            "fd_max_rel_err": worst, "fd_directions": fd_dirs,
            "note": "the 64-kappa batch; centred FD (h = 1e-6, float64) on the first kappa's gradient; "
                    "the reference has no per-element diffusivity (and JAX is absent), so there is no "
                    "reference jax.grad to compare with"}


def profile_apply(args):
    """Stand-alone applies of the workload (no L2 flush), for a profiler's
    capture of one kernel: `--profile-apply fp64` runs the float64 apply,
    `fp32` the float32 one, each `--profile-reps` times."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    m, bc, _ = workload_arrays(pm.build_mesh_2d, pm.uniform_rectangle_mesh_2d)
    op = m.device_operator(bc, TAU_SCALE)
    dt = torch.float64 if args.profile_apply == "fp64" else torch.float32
    u = torch.randn(op.n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1)).to(dt)
    y = torch.empty_like(u)
    for _ in range(args.profile_reps):
        op.apply(u, alpha=ALPHA, out=y)
    torch.cuda.synchronize()
    print(f"{args.profile_reps} {args.profile_apply} applies done", flush=True)


def profile_kernels(args):
    """Short runs of the other kernels for a profiler's per-kernel captures:
    `cg-fp64` / `cg-fp32`: block-Jacobi PCG on the workload with the
    iteration kernels launched eagerly (DDG_CG_EAGER=1, which the caller
    sets; conditional graphs hide their kernels from profilers), including
    the block-Jacobi set-up; `mg`: V-cycle applies of the pressure-Poisson
    workload's hp-multigrid; `serving`: a 64-request stream through the
    pools; `adjoint`: one gradient of the differentiation workload;
    `curved`: nodal then cubature applies of the curved-element workload."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    what = args.profile_kernels
    if what.startswith("cg-"):
        m, bc, f = workload_arrays(pm.build_mesh_2d, pm.uniform_rectangle_mesh_2d)
        op = m.device_operator(bc, TAU_SCALE)
        op.pc_build(ALPHA)
        dt = torch.float64 if what == "cg-fp64" else torch.float32
        b = torch.as_tensor(f.T.reshape(-1).copy(), device="cuda").to(dt)
        x = torch.zeros_like(b)
        st = op.cg(b, x, tol=1e-12, maxiter=args.profile_maxiter, pc=True, alpha=ALPHA,
                   precision="fp64" if what == "cg-fp64" else "fp32")
        print(what, st, flush=True)
    elif what == "mg":
        from ddg_b200.dg2d import multigrid as pmg
        VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 2.0, 16, 32)
        base = pm.build_mesh_2d(VX, VY, E, 3)

        def nbc(mm):
            return np.where(mm.EToE == np.arange(mm.K)[:, None], ps.BC_NEUMANN, 0).astype(np.int32)
        mg, fin = pmg.make_sipg_hpmg_preconditioner(base, 3, bc_fn=nbc, regularize=True, tau_scale=TAU_SCALE)
        v = torch.randn(fin.K * fin.Np, dtype=torch.float64, device="cuda")
        mg.apply_device(v)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()    # the V-cycles only (not the set-up's probing)
        for _ in range(args.profile_reps):
            mg.apply_device(v)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        print("mg done", flush=True)
    elif what == "serving":
        from ddg_b200 import serving
        eng = serving.ServingEngine(degrees=(2, 3, 4), capacity=1_000_000, max_requests=128, pairs=4)
        done = eng.run(serving.make_requests(count=64, seed=0), realtime=False)
        eng.close()
        print("serving", len(done), flush=True)
    elif what == "curved":
        from ddg_b200.dg2d import cubature as pcub
        from ddg_b200.dg2d import curved as pcur
        m, bc, cub = curved_workload(pm.build_mesh_2d, pm.channel_with_circle_mesh_2d, pcur.apply_circular_hole_2d,
                                     pcub.attach_cubature)
        op = m.curved_operator(bc, TAU_SCALE, cub)
        u = torch.randn(op.n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
        for quad in ("nodal", "cubature"):
            for _ in range(args.profile_reps):
                op.apply(u, alpha=ALPHA, quad=quad)
        torch.cuda.synchronize()
        print("curved applies done", flush=True)
    elif what == "adjoint":
        from ddg_b200 import adjoint
        VX, VY, E = pm.uniform_rectangle_mesh_2d(0.0, 1.0, 0.0, 1.0, 64, 64)
        m = pm.build_mesh_2d(VX, VY, E, 4)
        bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
        op = m.device_operator(bc, TAU_SCALE)
        f = torch.as_tensor((np.sin(np.pi * m.x) * np.sin(np.pi * m.y)).T.reshape(-1).copy(), device="cuda")
        G = torch.as_tensor(0.5 * np.random.default_rng(2).standard_normal((1, m.K)), device="cuda")
        L, grads, its = adjoint.loss_and_grad(op, G, f, torch.zeros_like(f), tol=1e-8, maxiter=4000)
        print("adjoint", its, flush=True)


def profile_solves(args):
    """One float64 and one mixed block-Jacobi PCG solve of the workload."""
    import torch
    from ddg_b200.dg2d import mesh as pm
    from ddg_b200.dg2d import sipg as ps
    m, bc, f = workload_arrays(pm.build_mesh_2d, pm.uniform_rectangle_mesh_2d)
    pc = ps.make_helmholtz_block_jacobi_preconditioner(m, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE)
    for prec in ("fp64", "mixed"):
        cfg = ps.IterativeConfig(tol=args.solve_tol, maxiter=args.profile_maxiter, precision=prec,
                                 inner_tol=args.inner_tol)
        t0 = time.perf_counter()
        _, info = ps.solve_sipg_helmholtz_2d(m, f, alpha=ALPHA, nu=1.0, bc_types=bc, tau_scale=TAU_SCALE,
                                             preconditioner=pc, iterative=cfg, return_info=True)
        torch.cuda.synchronize()
        print(prec, info, f"{time.perf_counter() - t0:.3f} s", flush=True)


# ------------------------------------------------------------ CPU legs

def cpu_baseline(budget_s=15.0):
    """The oracle's float64 apply on the host cores, bounded sample; then the
    oracle's float64 block-Jacobi PCG solve (C + OpenMP apply, numpy block
    inverses, the reference's CG stopping rule) of the 64 x 64 version of the
    workload, timed, and the GPU solutions of the same system graded
    against it."""
    from oracle import cbuild
    from oracle import mesh as om
    from oracle import sipg as osp
    out = cbuild.time_apply(KX, KY, NDEG, TAU_SCALE, ALPHA, budget_s=budget_s)
    m, bc, f = workload_arrays(om.build_mesh_2d, om.uniform_rectangle_mesh_2d, SMALL, SMALL)
    A = cbuild.CApply(m, bc, TAU_SCALE, ALPHA)
    t0 = time.perf_counter()
    pc = osp.block_jacobi_from_blocks(osp.extract_block_diag_matfree(A, m))
    b = osp._rhs(m, f, bc, None, None, TAU_SCALE)
    x, its = osp.cg(A, b, tol=1e-10, maxiter=20000, M=pc)
    dt = time.perf_counter() - t0
    u = x.reshape(m.K, m.Np).T
    solve = {"workload": f"{SMALL}x{SMALL} quads -> {2 * SMALL * SMALL} triangles, N={NDEG}, {m.K * m.Np} DOFs, "
                         "same BCs, alpha, tau_scale and RHS as the full workload",
             "oracle_block_jacobi_pcg": {"iterations": int(its), "solve_s": dt, "tol": 1e-10,
                                         "cores": len(os.sched_getaffinity(0))}}
    for name, ug in SMALL_SOLVES.items():
        solve[f"rel_l2_err_{name}_vs_oracle"] = float(np.linalg.norm(ug - u) / np.linalg.norm(u))
    out["solve"] = solve
    if CURVED_SAMPLE:
        out["curved"] = cpu_curved(budget_s=min(budget_s, 10.0))
    return out


def cpu_curved(budget_s=10.0):
    """The oracle's float64 cubature apply (numpy, batched over elements) on
    the cylinder workload's elements, timed on a bounded sample: whole
    applies of a 64 x 64-cell version of the same mesh."""
    from oracle import cubature as ocub
    from oracle import curved as ocur
    from oracle import mesh as om
    from oracle import sipg as osp
    VX, VY, E = ocur.channel_with_circle_mesh_2d(0.0, 32.0, 0.0, 32.0, 64, 64, cx=16.0, cy=16.0, radius=1.0,
                                                 R_outer=2.0, n_radial=8, radial_growth=1.2)
    m = ocur.apply_circular_hole_2d(om.build_mesh_2d(VX, VY, E, NDEG), cx=16.0, cy=16.0, radius=1.0)
    cub = ocub.attach_cubature(m)
    bc = np.where(m.EToE == np.arange(m.K)[:, None], 1, 0).astype(np.int32)
    u = np.random.default_rng(4).standard_normal((m.Np, m.K))
    ts, t_end = [], time.perf_counter() + budget_s
    while time.perf_counter() < t_end or len(ts) < 3:
        t0 = time.perf_counter()
        osp.apply(m, u, bc_types=bc, tau_scale=TAU_SCALE, cub=cub)
        ts.append(time.perf_counter() - t0)
    t = float(np.median(ts))
    v = m.K * m.Np / t / 1e9
    return {"value": v, "unit": "GDOF/s", "kind": "port", "cores": 1,
            "sample": f"{len(ts)} cubature applies of the {m.K}-element version of the cylinder mesh by the "
                      f"oracle (numpy), median {t * 1e3:.1f} ms",
            "gpu_over_cpu": CURVED_SAMPLE["gdofs_cubature"] / v}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from oracle import cbuild
    step, ndof, nt = cbuild.apply_stepper(KX, KY, NDEG, TAU_SCALE, ALPHA)
    per = max(1, -(-50 // max(1, args.steps)))      # at least 50 timed applies in all
    for _ in range(args.warmup * per):
        step()
    ts = [step() for _ in range(args.steps * per)]
    t = float(np.median(ts))
    v = ndof / t / 1e9
    cb = {"value": v, "unit": "GDOF/s", "cores": nt, "kind": "port",
          "sample": f"{len(ts)} timed float64 applies ({per} per step, after {args.warmup * per} warm-up applies) of the "
                    f"full {2 * KX * KY}-element N={NDEG} mesh; C+OpenMP restatement of the reference operator; "
                    f"median {t * 1e3:.2f} ms",
          "median_ms": t * 1e3}
    return {"metric": METRIC, "value": v, "unit": "GDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * (KX * KY * 2 * 15) / (v * 1e9),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": "precision: Helmholtz k^2=5, 256x256 quads -> 131072 triangles, N=4, "
                                   "1,966,080 DOFs, Dirichlet x / Neumann y, tau_scale=0.5",
                       "step": "one float64 operator apply on the host cores"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solve-tol", type=float, default=1e-10)
    ap.add_argument("--inner-tol", type=float, default=0.7)
    ap.add_argument("--solve-reps", type=int, default=3)
    ap.add_argument("--skip-solves", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-workloads", action="store_true",
                    help="leave out the multigrid, serving and adjoint legs")
    ap.add_argument("--serving-requests", type=int, default=4096)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--profile-maxiter", type=int, default=20000)
    ap.add_argument("--profile-solves", action="store_true",
                    help="only the float64 and mixed solves, one each (for a profiler's launch list)")
    ap.add_argument("--profile-apply", choices=["fp64", "fp32"], default=None,
                    help="only stand-alone applies of one precision (for a profiler's capture of that kernel)")
    ap.add_argument("--profile-reps", type=int, default=5)
    ap.add_argument("--profile-kernels", choices=["cg-fp64", "cg-fp32", "mg", "serving", "adjoint", "curved"],
                    default=None,
                    help="only a short run of those kernels (for a profiler's per-kernel capture)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.profile_solves:
        profile_solves(args)
        return
    if args.profile_apply:
        profile_apply(args)
        return
    if args.profile_kernels:
        profile_kernels(args)
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
