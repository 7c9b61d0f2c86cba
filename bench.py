"""Benchmark of the C3D10 solve path on B200 -- one JSON line on stdout (rank 0).

Workload (default): the 200,340-element structured C3D10 I-beam (L = 4 m, 337,585 nodes,
1,012,755 DOFs, seeded 5 % corner jitter, root clamped, 50 kN tip shear), assembled on the
GPU, smoothed-aggregation AMG built once; one *step* is one solve K u = F to a true relative
residual of 1e-8:

* ``value``  -- DOF/s of the mixed-precision solve (FP64 PCG with an FP32 AMG V-cycle, FP64
                dots and coarsest solve, stopped on the true FP64 residual), device-resident
                F/u, CUDA events on the launching stream;
* ``fp64``   -- the same with the plain FP64 AMG-PCG, for the mixed vs FP64 ratio;
* ``e2e``    -- the same metric through the public API ``solve_c3d10_system`` with host
                (numpy) F and u, the host<->device copies inside the timed region;
* ``roofline`` -- the fine-level FP32 BSR3 SpMV (the kernel class that every fused V-cycle
                stage and the PCG SpMV are built from), algorithmic bytes per launch /
                event-timed launch duration vs the measured HBM copy bandwidth;
* ``cpu_baseline`` -- the reference's own CPU algorithm for this solve (scipy ``cg`` with the
                point-Jacobi preconditioner, solid_solver.py:197-266, restated in the oracle),
                timed on a bounded sample of iterations on this host and extrapolated to the
                iteration count that algorithm needs at this size (measured by the GPU
                Jacobi-PCG, which reproduces scipy's count).

``--impl reference`` runs only that CPU baseline, as the reference arm.  With N > 1 GPUs
(torchrun) every rank solves its own replica (the solve does not shard): weak scaling,
value = sum over ranks of DOF/s, timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "C3D10 solve time & DOF/s, mixed vs FP64 GPU at rel.res 1e-8; adjoint grad ms"
# Jacobi-PCG iterations to rel. res 1e-8 on the default I-beam, measured on a B200 by this
# script's GPU arm (``jacobi_pcg_iterations`` in its output); used by the CPU-only
# reference arm, which cannot afford to run the solve to convergence.
JACOBI_ITERS_IBEAM = 48507


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--slices", type=int, default=315, help="I-beam slices (315 -> 200,340 elements)")
    ap.add_argument("--cpu-iters", type=int, default=12, help="scipy cg iterations in the CPU sample")
    ap.add_argument("--skip-jacobi", action="store_true", help="do not measure the Jacobi iteration count")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-multi", action="store_true", help="do not time the batched load cases")
    ap.add_argument("--skip-adjoint", action="store_true", help="do not run the adjoint workload")
    ap.add_argument("--fd-elements", type=int, default=50, help="elements of the finite-difference check")
    ap.add_argument("--skip-frame", action="store_true", help="do not run the beam-frame workload")
    ap.add_argument("--frame-n", type=int, default=70, help="space frame of n x n x n nodes (70: 2,058,000 DOFs)")
    ap.add_argument("--cases", type=int, default=32, help="load cases of the batched (multi-RHS) solve")
    ap.add_argument("--order", choices=["native", "scrambled", "rcm"], default="native",
                    help="profiling mode: node numbering -- the generator's, a seeded random one, or RCM of that")
    ap.add_argument("--only", choices=["solve-mixed", "solve-fp64", "solve-multi", "spmv32", "spmv64", "frame"],
                    default=None,
                    help="profiling mode: run only this operation (warmup + steps times) and print its time")
    return ap.parse_args()


def run_only(args):
    """Profiling mode used by the ncu recipes in profiles/: one operation, nothing else."""
    import torch

    if args.only == "frame":
        print(json.dumps({"only": "frame", **frame_workload(args, torch.cuda.current_stream())}))
        return

    from wnfea_b200 import _lib
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof

    m, meta = build_model(args.slices)
    if args.order != "native":
        m = renumber(m, args.order)
    K, F_np, _ = assemble_c3d10_sparse_3dof(m)
    s = K.system
    st = torch.cuda.current_stream().cuda_stream
    n = 3 * s.n_nodes
    if args.only == "solve-multi":
        from wnfea_b200.mesh import tip_load_cases

        s.amg_setup()
        Fm = torch.from_numpy(tip_load_cases(m.mesh_nodes, n_cases=args.cases, seed=0)).cuda()
        Um = torch.empty_like(Fm)
        info = {}

        def op():
            info.update(s.solve_multi_device(Fm, Um, rtol=1e-8, precision=1, stream=st))
    elif args.only.startswith("solve"):
        s.amg_setup()
        F = torch.from_numpy(F_np).cuda()
        u = torch.empty_like(F)
        prec = 1 if args.only == "solve-mixed" else 0

        info = {}

        def op():
            prm = _lib.SolveParams(1e-8, 2000, 2, prec, 0.0, 10, 8, 1)
            stt = _lib.SolveStats()
            _lib.call("wn_solve_device", s.handle, F.data_ptr(), u.data_ptr(), prm, stt, st)
            info.update(iterations=stt.iterations, outer=stt.outer_iterations, rel_res=stt.rel_res,
                        device_ms=stt.solve_seconds * 1e3)
    else:
        prec = 1 if args.only == "spmv32" else 0
        dt = torch.float32 if prec else torch.float64
        x = torch.randn(n, dtype=torch.float64, device="cuda").to(dt)
        y = torch.empty_like(x)

        def op():
            _lib.call("wn_spmv_solid_device", s.handle, prec, x.data_ptr(), y.data_ptr(), st)
    for _ in range(args.warmup):
        op()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        op()
    torch.cuda.synchronize()
    out = {"only": args.only, "order": args.order, "ms_per_op": (time.perf_counter() - t0) * 1e3 / args.steps,
           "elements": meta["n_elements"], "nnz_blocks": s.nnzb}
    if args.only in ("solve-mixed", "solve-fp64"):
        out.update(info)
    if args.only == "solve-multi":
        out.update({"cases": args.cases, "iterations": info["iterations"], "outer": info["outer_iterations"],
                    "status": info["status"], "max_rel_res": info["rel_res"],
                    "device_ms": info["solve_seconds"] * 1e3,
                    "case_iterations": [int(v) for v in info["case_iterations"]]})
    print(json.dumps(out))


def renumber(m, order):
    """The I-beam with a seeded random node numbering (an arbitrary mesher's), or RCM of it."""
    n = len(m.mesh_nodes)
    perm = np.random.default_rng(0).permutation(n)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)
    m.mesh_nodes = m.mesh_nodes[perm].copy()
    m.solid_elements = inv[m.solid_elements].astype(np.int32)
    for item in list(m.supports) + list(m.loads):
        if not item.is_geometry_node:
            item.node_id = int(inv[item.node_id])
    if order == "rcm":
        from wnfea_b200.rcm import apply_rcm_to_model

        m = apply_rcm_to_model(m)[0]
    return m


def build_model(slices):
    from wnfea_b200.mesh import generate_c3d10_ibeam_structured

    m, meta = generate_c3d10_ibeam_structured(n_slices=slices, length=4.0 * slices / 315, seed=0)
    return m, meta


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax = max(smax, float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(name):
    """dram bytes per launch recorded in a committed ncu summary (profiles/<name>), if any."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("dram_bytes_per_launch_full_size:"):
            return float(ln.split(":", 1)[1])
    return None


def cpu_jacobi_sample(Kcsr, F, iters):
    """Seconds per iteration of the reference's CPU solve algorithm (oracle restatement of
    solve_c3d10_pcg's Jacobi branch: scipy cg + point Jacobi) on this host."""
    from scipy.sparse.linalg import LinearOperator, cg

    d = Kcsr.diagonal()
    dinv = np.where(np.abs(d) > 1e-12, 1.0 / d, 1.0)
    M = LinearOperator(Kcsr.shape, matvec=lambda v: dinv * v, dtype=np.float64)
    t0 = time.perf_counter()
    cg(Kcsr, F, M=M, rtol=1e-30, maxiter=iters)
    return (time.perf_counter() - t0) / iters


def run_reference(args):
    import scipy.sparse as sp  # noqa: F401

    from oracle import solid
    from wnfea_b200.model import solid_element_props, solid_fixed_dofs, solid_load_vector

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    m, meta = build_model(args.slices)
    ndof = meta["n_dofs"]
    K, F, _ = solid.assemble(m.mesh_nodes, m.solid_elements, solid_element_props(m), solid_load_vector(m),
                             solid_fixed_dofs(m))
    its = JACOBI_ITERS_IBEAM if (args.slices == 315 and JACOBI_ITERS_IBEAM) else None
    per_iter = []
    for _ in range(args.warmup):
        cpu_jacobi_sample(K, F, 2)
    for _ in range(args.steps):
        per_iter.append(cpu_jacobi_sample(K, F, args.cpu_iters))
    t_it = statistics.median(per_iter)
    if its is None:
        line = {"impl": "reference", "unavailable": "Jacobi-PCG iteration count for this size not measured yet"}
        print(json.dumps(line))
        return
    solve_s = t_it * its
    v = ndof / solve_s
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "DOF/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"C3D10 I-beam {meta['n_elements']} el / {ndof} DOFs, Jacobi-PCG (scipy cg) to 1e-8",
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": v, "unit": "DOF/s", "cores": 1, "kind": "port",
                         "sample": f"{args.cpu_iters} scipy cg iterations per step, x {its} iterations"},
        "e2e": {"value": v, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def internal_force(m, s, stream):
    """Matrix-free C3D10 internal force f_int(u) on the I-beam: the device-resident kernel
    (event-timed) and the reference-signature call with host buffers
    (``wn_c3d10_internal_forces``: 6-DOF stride, copies in and out inside the timed region --
    the form of the reference's HIP measurement)."""
    import torch

    from wnfea_b200 import _lib
    from wnfea_b200.model import solid_element_props

    n = s.n_nodes
    rng = np.random.default_rng(1)
    u = torch.from_numpy(rng.standard_normal(3 * n) * 1e-4).cuda()
    f = torch.empty_like(u)
    sptr = stream.cuda_stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(3):
        _lib.call("wn_fint_c3d10_device", s.handle, u.data_ptr(), f.data_ptr(), sptr)
    ev[0].record(stream)
    for _ in range(20):
        _lib.call("wn_fint_c3d10_device", s.handle, u.data_ptr(), f.data_ptr(), sptr)
    ev[1].record(stream)
    torch.cuda.synchronize()
    dev_ms = ev[0].elapsed_time(ev[1]) / 20
    nodes = np.ascontiguousarray(m.mesh_nodes, dtype=np.float64)
    conn = np.ascontiguousarray(m.solid_elements, dtype=np.int32)
    props = np.ascontiguousarray(solid_element_props(m))
    U6 = np.zeros(6 * n)
    U6.reshape(-1, 6)[:, :3] = u.cpu().numpy().reshape(-1, 3)
    F6 = np.zeros(6 * n)
    _lib.call("wn_c3d10_internal_forces", _lib.ptr(nodes), _lib.ptr(conn), _lib.ptr(props), _lib.ptr(U6), _lib.ptr(F6),
              len(conn), n)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        F6.fill(0.0)
        _lib.call("wn_c3d10_internal_forces", _lib.ptr(nodes), _lib.ptr(conn), _lib.ptr(props), _lib.ptr(U6),
                  _lib.ptr(F6), len(conn), n)
    host_ms = (time.perf_counter() - t0) * 1e3 / reps
    agree = float(np.abs(F6.reshape(-1, 6)[:, :3].ravel() - f.cpu().numpy()).max() / np.abs(f.cpu().numpy()).max())
    ne = len(conn)
    return {"elements": ne, "device_ms": dev_ms, "device_elements_per_s": ne / (dev_ms * 1e-3),
            "host_buffers_ms": host_ms, "host_buffers_elements_per_s": ne / (host_ms * 1e-3),
            "host_vs_device_max_rel_diff": agree,
            "reference_published": "8.50 ms for 213,358 elements incl. host copies (25.1 M elem/s), RX 7800 XT, "
                                   "HIP; not rerunnable here"}


def frame_workload(args, stream):
    """Linear static solve of an n x n x n space frame (beams along x, y, z at 1 m, 0.1 x 0.1 m
    sections, steel, bottom plane clamped, seeded top-plane loads): stiffness at U = 0 by the
    beam tangent kernel, AMG over the 6 rigid modes of beam nodes + PCG to true rel. res 1e-8,
    device-resident F / U, mixed (FP32 V-cycle) and FP64."""
    import torch

    from wnfea_b200.beam import frame_linear_system
    from wnfea_b200.frames import generate_space_frame

    n = args.frame_n
    t0 = time.perf_counter()
    m = generate_space_frame(n, n, n, seed=0)
    frame, system, F_np = frame_linear_system(m)
    build_s = time.perf_counter() - t0
    setup_s = system.amg_setup()
    F = torch.from_numpy(F_np).cuda()
    U = torch.empty_like(F)
    out = {"workload": f"space frame {n}^3 nodes, {len(m.mesh_elements)} beams, {F.numel()} DOFs",
           "dofs": int(F.numel()), "build_and_tangent_s": build_s, "amg_setup_s": setup_s,
           "reference_published": "2.06 M DOFs, 3.32 s solve, RX 7800 XT, HIP AMG-PCG (different frame and "
                                  "hardware; context only)"}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for prec in ("mixed_fp32", "fp64"):
        system.solve_device(F, U, rtol=1e-8, precision=prec, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        reps = 3
        ev[0].record(stream)
        for _ in range(reps):
            st = system.solve_device(F, U, rtol=1e-8, precision=prec, stream=stream.cuda_stream)
        ev[1].record(stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / reps
        out[prec] = {"solve_ms": ms, "dof_per_s": F.numel() / (ms * 1e-3), "iterations": st["iterations"],
                     "outer": st["outer_iterations"], "rel_res": st["rel_res"], "status": st["status"],
                     "levels": st["n_levels"]}
    system.close()
    frame.close()
    return out


def batched_cases(args, m, s, stream, ms_single):
    """Load cases solved together: tip forces of magnitude U[10, 100] kN along directions
    uniform on the sphere (seeded), one multi-RHS solve of the batch (FP64 PCG, FP32 V-cycle,
    per-case true residual 1e-8), device-resident F and U."""
    import torch

    from wnfea_b200.mesh import tip_load_cases

    Fm = torch.from_numpy(tip_load_cases(m.mesh_nodes, n_cases=args.cases, seed=0)).cuda()
    Um = torch.empty_like(Fm)
    sptr = stream.cuda_stream
    s.solve_multi_device(Fm, Um, rtol=1e-8, precision=1, stream=sptr)  # warm-up (workspace, graph)
    reps = max(1, min(args.steps, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        info = s.solve_multi_device(Fm, Um, rtol=1e-8, precision=1, stream=sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    ndof = 3 * s.n_nodes
    return {"cases": args.cases, "ms_per_batch": ms, "ms_per_case": ms / args.cases,
            "case_dof_per_s": args.cases * ndof / (ms * 1e-3),
            "speedup_vs_single_case_solves": args.cases * ms_single / ms,
            "batched_iterations": info["iterations"], "outer_passes": info["outer_iterations"],
            "status": info["status"], "max_case_rel_res": info["rel_res"],
            "case_iterations_min_max": [int(info["case_iterations"].min()), int(info["case_iterations"].max())],
            "workload": "same I-beam, tip forces U[10, 100] kN, direction uniform on the sphere (seed 0)"}


def adjoint_workload(args, stream):
    """Compliance adjoint on the 2 x 1 x 0.5 m block (60 x 30 x 15 hexes, 162,000 C3D10,
    per-element E log-uniform in [1, 210] GPa, seed 0; bottom clamped, 10 kN/m^2 top pressure):
    mixed-precision forward solve, dC/dE and dC/dF through torch.autograd, and a central
    finite-difference check on seeded elements (h = 1e-3 E_e, FP64 solves to 1e-12)."""
    import torch

    from wnfea_b200.autograd import ComplianceProblem
    from wnfea_b200.mesh import generate_c3d10_pressure_block
    from wnfea_b200.model import solid_element_props, solid_load_vector

    mb, meta = generate_c3d10_pressure_block(seed=0)
    props = solid_element_props(mb)
    prob = ComplianceProblem.from_model(mb, precision="mixed_fp32", rtol=1e-8, reuse_hierarchy=True)
    E = torch.from_numpy(props[:, 0].copy()).cuda().requires_grad_(True)
    F = torch.from_numpy(solid_load_vector(mb)).cuda().requires_grad_(True)
    t0 = time.perf_counter()
    C = prob.compliance(E, F)  # first forward builds the hierarchy
    C.backward()
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t0
    setup_s = prob.last_stats["setup_seconds"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(reps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    Ed, Fd = E.detach(), F.detach()
    solve_ms = timed(lambda: prob.solve(Ed, Fd), 3)
    it_mixed = prob.last_stats["iterations"]
    u, Fb = prob.solve(Ed, Fd)
    grad_ms = timed(lambda: prob.gradient(u), 20)
    g_mixed = prob.gradient(u)[0].cpu().numpy()

    def fwd_bwd():
        E.grad = None
        F.grad = None
        prob.compliance(E, F).backward()

    autograd_ms = timed(fwd_bwd, 3)
    # finite differences: FP64 solves to a true residual of 1e-12 (same hierarchy)
    prob.precision, prob.rtol = "fp64", 1e-12
    u64, Fb64 = prob.solve(Ed, Fd)
    g64 = prob.gradient(u64)[0].cpu().numpy()
    rng = np.random.default_rng(0)
    els = rng.choice(len(props), size=args.fd_elements, replace=False)
    errs = []
    t0 = time.perf_counter()
    for e in els:
        h = 1e-3 * float(props[e, 0])
        c = []
        for sg in (1.0, -1.0):
            Ep = Ed.clone()
            Ep[e] += sg * h
            up, Fbp = prob.solve(Ep, Fd)
            c.append(float(torch.dot(Fbp, up)))
        fd = (c[0] - c[1]) / (2 * h)
        errs.append(abs(fd - g64[e]) / abs(g64[e]))
    fd_s = time.perf_counter() - t0
    prob.precision, prob.rtol = "mixed_fp32", 1e-8
    ndof = 3 * len(mb.mesh_nodes)
    return {"workload": f"C3D10 block 60x30x15 hexes, {meta['n_elements']} el / {ndof} DOFs, E log-uniform "
                        "[1, 210] GPa (seed 0), bottom clamped, 10 kN/m^2 top pressure",
            "grad_kernel_ms": grad_ms, "autograd_forward_backward_ms": autograd_ms,
            "forward_solve_ms": solve_ms, "forward_iterations": it_mixed, "amg_setup_s": setup_s,
            "first_forward_backward_s": first_s,
            "fd_check": {"elements": int(args.fd_elements), "h": "1e-3 E_e", "solves": "FP64 to rel.res 1e-12",
                         "max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs)),
                         "seconds": fd_s},
            "mixed_vs_fp64_gradient_max_rel_diff": float(np.max(np.abs(g_mixed - g64)) / np.max(np.abs(g64)))}


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from wnfea_b200 import _lib
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_system

    m, meta = build_model(args.slices)
    ndof = meta["n_dofs"]
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # assembly (device time)
    t0 = time.perf_counter()
    K, F_np, fixed = assemble_c3d10_sparse_3dof(m)
    t_asm_wall = time.perf_counter() - t0
    s = K.system
    props = np.ascontiguousarray(s.props)
    d_props = torch.from_numpy(props).cuda()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(2):
        _lib.call("wn_assemble_c3d10_device", s.handle, d_props.data_ptr(), 1, sptr)
    ev[0].record(stream)
    for _ in range(3):
        _lib.call("wn_assemble_c3d10_device", s.handle, d_props.data_ptr(), 1, sptr)
    ev[1].record(stream)
    torch.cuda.synchronize()
    assembly_ms = ev[0].elapsed_time(ev[1]) / 3
    t0 = time.perf_counter()
    s.amg_setup()
    setup_s = time.perf_counter() - t0

    F = torch.from_numpy(F_np).cuda()
    u = torch.empty_like(F)
    rtol = 1e-8

    def solve(precision, precond=2, max_iter=2000):
        prm = _lib.SolveParams(rtol, max_iter, precond, precision, 0.0, 10, 8, 1)
        st = _lib.SolveStats()
        _lib.call("wn_solve_device", s.handle, F.data_ptr(), u.data_ptr(), prm, st, sptr)
        return st

    def timed(precision):
        for _ in range(args.warmup):
            solve(precision)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        launches, iters, outer, rels = 0, [], [], []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                st = solve(precision)
                launches += st.kernel_launches
                iters.append(st.iterations)
                outer.append(st.outer_iterations)
                rels.append(st.rel_res)
                if st.status != 0:
                    raise RuntimeError(f"solve did not converge: status {st.status}")
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, launches, iters, outer, max(rels), clk.summary()

    ms_mixed, launches, it_m, out_m, rel_m, clocks = timed(1)
    u_mixed = u.clone()
    ms_64, launches64, it_64, _, rel_64, clocks64 = timed(0)
    u_diff = float(torch.linalg.norm(u - u_mixed) / torch.linalg.norm(u))

    # end to end through the public API with host buffers
    for _ in range(1):
        solve_c3d10_system(K, F_np, method="pcg", rtol=rtol, precision="mixed_fp32")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        u_np, st = solve_c3d10_system(K, F_np, method="pcg", rtol=rtol, precision="mixed_fp32")
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps

    # adjoint gradient (dC/dE per element, dC/dF) on the converged field
    gE = torch.empty(s.n_el, dtype=torch.float64, device="cuda")
    gF = torch.empty_like(F)
    for _ in range(3):
        _lib.call("wn_adjoint_compliance_device", s.handle, u.data_ptr(), gE.data_ptr(), gF.data_ptr(), sptr)
    ev[0].record(stream)
    for _ in range(10):
        _lib.call("wn_adjoint_compliance_device", s.handle, u.data_ptr(), gE.data_ptr(), gF.data_ptr(), sptr)
    ev[1].record(stream)
    torch.cuda.synchronize()
    adjoint_ms = ev[0].elapsed_time(ev[1]) / 10

    fint = internal_force(m, s, stream)
    multi = None if args.skip_multi else batched_cases(args, m, s, stream, ms_mixed)
    adjoint = None if args.skip_adjoint else adjoint_workload(args, stream)
    frame_res = None if args.skip_frame else frame_workload(args, stream)

    # roofline: fine-level BSR3 SpMV, FP32 and FP64, event-timed on this stream
    nb, n_nodes = s.nnzb, s.n_nodes
    x64 = torch.randn(3 * n_nodes, dtype=torch.float64, device="cuda")
    y64 = torch.empty_like(x64)
    x32, y32 = x64.float(), torch.empty(3 * n_nodes, dtype=torch.float32, device="cuda")

    def spmv_ms(prec, x, y, reps=50):
        for _ in range(5):
            _lib.call("wn_spmv_solid_device", s.handle, prec, x.data_ptr(), y.data_ptr(), sptr)
        ev[0].record(stream)
        for _ in range(reps):
            _lib.call("wn_spmv_solid_device", s.handle, prec, x.data_ptr(), y.data_ptr(), sptr)
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    def spmv_bytes(sz):
        return nb * (9 * sz + 4) + 4 * (n_nodes + 1) + 2 * 3 * n_nodes * sz

    peak, peak_kind = measured_peaks()
    t32 = spmv_ms(1, x32, y32)
    t64 = spmv_ms(0, x64, y64)
    ach32 = spmv_bytes(4) / (t32 * 1e-3) / 1e9
    ach64 = spmv_bytes(8) / (t64 * 1e-3) / 1e9

    jacobi_iters = None
    if not args.skip_jacobi and rank == 0:
        st = solve(0, precond=1, max_iter=200000)
        jacobi_iters = st.iterations if st.status == 0 else None

    cpu = None
    if not args.skip_cpu and rank == 0 and world == 1:
        Kc = K.tocsr()
        t_it = cpu_jacobi_sample(Kc, F_np, args.cpu_iters)
        its = jacobi_iters or JACOBI_ITERS_IBEAM
        if its:
            cpu = {"value": ndof / (t_it * its), "unit": "DOF/s", "cores": 1, "kind": "port",
                   "sample": f"{args.cpu_iters} iterations of scipy cg + Jacobi on the full matrix "
                             f"({t_it * 1e3:.1f} ms/iter, 1 thread), x {its} iterations to 1e-8",
                   "solve_s": t_it * its}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = world * ndof / (ms_mixed * 1e-3)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "DOF/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (AMG, SpMV, vectors) + f64 (residual, dots, coarse Cholesky)",
        "data": "synthetic",
        "config": {
            "workload": f"C3D10 I-beam {meta['n_elements']} el / {meta['n_nodes']} nodes / {ndof} DOFs, "
                        "FP64 PCG + FP32 SA-AMG V-cycle to true rel.res 1e-8",
            "elements": meta["n_elements"], "dofs": ndof, "nnz_blocks": nb, "rtol": rtol,
            "preconditioner": "smoothed-aggregation AMG, Chebyshev(2)", "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (FP32 K 0.31 GB, FP64 K 0.61 GB per step)",
        },
        "iterations": {"mixed_inner": it_m[-1], "mixed_outer": out_m[-1], "fp64": it_64[-1]},
        "rel_res": {"mixed": rel_m, "fp64": rel_64},
        "fp64": {"value": world * ndof / (ms_64 * 1e-3), "ms_per_step": ms_64, "clocks": clocks64},
        "speedup_mixed_vs_fp64": ms_64 / ms_mixed,
        "u_rel_diff_mixed_vs_fp64": u_diff,
        "assembly_ms": assembly_ms,
        "assembly_wall_s_first_call": t_asm_wall,
        "amg_setup_s": setup_s,
        "adjoint_grad_ms": adjoint["grad_kernel_ms"] if adjoint else None,
        "adjoint_grad_ms_ibeam_field": adjoint_ms,
        "adjoint": adjoint,
        "multi_rhs": multi,
        "internal_force": fint,
        "beam_frame": frame_res,
        "jacobi_pcg_iterations": jacobi_iters,
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                     "traffic": ncu_traffic("k_stream_spmv_f32_ibeam200k.txt"), "peak_kind": peak_kind,
                     "kernel": "k_stream_spmv<float> (fine-level FP32 BSR3 SpMV streamed from the tile-major "
                               "pack by bulk async copies)",
                     "algorithmic_bytes": spmv_bytes(4), "launch_ms": t32},
        "roofline_fp64_spmv": {"achieved": ach64, "frac": ach64 / peak, "launch_ms": t64,
                               "algorithmic_bytes": spmv_bytes(8)},
        "cpu_baseline": cpu,
        "e2e": {"value": world * ndof / e2e_s, "unit": "DOF/s", "h2d_bytes_per_step": 8 * ndof,
                "d2h_bytes_per_step": 8 * ndof, "api": "solve_c3d10_system(K, F numpy) -> u numpy"},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.only:
        run_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
