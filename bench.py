"""Benchmark of the FP64 R+K element-assembly path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 64]

Workload (one "step" = one FP64 R+K iterate, constitutive update included):
J2 finite-strain plasticity on a 64^3-cell unit cube, 6 quadratic tets per
cell (1,572,864 elements, 4-point rule, 6,291,456 quadrature points,
2,146,689 nodes, 6,440,067 DOFs, ~546 M CSR non-zeros), seeded synthetic
displacement at the onset of yield.  Metric: quadrature points per second.

ours:      the sm_100a path through the C ABI.  `value` is device-timed (CUDA
           events on the launching stream) with inputs resident in HBM; the K
           values (4.4 GB) exceed L2, so no L2 flush is needed.  `e2e` times
           the host-buffer entry point (pinned u in, R and K out) end to end.
reference: the reference's element algorithm (4-nested
           compute_stiffness_matrix) restated as the CPU oracle -- the
           reference itself cannot be built here -- on all host threads, on a
           bounded element sample of the same workload per step.
Multi-GPU (torchrun): each rank assembles its own copy of the workload
(weak scaling, no data-path collective); time = max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pgfem-3d_b200"))

METRIC = "quad-points/sec for FP64 R+K assembly, % roofline; surrogate vs plain Newton"
UNIT = "qp/s"
# Algorithmic figures per R+K iterate of the J2 quadratic-tet workload:
# canonical B-form flop count per quadrature point and the byte count
# (x, u, connectivity, state read n + write n+1 at 160 B/qp, K values, R).
FLOP_PER_QP = 10.6e3


def alg_bytes(nn, ndof, ne, nqp, nnz):
    return 24.0 * nn + 8.0 * ndof + 40.0 * ne + 160.0 * nqp + 8.0 * nnz + 8.0 * ndof


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem,clocks.max.mem")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for ln in open(self.f.name):
            t = [x.strip() for x in ln.split(",")]
            if len(t) >= 9:
                rows.append(t)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        mem = [float(r[9]) for r in rows if len(r) > 10 and r[9].replace(".", "").isdigit()]
        mem_mx = [float(r[10]) for r in rows if len(r) > 10 and r[10].replace(".", "").isdigit()]
        ecc = None
        try:
            ecc = subprocess.run(["nvidia-smi", "--query-gpu=ecc.mode.current", "--format=csv,noheader",
                                  "-i", str(self.index)], capture_output=True, text=True, timeout=10).stdout.strip()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None,
                "mem_mhz": statistics.median(mem) if mem else None, "mem_max_mhz": max(mem_mx) if mem_mx else None,
                "ecc": ecc or None}


def dist_setup(ngpus, backend=None):
    """One process per GPU (torchrun environment).  The backend is NCCL on the
    GPUs; `gloo` (or PGFEM_DIST_BACKEND=gloo) runs the same host logic on CPU."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or os.environ.get("PGFEM_DIST_BACKEND", "nccl")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return ws, rank, local


def allreduce_max(x, ws):
    """Max over ranks (device timings are reported as the slowest rank's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rve_shard(nrve, ws, rank):
    """RVEs assembled by `rank`: a contiguous block of the batch, sizes within
    one of each other (the RVEs are independent: no data-path collective)."""
    base, extra = divmod(nrve, ws)
    lo = rank * base + min(rank, extra)
    return list(range(lo, lo + base + (1 if rank < extra else 0)))


def allreduce_sum(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def measured_hbm_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
        except Exception:
            pass
    return 6650.0, "fallback"


def traffic_per_launch():
    """dram bytes of one R+K iterate's two kernels (point updates, then the
    assembly) from the committed ncu summary of the J2 quadratic-tet workload."""
    path = os.path.join(ROOT, "profiles", "k_assemble_p2m_j2_p2_traffic.txt")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(ln.split(":")[1])
            except ValueError:
                return None
    return None


def cpu_baseline_sample(p, target_s, nthreads=1, bform=False):
    """Time the CPU oracle on the first S elements of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    P, mat = oracle.from_workload(p)
    e1 = 64
    t0 = time.perf_counter()
    P.assemble(mat, p.u, state_n=p.state, e1=e1, nthreads=nthreads, bform=bform)
    dt = time.perf_counter() - t0
    S = int(min(p.ne, max(e1, e1 * target_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    err, R, K, _ = P.assemble(mat, p.u, state_n=p.state, e1=S, nthreads=nthreads, bform=bform)
    t = time.perf_counter() - t0
    return S * p.nint / t, S, t


def run_ours(args, ws, rank, local):
    import torch

    import pgfem_gpu as pg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    he = args.workload == "he_p1"
    tf = args.workload == "he3f_p2"  # the three-field element on the config-2 mesh
    p = wl.he_p1(n=10, seed=0) if he else wl.j2_p2(n=args.n, seed=1)
    if tf:
        p.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.45)
        p.state = None
    log("[rank %d] setup (mesh, DOFs, CSR pattern %d nnz) %.1f s" % (rank, p.nnz, time.perf_counter() - t0))
    t0 = time.perf_counter()
    ctx = p.context()
    log("[rank %d] context (device copy + element->CSR map) %.1f s, %.2f GB on device"
        % (rank, time.perf_counter() - t0, ctx.device_bytes() / 1e9))
    ctx.set_scatter_mode({"atomic": pg.SCATTER_ATOMIC, "colour": pg.SCATTER_COLOUR}[args.scatter])
    if tf:  # element pressure 0 and volume 1 (the reference's initial values)
        ctx.set_three_field(np.zeros(p.ne), np.ones(p.ne))
    fp64_peak = pg.fp64_peak_tflops()
    hbm_peak, hbm_src = measured_hbm_gbs()

    stream = torch.cuda.current_stream()
    d_u = torch.from_numpy(p.u).to(dev)
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    sh = stream.cuda_stream

    def step():
        ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st = ctx.read_status(clear=True)
    assert st.ok(), st.as_dict()
    graph = None
    if he:
        # the small linear-tet step is launch-bound: its launches (zero fills, u
        # expansion, point updates, assembly) replayed from one CUDA graph
        graph = ctx.graph_create(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr())
        step = lambda: graph.launch(sh)  # noqa: E731
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
    ctx.set_timing(True)
    ctx.kernel_time(reset=True)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    for _ in range(max(3, args.warmup)):  # keep the GPU loaded while the sampler starts
        step()
    ctx.kernel_time(reset=True)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = clk.stop()
    ms_total = e0.elapsed_time(e1)
    kms, kcalls = ctx.kernel_time(reset=True)
    if graph is not None:  # the graph records no kernel events: time three direct calls
        for _ in range(3):
            ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh)
        torch.cuda.synchronize()
        kms, kcalls = ctx.kernel_time(reset=True)
    ctx.set_timing(False)
    st = ctx.read_status(clear=True)
    assert st.ok(), st.as_dict()
    ms_total = allreduce_max(ms_total, ws)
    ms_step = ms_total / args.steps
    value = ws * p.nqp * args.steps / (ms_total * 1e-3)
    yielded = None if (he or tf) else float((ctx.get_state(1)[:, 9] > 0).mean())

    # end to end through the host-buffer entry point (pinned host memory)
    u_h = torch.from_numpy(p.u).pin_memory().numpy()
    R_h = torch.empty(p.ndof, dtype=torch.float64).pin_memory().numpy()
    K_h = torch.empty(p.nnz, dtype=torch.float64).pin_memory().numpy()
    ctx.assemble_RK(u_h, R=R_h, K=K_h)
    n_e2e = max(1, min(args.steps, 5))
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        _, _, st = ctx.assemble_RK(u_h, R=R_h, K=K_h)
    e2e_s = allreduce_max(time.perf_counter() - t0, ws)
    assert st.ok()
    e2e_value = ws * p.nqp * n_e2e / e2e_s

    # roofline of the assembly kernels (quadratic tets: the point-update kernel
    # and the R+K assembly kernel together; linear tets: the fused kernel)
    k_ms = kms / max(kcalls, 1)
    # (the three-field element: the B-form count without the return map)
    flops = (2.5e3 if he else FLOP_PER_QP - (600.0 if tf else 0.0)) * p.nqp
    nbytes = alg_bytes(p.X.shape[0], p.ndof, p.ne, p.nqp, p.nnz)
    t_fp64 = flops / (fp64_peak * 1e12)
    t_hbm = nbytes / (hbm_peak * 1e9)
    if t_fp64 >= t_hbm:
        roof = {"bound": "fp64", "achieved": flops / (k_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                "peak_source": "measured this run (FP64 FMA-chain probe, every SM)"}
    else:
        roof = {"bound": "hbm", "achieved": nbytes / (k_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "peak_source": hbm_src}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["kernel"] = ("k_assemble<4,1,0> (fused R+K)" if he else
                      "k_qp_update<10,4,0,1,1> + k_assemble_p2m<0,1> (three-field point updates, then the condensed "
                      "R+K on the FP64 tensor cores)" if tf else
                      "k_qp_update<10,4,1,1> + k_assemble_p2m<1> (point updates, then R+K on the FP64 tensor cores)")
    roof["traffic"] = None if (he or tf) else traffic_per_launch()
    roof["kernel_ms"] = k_ms
    roof["roofline_ms"] = 1e3 * max(t_fp64, t_hbm)
    roof["frac_of_roofline_step"] = max(t_fp64, t_hbm) / (ms_step * 1e-3)
    roof["alg_flops"] = flops
    roof["alg_bytes"] = nbytes
    roof["hbm_achieved_gbs"] = nbytes / (k_ms * 1e-3) / 1e9
    roof["hbm_peak_gbs"] = hbm_peak

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded splitmix64)",
           "config": {"workload": ("compressible neo-Hookean, linear tets, 10^3 cells x 6 (%d elements, %d DOFs, "
                                   "%d CSR non-zeros), one R+K iterate replayed from a CUDA graph" %
                                   (p.ne, p.ndof, p.nnz)) if he else
                                  ("three-field (CM3F) compressible neo-Hookean, one pressure and one volume per "
                                   "element, quadratic tets, %d^3 cells x 6 (%d elements, %d quadrature points, %d "
                                   "DOFs, %d CSR non-zeros), one condensed R+K iterate" %
                                   (args.n, p.ne, p.nqp, p.ndof, p.nnz)) if tf else
                                  ("J2 finite-strain plasticity, quadratic tets, %d^3 cells x 6 (%d elements, "
                                   "%d quadrature points, %d DOFs, %d CSR non-zeros), one R+K iterate" %
                                   (args.n, p.ne, p.nqp, p.ndof, p.nnz)),
                      "elements": p.ne, "quad_points": p.nqp, "dofs": p.ndof, "nnz": p.nnz,
                      "yielded_fraction": yielded, "parallelism": "replicas%d" % ws if ws > 1 else "1 GPU",
                      "l2": "inputs larger than L2 (K values %.2f GB)" % (8e-9 * p.nnz),
                      "scatter": args.scatter},
           "roofline": roof, "clocks": clocks,
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * p.ndof,
                   "d2h_bytes_per_step": 8 * (p.ndof + p.nnz), "steps": n_e2e},
           "gpu_launches": args.steps * ctx.launches_per_assembly()}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline and not tf:
        v, S, t = cpu_baseline_sample(p, args.cpu_seconds, nthreads=1)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": "first %d elements (%d qp) of the same workload, %.1f s, reference "
                                         "4-nested element algorithm, 1 thread (one reference MPI rank)" %
                                         (S, S * p.nint, t)}
        nth = os.cpu_count() or 1
        v2, S2, t2 = cpu_baseline_sample(p, args.cpu_seconds / 2, nthreads=nth, bform=True)
        out["cpu_best"] = {"value": v2, "unit": UNIT, "cores": nth, "kind": "port",
                           "sample": "first %d elements, B-matrix form, %d threads (element colours), %.1f s"
                                     % (S2, nth, t2)}
    if graph is not None:
        graph.destroy()
    ctx.close()
    return out


# Declared FP64 work of the CP local update (survey figures for this model):
# one Newton iteration (residual with 12 power laws at 40 flop each, 10x10
# Jacobian, LU solve, one line-search residual) and the per-point fixed work
# (set-up, consistent dM/dF with 9 right-hand sides).
FLOP_CP_ITER = 10.0e3
FLOP_CP_POINT = 8.0e3


def cp_roofline(kernel_ms, iters, nqp, fp64_peak):
    flops = FLOP_CP_ITER * float(np.sum(iters)) + FLOP_CP_POINT * nqp
    ach = flops / (kernel_ms * 1e-3) / 1e12
    return {"bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
            "peak_source": "measured this run (FP64 FMA-chain probe, every SM)", "frac": ach / fp64_peak,
            "traffic": None, "kernel": "k_cp_update (local Newton)", "kernel_ms": kernel_ms, "alg_flops": flops,
            "flop_model": "%.0f per Newton iteration + %.0f per point" % (FLOP_CP_ITER, FLOP_CP_POINT)}


def cp_e2e(ctx, p, u, ws, nsteps):
    """Host-buffer path (pinned u in, R and K out) of the same R+K iterate."""
    import torch
    u_h = torch.from_numpy(u).pin_memory().numpy()
    R_h = torch.empty(p.ndof, dtype=torch.float64).pin_memory().numpy()
    K_h = torch.empty(p.nnz, dtype=torch.float64).pin_memory().numpy()
    ctx.reset_state()
    ctx.assemble_RK(u_h, dt=p.dt, R=R_h, K=K_h)
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        ctx.reset_state()
        _, _, st = ctx.assemble_RK(u_h, dt=p.dt, R=R_h, K=K_h)
    e2e_s = allreduce_max(time.perf_counter() - t0, ws)
    assert st.ok(), st.as_dict()
    return {"value": ws * p.nqp * nsteps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * p.ndof,
            "d2h_bytes_per_step": 8 * (p.ndof + p.nnz), "steps": nsteps}


def run_cp(args, ws, rank, local):
    """Config 3: FCC crystal plasticity, 48^3 cells x 6 linear tets, one R+K
    iterate at load step `--cp-step` of the 1 % tension ramp (the state of the
    previous step is produced on the GPU first)."""
    import torch

    import pgfem_gpu as pg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    p = wl.cp_p1(n=args.cp_n, seed=2)
    ctx = p.context()
    log("[rank %d] CP setup %.1f s, %d elements" % (rank, time.perf_counter() - t0, p.ne))
    for s in range(1, args.cp_step):
        _, _, st = ctx.assemble_RK(p.displacement(s), dt=p.dt)
        assert st.ok(), st.as_dict()
        ctx.commit_state()
    u = p.displacement(args.cp_step)
    stream = torch.cuda.current_stream()
    d_u = torch.from_numpy(u).to(dev)
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    sh = stream.cuda_stream

    def step():
        ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh, dt=p.dt)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st = ctx.read_status(clear=True)
    assert st.ok(), st.as_dict()
    fp64_peak = pg.fp64_peak_tflops()
    ctx.set_timing(True)
    ctx.kernel_time(reset=True)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = allreduce_max(e0.elapsed_time(e1), ws)
    kms, kc = ctx.kernel_time(reset=True)
    ctx.set_timing(False)
    it = ctx.cp_iterations()
    out = {"metric": METRIC, "value": ws * p.nqp * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded splitmix64)",
           "config": {"workload": "FCC crystal plasticity, %d^3 cells x 6 linear tets (%d elements, 1 point each), "
                                  "512 Voronoi grains, R+K at load step %d of %d (1 %% tension ramp, dt 0.1 s), "
                                  "cold-start local Newton to 1e-10" % (args.cp_n, p.ne, args.cp_step, wl.CP_STEPS),
                      "local_newton_ms": kms / max(kc, 1),
                      "iterations_hist": np.bincount(it).tolist(), "iterations_mean": float(it.mean()),
                      "l2": "one R+K iterate touches 0.4 GB (K 0.12 GB, point records 0.55 GB) > L2"},
           "roofline": cp_roofline(kms / max(kc, 1), it, p.nqp, fp64_peak), "clocks": clocks,
           "e2e": cp_e2e(ctx, p, u, ws, max(1, min(args.steps, 3))),
           "gpu_launches": args.steps * ctx.launches_per_assembly()}
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        P, mat = oracle.from_workload(p)
        sn = ctx.get_state(0)
        e1_ = 256
        t0 = time.perf_counter()
        P.assemble(mat, u, state_n=sn, dt=p.dt, e1=e1_)
        dt_ = time.perf_counter() - t0
        S = int(min(p.ne, max(e1_, e1_ * args.cpu_seconds / max(dt_, 1e-6))))
        t0 = time.perf_counter()
        P.assemble(mat, u, state_n=sn, dt=p.dt, e1=S)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": S / t, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": "first %d elements of the same step, reference element algorithm + "
                                         "restated CP local Newton, 1 thread, %.1f s" % (S, t)}
    ctx.close()
    return out


def run_cp_warm(args, ws, rank, local):
    """Config 4: the config-3 local update started from the learned guess.  The
    network is trained here, on the GPU, from plain-Newton pairs of 20 other
    seeded meshes (seeds 100..119, 32^3 cells, one load step each); then the
    same R+K iterate as config 3 is timed with the plain cold start and with
    the warm start, both to the 1e-10 local residual."""
    import torch

    import pgfem_gpu as pg
    import surrogate as sg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    x, t, info = sg.generate_pairs(n=args.train_n)
    net, hist, train_s = sg.train(x, t, seed=1, epochs=args.train_epochs, batch=8192, lr=2e-3, lr_min=2e-5)
    del x, t
    torch.cuda.empty_cache()
    log("[rank %d] %d training pairs in %.1f s, trained in %.2f s, loss %.4f -> %.4f"
        % (rank, info["pairs"], info["seconds"], train_s, hist[0], hist[-1]))
    p = wl.cp_p1(n=args.cp_n, seed=2)
    ctx = p.context()
    for s in range(1, args.cp_step):
        _, _, st = ctx.assemble_RK(p.displacement(s), dt=p.dt)
        assert st.ok(), st.as_dict()
        ctx.commit_state()
    u = p.displacement(args.cp_step)
    stream = torch.cuda.current_stream()
    d_u = torch.from_numpy(u).to(dev)
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    sh = stream.cuda_stream

    def step():
        ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh, dt=p.dt)

    def timed():
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        st = ctx.read_status(clear=True)
        assert st.ok(), st.as_dict()
        ctx.set_timing(True)
        ctx.kernel_time(reset=True)
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = allreduce_max(e0.elapsed_time(e1), ws)
        kms, kc = ctx.kernel_time(reset=True)
        ctx.set_timing(False)
        st = ctx.read_status(clear=True)
        assert st.ok(), st.as_dict()
        return ms / args.steps, kms / max(kc, 1), ctx.cp_iterations()

    fp64_peak = pg.fp64_peak_tflops()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    # plain and warm runs alternate; the speed-ups are reported as the median
    # and the range over the repeats
    runs = []
    ctx.set_cp_warm_limit(args.warm_k)
    for r in range(max(1, args.repeats)):
        ctx.set_cp_surrogate(None)
        ms_c, upd_c, it_c = timed()
        if r == 0:
            R_c = d_R.cpu().numpy()
            s_c = ctx.get_state(1)
        ctx.set_cp_surrogate(net)
        ms_w, upd_w, it_w = timed()
        runs.append((ms_c, ms_w, upd_c, upd_w))
    clocks = clk.stop()
    runs = np.array(runs)
    ms_c, ms_w, upd_c, upd_w = (float(np.median(runs[:, k])) for k in range(4))
    sp_it, sp_upd = runs[:, 0] / runs[:, 1], runs[:, 2] / runs[:, 3]
    launches = ctx.launches_per_assembly()  # with the network attached
    fb = ctx.cp_fallbacks()
    R_w = d_R.cpu().numpy()
    s_w = ctx.get_state(1)
    # the warm start converges to the same point solution (both meet 1e-10)
    state_rel = float(np.abs(s_w - s_c).max() / np.abs(s_c).max())
    R_rel = float(np.linalg.norm(R_w - R_c) / np.linalg.norm(R_c))
    # surrogate error on this step, judged by the converged plain Newton
    xx = torch.empty((p.ne, pg.MLP_IN), dtype=torch.float32, device=dev)
    tt = torch.empty((p.ne, pg.MLP_OUT), dtype=torch.float32, device=dev)
    ctx.set_cp_surrogate(None)
    step()
    ctx.cp_training_pairs(xx.data_ptr(), tt.data_ptr())
    yy = torch.empty_like(tt)
    net.predict_device(p.ne, xx.data_ptr(), yy.data_ptr(), sh)
    torch.cuda.synchronize()
    pred_err = float(torch.linalg.norm(yy - tt) / torch.linalg.norm(tt))
    ctx.set_cp_surrogate(net)
    e2e_w = cp_e2e(ctx, p, u, ws, max(1, min(args.steps, 3)))
    out = {"metric": METRIC, "value": ws * p.nqp / (ms_w * 1e-3), "unit": UNIT, "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_w, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 (network bf16 x bf16 -> f32)",
           "data": "synthetic (seeded splitmix64)",
           "config": {"workload": "FCC crystal plasticity, %d^3 cells x 6 linear tets (%d points), 512 grains, R+K "
                                  "at load step %d of %d, local Newton to 1e-10 started from the learned guess "
                                  "(cold-start fallback after %d iterations)"
                                  % (args.cp_n, p.ne, args.cp_step, wl.CP_STEPS, args.warm_k),
                      "plain_value": ws * p.nqp / (ms_c * 1e-3), "plain_ms_per_step": ms_c,
                      "repeats": int(len(runs)),
                      "speedup_rk_iterate": float(np.median(sp_it)),
                      "speedup_rk_iterate_range": [float(sp_it.min()), float(sp_it.max())],
                      "local_update_ms": {"plain": upd_c, "warm": upd_w},
                      "speedup_local_update": float(np.median(sp_upd)),
                      "speedup_local_update_range": [float(sp_upd.min()), float(sp_upd.max())],
                      "speedup_runs": [[float(a), float(b)] for a, b in zip(sp_it, sp_upd)],
                      "iterations_mean": {"plain": float(it_c.mean()), "warm": float(it_w.mean())},
                      "iterations_hist": {"plain": np.bincount(it_c).tolist(), "warm": np.bincount(it_w).tolist()},
                      "fallbacks": fb, "warm_vs_plain_state_rel": state_rel, "warm_vs_plain_R_rel": R_rel,
                      "network": {"params": pg.Mlp.num_params(), "train_pairs": info["pairs"],
                                  "train_seeds": "100..119 (%d^3 cells, one load step each)" % args.train_n,
                                  "pair_generation_s": info["seconds"], "train_s": train_s,
                                  "epochs": args.train_epochs, "loss_first_last": [float(hist[0]), float(hist[-1])],
                                  "prediction_rel_err": pred_err}},
           "roofline": cp_roofline(upd_w, it_w, p.nqp, fp64_peak), "clocks": clocks, "e2e": e2e_w,
           "gpu_launches": args.steps * launches}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        P, mat = oracle.from_workload(p)
        sn = ctx.get_state(0)
        S = 20000
        t0 = time.perf_counter()
        P.assemble(mat, u, state_n=sn, dt=p.dt, e1=S)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": S / t, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": "first %d elements of the same step, reference element algorithm + "
                                         "restated CP local Newton (cold start), 1 thread, %.1f s" % (S, t)}
    ctx.close()
    return out


FLOP_PER_QP_P1 = 3.1e3  # linear-tet B-form (~2.5 k) + J2 return map (~0.6 k) per point


def run_rve(args, ws, rank, local):
    """Config 5: FE2 micro-RVE batch -- `--nrve` independent periodic unit
    cells of uneven size (n_r^3 cells x 6 linear tets, n_r uniform in 8..24),
    each with its own macro deformation, assembled (R+K, J2 update) in ONE
    persistent work-stealing launch replayed from a captured CUDA graph, with
    the block size and steal size picked by the autotuner."""
    import torch

    import pgfem_gpu as pg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    shard = rve_shard(args.nrve, ws, rank)
    p = wl.rve_batch(nrve=args.nrve, subset=shard)
    log("[rank %d] RVEs %d..%d of %d: %d elements, %d DOFs, %d nnz, built in %.1f s"
        % (rank, shard[0], shard[-1], args.nrve, p.ne, p.ndof, p.nnz, time.perf_counter() - t0))
    ctx = p.context()
    fp64_peak = pg.fp64_peak_tflops()
    hbm_peak, hbm_src = measured_hbm_gbs()
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    d_u = torch.from_numpy(p.u).to(dev)
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    epb, grab, tune_ms = ctx.autotune(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), reps=3)
    log("[rank %d] autotune: %d elements per block, steal %d blocks, %.3f ms (%.1f s)"
        % (rank, epb, grab, tune_ms, time.perf_counter() - t0))
    ctx.set_schedule(0, 0)
    ctx.set_timing(True)
    ctx.kernel_time(reset=True)
    for _ in range(3):
        ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh)
    static_kms, n_ = ctx.kernel_time(reset=True)
    ctx.set_timing(False)
    ctx.set_schedule(epb, grab)
    g = ctx.graph_create(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr())
    for _ in range(args.warmup):
        g.launch(sh)
    torch.cuda.synchronize()
    st = ctx.read_status(clear=True)
    assert st.ok(), st.as_dict()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    for _ in range(max(3, args.warmup)):
        g.launch(sh)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        g.launch(sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = clk.stop()
    ms_step = allreduce_max(e0.elapsed_time(e1), ws) / args.steps
    # kernel-only time of the tuned launch (events around the assembly kernel)
    ctx.set_timing(True)
    ctx.kernel_time(reset=True)
    for _ in range(3):
        ctx.assemble_RK_device(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), sh)
    kms, kc = ctx.kernel_time(reset=True)
    k_ms = kms / max(kc, 1)
    ctx.set_timing(False)
    # per-RVE reference check on the smallest and the largest RVE
    R_all = d_R.cpu().numpy()
    K_all = d_K.cpu().numpy()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    checks = []
    for r in sorted({int(np.argmin(p.n_r)), int(np.argmax(p.n_r))}):
        q = p.rve(r)
        P, mat = oracle.from_workload(q)
        err, Ro, Ko, _ = P.assemble(mat, q.u, state_n=q.state, nthreads=os.cpu_count() or 1)
        d0, d1 = p.dof_off[r], p.dof_off[r + 1]
        checks.append({"rve": r, "n": int(p.n_r[r]),
                       "R_rel": float(np.linalg.norm(R_all[d0:d1] - Ro) / np.linalg.norm(Ro)),
                       "K_rel": float(np.linalg.norm(K_all[p.Ap[d0]:p.Ap[d1]] - Ko) / np.linalg.norm(Ko))})
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        q = p.rve(int(np.argmin(p.n_r)))
        P, mat = oracle.from_workload(q)
        t0 = time.perf_counter()
        P.assemble(mat, q.u, state_n=q.state, nthreads=1)
        t1 = time.perf_counter() - t0
        cpu_base = {"value": q.nqp / t1, "unit": UNIT, "cores": 1, "kind": "port",
                    "sample": "the smallest RVE (%d^3 cells, %d elements), reference element algorithm, 1 thread, "
                              "%.2f s" % (q.meta["n"], q.ne, t1)}
    else:
        cpu_base = None
    # end to end: pinned host u in, R and K out, through the captured graph
    u_h = torch.from_numpy(p.u).pin_memory()
    R_h = torch.empty(p.ndof, dtype=torch.float64).pin_memory()
    K_h = torch.empty(p.nnz, dtype=torch.float64).pin_memory()
    n_e2e = max(1, min(args.steps, 5))
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        d_u.copy_(u_h, non_blocking=True)
        g.launch(sh)
        R_h.copy_(d_R, non_blocking=True)
        K_h.copy_(d_K, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, ws)
    g.destroy()
    flops = FLOP_PER_QP_P1 * p.nqp
    nbytes = 24.0 * p.X.shape[0] + 16.0 * p.ndof + 16.0 * p.ne + 160.0 * p.nqp + 8.0 * p.nnz
    t_fp64 = flops / (fp64_peak * 1e12)
    t_hbm = nbytes / (hbm_peak * 1e9)
    if t_fp64 >= t_hbm:
        roof = {"bound": "fp64", "achieved": flops / (k_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                "peak_source": "measured this run (FP64 FMA-chain probe, every SM)"}
    else:
        roof = {"bound": "hbm", "achieved": nbytes / (k_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "peak_source": hbm_src}
    roof.update({"frac": roof["achieved"] / roof["peak"], "traffic": None, "kernel_ms": k_ms,
                 "roofline_ms": 1e3 * max(t_fp64, t_hbm), "alg_flops": flops, "alg_bytes": nbytes})
    nqp_all = allreduce_sum(p.nqp, ws)
    out = {"metric": METRIC, "value": nqp_all / (ms_step * 1e-3), "unit": UNIT, "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
           "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded splitmix64)",
           "config": {"parallelism": "RVEs sharded over %d ranks, no collective" % ws if ws > 1 else "1 GPU",
                      "workload": "FE2 micro-RVE batch: %d periodic unit cells, n^3 cells x 6 linear tets with n "
                                  "uniform in 8..24 (%d elements, %d DOFs, %d nnz), J2, per-RVE macro F = I + "
                                  "sym(U(-0.02, 0.02)), one R+K iterate per step as one persistent work-stealing "
                                  "launch replayed from a CUDA graph" % (args.nrve, p.ne, p.ndof, p.nnz),
                      "autotune": {"elems_per_block": epb, "steal_blocks": grab, "tuned_ms": tune_ms,
                                   "static_schedule_kernel_ms": static_kms / max(n_, 1)},
                      "rve_checks_vs_oracle": checks,
                      "l2": "inputs larger than L2 (K values %.2f GB)" % (8e-9 * p.nnz)},
           "roofline": roof, "clocks": clocks,
           "e2e": {"value": nqp_all * n_e2e / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * p.ndof,
                   "d2h_bytes_per_step": 8 * (p.ndof + p.nnz), "steps": n_e2e},
           "gpu_launches": args.steps * ctx.launches_per_assembly()}
    if cpu_base:
        out["cpu_baseline"] = cpu_base
    ctx.close()
    return out


NR_METRIC = "Newton-Raphson load steps/sec (device assembly + GMRES), SpMV % of HBM roofline"


def run_nr(args, ws, rank, local):
    """One Newton-Raphson load step on the device (the consumer of K): J2
    quadratic tets, `--nr-n`^3 cells, x = 0 face fixed, x = 1 face pulled to
    `--nr-stretch` in one step from the linear predictor u_x = stretch x; each
    Newton iteration assembles R and K on the device and solves K du = -R with
    GMRES(kdim) + diagonal scaling (pgfem_gpu_newton_step).  A step = state
    reset, u = predictor, the whole Newton loop.  Roofline: the CSR SpMV that dominates the
    solve, timed alone on the step's K (HBM-bound: 12 bytes per non-zero)."""
    import torch

    import pgfem_gpu as pg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    p = wl.tension(n=args.nr_n, nne=10, model="j2", stretch=args.nr_stretch, predictor=True)
    ctx = p.context()
    solver = pg.Solver(p.Ap, p.Ai, p.ndof, maxit=args.nr_maxit, kdim=args.nr_kdim, tol=args.nr_tol)
    log("[rank %d] tension J2 P2 n=%d: %d elements, %d DOFs, %d nnz, set up in %.1f s"
        % (rank, args.nr_n, p.ne, p.ndof, p.nnz, time.perf_counter() - t0))
    hbm_peak, hbm_src = measured_hbm_gbs()
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    d_u0 = torch.from_numpy(p.u.copy()).to(dev)
    d_u = torch.empty_like(d_u0)
    d_p = torch.from_numpy(p.u_presc.copy()).to(dev)
    infos = []

    def step():
        ctx.reset_state()
        d_u.copy_(d_u0)
        info = solver.newton_step(ctx, d_u.data_ptr(), d_p.data_ptr(), iter_max=20, nor_min=args.nr_nor_min,
                                  stream=sh)
        assert info.converged and info.elem_failures == 0, (info.iters, info.history())
        return info

    for _ in range(args.warmup):
        infos.append(step())
    nsteps = max(1, min(args.steps, args.nr_steps))
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nsteps):
        infos.append(step())
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = clk.stop()
    ms_step = allreduce_max(e0.elapsed_time(e1), ws) / nsteps
    info = infos[-1]
    # split: the assemblies of the step, timed alone
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    ctx.set_timing(True)
    ctx.kernel_time(reset=True)
    for _ in range(3):
        ctx.assemble_RK_device(d_u.data_ptr(), d_p.data_ptr(), d_R.data_ptr(), d_K.data_ptr(), sh)
    kms, kc = ctx.kernel_time(reset=True)
    ctx.set_timing(False)
    asm_ms = kms / max(kc, 1)
    # SpMV alone on the converged K (inputs larger than L2 when 12 nnz > 126 MB)
    d_x = torch.rand(p.ndof, dtype=torch.float64, device=dev)
    d_y = torch.empty_like(d_x)
    for _ in range(5):
        solver.spmv(d_K.data_ptr(), d_x.data_ptr(), d_y.data_ptr(), sh)
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    nsp = 50
    s0.record(stream)
    for _ in range(nsp):
        solver.spmv(d_K.data_ptr(), d_x.data_ptr(), d_y.data_ptr(), sh)
    s1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = s0.elapsed_time(s1) / nsp
    spmv_bytes = 12.0 * p.nnz + 4.0 * (p.ndof + 1) + 16.0 * p.ndof
    roof = {"bound": "hbm", "achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
            "peak_source": hbm_src, "kernel": "k_spmv (CSR, warp per row)", "kernel_ms": spmv_ms,
            "alg_bytes": spmv_bytes, "traffic": None}
    roof["frac"] = roof["achieved"] / roof["peak"]
    # kernels of one step: per assembly its kernels + the norm (2); per solve the
    # negation, the diagonal scaling and the final residual (5); per GMRES cycle
    # 6; per queued Arnoldi step 11 (steps are queued 8 at a time, so a cycle
    # queues at most 7 beyond its last step)
    solves = info.iters
    cycles = solves + info.lin_iters // max(args.nr_kdim, 1)
    launches = (info.iters + 1) * (ctx.launches_per_assembly() + 2) + 5 * solves + 6 * cycles \
        + 11 * (info.lin_iters + 7 * cycles)
    out = {"metric": NR_METRIC, "value": 1e3 / ms_step, "unit": "steps/s", "n_gpus": ws, "steps": nsteps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (structured mesh, uniaxial tension)",
           "config": {"workload": "one Newton-Raphson load step, J2 quadratic tets, %d^3 cells x 6 (%d elements, "
                                  "%d DOFs, %d nnz), uniaxial stretch %.4g in one step from the linear "
                                  "predictor, full Newton to ||R||/||R0|| <= %.0e, GMRES(%d) + diagonal "
                                  "scaling to %.0e"
                                  % (args.nr_n, p.ne, p.ndof, p.nnz, args.nr_stretch, args.nr_nor_min,
                                     args.nr_kdim, args.nr_tol),
                      "newton_iterations": info.iters, "linear_iterations": info.lin_iters,
                      "residual_history": info.history(),
                      "assembly_ms": asm_ms, "assembly_share": info.iters and (info.iters + 1) * asm_ms / ms_step,
                      "spmv_ms": spmv_ms,
                      "l2": "K values + column ids %.0f MB (L2 126 MB)" % (12e-6 * p.nnz),
                      "parallelism": "replicas%d" % ws if ws > 1 else "1 GPU"},
           "roofline": roof, "clocks": clocks,
           "e2e": {"value": 1e3 / ms_step, "unit": "steps/s", "h2d_bytes_per_step": 8 * len(p.u_presc),
                   "d2h_bytes_per_step": 0, "note": "the step's input is the prescribed value (the predictor and "
                                                    "the state are reset on the device); nothing returns to the "
                                                    "host but the convergence flags"},
           "gpu_launches": int(nsteps * launches)}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        from scipy.sparse import csr_matrix
        from scipy.sparse.linalg import LinearOperator, bicgstab
        P, mat = oracle.from_workload(p)
        nth = os.cpu_count() or 1
        t0 = time.perf_counter()
        P.assemble(mat, p.u, p.u_presc, state_n=p.state, nthreads=nth)
        t_asm = time.perf_counter() - t0
        Km = csr_matrix((d_K.cpu().numpy(), p.Ai, p.Ap), shape=(p.ndof, p.ndof))
        dinv = 1.0 / Km.diagonal()
        M = LinearOperator(Km.shape, matvec=lambda v: dinv * v)
        b = np.random.default_rng(0).normal(size=p.ndof)
        nit = 20
        t0 = time.perf_counter()
        bicgstab(Km, b, rtol=1e-30, maxiter=nit, M=M)
        t_it = (time.perf_counter() - t0) / nit
        t_cpu = (info.iters + 1) * t_asm + info.lin_iters * t_it
        out["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "steps/s", "cores": nth, "kind": "port",
                               "sample": "one R+K assembly of the step (CPU oracle, %d threads, %.2f s) and %d "
                                         "BiCGSTAB iterations (scipy, diagonal scaling, %.3f s each), scaled to "
                                         "the step's %d assemblies and %d linear iterations"
                                         % (nth, t_asm, nit, t_it, info.iters + 1, info.lin_iters)}
    solver.close()
    ctx.close()
    return out


def run_transient(args, ws, rank, local):
    """The transient (inertia, mid-point rule) element on the device
    (pgfem_gpu_assemble_RK_transient_device): `cp_tr` -- crystal plasticity on
    the config-3 mesh (`--cp-n`), states at t_{n-1}, t_n from two committed load
    steps of the tension ramp, u_{n+1} the third step; `he3f_tr` -- the
    three-field neo-Hookean element on the config-2 mesh (`--n`), P and theta
    histories set.  A step = one transient R+K call (alpha 0.5, rho 7.85e-9,
    dt 0.1); the quasi-static R+K at u_{n+1} is timed beside it."""
    import torch

    import pgfem_gpu as pg
    import workloads as wl
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cp = args.workload == "cp_tr"
    t0 = time.perf_counter()
    alpha, dt1, dt0, rho = 0.5, 0.1, 0.1, 7.85e-9

    def problem(n):
        if cp:
            q = wl.cp_p1(n=n, seed=2)
            us = [q.displacement(3), q.displacement(2), q.displacement(1)]
            return q, us, None, None
        q = wl.j2_p2(n=n, seed=1)
        q.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.45)
        q.state = None
        r = np.random.default_rng(4)
        us = [q.u, 0.7 * q.u, 0.4 * q.u]
        Ps = [np.zeros(q.ne), 5.0 * r.uniform(-1, 1, q.ne), 2.0 * r.uniform(-1, 1, q.ne)]
        ths = [np.ones(q.ne), 1.0 + 1e-3 * r.uniform(-1, 1, q.ne), 1.0 + 1e-3 * r.uniform(-1, 1, q.ne)]
        return q, us, Ps, ths

    p, us, Ps, ths = problem(args.cp_n if cp else args.n)
    ctx = p.context()
    if cp:
        for k in (1, 2):
            _, _, st = ctx.assemble_RK(p.displacement(k), dt=p.dt)
            assert st.ok(), st.as_dict()
            ctx.commit_state()
        dt1 = dt0 = p.dt
    else:
        ctx.set_three_field(Ps[0], ths[0])
        ctx.set_three_field_history(Ps[1], ths[1], Ps[2], ths[2])
    log("[rank %d] %s setup %.1f s, %d elements, %d nnz" % (rank, args.workload, time.perf_counter() - t0, p.ne,
                                                          p.nnz))
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    d_us = [torch.from_numpy(np.ascontiguousarray(u)).to(dev) for u in us]
    d_R = torch.empty(p.ndof, dtype=torch.float64, device=dev)
    d_K = torch.empty(p.nnz, dtype=torch.float64, device=dev)
    ptrs = [d.data_ptr() for d in d_us]

    def step():
        ctx.assemble_RK_transient_device(ptrs, [0, 0, 0], alpha, dt1, dt0, rho, d_R.data_ptr(), d_K.data_ptr(), sh)

    def quasi():
        ctx.assemble_RK_device(ptrs[0], None, d_R.data_ptr(), d_K.data_ptr(), sh, dt=dt1)

    def timed(fn, n):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st = ctx.read_status(clear=True)
    assert st.ok(), st.as_dict()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    ms = allreduce_max(timed(step, args.steps), ws)
    clocks = clk.stop()
    ms_qs = timed(quasi, 3)
    # end to end: the host-buffer call (three displacement vectors in, R and K out)
    t0 = time.perf_counter()
    ne2 = 2
    for _ in range(ne2):
        ctx.assemble_RK_transient(us[0], us[1], us[2], alpha, dt1, dt0, rho)
    e2e_s = (time.perf_counter() - t0) / ne2
    nqp = p.ne * (1 if cp else 4)
    out = {"metric": "quad-points/sec for the FP64 transient (mid-point rule) R+K", "value": nqp / (ms * 1e-3),
           "unit": "qp/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded splitmix64 mesh perturbation / load ramp)",
           "config": {"workload": ("crystal plasticity, linear tets, %d^3 cells x 6 (%d elements), transient R+K "
                                   "with the mid-point plastic state" % (args.cp_n, p.ne)) if cp else
                                  ("three-field neo-Hookean, quadratic tets, %d^3 cells x 6 (%d elements, %d qp, "
                                   "%d nnz), transient R+K: two condensed assemblies + correction + inertia"
                                   % (args.n, p.ne, nqp, p.nnz)),
                      "alpha": alpha, "dt": [dt1, dt0], "rho": rho, "quasi_static_ms": ms_qs,
                      "transient_over_quasi_static": ms / ms_qs,
                      "l2": "inputs larger than L2 (K values %.2f GB)" % (8e-9 * p.nnz),
                      "parallelism": "replicas%d" % ws if ws > 1 else "1 GPU"},
           "roofline": None,
           "roofline_note": "the transient call runs the quasi-static kernels (CP: one point update and the "
                            "mid-point element; three-field: two condensed assemblies), whose rooflines are the "
                            "cp_p1 and he3f_p2 lines; this line reports its cost against the quasi-static iterate",
           "clocks": clocks,
           "e2e": {"value": nqp / e2e_s, "unit": "qp/s", "h2d_bytes_per_step": 3 * 8 * p.ndof,
                   "d2h_bytes_per_step": 8 * (p.ndof + p.nnz), "timer": "host wall clock around the synchronous call"}}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        n_s = 16 if cp else 12
        q, qus, qPs, qths = problem(n_s)
        P, mat = oracle.from_workload(q)
        t0 = time.perf_counter()
        if cp:
            _, _, _, s1 = P.assemble(mat, q.displacement(1), state_n=q.state, dt=q.dt, want_K=False)
            _, _, _, s2 = P.assemble(mat, q.displacement(2), state_n=s1, dt=q.dt, want_K=False)
            t0 = time.perf_counter()
            oracle.assemble_transient_cp(P, mat, qus[0], qus[1], qus[2], alpha, q.dt, q.dt, rho, s1, s2)
        else:
            P.assemble_3f_transient(mat, qus, qPs, qths, alpha, dt1, dt0, rho)
        t_cpu = time.perf_counter() - t0
        nq = q.ne * (1 if cp else 4)
        out["cpu_baseline"] = {"value": nq / t_cpu, "unit": "qp/s", "cores": 1, "kind": "port",
                               "sample": "the same transient call on the %d^3-cell mesh (%d qp), oracle, 1 thread, "
                                         "%.2f s" % (n_s, nq, t_cpu)}
    ctx.close()
    return out


def run_reference(args, ws, rank):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if rank != 0:
        return None
    nth = os.cpu_count() or 1
    # the same workload restricted to an element sample: the first cells of
    # the n^3 mesh in element order (identical per-element work), built by the
    # oracle's own mesher, DOF numbering and CSR pattern (no product code)
    P, mat, u, state = oracle.j2_p2_problem(args.n, seed=1, max_cells_z=args.ref_layers)

    class _W:  # the attributes the timing below reads
        pass
    p = _W()
    p.u, p.state, p.ne, p.nint = u, state, int(P.conn.shape[0]), 4
    per_step = min(10.0, 150.0 / max(1, args.steps + args.warmup))
    t0 = time.perf_counter()
    P.assemble(mat, p.u, state_n=p.state, e1=min(p.ne, 256), nthreads=nth)
    dt = time.perf_counter() - t0
    S = int(min(p.ne, max(256, 256 * per_step / max(dt, 1e-6))))
    for _ in range(args.warmup):
        P.assemble(mat, p.u, state_n=p.state, e1=min(S, 256), nthreads=nth)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        err, R, K, _ = P.assemble(mat, p.u, state_n=p.state, e1=S, nthreads=nth)
        ts.append(time.perf_counter() - t0)
        assert err == 0
    value = S * p.nint * len(ts) / sum(ts)
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(ts) / len(ts), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded splitmix64)",
            "impl": "reference",
            "config": {"workload": "J2 finite-strain plasticity, quadratic tets, %d^3 cells x 6, one R+K iterate "
                                   "(element sample per step)" % args.n, "sample_elements": S},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port",
                             "sample": "first %d elements per step, reference 4-nested element algorithm "
                                       "(CPU oracle; the reference needs MPI, GCM, TTL, hypre, msnet and "
                                       "cannot be built here), %d threads over element colours" % (S, nth)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-layers", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scatter", default="atomic", choices=["atomic", "colour"])
    ap.add_argument("--workload", default="j2_p2", choices=["j2_p2", "he3f_p2", "he_p1", "cp_p1", "cp_warm", "cp_tr", "he3f_tr", "rve_batch",
                                                         "nr_step"])
    ap.add_argument("--nr-n", type=int, default=16)
    ap.add_argument("--nr-stretch", type=float, default=0.003)
    ap.add_argument("--nr-tol", type=float, default=1e-8)
    ap.add_argument("--nr-maxit", type=int, default=20000)
    ap.add_argument("--nr-nor-min", type=float, default=1e-8)
    ap.add_argument("--nr-steps", type=int, default=1)
    ap.add_argument("--nr-kdim", type=int, default=100)
    ap.add_argument("--nrve", type=int, default=256)
    ap.add_argument("--train-n", type=int, default=32)
    ap.add_argument("--train-epochs", type=int, default=30)
    ap.add_argument("--warm-k", type=int, default=6)
    ap.add_argument("--repeats", type=int, default=5, help="cp_warm: alternating plain / warm runs (median, range)")
    ap.add_argument("--cp-n", type=int, default=48)
    ap.add_argument("--cp-step", type=int, default=10)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        out = run_reference(args, ws, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    ws, rank, local = dist_setup(args.gpus)
    if args.workload == "cp_p1":
        out = run_cp(args, ws, rank, local)
    elif args.workload == "cp_warm":
        out = run_cp_warm(args, ws, rank, local)
    elif args.workload == "rve_batch":
        out = run_rve(args, ws, rank, local)
    elif args.workload == "nr_step":
        out = run_nr(args, ws, rank, local)
    elif args.workload in ("cp_tr", "he3f_tr"):
        out = run_transient(args, ws, rank, local)
    else:
        out = run_ours(args, ws, rank, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
