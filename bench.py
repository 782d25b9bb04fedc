"""Benchmark: solved DOF/s of the weighted-quadrature elasticity solve.

Workload (one step = one complete Jacobi-PCG solve): the unit-cube NURBS patch
of degree 3 with 64 x 64 x 64 elements (67^3 control points, 902,289 dofs),
interior control points perturbed U(-0.2h, 0.2h), geometry weights
U(0.8, 1.2), E=1, nu=0.3, clamped at z=0, body force (0, 0, -1), solved to
||r|| <= 1e-9 ||b|| (relative error <= 1e-8 against a 1e-12 FP64 solution)
by Jacobi-PCG with the FP32 operator and FP32 Krylov vectors, and FP64
true-residual replacement (reliable updates).  Synthetic, seeded inputs; the
operator data (1.27 GB) is far larger than L2, so no L2 flush is needed
between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0).  Under torchrun each rank solves its own
replica (no collective in the data path: replicas only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("solved DOF/s at rel.err<=1e-8 (mixed vs plain FP64, 1 B200); "
          "serve p50/p99 ms")
WORKLOAD = {"workload": "WQ elasticity PCG, unit-cube NURBS patch p=3 64^3 "
                        "elements, perturbed +-0.2h, weights U(0.8,1.2), "
                        "E=1 nu=0.3, clamped z=0, body force (0,0,-1)",
            "nel": [64, 64, 64], "p": 3, "seed": 20261203,
            "l2": "operator data (1.27 GB) larger than L2: no flush needed"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nel", type=int, nargs=3, default=[64, 64, 64])
    ap.add_argument("--p", type=int, default=3)
    ap.add_argument("--rtol", type=float, default=1e-9)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=25.0,
                    help="Poisson arrival rate of the serving stream (requests/s)")
    ap.add_argument("--serve-rate-high", type=float, default=80.0,
                    help="second serving stream near saturation (requests/s; 0: none)")
    ap.add_argument("--serve-rate-capacity", type=float, default=160.0,
                    help="third serving stream above the 80/s point, to show the "
                         "sustained capacity (requests/s; 0: none)")
    ap.add_argument("--serve-budget-gb", type=float, default=32.0)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-precond", default="fd", choices=["jacobi", "fd"],
                    help="preconditioner of the served solves")
    ap.add_argument("--serve-method", default="bicgstab", choices=["cg", "bicgstab"],
                    help="Krylov method of the served solves")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the assembly, gradient and p=4 block measurements")
    ap.add_argument("--only-extra", action="store_true",
                    help="run only the assembly, mass, gradient, volume and p=4 block "
                         "measurements (one JSON line with other_configs)")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name):
    """Bytes per launch read from a committed ncu summary (profiles/), if any:
    a line 'traffic_bytes_per_launch: <float>'."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Each rank solves its own replica of the workload (replicas only: no
    collective in the data path), seeded by its rank."""
    return WORKLOAD["seed"] + rank


def aggregate_rate(units_per_rank, ms_max, ws, steps=1):
    """Whole-job throughput: the units all ranks processed divided by the
    slowest rank's time (max over ranks)."""
    return ws * units_per_rank * steps / (ms_max / 1e3)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------ CPU baseline
def cpu_reference_rate(args, iters_fp64, iters_source, sample_iters=10):
    """The reference's algorithm on the host cores: the restated
    mf_wq_get_ku_3d with the rank-one sparse products of
    tensor3d_sparsedot_vector (oracle/oracle_wq.c, OpenMP over all cores)
    inside the Jacobi-PCG loop of wq_mf_cg_3d; `sample_iters` consecutive
    iterations (apply and vector work) of the full workload are timed as one
    loop; solved DOF/s = n_free / (iterations to converge x seconds per
    iteration)."""
    import oracle.wq_cpu as wc
    from yeti_b200.patches import cube_patch
    P = cube_patch(tuple(args.nel), args.p, perturb=0.2, wrange=(0.8, 1.2),
                   seed=WORKLOAD["seed"])
    res = wc.time_reference_cg(P, 1.0, 0.3, {"w0": (0, 1, 2)}, iters=sample_iters,
                               seed=WORKLOAD["seed"])
    t_iter = res["seconds_per_iteration"]
    nfree = res["nfree"]
    return {"value": nfree / (iters_fp64 * t_iter), "unit": "DOF/s",
            "cores": res["threads"], "kind": "port",
            "seconds_per_iteration": t_iter, "iterations": int(iters_fp64),
            "sample": (f"{sample_iters} consecutive Jacobi-PCG iterations (operator apply "
                       f"with the reference's rank-one sparse products, dots, updates, "
                       f"z = r/diag) of the full {args.nel} p={args.p} workload timed as "
                       f"one loop: {t_iter:.3f} s per iteration on {res['threads']} "
                       f"threads; x {int(iters_fp64)} iterations to converge "
                       f"({iters_source})")}


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    iters = ITERS_FP64_DEFAULT
    vals = []
    base = None
    for _ in range(args.warmup + args.steps):
        base = cpu_reference_rate(args, iters, ITERS_SOURCE)
        vals.append(base["value"])
    v = statistics.median(vals[args.warmup:]) if args.steps else vals[-1]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "DOF/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, nel=args.nel, p=args.p),
            "cpu_baseline": dict(base, value=v),
            "e2e": {"value": v, "unit": "DOF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def serve_stream(args, device, rate=None):
    """The serving workload: a seeded stream of requests (cube-like NURBS
    patches, p in {2,3}, 4..32 elements per direction, 1..8 Gaussian
    right-hand sides, FP64 preconditioned Krylov solves to 1e-8:
    --serve-method, --serve-precond) with Poisson arrivals at --serve-rate,
    through the persistent loop (yeti_b200.serve.Server)."""
    from yeti_b200.serve import Server, run_stream, synthetic_requests
    reqs = synthetic_requests(args.serve_requests, seed=WORKLOAD["seed"] + 7)
    budget = int(args.serve_budget_gb * (1 << 30))
    with Server(device=device, hbm_budget_bytes=budget, max_active=128) as srv:
        rate = args.serve_rate if rate is None else rate
        out = run_stream(srv, reqs, rate, seed=WORKLOAD["seed"] + 8, rtol=1e-8,
                         precond=args.serve_precond, method=args.serve_method)
        st = srv.stats()
    lat = out["latency_ms"]
    its = [sum(r["iterations"]) for r in out["results"] if r is not None]
    return {"requests": len(reqs), "completed": int(len(lat)), "errors": len(out["errors"]),
            "arrival_rate_per_s": rate, "offered_s": out["offered_s"],
            "wall_s": out["wall_s"],
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "solved_dof_per_s": out["solved_dofs"] / out["wall_s"],
            "completed_per_s": len(lat) / out["wall_s"],
            "cg_iterations_total": int(sum(its)), "peak_active": st["peak_active"],
            "thread_ms": {"setup": st["setup_ms"], "retire": st["retire_ms"],
                          "poll": st["poll_ms"]},
            "max_active": 128, "hbm_budget_bytes": budget, "rtol": 1e-8,
            "precision": "FP64 operator and Krylov vectors",
            "preconditioner": args.serve_precond, "method": args.serve_method}


def _median_ms(fn, reps, sync, with_min=False):
    """Median wall time of fn() in ms (with_min: also the fastest call; on a
    shared host the calls that allocate and copy host buffers vary by tens of
    ms from run to run, the minimum is the call's own cost)."""
    ts = []
    for _ in range(reps):
        sync()
        t0 = time.perf_counter()
        fn()
        sync()
        ts.append((time.perf_counter() - t0) * 1e3)
    if with_min:
        return float(np.median(ts)), float(np.min(ts))
    return float(np.median(ts))


def _system_args(name):
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES
    d = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))
    return [d[k] if d[k].ndim else d[k][()] for k in SYSTEM_ARG_NAMES]


def _event_ms(fn, reps):
    """Median device time of fn() between two CUDA events on the current
    stream (the library's), after one warm call."""
    import torch
    fn()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def fp64_peak_tflops():
    """Measured FP64 GEMM rate (cuBLAS DGEMM 8192^3, best of 5): the FP64
    denominator of the Gauss kernels' compute rooflines."""
    import torch
    n = 8192
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    B = torch.randn_like(A)
    for _ in range(2):
        A @ B
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        A @ B
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del A, B
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def stiffness_flops(nq, nn, nel):
    """FP64 operations of k_u1_stiffness: per (point, node pair) the nine
    B_i^T D B_j entries (72), per (point, node) the basis stage (60)."""
    return nel * nq * (nn * (nn + 1) // 2 * 72 + nn * 60)


def stiffness_sf_flops(n, g, nel):
    """FP64 operations of k_u1_stiffness_sf per its loops (a multiply-add
    counts 2): the per-point geometry pass (nn sums of 16 values), then per
    pair i3 <= j3 of w indices the w, v and u contractions of the nine G_rs,
    and per written node pair the 3x3 block (about 40)."""
    n1, n2, n3 = n
    nn, nq = n1 * n2 * n3, g ** 3
    step1 = 9 * g ** 3 * 31
    step2 = 18 * n2 * g * (6 * g + 6 * n2 * g)
    step3 = 9 * n1 * n2 ** 2 * (6 * g + 4 * n1 * g)
    per_elem = (n3 * (n3 + 1) // 2 * (step1 + step2 + step3) + nn * (nn + 1) // 2 * 40 +
                nq * nn * 36)
    return nel * per_elem


def assembly_beyond_p2(device, seed):
    """U1 COO assembly of perturbed rational cubes of degree 3 and 4 with the
    pair kernel (bit-identical to the oracle) and the sum-factorised kernel,
    device times of the element kernels from the context's CUDA-event
    timers, and the oracle (OpenMP) on the same model."""
    import oracle
    from yeti_b200._lib import Context
    from yeti_b200.patches import cube_patch, u1_system_args
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    ctx = Context(device)
    out = {}
    for tag, nel, p in (("p3_16x16x16", (16, 16, 16), 3), ("p4_12x12x12", (12, 12, 12), 4)):
        args = u1_system_args(cube_patch(nel, p, perturb=0.1, wrange=(0.8, 1.2), seed=seed),
                              E=1.0, nu=0.3)
        nelt = nel[0] * nel[1] * nel[2]
        nn, g = (p + 1) ** 3, p + 1
        r = {"elements": nelt, "nb_data": int(args[1])}
        for kern, name in (("pairs", "k_u1_stiffness"), ("sumfact", "k_u1_stiffness_sf")):
            sys_linmat_lindef_static(*args, ctx=ctx, device_out=True, element_kernel=kern)
            ctx.set_timing(True)
            reps = 3
            for _ in range(reps):
                sys_linmat_lindef_static(*args, ctx=ctx, device_out=True, element_kernel=kern)
            r[f"{kern}_kernel_ms_events"] = ctx.kernel_ms(name) / reps
            ctx.set_timing(False)
        k_p = sys_linmat_lindef_static(*args, ctx=ctx)[0]
        k_s = sys_linmat_lindef_static(*args, ctx=ctx, element_kernel="sumfact")[0]
        t0 = time.perf_counter()
        k_o = oracle.sys_linmat_lindef_static(*args)[0]
        r["cpu_oracle_ms"] = (time.perf_counter() - t0) * 1e3
        r["cpu_cores"] = oracle.threads()
        r["pairs_bit_identical"] = bool(np.array_equal(k_p, k_o))
        r["sumfact_max_rel_diff_vs_oracle"] = float(np.abs(k_s - k_o).max() / np.abs(k_o).max())
        r["pairs_gflop"] = stiffness_flops(g ** 3, nn, nelt) / 1e9
        r["sumfact_gflop"] = stiffness_sf_flops((p + 1,) * 3, g, nelt) / 1e9
        r["sumfact_speedup_vs_pairs"] = r["pairs_kernel_ms_events"] / r["sumfact_kernel_ms_events"]
        # the COO output (value + row + col, 16 B a slot) is the HBM floor
        r["sumfact_hbm_gbs_output"] = int(args[1]) * 16 / (r["sumfact_kernel_ms_events"] / 1e3) / 1e9
        del k_p, k_s, k_o
        out[tag] = r
    ctx.close()
    return out


def gradient_flops(nq, nn, nel, nadj=1):
    """FP64 operations of k_u1_grad: per (point, control point, component)
    the interior-work derivative terms (dJ, the strain variation, dAAI, the
    81-term dAAE, the 36 dC products: about 1150 with one adjoint)."""
    return nel * nq * nn * 3 * 1150 * nadj


def extra_configs(args, device):
    """The other configurations of the path, each beside its CPU oracle:
    U1 Gauss assembly of the p=2 16x4x4 cantilever (COO), the compliance
    shape gradient of the p=2 32x32x2 quarter annulus, and the p=4
    128x128x32 WQ block (200 FP32 applies and a mixed solve)."""
    import torch
    import oracle
    from yeti_b200.gradient import grad_from_system_args, _solve
    from yeti_b200.patches import cube_patch
    from yeti_b200.stiffmtrx_elemstorage import sys_linmat_lindef_static
    from yeti_b200.wq import WQElasticity
    sync = torch.cuda.synchronize
    out = {}
    # C1: assembly (parity: bit-identical COO and F)
    a1 = _system_args("cantilever_p2_16x4x4")
    sys_linmat_lindef_static(*a1, device_out=True)
    t_gpu = _median_ms(lambda: sys_linmat_lindef_static(*a1, device_out=True), 20, sync)
    t_gpu_host, t_gpu_host_min = _median_ms(lambda: sys_linmat_lindef_static(*a1), 15, sync, True)
    kd, kr, kc, F = sys_linmat_lindef_static(*a1)
    t0 = time.perf_counter()
    ko, _, _, Fo = oracle.sys_linmat_lindef_static(*a1)
    t_cpu = (time.perf_counter() - t0) * 1e3
    # the whole C1 path: assembly, K = Kside + Kside^T, sparse direct solve of
    # the free dofs (scipy, on the host, as the reference does); displacement
    # against the same path on the oracle's COO
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    X1 = np.asarray(a1[2], dtype=np.float64)
    t_solve = _median_ms(lambda: _solve(a1, X1), 5, sync)
    U1, _ = _solve(a1, X1)
    n1 = Fo.size
    t0 = time.perf_counter()
    ko2, ro2, co2, Fo2 = oracle.sys_linmat_lindef_static(*a1)
    K1 = sp.coo_matrix((ko2, (ro2, co2)), shape=(n1, n1)).tocsc()
    K1 = K1 + K1.T
    idof1 = np.asarray(a1[26])[:int(a1[27])] - 1
    Uo = np.zeros(n1)
    Uo[idof1] = spla.spsolve(K1[idof1, :][:, idof1], Fo2[idof1])
    t_cpu_solve = (time.perf_counter() - t0) * 1e3
    peak64 = fp64_peak_tflops()
    t_ev = _event_ms(lambda: sys_linmat_lindef_static(*a1, device_out=True), 20)
    fl1 = stiffness_flops(27, 27, 256)
    from yeti_b200._lib import Context
    tctx = Context(device)
    tctx.set_timing(True)
    for _ in range(20):
        sys_linmat_lindef_static(*a1, device_out=True, ctx=tctx)
    t_k1 = tctx.kernel_ms("k_u1_stiffness") / 20
    tctx.set_timing(False)
    out["fp64_gemm_tflops_measured"] = peak64
    out["assembly_p2_16x4x4"] = {
        "nb_data": int(kd.size), "gpu_ms_device_out": t_gpu, "gpu_ms_host_buffers": t_gpu_host,
        "gpu_ms_host_buffers_min": t_gpu_host_min,
        "gpu_ms_events_device_out": t_ev, "k_u1_stiffness_ms_events": t_k1,
        "stiffness_gflop": fl1 / 1e9,
        "fp64_frac_of_measured_dgemm": fl1 / (t_k1 / 1e3) / 1e12 / peak64,
        "cpu_oracle_ms": t_cpu, "cpu_cores": oracle.threads(),
        "bit_identical": bool(np.array_equal(kd, ko) and np.array_equal(F, Fo)),
        "assemble_and_solve_ms": t_solve, "cpu_oracle_assemble_and_solve_ms": t_cpu_solve,
        "displacement_max_rel_diff_vs_oracle": float(np.abs(U1 - Uo).max() / np.abs(Uo).max()),
        "tip_min_uz": float(U1[2::3].min())}
    # consistent mass matrix of the same model (parity: bit-identical COO)
    from yeti_b200.massmtrx import build_cmassmatrix
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES as _SAN
    d1 = dict(zip(_SAN, a1))
    m_in = [d1["activeElement"], d1["nb_data"], np.asarray(d1["COORDS3D"], dtype=np.float64),
            d1["IEN"], d1["nb_elem_patch"], d1["Nkv"], d1["Ukv"], d1["Nijk"], d1["weight"],
            d1["Jpqr"], d1["ELT_TYPE"], d1["PROPS"], d1["JPROPS"], np.full(1, 7.85),
            d1["TENSOR"], d1["ind_dof_free"], d1["nb_dof_free"], d1["MCRD"], d1["NBINT"],
            d1["NNODE"]]
    build_cmassmatrix(*m_in, device_out=True)
    t_m = _median_ms(lambda: build_cmassmatrix(*m_in, device_out=True), 20, sync)
    md = build_cmassmatrix(*m_in)[0]
    t0 = time.perf_counter()
    mo = oracle.build_cmassmatrix(m_in)[0]
    t_mo = (time.perf_counter() - t0) * 1e3
    out["mass_matrix_p2_16x4x4"] = {"gpu_ms_device_out": t_m, "cpu_oracle_ms": t_mo,
                                    "cpu_cores": oracle.threads(), "bit_identical": bool(np.array_equal(md, mo))}

    asm = assembly_beyond_p2(device, WORKLOAD["seed"] + 7)
    for tag, r in asm.items():
        r["pairs_fp64_frac_of_measured_dgemm"] = (r["pairs_gflop"] / (r["pairs_kernel_ms_events"] / 1e3)
                                                  / 1e3 / peak64)
        r["sumfact_fp64_frac_of_measured_dgemm"] = (r["sumfact_gflop"] / (r["sumfact_kernel_ms_events"] / 1e3)
                                                    / 1e3 / peak64)
        out["assembly_" + tag] = r
    # C3: shape gradient (adjoint kernel; parity vs the CPU oracle)
    a3 = _system_args("quarter_annulus_p2_32x32x2")
    U, _ = _solve(a3, np.asarray(a3[2], dtype=np.float64))
    sol = U.reshape(-1, 3).T
    adj = 0.5 * sol[None]
    grad_from_system_args(a3, sol, adj)
    t_g, t_g_min = _median_ms(lambda: grad_from_system_args(a3, sol, adj), 15, sync, True)
    gi, ge = grad_from_system_args(a3, sol, adj)
    t_gev = _event_ms(lambda: grad_from_system_args(a3, sol, adj), 5)
    tctx.set_timing(True)
    for _ in range(5):
        grad_from_system_args(a3, sol, adj, ctx=tctx)
    t_k3 = tctx.kernel_ms("k_u1_grad") / 5
    tctx.set_timing(False)
    fl3 = gradient_flops(27, 27, 2048)
    t0 = time.perf_counter()
    oi, oe = oracle.grad_lin_elast_work(a3, sol, adj)
    t_go = (time.perf_counter() - t0) * 1e3
    ref = np.concatenate([oi.ravel(), oe.ravel()])
    got = np.concatenate([gi.ravel(), ge.ravel()])
    out["gradient_p2_32x32x2"] = {
        "nb_cp": int(sol.shape[1]), "gpu_ms_host_buffers": t_g, "gpu_ms_host_buffers_min": t_g_min,
        "gpu_ms_events": t_gev,
        "k_u1_grad_ms_events": t_k3, "gradient_gflop": fl3 / 1e9,
        "fp64_frac_of_measured_dgemm": fl3 / (t_k3 / 1e3) / 1e12 / peak64,
        "cpu_oracle_ms": t_go,
        "cpu_cores": oracle.threads(), "max_rel_diff_vs_oracle": float(np.abs(got - ref).max() / np.abs(ref).max())}
    # volume and its shape gradient on the C3 geometry (the constraint of the
    # shape optimisation beside the compliance)
    from yeti_b200.stiffmtrx_elemstorage import SYSTEM_ARG_NAMES
    from yeti_b200.volume import volume_and_gradient
    d3 = dict(zip(SYSTEM_ARG_NAMES, a3))
    A3 = [np.ones(np.atleast_1d(d3["nb_elem_patch"]).size, dtype=np.int64),
          np.asarray(d3["COORDS3D"], dtype=np.float64), d3["IEN"], d3["nb_elem_patch"],
          d3["Nkv"], d3["Ukv"], d3["Nijk"], d3["weight"], d3["Jpqr"], d3["ELT_TYPE"],
          d3["PROPS"], d3["JPROPS"], d3["TENSOR"], d3["MCRD"], d3["NBINT"], d3["NNODE"]]
    volume_and_gradient(A3)
    t_v, t_v_min = _median_ms(lambda: volume_and_gradient(A3), 15, sync, True)
    v_gpu, g_gpu = volume_and_gradient(A3)
    t0 = time.perf_counter()
    v_cpu, g_cpu = oracle.volume(A3)
    t_vo = (time.perf_counter() - t0) * 1e3
    out["volume_gradient_p2_32x32x2"] = {
        "volume": v_gpu, "gpu_ms_host_buffers": t_v, "gpu_ms_host_buffers_min": t_v_min,
        "cpu_oracle_ms": t_vo, "cpu_cores": oracle.threads(),
        "bit_identical": bool(v_gpu == v_cpu and np.array_equal(g_gpu, g_cpu))}
    # C5: p=4 128x128x32 WQ block
    P = cube_patch((128, 128, 32), 4, size=(4.0, 4.0, 1.0), perturb=0.1, wrange=(0.8, 1.2),
                   seed=WORKLOAD["seed"] + 5)
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1, 2)}, precisions="both")
    dev = torch.device("cuda", device)
    u32 = torch.randn(op.ndof, dtype=torch.float32, device=dev)
    k32 = torch.empty_like(u32)
    for _ in range(3):
        op.apply_device(u32, k32, "f32")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(200):
        op.apply_device(u32, k32, "f32")
    e1.record()
    sync()
    t_app = e0.elapsed_time(e1) / 200 / 1e3
    alg = op.nqp * 45 * 4 + 2 * op.ndof * 4
    peak, kind = measured_peaks()
    b = torch.from_numpy(op.eval_bodyforce_vector([0.0, 0.0, -1.0])).to(dev)
    xref, st_ref = op.pcg(b, rtol=1e-12, maxit=50000)
    sync()
    t0 = time.perf_counter()
    # rtol 1e-9, as on the 64^3 block: a 1e-8 residual leaves the error just
    # above the 1e-8 bar (1.04e-8 measured)
    x, st = op.pcg(b, rtol=1e-9, mixed=True, maxit=50000)
    sync()
    t_solve = time.perf_counter() - t0
    err = (torch.linalg.norm(x - xref) / torch.linalg.norm(xref)).item()
    op.pcg(b, rtol=1e-9, mixed=True, precond="fd")   # builds the plan
    sync()
    t0 = time.perf_counter()
    xf, stf = op.pcg(b, rtol=1e-9, mixed=True, precond="fd")
    sync()
    t_fd = time.perf_counter() - t0
    err_fd = (torch.linalg.norm(xf - xref) / torch.linalg.norm(xref)).item()
    out["wq_p4_128x128x32"] = {
        "ndof": op.ndof, "nqp": op.nqp, "rtol": 1e-9, "apply_f32_us": t_app * 1e6,
        "achieved_gbs": alg / t_app / 1e9, "peak_gbs": peak, "frac": alg / t_app / 1e9 / peak,
        "peak_kind": peak_kind_note(kind), "mixed_solve_s": t_solve,
        "iterations": st["iterations"], "rel_residual": st["rel_residual"],
        "rel_error_vs_fp64": err, "fp64_ref_rel_residual": st_ref["rel_residual"],
        "fd_mixed_solve_s": t_fd, "fd_iterations": stf["iterations"],
        "fd_rel_residual": stf["rel_residual"], "fd_rel_error_vs_fp64": err_fd}
    del op
    return out


def peak_kind_note(kind):
    return "of measured" if kind == "measured" else "of fallback"


# Iterations the FP64 Jacobi-PCG needs on the default workload to rtol 1e-9:
# the count of this bench's own FP64 leg on a B200 (the same operator and
# recurrence the CPU port runs; the CPU arithmetic differs only in rounding).
# The reference arm, which cannot run a full CPU solve (about 950 iterations
# of a quarter second) within its time limit, scales its timed iterations by
# it; the main arm's CPU baseline uses the count measured in the same run.
ITERS_FP64_DEFAULT = 952
ITERS_SOURCE = ("the FP64 Jacobi-PCG iteration count of this workload, measured by "
                "this bench's FP64 leg on a B200")


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    from yeti_b200 import _lib
    from yeti_b200.patches import cube_patch
    from yeti_b200.wq import WQElasticity

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = _lib.default_context(local)
    ctx.set_stream(torch.cuda.current_stream(dev))
    L = _lib.lib()
    if args.only_extra:
        if rank == 0:
            print(json.dumps({"other_configs": extra_configs(args, local)}), flush=True)
        return 0
    seed = replica_seed(rank)
    P = cube_patch(tuple(args.nel), args.p, perturb=0.2, wrange=(0.8, 1.2), seed=seed)
    t0 = time.perf_counter()
    op = WQElasticity(P, 1.0, 0.3, {"w0": (0, 1, 2)}, precisions="both", ctx=ctx)
    setup_s = time.perf_counter() - t0
    b_host = op.eval_bodyforce_vector([0.0, 0.0, -1.0])
    b = torch.from_numpy(b_host).to(dev)

    # roofline of the dominant kernel: the FP32 operator apply
    # (first kernels after the setup, so that a profiler can capture one
    # apply with only setup launches before it)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    u32 = torch.randn(op.ndof, dtype=torch.float32, device=dev)
    k32 = torch.empty_like(u32)
    for _ in range(5):
        op.apply_device(u32, k32, "f32")
    torch.cuda.synchronize()
    napp = 30
    e0.record()
    for _ in range(napp):
        op.apply_device(u32, k32, "f32")
    e1.record()
    torch.cuda.synchronize()
    t_app = e0.elapsed_time(e1) / napp / 1e3
    alg_bytes = op.nqp * 45 * 4 + 2 * op.ndof * 4
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / t_app / 1e9
    u64 = u32.double()
    k64 = torch.empty_like(u64)
    op.apply_device(u64, k64, "f64")
    e0.record()
    for _ in range(10):
        op.apply_device(u64, k64, "f64")
    e1.record()
    torch.cuda.synchronize()
    t_app64 = e0.elapsed_time(e1) / 10 / 1e3


    # FP64 reference solution (untimed, tight) and the plain FP64 solve
    xref, st_ref = op.pcg(b, rtol=1e-12)
    torch.cuda.synchronize()
    x64, st64 = op.pcg(b, rtol=args.rtol)
    err64 = (torch.linalg.norm(x64 - xref) / torch.linalg.norm(xref)).item()

    def step():
        x, st = op.pcg(b, rtol=args.rtol, mixed=True)
        return x, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(ws)
    clocks = ClockSampler(local)
    clocks.start()
    l0 = L.yeti_kernel_launches()
    torch.cuda.synchronize()
    e0.record()
    stats = []
    torch.cuda.nvtx.range_push("timed_mixed_solves")
    for _ in range(args.steps):
        x, st = step()
        stats.append(st)
    torch.cuda.nvtx.range_pop()
    e1.record()
    torch.cuda.synchronize()
    launches = L.yeti_kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(ms, ws)
    barrier(ws)
    err = (torch.linalg.norm(x - xref) / torch.linalg.norm(xref)).item()
    value = aggregate_rate(op.nfree, ms, ws, args.steps)

    # plain FP64 throughput for the same tolerance (device-resident)
    e0.record()
    for _ in range(max(1, args.steps)):
        op.pcg(b, rtol=args.rtol)
    e1.record()
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1) / max(1, args.steps)

    # the same solves with the fast-diagonalisation preconditioner (the
    # reference's FD branch of wq_mf_cg_3d, 'JM'), device-resident
    fd = {}
    for mixed in (False, True):
        op.pcg(b, rtol=args.rtol, mixed=mixed, precond="fd")   # builds the plan
        torch.cuda.synchronize()
        # each solve timed alone, the median kept: one host stall between
        # two calls on a shared machine would otherwise double a 17 ms mean
        tf = []
        for _ in range(max(3, args.steps)):
            e0.record()
            xf, stf = op.pcg(b, rtol=args.rtol, mixed=mixed, precond="fd")
            e1.record()
            torch.cuda.synchronize()
            tf.append(e0.elapsed_time(e1))
        msf = float(np.median(tf))
        fd["mixed" if mixed else "fp64"] = {
            "value": ws * op.nfree / (msf / 1e3), "ms_per_step": msf,
            "iterations": stf["iterations"], "outer_iterations": stf["outer_iterations"],
            "solve_ms_device": stf["solve_ms"], "rel_residual": stf["rel_residual"],
            "rel_error_vs_fp64_ref": (torch.linalg.norm(xf - xref) / torch.linalg.norm(xref)).item()}
    fd["mixed_over_jacobi_mixed"] = fd["mixed"]["value"] / value
    fd["preconditioner"] = ("fast diagonalisation per displacement component, a[c][d] = mean "
                            "coefficient diagonal ('JM'); FP32 in the mixed solve")

    # end to end through the public API with pinned host buffers
    bh = torch.empty(op.ndof, dtype=torch.float64, pin_memory=True)
    bh.copy_(torch.from_numpy(b_host))
    bh_np = bh.numpy()
    torch.cuda.synchronize()
    e0.record()
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        xh, _ = op.pcg(bh_np, rtol=args.rtol, mixed=True)
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), ws)
    wall_e2e = time.perf_counter() - t_wall

    serve = None
    if not args.no_serve and args.serve_requests > 0:
        serve = serve_stream(args, local)
        if args.serve_rate_high > 0:
            serve["high_rate"] = serve_stream(args, local, args.serve_rate_high)
        if args.serve_rate_capacity > 0:
            serve["capacity_rate"] = serve_stream(args, local, args.serve_rate_capacity)
    extra = None
    if rank == 0 and ws == 1 and not args.no_extra:
        extra = extra_configs(args, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_rate(args, st64["iterations"],
                                     "the FP64 Jacobi-PCG iterations of this run's FP64 leg")
        except Exception as exc:  # report, do not hide
            cpu = {"value": None, "error": repr(exc)[:200]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "precision": "FP32 operator + inner PCG, FP64 residual and refinement",
            "data": "synthetic",
            "config": dict(WORKLOAD, nel=args.nel, p=args.p, rtol=args.rtol,
                           parallelism=f"replicas x{ws}", ndof=op.ndof,
                           nfree=op.nfree, nqp=op.nqp),
            "solve": {"iterations": stats[-1]["iterations"],
                      "outer_iterations": stats[-1]["outer_iterations"],
                      "fp64_applies": stats[-1]["fp64_applies"],
                      "rel_residual": stats[-1]["rel_residual"],
                      "rel_residual_inf": stats[-1]["rel_residual_inf"],
                      "rel_error_vs_fp64_ref": err,
                      "ref_rel_residual": st_ref["rel_residual"]},
            "fp64": {"value": ws * op.nfree / (ms64 / 1e3), "ms_per_step": ms64,
                     "iterations": st64["iterations"], "rel_error_vs_fp64_ref": err64},
            "mixed_over_fp64": (value / ws) / (op.nfree / (ms64 / 1e3)),
            "fd_pcg": fd,
            "setup_s": setup_s,
            "e2e": {"value": ws * op.nfree * args.steps / (ms_e2e / 1e3), "unit": "DOF/s",
                    "h2d_bytes_per_step": 2 * op.ndof * 8,
                    "d2h_bytes_per_step": op.ndof * 8,
                    "wall_s": wall_e2e},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": f"k_wq_apply_stream<float,{args.p}>",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (profiled_traffic("k_wq_apply_stream_f32_p3_64cube.txt")
                                     if list(args.nel) == [64, 64, 64] and args.p == 3 else None),
                         "alg_bytes_per_launch": alg_bytes,
                         "apply_us": t_app * 1e6, "apply_f64_us": t_app64 * 1e6,
                         "f64_frac": (op.nqp * 45 * 8 + 2 * op.ndof * 8) / t_app64 / 1e9 / peak},
            "cpu_baseline": cpu,
            "clocks": clk,
            "serve": serve,
            "other_configs": extra,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
