"""Benchmark of the fused element loop (Gauss-point update + f_int + K assembly).

Workload: the viscoelastic scale-up configuration -- unit cube, 64x64x64 Hexa8 (262,144
elements, 2,097,152 Gauss points), interior nodes jittered +-5% (seed 0), Neo-Hookean ground
state (mu = 1, K = 100) with 3 generalized-Maxwell branches (beta = 0.3, 0.2, 0.1;
tau = 0.01, 0.1, 1 s), FP32 Gauss-point state with FP64 det F / ln J and FP64 K / f_int
(CEOS_MIXED), cyclic simple shear of amplitude 0.3 at 1 Hz with dt = 0.025 s.  One step = one
Newton evaluation of the whole mesh through the C ABI (the work the reference does in
SolveConstitutiveModel + InternalForce + TangentStiffnessMatrix per iteration).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload fe2-surrogate [--n-train 200000] [--epochs 2000]
  python bench.py --workload fe2-batch [--n-rve 4096]
  python bench.py --workload j2-plate

The second form runs the learned-surrogate experiment instead (training data from the batched
RVE solver, training, validation error, a 4^3 macro head-to-head of surrogate and direct FE^2,
and the 32^3 surrogate macro run) and prints its own JSON record.

--impl reference times the reference's CPU element loop: the Fortran is not buildable here
(no Fortran compiler, no MKL), so its FP64 C++ restatement (oracle/) runs on all host cores
on a bounded slab of the same mesh.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ceos-eems_b200"))

NX = 64
PRONY = [1.0, 100.0, 3, 0.3, 0.01, 0.2, 0.1, 0.1, 1.0, 0.0, 1.0]
DT = 0.025
WORKLOAD = "visco-Prony 64^3 Hexa8 (262144 elements, 2097152 GPs), cyclic simple shear"
METRIC = "GP updates/s"
UNIT = "GP updates/s"


def shear_u(X, t):
    gamma = 0.3 * np.sin(2.0 * np.pi * t)
    U = np.zeros_like(X)
    U[:, 0] = gamma * X[:, 2]
    return U.reshape(-1)


def cpu_slab(X, conn, nz_layers):
    """The first nz_layers element layers of the mesh with nodes renumbered compactly."""
    nx = round((conn.shape[0]) ** (1.0 / 3.0))
    ne = nx * nx * nz_layers
    c = conn[:ne]
    used = np.unique(c)
    newid = np.zeros(X.shape[0] + 1, np.int64)
    newid[used] = np.arange(1, used.size + 1)
    return X[used - 1], newid[c].astype(np.int32)


def run_cpu_sample(X, conn, threads, nz_layers=4, reps=1):
    """Time the oracle (reference CPU element loop restated in FP64 C++) on a slab."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    Xs, cs = cpu_slab(X, conn, nz_layers)
    m = O.Model(Xs, cs, [O.VISCO_PRONY], PRONY)
    U = shear_u(Xs, 2 * DT)
    m.evaluate_sample(DT, shear_u(Xs, DT), cs.shape[0], threads)  # one increment of history
    m.commit()
    m.set_time_old(DT)
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        m.evaluate_sample(2 * DT, U, cs.shape[0], threads)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    n_gp = 8 * cs.shape[0]
    return n_gp / best, n_gp, best, m


def run_cpu_single(X, conn, nz_layers=4):
    """The oracle's element loop on one thread (the reference's serial loop) over the first nz_layers
    element layers, after one committed increment; returns (GP updates/s, GPs, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    Xs, cs = cpu_slab(X, conn, nz_layers)
    m = O.Model(Xs, cs, [O.VISCO_PRONY], PRONY)
    m.evaluate_sample(DT, shear_u(Xs, DT), cs.shape[0], 1)
    m.commit()
    m.set_time_old(DT)
    t0 = time.perf_counter()
    m.evaluate_sample(2 * DT, shear_u(Xs, 2 * DT), cs.shape[0], 1)
    secs = time.perf_counter() - t0
    n_gp = 8 * cs.shape[0]
    return n_gp / secs, n_gp, secs


def clocks_sampler_start(path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except OSError:
        return None


def clocks_summary(path, dev):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for ln in open(path):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9 or not f[0].isdigit() or int(f[0]) != dev:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
    except OSError:
        pass
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def max_over_ranks(x, world, device):
    """The largest x over all ranks (the job is as slow as its slowest rank); x itself when world == 1.
    device: where the reduction tensor lives ("cuda:k" under NCCL, "cpu" under gloo)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds):
    """Aggregate throughput of N replicas that each processed units_per_rank in the max-over-ranks time."""
    return world * units_per_rank / seconds


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the element kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "element_loop_visco_prony_64cube.json")
    try:
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except Exception:
        return None


def algorithmic_bytes(n_nodes, n_elem, n_gp, n_dof, nnz, nb=3):
    nodes = 48 * n_nodes                  # X + U, FP64
    connectivity = 32 * n_elem            # 8 int32 node ids
    state = n_gp * (6 + 6 * nb) * 4 * 2   # FP32 state read + write
    fint = 8 * n_dof
    kval = 8 * nnz
    return nodes + connectivity + state + fint + kval


def run_j2_plate(args):
    """Finite-strain J2 plate: 96 x 96 x 48 Hexa8 (442,368 elements, 3.54 M Gauss points), jitter 5 %,
    E = 200 GPa, nu = 0.3, sigma_y0 = 250 MPa, H = 1 GPa with E and sigma_y scaled per element by a
    log-uniform factor in [0.9, 1.1]; uniaxial tension along x with lateral contraction, evaluated at
    2.5 % strain from the committed state of 1.25 % (every point plastic).  One step = one evaluation
    (return mapping, f_int, K) in mixed precision; GP updates/s, device-resident."""
    import torch
    import ceos_b200 as G
    from ceos_b200 import meshgen
    nx, ny, nz = 96, 96, 48
    X, conn = meshgen.structured_box(nx, ny, nz, lx=2.0, ly=2.0, lz=1.0, jitter=0.05, seed=0)
    rng = np.random.default_rng(3)
    ne = conn.shape[0]
    fac = np.exp(rng.uniform(np.log(0.9), np.log(1.1), (ne, 2)))
    params = np.zeros((ne, 4))
    params[:, 0] = 200e3 * fac[:, 0]   # MPa
    params[:, 1] = 0.3
    params[:, 2] = 250.0 * fac[:, 1]
    params[:, 3] = 1e3
    g = G.ElementLoop(X, conn, G.J2_FINITE, params, per_element=True, precision=G.MIXED)

    def U_at(eps):
        U = np.zeros_like(X)
        U[:, 0] = eps * X[:, 0]
        U[:, 1] = -0.5 * eps * X[:, 1]
        U[:, 2] = -0.5 * eps * X[:, 2]
        return U.reshape(-1)
    _, _, rc, _ = g.evaluate(0.0, U_at(0.0125), tangent=False)
    assert rc == 0, rc
    g.commit()
    dU = torch.tensor(U_at(0.025), dtype=torch.float64, device="cuda")
    dfint = torch.zeros(g.n_dof, dtype=torch.float64, device="cuda")
    dK = torch.zeros(g.nnz, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            g.evaluate_device(0.0, dU, dfint, dK, stream=sp)
    torch.cuda.synchronize()
    assert g.status()[0] == 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        g.evaluate_device(0.0, dU, dfint, dK, stream=sp)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    g.set_options(G.OPT_TIME_KERNELS)
    g.evaluate_device(0.0, dU, dfint, dK, stream=sp)
    k_ms, c_ms = g.kernel_time_ms()
    g.set_options(0)
    st = g.state(1)
    n_gp = 8 * ne
    alg = 48 * g.n_nodes + 32 * ne + 16 * ne + n_gp * 7 * 4 * 2 + 8 * g.n_dof + 8 * g.nnz
    peak, kind = measured_peak_hbm()
    rec = {"metric": "GP updates/s", "value": n_gp / (ms * 1e-3), "unit": "GP updates/s", "higher_is_better": True,
           "n_gpus": 1, "steps": args.steps, "ms_per_step": ms, "dtype": "f32+f64", "data": "synthetic",
           "plastic_points": int((st[:, :, 6] > 0).sum()), "gauss_points": n_gp,
           "roofline": {"bound": "hbm", "achieved": alg / (k_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (k_ms * 1e-3) / 1e9 / peak, "peak_kind": kind, "kernel_ms": k_ms,
                        "conversion_kernel_ms": c_ms, "algorithmic_bytes_per_launch": alg},
           "config": {"workload": "finite-strain J2 plate 96x96x48 Hexa8 (442,368 elements, 3.54 M GPs), per-element "
                                  "E and sigma_y x U_log[0.9,1.1], uniaxial tension at 2.5 % from 1.25 % committed"}}
    print(json.dumps(rec), flush=True)


def run_fe2_batch(args):
    """Batched FE^2: n_rve periodic fibre RVEs of uneven size n in {6..12}, vf U[0.1, 0.4], F = I + G
    with |G_ij| <= 0.15, solved to 1e-8 with homogenized P and the 9x9 tangent, one batch on the GPU."""
    import torch
    from ceos_b200 import fe2
    n, vf = fe2.sample_rve_family(args.n_rve, seed=4)
    Fb = fe2.sample_macro_F(args.n_rve, seed=5)
    t0 = time.perf_counter()
    b = fe2.BatchedRVE(n, vf)
    t_create = time.perf_counter() - t0
    b.set_allow_failures(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = b.solve(Fb, tangent=True)
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t0
    ok = ~out["failed"]
    rec = {"metric": "RVE solves/s (P and 9x9 tangent)", "value": float(args.n_rve / t_solve), "unit": "RVE/s",
           "higher_is_better": True, "n_gpus": 1, "dtype": "f64 element loop / f32 MINRES with f64 refinement",
           "data": "synthetic", "solve_s": t_solve, "setup_s": t_create, "failed_rves": int((~ok).sum()),
           "newton_iters_mean": float(out["newton_iters"][ok].mean()), "newton_iters_max": int(out["newton_iters"].max()),
           "minres_iters_mean": float(out["cg_iters"][ok].mean()),
           "elements": int(b.n_elem), "reduced_dofs": int(b.n_red),
           "config": {"workload": f"batched FE2: {args.n_rve} periodic fibre RVEs, n U{{6..12}}, vf U[0.1,0.4], "
                                  "mu_f/mu_m=50, K/mu=100, F = I + G, |G_ij| <= 0.15, tol 1e-8, P + tangent"}}
    print(json.dumps(rec), flush=True)
    b.close()


def run_fe2_surrogate(args):
    """Learned surrogate against direct batched FE^2 (all on the GPU, no oracle)."""
    from ceos_b200 import fe2_surrogate as FS
    rec = {"metric": "FE2 macro step time: surrogate vs direct", "unit": "s", "higher_is_better": False,
           "dtype": "bf16 training / f32 inference / f64 RVE", "data": "synthetic"}
    F, vf = FS.sample_points(args.n_train, seed=1, small_fraction=0.5)
    P, _, st = FS.rve_stresses(F, vf, batch=8192)
    Fv, vfv = FS.sample_points(4096, seed=99)
    Pv, _, _ = FS.rve_stresses(Fv, vfv, batch=4096)
    Ft, vft = FS.sample_points(8192, seed=7)
    _, _, st_tan = FS.rve_stresses(Ft, vft, batch=8192, tangent=True)
    sur, hist, t_train = FS.fit(F, vf, P, epochs=args.epochs, batch=2048, lr0=3e-3, lr1=3e-6)
    Pp, fl = FS.predict_P(sur, Fv, vfv)
    rec["training"] = {"samples": int(args.n_train), "rve_n_cells": 6, "data_s": st["seconds"],
                       "rve_per_s": st["rve_per_s"], "rve_per_s_with_tangent": st_tan["rve_per_s"],
                       "failed_rves": st["failed"], "epochs": args.epochs, "batch": 2048,
                       "adam_steps": args.epochs * (args.n_train // 2048), "train_s": t_train,
                       "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1])}
    rec["validation_stress_error"] = FS.stress_errors(Pp[~fl], Pv[~fl])
    rec["validation_out_of_range"] = int(fl.sum())
    print(json.dumps({"partial": "training", "training": rec["training"],
                      "validation": rec["validation_stress_error"]}), file=sys.stderr, flush=True)
    small = FS.macro_compare(sur, nx=4)
    rec["macro_4cube"] = {k: small[k] for k in ("direct", "surrogate", "stress_error_per_step",
                                                "constitutive_error_per_step")}
    rec["speedup_4cube_in_range_steps"] = [d / s for d, s, fb in zip(small["direct"]["step_s"], small["surrogate"]["step_s"],
                                                                    small["surrogate"]["fallback_points"]) if fb == 0]
    print(json.dumps({"partial": "4cube", "macro_4cube": rec["macro_4cube"],
                      "speedup": rec["speedup_4cube_in_range_steps"]}), file=sys.stderr, flush=True)
    big = FS.macro_surrogate_run(sur, nx=32)
    evals = np.array(big["newton"]) + 1  # material evaluations per step
    st_b = big["stats"]
    other = (st_b["loop_s"] + st_b["solve_s"]) / max(1, len(big["newton"]))
    direct_est = evals * (big["n_gp"] / st_tan["rve_per_s"]) + other
    rec["macro_32cube"] = {"surrogate": {k: big[k] for k in ("step_s", "newton", "fallback_points", "stopped")},
                           "surrogate_stats": st_b,
                           "direct_step_s_estimated": direct_est.tolist(),
                           "direct_estimate": "material evaluations per step x 262,144 RVE solves (with tangent) at "
                                              "the measured batched throughput, plus the surrogate run's element-loop "
                                              "and solve time per step"}
    s32 = np.array(big["step_s"])
    rec["value"] = float(s32.mean()) if s32.size else None
    rec["speedup_32cube_estimated"] = float(np.mean(direct_est / s32)) if s32.size else None

    rec["config"] = {"workload": "FE2 uniaxial stretch to 1.2 in 10 increments; macro 32^3 Hexa8 (262,144 GPs) and "
                                 "4^3 head-to-head; periodic fibre RVEs n=6, vf U[0.1,0.4], mu_f/mu_m=50, K/mu=100",
                     "surrogate": "MLP 7-128x4-1 softplus energy of (C, vf)"}
    print(json.dumps(rec), flush=True)
    sur.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="element-loop",
                    choices=["element-loop", "fe2-surrogate", "fe2-batch", "j2-plate"])
    ap.add_argument("--n-rve", type=int, default=4096)
    ap.add_argument("--n-train", type=int, default=200000)
    ap.add_argument("--epochs", type=int, default=2000)
    args = ap.parse_args()
    if args.workload == "fe2-surrogate":
        return run_fe2_surrogate(args)
    if args.workload == "fe2-batch":
        return run_fe2_batch(args)
    if args.workload == "j2-plate":
        return run_j2_plate(args)
    warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from ceos_b200 import meshgen
    X, conn = meshgen.structured_box(args.nx, args.nx, args.nx, jitter=0.05, seed=0)
    n_elem, n_gp = conn.shape[0], 8 * conn.shape[0]
    workload = WORKLOAD if args.nx == 64 else (f"visco-Prony {args.nx}^3 Hexa8 ({int(n_elem)} elements, "
                                               f"{int(n_gp)} GPs), cyclic simple shear")
    config = {"workload": workload, "mesh": f"{args.nx}^3 Hexa8", "elements": int(n_elem), "gauss_points": int(n_gp),
              "material": "Neo-Hookean mu=1 K=100 + 3 Maxwell branches (0.3,0.01s),(0.2,0.1s),(0.1,1s)",
              "precision": "FP32 element arithmetic/state, FP64 detF/lnJ/K/f_int",
              "l2": "inputs larger than L2 (K 262 MB + state 403 MB per step)", "parallelism": f"replicas x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        reps = max(1, min(args.steps, 3))
        rate, n_sample, secs, _ = run_cpu_sample(X, conn, threads, nz_layers=args.nx, reps=reps)
        sample = f"whole mesh ({n_sample // 8} elements, {n_sample} GPs) per step, FP64, best of {reps}"
        r1, g1, s1 = run_cpu_single(X, conn, nz_layers=min(4, args.nx))
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": warmup, "ms_per_step": secs * 1e3 * n_gp / n_sample,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                                 "single_thread": {"value": r1, "unit": UNIT, "cores": 1,
                                                   "sample": f"{g1 // 8} elements (first element layers), "
                                                             f"serial loop, {s1:.2f} s"}},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "reference Fortran not buildable (no Fortran compiler/MKL); FP64 C++ restatement of its "
                        "serial element loop with linear-search assembly, OpenMP over element colours"}
        print(json.dumps(line))
        return

    import torch
    import ceos_b200 as G
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = local_rank
    torch.cuda.set_device(dev)

    g = G.ElementLoop(X, conn, G.VISCO_PRONY, PRONY, precision=G.MIXED, device=dev)
    n_dof, nnz = g.n_dof, g.nnz
    # two committed increments of cyclic shear give the Maxwell branches a non-trivial history
    for k in (1, 2):
        t = k * DT
        _, _, rc, _ = g.evaluate(t, shear_u(X, t), tangent=False)
        assert rc == 0, rc
        g.commit()
    t_eval = 3 * DT
    U_host = shear_u(X, t_eval)
    dU = torch.tensor(U_host, dtype=torch.float64, device=f"cuda:{dev}")
    dfint = torch.zeros(n_dof, dtype=torch.float64, device=f"cuda:{dev}")
    dK = torch.zeros(nnz, dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    def step():
        g.evaluate_device(t_eval, dU, dfint, dK, stream=sp)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step()
    torch.cuda.synchronize()
    rc, nf = g.status()
    assert rc == 0, ("element failures", rc, nf)

    clk_path = os.path.join(os.environ.get("CEOS_BENCH_CLOCKS_DIR", tempfile.gettempdir()),
                            f"ceos_bench_clocks_r{rank}_{os.getpid()}.csv")
    os.makedirs(os.path.dirname(clk_path), exist_ok=True)
    sampler = clocks_sampler_start(clk_path)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, f"cuda:{dev}")
    # kernel-only durations for the roofline (events around the element-loop launch)
    g.set_options(G.OPT_TIME_KERNELS)
    kms, cms = [], []
    for _ in range(max(5, min(args.steps, 20))):
        g.evaluate_device(t_eval, dU, dfint, dK, stream=sp)
        k_ms, c_ms = g.kernel_time_ms()
        kms.append(k_ms)
        cms.append(c_ms)
    g.set_options(0)
    if sampler:
        sampler.terminate()
        sampler.wait()
    clocks = clocks_summary(clk_path, dev)

    # end to end through the C ABI with pinned host buffers: H2D of U, D2H of f_int and K
    U_pin = torch.from_numpy(U_host).pin_memory()
    f_pin = torch.zeros(n_dof, dtype=torch.float64).pin_memory()
    K_pin = torch.zeros(nnz, dtype=torch.float64).pin_memory()
    lib = G.lib()
    import ctypes as C
    nfail = C.c_int(0)

    def e2e_step():
        return lib.ceos_evaluate(g.handle, t_eval, C.c_void_p(U_pin.data_ptr()), C.c_void_p(f_pin.data_ptr()),
                                 C.c_void_p(K_pin.data_ptr()), C.byref(nfail))

    for _ in range(2):
        assert e2e_step() == 0
    e2e_steps = max(3, min(args.steps, 10))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, world, f"cuda:{dev}")
    # sanity: the device result equals the host result (up to the summation order of the atomics)
    assert torch.allclose(dfint.cpu(), f_pin, rtol=1e-10, atol=1e-12 * float(f_pin.abs().max()))

    ms_step = ms / args.steps
    value = whole_job_rate(n_gp * args.steps, world, ms * 1e-3)
    alg = algorithmic_bytes(g.n_nodes, n_elem, n_gp, n_dof, nnz)
    kmean = float(np.mean(kms)) * 1e-3
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / kmean / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic", "config": config,
            "e2e": {"value": whole_job_rate(n_gp, world, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 8 * n_dof,
                    "d2h_bytes_per_step": 8 * (n_dof + nnz)},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(), "peak_kind": peak_kind,
                         "kernel": "element_loop_kernel<float,101,1>", "kernel_ms": kmean * 1e3,
                         "conversion_kernel_ms": float(np.mean(cms)),
                         "algorithmic_bytes_per_launch": alg},
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, n_sample, secs, m = run_cpu_sample(X, conn, threads, nz_layers=args.nx)
        r1, g1, s1 = run_cpu_single(X, conn, nz_layers=min(4, args.nx))
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"one evaluation of the whole mesh ({n_sample // 8} elements), FP64 "
                                          f"oracle on {threads} threads, {secs:.2f} s",
                                "single_thread": {"value": r1, "unit": UNIT, "cores": 1,
                                                  "sample": f"{g1 // 8} elements (first element layers), "
                                                            f"serial loop, {s1:.2f} s"}}
        # error of the measured evaluation against the FP64 oracle at the same state: the oracle has
        # the same history (increments at DT and 2 DT committed) and evaluates the timed U at 3 DT
        m.commit()
        m.set_time_old(2 * DT)
        f_o, k_o, rc_o, _ = m.evaluate(t_eval, U_host)
        if rc_o == 0:
            f_g, k_g = f_pin.numpy(), K_pin.numpy()
            line["error_vs_fp64_oracle"] = {
                "f_int_rel": float(np.abs(f_g - f_o).max() / np.abs(f_o).max()),
                "K_rel": float(np.abs(k_g - k_o).max() / np.abs(k_o).max()),
                "K_rel_fro": float(np.linalg.norm(k_g - k_o) / np.linalg.norm(k_o)),
                "what": "max |GPU - oracle| / max |oracle| over all f_int and K entries of the timed evaluation "
                        f"(mixed precision GPU vs FP64 oracle, {args.nx}^3 mesh, same Gauss-point history)"}
    if rank == 0:
        print(json.dumps(line))
    g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
