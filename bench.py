"""Benchmark of the fused element loop (Gauss-point update + f_int + K assembly).

Default workload (one step = one Newton evaluation of the whole mesh through the C ABI: the work
the reference does in SolveConstitutiveModel + InternalForce + TangentStiffnessMatrix per
iteration): the finite-strain J2 plate -- 96 x 96 x 48 Hexa8 (442,368 elements, 3,538,944
Gauss points) on [0,2]x[0,2]x[0,1], interior nodes jittered +-5 % (seed 0), E = 200 GPa,
nu = 0.3, sigma_y0 = 250 MPa, H = 1 GPa with E and sigma_y0 scaled per element by a log-uniform
factor in [0.9, 1.1] (seed 3), multiplicative J2 with FP32 element arithmetic and state and FP64
det F / ln J / return-mapping scalar / K / f_int (CEOS_MIXED); uniaxial tension along x with
lateral contraction, evaluated at 2.5 % strain from the committed state of 1.25 % (every point
plastic), i.e. one Newton evaluation in the middle of the 50-increment load to 5 %.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload visco          # 64^3 visco-Prony cyclic shear
  python bench.py --workload fe2-batch [--n-rve 4096]
  python bench.py --workload fe2-surrogate [--n-train 200000] [--epochs 2000]

--impl reference times the reference's CPU element loop: the Fortran is not buildable here (no
Fortran compiler, no MKL), so its FP64 C++ restatement (oracle/) runs on all host cores, every
step a bounded slab of the same mesh.
"""
import argparse
import ctypes as C
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

METRIC = "GP updates/s"
UNIT = "GP updates/s"
PRONY = [1.0, 100.0, 3, 0.3, 0.01, 0.2, 0.1, 0.1, 1.0, 0.0, 1.0]
DT = 0.025
MODEL_J2_FINITE, MODEL_VISCO_PRONY = 102, 101


# ---------------------------------------------------------------------------------------------
# Workloads: mesh, material, load history and algorithmic bytes of one evaluation
# ---------------------------------------------------------------------------------------------
class Workload:
    """One element-loop configuration.  history: committed (time, U) evaluations before the timed
    one; (t_eval, U_eval) the evaluation every step repeats."""

    def __init__(self, name, nx):
        from ceos_b200 import meshgen
        self.name = name
        if name == "j2-plate":
            self.nx, self.ny, self.nz = nx, nx, max(1, nx // 2)
            self.X, self.conn = meshgen.structured_box(self.nx, self.ny, self.nz, lx=2.0, ly=2.0, lz=1.0,
                                                       jitter=0.05, seed=0)
            ne = self.conn.shape[0]
            rng = np.random.default_rng(3)
            fac = np.exp(rng.uniform(np.log(0.9), np.log(1.1), (ne, 2)))
            P = np.zeros((ne, 4))
            P[:, 0] = 200e3 * fac[:, 0]   # MPa
            P[:, 1] = 0.3
            P[:, 2] = 250.0 * fac[:, 1]
            P[:, 3] = 1e3
            self.model, self.params, self.per_element = MODEL_J2_FINITE, P, True
            self.history = [(1.0, self.tension(0.0125))]
            self.t_eval, self.U_eval = 2.0, self.tension(0.025)
            self.label = (f"finite-strain J2 plate {self.nx}x{self.ny}x{self.nz} Hexa8 ({ne} elements, {8 * ne} GPs), "
                          "per-element E and sigma_y x U_log[0.9,1.1], uniaxial tension at 2.5 % from 1.25 % committed")
            self.material = "multiplicative J2: E=200 GPa (x per element), nu=0.3, sigma_y0=250 MPa (x per element), H=1 GPa"
            self.state_bytes_per_gp = 7 * 4 * 2      # Cp^-1 (6) + alpha, FP32, read + write
            self.param_bytes_per_elem = 4 * 4        # E, nu, sigma_y0, H (FP32) per element
        elif name == "visco":
            self.nx = self.ny = self.nz = nx
            self.X, self.conn = meshgen.structured_box(nx, nx, nx, jitter=0.05, seed=0)
            ne = self.conn.shape[0]
            self.model, self.params, self.per_element = MODEL_VISCO_PRONY, PRONY, False
            self.history = [(k * DT, self.shear(k * DT)) for k in (1, 2)]
            self.t_eval, self.U_eval = 3 * DT, self.shear(3 * DT)
            self.label = f"visco-Prony {nx}^3 Hexa8 ({ne} elements, {8 * ne} GPs), cyclic simple shear"
            self.material = "Neo-Hookean mu=1 K=100 + 3 Maxwell branches (0.3,0.01s),(0.2,0.1s),(0.1,1s)"
            self.state_bytes_per_gp = (6 + 6 * 3) * 4 * 2
            self.param_bytes_per_elem = 0
        else:
            raise ValueError(name)
        self.n_elem = self.conn.shape[0]
        self.n_gp = 8 * self.n_elem

    def tension(self, eps):
        U = np.zeros_like(self.X)
        U[:, 0] = eps * self.X[:, 0]
        U[:, 1] = -0.5 * eps * self.X[:, 1]
        U[:, 2] = -0.5 * eps * self.X[:, 2]
        return U.reshape(-1)

    def shear(self, t):
        U = np.zeros_like(self.X)
        U[:, 0] = 0.3 * np.sin(2.0 * np.pi * t) * self.X[:, 2]
        return U.reshape(-1)

    def algorithmic_bytes(self, n_nodes, n_dof, nnz):
        """Each input read once, each output written once: nodes (X + U, FP64), connectivity (8 int32),
        per-element properties, Gauss-point state read + write, f_int and K values (FP64)."""
        return (48 * n_nodes + 32 * self.n_elem + self.param_bytes_per_elem * self.n_elem
                + self.state_bytes_per_gp * self.n_gp + 8 * n_dof + 8 * nnz)

    def slab(self, nz_layers):
        """The first nz_layers element layers with nodes renumbered compactly: (X, conn, params)."""
        ne = self.nx * self.ny * min(nz_layers, self.nz)
        c = self.conn[:ne]
        used = np.unique(c)
        newid = np.zeros(self.X.shape[0] + 1, np.int64)
        newid[used] = np.arange(1, used.size + 1)
        P = self.params[:ne] if self.per_element else self.params
        return self.X[used - 1], newid[c].astype(np.int32), P, used


def oracle_model(w, X, conn, params):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O.Model(X, conn, [w.model], params, per_element=w.per_element)


def oracle_with_history(w, X, conn, params, used, threads):
    """The FP64 oracle on (a slab of) the workload, with the workload's committed history applied."""
    m = oracle_model(w, X, conn, params)
    idx = np.stack([3 * (used - 1) + d for d in range(3)], axis=1).reshape(-1)
    t_old = 0.0
    for t, U in w.history:
        m.set_time_old(t_old)
        m.evaluate_sample(t, U[idx], conn.shape[0], threads, tangent=False)
        m.commit()
        t_old = t
    m.set_time_old(t_old)
    return m, w.U_eval[idx]


def cpu_layers_for(w, target_gps):
    return max(1, min(w.nz, int(round(target_gps / (8 * w.nx * w.ny)))))


# ---------------------------------------------------------------------------------------------
# clocks, ranks, peaks, profile traffic
# ---------------------------------------------------------------------------------------------
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


class Clocks:
    """nvidia-smi clock sampling around a timed region: with Clocks(dev) as c: ...; c.summary."""

    def __init__(self, dev=0, tag="x"):
        self.dev = dev
        self.path = os.path.join(os.environ.get("CEOS_BENCH_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"ceos_bench_clocks_{tag}_{os.getpid()}.csv")
        self.summary = None

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        self.p = clocks_sampler_start(self.path)
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            self.p.wait()
        self.summary = clocks_summary(self.path, self.dev)
        return False


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


# B^T D B of one Hexa8 element in the node-pair form: 63 FMA per node and Gauss point for D B_b (54) and
# sigma g_b (9), 27 per off-diagonal block and 18 per diagonal block per Gauss point (28 + 8 blocks), over
# 8 Gauss points; the geometric dots g_a . sigma g_b (1,440 more) are left out of this floor
FMA_PER_ELEMENT_BDB = 8 * (8 * 63 + 28 * 27 + 8 * 18)


def fma_roofline(n_elem, element_ms, clocks, dev):
    """The element loop's other bound: the FP32 FMAs of its B^T D B contraction per element pass against
    the FP32 pipe's peak (128 FMA per clock per SM) at the SM clock sampled during the timed region."""
    import torch
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    peak = sms * 128 * mhz * 1e6 / 1e12
    achieved = FMA_PER_ELEMENT_BDB * n_elem / (element_ms * 1e-3) / 1e12
    return {"bound": "fp32_fma", "unit": "TFMA/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "fma_per_element": FMA_PER_ELEMENT_BDB, "floor_ms": FMA_PER_ELEMENT_BDB * n_elem / (peak * 1e12) * 1e3,
            "what": "B^T D B contraction FMAs of one element pass / its CUDA-event time, against 128 FMA per clock "
                    "per SM at the sampled SM clock (the Gauss-point update and phase-A geometry are extra work)"}


def conversion_roofline(workload, n_elem, conv_ms, peak):
    """The conversion pass is HBM-bound: its DRAM bytes (the committed ncu capture, scaled by elements)
    over its CUDA-event time, against the copy peak."""
    p = os.path.join(ROOT, "profiles", "element_loop_traffic.json")
    try:
        with open(p) as f:
            per = json.load(f)[workload]["kernel_dram_bytes_per_element"]["csr_convert_kernel"]
    except Exception:
        return None
    if not conv_ms or conv_ms <= 0:
        return None
    b = per * n_elem
    a = b / (conv_ms * 1e-3) / 1e9
    return {"bound": "hbm", "unit": "GB/s", "dram_bytes": b, "achieved": a, "peak": peak, "frac": a / peak,
            "what": "csr_convert_kernel: DRAM bytes of one launch (ncu capture, scaled by elements) / its CUDA-event "
                    "time (FP32 blocks read and re-zeroed, FP64 K written)"}


def profile_traffic(workload, n_elem):
    """DRAM bytes of one evaluation (all its kernels) from the committed ncu summary, scaled by elements."""
    p = os.path.join(ROOT, "profiles", "element_loop_traffic.json")
    try:
        with open(p) as f:
            rec = json.load(f)[workload]
        return rec["dram_bytes_per_element"] * n_elem, rec.get("captured_on")
    except Exception:
        return None, None


# ---------------------------------------------------------------------------------------------
# reference arm and CPU baseline: the FP64 oracle on host cores
# ---------------------------------------------------------------------------------------------
def run_reference(args, w, config):
    """--impl reference: exactly W warm-up and K timed steps; each step one evaluation of a bounded
    slab of the workload's mesh by the FP64 restatement of the reference element loop on all host
    threads."""
    threads = os.cpu_count() or 1
    layers = cpu_layers_for(w, args.ref_sample_gps)
    Xs, cs, Ps, used = w.slab(layers)
    m, U = oracle_with_history(w, Xs, cs, Ps, used, threads)
    n_gp = 8 * cs.shape[0]
    for _ in range(args.warmup):
        m.evaluate_sample(w.t_eval, U, cs.shape[0], threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, rc = m.evaluate_sample(w.t_eval, U, cs.shape[0], threads)
        times.append(time.perf_counter() - t0)
        assert rc == 0, rc
    secs = float(np.mean(times))
    rate = n_gp / secs
    sample = (f"each step: one FP64 evaluation (update + f_int + K) of the first {layers} element layers "
              f"({cs.shape[0]} elements, {n_gp} GPs) on {threads} threads; {args.steps} timed steps after "
              f"{args.warmup} warm-up, mean {secs:.3f} s")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran not buildable (no Fortran compiler/MKL); FP64 C++ restatement of its "
                    "element loop with linear-search assembly, OpenMP over element colours"}
    print(json.dumps(line), flush=True)


def run_cpu_single(w, nz_layers):
    """The oracle's element loop on one thread (the reference's serial loop) on the first element layers."""
    Xs, cs, Ps, used = w.slab(nz_layers)
    m, U = oracle_with_history(w, Xs, cs, Ps, used, 1)
    t0 = time.perf_counter()
    m.evaluate_sample(w.t_eval, U, cs.shape[0], 1)
    secs = time.perf_counter() - t0
    n_gp = 8 * cs.shape[0]
    return n_gp / secs, n_gp, secs


# ---------------------------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------------------------
def run_element_loop(args, w, config, world, rank, local_rank):
    import torch
    import ceos_b200 as G
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = local_rank
    torch.cuda.set_device(dev)
    g = G.ElementLoop(w.X, w.conn, w.model, w.params, per_element=w.per_element, precision=G.MIXED, device=dev)
    g.set_assembly(args.assembly)
    n_dof, nnz = g.n_dof, g.nnz
    t_old = 0.0
    for t, U in w.history:
        g.set_committed_time(t_old)
        _, _, rc, _ = g.evaluate(t, U, tangent=False)
        assert rc == 0, rc
        g.commit()
        t_old = t
    g.set_committed_time(t_old)
    dU = torch.tensor(w.U_eval, dtype=torch.float64, device=f"cuda:{dev}")
    dfint = torch.zeros(n_dof, dtype=torch.float64, device=f"cuda:{dev}")
    dK = torch.zeros(nnz, dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    def step():
        g.evaluate_device(w.t_eval, dU, dfint, dK, stream=sp)

    warmup = max(args.warmup, 3)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step()
    torch.cuda.synchronize()
    rc, nf = g.status()
    assert rc == 0, ("element failures", rc, nf)

    with Clocks(dev, f"r{rank}") as clk:
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
        # kernel durations for the roofline: events on the launching stream around each kernel
        g.set_options(G.OPT_TIME_KERNELS)
        kms, cms = [], []
        for _ in range(max(5, min(args.steps, 20))):
            g.evaluate_device(w.t_eval, dU, dfint, dK, stream=sp)
            k_ms, c_ms = g.kernel_time_ms()
            kms.append(k_ms)
            cms.append(c_ms)
        g.set_options(0)
    clocks = clk.summary

    # end to end through the C ABI with pinned host buffers: H2D of U, D2H of f_int and K every step
    U_pin = torch.from_numpy(np.ascontiguousarray(w.U_eval)).pin_memory()
    f_pin = torch.zeros(n_dof, dtype=torch.float64).pin_memory()
    K_pin = torch.zeros(nnz, dtype=torch.float64).pin_memory()
    lib = G.lib()
    nfail = C.c_int(0)

    def e2e_step():
        return lib.ceos_evaluate(g.handle, w.t_eval, C.c_void_p(U_pin.data_ptr()), C.c_void_p(f_pin.data_ptr()),
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
    # the device result equals the host result (up to the summation order of the atomics)
    assert torch.allclose(dfint.cpu(), f_pin, rtol=1e-9, atol=1e-9 * float(f_pin.abs().max()))

    ms_step = ms / args.steps
    value = whole_job_rate(w.n_gp * args.steps, world, ms * 1e-3)
    alg = w.algorithmic_bytes(g.n_nodes, n_dof, nnz)
    k_mean, c_mean = float(np.mean(kms)), float(np.mean(cms))
    eval_s = (k_mean + c_mean) * 1e-3
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / eval_s / 1e9
    traffic, traffic_src = profile_traffic(w.name, w.n_elem)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic", "config": config,
            "e2e": {"value": whole_job_rate(w.n_gp, world, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 8 * n_dof,
                    "d2h_bytes_per_step": 8 * (n_dof + nnz), "ms_per_step": e2e_s * 1e3,
                    "call": "ceos_evaluate (host U in, host f_int and K out, pinned buffers)"},
            "gpu_launches": g.launches_per_evaluation() * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                         "peak_kind": peak_kind, "kernel": g.kernel_names(), "kernel_ms": k_mean + c_mean,
                         "algorithmic_bytes_per_launch": alg,
                         "kernel_split_ms": {"element_loop": k_mean, "conversion": c_mean},
                         "compute": fma_roofline(w.n_elem, k_mean, clocks, dev),
                         "conversion": (conversion_roofline(w.name, w.n_elem, c_mean, peak)
                                        if getattr(args, "assembly", "two-pass") == "two-pass" else None),
                         "what": "algorithmic bytes of one evaluation / device time of all its kernels (the "
                                 "element loop and the K conversion, CUDA events on the launching stream)"},
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        # CPU baseline: one FP64 evaluation of the whole mesh on all host threads (the same oracle
        # evaluation gives the error of the timed GPU evaluation)
        used = np.arange(1, w.X.shape[0] + 1)
        m, U = oracle_with_history(w, w.X, w.conn, w.params, used, threads)
        t0 = time.perf_counter()
        f_o, k_o, rc_o = m.evaluate_sample(w.t_eval, U, w.n_elem, threads)
        secs = time.perf_counter() - t0
        r1, g1, s1 = run_cpu_single(w, nz_layers=cpu_layers_for(w, 131072))
        line["cpu_baseline"] = {"value": w.n_gp / secs, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"one FP64 evaluation of the whole mesh ({w.n_elem} elements) on "
                                          f"{threads} threads, {secs:.2f} s",
                                "single_thread": {"value": r1, "unit": UNIT, "cores": 1,
                                                  "sample": f"{g1 // 8} elements (first element layers), "
                                                            f"serial loop, {s1:.2f} s"}}
        if rc_o == 0:
            f_g, k_g = f_pin.numpy(), K_pin.numpy()
            line["error_vs_fp64_oracle"] = {
                "f_int_rel": float(np.abs(f_g - f_o).max() / np.abs(f_o).max()),
                "K_rel": float(np.abs(k_g - k_o).max() / np.abs(k_o).max()),
                "K_rel_fro": float(np.linalg.norm(k_g - k_o) / np.linalg.norm(k_o)),
                "what": "max |GPU - oracle| / max |oracle| over all f_int and K entries of the timed evaluation "
                        "(mixed precision GPU vs FP64 oracle, whole mesh, same Gauss-point history)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.destroy_process_group()


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
    with Clocks(0, "fe2") as clk:
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
           "elements": int(b.n_elem), "reduced_dofs": int(b.n_red), "clocks": clk.summary,
           "config": {"workload": f"batched FE2: {args.n_rve} periodic fibre RVEs, n U{{6..12}}, vf U[0.1,0.4], "
                                  "mu_f/mu_m=50, K/mu=100, F = I + G, |G_ij| <= 0.15, tol 1e-8, P + tangent"}}
    print(json.dumps(rec), flush=True)
    b.close()


def run_fe2_surrogate(args):
    """Learned surrogate against direct batched FE^2 (all on the GPU, no oracle)."""
    from ceos_b200 import fe2_surrogate as FS
    with Clocks(0, "sur") as clk:
        rec = FS.experiment(n_train=args.n_train, epochs=args.epochs, log=sys.stderr)
    rec["clocks"] = clk.summary
    print(json.dumps(rec), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=None, help="mesh size (96 for j2-plate: nx x nx x nx/2; 64 for visco)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--assembly", default="two-pass", choices=["two-pass", "fused", "banded"],
                    help="mixed-precision K assembly of the element-loop workloads")
    ap.add_argument("--ref-sample-gps", type=int, default=600000,
                    help="Gauss points per step of the reference arm's bounded sample")
    ap.add_argument("--workload", default="j2-plate",
                    choices=["j2-plate", "visco", "element-loop", "fe2-surrogate", "fe2-batch"])
    ap.add_argument("--n-rve", type=int, default=4096)
    ap.add_argument("--n-train", type=int, default=200000)
    ap.add_argument("--epochs", type=int, default=2000)
    args = ap.parse_args()
    if args.workload == "fe2-surrogate":
        return run_fe2_surrogate(args)
    if args.workload == "fe2-batch":
        return run_fe2_batch(args)
    name = "visco" if args.workload in ("visco", "element-loop") else "j2-plate"
    nx = args.nx or (96 if name == "j2-plate" else 64)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return
    w = Workload(name, nx)
    config = {"workload": w.label, "mesh": f"{w.nx}x{w.ny}x{w.nz} Hexa8", "elements": int(w.n_elem),
              "gauss_points": int(w.n_gp), "material": w.material,
              "precision": "FP32 element arithmetic/state, FP64 detF/lnJ/return mapping/K/f_int",
              "l2": "inputs larger than L2 (K and the Gauss-point state are each larger than the 126 MB L2)",
              "parallelism": f"replicas x{args.gpus}", "assembly": args.assembly}
    if args.impl == "reference":
        return run_reference(args, w, config)
    return run_element_loop(args, w, config, world, rank, local_rank)


if __name__ == "__main__":
    main()
