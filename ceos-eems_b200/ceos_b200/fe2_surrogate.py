"""Training data, fitting and error of the learned FE^2 surrogate, all on the GPU.

Training pairs (C, vf) -> S come from the batched RVE solver itself (ceos_fe2_*): F = I + G with
G_ij uniform in [-amp, amp] (det F > 0) and vf uniform in vf_range, one fixed RVE resolution
n_cells (the homogenized response depends on the resolution, so the surrogate stands in for the
RVE family of that resolution).  The RVE solver is also the reference the surrogate's error is measured against."""
import time

import numpy as np

from . import fe2 as FE2
from .surrogate import Surrogate, init_params, training_targets, voigt_C


def sample_points(n, seed, amp=0.15, vf_range=(0.1, 0.4), small_fraction=0.0, path_fraction=0.0, axis=2,
                  stretch_range=(0.97, 1.26), path_amp=0.05):
    """F = I + G, G_ij uniform in [-amp, amp] (det F > 0); a share small_fraction of the points has its
    G scaled by a uniform factor in [0, 1] (more small strains, same range); vf uniform.  A share
    path_fraction (the last points) follows the macro uniaxial load path instead: stretch lam along
    `axis` uniform in stretch_range, lam^-1/2 (+-3 %) across it (the nearly isochoric contraction of
    K/mu = 100 phases), times I + G with |G_ij| <= path_amp (the spread of the local deformation
    around the macro one)."""
    F = FE2.sample_macro_F(n, seed=seed, amp=amp)
    rng = np.random.default_rng(seed + 7919)
    vf = rng.uniform(vf_range[0], vf_range[1], n)
    k = int(round(small_fraction * n))
    if k:
        F[:k] = np.eye(3) + rng.uniform(0.0, 1.0, (k, 1, 1)) * (F[:k] - np.eye(3))
    m = int(round(path_fraction * n))
    if m:
        lam = rng.uniform(stretch_range[0], stretch_range[1], m)
        lat = (lam ** -0.5)[:, None] * rng.uniform(0.97, 1.03, (m, 2))
        D = np.zeros((m, 3, 3))
        others = [d for d in range(3) if d != axis]
        D[:, axis, axis] = lam
        D[:, others[0], others[0]] = lat[:, 0]
        D[:, others[1], others[1]] = lat[:, 1]
        G = rng.uniform(-path_amp, path_amp, (m, 3, 3))
        F[n - m:] = np.einsum("nij,njk->nik", np.eye(3) + G, D)
    return F, vf


def rve_stresses(F, vf, n_cells=6, batch=4096, tangent=False, **rve_args):
    """First Piola stress (and tangent) of the RVEs at (F, vf), solved in batches on the GPU.
    RVEs that cannot converge come back as NaN.  Returns (P [n,3,3], A [n,9,9] or None, stats)."""
    n = len(vf)
    P = np.full((n, 3, 3), np.nan)
    A = np.full((n, 9, 9), np.nan) if tangent else None
    b = None
    t0 = time.perf_counter()
    newton, failed, minres = 0, 0, 0
    for s0 in range(0, n, batch):
        k = min(batch, n - s0)
        if b is None or b.n_rve != k:
            if b is not None:
                b.close()
            b = FE2.BatchedRVE(np.full(k, n_cells, np.int32), vf[s0:s0 + k], **rve_args)
            b.set_allow_failures(True)
        else:
            b.set_fractions(vf[s0:s0 + k])
        out = b.solve(F[s0:s0 + k], tangent=tangent)
        P[s0:s0 + k] = out["P"]
        if tangent:
            A[s0:s0 + k] = out["A"]
        newton += int(out["newton_iters"][out["newton_iters"] > 0].sum())
        minres += int(out["cg_iters"].sum())
        failed += int(out["failed"].sum())
    if b is not None:
        b.close()
    secs = time.perf_counter() - t0
    return P, A, {"seconds": secs, "rve_per_s": n / secs, "failed": failed, "newton_total": newton,
                  "minres_total": minres}


def fit(F, vf, P, epochs=150, batch=2048, lr0=3e-3, lr1=2e-5, seed=0, s_C=0.15, vf0=0.25, s_vf=0.15,
        relative=0.2, box_margin=0.005):
    """Train a surrogate on the finite samples; the training box of the range check is the
    component-wise extent of the training inputs widened by box_margin of that extent on either side
    (the sampled extremes fall just inside the sampling ranges: without a margin a macro point whose
    fibre fraction lies 1e-6 beyond the smallest sampled one would be sent to an RVE solve for
    nothing).  relative > 0 weights every sample by
    1 / (|S|^2 / mean|S|^2 + relative), so the loss measures relative stress error (small stresses of
    nearly isochoric states count as much as the large volumetric ones) with a floor.
    Returns (Surrogate, loss history, seconds)."""
    ok = np.all(np.isfinite(P.reshape(len(P), -1)), axis=1)
    F, vf, P = F[ok], vf[ok], P[ok]
    C6 = voigt_C(F)
    S = np.linalg.solve(F, P)
    s_scale = float(np.sqrt(np.mean(S ** 2)))
    s_W = s_scale * s_C
    sur = Surrogate(batch_max=batch)
    sur.set_params(init_params(seed))
    sur.set_scaling(s_C, s_W, vf0, s_vf)
    x = sur.inputs(C6, vf)
    lo, hi = x.min(axis=0), x.max(axis=0)
    pad = box_margin * (hi - lo)
    sur.set_scaling(s_C, s_W, vf0, s_vf, lo=lo - pad, hi=hi + pad)
    t, w = training_targets(F, P, s_C, s_W)
    sw = None
    if relative > 0:
        tn = np.sum(w * t * t, axis=1)
        sw = 1.0 / (tn / tn.mean() + relative)
        sw /= sw.mean()
    t0 = time.perf_counter()
    hist = sur.train(x, t, w, epochs, batch, lr0, lr1, seed, sw=sw)
    sur.set_reference(float(vf.min()), float(vf.max()))
    return sur, hist, time.perf_counter() - t0


def predict_P(sur, F, vf):
    """Surrogate first Piola stress [n,3,3] and out-of-range flags."""
    S6, _, flags = sur.evaluate(voigt_C(F), vf)
    S = np.zeros((len(vf), 3, 3))
    for p, (i, j) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]):
        S[:, i, j] = S6[:, p]
        S[:, j, i] = S6[:, p]
    return F @ S, flags


def stress_errors(P_pred, P_ref):
    """Relative stress errors: aggregate sqrt(sum |dP|^2 / sum |P|^2) and per-point |dP|/|P|."""
    ok = np.all(np.isfinite(P_ref.reshape(len(P_ref), -1)), axis=1)
    d = np.linalg.norm((P_pred - P_ref)[ok].reshape(ok.sum(), -1), axis=1)
    r = np.linalg.norm(P_ref[ok].reshape(ok.sum(), -1), axis=1)
    return {"aggregate": float(np.sqrt(np.sum(d ** 2) / np.sum(r ** 2))),
            "median": float(np.median(d / r)), "p95": float(np.percentile(d / r, 95)),
            "max": float(np.max(d / r)), "n": int(ok.sum())}


def macro_compare(sur, nx=4, n_cells=6, stretch=1.2, n_steps=10, seed=11, tol=1e-6, axis=2):
    """Uniaxial macro stretch on an nx^3 mesh with the surrogate (RVE fallback outside its box)
    and with RVE solves at every point; per-step wall times, Newton iterations, fallback points
    and the relative error of the Gauss-point first Piola stresses of the surrogate run against
    the direct run after every step."""
    import sys

    from . import CeosError
    from . import macro as M
    vf = np.random.default_rng(seed).uniform(0.1, 0.4, nx ** 3)
    res, fields, const_err = {}, {}, []
    for mode in ("direct", "surrogate"):
        m = M.MacroFE2(nx, vf, n_cells=n_cells, surrogate=sur, axis=axis)
        L = m.X[:, axis].max() - m.X[:, axis].min()
        times, its, fbs, Ps, failed = [], [], [], [], None
        for k in range(1, n_steps + 1):
            fb0 = m.stats["fallback_points"]
            t0 = time.perf_counter()
            try:
                its.append(m.newton_step((stretch - 1.0) * L * k / n_steps, mode, tol))
            except CeosError as e:  # an RVE (or the macro Newton) that cannot converge ends this run
                failed = {"step": k, "stretch": 1.0 + (stretch - 1.0) * k / n_steps, "reason": str(e)}
                print(f"macro {mode}: step {k} failed: {e}", file=sys.stderr, flush=True)
                break
            times.append(time.perf_counter() - t0)
            fbs.append(m.stats["fallback_points"] - fb0)
            Ps.append(m.gp_first_piola())
            if mode == "direct":  # the surrogate's response at the direct run's own deformation
                Fq = m._gp_F_host()
                Pq, flq = predict_P(sur, Fq, np.tile(vf, 8))
                const_err.append({"in_range": stress_errors(Pq[~flq], Ps[-1][~flq])["aggregate"] if (~flq).any()
                                  else None, "out_of_range_points": int(flq.sum())})
            print(f"macro {mode}: step {k} {times[-1]:.2f}s newton {its[-1]} fallback {fbs[-1]}", file=sys.stderr,
                  flush=True)
        res[mode] = {"step_s": times, "newton": its, "fallback_points": fbs, "stats": dict(m.stats),
                     "failed": failed}
        fields[mode] = Ps
        m.close()
    # field error: the two macro solutions differ wherever the constitutive responses do
    res["stress_error_per_step"] = [stress_errors(Psu, Pd)["aggregate"]
                                    for Pd, Psu in zip(fields["direct"], fields["surrogate"])]
    # constitutive error: surrogate against RVE solves at the same deformation gradients
    res["constitutive_error_per_step"] = const_err
    return res


def macro_surrogate_run(sur, nx=32, stretch=1.2, n_steps=10, seed=12, tol=1e-6, max_fallback=4096, n_cells=6,
                        axis=2, pool_size=4096):
    """Surrogate macro run on nx^3 cells; stops at a step that would send more than max_fallback
    points to RVE solves (FallbackLimit) or whose RVE or macro solve fails.  Returns per-step times
    and the steps done."""
    from . import CeosError
    from . import macro as M
    vf = np.random.default_rng(seed).uniform(0.1, 0.4, nx ** 3)
    m = M.MacroFE2(nx, vf, n_cells=n_cells, surrogate=sur, axis=axis)
    m.max_fallback = max_fallback
    m.pool_size = pool_size
    L = m.X[:, axis].max() - m.X[:, axis].min()
    times, its, fbs, stopped = [], [], [], None
    for k in range(1, n_steps + 1):
        fb0 = m.stats["fallback_points"]
        t0 = time.perf_counter()
        try:
            its.append(m.newton_step((stretch - 1.0) * L * k / n_steps, "surrogate", tol))
        except (M.FallbackLimit, CeosError) as e:
            stopped = {"step": k, "reason": str(e)}
            break
        times.append(time.perf_counter() - t0)
        fbs.append(m.stats["fallback_points"] - fb0)
    out = {"step_s": times, "newton": its, "fallback_points": fbs, "stopped": stopped, "n_gp": m.n_gp,
           "stats": dict(m.stats)}
    m.close()
    return out


def experiment(n_train=200000, epochs=2000, log=None, nx_direct=8, nx_big=32, path_fraction=0.4):
    """The learned-surrogate experiment: training data from the batched RVE solver (the cube of
    |G_ij| <= 0.15 and the macro load path), training, held-out stress error, a head-to-head of
    surrogate and direct FE^2 on an nx_direct^3 macro mesh (both measured), and the nx_big^3
    surrogate macro run.  The macro load is uniaxial stretch to 1.2 along the fibres (z).  Returns one
    JSON-ready record."""
    import json

    rec = {"metric": "FE2 macro step time: surrogate vs direct", "unit": "s", "higher_is_better": False,
           "dtype": "bf16 training / f32 inference / f64 RVE", "data": "synthetic"}
    F, vf = sample_points(n_train, seed=1, small_fraction=0.3, path_fraction=path_fraction)
    P, _, st = rve_stresses(F, vf, batch=8192)
    Fv, vfv = sample_points(4096, seed=99, path_fraction=path_fraction)
    Pv, _, _ = rve_stresses(Fv, vfv, batch=4096)
    Ft, vft = sample_points(8192, seed=7)
    _, _, st_tan = rve_stresses(Ft, vft, batch=8192, tangent=True)
    sur, hist, t_train = fit(F, vf, P, epochs=epochs, batch=2048, lr0=3e-3, lr1=3e-6)
    Pp, fl = predict_P(sur, Fv, vfv)
    rec["training"] = {"samples": int(n_train), "path_fraction": path_fraction, "rve_n_cells": 6,
                       "data_s": st["seconds"], "rve_per_s": st["rve_per_s"],
                       "rve_per_s_with_tangent": st_tan["rve_per_s"], "failed_rves": st["failed"], "epochs": epochs,
                       "batch": 2048, "adam_steps": epochs * (n_train // 2048), "train_s": t_train,
                       "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1])}
    rec["validation_stress_error"] = stress_errors(Pp[~fl], Pv[~fl])
    rec["validation_out_of_range"] = int(fl.sum())
    if log:
        print(json.dumps({"partial": "training", "training": rec["training"],
                          "validation": rec["validation_stress_error"]}), file=log, flush=True)
    h2h = macro_compare(sur, nx=nx_direct)
    rec[f"macro_{nx_direct}cube"] = {k: h2h[k] for k in ("direct", "surrogate", "stress_error_per_step",
                                                         "constitutive_error_per_step")}
    rec["speedup_head_to_head"] = [d / s for d, s in zip(h2h["direct"]["step_s"], h2h["surrogate"]["step_s"])]
    if log:
        print(json.dumps({"partial": "head_to_head", "macro": rec[f"macro_{nx_direct}cube"],
                          "speedup": rec["speedup_head_to_head"]}), file=log, flush=True)
    big = macro_surrogate_run(sur, nx=nx_big)
    s_big = np.array(big["step_s"])
    rec[f"macro_{nx_big}cube"] = {"surrogate": {k: big[k] for k in ("step_s", "newton", "fallback_points", "stopped")},
                                  "surrogate_stats": big["stats"]}
    rec["value"] = float(s_big.mean()) if s_big.size else None
    rec["config"] = {"workload": f"FE2 uniaxial stretch to 1.2 along the fibres in 10 increments; macro {nx_big}^3 "
                                 f"Hexa8 ({8 * nx_big ** 3} GPs) with the surrogate and a measured {nx_direct}^3 "
                                 "head-to-head against direct FE2; periodic fibre RVEs n=6, vf U[0.1,0.4], "
                                 "mu_f/mu_m=50, K/mu=100",
                     "surrogate": "MLP 7-128x4-1 softplus energy of (C, vf)"}
    sur.close()
    return rec
