"""What the trained network gains over the method without it: a surrogate trained on the GPU from
RVE solves (40,000 samples, seconds of data and training) against direct FE^2 on the same macro
problem (2^3 macro cells, uniaxial stretch to 1.05 along the fibres in 3 steps).

The training samples cover that load range: a strain cube |G_ij| <= 0.06 (30 % of it scaled towards
small strains) and the uniaxial path along the fibres up to stretch 1.07 with nearly isochoric
contraction and +-2 % local perturbations.  Bars:
- the surrogate macro step is at least 10x faster than the direct one;
- the held-out stress error, the constitutive error (surrogate vs RVE solves at the direct run's own
  Gauss-point deformations) and the Gauss-point stress field against the direct run all stay under 1 %.
"""
import numpy as np
import pytest

from ceos_b200 import fe2_surrogate as FS

pytestmark = pytest.mark.gpu


def test_surrogate_macro_step_gain_over_direct_fe2():
    n, n_val = 40000, 2000
    F, vf = FS.sample_points(n, seed=21, amp=0.06, small_fraction=0.3, path_fraction=0.5,
                             stretch_range=(0.99, 1.07), path_amp=0.02)
    P, _, st = FS.rve_stresses(F, vf, n_cells=6)
    assert st["failed"] <= n // 200
    k = n - n_val
    sur, hist, _ = FS.fit(F[:k], vf[:k], P[:k], epochs=3000, batch=2048)
    assert hist[-1] < 0.05 * hist[0]
    Pp, flags = FS.predict_P(sur, F[k:], vf[k:])
    val = FS.stress_errors(Pp[~flags], P[k:][~flags])
    assert val["aggregate"] < 0.01, val
    res = FS.macro_compare(sur, nx=2, n_cells=6, stretch=1.05, n_steps=3, seed=3, axis=2)
    assert res["direct"]["failed"] is None and res["surrogate"]["failed"] is None
    t_direct = np.median(res["direct"]["step_s"][1:])
    t_sur = np.median(res["surrogate"]["step_s"][1:])
    assert t_direct >= 10.0 * t_sur, (t_direct, t_sur)
    assert sum(res["surrogate"]["fallback_points"]) == 0
    const = [c["in_range"] for c in res["constitutive_error_per_step"]]
    assert max(const) < 0.01, const
    assert max(res["stress_error_per_step"]) < 0.01, res["stress_error_per_step"]
    sur.close()
