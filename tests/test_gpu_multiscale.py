"""The device passes of the coarse-to-fine warm start (pdot_points_max_sqdist,
pdot_points_c_transform through pdot/multiscale.py) against brute force on the
host. Both read FP32 coordinates and compute in FP64, so the references round
the points to FP32 first; the results agree to FP64 rounding (1e-13)."""
import numpy as np
import pytest

from pdot import instances, multiscale

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("np_,nc,dim", [(50, 17, 2), (1000, 300, 2), (257, 513, 3), (5, 1, 1)])
def test_c_transform_matches_brute_force(cuda, np_, nc, dim):
    rng = np.random.default_rng(np_ + nc)
    pts = rng.uniform(0, 1, (np_, dim)).astype(np.float32)
    cen = rng.uniform(0, 1, (nc, dim))
    dual = rng.normal(0, 0.1, nc)
    got = multiscale.c_transform(pts, cen, dual, 0.7)
    p64 = pts.astype(np.float64)
    ref = (0.7 * ((p64[:, None, :] - cen[None, :, :]) ** 2).sum(-1) - dual[None, :]).min(axis=1)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("m,n,dim", [(2, 2, 2), (300, 700, 2), (1025, 257, 3), (7, 3, 1)])
def test_max_sq_distance_matches_brute_force(cuda, m, n, dim):
    rng = np.random.default_rng(m * n)
    xs = rng.uniform(-1, 2, (m, dim))
    ys = rng.uniform(0, 1, (n, dim))
    x32, y32 = xs.astype(np.float32).astype(np.float64), ys.astype(np.float32).astype(np.float64)
    ref = float(((x32[:, None, :] - y32[None, :, :]) ** 2).sum(-1).max())
    assert multiscale.max_sq_distance(xs, ys) == pytest.approx(ref, rel=1e-13)


def test_coarse_to_fine_warm_start_solves_the_fine_problem(cuda):
    """The whole pipeline on a small point cloud: the extended duals are finite,
    and the fine solve from them (plan recovered from the duals) ends optimal."""
    import pdot

    xs, ys, a, b = instances.gauss_mixture_instance(400, 300, seed=2)
    u, v, info = multiscale.coarse_to_fine_duals(xs, ys, a, b, G=8)
    assert info["coarse_termination"] == "OPTIMAL"
    assert u.shape == (400,) and v.shape == (300,)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(v))
    prob = pdot.OptimalTransportProblem(None, a, b)
    pts = (xs.astype(np.float32), ys.astype(np.float32))
    out = pdot.optimize(pdot.default_parameters(1e-4), prob, precision="f32", cost="sqeuclid", points=pts,
                        warm_start=(u, v), recover_plan=(3e-4, 100))
    assert out.termination_reason == pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


@pytest.mark.parametrize("coarse", [False, True])
def test_learned_point_cloud_warm_starts_solve_the_fine_problem(cuda, coarse):
    """The packaged network's warm starts for a point cloud: its 32 x 32 grid
    duals extended to every point, or first to the cells of a 16 x 16 coarse
    solve that they warm-start. The duals are finite and the fine solve from
    them ends optimal."""
    import pdot
    from pdot import learned

    xs, ys, a, b = instances.gauss_mixture_instance(400, 300, seed=3)
    st = learned.WarmStarter(device=0)
    if coarse:
        u, v, info = multiscale.learned_coarse_to_fine_duals(xs, ys, a, b, st, G=16)
        assert info["coarse_termination"] == "OPTIMAL"
    else:
        u, v, info = multiscale.learned_to_fine_duals(xs, ys, a, b, st)
    assert u.shape == (400,) and v.shape == (300,)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(v))
    prob = pdot.OptimalTransportProblem(None, a, b)
    pts = (xs.astype(np.float32), ys.astype(np.float32))
    out = pdot.optimize(pdot.default_parameters(1e-4), prob, precision="f32", cost="sqeuclid", points=pts,
                        warm_start=(u, v), recover_plan=(3e-4, 100))
    assert out.termination_reason == pdot.TerminationReason.TERMINATION_REASON_OPTIMAL
