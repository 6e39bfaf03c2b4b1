"""Host-side checks of the learned-sensor pieces (no GPU): the numpy network against finite differences, the
C oracle's forward against numpy, the PP activation on smooth and rough fields, the parameter layout, and
the viscosity RHS with the sensor switched off against the plain RHS."""
import numpy as np

from dgkernel_b200 import sensor as SN
from oracle import burgers_ref as b
from oracle import mlp_ref as MR
from oracle import oracle as O


def test_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin = 10
    p = SN.init_params(nin, seed=3).astype(np.float64) + rng.normal(size=SN.mlp_param_count(nin)) * 0.05
    X = rng.normal(size=(17, nin))
    y = rng.uniform(size=17)
    loss, g = MR.loss_grad(p, X, y, nin)
    for k in rng.choice(len(p), 40, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (MR.loss_grad(p + e, X, y, nin)[0] - MR.loss_grad(p - e, X, y, nin)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-7 + 1e-5 * abs(g[k]), k


def test_c_forward_matches_numpy():
    rng = np.random.default_rng(1)
    p = rng.normal(size=SN.mlp_param_count(35)) * 0.3
    X = rng.normal(size=(4, 35))
    want = MR.forward(p, X, 35)[0]
    got = [O.lib().ora_mlp_forward1(35, np.ascontiguousarray(p), np.ascontiguousarray(x)) for x in X]
    assert np.max(np.abs(np.array(got) - want)) < 1e-14


def test_parameter_layout_and_init():
    assert SN.mlp_param_count(35) == 32 * 35 + 32 + 32 * 32 + 32 + 32 + 1 == 2241
    p = SN.init_params(35)
    W1, b1, W2, b2, w3, b3 = MR.unpack(p, 35)
    assert np.all(b1 == 0) and np.all(b2 == 0) and b3 == 0
    assert np.abs(W1).max() <= np.sqrt(6 / 67) and np.abs(W1).std() > 0.05
    assert np.array_equal(p, SN.init_params(35))


def test_pp_sensor_smooth_and_rough():
    prob = b.Problem(4, 6, 1, "smooth")
    av = O.AVState(prob)
    S, sig, feat = av.sensor(prob.u0)
    assert np.all(sig == 0.0) and S.max() < av.s0 - av.kappa  # resolved smooth field: no activation
    np.testing.assert_allclose(np.linalg.norm(feat, axis=1), 1.0, rtol=1e-12)
    rough = prob.u0.copy()
    rough[::7, 5] += 0.3  # a node-scale jump in every 7th element
    S2, sig2, _ = av.sensor(rough)
    assert np.all(sig2[::7] > 0.5) and np.all(S2[::7] > S[::7])
    assert O.mode_degrees(4).tolist().count(4) == 15


def test_viscosity_rhs_without_sensor_is_the_plain_rhs():
    prob = b.Problem(3, 4, 1, "sine")
    av = O.AVState(prob)
    r, eps = av.rhs(prob.u0, "none")
    assert np.all(eps == 0)
    assert np.max(np.abs(r - O.RunState(prob).rhs(prob.u0))) < 1e-13
