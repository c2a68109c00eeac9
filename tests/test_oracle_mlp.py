"""CPU checks of the proposal network's restatement (oracle/mlp.py): the FP64 gradient equals
central finite differences of the FP64 loss; the loss is invariant to a constant shift of h and
is minimised at e^{h_b} ~ sqrt(C_b / W_b); BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import mlp


def _data(G=2, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(G * 256, 16)).astype(np.float32)
    w = rng.uniform(0.1, 1.0, G * 256).astype(np.float32)
    c = rng.uniform(0.1, 1.0, G * 256).astype(np.float32)
    return x, w, c


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 0.0], np.float32)
    got = mlp.bf16(v)
    assert got[0] == 1.0 and got[1] == 1.0          # tie rounds to even
    assert got[2] == 1.0078125
    assert abs(got[3] + 3.140625) < 1e-12


def test_fp64_gradient_matches_finite_differences():
    x, w, c = _data()
    p = mlp.init_params(3).astype(np.float64)
    L, _, g, _ = mlp.loss_and_grad(p, x, w, c, bf=False)
    rng = np.random.default_rng(0)
    for idx in list(rng.choice(mlp.N_PARAM, 25, replace=False)) + [mlp.OB3, mlp.OW3, mlp.OB1]:
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[idx] += e
        pm[idx] -= e
        fd = (mlp.loss_and_grad(pp, x, w, c, bf=False)[0] - mlp.loss_and_grad(pm, x, w, c, bf=False)[0]) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, g[idx])


def test_loss_shift_invariance_and_optimum():
    x, w, c = _data(G=1)
    p = mlp.init_params(4)
    L0 = mlp.loss_and_grad(p, x, w, c, bf=False)[0]
    p2 = p.copy()
    p2[mlp.OB3] += 3.0
    assert abs(mlp.loss_and_grad(p2, x, w, c, bf=False)[0] - L0) < 1e-9
    # the optimum of log sum W e^h + log sum C e^-h over free h is 2 log sum sqrt(W C)
    h = 0.5 * np.log(c.astype(np.float64) / w)
    opt = np.log((w * np.exp(h)).sum()) + np.log((c * np.exp(-h)).sum())
    assert abs(opt - 2 * np.log(np.sqrt(w.astype(np.float64) * c).sum())) < 1e-9
    assert L0 >= opt - 1e-12
