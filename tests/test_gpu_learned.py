"""The learned k-proposal on the GPU.

* the exact Gaussian sampler ("gauss_iid"): never m = 0, deterministic per (seed, step), and its
  |k|-bin histogram over many draws matches the bin masses W_b (chi-square bound);
* importance weights keep the estimator unbiased: with a network that reweights the bins
  strongly, the mean RBE force over many k-sets converges to the FP64 Ewald k-space force of the
  oracle, within 4 standard errors;
* training lowers the force variance: the trained proposal's group loss falls below the Gaussian's
  on its training data, and on fresh k-sets the measured RBE noise (two independent k-sets at the
  same positions) is lower than the Gaussian's at the same P.
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems
from oracle import mlp
from tests.helpers import make_ff, to_dev

pytestmark = pytest.mark.gpu


def _cfg(proposal, P, dt=0.0, seed=11):
    cfg = systems.electrolyte_config(P=P, precision="fp32", seed=seed, ensemble="NVE", dt=dt)
    cfg["hyper_parameters"]["coulomb"]["proposal"] = proposal
    return cfg


def _kappa_bins(m, L, alpha):
    k = 2 * np.pi * m / L
    kap = np.sqrt((k ** 2).sum(1)) / (2 * np.sqrt(alpha))
    return np.minimum((kap * (256 / 6.0)).astype(int), 255)


def test_iid_sampler_law_and_determinism(cuda):
    s = systems.electrolyte(3000, seed=4)
    P = 1000
    cfg = _cfg("gauss_iid", P)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    L = (s["hi"] - s["lo"])[0]
    a = ff.sample_k(5, P)
    b = ff.sample_k(5, P)
    assert np.array_equal(a, b)
    draws = np.concatenate([ff.sample_k(st, P) for st in range(200)])
    assert not np.any(np.all(draws == 0, axis=1))
    # bin masses W_b of p(m) ~ exp(-pi^2 |m|^2 / (alpha L^2)), m != 0, by direct summation
    M = int(np.ceil(6 * np.sqrt(alpha) * L / np.pi))
    g = np.exp(-np.pi ** 2 * np.arange(-M, M + 1) ** 2 / (alpha * L * L))
    mm = np.arange(-M, M + 1)
    mx, my, mz = np.meshgrid(mm, mm, mm, indexing="ij")
    w = (g[:, None, None] * g[None, :, None] * g[None, None, :]).ravel()
    allm = np.stack([mx.ravel(), my.ravel(), mz.ravel()], 1)
    keep = np.any(allm != 0, axis=1)
    W = np.bincount(_kappa_bins(allm[keep], L, alpha), weights=w[keep], minlength=256)
    W /= W.sum()
    obs = np.bincount(_kappa_bins(draws, L, alpha), minlength=256)
    n = len(draws)
    sel = W * n > 20
    chi2 = (((obs[sel] - n * W[sel]) ** 2) / (n * W[sel])).sum()
    dof = sel.sum() - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_learned_weights_unbiased(cuda, oracle_lib):
    import torch
    s = systems.electrolyte(1500, seed=6)
    P = 64
    cfg = _cfg("learned", P)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    cfg["hyper_parameters"]["neighbor"]["cut_off"] = 0.5     # empty near list: the force is the k-space part
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    # a network that strongly reweights |k|: h = 2 tanh(2 tanh(4 kappa / 3)), up to e^1.9 between bins
    p = np.zeros(mlp.N_PARAM, np.float32)
    p[mlp.OW1 + 0 * 16 + 0] = 4.0
    p[mlp.OW2 + 0 * 64 + 0] = 2.0
    p[mlp.OW3 + 0] = 2.0
    ff.proposal_params(p)
    L = s["hi"] - s["lo"]
    ref, _ = oracle_lib.ewald_kspace(s["pos"], s["charge"], L, alpha, kcut=2 * np.sqrt(alpha) * 6.2)
    q = s["charge"] != 0
    nsteps = 300
    acc = np.zeros_like(ref)
    acc2 = np.zeros(q.sum())
    for _ in range(nsteps):
        ff.step(1)
        torch.cuda.synchronize()
        f = ff.far_force()
        acc += f
        acc2 += ((f - ref)[q] ** 2).sum(1)
    assert ff.status() == 0
    mean = acc / nsteps
    err = np.sqrt(((mean - ref)[q] ** 2).sum(1).mean())
    sigma = np.sqrt(acc2.mean() / nsteps)            # per-step RMS deviation
    assert err <= 4 * sigma / np.sqrt(nsteps), (err, sigma)


def _noise(ff, nsteps, torch):
    """Per-atom RMS of the RBE estimator: k-sets of consecutive steps at fixed positions (dt = 0)."""
    prev, acc, n = None, 0.0, 0
    for _ in range(nsteps):
        ff.step(1)
        torch.cuda.synchronize()
        f = ff.far_force()
        if prev is not None:
            acc += ((f - prev) ** 2).sum(1).sum() / 2.0
            n += 1
        prev = f
    return acc, n


def test_training_lowers_force_variance(cuda):
    import torch
    s = systems.electrolyte(20000, seed=8)
    P = 200
    q = s["charge"] != 0
    cfg = _cfg("learned", P, dt=0.0)
    cfg["hyper_parameters"]["neighbor"]["cut_off"] = 0.5
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    rep = ff.train_proposal(n_snapshots=24, steps_between=0, k_per_snapshot=8192, iterations=400,
                            learning_rate=3e-3, seed=3)
    assert ff.status() == 0
    assert rep["loss_final"] < rep["loss_gauss"], rep
    assert rep["loss_optimum"] <= rep["loss_final"] + 1e-6, rep
    acc_l, n_l = _noise(ff, 60, torch)
    cfg_g = _cfg("gauss_iid", P, dt=0.0)
    cfg_g["hyper_parameters"]["neighbor"]["cut_off"] = 0.5
    dev_g = to_dev(s, cuda)
    ffg = make_ff(cfg_g, s, dev_g)
    acc_g, n_g = _noise(ffg, 60, torch)
    var_l = acc_l / (n_l * q.sum())
    var_g = acc_g / (n_g * q.sum())
    print(f"train report {rep}; measured variance learned/gauss = {var_l / var_g:.4f}")
    assert var_l < var_g, (var_l, var_g, rep)


def test_learned_proposal_on_cvff_molecules(cuda):
    """The learned proposal on a CVFF system (REAL units, special bonds, RBL near field): training
    lowers its loss below the Gaussian's, and graph-replayed MD steps with the trained proposal
    keep every status bit clear and the forces finite."""
    import torch
    s = systems.molecular(n_chain=125, chain_len=10, n_ion_pairs=40, seed=9)
    cfg = systems.molecular_config(P=64, precision="fp32", neighbor="RBL", cutoff=8.0, r_core=4.0, sample_num=60,
                                   special=(0.0, 0.0, 0.5))
    cfg["hyper_parameters"]["coulomb"]["proposal"] = "learned"
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
                    s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"])
    rep = ff.train_proposal(n_snapshots=16, steps_between=2, k_per_snapshot=4096, iterations=200,
                            learning_rate=3e-3, seed=4)
    assert ff.status() == 0
    assert rep["loss_final"] < rep["loss_gauss"], rep
    ff.Execute()
    ff.step(20)
    torch.cuda.synchronize()
    assert ff.status() == 0
    assert torch.isfinite(dev["force"]).all() and torch.isfinite(dev["pos"]).all()
    ff.close()
