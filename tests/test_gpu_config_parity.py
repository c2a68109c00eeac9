"""Oracle parity at the benchmark configurations' own sizes.

Each configuration the benchmark runs is checked against the CPU oracle on the same inputs:
* the 1,000,000-atom electrolyte (LJ + erfc near + RBE with an injected P = 500 k-set), FP32
  and FP64, and in FP64 also after MD steps with the Verlet skin of the benchmark (list reuse);
* the 256,000-atom Johnson EAM crystal, FP32 and FP64;
* the 30,000-atom SPC/E water (near + RBE P = 200 + intramolecular terms), FP32;
* the 4,000-atom LJ FCC at rc 2.5 in FP64, including a short NVE trajectory;
* 16 replicas of the 512-replica batch (the smallest, the largest and 14 more), FP32, each with
  its own injected k-set.

Bars, as in the small parity tests: neighbour pair sets bit-exact per atom at rc (the
reference's per-call list, ComputeNeighboursWorklet, rbmd/framework/run/worklet/RunWorklet.cpp:
40-96); forces max_i |dF_i| / rms|F| <= 1e-5 in FP32 and <= 1e-11 in FP64 against the oracle's
reference-precision pair terms (RunWorklet.cpp:170-417) plus its FP64 RBE terms
(RunWorklet.cpp:1508-1677).  The k-space term is evaluated by the oracle on the charged atoms
only (uncharged atoms contribute nothing to rho_k and receive no k-space force).
"""
import numpy as np
import pytest

from copy_gpu_b200 import Box, systems
from tests.helpers import make_ff, pair_sets_equal, rel_err, to_dev

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "fp64": 1e-11}


def _posr(pos, prec):
    return pos.astype(np.float32) if prec == "fp32" else pos.astype(np.float64)


def _kspace(pos, charge, L, alpha, qqr2e, m, origin=(0.0, 0.0, 0.0), oracle=None, prec="fp64"):
    """RBE force of the charged atoms (FP64, or the reference's FP32 terms), scattered back to all
    atoms."""
    q = np.nonzero(charge != 0)[0]
    out = np.zeros((pos.shape[0], 3))
    if len(q) == 0:
        return out
    rho = oracle.rhok(pos[q], charge[q], L, m, origin=origin, prec=prec)
    out[q] = oracle.rbe_force(pos[q], charge[q], L, alpha, qqr2e, m, rho, origin=origin, prec=prec)
    return out


def _run(cfg, s, cuda, m=None, boxes=None, offsets=None, cap=160, steps=0):
    import torch
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev, boxes=boxes, offsets=offsets)
    if m is not None:
        ff.set_ksamples(m)
    ff.Execute()
    if steps:
        ff.step(steps)
    torch.cuda.synchronize()
    assert ff.status() == 0
    c, ids = ff.neighbors(cap) if not steps else (None, None)
    out = dict(force=dev["force"].cpu().numpy(), pos=dev["pos"].cpu().numpy(), counts=c, ids=ids)
    ff.close()
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_electrolyte_1m_pairs_and_force(cuda, oracle_lib, prec):
    s = systems.electrolyte(1_000_000, seed=3)
    P = 500
    cfg = systems.electrolyte_config(P=P, precision=prec, seed=5, ensemble="NVE")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, 7, 0, 0, P)
    g = _run(cfg, s, cuda, m)
    pr = _posr(s["pos"], prec)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 2.5, prec, cap=128)
    bad = pair_sets_equal(g["counts"], g["ids"], nl[0], nl[1])
    assert bad == -1, f"neighbour pair set of atom {bad} differs"
    near = oracle_lib.near_force(pr, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                                 sigma=s["sigma"], with_coul=True, alpha=alpha, coul_scale=1.0, prec=prec, sum_mode=1)
    del nl
    ref = near + _kspace(s["pos"], s["charge"], L, alpha, 1.0, m, oracle=oracle_lib)
    err = rel_err(g["force"], ref)
    assert err <= TOL[prec], f"1M electrolyte force rel err {err:.3e} > {TOL[prec]}"


def test_electrolyte_1m_skin_steps_fp64(cuda, oracle_lib):
    """The benchmark's Verlet skin (0.3) with list reuse: after NVE steps the force equals a fresh
    oracle evaluation (per-call list at rc) at the device's positions."""
    s = systems.electrolyte(1_000_000, seed=3)
    P = 500
    cfg = systems.electrolyte_config(P=P, precision="fp64", seed=5, ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, 7, 0, 0, P)
    g = _run(cfg, s, cuda, m, steps=6)
    x = g["pos"]
    nl = oracle_lib.neighbors(x, s["lo"], s["hi"], 2.5, "fp64", cap=128)
    near = oracle_lib.near_force(x, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                                 sigma=s["sigma"], with_coul=True, alpha=alpha, coul_scale=1.0, prec="fp64")
    del nl
    ref = near + _kspace(x, s["charge"], L, alpha, 1.0, m, oracle=oracle_lib)
    err = rel_err(g["force"], ref)
    assert err <= TOL["fp64"], f"1M electrolyte (skin, 6 steps) force rel err {err:.3e}"


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_eam_256k_pairs_and_force(cuda, oracle_lib, tmp_path, prec):
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=40, seed=13)
    cfg = systems.eam_config(pot, precision=prec)
    g = _run(cfg, s, cuda, cap=96)
    pr = _posr(s["pos"], prec)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 5.0, prec, cap=96)
    bad = pair_sets_equal(g["counts"], g["ids"], nl[0], nl[1])
    assert bad == -1, f"neighbour pair set of atom {bad} differs"
    ref, _ = oracle_lib.eam_force(pot, pr, s["lo"], s["hi"], 5.0, nl, prec=prec, sum_mode=1)
    err = rel_err(g["force"], ref)
    assert err <= TOL[prec], f"256k EAM force rel err {err:.3e} > {TOL[prec]}"


def test_water_30k_pairs_and_force(cuda, oracle_lib):
    s = systems.water(n_mol=10000, seed=9)
    P = 200
    cfg = systems.water_config(P=P, precision="fp32")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    rc = cfg["hyper_parameters"]["neighbor"]["cut_off"]
    qqr2e = 332.06371
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, 5, 0, 0, P)
    g = _run(cfg, s, cuda, m, cap=640)
    pr = _posr(s["pos"], "fp32")
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], rc, "fp32", cap=640)
    bad = pair_sets_equal(g["counts"], g["ids"], nl[0], nl[1])
    assert bad == -1, f"neighbour pair set of atom {bad} differs"
    near = oracle_lib.near_force(pr, s["lo"], s["hi"], rc, nl, type=s["type"], mol=s["molecule"],
                                 charge=s["charge"], eps=s["eps"], sigma=s["sigma"], with_coul=True, alpha=alpha,
                                 coul_scale=qqr2e, prec="fp32", sum_mode=1)
    far = _kspace(s["pos"], s["charge"], L, alpha, qqr2e, m, oracle=oracle_lib)
    ex, _ = oracle_lib.water_extras(s["hoh"], s["pos"], s["charge"], s["lo"], s["hi"], *s["bond"], *s["angle"])
    ref = near + far + ex
    err = rel_err(g["force"], ref)
    # The k-space rule of the FP32 tests: no larger than the error of the reference's own FP32
    # k-space arithmetic (float cos(k.r) at |k.r| up to ~100 rad in this 67 A box) against FP64.
    far32 = _kspace(pr, s["charge"], L, alpha, qqr2e, m, oracle=oracle_lib, prec="fp32")
    err_ref = rel_err(near + far32 + ex, ref)
    assert err <= max(TOL["fp32"], err_ref), f"30k water force rel err {err:.3e} (reference FP32 k-space {err_ref:.3e})"


def test_lj_4000_fcc_fp64_pairs_force_and_trajectory(cuda, oracle_lib):
    """The CPU-runnable LJ configuration itself: 10^3 FCC cells, rho* 0.8442, T* 0.72, rc 2.5,
    velocity Verlet dt 0.005, FP64.  Pair sets and forces at the start, then 20 NVE steps
    (per-call lists, as the reference) against the oracle's velocity Verlet."""
    import torch
    s = systems.lj_fcc(ncell=10, seed=1)
    assert s["pos"].shape[0] == 4000
    cfg = systems.lj_config(cutoff=2.5, precision="fp64", ensemble="NVE")
    dt = cfg["execution"]["timestep"]
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    c, ids = ff.neighbors(128)
    nl = oracle_lib.neighbors(s["pos"], s["lo"], s["hi"], 2.5, "fp64")
    assert pair_sets_equal(c, ids, nl[0], nl[1]) == -1
    F = oracle_lib.near_force(s["pos"], s["lo"], s["hi"], 2.5, nl, prec="fp64")
    # the perfect lattice: every force vanishes by symmetry (rounding of about 1e-13 left), so the
    # start is checked in absolute terms against the nearest-neighbour pair force (about 4)
    assert np.abs(dev["force"].cpu().numpy() - F).max() <= 1e-11
    x, v = s["pos"].copy(), s["vel"].copy()
    lo, hi = s["lo"], s["hi"]
    m = s["mass"][:, None]
    for _ in range(20):
        v = v + 0.5 * F / m * dt
        x = x + v * dt   # one periodic wrap per axis, as the device's drift
        x = np.where(x < lo, x + (hi - lo), np.where(x > hi, x - (hi - lo), x))
        nl = oracle_lib.neighbors(x, lo, hi, 2.5, "fp64")
        F = oracle_lib.near_force(x, lo, hi, 2.5, nl, prec="fp64")
        v = v + 0.5 * F / m * dt
    ff.step(20)
    torch.cuda.synchronize()
    assert ff.status() == 0
    ff.close()
    assert np.abs(dev["pos"].cpu().numpy() - x).max() < 1e-9
    assert np.abs(dev["vel"].cpu().numpy() - v).max() < 1e-8
    assert rel_err(dev["force"].cpu().numpy(), F) < 1e-9


def test_batched_512_replicas_sample_fp32(cuda, oracle_lib):
    """The 512-replica batch in one launch, each replica with its own injected k-set (P = 100);
    16 replicas, the smallest and the largest among them, against stand-alone oracle runs."""
    r = systems.replicas(n_rep=512, seed=11)
    P = 100
    cfg = systems.electrolyte_config(P=P, precision="fp32", seed=5, ensemble="NVE")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    nrep = len(r["offsets"]) - 1
    assert nrep == 512
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(nrep)]
    ks = np.concatenate([oracle_lib.rbe_sample(alpha, r["hi"][k] - r["lo"][k], 9, 0, k, P) for k in range(nrep)])
    g = _run(cfg, r, cuda, ks, boxes=boxes, offsets=r["offsets"], cap=128)
    off = r["offsets"]
    sizes = np.diff(off)
    pick = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    pick |= set(int(k) for k in np.random.default_rng(2).choice(nrep, 14, replace=False))
    for k in sorted(pick):
        sl = slice(off[k], off[k + 1])
        x = r["pos"][sl]
        lo, hi = r["lo"][k], r["hi"][k]
        pr = _posr(x, "fp32")
        nl = oracle_lib.neighbors(pr, lo, hi, 2.5, "fp32", cap=128)
        # device lists hold caller (global) ids
        bad = pair_sets_equal(g["counts"][sl], g["ids"][sl] - off[k], nl[0], nl[1])
        assert bad == -1, f"replica {k}: neighbour pair set of atom {bad} differs"
        near = oracle_lib.near_force(pr, lo, hi, 2.5, nl, type=r["type"][sl], charge=r["charge"][sl], eps=r["eps"],
                                     sigma=r["sigma"], with_coul=True, alpha=alpha, prec="fp32", sum_mode=1)
        far = _kspace(x, r["charge"][sl], hi - lo, alpha, 1.0, ks[k * P:(k + 1) * P], origin=lo, oracle=oracle_lib)
        err = rel_err(g["force"][sl], near + far)
        assert err <= TOL["fp32"], f"replica {k} ({sizes[k]} atoms): force rel err {err:.3e}"
