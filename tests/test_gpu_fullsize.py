"""Size-independent properties at the benchmark sizes (the oracle is too slow there):

* Newton's third law: the total force of the 1,000,000-atom electrolyte (LJ + erfc near + RBE
  k-space with injected samples), of the 256,000-atom EAM crystal and of every replica of the
  512-replica batch sums to zero up to rounding (pair terms are exact negatives of each other;
  the RBE sum cancels as Re(rho) Im(rho) - Im(rho) Re(rho));
* translation invariance: shifting every atom by the same vector (wrapped into the box) gives
  the same forces, although cells, slots, list order and fixed-point phases all change.  In FP64
  runs to 1e-9; in FP32 runs the positions themselves round differently once shifted (an ulp of
  a 100-sigma coordinate is 8e-6 sigma, and r^-13 pair forces of close contacts amplify it), so
  the bar is 2e-3 there, and 5e-3 for the EAM crystal, whose forces at its equilibrium lattice
  constant come from the thermal displacements alone (rms 0.5 eV/A) while the rounding of 144 A
  coordinates (1.5e-5 A) times the pair curvature stays the same; a cell, slot or list error
  would be of order one;
* momentum conservation: NVE steps of the batch keep every replica's momentum.
"""
import numpy as np
import pytest

from copy_gpu_b200 import Box, systems
from tests.helpers import make_ff, rel_err, to_dev

pytestmark = pytest.mark.gpu

SHIFT = np.array([0.37, 1.91, 2.53])


def _shifted(s, shift):
    t = dict(s)
    lo, hi = np.asarray(s["lo"]), np.asarray(s["hi"])
    t["pos"] = lo + np.mod(s["pos"] + shift - lo, hi - lo)
    return t


def _forces(cfg, s, cuda, m=None, boxes=None, offsets=None):
    import torch
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev, boxes=boxes, offsets=offsets)
    if m is not None:
        ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    f = dev["force"].cpu().numpy()
    ff.close()
    return f


def _net(f):
    return np.abs(f.sum(0)).max() / np.sqrt((f ** 2).sum(1)).sum()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_electrolyte_1m_newton_and_translation(cuda, oracle_lib, prec):
    s = systems.electrolyte(1_000_000, seed=3)
    P = 500
    cfg = systems.electrolyte_config(P=P, precision=prec, seed=5, ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    m = oracle_lib.rbe_sample(alpha, s["hi"] - s["lo"], 7, 0, 0, P)
    f0 = _forces(cfg, s, cuda, m)
    assert _net(f0) < 1e-7, _net(f0)
    f1 = _forces(cfg, _shifted(s, SHIFT), cuda, m)
    assert rel_err(f1, f0) < (2e-3 if prec == "fp32" else 1e-9), rel_err(f1, f0)


def test_eam_256k_newton_and_translation(cuda, tmp_path):
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=40, seed=13)
    cfg = systems.eam_config(pot, precision="fp32")
    f0 = _forces(cfg, s, cuda)
    assert _net(f0) < 1e-7, _net(f0)
    f1 = _forces(cfg, _shifted(s, SHIFT), cuda)
    assert rel_err(f1, f0) < 5e-3, rel_err(f1, f0)


def test_batched_512_newton_and_momentum(cuda):
    import torch
    r = systems.replicas(n_rep=512, seed=11)
    cfg = systems.electrolyte_config(P=100, precision="fp32", seed=5, ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(512)]
    off = r["offsets"]
    dev = to_dev(r, cuda)
    ff = make_ff(cfg, r, dev, boxes=boxes, offsets=off)
    ff.Execute()
    torch.cuda.synchronize()
    f = dev["force"].cpu().numpy()
    worst = max(_net(f[off[k]:off[k + 1]]) for k in range(512))
    assert worst < 1e-6, worst
    mass = r["mass"][:, None]
    p0 = np.add.reduceat(mass * dev["vel"].cpu().numpy(), off[:-1], axis=0)
    ff.step(10)
    torch.cuda.synchronize()
    assert ff.status() == 0
    p1 = np.add.reduceat(mass * dev["vel"].cpu().numpy(), off[:-1], axis=0)
    scale = np.add.reduceat(mass[:, 0] * np.linalg.norm(dev["vel"].cpu().numpy(), axis=1), off[:-1])
    drift = (np.abs(p1 - p0).max(1) / scale).max()
    assert drift < 1e-7, drift
