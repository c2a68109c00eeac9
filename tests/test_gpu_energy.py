"""Thermo energies of rbmd_force_energy against independent restatements (FP64 runs).

The reference reports per-atom averages in ThermoOutput (rbmd/framework/output/ThermoOutput.cpp:
152-300); the library returns totals, so each term here is the reference's sum before its
division by N:
* LJ: 0.5 sum_{i != j} 4 eps (s^6 - 1) s^6 over minimum-image pairs with d^2 < rc^2, d^2 > 1e-4,
  same-molecule pairs skipped (ExecForceFunction.h:296-312, OutPutWorklet.cpp:139-188);
* real-space Coulomb: 0.5 sum q_i q_j erfc(sqrt(alpha) d) / d for 0.01 < d < rc
  (ExecForceFunction.h:315-329), times qqr2e;
* self: -sqrt(alpha / pi) qqr2e sum q^2 (ThermoOutput.cpp:208-215);
* k-space with the EWALD cube: (2 pi / V) qqr2e sum_{m in [-K, K]^3, m != 0} e^{-k^2/4 alpha}
  |rho(k)|^2 / k^2 (ThermoOutput.cpp:218-252); with RBE the per-step estimate
  (S/P) sum_l (2 pi / V) |rho_l|^2 / k_l^2 is unbiased for the converged Ewald k-space energy;
* kinetic 0.5 sum m v^2 mvv2e and T = 2 KE / ((3N - 3) kB) (ExecutionNVT.cpp:749-786);
* EAM embedding + pair against the oracle's FP64 EAM energy; water bond and angle energies
  against the oracle's harmonic terms.
"""
import math

import numpy as np
import pytest

from copy_gpu_b200 import systems
from tests.helpers import make_ff, to_dev

pytestmark = pytest.mark.gpu


def _min_image_pairs(pos, L, rc):
    d = pos[None, :, :] - pos[:, None, :]
    d -= L * np.round(d / L)
    d2 = (d ** 2).sum(-1)
    return d2, (d2 < rc * rc) & (d2 > 1e-4)


def _electrolyte(cuda, n, coulomb, P, kmax=2, seed=21):
    s = systems.electrolyte(n, seed=seed)
    cfg = systems.electrolyte_config(P=P, precision="fp64", ensemble="NVE", dt=0.0, coulomb=coulomb,
                                     kmax=kmax, seed=seed)
    cfg["outputs"] = {"thermo_out": {"interval": 1}}
    dev = to_dev(s, cuda)
    return s, cfg, dev, make_ff(cfg, s, dev)


def test_electrolyte_energies_ewald_cube(cuda, oracle_lib):
    from scipy.special import erfc
    import torch
    n, K = 1500, 3
    s, cfg, dev, ff = _electrolyte(cuda, n, "EWALD", P=1, kmax=K)
    ff.Execute()
    ff.step(1)
    torch.cuda.synchronize()
    assert ff.status() == 0
    e = ff.energy()
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    rc = cfg["hyper_parameters"]["neighbor"]["cut_off"]
    L = s["hi"] - s["lo"]
    x, q = s["pos"], s["charge"]
    d2, m = _min_image_pairs(x, L, rc)
    inv6 = np.where(m, 1.0 / np.where(m, d2, 1.0) ** 3, 0.0)
    e_lj = 0.5 * (4.0 * (inv6 - 1.0) * inv6)[m].sum()
    assert abs(e["lj"] - e_lj) <= 1e-10 * abs(e_lj), (e["lj"], e_lj)
    d = np.sqrt(d2)
    mc = (d < rc) & (d > 0.01)
    qq = q[:, None] * q[None, :]
    e_real = 0.5 * (qq * erfc(math.sqrt(alpha) * np.where(mc, d, 1.0)) / np.where(mc, d, 1.0))[mc].sum()
    assert abs(e["coul_real"] - e_real) <= 1e-10 * abs(e_real) + 1e-12, (e["coul_real"], e_real)
    assert abs(e["coul_self"] + math.sqrt(alpha / math.pi) * (q * q).sum()) < 1e-9
    r = np.arange(-K, K + 1)
    mk = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    mk = mk[np.any(mk != 0, axis=1)].astype(np.int32)
    rho = oracle_lib.rhok(x, q, L, mk)
    k = 2 * np.pi * mk / L
    k2 = (k ** 2).sum(1)
    e_k = 2 * np.pi / np.prod(L) * (np.exp(-k2 / (4 * alpha)) * (rho ** 2).sum(1) / k2).sum()
    assert abs(e["coul_kspace"] - e_k) <= 1e-10 * abs(e_k), (e["coul_kspace"], e_k)
    ke = 0.5 * (s["mass"][:, None] * s["vel"] ** 2).sum()
    assert abs(e["kinetic"] - ke) <= 1e-12 * ke
    assert abs(e["temperature"] - 2 * ke / (3 * n - 3)) <= 1e-12 * e["temperature"]


def test_rbe_kspace_energy_unbiased(cuda, oracle_lib):
    import torch
    n, P, nsteps = 1500, 100, 400
    s, cfg, dev, ff = _electrolyte(cuda, n, "RBE", P=P, seed=23)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    _, e_ref = oracle_lib.ewald_kspace(s["pos"], s["charge"], L, alpha, kcut=2 * np.sqrt(alpha) * 6.2)
    ff.Execute()
    vals = []
    for _ in range(nsteps):
        ff.step(1)
        torch.cuda.synchronize()
        vals.append(ff.energy()["coul_kspace"])
    assert ff.status() == 0
    vals = np.array(vals)
    se = vals.std(ddof=1) / math.sqrt(nsteps)
    assert abs(vals.mean() - e_ref) <= 4 * se, (vals.mean(), e_ref, se)


def test_eam_energy_matches_oracle(cuda, oracle_lib, tmp_path):
    import torch
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=6, seed=7)
    cfg = systems.eam_config(pot, precision="fp64")
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    e = ff.energy()
    nl = oracle_lib.neighbors(s["pos"], s["lo"], s["hi"], 5.0, "fp64")
    ref = oracle_lib.eam_energy(pot, s["pos"], s["lo"], s["hi"], 5.0, nl)
    got = e["eam_embed"] + e["eam_pair"]
    assert abs(got - ref) <= 1e-10 * abs(ref), (got, ref)


def test_water_bond_angle_energies(cuda, oracle_lib):
    import torch
    s = systems.water(n_mol=200, seed=4)
    cfg = systems.water_config(P=16, precision="fp64")
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    e = ff.energy()
    _, (eb, ea) = oracle_lib.water_extras(s["hoh"], s["pos"], s["charge"], s["lo"], s["hi"], *s["bond"],
                                          *s["angle"])
    assert abs(e["bond"] - eb) <= 1e-10 * abs(eb) + 1e-12, (e["bond"], eb)
    assert abs(e["angle"] - ea) <= 1e-10 * abs(ea) + 1e-12, (e["angle"], ea)
    # energy of the removed intramolecular bare Coulomb pairs (ComputeSpecialCoulWorklet)
    hoh = s["hoh"]
    bonds = np.concatenate([hoh[:, [0, 1]], hoh[:, [2, 1]]])
    _, eo = oracle_lib.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], bonds,
                                  np.zeros(len(bonds), np.int32), np.array([s["bond"]]), hoh,
                                  np.zeros(len(hoh), np.int32), np.array([s["angle"]]))
    assert abs(e["coul_special"] - eo["coul_special"]) <= 1e-10 * abs(eo["coul_special"]), \
        (e["coul_special"], eo["coul_special"])
