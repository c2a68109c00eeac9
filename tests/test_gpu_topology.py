"""GPU parity of the general CVFF topology path (rbmd_force_set_topology) against the oracle.

The total force of flexible chain molecules with ions (REAL units) is compared with the oracle's
near pass (special-bond LJ weights, erfc Coulomb x qqr2e) + RBE far force (injected k-samples)
+ CVFF intramolecular terms (Coulomb correction, bonds, angles, harmonic dihedrals):
max_i |dF_i| / rms|F| <= 1e-5 in FP32 and <= 1e-11 in FP64, for the Verlet list and for RBL
(near part after mean removal), with and without special bonds, and on 5-rings whose special
weights differ by direction (the reference's last-occurrence rule).  The bonded and correction
energies match the oracle's sums, and water given as a general topology reproduces the water
path bit for bit in FP64.
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems
from tests.helpers import make_ff, rel_err, to_dev
from tests.test_topology_host import _ring5

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "fp64": 1e-11}
QQR2E = 332.06371


def _posr(pos, prec):
    return pos.astype(np.float32) if prec == "fp32" else pos.astype(np.float64)


def _run(s, cfg, cuda, m=None):
    import torch
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
                    s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"])
    if m is not None:
        ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    f = dev["force"].cpu().numpy()
    e = ff.energy()
    ff.close()
    return f, e


def _reference(oracle_lib, s, cfg, prec, m, pice=None):
    hp = cfg["hyper_parameters"]
    rc, alpha = hp["neighbor"]["cut_off"], hp["coulomb"]["alpha"]
    wts = hp.get("extend", {}).get("special_bonds")
    n = len(s["pos"])
    sp = oracle_lib.special_lists(n, s["bonds"], wts) if wts is not None else None
    pr = _posr(s["pos"], prec)
    if hp["neighbor"]["type"] == "RBL":
        rs = hp["neighbor"]["r_core"]
        rl = oracle_lib.rbl_list(pr, s["lo"], s["hi"], rc, rs, pice, 400, 400, prec=prec)
        near = oracle_lib.rbl_near(pr, s["lo"], s["hi"], rc, rs, pice, rl, 400, type=s["type"],
                                   mol=s["molecule"], charge=s["charge"], eps=s["eps"], sigma=s["sigma"],
                                   with_coul=True, alpha=alpha, qqr2e=QQR2E, prec=prec, special=sp)
    else:
        nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], rc, prec)
        near = oracle_lib.near_force(pr, s["lo"], s["hi"], rc, nl, type=s["type"], mol=s["molecule"],
                                     charge=s["charge"], eps=s["eps"], sigma=s["sigma"], with_coul=True,
                                     alpha=alpha, coul_scale=QQR2E, prec=prec, special=sp)
    L = s["hi"] - s["lo"]
    rho = oracle_lib.rhok(s["pos"], s["charge"], L, m, prec="fp64")
    far = oracle_lib.rbe_force(s["pos"], s["charge"], L, alpha, QQR2E, m, rho, prec="fp64")
    intra, e = oracle_lib.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"],
                                     s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
                                     s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"],
                                     special=sp)
    return near + far + intra, e


def _ksamples(oracle_lib, s, cfg, seed=4):
    hp = cfg["hyper_parameters"]["coulomb"]
    return oracle_lib.rbe_sample(hp["alpha"], s["hi"] - s["lo"], seed=seed, step=0, rep=0,
                                 P=hp["coulomb_sample_num"])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("special", [(0.0, 0.0, 0.5), None])
def test_topology_verlet_matches_oracle(cuda, oracle_lib, prec, special):
    s = systems.molecular(n_chain=64, chain_len=12, n_ion_pairs=16, seed=21)
    cfg = systems.molecular_config(P=64, precision=prec, special=special)
    m = _ksamples(oracle_lib, s, cfg)
    f, e = _run(s, cfg, cuda, m)
    ref, eref = _reference(oracle_lib, s, cfg, prec, m)
    assert rel_err(f, ref) <= TOL[prec], rel_err(f, ref)
    for k in ("bond", "angle", "dihedral", "coul_special"):
        assert abs(e[k] - eref[k]) <= 1e-9 * max(1.0, abs(eref[k])), (k, e[k], eref[k])
    if special is None:
        assert e["dihedral"] == 0.0


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_topology_rbl_matches_oracle(cuda, oracle_lib, prec):
    """RBL near field with special-bond weights (ComputeNearForceRBLERFSpecialBondsWorklet)."""
    s = systems.molecular(n_chain=125, chain_len=12, n_ion_pairs=40, seed=23)
    cfg = systems.molecular_config(P=64, precision=prec, neighbor="RBL", cutoff=8.0, r_core=4.0, sample_num=60)
    m = _ksamples(oracle_lib, s, cfg)
    import torch
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
                    s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"])
    ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pice = ff.rbl_lists()[2][2]
    assert pice > 1
    f = dev["force"].cpu().numpy()
    ff.close()
    ref, _ = _reference(oracle_lib, s, cfg, prec, m, pice=pice)
    assert rel_err(f, ref) <= TOL[prec], rel_err(f, ref)


def test_topology_ring_direction_dependent_weights(cuda, oracle_lib):
    """5-rings with special_bonds [0, 0.25, 0.5]: w(i, j) != w(j, i) for some pairs (last
    occurrence in the traversal); the GPU reproduces the oracle's direction-dependent forces."""
    s = _ring5(n_ring=27, cell=7.0, seed=6)
    s["vel"] = np.zeros_like(s["pos"])
    cfg = systems.molecular_config(P=32, precision="fp64", special=(0.0, 0.25, 0.5), cutoff=6.0)
    m = _ksamples(oracle_lib, s, cfg)
    f, _ = _run(s, cfg, cuda, m)
    ref, _ = _reference(oracle_lib, s, cfg, "fp64", m)
    assert rel_err(f, ref) <= TOL["fp64"], rel_err(f, ref)


def test_water_as_topology_equals_water_path(cuda):
    """Water given as bonds + angles (no special bonds) takes the general path; its forces equal
    the water-specific path's bit for bit in FP64, apart from the summation order of the bonded
    terms (at most a few ulp)."""
    import torch
    s = systems.water(n_mol=400, seed=5)
    cfg = systems.water_config(P=16, precision="fp64")
    del cfg["hyper_parameters"]["extend"]["special_bonds"]
    cfg["hyper_parameters"]["extend"]["fix_shake"] = "null"
    out = []
    for general in (False, True):
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        if general:
            hoh = s["hoh"]
            bonds = np.concatenate([hoh[:, [0, 1]], hoh[:, [2, 1]]])
            ff.set_topology(s["molecule"], bonds, np.zeros(len(bonds), np.int32), np.array([s["bond"]]), hoh,
                            np.zeros(len(hoh), np.int32), np.array([s["angle"]]))
        ff.Execute()
        torch.cuda.synchronize()
        assert ff.status() == 0
        out.append((dev["force"].cpu().numpy(), ff.energy()))
        ff.close()
    assert rel_err(out[1][0], out[0][0]) <= 1e-13
    for k in ("bond", "angle", "lj", "coul_real"):
        assert abs(out[1][1][k] - out[0][1][k]) <= 1e-12 * max(1.0, abs(out[0][1][k])), k


def test_topology_nve_energy_conservation_fp64(cuda):
    """Flexible chains (bonds, angles, dihedrals, special bonds 0 / 0 / 0.5, intramolecular
    Coulomb correction) with LJ + erfc + Ewald k-space (deterministic), FP64, Verlet skin and
    CUDA-graph steps: 2000 Berendsen steps relax the lattice-grown chains, then 2000 NVE steps of
    0.5 fs keep the total energy (kinetic + LJ + Coulomb real / k-space / self / correction +
    bonded) within 1 % of the kinetic energy of its start value.  A force that is not minus the
    gradient of the energy (a sign, a weight or a missing term) drifts by far more."""
    import copy
    import torch
    s = systems.molecular(n_chain=64, chain_len=12, n_ion_pairs=0, seed=21)
    cfg = systems.molecular_config(precision="fp64", cutoff=10.0, special=(0.0, 0.0, 0.5), dt=0.5)
    cfg["hyper_parameters"]["coulomb"] = {"type": "EWALD", "alpha": 0.09, "kmax": 6}
    cfg["hyper_parameters"]["neighbor"]["skin"] = 1.0
    nvt = copy.deepcopy(cfg)
    nvt["execution"].update({"ensemble": "NVT", "temp_ctrl_type": "BERENDSEN", "temperature": [298.0, 298.0, 10.0]})
    dev = to_dev(s, cuda)
    topo = (s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
            s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"])
    ff = make_ff(nvt, s, dev)
    ff.set_topology(*topo)
    ff.Execute()
    ff.step(2000)
    ff.sync_velocities()
    torch.cuda.synchronize()
    assert ff.status() == 0
    ff.close()
    ff = make_ff(cfg, s, dev)
    ff.set_topology(*topo)
    keys = ("lj", "coul_real", "coul_kspace", "coul_self", "bond", "angle", "dihedral", "coul_special")

    def total():
        ff.step(1)
        ff.Execute()
        e = ff.energy()
        return e["kinetic"] + sum(e[k] for k in keys), e

    e0, d0 = total()
    assert all(d0[k] != 0.0 for k in keys), d0
    for _ in range(4):
        ff.step(500)
        torch.cuda.synchronize()
        assert ff.status() == 0
        e, d = total()
        assert abs(e - e0) <= 1e-2 * d0["kinetic"], (e, e0, d0["kinetic"], d)
    ff.close()


def test_topology_original_neighbor_type(cuda, oracle_lib):
    """neighbor.type "ORIGINAL" with special bonds (ComputeSpecialBondsLJWorklet, RunWorklet.cpp:
    570-632): pairs d^2 < rc^2 with special-bond LJ weights, FP64, against the oracle."""
    s = systems.molecular(n_chain=64, chain_len=12, n_ion_pairs=16, seed=28)
    cfg = systems.molecular_config(P=32, precision="fp64", special=(0.0, 0.0, 0.5))
    cfg["hyper_parameters"]["neighbor"]["type"] = "ORIGINAL"
    m = _ksamples(oracle_lib, s, cfg)
    f, _ = _run(s, cfg, cuda, m)
    hp = cfg["hyper_parameters"]
    rc, alpha = hp["neighbor"]["cut_off"], hp["coulomb"]["alpha"]
    sp = oracle_lib.special_lists(len(s["pos"]), s["bonds"], [0.0, 0.0, 0.5])
    nl = oracle_lib.neighbors(s["pos"], s["lo"], s["hi"], rc, "fp64", original=True)
    near = oracle_lib.near_force(s["pos"], s["lo"], s["hi"], rc, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                                 sigma=s["sigma"], with_coul=True, alpha=alpha, coul_scale=QQR2E, prec="fp64",
                                 special=sp)
    L = s["hi"] - s["lo"]
    far = oracle_lib.rbe_force(s["pos"], s["charge"], L, alpha, QQR2E, m, oracle_lib.rhok(s["pos"], s["charge"], L, m))
    intra, _ = oracle_lib.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"], s["bond_type"],
                                     s["bond_coeffs"], s["angles"], s["angle_type"], s["angle_coeffs"], s["dihedrals"],
                                     s["dihedral_type"], s["dihedral_coeffs"], special=sp)
    assert rel_err(f, near + far + intra) <= TOL["fp64"]


def test_topology_batched_replicas_equal_single(cuda):
    """Two molecular replicas of different sizes and boxes in one batch (Ewald k-space, so both
    runs use the same k-vectors): the bonded terms, special weights and Coulomb correction of
    each replica equal the single-replica run's forces (FP64)."""
    import torch
    from copy_gpu_b200 import Box
    sa = systems.molecular(n_chain=27, chain_len=10, n_ion_pairs=4, seed=31)
    sb = systems.molecular(n_chain=64, chain_len=8, n_ion_pairs=8, seed=32)
    cfg = systems.molecular_config(precision="fp64", cutoff=8.0, special=(0.0, 0.0, 0.5))
    cfg["hyper_parameters"]["coulomb"] = {"type": "EWALD", "alpha": 0.09, "kmax": 3}
    topo_keys = ("bonds", "bond_type", "bond_coeffs", "angles", "angle_type", "angle_coeffs", "dihedrals",
                 "dihedral_type", "dihedral_coeffs")

    def single(s):
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        ff.set_topology(s["molecule"], *[s[k] for k in topo_keys])
        ff.Execute()
        torch.cuda.synchronize()
        assert ff.status() == 0
        f = dev["force"].cpu().numpy()
        ff.close()
        return f

    fa, fb = single(sa), single(sb)
    na = len(sa["pos"])
    b = {k: np.concatenate([sa[k], sb[k]]) for k in ("pos", "vel", "mass", "charge", "type")}
    b["molecule"] = np.concatenate([sa["molecule"], sb["molecule"] + sa["molecule"].max() + 1]).astype(np.int32)
    b.update(eps=sa["eps"], sigma=sa["sigma"], lo=sa["lo"], hi=sa["hi"])
    offs = np.array([0, na, na + len(sb["pos"])])
    boxes = [Box(tuple(sa["lo"]), tuple(sa["hi"])), Box(tuple(sb["lo"]), tuple(sb["hi"]))]
    dev = to_dev(b, cuda)
    ff = make_ff(cfg, b, dev, boxes=boxes, offsets=offs)
    ff.set_topology(b["molecule"], np.concatenate([sa["bonds"], sb["bonds"] + na]),
                    np.concatenate([sa["bond_type"], sb["bond_type"]]), sa["bond_coeffs"],
                    np.concatenate([sa["angles"], sb["angles"] + na]),
                    np.concatenate([sa["angle_type"], sb["angle_type"]]), sa["angle_coeffs"],
                    np.concatenate([sa["dihedrals"], sb["dihedrals"] + na]),
                    np.concatenate([sa["dihedral_type"], sb["dihedral_type"]]), sa["dihedral_coeffs"])
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    f = dev["force"].cpu().numpy()
    ff.close()
    assert rel_err(f[:na], fa) <= 1e-12 and rel_err(f[na:], fb) <= 1e-12


def test_topology_needs_cvff(cuda):
    """Only force_field CVFF carries bonded terms: set_topology on LJ/CUT/COUL/LONG is an error,
    not a silent no-op."""
    from copy_gpu_b200 import Box, ForceField, RbmdError
    s = systems.molecular(n_chain=8, chain_len=6, n_ion_pairs=2, seed=33)
    cfg = systems.molecular_config(precision="fp64")
    cfg["hyper_parameters"]["force_field"]["type"] = "LJ/CUT/COUL/LONG"
    ff = ForceField(cfg, Box(tuple(s["lo"]), tuple(s["hi"])))
    with pytest.raises(RbmdError):
        ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"])
    ff.close()


def test_special_bonds_integer_compat(cuda):
    """compat.special_bonds_integer reads extend.special_bonds as the reference does (integers:
    [0, 0, 0.5] acts as [0, 0, 0]); by default the 0.5 weight reaches the 1-4 LJ pairs."""
    s = systems.molecular(n_chain=27, chain_len=8, n_ion_pairs=4, seed=34)
    f = {}
    for name, special, compat in (("half", (0.0, 0.0, 0.5), False), ("zero", (0.0, 0.0, 0.0), False),
                                  ("compat", (0.0, 0.0, 0.5), True)):
        cfg = systems.molecular_config(P=8, precision="fp64", special=special)
        if compat:
            cfg["compat"] = {"special_bonds_integer": True}
        m = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1], [2, 0, 0]],
                     np.int32)
        f[name], _ = _run(s, cfg, cuda, m)
    assert np.array_equal(f["compat"], f["zero"])
    assert not np.array_equal(f["half"], f["zero"])


def test_water_special_bonds_zero_equals_exclusion_rbl(cuda):
    """The reference's H2O example shape (CVFF, RBL, special_bonds [0, 0, 0], rbmd/examples/H2O):
    water given as a general topology takes the special-bond path, where every intramolecular
    pair is a 1-2 or 1-3 partner with weight 0; its forces equal those of the molecule-exclusion
    water path to summation order (FP64)."""
    import torch
    s = systems.water(n_mol=400, seed=6)
    out = []
    for general in (False, True):
        cfg = systems.water_config(P=16, precision="fp64")
        cfg["hyper_parameters"]["neighbor"] = {"type": "RBL", "cut_off": 10.0, "r_core": 5.0,
                                               "neighbor_sample_num": 100}
        if not general:
            del cfg["hyper_parameters"]["extend"]["special_bonds"]
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        if general:
            hoh = s["hoh"]
            bonds = np.concatenate([hoh[:, [0, 1]], hoh[:, [2, 1]]])
            ff.set_topology(s["molecule"], bonds, np.zeros(len(bonds), np.int32), np.array([s["bond"]]), hoh,
                            np.zeros(len(hoh), np.int32), np.array([s["angle"]]))
        ff.Execute()
        torch.cuda.synchronize()
        assert ff.status() == 0
        out.append(dev["force"].cpu().numpy())
        ff.close()
    assert rel_err(out[1], out[0]) <= 1e-12
