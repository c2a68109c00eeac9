"""GPU parity of the RBL near field (neighbor.type "RBL") against the CPU oracle.

Bars:
* lists: per atom the core pairs and the kept shell pairs equal the oracle's, in the same order
  (the reference's traversal order decides which shell pairs are kept), FP32 and FP64;
* pice_num and the reference's rs_num / rc_num equal the oracle's;
* forces (near part after mean removal, plus the RBE far part with injected k-samples):
  max_i |dF_i| / rms|F| <= 1e-5 in FP32 and <= 1e-11 in FP64, in the default mode (G at the
  configured alpha, shell Coulomb x pice) and with the reference's ERF table and dropped shell
  Coulomb (compat flags);
* EAM over RBL lists, and the Verlet EAM force with the reference's reversed pair vector.
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems
from tests.helpers import make_ff, rel_err, to_dev

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "fp64": 1e-11}
RS, RC, SAMPLE = 1.25, 2.5, 10


def _posr(pos, prec):
    return pos.astype(np.float32) if prec == "fp32" else pos.astype(np.float64)


def _rbl_cfg(prec, compat=None, P=32):
    cfg = systems.electrolyte_config(P=P, precision=prec)
    cfg["hyper_parameters"]["neighbor"] = {"type": "RBL", "cut_off": RC, "r_core": RS,
                                           "neighbor_sample_num": SAMPLE}
    if compat:
        cfg["compat"] = compat
    return cfg


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_rbl_lists_match_oracle(cuda, oracle_lib, prec):
    import torch
    s = systems.electrolyte(3000, seed=21)
    cfg = _rbl_cfg(prec)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    m = oracle_lib.rbe_sample(alpha, s["hi"] - s["lo"], seed=3, step=0, rep=0, P=32)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    ncore, nshell, sizes = ff.rbl_lists()
    rs_num, rc_num, pice = oracle_lib.rbl_sizes(len(s["pos"]), s["lo"], s["hi"], RS, RC, SAMPLE, prec=prec)
    assert sizes[:3] == (rs_num, rc_num, pice)
    assert pice > 1
    pr = _posr(s["pos"], prec)
    oc, osh, oids, _ = oracle_lib.rbl_list(pr, s["lo"], s["hi"], RC, RS, pice, 96, 96, prec=prec)
    assert np.array_equal(ncore, oc) and np.array_equal(nshell, osh)
    cap = int((ncore + nshell).max()) + 1
    counts, ids = ff.neighbors(cap)
    for i in range(len(pr)):
        ref = np.concatenate([oids[i, :oc[i]], oids[i, 96:96 + osh[i]]])
        assert np.array_equal(ids[i, :counts[i]], ref), f"atom {i}"


@pytest.mark.parametrize("prec,compat", [("fp32", None), ("fp64", None),
                                         ("fp32", {"rbl_erf_table": True, "rbl_drop_shell_coulomb": True}),
                                         ("fp64", {"rbl_drop_shell_coulomb": True})])
def test_rbl_force_matches_oracle(cuda, oracle_lib, prec, compat):
    import torch
    s = systems.electrolyte(3000, seed=22)
    P = 48
    cfg = _rbl_cfg(prec, compat, P=P)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, seed=8, step=0, rep=0, P=P)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pice = ff.rbl_lists()[2][2]
    pr = _posr(s["pos"], prec)
    rl = oracle_lib.rbl_list(pr, s["lo"], s["hi"], RC, RS, pice, 96, 96, prec=prec)
    compat = compat or {}
    near = oracle_lib.rbl_near(pr, s["lo"], s["hi"], RC, RS, pice, rl, 96, type=s["type"], charge=s["charge"],
                               eps=s["eps"], sigma=s["sigma"], with_coul=True, alpha=alpha, qqr2e=1.0,
                               table_mode=int(compat.get("rbl_erf_table", False)),
                               shell_coul=0 if compat.get("rbl_drop_shell_coulomb") else 1, prec=prec)
    rho = oracle_lib.rhok(s["pos"], s["charge"], L, m, prec="fp64")
    far = oracle_lib.rbe_force(s["pos"], s["charge"], L, alpha, 1.0, m, rho, prec="fp64")
    err = rel_err(dev["force"].cpu().numpy(), near + far)
    assert err <= TOL[prec], f"RBL total force rel err {err:.3e}"


def test_rbl_lj_only_mean_removed(cuda, oracle_lib):
    """LJ/CUT over RBL lists (ComputeLJForceRBLWorklet): forces match and sum to zero."""
    import torch
    s = systems.lj_fcc(ncell=8, seed=6)
    cfg = systems.lj_config(cutoff=RC, precision="fp32")
    cfg["hyper_parameters"]["neighbor"] = {"type": "RBL", "cut_off": RC, "r_core": RS, "neighbor_sample_num": 12}
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pice = ff.rbl_lists()[2][2]
    pr = s["pos"].astype(np.float32)
    rl = oracle_lib.rbl_list(pr, s["lo"], s["hi"], RC, RS, pice, 96, 96)
    ref = oracle_lib.rbl_near(pr, s["lo"], s["hi"], RC, RS, pice, rl, 96)
    got = dev["force"].cpu().numpy()
    assert rel_err(got, ref) <= 1e-5
    assert np.abs(got.sum(0)).max() <= 1e-9 * len(got) * np.abs(got).max()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_rbl_eam_matches_oracle(cuda, oracle_lib, tmp_path, prec):
    import torch
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=8, seed=7)
    cfg = systems.eam_config(pot, precision=prec)
    cfg["hyper_parameters"]["neighbor"] = {"type": "RBL", "cut_off": 5.0, "r_core": 3.0, "neighbor_sample_num": 20}
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pice = ff.rbl_lists()[2][2]
    rs_num, rc_num, pice_ref = oracle_lib.rbl_sizes(len(s["pos"]), s["lo"], s["hi"], 3.0, 5.0, 20, eam=True, prec=prec)
    assert pice == pice_ref and pice > 1
    pr = _posr(s["pos"], prec)
    rl = oracle_lib.rbl_list(pr, s["lo"], s["hi"], 5.0, 3.0, pice, 96, 96, prec=prec)
    ref, _ = oracle_lib.rbl_eam(pot, pr, s["lo"], s["hi"], 5.0, 3.0, pice, rl, 96, prec=prec)
    err = rel_err(dev["force"].cpu().numpy(), ref)
    assert err <= (1e-5 if prec == "fp32" else 1e-11), err


def test_eam_verlet_reference_pair_vector(cuda, oracle_lib, tmp_path):
    """compat.eam_verlet_pair_vector reproduces the reference's reversed Verlet EAM force."""
    import torch
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=6, seed=5)
    cfg = systems.eam_config(pot, precision="fp64")
    cfg["compat"] = {"eam_verlet_pair_vector": True}
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    nl = oracle_lib.neighbors(s["pos"], s["lo"], s["hi"], 5.0, "fp64")
    ref, _ = oracle_lib.eam_force(pot, s["pos"], s["lo"], s["hi"], 5.0, nl, prec="fp64", ref_sign=True)
    assert rel_err(dev["force"].cpu().numpy(), ref) <= 1e-11


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("system", ["electrolyte", "molecular"])
def test_rbl_warp_list_identical(cuda, prec, system):
    """tuning.rbl_list "warp" (one warp per atom over the flattened stencil, ballot-ordered shell
    selection) and "thread" (one thread per atom) build identical lists, entry for entry, and so
    identical forces; the molecular case has 125-cell stencils (num_cycles 2) and special bonds."""
    import torch
    if system == "electrolyte":
        s = systems.electrolyte(3000, seed=24)
        base = _rbl_cfg(prec)
    else:
        s = systems.molecular(n_chain=343, chain_len=12, n_ion_pairs=40, step=1.5, cell=6.0, seed=25)
        base = systems.molecular_config(P=32, precision=prec, neighbor="RBL", cutoff=12.0, r_core=6.0,
                                        sample_num=100, special=(0.0, 0.0, 0.0))
    out = []
    for mode in ("thread", "warp"):
        cfg = dict(base)
        cfg["tuning"] = {"rbl_list": mode}
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        if system == "molecular":
            ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"],
                            s["angle_type"], s["angle_coeffs"], s["dihedrals"], s["dihedral_type"],
                            s["dihedral_coeffs"])
        ff.Execute()   # the device sampler draws the same seeded k-set in both runs
        torch.cuda.synchronize()
        assert ff.status() == 0
        ncore, nshell, sizes = ff.rbl_lists()
        counts, ids = ff.neighbors(int((ncore + nshell).max()) + 1)
        out.append((ncore, nshell, counts, ids, dev["force"].cpu().numpy()))
        ff.close()
    assert out[1][0].sum() > 0 and out[1][1].sum() > 0
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
def test_rbl_force_lanes_parity(cuda, oracle_lib, lanes):
    """tuning.rbl_lanes G > 1 (G lanes per atom, FP64 butterfly of the lane sums) equals one
    thread per atom to summation-order rounding in FP64 (molecular system with special bonds),
    and the FP32 electrolyte matches the oracle."""
    import torch
    s = systems.molecular(n_chain=343, chain_len=12, n_ion_pairs=40, step=1.5, cell=6.0, seed=26)
    forces = []
    for g in (1, lanes):
        cfg = systems.molecular_config(P=16, precision="fp64", neighbor="RBL", cutoff=12.0, r_core=6.0,
                                       sample_num=100, special=(0.0, 0.0, 0.5))
        cfg["tuning"] = {"rbl_lanes": g}
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        ff.set_topology(s["molecule"], s["bonds"], s["bond_type"], s["bond_coeffs"], s["angles"], s["angle_type"],
                        s["angle_coeffs"], s["dihedrals"], s["dihedral_type"], s["dihedral_coeffs"])
        ff.Execute()
        torch.cuda.synchronize()
        assert ff.status() == 0
        forces.append(dev["force"].cpu().numpy())
        ff.close()
    assert rel_err(forces[1], forces[0]) < 1e-12
    se = systems.electrolyte(3000, seed=27)
    P = 32
    cfg = _rbl_cfg("fp32", P=P)
    cfg["tuning"] = {"rbl_lanes": lanes, "rbl_list": "thread"}
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = se["hi"] - se["lo"]
    m = oracle_lib.rbe_sample(alpha, L, seed=9, step=0, rep=0, P=P)
    dev = to_dev(se, cuda)
    ff = make_ff(cfg, se, dev)
    ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pice = ff.rbl_lists()[2][2]
    f = dev["force"].cpu().numpy()
    ff.close()
    pr = _posr(se["pos"], "fp32")
    rl = oracle_lib.rbl_list(pr, se["lo"], se["hi"], RC, RS, pice, 96, 96, prec="fp32")
    near = oracle_lib.rbl_near(pr, se["lo"], se["hi"], RC, RS, pice, rl, 96, type=se["type"], charge=se["charge"],
                               eps=se["eps"], sigma=se["sigma"], with_coul=True, alpha=alpha, qqr2e=1.0, prec="fp32")
    rho = oracle_lib.rhok(se["pos"], se["charge"], L, m, prec="fp64")
    far = oracle_lib.rbe_force(se["pos"], se["charge"], L, alpha, 1.0, m, rho, prec="fp64")
    assert rel_err(f, near + far) <= TOL["fp32"]


@pytest.mark.parametrize("mode", ["thread", "warp"])
def test_rbl_lists_atoms_outside_box(cuda, oracle_lib, mode):
    """Atoms up to one r_core outside the box are binned into the boundary cells; the list builds
    skip stencil cells beyond rc from the atom, with boundary cells open on their outer side, so
    the lists still equal the oracle's entry for entry."""
    import torch
    rng = np.random.default_rng(12)
    L = 12.0
    n = 2000
    pos = rng.uniform(0, L, size=(n, 3))
    pos[:150] += rng.uniform(-RS, RS, size=(150, 3))
    s = dict(pos=pos, vel=np.zeros_like(pos), mass=np.ones(n), charge=np.zeros(n), type=np.zeros(n, np.int32),
             molecule=None, lo=np.zeros(3), hi=np.full(3, L), eps=np.ones(1), sigma=np.ones(1))
    cfg = systems.lj_config(cutoff=RC, precision="fp32")
    cfg["hyper_parameters"]["neighbor"] = {"type": "RBL", "cut_off": RC, "r_core": RS, "neighbor_sample_num": SAMPLE}
    cfg["tuning"] = {"rbl_list": mode}
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    ncore, nshell, sizes = ff.rbl_lists()
    pice = sizes[2]
    pr = pos.astype(np.float32)
    oc, osh, oids, _ = oracle_lib.rbl_list(pr, s["lo"], s["hi"], RC, RS, pice, 96, 96)
    assert np.array_equal(ncore, oc) and np.array_equal(nshell, osh)
    counts, ids = ff.neighbors(int((ncore + nshell).max()) + 1)
    for i in range(n):
        ref = np.concatenate([oids[i, :oc[i]], oids[i, 96:96 + osh[i]]])
        assert np.array_equal(ids[i, :counts[i]], ref), f"atom {i}"
    ff.close()
