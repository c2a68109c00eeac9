"""LAMMPS data files through the C ABI (rbmd_data_read / rbmd_data_write): exact round trips in
every atom style, the reference's conventions (1-based ids stored by id, LJ masses forced to 1),
malformed files rejected with RBMD_ERR_FILE, and the reference's own example inputs (read when the
reference checkout is present; their JSON configurations are accepted by rbmd_force_create)."""
import os

import numpy as np
import pytest

import copy_gpu_b200 as c
from copy_gpu_b200 import systems

REF = os.path.join(os.environ.get("RBMD_REFERENCE", "/root/reference"), "rbmd", "res", "json_files")


@pytest.mark.parametrize("style", ["atomic", "charge", "full"])
def test_roundtrip_exact(tmp_path, style):
    rng = np.random.default_rng(1)
    n = 97
    d = dict(pos=rng.uniform(-1, 9, (n, 3)), vel=rng.normal(size=(n, 3)), charge=rng.normal(size=n),
             type=rng.integers(0, 3, n).astype(np.int32), molecule=rng.integers(0, 20, n).astype(np.int32),
             image=rng.integers(-2, 3, (n, 3)).astype(np.int32), mass_by_type=np.array([1.5, 2.0, 16.0]),
             eps=np.array([0.1, 0.2, 0.3]), sigma=np.array([1.0, 2.0, 3.0]), lo=np.array([-1.0, -1, -1]),
             hi=np.array([9.0, 9.5, 10.0]), bonds=rng.integers(0, n, (30, 2)).astype(np.int32),
             angles=rng.integers(0, n, (10, 3)).astype(np.int32))
    p = tmp_path / f"{style}.data"
    c.write_data(p, style, d)
    r = c.read_data(p, style, unit="REAL")
    assert np.array_equal(r["pos"], d["pos"]) and np.array_equal(r["vel"], d["vel"])
    assert np.array_equal(r["type"], d["type"]) and np.array_equal(r["image"], d["image"])
    if style != "atomic":
        assert np.array_equal(r["charge"], d["charge"])
    if style == "full":
        assert np.array_equal(r["molecule"], d["molecule"])
    assert np.array_equal(r["mass"], d["mass_by_type"][d["type"]])
    assert np.array_equal(r["eps"], d["eps"]) and np.array_equal(r["sigma"], d["sigma"])
    assert np.array_equal(r["bonds"], d["bonds"]) and np.array_equal(r["angles"], d["angles"])
    assert np.array_equal(r["lo"], d["lo"]) and np.array_equal(r["hi"], d["hi"])
    lj = c.read_data(p, style, unit="LJ")
    assert np.all(lj["mass"] == 1.0)                 # ModelFileInitCondition.cpp:293-298


def test_malformed_files_rejected(tmp_path):
    p = tmp_path / "bad.data"
    p.write_text("title\n\n3 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n1 1 0 0 0\n7 1 0 0 0\n")
    with pytest.raises(c.RbmdError, match="ERR_FILE"):
        c.read_data(p, "atomic")
    with pytest.raises(c.RbmdError, match="ERR_FILE"):
        c.read_data(tmp_path / "missing.data", "atomic")


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout absent")
def test_reference_example_inputs():
    w = c.read_data(os.path.join(REF, "H2O", "rbmd.data"), "full", unit="REAL")
    assert len(w["pos"]) == 300 and len(w["bonds"]) == 200 and len(w["angles"]) == 100
    assert np.allclose(w["mass_by_type"], [15.9994, 1.008])
    assert np.allclose(w["eps"], [0.1553, 0.0]) and np.allclose(w["sigma"], [3.166, 0.0])
    # first Atoms line of the file: "39 13 2 0.41 6.461243940069542 8.25774974714983 5.247946382705338 0 0 0"
    assert w["type"][38] == 1 and w["molecule"][38] == 12 and w["charge"][38] == 0.41
    assert w["pos"][38][0] == 6.461243940069542
    assert abs(w["charge"].sum()) < 1e-9 and w["has_velocities"]
    s = c.read_data(os.path.join(REF, "LJ_salt", "box_102030", "rbmd.data"), "charge", unit="LJ")
    assert len(s["pos"]) == 6000 and np.all(s["mass"] == 1.0)
    assert np.allclose(s["hi"] - s["lo"], [10, 20, 30]) and abs(s["charge"].sum()) < 1e-9
    for cfg in ("H2O/rbmd.json", "LJ_salt/rbmd.json", "LJ/rbmd.json"):
        text = open(os.path.join(REF, cfg), encoding="utf-8-sig").read()
        ff = c.ForceField(text, c.Box((0.0, 0.0, 0.0), (30.0, 30.0, 30.0)))
        ff.close()


def test_setfl_and_funcfl_files_load(tmp_path):
    """EAM potential files: funcfl (the reference's format) and single-element setfl are read
    when the handle is created (no device needed); a truncated file is rejected."""
    pf = systems.write_johnson_funcfl(str(tmp_path / "j.eam"))
    ps = systems.write_johnson_setfl(str(tmp_path / "j.eam.alloy"))
    box = c.Box((0.0, 0.0, 0.0), (20.0, 20.0, 20.0))
    for path in (pf, ps):
        c.ForceField(systems.eam_config(path), box).close()
    bad = tmp_path / "bad.eam.alloy"
    bad.write_text("".join(open(ps).readlines()[:9]))
    with pytest.raises(c.RbmdError, match="ERR_FILE"):
        c.ForceField(systems.eam_config(str(bad)), box)


def test_molecular_roundtrip_with_topology(tmp_path):
    """A flexible-chain system with bond / angle / dihedral types and harmonic coefficients writes
    (rbmd_data_write_arrays) and reads back identically: a checkpoint of a CVFF system."""
    from copy_gpu_b200 import systems
    s = systems.molecular(n_chain=20, chain_len=10, n_ion_pairs=5, seed=7)
    d = dict(s)
    d["mass_by_type"] = np.array([12.011, 15.999, 15.035, 6.94, 140.0])
    p = tmp_path / "mol.data"
    c.write_data(p, "full", d)
    r = c.read_data(p, "full", unit="REAL")
    for k in ("pos", "vel", "charge", "type", "molecule", "bonds", "bond_type", "angles", "angle_type",
              "dihedrals", "dihedral_type", "bond_coeffs", "angle_coeffs", "dihedral_coeffs"):
        assert np.array_equal(r[k], d[k]), k
