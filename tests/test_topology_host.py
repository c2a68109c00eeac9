"""CPU checks of the general CVFF topology: the oracle's special-bond lists, bonded terms and the
data reader's Dihedrals sections.

* special lists follow ModelFileInitCondition::SetSpecialBonds: traversal order through the
  bond multimap, duplicates kept, and in rings the last occurrence of a partner decides its
  weight (the pair loops overwrite on every match);
* the oracle's CVFF forces (bonds, angles, harmonic dihedrals, intramolecular Coulomb
  correction) are minus the gradient of its energies (central differences, FP64);
* on water the general terms reproduce the water-specific oracle exactly;
* the data reader returns Dihedral Coeffs (K, sign, multiplicity) and Dihedrals, and reads the
  reference's polymer-electrolyte input when the reference tree is present.
"""
import os

import numpy as np
import pytest

import oracle
from copy_gpu_b200 import systems


def _ring5(n_ring=8, cell=7.0, seed=4):
    """Five-membered rings (side 1.5) on a lattice, random orientations, neutral charges."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(n_ring ** (1 / 3)))
    L = m * cell
    R = 1.5 / (2 * np.sin(np.pi / 5))
    ang = 2 * np.pi * np.arange(5) / 5
    loc = np.stack([R * np.cos(ang), R * np.sin(ang), np.zeros(5)], 1)
    pos, bonds, angles, dihs = [], [], [], []
    for r in range(n_ring):
        ijk = np.array(np.unravel_index(r, (m, m, m)), float)
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        base = 5 * r
        pos.append((ijk + 0.5) * cell + loc @ q.T + rng.normal(scale=0.03, size=(5, 3)))
        for k in range(5):
            bonds.append((base + k, base + (k + 1) % 5))
            angles.append((base + k, base + (k + 1) % 5, base + (k + 2) % 5))
            dihs.append((base + k, base + (k + 1) % 5, base + (k + 2) % 5, base + (k + 3) % 5))
    n = 5 * n_ring
    return dict(pos=np.mod(np.concatenate(pos), L), lo=np.zeros(3), hi=np.full(3, L),
                charge=np.tile([0.2, -0.1, -0.1, 0.1, -0.1], n_ring), molecule=np.repeat(np.arange(n_ring), 5),
                type=np.zeros(n, np.int32), mass=np.full(n, 12.0), eps=np.array([0.066]), sigma=np.array([3.5]),
                bonds=np.array(bonds, np.int32), bond_type=np.zeros(len(bonds), np.int32),
                bond_coeffs=np.array([[300.0, 1.5]]), angles=np.array(angles, np.int32),
                angle_type=np.zeros(len(angles), np.int32), angle_coeffs=np.array([[60.0, 108.0]]),
                dihedrals=np.array(dihs, np.int32), dihedral_type=np.zeros(len(dihs), np.int32),
                dihedral_coeffs=np.array([[0.4, -1, 2]]))


def _last_weight(sp, i, j):
    off, ids, w = sp
    r = 1.0
    for k in range(off[i], off[i + 1]):
        if ids[k] == j:
            r = w[k]
    return r


def test_special_lists_chain_and_bondless():
    off, ids, w = oracle.special_lists(6, [[0, 1], [1, 2], [2, 3], [3, 4]], [0.0, 0.25, 0.5])
    got = {a: list(zip(ids[off[a]:off[a + 1]].tolist(), w[off[a]:off[a + 1]].tolist())) for a in range(6)}
    assert got[0] == [(1, 0.0), (2, 0.25), (3, 0.5)]
    assert got[1] == [(0, 0.0), (2, 0.0), (3, 0.25), (4, 0.5)]
    assert got[2] == [(1, 0.0), (0, 0.25), (3, 0.0), (4, 0.25)]
    assert got[5] == [(5, 1.0)]   # no bonds: the atom itself with weight 1


def test_special_lists_ring_last_occurrence():
    """5-ring 0-1-2-3-4-0: atom 0 meets 3 first as a 1-4 partner (via 1, 2) and later as a 1-3
    partner (via 4), and 2 first as 1-3 and later as 1-4: the later weight is the one kept."""
    sp = oracle.special_lists(5, [[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]], [0.0, 0.25, 0.5])
    off, ids, w = sp
    assert ids[off[0]:off[1]].tolist() == [1, 2, 3, 4, 3, 2]
    assert _last_weight(sp, 0, 3) == 0.25 and _last_weight(sp, 0, 2) == 0.5
    assert _last_weight(sp, 0, 1) == 0.0 and _last_weight(sp, 0, 4) == 0.0
    # the weight of a pair then depends on which end looks: w(1, 3) = w13 but w(3, 1) = w14, so
    # in rings with w13 != w14 the reference's pair forces are not equal and opposite
    assert _last_weight(sp, 1, 3) == 0.25 and _last_weight(sp, 3, 1) == 0.5


def _energy(s, pos, special):
    _, e = oracle.cvff_terms(pos, s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"], s["bond_type"],
                             s["bond_coeffs"], s["angles"], s["angle_type"], s["angle_coeffs"], s["dihedrals"],
                             s["dihedral_type"], s["dihedral_coeffs"], special=special)
    return e["bond"] + e["angle"] + e["dihedral"] + e["coul_special"], e


@pytest.mark.parametrize("kind", ["chains", "rings", "chains_nospecial"])
def test_cvff_forces_are_minus_gradient(kind):
    s = _ring5() if kind == "rings" else systems.molecular(n_chain=6, chain_len=9, n_ion_pairs=2, seed=8)
    n = len(s["pos"])
    # rings: w13 = w14 keeps the weights symmetric (see the test above), so the forces derive
    # from one energy
    w = [0.0, 0.5, 0.5] if kind == "rings" else [0.0, 0.3, 0.5]
    special = None if kind == "chains_nospecial" else oracle.special_lists(n, s["bonds"], w)
    f, e = oracle.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], s["bonds"], s["bond_type"],
                             s["bond_coeffs"], s["angles"], s["angle_type"], s["angle_coeffs"], s["dihedrals"],
                             s["dihedral_type"], s["dihedral_coeffs"], special=special)
    assert all(abs(v) > 0 for k, v in e.items() if not (k == "dihedral" and special is None))
    if special is None:
        assert e["dihedral"] == 0.0   # dihedrals only with special bonds, as the reference
    h = 1e-6
    rng = np.random.default_rng(1)
    for a in rng.choice(n, 12, replace=False):
        for d in range(3):
            p = s["pos"].copy()
            p[a, d] += h
            ep, _ = _energy(s, p, special)
            p[a, d] -= 2 * h
            em, _ = _energy(s, p, special)
            g = -(ep - em) / (2 * h)
            assert abs(g - f[a, d]) <= 1e-5 * max(1.0, abs(f[a, d])), (a, d, g, f[a, d])


def test_cvff_terms_reproduce_water_extras():
    s = systems.water(n_mol=60, seed=2)
    n = len(s["pos"])
    hoh = s["hoh"]
    bonds = np.concatenate([hoh[:, [0, 1]], hoh[:, [2, 1]]])
    fw, ew = oracle.water_extras(hoh, s["pos"], s["charge"], s["lo"], s["hi"], *s["bond"], *s["angle"])
    f, e = oracle.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], bonds,
                             np.zeros(len(bonds), np.int32), np.array([s["bond"]]), hoh,
                             np.zeros(len(hoh), np.int32), np.array([s["angle"]]))
    assert np.abs(f - fw).max() <= 1e-12 * np.abs(fw).max()
    assert abs(e["bond"] - ew[0]) <= 1e-12 * abs(ew[0]) and abs(e["angle"] - ew[1]) <= 1e-12 * abs(ew[1])
    # with special_bonds [0, 0, 0] every intramolecular water pair is special with weight 0, so
    # the general correction equals the plain one
    sp = oracle.special_lists(n, bonds, [0.0, 0.0, 0.0])
    f2, _ = oracle.cvff_terms(s["pos"], s["lo"], s["hi"], s["charge"], s["molecule"], bonds,
                              np.zeros(len(bonds), np.int32), np.array([s["bond"]]), hoh,
                              np.zeros(len(hoh), np.int32), np.array([s["angle"]]), special=sp)
    assert np.abs(f2 - fw).max() <= 1e-12 * np.abs(fw).max()


DATA = """LAMMPS data file with dihedrals

6 atoms
2 atom types
5 bonds
1 bond types
4 angles
1 angle types
3 dihedrals
2 dihedral types

0 10 xlo xhi
0 10 ylo yhi
0 10 zlo zhi

Masses

1 12.0
2 16.0

Pair Coeffs # lj/cut/coul/long

1 0.1 3.4
2 0.2 3.0

Bond Coeffs # harmonic

1 300 1.5

Angle Coeffs # harmonic

1 50 109.5

Dihedral Coeffs # harmonic

1 0.15 1 3
2 0.3 -1 2

Atoms # full

1 1 1 0.1 1 1 1
2 1 2 -0.1 2 1 1
3 1 1 0.1 3 1 1
4 1 2 -0.1 4 1 1
5 1 1 0.1 5 1 1
6 1 2 -0.1 6 1 1

Bonds

1 1 1 2
2 1 2 3
3 1 3 4
4 1 4 5
5 1 5 6

Angles

1 1 1 2 3
2 1 2 3 4
3 1 3 4 5
4 1 4 5 6

Dihedrals

1 1 1 2 3 4
2 2 2 3 4 5
3 1 3 4 5 6
"""


def test_data_reader_dihedrals(tmp_path):
    from copy_gpu_b200 import read_data
    p = tmp_path / "mol.data"
    p.write_text(DATA)
    d = read_data(p, "full", "REAL")
    assert d["dihedrals"].tolist() == [[0, 1, 2, 3], [1, 2, 3, 4], [2, 3, 4, 5]]
    assert d["dihedral_type"].tolist() == [0, 1, 0]
    assert np.array_equal(d["dihedral_coeffs"], [[0.15, 1, 3], [0.3, -1, 2]])
    assert d["bond_type"].tolist() == [0] * 5 and d["angle_type"].tolist() == [0] * 4


PEO = os.path.join(os.environ.get("RBMD_REFERENCE", "/root/reference"), "rbmd", "res", "json_files", "PEO", "rbmd.data")


@pytest.mark.skipif(not os.path.exists(PEO), reason="reference tree not present")
def test_data_reader_reference_polymer_electrolyte():
    """The reference's PEO/LiTFSI input (rbmd/res/json_files/PEO/rbmd.data): header counts,
    coefficient rows and the first/last topology lines as the file states them."""
    from copy_gpu_b200 import read_data
    d = read_data(PEO, "full", "REAL")
    assert len(d["pos"]) == 4322 and len(d["bonds"]) == 3921 and len(d["angles"]) == 7080
    assert len(d["dihedrals"]) == 7197 and d["dihedral_coeffs"].shape == (16, 3)
    assert d["dihedral_coeffs"][0].tolist() == [0.0467, 1, 3]
    assert d["bonds"][0].tolist() == [1304, 1305] and d["dihedrals"][-1].tolist() == [839, 834, 840, 843]
    # the special lists and the oracle's intramolecular terms evaluate on it
    sp = oracle.special_lists(len(d["pos"]), d["bonds"], [0.0, 0.0, 0.0])
    f, e = oracle.cvff_terms(d["pos"], d["lo"], d["hi"], d["charge"], d["molecule"], d["bonds"], d["bond_type"],
                             d["bond_coeffs"], d["angles"], d["angle_type"], d["angle_coeffs"], d["dihedrals"],
                             d["dihedral_type"], d["dihedral_coeffs"], special=sp)
    assert np.isfinite(f).all() and all(np.isfinite(v) for v in e.values())
    assert abs(f.sum(0)).max() < 1e-6 * np.abs(f).max()


@pytest.mark.skipif(not os.path.exists(PEO), reason="reference tree not present")
def test_reference_polymer_electrolyte_roundtrip(tmp_path):
    """The reference's PEO/LiTFSI input written back with rbmd_data_write_arrays (every section,
    11 bond / 19 angle / 16 dihedral types with their coefficients) reads back identically."""
    from copy_gpu_b200 import read_data, write_data
    d = read_data(PEO, "full", "REAL")
    p = tmp_path / "peo.data"
    write_data(p, "full", d)
    r = read_data(p, "full", "REAL")
    for k in ("pos", "vel", "charge", "type", "molecule", "image", "mass", "eps", "sigma", "bonds", "bond_type",
              "bond_coeffs", "angles", "angle_type", "angle_coeffs", "dihedrals", "dihedral_type",
              "dihedral_coeffs", "lo", "hi"):
        assert np.array_equal(r[k], d[k]), k
