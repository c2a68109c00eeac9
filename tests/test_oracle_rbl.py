"""CPU checks of the oracle's RBL restatement, the reference ERF table and the EAM force sign.

* ERF table: the oracle's reconstruction equals the reference's own table
  (tests/golden/erf_table.csv, made by tests/golden/make_erf_table.py from the reference's
  Gnear_table_*.txt) exactly for nearly every entry and within one unit of the printed sixth
  significant digit for all.
* RBL sizes: the reference's formulas (ExecutionMD.cpp:467-486) evaluated independently here.
* RBL list: with pice = 1 the core and shell pairs together are the full list at rc (minus pairs
  within 1e-4 of r_core^2, which neither predicate takes); with pice = k the shell list is every
  k-th shell pair of the full list's traversal order.
* EAM: forces are -grad E by central finite differences of the FP64 energy for the default pair
  vector, and exactly reversed for the reference's Verlet pair vector.
"""
import csv
import os

import numpy as np
import pytest

from copy_gpu_b200 import systems

HERE = os.path.dirname(os.path.abspath(__file__))


def test_erf_table_matches_reference_golden(oracle_lib):
    """The reconstructed table equals the reference's 6-digit literals as floats for at least 97 %
    of the entries, and is within one unit of their sixth digit (1e-5 relative) everywhere."""
    rows = list(csv.DictReader(open(os.path.join(HERE, "golden", "erf_table.csv"))))
    assert len(rows) > 800
    worst, exact = 0.0, 0
    for r in rows:
        g = oracle_lib.rbl_table_g(np.float32(float(r["distance"])))
        ref = np.float32(float(r["g"]))
        exact += np.float32(g) == ref
        worst = max(worst, abs(g - float(ref)) / abs(float(ref)))
    assert worst <= 1e-5, worst
    assert exact >= 0.97 * len(rows), (exact, len(rows))


def _sizes_by_hand(n, L, rs, rc, sample, eam=False):
    f32 = np.float32
    rho = f32(n) / (f32(L) * f32(L) * f32(L))
    pif = float(f32(np.pi))
    coeff = 1 if eam else int(np.round(f32(1.0 + (0.05 / float(rho) - 0.05))))
    cs = np.ceil(4.0 / 3.0 * pif * float(f32(rs)) ** 3)
    cc = np.ceil(4.0 / 3.0 * pif * float(f32(rc)) ** 3)
    rf = float(rho if eam else f32(coeff) * rho)
    rs_num = int(rf * cs + 1)
    rc_num = int(rf * cc + 1)
    rate = f32(sample) / f32(rc_num - rs_num)
    return rs_num, rc_num, int(np.ceil(1.0 / float(rate)))


@pytest.mark.parametrize("n,L,rs,rc,sample,eam", [(30000, 66.88, 5.0, 12.0, 100, False),
                                                   (3000, 15.536, 1.25, 2.5, 10, False),
                                                   (4000, 14.46, 3.0, 5.0, 20, True)])
def test_rbl_sizes(oracle_lib, n, L, rs, rc, sample, eam):
    got = oracle_lib.rbl_sizes(n, (0, 0, 0), (L, L, L), rs, rc, sample, eam=eam)
    assert got == _sizes_by_hand(n, L, rs, rc, sample, eam)


def test_rbl_list_pice1_is_full_list(oracle_lib):
    s = systems.electrolyte(1500, seed=8)
    pos = s["pos"].astype(np.float32)
    rs, rc = 1.25, 2.5
    ncore, nshell, ids, codes = oracle_lib.rbl_list(pos, s["lo"], s["hi"], rc, rs, 1, 64, 128)
    counts, fids, _ = oracle_lib.neighbors(pos, s["lo"], s["hi"], rc, rs=rs)
    for i in range(len(pos)):
        mine = np.concatenate([ids[i, :ncore[i]], ids[i, 64:64 + nshell[i]]])
        full = fids[i, :counts[i]]
        assert set(mine.tolist()) <= set(full.tolist())
        assert len(full) - len(mine) <= 2     # pairs within 1e-4 of rs^2 belong to neither part
    assert ncore.sum() + nshell.sum() >= counts.sum() - len(pos) // 50


def test_rbl_shell_is_every_pice_th_in_traversal_order(oracle_lib):
    s = systems.electrolyte(1500, seed=9)
    pos = s["pos"].astype(np.float32)
    rs, rc, pice = 1.25, 2.5, 3
    ncore, nshell, ids, codes = oracle_lib.rbl_list(pos, s["lo"], s["hi"], rc, rs, pice, 64, 64)
    _, n1, ids1, codes1 = oracle_lib.rbl_list(pos, s["lo"], s["hi"], rc, rs, 1, 64, 192)
    for i in range(len(pos)):
        all_shell = ids1[i, 64:64 + n1[i]]
        assert np.array_equal(ids[i, 64:64 + nshell[i]], all_shell[::pice])
        assert np.array_equal(codes[i, 64:64 + nshell[i]], codes1[i, 64:64 + n1[i]][::pice])


def test_rbl_near_pice1_equals_full_list_lj(oracle_lib):
    s = systems.lj_fcc(ncell=5, seed=4)
    pos = s["pos"].astype(np.float32)
    rs, rc = 1.25, 2.5
    rl = oracle_lib.rbl_list(pos, s["lo"], s["hi"], rc, rs, 1, 64, 128)
    f_rbl = oracle_lib.rbl_near(pos, s["lo"], s["hi"], rc, rs, 1, rl, 64, remove_mean=False)
    nl = oracle_lib.neighbors(pos, s["lo"], s["hi"], rc, rs=rs)
    f_full = oracle_lib.near_force(pos, s["lo"], s["hi"], rc, nl, sum_mode=1)
    # identical except for pairs within 1e-4 of rs^2 (none in a jittered FCC lattice)
    assert np.abs(f_rbl - f_full).max() <= 1e-5 * np.abs(f_full).max()


def test_eam_force_is_minus_grad_energy(oracle_lib, tmp_path):
    pot = systems.write_johnson_funcfl(str(tmp_path / "j.eam"))
    s = systems.eam_fcc(ncell=4, seed=3)
    pos = s["pos"].astype(np.float64)
    nl = oracle_lib.neighbors(pos, s["lo"], s["hi"], 5.0, "fp64")
    f, _ = oracle_lib.eam_force(pot, pos, s["lo"], s["hi"], 5.0, nl, prec="fp64")
    f_ref, _ = oracle_lib.eam_force(pot, pos, s["lo"], s["hi"], 5.0, nl, prec="fp64", ref_sign=True)
    assert np.array_equal(f, -f_ref)
    h = 1e-5
    for a, d in [(0, 0), (7, 1), (100, 2)]:
        e = []
        for sgn in (1, -1):
            p = pos.copy()
            p[a, d] += sgn * h
            e.append(oracle_lib.eam_energy(pot, p, s["lo"], s["hi"], 5.0,
                                           oracle_lib.neighbors(p, s["lo"], s["hi"], 5.0, "fp64")))
        fd = -(e[0] - e[1]) / (2 * h)
        assert abs(fd - f[a, d]) <= 1e-5 * max(1.0, abs(fd)), (a, d, fd, f[a, d])
