"""The oracle pinned to the reference's own code.

oracle/_ref/libref.so is RBMD's force-path code compiled from the reference tree
(oracle/build_ref.sh: ExecForceFunction, ExecPointLocator, ContPointLocator's grid setters and
BinPointsWorklet, ExecTopology, ExecStaticTable with the ERFTable.h arrays, RBEPSAMPLE and every
worklet struct of RunWorklet.cpp, against the VTK-m stand-in in oracle/ref_shim).  These tests
feed identical FP32 inputs to it and to the oracle's restatement (oracle/oracle.cpp) and require:

* grid dims, num_cycles, cell order and bounds: identical;
* Verlet lists (ComputeNeighboursWorklet) and RBL lists (ComputeRBLNeighboursOnceWorklet):
  identical ids in identical traversal order, offsets matching the oracle's shift codes;
* near forces (ComputeNearForceVerletWorklet, ComputeLJForceVerletWorklet, the RBL LJ worklet),
  structure-factor terms, the RBE normaliser S, the RBE force (ComputeNewRBEForceWorklet), EAM
  F'(rho) and forces (ComputeEAMfpVerletWorklet / ComputeEAMForceVerletWorklet, and the ORIGINAL
  type's ComputeEAMrho/fp/forceWorklet): bit for bit (the oracle in its reference-order
  accumulation);
* the RBE sampler: the oracle's seeded sampler (which the device sampler reproduces exactly) and
  RBEPSAMPLE::Fetch_P_Sample run on the same uniforms give identical k-sets;
* the RBL ERF table and the RBL erfc force: the oracle's reconstruction of the table equals the
  reference's arrays for at least 98 % of the entries and within 1e-5 relative for all.

Skipped where the reference tree is absent (the library cannot be built there).
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems


@pytest.fixture(scope="module")
def ref(oracle_lib):
    from oracle import ref as r
    if not r.build():
        pytest.skip("reference tree not present: oracle/_ref cannot be built")
    return r


def _jittered_lj(n_cell=6, seed=2):
    s = systems.lj_fcc(ncell=n_cell, seed=seed)
    rng = np.random.default_rng(seed)
    L = s["hi"] - s["lo"]
    s["pos"] = s["lo"] + np.mod(s["pos"] + rng.normal(scale=0.08, size=s["pos"].shape) - s["lo"], L)
    return s


def _edge_box():
    rng = np.random.default_rng(4)
    L = 7.6
    pos = rng.uniform(0, L, size=(300, 3))
    pos[:8] = np.array([[0, 0, 0], [L, 0, 0], [0, L, 0], [0, 0, L], [L, L, L], [L / 2, 0, L],
                        [2.5, 2.5, 2.5], [5.0, 5.0, 5.0]])
    pos[9] = np.array([1.0, 3.0, 3.0])
    pos[8] = pos[9] + np.array([2.5, 0, 0])
    pos[10] = np.array([-0.2, 3.0, 7.9])              # outside the box on two faces
    return dict(pos=pos, lo=np.zeros(3), hi=np.full(3, L))


CASES = {
    "electrolyte": lambda: systems.electrolyte(3000, seed=3),
    "lj_fcc": _jittered_lj,
    "edges": _edge_box,
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("rc,rs", [(2.5, 2.5), (2.5, 1.25)])
def test_grid_and_cells(oracle_lib, ref, case, rc, rs):
    import ctypes
    s = CASES[case]()
    pr = s["pos"].astype(np.float32)
    dims_r, nc_r = ref.grid(s["lo"], s["hi"], rc, rs)
    pid_r, low_r, up_r = ref.cells(pr, s["lo"], s["hi"], rc, rs)
    ncell = int(np.prod(dims_r))
    dims = np.zeros(3, np.int32)
    pid = np.zeros(len(pr), np.int32)
    low = np.zeros(ncell, np.int32)
    up = np.zeros(ncell, np.int32)
    D, I = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    oracle_lib.lib().oracle_cells_f32(ctypes.c_int64(len(pr)), pr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      np.asarray(s["lo"], np.float64).ctypes.data_as(D),
                                      np.asarray(s["hi"], np.float64).ctypes.data_as(D), ctypes.c_double(rc),
                                      ctypes.c_double(rs), dims.ctypes.data_as(I), pid.ctypes.data_as(I),
                                      low.ctypes.data_as(I), up.ctypes.data_as(I))
    assert np.array_equal(dims, dims_r)
    assert np.array_equal(pid, pid_r) and np.array_equal(low, low_r) and np.array_equal(up, up_r)


def _codes_to_sign(codes):
    c = np.stack([(codes >> (2 * d)) & 3 for d in range(3)], axis=-1)
    return np.where(c == 1, 1, np.where(c == 2, -1, 0))


@pytest.mark.parametrize("case", sorted(CASES))
def test_verlet_lists(oracle_lib, ref, case):
    s = CASES[case]()
    pr = s["pos"].astype(np.float32)
    c_o, ids_o, codes_o = oracle_lib.neighbors(pr, s["lo"], s["hi"], 2.5, "fp32")
    c_r, ids_r, off_r = ref.neighbors(pr, s["lo"], s["hi"], 2.5)
    assert np.array_equal(c_o, c_r)
    w = int(c_o.max())
    used = np.arange(w)[None, :] < c_o[:, None]
    assert np.array_equal(np.where(used, ids_o[:, :w], -1), np.where(used, ids_r[:, :w], -1))
    # the reference's coordinate offset dxdydz * (wrapped - unwrapped cell) against the code
    assert np.array_equal(np.where(used[..., None], np.sign(off_r[:, :w]), 0),
                          np.where(used[..., None], _codes_to_sign(codes_o[:, :w]), 0))


def test_near_forces(oracle_lib, ref):
    s = systems.electrolyte(3000, seed=3)
    pr = s["pos"].astype(np.float32)
    alpha = systems.electrolyte_alpha()
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 2.5, "fp32")
    rl = ref.neighbors(pr, s["lo"], s["hi"], 2.5)
    for with_coul in (False, True):
        fo = oracle_lib.near_force(pr, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"], eps=s["eps"],
                                   sigma=s["sigma"], with_coul=with_coul, alpha=alpha, prec="fp32", sum_mode=0)
        fr = ref.near_force(pr, s["lo"], s["hi"], 2.5, rl, type=s["type"], charge=s["charge"], eps=s["eps"],
                            sigma=s["sigma"], alpha=alpha, with_coul=with_coul)
        assert np.array_equal(fo.astype(np.float32), fr), f"with_coul={with_coul}"


def test_near_forces_water_molecules(oracle_lib, ref):
    """Molecule exclusion of the LJ term, several types, REAL-unit charges (no qqr2e on this
    path, as the reference's Verlet worklet)."""
    s = systems.water(n_mol=300, seed=2)
    pr = s["pos"].astype(np.float32)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 8.0, "fp32")
    rl = ref.neighbors(pr, s["lo"], s["hi"], 8.0)
    fo = oracle_lib.near_force(pr, s["lo"], s["hi"], 8.0, nl, type=s["type"], mol=s["molecule"], charge=s["charge"],
                               eps=s["eps"], sigma=s["sigma"], with_coul=True, alpha=0.09, prec="fp32", sum_mode=0)
    fr = ref.near_force(pr, s["lo"], s["hi"], 8.0, rl, type=s["type"], mol=s["molecule"], charge=s["charge"],
                        eps=s["eps"], sigma=s["sigma"], alpha=0.09, with_coul=True)
    assert np.array_equal(fo.astype(np.float32), fr)


def test_rbe_terms_normaliser_and_force(oracle_lib, ref):
    s = systems.electrolyte(3000, seed=3)
    pr = s["pos"].astype(np.float32)
    alpha = systems.electrolyte_alpha()
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, 5, 0, 0, 64)
    rho_o = oracle_lib.rhok(pr, s["charge"], L, m, prec="fp32")
    rho_r = ref.rhok(pr, s["charge"], L, m)
    assert np.array_equal(rho_o, rho_r)
    rho32 = rho_r.astype(np.float32)
    f_r, S_r = ref.rbe_force(pr, s["charge"], s["lo"], s["hi"], alpha, m, rho32)
    assert np.float32(S_r) == np.float32(oracle_lib.rbe_S(alpha, L, "fp32"))
    f_o = oracle_lib.rbe_force(pr, s["charge"], L, alpha, 1.0, m, rho32.astype(np.float64), prec="fp32")
    assert np.array_equal(f_o.astype(np.float32), f_r)


def test_eam_passes(oracle_lib, ref, tmp_path):
    """F'(rho) and forces of the Verlet EAM worklets; the reference's pair vector (p_j - p_i) gives
    its forces bit for bit, the physical sign exactly their negation (compat flag
    eam_verlet_pair_vector)."""
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=6, seed=5)
    pr = s["pos"].astype(np.float32)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 5.0, "fp32")
    rl = ref.neighbors(pr, s["lo"], s["hi"], 5.0)
    f_r, fp_r = ref.eam(oracle_lib.eam_tables(pot), pr, s["lo"], s["hi"], 5.0, rl)
    f_o, fp_o = oracle_lib.eam_force(pot, pr, s["lo"], s["hi"], 5.0, nl, prec="fp32", sum_mode=0, ref_sign=True)
    assert np.array_equal(fp_o.astype(np.float32), fp_r)
    assert np.array_equal(f_o.astype(np.float32), f_r)
    f_p, _ = oracle_lib.eam_force(pot, pr, s["lo"], s["hi"], 5.0, nl, prec="fp32", sum_mode=0, ref_sign=False)
    assert np.array_equal(f_p.astype(np.float32), -f_r)


def test_eam_original_neighbor_type(oracle_lib, ref, tmp_path):
    """The ORIGINAL type's EAM (cells walked on the fly, ComputeEAMrho/fp/forceWorklet) equals the
    oracle over the ORIGINAL pair set with the physical pair vector p_i - p_j, bit for bit."""
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=6, seed=9)
    pr = s["pos"].astype(np.float32)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 5.0, "fp32", original=True)
    f_o, fp_o = oracle_lib.eam_force(pot, pr, s["lo"], s["hi"], 5.0, nl, prec="fp32", sum_mode=0, ref_sign=False)
    f_r, fp_r = ref.eam_original(oracle_lib.eam_tables(pot), pr, s["lo"], s["hi"], 5.0)
    assert np.array_equal(fp_o.astype(np.float32), fp_r)
    assert np.array_equal(f_o.astype(np.float32), f_r)


@pytest.mark.parametrize("L,alpha,P", [(107.72, None, 500), (66.88, 0.09, 200), (15.5, None, 64)])
def test_sampler_same_draws(oracle_lib, ref, L, alpha, P):
    alpha = alpha or systems.electrolyte_alpha()
    box = np.full(3, L)
    for seed in range(40):
        m, trace = oracle_lib.rbe_sample_trace(alpha, box, seed, 3, 1, P)
        m_r, used = ref.rbe_sample(alpha, box, P, trace)
        assert used == len(trace), (seed, used, len(trace))
        assert np.array_equal(m, m_r), seed


def test_sampler_reference_test_mode(ref):
    """velocity_type TEST: U = 0.5 everywhere, so every sample is round(sigma_d sqrt(2 ln 2) cos(pi))
    and the chain never moves (the reference's degenerate but reproducible k-set)."""
    alpha, L, P = 0.09, np.array([30.0, 40.0, 50.0]), 16
    m, _ = ref.rbe_sample(alpha, L, P)
    sigma = np.sqrt(alpha / 2.0) * L / np.pi
    expect = np.round(-sigma * np.sqrt(2.0 * np.log(2.0))).astype(np.int32)
    assert np.array_equal(m, np.tile(expect, (P, 1)))


def test_rbl_lists_and_forces(oracle_lib, ref):
    s = systems.electrolyte(3000, seed=8)
    pr = s["pos"].astype(np.float32)
    lo, hi = s["lo"], s["hi"]
    rs, rc = 1.25, 2.5
    rs_num, _, pice = oracle_lib.rbl_sizes(3000, lo, hi, rs, rc, 10)
    ol = oracle_lib.rbl_list(pr, lo, hi, rc, rs, pice, rs_num, 128)
    rl = ref.rbl_list(pr, lo, hi, rc, rs, rs_num, pice, cap=rs_num + 128)
    assert np.array_equal(ol[0], rl[0]) and np.array_equal(ol[1], rl[1])
    for i in range(len(pr)):
        assert np.array_equal(ol[2][i, :ol[0][i]], rl[2][i, :rl[0][i]]), i
        assert np.array_equal(ol[2][i, rs_num:rs_num + ol[1][i]], rl[2][i, rs_num:rs_num + rl[1][i]]), i
    kw = dict(type=s["type"], charge=s["charge"], eps=s["eps"], sigma=s["sigma"])
    fo = oracle_lib.rbl_near(pr, lo, hi, rc, rs, pice, ol, rs_num, with_coul=False, table_mode=1, shell_coul=0,
                             remove_mean=False, prec="fp32", sum_mode=0, **kw)
    fr = ref.rbl_near(pr, lo, hi, rc, rs, rs_num, pice, rl, with_coul=False, **kw)
    assert np.array_equal(fo.astype(np.float32), fr)
    fo = oracle_lib.rbl_near(pr, lo, hi, rc, rs, pice, ol, rs_num, with_coul=True, alpha=0.1, qqr2e=1.0, table_mode=1,
                             shell_coul=0, remove_mean=False, prec="fp32", sum_mode=0, **kw)
    fr = ref.rbl_near(pr, lo, hi, rc, rs, rs_num, pice, rl, alpha=0.1, qqr2e=1.0, with_coul=True, **kw)
    assert np.abs(fo - fr).max() <= 1e-5 * np.abs(fr).max()


def test_rbl_erf_table(oracle_lib, ref):
    lo = np.float32(0.1).view(np.uint32) & ~np.uint32(0x7FFF)
    hi = np.float32(12.0).view(np.uint32)
    edges = np.arange(lo, hi, 0x8000, dtype=np.uint32)
    d = (edges + np.uint32(0x4000)).view(np.float32)
    d = d[(d >= 0.1) & (d < 12.0)]
    g_r = ref.erf_table(d)
    g_o = np.array([oracle_lib.rbl_table_g(x) for x in d], np.float32)
    assert (g_o == g_r).sum() >= 0.98 * len(d)
    assert (np.abs(g_o - g_r) / np.abs(g_r)).max() <= 1e-5
