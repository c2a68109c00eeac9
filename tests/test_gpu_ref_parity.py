"""The B200 path against the reference's own code (oracle/_ref/libref.so: RBMD's worklets and
force functions compiled from the reference tree; see tests/test_oracle_ref_pin.py).

* neighbour pair sets: the device list equals ComputeNeighboursWorklet's, atom for atom;
* near forces (LJ + erfc Coulomb, LJ units, qqr2e = 1): within the FP32 bar (1e-5 of the rms force,
  max-norm) of ComputeNearForceVerletWorklet's float sums;
* EAM with the reference's Verlet pair vector (compat.eam_verlet_pair_vector): within the FP32 bar
  of ComputeEAMfpVerletWorklet / ComputeEAMForceVerletWorklet; neighbor.type ORIGINAL EAM within
  the FP32 bar of the on-the-fly worklets (ComputeEAMrho/fp/forceWorklet);
* RBE k-space with injected samples: the device error against the FP64 oracle is no larger than
  the reference's own FP32 k-space error (ComputePnumberChargeStructureFactorWorklet +
  ComputeNewRBEForceWorklet) and at most 1e-5;
* the device k-sampler equals RBEPSAMPLE::Fetch_P_Sample run on the same uniforms.

Skipped where oracle/_ref was not built (no reference tree where the repository was built).
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems
from tests.helpers import make_ff, pair_sets_equal, rel_err, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as r
    if not r.available():
        pytest.skip("oracle/_ref/libref.so not built")
    return r


def _run(cfg, s, cuda, m=None):
    import torch
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    if m is not None:
        ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    c, ids = ff.neighbors(256)
    f = dev["force"].cpu().numpy()
    return ff, c, ids, f


def test_pairs_and_near_force_vs_reference(cuda, ref, oracle_lib):
    """LJ/CUT/COUL/LONG with injected k-samples: the device force minus the oracle's FP64 RBE term
    against the reference's near worklet."""
    s = systems.electrolyte(6000, seed=21)
    P = 32
    cfg = systems.electrolyte_config(P=P, precision="fp32")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, seed=8, step=0, rep=0, P=P)
    ff, c, ids, f = _run(cfg, s, cuda, m)
    ff.close()
    pr = s["pos"].astype(np.float32)
    rl = ref.neighbors(pr, s["lo"], s["hi"], 2.5)
    assert pair_sets_equal(c, ids, rl[0], rl[1]) == -1
    fr = ref.near_force(pr, s["lo"], s["hi"], 2.5, rl, type=s["type"], charge=s["charge"], eps=s["eps"],
                        sigma=s["sigma"], alpha=alpha, with_coul=True).astype(np.float64)
    far = oracle_lib.rbe_force(s["pos"], s["charge"], L, alpha, 1.0, m, oracle_lib.rhok(s["pos"], s["charge"], L, m))
    assert rel_err(f - far, fr) <= 1e-5, rel_err(f - far, fr)


def test_eam_vs_reference(cuda, ref, oracle_lib, tmp_path):
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=8, seed=5)
    cfg = systems.eam_config(pot, precision="fp32")
    cfg["compat"] = {"eam_verlet_pair_vector": True}
    ff, c, ids, f = _run(cfg, s, cuda)
    ff.close()
    pr = s["pos"].astype(np.float32)
    rl = ref.neighbors(pr, s["lo"], s["hi"], 5.0)
    assert pair_sets_equal(c, ids, rl[0], rl[1]) == -1
    fr, _ = ref.eam(oracle_lib.eam_tables(pot), pr, s["lo"], s["hi"], 5.0, rl)
    assert rel_err(f, fr.astype(np.float64)) <= 1e-5, rel_err(f, fr)


@pytest.mark.parametrize("compat", [False, True])
def test_eam_original_neighbor_type_vs_reference(cuda, ref, oracle_lib, tmp_path, compat):
    """neighbor.type ORIGINAL with EAM (ExecutionMD::ComputeOriginalEAMForce): the reference's
    on-the-fly worklets use p_i - p_j, so the result is the physical force with or without
    compat.eam_verlet_pair_vector (that flag reproduces only the Verlet worklet's reversal)."""
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=8, seed=7)
    cfg = systems.eam_config(pot, precision="fp32")
    cfg["hyper_parameters"]["neighbor"]["type"] = "ORIGINAL"
    if compat:
        cfg["compat"] = {"eam_verlet_pair_vector": True}
    ff, _, _, f = _run(cfg, s, cuda)
    ff.close()
    fr, _ = ref.eam_original(oracle_lib.eam_tables(pot), s["pos"].astype(np.float32), s["lo"], s["hi"], 5.0)
    assert rel_err(f, fr.astype(np.float64)) <= 1e-5, rel_err(f, fr)


def test_rbe_kspace_vs_reference(cuda, ref, oracle_lib):
    """Real-space cutoff below the closest pair: the force is the RBE k-space term alone."""
    n, P = 3000, 128
    s = systems.electrolyte(n, seed=3)
    cfg = systems.electrolyte_config(P=P, precision="fp32")
    cfg["hyper_parameters"]["neighbor"]["cut_off"] = 0.5
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    m = oracle_lib.rbe_sample(alpha, L, seed=42, step=3, rep=0, P=P)
    ff, _, _, f = _run(cfg, s, cuda, m)
    ff.close()
    rho64 = oracle_lib.rhok(s["pos"], s["charge"], L, m)
    exact = oracle_lib.rbe_force(s["pos"], s["charge"], L, alpha, 1.0, m, rho64)
    pr = s["pos"].astype(np.float32)
    rho_r = ref.rhok(pr, s["charge"], L, m).astype(np.float32)
    f_ref, _ = ref.rbe_force(pr, s["charge"], s["lo"], s["hi"], alpha, m, rho_r)
    err_dev = rel_err(f, exact)
    err_ref = rel_err(f_ref.astype(np.float64), exact)
    assert err_dev <= min(err_ref, 1e-5) or err_dev <= 1e-6, (err_dev, err_ref)


def test_device_sampler_vs_reference_sampler(cuda, ref, oracle_lib):
    n, P = 2000, 200
    s = systems.electrolyte(n, seed=3)
    cfg = systems.electrolyte_config(P=P, precision="fp32")
    cfg["hyper_parameters"]["coulomb"]["seed"] = 99
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    L = s["hi"] - s["lo"]
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    for step in (0, 5, 77):
        got = ff.sample_k(step, P)
        _, trace = oracle_lib.rbe_sample_trace(alpha, L, 99, step, 0, P)
        m_r, used = ref.rbe_sample(alpha, L, P, trace)
        assert used == len(trace)
        assert np.array_equal(got, m_r), f"step {step}"
    ff.close()
