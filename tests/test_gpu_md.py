"""GPU parity of full MD steps (ExecutionNVT::Solve order) against oracle-driven steps, plus the
Verlet-skin, EAM, batched-replica and status paths.

Bars: FP64 trajectories agree with the oracle to <= 1e-9 absolute in positions after several
steps (forces agree to <= 1e-11 relative per step; the residual is summation order); FP32 EAM
forces <= 1e-5 relative (norm-wise, vs the oracle's reference-precision terms summed exactly).
"""
import math
import os

import numpy as np
import pytest

from copy_gpu_b200 import Box, systems
from tests.helpers import jitter, make_ff, rel_err, to_dev

pytestmark = pytest.mark.gpu


def _wrap(x, lo, hi):
    L = hi - lo
    x = np.where(x < lo, x + L, x)
    x = np.where(x > hi, x - L, x)
    return x


def _oracle_lj_force(o, pos, s, rc):
    nl = o.neighbors(pos, s["lo"], s["hi"], rc, "fp64")
    return o.near_force(pos, s["lo"], s["hi"], rc, nl, type=s["type"], eps=s["eps"], sigma=s["sigma"],
                        prec="fp64")


def test_lj_nve_trajectory_fp64(cuda, oracle_lib):
    import torch
    s = systems.lj_fcc(ncell=6, seed=3)
    s["pos"] = jitter(s["pos"], s["lo"], s["hi"], 0.03, seed=1)
    cfg = systems.lj_config(cutoff=2.5, precision="fp64", ensemble="NVE")
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    nsteps, dt = 10, cfg["execution"]["timestep"]
    ff.step(nsteps)
    torch.cuda.synchronize()
    assert ff.status() == 0
    x, v, m = s["pos"].copy(), s["vel"].copy(), s["mass"][:, None]
    F = _oracle_lj_force(oracle_lib, x, s, 2.5)
    for _ in range(nsteps):
        v = v + 0.5 * F / m * dt * 1.0
        x = _wrap(x + v * dt, s["lo"], s["hi"])
        F = _oracle_lj_force(oracle_lib, x, s, 2.5)
        v = v + 0.5 * F / m * dt * 1.0
    assert np.abs(dev["pos"].cpu().numpy() - x).max() < 1e-9
    assert np.abs(dev["vel"].cpu().numpy() - v).max() < 1e-8


def test_lj_nve_energy_conservation_fp64(cuda):
    """FP64 LJ (4000 atoms from FCC at rho 0.8442, T 0.72, rc 4.0 + skin 0.3, list reuse,
    CUDA-graph steps): after 200 steps of melting, 2000 NVE steps of dt = 0.005 keep the total
    energy (kinetic + LJ) within 2e-4 of its value.  The reference's LJ is truncated without a
    shift, so the energy jumps by 4 (rc^-12 - rc^-6) = -1e-3 whenever a pair crosses rc; at
    rc = 4.0 that noise stays well inside the bar, which therefore tests the integrator and the
    list reuse."""
    import torch
    s = systems.lj_fcc(ncell=10, seed=4)
    cfg = systems.lj_config(cutoff=4.0, precision="fp64", ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    ff.step(200)
    torch.cuda.synchronize()

    def total():
        ff.Execute()
        e = ff.energy()
        return e["kinetic"] + e["lj"]

    e0 = total()
    for _ in range(4):
        ff.step(500)
        torch.cuda.synchronize()
        assert ff.status() == 0
        e = total()
        assert abs(e - e0) <= 2e-4 * abs(e0), (e, e0)


def test_langevin_reaches_target_temperature(cuda):
    """temp_ctrl_type LANGEVIN (physical form: per-atom, per-step noise, the atom's mass,
    kBT = kB T0): an ideal gas (LJ epsilon 0) of 19,652 atoms started at T = 0.72 settles at the
    target T0 = 1.5 within 2 % (the full-step velocities of this kick-drift-kick form sample the
    target exactly for free particles; the tolerance is statistical)."""
    import torch
    s = systems.lj_fcc(ncell=17, seed=6)
    s["eps"] = np.array([0.0])
    cfg = systems.lj_config(cutoff=2.5, precision="fp64", ensemble="NVT")
    cfg["execution"].update({"temp_ctrl_type": "LANGEVIN", "temperature": [1.5, 1.5, 0.5],
                             "langevin_gamma": 10.0, "timestep": 0.005})
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    ff.step(600)
    temps = []
    for _ in range(40):
        ff.step(10)
        torch.cuda.synchronize()
        temps.append(ff.energy()["temperature"])
    assert ff.status() == 0
    assert abs(np.mean(temps) / 1.5 - 1.0) < 0.02, np.mean(temps)


def test_langevin_reference_form(cuda):
    """compat.langevin_reference reproduces the reference's UnderdampedLangevinWorklet
    (RunWorklet.cpp:1700-1728 with ExecutionNVT.cpp:735-747): F += -gamma v + sqrt(2 gamma / dt) xi
    with m = 1, kBT = 1, gamma = 100 and one xi vector shared by every atom."""
    import torch
    s = systems.lj_fcc(ncell=6, seed=7)
    forces = []
    for tctrl in ("", "LANGEVIN"):
        cfg = systems.lj_config(cutoff=2.5, precision="fp64", ensemble="NVT")
        cfg["execution"]["temp_ctrl_type"] = tctrl
        cfg["compat"] = {"langevin_reference": True}
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        ff.Execute()
        torch.cuda.synchronize()
        forces.append(dev["force"].cpu().numpy())
    gamma, dt = 100.0, cfg["execution"]["timestep"]
    noise = forces[1] - forces[0] + gamma * s["vel"]
    assert np.abs(noise - noise[0]).max() < 1e-9 * np.abs(noise).max()
    xi = noise[0] / np.sqrt(2.0 * gamma / dt)
    assert 1e-3 < np.linalg.norm(xi) < 8.0, xi


def test_skin_list_reuse_same_forces(cuda, oracle_lib):
    """Skin 0.3: the list is rebuilt only when an atom moved more than skin/2, and the forces of
    every step equal a fresh evaluation at the same positions (pairs within rc are unchanged).
    Trajectories themselves are not compared: the truncated (unshifted) LJ force jumps at rc,
    so summation-order rounding between two cell grids grows into visible differences."""
    import torch
    s = systems.lj_fcc(ncell=6, seed=4)
    cfg = systems.lj_config(cutoff=2.5, skin=0.3, precision="fp64", ensemble="NVE")
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    for _ in range(4):
        ff.step(10)
        torch.cuda.synchronize()
        assert ff.status() == 0
        x = dev["pos"].cpu().numpy()
        nl = oracle_lib.neighbors(x, s["lo"], s["hi"], 2.5, "fp64")
        ref = oracle_lib.near_force(x, s["lo"], s["hi"], 2.5, nl, prec="fp64")
        assert rel_err(dev["force"].cpu().numpy(), ref) < 1e-12
    assert 2 <= ff.list_builds() < 41


def test_electrolyte_rbe_steps_fp64(cuda, oracle_lib):
    """Two steps with the on-device sampler: the oracle draws the same k-samples per step."""
    import torch
    n, P = 2000, 48
    s = systems.electrolyte(n, seed=8)
    cfg = systems.electrolyte_config(P=P, precision="fp64", seed=77, ensemble="NVE")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    dt = cfg["execution"]["timestep"]
    L = s["hi"] - s["lo"]
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()                       # step counter 0: samples of step 0
    ff.step(2)                         # steps 0 and 1 of the step counter
    torch.cuda.synchronize()
    assert ff.status() == 0

    def force(x, step):
        nl = oracle_lib.neighbors(x, s["lo"], s["hi"], 2.5, "fp64")
        near = oracle_lib.near_force(x, s["lo"], s["hi"], 2.5, nl, type=s["type"], charge=s["charge"],
                                     eps=s["eps"], sigma=s["sigma"], with_coul=True, alpha=alpha, prec="fp64")
        m = oracle_lib.rbe_sample(alpha, L, 77, step, 0, P)
        rho = oracle_lib.rhok(x, s["charge"], L, m)
        return near + oracle_lib.rbe_force(x, s["charge"], L, alpha, 1.0, m, rho)

    x, v, m = s["pos"].copy(), s["vel"].copy(), s["mass"][:, None]
    F = force(x, 0)
    for step in range(2):
        v = v + 0.5 * F / m * dt
        x = _wrap(x + v * dt, s["lo"], s["hi"])
        F = force(x, step)
        v = v + 0.5 * F / m * dt
    assert np.abs(dev["pos"].cpu().numpy() - x).max() < 1e-9
    assert rel_err(dev["force"].cpu().numpy(), F) < 1e-10


def test_water_shake_rattle_step_fp64(cuda, oracle_lib):
    import torch
    s = systems.water(n_mol=300, seed=2)
    P = 32
    cfg = systems.water_config(P=P, precision="fp64", shake_tol=1e-10)
    cfg["execution"]["ensemble"] = "NVE"
    cfg["hyper_parameters"]["extend"]["shake_max_iter"] = 500
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    rc = cfg["hyper_parameters"]["neighbor"]["cut_off"]
    dt = cfg["execution"]["timestep"]
    fmt2v, qqr2e = 4.186e-4, 332.06371
    L = s["hi"] - s["lo"]
    m_k = oracle_lib.rbe_sample(alpha, L, 5, 0, 0, P)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_ksamples(m_k)
    ff.Execute()
    F_dev0 = dev["force"].cpu().numpy().copy()

    def force(x):
        nl = oracle_lib.neighbors(x, s["lo"], s["hi"], rc, "fp64")
        near = oracle_lib.near_force(x, s["lo"], s["hi"], rc, nl, type=s["type"], mol=s["molecule"],
                                     charge=s["charge"], eps=s["eps"], sigma=s["sigma"], with_coul=True,
                                     alpha=alpha, coul_scale=qqr2e, prec="fp64")
        rho = oracle_lib.rhok(x, s["charge"], L, m_k)
        far = oracle_lib.rbe_force(x, s["charge"], L, alpha, qqr2e, m_k, rho)
        ex, _ = oracle_lib.water_extras(s["hoh"], x, s["charge"], s["lo"], s["hi"], *s["bond"], *s["angle"])
        return near + far + ex

    F0 = force(s["pos"])
    assert rel_err(F_dev0, F0) < 1e-10
    ff.step(1)
    torch.cuda.synchronize()
    assert ff.status() == 0
    m = s["mass"][:, None]
    x_old, v_old = s["pos"].copy(), s["vel"].copy()
    v = v_old + 0.5 * F0 / m * dt * fmt2v
    x = _wrap(x_old + v * dt, s["lo"], s["hi"])
    x, v, _, bad, _ = oracle_lib.shake(s["hoh"], x_old, v_old, F0, s["mass"], s["lo"], s["hi"], dt, fmt2v,
                                       tol=1e-10, max_iter=500)
    assert bad == 0
    F1 = force(x)
    v = oracle_lib.rattle(s["hoh"], x, v, F1, s["mass"], s["lo"], s["hi"], dt, fmt2v)
    got_x = dev["pos"].cpu().numpy()
    got_v = dev["vel"].cpu().numpy()
    assert np.abs(got_x - x).max() < 1e-9
    assert np.abs(got_v - v).max() < 1e-9
    # constraints hold: O-H = 1.0, H-H from 109.47 deg
    hoh = s["hoh"]
    d01 = np.linalg.norm(got_x[hoh[:, 1]] - got_x[hoh[:, 0]], axis=1)
    assert np.abs(d01 - 1.0).max() < 1e-6


def test_shake_nonconvergence_flag(cuda):
    import torch
    from copy_gpu_b200 import FLAG_SHAKE_NOCONV
    s = systems.water(n_mol=64, seed=3)
    cfg = systems.water_config(P=16, precision="fp64", shake_tol=0.0)
    cfg["hyper_parameters"]["extend"]["shake_max_iter"] = 3
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    ff.step(1)
    torch.cuda.synchronize()
    assert ff.status() & FLAG_SHAKE_NOCONV


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_eam_johnson(cuda, oracle_lib, tmp_path, prec):
    import torch
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=8, seed=5)
    cfg = systems.eam_config(pot, precision=prec)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    pr = s["pos"].astype(np.float32 if prec == "fp32" else np.float64)
    nl = oracle_lib.neighbors(pr, s["lo"], s["hi"], 5.0, prec)
    ref, _ = oracle_lib.eam_force(pot, pr, s["lo"], s["hi"], 5.0, nl, prec=prec, sum_mode=1)
    err = rel_err(dev["force"].cpu().numpy(), ref)
    assert err < (1e-5 if prec == "fp32" else 1e-11), err


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_eam_setfl_matches_analytic_johnson(cuda, tmp_path, prec):
    """A single-element setfl file of Johnson's EAM (tables on the file grid, r*phi given
    directly) reproduces the analytic forces F_i = -sum_j [(F'(rho_i) + F'(rho_j)) f'(r) + phi'(r)]
    (r_i - r_j) / r, FP64 in numpy over all minimum-image pairs within the cutoff.  The spline
    tables are float (as the reference's): their derivative coefficients carry rounding of about
    4e-5 relative (a difference of values divided by dr = 1e-3), which the near-cancelling pair
    terms of a crystal amplify to 4e-4 of the rms force, in FP32 and FP64 runs alike; the bar is
    1e-3.  A table offset by one grid point (the funcfl reader's quirk) would give 8e-3.  The
    crystal is stressed (phi_e = 0.59 eV instead of the benchmark's equilibrium 0.2235 eV), so
    its forces stand well above the tables' rounding; at equilibrium only the thermal
    displacements are left and the same rounding reads 2.5e-3 of their rms."""
    import torch
    p = dict(systems.JOHNSON_CU, phi_e=0.59)
    path = systems.write_johnson_setfl(str(tmp_path / "johnson.eam.alloy"), p)
    s = systems.eam_fcc(ncell=6, seed=8)
    cfg = systems.eam_config(path, precision=prec)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    got = dev["force"].cpu().numpy()
    x = s["pos"]
    L = s["hi"] - s["lo"]
    d = x[:, None, :] - x[None, :, :]            # r_i - r_j
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))
    inside = (r < p["cutoff"]) & (r > 0.1)
    rs = np.where(inside, r, 1.0)
    f, fp, phi, phip = systems.johnson_terms(rs, p)
    rho = np.where(inside, f, 0.0).sum(1)
    Fp = -p["Ec"] / (2.0 * np.sqrt(rho * p["rho_e"]))
    coef = np.where(inside, (Fp[:, None] + Fp[None, :]) * fp + phip, 0.0) / rs
    ref = -(coef[:, :, None] * d).sum(1)
    err = rel_err(got, ref)
    assert err < 1e-3, err


def test_batched_replicas_match_single(cuda):
    """Replica 0 advanced inside a batch equals replica 0 advanced alone (its sampler stream is
    keyed by replica index 0 in both runs)."""
    import torch
    r = systems.replicas(n_rep=6, nmin=500, nmax=1500, seed=5)
    P = 24
    cfg = systems.electrolyte_config(P=P, precision="fp64", seed=31, ensemble="NVE")
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(6)]
    dev = to_dev(r, cuda)
    ff = make_ff(cfg, r, dev, boxes=boxes, offsets=r["offsets"])
    ff.Execute()
    ff.step(3)
    torch.cuda.synchronize()
    assert ff.status() == 0
    got = dev["pos"].cpu().numpy()
    off = r["offsets"]
    sl = slice(off[0], off[1])
    n0 = off[1]
    s0 = {key: (val[sl] if isinstance(val, np.ndarray) and val.shape[:1] == (off[-1],) else val)
          for key, val in r.items()}
    s0["lo"], s0["hi"] = r["lo"][0], r["hi"][0]
    assert s0["pos"].shape[0] == n0
    dev0 = to_dev(s0, cuda)
    ff0 = make_ff(cfg, s0, dev0)
    ff0.Execute()
    ff0.step(3)
    torch.cuda.synchronize()
    assert np.abs(dev0["pos"].cpu().numpy() - got[sl]).max() < 1e-12


def test_per_replica_rebuild_matches_single(cuda):
    """With a Verlet skin each replica rebuilds its own list when its own atoms moved more than
    skin/2: after 60 FP32 steps replica 0 of a batch matches replica 0 advanced alone (1e-6 in
    positions; its k-sampler stream is keyed by replica index 0 in both runs), the batch rebuilt
    as many replica lists as the replicas alone did, and fewer than one rebuild of every replica
    per step on which any replica rebuilds."""
    import torch
    r = systems.replicas(n_rep=4, nmin=700, nmax=1600, seed=21)
    cfg = systems.electrolyte_config(P=16, precision="fp32", seed=9, ensemble="NVE")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    cfg["tuning"] = {"list_block": 128, "force_block": 128}
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(4)]
    dev = to_dev(r, cuda)
    ff = make_ff(cfg, r, dev, boxes=boxes, offsets=r["offsets"])
    ff.Execute()
    ff.step(60)
    torch.cuda.synchronize()
    assert ff.status() == 0
    got = dev["pos"].cpu().numpy()
    builds_batch = ff.list_builds()
    off = r["offsets"]
    singles = []
    for k in range(4):
        sl = slice(off[k], off[k + 1])
        sk = {key: (val[sl] if isinstance(val, np.ndarray) and val.shape[:1] == (off[-1],) else val)
              for key, val in r.items()}
        sk["lo"], sk["hi"] = r["lo"][k], r["hi"][k]
        devk = to_dev(sk, cuda)
        ffk = make_ff(cfg, sk, devk)
        ffk.Execute()
        ffk.step(60)
        torch.cuda.synchronize()
        singles.append(ffk.list_builds())
        if k == 0:   # the k-sampler streams are keyed by replica index: only replica 0 matches alone
            assert np.abs(devk["pos"].cpu().numpy() - got[sl]).max() < 1e-6
    assert abs(builds_batch - sum(singles)) <= 2, (builds_batch, singles)
    assert builds_batch < 4 * max(singles), (builds_batch, singles)


def test_batched_replicas_injected_k(cuda, oracle_lib):
    """With injected k-samples every replica's force equals its stand-alone force."""
    import torch
    r = systems.replicas(n_rep=5, nmin=600, nmax=1200, seed=6)
    P = 20
    cfg = systems.electrolyte_config(P=P, precision="fp64", seed=3)
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    boxes = [Box(tuple(r["lo"][k]), tuple(r["hi"][k])) for k in range(5)]
    ks = np.concatenate([oracle_lib.rbe_sample(alpha, r["hi"][k] - r["lo"][k], 9, 0, k, P) for k in range(5)])
    dev = to_dev(r, cuda)
    ff = make_ff(cfg, r, dev, boxes=boxes, offsets=r["offsets"])
    ff.set_ksamples(ks)
    ff.Execute()
    torch.cuda.synchronize()
    F = dev["force"].cpu().numpy()
    off = r["offsets"]
    for k in range(5):
        sl = slice(off[k], off[k + 1])
        x = r["pos"][sl]
        L = r["hi"][k] - r["lo"][k]
        nl = oracle_lib.neighbors(x, r["lo"][k], r["hi"][k], 2.5, "fp64")
        near = oracle_lib.near_force(x, r["lo"][k], r["hi"][k], 2.5, nl, type=r["type"][sl],
                                     charge=r["charge"][sl], eps=r["eps"], sigma=r["sigma"],
                                     with_coul=True, alpha=alpha, prec="fp64")
        m = ks[k * P:(k + 1) * P]
        rho = oracle_lib.rhok(x, r["charge"][sl], L, m, origin=r["lo"][k])
        far = oracle_lib.rbe_force(x, r["charge"][sl], L, alpha, 1.0, m, rho, origin=r["lo"][k])
        assert rel_err(F[sl], near + far) < 1e-11


def test_nonfinite_position_flag(cuda):
    import torch
    from copy_gpu_b200 import FLAG_NONFINITE
    s = systems.lj_fcc(ncell=4)
    s["pos"][7, 1] = np.nan
    cfg = systems.lj_config(precision="fp32")
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() & FLAG_NONFINITE


def test_list_capacity_regrowth(cuda, oracle_lib):
    """An initial list capacity of 4 overflows; the library grows it and recomputes."""
    import torch
    s = systems.lj_fcc(ncell=5, seed=9)
    s["pos"] = jitter(s["pos"], s["lo"], s["hi"], 0.05, seed=2)
    cfg = systems.lj_config(precision="fp64")
    cfg["hyper_parameters"]["neighbor"]["capacity"] = 4
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    torch.cuda.synchronize()
    assert ff.status() == 0
    nl = oracle_lib.neighbors(s["pos"], s["lo"], s["hi"], 2.5, "fp64")
    ref = oracle_lib.near_force(s["pos"], s["lo"], s["hi"], 2.5, nl, prec="fp64")
    assert rel_err(dev["force"].cpu().numpy(), ref) < 1e-11
    ff.step(3)
    torch.cuda.synchronize()
    assert ff.status() == 0


@pytest.mark.parametrize("proposal", ["gauss", "learned"])
def test_cuda_graph_replay_is_bit_identical(cuda, proposal):
    """rbmd_force_step replays a captured step (one graph launch per step); positions and
    velocities after 25 steps equal those of direct launches bit for bit (every kernel is
    deterministic and the samplers read the step index from the device counter)."""
    import torch
    from oracle import mlp
    out = []
    for graph in (True, False):
        s = systems.electrolyte(3000, seed=17)
        cfg = systems.electrolyte_config(P=48, precision="fp32", seed=5)
        cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
        cfg["hyper_parameters"]["coulomb"]["proposal"] = proposal
        cfg["execution"]["cuda_graph"] = graph
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        if proposal == "learned":
            ff.proposal_params(mlp.init_params(2, scale=0.5))
        ff.Execute()
        ff.step(25)
        ff.sync_velocities()
        torch.cuda.synchronize()
        assert ff.status() == 0
        out.append((dev["pos"].cpu().numpy(), dev["vel"].cpu().numpy(), ff.list_builds()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


@pytest.mark.parametrize("skin", [0.0, 1.0])
def test_cuda_graph_water_shake(cuda, skin):
    """SHAKE water through graph replay equals direct launches bit for bit; with a Verlet skin the
    captured steps hold the cell sort and list build in a conditional node and re-gather the slot
    caches after it on list-reuse steps."""
    import torch
    out = []
    for graph in (True, False):
        s = systems.water(n_mol=300, seed=4)
        cfg = systems.water_config(P=32, precision="fp32")
        cfg["hyper_parameters"]["neighbor"]["skin"] = skin
        cfg["execution"]["cuda_graph"] = graph
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        ff.Execute()
        ff.step(40)
        ff.sync_velocities()
        torch.cuda.synchronize()
        assert ff.status() == 0
        out.append((dev["pos"].cpu().numpy(), ff.list_builds()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and (skin == 0 or out[0][1] >= 2)


def test_graph_steps_and_state_changes(cuda):
    """execution.graph_steps: 8 steps per graph launch give the same trajectory bit for bit as one
    step per graph launch; a k-set injected between step() calls reaches the replayed steps
    (the captured graphs are dropped when host-side state they depend on changes)."""
    import torch
    out = []
    for gs in (1, 8, None):
        s = systems.electrolyte(3000, seed=18)
        cfg = systems.electrolyte_config(P=32, precision="fp32", seed=5)
        cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
        if gs is None:
            cfg["execution"]["cuda_graph"] = False
        else:
            cfg["execution"]["graph_steps"] = gs
        dev = to_dev(s, cuda)
        ff = make_ff(cfg, s, dev)
        ff.Execute()
        ff.step(20)
        m = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0]] * 8, np.int32)
        ff.set_ksamples(m)
        ff.step(20)
        ff.sync_velocities()
        torch.cuda.synchronize()
        assert ff.status() == 0
        out.append((dev["pos"].cpu().numpy(), dev["vel"].cpu().numpy()))
        ff.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])


def test_water_shake_nve_energy_conservation_fp64(cuda):
    """SPC/E water with SHAKE/RATTLE, LJ + erfc + Ewald k-space (deterministic), FP64, skin 1 A,
    CUDA-graph steps of 2 fs: after 300 Berendsen steps, 1000 NVE steps keep the total energy
    (kinetic + LJ + Coulomb real / k-space / self / intramolecular correction + bond + angle)
    within 1e-3 of the kinetic energy (measured at 10,000 molecules: 1.2e-4 over 2000 steps)."""
    import copy
    import torch
    s = systems.water(n_mol=2000, seed=9)
    cfg = systems.water_config(P=200, precision="fp64", shake_tol=1e-6)
    cfg["hyper_parameters"]["coulomb"] = {"type": "EWALD", "alpha": 0.09, "kmax": 5}
    cfg["hyper_parameters"]["neighbor"]["skin"] = 1.0
    nvt = copy.deepcopy(cfg)
    nvt["execution"].update({"ensemble": "NVT", "temp_ctrl_type": "BERENDSEN",
                             "temperature": [298.0, 298.0, 100.0]})
    cfg["execution"]["ensemble"] = "NVE"
    dev = to_dev(s, cuda)
    ff = make_ff(nvt, s, dev)
    ff.Execute()
    ff.step(300)
    ff.sync_velocities()
    torch.cuda.synchronize()
    assert ff.status() == 0
    ff.close()
    ff = make_ff(cfg, s, dev)
    keys = ("lj", "coul_real", "coul_kspace", "coul_self", "bond", "angle", "coul_special")

    def total():
        ff.step(1)
        ff.Execute()
        e = ff.energy()
        return e["kinetic"] + sum(e[k] for k in keys), e

    e0, d0 = total()
    for _ in range(5):
        ff.step(200)
        torch.cuda.synchronize()
        assert ff.status() == 0
        e, _ = total()
        assert abs(e - e0) <= 1e-3 * d0["kinetic"], (e, e0, d0["kinetic"])
    ff.close()


def test_eam_nve_energy_conservation_fp64(cuda, tmp_path):
    """Johnson EAM (funcfl tables), FP64, skin 0.3, CUDA-graph steps of 1 fs: after 200 steps,
    1000 NVE steps keep kinetic + embedding + pair energy within 1e-3 of the kinetic energy
    (measured at 256,000 atoms: 4.8e-4 over the 1000 steps; the tables are not shifted to zero
    at the cutoff)."""
    import torch
    pot = systems.write_johnson_funcfl(str(tmp_path / "johnson.eam"))
    s = systems.eam_fcc(ncell=12, seed=13)
    cfg = systems.eam_config(pot, precision="fp64")
    cfg["hyper_parameters"]["neighbor"]["skin"] = 0.3
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    ff.step(200)
    torch.cuda.synchronize()

    def total():
        ff.step(1)
        ff.Execute()
        e = ff.energy()
        return e["kinetic"] + e["eam_embed"] + e["eam_pair"], e

    e0, d0 = total()
    for _ in range(5):
        ff.step(200)
        torch.cuda.synchronize()
        assert ff.status() == 0
        e, _ = total()
        assert abs(e - e0) <= 1e-3 * d0["kinetic"], (e, e0, d0["kinetic"])
    ff.close()
