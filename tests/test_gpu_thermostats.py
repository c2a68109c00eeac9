"""NVT thermostats against a restatement of the reference's step (FP64).

ExecutionNVT::Solve (rbmd/framework/run/ExecutionNVT.cpp:133-159): kick, drift + wrap, force,
kick, ComputeTempe (:749-786, dof 3n - 3 without SHAKE), then UpdateVelocityByTempConType
(:256-290):
* NOSE_HOOVER: v += dt/2 (F/m - xi v) fmt2v with the current xi
  (UpdateVelocityNoseHooverWorklet, RunWorklet.cpp:1784-1804), then
  xi += dt/2 (T/T0 - 1) / tauT with tauT = 0.1 dt;
* TEMP_RESCALE: v *= sqrt(T0 / T);
* BERENDSEN: v *= sqrt(1 + dt/Tdamp (T0/T - 1)), Tdamp = temperature[2].
Three steps of an LJ crystal started well below the target T0 = 1.5 (so every thermostat acts on
every step), positions and velocities to 1e-9, the device temperature to 1e-12 relative.
"""
import numpy as np
import pytest

from copy_gpu_b200 import systems
from tests.helpers import jitter, make_ff, to_dev

pytestmark = pytest.mark.gpu


def _force(o, x, s):
    nl = o.neighbors(x, s["lo"], s["hi"], 2.5, "fp64")
    return o.near_force(x, s["lo"], s["hi"], 2.5, nl, prec="fp64")


@pytest.mark.parametrize("tctrl", ["NOSE_HOOVER", "TEMP_RESCALE", "BERENDSEN"])
def test_thermostat_steps_match_reference_restatement(cuda, oracle_lib, tctrl):
    import torch
    s = systems.lj_fcc(ncell=5, seed=11)
    s["pos"] = jitter(s["pos"], s["lo"], s["hi"], 0.04, seed=3)
    T0, Tdamp = 1.5, 0.1
    cfg = systems.lj_config(cutoff=2.5, precision="fp64", ensemble="NVT")
    cfg["execution"].update({"temp_ctrl_type": tctrl, "temperature": [T0, T0, Tdamp]})
    dt = cfg["execution"]["timestep"]
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.Execute()
    nsteps = 3
    ff.step(nsteps)
    ff.sync_velocities()
    torch.cuda.synchronize()
    assert ff.status() == 0
    T_dev = ff.energy()["temperature"]
    ff.close()

    lo, hi = s["lo"], s["hi"]
    L = hi - lo
    x, v = s["pos"].copy(), s["vel"].copy()
    m = s["mass"][:, None]
    n = x.shape[0]
    F = _force(oracle_lib, x, s)
    xi = 0.0
    T, Ts = None, []
    for _ in range(nsteps):
        v = v + 0.5 * dt * F / m
        x = x + v * dt
        x = np.where(x < lo, x + L, np.where(x > hi, x - L, x))
        F = _force(oracle_lib, x, s)
        v = v + 0.5 * dt * F / m
        T = 0.5 * (m[:, 0] * (v ** 2).sum(1)).sum() / ((3 * n - 3) / 2.0)
        Ts.append(T)
        if tctrl == "NOSE_HOOVER":
            v = v + 0.5 * dt * (F / m - xi * v)
            xi += 0.5 * dt * (T / T0 - 1.0) / (0.1 * dt)
        elif tctrl == "TEMP_RESCALE":
            v = v * np.sqrt(T0 / T)
        else:
            v = v * np.sqrt(1.0 + dt / Tdamp * (T0 / T - 1.0))
    assert Ts[0] < 0.9 * T0      # the thermostat had work to do
    assert np.abs(dev["pos"].cpu().numpy() - x).max() < 1e-9
    assert np.abs(dev["vel"].cpu().numpy() - v).max() < 1e-9
    assert abs(T_dev - T) <= 1e-12 * T, (T_dev, T)
