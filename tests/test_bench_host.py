"""Host-side pieces of bench.py that need no GPU: the secondary configurations it builds and the
CPU oracle leg that times them (run here on small versions of the same systems)."""
import numpy as np
import pytest

import bench
from copy_gpu_b200 import systems


@pytest.mark.parametrize("name", ["lj", "water", "eam", "batched"])
def test_config_systems(tmp_path, name):
    s, cfg, boxes, offs, desc = bench.config_system(name, str(tmp_path))
    n = s["pos"].shape[0]
    assert desc and cfg["hyper_parameters"]["neighbor"]["cut_off"] > 0
    assert np.all(s["pos"] >= (s["lo"] if s["lo"].ndim == 1 else s["lo"].min(0)) - 1e-9)
    if name == "batched":
        assert len(boxes) == 512 and offs[-1] == n
    else:
        assert boxes is None and offs is None
    if name == "eam":
        assert cfg["hyper_parameters"]["force_field"]["type"] == "EAM"


@pytest.mark.parametrize("name", ["lj", "water", "eam", "batched"])
def test_cpu_config_eval_small(tmp_path, name, oracle_lib):
    s, cfg, boxes, offs, _ = bench.config_system(name, str(tmp_path))
    if name == "water":
        s = systems.water(n_mol=300, seed=2)
    elif name == "eam":
        s = systems.eam_fcc(ncell=6, seed=2)
    sec, atoms = bench.cpu_config_eval(name, s, cfg, offs, str(tmp_path))
    assert sec > 0 and atoms > 0
    if name == "batched":
        assert atoms == int(offs[16])
    else:
        assert atoms == s["pos"].shape[0]
