"""Host-side pieces of bench.py that need no GPU: the secondary configurations it builds and the
CPU oracle leg that times them (run here on small versions of the same systems)."""
import numpy as np
import pytest

import bench
from copy_gpu_b200 import systems


@pytest.mark.parametrize("name", ["lj", "water", "eam", "batched", "molecular", "molecular_verlet"])
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
    if name.startswith("molecular"):
        assert cfg["hyper_parameters"]["neighbor"]["type"] == ("RBL" if name == "molecular" else "VERLETLIST")
        assert len(s["dihedrals"]) > 0 and abs(s["charge"].sum()) < 1e-9


@pytest.mark.parametrize("name", ["lj", "water", "eam", "batched", "molecular"])
def test_cpu_config_eval_small(tmp_path, name, oracle_lib):
    if name == "molecular":   # the workload's configuration on a small system of the same kind
        cfg = systems.molecular_config(P=100, cutoff=12.0, alpha=0.074, neighbor="RBL", special=(0.0, 0.0, 0.0),
                                       precision="fp32", r_core=6.0, sample_num=100)
        s = systems.molecular(n_chain=64, chain_len=12, n_ion_pairs=16, step=1.5, cell=6.0, seed=3)
        sec, atoms = bench.cpu_config_eval(name, s, cfg, None, str(tmp_path))
        assert sec > 0 and atoms == s["pos"].shape[0]
        return
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
