"""C-ABI and host-logic tests that need no GPU: the library loads, exports every symbol
include/rbmd_force.h declares, and parses RBMD configuration text (accepting the reference's
keys, rejecting malformed input with status codes instead of exiting)."""
import json
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "rbmd_force.h")).read()
    return sorted(set(re.findall(r"^RBMD_API\s+[\w\s\*]+?\b(rbmd_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_header_symbol():
    import copy_gpu_b200 as c
    lib = c.library()
    syms = header_symbols()
    assert len(syms) >= 20
    for name in syms:
        assert hasattr(lib, name), name
    assert sorted(c.EXPORTED) == syms
    assert "sm_100a" in c.version()


def test_library_is_sm100a_only():
    """The shared object carries an sm_100a cubin (checked through cuobjdump's listing of the
    embedded ELF architectures, not its code)."""
    import shutil
    import subprocess
    import copy_gpu_b200 as c
    tool = shutil.which("cuobjdump") or "/usr/local/cuda/bin/cuobjdump"
    if not os.path.exists(tool):
        pytest.skip("cuobjdump not available")
    out = subprocess.run([tool, "--list-elf", c.LIB_PATH], capture_output=True, text=True).stdout
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def _box(L=10.0):
    from copy_gpu_b200 import Box
    return Box((0.0, 0.0, 0.0), (L, L, L))


def test_create_accepts_reference_keys():
    from copy_gpu_b200 import ForceField, systems
    for cfg in (systems.lj_config(), systems.electrolyte_config(), systems.water_config()):
        ff = ForceField(cfg, _box(30.0))
        ff.close()


def test_create_accepts_comments_and_verlet_list_spelling():
    from copy_gpu_b200 import ForceField
    text = """{
      // RBMD files carry comments
      "init_configuration": {"read_data": {"file": "x.data", "unit": "LJ", "atom_style": "charge"}},
      "hyper_parameters": {
        "force_field": {"type": "LJ/CUT/COUL/LONG"},
        "neighbor": {"type": "VERLET-LIST", "cut_off": 2.5, "r_core": 1.0, "neighbor_sample_num": 10},
        "coulomb": {"type": "RBE", "coulomb_sample_num": 100, "alpha": 0.5, "kmax": 2},
        /* block comment */
        "extend": {"fix_shake": "null", "special_bonds": [0, 0, 0]}
      },
      "execution": {"ensemble": "NVT", "temperature": [1.0, 1.0, 0.5], "temp_ctrl_type": "BERENDSEN",
                    "timestep": 0.002, "num_steps": 10}
    }"""
    ff = ForceField(text, _box())
    ff.close()


@pytest.mark.parametrize("bad", [
    "{not json",
    json.dumps({"hyper_parameters": {"force_field": {"type": "LJ/CUT"}, "neighbor": {"type": "VERLETLIST"}}}),
    json.dumps({"hyper_parameters": {"force_field": {"type": "TERSOFF"},
                                     "neighbor": {"type": "VERLETLIST", "cut_off": 2.5}}}),
    json.dumps({"hyper_parameters": {"force_field": {"type": "LJ/CUT/COUL/LONG"},
                                     "neighbor": {"type": "VERLETLIST", "cut_off": 2.5},
                                     "coulomb": {"type": "PPPM", "coulomb_sample_num": 10, "alpha": 0.3}}}),
])
def test_create_rejects_bad_config(bad):
    from copy_gpu_b200 import ForceField, RbmdError
    with pytest.raises(RbmdError, match="ERR_CONFIG"):
        ForceField(bad, _box())


def test_create_rejects_degenerate_box():
    from copy_gpu_b200 import Box, ForceField, RbmdError, systems
    with pytest.raises(RbmdError, match="ERR_ARG"):
        ForceField(systems.lj_config(), Box((0, 0, 0), (5.0, 0.0, 5.0)))


def test_missing_potential_file_is_an_error():
    from copy_gpu_b200 import ForceField, RbmdError, systems
    with pytest.raises(RbmdError, match="ERR_FILE"):
        ForceField(systems.eam_config("/nonexistent/potential.eam"), _box(40.0))


def test_pair_coeff_bounds():
    from copy_gpu_b200 import ForceField, RbmdError, systems
    ff = ForceField(systems.lj_config(), _box())
    ff.set_pair_coeffs([1.0, 0.5], [1.0, 1.2])
    with pytest.raises(RbmdError):
        ff.set_pair_coeffs(np.ones(17), np.ones(17))
    ff.close()


def test_as_7_1_26_erfc_bound():
    """The FP32 real-space kernel evaluates erfc with Abramowitz & Stegun 7.1.26 reusing
    exp(-x^2); its published bound |err| <= 1.5e-7 holds over the range the cutoff produces."""
    p, a = 0.3275911, (0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429)
    x = np.linspace(0.0, 6.0, 20001)
    t = 1.0 / (1.0 + p * x)
    poly = a[4]
    for c in reversed(a[:4]):
        poly = poly * t + c
    approx = poly * t * np.exp(-x * x)
    exact = np.array([math.erfc(v) for v in x])
    assert np.abs(approx - exact).max() <= 1.5e-7


def test_struct_layouts_match_the_header(tmp_path):
    """Every public struct of include/rbmd_force.h has the size and field offsets of its ctypes
    mirror in copy_gpu_b200 (a C program compiled against the header prints them)."""
    import ctypes
    import shutil
    import subprocess
    import copy_gpu_b200 as c
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"rbmd_box": c.rbmd_box, "rbmd_atoms_dev": c.rbmd_atoms_dev, "rbmd_energy": c.rbmd_energy,
               "rbmd_topology": c.rbmd_topology, "rbmd_train_opts": c.rbmd_train_opts,
               "rbmd_train_report": c.rbmd_train_report, "rbmd_data_info": c.rbmd_data_info,
               "rbmd_data_arrays": c.rbmd_data_arrays}
    lines = ['#include <stdio.h>', '#include "rbmd_force.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-std=c11", "-I", inc, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        name, what, val = line.split()
        cls = structs[name]
        got = ctypes.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert got == int(val), (name, what, got, val)
