"""copy_gpu_b200 -- RBMD's per-timestep force path on B200 (sm_100a), behind a C ABI.

The compute lives in ``librbmd_b200.so`` (CUDA kernels + C++ host driver, declared in
``include/rbmd_force.h``).  This module is the thin Python host mirror of the reference's
force-field interface: :class:`ForceField` is configured from RBMD's JSON text and exposes
``Init`` / ``Execute`` like the HIP tree's ``class Force``
(rbmd-gpu-clone/rbmd-gpu/src/force/include/force.h:8-25) plus the full step of
``ExecutionNVT::Solve`` (rbmd/framework/run/ExecutionNVT.cpp:133-159).

There is no CPU fallback: importing works without a GPU (for building and symbol checks), but
every compute call requires the CUDA library and a device and raises otherwise.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librbmd_b200.so")

RBMD_OK = 0
RBMD_ERR_ARG, RBMD_ERR_CONFIG, RBMD_ERR_CUDA, RBMD_ERR_STATE, RBMD_ERR_DEVICE, RBMD_ERR_FILE = 1, 2, 3, 4, 5, 6
STATUS_NAMES = {1: "ERR_ARG", 2: "ERR_CONFIG", 3: "ERR_CUDA", 4: "ERR_STATE", 5: "ERR_DEVICE",
                6: "ERR_FILE"}
FLAG_LIST_OVERFLOW = 0x01
FLAG_CELL_OVERFLOW = 0x02
FLAG_SHAKE_NOCONV = 0x04
FLAG_NONFINITE = 0x08
FLAG_OUT_OF_BOX = 0x10
FLAG_SAMPLER = 0x20
FLAG_SHAKE_SINGULAR = 0x40

# every symbol include/rbmd_force.h declares
EXPORTED = [
    "rbmd_force_create", "rbmd_force_set_pair_coeffs", "rbmd_force_load_funcfl",
    "rbmd_force_set_water", "rbmd_force_set_topology", "rbmd_force_bind", "rbmd_force_set_ksamples",
    "rbmd_force_set_kweights", "rbmd_force_get_ksamples", "rbmd_force_sample_k",
    "rbmd_force_compute", "rbmd_force_autotune", "rbmd_force_compute_host", "rbmd_force_compute_host_f32",
    "rbmd_force_step",
    "rbmd_force_sync_velocities", "rbmd_force_energy", "rbmd_force_status",
    "rbmd_force_get_neighbors", "rbmd_force_get_rbl", "rbmd_force_get_rhok", "rbmd_force_profile",
    "rbmd_force_phase_ms", "rbmd_force_list_builds", "rbmd_force_launch_count",
    "rbmd_force_train_proposal", "rbmd_force_proposal_params", "rbmd_force_get_far",
    "rbmd_force_destroy", "rbmd_rhok_noalloc", "rbmd_proposal_mlp_eval", "rbmd_data_read",
    "rbmd_data_atoms", "rbmd_data_types", "rbmd_data_topology", "rbmd_data_dihedrals", "rbmd_data_free",
    "rbmd_data_write", "rbmd_data_write_arrays",
    "rbmd_version",
    "rbmd_last_error",
]


class RbmdError(RuntimeError):
    pass


class rbmd_box(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3)]


class rbmd_atoms_dev(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int64),
        ("n_replicas", ctypes.c_int32),
        ("replica_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("pos", ctypes.c_void_p),
        ("vel", ctypes.c_void_p),
        ("force", ctypes.c_void_p),
        ("mass", ctypes.c_void_p),
        ("charge", ctypes.c_void_p),
        ("type", ctypes.c_void_p),
        ("molecule", ctypes.c_void_p),
        ("image", ctypes.c_void_p),
    ]


class rbmd_energy(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "lj", "coul_real", "coul_kspace", "coul_self", "eam_embed", "eam_pair", "bond", "angle",
        "kinetic", "temperature", "dihedral", "coul_special")]


class rbmd_data_info(ctypes.Structure):
    _fields_ = [("n_atoms", ctypes.c_int64), ("n_bonds", ctypes.c_int64), ("n_angles", ctypes.c_int64),
                ("n_atom_types", ctypes.c_int32), ("n_bond_types", ctypes.c_int32), ("n_angle_types", ctypes.c_int32),
                ("has_velocities", ctypes.c_int32), ("has_pair_coeffs", ctypes.c_int32), ("has_masses", ctypes.c_int32),
                ("box", rbmd_box), ("n_dihedrals", ctypes.c_int64), ("n_dihedral_types", ctypes.c_int32)]


class rbmd_data_arrays(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "pos", "vel", "charge", "type", "molecule", "image", "mass_by_type", "epsilon", "sigma",
        "bonds", "bond_type", "bond_coeffs", "angles", "angle_type", "angle_coeffs",
        "dihedrals", "dihedral_type", "dihedral_coeffs")]


class rbmd_topology(ctypes.Structure):
    _fields_ = [("n_atoms", ctypes.c_int64), ("molecule", ctypes.c_void_p),
                ("n_bonds", ctypes.c_int64), ("bonds", ctypes.c_void_p), ("bond_type", ctypes.c_void_p),
                ("n_bond_types", ctypes.c_int32), ("bond_coeffs", ctypes.c_void_p),
                ("n_angles", ctypes.c_int64), ("angles", ctypes.c_void_p), ("angle_type", ctypes.c_void_p),
                ("n_angle_types", ctypes.c_int32), ("angle_coeffs", ctypes.c_void_p),
                ("n_dihedrals", ctypes.c_int64), ("dihedrals", ctypes.c_void_p), ("dihedral_type", ctypes.c_void_p),
                ("n_dihedral_types", ctypes.c_int32), ("dihedral_coeffs", ctypes.c_void_p)]


class rbmd_train_opts(ctypes.Structure):
    _fields_ = [("n_snapshots", ctypes.c_int32), ("steps_between", ctypes.c_int32),
                ("k_per_snapshot", ctypes.c_int32), ("iterations", ctypes.c_int32),
                ("learning_rate", ctypes.c_float), ("seed", ctypes.c_uint64)]


class rbmd_train_report(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "loss_gauss", "loss_first", "loss_final", "loss_optimum", "variance_ratio", "seconds")]


_lib = None


def library() -> ctypes.CDLL:
    """Load the CUDA force library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RbmdError(f"{LIB_PATH} is missing: run `python -m copy_gpu_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P, I32, I64, D, V = ctypes.POINTER, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    sig = {
        "rbmd_force_create": (I32, [ctypes.c_char_p, I32, P(rbmd_box), P(V)]),
        "rbmd_force_set_pair_coeffs": (I32, [V, I32, P(D), P(D)]),
        "rbmd_force_load_funcfl": (I32, [V, ctypes.c_char_p]),
        "rbmd_force_set_water": (I32, [V, I64, P(I32), D, D, D, D]),
        "rbmd_force_set_topology": (I32, [V, P(rbmd_topology)]),
        "rbmd_force_bind": (I32, [V, P(rbmd_atoms_dev)]),
        "rbmd_force_set_ksamples": (I32, [V, P(I32), I32]),
        "rbmd_force_set_kweights": (I32, [V, P(D)]),
        "rbmd_force_get_ksamples": (I32, [V, P(I32), I32]),
        "rbmd_force_sample_k": (I32, [V, I64, P(I32), I32]),
        "rbmd_force_compute": (I32, [V, V]),
        "rbmd_force_autotune": (I32, [V, V, P(I32), P(I32)]),
        "rbmd_force_compute_host": (I32, [V, P(D), P(D), V]),
        "rbmd_force_compute_host_f32": (I32, [V, P(ctypes.c_float), P(ctypes.c_float), V]),
        "rbmd_force_step": (I32, [V, I32, V]),
        "rbmd_force_sync_velocities": (I32, [V, V]),
        "rbmd_force_energy": (I32, [V, P(rbmd_energy), V]),
        "rbmd_force_status": (I32, [V, P(ctypes.c_uint32), I32, V]),
        "rbmd_force_get_neighbors": (I32, [V, P(I32), P(I32), I64]),
        "rbmd_force_get_rbl": (I32, [V, P(I32), P(I32), P(I64)]),
        "rbmd_force_get_rhok": (I32, [V, P(D), I32]),
        "rbmd_force_profile": (I32, [V, I32]),
        "rbmd_force_phase_ms": (I32, [V, P(D), P(I64), I32]),
        "rbmd_force_list_builds": (I32, [V, P(I64)]),
        "rbmd_force_launch_count": (I32, [V, P(I32)]),
        "rbmd_force_destroy": (None, [V]),
        "rbmd_rhok_noalloc": (I32, [V, V, I32, P(rbmd_box), V, I32, V, V]),
        "rbmd_proposal_mlp_eval": (I32, [V, V, V, V, I32, I32, V, V, V, V, V]),
        "rbmd_force_train_proposal": (I32, [V, P(rbmd_train_opts), P(rbmd_train_report), V]),
        "rbmd_force_proposal_params": (I32, [V, P(ctypes.c_float), P(ctypes.c_float)]),
        "rbmd_force_get_far": (I32, [V, P(D)]),
        "rbmd_data_read": (I32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, P(V), P(rbmd_data_info)]),
        "rbmd_data_atoms": (I32, [V, V, V, V, V, V, V, V]),
        "rbmd_data_types": (I32, [V, V, V, V]),
        "rbmd_data_topology": (I32, [V, V, V, V, V, V, V]),
        "rbmd_data_dihedrals": (I32, [V, V, V, V]),
        "rbmd_data_free": (None, [V]),
        "rbmd_data_write_arrays": (I32, [ctypes.c_char_p, ctypes.c_char_p, P(rbmd_data_info), P(rbmd_data_arrays)]),
        "rbmd_data_write": (I32, [ctypes.c_char_p, ctypes.c_char_p, P(rbmd_data_info), V, V, V, V, V, V, V, V, V,
                                  V, V]),
        "rbmd_version": (ctypes.c_char_p, []),
        "rbmd_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(st: int, what: str) -> None:
    if st != RBMD_OK:
        msg = library().rbmd_last_error().decode(errors="replace")
        raise RbmdError(f"{what} failed: {STATUS_NAMES.get(st, st)} {msg}")


def _ptr(t, ctype):
    import numpy as np
    if isinstance(t, np.ndarray):
        return t.ctypes.data_as(ctypes.POINTER(ctype))
    return ctypes.cast(t, ctypes.POINTER(ctype))


@dataclass
class Box:
    lo: tuple
    hi: tuple

    def c(self) -> rbmd_box:
        b = rbmd_box()
        for d in range(3):
            b.lo[d] = float(self.lo[d])
            b.hi[d] = float(self.hi[d])
        return b


class ForceField:
    """Force path selected by RBMD's configuration (force_field / neighbor / coulomb keys).

    Mirrors ``ExecutionNVT::ComputeAllForce`` (rbmd/framework/run/ExecutionNVT.cpp:185-222):
    ``LJ/CUT`` -> LJ over the full Verlet list; ``LJ/CUT/COUL/LONG`` -> far (RBE or EWALD) plus
    near (LJ + erfc); ``CVFF`` -> the same plus intramolecular Coulomb removal, bonds and angles;
    ``EAM`` -> the two EAM passes.  Atom arrays are torch CUDA tensors owned by the caller.
    """

    def __init__(self, config, boxes):
        if isinstance(config, dict):
            config = json.dumps(config)
        if isinstance(boxes, Box):
            boxes = [boxes]
        self.config_text = config
        self.boxes = list(boxes)
        lib = library()
        arr = (rbmd_box * len(self.boxes))(*[b.c() for b in self.boxes])
        h = ctypes.c_void_p()
        _check(lib.rbmd_force_create(config.encode(), len(self.boxes), arr, ctypes.byref(h)),
               "rbmd_force_create")
        self._h = h
        self._keep = []

    # ---- configuration --------------------------------------------------------------
    def set_pair_coeffs(self, eps, sigma):
        import numpy as np
        e = np.ascontiguousarray(eps, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        _check(library().rbmd_force_set_pair_coeffs(self._h, len(e), _ptr(e, ctypes.c_double),
                                                    _ptr(s, ctypes.c_double)), "set_pair_coeffs")

    def load_funcfl(self, path):
        _check(library().rbmd_force_load_funcfl(self._h, str(path).encode()), "load_funcfl")

    def set_water(self, hoh, bond_k, bond_r0, angle_k, angle_theta0_deg):
        import numpy as np
        t = np.ascontiguousarray(hoh, dtype=np.int32).reshape(-1)
        _check(library().rbmd_force_set_water(self._h, len(t) // 3, _ptr(t, ctypes.c_int32),
                                              float(bond_k), float(bond_r0), float(angle_k),
                                              float(angle_theta0_deg)), "set_water")

    def set_topology(self, molecule, bonds=None, bond_type=None, bond_coeffs=None, angles=None, angle_type=None,
                     angle_coeffs=None, dihedrals=None, dihedral_type=None, dihedral_coeffs=None):
        """General CVFF topology (rbmd_force_set_topology): 0-based atom ids, per-type harmonic
        coefficients bond (k, r0), angle (k, theta0 degrees), dihedral (K, sign, multiplicity)."""
        import numpy as np
        c = lambda a, t, w: np.zeros((0, w) if w else 0, t) if a is None else np.ascontiguousarray(a, t)  # noqa
        mol = c(molecule, np.int32, 0)
        b, bt, bc = c(bonds, np.int32, 2), c(bond_type, np.int32, 0), c(bond_coeffs, np.float64, 2)
        a, at, ac = c(angles, np.int32, 3), c(angle_type, np.int32, 0), c(angle_coeffs, np.float64, 2)
        d, dt, dc = c(dihedrals, np.int32, 4), c(dihedral_type, np.int32, 0), c(dihedral_coeffs, np.float64, 3)
        keep = [mol, b, bt, bc, a, at, ac, d, dt, dc]
        vp = lambda x: x.ctypes.data_as(ctypes.c_void_p) if x.size else None   # noqa: E731
        t = rbmd_topology(len(mol), vp(mol), len(b), vp(b), vp(bt), len(bc), vp(bc), len(a), vp(a), vp(at),
                          len(ac), vp(ac), len(d), vp(d), vp(dt), len(dc), vp(dc))
        _check(library().rbmd_force_set_topology(self._h, ctypes.byref(t)), "set_topology")
        del keep

    def Init(self, pos, force, *, vel=None, mass=None, charge=None, type=None, molecule=None,
             image=None, replica_offsets=None):
        """Bind caller-owned device tensors (ExecutionMD::Init, ExecutionMD.cpp:117-134)."""
        import numpy as np
        import torch
        for t in (pos, force):
            if not (isinstance(t, torch.Tensor) and t.is_cuda):
                raise RbmdError("ForceField.Init needs CUDA tensors (no CPU fallback)")
        a = rbmd_atoms_dev()
        a.n_atoms = pos.shape[0]
        nrep = len(self.boxes)
        a.n_replicas = nrep
        if nrep > 1:
            off = np.ascontiguousarray(replica_offsets, dtype=np.int64)
            self._keep.append(off)
            a.replica_offsets = off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        else:
            a.replica_offsets = None

        def p(t, dt):
            if t is None:
                return None
            if t.dtype != dt or not t.is_contiguous() or not t.is_cuda:
                raise RbmdError(f"tensor must be contiguous CUDA {dt}")
            self._keep.append(t)
            return t.data_ptr()
        a.pos = p(pos, torch.float64)
        a.force = p(force, torch.float64)
        a.vel = p(vel, torch.float64)
        a.mass = p(mass, torch.float64)
        a.charge = p(charge, torch.float64)
        a.type = p(type, torch.int32)
        a.molecule = p(molecule, torch.int32)
        a.image = p(image, torch.int32)
        _check(library().rbmd_force_bind(self._h, ctypes.byref(a)), "rbmd_force_bind")
        self.n = int(pos.shape[0])

    bind = Init

    # ---- work ---------------------------------------------------------------------------
    @staticmethod
    def _stream(stream):
        if stream is None:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        return ctypes.c_void_p(int(stream))

    def Execute(self, stream=None):
        """One force evaluation (Force::Execute / ExecutionNVT::ComputeForce)."""
        _check(library().rbmd_force_compute(self._h, self._stream(stream)), "rbmd_force_compute")

    compute = Execute

    def autotune(self, stream=None):
        """Pick the fastest threads-per-block of the list build and force pass; returns both."""
        a, b = ctypes.c_int32(), ctypes.c_int32()
        _check(library().rbmd_force_autotune(self._h, self._stream(stream), ctypes.byref(a), ctypes.byref(b)),
               "autotune")
        return int(a.value), int(b.value)

    def compute_host(self, pos_host, force_host, stream=None):
        """Force of host positions into host forces: float64 arrays use rbmd_force_compute_host,
        float32 arrays (the reference's Vec3f layout) rbmd_force_compute_host_f32."""
        import numpy as np
        if pos_host.dtype == np.float32:
            if force_host.dtype != np.float32:
                raise RbmdError("compute_host: float32 positions need float32 forces")
            _check(library().rbmd_force_compute_host_f32(self._h, _ptr(pos_host, ctypes.c_float),
                                                         _ptr(force_host, ctypes.c_float),
                                                         self._stream(stream)), "compute_host_f32")
            return
        _check(library().rbmd_force_compute_host(self._h, _ptr(pos_host, ctypes.c_double),
                                                 _ptr(force_host, ctypes.c_double),
                                                 self._stream(stream)), "compute_host")

    def step(self, n_steps=1, stream=None):
        _check(library().rbmd_force_step(self._h, int(n_steps), self._stream(stream)), "rbmd_force_step")

    def sync_velocities(self, stream=None):
        _check(library().rbmd_force_sync_velocities(self._h, self._stream(stream)), "sync_velocities")

    # ---- k-space -------------------------------------------------------------------------
    def set_ksamples(self, m):
        import numpy as np
        if m is None:
            _check(library().rbmd_force_set_ksamples(self._h, None, 0), "set_ksamples")
            return
        a = np.ascontiguousarray(m, dtype=np.int32).reshape(-1, 3)
        P = a.shape[0] // len(self.boxes)
        _check(library().rbmd_force_set_ksamples(self._h, _ptr(a, ctypes.c_int32), P), "set_ksamples")

    def set_kweights(self, w):
        import numpy as np
        if w is None:
            _check(library().rbmd_force_set_kweights(self._h, None), "set_kweights")
            return
        a = np.ascontiguousarray(w, dtype=np.float64)
        _check(library().rbmd_force_set_kweights(self._h, _ptr(a, ctypes.c_double)), "set_kweights")

    def get_ksamples(self, P):
        import numpy as np
        out = np.zeros((len(self.boxes) * P, 3), dtype=np.int32)
        _check(library().rbmd_force_get_ksamples(self._h, _ptr(out, ctypes.c_int32), P), "get_ksamples")
        return out

    def sample_k(self, step, P):
        import numpy as np
        out = np.zeros((len(self.boxes) * P, 3), dtype=np.int32)
        _check(library().rbmd_force_sample_k(self._h, int(step), _ptr(out, ctypes.c_int32), P), "sample_k")
        return out

    def get_rhok(self, P):
        import numpy as np
        out = np.zeros((len(self.boxes) * P, 2), dtype=np.float64)
        _check(library().rbmd_force_get_rhok(self._h, _ptr(out, ctypes.c_double), P), "get_rhok")
        return out

    # ---- learned k-proposal ---------------------------------------------------------------
    def train_proposal(self, n_snapshots=200, steps_between=10, k_per_snapshot=16384, iterations=1500,
                       learning_rate=3e-3, seed=1, stream=None):
        """Train the learned proposal on the bound system; returns the report as a dict."""
        o = rbmd_train_opts(n_snapshots, steps_between, k_per_snapshot, iterations, learning_rate, seed)
        r = rbmd_train_report()
        _check(library().rbmd_force_train_proposal(self._h, ctypes.byref(o), ctypes.byref(r),
                                                    self._stream(stream)), "train_proposal")
        return {k: getattr(r, k) for k, _ in rbmd_train_report._fields_}

    def proposal_params(self, new=None):
        """Current network parameters (5313 floats); with `new`, replace them first."""
        import numpy as np
        out = np.zeros(5313, dtype=np.float32)
        src = None if new is None else np.ascontiguousarray(new, dtype=np.float32)
        _check(library().rbmd_force_proposal_params(self._h, None if src is not None else _ptr(out, ctypes.c_float),
                                                    None if src is None else _ptr(src, ctypes.c_float)),
               "proposal_params")
        return src if src is not None else out

    def far_force(self):
        """k-space force of the last compute, [n_atoms, 3]."""
        import numpy as np
        out = np.zeros((self.n, 3), dtype=np.float64)
        _check(library().rbmd_force_get_far(self._h, _ptr(out, ctypes.c_double)), "get_far")
        return out

    # ---- diagnostics ----------------------------------------------------------------------
    def neighbors(self, cap):
        import numpy as np
        counts = np.zeros(self.n, dtype=np.int32)
        ids = np.full((self.n, cap), -1, dtype=np.int32)
        st = library().rbmd_force_get_neighbors(self._h, _ptr(counts, ctypes.c_int32),
                                                _ptr(ids, ctypes.c_int32), cap)
        if st not in (RBMD_OK, 1):
            _check(st, "get_neighbors")
        return counts, ids

    def rbl_lists(self):
        """RBL counts per caller atom and the list sizes: (ncore, nshell, sizes) with sizes =
        (rs_num, rc_num, pice_num, core_cap, shell_cap)."""
        import numpy as np
        ncore = np.zeros(self.n, dtype=np.int32)
        nshell = np.zeros(self.n, dtype=np.int32)
        sizes = np.zeros(5, dtype=np.int64)
        _check(library().rbmd_force_get_rbl(self._h, _ptr(ncore, ctypes.c_int32), _ptr(nshell, ctypes.c_int32),
                                            _ptr(sizes, ctypes.c_int64)), "get_rbl")
        return ncore, nshell, tuple(int(v) for v in sizes)

    def energy(self, stream=None):
        e = rbmd_energy()
        _check(library().rbmd_force_energy(self._h, ctypes.byref(e), self._stream(stream)), "energy")
        return {k: getattr(e, k) for k, _ in rbmd_energy._fields_}

    def status(self, clear=False, stream=None):
        f = ctypes.c_uint32()
        _check(library().rbmd_force_status(self._h, ctypes.byref(f), int(clear), self._stream(stream)),
               "status")
        return int(f.value)

    PHASES = ("integrate", "cell_sort", "kspace", "neighbor_list", "force", "molecular", "sampler",
              "rbe_force")

    def profile(self, enable=True):
        _check(library().rbmd_force_profile(self._h, int(enable)), "profile")

    def phase_ms(self):
        import numpy as np
        ms = np.zeros(len(self.PHASES))
        cnt = np.zeros(len(self.PHASES), np.int64)
        _check(library().rbmd_force_phase_ms(self._h, _ptr(ms, ctypes.c_double),
                                             _ptr(cnt, ctypes.c_int64), len(self.PHASES)), "phase_ms")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PHASES)}

    def list_builds(self):
        k = ctypes.c_int64()
        _check(library().rbmd_force_list_builds(self._h, ctypes.byref(k)), "list_builds")
        return int(k.value)

    def launches_per_step(self):
        k = ctypes.c_int32()
        _check(library().rbmd_force_launch_count(self._h, ctypes.byref(k)), "launch_count")
        return int(k.value)

    def close(self):
        if getattr(self, "_h", None):
            library().rbmd_force_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def version() -> str:
    return library().rbmd_version().decode()


# ---- LAMMPS data files ----------------------------------------------------------------------
def read_data(path, atom_style, unit="LJ"):
    """Read a LAMMPS data file as the reference's read_data does (rbmd_data_read); returns a dict
    of numpy arrays (0-based types, molecules and ids) and the box."""
    import numpy as np
    lib = library()
    h = ctypes.c_void_p()
    info = rbmd_data_info()
    _check(lib.rbmd_data_read(str(path).encode(), atom_style.encode(), unit.encode(), ctypes.byref(h),
                              ctypes.byref(info)), "rbmd_data_read")
    try:
        n, nt = info.n_atoms, info.n_atom_types
        out = dict(pos=np.zeros((n, 3)), vel=np.zeros((n, 3)), charge=np.zeros(n), type=np.zeros(n, np.int32),
                   molecule=np.zeros(n, np.int32), mass=np.zeros(n), image=np.zeros((n, 3), np.int32))
        dp = lambda a: a.ctypes.data_as(ctypes.c_void_p)   # noqa: E731
        _check(lib.rbmd_data_atoms(h, dp(out["pos"]), dp(out["vel"]), dp(out["charge"]), dp(out["type"]),
                                   dp(out["molecule"]), dp(out["mass"]), dp(out["image"])), "rbmd_data_atoms")
        out["mass_by_type"] = np.zeros(nt)
        if info.has_pair_coeffs:
            out["eps"], out["sigma"] = np.zeros(nt), np.zeros(nt)
            _check(lib.rbmd_data_types(h, dp(out["mass_by_type"]), dp(out["eps"]), dp(out["sigma"])), "types")
        else:
            _check(lib.rbmd_data_types(h, dp(out["mass_by_type"]), None, None), "types")
        out["bonds"] = np.zeros((info.n_bonds, 2), np.int32)
        out["angles"] = np.zeros((info.n_angles, 3), np.int32)
        out["bond_coeffs"] = np.zeros((max(info.n_bond_types, 0), 2))
        out["angle_coeffs"] = np.zeros((max(info.n_angle_types, 0), 2))
        out["bond_type"] = np.zeros(info.n_bonds, np.int32)
        out["angle_type"] = np.zeros(info.n_angles, np.int32)
        _check(lib.rbmd_data_topology(h, dp(out["bonds"]), dp(out["bond_type"]), dp(out["angles"]),
                                      dp(out["angle_type"]), dp(out["bond_coeffs"]), dp(out["angle_coeffs"])),
               "topology")
        out["dihedrals"] = np.zeros((info.n_dihedrals, 4), np.int32)
        out["dihedral_type"] = np.zeros(info.n_dihedrals, np.int32)
        out["dihedral_coeffs"] = np.zeros((max(info.n_dihedral_types, 0), 3))
        _check(lib.rbmd_data_dihedrals(h, dp(out["dihedrals"]), dp(out["dihedral_type"]),
                                       dp(out["dihedral_coeffs"])), "dihedrals")
        out["lo"] = np.array(info.box.lo[:])
        out["hi"] = np.array(info.box.hi[:])
        out["has_velocities"] = bool(info.has_velocities)
        return out
    finally:
        lib.rbmd_data_free(h)


def write_data(path, atom_style, d):
    """Write arrays in the dict form of read_data as a LAMMPS data file (rbmd_data_write_arrays):
    bonds, angles and dihedrals with their types and coefficients when the dict holds them."""
    import numpy as np
    info = rbmd_data_info()
    n = d["pos"].shape[0]
    info.n_atoms = n
    mt = np.ascontiguousarray(d.get("mass_by_type", np.ones(int(d["type"].max()) + 1)), np.float64)
    info.n_atom_types = len(mt)
    c = lambda a, t: None if a is None else np.ascontiguousarray(a, t)   # noqa: E731
    bonds, angles, dihs = c(d.get("bonds"), np.int32), c(d.get("angles"), np.int32), c(d.get("dihedrals"), np.int32)
    bc, ac, dc = (c(d.get(k), np.float64) for k in ("bond_coeffs", "angle_coeffs", "dihedral_coeffs"))
    info.n_bonds = 0 if bonds is None else len(bonds)
    info.n_angles = 0 if angles is None else len(angles)
    info.n_dihedrals = 0 if dihs is None else len(dihs)
    info.n_bond_types = len(bc) if bc is not None and len(bc) else 1
    info.n_angle_types = len(ac) if ac is not None and len(ac) else 1
    info.n_dihedral_types = len(dc) if dc is not None and len(dc) else 1
    info.box = rbmd_box(tuple(d["lo"]), tuple(d["hi"]))
    keep = dict(pos=c(d["pos"], np.float64), vel=c(d.get("vel"), np.float64), charge=c(d.get("charge"), np.float64),
                type=c(d["type"], np.int32), molecule=c(d.get("molecule"), np.int32), image=c(d.get("image"), np.int32),
                mass_by_type=mt, epsilon=c(d.get("eps"), np.float64), sigma=c(d.get("sigma"), np.float64),
                bonds=bonds if info.n_bonds else None, bond_type=c(d.get("bond_type"), np.int32),
                bond_coeffs=bc if bc is not None and len(bc) else None,
                angles=angles if info.n_angles else None, angle_type=c(d.get("angle_type"), np.int32),
                angle_coeffs=ac if ac is not None and len(ac) else None,
                dihedrals=dihs if info.n_dihedrals else None, dihedral_type=c(d.get("dihedral_type"), np.int32),
                dihedral_coeffs=dc if dc is not None and len(dc) else None)
    arrs = rbmd_data_arrays(**{k: (None if v is None else v.ctypes.data_as(ctypes.c_void_p).value)
                               for k, v in keep.items()})
    _check(library().rbmd_data_write_arrays(str(path).encode(), atom_style.encode(), ctypes.byref(info),
                                            ctypes.byref(arrs)), "rbmd_data_write")
