"""CPU oracle for RBMD's force path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper around ``oracle/liboracle.so`` (built from ``oracle/oracle.cpp`` by
``oracle/build.sh``).  Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` use it, always as the checker or the timed CPU reference, never as the product.

Parity status: the reference (VTK-m 1.9, not vendored) cannot be built here; the oracle is a
restatement of its code (file:line cited in oracle.cpp) pinned by the reference's own data
(funcfl potentials, the ERF table) and by analytic known answers, see tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force=False):
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["sh", os.path.join(_HERE, "build.sh")], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.oracle_rbe_S_f32.restype = ctypes.c_double
        _lib.oracle_rbe_S_f64.restype = ctypes.c_double
        _lib.oracle_ewald_kspace_f64.restype = ctypes.c_double
        _lib.oracle_ewald_real_f64.restype = ctypes.c_double
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


D, F, I32 = ctypes.c_double, ctypes.c_float, ctypes.c_int32


def _real(prec):
    return (np.float32, F, "f32") if prec == "fp32" else (np.float64, D, "f64")


def neighbors(pos, lo, hi, cutoff, prec="fp32", cap=None, rs=None, original=False):
    """Full Verlet list (ComputeNeighboursWorklet semantics; original=True: the pairs the
    "ORIGINAL" neighbour type visits, d^2 < rc^2).  Returns counts, ids, codes."""
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    n = x.shape[0]
    lo = np.ascontiguousarray(lo, dtype=np.float64)
    hi = np.ascontiguousarray(hi, dtype=np.float64)
    rs = cutoff if rs is None else rs
    if cap is None:
        vol = np.prod(hi - lo)
        cap = int(2.0 * n / vol * 4.0 / 3.0 * np.pi * cutoff ** 3) + 64
    while True:
        counts = np.zeros(n, np.int32)
        ids = np.full((n, cap), -1, np.int32)
        codes = np.zeros((n, cap), np.int32)
        dims = np.zeros(3, np.int32)
        rc = getattr(lib(), "oracle_neighbors_" + sfx)(
            ctypes.c_int64(n), _p(x, ct), _p(lo, D), _p(hi, D), D(cutoff), D(rs), ctypes.c_int64(cap),
            _p(counts, I32), _p(ids, I32), _p(codes, I32), _p(dims, I32), int(original))
        if rc == 0:
            return counts, ids, codes
        cap = int(counts.max()) + 8


def near_force(pos, lo, hi, cutoff, nl, *, type=None, mol=None, charge=None, eps=(1.0,), sigma=(1.0,),
               with_lj=True, with_coul=False, alpha=0.0, coul_scale=1.0, sum_mode=1, prec="fp32", special=None):
    """special = (off, ids, w) from special_lists: LJ pairs weighted by their special-bond weight
    instead of the same-molecule exclusion."""
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    n = x.shape[0]
    counts, ids, codes = nl
    cap = ids.shape[1]
    out = np.zeros((n, 3))
    t = None if type is None else np.ascontiguousarray(type, dtype=np.int32)
    m = None if mol is None else np.ascontiguousarray(mol, dtype=np.int32)
    q = None if charge is None else np.ascontiguousarray(charge, dtype=np.float64)
    e = np.ascontiguousarray(eps, dtype=np.float64)
    s = np.ascontiguousarray(sigma, dtype=np.float64)
    if special is not None:
        so, si, sw = special
        getattr(lib(), "oracle_near_sp_" + sfx)(
            ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
            D(cutoff), _p(t, I32), _p(q, D), len(e), _p(e, D), _p(s, D), ctypes.c_int64(cap),
            _p(counts, I32), _p(ids, I32), _p(codes, I32), int(with_coul), D(alpha), D(coul_scale),
            _p(so, ctypes.c_int64), _p(si, I32), _p(sw, D), _p(out, D))
        return out
    getattr(lib(), "oracle_near_" + sfx)(
        ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
        D(cutoff), _p(t, I32), _p(m, I32), _p(q, D), len(e), _p(e, D), _p(s, D), ctypes.c_int64(cap),
        _p(counts, I32), _p(ids, I32), _p(codes, I32), int(with_lj), int(with_coul), D(alpha),
        D(coul_scale), int(sum_mode), _p(out, D))
    return out


def rbe_sample(alpha, L, seed, step, rep, P):
    out = np.zeros((P, 3), np.int32)
    Lb = np.ascontiguousarray(L, dtype=np.float64)
    lib().oracle_rbe_sample(D(alpha), _p(Lb, D), ctypes.c_uint64(seed), ctypes.c_int64(step),
                            int(rep), int(P), _p(out, I32))
    return out


def rbe_sample_trace(alpha, L, seed, step, rep, P):
    """rbe_sample plus the uniforms it used, in the order RBEPSAMPLE consumes them."""
    out = np.zeros((P, 3), np.int32)
    Lb = np.ascontiguousarray(L, dtype=np.float64)
    f = lib().oracle_rbe_sample_trace
    f.restype = ctypes.c_int64
    cap = 16 * P + 64
    while True:
        tr = np.zeros(cap)
        k = f(D(alpha), _p(Lb, D), ctypes.c_uint64(seed), ctypes.c_int64(step), int(rep), int(P), _p(out, I32),
              _p(tr, D), ctypes.c_int64(cap))
        if k <= cap:
            return out, tr[:k]
        cap = int(k)


def rbe_S(alpha, box, prec="fp64"):
    b = np.ascontiguousarray(box, dtype=np.float64)
    return getattr(lib(), "oracle_rbe_S_" + ("f32" if prec == "fp32" else "f64"))(D(alpha), _p(b, D))


def rhok(pos, charge, box, m, origin=(0, 0, 0), prec="fp64"):
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    m = np.ascontiguousarray(m, dtype=np.int32)
    out = np.zeros((m.shape[0], 2))
    getattr(lib(), "oracle_rhok_" + sfx)(
        ctypes.c_int64(x.shape[0]), _p(x, ct), _p(np.ascontiguousarray(charge, np.float64), D),
        _p(np.ascontiguousarray(box, np.float64), D), _p(np.ascontiguousarray(origin, np.float64), D),
        m.shape[0], _p(m, I32), _p(out, D))
    return out


def rbe_force(pos, charge, box, alpha, qqr2e, m, rho, origin=(0, 0, 0), weights=None, S=0.0, prec="fp64"):
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    m = np.ascontiguousarray(m, dtype=np.int32)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    out = np.zeros((x.shape[0], 3))
    getattr(lib(), "oracle_rbe_force_" + sfx)(
        ctypes.c_int64(x.shape[0]), _p(x, ct), _p(np.ascontiguousarray(charge, np.float64), D),
        _p(np.ascontiguousarray(box, np.float64), D), _p(np.ascontiguousarray(origin, np.float64), D),
        D(alpha), D(qqr2e), m.shape[0], _p(m, I32), _p(rho, D), _p(w, D), D(S), _p(out, D))
    return out


def ewald_kspace(pos, charge, box, alpha, kcut, qqr2e=1.0):
    x = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.zeros_like(x)
    e = lib().oracle_ewald_kspace_f64(ctypes.c_int64(x.shape[0]), _p(x, D),
                                      _p(np.ascontiguousarray(charge, np.float64), D),
                                      _p(np.ascontiguousarray(box, np.float64), D), D(alpha), D(kcut),
                                      D(qqr2e), _p(out, D))
    return out, e


def ewald_real(pos, lo, hi, cutoff, charge, alpha, nl, qqr2e=1.0):
    x = np.ascontiguousarray(pos, dtype=np.float64)
    counts, ids, codes = nl
    out = np.zeros_like(x)
    e = lib().oracle_ewald_real_f64(ctypes.c_int64(x.shape[0]), _p(x, D),
                                    _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
                                    D(cutoff), _p(np.ascontiguousarray(charge, np.float64), D), D(alpha),
                                    D(qqr2e), ctypes.c_int64(ids.shape[1]), _p(counts, I32), _p(ids, I32),
                                    _p(codes, I32), _p(out, D))
    return out, e


def eam_tables(path):
    meta = np.zeros(6)
    rc = lib().oracle_eam_tables(str(path).encode(), _p(meta, D), None, None, None, ctypes.c_int64(0))
    if rc:
        raise RuntimeError(f"oracle_eam_tables({path}) -> {rc}")
    nrho, nr = int(meta[0]), int(meta[1])
    rows = max(nrho, nr) + 1
    fr = np.zeros((rows, 7), np.float32)
    rr = np.zeros((rows, 7), np.float32)
    zr = np.zeros((rows, 7), np.float32)
    lib().oracle_eam_tables(str(path).encode(), _p(meta, D), _p(fr, F), _p(rr, F), _p(zr, F),
                            ctypes.c_int64(rows))
    return dict(nrho=nrho, nr=nr, drho=meta[2], dr=meta[3], rhomax=meta[4], cut=meta[5],
                frho=fr[:nrho + 1], rhor=rr[:nrho + 1], z2r=zr[:nr + 1])


def eam_force(path, pos, lo, hi, cutoff, nl, prec="fp32", sum_mode=1, ref_sign=False):
    """EAM forces over a full list.  ref_sign=True uses the reference's Verlet pair vector
    p_j - p_i (reversed forces); the default p_i - p_j is the sign for which F = -grad E."""
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    counts, ids, codes = nl
    n = x.shape[0]
    fp = np.zeros(n)
    out = np.zeros((n, 3))
    rc = getattr(lib(), "oracle_eam_force_" + sfx)(
        str(path).encode(), ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D),
        _p(np.asarray(hi, np.float64), D), D(cutoff), ctypes.c_int64(ids.shape[1]), _p(counts, I32),
        _p(ids, I32), _p(codes, I32), int(sum_mode), _p(fp, D), _p(out, D), int(ref_sign))
    if rc:
        raise RuntimeError(f"oracle eam_force -> {rc}")
    return out, fp


def eam_energy(path, pos, lo, hi, cutoff, nl):
    """FP64 EAM total energy (embedding + pair) over a full list."""
    x = np.ascontiguousarray(pos, dtype=np.float64)
    counts, ids, codes = nl
    f = lib().oracle_eam_energy_f64
    f.restype = ctypes.c_double
    return f(str(path).encode(), ctypes.c_int64(x.shape[0]), _p(x, D), _p(np.asarray(lo, np.float64), D),
             _p(np.asarray(hi, np.float64), D), D(cutoff), ctypes.c_int64(ids.shape[1]), _p(counts, I32),
             _p(ids, I32), _p(codes, I32))


def rbl_sizes(n, lo, hi, rs, rc, sample_num, eam=False, prec="fp32"):
    """(rs_num, rc_num, pice_num) of the reference's RBL list sizing."""
    out = np.zeros(3, np.int64)
    lib().oracle_rbl_sizes(ctypes.c_int64(n), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
                           D(rs), D(rc), D(sample_num), int(eam), int(prec == "fp64"),
                           out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return tuple(int(v) for v in out)


def rbl_list(pos, lo, hi, cutoff, rs, pice, core_cap, shell_cap, prec="fp32"):
    """RBL core list + every pice-th shell pair in the reference's traversal order.
    Returns (ncore, nshell, ids[n, core_cap + shell_cap], codes)."""
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    n = x.shape[0]
    ncore = np.zeros(n, np.int32)
    nshell = np.zeros(n, np.int32)
    ids = np.full((n, core_cap + shell_cap), -1, np.int32)
    codes = np.zeros((n, core_cap + shell_cap), np.int32)
    getattr(lib(), "oracle_rbl_list_" + sfx)(
        ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
        D(cutoff), D(rs), ctypes.c_int64(pice), ctypes.c_int64(core_cap), ctypes.c_int64(shell_cap),
        _p(ncore, I32), _p(nshell, I32), _p(ids, I32), _p(codes, I32))
    return ncore, nshell, ids, codes


def rbl_table_g(dis):
    """G of the reference's ERF table for a float distance (alpha 0.1, one value per bucket)."""
    f = lib().oracle_rbl_table_g
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float]
    return float(f(float(dis)))


def rbl_near(pos, lo, hi, cutoff, rs, pice, rl, core_cap, *, type=None, mol=None, charge=None, eps=(1.0,),
             sigma=(1.0,), with_coul=False, alpha=0.0, qqr2e=1.0, table_mode=0, shell_coul=1,
             remove_mean=True, prec="fp32", special=None, sum_mode=1):
    """sum_mode 1: pair terms summed in FP64; 0 (FP32 only): the reference's float accumulators."""
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    n = x.shape[0]
    ncore, nshell, ids, codes = rl
    shell_cap = ids.shape[1] - core_cap
    out = np.zeros((n, 3))
    t = None if type is None else np.ascontiguousarray(type, dtype=np.int32)
    m = None if mol is None else np.ascontiguousarray(mol, dtype=np.int32)
    q = None if charge is None else np.ascontiguousarray(charge, dtype=np.float64)
    if special is not None:
        so, si, sw = special
        getattr(lib(), "oracle_rbl_near_sp_" + sfx)(
            ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
            D(cutoff), D(rs), ctypes.c_int64(pice), _p(t, I32), _p(q, D),
            _p(np.ascontiguousarray(eps, np.float64), D), _p(np.ascontiguousarray(sigma, np.float64), D),
            ctypes.c_int64(core_cap), ctypes.c_int64(shell_cap), _p(ncore, I32), _p(nshell, I32), _p(ids, I32),
            _p(codes, I32), int(with_coul), D(alpha), D(qqr2e), int(table_mode), int(shell_coul),
            int(remove_mean), _p(so, ctypes.c_int64), _p(si, I32), _p(sw, D), _p(out, D))
        return out
    name = "oracle_rbl_near_ref_f32" if (sum_mode == 0 and sfx == "f32") else "oracle_rbl_near_" + sfx
    getattr(lib(), name)(
        ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
        D(cutoff), D(rs), ctypes.c_int64(pice), _p(t, I32), _p(m, I32), _p(q, D),
        _p(np.ascontiguousarray(eps, np.float64), D), _p(np.ascontiguousarray(sigma, np.float64), D),
        ctypes.c_int64(core_cap), ctypes.c_int64(shell_cap), _p(ncore, I32), _p(nshell, I32), _p(ids, I32),
        _p(codes, I32), int(with_coul), D(alpha), D(qqr2e), int(table_mode), int(shell_coul), int(remove_mean),
        _p(out, D))
    return out


def rbl_eam(path, pos, lo, hi, cutoff, rs, pice, rl, core_cap, remove_mean=True, prec="fp32"):
    dt, ct, sfx = _real(prec)
    x = np.ascontiguousarray(pos, dtype=dt)
    n = x.shape[0]
    ncore, nshell, ids, codes = rl
    fp = np.zeros(n)
    out = np.zeros((n, 3))
    rc = getattr(lib(), "oracle_rbl_eam_" + sfx)(
        str(path).encode(), ctypes.c_int64(n), _p(x, ct), _p(np.asarray(lo, np.float64), D),
        _p(np.asarray(hi, np.float64), D), D(cutoff), D(rs), ctypes.c_int64(pice), ctypes.c_int64(core_cap),
        ctypes.c_int64(ids.shape[1] - core_cap), _p(ncore, I32), _p(nshell, I32), _p(ids, I32), _p(codes, I32),
        int(remove_mean), _p(fp, D), _p(out, D))
    if rc:
        raise RuntimeError(f"oracle rbl_eam -> {rc}")
    return out, fp


def shake(hoh, pos_old, vel_old, force, mass, lo, hi, dt, fmt2v, tol=1e-5, max_iter=5000, image=None):
    """Returns (pos, vel, image, nonconverged, iterations) after SHAKE (positions) from old state."""
    h = np.ascontiguousarray(hoh, np.int32).reshape(-1)
    x = np.array(pos_old, dtype=np.float64, copy=True)
    v = np.array(vel_old, dtype=np.float64, copy=True)
    img = None if image is None else np.array(image, dtype=np.int32, copy=True)
    it = np.zeros(len(h) // 3, np.int32)
    bad = lib().oracle_shake_f64(ctypes.c_int64(len(h) // 3), _p(h, I32), _p(x, D), _p(v, D),
                                 _p(np.ascontiguousarray(force, np.float64), D),
                                 _p(np.ascontiguousarray(mass, np.float64), D), _p(img, I32),
                                 _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
                                 D(dt), D(fmt2v), D(tol), int(max_iter), _p(it, I32))
    return x, v, img, bad, it


def rattle(hoh, pos, vel_old, force, mass, lo, hi, dt, fmt2v):
    h = np.ascontiguousarray(hoh, np.int32).reshape(-1)
    v = np.array(vel_old, dtype=np.float64, copy=True)
    lib().oracle_rattle_f64(ctypes.c_int64(len(h) // 3), _p(h, I32), _p(np.ascontiguousarray(pos, np.float64), D),
                            _p(v, D), _p(np.ascontiguousarray(force, np.float64), D),
                            _p(np.ascontiguousarray(mass, np.float64), D),
                            _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D), D(dt), D(fmt2v))
    return v


def water_extras(hoh, pos, charge, lo, hi, bond_k, bond_r0, angle_k, angle_t0):
    h = np.ascontiguousarray(hoh, np.int32).reshape(-1)
    out = np.zeros((np.asarray(pos).shape[0], 3))
    e = np.zeros(2)
    lib().oracle_water_extras_f64(ctypes.c_int64(len(h) // 3), _p(h, I32),
                                  _p(np.ascontiguousarray(pos, np.float64), D),
                                  _p(np.ascontiguousarray(charge, np.float64), D),
                                  _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
                                  D(bond_k), D(bond_r0), D(angle_k), D(angle_t0), _p(out, D), _p(e, D))
    return out, e


def special_lists(n, bonds, weights):
    """Per-atom special-bond lists (off[n+1], ids, w) as ModelFileInitCondition::SetSpecialBonds
    builds them, duplicates included."""
    b = np.ascontiguousarray(bonds, np.int32).reshape(-1)
    w3 = np.ascontiguousarray(weights, np.float64)
    off = np.zeros(n + 1, np.int64)
    cap = 0
    while True:
        ids = np.zeros(max(cap, 1), np.int32)
        w = np.zeros(max(cap, 1))
        m = lib().oracle_special_lists
        m.restype = ctypes.c_int64
        tot = m(ctypes.c_int64(n), ctypes.c_int64(len(b) // 2), _p(b, I32), _p(w3, D), ctypes.c_int64(cap),
                _p(off, ctypes.c_int64), _p(ids, I32), _p(w, D))
        if tot <= cap:
            return off, ids[:tot], w[:tot]
        cap = int(tot)


def cvff_terms(pos, lo, hi, charge, mol, bonds, bond_type, bond_coeffs, angles, angle_type, angle_coeffs,
               dihedrals=None, dihedral_type=None, dihedral_coeffs=None, special=None):
    """FP64 CVFF intramolecular forces (special Coulomb, bonds, angles, dihedrals with special
    lists) and energies {bond, angle, dihedral, special Coulomb}."""
    x = np.ascontiguousarray(pos, np.float64)
    n = x.shape[0]
    out = np.zeros((n, 3))
    e = np.zeros(4)
    c = lambda a, t: None if a is None else np.ascontiguousarray(a, t)   # noqa: E731
    b, bt, bc = c(bonds, np.int32), c(bond_type, np.int32), c(bond_coeffs, np.float64)
    a, at, ac = c(angles, np.int32), c(angle_type, np.int32), c(angle_coeffs, np.float64)
    d, dt_, dc = c(dihedrals, np.int32), c(dihedral_type, np.int32), c(dihedral_coeffs, np.float64)
    so, si, sw = special if special is not None else (None, None, None)
    lib().oracle_cvff_terms_f64(
        ctypes.c_int64(n), _p(x, D), _p(np.asarray(lo, np.float64), D), _p(np.asarray(hi, np.float64), D),
        _p(np.ascontiguousarray(charge, np.float64), D), _p(np.ascontiguousarray(mol, np.int32), I32),
        ctypes.c_int64(0 if b is None else len(b)), _p(b, I32), _p(bt, I32), _p(bc, D),
        ctypes.c_int64(0 if a is None else len(a)), _p(a, I32), _p(at, I32), _p(ac, D),
        ctypes.c_int64(0 if d is None else len(d)), _p(d, I32), _p(dt_, I32), _p(dc, D),
        _p(so, ctypes.c_int64), _p(si, I32), _p(sw, D), _p(out, D), _p(e, D))
    return out, dict(bond=e[0], angle=e[1], dihedral=e[2], coul_special=e[3])


def set_threads(n):
    lib().oracle_set_threads(int(n))


def num_threads():
    return lib().oracle_num_threads()
