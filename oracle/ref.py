"""ctypes access to oracle/_ref/libref.so: RBMD's own force-path code compiled from the reference
tree (oracle/build_ref.sh, oracle/ref_harness.cpp, VTK-m stand-in in oracle/ref_shim).

Test infrastructure only: it pins the oracle's restatement to the reference's code.  All
arithmetic is the reference's FP32 (Real = float).  available() is False where the library was
not built (no reference tree on this machine); build() needs the tree.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref.so")
_lib = None

F = ctypes.POINTER(ctypes.c_float)
D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)


def _sources():
    out = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "build_ref.sh")]
    for root, _, files in os.walk(os.path.join(HERE, "ref_shim")):
        out += [os.path.join(root, f) for f in files]
    return out


def build(reference=None, force=False):
    """Compile the reference's code (again when the harness or the stand-in changed); returns
    False when no reference tree is present and nothing is built."""
    ref = reference or os.environ.get("RBMD_REFERENCE", "/root/reference")
    present = os.path.exists(os.path.join(ref, "rbmd", "framework", "run", "worklet", "RunWorklet.cpp"))
    if os.path.exists(LIB) and not force:
        t = os.path.getmtime(LIB)
        if not present or all(os.path.getmtime(f) <= t for f in _sources()):
            return True
    if not present:
        return False
    subprocess.run([os.path.join(HERE, "build_ref.sh"), ref], check=True)
    return True


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libref.so is not built (oracle/build_ref.sh needs the reference tree)")
        _lib = ctypes.CDLL(LIB)
        _lib.ref_rbe_force.restype = ctypes.c_double
        _lib.ref_rbe_sample.restype = ctypes.c_int64
        _lib.ref_neighbors.restype = ctypes.c_int32
        _lib.ref_rbl_list.restype = ctypes.c_int32
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def grid(lo, hi, cutoff, rs=None):
    dims = np.zeros(3, np.int32)
    nc = np.zeros(1, np.int32)
    lib().ref_grid(_p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                   ctypes.c_double(cutoff if rs is None else rs), _p(dims, I32), _p(nc, I32))
    return dims, int(nc[0])


def cells(pos, lo, hi, cutoff, rs=None):
    x = _f32(pos)
    dims, _ = grid(lo, hi, cutoff, rs)
    ncell = int(np.prod(dims))
    pid = np.zeros(x.shape[0], np.int32)
    lower = np.zeros(ncell, np.int32)
    upper = np.zeros(ncell, np.int32)
    lib().ref_cells(ctypes.c_int64(x.shape[0]), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                    ctypes.c_double(cutoff if rs is None else rs), _p(pid, I32), _p(lower, I32), _p(upper, I32))
    return pid, lower, upper


def neighbors(pos, lo, hi, cutoff, cap=None, rs=None):
    """ComputeNeighboursWorklet over every atom: (counts, ids, offsets[n, cap, 3])."""
    x = _f32(pos)
    n = x.shape[0]
    if cap is None:
        cap = int(2.0 * n / np.prod(np.asarray(hi) - np.asarray(lo)) * 4.0 / 3.0 * np.pi * cutoff ** 3) + 64
    while True:
        counts = np.zeros(n, np.int32)
        ids = np.full((n, cap), -1, np.int32)
        off = np.zeros((n, cap, 3), np.float32)
        mx = lib().ref_neighbors(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D),
                                 ctypes.c_double(cutoff), ctypes.c_double(cutoff if rs is None else rs),
                                 ctypes.c_int64(cap), _p(counts, I32), _p(ids, I32), _p(off, F))
        if mx <= cap:
            return counts, ids, off
        cap = int(mx) + 8


def near_force(pos, lo, hi, cutoff, nl, *, type=None, mol=None, charge=None, eps=(1.0,), sigma=(1.0,),
               alpha=0.0, with_coul=False):
    """ComputeNearForceVerletWorklet (with_coul) or ComputeLJForceVerletWorklet over nl
    (from neighbors()); float32 forces.  mol None: every atom its own molecule."""
    x = _f32(pos)
    n = x.shape[0]
    counts, ids, off = nl
    t = _i32(np.zeros(n) if type is None else type)
    m = _i32(np.arange(n) if mol is None else mol)
    q = _f32(np.zeros(n) if charge is None else charge)
    e, s = _f32(eps), _f32(sigma)
    out = np.zeros((n, 3), np.float32)
    lib().ref_near_force(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                         _p(t, I32), _p(m, I32), _p(q, F), len(e), _p(e, F), _p(s, F), ctypes.c_double(alpha),
                         int(with_coul), ctypes.c_int64(ids.shape[1]), _p(_i32(counts), I32), _p(_i32(ids), I32),
                         _p(_f32(off), F), _p(out, F))
    return out


def rhok(pos, charge, box, m):
    """Structure-factor terms of ComputePnumberChargeStructureFactorWorklet, summed per k in FP64."""
    x = _f32(pos)
    mm = _i32(m)
    out = np.zeros((mm.shape[0], 2))
    lib().ref_rhok(ctypes.c_int64(x.shape[0]), _p(x, F), _p(_f32(charge), F), _p(_f64(box), D), mm.shape[0],
                   _p(mm, I32), _p(out, D))
    return out


def rbe_force(pos, charge, lo, hi, alpha, m, rho):
    """ComputeNewRBEForceWorklet (before the qqr2e rescale) with rho as float; returns (force, S)."""
    x = _f32(pos)
    mm = _i32(m)
    out = np.zeros((x.shape[0], 3), np.float32)
    S = lib().ref_rbe_force(ctypes.c_int64(x.shape[0]), _p(x, F), _p(_f32(charge), F), _p(_f64(lo), D),
                            _p(_f64(hi), D), ctypes.c_double(alpha), mm.shape[0], _p(mm, I32), _p(_f32(rho), F),
                            _p(out, F))
    return out, S


def eam(tables, pos, lo, hi, cutoff, nl):
    """ComputeEAMfpVerletWorklet + ComputeEAMForceVerletWorklet with the given spline tables
    (dict as oracle.eam_tables returns); returns (force, fp) in float32."""
    x = _f32(pos)
    n = x.shape[0]
    counts, ids, off = nl
    fp = np.zeros(n, np.float32)
    out = np.zeros((n, 3), np.float32)
    fr, rr, zr = _f32(tables["frho"]), _f32(tables["rhor"]), _f32(tables["z2r"])
    lib().ref_eam(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                  int(tables["nrho"]), ctypes.c_double(tables["drho"]), int(tables["nr"]), ctypes.c_double(tables["dr"]),
                  ctypes.c_double(tables["rhomax"]), _p(fr, F), ctypes.c_int64(fr.shape[0]), _p(rr, F),
                  ctypes.c_int64(rr.shape[0]), _p(zr, F), ctypes.c_int64(zr.shape[0]), ctypes.c_int64(ids.shape[1]),
                  _p(_i32(counts), I32), _p(_i32(ids), I32), _p(_f32(off), F), _p(fp, F), _p(out, F))
    return out, fp


def rbe_sample(alpha, L, P, uniforms=None):
    """RBEPSAMPLE::Fetch_P_Sample on an injected uniform stream (None: the reference's TEST mode,
    U = 0.5 throughout).  Returns (m[P, 3] as int32, number of uniforms consumed)."""
    u = None if uniforms is None else _f64(uniforms)
    out = np.zeros((P, 3), np.float32)
    used = lib().ref_rbe_sample(ctypes.c_double(alpha), _p(_f64(L), D), int(P), int(u is not None), _p(u, D),
                                ctypes.c_int64(0 if u is None else u.shape[0]), _p(out, F))
    return out.astype(np.int32), int(used)


def gnear(alpha, dis):
    d = _f32(dis)
    out = np.zeros_like(d)
    lib().ref_gnear(ctypes.c_int64(d.shape[0]), ctypes.c_double(alpha), _p(d, F), _p(out, F))
    return out


def rbl_list(pos, lo, hi, cutoff, rs, rs_num, pice, cap=None):
    """ComputeRBLNeighboursOnceWorklet: (ncore, nshell, ids[n, cap], offsets[n, cap, 3]) with the
    core pairs at [0, ncore) and the kept shell pairs at [rs_num, rs_num + nshell)."""
    x = _f32(pos)
    n = x.shape[0]
    cap = cap or rs_num + 64
    while True:
        ncore = np.zeros(n, np.int32)
        nshell = np.zeros(n, np.int32)
        ids = np.full((n, cap), -1, np.int32)
        off = np.zeros((n, cap, 3), np.float32)
        mx = lib().ref_rbl_list(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D),
                                ctypes.c_double(cutoff), ctypes.c_double(rs), int(rs_num), int(pice),
                                ctypes.c_int64(cap), _p(ncore, I32), _p(nshell, I32), _p(ids, I32), _p(off, F))
        if mx <= cap:
            return ncore, nshell, ids, off
        cap = int(mx) + 8


def rbl_near(pos, lo, hi, cutoff, rs, rs_num, pice, rl, *, type=None, mol=None, charge=None, eps=(1.0,),
             sigma=(1.0,), alpha=0.0, qqr2e=1.0, with_coul=False):
    """ComputeNearForceRBLERFWorklet (with_coul) or ComputeLJForceRBLWorklet over rl (from
    rbl_list), before the mean removal; float32 forces."""
    x = _f32(pos)
    n = x.shape[0]
    ncore, nshell, ids, off = rl
    t = _i32(np.zeros(n) if type is None else type)
    m = _i32(np.arange(n) if mol is None else mol)
    q = _f32(np.zeros(n) if charge is None else charge)
    e, s = _f32(eps), _f32(sigma)
    out = np.zeros((n, 3), np.float32)
    lib().ref_rbl_near(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                       ctypes.c_double(rs), int(rs_num), int(pice), ctypes.c_double(qqr2e), _p(t, I32), _p(m, I32),
                       _p(q, F), len(e), _p(e, F), _p(s, F), ctypes.c_double(alpha), int(with_coul),
                       ctypes.c_int64(ids.shape[1]), _p(_i32(ncore), I32), _p(_i32(nshell), I32), _p(_i32(ids), I32),
                       _p(_f32(off), F), _p(out, F))
    return out


def erf_table(dis):
    """G from the reference's RBL Coulomb table (ExecStaticTable over model/ERFTable.h)."""
    d = _f32(dis)
    out = np.zeros_like(d)
    lib().ref_erf_table(ctypes.c_int64(d.shape[0]), _p(d, F), _p(out, F))
    return out


def eam_original(tables, pos, lo, hi, cutoff):
    """The ORIGINAL neighbour type's EAM worklets (cells walked on the fly); (force, fp) float32."""
    x = _f32(pos)
    n = x.shape[0]
    fp = np.zeros(n, np.float32)
    out = np.zeros((n, 3), np.float32)
    fr, rr, zr = _f32(tables["frho"]), _f32(tables["rhor"]), _f32(tables["z2r"])
    lib().ref_eam_original(ctypes.c_int64(n), _p(x, F), _p(_f64(lo), D), _p(_f64(hi), D), ctypes.c_double(cutoff),
                           int(tables["nrho"]), ctypes.c_double(tables["drho"]), int(tables["nr"]),
                           ctypes.c_double(tables["dr"]), ctypes.c_double(tables["rhomax"]), _p(fr, F),
                           ctypes.c_int64(fr.shape[0]), _p(rr, F), ctypes.c_int64(rr.shape[0]), _p(zr, F),
                           ctypes.c_int64(zr.shape[0]), _p(fp, F), _p(out, F))
    return out, fp
