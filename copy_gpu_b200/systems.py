"""Seeded synthetic systems in the shapes of the benchmark configurations.

No dataset or checkpoint is used: every system is generated from a seed.  Each generator returns
a dict of numpy arrays (positions FP64 [N,3], velocities, masses, charges, types, molecule ids,
box lo/hi) plus the RBMD JSON configuration that selects the matching force path.

* ``lj_fcc``        -- FCC Lennard-Jones fluid start (4000 atoms at rho*=0.8442, T*=0.72).
* ``electrolyte``   -- primitive-model 1:1 electrolyte: +/-1 ions plus neutral LJ solvent (10 %
                       ions), rho=0.8 sigma^-3, Bjerrum length 1 (qqr2e = 1 at T = 1).
* ``replicas``      -- many electrolyte replicas with uniform-random atom counts.
* ``water``         -- rigid 3-site water (SPC/E charges) at 1.0 g/cm^3, random orientations.
* ``eam_fcc``       -- FCC metal with Gaussian thermal displacements, plus ``write_johnson_funcfl``
                       which tabulates Johnson's analytic EAM as a funcfl file.
* ``molecular``     -- flexible chain molecules with bonds, angles and dihedrals of several types
                       plus free ions, REAL units (the shape of a polymer electrolyte input).
"""
from __future__ import annotations

import json
import math

import numpy as np


def _maxwell(rng, n, T, mass, kB=1.0, mvv2e=1.0):
    v = rng.normal(size=(n, 3)) * np.sqrt(kB * T / (mass[:, None] * mvv2e))
    p = (v * mass[:, None]).sum(0) / mass.sum()
    return v - p


def _lattice_points(n, L, rng, jitter=0.0):
    """n points on the smallest simple-cubic lattice holding them, random subset, small jitter."""
    m = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    while m ** 3 < n:
        m += 1
    a = L / m
    idx = rng.permutation(m ** 3)[:n]
    ijk = np.stack(np.unravel_index(idx, (m, m, m)), axis=1).astype(np.float64)
    x = (ijk + 0.5) * a + rng.uniform(-jitter, jitter, size=(n, 3)) * a
    return np.mod(x, L)


def lj_config(cutoff=2.5, skin=0.0, dt=0.005, T=0.72, ensemble="NVE", precision="fp64"):
    return {
        "init_configuration": {"read_data": {"unit": "LJ", "atom_style": "atomic", "velocity_type": "GAUSS"}},
        "hyper_parameters": {
            "force_field": {"type": "LJ/CUT"},
            "neighbor": {"type": "VERLETLIST", "cut_off": cutoff, "skin": skin},
        },
        "execution": {"ensemble": ensemble, "temperature": [T, T, 1.0], "temp_ctrl_type": "BERENDSEN",
                      "timestep": dt, "num_steps": 1000},
        "precision": precision,
    }


def lj_fcc(ncell=10, rho=0.8442, T=0.72, seed=1):
    """FCC lattice of 4*ncell^3 atoms at reduced density rho, Maxwell velocities at T."""
    rng = np.random.default_rng(seed)
    a = (4.0 / rho) ** (1.0 / 3.0)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + basis[None]) * a).reshape(-1, 3).astype(np.float64)
    L = a * ncell
    n = pos.shape[0]
    mass = np.ones(n)
    return dict(pos=pos, vel=_maxwell(rng, n, T, mass), mass=mass, charge=np.zeros(n),
                type=np.zeros(n, np.int32), molecule=None, lo=np.zeros(3), hi=np.full(3, L),
                eps=np.array([1.0]), sigma=np.array([1.0]))


def electrolyte_alpha(cutoff=2.5, tol=1e-5):
    """Smallest Gaussian exponent alpha with erfc(sqrt(alpha) * rc) <= tol (bisection)."""
    lo, hi = 0.0, 50.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.erfc(math.sqrt(mid) * cutoff) <= tol:
            hi = mid
        else:
            lo = mid
    return hi


def electrolyte_config(P=500, cutoff=2.5, alpha=None, dt=0.005, T=1.0, precision="fp32",
                       seed=7, coulomb="RBE", kmax=2, ensemble="NVT"):
    if alpha is None:
        alpha = electrolyte_alpha(cutoff)
    return {
        "init_configuration": {"read_data": {"unit": "LJ", "atom_style": "charge", "velocity_type": "GAUSS"}},
        "hyper_parameters": {
            "force_field": {"type": "LJ/CUT/COUL/LONG"},
            "neighbor": {"type": "VERLETLIST", "cut_off": cutoff},
            "coulomb": {"type": coulomb, "coulomb_sample_num": P, "alpha": alpha, "kmax": kmax, "seed": seed},
        },
        "execution": {"ensemble": ensemble, "temperature": [T, T, 0.5], "temp_ctrl_type": "BERENDSEN",
                      "timestep": dt, "num_steps": 1000},
        "precision": precision,
    }


def electrolyte(n, rho=0.8, ion_frac=0.1, T=1.0, seed=3, jitter=0.1):
    """Primitive-model 1:1 electrolyte: n atoms in a cubic box at density rho."""
    rng = np.random.default_rng(seed)
    L = (n / rho) ** (1.0 / 3.0)
    pos = _lattice_points(n, L, rng, jitter)
    nion = int(round(ion_frac * n))
    nion -= nion % 2
    charge = np.zeros(n)
    typ = np.zeros(n, np.int32)
    ions = rng.permutation(n)[:nion]
    charge[ions[: nion // 2]] = 1.0
    charge[ions[nion // 2:]] = -1.0
    typ[ions[: nion // 2]] = 1
    typ[ions[nion // 2:]] = 2
    mass = np.ones(n)
    return dict(pos=pos, vel=_maxwell(rng, n, T, mass), mass=mass, charge=charge, type=typ,
                molecule=None, lo=np.zeros(3), hi=np.full(3, L), eps=np.ones(3), sigma=np.ones(3))


def replicas(n_rep=512, nmin=500, nmax=8000, rho=0.8, ion_frac=0.1, T=1.0, seed=11):
    """Independent electrolyte replicas with atom counts uniform in [nmin, nmax]."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(nmin, nmax + 1, size=n_rep)
    parts = [electrolyte(int(c), rho, ion_frac, T, seed=seed * 1000 + r) for r, c in enumerate(counts)]
    off = np.zeros(n_rep + 1, np.int64)
    off[1:] = np.cumsum(counts)
    cat = lambda k: np.concatenate([p[k] for p in parts])
    return dict(pos=cat("pos"), vel=cat("vel"), mass=cat("mass"), charge=cat("charge"),
                type=cat("type"), molecule=None, offsets=off,
                lo=np.stack([p["lo"] for p in parts]), hi=np.stack([p["hi"] for p in parts]),
                eps=np.ones(3), sigma=np.ones(3))


# ------------------------------------------------------------------------------------------
# water
# ------------------------------------------------------------------------------------------
WATER_MASS = (15.9994, 1.008)
SPCE_CHARGE = (-0.8476, 0.4238)


def water_config(P=200, cutoff=10.0, alpha=0.09, dt=2.0, T=298.0, shake_tol=1e-6, precision="fp32",
                 seed=5, compat_no_qqr2e=False):
    """CVFF water: LJ (O-O only) + erfc near Coulomb + RBE, SHAKE, REAL units.  alpha is the
    Gaussian exponent of erfc(sqrt(alpha) r): an Ewald splitting beta = 0.3 A^-1 is alpha = 0.09."""
    return {
        "init_configuration": {"read_data": {"unit": "REAL", "atom_style": "full", "velocity_type": "GAUSS"}},
        "hyper_parameters": {
            "force_field": {"type": "CVFF"},
            "neighbor": {"type": "VERLETLIST", "cut_off": cutoff},
            "coulomb": {"type": "RBE", "coulomb_sample_num": P, "alpha": alpha, "kmax": 2, "seed": seed},
            "extend": {"fix_shake": "true", "special_bonds": [0, 0, 0], "shake_tolerance": shake_tol},
        },
        "execution": {"ensemble": "NVT", "temperature": [T, T, 100.0], "temp_ctrl_type": "BERENDSEN",
                      "timestep": dt, "num_steps": 1000},
        "compat": {"verlet_coul_no_qqr2e": bool(compat_no_qqr2e)},
        "precision": precision,
    }


def water(n_mol=10000, density=1.0, T=298.0, seed=9):
    """Rigid 3-site water molecules on a cubic lattice with random orientations.
    Atom order per molecule: H, O, H (the reference's angle-triple order)."""
    rng = np.random.default_rng(seed)
    vol_per_mol = 18.0154 / (6.02214076e23 * density) * 1e24   # A^3
    L = (n_mol * vol_per_mol) ** (1.0 / 3.0)
    O = _lattice_points(n_mol, L, rng, 0.05)
    th = math.radians(109.47) / 2.0
    loc = np.array([[math.sin(th), math.cos(th), 0.0], [0.0, 0.0, 0.0], [-math.sin(th), math.cos(th), 0.0]])
    q = rng.normal(size=(n_mol, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    pos = O[:, None, :] + np.einsum("mij,aj->mai", R, loc)
    pos = np.mod(pos.reshape(-1, 3), L)
    n = 3 * n_mol
    typ = np.tile(np.array([1, 0, 1], np.int32), n_mol)          # 0 = O, 1 = H
    charge = np.tile(np.array([SPCE_CHARGE[1], SPCE_CHARGE[0], SPCE_CHARGE[1]]), n_mol)
    mass = np.where(typ == 0, WATER_MASS[0], WATER_MASS[1]).astype(np.float64)
    mol = np.repeat(np.arange(n_mol, dtype=np.int32), 3)
    kB, mvv2e = 1.9872067e-3, 1.0 / 4.186e-4
    vel = _maxwell(rng, n, T, mass, kB, mvv2e)
    # rigid molecules: remove the relative motion along the bonds by giving each molecule its
    # centre-of-mass velocity only
    vm = (vel.reshape(n_mol, 3, 3) * mass.reshape(n_mol, 3, 1)).sum(1) / mass.reshape(n_mol, 3).sum(1, keepdims=True)
    vel = np.repeat(vm, 3, axis=0)
    hoh = np.arange(n, dtype=np.int32).reshape(n_mol, 3)
    return dict(pos=pos, vel=vel, mass=mass, charge=charge, type=typ, molecule=mol,
                lo=np.zeros(3), hi=np.full(3, L), hoh=hoh,
                eps=np.array([0.1553, 0.0]), sigma=np.array([3.166, 0.0]),
                bond=(450.0, 1.0), angle=(55.0, 109.47))


# ------------------------------------------------------------------------------------------
# EAM
# ------------------------------------------------------------------------------------------
# phi_e solves dE/da = 0 at a = 3.615 A for the three FCC neighbour shells inside the 5.0 A
# cutoff (E per atom = F(rho) + 1/2 sum phi; stable: d2E/da2 = 4.2 eV/A^2, E = -2.29 eV per atom),
# so the benchmark crystal starts at the potential's equilibrium lattice constant.
JOHNSON_CU = dict(re=2.556, fe=1.0, rho_e=12.0, phi_e=0.2235, Ec=3.54, beta=5.85, gamma=8.0,
                  cutoff=5.0, npts=5000, rho_max=30.0, mass=63.546, a=3.615)


def write_johnson_funcfl(path, p=JOHNSON_CU):
    """Tabulate Johnson's analytic EAM as a funcfl file (LAMMPS layout, which RBMD reads):
    f(r) = fe exp(-beta (r/re - 1)), phi(r) = phi_e exp(-gamma (r/re - 1)),
    F(rho) = -Ec sqrt(rho / rho_e); Z(r) = sqrt(r phi(r) / (27.2 * 0.529)).
    nrho = nr = npts (the reference reads rho(r) with the nrho count)."""
    n = int(p["npts"])
    dr = p["cutoff"] / n
    drho = p["rho_max"] / n
    r = np.arange(n) * dr
    rho = np.arange(n) * drho
    F = -p["Ec"] * np.sqrt(rho / p["rho_e"])
    phi = p["phi_e"] * np.exp(-p["gamma"] * (r / p["re"] - 1.0))
    Z = np.sqrt(np.maximum(r * phi, 0.0) / (27.2 * 0.529))
    f = p["fe"] * np.exp(-p["beta"] * (r / p["re"] - 1.0))
    with open(path, "w") as fh:
        fh.write("Johnson analytic EAM (Cu-like), generated\n")
        fh.write(f"29 {p['mass']:.3f} {p['a']:.4f} FCC\n")
        fh.write(f"{n} {drho:.16e} {n} {dr:.16e} {p['cutoff']:.6f}\n")
        for arr in (F, Z, f):
            for k in range(0, n, 5):
                fh.write(" ".join(f"{v:.16e}" for v in arr[k:k + 5]) + "\n")
    return path


def johnson_terms(r, p=JOHNSON_CU):
    """Johnson's f(r), phi(r) and their derivatives (analytic, for checks)."""
    f = p["fe"] * np.exp(-p["beta"] * (r / p["re"] - 1.0))
    phi = p["phi_e"] * np.exp(-p["gamma"] * (r / p["re"] - 1.0))
    return f, -p["beta"] / p["re"] * f, phi, -p["gamma"] / p["re"] * phi


def write_johnson_setfl(path, p=JOHNSON_CU):
    """The same Johnson EAM as a single-element setfl (eam/alloy) file: F(rho) and rho(r) on the
    file grids, then r * phi(r)."""
    n = int(p["npts"])
    dr = p["cutoff"] / n
    drho = p["rho_max"] / n
    r = np.arange(n) * dr
    rho = np.arange(n) * drho
    F = -p["Ec"] * np.sqrt(rho / p["rho_e"])
    f, _, phi, _ = johnson_terms(r, p)
    with open(path, "w") as fh:
        fh.write("Johnson analytic EAM (Cu-like), generated\n\n\n")
        fh.write("1 Cu\n")
        fh.write(f"{n} {drho:.16e} {n} {dr:.16e} {p['cutoff']:.6f}\n")
        fh.write(f"29 {p['mass']:.3f} {p['a']:.4f} fcc\n")
        for arr in (F, f, r * phi):
            for k in range(0, n, 5):
                fh.write(" ".join(f"{v:.16e}" for v in arr[k:k + 5]) + "\n")
    return path


def eam_config(potential_file, cutoff=5.0, dt=1.0, precision="fp32"):
    return {
        "init_configuration": {"read_data": {"unit": "METAL", "atom_style": "atomic", "velocity_type": "GAUSS"}},
        "hyper_parameters": {
            "force_field": {"type": "EAM", "potential_file": str(potential_file)},
            "neighbor": {"type": "VERLETLIST", "cut_off": cutoff},
        },
        "execution": {"ensemble": "NVE", "temperature": [300.0, 300.0, 100.0], "temp_ctrl_type": "",
                      "timestep": dt / 1000.0, "num_steps": 1000},
        "precision": precision,
    }


def eam_fcc(ncell=40, a=3.615, T=300.0, k_eff=1.5, mass=63.546, seed=13):
    """FCC crystal with Gaussian displacements of variance kT/k_eff per axis (k_eff in eV/A^2)."""
    rng = np.random.default_rng(seed)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + basis[None]) * a).reshape(-1, 3).astype(np.float64)
    kT = 8.617343e-5 * T
    pos += rng.normal(scale=math.sqrt(kT / k_eff), size=pos.shape)
    L = a * ncell
    pos = np.mod(pos, L)
    n = pos.shape[0]
    m = np.full(n, mass)
    vel = _maxwell(rng, n, T, m, kB=8.617343e-5, mvv2e=1.0364269e-4)
    return dict(pos=pos, vel=vel, mass=m, charge=np.zeros(n), type=np.zeros(n, np.int32),
                molecule=None, lo=np.zeros(3), hi=np.full(3, L), eps=np.ones(1), sigma=np.ones(1))


# ------------------------------------------------------------------------------------------
# flexible molecules
# ------------------------------------------------------------------------------------------
def molecular_config(P=100, cutoff=8.0, alpha=0.09, neighbor="VERLETLIST", special=(0.0, 0.0, 0.5), dt=0.5,
                     T=298.0, precision="fp64", seed=5, r_core=4.0, sample_num=100):
    """CVFF with a full topology: LJ + erfc near Coulomb + RBE, special-bond weights, REAL units.
    special=None leaves out extend.special_bonds (same-molecule LJ exclusion, no dihedrals)."""
    nb = {"type": neighbor, "cut_off": cutoff}
    if neighbor == "RBL":
        nb.update({"r_core": r_core, "neighbor_sample_num": sample_num})
    cfg = {
        "init_configuration": {"read_data": {"unit": "REAL", "atom_style": "full", "velocity_type": "GAUSS"}},
        "hyper_parameters": {
            "force_field": {"type": "CVFF"},
            "neighbor": nb,
            "coulomb": {"type": "RBE", "coulomb_sample_num": P, "alpha": alpha, "kmax": 2, "seed": seed},
        },
        "execution": {"ensemble": "NVE", "temperature": [T, T, 100.0], "timestep": dt, "num_steps": 1000},
        "precision": precision,
    }
    if special is not None:
        cfg["hyper_parameters"]["extend"] = {"special_bonds": list(special)}
    return cfg


def molecular(n_chain=64, chain_len=12, n_ion_pairs=16, step=1.6, cell=8.0, T=298.0, seed=21):
    """Chains grown as self-avoiding walks (step `step`, 90 or 180 degree turns, no U-turns, small jitter),
    one chain per cell of a cubic lattice of spacing `cell`, plus +/-1 ion pairs in free cells.
    Backbone types alternate 0/1 (charges +0.2/-0.2, one end group type 2 carries the rest so
    every chain is neutral); ions are types 3 (+1) and 4 (-1), each its own molecule.  Bonds,
    angles and dihedrals follow the chain; their types depend on the end atom types, so several
    coefficient rows are used.  Returns arrays plus per-type coefficient tables."""
    rng = np.random.default_rng(seed)
    n_sites = n_chain + 2 * n_ion_pairs
    m = int(math.ceil(n_sites ** (1.0 / 3.0) - 1e-9))
    while m ** 3 < n_sites:
        m += 1
    L = m * cell
    order = rng.permutation(m ** 3)[:n_sites]
    corners = np.stack(np.unravel_index(order, (m, m, m)), axis=1).astype(np.float64) * cell
    g = int(cell / step) - 1   # sublattice points per axis inside a cell, one step of margin
    pos, typ, q, mol, bonds, angles, dihs = [], [], [], [], [], [], []
    moves = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])
    for c in range(n_chain):
        while True:   # self-avoiding walk on the g^3 sublattice of the cell
            p = [rng.integers(0, g, size=3)]
            seen = {tuple(p[0])}
            ok = True
            for _ in range(chain_len - 1):
                cand = [p[-1] + mv for mv in moves]
                # inside the cell, unvisited, and at least sqrt(2) steps from every site three or
                # more bonds back (no U-turns: keeps 1-4 and farther pairs off the LJ wall)
                cand = [x for x in cand if (x >= 0).all() and (x < g).all() and tuple(x) not in seen
                        and all(((x - y) ** 2).sum() >= 2 for y in p[:-2])]
                if not cand:
                    ok = False
                    break
                x = cand[rng.integers(len(cand))]
                p.append(x)
                seen.add(tuple(x))
            if ok:
                break
        base = len(pos)
        for k, x in enumerate(p):
            pos.append(corners[c] + (x + 0.5) * step + rng.normal(scale=0.05, size=3))
            t = 2 if k == chain_len - 1 else k % 2
            typ.append(t)
            q.append(0.2 if t == 0 else -0.2)
            mol.append(c)
        q[-1] = -sum(q[base:-1])
        for k in range(chain_len - 1):
            bonds.append((base + k, base + k + 1))
        for k in range(chain_len - 2):
            angles.append((base + k, base + k + 1, base + k + 2))
        for k in range(chain_len - 3):
            dihs.append((base + k, base + k + 1, base + k + 2, base + k + 3))
    for i in range(2 * n_ion_pairs):
        pos.append(corners[n_chain + i] + rng.uniform(0.3, 0.7, size=3) * cell)
        typ.append(3 + (i % 2))
        q.append(1.0 if i % 2 == 0 else -1.0)
        mol.append(n_chain + i)
    pos = np.mod(np.array(pos), L)
    typ = np.array(typ, np.int32)
    bonds, angles, dihs = (np.array(a, np.int32).reshape(-1, w) for a, w in ((bonds, 2), (angles, 3), (dihs, 4)))
    bond_type = (typ[bonds[:, 0]] + typ[bonds[:, 1]]).astype(np.int32)            # 0..3
    angle_type = (typ[angles[:, 0]] + typ[angles[:, 2]]).astype(np.int32) % 3      # 0..2
    dih_type = (typ[dihs[:, 0]] + typ[dihs[:, 3]]).astype(np.int32) % 3            # 0..2
    mass = np.array([12.011, 15.999, 15.035, 6.94, 140.0])[typ]
    n = len(typ)
    return dict(pos=pos, vel=_maxwell(rng, n, T, mass, 1.9872067e-3, 1.0 / 4.186e-4), mass=mass,
                charge=np.array(q), type=typ, molecule=np.array(mol, np.int32), lo=np.zeros(3),
                hi=np.full(3, L), eps=np.array([0.066, 0.14, 0.17, 0.018, 0.2]),
                sigma=np.array([3.5, 2.9, 3.9, 2.1, 4.0]),
                bonds=bonds, bond_type=bond_type,
                bond_coeffs=np.array([[300.0, step], [320.0, step], [280.0, 1.05 * step], [310.0, step]]),
                angles=angles, angle_type=angle_type,
                angle_coeffs=np.array([[50.0, 109.5], [60.0, 112.0], [45.0, 95.0]]),
                dihedrals=dihs, dihedral_type=dih_type,
                dihedral_coeffs=np.array([[0.15, 1, 3], [0.3, -1, 2], [0.08, 1, 1]]))


def to_json(cfg) -> str:
    return json.dumps(cfg)
