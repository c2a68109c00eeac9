"""Shared helpers for the parity tests: move a generated system onto the device and bind it."""
from __future__ import annotations

import numpy as np


def to_dev(sysd, device, with_vel=True):
    import torch
    n = sysd["pos"].shape[0]
    t = dict(
        pos=torch.tensor(sysd["pos"], dtype=torch.float64, device=device).contiguous(),
        force=torch.zeros((n, 3), dtype=torch.float64, device=device),
        charge=torch.tensor(sysd["charge"], dtype=torch.float64, device=device),
        type=torch.tensor(sysd["type"], dtype=torch.int32, device=device),
        mass=torch.tensor(sysd["mass"], dtype=torch.float64, device=device),
    )
    if with_vel:
        t["vel"] = torch.tensor(sysd["vel"], dtype=torch.float64, device=device).contiguous()
        t["image"] = torch.zeros((n, 3), dtype=torch.int32, device=device)
    if sysd.get("molecule") is not None:
        t["molecule"] = torch.tensor(sysd["molecule"], dtype=torch.int32, device=device)
    return t


def make_ff(cfg, sysd, dev, boxes=None, offsets=None):
    from copy_gpu_b200 import Box, ForceField
    if boxes is None:
        boxes = [Box(tuple(sysd["lo"]), tuple(sysd["hi"]))]
    ff = ForceField(cfg, boxes)
    ff.set_pair_coeffs(sysd["eps"], sysd["sigma"])
    if "hoh" in sysd:
        ff.set_water(sysd["hoh"], sysd["bond"][0], sysd["bond"][1], sysd["angle"][0], sysd["angle"][1])
    ff.Init(dev["pos"], dev["force"], vel=dev.get("vel"), mass=dev.get("mass"), charge=dev["charge"],
            type=dev["type"], molecule=dev.get("molecule"), image=dev.get("image"),
            replica_offsets=offsets)
    return ff


def pair_sets_equal(c_a, ids_a, c_b, ids_b):
    """Per-atom neighbour sets (as sorted lists) identical; returns the first mismatching atom or -1."""
    if not np.array_equal(c_a, c_b):
        return int(np.nonzero(c_a != c_b)[0][0])
    for i in range(len(c_a)):
        a = np.sort(ids_a[i, :c_a[i]])
        b = np.sort(ids_b[i, :c_b[i]])
        if not np.array_equal(a, b):
            return i
    return -1


def rel_err(f, ref):
    """max_i |f_i - ref_i| / rms_i |ref_i|  (norm-wise, per-atom force vectors)."""
    rms = np.sqrt((ref ** 2).sum(1).mean())
    return float(np.sqrt(((f - ref) ** 2).sum(1)).max() / rms)


def jitter(pos, lo, hi, scale, seed):
    rng = np.random.default_rng(seed)
    p = pos + rng.normal(scale=scale, size=pos.shape)
    return lo + np.mod(p - lo, hi - lo)
