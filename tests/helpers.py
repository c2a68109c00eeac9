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


def pair_sets_equal(c_a, ids_a, c_b, ids_b, rows=1 << 16):
    """Per-atom neighbour sets (as sorted lists) identical; returns the first mismatching atom or -1.
    Rows are compared in blocks (sorted with the unused tail padded), so that a million atoms take
    seconds."""
    c_a = np.asarray(c_a)
    c_b = np.asarray(c_b)
    if not np.array_equal(c_a, c_b):
        return int(np.nonzero(c_a != c_b)[0][0])
    w = int(c_a.max()) if len(c_a) else 0
    if w == 0:
        return -1
    big = np.iinfo(np.int32).max
    for r0 in range(0, len(c_a), rows):
        r1 = min(len(c_a), r0 + rows)
        tail = np.arange(w)[None, :] >= c_a[r0:r1, None]
        a = np.where(tail, big, ids_a[r0:r1, :w]).astype(np.int64)
        b = np.where(tail, big, ids_b[r0:r1, :w]).astype(np.int64)
        a.sort(axis=1)
        b.sort(axis=1)
        bad = np.nonzero((a != b).any(axis=1))[0]
        if len(bad):
            return r0 + int(bad[0])
    return -1


def rel_err(f, ref):
    """max_i |f_i - ref_i| / rms_i |ref_i|  (norm-wise, per-atom force vectors)."""
    rms = np.sqrt((ref ** 2).sum(1).mean())
    return float(np.sqrt(((f - ref) ** 2).sum(1)).max() / rms)


def jitter(pos, lo, hi, scale, seed):
    rng = np.random.default_rng(seed)
    p = pos + rng.normal(scale=scale, size=pos.shape)
    return lo + np.mod(p - lo, hi - lo)
