"""rbmd_rhok_noalloc: structure factors for callers that cannot allocate device memory when
they need them (an engine that owns all device memory through its own pool or a fixed budget,
or a step loop that cannot take the device-wide synchronisation of cudaFree).

The entry point keeps its scratch in a static device array of the library, so it is checked
here through the C ABI against the structure factors of the regular force path (same atoms,
same k-samples), on two calls in a row (the second reuses the scratch the first left behind),
with the FP32 tolerance of the other k-space tests.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5   # max |rho - rho_ref| / max |rho_ref|, as for the FP32 k-space parity tests


def test_rhok_noalloc_matches_force_path(cuda, oracle_lib):
    import torch
    import copy_gpu_b200 as c
    from copy_gpu_b200 import systems
    from tests.helpers import make_ff, to_dev

    n, P = 3000, 96
    s = systems.electrolyte(n, seed=12)
    cfg = systems.electrolyte_config(P=P, precision="fp32")
    alpha = cfg["hyper_parameters"]["coulomb"]["alpha"]
    m = oracle_lib.rbe_sample(alpha, s["hi"] - s["lo"], seed=4, step=0, rep=0, P=P)
    dev = to_dev(s, cuda)
    ff = make_ff(cfg, s, dev)
    ff.set_ksamples(m)
    ff.Execute()
    torch.cuda.synchronize()
    ref = ff.get_rhok(P)
    scale = np.abs(ref).max()

    lib = c.library()
    box = c.Box(tuple(s["lo"]), tuple(s["hi"])).c()
    m_dev = torch.tensor(m, dtype=torch.int32, device=cuda).contiguous()
    stream = torch.cuda.current_stream()
    for call in range(2):
        rho = torch.full((P, 2), float("nan"), dtype=torch.float64, device=cuda)
        st = lib.rbmd_rhok_noalloc(dev["pos"].data_ptr(), dev["charge"].data_ptr(), n, ctypes.byref(box),
                                   m_dev.data_ptr(), P, rho.data_ptr(), stream.cuda_stream)
        assert st == c.RBMD_OK, lib.rbmd_last_error()
        torch.cuda.synchronize()
        got = rho.cpu().numpy()
        err = np.abs(got - ref).max() / scale
        assert err <= TOL, f"call {call}: rel err {err:.3e}"
        # and against the FP64 oracle (phase origin at the box's lo corner, as here)
        ref64 = oracle_lib.rhok(s["pos"], s["charge"], s["hi"] - s["lo"], m, origin=s["lo"])
        assert np.abs(got - ref64).max() / np.abs(ref64).max() <= TOL


def test_rhok_noalloc_at_its_limits(cuda, oracle_lib):
    """The fixed scratch at its stated limits (n = 262144 atoms, all charged: 128 chunks, the
    partials at the 4 MiB offset; P = 1024: a 1024-thread block) and a P that is not a multiple
    of 32 (a partly filled last warp), against the FP64 oracle, two calls in a row each."""
    import torch
    import copy_gpu_b200 as c

    lib = c.library()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(31)
    for n, P in ((262144, 1024), (5000, 77)):
        L = np.array([60.0, 64.0, 70.0])
        lo = np.array([-3.0, 1.5, 0.25])
        pos = lo + rng.random((n, 3)) * L
        q = rng.choice([-1.0, 1.0], size=n)
        m = rng.integers(-12, 13, size=(P, 3)).astype(np.int32)
        m[np.all(m == 0, axis=1)] = (1, 0, 0)
        ref64 = oracle_lib.rhok(pos, q, L, m, origin=lo)
        box = c.Box(tuple(lo), tuple(lo + L)).c()
        x_d = torch.tensor(pos, dtype=torch.float64, device=cuda).contiguous()
        q_d = torch.tensor(q, dtype=torch.float64, device=cuda)
        m_d = torch.tensor(m, dtype=torch.int32, device=cuda).contiguous()
        for call in range(2):
            rho = torch.full((P, 2), float("nan"), dtype=torch.float64, device=cuda)
            st = lib.rbmd_rhok_noalloc(x_d.data_ptr(), q_d.data_ptr(), n, ctypes.byref(box), m_d.data_ptr(), P,
                                       rho.data_ptr(), stream.cuda_stream)
            assert st == c.RBMD_OK, lib.rbmd_last_error()
            torch.cuda.synchronize()
            err = np.abs(rho.cpu().numpy() - ref64).max() / np.abs(ref64).max()
            assert err <= TOL, f"n={n} P={P} call {call}: rel err {err:.3e}"


def test_rhok_noalloc_rejects_oversize(cuda):
    import torch
    import copy_gpu_b200 as c
    lib = c.library()
    box = c.Box((0.0, 0.0, 0.0), (10.0, 10.0, 10.0)).c()
    x = torch.zeros((8, 3), dtype=torch.float64, device=cuda)
    q = torch.zeros(8, dtype=torch.float64, device=cuda)
    m = torch.ones((8, 3), dtype=torch.int32, device=cuda)
    rho = torch.zeros((8, 2), dtype=torch.float64, device=cuda)
    # sizes beyond the fixed scratch are refused before anything is launched
    assert lib.rbmd_rhok_noalloc(x.data_ptr(), q.data_ptr(), 262145, ctypes.byref(box), m.data_ptr(), 8,
                                 rho.data_ptr(), None) == c.RBMD_ERR_ARG
    assert b"exceed" in lib.rbmd_last_error()
    assert lib.rbmd_rhok_noalloc(x.data_ptr(), q.data_ptr(), 8, ctypes.byref(box), m.data_ptr(), 1025,
                                 rho.data_ptr(), None) == c.RBMD_ERR_ARG
    # every refusal leaves its own message (not a stale one from an earlier call)
    flat = c.Box((0.0, 0.0, 0.0), (10.0, 0.0, 10.0)).c()
    assert lib.rbmd_rhok_noalloc(x.data_ptr(), q.data_ptr(), 8, ctypes.byref(flat), m.data_ptr(), 8,
                                 rho.data_ptr(), None) == c.RBMD_ERR_ARG
    assert b"not positive" in lib.rbmd_last_error()
    assert lib.rbmd_rhok_noalloc(x.data_ptr(), q.data_ptr(), 0, ctypes.byref(box), m.data_ptr(), 8,
                                 rho.data_ptr(), None) == c.RBMD_ERR_ARG
    assert b"non-positive size" in lib.rbmd_last_error()
