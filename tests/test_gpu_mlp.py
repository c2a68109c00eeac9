"""The tcgen05 proposal network against its CPU restatement (oracle/mlp.py, FP64 with the same
BF16 roundings): outputs h to 1e-3 of max|h| (the tensor-core pass and the CUDA-core forward
pass of the sampler), group losses to 1e-4, and the parameter gradient
of the mean group loss to 2e-3 norm-wise (FP32 accumulation order and tanhf are the only
differences)."""
import ctypes

import numpy as np
import pytest

from oracle import mlp

pytestmark = pytest.mark.gpu


def _run(cuda, params, x, w, c, train):
    import torch
    import copy_gpu_b200 as cg
    G = x.shape[0] // 256
    P = torch.tensor(params, dtype=torch.float32, device=cuda)
    X = torch.tensor(x, dtype=torch.float32, device=cuda)
    W = torch.tensor(w, dtype=torch.float32, device=cuda)
    C = torch.tensor(c, dtype=torch.float32, device=cuda)
    H = torch.zeros(G * 256, dtype=torch.float32, device=cuda)
    L = torch.zeros(G, dtype=torch.float64, device=cuda)
    GR = torch.zeros(mlp.N_PARAM, dtype=torch.float32, device=cuda)
    ST = torch.zeros(1, dtype=torch.int32, device=cuda)
    st = cg.library().rbmd_proposal_mlp_eval(P.data_ptr(), X.data_ptr(), W.data_ptr(), C.data_ptr(), G, int(train),
                                             H.data_ptr(), L.data_ptr(), GR.data_ptr(), ST.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream)
    assert st == 0, cg.library().rbmd_last_error()
    assert int(ST.item()) == 0, "MLP kernel wait timed out"
    return H.cpu().numpy(), L.cpu().numpy(), GR.cpu().numpy()


@pytest.mark.parametrize("G,seed", [(1, 0), (3, 1), (40, 2)])
def test_mlp_forward_backward_matches_oracle(cuda, G, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(G * 256, 16)).astype(np.float32)
    w = rng.uniform(0.01, 1.0, G * 256).astype(np.float32)
    c = rng.uniform(0.01, 1.0, G * 256).astype(np.float32)
    p = mlp.init_params(seed + 7)
    h, L, g = _run(cuda, p, x, w, c, train=True)
    Lr, Lg, gr, hr = mlp.loss_and_grad(p, x, w, c, bf=True)
    assert np.abs(h - hr).max() <= 1e-3 * np.abs(hr).max()
    assert np.abs(L - Lg).max() <= 1e-4 * max(1.0, np.abs(Lg).max())
    err = np.linalg.norm(g - gr) / np.linalg.norm(gr)
    assert err <= 2e-3, err
    # forward-only launch returns the same outputs
    h2, _, _ = _run(cuda, p, x, w, c, train=False)
    assert np.array_equal(h, h2)
    # the sampler's per-step forward pass on the CUDA cores (train < 0): same roundings, other
    # summation order
    h3, _, _ = _run(cuda, p, x, w, c, train=-1)
    assert np.abs(h3 - hr).max() <= 1e-3 * np.abs(hr).max()
    assert np.abs(h3 - h).max() <= 1e-3 * np.abs(h).max()
