"""Learned closure: the tensor-core (tcgen05) products, forward and backward passes against
the NumPy oracle (oracle/mlp_oracle.py), BF16 operands with FP32 accumulation."""
import ctypes

import numpy as np
import pytest

import mlp_oracle as mo


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    W = [rng.standard_normal((8, 8)) * 0.4 for _ in range(3)]
    b = [rng.standard_normal(8) * 0.1 for _ in range(3)]
    X = rng.standard_normal((5, 8))
    T = rng.standard_normal((5, 8))
    # exact-arithmetic variant of the oracle (no BF16 rounding) for the finite-difference check
    def fwd(W, b):
        a = X
        for l in range(3):
            z = a @ W[l].T + b[l]
            a = z if l == 2 else mo.gelu(z)
        return a
    def loss(W, b):
        return np.mean((fwd(W, b) - T) ** 2)
    a, ins, pres = X, [], []
    for l in range(3):
        ins.append(a)
        z = a @ W[l].T + b[l]
        pres.append(z)
        a = z if l == 2 else mo.gelu(z)
    dY = 2 * (a - T) / a.size
    g = dY
    for l in range(2, -1, -1):
        G = g if l == 2 else g * mo.gelu_grad(pres[l])
        dW = G.T @ ins[l]
        eps = 1e-6
        W2 = [w.copy() for w in W]
        W2[l][1, 2] += eps
        num = (loss(W2, b) - loss(W, b)) / eps
        assert abs(num - dW[1, 2]) < 1e-5 * max(1.0, abs(num))
        g = G @ W[l]


def _cuda():
    import torch
    return torch


def _t(a, dtype="f32"):
    torch = _cuda()
    dt = {"f32": torch.float32, "bf16": torch.bfloat16}[dtype]
    return torch.tensor(np.asarray(a, np.float32), dtype=dt, device="cuda").contiguous()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    torch = _cuda()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.gpu
@pytest.mark.parametrize("M,K", [(128, 128), (256, 128), (200, 64), (128, 384)])
def test_tcgen05_gemm_tile(M, K):
    torch = _cuda()
    from sailfish_b200._lib import lib
    rng = np.random.default_rng(M + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((128, K)).astype(np.float32)
    bias = rng.standard_normal(128).astype(np.float32)
    tA, tB, tb = _t(A), _t(B, "bf16"), _t(bias)
    O = torch.zeros((M, 128), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sf_mlp_gemm(M, K, _p(tA), 0, K, 1, _p(tB), 1, K, 1, _p(tb), 0, _p(O), 128, None, 0,
                         _p(err), _stream())
    assert rc == 0, lib.sf_mlp_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref, _ = mo.gemm(A, mo.bf16(B), bias)
    got = O.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=2e-5, atol=2e-4 * np.abs(ref).max())


class Net:
    def __init__(self, seed=1):
        rng = np.random.default_rng(seed)
        self.W = [mo.bf16(rng.standard_normal((128, 128)) / np.sqrt(128)) for _ in range(5)]
        self.b = [rng.standard_normal(128) * 0.05 for _ in range(5)]

    def device(self):
        from sailfish_b200._lib import MlpParams
        self.tW = [_t(w, "bf16") for w in self.W]
        self.tb = [_t(b) for b in self.b]
        P = MlpParams()
        for l in range(5):
            P.W[l] = self.tW[l].data_ptr()
            P.b[l] = self.tb[l].data_ptr()
        return P


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gelu", "relu"])
def test_mlp_forward_and_backward_match_oracle(kind):
    torch = _cuda()
    from sailfish_b200._lib import lib, MLP_ACT
    n = 256
    rng = np.random.default_rng(3)
    X = rng.standard_normal((n, 128)).astype(np.float32)
    dY = (rng.standard_normal((n, 128)) * 1e-2).astype(np.float32)
    net = Net()
    P = net.device()
    P.act = MLP_ACT[kind]
    tX, tdY = _t(X), _t(dY)
    Y = torch.zeros((n, 128), device="cuda")
    acts = torch.zeros((4, n, 128), device="cuda")
    pre = torch.zeros((5, n, 128), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.sf_mlp_forward(ctypes.byref(P), n, _p(tX), _p(Y), _p(acts), _p(pre), _p(err),
                              _stream()) == 0, lib.sf_mlp_last_error()
    dW = [torch.zeros((128, 128), device="cuda") for _ in range(5)]
    db = [torch.zeros(128, device="cuda") for _ in range(5)]
    work = torch.zeros((2, n, 128), device="cuda")
    pdW = (ctypes.c_void_p * 5)(*[t.data_ptr() for t in dW])
    pdb = (ctypes.c_void_p * 5)(*[t.data_ptr() for t in db])
    assert lib.sf_mlp_backward(ctypes.byref(P), n, _p(tX), _p(acts), _p(pre), _p(tdY), pdW, pdb,
                               _p(work), _p(err), _stream()) == 0, lib.sf_mlp_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref, ins, pres = mo.forward(net.W, net.b, X, kind)
    got = Y.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-2 * np.abs(ref).max())
    rdW, rdb = mo.backward(net.W, ins, pres, dY, kind)
    for l in range(5):
        g = dW[l].cpu().numpy()
        assert np.abs(g - rdW[l]).max() <= 3e-2 * np.abs(rdW[l]).max(), l
        np.testing.assert_allclose(db[l].cpu().numpy(), rdb[l], rtol=0, atol=3e-2 * np.abs(rdb[l]).max())
