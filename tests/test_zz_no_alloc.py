"""The allocation-free backward pass (sf_mlp_backward_static) against the one with a
caller-provided scratch buffer (sf_mlp_backward), through the C ABI.

It serves callers that cannot allocate device memory where they train, for example an
application that owns every device byte through its own pool, or a latency-critical loop that
may not call an allocator.  Its scratch is a fixed array inside the library shared by all
calls, so this test makes two calls in a row (the second one runs over the first one's
leftovers) and checks both.  The file name sorts last so that a run stopping at the first
failure has run every other test first."""
import ctypes

import numpy as np
import pytest


@pytest.mark.gpu
def test_static_scratch_backward_matches_buffer_backward():
    import torch
    from sailfish_b200._lib import lib, MlpParams

    def t(a, dt=torch.float32):
        return torch.tensor(np.asarray(a, np.float32), dtype=dt, device="cuda").contiguous()

    p = lambda x: ctypes.c_void_p(x.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(11)
    W = [t(rng.standard_normal((128, 128)) / np.sqrt(128), torch.bfloat16) for _ in range(5)]
    b = [t(rng.standard_normal(128) * 0.05) for _ in range(5)]
    P = MlpParams()
    for l in range(5):
        P.W[l], P.b[l] = W[l].data_ptr(), b[l].data_ptr()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")

    for call, n in enumerate((512, 384)):
        X = t(rng.standard_normal((n, 128)))
        dY = t(rng.standard_normal((n, 128)) * 1e-2)
        Y = torch.zeros((n, 128), device="cuda")
        acts = torch.zeros((4, n, 128), device="cuda")
        pre = torch.zeros((5, n, 128), device="cuda")
        assert lib.sf_mlp_forward(ctypes.byref(P), n, p(X), p(Y), p(acts), p(pre), p(err), stream) == 0

        grads = {}
        for name in ("buffer", "static"):
            dW = [torch.full((128, 128), float("nan"), device="cuda") for _ in range(5)]
            db = [torch.full((128,), float("nan"), device="cuda") for _ in range(5)]
            pdW = (ctypes.c_void_p * 5)(*[x.data_ptr() for x in dW])
            pdb = (ctypes.c_void_p * 5)(*[x.data_ptr() for x in db])
            if name == "buffer":
                work = torch.zeros((2, n, 128), device="cuda")
                rc = lib.sf_mlp_backward(ctypes.byref(P), n, p(X), p(acts), p(pre), p(dY), pdW, pdb,
                                         p(work), p(err), stream)
            else:
                rc = lib.sf_mlp_backward_static(ctypes.byref(P), n, p(X), p(acts), p(pre), p(dY),
                                                pdW, pdb, p(err), stream)
            assert rc == 0, lib.sf_mlp_last_error()
            torch.cuda.synchronize()
            grads[name] = ([x.cpu().numpy() for x in dW], [x.cpu().numpy() for x in db])
        assert int(err.item()) == 0
        for l in range(5):
            a, s_ = grads["buffer"][0][l], grads["static"][0][l]
            assert np.isfinite(s_).all(), (call, l)
            assert np.abs(a - s_).max() <= 1e-5 * max(np.abs(a).max(), 1e-30), (call, l)
            np.testing.assert_allclose(grads["static"][1][l], grads["buffer"][1][l], rtol=1e-5,
                                       atol=1e-6 * np.abs(grads["buffer"][1][l]).max())

    # sizes beyond the fixed scratch are refused, before any work is queued
    rc = lib.sf_mlp_backward_static(ctypes.byref(P), 4096, None, None, None, None, None, None,
                                    None, stream)
    assert rc != 0 and b"2048" in lib.sf_mlp_last_error()
