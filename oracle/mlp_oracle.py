"""MLP closure oracle (TEST INFRASTRUCTURE): forward and backward of the per-column network in
NumPy FP64, with the operands of every dense product rounded to BF16 as the tensor-core
kernels stage them (sailfish_b200/csrc/sf_mlp.cu).  The closure has no counterpart in the
reference; this is the CPU check of the CUDA kernels' products and gradients."""
import numpy as np

WIDTH = 128
C_GELU = 0.7978845608028654


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = C_GELU * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * x * x)


def relu(x):
    return np.maximum(x, 0.0)


def relu_grad(x):
    return (x > 0.0).astype(np.float64)


ACTS = {"gelu": (gelu, gelu_grad), "relu": (relu, relu_grad)}


def gemm(A, B, bias=None, act=False, kind="gelu"):
    """act(bf16(A) bf16(B)^T + bias), act GELU (tanh form) or ReLU."""
    z = bf16(A) @ bf16(B).T
    if bias is not None:
        z = z + bias
    return (ACTS[kind][0](z) if act else z), z


def forward(W, b, X, kind="gelu"):
    """Returns output, list of layer inputs, list of pre-activations."""
    a = np.asarray(X, np.float64)
    ins, pres = [], []
    for l in range(len(W)):
        last = l == len(W) - 1
        ins.append(a)
        a, z = gemm(a, W[l], b[l], act=not last, kind=kind)
        pres.append(z)
        if not last:
            a = a.astype(np.float32).astype(np.float64)   # activations are stored in FP32
    return a, ins, pres


def backward(W, ins, pres, dY, kind="gelu"):
    """Gradients (dW, db) for output gradient dY, products with BF16-rounded operands."""
    L = len(W)
    dW, db = [None] * L, [None] * L
    g = np.asarray(dY, np.float64)
    for l in range(L - 1, -1, -1):
        G = g if l == L - 1 else g * ACTS[kind][1](pres[l])
        G = G.astype(np.float32).astype(np.float64)
        dW[l] = bf16(G).T @ bf16(ins[l])
        db[l] = G.sum(axis=0)
        if l > 0:
            g = (bf16(G) @ bf16(W[l])).astype(np.float32).astype(np.float64)
    return dW, db
