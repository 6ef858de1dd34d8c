"""FP64 numpy restatement of the learned smoother's MLP (test infrastructure).

Forward and backward of 29 -> 64 -> 64 -> 20 with the tanh-form GELU, on the BF16
rounding of the weights (the product computes with BF16 weights and FP32
accumulation), and the loss mean_b ||o_b - y_b||^2.  Used as the oracle of
the GPU gradient kernels.  Parameter layout:
W1 [64][29], b1 [64], W2 [64][64], b2 [64], W3 [20][64], b3 [20].
"""
import numpy as np

NIN, NH, NOUT = 29, 64, 20
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NOUT, NH)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16_round(w):
    """Round float32 values to bfloat16 (round to nearest even) and back."""
    a = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    a = (a + 0x7FFF + lsb) & 0xFFFF0000
    return a.astype(np.uint32).view(np.float32)


def unpack(w):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(w[off:off + n], np.float64).reshape(shape)
        off += n
    return out


C_GELU = np.sqrt(2 / np.pi)


def gelu(x):
    """GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))."""
    return 0.5 * x * (1 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * C_GELU * (1 + 3 * 0.044715 * x * x)


def forward(w, X, bf16_activations=False):
    """bf16_activations: round the inputs and both hidden activations to BF16,
    as the tensor-core path does (its MMA operands are BF16)."""
    p = unpack(bf16_round(w))
    r = (lambda a: bf16_round(np.asarray(a, np.float32)).astype(np.float64)) if bf16_activations else (lambda a: a)
    a1 = r(X) @ p["W1"].T + p["b1"]
    h1 = r(gelu(a1))
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = r(gelu(a2))
    return h2 @ p["W3"].T + p["b3"], (a1, h1, a2, h2, p)


def loss_and_grad(w, X, Y):
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    o, (a1, h1, a2, h2, p) = forward(w, X)
    n = X.shape[0]
    d = o - Y
    loss = float((d * d).sum() / n)
    do = 2 * d / n
    g = {"W3": do.T @ h2, "b3": do.sum(0)}
    dh2 = (do @ p["W3"]) * gelu_grad(a2)
    g["W2"], g["b2"] = dh2.T @ h1, dh2.sum(0)
    dh1 = (dh2 @ p["W2"]) * gelu_grad(a1)
    g["W1"], g["b1"] = dh1.T @ X, dh1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])
