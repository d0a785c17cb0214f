"""CPU oracle of the warm-start network (test infrastructure only).

FP64 numpy restatement of the GPU definitions in qkrylov_b200's warm-start
kernels: inputs (spins as +-1, bit set = +1, then J2), two hidden layers of
128 with the tanh form of GELU, outputs (log-amplitude o0, sign logit o1); weights
rounded to BF16 (round to nearest even) as the GPU products see them,
biases in FP32; per-sample loss w [(o0 - a)^2 + c_sign softplus(-y o1)]
averaged over the samples, and its gradient by backpropagation (the
gradient of a weight is taken at its BF16 value).  Parameter layout:
W1 [128][nsites+1], W2 [128][128], W3 [2][128], b1, b2, b3.  There is no
counterpart in the reference; parity here means GPU against this file.
"""
import numpy as np
from scipy.special import erf

HID = 128


def n_params(nsites):
    ki = nsites + 1
    return HID * ki + HID * HID + 2 * HID + HID + HID + 2


def split(p, nsites):
    ki = nsites + 1
    o = 0
    W1 = p[o:o + HID * ki].reshape(HID, ki); o += HID * ki
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    W3 = p[o:o + 2 * HID].reshape(2, HID); o += 2 * HID
    b1 = p[o:o + HID]; o += HID
    b2 = p[o:o + HID]; o += HID
    b3 = p[o:o + 2]
    return W1, W2, W3, b1, b2, b3


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


GELU_C, GELU_K = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """tanh form of GELU (Hendrycks & Gimpel 2016), the network's activation."""
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_K * z ** 3)))


def gelu_d(z):
    t = np.tanh(GELU_C * (z + GELU_K * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_K * z * z)


def gelu_exact(z):
    """GELU with the Gaussian CDF (for the approximation bound test)."""
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def inputs(states, j2, nsites):
    s = np.asarray(states, dtype=np.uint64)
    X = np.empty((s.size, nsites + 1))
    for b in range(nsites):
        X[:, b] = np.where((s >> np.uint64(b)) & np.uint64(1), 1.0, -1.0)
    X[:, nsites] = np.float32(np.broadcast_to(j2, s.shape))  # the GPU reads J2 as float32
    return X


def forward(p, X, nsites, round_bf16=True, act_bf16=False):
    """act_bf16: round the inputs of the two hidden-layer products to BF16,
    as the tensor-core inference kernel does (it keeps FP32 accumulation)."""
    W1, W2, W3, b1, b2, b3 = split(np.asarray(p, np.float32), nsites)
    if round_bf16:
        W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    W1, W2, W3 = (np.asarray(w, np.float64) for w in (W1, W2, W3))
    b1, b2, b3 = (np.asarray(b, np.float64) for b in (b1, b2, b3))
    Z1 = (bf16(X) if act_bf16 else X) @ W1.T + b1
    H1 = gelu(Z1)
    Z2 = (bf16(H1) if act_bf16 else H1) @ W2.T + b2
    H2 = gelu(Z2)
    O = H2 @ W3.T + b3
    return dict(W1=W1, W2=W2, W3=W3, Z1=Z1, H1=H1, Z2=Z2, H2=H2, O=O)


def loss_grad(p, states, j2, targets, nsites, c_sign=1.0, round_bf16=True):
    X = inputs(states, j2, nsites)
    f = forward(p, X, nsites, round_bf16)
    O = f["O"]
    t = np.asarray(targets, np.float64)
    a, y, w = t[:, 0], t[:, 1], t[:, 2]
    n = X.shape[0]
    e = O[:, 0] - a
    m = -y * O[:, 1]
    sp = np.where(m > 20, m, np.log1p(np.exp(np.minimum(m, 20))))
    loss = np.mean(w * (e * e + c_sign * sp))
    dO = np.empty_like(O)
    dO[:, 0] = w * 2 * e / n
    dO[:, 1] = w * c_sign * (1 / (1 + np.exp(-m))) * (-y) / n
    dW3 = dO.T @ f["H2"]
    db3 = dO.sum(0)
    dZ2 = (dO @ f["W3"]) * gelu_d(f["Z2"])
    dW2 = dZ2.T @ f["H1"]
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ f["W2"]) * gelu_d(f["Z1"])
    dW1 = dZ1.T @ X
    db1 = dZ1.sum(0)
    g = np.concatenate([dW1.ravel(), dW2.ravel(), dW3.ravel(), db1, db2, db3])
    return loss, g


def marshall_mask(nsites):
    return sum(1 << b for b in range(1, nsites, 2))


def start_vector(p, states, j2, nsites, act_bf16=False):
    X = inputs(states, j2, nsites)
    O = forward(p, X, nsites, act_bf16=act_bf16)["O"]
    s = np.asarray(states, dtype=np.uint64)
    mm = np.uint64(marshall_mask(nsites))
    par = np.array([bin(int(v)).count("1") & 1 for v in (s & mm)])
    M = np.where(par == 1, -1.0, 1.0)
    return M * np.exp(O[:, 0] - O[:, 0].max()) * np.tanh(O[:, 1])
