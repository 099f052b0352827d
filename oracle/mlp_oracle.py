"""TEST INFRASTRUCTURE ONLY — FP64 numpy restatement of the closure network.

Mirrors lbm-c_b200/csrc/mlp.cuh / mlp.cu: the six strain features, the
6 -> 32 -> 32 -> 1 SiLU network with the parameter layout W1[32x6], b1,
W2[32x32], b2, W3, b3, the mean-squared-error loss and its gradient, and
(forward_step) the BF16-activation form the step kernel evaluates.  The
tests feed it the GPU's BF16-rounded parameters, so the two compute the same
function; the GPU accumulates in FP32.
"""
import numpy as np

H, IN = 32, 6
W1, B1 = 0, H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
PARAMS = B3 + 1


def strain_features(S, rho):
    """Six invariants of S (xx, yy, zz, xy, yz, xz) and rho - 1, as
    lbm-c_b200/csrc/mlp.cuh strain_features defines them."""
    S = np.asarray(S, np.float64).reshape(-1, 6)
    rho = np.ones(len(S)) if rho is None else np.asarray(rho, np.float64).reshape(-1)
    xx, yy, zz, xy, yz, xz = S.T
    d2 = xx * xx + yy * yy + zz * zz
    ss = d2 + 2 * (xy * xy + yz * yz + xz * xz)
    sabs = np.abs(xx) + np.abs(yy) + np.abs(zz) + 2 * (np.abs(xy) + np.abs(yz) + np.abs(xz))
    det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz)
    return np.stack([0.5 * np.log(2 * ss + 1e-24), np.log(1e-12 + sabs),
                     np.copysign(np.log(1 + np.abs(det) * 1e9), det),
                     (xx + yy + zz) * 1e3, 0.5 * np.log(d2 + 1e-24), (rho - 1) * 1e2], 1)


def silu(x):
    return x / (1 + np.exp(-x))


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(H, IN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3],
            p[B3])


def forward(p, x):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    a1 = x @ w1.T + b1
    h1 = silu(a1)
    a2 = h1 @ w2.T + b2
    h2 = silu(a2)
    return h2 @ w3 + b3, (a1, h1, a2, h2)


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    shape = np.shape(a)
    b = np.ascontiguousarray(a, np.float32).reshape(-1).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(shape)


def silu_bf16(z):
    """The in-step SiLU: h = bf16(z / 2), bf16(h + h t) with t = tanh(h) in
    BF16 (the GPU uses the hardware tanh approximation here)."""
    h = bf16(0.5 * z)
    return bf16(h + h * bf16(np.tanh(h)))


def forward_step(p, x):
    """The network as the step kernel evaluates it on the tensor cores:
    BF16 weights, inputs and activations, FP32 (here FP64) accumulation."""
    w1, b1, w2, b2, w3, b3 = (bf16(a) for a in unpack(p))
    a1 = silu_bf16(bf16(x) @ w1.T + b1)
    a2 = silu_bf16(a1 @ w2.T + b2)
    return a2 @ w3 + b3


def loss_and_grad(p, x, t):
    """Mean squared error and its gradient in the parameter layout."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    n = len(x)
    y, (a1, h1, a2, h2) = forward(p, x)
    r = y - t
    loss = np.mean(r * r)
    dy = 2 * r / n
    g = np.zeros(PARAMS)

    def dsilu(a):
        s = 1 / (1 + np.exp(-a))
        return s + a * s * (1 - s)
    g[W3:B3] = dy @ h2
    g[B3] = dy.sum()
    d2 = (dy[:, None] * w3[None, :]) * dsilu(a2)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * dsilu(a1)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(0)
    return loss, g
