"""Reference MLP for the learned star-pressure guess -- TEST INFRASTRUCTURE ONLY.

Float64 numpy forward pass, analytic backward pass of the mean-squared
loss, finite-difference gradients, the feature map and a replica of the
device input generator (splitmix64), all following the parameter layout of
flash5_b200/csrc/riemann_exact.cu: W1[64][8], b1[64], W2[64][64], b2[64],
w3[64], b3.
"""
import numpy as np

NIN, NH = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[OFF_W1:OFF_B1].reshape(NH, NIN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def forward(w, X):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    H1 = np.maximum(X @ W1.T + b1, 0.0)
    H2 = np.maximum(H1 @ W2.T + b2, 0.0)
    return H2 @ w3 + b3, H1, H2


def loss_and_grad(w, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    y, H1, H2 = forward(w, X)
    r = y - T
    n = len(T)
    loss = float((r * r).mean())
    dy = 2.0 * r / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = H2.T @ dy
    g[OFF_B3] = dy.sum()
    dH2 = np.outer(dy, w3) * (H2 > 0)
    g[OFF_W2:OFF_B2] = (dH2.T @ H1).ravel()
    g[OFF_B2:OFF_W3] = dH2.sum(0)
    dH1 = (dH2 @ W2) * (H1 > 0)
    g[OFF_W1:OFF_B1] = (dH1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dH1.sum(0)
    return loss, g


def fd_grad(w, X, T, idx, h=1e-6):
    w = np.asarray(w, dtype=np.float64).copy()
    out = []
    for i in idx:
        w[i] += h
        lp, _ = loss_and_grad(w, X, T)
        w[i] -= 2 * h
        lm, _ = loss_and_grad(w, X, T)
        w[i] += h
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even)."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def forward_bf16(w, X):
    """Forward pass with BF16 weights and activations, FP32-like accumulation."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    W1, W2 = bf16(W1).astype(np.float64), bf16(W2).astype(np.float64)
    H1 = np.maximum(bf16(X).astype(np.float64) @ W1.T + b1, 0.0)
    H1 = bf16(H1).astype(np.float64)
    H2 = np.maximum(H1 @ W2.T + b2, 0.0)
    H2 = bf16(H2).astype(np.float64)
    return H2 @ w3 + b3


def two_rarefaction(L, R, g):
    z = (g - 1.0) / (2.0 * g)
    num = L[3] + R[3] - 0.5 * (g - 1.0) * (R[1] - L[1])
    return (num / (L[3] / L[2] ** z + R[3] / R[2] ** z)) ** (1.0 / z)


def features(S):
    """Feature map of riemann_exact.cu for states S[7][n] (non-vacuum),
    evaluated in float64 (the device evaluates it in FP32)."""
    dl, ul, pl, dr, ur, pr, g = S
    cl, cr = np.sqrt(g * pl / dl), np.sqrt(g * pr / dr)
    ptr = two_rarefaction((dl, ul, pl, cl), (dr, ur, pr, cr), g)
    ppv = np.maximum(0.5 * (pl + pr) - 0.125 * (ur - ul) * (dl + dr) * (cl + cr), 1e-6 * np.minimum(pl, pr))
    gL = np.sqrt(2.0 / ((g + 1.0) * dl) / (ppv + (g - 1.0) / (g + 1.0) * pl))
    gR = np.sqrt(2.0 / ((g + 1.0) * dr) / (ppv + (g - 1.0) / (g + 1.0) * pr))
    pts = np.maximum((gL * pl + gR * pr - (ur - ul)) / (gL + gR), 1e-30)
    f = np.stack([np.log(pr / pl) / np.log(1e4), np.log(dr / dl) / np.log(1e3), ul / cl * 0.2, ur / cr * 0.2,
                  (g - 1.5333333333333333) * 7.5, (ur - ul) / (cl + cr), np.log(ptr / pl) / np.log(1e4),
                  np.log(pts / ptr) / np.log(1e4)], axis=1)
    return f, ptr


M64 = (1 << 64) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def generate(seed, idx):
    """Replica of k_generate for the given sample indices."""
    out = np.zeros((7, len(idx)))
    for c, i in enumerate(idx):
        u = [(splitmix64(seed ^ splitmix64(i * 8 + k)) >> 11) * (1.0 / 9007199254740992.0) for k in range(5)]
        g = 1.4 if u[0] < 0.5 else 5.0 / 3.0
        pr = np.exp(np.log(1e-4) + u[1] * (np.log(1e4) - np.log(1e-4)))
        dr = np.exp(np.log(1e-3) + u[2] * (np.log(1e3) - np.log(1e-3)))
        cl, cr = np.sqrt(g), np.sqrt(g * pr / dr)
        out[:, c] = (1.0, (2 * u[3] - 1) * 5 * cl, 1.0, dr, (2 * u[4] - 1) * 5 * cr, pr, g)
    return out
