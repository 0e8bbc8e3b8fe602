"""CPU oracle: the learned match filter's 8-64-64-1 MLP in float64.

TEST INFRASTRUCTURE ONLY (imported by tests/ and bench.py; never by the fieldstitch_b200
package).

The network has no counterpart in the reference (PlaneSite accepts guided candidates by the ratio
test of app/planesite/matching.py:142-146 and verifies them with a RANSAC homography,
matching.py:205-233). This module restates the network the CUDA kernels implement: parameter
layout W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3, mu[8], sigma[8]; forward
x_n = (x - mu) / sigma, h1 = relu(W1 x_n + b1), h2 = relu(W2 h1 + b2), z = w3 . h2 + b3,
p = sigmoid(z); loss = mean binary cross-entropy (with logits); and its exact gradient
(backpropagation), which tests/test_oracle_mlp.py checks against central finite differences.
``forward_bf16`` rounds the normalised inputs, the weights and the hidden activations to bfloat16
(round to nearest even) the way the BF16 inference kernel does, accumulating in float64.
"""
import numpy as np

NF, H = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * NF
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
N_TRAIN = OFF_B3 + 1
OFF_MU = N_TRAIN
OFF_SIG = OFF_MU + NF
N_PARAM = OFF_SIG + NF


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, NF), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3], p[OFF_MU:OFF_SIG], p[OFF_SIG:N_PARAM])


def init_params(mu, sigma, seed=0):
    """He-normal hidden layers, small output layer, zero biases (float32 vector)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM, np.float64)
    p[OFF_W1:OFF_B1] = rng.normal(0.0, np.sqrt(2.0 / NF), H * NF)
    p[OFF_W2:OFF_B2] = rng.normal(0.0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0.0, np.sqrt(1.0 / H), H)
    p[OFF_MU:OFF_SIG] = mu
    p[OFF_SIG:N_PARAM] = np.where(np.asarray(sigma) > 1e-6, sigma, 1.0)
    return p.astype(np.float32)


def forward(p, x):
    W1, b1, W2, b2, w3, b3, mu, sig = unpack(p)
    xn = (np.asarray(x, np.float64) - mu) / sig
    a1 = xn @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return z, {"xn": xn, "h1": h1, "h2": h2}


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def loss(p, x, y):
    z, _ = forward(p, x)
    y = np.asarray(y, np.float64)
    return float(np.mean(np.maximum(z, 0.0) - z * y + np.log1p(np.exp(-np.abs(z)))))


def grad(p, x, y):
    """Mean BCE loss and its gradient with respect to the trainable parameters (N_TRAIN)."""
    W1, b1, W2, b2, w3, b3, mu, sig = unpack(p)
    z, c = forward(p, x)
    y = np.asarray(y, np.float64)
    n = len(y)
    dz = (sigmoid(z) - y) / n
    d2 = (dz[:, None] * w3[None, :]) * (c["h2"] > 0)
    d1 = (d2 @ W2) * (c["h1"] > 0)
    g = np.zeros(N_TRAIN, np.float64)
    g[OFF_W1:OFF_B1] = (d1.T @ c["xn"]).reshape(-1)
    g[OFF_B1:OFF_W2] = d1.sum(0)
    g[OFF_W2:OFF_B2] = (d2.T @ c["h1"]).reshape(-1)
    g[OFF_B2:OFF_W3] = d2.sum(0)
    g[OFF_W3:OFF_B3] = c["h2"].T @ dz
    g[OFF_B3] = dz.sum()
    l = float(np.mean(np.maximum(z, 0.0) - z * y + np.log1p(np.exp(-np.abs(z)))))
    return l, g


def bf16(a):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, x):
    W1, b1, W2, b2, w3, b3, mu, sig = unpack(p)
    xn = bf16(((np.asarray(x, np.float32) - mu.astype(np.float32)) / sig.astype(np.float32)).astype(np.float32))
    h1 = bf16(np.maximum(xn @ bf16(W1).T + b1, 0.0))
    h2 = bf16(np.maximum(h1 @ bf16(W2).T + b2, 0.0))
    return sigmoid(h2 @ bf16(w3) + b3)


def adam(p, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on the trainable slice (t = 1 for the first step); returns new (p, m, v)."""
    p = np.array(p, np.float64)
    m = b1 * np.asarray(m, np.float64) + (1 - b1) * g
    v = b2 * np.asarray(v, np.float64) + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    p[:N_TRAIN] -= lr * mh / (np.sqrt(vh) + eps)
    return p, m, v
