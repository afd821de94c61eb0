"""Oracle of the learned path-guiding network: a float64 numpy restatement of its forward pass, of
the von Mises-Fisher mixture head and of the importance-weighted negative log-likelihood with its
analytic gradient. Test infrastructure only: it checks the GPU kernels (FP32 training passes and the
BF16 tensor-core inference) and is never part of the product.

The network maps 8 inputs through 4 hidden ReLU layers of 64 to 40 outputs, 8 lobes x (weight
logit, direction[3], concentration); parameters are stored per layer as W (out x in, row-major)
followed by b. The concentration is softplus(s) + 0.05, clamped at 2000. No reference counterpart:
the reference has no path guiding; this oracle is pinned by finite differences of its own loss.
"""
import numpy as np

N_IN, N_HID, N_LOBES, N_OUT, N_LAYERS = 8, 64, 8, 40, 5
DIMS = [(N_IN, N_HID), (N_HID, N_HID), (N_HID, N_HID), (N_HID, N_HID), (N_HID, N_OUT)]
KAPPA_MIN, KAPPA_MAX = 0.05, 2000.0


def num_params():
    return sum(o * i + o for i, o in DIMS)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    layers, off = [], 0
    for i, o in DIMS:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        layers.append((W, b))
    return layers


def bf16(a):
    """Round to bfloat16 (nearest even) and back, as the tensor-core inference stores operands."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, x, quantize=False):
    """Raw outputs (n x 40) and the hidden activations; quantize emulates the BF16 inference
    (BF16 weights and layer inputs, accumulation in float64 here, FP32 on the GPU, FP32 biases)."""
    h = np.asarray(x, dtype=np.float64)
    hs = []
    for l, (W, b) in enumerate(unpack(p)):
        if quantize:
            h, W = bf16(h), bf16(W)
            b = np.asarray(b, dtype=np.float32).astype(np.float64)
        z = h @ W.T + b
        if l + 1 < N_LAYERS:
            h = np.maximum(z, 0.0)
            hs.append(h)
        else:
            h = z
    return h, hs


def mixture(o):
    o = np.asarray(o, dtype=np.float64).reshape(-1, N_LOBES, 5)
    a = o[:, :, 0]
    logw = a - np.logaddexp.reduce(a, axis=1, keepdims=True)
    m = o[:, :, 1:4]
    n = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(n > 1e-12, m / np.maximum(n, 1e-300), np.array([0.0, 0.0, 1.0]))
    s = o[:, :, 4]
    kap = np.minimum(np.logaddexp(0.0, s) + KAPPA_MIN, KAPPA_MAX)
    return logw, mu, kap, n[:, :, 0]


def log_vmf(kap, c):
    return np.log(kap) - np.log(2 * np.pi) - np.log1p(-np.exp(-2 * kap)) + kap * (c - 1.0)


def log_density(o, k):
    logw, mu, kap, _ = mixture(o)
    k = np.asarray(k, dtype=np.float64).reshape(-1, 1, 3)
    c = np.clip((mu * k).sum(axis=2), -1.0, 1.0)
    return np.logaddexp.reduce(logw + log_vmf(kap, c), axis=1)


def head_grad(o, k):
    """d log q / d o for every sample (n x 40)."""
    o = np.asarray(o, dtype=np.float64).reshape(-1, N_LOBES, 5)
    logw, mu, kap, n = mixture(o)
    k = np.asarray(k, dtype=np.float64).reshape(-1, 1, 3)
    c = (mu * k).sum(axis=2)
    l = logw + log_vmf(kap, c)
    logq = np.logaddexp.reduce(l, axis=1, keepdims=True)
    r = np.exp(l - logq)
    g = np.zeros_like(o)
    g[:, :, 0] = r - np.exp(logw)
    coef = np.where(n > 1e-12, r * kap / np.maximum(n, 1e-300), 0.0)[:, :, None]
    g[:, :, 1:4] = coef * (k - c[:, :, None] * mu)
    e = np.exp(-2 * kap)
    dlogf = 1 / kap - 2 * e / (1 - e) + (c - 1)
    s = o[:, :, 4]
    dk = np.where(np.logaddexp(0.0, s) + KAPPA_MIN < KAPPA_MAX, 1 / (1 + np.exp(-s)), 0.0)
    g[:, :, 4] = r * dlogf * dk
    return g.reshape(-1, N_OUT)


def loss_grad(p, x, k, w):
    """sum_b -w_b log q(k_b | x_b) and its gradient with respect to the parameters."""
    layers = unpack(p)
    out, hs = forward(p, x)
    logq = log_density(out, k)
    loss = float(-(np.asarray(w, dtype=np.float64) * logq).sum())
    delta = -np.asarray(w, dtype=np.float64)[:, None] * head_grad(out, k)
    grads = [None] * N_LAYERS
    inputs = [np.asarray(x, dtype=np.float64)] + hs
    for l in range(N_LAYERS - 1, -1, -1):
        W, _ = layers[l]
        grads[l] = (delta.T @ inputs[l], delta.sum(axis=0))
        if l > 0:
            delta = (delta @ W) * (hs[l - 1] > 0)
    flat = []
    for gW, gb in grads:
        flat.append(gW.ravel())
        flat.append(gb)
    return loss, np.concatenate(flat)


def random_params(seed):
    rng = np.random.default_rng(seed)
    parts = []
    for l, (i, o) in enumerate(DIMS):
        lim = np.sqrt(6.0 / i) * (0.1 if l + 1 == N_LAYERS else 1.0)
        parts.append(rng.uniform(-lim, lim, size=o * i))
        parts.append(rng.normal(0.0, 0.3, size=o))
    return np.concatenate(parts)
