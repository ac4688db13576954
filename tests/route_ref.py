"""CPU restatement of the router network (test infrastructure only).

The 8-64-64-1 MLP of temporal-lightfield-reconstruction_b200/csrc/tlfr_route.cu:
ReLU hidden layers, sigmoid output, mean binary cross-entropy.  The device
multiplies BF16 operands with FP32 accumulation; `forward`/`gradient` with
bf16=True round at the same points (standardised inputs, weights, h1, h2, the
backpropagated dh2 and dh1), so their results agree with the device up to the
order of FP32 summation.  bf16=False is the same network without rounding, in
float64, used to check the backward formulas by finite differences.

Parameter block layout (float32): W1 [64][16] (columns 8..15 zero), b1 [64],
W2 [64][64], b2 [64], W3 [64], b3, then mean [8], inv_std [8].
"""
import numpy as np

F, K1, H = 8, 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * K1
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NUM_TRAIN = OFF_B3 + 1
OFF_MEAN = NUM_TRAIN
OFF_INVSTD = OFF_MEAN + F
NUM_PARAMS = OFF_INVSTD + F


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p, dtype=np.float32):
    p = np.asarray(p, dtype)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(H, K1), b1=p[OFF_B1:OFF_W2], W2=p[OFF_W2:OFF_B2].reshape(H, H),
                b2=p[OFF_B2:OFF_W3], W3=p[OFF_W3:OFF_B3], b3=p[OFF_B3], mean=p[OFF_MEAN:OFF_INVSTD],
                inv_std=p[OFF_INVSTD:NUM_PARAMS])


def _r(a, on):
    return bf16(a) if on else a


def forward(p, feats, bf=True):
    dt = np.float32 if bf else np.float64
    q = unpack(p, dt)
    x = np.zeros((feats.shape[0], K1), dt)
    x[:, :F] = (feats.astype(dt) - q["mean"]) * q["inv_std"]
    x = _r(x, bf)
    W1, W2, W3 = (_r(q[k].astype(dt), bf) for k in ("W1", "W2", "W3"))
    h1 = _r(np.maximum(x.astype(np.float64) @ W1.T.astype(np.float64) + q["b1"], 0).astype(dt), bf)
    h2 = _r(np.maximum(h1.astype(np.float64) @ W2.T.astype(np.float64) + q["b2"], 0).astype(dt), bf)
    y = h2.astype(np.float64) @ W3.astype(np.float64) + float(q["b3"])
    prob = 1.0 / (1.0 + np.exp(-y))
    return dict(x=x, h1=h1, h2=h2, y=y, p=prob, W1=W1, W2=W2, W3=W3)


def loss(p, feats, labels, bf=True):
    f = forward(p, feats, bf)
    pr = np.clip(f["p"], 1e-7, 1 - 1e-7)
    return float(-np.mean(labels * np.log(pr) + (1 - labels) * np.log(1 - pr)))


def gradient(p, feats, labels, bf=True):
    """Gradient of the mean cross-entropy over the trainable prefix (float64)."""
    f = forward(p, feats, bf)
    n = feats.shape[0]
    dy = (f["p"] - labels) / n
    h1, h2, x = (f[k].astype(np.float64) for k in ("h1", "h2", "x"))
    W2, W3 = f["W2"].astype(np.float64), f["W3"].astype(np.float64)
    g = np.zeros(NUM_TRAIN, np.float64)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    dh2 = dy[:, None] * W3[None, :]
    if bf:
        dh2 = bf16(dh2.astype(np.float32)).astype(np.float64)
    dh2 = dh2 * (h2 > 0)
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = dh2 @ W2
    if bf:
        dh1 = bf16(dh1.astype(np.float32)).astype(np.float64)
    dh1 = dh1 * (h1 > 0)
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).ravel()
    g[OFF_W1:OFF_B1] = (dh1.T @ x).ravel()
    return g


def init_params(seed=1, mean=None, inv_std=None):
    """A random parameter block (not the device's initialiser; for tests)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NUM_PARAMS, np.float32)
    W1 = np.zeros((H, K1), np.float32)
    W1[:, :F] = rng.uniform(-1, 1, (H, F)) * np.sqrt(6 / F)
    p[OFF_W1:OFF_B1] = W1.ravel()
    p[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, H)
    p[OFF_W2:OFF_B2] = rng.uniform(-1, 1, H * H) * np.sqrt(6 / H)
    p[OFF_B2:OFF_W3] = rng.uniform(-0.1, 0.1, H)
    p[OFF_W3:OFF_B3] = rng.uniform(-1, 1, H) * np.sqrt(3 / H)
    p[OFF_B3] = 0.05
    p[OFF_MEAN:OFF_INVSTD] = 0 if mean is None else mean
    p[OFF_INVSTD:NUM_PARAMS] = 1 if inv_std is None else inv_std
    return p


def psnr(a, b):
    """PSNR in dB of RGB images in [0, 1]."""
    d = np.asarray(a, np.float64)[..., :3] - np.asarray(b, np.float64)[..., :3]
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)
