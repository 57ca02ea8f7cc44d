"""Float64 restatement of the path-guiding network (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA guide
kernels (raymond_b200/csrc/guide.cu, raymond_b200/csrc/device/guide.cuh); the
product never imports it.  The guide has no counterpart in the reference, so
this file restates the project's own specification of it:

* inputs: one-blob encoding (quartic kernel (1 - d^2)^2, unit bin width) of
  position x, y, z (32 bins each) and of the normal's and view direction's
  theta / pi, phi / 2 pi (16 bins each) -> 160 values, rounded to bf16;
* MLP 160 -> 64 -> 64 -> 64 -> 48, ReLU between layers, weights rounded to
  bf16 from the FP32 master copy, biases FP32, hidden activations rounded to
  bf16 (the tensor-core kernels keep them as bf16 in shared memory);
* outputs, per lobe j: 4j+0 / 4j+1 mean direction angles through a sigmoid
  (theta in [0, pi], phi in [0, 2 pi]), 4j+2 log concentration clamped to
  [-3, 5], 4j+3 mixture logit (softmax); 32: selection probability
  alpha = 0.02 + 0.48 sigmoid(z);
* loss of a record (features, direction w, BSDF pdf pb, target y), with
  y' = min(y / mean(y), 100) and the mean over the batch: the mixture's
  parameters descend -y' log q(w); the selection probability descends
  -y' log(alpha q(w) + (1 - alpha) pb) with q held fixed; the reported loss
  is the latter.

`forward` / `loss_and_grad` emulate the device's bf16 roundings where asked
(`emulate_bf16`), so the GPU outputs can be compared element by element;
with it off they are plain float64 functions whose gradient the finite
difference test checks.
"""
from __future__ import annotations

import numpy as np

LOBES = 8
INPUTS, HIDDEN, OUTPUTS = 160, 64, 48
LOG_KAPPA_MIN, LOG_KAPPA_MAX = -3.0, 5.0
ALPHA_MIN, ALPHA_MAX = 0.02, 0.5
LAYERS = [(INPUTS, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, OUTPUTS)]
PARAMS = sum(i * o + o for i, o in LAYERS)


def bf16(x) -> np.ndarray:
    """Round float32 values to bf16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
    """[(W [out][in], b [out])] per layer from the flat parameter vector."""
    p = np.asarray(params, np.float64)
    out, off = [], 0
    for i, o in LAYERS:
        W = p[off:off + i * o].reshape(o, i)
        off += i * o
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def encode(features: np.ndarray, emulate_bf16: bool = True) -> np.ndarray:
    """One-blob inputs (n, 160) of features (n, 7), in the device's float32 arithmetic."""
    f = np.asarray(features, np.float32).reshape(-1, 7)
    cols = []
    for feat, bins in [(0, 32), (1, 32), (2, 32), (3, 16), (4, 16), (5, 16), (6, 16)]:
        centres = (np.arange(bins, dtype=np.float32) + np.float32(0.5))
        d = f[:, feat:feat + 1] * np.float32(bins) - centres[None, :]
        x = np.maximum(np.float32(0), np.float32(1) - d * d)
        cols.append(x * x)
    x = np.concatenate(cols, axis=1)
    return bf16(x) if emulate_bf16 else x.astype(np.float64)


def forward(params: np.ndarray, features: np.ndarray, emulate_bf16: bool = True):
    """Raw outputs (n, 48) and the per-layer inputs (for the backward pass)."""
    layers = unpack(params)
    h = encode(features, emulate_bf16)
    acts = [h]
    for li, (W, b) in enumerate(layers):
        Wq = bf16(W) if emulate_bf16 else W
        z = h @ Wq.T + b[None, :]
        if li < 3:
            h = np.maximum(z, 0.0)
            if emulate_bf16:
                h = bf16(h)
            acts.append(h)
        else:
            h = z
    return h, acts


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def decode(o: np.ndarray) -> dict[str, np.ndarray]:
    """Mixture parameters of raw outputs (n, 48)."""
    o = np.asarray(o, np.float64).reshape(-1, OUTPUTS)
    st = _sigmoid(o[:, 0:32:4])
    sp = _sigmoid(o[:, 1:32:4])
    theta, phi = np.pi * st, 2 * np.pi * sp
    lk_raw = o[:, 2:32:4]
    clamped = (lk_raw < LOG_KAPPA_MIN) | (lk_raw > LOG_KAPPA_MAX)
    lk = np.clip(lk_raw, LOG_KAPPA_MIN, LOG_KAPPA_MAX)
    logits = o[:, 3:32:4]
    lam = np.exp(logits - logits.max(axis=1, keepdims=True))
    lam /= lam.sum(axis=1, keepdims=True)
    asig = _sigmoid(o[:, 32])
    mu = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=-1)
    return dict(st=st, sp=sp, theta=theta, phi=phi, log_kappa=lk, clamped=clamped, kappa=np.exp(lk), lam=lam,
                alpha_sig=asig, alpha=ALPHA_MIN + (ALPHA_MAX - ALPHA_MIN) * asig, mu=mu)


def vmf_norm(kappa):
    return kappa / (2 * np.pi * -np.expm1(-2 * kappa))


def mixture_pdf(d: dict[str, np.ndarray], w: np.ndarray) -> np.ndarray:
    """q of one decoded mixture (d of n = 1) at directions w (m, 3): shape (1, m)."""
    w = np.asarray(w, np.float64).reshape(-1, 3)
    cos = np.einsum("njc,mc->nmj", d["mu"], w)
    v = vmf_norm(d["kappa"])[:, None, :] * np.exp(d["kappa"][:, None, :] * (cos - 1))
    return (d["lam"][:, None, :] * v).sum(-1)


def _targets(records: np.ndarray):
    rec = np.asarray(records, np.float64).reshape(-1, 12)
    n = rec.shape[0]
    y32 = np.asarray(records, np.float32).reshape(-1, 12)[:, 11]
    sum_y = np.float64(y32.astype(np.float64).sum())
    yn = np.minimum(rec[:, 11] * (n / sum_y), 100.0) if sum_y > 0 else np.zeros(n)
    return rec, n, yn


def _record_pdfs(d, w):
    cos = np.einsum("njc,nc->nj", d["mu"], w)
    v = vmf_norm(d["kappa"]) * np.exp(d["kappa"] * (cos - 1))
    return cos, v, (d["lam"] * v).sum(1)


def loss_and_grad(params: np.ndarray, records: np.ndarray, emulate_bf16: bool = True):
    """Mean loss over records (n, 12) and the descent direction with respect
    to the flat parameters (float64 backward through the forward's values)."""
    rec, n, yn = _targets(records)
    w, pb = rec[:, 7:10], rec[:, 10]
    out, acts = forward(params, rec[:, 0:7].astype(np.float32), emulate_bf16)
    d = decode(out)
    cos, v, q = _record_pdfs(d, w)
    a = d["alpha"]
    pmix = np.maximum(a * q + (1 - a) * pb, 1e-20)
    loss = float(np.mean(-yn * np.log(pmix)))
    # d / d outputs
    g = np.zeros_like(out)
    g[:, 32] = -yn / pmix / n * (q - pb) * (ALPHA_MAX - ALPHA_MIN) * d["alpha_sig"] * (1 - d["alpha_sig"])
    gq = (-yn / np.maximum(q, 1e-20) / n)[:, None]
    g[:, 3:32:4] = gq * d["lam"] * (v - q[:, None])
    gv = gq * d["lam"]
    k = d["kappa"]
    dlogC = 1 / k - 2 / np.expm1(2 * k)
    g[:, 2:32:4] = np.where(d["clamped"], 0.0, gv * v * (dlogC + cos - 1) * k)
    gmu = gv * v * k
    th, ph = d["theta"], d["phi"]
    dth = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], -1)
    dph = np.stack([-np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph), np.zeros_like(th)], -1)
    g[:, 0:32:4] = gmu * np.einsum("nc,njc->nj", w, dth) * np.pi * d["st"] * (1 - d["st"])
    g[:, 1:32:4] = gmu * np.einsum("nc,njc->nj", w, dph) * 2 * np.pi * d["sp"] * (1 - d["sp"])
    # backward through the layers
    layers = unpack(params)
    grads = []
    delta = g
    for li in range(3, -1, -1):
        W, _ = layers[li]
        Wq = bf16(W) if emulate_bf16 else W
        x = acts[li]
        grads.append((delta.T @ x, delta.sum(0)))
        if li > 0:
            delta = (delta @ Wq) * (x > 0)
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def mixture_pdf_at_records(params: np.ndarray, records: np.ndarray, emulate_bf16: bool = False) -> np.ndarray:
    rec = np.asarray(records, np.float64).reshape(-1, 12)
    out, _ = forward(params, rec[:, 0:7].astype(np.float32), emulate_bf16)
    return _record_pdfs(decode(out), rec[:, 7:10])[2]


def surrogate(params: np.ndarray, records: np.ndarray, q_fixed: np.ndarray, emulate_bf16: bool = False) -> float:
    """The scalar whose gradient loss_and_grad returns, with the mixture's pdf
    in the selection term held at `q_fixed` (per record):
    mean(-y' log q(w)) + mean(-y' log(alpha q_fixed + (1 - alpha) pb))."""
    rec, n, yn = _targets(records)
    out, _ = forward(params, rec[:, 0:7].astype(np.float32), emulate_bf16)
    d = decode(out)
    q = _record_pdfs(d, rec[:, 7:10])[2]
    pmix = np.maximum(d["alpha"] * q_fixed + (1 - d["alpha"]) * rec[:, 10], 1e-20)
    return float(np.mean(-yn * np.log(np.maximum(q, 1e-20))) + np.mean(-yn * np.log(pmix)))


def init_params(seed: int = 0) -> np.ndarray:
    """A seeded Xavier-uniform initialisation with the device's output biases
    (log concentration 1, selection probability 0.2)."""
    rng = np.random.default_rng(seed)
    parts = []
    for li, (i, o) in enumerate(LAYERS):
        a = np.sqrt(6.0 / (i + o))
        b = np.zeros(o)
        if li == 3:
            b[2:32:4] = 1.0
            s = (0.2 - ALPHA_MIN) / (ALPHA_MAX - ALPHA_MIN)
            b[32] = np.log(s / (1 - s))
        parts += [rng.uniform(-a, a, i * o), b]
    return np.concatenate(parts).astype(np.float32)


def adam_step(params, grad, m, v, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba 2015, bias-corrected moments) in float64
    with the device's FP32 coefficients (beta and 1 - beta rounded to float:
    1 - 0.999f is 9.9998713e-4): returns the new parameters and moments."""
    b1, b2 = np.float32(beta1), np.float32(beta2)
    c1, c2 = float(np.float32(1) - b1), float(np.float32(1) - b2)
    b1, b2 = float(b1), float(b2)
    g = np.asarray(grad, np.float64)
    m = b1 * np.asarray(m, np.float64) + c1 * g
    v = b2 * np.asarray(v, np.float64) + c2 * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return np.asarray(params, np.float64) - lr * mh / (np.sqrt(vh) + eps), m, v


def weight_mask() -> np.ndarray:
    """True at the flat parameters that are weights (False at biases)."""
    return np.concatenate([np.concatenate([np.ones(i * o, bool), np.zeros(o, bool)]) for i, o in LAYERS])
