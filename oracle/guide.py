"""CPU restatement of the path-guiding network — TEST INFRASTRUCTURE ONLY.

Only tests/ (and the bench's CPU baseline leg) may import this module; the
product path evaluates and trains the network on the GPU (rt_guide.cuh /
rt_guide.cu) and fails without the CUDA library.

The reference has no learned proposal: its diffuse bounce is the cosine lobe
(renderer.rs:545-571, pdf.rs:12-41).  This file restates the published methods
the GPU network is built from, at the GPU's rounding points:
  * hash-grid encoding: Müller et al. 2022 ("Instant neural graphics
    primitives"): 16 levels × 2 features, 2^19 entries per level (read as
    BF16; the float32 master is what Adam updates), dense
    indexing where (res+1)^3 fits, else x ⊕ 2654435761·y ⊕ 805459861·z;
    trilinear weights and sums in float32, in corner order 0..7;
  * one-blob encoding of the outgoing direction ω_o (Müller et al. 2019,
    "Neural importance sampling"), 16 bins for θ/π and 16 for φ/2π; the
    normal enters only the cosine lobe of the mixture;
  * a 64-64-64-64-48 ReLU MLP without biases, BF16 weights, inputs and
    activations (round to nearest even) with products summed exactly here
    (float64) and rounded to float32 — the GPU sums in float32 on the tensor
    cores, so outputs agree to float32 rounding and an occasional one-ulp
    BF16 flip;
  * 8 von Mises–Fisher lobes and a guide fraction α = amax·sigmoid, mixed
    with the cosine lobe by one-sample MIS; loss −w·log p and its analytic
    gradient; Adam (Kingma & Ba 2015) with bias-corrected moments.
Parity: this oracle has no reference counterpart to pin against; the GPU
kernels are checked against it (forward outputs, densities, gradients, Adam).
"""
import numpy as np

LEVELS, TSIZE, NIN, NHID, NOUT, NOUTP, NLOBE = 16, 1 << 19, 64, 64, 41, 48, 8
N_MLP = 3 * NHID * NIN + NOUTP * NHID
N_PARAMS = N_MLP + LEVELS * TSIZE * 2
LOGK_LO = -5.0
AMAX, LKMAX = 0.9, 7.0            # caps of α and log κ used when a call names none
f32 = np.float32


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), kept as float32."""
    x = np.ascontiguousarray(x, dtype=f32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(f32)


def resolutions(min_res=16, scale=1.447):
    out, r = [], float(min_res)
    for _ in range(LEVELS):
        out.append(max(2, int(np.floor(r))))
        r *= scale
    return out


def grid_index(res, x, y, z):
    n1 = res + 1
    if n1 ** 3 <= TSIZE:
        return (x + np.uint32(n1) * (y + np.uint32(n1) * z)).astype(np.uint32)
    with np.errstate(over="ignore"):
        return ((x ^ (y * np.uint32(2654435761)) ^ (z * np.uint32(805459861))) & np.uint32(TSIZE - 1)).astype(np.uint32)


def _cells(res, pn):
    x = (pn * f32(res)).astype(f32)
    c = np.minimum(np.floor(x).astype(np.uint32), np.uint32(res - 1))
    return c, (x - c.astype(f32)).astype(f32)


def _corner_weight(c, f):
    wx = f[:, 0] if c & 1 else (f32(1) - f[:, 0])
    wy = f[:, 1] if c & 2 else (f32(1) - f[:, 1])
    wz = f[:, 2] if c & 4 else (f32(1) - f[:, 2])
    return ((wx * wy).astype(f32) * wz).astype(f32)


def normalise(P, lo, inv):
    return np.clip(((np.asarray(P, f32) - np.asarray(lo, f32)).astype(f32) * np.asarray(inv, f32)).astype(f32), 0, 1)


def encode(params, res, lo, inv, P, WO):
    """(n, 64) BF16-rounded inputs: hash-grid features of P (from the BF16
    copy of the table the GPU gathers from), one-blob of the unit outgoing
    directions WO."""
    table = bf16(params[N_MLP:]).reshape(LEVELS, TSIZE, 2)
    pn = normalise(P, lo, inv)
    n = len(pn)
    enc = np.zeros((n, NIN), f32)
    for l in range(LEVELS):
        cells = [_cells(res[l], pn[:, a]) for a in range(3)]
        ci = np.stack([c for c, _ in cells], 1)
        fr = np.stack([f for _, f in cells], 1)
        a0 = np.zeros(n, f32)
        a1 = np.zeros(n, f32)
        for c in range(8):
            idx = grid_index(res[l], ci[:, 0] + np.uint32(c & 1), ci[:, 1] + np.uint32((c >> 1) & 1),
                             ci[:, 2] + np.uint32(c >> 2))
            w = _corner_weight(c, fr)
            v = table[l, idx]
            a0 = (a0 + (w * v[:, 0]).astype(f32)).astype(f32)
            a1 = (a1 + (w * v[:, 1]).astype(f32)).astype(f32)
        enc[:, 2 * l] = a0
        enc[:, 2 * l + 1] = a1
    th, ph = blob_angles(WO)
    for k in range(16):
        d0 = (f32(16) * th - f32(k + 0.5)).astype(f32)
        d1 = (f32(16) * ph - f32(k + 0.5)).astype(f32)
        enc[:, 32 + k] = np.exp(f32(-0.5) * d0 * d0)
        enc[:, 48 + k] = np.exp(f32(-0.5) * d1 * d1)
    return bf16(enc)


def blob_angles(D):
    """θ/π and φ/2π of unit directions D (n, 3), float32 as the GPU forms them."""
    D = np.asarray(D, f32)
    th = (np.arccos(np.clip(D[:, 2], -1, 1)).astype(f32) * f32(0.318309886)).astype(f32)
    ph = ((np.arctan2(D[:, 1], D[:, 0]).astype(f32) + f32(3.14159265)) * f32(0.159154943)).astype(f32)
    return th, ph


def weights(params):
    W = []
    for l in range(4):
        rows = NOUTP if l == 3 else NHID
        W.append(bf16(params[l * NHID * NIN:l * NHID * NIN + rows * NIN].reshape(rows, NIN)))
    return W


def _mm(a, b):
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(f32)


def forward(params, X):
    """Outputs (n, 48) and the activations (X, H1, H2, H3)."""
    W = weights(params)
    H1 = bf16(np.maximum(_mm(X, W[0].T), 0))
    H2 = bf16(np.maximum(_mm(H1, W[1].T), 0))
    H3 = bf16(np.maximum(_mm(H2, W[2].T), 0))
    return _mm(H3, W[3].T), (X, H1, H2, H3)


def mixture(o, amax=AMAX, lkmax=LKMAX):
    """Per-row mixture: mu (n, 8, 3), kappa (n, 8), pi (n, 8), alpha (n,)."""
    o = np.asarray(o, np.float64)[:, :NOUT]
    lob = o[:, :40].reshape(-1, NLOBE, 5)
    v = lob[:, :, :3]
    ln = np.linalg.norm(v, axis=2)
    mu = np.where(ln[..., None] > 1e-12, v / np.maximum(ln, 1e-300)[..., None], np.array([0.0, 0.0, 1.0]))
    k = np.exp(np.clip(lob[:, :, 3], LOGK_LO, lkmax))
    lg = lob[:, :, 4]
    e = np.exp(lg - lg.max(1, keepdims=True))
    pi = e / e.sum(1, keepdims=True)
    alpha = amax / (1 + np.exp(-o[:, 40]))
    return mu, k, pi, alpha, ln


def vmf_norm(k):
    return k / (2 * np.pi * -np.expm1(-2 * k))


def guide_pdf(o, N, D, amax=AMAX, lkmax=LKMAX):
    """Density of the one-sample mixture (guide and cosine lobe about N) at unit D."""
    mu, k, pi, a, _ = mixture(o, amax, lkmax)
    D = np.asarray(D, np.float64)
    c = np.einsum("nlj,nj->nl", mu, D)
    pg = (pi * vmf_norm(k) * np.exp(k * (c - 1))).sum(1)
    pb = np.maximum((np.asarray(N, np.float64) * D).sum(1), 0) / np.pi
    return a * pg + (1 - a) * pb


def loss_grad(o, N, D, w, scale, amax=AMAX, lkmax=LKMAX):
    """−w·log p_mix per row and the training gradient (n, 41), times scale:
    the lobe outputs descend −w·log p_vmf (the vMF mixture alone), the α
    output descends −w·log p_mix with the lobes fixed; densities floored at
    1e-8."""
    o = np.asarray(o, np.float64)[:, :NOUT]
    mu, k, pi, a, ln = mixture(o, amax, lkmax)
    D = np.asarray(D, np.float64)
    N = np.asarray(N, np.float64)
    w = np.asarray(w, np.float64)
    c = np.einsum("nlj,nj->nl", mu, D)
    f = vmf_norm(k) * np.exp(k * (c - 1))
    pg = (pi * f).sum(1)
    pb = np.maximum((N * D).sum(1), 0) / np.pi
    sg = 1 / (1 + np.exp(-o[:, 40]))
    p = np.maximum(a * pg + (1 - a) * pb, 1e-8)
    loss = -w * np.log(p)
    dp = -w / p * scale
    g = np.zeros((len(o), NOUT))
    g[:, 40] = dp * (pg - pb) * amax * sg * (1 - sg)
    dq = -w / np.maximum(pg, 1e-8) * scale
    gpi = dq[:, None] * f
    gs = (pi * gpi).sum(1, keepdims=True)
    lob = np.zeros((len(o), NLOBE, 5))
    lob[:, :, 4] = pi * (gpi - gs)
    df = dq[:, None] * pi * f
    lk = o[:, :40].reshape(-1, NLOBE, 5)[:, :, 3]
    with np.errstate(over="ignore"):
        dlk = 1 / k - 2 / np.expm1(2 * k) + (c - 1)
    lob[:, :, 3] = np.where((lk > LOGK_LO) & (lk < lkmax), df * dlk * k, 0)
    cm = np.where(ln > 1e-12, df * k / np.maximum(ln, 1e-300), 0)
    lob[:, :, :3] = cm[..., None] * (D[:, None, :] - mu * c[..., None])
    g[:, :40] = lob.reshape(-1, 40)
    return loss, g


def loss_and_grad(params, res, lo, inv, samples, amax=AMAX, lkmax=LKMAX):
    """Σ loss (−w·log p_mix) of samples (n × 13: position, normal, ω_o,
    direction, weight) and the training gradient over all parameters
    (loss_grad's objectives over n), following the GPU's rounding points: dO, dZ in BF16, weight gradients summed exactly,
    hash-grid gradients as float32 products scattered per corner."""
    s = np.asarray(samples, f32).reshape(-1, 13)
    n = len(s)
    P, N, WO, D, w = s[:, 0:3], s[:, 3:6], s[:, 6:9], s[:, 9:12], s[:, 12]
    X = encode(params, res, lo, inv, P, WO)
    O, (X, H1, H2, H3) = forward(params, X)
    W = weights(params)
    valid = w > 0
    loss, g = loss_grad(O, N, D, w, 1.0 / n, amax, lkmax)
    g[~valid] = 0
    dO = np.zeros((n, NOUTP), f32)
    dO[:, :NOUT] = g.astype(f32)
    dO = bf16(dO)
    dZ3 = bf16(_mm(dO, W[3]) * (H3 > 0))
    dZ2 = bf16(_mm(dZ3, W[2]) * (H2 > 0))
    dZ1 = bf16(_mm(dZ2, W[1]) * (H1 > 0))
    dX = _mm(dZ1, W[0])
    grad = np.zeros(N_PARAMS, np.float64)
    for l, (dz, h) in enumerate(((dZ1, X), (dZ2, H1), (dZ3, H2), (dO, H3))):
        gw = dz.astype(np.float64).T @ h.astype(np.float64)
        grad[l * NHID * NIN:l * NHID * NIN + gw.size] = gw.reshape(-1)
    gt = np.zeros((LEVELS, TSIZE, 2), np.float64)
    pn = normalise(P, lo, inv)
    for l in range(LEVELS):
        cells = [_cells(res[l], pn[:, a]) for a in range(3)]
        ci = np.stack([c for c, _ in cells], 1)
        fr = np.stack([f for _, f in cells], 1)
        for c in range(8):
            idx = grid_index(res[l], ci[:, 0] + np.uint32(c & 1), ci[:, 1] + np.uint32((c >> 1) & 1),
                             ci[:, 2] + np.uint32(c >> 2))
            wc = _corner_weight(c, fr)
            for ft in range(2):
                np.add.at(gt[l, :, ft], idx[valid], (wc * dX[:, 2 * l + ft]).astype(f32)[valid])
    grad[N_MLP:] = gt.reshape(-1)
    return float(loss[valid].sum()), grad.astype(f32)


def adam(params, m, v, g, t, lr=1e-2, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step in float32 with the GPU's operation order; returns (p, m, v)."""
    b1, b2, lr, eps = f32(b1), f32(b2), f32(lr), f32(eps)
    bc1, bc2 = f32(1.0 - float(b1) ** t), f32(1.0 - float(b2) ** t)
    m = (b1 * m + (f32(1) - b1) * g).astype(f32)
    v = (b2 * v + (f32(1) - b2) * (g * g).astype(f32)).astype(f32)
    step = ((lr * (m / bc1).astype(f32)).astype(f32) / (np.sqrt((v / bc2).astype(f32)) + eps)).astype(f32)
    return (params - step).astype(f32), m, v


def init_params(seed=1):
    """Glorot-uniform weights (output rows 41..47 zero) and a U(−1e-4, 1e-4)
    table, from a numpy generator (any parameter vector serves the checks)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, f32)
    for l in range(4):
        rows, fo = (NOUTP, NOUT) if l == 3 else (NHID, NHID)
        lim = np.sqrt(6.0 / (NIN + fo))
        W = rng.uniform(-lim, lim, (rows, NIN)).astype(f32)
        if l == 3:
            W[NOUT:] = 0
        p[l * NHID * NIN:l * NHID * NIN + rows * NIN] = W.reshape(-1)
    p[N_MLP:] = rng.uniform(-1e-4, 1e-4, N_PARAMS - N_MLP).astype(f32)
    return p

