"""CPU oracle of the path-guiding network (test infrastructure only).

azimuth has no learned component, so there is no reference code to pin this
part to: this module restates the network of azimuth_b200's path guide in
numpy float64, from its published definitions, and the tests compare the CUDA
kernels with it:

* multiresolution hash-grid encoding (Mueller, Evans, Schied, Keller, "Instant
  Neural Graphics Primitives with a Multiresolution Hash Encoding", SIGGRAPH
  2022): 16 levels, 2^19 entries, 2 features per entry, resolutions
  floor(16 * 2^(7 l / 15)) from 16 to 2048, dense indexing while (res+1)^3 fits
  the table, spatial hash x * 1 ^ y * 2654435761 ^ z * 805459861 otherwise,
  trilinear interpolation;
* a 64-64-64-64 MLP (three ReLU hidden layers and a linear output layer with
  bias) over [grid features (32), normal (3), outgoing direction (3), 1, 0...];
* the proposal: per lobe k a mean direction (normalised outputs 5k..5k+2),
  kappa = exp(clamp(o[5k+3], -3, 5)), mixture weight softmax(o[5k+4]);
  alpha = 0.05 + 0.75 sigmoid(o[40]); density
  q(w) = alpha sum_k pi_k vMF(w; mu_k, kappa_k) + (1 - alpha) max(0, n.w) / pi;
* the loss -w log q(wi) (the KL-divergence estimator of Mueller, McWilliams,
  Rousselle, Gross, Novak, "Neural Importance Sampling", ToG 2019) and its
  gradients.

With `bf16=True` the forward and backward passes round to bfloat16 exactly
where the tensor-core kernels do (network inputs, weights, hidden
activations, the backward's dY and weights), so the comparison with the GPU
is limited by FP32 accumulation order only; with `bf16=False` everything is
float64 (used for the finite-difference checks).
"""
import numpy as np

LEVELS = 16
LOG2_T = 19
T = 1 << LOG2_T
WIDTH = 64
LOBES = 8
LOGK_MIN, LOGK_MAX = -3.0, 5.0
ALPHA_MIN, ALPHA_SPAN = 0.05, 0.75


def level_res():
    return np.array([int(np.floor(16.0 * 2.0 ** (7.0 * l / 15.0))) for l in range(LEVELS)], np.int64)


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def grid_index(x, y, z, res):
    n1 = res + 1
    if n1 ** 3 <= T:
        return (x + n1 * (y + n1 * z)).astype(np.int64)
    h = (x.astype(np.uint64) * np.uint64(1)) ^ (y.astype(np.uint64) * np.uint64(2654435761)) ^ \
        (z.astype(np.uint64) * np.uint64(805459861))
    return (h & np.uint64(0xFFFFFFFF) & np.uint64(T - 1)).astype(np.int64)


def corners(p01, l, res):
    """Corner indices (n, 8) into level l's table and trilinear weights (n, 8)."""
    r = int(res[l])
    x = (p01.astype(np.float32) * np.float32(r))
    i = np.minimum(np.floor(x).astype(np.int64), r - 1)
    f = x.astype(np.float64) - i
    idx = np.empty((len(p01), 8), np.int64)
    w = np.empty((len(p01), 8), np.float64)
    for k in range(8):
        d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
        c = i + d
        idx[:, k] = grid_index(c[:, 0], c[:, 1], c[:, 2], r)
        w[:, k] = np.prod(np.where(d == 1, f, 1.0 - f), axis=1)
    return idx, w


def normalise_positions(pos, lo, inv_ext):
    p = (np.asarray(pos, np.float32) - np.asarray(lo, np.float32)) * np.asarray(inv_ext, np.float32)
    return np.clip(p, 0.0, 1.0).astype(np.float32)


def encode(grid, p01, n, wo, res):
    """Network inputs (n, 64): grid features of every level, normal, wo, 1."""
    N = len(p01)
    x = np.zeros((N, WIDTH))
    for l in range(LEVELS):
        idx, w = corners(p01, l, res)
        feat = grid[l][idx]                       # (N, 8, 2)
        x[:, 2 * l:2 * l + 2] = np.einsum("nk,nkf->nf", w, feat)
    x[:, 32:35] = n
    x[:, 35:38] = wo
    x[:, 38] = 1.0
    return x


def forward(params, x, bf=True):
    """Raw outputs (N, 64) and each layer's input (list of 4 arrays)."""
    mlp, bias = params["mlp"], params["bias"]
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    a = r(x)
    inputs = []
    for l in range(4):
        inputs.append(a)
        z = a @ r(mlp[l])
        if l < 3:
            a = r(np.maximum(z, 0.0))
        else:
            out = z + bias
    return out, inputs


def decode(o):
    """Proposal parameters of raw outputs o (N, 64)."""
    lg = o[:, 4:40:5]
    e = np.exp(lg - lg.max(axis=1, keepdims=True))
    pi = e / e.sum(axis=1, keepdims=True)
    m = np.stack([o[:, 5 * k:5 * k + 3] for k in range(LOBES)], axis=1)       # (N, 8, 3)
    ln = np.sqrt((m * m).sum(axis=2) + 1e-12)
    mu = m / ln[..., None]
    lk = o[:, 3:40:5]
    kap = np.exp(np.clip(lk, LOGK_MIN, LOGK_MAX))
    s = 1.0 / (1.0 + np.exp(-o[:, 40]))
    alpha = ALPHA_MIN + ALPHA_SPAN * s
    return dict(pi=pi, mu=mu, len=ln, lk=lk, kap=kap, s=s, alpha=alpha)


def vmf_pdf(mu, kap, w):
    """vMF density on the sphere: kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu.w - 1))."""
    c = (mu * w[:, None, :]).sum(axis=2)
    return kap / (2.0 * np.pi * -np.expm1(-2.0 * kap)) * np.exp(kap * (c - 1.0)), c


def mixture_pdf(o, n, wi):
    d = decode(o)
    f, _ = vmf_pdf(d["mu"], d["kap"], wi)
    qv = (d["pi"] * f).sum(axis=1)
    pc = np.maximum(0.0, (n * wi).sum(axis=1)) / np.pi
    return d["alpha"] * qv + (1.0 - d["alpha"]) * pc


def loss_and_grad(o, n, wi, w):
    """Loss sum_i -w_i log q_i(wi_i) and its gradient (N, 64) w.r.t. the raw outputs."""
    d = decode(o)
    f, c = vmf_pdf(d["mu"], d["kap"], wi)
    pi, kap, mu, alpha, s = d["pi"], d["kap"], d["mu"], d["alpha"], d["s"]
    qv = (pi * f).sum(axis=1)
    pc = np.maximum(0.0, (n * wi).sum(axis=1)) / np.pi
    q = np.maximum(alpha * qv + (1.0 - alpha) * pc, 1e-30)
    loss = float((-w * np.log(q)).sum())
    g = -w / q
    do = np.zeros_like(o)
    do[:, 40] = g * (qv - pc) * ALPHA_SPAN * s * (1.0 - s)
    gp = g[:, None] * alpha[:, None] * f
    dot = (pi * gp).sum(axis=1, keepdims=True)
    do[:, 4:40:5] = pi * (gp - dot)
    gf = g[:, None] * alpha[:, None] * pi * f
    with np.errstate(over="ignore"):
        dlk = 1.0 / kap - 2.0 / np.expm1(2.0 * kap) + (c - 1.0)
    inside = (d["lk"] > LOGK_MIN) & (d["lk"] < LOGK_MAX)
    do[:, 3:40:5] = np.where(inside, gf * dlk * kap, 0.0)
    gm = (gf * kap)[..., None] * wi[:, None, :]
    pr = (gm * mu).sum(axis=2, keepdims=True)
    dm = (gm - pr * mu) / d["len"][..., None]
    for k in range(LOBES):
        do[:, 5 * k:5 * k + 3] = dm[:, k]
    return loss, do


def backward(params, inputs, do, bf=True):
    """Gradients of the MLP weights (4, 64, 64), the bias (64) and the inputs' first 32 columns."""
    mlp = params["mlp"]
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    dmlp = np.zeros((4, WIDTH, WIDTH))
    dbias = do.sum(axis=0)
    dy = r(do)
    enc = None
    for l in range(3, -1, -1):
        dmlp[l] = inputs[l].T @ dy
        dx = dy @ r(mlp[l]).T
        if l > 0:
            dy = r(np.where(inputs[l] > 0.0, dx, 0.0))
        else:
            enc = dx[:, :32]
    return dmlp, dbias, enc


def rows_split(rows):
    rows = np.asarray(rows, np.float64)
    return rows[:, 0:3], rows[:, 3], rows[:, 4:7], rows[:, 8:11], rows[:, 12:15]


def evaluate(params, grid16, rows, lo, inv_ext, bf=True):
    """Outputs, loss and all gradients for rows of the GuideRow layout (N, 16)."""
    pos, w, n, wo, wi = rows_split(rows)
    res = level_res()
    p01 = normalise_positions(pos, lo, inv_ext)
    x = encode(grid16, p01, n, wo, res)
    o, inputs = forward(params, x, bf)
    loss, do = loss_and_grad(o, n, wi, w)
    dmlp, dbias, enc = backward(params, inputs, do, bf)
    return dict(outputs=o, loss=loss, mlp_grad=dmlp, bias_grad=dbias, enc_grad=enc, x=x)


def sample_vmf(mu, kap, u1, u2):
    """Direction from a vMF lobe: cos theta = 1 + log(u1 + (1 - u1) exp(-2 kappa)) / kappa."""
    ct = np.clip(1.0 + np.log(u1 + (1.0 - u1) * np.exp(-2.0 * kap)) / kap, -1.0, 1.0)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = 2.0 * np.pi * u2
    a = np.where(np.abs(mu[:, 0:1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    u = np.cross(a, mu)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(mu, u)
    return u * (st * np.cos(ph))[:, None] + v * (st * np.sin(ph))[:, None] + mu * ct[:, None]
