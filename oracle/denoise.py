"""CPU oracle for the learned denoiser (test infrastructure only).

The denoiser has no counterpart in the reference, so this restates the
product's own definition of it in numpy, operation by operation, to check the
CUDA kernels (fornos_b200/csrc/fk_denoise.cu):

* features: dense W x H image of 3 float4 planes per pixel,
  (AO, octahedral BN.xy, coverage), (position / R, mapping distance / R),
  (octahedral normal.xy, texel spacing, 0); float32 arithmetic in the
  kernel's order, so the image is bit-exact;
* rows: 25 neighbours x 10 features (positions relative to the centre in
  units of its texel spacing, clamped to +-4), bf16-rounded (round to nearest
  even), padded to 256 columns; bit-exact;
* forward / backward of the MLP 250 -> 64 -> 64 -> 4 with tanh-form GELU.  With
  `bf16=True` the activations, the output gradient and the pre-activation
  gradients are rounded to bf16 at the points where the kernels feed them to
  the tensor cores, and products are accumulated in float64; the kernels
  accumulate in float32, so agreement is to accumulation-order rounding.  With
  `bf16=False` and float64 inputs it is the exact network, which the finite-
  difference test pins;
* Adam with float32 master weights in the kernel's operation order (bit-exact
  given the same gradient).
"""
import numpy as np

INPUTS, K1, HIDDEN, OUT = 250, 256, 64, 4
LAYOUT = {"w1": (0, (64, 256)), "b1": (16384, (64,)), "w2": (16448, (64, 64)), "b2": (20544, (64,)),
          "w3": (20608, (4, 64)), "b3": (20864, (4,))}
PARAMS = 20868
MISS = 0xFFFFFFFF
K0 = np.float32(0.7978845608028654)
KC = np.float32(0.044715)
K3 = np.float32(3.0) * KC
f32 = np.float32


def bf16(x):
    """float32 -> nearest-even bf16, returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p, dtype=np.float32):
    p = np.asarray(p, dtype)
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in LAYOUT.items()}


def init_params(seed):
    """He-style initialisation used to start training (W1's pad columns zero)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    q = unpack(p)
    q["w1"][:, :INPUTS] = rng.normal(0, np.sqrt(2.0 / INPUTS), (HIDDEN, INPUTS))
    q["w2"][:] = rng.normal(0, np.sqrt(2.0 / HIDDEN), (HIDDEN, HIDDEN))
    q["w3"][:] = rng.normal(0, 0.1 * np.sqrt(1.0 / HIDDEN), (OUT, HIDDEN))
    return p


def gelu(z):
    """tanh-form GELU and its derivative, in the kernel's float32 order (works
    in float64 for float64 input)."""
    t = z.dtype.type
    k0, kc, k3 = t(K0), t(KC), t(K3)
    z2 = z * z
    u = k0 * (z + kc * (z2 * z))
    th = np.tanh(u)
    half, one = t(0.5), t(1.0)
    dz = half * (one + th) + (half * z) * ((one - th * th) * (k0 * (one + k3 * z2)))
    return (half * z) * (one + th), dz


def oct_encode(v):
    v = np.asarray(v, np.float32)
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    s = (np.abs(x) + np.abs(y)) + np.abs(z)
    ok = (s > 0) & np.isfinite(s)
    with np.errstate(all="ignore"):
        px, py = x / s, y / s
        sx = np.where(px >= 0, f32(1), f32(-1))
        sy = np.where(py >= 0, f32(1), f32(-1))
        qx = (f32(1) - np.abs(py)) * sx
        qy = (f32(1) - np.abs(px)) * sy
    neg = z < 0
    ox = np.where(neg, qx, px)
    oy = np.where(neg, qy, py)
    return np.where(ok, ox, 0).astype(np.float32), np.where(ok, oy, 0).astype(np.float32)


def features(w, h, indices, tidx, coords, ao, bn3, pos3, nrm3, max_d):
    """(3, W*H, 4) float32 image."""
    f = np.zeros((3, w * h, 4), np.float32)
    idx = np.asarray(indices, np.uint32)
    keep = (idx < w * h) & (np.asarray(tidx) != MISS)
    p = idx[keep]
    r = f32(max_d)
    obx, oby = oct_encode(np.asarray(bn3, np.float32).reshape(-1, 3)[keep])
    onx, ony = oct_encode(np.asarray(nrm3, np.float32).reshape(-1, 3)[keep])
    pos = np.asarray(pos3, np.float32).reshape(-1, 3)[keep]
    f[0, p] = np.stack([np.asarray(ao, np.float32)[keep], obx, oby, np.ones_like(obx)], 1)
    f[1, p] = np.stack([pos[:, 0] / r, pos[:, 1] / r, pos[:, 2] / r,
                        np.asarray(coords, np.float32).reshape(-1, 4)[keep, 0] / r], 1)
    f[2, p] = np.stack([onx, ony, np.zeros_like(onx), np.zeros_like(onx)], 1)
    # texel spacing: mean distance to the covered 4-neighbours (right, left, down, up)
    x, y = (p % w).astype(np.int64), (p // w).astype(np.int64)
    total = np.zeros(len(p), np.float32)
    k = np.zeros(len(p), np.int64)
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        nx, ny = x + dx, y + dy
        ok = (nx >= 0) & (ny >= 0) & (nx < w) & (ny < h)
        q = np.where(ok, ny * w + nx, 0)
        ok &= f[0, q, 3] > 0
        d = f[1, q, :3] - f[1, p, :3]
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        total = np.where(ok, total + dist, total).astype(np.float32)
        k += ok
    with np.errstate(all="ignore"):
        f[2, p, 2] = np.where(k > 0, total / k.astype(np.float32), 0)
    return f


def rows(f, w, h, pixels):
    """(M, 256) float32 holding bf16 values."""
    pixels = np.asarray(pixels, np.int64)
    m = len(pixels)
    out = np.zeros((m, 25, 10), np.float32)
    valid = pixels < w * h
    cx, cy = pixels % w, pixels // w
    for j in range(25):
        dx, dy = j % 5 - 2, j // 5 - 2
        x, y = cx + dx, cy + dy
        ok = valid & (x >= 0) & (y >= 0) & (x < w) & (y < h)
        q = np.where(ok, y * w + x, 0)
        a = f[0, q]
        ok &= a[:, 3] > 0
        pc = np.where(valid, pixels, 0)
        b, n, c, sp = f[1, q], f[2, q], f[1, pc], f[2, pc, 2]
        with np.errstate(all="ignore"):
            rel = [np.where(sp > 0, np.clip((b[:, k] - c[:, k]) / sp, f32(-4), f32(4)), 0) for k in range(3)]
        v = np.stack([a[:, 0], a[:, 1], a[:, 2], rel[0], rel[1], rel[2], n[:, 0], n[:, 1], b[:, 3],
                      np.ones(m, np.float32)], 1)
        out[:, j] = np.where(ok[:, None], v, 0)
    x = np.zeros((m, K1), np.float32)
    x[:, :INPUTS] = out.reshape(m, INPUTS)
    return bf16(x)


def _mm(a, b, dtype):
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(dtype)


def forward(params, x, bf=True):
    """Network outputs (M, 4) and the cache for backward."""
    dt = np.float32 if bf else np.float64
    q = unpack(params, dt)
    r = bf16 if bf else (lambda v: v)
    w1, w2, w3 = r(q["w1"]), r(q["w2"]), r(q["w3"])
    x = np.asarray(x, dt)
    z1 = _mm(x, w1.T, dt) + q["b1"]
    a1, d1 = gelu(z1)
    a1 = r(a1)
    z2 = _mm(a1, w2.T, dt) + q["b2"]
    a2, d2 = gelu(z2)
    a2 = r(a2)
    y = _mm(a2, w3.T, dt) + q["b3"]
    return y, dict(x=x, a1=a1, a2=a2, d1=d1, d2=d2, w1=w1, w2=w2, w3=w3, dt=dt, r=r)


def backward(params, x, t, bf=True):
    """(gradient of the mean squared error, loss) for rows x with targets t."""
    y, c = forward(params, x, bf)
    dt, r = c["dt"], c["r"]
    t = np.asarray(t, dt)
    b = len(x)
    scale = dt(2.0) / (dt(4.0) * dt(b))
    e = y - t
    loss = float(np.mean(e.astype(np.float64) ** 2))
    dy = scale * e
    dyb = r(dy)
    da2 = _mm(dyb, c["w3"], dt)
    dz2 = da2 * c["d2"]
    dz2b = r(dz2)
    da1 = _mm(dz2b, c["w2"], dt)
    dz1 = da1 * c["d1"]
    dz1b = r(dz1)
    g = np.zeros(PARAMS, dt)
    gq = unpack(g, dt)
    gq["w1"][:] = _mm(dz1b.T, c["x"], dt)
    gq["w1"][:, INPUTS:] = 0
    gq["b1"][:] = dz1.astype(np.float64).sum(0)
    gq["w2"][:] = _mm(dz2b.T, c["a1"], dt)
    gq["b2"][:] = dz2.astype(np.float64).sum(0)
    gq["w3"][:] = _mm(dyb.T, c["a2"], dt)
    gq["b3"][:] = dy.astype(np.float64).sum(0)
    return g, loss


def loss_of(params, x, t):
    """Exact (float64, unrounded) mean squared error, for finite differences."""
    y, _ = forward(np.asarray(params, np.float64), np.asarray(x, np.float64), bf=False)
    return float(np.mean((y - np.asarray(t, np.float64)) ** 2))


def adam(params, m, v, g, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (step counts from 1) in the kernel's float32 order;
    returns new (params, m, v).  W1's pad columns are left untouched."""
    p, m, v, g = (np.array(a, np.float32) for a in (params, m, v, g))
    b1, b2, lr, eps = f32(beta1), f32(beta2), f32(lr), f32(eps)
    c1 = f32(1.0 / (1.0 - float(b1) ** step))
    c2 = f32(1.0 / (1.0 - float(b2) ** step))
    upd = np.ones(PARAMS, bool)
    upd[:LAYOUT["b1"][0]] = (np.arange(LAYOUT["b1"][0]) % K1) < INPUTS
    m2 = b1 * m + (f32(1) - b1) * g
    v2 = b2 * v + (f32(1) - b2) * (g * g)
    mh, vh = m2 * c1, v2 * c2
    p2 = p - lr * mh / (np.sqrt(vh) + eps)
    return np.where(upd, p2, p), np.where(upd, m2, m), np.where(upd, v2, v)


def apply(params, f, w, h, indices, tidx, ao_in, bn_in):
    """Denoised (AO, BN) of every texel of a map."""
    x = rows(f, w, h, indices)
    y, _ = forward(params, x)
    ao_in = np.asarray(ao_in, np.float32)
    bn = np.asarray(bn_in, np.float32).reshape(-1, 3).copy()
    bn[~np.isfinite(bn).all(1)] = 0
    ao = np.clip(ao_in + y[:, 0], f32(0), f32(1))
    vv = bn + y[:, 1:4]
    d = (vv[:, 0] * vv[:, 0] + vv[:, 1] * vv[:, 1]) + vv[:, 2] * vv[:, 2]
    with np.errstate(all="ignore"):
        inv = f32(1) / np.sqrt(d)
    out = np.where((d > 0)[:, None], vv * inv[:, None], 0).astype(np.float32)
    miss = np.asarray(tidx) == MISS
    ao[miss] = 1
    out[miss] = 0
    return ao.astype(np.float32), out
