"""CPU restatement of the learned far-field e-map surrogate (test infrastructure).

Checker only: the tests compare the CUDA kernels against these numpy
functions on small seeded cases; nothing on the product path imports this
module.  The surrogate has no counterpart in the reference.  Its exact part
uses the reference's binned kernel

    phi(r) = min(1/r, 2) * invEps[min(int(100 r), 8191)]

(fastgrid_master/fastgrid/electrostatics/Cpu.cpp:59-82, table
InputDataLoader.cpp:715-742) and splits it as

    e(p) = sum_{r<a} w (phi - psi) + sum_all w psi + (binning noise beyond a),

psi(r) = tau(min(r - 0.005, 81.91)) / r for r >= a (tau = 332/eps as a
6-term series in E = exp(-0.3153767175 x)), psi(r) = A + B r^2 + C r^4 for
r < a, matching value, slope and curvature at a.

The corrector network mirrors the GPU's arithmetic: BF16 inputs, weights and
hidden activations (round to nearest even), FP32/FP64 accumulation, leaky
ReLU with slope 1/8, 3x3x3 zero-padded convolutions, no biases.
"""
import numpy as np

LAMBDA = 0.3153767175
SHIFT = 0.005
XMAX = 81.91
SLOPE = 0.125
N_IN, N_CH = 8, 32
W1, W2, W3 = 27 * N_IN * N_CH, 27 * N_CH * N_CH, 27 * N_CH


def ddd_table():
    d = np.arange(8192, dtype=np.float64) / 100.0
    E = np.exp(-LAMBDA * d)
    return (332.0 + (332 * 7.7839) * E) / (78.4 + -66.57180475 * E)


def series_coeffs():
    a, rho, g0 = 7.7839, 66.57180475 / 78.4, 332.0 / 78.4
    poly = [g0]
    rp = 1.0
    for _ in range(1, 6):
        prev = rp
        rp *= rho
        poly.append(g0 * (rp + a * prev))
    return np.array(poly)


def tau(x, poly=None):
    poly = series_coeffs() if poly is None else poly
    E = np.exp(-LAMBDA * np.asarray(x, dtype=np.float64))
    t = np.full_like(E, poly[5])
    for n in range(4, -1, -1):
        t = t * E + poly[n]
    return t


def g_outer(r):
    r = np.asarray(r, dtype=np.float64)
    return tau(np.minimum(r - SHIFT, XMAX)) / r


def split_coeffs(a):
    """(A, B, C) of psi inside a (central differences of g at a, step 1e-3)."""
    h = 1e-3
    gm, g0, gp = g_outer(a - h), g_outer(a), g_outer(a + h)
    g1, g2 = (gp - gm) / (2 * h), (gp - 2 * g0 + gm) / (h * h)
    C = (a * g2 - g1) / (8 * a ** 3)
    B = (g2 - 12 * C * a * a) / 2
    A = g0 - B * a * a - C * a ** 4
    return float(A), float(B), float(C)


def psi(r, a):
    A, B, C = split_coeffs(a)
    r = np.asarray(r, dtype=np.float64)
    inner = A + B * r * r + C * r ** 4
    with np.errstate(divide="ignore"):
        outer = g_outer(np.maximum(r, 1e-12))
    return np.where(r < a, inner, outer)


def points(nx, ny, nz, h):
    """Grid-centred coordinates of all points, x fastest (P, 3)."""
    x = (np.arange(nx) - nx // 2) * h
    y = (np.arange(ny) - ny // 2) * h
    z = (np.arange(nz) - nz // 2) * h
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def direct(pts, xyzw, tab=None):
    """Exact e-map at pts (FP64)."""
    tab = ddd_table() if tab is None else tab
    out = np.zeros(len(pts))
    for i0 in range(0, len(pts), 256):
        p = pts[i0:i0 + 256]
        d = p[:, None, :] - xyzw[None, :, :3]
        r = np.sqrt((d * d).sum(-1))
        with np.errstate(divide="ignore"):
            inv = np.minimum(1.0 / r, 2.0)
        b = np.minimum((r * 100.0).astype(np.int64), 8191)
        out[i0:i0 + 256] = (xyzw[None, :, 3] * inv * tab[b]).sum(1)
    return out


def near_field(pts, xyzw, a, tab=None):
    """sum over atoms within a of w (phi(r) - psi(r))."""
    tab = ddd_table() if tab is None else tab
    A, B, C = split_coeffs(a)
    out = np.zeros(len(pts))
    for i0 in range(0, len(pts), 256):
        p = pts[i0:i0 + 256]
        d = p[:, None, :] - xyzw[None, :, :3]
        r2 = (d * d).sum(-1)
        r = np.sqrt(r2)
        with np.errstate(divide="ignore"):
            inv = np.minimum(1.0 / r, 2.0)
        b = np.minimum((r * 100.0).astype(np.int64), 8191)
        term = inv * tab[b] - (A + B * r2 + C * r2 * r2)
        out[i0:i0 + 256] = (np.where(r < a, term, 0.0) * xyzw[None, :, 3]).sum(1)
    return out


def geometry(nx, ny, nz, h, coarse=1.5, halo=2):
    R = max(1, int(round(coarse / h)))
    nc = [max(2, (n - 1 + R - 1) // R + 1) for n in (nx, ny, nz)]
    return R, nc, halo


def coarse_field(xyzw, nx, ny, nz, h, a, coarse=1.5):
    """Far field sum_all w psi on the coarse nodes incl. a 2-node halo: (Nz, Ny, Nx)."""
    R, nc, H = geometry(nx, ny, nz, h, coarse)
    ax = [((np.arange(-H, c + H) * R) - n // 2) * h for c, n in zip(nc, (nx, ny, nz))]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    out = np.zeros(len(nodes))
    for i0 in range(0, len(nodes), 256):
        p = nodes[i0:i0 + 256]
        d = p[:, None, :] - xyzw[None, :, :3]
        r = np.sqrt((d * d).sum(-1))
        out[i0:i0 + 256] = (psi(r, a) * xyzw[None, :, 3]).sum(1)
    return out.reshape(len(ax[2]), len(ax[1]), len(ax[0]))


def features_and_flin(field, nx, ny, nz, h, coarse=1.5, s_in=1.0):
    """Corrector inputs (P, 8) and the trilinear far field (P,), FP64."""
    R, nc, H = geometry(nx, ny, nz, h, coarse)
    f = field
    c = f[H:H + nc[2], H:H + nc[1], H:H + nc[0]]

    def sh(dz, dy, dx):
        return f[H + dz:H + dz + nc[2], H + dy:H + dy + nc[1], H + dx:H + dx + nc[0]]

    d2 = [sh(0, 0, 1) - 2 * c + sh(0, 0, -1), sh(0, 1, 0) - 2 * c + sh(0, -1, 0), sh(1, 0, 0) - 2 * c + sh(-1, 0, 0)]
    d4 = [sh(0, 0, 2) - 4 * sh(0, 0, 1) + 6 * c - 4 * sh(0, 0, -1) + sh(0, 0, -2),
          sh(0, 2, 0) - 4 * sh(0, 1, 0) + 6 * c - 4 * sh(0, -1, 0) + sh(0, -2, 0),
          sh(2, 0, 0) - 4 * sh(1, 0, 0) + 6 * c - 4 * sh(-1, 0, 0) + sh(-2, 0, 0)]
    ix, iy, iz = np.arange(nx), np.arange(ny), np.arange(nz)
    I = np.minimum(ix // R, nc[0] - 2)
    J = np.minimum(iy // R, nc[1] - 2)
    K = np.minimum(iz // R, nc[2] - 2)
    u = (ix - I * R) / R
    v = (iy - J * R) / R
    w = (iz - K * R) / R
    Kz, Jy, Ix = np.meshgrid(K, J, I, indexing="ij")
    W, V, U = np.meshgrid(w, v, u, indexing="ij")
    wx, wy, wz = [1 - U, U], [1 - V, V], [1 - W, W]

    def interp(arr):
        s = 0
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    s = s + wx[di] * wy[dj] * wz[dk] * arr[Kz + dk, Jy + dj, Ix + di]
        return s

    def deriv(arr, axis):
        s = 0
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    wt = [(wy[dj] * wz[dk]) * (1 if di else -1), (wx[di] * wz[dk]) * (1 if dj else -1),
                          (wx[di] * wy[dj]) * (1 if dk else -1)][axis]
                    s = s + wt * arr[Kz + dk, Jy + dj, Ix + di]
        return s

    F = interp(c)
    D = [interp(d2[k]) for k in range(3)]
    Q = [interp(d4[k]) for k in range(3)]
    G = [deriv(d2[k], k) for k in range(3)]
    b = [U * (1 - U), V * (1 - V), W * (1 - W)]
    fr = [U, V, W]
    feats = [b[0] * D[0], b[1] * D[1], b[2] * D[2], D[0], D[1], D[2],
             sum(b[k] * (2 * fr[k] - 1) * G[k] for k in range(3)), sum(b[k] * Q[k] for k in range(3))]
    feat = np.stack([x.ravel() for x in feats], axis=1) * s_in
    return feat, F.ravel()


# --------------------------------------------------------------------------
# Corrector network (BF16 emulation)
# --------------------------------------------------------------------------
def bf16(x):
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64).reshape(np.shape(x))


def split_weights(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[:W1].reshape(27, N_IN, N_CH), w[W1:W1 + W2].reshape(27, N_CH, N_CH),
            w[W1 + W2:].reshape(27, N_CH, 1))


def _offsets():
    return [(t // 9, (t // 3) % 3, t % 3) for t in range(27)]


def conv(x, W):
    """x (nz, ny, nx, Cin), W (27, Cin, Cout): 3x3x3 zero-padded convolution."""
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, W.shape[2]))
    for t, (dz, dy, dx) in enumerate(_offsets()):
        out += xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :] @ W[t]
    return out


def conv_t(g, W):
    """Adjoint of conv with respect to its input."""
    nz, ny, nx, _ = g.shape
    gp = np.pad(g, ((1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((nz, ny, nx, W.shape[1]))
    for t, (dz, dy, dx) in enumerate(_offsets()):
        out += gp[2 - dz:2 - dz + nz, 2 - dy:2 - dy + ny, 2 - dx:2 - dx + nx, :] @ W[t].T
    return out


def conv_w(x, g):
    """Gradient of sum(g * conv(x, W)) with respect to W: (27, Cin, Cout)."""
    nz, ny, nx, cin = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    G = g.reshape(-1, g.shape[-1])
    out = np.zeros((27, cin, g.shape[-1]))
    for t, (dz, dy, dx) in enumerate(_offsets()):
        out[t] = xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :].reshape(-1, cin).T @ G
    return out


def leaky(x):
    return np.where(x > 0, x, SLOPE * x)


def net_forward(feat, w, shape, emulate_bf16=True):
    """feat (P, 8) -> (o (P,), cache); shape = (nz, ny, nx)."""
    q = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1_, W2_, W3_ = [q(x) for x in split_weights(w)]
    f = q(feat).reshape(*shape, N_IN)
    a1 = q(leaky(conv(f, W1_)))
    a2 = q(leaky(conv(a1, W2_)))
    o = conv(a2, W3_)[..., 0]
    return o.ravel(), (f, a1, a2, W1_, W2_, W3_)


def net_grad(feat, w, shape, target, s_out=1.0, emulate_bf16=True):
    """(o, loss, grad (35424,)) for loss = mean((o - target / s_out)^2)."""
    q = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    o, (f, a1, a2, W1_, W2_, W3_) = net_forward(feat, w, shape, emulate_bf16)
    n = o.size
    e = o - np.asarray(target, dtype=np.float64) / s_out
    loss = float((e * e).mean())
    dO = q(2.0 * e / n).reshape(*shape, 1)
    dW3 = conv_w(a2, dO)
    dZ2 = q(conv_t(dO, W3_) * np.where(a2 > 0, 1.0, SLOPE))
    dW2 = conv_w(a1, dZ2)
    dZ1 = q(conv_t(dZ2, W2_) * np.where(a1 > 0, 1.0, SLOPE))
    dW1 = conv_w(f, dZ1)
    return o, loss, np.concatenate([dW1.ravel(), dW2.ravel(), dW3.ravel()])
