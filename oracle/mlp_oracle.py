"""CPU oracle of the learned closure (test infrastructure only; nothing in the library calls it).

The learned closure replaces the liquid closure's per-cell velocity correction
    du = beta_applied * duRepair + duEOS
(reference src/liquid_closure.cpp:380-389 for the repair kick beta * (P_ref - P_red) / gamma,
:401-436 for the EOS kick; the reference returns both as LiquidClosureResult::duRepairX/Y,
duEOSX/Y, include/liquid_closure.h:29-44) by a stencil MLP. The reference has no network, so
this file restates the library's own definition of it, in float64:

  features  75 per cell: a 5x5 stencil (dy outer, dx inner, offsets -2..2) of N/gamma - 1,
            Ux - <Ux>, Uy - <Uy> of the red cell fields, <.> the mean over the stencil points
            inside the walls; wrapped on periodic axes; a stencil point beyond a wall gives
            N term -1 and velocity terms 0. Cell index c = iy + Ny * ix.
  kick      the network's kick per cell, zero in cells whose stencil crosses a wall (bulk
            only), less sum_c N_c kick_c / n (momentum conserving)
  network   z1 = W1 bf(x) + b1, a1 = gelu(z1), z2 = W2 bf(a1) + b2, a2 = gelu(z2),
            output = W3 a2 + b3, kick = output * scale; GELU in the tanh form of Hendrycks
            and Gimpel, z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))) / 2; every weight
            and bias rounded to BF16 (bf: round to nearest even); the operands of the two
            64-wide layers (x, a1) are BF16 too, a2 is not
  loss      mean over rows and both outputs of (output - target / scale)^2; gradients pass
            straight through the roundings (loss_grad); the tensor-core training kernel
            also rounds its backward operands dz2, dz1 to BF16 (loss_grad_tc)
  Adam      m = b1 m + (1 - b1) g; v = b2 v + (1 - b2) g^2;
            p -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)

Parameter layout (one float32 array): W1[64][75], b1[64], W2[64][64], b2[64], W3[2][64],
b3[2], scale.
"""
import numpy as np

FEAT, HID, OUT = 75, 64, 2
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * FEAT
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
OFF_SCALE = OFF_B3 + OUT
N_PARAMS = OFF_SCALE + 1


def bf16(a):
    """float32 -> nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    p = bf16(np.asarray(params, np.float32)[:OFF_SCALE])
    W1 = p[OFF_W1:OFF_B1].reshape(HID, FEAT)
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(HID, HID)
    b2 = p[OFF_B2:OFF_W3]
    W3 = p[OFF_W3:OFF_B3].reshape(OUT, HID)
    b3 = p[OFF_B3:OFF_SCALE]
    return W1, b1, W2, b2, W3, b3, float(np.float32(params[OFF_SCALE]))


_C = np.sqrt(2.0 / np.pi)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(_C * (z + 0.044715 * z ** 3)))


def gelu_d(z):
    t = np.tanh(_C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3 * 0.044715 * z * z)


def forward(X, params):
    """Network outputs (before the scale) and the intermediates."""
    W1, b1, W2, b2, W3, b3, _ = unpack(params)
    X = bf16(np.asarray(X, np.float32))
    z1 = X @ W1.T + b1
    a1 = bf16(gelu(z1).astype(np.float32))
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    out = a2 @ W3.T + b3
    return out, (X, z1, a1, z2, a2)


def predict(X, params):
    out, _ = forward(X, params)
    return out * unpack(params)[6]


def loss_grad(X, Y, params):
    """(loss, gradient over the parameter array; the scale's entry 0). The gradient is taken
    with respect to the BF16-rounded weights (straight through to the FP32 masters)."""
    W1, b1, W2, b2, W3, b3, scale = unpack(params)
    out, (X, z1, a1, z2, a2) = forward(X, params)
    e = out - np.asarray(Y, np.float64) / scale
    m = e.size
    loss = float(np.sum(e * e) / m)
    d3 = 2.0 * e / m
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = (d3.T @ a2).ravel()
    g[OFF_B3:OFF_SCALE] = d3.sum(0)
    d2 = (d3 @ W3) * gelu_d(z2)
    g[OFF_W2:OFF_B2] = (d2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2) * gelu_d(z1)
    g[OFF_W1:OFF_B1] = (d1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def loss_grad_tc(X, Y, params):
    """loss_grad as the tensor-core training kernel takes it: the backward products run on BF16
    operands, so dz2 and dz1 are rounded to BF16 (through FP32) before they multiply; the
    output layer's gradient stays in FP32 (here float64). Biases are the weights of a constant
    input column, so their gradients are the sums of the same rounded dz."""
    W1, b1, W2, b2, W3, b3, scale = unpack(params)
    out, (X, z1, a1, z2, a2) = forward(X, params)
    e = out - np.asarray(Y, np.float64) / scale
    m = e.size
    loss = float(np.sum(e * e) / m)
    d3 = 2.0 * e / m
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = (d3.T @ a2).ravel()
    g[OFF_B3:OFF_SCALE] = d3.sum(0)
    d2 = bf16(((d3 @ W3) * gelu_d(z2)).astype(np.float32))
    g[OFF_W2:OFF_B2] = (d2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = bf16(((d2 @ W2) * gelu_d(z1)).astype(np.float32))
    g[OFF_W1:OFF_B1] = (d1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def adam_step(params, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trained entries (everything but the scale); returns new arrays."""
    p = np.asarray(params, np.float64).copy()
    m = b1 * m + (1.0 - b1) * g
    v = b2 * v + (1.0 - b2) * g * g
    upd = lr * (m / (1.0 - b1 ** t)) / (np.sqrt(v / (1.0 - b2 ** t)) + eps)
    p[:OFF_SCALE] -= upd[:OFF_SCALE]
    return p, m, v


def features(N, Ux, Uy, Nx, Ny, perx, pery, gamma):
    """Stencil features of every cell: [Nx * Ny, 75] (N, Ux, Uy indexed by c = iy + Ny * ix)."""
    N = np.asarray(N, np.float64).reshape(Nx, Ny)
    Ux = np.asarray(Ux, np.float64).reshape(Nx, Ny)
    Uy = np.asarray(Uy, np.float64).reshape(Nx, Ny)
    ix, iy = np.meshgrid(np.arange(Nx), np.arange(Ny), indexing="ij")
    F = np.zeros((Nx, Ny, FEAT))
    ins = np.zeros((Nx, Ny, 25), bool)
    k = 0
    for dy in range(-2, 3):
        for dx in range(-2, 3):
            jx, jy = ix + dx, iy + dy
            inside = np.ones_like(jx, bool)
            if perx:
                jx = jx % Nx
            else:
                inside &= (jx >= 0) & (jx < Nx)
            if pery:
                jy = jy % Ny
            else:
                inside &= (jy >= 0) & (jy < Ny)
            qx, qy = np.clip(jx, 0, Nx - 1), np.clip(jy, 0, Ny - 1)
            F[..., k] = np.where(inside, N[qx, qy] / gamma - 1.0, -1.0)
            F[..., 25 + k] = np.where(inside, Ux[qx, qy], 0.0)
            F[..., 50 + k] = np.where(inside, Uy[qx, qy], 0.0)
            ins[..., k] = inside
            k += 1
    cnt = ins.sum(-1, keepdims=True)
    for ch in (1, 2):
        U = F[..., 25 * ch:25 * ch + 25]
        F[..., 25 * ch:25 * ch + 25] = np.where(ins, U - U.sum(-1, keepdims=True) / cnt, 0.0)
    return F.reshape(Nx * Ny, FEAT)


def bulk_mask(Nx, Ny, perx, pery):
    """Cells whose 5x5 stencil stays inside the walls (c = iy + Ny * ix)."""
    ix, iy = np.meshgrid(np.arange(Nx), np.arange(Ny), indexing="ij")
    m = np.ones((Nx, Ny), bool)
    if not perx:
        m &= (ix >= 2) & (ix < Nx - 2)
    if not pery:
        m &= (iy >= 2) & (iy < Ny - 2)
    return m.reshape(-1)


def conserving(kick, N):
    """The kick per cell less its particle mean: kick - sum_c N_c kick_c / sum_c N_c."""
    N = np.asarray(N, np.float64)
    return kick - (N[:, None] * kick).sum(0) / N.sum()


def init(seed):
    """Glorot-uniform weights, zero biases, scale 0 (same law as mpcd_learned_init; the draws
    differ)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for off, fo, fi in ((OFF_W1, HID, FEAT), (OFF_W2, HID, HID), (OFF_W3, OUT, HID)):
        b = np.sqrt(6.0 / (fi + fo))
        p[off:off + fo * fi] = rng.uniform(-b, b, fo * fi)
    return p
