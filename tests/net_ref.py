"""NumPy restatement of the refine-flag forecaster (amrlbm_net.cu), the
checker of its forward pass and gradients: the same layers, the same BF16
rounding of weights, inputs, activations and back-propagated products, FP64
arithmetic. Test infrastructure only."""
import numpy as np

CIN, CH, TILE = 4, 32, 18
K1, K2 = CIN * 9, CH * 9
O_W1 = 0
O_B1 = O_W1 + K1 * CH
O_W2 = O_B1 + CH
O_B2 = O_W2 + K2 * CH
O_W3 = O_B2 + CH
O_B3 = O_W3 + K2 * CH
O_WD = O_B3 + CH
O_BD = O_WD + CH
NPARAM = O_BD + 1


EXACT = False  # True: no BF16 or FP32 rounding (for finite-difference checks)


def bf16(a):
    """Round to BF16 (nearest, ties to even), returned as float64."""
    if EXACT:
        return np.asarray(a, dtype=np.float64)
    b = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def im2col(a):
    """[n, H, W, c] -> [n, H, W, 9*c], column o*c + ci, o = (dy+1)*3 + (dx+1)."""
    n, H, W, c = a.shape
    ap = np.pad(a, ((0, 0), (1, 1), (1, 1), (0, 0)))
    cols = np.zeros((n, H, W, 9, c))
    for o in range(9):
        dy, dx = o // 3 - 1, o % 3 - 1
        cols[..., o, :] = ap[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]
    return cols.reshape(n, H, W, 9 * c)


def col2im(dcol, c):
    n, H, W, _ = dcol.shape
    d = dcol.reshape(n, H, W, 9, c)
    out = np.zeros((n, H + 2, W + 2, c))
    for o in range(9):
        dy, dx = o // 3 - 1, o % 3 - 1
        out[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] += d[..., o, :]
    return out[:, 1:H + 1, 1:W + 1, :]


def loss_and_grad(p, x, y, pos_weight=1.0):
    p = np.asarray(p, dtype=np.float64)
    W = [p[O_W1:O_B1].reshape(K1, CH), p[O_W2:O_B2].reshape(K2, CH), p[O_W3:O_B3].reshape(K2, CH)]
    b = [p[O_B1:O_W2], p[O_B2:O_W3], p[O_B3:O_WD]]
    wd, bd = p[O_WD:O_BD], p[O_BD]
    n = len(x)
    a = bf16(np.transpose(np.asarray(x, dtype=np.float64 if EXACT else np.float32), (0, 2, 3, 1)))
    cols, acts = [], []
    for l in range(3):
        col = im2col(a)
        z = col @ bf16(W[l]) + b[l]
        af = np.maximum(z if EXACT else z.astype(np.float32).astype(np.float64), 0.0)
        cols.append(col)
        acts.append(af)
        a = bf16(af)
    a3 = acts[2].reshape(n, -1, CH)
    arg = np.argmax(a3, axis=1)
    pooled = a3.max(axis=1)
    z = pooled @ wd + bd
    wt = np.where(y > 0.5, pos_weight, 1.0)
    loss = np.mean(wt * (np.log1p(np.exp(-np.abs(z))) + np.maximum(z, 0) - z * y))
    dlogit = wt * (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = np.zeros(NPARAM)
    g[O_WD:O_BD] = pooled.T @ dlogit
    g[O_BD] = dlogit.sum()
    dpool = dlogit[:, None] * wd[None, :]
    dA = np.zeros_like(a3)
    for i in range(n):
        dA[i, arg[i], np.arange(CH)] = dpool[i]
    dA = dA.reshape(acts[2].shape)
    for l in (2, 1, 0):
        dz = np.where(acts[l] > 0, dA, 0.0)
        dzb = bf16(dz)
        g[[O_B1, O_B2, O_B3][l]:[O_B1, O_B2, O_B3][l] + CH] = dz.reshape(-1, CH).sum(axis=0)
        col = cols[l].reshape(-1, cols[l].shape[-1])
        dW = col.T @ dzb.reshape(-1, CH)
        off = [O_W1, O_W2, O_W3][l]
        g[off:off + dW.size] = dW.ravel()
        if l == 0:
            break
        dcol = dzb.reshape(-1, CH) @ bf16(W[l]).T
        dA = col2im(dcol.reshape(cols[l].shape), CH)
    return loss, g, z
