"""Oracle (test infrastructure only: imported by tests, never by the library) for the learned warm start's network:
FP64 numpy restatements of the 3x3 convolution (forward, data gradient, weight and bias gradients), f x f average
pooling, nearest upsampling, the FP32 head, and the whole encoder-decoder forward and backward pass with the
activations rounded to BF16 where the device stores them.

There is no reference implementation to pin this against (the reference has no learned component); the oracle is
the textbook definition of each operation, and the tests check the device kernels against it and against finite
differences of its own loss.

Layouts follow the device: NHWC activations, weights [c_out][9][c_in] with tap = 3 ky + kx reading the pixel at
offset (ky - 1, kx - 1), zero padding 1.
"""
import numpy as np


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shifted(x, dy, dx):
    """x[n, y + dy, x + dx, c] with zeros outside the image."""
    n, h, w, c = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(h, h - dy)
    xs, xe = max(0, -dx), min(w, w - dx)
    out[:, ys:ye, xs:xe, :] = x[:, ys + dy:ye + dy, xs + dx:xe + dx, :]
    return out


def conv_fwd(x, w, b=None, relu=False):
    """y[p][n] = sum_{tap, c} x[p + off(tap)][c] w[n][tap][c] + b[n]"""
    cout = w.shape[0]
    y = np.zeros(x.shape[:3] + (cout,))
    for tap in range(9):
        y += _shifted(x, tap // 3 - 1, tap % 3 - 1) @ w[:, tap, :].T
    if b is not None:
        y += b
    return np.maximum(y, 0.0) if relu else y


def conv_dgrad(dz, w):
    """dx[p][c] = sum_{tap, n} dz[p - off(tap)][n] w[n][tap][c]"""
    dx = np.zeros(dz.shape[:3] + (w.shape[2],))
    for tap in range(9):
        dx += _shifted(dz, -(tap // 3 - 1), -(tap % 3 - 1)) @ w[:, tap, :]
    return dx


def conv_wgrad(x, dz):
    """dw[n][tap][c] = sum_p dz[p][n] x[p + off(tap)][c]; db[n] = sum_p dz[p][n]"""
    cout, cin = dz.shape[-1], x.shape[-1]
    dw = np.zeros((cout, 9, cin))
    dzf = dz.reshape(-1, cout)
    for tap in range(9):
        dw[:, tap, :] = dzf.T @ _shifted(x, tap // 3 - 1, tap % 3 - 1).reshape(-1, cin)
    return dw, dzf.sum(axis=0)


POOL = 4   # pooling / upsampling factor of the network


def pool(x, f=POOL):
    n, h, w, c = x.shape
    return x.reshape(n, h // f, f, w // f, f, c).sum(axis=(2, 4)) / (f * f)


def pool_bwd(dy, f=POOL):
    return np.repeat(np.repeat(dy, f, axis=1), f, axis=2) / (f * f)


def up(x, f=POOL):
    return np.repeat(np.repeat(x, f, axis=1), f, axis=2)


def up_bwd(dy, f=POOL):
    n, h, w, c = dy.shape
    return dy.reshape(n, h // f, f, w // f, f, c).sum(axis=(2, 4))


def head_fwd(x, wh, bh):
    """out[p] = sum_{tap, c} x[p + off(tap)][c] wh[tap][c] + bh"""
    return conv_fwd(x, wh.reshape(1, 9, -1), np.array([bh]))[..., 0]


def head_bwd(x, wh, dout):
    dz = dout[..., None]
    dx = conv_dgrad(dz, wh.reshape(1, 9, -1))
    dw, db = conv_wgrad(x, dz)
    return dx, dw.reshape(-1), db[0]


LAYERS = [(32, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128), (128, 256), (256, 256), (384, 128),
          (128, 128), (192, 64), (64, 64), (96, 32), (32, 32)]


def unpack(theta):
    convs, off = [], 0
    for ci, co in LAYERS:
        w = theta[off:off + 9 * ci * co].reshape(co, 9, ci).astype(np.float64)
        off += 9 * ci * co
        b = theta[off:off + co].astype(np.float64)
        off += co
        convs.append((w, b))
    heads = []
    for _ in range(2):
        heads.append((theta[off:off + 9 * 32].astype(np.float64), float(theta[off + 9 * 32])))
        off += 9 * 32 + 1
    return convs, heads


def _exact(a):
    return np.asarray(a, dtype=np.float64)


def net_forward(theta, x, quantize=True):
    """The encoder-decoder on x [N, H, W, 32]; with quantize, BF16 weights and BF16-rounded stored activations as
    on the device (FP64 arithmetic otherwise exact). Returns the output and the tape for net_backward."""
    bf16 = globals()["bf16"] if quantize else _exact
    convs, heads = unpack(theta)
    wq = [(bf16(w), b) for w, b in convs]
    tape = {"q": quantize}

    def conv(l, a, skip=None):
        inp = a if skip is None else np.concatenate([a, skip], axis=-1)
        y = bf16(conv_fwd(inp, wq[l][0], wq[l][1], relu=True))
        tape[l] = (inp, y)
        return y

    s0 = conv(1, conv(0, x))
    s1 = conv(3, conv(2, bf16(pool(s0))))
    s2 = conv(5, conv(4, bf16(pool(s1))))
    bb = conv(7, conv(6, bf16(pool(s2))))
    d2 = conv(9, conv(8, up(bb), s2))
    d1 = conv(11, conv(10, up(d2), s1))
    d0 = conv(13, conv(12, up(d1), s0))
    out = [head_fwd(d0, wh, bh) for wh, bh in heads]
    tape["head"] = d0
    if quantize:
        out = [o.astype(np.float32).astype(np.float64) for o in out]
    return out, (tape, wq, heads)


def net_backward(theta, tape_all, dout):
    """Gradient of sum_h sum(out[h] * dout[h]) with respect to theta (same order), BF16-rounded data gradients as
    stored on the device."""
    tape, wq, heads = tape_all
    bf16 = globals()["bf16"] if tape["q"] else _exact
    grads = [None] * len(LAYERS)
    d0 = tape["head"]
    g = 0.0
    ghead = []
    for (wh, _), do in zip(heads, dout):
        gx, gwh, gbh = head_bwd(d0, wh, do)
        g = g + gx
        ghead.append((gwh, gbh))
    g = bf16(g)

    def conv_back(l, dy, need_dx=True):
        inp, y = tape[l]
        dz = bf16(np.where(y > 0.0, dy, 0.0))
        dw, db = conv_wgrad(inp, dz)
        grads[l] = (dw, db)
        return bf16(conv_dgrad(dz, wq[l][0])) if need_dx else None

    def split(d, c1):
        return d[..., :c1], d[..., c1:]

    d = conv_back(13, g)
    du0, ds0 = split(conv_back(12, d), 64)
    d = bf16(up_bwd(du0))
    d = conv_back(11, d)
    du1, ds1 = split(conv_back(10, d), 128)
    d = bf16(up_bwd(du1))
    d = conv_back(9, d)
    du2, ds2 = split(conv_back(8, d), 256)
    d = bf16(up_bwd(du2))
    d = conv_back(7, d)
    d = conv_back(6, d)
    d = bf16(bf16(pool_bwd(d)) + ds2)
    d = conv_back(5, d)
    d = conv_back(4, d)
    d = bf16(bf16(pool_bwd(d)) + ds1)
    d = conv_back(3, d)
    d = conv_back(2, d)
    d = bf16(bf16(pool_bwd(d)) + ds0)
    d = conv_back(1, d)
    conv_back(0, d, need_dx=False)
    out = []
    for dw, db in grads:
        out.append(dw.reshape(-1))
        out.append(db)
    for gwh, gbh in ghead:
        out.append(gwh)
        out.append(np.array([gbh]))
    return np.concatenate(out)
