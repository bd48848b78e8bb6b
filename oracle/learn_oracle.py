"""CPU restatement of the learned ionosphere preconditioner's network
(gamera_cube_b200/csrc/gcs_learn.cu): forward, loss and parameter gradients.

Test infrastructure only: the GPU kernels are checked against it.  With
``bf16=True`` it rounds where the GPU kernels round -- weights, activations
and the gradient fed to each convolution's backward pass to BF16, products
accumulated in higher precision -- so it agrees with the device gradients
to BF16 noise; with ``bf16=False`` it is the exact float64 network, whose
gradients are pinned against central finite differences.

Layout: tensors [batch][channel][H][W], periodic in W, zero-padded in H.
Packed parameters: for every convolution (in graph order) and output
channel, the 9 Cin weights [ci][tap] (tap = 3 (dh+1) + (dw+1)), then the
bias.  The network has no counterpart in the reference.
"""
import numpy as np

WIDTHS = (16, 32, 48, 64)
IN_CHANNELS = 4


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + (((u >> 16) & 1) + 0x7FFF)) & 0xFFFF0000
    return u.view(np.float32)


def graph(widths=WIDTHS, in_channels=IN_CHANNELS):
    """Ops of the network: ('conv', src, dst, cin, cout, relu, skip, final),
    ('pool', src, dst), ('up', src, dst); tensor 0 is the input."""
    chans = [in_channels]
    ops = []

    def conv(src, cout, relu, skip, final=False):
        chans.append(cout)
        ops.append(("conv", src, len(chans) - 1, chans[src], cout, relu, skip, final))
        return len(chans) - 1

    def pool(src):
        chans.append(chans[src])
        ops.append(("pool", src, len(chans) - 1))
        return len(chans) - 1

    def up(src):
        chans.append(chans[src])
        ops.append(("up", src, len(chans) - 1))
        return len(chans) - 1

    levels = len(widths)
    e = [0] * levels
    h = 0
    for lvl in range(levels):
        if lvl > 0:
            h = pool(e[lvl - 1])
        h = conv(h, widths[lvl], True, -1)
        e[lvl] = conv(h, widths[lvl], True, -1)
    h = e[-1]
    for lvl in range(levels - 2, -1, -1):
        h = up(h)
        h = conv(h, widths[lvl], True, e[lvl])
        h = conv(h, widths[lvl], True, -1)
    conv(h, 1, False, -1, True)
    return ops


def unpack(params, ops):
    """Packed parameter vector -> list of (W [cout][cin][9], b [cout]) per conv."""
    out, o = [], 0
    for op in ops:
        if op[0] != "conv":
            continue
        cin, cout = op[3], op[4]
        blk = np.asarray(params[o:o + cout * (9 * cin + 1)], dtype=np.float64)
        blk = blk.reshape(cout, 9 * cin + 1)
        out.append((blk[:, :9 * cin].reshape(cout, cin, 9), blk[:, 9 * cin].copy()))
        o += cout * (9 * cin + 1)
    assert o == len(params)
    return out


def pack(grads):
    return np.concatenate([np.concatenate([gw.reshape(gw.shape[0], -1), gb[:, None]], axis=1)
                           .ravel() for gw, gb in grads])


def shift(x, dh, dw):
    """y[..., h, w] = x[..., h + dh, (w + dw) mod W], zero outside 0 <= h + dh < H."""
    y = np.roll(x, -dw, axis=-1)
    out = np.zeros_like(y)
    H = x.shape[-2]
    if dh == 0:
        out[...] = y
    elif dh > 0:
        out[..., :H - dh, :] = y[..., dh:, :]
    else:
        out[..., -dh:, :] = y[..., :H + dh, :]
    return out


def taps():
    return [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def conv_forward(x, W, b):
    """sum_{ci,t} W[co, ci, t] x[ci](shifted by tap t) + b[co]."""
    y = np.zeros((x.shape[0], W.shape[0]) + x.shape[2:], dtype=np.float64)
    for t, (dh, dw) in enumerate(taps()):
        xs = shift(x, dh, dw).astype(np.float64)
        y += np.einsum("oc,bchw->bohw", W[:, :, t], xs)
    return y + b[None, :, None, None]


def conv_wgrad(x, gm):
    gW = np.zeros((gm.shape[1], x.shape[1], 9))
    for t, (dh, dw) in enumerate(taps()):
        xs = shift(x, dh, dw).astype(np.float64)
        gW[:, :, t] = np.einsum("bohw,bchw->oc", gm.astype(np.float64), xs)
    return gW, gm.astype(np.float64).sum(axis=(0, 2, 3))


def conv_dgrad(gm, W):
    gx = np.zeros((gm.shape[0], W.shape[1]) + gm.shape[2:], dtype=np.float64)
    for t, (dh, dw) in enumerate(taps()):
        gx += shift(np.einsum("oc,bohw->bchw", W[:, :, t], gm.astype(np.float64)), -dh, -dw)
    return gx


def pool_fwd(x):
    return 0.25 * (x[..., 0::2, 0::2] + x[..., 0::2, 1::2] + x[..., 1::2, 0::2] +
                   x[..., 1::2, 1::2])


def pool_back(g):
    return 0.25 * np.repeat(np.repeat(g, 2, axis=-2), 2, axis=-1)


def up_fwd(x):
    return np.repeat(np.repeat(x, 2, axis=-2), 2, axis=-1)


def up_back(g):
    return g[..., 0::2, 0::2] + g[..., 0::2, 1::2] + g[..., 1::2, 0::2] + g[..., 1::2, 1::2]


def forward(params, x, ops=None, bf16_mode=True):
    """Activations of every tensor; the last conv's output is the prediction
    [B][1][H][W]."""
    ops = ops or graph()
    rnd = bf16 if bf16_mode else (lambda v: np.asarray(v, dtype=np.float64))
    weights = unpack(params, ops)
    if bf16_mode:
        weights = [(bf16(W).astype(np.float64), bf16(b).astype(np.float64)) for W, b in weights]
    acts = {0: rnd(x)}
    ci = 0
    for op in ops:
        if op[0] == "conv":
            _, src, dst, cin, cout, relu, skip, final = op
            W, b = weights[ci]
            ci += 1
            y = conv_forward(acts[src], W, b)
            if skip >= 0:
                y = y + acts[skip]
            if relu:
                y = np.maximum(y, 0.0)
            acts[dst] = y if final else rnd(y)
        elif op[0] == "pool":
            acts[op[2]] = rnd(pool_fwd(np.asarray(acts[op[1]], dtype=np.float64)))
        else:
            acts[op[2]] = up_fwd(acts[op[1]])
    return acts, weights


def loss_and_grads(params, x, target, R, npl, ops=None, bf16_mode=True):
    """Loss sum over h < R, w < npl of (out - target)^2 / (B R npl) and the
    packed parameter gradient."""
    ops = ops or graph()
    acts, weights = forward(params, x, ops, bf16_mode)
    out = acts[max(acts)][:, 0]
    B = x.shape[0]
    scale = 1.0 / (B * R * npl)
    mask = np.zeros(out.shape[1:])
    mask[:R, :npl] = 1.0
    d = (out - target) * mask
    loss = float(np.sum(d * d) * scale)
    if bf16_mode:
        # the device's loss gradient is FP32
        grads = {max(acts): (2.0 * d * scale).astype(np.float32)[:, None].astype(np.float64)}
    else:
        grads = {max(acts): (2.0 * d * scale)[:, None]}
    pgrads = [None] * len(weights)
    ci = len(weights)
    for op in reversed(ops):
        if op[0] == "conv":
            _, src, dst, cin, cout, relu, skip, final = op
            ci -= 1
            g = grads.get(dst, np.zeros_like(acts[dst], dtype=np.float64))
            gm = g * (acts[dst] > 0) if relu else g
            if bf16_mode:
                gm = gm.astype(np.float32).astype(np.float64)
            if skip >= 0:
                grads[skip] = grads.get(skip, 0.0) + gm
            gin = bf16(gm) if bf16_mode else gm
            pgrads[ci] = conv_wgrad(acts[src], gin)
            if src != 0:
                W = weights[ci][0]
                grads[src] = grads.get(src, 0.0) + conv_dgrad(gin, W)
        elif op[0] == "pool":
            g = grads.get(op[2])
            if g is not None:
                grads[op[1]] = grads.get(op[1], 0.0) + pool_back(g)
        else:
            g = grads.get(op[2])
            if g is not None:
                grads[op[1]] = grads.get(op[1], 0.0) + up_back(g)
    return loss, pack(pgrads)


def param_count(ops=None):
    ops = ops or graph()
    return sum(op[4] * (9 * op[3] + 1) for op in ops if op[0] == "conv")
