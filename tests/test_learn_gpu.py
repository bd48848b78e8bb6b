"""The learned preconditioner's network on the GPU against the CPU oracle
(oracle/learn_oracle.py, rounding to BF16 where the kernels do): forward
output, loss and every parameter gradient.  BF16 activations round
differently where the two accumulation orders straddle a rounding boundary,
so gradients agree to 2e-2 of each convolution's largest gradient and the
loss to 1e-2."""
import ctypes as C

import numpy as np
import pytest

from oracle import learn_oracle as lo

pytestmark = pytest.mark.gpu


def glib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def make_net(R, npl, batch, seed):
    L = glib()
    net = C.c_void_p()
    assert L.gcs_mi_net_create(R, npl, batch, seed, C.byref(net)) == 0, \
        L.gcs_last_error().decode()
    H0, W0, nparam, cin = (C.c_int() for _ in range(4))
    L.gcs_mi_net_info(net, C.byref(H0), C.byref(W0), C.byref(nparam), C.byref(cin))
    return net, H0.value, W0.value, nparam.value, cin.value


def get_params(net, n, gradients=0):
    out = np.zeros(n, dtype=np.float32)
    assert glib().gcs_mi_net_get_params(net, out.ctypes.data_as(C.POINTER(C.c_float)), n,
                                        gradients) == 0
    return out


def test_gradients_against_oracle():
    import torch
    L = glib()
    R, npl, B = 14, 30, 2
    net, H0, W0, nparam, cin = make_net(R, npl, B, 3)
    try:
        assert (H0, W0, cin) == (16, 32, 4)
        assert nparam == lo.param_count()
        rng = np.random.default_rng(5)
        params = get_params(net, nparam)
        # biases away from zero so that the ReLUs are active in both signs
        ops = lo.graph()
        o = 0
        for op in ops:
            if op[0] != "conv":
                continue
            cinl, coutl = op[3], op[4]
            for co in range(coutl):
                params[o + co * (9 * cinl + 1) + 9 * cinl] = rng.normal(scale=0.1)
            o += coutl * (9 * cinl + 1)
        assert L.gcs_mi_net_set_params(net, params.ctypes.data_as(C.POINTER(C.c_float)),
                                       nparam) == 0
        x = rng.normal(size=(B, cin, H0, W0)).astype(np.float32)
        target = rng.normal(size=(B, H0, W0)).astype(np.float32)
        xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(target).cuda()
        out = torch.zeros((B, H0, W0), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        assert L.gcs_mi_net_forward(net, C.c_void_p(xd.data_ptr()), B,
                                    C.c_void_p(out.data_ptr())) == 0
        loss = C.c_float()
        assert L.gcs_mi_net_train_step(net, C.c_void_p(xd.data_ptr()),
                                       C.c_void_p(td.data_ptr()), B, 0.0, 0,
                                       C.byref(loss)) == 0, L.gcs_last_error().decode()
        grads = get_params(net, nparam, gradients=1)
        torch.cuda.synchronize()
        pred = out.cpu().numpy()
    finally:
        L.gcs_mi_net_destroy(net)
    acts, _ = lo.forward(params, x, ops, bf16_mode=True)
    ref_pred = acts[max(acts)][:, 0]
    assert np.abs(pred - ref_pred).max() <= 2e-2 * np.abs(ref_pred).max()
    ref_loss, ref_grads = lo.loss_and_grads(params, x, target, R, npl, ops, bf16_mode=True)
    assert loss.value == pytest.approx(ref_loss, rel=1e-2)
    o = 0
    for op in ops:
        if op[0] != "conv":
            continue
        n = op[4] * (9 * op[3] + 1)
        g, r = grads[o:o + n], ref_grads[o:o + n]
        assert np.abs(g - r).max() <= 2e-2 * np.abs(r).max() + 1e-12, (op, np.abs(g - r).max(),
                                                                       np.abs(r).max())
        o += n


def test_training_reduces_loss():
    """Adam steps on a fixed batch lower the loss of a learnable map (the
    3x3 periodic box average of the first input channel): the training path
    runs end to end on the device."""
    import torch
    L = glib()
    R, npl, B = 22, 40, 4
    net, H0, W0, nparam, cin = make_net(R, npl, B, 9)
    try:
        rng = np.random.default_rng(2)
        xh = rng.normal(size=(B, cin, H0, W0)).astype(np.float32)
        first = xh[:, 0]
        th = sum(np.roll(np.roll(first, a, axis=-2), b, axis=-1)
                 for a in (-1, 0, 1) for b in (-1, 0, 1)) / 9.0
        x = torch.from_numpy(xh).cuda()
        t = torch.from_numpy(th.astype(np.float32)).cuda()
        torch.cuda.synchronize()
        losses = []
        for _ in range(80):
            loss = C.c_float()
            assert L.gcs_mi_net_train_step(net, C.c_void_p(x.data_ptr()),
                                           C.c_void_p(t.data_ptr()), B, 2e-3, 1,
                                           C.byref(loss)) == 0
            losses.append(loss.value)
    finally:
        L.gcs_mi_net_destroy(net)
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0]
