"""Training of the learned ionosphere preconditioner (gcs_learn.cu).

A training triple is (conductance, field-aligned current, potential) on the
polar grid: the seeded conductance of the production case (Pedersen 2-20 S
with an auroral ridge, Hall = 1.5 Pedersen), a potential, and the FAC that
the conductance-tensor operator maps that potential to.  Potentials are
either random smooth fields (their FAC side is obtained by applying the
operator with the library's bitwise apply), or the solved potential of a
Region-1/2 FAC pattern.  The network learns the map from the (row-scaled,
unit-RMS) residual to the (unit-RMS) potential correction, with the
conductance and geometry as extra input channels; longitude rotations and
sign flips augment the pool.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import abi, cases

P = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(P)


def smooth_potential(rng, nt, npl, max_colatitude):
    """Random multi-scale potential: pole value single-valued, zero at the
    low-latitude boundary."""
    theta = np.linspace(0.0, max_colatitude, nt)[:, None]
    phi = (2.0 * math.pi / npl) * np.arange(npl)[None, :]
    x = theta / max_colatitude
    e = np.zeros((nt, npl))
    for m in range(0, int(rng.integers(4, 24))):
        for q in range(1, int(rng.integers(2, 8))):
            amp = rng.normal() / (1.0 + m + q) ** rng.uniform(0.5, 1.5)
            prof = np.sin(math.pi * q * x + rng.uniform(0, 2 * math.pi)) * (1.0 - x)
            if m > 0:
                prof = prof * np.sin(np.minimum(x, 0.5) * math.pi) ** min(m, 3)
            e += amp * prof * np.cos(m * phi + rng.uniform(0, 2 * math.pi))
    for _ in range(int(rng.integers(0, 6))):
        t0, p0 = rng.uniform(0.1, 0.9), rng.uniform(0, 2 * math.pi)
        wt, wp = rng.uniform(0.02, 0.15), rng.uniform(0.05, 0.6)
        dp = np.angle(np.exp(1j * (phi - p0)))
        e += rng.normal() * np.exp(-((x - t0) / wt) ** 2 - (dp / wp) ** 2)
    e[-1] = 0.0
    e[0] = e[0].mean()
    return e * 1e3


def features(config, pedersen, hall):
    nt = config.colatitude_count
    theta = np.linspace(0.0, config.maximum_colatitude, nt)
    sp, sh = pedersen[1:nt - 1], hall[1:nt - 1]
    s = np.broadcast_to(np.sin(theta[1:nt - 1])[:, None], sp.shape)
    return np.stack([np.log(sp / 5.0), sh / sp, s]).astype(np.float32)


class Pool:
    """Training samples: inputs [4][R][np] (residual channel unit RMS) and
    targets [R][np] (unit RMS)."""

    def __init__(self, lib, npl=361, nt=181, max_colatitude_deg=45.0, random_fields=384,
                 solved=16, conductances=16, seed=1234):
        rng = np.random.default_rng(seed)
        self.npl, self.nt = npl, nt
        inputs, targets = [], []
        cond = [cases.mi_case(npl, nt, seed=seed + 17 * c,
                              max_colatitude_deg=max_colatitude_deg) for c in range(conductances)]
        self.triples = 0
        for k in range(random_fields):
            case = cond[k % len(cond)]
            cfg = case.config
            e = smooth_potential(rng, nt, npl, cfg.maximum_colatitude)
            ap = np.zeros_like(e)
            if lib.gamera_mi_apply_conductance_tensor(C.byref(cfg), _ptr(case.pedersen),
                                                      _ptr(case.hall), _ptr(e), _ptr(ap)) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            self._add(inputs, targets, ap[1:nt - 1], e[1:nt - 1],
                      features(cfg, case.pedersen, case.hall))
        for k in range(solved):
            case = cases.mi_case(npl, nt, seed=seed + 1000 + k,
                                 max_colatitude_deg=max_colatitude_deg, max_iterations=20000)
            pot = case.potential.copy()
            st = abi.MiSolverStats()
            if lib.gamera_mi_solve_conductance_tensor(C.byref(case.config), _ptr(case.fac),
                                                      _ptr(case.pedersen), _ptr(case.hall),
                                                      _ptr(pot), C.byref(st)) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            th = np.linspace(0.0, case.config.maximum_colatitude, nt)[1:nt - 1]
            c = np.cos(th)
            inc = case.config.hemisphere * 2.0 * c / np.sqrt(1.0 + 3.0 * c * c)
            u = -(case.config.ionosphere_radius_m ** 2) * case.fac[1:nt - 1] * inc[:, None]
            self._add(inputs, targets, u, pot[1:nt - 1],
                      features(case.config, case.pedersen, case.hall))
        self.inputs = np.stack(inputs)
        self.targets = np.stack(targets)

    def _add(self, inputs, targets, r, e, feat):
        r = r / max(np.sqrt(np.mean(r * r)), 1e-300)
        e = e / max(np.sqrt(np.mean(e * e)), 1e-300)
        inputs.append(np.concatenate([r[None].astype(np.float32), feat]))
        targets.append(e.astype(np.float32))
        self.triples += 1

    def batch(self, rng, B, H0, W0):
        """B augmented samples on the padded grid: random longitude rotation
        and sign; periodic continuation in the padding columns."""
        R, npl = self.nt - 2, self.npl
        x = np.zeros((B, 4, H0, W0), dtype=np.float32)
        t = np.zeros((B, H0, W0), dtype=np.float32)
        cols = np.arange(W0) % npl
        for b in range(B):
            k = int(rng.integers(len(self.inputs)))
            sh = int(rng.integers(npl))
            sg = 1.0 if rng.random() < 0.5 else -1.0
            xi = np.roll(self.inputs[k], sh, axis=-1)
            ti = np.roll(self.targets[k], sh, axis=-1)
            x[b, :, :R] = xi[:, :, cols]
            x[b, 0, :R] *= sg
            t[b, :R] = sg * ti[:, cols]
        return x, t


def train(lib, net, pool, steps=2000, batch=8, lr=1e-3, seed=7, log_every=0):
    """Adam with cosine decay on augmented pool batches; returns the losses."""
    import torch
    H0, W0 = C.c_int(), C.c_int()
    lib.gcs_mi_net_info(net, C.byref(H0), C.byref(W0), None, None)
    rng = np.random.default_rng(seed)
    losses = []
    t0 = time.perf_counter()
    for it in range(steps):
        x, t = pool.batch(rng, batch, H0.value, W0.value)
        xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
        torch.cuda.synchronize()
        rate = lr * 0.5 * (1.0 + math.cos(math.pi * it / steps))
        loss = C.c_float()
        if lib.gcs_mi_net_train_step(net, C.c_void_p(xd.data_ptr()), C.c_void_p(td.data_ptr()),
                                     batch, rate, 1, C.byref(loss)) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        losses.append(loss.value)
        if log_every and (it % log_every == 0 or it == steps - 1):
            print("step %5d loss %.4f  %.1fs" % (it, loss.value, time.perf_counter() - t0),
                  flush=True)
    return losses


def create_net(lib, config, batch=8, seed=3):
    net = C.c_void_p()
    if lib.gcs_mi_net_create(config.colatitude_count - 2, config.longitude_count, batch, seed,
                             C.byref(net)) != 0:
        raise RuntimeError(lib.gcs_last_error().decode())
    return net


def solve(lib, net, case, guess=None):
    """Learned (net) or Jacobi (net None) FGMRES solve of a case; returns
    (rc, potential, stats, fallback, seconds)."""
    pot = (case.potential if guess is None else guess).copy()
    st = abi.MiSolverStats()
    fb = C.c_int()
    t = time.perf_counter()
    rc = lib.gcs_mi_solve_conductance_tensor_learned(
        net, C.byref(case.config), _ptr(case.fac), _ptr(case.pedersen), _ptr(case.hall),
        _ptr(pot), C.byref(st), C.byref(fb))
    return rc, pot, st, fb.value, time.perf_counter() - t
