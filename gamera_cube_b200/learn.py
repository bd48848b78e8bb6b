"""Training of the learned ionosphere preconditioner (gcs_learn.cu).

A training triple is (conductance, field-aligned current, potential) on the
polar grid: the seeded conductance of the production case (Pedersen 2-20 S
with an auroral ridge, Hall = 1.5 Pedersen), a potential, and the FAC that
the conductance-tensor operator maps that potential to.  Potentials are
either random smooth fields (their FAC side is obtained by applying the
operator with the library's bitwise apply), or the solved potential of a
Region-1/2 FAC pattern.  The network is the flexible right preconditioner
of the learned solve: it learns the map from v = L A e (L the linear
two-level left preconditioner, at unit RMS) back to the potential e (in the
same units), with the conductance and geometry as extra input channels;
longitude rotations and sign flips augment the pool.
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


def scaled_operator(config, pedersen, hall):
    """The reduced conductance-tensor system with its rows scaled as in the
    learned solve (interior rows by sin(theta), the pole by ps / sqrt(np)):
    returns (A' as a scipy CSR matrix, ring prolongation E).  Stencil as
    nonorthogonal_mi.c:776-900."""
    import scipy.sparse as sp
    nt, npl = config.colatitude_count, config.longitude_count
    R, n = nt - 2, 1 + (nt - 2) * npl
    dth = config.maximum_colatitude / (nt - 1)
    dph = 2.0 * math.pi / npl
    th = dth * np.arange(nt)

    def inc2(a):
        c = np.cos(a)
        return 4.0 * c * c / (1.0 + 3.0 * c * c)

    cinc = config.hemisphere * 2.0 * np.cos(th) / np.sqrt(1.0 + 3.0 * np.cos(th) ** 2)
    P, H = pedersen, hall
    i = np.arange(1, nt - 1)[:, None]
    j = np.arange(npl)[None, :]
    jm, jp = (j - 1) % npl, (j + 1) % npl
    ti = th[i]
    lower = np.sin(ti - dth / 2) * 0.5 * (P[i, j] + P[i - 1, j]) / (inc2(ti - dth / 2) * dth * dth)
    upper = np.sin(ti + dth / 2) * 0.5 * (P[i, j] + P[i + 1, j]) / (inc2(ti + dth / 2) * dth * dth)
    llo = 0.5 * (P[i, j] + P[i, jm]) / (np.sin(ti) * dph * dph)
    lup = 0.5 * (P[i, j] + P[i, jp]) / (np.sin(ti) * dph * dph)
    f12 = -H / cinc[:, None]
    dft = (f12[i + 1, j] - f12[i - 1, j]) / (2.0 * dth)
    dfp = (f12[i, jp] - f12[i, jm]) / (2.0 * dph)
    s = np.sin(ti)
    q = 1 + (i - 1) * npl + j
    below = np.where(i == 1, 0, q - npl)
    entries = [(q, (lower + upper + llo + lup) / s), (below, (-lower - dfp / (2 * dth)) / s),
               (1 + (i - 1) * npl + jm, (-llo + dft / (2 * dph)) / s),
               (1 + (i - 1) * npl + jp, (-lup - dft / (2 * dph)) / s)]
    rows, cols, vals = [], [], []
    for c, v in entries:
        rows.append(np.broadcast_to(q, v.shape).ravel())
        cols.append(np.broadcast_to(c, v.shape).ravel())
        vals.append(v.ravel())
    upm = (i + 2 < nt) & np.ones_like(q, dtype=bool)
    rows.append(q[upm])
    cols.append((q + npl)[upm])
    vals.append(((-upper + dfp / (2 * dth)) / s)[upm])
    ppm = P[0].mean()
    pe = np.sin(0.5 * dth) * 0.5 * (ppm + P[1]) / (inc2(0.5 * dth) * dth * dth)
    ps = npl * (np.sin(0.5 * dth) * config.pedersen_siemens / (inc2(0.5 * dth) * dth * dth))
    s0 = ps / math.sqrt(npl)
    rows += [np.array([0]), np.zeros(npl, dtype=np.int64)]
    cols += [np.array([0]), 1 + np.arange(npl)]
    vals += [np.array([pe.sum() / s0]), -pe / s0]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    E = sp.csr_matrix((np.ones(n), (np.arange(n),
                                    np.concatenate([[0], 1 + np.repeat(np.arange(R), npl)]))),
                      shape=(n, R + 1))
    return A, E


def two_level(A, E, T, v, omega=0.7):
    """The learned solve's linear left preconditioner L v: a coarse
    correction on ring means, two damped Jacobi steps, the coarse correction
    again (as lp_left in gcs_learn.cu)."""
    D = A.diagonal()
    z = E @ T.solve(E.T @ v)
    for _ in range(2):
        z = z + omega * (v - A @ z) / D
    return z + E @ T.solve(E.T @ (v - A @ z))


def reduce(field):
    """Natural nt x np field -> reduced vector (pole, interior rows)."""
    return np.concatenate([[field[0, 0]], field[1:-1].ravel()])


def features(config, pedersen, hall):
    nt = config.colatitude_count
    theta = np.linspace(0.0, config.maximum_colatitude, nt)
    sp, sh = pedersen[1:nt - 1], hall[1:nt - 1]
    s = np.broadcast_to(np.sin(theta[1:nt - 1])[:, None], sp.shape)
    return np.stack([np.log(sp / 5.0), sh / sp, s]).astype(np.float32)


class Pool:
    """Training samples: inputs [4][R][np] (first channel unit RMS) and
    targets [R][np] (unit RMS)."""

    def __init__(self, lib, npl=361, nt=181, max_colatitude_deg=45.0, random_fields=384,
                 solved=16, conductances=16, seed=1234, hall_ratio=1.5):
        rng = np.random.default_rng(seed)
        self.npl, self.nt = npl, nt
        inputs, targets = [], []
        cond = [cases.mi_case(npl, nt, seed=seed + 17 * c, hall_ratio=hall_ratio,
                              max_colatitude_deg=max_colatitude_deg) for c in range(conductances)]
        self.triples = 0
        ops = {}
        for k in range(random_fields):
            case = cond[k % len(cond)]
            cfg = case.config
            if k % len(cond) not in ops:
                ops[k % len(cond)] = self._operator(case)
            e = smooth_potential(rng, nt, npl, cfg.maximum_colatitude)
            A, E, T = ops[k % len(cond)]
            self._add(inputs, targets, A, E, T, A @ reduce(e), reduce(e),
                      features(cfg, case.pedersen, case.hall))
        for k in range(solved):
            case = cases.mi_case(npl, nt, seed=seed + 1000 + k, hall_ratio=hall_ratio,
                                 max_colatitude_deg=max_colatitude_deg, max_iterations=20000)
            pot = case.potential.copy()
            st = abi.MiSolverStats()
            if lib.gamera_mi_solve_conductance_tensor(C.byref(case.config), _ptr(case.fac),
                                                      _ptr(case.pedersen), _ptr(case.hall),
                                                      _ptr(pot), C.byref(st)) != 0:
                raise RuntimeError(lib.gcs_last_error().decode())
            A, E, T = self._operator(case)
            e = reduce(pot)
            self._add(inputs, targets, A, E, T, A @ e, e,
                      features(case.config, case.pedersen, case.hall))
        self.inputs = np.stack(inputs)
        self.targets = np.stack(targets)

    @staticmethod
    def _operator(case):
        import scipy.sparse.linalg as spl
        A, E = scaled_operator(case.config, case.pedersen, case.hall)
        T = spl.splu((E.T @ A @ E).tocsc())
        return A, E, T

    def _add(self, inputs, targets, A, E, T, r, e, feat):
        """The pair the network sees as the right preconditioner of the
        learned solve: v = L r (L the two-level left preconditioner) at unit
        RMS, and the error e with L A e = v at unit RMS (a right
        preconditioner's output scale does not matter to flexible GMRES, and
        unit-RMS targets keep the training stable)."""
        v = two_level(A, E, T, r)
        sv = 1.0 / max(np.sqrt(np.mean(v * v)), 1e-300)
        se = 1.0 / max(np.sqrt(np.mean(e * e)), 1e-300)
        R, npl = self.nt - 2, self.npl
        vi = (sv * v[1:]).reshape(R, npl)
        ei = (se * e[1:]).reshape(R, npl)
        inputs.append(np.concatenate([vi[None].astype(np.float32), feat]))
        targets.append(ei.astype(np.float32))
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


def solve(lib, net, case, method=0, guess=None):
    """Learned-solve call for a case (method 0 two-level + network, 1 Jacobi,
    2 two-level); returns (rc, potential, stats, fallback, seconds)."""
    pot = (case.potential if guess is None else guess).copy()
    st = abi.MiSolverStats()
    fb = C.c_int()
    t = time.perf_counter()
    rc = lib.gcs_mi_solve_conductance_tensor_learned(
        net, method, C.byref(case.config), _ptr(case.fac), _ptr(case.pedersen), _ptr(case.hall),
        _ptr(pot), C.byref(st), C.byref(fb))
    return rc, pot, st, fb.value, time.perf_counter() - t
