"""FP32-bulk precision variant against the plain FP64 path.

`compare_bulk(lib, kind, nr, n, steps)` advances two copies of one
device-built case, the plain FP64 path and the FP32-bulk path, through the
same time levels: the FP64 copy runs the reference Earth driver's dt rule
on the device, and the FP32 copy replays each step's dt and predictor ratio
from it.  It returns, over the active cells, the maximum and RMS error of
every state variable relative to that variable's maximum magnitude, and the
maximum |div B| (face-flux divergence over the largest |face flux|) of both
copies.  `compare_bulk_sequential` does the same with one context on the
GPU at a time, for the largest cases.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .host import HostStorage

VARIABLES = ["rho", "mx", "my", "mz", "energy", "bx", "by", "bz"]


def _download(lib, ctx):
    act = (C.c_size_t * 3)()
    g = C.c_size_t()
    if lib.gcs_context_dims(ctx, act, C.byref(g)) != 0:
        raise RuntimeError("dims")
    hs = HostStorage(list(act), g.value)
    if lib.gcs_context_download_state(ctx, hs.storage, 0) != 0:
        raise RuntimeError("download")
    return hs, [act[0], act[1], act[2]], g.value


def div_b(hs, act, g):
    worst, scale = 0.0, 0.0
    I, J, K = (slice(g, g + act[0]), slice(g, g + act[1]), slice(g, g + act[2]))
    for f in range(6):
        a = hs.arrays(f)
        p0, p1, p2 = a["face_flux0"], a["face_flux1"], a["face_flux2"]
        dv = ((p0[g + 1:g + act[0] + 1, J, K] - p0[I, J, K]) +
              (p1[I, g + 1:g + act[1] + 1, K] - p1[I, J, K]) +
              (p2[I, J, g + 1:g + act[2] + 1] - p2[I, J, K]))
        worst = max(worst, float(np.abs(dv).max()))
        scale = max(scale, float(np.abs(p0).max()), float(np.abs(p1).max()),
                    float(np.abs(p2).max()))
    return worst / scale


def _errors(a, b, act, g):
    sl = (slice(g, g + act[0]), slice(g, g + act[1]), slice(g, g + act[2]))
    out = {}
    for q, name in enumerate(VARIABLES):
        arr, comp = ("conserved", q) if q < 5 else ("cell_magnetic", q - 5)
        dmax = smax = d2 = s2 = 0.0
        for f in range(6):
            x = a.arrays(f)[arr][sl][..., comp]
            y = b.arrays(f)[arr][sl][..., comp]
            dmax = max(dmax, float(np.abs(x - y).max()))
            smax = max(smax, float(np.abs(x).max()))
            d2 += float(((x - y) ** 2).sum())
            s2 += float((x ** 2).sum())
        out[name] = {"linf": dmax / smax if smax else 0.0,
                     "l2": (d2 / s2) ** 0.5 if s2 else 0.0}
    return out


def compare_bulk_sequential(lib, kind, nr, n, steps, seed=7, fraction=0.5,
                            b0_threshold=None, stream_time=None):
    """compare_bulk for cases too large for two contexts on one GPU
    (6 x 192x192x384: about 155 GB in FP64): the FP64 run goes first and
    records each step's dt and predictor ratio, its final state is copied to
    the host and the context released; then the FP32-bulk copy is built and
    replays the same time levels.  Also returns both runs' device time per
    step (CUDA events around the stepping loops, the FP64 loop including its
    per-step read-back of dt)."""
    import time
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(kind, C.byref(opts), C.byref(ts))
    ref = lib.gcs_context_create_case(kind, nr, n, seed)
    if not ref:
        raise RuntimeError(lib.gcs_last_error().decode())
    levels = []
    try:
        dt0 = C.c_double()
        if lib.gcs_context_timestep(ref, C.byref(ts), C.byref(dt0)) != 0:
            raise RuntimeError("timestep")
        dt, ratio = fraction * dt0.value, 0.0
        t0 = time.perf_counter()
        for step in range(steps):
            if step > 0:
                d, r = C.c_double(), C.c_double()
                lib.gcs_context_params(ref, C.byref(d), C.byref(r), None, None)
                dt, ratio = d.value, r.value
            levels.append((ratio, dt))
            if lib.gcs_context_run(ref, C.byref(opts), C.byref(ts), fraction, 1, 1) != 0 \
                    or lib.gcs_context_sync(ref) != 0:
                raise RuntimeError("FP64 step %d failed" % step)
        fp64_s = time.perf_counter() - t0
        a, act, g = _download(lib, ref)
        fp64_bytes = lib.gcs_context_device_bytes(ref)
    finally:
        lib.gcs_context_destroy(ref)
    bulk = lib.gcs_context_create_case(kind, nr, n, seed)
    if not bulk:
        raise RuntimeError(lib.gcs_last_error().decode())
    try:
        if b0_threshold is not None and \
                lib.gcs_context_set_bulk_threshold(bulk, b0_threshold) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        if lib.gcs_context_set_precision(bulk, 1) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        split = lib.gcs_context_bulk_split(bulk)
        lib.gcs_context_sync(bulk)
        t0 = time.perf_counter()
        for step, (ratio, dt) in enumerate(levels):
            if lib.gcs_context_step(bulk, C.byref(opts), ratio, dt) != 0:
                raise RuntimeError("FP32-bulk step %d failed" % step)
        if lib.gcs_context_sync(bulk) != 0:
            raise RuntimeError("FP32-bulk run failed")
        bulk_s = time.perf_counter() - t0
        b, _, _ = _download(lib, bulk)
        bulk_bytes = lib.gcs_context_device_bytes(bulk)
    finally:
        lib.gcs_context_destroy(bulk)
    out = {"steps": steps, "fp64_layers": split, "radial_layers": nr + 8,
           "div_b_fp64": div_b(a, act, g), "div_b_bulk": div_b(b, act, g),
           "fp64_ms_per_step_wall": fp64_s / steps * 1e3,
           "bulk_ms_per_step_wall": bulk_s / steps * 1e3,
           "fp64_device_bytes": fp64_bytes, "bulk_device_bytes": bulk_bytes}
    out.update(_errors(a, b, act, g))
    return out


def compare_bulk(lib, kind, nr, n, steps, seed=7, fraction=0.5, b0_threshold=None):
    opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
    lib.gcs_case_options(kind, C.byref(opts), C.byref(ts))
    ref = lib.gcs_context_create_case(kind, nr, n, seed)
    bulk = lib.gcs_context_create_case(kind, nr, n, seed)
    if not ref or not bulk:
        raise RuntimeError(lib.gcs_last_error().decode())
    try:
        if b0_threshold is not None and \
                lib.gcs_context_set_bulk_threshold(bulk, b0_threshold) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        if lib.gcs_context_set_precision(bulk, 1) != 0:
            raise RuntimeError(lib.gcs_last_error().decode())
        split = lib.gcs_context_bulk_split(bulk)
        dt0 = C.c_double()
        if lib.gcs_context_timestep(ref, C.byref(ts), C.byref(dt0)) != 0:
            raise RuntimeError("timestep")
        dt, ratio = fraction * dt0.value, 0.0
        for step in range(steps):
            if step > 0:
                d, r = C.c_double(), C.c_double()
                lib.gcs_context_params(ref, C.byref(d), C.byref(r), None, None)
                dt, ratio = d.value, r.value
            if lib.gcs_context_run(ref, C.byref(opts), C.byref(ts), fraction, 1, 1) != 0 \
                    or lib.gcs_context_sync(ref) != 0:
                raise RuntimeError("FP64 step %d failed" % step)
            if lib.gcs_context_step(bulk, C.byref(opts), ratio, dt) != 0:
                raise RuntimeError("FP32-bulk step %d failed" % step)
        a, act, g = _download(lib, ref)
        b, _, _ = _download(lib, bulk)
    finally:
        lib.gcs_context_destroy(ref)
        lib.gcs_context_destroy(bulk)
    out = {"steps": steps, "fp64_layers": split, "div_b_fp64": div_b(a, act, g),
           "div_b_bulk": div_b(b, act, g)}
    out.update(_errors(a, b, act, g))
    return out
