"""Generate the golden vectors of tests/golden/ from the unmodified reference.

Run in a container that has the reference sources (it builds
oracle/_ref/libgamera_ref.so from them):

    make -C oracle ref && python tests/golden/make_golden.py

For each case the script records, after each of a few reference steps, the
per-face sum, sum of absolute values and a fixed strided sample of every
state array.  The values come only from the reference library through the
reference's own public API; the CPU restatement and the CUDA library are
checked against them by tests/test_oracle.py and tests/test_step_parity.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import refbind  # noqa: E402

ARRAYS = ["conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic",
          "face_flux0", "face_flux1", "face_flux2", "old_face_flux0",
          "old_face_flux1", "old_face_flux2"]

# (name, kind, nr, n, steps, driver dt)
CASES = [("uniform", refbind.FX_UNIFORM, 0, 0, 2, False),
         ("shock", refbind.FX_SHOCK, 0, 0, 3, False),
         ("wind", refbind.FX_WIND, 12, 10, 2, True)]
SEED = 7
SAMPLES = 61


def sample_indices(size):
    return np.linspace(0, size - 1, SAMPLES).astype(np.int64)


def record(case, prefix, out):
    for f in range(6):
        arr = case.arrays(f)
        for name in ARRAYS:
            flat = np.ascontiguousarray(arr[name]).reshape(-1)
            key = "%s/f%d/%s" % (prefix, f, name)
            out[key + "/sum"] = np.array([flat.sum(), np.abs(flat).sum()])
            out[key + "/sample"] = flat[sample_indices(flat.size)]


def main():
    out = {}
    for name, kind, nr, n, steps, driver in CASES:
        case = refbind.Case(kind, nr, n, SEED)
        record(case, "%s/step0" % name, out)
        dt_prev = 0.0
        dts = []
        for s in range(steps):
            if driver:
                local = case.local_timestep()
                dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local,
                                                            1.25 * dt_prev)
                ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
            else:
                dt, ratio = case.dt, case.ratio
            assert case.step(ratio, dt) == 0
            dts.append((ratio, dt))
            dt_prev = dt
            record(case, "%s/step%d" % (name, s + 1), out)
        out["%s/dts" % name] = np.array(dts)
        case.close()
    path = os.path.join(HERE, "reference_steps.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
