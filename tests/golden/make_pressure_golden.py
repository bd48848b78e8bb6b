"""Golden vectors of the post-step pressure control
(nonorthogonal_step.c:74-171) from the unmodified reference.

Run in a container that has the reference sources:

    make -C oracle ref && python tests/golden/make_pressure_golden.py

On the reference's wind case (12 radial x 10 x 10 cells per face, seed 7)
after one reference step, with parameters that make both branches fire
(tests/pressure_util.py), the script records the counts, the maxima and,
per face, the sums and a strided sample of the controlled conserved array.
tests/test_pressure_host.py checks the oracle against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import refbind  # noqa: E402
from tests import pressure_util as pu  # noqa: E402
from tests.golden.make_golden import sample_indices  # noqa: E402


def main():
    case = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    act = list(case.active)
    light, thr, low_sound = pu.parameters([case.arrays(f) for f in range(6)], case.ghost, act)
    rc, low, hot, ms, mp = pu.apply_faces(case.lib.gamera_no_apply_pressure_control,
                                          case.storage, case.grid, case.ghost, act, pu.DT,
                                          light, thr, low_sound)
    assert rc == 0 and low > 0 and hot > 0
    out = {"params": np.array([light, thr, low_sound, pu.DT]),
           "counts": np.array([low, hot]), "maxima": np.array([ms, mp])}
    for f in range(6):
        flat = np.ascontiguousarray(case.arrays(f)["conserved"]).reshape(-1)
        out["f%d/sum" % f] = np.array([flat.sum(), np.abs(flat).sum()])
        out["f%d/sample" % f] = flat[sample_indices(flat.size)]
    np.savez_compressed(os.path.join(HERE, "reference_pressure.npz"), **out)
    print("low %d hot %d of %d cells" % (low, hot, 6 * act[0] * act[1] * act[2]))


if __name__ == "__main__":
    main()
