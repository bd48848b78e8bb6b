"""The analysis-frame restatement (oracle/analysis_oracle.py) pinned to the
reference: frames recorded through the reference library's own
gamera_no_conserved_to_primitive on a reference-built, reference-stepped
case (tests/golden/make_analysis_golden.py), against the restatement's frame
of the same case built and stepped by the CPU restatement (which equals the
reference bit for bit, tests/test_oracle.py).  Bitwise."""
import ctypes as C
import os

import numpy as np

from oracle import analysis_oracle, oracle_cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_analysis.npz")
GAMMA = 5.0 / 3.0


def restated_frames(case):
    out = []
    for f in range(6):
        a = case.arrays(f)
        n = int(np.prod(a["cell_magnetic"].shape[:3]))
        b0 = np.ctypeslib.as_array(C.cast(case.background[f].cell_magnetic,
                                          C.POINTER(C.c_double)),
                                   shape=(3 * n,)).reshape(a["cell_magnetic"].shape)
        out.append(analysis_oracle.frame(a["conserved"], a["cell_magnetic"], b0,
                                         case.ghost, GAMMA))
    return np.stack(out)


def test_restated_frame_equals_reference_golden():
    case = oracle_cases.Case("wind", 12, 10, 7)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    want = np.load(GOLDEN)["frames"]
    np.testing.assert_array_equal(restated_frames(case), want)
