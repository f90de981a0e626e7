"""Seeded states for the sea-ice adjustment tests (icesnow.cpp:15-85): a
synthetic domain's AT with a band of surface water below the freezing point,
a patch of super-cooled water at every level (land columns included), values
at and one ulp either side of the freezing point, and a QICE field with ice
over warm and over cold water (used by the build without FRC_CORE, where
QICE carries over)."""
import numpy as np

TBICE = -1.8
# (frc_core, tracer steps before the adjustment, seed); a case with steps > 0
# runs the stepon.cpp:69-77 order tracer_ -> icesnow_ -> convadj_ (first step)
ICE_CASES = [(1, 0, 5), (0, 0, 6), (1, 2, 7), (0, 2, 8)]


def cold_state(inp, seed):
    rng = np.random.default_rng(seed)
    at = inp["AT"].copy()
    km, jmt, imt = at.shape[1:]
    south = slice(jmt - 16, jmt)          # j = 0 is the northern edge
    at[0, 0, south] = rng.uniform(-3.0, -0.5, size=(16, imt))
    at[0, km // 2:, 5:15, 3:12] = rng.uniform(-2.6, -1.6, size=(km - km // 2, 10, 9))
    edge = [TBICE, np.nextafter(TBICE, 0.0), np.nextafter(TBICE, -10.0), TBICE - 1e-12, TBICE + 1e-12]
    at[0, 0, 10, 5:5 + len(edge)] = edge
    at[0, 0, jmt - 10, 5:5 + len(edge)] = edge
    qice = np.zeros((jmt, imt))
    qice[4:20] = rng.uniform(0.0, 0.6, size=(16, imt))
    qice[jmt - 12:jmt - 4, : imt // 2] = rng.uniform(0.0, 0.3, size=(8, imt // 2))
    qice[rng.uniform(size=(jmt, imt)) < 0.2] = 0.0
    return at, qice
