"""Regenerates the committed oracle fixtures of tests/golden/.

c1_muscl_ppm_fct.npz: the analytic dwarf configuration (20x20x10 doubly
periodic, the analytic driver's T field and flow, dt = 1000 s, valuesAB
frozen as in src/fesom_analytic.F90:335) advanced 10 steps with
MUSCL/PPM/FCT by the CPU oracle, with the reference's pre-remap
nod_in_elem2D rings.  The reference ships no run of these schemes
(lib/tracer_init_from_mesh.F90:172-174, src/fesom_analytic.F90:275-277 hard
code UPW1/UPW1/NONE), so this fixture pins the oracle against itself.

Usage: python tests/golden/make_fixtures.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import pyoracle  # noqa: E402


def main():
    o = pyoracle.Oracle()
    m = pyoracle.OracleMesh(o, 20, 20, 10, periodic=True, full_rings=False)
    T, S, uv, w = m.analytic_fields()
    TAB = T.copy(order="F")
    stats = []
    for _ in range(10):
        m.step(T, TAB, uv, w, 1000.0, "MUSCL", "PPM", "FCT")
        stats.append(m.stats(T))
    np.savez_compressed(Path(__file__).with_name("c1_muscl_ppm_fct.npz"), T_final=T, nsteps=10,
                        stats=np.array(stats))


if __name__ == "__main__":
    main()
