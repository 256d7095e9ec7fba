"""Converts the reference's golden membrane-potential traces into a fixture.

Source: test/lif_unit{1,2,3,4}_test_v.std of the BSim project — 1000 rows (one per
simulation cycle, dt = 0.1 ms) of 30 values printed with "%.10lf \\t" (the v of the
3x10 LIF_brian nets built in test/gpu/lif_unit{1..4}_test.cpp). The traces are kept
verbatim as float64 so that tests can compare at the printed precision.

Run:  python tests/golden/make_golden.py /path/to/BSim
"""
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    raise SystemExit("usage: make_golden.py <root of the BSim project>")
ref = sys.argv[1]
out = {}
for k in (1, 2, 3, 4):
    path = os.path.join(ref, "test", "lif_unit%d_test_v.std" % k)
    rows = [np.array(line.split(), dtype=np.float64) for line in open(path) if line.strip()]
    out["unit%d" % k] = np.stack(rows)
np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "lif_unit_v.npz"), **out)
print({k: v.shape for k, v in out.items()})
