"""The statistics restatement (oracle/stats.py) against values from the
reference's own massPy / analysis code (tests/golden/gen_stats_golden.py)."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import stats as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "stats_*.npz")))


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_stats_restatement_matches_reference_post(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    st = {k: z[k] for k in z.files if k != "meta"}
    got = S.statistics(st, meta["LX"], meta["LY"])
    want = meta["stats"]
    for k, v in want.items():
        if isinstance(v, int) or k.startswith("defects"):
            assert got[k] == v, k
        else:
            assert got[k] == pytest.approx(v, rel=1e-12), k


def test_count_defects_periodic_clusters():
    w = np.zeros((6, 5))
    w[0, 0] = w[5, 0] = 0.5     # one cluster across the x wrap
    w[2, 2] = -0.5
    w[2, 3] = 0.5               # touching opposite signs stay separate
    w[4, 4] = w[4, 0] = -0.45   # one cluster across the y wrap
    assert S.count_defects(w) == (2, 2)
