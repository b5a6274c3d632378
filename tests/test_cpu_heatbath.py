"""KAT-5: the oracle's restatement of the reference's pseudo-heatbath (phbup / su2up /
sprd1 G/heatbath.f90:33-467 with the staples of G/gaugetools.f90:39-345, in the order of
C/cfgsprops.f90 sweep :1973-2001) reproduces its committed record: the plaquette after
each of 200 sweeps on 8^4 at beta = 6.0 from a cold start with lagfib seed (0, 7),
bit for bit.  The links stay in SU(3) to rounding."""
import json
from pathlib import Path

import numpy as np

import oracle

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())


def test_kat5_heatbath_reproduces_record():
    rec = GOLDEN["kat5_heatbath"]
    ol = oracle.OracleLattice(*rec["dims"], bc=(1, 1, 1, -1))
    u = ol.coldstart()
    oracle.initlagfib(0, rec["iseed"])
    plaq = ol.heatbath(u, rec["beta"], len(rec["plaquette"]))
    assert np.array_equal(plaq, np.array(rec["plaquette"]))
    nv = ol.nvhalf
    m = u.reshape(16, 2, 4, ol.ntotal, 18)[..., :nv, :]
    m = (m[..., 0::2] + 1j * m[..., 1::2]).reshape(-1, 3, 3)
    assert np.abs(m @ np.conj(np.swapaxes(m, -1, -2)) - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(m) - 1).max() < 1e-13
