"""Failure detection on the host, without a GPU: a corrupted masked numbering
handed in from outside is caught by bp_ogs_check before any device work.

The numbering checked first is the reference's own (tests/golden/, written by
its mesh/ogs set-up), then copies with one entry broken in each way the check
names.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_hex_3x3x2_p5.npz")


@pytest.fixture(scope="module")
def numbering():
    g = np.load(GOLDEN)
    return g["GlobalToLocal"], g["rowStartsT"], g["colIdsT"], int(g["Ngather"][0])


def test_reference_numbering_passes(bp, numbering):
    g2l, rs, ci, ng = numbering
    bp.ogs_check(g2l, rs, ci, ng)
    g2l2, rs2, ci2 = bp.box_numbering(3, 3, 2, 5)
    bp.ogs_check(g2l2, rs2, ci2, ng)


def _broken(numbering, what):
    g2l, rs, ci, ng = (a.copy() if isinstance(a, np.ndarray) else a for a in numbering)
    if what == "row out of range":
        g2l[np.flatnonzero(g2l >= 0)[7]] = ng
    elif what == "below -1":
        g2l[3] = -2
    elif what == "moved node":
        l = np.flatnonzero(g2l >= 0)[11]
        g2l[l] = (g2l[l] + 1) % ng
    elif what == "masked node":
        g2l[np.flatnonzero(g2l >= 0)[5]] = -1
    elif what == "swapped columns":
        r = int(np.flatnonzero(np.diff(rs) >= 2)[0])
        ci[rs[r]], ci[rs[r] + 1] = ci[rs[r] + 1], ci[rs[r]]
    elif what == "empty row":
        rs[4] = rs[5]
    elif what == "first row start":
        rs[0] = 1
    return g2l, rs, ci, ng


@pytest.mark.parametrize("what,message", [
    ("row out of range", "outside \\[-1, Ngather"), ("below -1", "outside \\[-1, Ngather"),
    ("moved node", "is not a local node of row"), ("masked node", "unmasked entries"),
    ("swapped columns", "do not ascend"), ("empty row", "is empty"), ("first row start", "rowStarts\\[0\\]")])
def test_corrupted_numbering_is_rejected(bp, numbering, what, message):
    g2l, rs, ci, ng = _broken(numbering, what)
    with pytest.raises(bp.BPError, match=message) as e:
        bp.ogs_check(g2l, rs, ci, ng)
    assert e.value.code == bp.BP_ERROR_ARG
