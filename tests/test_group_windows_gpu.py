"""The parity suites again, with whole-window probing by groups of lanes.

Tables that fit in L2 probe whole windows with one key per lane by default
(wc_lane_ops); tables in DRAM use groups of lanes per window.  The parity
tests' tables are small, so this module re-collects the golden and table
tests with the lane kernel switched off, so that the group kernel keeps
being checked against the same oracle and fixtures on every operation."""
import pytest

import warpcore_b200 as wc
from tests.test_golden_gpu import *  # noqa: F401,F403  (re-collected below)
from tests.test_tables_gpu import *  # noqa: F401,F403

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _group_windows():
    prev = wc.set_lane_ops(0)
    yield
    wc.set_lane_ops(prev)


def test_lane_mask_round_trip():
    assert wc.set_lane_ops(0xD) == 0
    assert wc.set_lane_ops(0) == 0xD
