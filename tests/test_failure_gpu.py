"""Failure detection without a GPU fault: a bounded device wait that runs out reports
DM_ETIMEOUT, and the context stays usable for the next call."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_clique_wait_times_out_then_recovers(dm, orc, gpu):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    with pytest.raises(dm.DMError) as e:
        dm.count_cliques(g, 4, dm.Options(test_flags=dm.TEST_STALL_AT_EXIT, timeout_ms=300))
    assert e.value.status == -7
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    assert dm.count_cliques(g, 4)[0] == orc.clique_dfs(og, 4)


def test_motif_wait_times_out_then_recovers(dm, orc, gpu):
    g = dm.Graph.load_edgelist(GOLDEN / "citeseer.edgelist")
    d = dm.Dictionary.generate(3)
    with pytest.raises(dm.DMError) as e:
        dm.count_motifs(g, 3, d, dm.Options(test_flags=dm.TEST_STALL_AT_EXIT, timeout_ms=300))
    assert e.value.status == -7
    og = orc.OracleGraph.load(GOLDEN / "citeseer.edgelist")
    got, _ = dm.count_motifs(g, 3, d)
    assert np.array_equal(got, orc.motifs(og, 3, d.tables()[0], d.n_classes))


def test_bad_options_rejected(dm, gpu):
    g = dm.Graph.load_edgelist(GOLDEN / "test.edgelist")
    for bad in (dm.Options(mode=9), dm.Options(rank=3, world_size=2), dm.Options(vwarp=5),
                dm.Options(scheduler=dm.SCHED_LEARNED)):
        with pytest.raises(dm.DMError) as e:
            dm.count_cliques(g, 3, bad)
        assert e.value.status == -1
