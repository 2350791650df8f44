"""The batched sweep's contracted tail (sweep.cu).  Once a Boruvka round's root list is
short, the next round (the table round) reduces every live (edge, MST) pair into an
(MST, root pair) -> lightest-key table, the table's entries make that round's offers,
and the rounds after it walk the entries instead of the edges.

On every reference fixture, against the reference's trees and the oracle:
* the tail never taken, taken at the earliest round (the table round is round 2),
  taken at the default point, and a table far too small for its entries (it
  overflows: the round walks its edges again and the sweep finishes on the edge
  worklist) all give the reference's trees, labels and weights bit for bit;
* the per-round trace (cs_sweep_trace, flag bits 1-2) shows which path each round
  took, so each setting is known to have run the path it names.
At n = 200,000 the same settings give the plain path's trees."""
import numpy as np
import pytest

import coresg_b200 as cs
from conftest import golden_names, load_golden
from test_extract_gpu import check_tree, resident

pytestmark = pytest.mark.gpu

WALK_EDGES, WALK_TABLE, WALK_TAIL = 0, 1, 2
DEFAULT = 0xFFFFFFFF
SETTINGS = {
    "never": (0, 0),
    "earliest": (1, 0),
    "default": (DEFAULT, 0),
    "overflow": (1, 1024),
}


def walks(g):
    """What phase A walked in each round of the last sweep's first pass."""
    return [int(t[5]) >> 1 for t in g.sweep_trace()]


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("setting", list(SETTINGS))
def test_tail_settings_match_reference(gpu_ctx, oracle, name, setting):
    z = load_golden(name)
    g = resident(gpu_ctx, z)
    g.set_sweep_tail(*SETTINGS[setting])
    n = len(z["counts"])
    mp = [int(m) for m in z["mpts"]]
    res = g.all_msts(mp)
    for m, r in zip(mp, res):
        e = oracle.edges(m, z["ids"], z["dists"], z["counts"], z["bridges"])
        check_tree(oracle, z, e, r, m, n)
    w = walks(g)
    if setting == "never":
        assert set(w) == {WALK_EDGES}
    elif setting == "earliest" and len(w) > 3:
        # the first round that may arm is round 1, so round 2 is the table round
        assert w[2] == WALK_TABLE and w.count(WALK_TABLE) == 1 and WALK_TAIL in w[3:]
    if setting == "overflow" and name == "coresg_n6000_d16_k32":
        # thousands of (MST, root pair) entries in a 1024-slot table: the table round
        # overflows and no round walks tail entries
        assert w[2] == WALK_TABLE and WALK_TAIL not in w


def test_tail_default_runs_on_the_largest_fixture(gpu_ctx):
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    g.all_msts([1, 8, 32])
    w = walks(g)
    assert w.count(WALK_TABLE) == 1 and WALK_TAIL in w


@pytest.mark.parametrize("setting", ["never", "earliest", "overflow"])
def test_tail_settings_match_plain_at_scale(gpu_ctx, setting):
    from coresg_b200.datagen import gaussian_mixture

    pts = gaussian_mixture(200_000, 16, 30, (0.2, 1.0), 0.05, seed=78)
    g = cs.CoreSG(gpu_ctx, 16, 32)
    g.build(pts)
    g.set_sweep_tail(*SETTINGS[setting])
    g.sweep_device(list(range(1, 33)))
    w = walks(g)
    if setting == "earliest":
        assert w[2] == WALK_TABLE and WALK_TAIL in w[3:]
    if setting == "overflow":
        assert w[2] == WALK_TABLE and WALK_TAIL not in w
    for m in (1, 2, 7, 16, 32):
        plain, swept = g.mst(m), g.sweep_fetch(m - 1)
        assert swept.edges.tobytes() == plain.edges.tobytes()
        assert np.array_equal(swept.component, plain.component) and swept.weight == plain.weight
