"""GPU anti-hub bridges against the reference: on the reference's own k-NN graph
the selected anti-hubs (order included), the bridge edges with base distances, the
repair count and the k-NN component count are identical; cs_mrd_block equals the
reference's dense MRD rows bit for bit."""
import numpy as np
import pytest

import coresg_b200 as cs
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names())
def test_bridges_match_reference(gpu_ctx, name):
    z = load_golden(name)
    g = cs.CoreSG(gpu_ctx, int(z["dim"]), int(z["k"]))
    g.set_points(z["points"])
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    st = g.select_bridges()
    assert st["knn_components"] == int(z["ncomp_knn"])
    assert np.array_equal(g.selected(), z["selected"])
    assert st["repair"] == int(z["repair"])
    assert g.missing_edges().tobytes() == z["bridges"].tobytes()


def test_mrd_block_matches_oracle(gpu_ctx, oracle):
    z = load_golden("coresg_n2000_d40_k10")
    sel = z["selected"][:200]
    pts = z["padded"][sel]
    core = oracle.core(z["dists"], z["counts"], int(z["k"]))[sel]
    for r0, r1 in ((0, 200), (17, 91)):
        got = gpu_ctx.mrd_block(pts, core, r0, r1)
        want = oracle.mrd_block(pts, core, r0, r1)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_full_build_on_device(gpu_ctx, oracle):
    """CoreSG::build end to end on the device: NN-Descent, then bridges; the bridges
    equal the oracle's bridge computation on the device-built k-NN graph."""
    z = load_golden("coresg_n3000_d24_k16")
    g = cs.CoreSG(gpu_ctx, 24, 16)
    st = g.build(z["points"])
    ids, dists, flags, counts = g.knn()
    br, nsel, nrep = oracle.bridges(z["padded"], 24, ids, dists, counts)
    assert st["selected"] == nsel and st["repair"] == nrep
    assert g.missing_edges().tobytes() == br.tobytes()
