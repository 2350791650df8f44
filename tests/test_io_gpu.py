"""CORESG01 interoperability with the reference's CoreSG::save / CoreSG::load
(src/io.cpp:195-330): a file written by the engine loads in the reference and
vice versa, with identical state and identical extractions."""
import os

import numpy as np
import pytest

import coresg_b200 as cs
from checkers import Reference
from conftest import edge_keys, load_golden

pytestmark = pytest.mark.gpu


def test_engine_save_load_roundtrip(gpu_ctx, tmp_path):
    z = load_golden("coresg_n3000_d24_k16")
    g = cs.CoreSG(gpu_ctx, 24, 16)
    g.set_points(z["points"])
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    path = str(tmp_path / "a.coresg")
    g.save(path)
    h = cs.CoreSG.load(gpu_ctx, path)
    for a, b in zip(g.knn(), h.knn()):
        assert np.array_equal(a, b)
    assert h.missing_edges().tobytes() == z["bridges"].tobytes()
    assert np.array_equal(edge_keys(h.mst(8).edges), z["mst_keys_8"])


@pytest.mark.skipif(not Reference.available(), reason="reference not built (oracle/_ref)")
def test_files_interoperate_with_the_reference(gpu_ctx, tmp_path):
    z = load_golden("coresg_n6000_d16_k32")
    ref = Reference()
    # reference -> engine
    sg = ref.from_state(z["padded"], 16, z["ids"], z["dists"], z["flags"], z["counts"], z["bridges"])
    p1 = str(tmp_path / "ref.coresg")
    sg.save(p1)
    g = cs.CoreSG.load(gpu_ctx, p1)
    ids, dists, flags, counts = g.knn()
    assert np.array_equal(ids, z["ids"]) and np.array_equal(dists.view(np.uint32), z["dists"].view(np.uint32))
    assert np.array_equal(counts, z["counts"])
    assert g.missing_edges().tobytes() == z["bridges"].tobytes()
    r = g.all_msts([3, 16])
    assert np.array_equal(edge_keys(r[0].edges), z["mst_keys_3"])
    assert np.array_equal(edge_keys(r[1].edges), z["mst_keys_16"])
    # engine -> reference: byte-identical file
    p2 = str(tmp_path / "eng.coresg")
    g.save(p2)
    assert open(p1, "rb").read() == open(p2, "rb").read()
    back = ref.lib.ref_load(p2.encode(), 4)
    assert back
    ref.lib.ref_free(back)


def test_sweep_results_straight_to_tsv(gpu_ctx, tmp_path):
    """cs_sweep_write_tsv writes a sweep's tree and labels from the device in the
    reference's TSV formats: the same bytes as the host writers (pinned to the
    reference's own writers by test_tsv.py) on the fetched results."""
    z = load_golden("coresg_n3000_d24_k16")
    g = cs.CoreSG(gpu_ctx, int(z["dim"]), int(z["k"]))
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    mp = [2, 8, 16]
    res = g.all_msts(mp)
    for j, r in enumerate(res):
        g.write_sweep_tsv(j, tmp_path / f"e{j}.tsv", tmp_path / f"l{j}.tsv")
        cs.write_edges_tsv(tmp_path / f"he{j}.tsv", r.edges)
        cs.write_labels_tsv(tmp_path / f"hl{j}.tsv", r.component)
        assert (tmp_path / f"e{j}.tsv").read_bytes() == (tmp_path / f"he{j}.tsv").read_bytes()
        assert (tmp_path / f"l{j}.tsv").read_bytes() == (tmp_path / f"hl{j}.tsv").read_bytes()
    g.write_sweep_tsv(0, tmp_path / "only_edges.tsv", None)
    assert (tmp_path / "only_edges.tsv").read_bytes() == (tmp_path / "he0.tsv").read_bytes()
