"""The extraction's TSV outputs (coresg::write_edges_tsv / write_labels_tsv,
src/io.cpp:131-145) written by the engine are byte-identical to the reference's:
against the committed files the reference wrote (tests/golden/make_tsv_golden.py)
and, when the reference is built here, against it live."""
import os

import numpy as np
import pytest

import coresg_b200 as cs
from checkers import Reference
from conftest import GOLDEN

from golden.make_tsv_golden import tsv_cases  # noqa: E402


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def test_edges_and_labels_match_the_reference_files(tmp_path):
    e, lab = tsv_cases()
    cs.write_edges_tsv(tmp_path / "e.tsv", e)
    cs.write_labels_tsv(tmp_path / "l.tsv", lab)
    assert _read(tmp_path / "e.tsv") == _read(os.path.join(GOLDEN, "tsv_edges.tsv"))
    assert _read(tmp_path / "l.tsv") == _read(os.path.join(GOLDEN, "tsv_labels.tsv"))


@pytest.mark.skipif(not Reference.available(), reason="reference not built (oracle/_ref)")
def test_random_edges_match_the_live_reference(tmp_path):
    rng = np.random.default_rng(3)
    e = np.zeros(5000, cs.EDGE_DTYPE)
    e["u"] = rng.integers(0, 1 << 32, size=len(e), dtype=np.uint64).astype(np.uint32)
    e["v"] = rng.integers(0, 1 << 32, size=len(e), dtype=np.uint64).astype(np.uint32)
    # every float bit pattern class: normal, subnormal, zero, inf, a wide exponent range
    e["w"] = (rng.random(len(e)) * 10.0 ** rng.integers(-45, 38, size=len(e))).astype(np.float32)
    lab = rng.integers(0, 1 << 32, size=3000, dtype=np.uint64).astype(np.uint32)
    ref = Reference()
    ref.write_edges_tsv(tmp_path / "re.tsv", e)
    ref.write_labels_tsv(tmp_path / "rl.tsv", lab)
    cs.write_edges_tsv(tmp_path / "e.tsv", e)
    cs.write_labels_tsv(tmp_path / "l.tsv", lab)
    assert _read(tmp_path / "e.tsv") == _read(tmp_path / "re.tsv")
    assert _read(tmp_path / "l.tsv") == _read(tmp_path / "rl.tsv")


def test_unwritable_path_is_an_error(tmp_path):
    with pytest.raises(cs.CsError, match="cannot write"):
        cs.write_edges_tsv(tmp_path / "missing" / "e.tsv", np.zeros(1, cs.EDGE_DTYPE))
