"""Writes the TSV golden files with the reference's own writers
(coresg::write_edges_tsv / write_labels_tsv, src/io.cpp:131-145) through the oracle
harness (oracle/_ref, built from the reference sources by oracle/Makefile).

    python tests/golden/make_tsv_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from checkers import EDGE_DTYPE, Reference  # noqa: E402


def tsv_cases():
    """Edges and labels covering the formatter's cases: zero, negative zero, a
    subnormal, the largest float, infinity, values needing all 9 digits, ids at the
    32-bit limit."""
    e = np.zeros(9, EDGE_DTYPE)
    e["u"] = [0, 2, 5, 8, 1, 3, 10, 4294967294, 12]
    e["v"] = [1, 3, 7, 9, 4, 6, 11, 4294967295, 13]
    e["w"] = np.array([0.0, -0.0, 1e-40, 3.4028235e38, np.inf, 0.1, 123456.789, 1.0, 2.5e-7], np.float32)
    lab = np.array([0, 5, 4294967295, 7, 1, 0], np.uint32)
    return e, lab


def main():
    e, lab = tsv_cases()
    ref = Reference()
    ref.write_edges_tsv(os.path.join(HERE, "tsv_edges.tsv"), e)
    ref.write_labels_tsv(os.path.join(HERE, "tsv_labels.tsv"), lab)


if __name__ == "__main__":
    main()
