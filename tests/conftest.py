import glob
import hashlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "incremental-core-sg_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_names(prefix="coresg_"):
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def load_golden(name):
    """A golden fixture plus its regenerated points (checked against the stored sha)."""
    from coresg_b200.datagen import gaussian_mixture, pad_rows

    z = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    n, dim, clusters, seed = (int(x) for x in z["spec"])
    pts = gaussian_mixture(n, dim, clusters, tuple(z["sigma"]), float(z["noise"]), seed=seed)
    assert hashlib.sha256(pts.tobytes()).digest() == z["points_sha"].tobytes(), "generator drifted"
    z["points"] = pts
    z["padded"] = pad_rows(pts)
    if "bridges" in z:
        from checkers import EDGE_DTYPE

        z["bridges"] = z["bridges"].view(EDGE_DTYPE)
    if "edges_full" in z:
        from checkers import EDGE_DTYPE

        z["edges_full"] = z["edges_full"].view(EDGE_DTYPE)
    return z


@pytest.fixture(scope="session")
def oracle():
    from checkers import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def gpu_ctx():
    import coresg_b200 as cs

    return cs.Context(0)


def edge_keys(e):
    return np.sort((e["u"].astype(np.uint64) << np.uint64(32)) | e["v"].astype(np.uint64))
