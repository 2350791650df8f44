"""Host logic that the benchmark workloads and the serving leg rest on, on the CPU:
the seeded mixtures (one seed, one matrix), the parameters of every named workload,
row padding and the uint8 quantisation, insertion batches drawn from a workload's
own clusters or from new ones, and the serving request stream (Poisson arrivals
inside the window, the request mix, the mpts range, log-uniform insert sizes, one
stream per seed)."""
import numpy as np
import pytest

from coresg_b200 import datagen
from coresg_b200.serving import CS_REQ_EPS_LABELS, CS_REQ_EXTRACT, CS_REQ_INSERT, percentile, request_stream


def test_mixture_is_reproducible():
    a = datagen.gaussian_mixture(4000, 16, 10, seed=3)
    b = datagen.gaussian_mixture(4000, 16, 10, seed=3)
    c = datagen.gaussian_mixture(4000, 16, 10, seed=4)
    assert a.dtype == np.float32 and a.shape == (4000, 16) and a.flags.c_contiguous
    assert a.tobytes() == b.tobytes()
    assert a.tobytes() != c.tobytes()


def test_mixture_noise_share_and_box():
    """Without noise every row lies near a centre; with 20 % noise (uniform over the
    clustered rows' bounding box) about that share lies far from every centre."""
    centres = np.random.default_rng(9).uniform(0.0, 10.0, size=(5, 8))
    x = datagen.gaussian_mixture(3000, 8, 5, sigma=(0.1, 0.1), noise=0.0, seed=9, centres=centres)
    d = np.min(np.linalg.norm(x[:, None, :].astype(np.float64) - centres[None], axis=2), axis=1)
    assert np.quantile(d, 0.99) < 0.1 * 8 ** 0.5 * 2.5  # chi(8) tail at sigma 0.1
    y = datagen.gaussian_mixture(3000, 8, 5, sigma=(0.1, 0.1), noise=0.2, seed=9, centres=centres)
    far = np.min(np.linalg.norm(y[:, None, :].astype(np.float64) - centres[None], axis=2), axis=1) > 1.0
    assert 0.15 < far.mean() < 0.21  # the 20 % noise rows, bar the few that land near a centre


@pytest.mark.parametrize("name,n,dim,clusters,k_max", [
    ("blobs60k_d24", 60_000, 24, 20, 32),
    ("blobs1m_d16", 1_000_000, 16, 50, 32),
    ("blobs2m_d32", 2_000_000, 32, 100, 24),
    ("blobs4m_d16", 4_000_000, 16, 200, 32),
    ("blobs1m_d128", 1_000_000, 128, 100, 16),
])
def test_named_workloads(name, n, dim, clusters, k_max):
    w = datagen.WORKLOADS[name]
    assert (w["n"], w["dim"], w["clusters"], w["k_max"]) == (n, dim, clusters, k_max)
    pts, w2 = datagen.workload(name, n=700)
    assert pts.shape == (700, dim) and w2["n"] == 700 and w2["dim"] == dim
    again, _ = datagen.workload(name, n=700)
    assert pts.tobytes() == again.tobytes()


def test_workload_parameters_of_the_insert_and_highdim_sets():
    w = datagen.WORKLOADS["blobs2m_d32"]
    assert w["sigma"] == (0.1, 1.5) and w["noise"] == 0.03
    w = datagen.WORKLOADS["blobs1m_d128"]
    assert w["sigma"] == (0.5, 2.0) and w["noise"] == 0.0


def test_pad_rows():
    x = np.arange(3 * 20, dtype=np.float32).reshape(3, 20)
    p = datagen.pad_rows(x)
    assert p.shape == (3, 24) and np.array_equal(p[:, :20], x) and not p[:, 20:].any()
    y = np.ones((2, 16), np.float32)
    assert datagen.pad_rows(y).shape == (2, 16)


def test_quantize_u8():
    x = np.linspace(-3.0, 5.0, 1000, dtype=np.float32).reshape(100, 10)
    q = datagen.quantize_u8(x)
    assert q.dtype == np.uint8 and q.min() == 0 and q.max() == 255
    flat = q.reshape(-1)
    assert np.all(np.diff(flat.astype(np.int32)) >= 0)  # order kept
    # at d = 128 every partial sum of squared uint8 differences is an integer below
    # 2^24, so a float32 sum in any order is the exact integer distance
    rng = np.random.default_rng(2)
    a = rng.integers(0, 256, size=(64, 128)).astype(np.int64)
    b = rng.integers(0, 256, size=(64, 128)).astype(np.int64)
    exact = ((a - b) ** 2).sum(axis=1)
    f32 = ((a.astype(np.float32) - b.astype(np.float32)) ** 2).astype(np.float32)
    seq = np.zeros(64, np.float32)
    for j in range(128):
        seq = (seq + f32[:, j]).astype(np.float32)
    assert np.array_equal(seq.astype(np.int64), exact)
    assert np.array_equal(f32.sum(axis=1, dtype=np.float32).astype(np.int64), exact)
    worst = np.full(128, 255, np.float32) ** 2
    assert float(worst.sum(dtype=np.float32)) == 128 * 255 ** 2


def test_insert_batches():
    w = datagen.WORKLOADS["blobs2m_d32"]
    centres = datagen.workload_centres(w)
    old = datagen.insert_batch(w, 2000, seed=5)
    new = datagen.insert_batch(w, 1500, seed=5, new_clusters=10)
    assert old.shape == (2000, 32) and new.shape == (1500, 32)
    assert old.tobytes() == datagen.insert_batch(w, 2000, seed=5).tobytes()
    # rows from the existing clusters lie near the workload's centres (sigma <= 1.5)
    d = np.min(np.linalg.norm(old[:, None, :].astype(np.float64) - centres[None], axis=2), axis=1)
    assert np.median(d) < 1.5 * 32 ** 0.5 * 1.2


def test_request_stream_mix_and_ranges():
    s = request_stream(20.0, 200.0, 32, seed=11)
    assert s == request_stream(20.0, 200.0, 32, seed=11)
    t = np.array([a.t for a in s])
    assert np.all(np.diff(t) > 0) and t[0] > 0 and t[-1] < 20.0
    assert abs(len(s) - 4000) < 4 * 4000 ** 0.5  # Poisson count
    kinds = np.array([a.kind for a in s])
    ins = kinds == CS_REQ_INSERT
    assert abs(ins.mean() - 0.10) < 0.02
    q = ~ins
    cuts = (kinds == CS_REQ_EPS_LABELS)[q]
    assert abs(cuts.mean() - 0.25) < 0.03
    assert set(kinds) <= {CS_REQ_INSERT, CS_REQ_EXTRACT, CS_REQ_EPS_LABELS}
    mp = np.array([a.mpts for a in s if a.kind != CS_REQ_INSERT])
    assert mp.min() == 1 and mp.max() == 32
    sizes = np.array([a.size for a in s if a.kind == CS_REQ_INSERT])
    assert sizes.min() >= 1_000 and sizes.max() <= 100_000
    # log-uniform: the median is near the geometric mean of the bounds
    assert 10 ** 3.6 < np.median(sizes) < 10 ** 4.4
    qs = np.array([a.quantile for a in s if a.kind == CS_REQ_EPS_LABELS])
    assert qs.min() >= 0.0 and qs.max() < 1.0


def test_percentile():
    xs = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert percentile(xs, 50) == 3.0
    assert percentile(xs, 99) == pytest.approx(float(np.percentile(xs, 99)))
    assert percentile([], 50) is None
