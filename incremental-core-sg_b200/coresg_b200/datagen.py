"""Seeded synthetic point sets with the shapes of the benchmark workloads.

A mixture of C isotropic Gaussians: centres uniform in [0, 10]^d, per-cluster
sigma log-uniform in [sigma_lo, sigma_hi], cluster of each point uniform, plus a
fraction of uniform noise over the bounding box of the clustered points; rows are
shuffled.  Everything is drawn from one numpy PCG64 stream, so a (shape, seed)
pair names the same float32 matrix on every machine.

The reference's own generator (make_blobs, src/io.cpp:151-179) draws centres from
N(0, separation^2) and sigma uniform in [0.15, 1.5]; the benchmark workloads use
the mixture above instead, and both the reference and this engine read the same
arrays, so the generator cannot drift between the two sides.
"""
from __future__ import annotations

import numpy as np

# Named workloads (points, dimension, clusters, sigma range, noise, k_max).
WORKLOADS = {
    # n=60,000 d=24, 20 clusters, sigma [0.2, 1.0], 5% noise, k_max=32
    "blobs60k_d24": dict(n=60_000, dim=24, clusters=20, sigma=(0.2, 1.0), noise=0.05, k_max=32, seed=20261204),
    # n=1,000,000 d=16, 50 clusters, sigma [0.2, 1.0], 5% noise, k_max=32
    "blobs1m_d16": dict(n=1_000_000, dim=16, clusters=50, sigma=(0.2, 1.0), noise=0.05, k_max=32, seed=20261205),
    # n=2,000,000 d=32, 100 clusters, sigma [0.1, 1.5], 3% noise, k_max=24
    "blobs2m_d32": dict(n=2_000_000, dim=32, clusters=100, sigma=(0.1, 1.5), noise=0.03, k_max=24, seed=20261206),
    # n=4,000,000 d=16, 200 clusters, sigma [0.2, 1.0], 5% noise, k_max=32
    "blobs4m_d16": dict(n=4_000_000, dim=16, clusters=200, sigma=(0.2, 1.0), noise=0.05, k_max=32, seed=20261207),
    # n=1,000,000 d=128, 100 clusters, sigma [0.5, 2.0], no noise, k_max=16
    "blobs1m_d128": dict(n=1_000_000, dim=128, clusters=100, sigma=(0.5, 2.0), noise=0.0, k_max=16, seed=20261208),
}


def gaussian_mixture(n: int, dim: int, clusters: int, sigma=(0.2, 1.0), noise: float = 0.05,
                     seed: int = 0, centres: np.ndarray | None = None) -> np.ndarray:
    """Return an (n, dim) float32 array drawn from the mixture described above.

    `centres` overrides the cluster centres (used to draw insertion batches from
    the clusters of an existing set)."""
    rng = np.random.default_rng(seed)
    if centres is None:
        centres = rng.uniform(0.0, 10.0, size=(clusters, dim))
    else:
        centres = np.asarray(centres, dtype=np.float64)
        clusters = centres.shape[0]
    lo, hi = np.log(sigma[0]), np.log(sigma[1])
    sig = np.exp(rng.uniform(lo, hi, size=clusters))
    n_noise = int(round(noise * n))
    n_clu = n - n_noise
    which = rng.integers(0, clusters, size=n_clu)
    pts = centres[which] + sig[which, None] * rng.standard_normal((n_clu, dim))
    if n_noise:
        lo_b = pts.min(axis=0) if n_clu else np.zeros(dim)
        hi_b = pts.max(axis=0) if n_clu else np.full(dim, 10.0)
        noise_pts = rng.uniform(lo_b, hi_b, size=(n_noise, dim))
        pts = np.concatenate([pts, noise_pts], axis=0)
    rng.shuffle(pts, axis=0)
    return np.ascontiguousarray(pts, dtype=np.float32)


def workload(name: str, n: int | None = None) -> tuple[np.ndarray, dict]:
    """Points of a named workload (optionally truncated/resized to `n` rows with
    the same mixture parameters) and its parameter dict."""
    w = dict(WORKLOADS[name])
    if n is not None:
        w["n"] = n
    pts = gaussian_mixture(w["n"], w["dim"], w["clusters"], w["sigma"], w["noise"], w["seed"])
    return pts, w


def quantize_u8(x: np.ndarray) -> np.ndarray:
    """uint8 variant of a float set: clamp(round(x*s + o), 0, 255) with s, o from
    the global range of x."""
    lo, hi = float(x.min()), float(x.max())
    s = 255.0 / (hi - lo) if hi > lo else 1.0
    return np.clip(np.rint((x - lo) * s), 0, 255).astype(np.uint8)


def pad_rows(x: np.ndarray) -> np.ndarray:
    """Zero-pad rows to a multiple of 8 floats (include/coresg/dataset.hpp:21)."""
    n, d = x.shape
    stride = (d + 7) & ~7
    if stride == d:
        return np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros((n, stride), dtype=np.float32)
    out[:, :d] = x
    return out


def workload_centres(w: dict) -> np.ndarray:
    """The cluster centres of a named workload's mixture (the first draw of its
    stream, as gaussian_mixture makes them)."""
    return np.random.default_rng(w["seed"]).uniform(0.0, 10.0, size=(w["clusters"], w["dim"]))


def insert_batch(w: dict, size: int, seed: int, new_clusters: int = 0) -> np.ndarray:
    """An insertion batch for workload `w`: drawn from its existing clusters, or
    from `new_clusters` fresh centres uniform in [0, 10]^d."""
    if new_clusters:
        return gaussian_mixture(size, w["dim"], new_clusters, w["sigma"], 0.0, seed)
    return gaussian_mixture(size, w["dim"], w["clusters"], w["sigma"], 0.0, seed, centres=workload_centres(w))
