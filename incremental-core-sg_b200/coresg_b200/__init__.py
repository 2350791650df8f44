"""B200 engine for the CORE-SG hot path (NN-Descent, core distances, MRD
reweighting, per-mpts MST extraction, anti-hub bridges).

The compute lives in libcoresg_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/coresg_b200.h); this package is its Python binding plus the seeded
synthetic-data generator used by the tests and the benchmark.
"""
from ._abi import (CS_ERR_CUDA, CS_ERR_INVALID, CS_ERR_OOM, CS_ERR_STATE, CS_ERR_TIMEOUT,  # noqa: F401
                   CS_ERR_UNSUPPORTED, CS_METRIC_COSINE, CS_METRIC_L2, CS_OK, EDGE_DTYPE, LIB_PATH,
                   Context, CoreSG, CsError, MstResult, device_allocs, device_count, device_props, header_symbols, lib, write_edges_tsv,
                   write_labels_tsv)
from .serving import (CS_REQ_EPS_LABELS, CS_REQ_EXTRACT, CS_REQ_INSERT, Pinned, Server,  # noqa: F401,E402
                      request_stream)
