/* Test infrastructure only: a plain-C restatement of the reference CPU algorithms on
 * the CORE-SG hot path, used as the correctness checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU baseline leg.  The product never
 * links or calls it.
 *
 * Each function cites the reference file:line it restates (paths relative to the
 * reference project root).  Pinned against the reference itself: tests/test_oracle.py
 * compares every function with the golden vectors in tests/golden/, which
 * tests/golden/make_golden.py produced by running the reference's own code
 * (oracle/ref_harness.cpp over the reference sources).
 */
#ifndef CORESG_ORACLE_H
#define CORESG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as coresg::Edge (include/coresg/types.hpp:20-33). */
typedef struct {
    uint32_t u;
    uint32_t v;
    float w;
} orc_edge;

/* Squared L2 in the association order of l2sqr_avx2 (include/coresg/distance.hpp:191-211). */
float orc_l2sqr(const float* a, const float* b, uint32_t stride);
/* MetricOp<L2>::finalize(rank) = IEEE sqrt (distance.hpp:259-265, :307-312). */
float orc_dist(const float* a, const float* b, uint32_t stride);

/* KnnGraph::core_dist for every node (include/coresg/knn_graph.hpp:157-163). */
void orc_core(const float* dists, const uint32_t* counts, uint32_t n, uint32_t k, uint32_t mpts,
              float* out);

/* collect_undirected / undirected_edges (src/knn_graph.cpp:132-200): node-major,
 * list order.  Returns the count; writes the edges when out != NULL. */
uint64_t orc_undirected(const uint32_t* ids, const float* dists, const uint32_t* counts,
                        uint32_t n, uint32_t k, orc_edge* out);

/* CoreSG::edges(mpts) (src/coresg.cpp:391-406, mutual_reachability_edges
 * src/knn_graph.cpp:219-235): k-NN edges reweighted, then bridges reweighted from
 * their base distance.  mpts 0 -> 1.  Returns the count. */
uint64_t orc_edges(uint32_t mpts, const uint32_t* ids, const float* dists, const uint32_t* counts,
                   uint32_t n, uint32_t k, const orc_edge* bridges, uint64_t n_bridges,
                   orc_edge* out);

/* Minimum spanning forest under the total order (float bits of w, edge index),
 * i.e. the order mst_boruvka selects by (src/mst.cpp:19-38, :79-151).  That order is
 * strict, so the forest is unique and equals the reference Boruvka's tree.
 * in_tree[m] (optional) marks chosen edges; labels[n] (optional) are the dense
 * component labels of UnionFind::labels (mst.cpp:48-59: numbered by first node).
 * exact_weight is the correctly rounded sum of the chosen weights. */
int orc_mst(const orc_edge* e, uint64_t m, uint32_t n, uint8_t* in_tree, uint32_t* labels,
            uint32_t* ncomp, uint64_t* nedges, double* exact_weight);

/* Kruskal under edge_less (w, u, v) (types.hpp:38-42, mst.cpp:61-77). */
int orc_mst_kruskal(const orc_edge* e, uint64_t m, uint32_t n, uint8_t* in_tree,
                    uint32_t* ncomp, uint64_t* nedges);

/* Correctly rounded double of the exact sum of `count` non-negative floats. */
double orc_exact_sum(const float* w, uint64_t count);

/* HubnessIndex::build reverse degrees (src/hubness.cpp:79-95). */
void orc_rdeg(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k, int32_t* rdeg);
/* compute_score, arithmetic mean (src/hubness.cpp:302-352). */
void orc_scores(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k,
                uint32_t k_for_score, const int32_t* rdeg, double* score);
/* antihub_budget (src/hubness.cpp:16-40). */
uint64_t orc_budget(uint32_t dim, uint64_t num_edges, uint32_t n, double multiplier,
                    double max_pair_ops, uint64_t min_selected, uint64_t max_selected);
/* HubnessIndex::select (src/hubness.cpp:424-521): budget lowest by (score, rdeg, id)
 * plus `per` lowest per component, sorted by the same order. */
uint64_t orc_select(const double* score, const int32_t* rdeg, uint32_t n, uint64_t budget,
                    const uint32_t* comp, uint32_t ncomp, uint32_t per, uint32_t* out);

/* ConnectivityTracker::rebuild + finalize (src/connectivity.cpp:24-79, :99-139). */
uint32_t orc_conn(const uint32_t* ids, const uint32_t* counts, uint32_t n, uint32_t k,
                  uint32_t* labels);

/* Dense MRD rows (src/cpu_backend.cpp:61-90) and Prim (src/mst.cpp:268-330). */
void orc_mrd_block(const float* pts, uint32_t m, uint32_t stride, const float* core, uint32_t r0,
                   uint32_t r1, float* out);
uint64_t orc_prim_dense(const float* mat, uint32_t m, orc_edge* out);

/* The bridge set of CoreSG::build for a given k-NN graph: connectivity, hubness,
 * selection, mst_over_subset with base distances, and repair_connectivity
 * (src/coresg.cpp:97-141, :355-470, :472-516; defaults of coresg.hpp:63-106 and
 * hubness.hpp:72-119).  Returns the edge count (writes at most `cap`). */
uint64_t orc_bridges(const float* padded, uint32_t n, uint32_t dim, uint32_t stride,
                     const uint32_t* ids, const float* dists, const uint32_t* counts, uint32_t k,
                     orc_edge* out, uint64_t cap, uint64_t* n_selected, uint64_t* n_repair);

/* Exact k nearest neighbours (rank space, ties by id) of the `nq` query nodes. */
void orc_brute_knn(const float* padded, uint32_t n, uint32_t stride, uint32_t k,
                   const uint32_t* queries, uint32_t nq, uint32_t* out_ids, float* out_dists);

#ifdef __cplusplus
}
#endif
#endif
