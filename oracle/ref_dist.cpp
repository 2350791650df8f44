// Test infrastructure only.  Exposes the reference's L2 metric_distance
// (include/coresg/distance.hpp:307-312 -> l2sqr_avx2 :191-211, finalize std::sqrt)
// compiled with the reference's own flags, so the oracle's restated arithmetic can
// be pinned against the exact bits the reference produces.
#include <cstdint>

#include "coresg/distance.hpp"

extern "C" float refd_metric_distance_l2(const float* a, const float* b, std::uint32_t stride) {
    return coresg::metric_distance(coresg::MetricKind::L2, a, b, stride);
}

/// metric_distance for any of the reference's metrics (0 L2, 1 cosine on normalised
/// rows, 2 L1, 3 inner product), with the reference's flags.
extern "C" float refd_metric_distance(int metric, const float* a, const float* b, std::uint32_t stride) {
    return coresg::metric_distance(static_cast<coresg::MetricKind>(metric), a, b, stride);
}
