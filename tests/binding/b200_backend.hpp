// Test infrastructure: declarations of the reference-side binding of the engine
// (b200_backend.cpp), compiled against the reference's headers by oracle/Makefile.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "coresg/backend.hpp"
#include "coresg/coresg.hpp"
#include "coresg/mst.hpp"
#include "coresg_b200.h"

namespace coresg {

/// The engine as a coresg::Backend over the given CUDA device ordinals (one context,
/// i.e. one slot, per device); the branch a maintainer adds to make_backend
/// (src/backend.cpp:52-65) returns it.
std::unique_ptr<Backend> make_b200_backend(const std::vector<int>& ids);

/// The extraction hook of CoreSG::mst / all_msts: a resident device copy of a
/// CoreSG's k-NN arrays and bridges (sync after build, insert or load) and the
/// engine's extraction over it, with MstResult outputs.
class B200Extractor {
public:
    explicit B200Extractor(int device);
    ~B200Extractor();
    B200Extractor(const B200Extractor&) = delete;
    B200Extractor& operator=(const B200Extractor&) = delete;

    void sync(const CoreSG& sg);
    MstResult mst(std::uint32_t mpts) const;
    std::vector<MstResult> all_msts(const std::vector<std::uint32_t>& mpts) const;

private:
    void check(cs_status st, const char* what) const;
    cs_ctx* ctx_ = nullptr;
    cs_graph* dev_ = nullptr;
    std::size_t n_ = 0;
};

}  // namespace coresg
