// The reference's bblock::System with its 2-body/3-body terms forwarded to the
// C ABI of mbx_b200 (include/mbx_b200.h): the drop-in boundary exercised from
// the reference's own C++ code.
//
// Test infrastructure.  oracle/build_ref_gpu.py compiles the reference's
// bblock/system.cpp with -DMBX_GPU_2B3B after inserting, at the top of
// System::Get2B and System::Get3B (bblock/system.cpp:2425, 2769), a forward
// to System::GpuTerm (declared next to Get3B in a copy of bblock/system.h,
// system.h:1279), and links it with this file and libmbx_b200.so.  Everything
// else in System (SetPBC, the 1-body and electrostatic terms, the public
// TwoBodyEnergy/ThreeBodyEnergy entries at system.cpp:2403-2423, 2727-2745)
// is the reference's unmodified code.
//
// GpuTerm follows the contract of Get2B/Get3B: return the term's energy, add
// dE/dx into grad_ for real atoms and the virial into virial_.  The library
// context of each System lives in a table keyed by the object, so the class
// layout of System is unchanged.
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "bblock/system.h"
#include "mbx_b200.h"

namespace {
std::mutex g_mu;
std::map<const bblock::System*, mbx_ctx*> g_ctx;
}  // namespace

namespace bblock {

double System::GpuTerm(int nbody, bool do_grads, bool use_ghost) {
    mbx_ctx* ctx = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        auto it = g_ctx.find(this);
        if (it == g_ctx.end()) {
            if (mbx_create(&ctx, 0, nullptr) != MBX_OK)
                throw CUException(__func__, __FILE__, __LINE__, "mbx_create failed (no CUDA device?)");
            g_ctx[this] = ctx;
        } else {
            ctx = it->second;
        }
    }
    // topology: monomer ids in internal order, first site of every monomer,
    // the first atom's tag (what AddClusters compares) and the local flags
    std::vector<const char*> ids(nummon_);
    std::vector<int> first(nummon_), tag(nummon_), local(nummon_);
    for (size_t m = 0; m < nummon_; ++m) {
        ids[m] = monomers_[m].c_str();
        first[m] = (int)first_index_[m];
        tag[m] = atom_tag_[first_index_[m]];
        local[m] = (int)islocal_[m];
    }
    if (mbx_set_topology(ctx, (int)nummon_, ids.data(), first.data(), tag.data(), local.data(), (int)numsites_))
        throw CUException(__func__, __FILE__, __LINE__, mbx_last_error(ctx));
    std::vector<const char*> i2, i3;
    for (auto& t : ignore_2b_poly_)
        for (auto& s : t) i2.push_back(s.c_str());
    for (auto& t : ignore_3b_poly_)
        for (auto& s : t) i3.push_back(s.c_str());
    if (mbx_set_config(ctx, cutoff2b_, cutoff3b_, use_pbc_ ? box_.data() : nullptr, (int)ignore_2b_poly_.size(),
                       i2.data(), (int)ignore_3b_poly_.size(), i3.data()))
        throw CUException(__func__, __FILE__, __LINE__, mbx_last_error(ctx));
    double e = 0.0;
    // xyz_ is already wrapped by SetPBC; the library wraps it again (a no-op)
    if (mbx_energy(ctx, nbody, xyz_.data(), use_ghost ? 1 : 0, &e, do_grads ? grad_.data() : nullptr,
                   virial_.data(), do_grads ? 0 : MBX_NO_GRADS))
        throw CUException(__func__, __FILE__, __LINE__, mbx_last_error(ctx));
    return e;
}

}  // namespace bblock

// Releases the library context of a System (called by the harness before the
// System is deleted).
extern "C" void mbxref_gpu_release(const void* sys) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_ctx.find(static_cast<const bblock::System*>(sys));
    if (it != g_ctx.end()) {
        mbx_destroy(it->second);
        g_ctx.erase(it);
    }
}
