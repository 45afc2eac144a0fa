// First-pass kernel instantiations for groups of 32 threads per record pair.
#include "sw_wavefront.cuh"
#include "sw_registry.h"

namespace swb {
namespace {
template <int R, int B>
constexpr WfKernel inst() {
    return WfKernel{32, R, B, (const void*)&sw_wavefront<32, R, B>, &wf_smem_bytes<32, R>,
                    (const void*)&sw_batch<32, R, B>};
}
}  // namespace

// rows per thread R (any even number; the two half-columns hold R/2 rows
// each) and the block size that leaves every shape register room without
// spilling (block sizes are multiples of 128 threads)
extern const WfKernel wf_table_t32[] = {
    inst<4, 768>(),  inst<6, 768>(),  inst<8, 768>(),  inst<10, 640>(), inst<12, 640>(),
    inst<16, 640>(), inst<20, 512>(), inst<24, 512>(), inst<28, 384>(), inst<32, 384>(),
    inst<40, 384>(), inst<48, 256>(), inst<56, 256>(), inst<64, 256>(),
};
extern const int wf_table_t32_n = sizeof(wf_table_t32) / sizeof(wf_table_t32[0]);

}  // namespace swb
