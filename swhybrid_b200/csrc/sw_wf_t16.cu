// First-pass kernel instantiations for groups of 16 thread(s) per record pair.
#include "sw_wavefront.cuh"
#include "sw_registry.h"

namespace swb {
namespace {
template <int R, int B>
constexpr WfKernel inst() {
    return WfKernel{16, R, B, (const void*)&sw_wavefront<16, R, B>, &wf_smem_bytes<16, R>};
}
}  // namespace

extern const WfKernel wf_table_t16[] = {
    inst<8, 768>(),  inst<16, 640>(), inst<24, 512>(), inst<32, 384>(),
    inst<40, 384>(), inst<48, 256>(), inst<56, 256>(), inst<64, 256>(),
};
extern const int wf_table_t16_n = sizeof(wf_table_t16) / sizeof(wf_table_t16[0]);

}  // namespace swb
