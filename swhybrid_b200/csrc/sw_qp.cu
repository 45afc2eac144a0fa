// Instantiations of the paired-query batched kernel (sw_qpair.cuh).
#include "sw_qpair.cuh"
#include "sw_registry.h"

namespace swb {
namespace {
template <int T, int R, int B>
constexpr QpKernel qinst() {
    return QpKernel{T, R, B, (const void*)&sw_qpbatch<T, R, B>, &qp_smem_bytes<T, R>};
}
}  // namespace

// block sizes as for the same shapes of the other first-pass kernels (no spills)
extern const QpKernel qp_table[] = {
    qinst<16, 64, 256>(), qinst<16, 48, 256>(), qinst<16, 32, 384>(), qinst<32, 32, 384>(),
    qinst<8, 64, 256>(),
};
extern const int qp_table_n = sizeof(qp_table) / sizeof(qp_table[0]);

const QpKernel* qp_kernels(int* n) {
    *n = qp_table_n;
    return qp_table;
}

}  // namespace swb
