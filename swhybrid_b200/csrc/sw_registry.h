// sw_registry.h -- table of compiled first-pass kernel shapes.
#pragma once
#include <cstddef>

namespace swb {

struct WfKernel {
    int T;                         // threads per record pair
    int R;                         // query rows per thread
    int block;                     // threads per block
    const void* fn;                // __global__ sw_wavefront<T, R, block> (plain)
    size_t (*smem)(int qlen);      // shared-memory bytes for a query length
    const void* batch_fn;          // __global__ sw_batch<T, R, block> (batched)
};

// All instantiated shapes (sw_wf_t*.cu).
const WfKernel* wf_kernels(int* n);

// Paired-query batched kernel shapes (sw_qp.cu).
struct QpKernel {
    int T, R, block;
    const void* fn;                // __global__ sw_qpbatch<T, R, block>
    size_t (*smem)(int rows);      // shared memory for a double stack of `rows` rows
};
const QpKernel* qp_kernels(int* n);
const QpKernel* find_qp(int T, int R);     // null when that shape is not compiled

}  // namespace swb
