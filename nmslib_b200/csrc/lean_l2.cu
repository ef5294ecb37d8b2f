// The lean search kernels for squared L2 (L2Sqr16Ext) indices.
#include "lean_kernel.cuh"

namespace nmsg {
void* lean_kernel_l2(const DevIndex& ix) { return lean_kernel_select<0>(ix); }
}  // namespace nmsg
