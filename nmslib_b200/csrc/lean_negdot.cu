// The lean search kernels for negative dot product indices.
#include "lean_kernel.cuh"

namespace nmsg {
void* lean_kernel_negdot(const DevIndex& ix) { return lean_kernel_select<2>(ix); }
}  // namespace nmsg
