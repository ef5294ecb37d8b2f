// The lean search kernels for cosine (NormCosine) indices.
#include "lean_kernel.cuh"

namespace nmsg {
void* lean_kernel_cos(const DevIndex& ix) { return lean_kernel_select<1>(ix); }
}  // namespace nmsg
