// Fused z pass (forward FFT, block multiply, inverse FFT), complex64 instantiation.
#include "mv_zbz.cuh"

namespace msc {
template int launch_zbz<float>(msc_plan*, float2*, const int*, int);
}  // namespace msc
