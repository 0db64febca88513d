// Fused z pass (forward FFT, block multiply, inverse FFT), complex128 instantiation.
#include "mv_zbz.cuh"

namespace msc {
template int launch_zbz<double>(msc_plan*, double2*, const int*, int);
}  // namespace msc
