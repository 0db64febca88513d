// Matvec kernel B, complex64 instantiation.
#include "mv_column.cuh"

namespace msc {
template int launch_zfft_block<float>(msc_plan*, float2*, const float2*, const int*);
}  // namespace msc
