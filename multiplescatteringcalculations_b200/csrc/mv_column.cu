// Matvec kernel B (block multiply), complex64 instantiation.
#include "mv_column.cuh"

namespace msc {
template int launch_block_mul<float>(msc_plan*, float2*, const int*);
}  // namespace msc
