// Matvec kernel B (block multiply), complex128 instantiation.
#include "mv_column.cuh"

namespace msc {
template int launch_block_mul<double>(msc_plan*, double2*, const int*);
}  // namespace msc
