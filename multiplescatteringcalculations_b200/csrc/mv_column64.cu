// Matvec kernel B, complex128 instantiation.
#include "mv_column.cuh"

namespace msc {
template int launch_zfft_block<double>(msc_plan*, double2*, const double2*, const int*);
}  // namespace msc
