// Instantiations of k_step / k_run for the single-type pair-parameter path.
#include "md_kernels.cuh"

namespace gdb {
GDB_DEFINE_NT(nt1, 1)
}  // namespace gdb
