// Instantiations of k_step / k_run for the two-type pair-parameter path.
#include "md_kernels.cuh"

namespace gdb {
GDB_DEFINE_NT(nt2, 2)
}  // namespace gdb
