// Instantiations of k_step / k_run for the general (up to 8 types) pair-parameter path.
#include "md_kernels.cuh"

namespace gdb {
GDB_DEFINE_NT(ntg, 0)
}  // namespace gdb
