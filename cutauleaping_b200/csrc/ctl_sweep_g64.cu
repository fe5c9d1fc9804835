// Sweep kernels for 64 lanes per simulation, in the three register budgets.
// Each group size has its own translation unit so the build compiles them in
// parallel.
#include "ctl_sweep_dev.cuh"

namespace ctl {
const void* sweep_kernel_g64(int minb) { return dev::sweep_kernel_ptr<64>(minb); }
}  // namespace ctl
