// Sweep kernels for 256 lanes per simulation, in the three register budgets.
// Each group size has its own translation unit so the build compiles them in
// parallel.
#include "ctl_sweep_dev.cuh"

namespace ctl {
const void* sweep_kernel_g256(int minb) { return dev::sweep_kernel_ptr<256>(minb); }
}  // namespace ctl
