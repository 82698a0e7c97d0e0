// Kernel instantiation: bulk precision double, species count 9 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(double, 9)
}  // namespace ccb
