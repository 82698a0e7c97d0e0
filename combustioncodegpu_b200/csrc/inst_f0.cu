// Kernel instantiation: bulk precision float, species count 0 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(float, 0)
}  // namespace ccb
