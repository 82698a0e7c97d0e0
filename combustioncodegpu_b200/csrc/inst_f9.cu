// Kernel instantiation: bulk precision float, species count 9 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(float, 9)
}  // namespace ccb
