// Kernel instantiation: bulk precision float, species count -1 (-1 = runtime).
#include "launch.cuh"
namespace ccb {
CCB_INSTANTIATE(float, -1)
}  // namespace ccb
