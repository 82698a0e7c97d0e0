// gxl::Time stand-in (oracle build only).
#pragma once
namespace gxl {
struct Time {
  double step_time = 0, elapsed_time = 0;
  void get_elapsed_time() {}
};
}  // namespace gxl
