// Prints TopOpt::StepOut's Output.txt entry (TopOpt.cpp:386-401) through
// the C++ mirror for fixed values, for comparison with the Python log.
#include <cstdio>
#include <vector>

#include "topopt_b200.hpp"

int main() {
  tpo::Compliance c({1.0}, 0.0, 1.0, true);
  tpo::Volume v({0.3}, 0.0, 1.0, false);
  c.value = 12.3456789;
  v.value = -0.00123456789012345;
  std::vector<tpo::Function_Base *> fns = {&c, &v};
  tpo::StepOut(stdout, 12.3456789, {-0.00123456789012345, 0.5}, 7, fns);
  return 0;
}
