// The test hook of lbx_test_fault (include/lbx.h), shared by the library's translation units.
#pragma once

namespace lbx {

struct TestFault {
  int kind = 0;   // lbx_test_fault_kind
  int param = 0;  // poll limit of the made-to-fail wait, or allocations left to fail
};

TestFault& test_fault();       // the process-wide setting (lbx_api.cu)
bool test_allocation_fails();  // true (and one failure used up) when an allocation is to fail

}  // namespace lbx
