// Library-wide error message for failures that have no engine handle
// (lbm_create, handle-free entry points); lbm_last_error(NULL) returns it.
#pragma once

#include <string>

namespace lbm {
void set_global_error(const std::string& msg);
}
