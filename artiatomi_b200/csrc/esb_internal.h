// Internal declarations shared by the translation units of libesb.
#pragma once

#include <string>

#include "../../include/esb.h"

namespace esb {

// Per-thread error message behind esb_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
inline int ok() { return ESB_OK; }

}  // namespace esb
