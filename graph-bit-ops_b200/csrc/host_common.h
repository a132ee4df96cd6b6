// Declarations shared by the host-only translation units of libgbo.
#pragma once

#include <string>

#include "gbo.h"

namespace gbo {
int fail(int status, const std::string& msg);
void clear_error();
}  // namespace gbo
