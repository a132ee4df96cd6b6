// Declarations shared by the host-only translation units of libgbo.
#pragma once

#include <string>

#include "gbo.h"

namespace gbo {
int fail(int status, const std::string& msg);
void clear_error();
bool inject_host_alloc_fails();  // gbo_debug_inject(GBO_INJECT_HOST_ALLOC)

#define GBO_HOST_TRY(call)          \
  do {                              \
    int s_ = (call);                \
    if (s_ != GBO_OK) return s_;    \
  } while (0)

// Matrix Market banner and size line (host_io.cpp).
struct MtxHeader {
  bool symmetric = false;  // 'symmetric'
  bool hermitian = false;
  bool skew = false;
  bool pattern = false, real = false, integer = false, complex_ = false;
  int nrows = 0, ncols = 0;
  long long nnz = 0;
};
int parse_mtx_header(const char* p, const char* end, MtxHeader* h, const char** entries);
// GRB_UTIL_REMOVE_SELFLOOP (readMtx.hpp:155): drop self-loops unless set to 0.
bool env_remove_self_loops();
}  // namespace gbo
