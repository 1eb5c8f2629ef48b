// The opaque C-ABI context (include/ppc_b200.h): one Session per ppcb_ctx.
#pragma once
#include "session.h"

struct ppcb_ctx {
  ppcb::Session s;
};

#include <string>

// records the message returned by ppcb_last_error() (defined in capi.cpp)
void ppcb_internal_set_error(const std::string& msg);
