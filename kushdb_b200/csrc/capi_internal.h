// Pieces of the extern "C" layer shared by the files that implement it
// (capi.cc, batch.cu, server.cc).
#pragma once

#include <string>

#include "../../include/kdb_b200.h"
#include "engine.h"

struct kdb_result {
  kdb::HostResult r;
};

kdb::Context* kdb_ctx_context(kdb_ctx* ctx);
void kdb_ctx_set_error(kdb_ctx* ctx, const std::string& msg);
