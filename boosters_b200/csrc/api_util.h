// api_util.h — the C ABI's shared error and configuration helpers, for entry
// points defined outside capi.cpp (noalloc.cu).
#pragma once
#include "../../include/boosters_c.h"

namespace bst {
// Sets the thread-local message bst_last_error() returns; returns `code`.
bst_status api_fail(bst_status code, const char* msg);
// GBDTConfig::validate (model/gbdt/config.rs:252-310) plus, for training,
// the engine's limits; sets the message on failure.
bst_status api_check_config(const bst_config* c, bool for_training);
void api_clear_error();
}  // namespace bst
