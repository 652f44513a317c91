#pragma once

#include "gpjson_b200.h"

namespace gpjson::detail {
// One engine context per process (created on first use on the current device).
gpj_ctx *engine_context();
}  // namespace gpjson::detail
