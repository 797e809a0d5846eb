// Matcher internals used by the serving loop (server.cpp).
#pragma once

#include <cstddef>
#include <string>

#include "../../include/r3dgpu.h"

namespace r3dgpu {

// Checks a pair like r3dgpu_match_stereo_batch does (options, sizes, masks,
// output buffer); throws Error with the matcher's message.
void validate_request(const r3dgpu_pair& p);

// Upper bound of the SGM scratch of this thread's workspace (0: the default).
void set_thread_scratch_budget(size_t bytes);

// Message that r3dgpu_last_error returns on this thread.
void set_thread_error(const std::string& message);

}  // namespace r3dgpu
