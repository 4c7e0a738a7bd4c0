// Shared host-side helpers for the C ABI: status messages.
#pragma once

#include <string>

namespace vt {

// Records the message returned by vt_last_message() on this thread and passes
// the status through.
int fail(int status, const std::string& msg);
void clear_message();

}  // namespace vt
