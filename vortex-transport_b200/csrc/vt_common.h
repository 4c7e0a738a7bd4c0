// Shared host-side helpers for the C ABI: status messages, pointer checks and
// the decoding of the stage kernels' first-error key.
#pragma once

#include <cstdint>
#include <string>

#include "../../include/vortex_b200.h"

namespace vt {

// The device-array entry points read the caller's state arrays as double2
// (two doubles per 16-byte access); a pointer that is not 16-byte aligned
// (for example a view starting one double into an array) is rejected with
// VT_ERR_INVALID before any device work instead of faulting in a kernel.
inline bool aligned_to(const void* p, uintptr_t bytes) { return (reinterpret_cast<uintptr_t>(p) % bytes) == 0; }

// Decodes the stage kernels' first-error key
//   (stage epoch << 40) | (((element * nfq + point) * 3 + side) * 4 + code),
// epoch = 4 * step + stage (record_error, vt_device.cuh).
inline vt_error_info decode_error_key(unsigned long long key, int nfq) {
  vt_error_info info{};
  const unsigned long long epoch = key >> 40;
  unsigned long long local = key & ((1ull << 40) - 1);
  info.code = static_cast<int>(local & 3ull);
  local >>= 2;
  info.side = static_cast<int>(local % 3ull);
  local /= 3ull;
  info.point = static_cast<int>(local % static_cast<unsigned long long>(nfq));
  info.element = static_cast<int>(local / static_cast<unsigned long long>(nfq));
  info.step = static_cast<int64_t>(epoch / 4);
  info.stage = static_cast<int>(epoch % 4);
  return info;
}

// Records the message returned by vt_last_message() on this thread and passes
// the status through.
int fail(int status, const std::string& msg);
void clear_message();

}  // namespace vt
