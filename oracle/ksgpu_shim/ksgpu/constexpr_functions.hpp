// Minimal stand-in for ksgpu's constexpr helpers (TEST INFRASTRUCTURE ONLY; see Array.hpp).
#pragma once

namespace ksgpu {

constexpr bool constexpr_is_log2(long n) { return (n > 0) && ((n & (n - 1)) == 0); }

}  // namespace ksgpu
