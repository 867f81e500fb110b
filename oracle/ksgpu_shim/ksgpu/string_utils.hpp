// Minimal stand-in for ksgpu's string helpers (TEST INFRASTRUCTURE ONLY; see Array.hpp).
#pragma once

#include <sstream>
#include <string>

namespace ksgpu {

// Human-readable byte count, e.g. "96.0 MB" (only used in the reference's str() methods).
inline std::string nbytes_to_str(long nbytes)
{
    const char *units[] = {"bytes", "KB", "MB", "GB", "TB"};
    double v = (double) nbytes;
    int u = 0;
    while ((v >= 1024.0) && (u < 4)) {
        v /= 1024.0;
        u++;
    }
    std::stringstream ss;
    ss.precision(1);
    ss << std::fixed << v << " " << units[u];
    return ss.str();
}

}  // namespace ksgpu
