// No-op logging shim for building the reference hydro path without spdlog.
//
// The reference routes its log output through spdlog (ramses/utils/Logger.hpp,
// macros RAMSES_INFO and friends).  spdlog is fetched by CMake over the network,
// which is not reachable here, and logging does no arithmetic on the hydro
// path, so every macro here expands to nothing.  This header replaces the
// reference's Logger.hpp only inside the oracle build (oracle/_ref).
#ifndef RAMSES_LOGGER_HPP
#define RAMSES_LOGGER_HPP

namespace ramses {
class Logger {
public:
    static void init() {}
    static int get_rank() { return 0; }
};
}  // namespace ramses

#define RG_SHIM_NOLOG(...) do { } while (0)
#define RAMSES_TRACE(...) RG_SHIM_NOLOG()
#define RAMSES_DEBUG(...) RG_SHIM_NOLOG()
#define RAMSES_INFO(...) RG_SHIM_NOLOG()
#define RAMSES_WARN(...) RG_SHIM_NOLOG()
#define RAMSES_ERROR(...) RG_SHIM_NOLOG()
#define RAMSES_CRITICAL(...) RG_SHIM_NOLOG()
#define RAMSES_TRACE_ALL(...) RG_SHIM_NOLOG()
#define RAMSES_DEBUG_ALL(...) RG_SHIM_NOLOG()
#define RAMSES_INFO_ALL(...) RG_SHIM_NOLOG()
#define RAMSES_WARN_ALL(...) RG_SHIM_NOLOG()
#define RAMSES_ERROR_ALL(...) RG_SHIM_NOLOG()

#endif
