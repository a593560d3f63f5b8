// Minimal stand-in for the spdlog logger type used by the reference's logger
// header. Logging is off in the oracle build (BIPP_LOG_LEVEL unset), so these
// members are compiled but never reached.
#pragma once
#include <string_view>

namespace spdlog {
namespace level {
enum level_enum { trace, debug, info, warn, err, critical, off };
}
class logger {
public:
  template <typename... Args>
  void log(level::level_enum, std::string_view, Args&&...) {}
};
}  // namespace spdlog
