// Out-of-line members of the reference's Logger (src/logger.hpp:24-141) for the
// oracle build. The reference implementation (src/logger.cpp) needs spdlog,
// which is absent; logging stays off, so every member is a no-op here.
#include "logger.hpp"

namespace bipp {

Logger::Logger() {}

auto Logger::convert_level(BippLogLevel) -> spdlog::level::level_enum {
  return spdlog::level::off;
}

auto Logger::log_timings() -> void {}

auto Logger::log_matrix(BippLogLevel, const std::string_view&, std::size_t, std::size_t,
                        const float*, std::size_t) -> void {}
auto Logger::log_matrix(BippLogLevel, const std::string_view&, std::size_t, std::size_t,
                        const double*, std::size_t) -> void {}
auto Logger::log_matrix(BippLogLevel, const std::string_view&, std::size_t, std::size_t,
                        const std::complex<float>*, std::size_t) -> void {}
auto Logger::log_matrix(BippLogLevel, const std::string_view&, std::size_t, std::size_t,
                        const std::complex<double>*, std::size_t) -> void {}

Logger globLogger;

}  // namespace bipp
