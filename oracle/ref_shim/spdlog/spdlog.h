// Stand-in for spdlog (empty submodule in the reference tree): every log call is a no-op.
#pragma once
#include <memory>
namespace spdlog {
template <typename... A> inline void trace(A&&...) {}
template <typename... A> inline void debug(A&&...) {}
template <typename... A> inline void info(A&&...) {}
template <typename... A> inline void warn(A&&...) {}
template <typename... A> inline void error(A&&...) {}
struct logger { void flush() {} };
inline std::shared_ptr<logger> default_logger() { static auto l = std::make_shared<logger>(); return l; }
}  // namespace spdlog
