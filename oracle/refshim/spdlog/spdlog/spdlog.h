// Logging stub used only to compile the reference sources as a parity oracle
// (TEST INFRASTRUCTURE): every spdlog call the reference makes is a no-op.
#ifndef ICEMPM_SPDLOG_STUB
#define ICEMPM_SPDLOG_STUB
namespace spdlog {
template <typename... A> inline void info(A &&...) {}
template <typename... A> inline void warn(A &&...) {}
template <typename... A> inline void error(A &&...) {}
template <typename... A> inline void critical(A &&...) {}
template <typename... A> inline void debug(A &&...) {}
}  // namespace spdlog
#endif
