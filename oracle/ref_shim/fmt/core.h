// Minimal stand-in for the fmt library's fmt::format, written for building the
// reference's hot-path sources as a test oracle (the reference's fmt submodule is not
// vendored).  Supports the placeholders those sources use: "{}", "{:.Nf}".
#pragma once
#include <cstdio>
#include <sstream>
#include <string>
#include <utility>

namespace fmt {
namespace detail {
inline void put(std::ostringstream& os, const std::string& spec, double v) {
  if (!spec.empty() && spec[0] == ':' && spec.size() > 2 && spec.back() == 'f') {
    char buf[64];
    std::snprintf(buf, sizeof(buf), ("%" + spec.substr(1)).c_str(), v);
    os << buf;
  } else {
    os << v;
  }
}
template <typename T> void put(std::ostringstream& os, const std::string&, const T& v) { os << v; }
inline void format_rest(std::ostringstream& os, const std::string& f, size_t pos) {
  os << f.substr(pos);
}
template <typename T, typename... Rest>
void format_rest(std::ostringstream& os, const std::string& f, size_t pos, const T& v,
                 Rest&&... rest) {
  size_t open = f.find('{', pos);
  if (open == std::string::npos) { os << f.substr(pos); return; }
  size_t close = f.find('}', open);
  os << f.substr(pos, open - pos);
  put(os, f.substr(open + 1, close - open - 1), v);
  format_rest(os, f, close + 1, std::forward<Rest>(rest)...);
}
}  // namespace detail
template <typename... Args> std::string format(const std::string& f, Args&&... args) {
  std::ostringstream os;
  detail::format_rest(os, f, 0, std::forward<Args>(args)...);
  return os.str();
}
}  // namespace fmt
