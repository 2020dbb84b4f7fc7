// Boost.StringAlgo is absent; the reference only calls replace_all on file names.
#pragma once
#include <string>
namespace boost {
inline void replace_all(std::string& s, const std::string& from, const std::string& to) {
  if (from.empty()) return;
  std::string::size_type p = 0;
  while ((p = s.find(from, p)) != std::string::npos) { s.replace(p, from.size(), to); p += to.size(); }
}
}
