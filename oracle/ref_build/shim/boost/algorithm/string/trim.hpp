// Stand-in for boost::algorithm::trim(std::string&) as used by the reference's
// Common/parameters.h:587.
#pragma once
#include <string>

namespace boost { namespace algorithm {
inline void trim(std::string& s) {
  const char* ws = " \t\r\n";
  const auto b = s.find_first_not_of(ws);
  if (b == std::string::npos) { s.clear(); return; }
  const auto e = s.find_last_not_of(ws);
  s = s.substr(b, e - b + 1);
}
}}  // namespace boost::algorithm
