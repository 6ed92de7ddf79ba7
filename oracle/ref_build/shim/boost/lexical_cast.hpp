// Stand-in for boost::lexical_cast<T>(std::string) as used by the reference's
// Common/parameters.h:588 (string -> float component of a Vec).
#pragma once
#include <sstream>
#include <stdexcept>
#include <string>

namespace boost {
template <typename T>
T lexical_cast(const std::string& text) {
  std::istringstream in(text);
  T out{};
  in >> out;
  if (in.fail()) throw std::runtime_error("bad lexical_cast: " + text);
  return out;
}
}  // namespace boost
