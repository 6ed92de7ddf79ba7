// Minimal stand-in for the one boost::property_tree feature the reference's
// Common/parameters.h uses (parameters.h:92-119): a flat "Section.key" -> string
// map with typed get<T>(path, default).  Test infrastructure only: it lets the
// reference headers compile in this container, which has no Boost.
#pragma once
#include <map>
#include <sstream>
#include <string>

namespace boost { namespace property_tree {
class ptree {
 public:
  std::map<std::string, std::string> values;

  template <typename T>
  T get(const std::string& path, const T& fallback) const {
    auto it = values.find(path);
    if (it == values.end()) return fallback;
    std::istringstream in(it->second);
    T out{};
    in >> out;
    if (in.fail()) return fallback;
    return out;
  }
  // get<std::string>(path, "literal") in parameters.h:112-118
  template <typename T>
  T get(const std::string& path, const char* fallback) const {
    auto it = values.find(path);
    if (it == values.end()) return T(fallback);
    return it->second;
  }
};
}}  // namespace boost::property_tree
