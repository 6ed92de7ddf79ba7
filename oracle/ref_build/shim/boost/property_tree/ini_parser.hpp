// Minimal INI reader standing in for boost::property_tree::ini_parser::read_ini
// as used by the reference's Common/parameters.h:94.  "[Section]" headers and
// "key = value" lines become "Section.key" entries; ';' and '#' start comments.
#pragma once
#include <fstream>
#include <stdexcept>
#include <string>
#include "ptree.hpp"

namespace boost { namespace property_tree { namespace ini_parser {
inline std::string shim_trim(const std::string& s) {
  const char* ws = " \t\r\n";
  const auto b = s.find_first_not_of(ws);
  if (b == std::string::npos) return "";
  const auto e = s.find_last_not_of(ws);
  return s.substr(b, e - b + 1);
}
inline void read_ini(const std::string& file_name, ptree& tree) {
  std::ifstream in(file_name);
  if (!in) throw std::runtime_error("cannot open INI file " + file_name);
  std::string line, section;
  while (std::getline(in, line)) {
    line = shim_trim(line);
    if (line.empty() || line[0] == ';' || line[0] == '#') continue;
    if (line.front() == '[' && line.back() == ']') {
      section = shim_trim(line.substr(1, line.size() - 2));
      continue;
    }
    const auto eq = line.find('=');
    if (eq == std::string::npos) continue;
    tree.values[section + "." + shim_trim(line.substr(0, eq))] = shim_trim(line.substr(eq + 1));
  }
}
}}}  // namespace boost::property_tree::ini_parser
