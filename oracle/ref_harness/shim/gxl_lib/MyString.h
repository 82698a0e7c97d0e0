// gxl string helpers stand-in (oracle build only), written from the call
// sites in BoundCond.cu, ChemData.cpp and Initialize.cu.
#pragma once
#include <algorithm>
#include <cctype>
#include <fstream>
#include <sstream>
#include <string>

namespace gxl {
enum class Case { lower, upper, keep };
inline void apply_case(std::string &s, Case c) {
  if (c == Case::lower) std::transform(s.begin(), s.end(), s.begin(), [](unsigned char ch) { return std::tolower(ch); });
  if (c == Case::upper) std::transform(s.begin(), s.end(), s.begin(), [](unsigned char ch) { return std::toupper(ch); });
}
inline std::istream &getline(std::ifstream &f, std::string &s, Case c = Case::keep) {
  std::getline(f, s);
  apply_case(s, c);
  return f;
}
inline void to_stringstream(const std::string &s, std::istringstream &line) {
  line.clear();
  line.str(s);
}
inline std::istream &getline_to_stream(std::ifstream &f, std::string &s, std::istringstream &line, Case c = Case::keep) {
  std::getline(f, s);
  apply_case(s, c);
  to_stringstream(s, line);
  return f;
}
inline void read_until(std::ifstream &f, std::string &s, const std::string &key, Case c = Case::keep) {
  while (std::getline(f, s)) {
    apply_case(s, c);
    if (s.rfind(key, 0) == 0) return;
  }
}
inline std::string to_upper(std::string s) {
  apply_case(s, Case::upper);
  return s;
}
inline void trim_left(std::string &s) {
  s.erase(s.begin(), std::find_if(s.begin(), s.end(), [](unsigned char ch) { return !std::isspace(ch); }));
}
}  // namespace gxl
