// Minimal stand-in for boost::filesystem (declarations the reference headers touch).
#pragma once
#include <string>
namespace boost { namespace filesystem {
class path {
 public:
  path() {}
  path(const std::string& s) : s_(s) {}
  path(const char* s) : s_(s) {}
  path operator/(const path& o) const { return path(s_ + "/" + o.s_); }
  std::string string() const { return s_; }
 private:
  std::string s_;
};
}}
