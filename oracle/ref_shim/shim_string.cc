// StringPrintf for the reference's util/cudacc.cc (its util/string.cc needs boost).
#include <cstdarg>
#include <cstdio>
#include <string>
namespace sensemap {
std::string StringPrintf(const char* format, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, format);
  vsnprintf(buf, sizeof(buf), format, ap);
  va_end(ap);
  return std::string(buf);
}
}  // namespace sensemap
