// Minimal stand-in for glog, enough for the reference's PatchMatch kernels to
// compile as a checker. CHECK failures abort with a message.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
namespace smvs_ref_shim {
struct Fatal {
  std::ostringstream s;
  Fatal(const char* f, int l, const char* c) { s << f << ":" << l << " check failed: " << c << " "; }
  ~Fatal() { std::cerr << s.str() << std::endl; std::abort(); }
  template <typename T> Fatal& operator<<(const T& v) { s << v; return *this; }
};
struct Null { template <typename T> Null& operator<<(const T&) { return *this; } };
}
#define CHECK(c) if (c) {} else smvs_ref_shim::Fatal(__FILE__, __LINE__, #c)
#define CHECK_EQ(a, b) CHECK((a) == (b))
#define CHECK_NE(a, b) CHECK((a) != (b))
#define CHECK_LE(a, b) CHECK((a) <= (b))
#define CHECK_LT(a, b) CHECK((a) < (b))
#define CHECK_GE(a, b) CHECK((a) >= (b))
#define CHECK_GT(a, b) CHECK((a) > (b))
#define CHECK_NOTNULL(p) (p)
#define LOG(x) smvs_ref_shim::Null()
#define VLOG(x) smvs_ref_shim::Null()
#define DCHECK(c) CHECK(c)
#define DCHECK_EQ(a, b) CHECK_EQ(a, b)
#define DCHECK_LT(a, b) CHECK_LT(a, b)
#define DCHECK_GE(a, b) CHECK_GE(a, b)
