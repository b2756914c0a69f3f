/* Minimal stand-in for glog's LOG()/CHECK() used when compiling the
 * reference's BSDF sources for the oracle cross-check: messages are dropped,
 * CHECK failures abort. */
#pragma once
#include <cstdlib>
#include <ostream>
#include <sstream>
namespace hk_glog_stub {
struct NullStream : std::ostringstream {};
struct CheckFail {
    ~CheckFail() { std::abort(); }
    template <class T> CheckFail &operator<<(const T &) { return *this; }
};
}
#define LOG(sev) hk_glog_stub::NullStream()
#define CHECK(c) if (c) {} else hk_glog_stub::CheckFail()
#define CHECK_EQ(a, b) CHECK((a) == (b))
#define CHECK_NE(a, b) CHECK((a) != (b))
#define CHECK_LT(a, b) CHECK((a) < (b))
#define CHECK_LE(a, b) CHECK((a) <= (b))
#define CHECK_GT(a, b) CHECK((a) > (b))
#define CHECK_GE(a, b) CHECK((a) >= (b))
#define DCHECK(c) CHECK(c)
template <class T> static inline T *hk_check_notnull(T *p) { if (!p) std::abort(); return p; }
#define CHECK_NOTNULL(p) hk_check_notnull(p)
