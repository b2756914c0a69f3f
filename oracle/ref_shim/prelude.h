/* Force-included when compiling the reference BSDF sources for the oracle
 * cross-check.  The reference targets MSVC: building with -DWIN32 selects its
 * Windows branches, whose CRT helpers are supplied here. */
#pragma once
#include <cmath>
#include <cstdint>
#include <type_traits>
static inline double _copysign(double a, double b) { return std::copysign(a, b); }
static inline unsigned char _BitScanReverse(unsigned long *idx, unsigned long v) {
    if (!v) return 0; *idx = 31u - (unsigned long)__builtin_clz((unsigned)v); return 1; }
static inline unsigned char _BitScanReverse64(unsigned long *idx, unsigned long long v) {
    if (!v) return 0; *idx = 63u - (unsigned long)__builtin_clzll(v); return 1; }
namespace std {
/* MSVC exposes the C float functions in namespace std; libstdc++ 13 does not. */
using ::sqrtf; using ::sinf; using ::cosf; using ::powf; using ::logf; using ::expf;
}
#include <cstdlib>
static inline void *_aligned_malloc(size_t size, size_t align) {
    void *p = nullptr; if (posix_memalign(&p, align < sizeof(void *) ? sizeof(void *) : align, size)) return nullptr; return p; }
static inline void _aligned_free(void *p) { free(p); }
