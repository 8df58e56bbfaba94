// Shared host-side helpers of libgg: status codes, thread-local error text.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/gg.h"

namespace gg {

void set_error(const char* fmt, ...);
const char* last_error();

// Return `code` after recording a formatted message.
int fail(int code, const char* fmt, ...);

#define GG_TRY_HOST(expr)         \
  do {                            \
    int r__ = (expr);             \
    if (r__ != GG_OK) return r__; \
  } while (0)

inline uint64_t mix64(uint64_t z) {
  // SplitMix64 output function (Steele, Lea & Flood, OOPSLA 2014).
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace gg
