// Force-included when the reference's src/main.cu is compiled here: its
// timestamp uses MSVC's localtime_s(tm*, const time_t*) (main.cu:29), which
// glibc spells localtime_r(const time_t*, tm*).
#pragma once
#include <ctime>

inline int localtime_s(std::tm* out, const std::time_t* t) {
  return localtime_r(t, out) ? 0 : 1;
}
