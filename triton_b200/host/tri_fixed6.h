// tri_fixed6.h -- the text printf("%.6f") gives for a double, without printf.
//
// The ASCII rasters (output_ascii.h:12-81 of the reference: fixed notation,
// six decimals) hold one such number per cell, 67 million per field at
// 8192^2, where the C library's formatter dominates the output time.  Here a
// finite v = m * 2^e is turned into N = round(v * 10^6) exactly in 128-bit
// integer arithmetic (m < 2^53 and 10^6 < 2^20, so m * 10^6 < 2^73), ties to
// even as glibc's printf rounds an exact decimal tie in the default rounding
// mode; the text is then the integer part of N / 10^6, a point and the six
// digits of N mod 10^6, with a minus sign for every value whose sign bit is
// set (printf gives "-0.000000" for -0.0 and for negatives that round to
// zero).  Values with N >= 2^64 (|v| above about 1.8e13), infinities and NaNs
// go to snprintf.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace trihost {

inline void append_fixed6_slow(std::string& out, double v) {
  char buf[512];
  const int n = std::snprintf(buf, sizeof(buf), "%.6f", v);
  out.append(buf, (size_t)n);
}

inline void append_fixed6(std::string& out, double v) {
  uint64_t bits;
  std::memcpy(&bits, &v, sizeof(bits));
  const bool neg = (bits >> 63) != 0;
  const int be = (int)((bits >> 52) & 0x7FF);
  uint64_t m = bits & ((1ull << 52) - 1);
  if (be == 0x7FF) return append_fixed6_slow(out, v);  // infinity or NaN
  int e;
  if (be == 0) {
    e = -1074;  // subnormal (or zero)
  } else {
    m |= 1ull << 52;
    e = be - 1075;
  }
  using u128 = unsigned __int128;
  const u128 p = (u128)m * 1000000u;  // v * 10^6 = p * 2^e exactly
  u128 n;
  if (e >= 0) {
    if (e > 54) return append_fixed6_slow(out, v);
    n = p << e;
  } else if (-e >= 128) {
    n = 0;  // p * 2^e < 2^-55: rounds to zero
  } else {
    const int sh = -e;
    u128 q = p >> sh;
    const u128 rem = p - (q << sh), half = (u128)1 << (sh - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    n = q;
  }
  if (n >> 64) return append_fixed6_slow(out, v);
  const uint64_t N = (uint64_t)n;
  uint64_t ip = N / 1000000u;
  uint32_t fp = (uint32_t)(N % 1000000u);
  char buf[32];
  int k = sizeof(buf);
  for (int i = 0; i < 6; i++) {
    buf[--k] = (char)('0' + fp % 10);
    fp /= 10;
  }
  buf[--k] = '.';
  do {
    buf[--k] = (char)('0' + ip % 10);
    ip /= 10;
  } while (ip);
  if (neg) buf[--k] = '-';
  out.append(buf + k, sizeof(buf) - (size_t)k);
}

}  // namespace trihost
