// Shared host helpers: status propagation, exact FP64->FP16 rounding, the CPython
// random.Random generator the reference planner is defined with.
#pragma once

#include <sys/mman.h>

#include <cstdint>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/trajsparsenufft.h"

namespace tsn {

// Error carried through the host library and turned into a tsn_status at the C boundary.
struct Error : std::runtime_error {
  tsn_status status;
  Error(tsn_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

[[noreturn]] inline void fail(tsn_status s, const std::string& what) { throw Error(s, what); }

void set_last_error(const std::string& text);

// Size a large host vector to n elements, asking the kernel for transparent huge pages before
// the first touch (multi-GB planner arrays otherwise fault in 4 KB at a time, which costs
// minutes of system time on virtualized hosts). Advisory: without THP it is a plain resize.
template <class T>
void resize_huge(std::vector<T>& v, size_t n) {
  if (n * sizeof(T) >= (size_t(64) << 20) && v.capacity() < n) {
    std::vector<T>().swap(v);
    v.reserve(n);
    const uintptr_t a = reinterpret_cast<uintptr_t>(v.data());
    const uintptr_t lo = (a + 0x1FFFFF) & ~uintptr_t(0x1FFFFF);
    const uintptr_t hi = (a + n * sizeof(T)) & ~uintptr_t(0x1FFFFF);
    if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_HUGEPAGE);
  }
  v.resize(n);
}

// Round an IEEE binary64 value to binary16, round-to-nearest-even, directly from the
// double bits (numpy's float64 -> float16 cast, used by compress_tile at
// src/export_gpu_case.py:52 and compress_tiles_vectorized at
// src/export_torchkbnufft_gpu_case.py:305). Going through float would double-round.
inline uint16_t f64_to_f16_bits(double v) {
  uint64_t b;
  std::memcpy(&b, &v, sizeof b);
  const uint16_t sign = static_cast<uint16_t>((b >> 48) & 0x8000u);
  const int64_t exp = static_cast<int64_t>((b >> 52) & 0x7FFu);
  const uint64_t man = b & 0xFFFFFFFFFFFFFull;
  if (exp == 0x7FF) return static_cast<uint16_t>(sign | 0x7C00u | (man ? 0x200u : 0u));
  if (exp == 0) return sign;  // zero or binary64 subnormal: far below half's range
  const int64_t e = exp - 1023;
  const uint64_t full = man | (1ull << 52);
  const int64_t shift = (e >= -14) ? 42 : 42 + (-14 - e);
  if (shift > 63) return sign;
  uint64_t q = full >> shift;
  const uint64_t rem = full & ((1ull << shift) - 1ull);
  const uint64_t halfway = 1ull << (shift - 1);
  if (rem > halfway || (rem == halfway && (q & 1ull))) ++q;
  if (e >= -14) {
    int64_t he = e + 15;
    if (q == 2048) {
      q = 1024;
      ++he;
    }
    if (he >= 31) return static_cast<uint16_t>(sign | 0x7C00u);
    return static_cast<uint16_t>(sign | (he << 10) | (q - 1024));
  }
  return static_cast<uint16_t>(sign | q);  // subnormal (q == 1024 encodes the smallest normal)
}

inline bool f16_bits_nonzero(uint16_t h) { return (h & 0x7FFFu) != 0; }

// Exact binary16 -> binary64 (sign, 5-bit exponent, 10-bit fraction; subnormals, inf, NaN).
inline double f16_bits_to_f64(uint16_t h) {
  const int e = (h >> 10) & 0x1F, m = h & 0x3FF;
  const double sign = (h & 0x8000u) ? -1.0 : 1.0;
  if (e == 0) return sign * std::ldexp(static_cast<double>(m), -24);
  if (e == 31) return m ? std::nan("") : sign * HUGE_VAL;
  return sign * std::ldexp(static_cast<double>(1024 + m), e - 25);
}

// CPython random.Random: MT19937 seeded by init_by_array over the 32-bit words of
// abs(seed) (a zero seed is the single word 0), random() = 53-bit double from two
// draws. The reference planner's tie-breaks are defined by this generator
// (src/nufft_layout_oracle.py:340-363, :383-413).
class PyRandom {
 public:
  explicit PyRandom(uint64_t seed) {
    uint32_t key[2];
    int len = 0;
    do {
      key[len++] = static_cast<uint32_t>(seed & 0xFFFFFFFFu);
      seed >>= 32;
    } while (seed != 0 && len < 2);
    init_by_array(key, len);
  }
  uint32_t next_u32() {
    if (idx_ >= 624) twist();
    uint32_t y = mt_[idx_++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9D2C5680u;
    y ^= (y << 15) & 0xEFC60000u;
    y ^= (y >> 18);
    return y;
  }
  double random() {
    const uint32_t a = next_u32() >> 5;
    const uint32_t b = next_u32() >> 6;
    return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0);
  }

 private:
  void init_genrand(uint32_t s) {
    mt_[0] = s;
    for (int i = 1; i < 624; ++i) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + static_cast<uint32_t>(i);
    idx_ = 624;
  }
  void init_by_array(const uint32_t* key, int len) {
    init_genrand(19650218u);
    int i = 1, j = 0;
    for (int k = (624 > len ? 624 : len); k; --k) {
      mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1664525u)) + key[j] + static_cast<uint32_t>(j);
      ++i;
      ++j;
      if (i >= 624) {
        mt_[0] = mt_[623];
        i = 1;
      }
      if (j >= len) j = 0;
    }
    for (int k = 623; k; --k) {
      mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1566083941u)) - static_cast<uint32_t>(i);
      ++i;
      if (i >= 624) {
        mt_[0] = mt_[623];
        i = 1;
      }
    }
    mt_[0] = 0x80000000u;
    idx_ = 624;
  }
  void twist() {
    for (int i = 0; i < 624; ++i) {
      const uint32_t y = (mt_[i] & 0x80000000u) | (mt_[(i + 1) % 624] & 0x7FFFFFFFu);
      uint32_t v = mt_[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908B0DFu;
      mt_[i] = v;
    }
    idx_ = 0;
  }
  uint32_t mt_[624];
  int idx_ = 624;
};

}  // namespace tsn
