// Exact, order-independent FP64 sums on the device, in the representation of the reference's
// ExactSum (runtime/include/autan/runtime/exact_sum.hpp:15-35, runtime/src/exact_sum.cpp:22-140):
// 68 fixed-point limbs of 32 bits held in int64 words, limb i weighing 2^(32 i - 1088), then the
// counts of +inf, -inf and NaN terms; the sum is rounded once, to nearest even. Integer additions
// are associative, so the words (and the rounded value) do not depend on the launch shape or on
// the order in which threads and blocks add their terms: repeated runs give the same bits.
//
// B200 layout: each warp merges the terms of its lanes that land on the same limb with shuffles
// before one shared-memory atomic per word; each block then adds its non-zero words to the global
// words with one atomic each.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace autan_b200 {

constexpr int kLimbs = 68;
constexpr int kWords = kLimbs + 3;  // limbs, +inf count, -inf count, NaN count
constexpr int kOffset = 1088;

// Adds the term t of every lane to `words` (shared or global memory). Every lane of the warp must
// call it (t = 0 adds nothing).
__device__ __forceinline__ void warp_exact_add(unsigned long long* words, double t) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(t));
  const int biased = static_cast<int>((bits >> 52) & 0x7ff);
  const unsigned long long fraction = bits & ((1ULL << 52) - 1);
  const bool negative = (bits >> 63) != 0;
  if (biased == 0x7ff) {
    atomicAdd(&words[fraction != 0 ? kLimbs + 2 : (negative ? kLimbs + 1 : kLimbs)], 1ULL);
  }
  const bool has = biased != 0x7ff && !(biased == 0 && fraction == 0);
  int limb = 0;
  long long p0 = 0, p1 = 0, p2 = 0;
  if (has) {
    const unsigned long long m = biased == 0 ? fraction : (fraction | (1ULL << 52));
    const int e = biased == 0 ? -1074 : biased - 1075;
    const int p = e + kOffset;
    limb = p >> 5;
    const int s = p & 31;
    const unsigned long long lo = (m & 0xffffffffULL) << s, hi = (m >> 32) << s;
    const long long sign = negative ? -1 : 1;
    p0 = sign * static_cast<long long>(lo & 0xffffffffULL);
    p1 = sign * static_cast<long long>((lo >> 32) + (hi & 0xffffffffULL));
    p2 = sign * static_cast<long long>(hi >> 32);
  }
  unsigned todo = __ballot_sync(full, has);
  while (todo != 0) {
    const int leader = __ffs(todo) - 1;
    const int li = __shfl_sync(full, limb, leader);
    const bool mine = has && limb == li;
    const unsigned group = __ballot_sync(full, mine);
    long long a = mine ? p0 : 0, b = mine ? p1 : 0, c = mine ? p2 : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a += __shfl_xor_sync(full, a, off);
      b += __shfl_xor_sync(full, b, off);
      c += __shfl_xor_sync(full, c, off);
    }
    if (lane == leader) {
      atomicAdd(&words[li], static_cast<unsigned long long>(a));
      atomicAdd(&words[li + 1], static_cast<unsigned long long>(b));
      atomicAdd(&words[li + 2], static_cast<unsigned long long>(c));
    }
    todo &= ~group;
  }
}

// warp_exact_add for terms that are never negative (squares): +0, positive, +inf or NaN. The
// shifted mantissa m << s (below 2^84) is cut into six 16-bit chunks; the lanes of one limb group
// sum each chunk with one redux.sync (32 terms below 2^16 sum below 2^21, exactly), and the leader
// adds chunk pairs to the group's three words: each addend is below 2^38, as in warp_exact_add.
// PRIVATE: `words` belong to this warp alone, so the leader's adds need no atomics.
template <bool PRIVATE = false>
__device__ __forceinline__ void warp_exact_add_nonneg(unsigned long long* words, double t) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(t));
  const int biased = static_cast<int>((bits >> 52) & 0x7ff);
  const unsigned long long fraction = bits & ((1ULL << 52) - 1);
  if (biased == 0x7ff) atomicAdd(&words[fraction != 0 ? kLimbs + 2 : kLimbs], 1ULL);
  const bool has = biased != 0x7ff && !(biased == 0 && fraction == 0);
  int limb = 0;
  unsigned long long lo = 0, hi = 0;
  if (has) {
    const unsigned long long m = biased == 0 ? fraction : (fraction | (1ULL << 52));
    const int e = biased == 0 ? -1074 : biased - 1075;
    const int p = e + kOffset;
    limb = p >> 5;
    const int s = p & 31;
    lo = m << s;
    hi = s == 0 ? 0ULL : m >> (64 - s);
  }
  unsigned todo = __ballot_sync(full, has);
  while (todo != 0) {
    const int leader = __ffs(todo) - 1;
    const int li = __shfl_sync(full, limb, leader);
    const bool mine = has && limb == li;
    const unsigned group = __ballot_sync(full, mine);
    const unsigned long long a = mine ? lo : 0ULL, b = mine ? hi : 0ULL;
    const unsigned s0 = __reduce_add_sync(full, static_cast<unsigned>(a & 0xffff));
    const unsigned s1 = __reduce_add_sync(full, static_cast<unsigned>((a >> 16) & 0xffff));
    const unsigned s2 = __reduce_add_sync(full, static_cast<unsigned>((a >> 32) & 0xffff));
    const unsigned s3 = __reduce_add_sync(full, static_cast<unsigned>(a >> 48));
    const unsigned s4 = __reduce_add_sync(full, static_cast<unsigned>(b & 0xffff));
    const unsigned s5 = __reduce_add_sync(full, static_cast<unsigned>(b >> 16));
    if (lane == leader) {
      const unsigned long long w0 = static_cast<unsigned long long>(s0) + (static_cast<unsigned long long>(s1) << 16);
      const unsigned long long w1 = static_cast<unsigned long long>(s2) + (static_cast<unsigned long long>(s3) << 16);
      const unsigned long long w2 = static_cast<unsigned long long>(s4) + (static_cast<unsigned long long>(s5) << 16);
      if constexpr (PRIVATE) {
        words[li] += w0;
        words[li + 1] += w1;
        words[li + 2] += w2;
      } else {
        atomicAdd(&words[li], w0);
        atomicAdd(&words[li + 1], w1);
        atomicAdd(&words[li + 2], w2);
      }
    }
    __syncwarp();
    todo &= ~group;
  }
}

// The rounded value of a word array (ExactSum::value, runtime/src/exact_sum.cpp:99-140).
__device__ inline double exact_value(const unsigned long long* in) {
  long long w[kWords];
  for (int i = 0; i < kWords; ++i) w[i] = static_cast<long long>(in[i]);
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  if (w[kLimbs + 2] > 0 || (w[kLimbs] > 0 && w[kLimbs + 1] > 0))
    return __longlong_as_double(0x7ff8000000000000LL);
  if (w[kLimbs] > 0) return inf;
  if (w[kLimbs + 1] > 0) return -inf;
  auto normalize = [&]() {
    for (int i = 0; i + 1 < kLimbs; ++i) {
      const long long carry = w[i] >> 32;
      w[i] -= carry * (1LL << 32);
      w[i + 1] += carry;
    }
  };
  normalize();
  const bool negative = w[kLimbs - 1] < 0;
  if (negative) {
    for (int i = 0; i < kLimbs; ++i) w[i] = -w[i];
    normalize();
  }
  int t = kLimbs - 1;
  while (t >= 0 && w[t] == 0) --t;
  if (t < 0) return 0.0;
  auto limb = [&](int k) { return k < 0 ? 0ULL : static_cast<unsigned long long>(w[k]); };
  const unsigned long long top = limb(t);
  if (top > 0xffffffffULL) return negative ? -inf : inf;
  const int b = 64 - __clzll(static_cast<long long>(top));
  const unsigned long long below = (limb(t - 1) << 32) | limb(t - 2);
  const unsigned long long lead = (top << (64 - b)) | (below >> b);
  bool sticky = (below & ((1ULL << b) - 1)) != 0;
  for (int k = t - 3; k >= 0 && !sticky; --k) sticky = limb(k) != 0;
  unsigned long long mantissa = lead >> 11;
  const unsigned long long rest = lead & 0x7ff;
  if (rest > 0x400 || (rest == 0x400 && (sticky || (mantissa & 1) != 0))) ++mantissa;
  int exponent = 32 * (t - 2) - kOffset + b + 11;
  if (mantissa == (1ULL << 53)) {
    mantissa >>= 1;
    ++exponent;
  }
  const double magnitude = ldexp(static_cast<double>(mantissa), exponent);
  return negative ? -magnitude : magnitude;
}

}  // namespace autan_b200
