// rng_math.cuh -- exact skip-ahead for the RANLUX generators (ranlxs/ranlxd).
//
// The reference's ranlxs/ranlxd (src/random/ranlxs.C, src/random/ranlxd.C,
// Luscher's generators) run four independent lanes.  Each lane is a
// subtract-with-borrow (SWB) generator on 48-bit words (two 24-bit digits,
// STEP at ranlxs.C:14-46):
//     x_n = x_{n-5} - x_{n-12} - c_{n-1}  (mod b),  b = 2^48,
//     c_n = 1 if that difference was negative.
// A SWB generator with lags (r, s) = (12, 5) is exactly a linear
// congruential generator Y_n = a * Y_{n-1} mod m with m = b^12 - b^5 + 1 =
// 2^576 - 2^240 + 1 and a = b^{-1} mod m (Marsaglia & Zaman 1991; Tezuka,
// L'Ecuyer & Couture 1993).  With
//     A_n = sum_{i=0..11} x_{n-i} b^{11-i}     (the last 12 words),
//     Y_n = A_n - floor(A_n / b^7) + c_n,
// one has b * Y_{n+1} = Y_n + m * x_{n+1} for every state, so jumping k
// steps is Y -> a^k Y mod m.  Conversely, for a state produced by at least
// 12 recurrence steps, the last 12 words are the first 12 base-b digits of
// Y/m: A_n = floor(b^12 Y_n / m), which reduces to
//     A_n = Y + floor(Y / b^7) - [ (Y mod b^7 + floor(Y / b^7)) b^5 < Y + floor(Y / b^7) ]
// and c_n = Y_n - A_n + floor(A_n / b^7).
//
// Numbers are little-endian arrays of 64-bit limbs; 576 bits = 9 limbs.
// All routines are __host__ __device__ so the host library and the device
// kernels run the same code (the host side is unit-tested against the
// reference's serial stream).
#pragma once

#include <stdint.h>

namespace nrcps {
namespace rng {

constexpr int kLimbs = 9;  // 576 bits
typedef unsigned __int128 u128;

struct U576 {
  uint64_t w[kLimbs];
};

constexpr uint64_t kMask48 = (1ull << 48) - 1;

__host__ __device__ inline void set_zero(uint64_t* a, int n) {
  for (int i = 0; i < n; ++i) a[i] = 0;
}

// r = a - b over n limbs; returns the borrow.
__host__ __device__ inline uint64_t sub_n(uint64_t* r, const uint64_t* a, const uint64_t* b, int n) {
  uint64_t borrow = 0;
  for (int i = 0; i < n; ++i) {
    uint64_t ai = a[i], bi = b[i];
    uint64_t d = ai - bi - borrow;
    borrow = (ai < bi) || (ai == bi && borrow) ? 1 : 0;
    r[i] = d;
  }
  return borrow;
}

// r = a + b over n limbs; returns the carry.
__host__ __device__ inline uint64_t add_n(uint64_t* r, const uint64_t* a, const uint64_t* b, int n) {
  uint64_t carry = 0;
  for (int i = 0; i < n; ++i) {
    u128 s = (u128)a[i] + b[i] + carry;
    r[i] = (uint64_t)s;
    carry = (uint64_t)(s >> 64);
  }
  return carry;
}

// Compare a and b over n limbs: -1, 0, 1.
__host__ __device__ inline int cmp_n(const uint64_t* a, const uint64_t* b, int n) {
  for (int i = n - 1; i >= 0; --i) {
    if (a[i] < b[i]) return -1;
    if (a[i] > b[i]) return 1;
  }
  return 0;
}

// r (n limbs) = a (n limbs) shifted left by s bits (truncating).
__host__ __device__ inline void shl_n(uint64_t* r, const uint64_t* a, int n, int s) {
  int ls = s / 64, bs = s % 64;
  for (int i = n - 1; i >= 0; --i) {
    uint64_t v = 0;
    int j = i - ls;
    if (j >= 0) {
      v = a[j] << bs;
      if (bs && j - 1 >= 0) v |= a[j - 1] >> (64 - bs);
    }
    r[i] = v;
  }
}

// r (n limbs) = a (n limbs) shifted right by s bits.
__host__ __device__ inline void shr_n(uint64_t* r, const uint64_t* a, int n, int s) {
  int ls = s / 64, bs = s % 64;
  for (int i = 0; i < n; ++i) {
    uint64_t v = 0;
    int j = i + ls;
    if (j < n) {
      v = a[j] >> bs;
      if (bs && j + 1 < n) v |= a[j + 1] << (64 - bs);
    }
    r[i] = v;
  }
}

// The modulus m = 2^576 - 2^240 + 1.
__host__ __device__ inline void modulus(uint64_t* m) {
  // 2^576 - 2^240 + 1: limbs 0..8 all ones above bit 240, i.e.
  // m = (2^576 - 1) - (2^240 - 1) + 1 - ... computed directly:
  // 2^576 - 2^240 = sum of bits 240..575; plus 1.
  for (int i = 0; i < kLimbs; ++i) m[i] = 0;
  for (int bit = 240; bit < 576; ++bit) m[bit / 64] |= 1ull << (bit % 64);
  m[0] |= 1ull;
}

// r = (a * b) mod m, a, b < m.
__host__ __device__ inline void mulmod(U576& r, const U576& a, const U576& b) {
  uint64_t p[2 * kLimbs + 2];
  set_zero(p, 2 * kLimbs + 2);
  for (int i = 0; i < kLimbs; ++i) {
    uint64_t carry = 0;
    for (int j = 0; j < kLimbs; ++j) {
      u128 t = (u128)a.w[i] * b.w[j] + p[i + j] + carry;
      p[i + j] = (uint64_t)t;
      carry = (uint64_t)(t >> 64);
    }
    p[i + kLimbs] = carry;
  }
  // Reduce with 2^576 = 2^240 - 1 (mod m): v = L + H * 2^240 - H, repeated.
  const int NL = 2 * kLimbs + 2;
  for (int it = 0; it < 4; ++it) {
    bool high = false;
    for (int i = kLimbs; i < NL; ++i) high |= (p[i] != 0);
    if (!high) break;
    uint64_t H[2 * kLimbs + 2], L[2 * kLimbs + 2], Hs[2 * kLimbs + 2];
    set_zero(H, NL);
    set_zero(L, NL);
    for (int i = 0; i < kLimbs; ++i) L[i] = p[i];
    for (int i = kLimbs; i < NL; ++i) H[i - kLimbs] = p[i];
    shl_n(Hs, H, NL, 240);
    add_n(p, L, Hs, NL);
    sub_n(p, p, H, NL);
  }
  uint64_t m[kLimbs];
  modulus(m);
  while (cmp_n(p, m, kLimbs) >= 0) sub_n(p, p, m, kLimbs);
  for (int i = 0; i < kLimbs; ++i) r.w[i] = p[i];
}

// Per-lane SWB state: 12 words, words[j] = x_{n-11+j} (oldest first), carry.
struct Lane {
  uint64_t words[12];
  uint32_t carry;
};

// Y = A - floor(A / b^7) + c,  A = sum_j words[j] b^j.
__host__ __device__ inline void encode(U576& Y, const Lane& s) {
  uint64_t A[kLimbs], As[kLimbs];
  set_zero(A, kLimbs);
  for (int j = 0; j < 12; ++j) {
    // place 48-bit word j at bit 48*j
    int bit = 48 * j, li = bit / 64, bi = bit % 64;
    A[li] |= s.words[j] << bi;
    if (bi > 16 && li + 1 < kLimbs) A[li + 1] |= s.words[j] >> (64 - bi);
  }
  shr_n(As, A, kLimbs, 336);
  sub_n(Y.w, A, As, kLimbs);
  uint64_t c[kLimbs];
  set_zero(c, kLimbs);
  c[0] = s.carry;
  add_n(Y.w, Y.w, c, kLimbs);
}

// Inverse of encode for states reached by >= 12 recurrence steps.
__host__ __device__ inline void decode(Lane& s, const U576& Y) {
  const int n = kLimbs + 1;
  uint64_t y[kLimbs + 1], yh[kLimbs + 1], yl[kLimbs + 1], P[kLimbs + 1], Q[kLimbs + 1], A[kLimbs + 1];
  for (int i = 0; i < kLimbs; ++i) y[i] = Y.w[i];
  y[kLimbs] = 0;
  shr_n(yh, y, n, 336);
  // yl = y mod 2^336
  for (int i = 0; i < n; ++i) yl[i] = y[i];
  for (int bit = 336; bit < 64 * n; ++bit) yl[bit / 64] &= ~(1ull << (bit % 64));
  add_n(P, yl, yh, n);
  shl_n(P, P, n, 240);
  add_n(Q, y, yh, n);
  add_n(A, y, yh, n);
  if (cmp_n(P, Q, n) < 0) {
    uint64_t one[kLimbs + 1];
    set_zero(one, n);
    one[0] = 1;
    sub_n(A, A, one, n);
  }
  for (int j = 0; j < 12; ++j) {
    int bit = 48 * j, li = bit / 64, bi = bit % 64;
    uint64_t v = A[li] >> bi;
    if (bi > 16) v |= A[li + 1] << (64 - bi);
    s.words[j] = v & kMask48;
  }
  // c = Y - A + floor(A / b^7)
  uint64_t As[kLimbs + 1], t[kLimbs + 1];
  shr_n(As, A, n, 336);
  sub_n(t, y, A, n);
  add_n(t, t, As, n);
  s.carry = (uint32_t)t[0];
}

// One SWB step on a lane held oldest-first with the write position `pos`
// (the slot of x_{n-12}); returns the new word.  Used by the host paths.
__host__ __device__ inline void swb_step(uint64_t* words, int pos, uint32_t* carry) {
  int j = pos + 7;
  if (j >= 12) j -= 12;
  int64_t d = (int64_t)words[j] - (int64_t)words[pos] - (int64_t)*carry;
  *carry = d < 0 ? 1u : 0u;
  words[pos] = (uint64_t)d & kMask48;
}

}  // namespace rng
}  // namespace nrcps
