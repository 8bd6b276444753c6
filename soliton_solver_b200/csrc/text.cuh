// text.cuh -- plain-text formatting of lattice arrays on the device (.dat bundles).
//
// The reference writes fields, densities and scalars as text with Python's
// format(v, ".{P}g") followed by a tab, a newline after each lattice row and a blank
// line after each component (core/io.py:44-240).  Here every value is formatted by one
// thread with an exact decimal conversion of the binary value (arbitrary-precision
// digits, round half to even at P significant digits, then the "g" presentation
// rules: scientific when the decimal exponent is < -4 or >= P, trailing zeros
// removed, at least two exponent digits, "nan", "inf", "-0"), so the bytes equal
// Python's.  Three passes: lengths, an exclusive scan of the lengths, and the write
// of each value's text at its offset.
#pragma once

#include <cstdint>

namespace ssb {

constexpr int TXT_MAX_P = 40;     // digits supported
constexpr int TXT_MAX_LEN = 48;   // longest value text: "-d.(39 digits)e-308"
constexpr int TXT_LIMBS = 36;     // 32-bit limbs of a fraction of up to 1152 bits

// Decimal digits of |v| (finite, nonzero): writes P significant digits (rounded half
// to even on the exact value) into d and returns the decimal exponent of d[0].
__device__ inline int exact_digits(double v, int P, int* d) {
  const uint64_t bits = (uint64_t)__double_as_longlong(v) & 0x7fffffffffffffffULL;
  int bexp = (int)(bits >> 52);
  uint64_t m = bits & 0xfffffffffffffULL;
  int e;
  if (bexp == 0) {
    e = -1074;
  } else {
    m |= 1ULL << 52;
    e = bexp - 1075;
  }
  // |v| = m * 2^e.  Collect P + 1 significant digits and a sticky flag.
  int nd = 0, X = 0;
  bool started = false, sticky = false;
  int dig[TXT_MAX_P + 2];
  auto push = [&](int digit, int pos_exp) {  // pos_exp: decimal exponent of this digit
    if (!started) {
      if (digit == 0) return;
      started = true;
      X = pos_exp;
    }
    if (nd < P + 1) dig[nd++] = digit;
    else if (digit) sticky = true;
  };
  // integer part
  if (e >= 0) {
    // m << e as little-endian limbs, then base-1e9 chunks by repeated division
    uint32_t L[TXT_LIMBS];
    for (int i = 0; i < TXT_LIMBS; ++i) L[i] = 0;
    const int ls = e / 32, bs = e % 32;
    const unsigned __int128 mm = (unsigned __int128)m << bs;
    L[ls] = (uint32_t)mm;
    L[ls + 1] = (uint32_t)(mm >> 32);
    if (ls + 2 < TXT_LIMBS) L[ls + 2] = (uint32_t)(mm >> 64);
    int top = ls + 2;
    uint32_t chunks[40];
    int nc = 0;
    while (top >= 0) {
      uint64_t rem = 0;
      for (int i = top; i >= 0; --i) {
        const uint64_t cur = (rem << 32) | L[i];
        L[i] = (uint32_t)(cur / 1000000000ULL);
        rem = cur % 1000000000ULL;
      }
      chunks[nc++] = (uint32_t)rem;
      while (top >= 0 && L[top] == 0) --top;
    }
    int total = 0;  // digits of the integer
    {
      uint32_t c = chunks[nc - 1];
      int lead = 0;
      while (c) { ++lead; c /= 10; }
      total = lead + 9 * (nc - 1);
    }
    int pos = total - 1;
    for (int ci = nc - 1; ci >= 0; --ci) {
      const uint32_t c = chunks[ci];
      const int w = ci == nc - 1 ? (total - 9 * (nc - 1)) : 9;
      uint32_t p10 = 1;
      for (int k = 1; k < w; ++k) p10 *= 10;
      for (int k = 0; k < w; ++k) {
        push((int)((c / p10) % 10), pos--);
        p10 /= 10;
      }
    }
  } else {
    const int k = -e;  // fraction bits
    const uint64_t ip = k >= 64 ? 0 : (m >> k);
    const uint64_t fr = k >= 64 ? m : (m & ((1ULL << k) - 1));
    if (ip) {
      int w = 0;
      uint64_t t = ip;
      char tmp[20];
      while (t) { tmp[w++] = (char)(t % 10); t /= 10; }
      for (int i = w - 1; i >= 0; --i) push(tmp[i], i);
    }
    // fraction fr / 2^k as limbs of a 32*NL-bit fixed-point number
    const int NL = (k + 31) / 32;
    const int sh = 32 * NL - k;  // left shift that aligns the fraction to the limb grid
    uint32_t f[TXT_LIMBS];
    for (int i = 0; i < NL; ++i) f[i] = 0;
    {
      const unsigned __int128 v2 = (unsigned __int128)fr << sh;  // fr < 2^53, sh < 32
      // the fraction's bits sit at the bottom of the NL-limb number
      f[0] = (uint32_t)v2;
      if (NL > 1) f[1] = (uint32_t)(v2 >> 32);
      if (NL > 2) f[2] = (uint32_t)(v2 >> 64);
    }
    int lo = 0;  // lowest nonzero limb (limbs below it stay zero)
    int pos = -1;
    bool nonzero = fr != 0;
    while (nonzero && nd < P + 1) {
      uint64_t carry = 0;
      for (int i = lo; i < NL; ++i) {
        const uint64_t t = (uint64_t)f[i] * 1000000000ULL + carry;
        f[i] = (uint32_t)t;
        carry = t >> 32;
      }
      const uint32_t c = (uint32_t)carry;  // next nine decimal digits
      uint32_t p10 = 100000000;
      for (int q = 0; q < 9; ++q) {
        push((int)((c / p10) % 10), pos--);
        p10 /= 10;
      }
      while (lo < NL && f[lo] == 0) ++lo;
      nonzero = lo < NL;
    }
    if (nonzero) sticky = true;
  }
  // round half to even at P digits
  bool up = false;
  if (nd > P) {
    const int nx = dig[P];
    up = nx > 5 || (nx == 5 && (sticky || (dig[P - 1] & 1)));
  }
  for (int i = nd; i < P; ++i) dig[i] = 0;
  if (up) {
    int i = P - 1;
    while (i >= 0 && dig[i] == 9) dig[i--] = 0;
    if (i >= 0) {
      ++dig[i];
    } else {
      dig[0] = 1;
      for (int j = 1; j < P; ++j) dig[j] = 0;
      ++X;
    }
  }
  for (int i = 0; i < P; ++i) d[i] = dig[i];
  return X;
}

// format(v, ".{P}g") of Python into buf; returns the length
__device__ inline int format_g(double v, int P, char* buf) {
  if (P < 1) P = 1;
  int n = 0;
  if (isnan(v)) {
    buf[0] = 'n'; buf[1] = 'a'; buf[2] = 'n';
    return 3;
  }
  const bool neg = signbit(v);
  if (neg) buf[n++] = '-';
  if (isinf(v)) {
    buf[n++] = 'i'; buf[n++] = 'n'; buf[n++] = 'f';
    return n;
  }
  if (v == 0.0) {
    buf[n++] = '0';
    return n;
  }
  int d[TXT_MAX_P];
  const int X = exact_digits(v, P, d);
  int last = P - 1;  // trailing zeros removed
  while (last > 0 && d[last] == 0) --last;
  if (X < -4 || X >= P) {
    buf[n++] = (char)('0' + d[0]);
    if (last > 0) {
      buf[n++] = '.';
      for (int i = 1; i <= last; ++i) buf[n++] = (char)('0' + d[i]);
    }
    buf[n++] = 'e';
    int ex = X;
    buf[n++] = ex < 0 ? '-' : '+';
    if (ex < 0) ex = -ex;
    if (ex >= 100) {
      buf[n++] = (char)('0' + ex / 100);
      ex %= 100;
      buf[n++] = (char)('0' + ex / 10);
      buf[n++] = (char)('0' + ex % 10);
    } else {
      buf[n++] = (char)('0' + ex / 10);
      buf[n++] = (char)('0' + ex % 10);
    }
  } else if (X >= 0) {
    for (int i = 0; i <= X; ++i) buf[n++] = (char)('0' + (i <= last ? d[i] : 0));
    if (last > X) {
      buf[n++] = '.';
      for (int i = X + 1; i <= last; ++i) buf[n++] = (char)('0' + d[i]);
    }
  } else {
    buf[n++] = '0';
    buf[n++] = '.';
    for (int i = 0; i < -X - 1; ++i) buf[n++] = '0';
    for (int i = 0; i <= last; ++i) buf[n++] = (char)('0' + d[i]);
  }
  return n;
}

struct TextLayout {
  long long n, row, block;  // newline after every `row` values, another after every `block`
  int digits;
};

__device__ inline int text_suffix(long long i, const TextLayout& L, char* s) {
  int k = 0;
  s[k++] = '\t';
  if (L.row > 0 && (i + 1) % L.row == 0) s[k++] = '\n';
  if (L.block > 0 && (i + 1) % L.block == 0) s[k++] = '\n';
  return k;
}

template <typename T>
__global__ void text_len_kernel(const T* __restrict__ v, TextLayout L, long long* __restrict__ len) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  char buf[TXT_MAX_LEN], s[4];
  len[i] = format_g((double)v[i], L.digits, buf) + text_suffix(i, L, s);
}

// exclusive scan, three kernels: per-block scan (1024 values per block) with block sums,
// a scan of the block sums by one block, and the add-back
__global__ void scan_block_kernel(long long* __restrict__ a, long long n, long long* __restrict__ sums) {
  __shared__ long long s[1024];
  const long long i = blockIdx.x * 1024LL + threadIdx.x;
  const long long x = i < n ? a[i] : 0;
  s[threadIdx.x] = x;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const long long t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) a[i] = s[threadIdx.x] - x;  // exclusive within the block
  if (threadIdx.x == 1023) sums[blockIdx.x] = s[1023];
}

__global__ void scan_sums_kernel(long long* __restrict__ sums, long long nb, long long* __restrict__ total) {
  __shared__ long long s[1024];
  __shared__ long long base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (long long c0 = 0; c0 < nb; c0 += 1024) {
    const long long i = c0 + threadIdx.x;
    const long long x = i < nb ? sums[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const long long t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) sums[i] = base + s[threadIdx.x] - x;
    __syncthreads();
    if (threadIdx.x == 1023) base += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = base;
}

__global__ void scan_add_kernel(long long* __restrict__ a, long long n, const long long* __restrict__ sums) {
  const long long i = blockIdx.x * 1024LL + threadIdx.x;
  if (i < n) a[i] += sums[blockIdx.x];
}

template <typename T>
__global__ void text_write_kernel(const T* __restrict__ v, TextLayout L, const long long* __restrict__ off,
                                  char* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  char buf[TXT_MAX_LEN + 4];
  int k = format_g((double)v[i], L.digits, buf);
  k += text_suffix(i, L, buf + k);
  char* o = out + off[i];
  for (int j = 0; j < k; ++j) o[j] = buf[j];
}

}  // namespace ssb
