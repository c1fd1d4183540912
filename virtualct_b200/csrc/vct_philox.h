// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).  Ten rounds of the
// paper's 4x32 S-P network with its published multipliers and Weyl key
// increments.  Usable from host and device so the host tests can check the
// known-answer vectors.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define VCT_HD __host__ __device__ __forceinline__
#else
#define VCT_HD inline
#endif

namespace vct {

struct Philox4 {
  uint32_t v[4];
};

VCT_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
#if defined(__CUDA_ARCH__)
  *lo = a * b;
  *hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *lo = (uint32_t)p;
  *hi = (uint32_t)(p >> 32);
#endif
}

// counter ctr (4 words), key (2 words).
VCT_HD Philox4 philox4x32_10(Philox4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;  // round multipliers (SC'11, Table 2)
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // key schedule increments
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, ctr.v[0], &hi0, &lo0);
    mulhilo32(M1, ctr.v[2], &hi1, &lo1);
    Philox4 n;
    n.v[0] = hi1 ^ ctr.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ ctr.v[3] ^ k1;
    n.v[3] = lo0;
    ctr = n;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// Uniform double in (0, 1) from two 32-bit words: 53 random bits, offset by
// half an ulp so neither end is reached (log(u) stays finite).
VCT_HD double u01_open(uint32_t hi, uint32_t lo) {
  uint64_t b = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)b + 0.5) * (1.0 / 9007199254740992.0);
}

}  // namespace vct
