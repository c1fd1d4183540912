// CPU check of the fast walk's paired-word accumulation (acc_words in
// virtualct_b200/csrc/vct_walk.cuh, __host__ __device__): for seeded records
// and weights, including the extremes (16-bit densities of 65535, weights of
// 2^31, a whole major step) and enough segments that the packed 64-bit sums wrap, the recovered
// per-element sums must equal the plain per-element 64-bit sums exactly.
//   acc_check <M> <segments> <seed>   prints "ok" or the first mismatch
#include "../../virtualct_b200/csrc/vct_walk.cuh"

#include <cstdio>
#include <cstdlib>

using namespace vct;

template <int M>
static int run(long nseg, unsigned long long seed) {
  constexpr int kWords = (M + 1) / 2;
  unsigned long long P[kWords] = {}, H[kWords] = {}, plain[8] = {};
  unsigned long long x = seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&x]() {  // xorshift64*
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return x * 0x2545F4914F6CDD1Dull;
  };
  for (long k = 0; k < nseg; k++) {
    unsigned short v[8];
    for (int m = 0; m < 8; m++) {
      const unsigned long long r = next();
      // one draw in four at the 16-bit maximum, the rest uniform
      v[m] = (r & 3) == 0 ? 0xffffu : (unsigned short)(r >> 16);
      if (m >= M) v[m] = 0;
    }
    const unsigned long long rq = next();
    const unsigned int q = (rq & 3) == 0 ? (1u << 31) : (unsigned int)((rq >> 20) & ((1u << 31) - 1));
    int4 w;
    w.x = (int)(v[0] | (unsigned)v[1] << 16);
    w.y = (int)(v[2] | (unsigned)v[3] << 16);
    w.z = (int)(v[4] | (unsigned)v[5] << 16);
    w.w = (int)(v[6] | (unsigned)v[7] << 16);
    acc_words<M>(w, q, P, H);
    for (int m = 0; m < M; m++) plain[m] += (unsigned long long)v[m] * q;
  }
  for (int i = 0; i < kWords; i++) {
    const unsigned long long lo = P[i] - (H[i] << 16);
    if (lo != plain[2 * i]) {
      printf("mismatch element %d: %llu vs %llu\n", 2 * i, lo, plain[2 * i]);
      return 1;
    }
    if (2 * i + 1 < M && H[i] != plain[2 * i + 1]) {
      printf("mismatch element %d: %llu vs %llu\n", 2 * i + 1, H[i], plain[2 * i + 1]);
      return 1;
    }
  }
  printf("ok\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 4) return 2;
  const int M = atoi(argv[1]);
  const long n = atol(argv[2]);
  const unsigned long long seed = strtoull(argv[3], nullptr, 10);
  switch (M) {
    case 1: return run<1>(n, seed);
    case 2: return run<2>(n, seed);
    case 3: return run<3>(n, seed);
    case 4: return run<4>(n, seed);
    case 5: return run<5>(n, seed);
    case 6: return run<6>(n, seed);
    case 7: return run<7>(n, seed);
    case 8: return run<8>(n, seed);
  }
  return 2;
}
