// tables.h -- host-built lookup tables uploaded once at initialize.
//
// The reference builds Poisson PMF tables on the device with expf/lgammaf and
// turns them into alias tables (src/cu/poisson.cu:9-34, lambda = n + beta for
// n < 100, 200 entries).  Here the tables are built on the host in double and
// stored as 32-bit CDF thresholds, so the device draw is a pure integer
// comparison and needs no device transcendental function.
#pragma once

#include <cmath>
#include <cstdint>

namespace gpulda {

// T[n][j] = min(floor(P(X <= j) * 2^32), 2^32-1) for X ~ Poisson(n + beta);
// guide[n][b] = first j with T[n][j] > b * 2^24 (capped at W-1).
inline void build_poisson_tables(float beta, uint32_t N, uint32_t W, uint32_t* cdf,
                                 uint8_t* guide) {
  for (uint32_t n = 0; n < N; ++n) {
    const double lam = (double)n + (double)beta;
    double p = std::exp(-lam);
    double c = 0.0;
    for (uint32_t j = 0; j < W; ++j) {
      c += p;
      double th = std::floor(c * 4294967296.0);
      cdf[n * W + j] = th >= 4294967295.0 ? 0xffffffffu : (uint32_t)th;
      p = p * lam / (double)(j + 1);
    }
    cdf[n * W + W - 1] = 0xffffffffu;
    uint32_t j = 0;
    for (uint32_t b = 0; b < 256; ++b) {
      const uint64_t lo = (uint64_t)b << 24;
      while (j < W - 1 && (uint64_t)cdf[n * W + j] <= lo) ++j;
      guide[n * 256 + b] = (uint8_t)j;
    }
  }
}

// lfac[k] = log(k!) for k < N.
inline void build_log_factorials(uint32_t N, double* lfac) {
  for (uint32_t k = 0; k < N; ++k) lfac[k] = std::lgamma((double)k + 1.0);
}

}  // namespace gpulda
