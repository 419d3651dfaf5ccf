// Seeded synthetic rating matrices, train/test split, CSR transpose and the raw
// binary CSR format. Host-only C++17; declarations in include/als_data.h.
//
// Generation model (one pure function of (seed, stream, index) per draw):
//   * item popularity: item at popularity rank r has weight (r+1)^-s; ranks are
//     mapped to item ids by a seeded permutation;
//   * user degree: lognormal or power law, clipped to [degree_min, degree_max],
//     scaled so that the total matches target_nnz;
//   * each user's items: weighted sampling without replacement (draw with
//     replacement, drop repeats -- the same law as successive sampling; users
//     rating more than half the catalogue use Gumbel top-k instead);
//   * rating: mu + <U_u, V_i> + noise, optionally rounded, clipped.
#include "../../include/als_data.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

enum Stream : uint64_t {
  kPerm = 1, kItemFactor = 2, kDegree = 3, kUserItems = 4, kUserFactor = 5,
  kNoise = 6, kSplit = 7, kInit = 8
};

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

inline uint64_t seed_of(uint64_t seed, uint64_t stream, uint64_t idx) {
  return mix64(mix64(seed + 0x9E3779B97F4A7C15ULL * (stream + 1)) ^
               (idx * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL));
}

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ULL;
    return mix64(s);
  }
  // uniform in (0, 1]
  double uni() { return ((next() >> 11) + 1) * 0x1.0p-53; }
  double normal() {
    double u1 = uni(), u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

int nthreads(int32_t req) {
  if (req > 0) return req;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Run body(i) for i in [0, count) on `threads` workers pulling chunks.
void parallel_for(int64_t count, int threads, int64_t chunk,
                  const std::function<void(int64_t, int64_t)> &body) {
  if (count <= 0) return;
  threads = (int)std::min<int64_t>(threads, (count + chunk - 1) / chunk);
  if (threads <= 1) {
    body(0, count);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= count) break;
        body(b, std::min(count, b + chunk));
      }
    });
  for (auto &th : pool) th.join();
}

double raw_degree(const als_synth_spec &s, int64_t u) {
  Rng r(seed_of(s.seed, kDegree, (uint64_t)u));
  if (s.degree_law == ALS_DEGREE_POWERLAW) {
    double a = s.degree_p1 > 1.0 ? s.degree_p1 : 2.0;
    return std::pow(r.uni(), -1.0 / (a - 1.0));
  }
  return std::exp(s.degree_p1 * r.normal());
}

int64_t clip_degree(const als_synth_spec &s, double x) {
  int64_t hi = s.degree_max > 0 ? std::min<int64_t>(s.degree_max, s.n) : s.n;
  int64_t lo = std::max<int64_t>(0, std::min(s.degree_min, hi));
  double v = std::nearbyint(x);
  if (!(v >= (double)lo)) return lo;  // also catches NaN
  if (v > (double)hi) return hi;
  return (int64_t)v;
}

}  // namespace

extern "C" {

int als_synth_degrees(const als_synth_spec *spec, int64_t *deg_out, int64_t *total_out) {
  if (!spec || !deg_out || spec->m <= 0 || spec->n <= 0) return -1;
  const als_synth_spec s = *spec;
  const int T = nthreads(s.threads);
  std::vector<double> raw((size_t)s.m);
  parallel_for(s.m, T, 1 << 16, [&](int64_t b, int64_t e) {
    for (int64_t u = b; u < e; ++u) raw[(size_t)u] = raw_degree(s, u);
  });
  auto total_for = [&](double c) {
    std::atomic<int64_t> total{0};
    parallel_for(s.m, T, 1 << 16, [&](int64_t b, int64_t e) {
      int64_t acc = 0;
      for (int64_t u = b; u < e; ++u) acc += clip_degree(s, c * raw[(size_t)u]);
      total.fetch_add(acc);
    });
    return total.load();
  };
  double c = (s.degree_law == ALS_DEGREE_POWERLAW) ? (double)std::max<int64_t>(1, s.degree_min) : 1.0;
  if (s.target_nnz > 0) {
    double lo = 1e-9, hi = 1e12;
    for (int it = 0; it < 100; ++it) {
      double mid = std::sqrt(lo * hi);
      if (total_for(mid) < s.target_nnz) lo = mid; else hi = mid;
      if (hi / lo < 1.0 + 1e-12) break;
    }
    c = hi;
  }
  int64_t total = 0;
  for (int64_t u = 0; u < s.m; ++u) {
    deg_out[u] = clip_degree(s, c * raw[(size_t)u]);
    total += deg_out[u];
  }
  if (total_out) *total_out = total;
  return 0;
}

int als_synth_fill(const als_synth_spec *spec, const int64_t *row_ptr, int32_t *col, float *val) {
  if (!spec || !row_ptr || !col || !val || spec->m <= 0 || spec->n <= 0) return -1;
  const als_synth_spec s = *spec;
  const int T = nthreads(s.threads);
  const int64_t n = s.n;
  const int k = std::max(1, s.planted_rank);

  // popularity rank -> item id
  std::vector<int32_t> perm((size_t)n);
  for (int64_t i = 0; i < n; ++i) perm[(size_t)i] = (int32_t)i;
  {
    Rng r(seed_of(s.seed, kPerm, 0));
    for (int64_t i = n - 1; i > 0; --i) {
      int64_t j = (int64_t)(r.next() % (uint64_t)(i + 1));
      std::swap(perm[(size_t)i], perm[(size_t)j]);
    }
  }
  std::vector<double> logw((size_t)n), cdf((size_t)n);
  double acc = 0.0;
  for (int64_t r = 0; r < n; ++r) {
    logw[(size_t)r] = -s.item_zipf_s * std::log((double)(r + 1));
    acc += std::exp(logw[(size_t)r]);
    cdf[(size_t)r] = acc;
  }
  const double wtotal = acc;

  // planted item factors
  std::vector<float> V((size_t)n * k);
  parallel_for(n, T, 4096, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      Rng r(seed_of(s.seed, kItemFactor, (uint64_t)i));
      for (int j = 0; j < k; ++j) V[(size_t)i * k + j] = (float)(s.factor_sigma * r.normal());
    }
  });

  parallel_for(s.m, T, 256, [&](int64_t b, int64_t e) {
    std::vector<uint64_t> seen((size_t)(n + 63) / 64, 0);
    std::vector<int32_t> ranks;
    std::vector<std::pair<double, int32_t>> keys;
    std::vector<float> U((size_t)k);
    for (int64_t u = b; u < e; ++u) {
      const int64_t off = row_ptr[u];
      const int64_t d = row_ptr[u + 1] - off;
      ranks.clear();
      if (d > 0) {
        Rng r(seed_of(s.seed, kUserItems, (uint64_t)u));
        if (2 * d > n) {  // Gumbel top-k over the whole catalogue
          keys.resize((size_t)n);
          for (int64_t q = 0; q < n; ++q)
            keys[(size_t)q] = {logw[(size_t)q] - std::log(-std::log(r.uni() * (1.0 - 1e-16))),
                               (int32_t)q};
          std::nth_element(keys.begin(), keys.begin() + (d - 1), keys.end(),
                           [](const std::pair<double, int32_t> &a,
                              const std::pair<double, int32_t> &c) { return a.first > c.first; });
          for (int64_t q = 0; q < d; ++q) ranks.push_back(keys[(size_t)q].second);
        } else {
          while ((int64_t)ranks.size() < d) {
            double x = r.uni() * wtotal;
            int64_t q = std::lower_bound(cdf.begin(), cdf.end(), x) - cdf.begin();
            if (q >= n) q = n - 1;
            uint64_t bit = 1ULL << (q & 63);
            if (seen[(size_t)q >> 6] & bit) continue;
            seen[(size_t)q >> 6] |= bit;
            ranks.push_back((int32_t)q);
          }
          for (int32_t q : ranks) seen[(size_t)q >> 6] = 0;
        }
      }
      for (int64_t q = 0; q < d; ++q) col[off + q] = perm[(size_t)ranks[(size_t)q]];
      std::sort(col + off, col + off + d);
      Rng ru(seed_of(s.seed, kUserFactor, (uint64_t)u));
      for (int j = 0; j < k; ++j) U[(size_t)j] = (float)(s.factor_sigma * ru.normal());
      for (int64_t q = 0; q < d; ++q) {
        const int64_t eidx = off + q;
        const float *v = &V[(size_t)col[eidx] * k];
        double dot = 0.0;
        for (int j = 0; j < k; ++j) dot += (double)U[(size_t)j] * (double)v[j];
        Rng rn(seed_of(s.seed, kNoise, (uint64_t)eidx));
        double x = s.mu + dot + s.noise_sigma * rn.normal();
        if (s.integer_ratings) x = std::nearbyint(x);
        x = std::min(s.rating_max, std::max(s.rating_min, x));
        val[eidx] = (float)x;
      }
    }
  });
  return 0;
}

int als_split(int64_t m, const int64_t *row_ptr, const int32_t *col, const float *val,
              double test_fraction, uint64_t seed, int64_t *train_cnt, int64_t *test_cnt,
              const int64_t *train_ptr, int32_t *train_col, float *train_val,
              const int64_t *test_ptr, int32_t *test_col, float *test_val, int32_t threads) {
  if (m < 0 || !row_ptr) return -1;
  const int T = nthreads(threads);
  auto is_test = [&](int64_t e) {
    Rng r(seed_of(seed, kSplit, (uint64_t)e));
    return r.uni() <= test_fraction;
  };
  if (!train_col) {
    if (!train_cnt || !test_cnt) return -1;
    parallel_for(m, T, 4096, [&](int64_t b, int64_t e) {
      for (int64_t u = b; u < e; ++u) {
        int64_t tr = 0, te = 0;
        for (int64_t q = row_ptr[u]; q < row_ptr[u + 1]; ++q) (is_test(q) ? te : tr)++;
        train_cnt[u] = tr;
        test_cnt[u] = te;
      }
    });
    return 0;
  }
  if (!col || !val || !train_ptr || !train_val || !test_ptr || !test_col || !test_val) return -1;
  parallel_for(m, T, 4096, [&](int64_t b, int64_t e) {
    for (int64_t u = b; u < e; ++u) {
      int64_t a = train_ptr[u], t = test_ptr[u];
      for (int64_t q = row_ptr[u]; q < row_ptr[u + 1]; ++q) {
        if (is_test(q)) { test_col[t] = col[q]; test_val[t] = val[q]; ++t; }
        else { train_col[a] = col[q]; train_val[a] = val[q]; ++a; }
      }
    }
  });
  return 0;
}

int als_csr_transpose(int64_t m, int64_t n, const int64_t *row_ptr, const int32_t *col,
                      const float *val, int64_t *col_ptr, int32_t *row_idx, float *val_t,
                      int32_t threads) {
  if (m < 0 || n < 0 || !row_ptr || !col_ptr) return -1;
  int T = std::min(nthreads(threads), 16);
  if (m < 4096) T = 1;
  // contiguous row ranges of roughly equal nnz, one per worker
  const int64_t nnz = row_ptr[m];
  std::vector<int64_t> rb((size_t)T + 1, m);
  rb[0] = 0;
  for (int t = 1; t < T; ++t) {
    int64_t target = nnz / T * t;
    rb[(size_t)t] = std::lower_bound(row_ptr, row_ptr + m + 1, target) - row_ptr;
    if (rb[(size_t)t] < rb[(size_t)t - 1]) rb[(size_t)t] = rb[(size_t)t - 1];
  }
  std::vector<std::vector<int64_t>> cnt((size_t)T, std::vector<int64_t>((size_t)n, 0));
  auto run = [&](const std::function<void(int)> &f) {
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) pool.emplace_back(f, t);
    for (auto &th : pool) th.join();
  };
  run([&](int t) {
    auto &c = cnt[(size_t)t];
    for (int64_t q = row_ptr[rb[(size_t)t]]; q < row_ptr[rb[(size_t)t + 1]]; ++q) c[(size_t)col[q]]++;
  });
  int64_t acc = 0;
  for (int64_t j = 0; j < n; ++j) {
    col_ptr[j] = acc;
    for (int t = 0; t < T; ++t) {
      int64_t c = cnt[(size_t)t][(size_t)j];
      cnt[(size_t)t][(size_t)j] = acc;
      acc += c;
    }
  }
  col_ptr[n] = acc;
  if (!row_idx) return 0;
  run([&](int t) {
    auto &pos = cnt[(size_t)t];
    for (int64_t u = rb[(size_t)t]; u < rb[(size_t)t + 1]; ++u)
      for (int64_t q = row_ptr[u]; q < row_ptr[u + 1]; ++q) {
        int64_t p = pos[(size_t)col[q]]++;
        row_idx[p] = (int32_t)u;
        if (val_t) val_t[p] = val[q];
      }
  });
  return 0;
}

int als_init_factors(int64_t rows, int32_t f, double sigma, uint64_t seed, float *out,
                     int32_t threads) {
  if (rows < 0 || f <= 0 || !out) return -1;
  parallel_for(rows, nthreads(threads), 4096, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      Rng r(seed_of(seed, kInit, (uint64_t)i));
      for (int j = 0; j < f; ++j) out[(size_t)i * f + j] = (float)(sigma * r.normal());
    }
  });
  return 0;
}

int als_load_csr_bin(const char *data_file, const char *row_file, const char *col_file,
                     float *data, int32_t *row, int32_t *col, int64_t m, int64_t nnz) {
  FILE *d = std::fopen(data_file, "rb"), *r = std::fopen(row_file, "rb"),
       *c = std::fopen(col_file, "rb");
  int rc = 0;
  if (!d || !r || !c) rc = -1;
  else if (std::fread(row, sizeof(int32_t), (size_t)(m + 1), r) != (size_t)(m + 1) ||
           std::fread(col, sizeof(int32_t), (size_t)nnz, c) != (size_t)nnz ||
           std::fread(data, sizeof(float), (size_t)nnz, d) != (size_t)nnz)
    rc = -1;
  if (d) std::fclose(d);
  if (r) std::fclose(r);
  if (c) std::fclose(c);
  return rc;
}

int als_save_csr_bin(const char *data_file, const char *row_file, const char *col_file,
                     const float *data, const int32_t *row, const int32_t *col, int64_t m,
                     int64_t nnz) {
  FILE *d = std::fopen(data_file, "wb"), *r = std::fopen(row_file, "wb"),
       *c = std::fopen(col_file, "wb");
  int rc = 0;
  if (!d || !r || !c) rc = -1;
  else if (std::fwrite(row, sizeof(int32_t), (size_t)(m + 1), r) != (size_t)(m + 1) ||
           std::fwrite(col, sizeof(int32_t), (size_t)nnz, c) != (size_t)nnz ||
           std::fwrite(data, sizeof(float), (size_t)nnz, d) != (size_t)nnz)
    rc = -1;
  if (d) std::fclose(d);
  if (r) std::fclose(r);
  if (c) std::fclose(c);
  return rc;
}

}  // extern "C"
