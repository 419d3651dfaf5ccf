/*
 * als_data.h -- seeded synthetic rating matrices and CSR utilities (host only).
 *
 * No counterpart in the reference: cuMF receives its rating blocks from Spark
 * (als/src/CuMFJNIInterface.cpp:78-99) and only ships a raw binary CSR reader
 * (loadCSRSparseMatrixBin, als/src/cuda/als.cu:914-933), which is mirrored here
 * as als_load_csr_bin. The generator exists so that the engine, the CPU oracle
 * and the reference's own kernels all see identical bytes.
 *
 * Every random draw is a pure function of (seed, stream, index), so the output
 * does not depend on the number of threads used to produce it.
 */
#ifndef ALS_DATA_H_
#define ALS_DATA_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ALS_DEGREE_LOGNORMAL = 0, ALS_DEGREE_POWERLAW = 1 };

typedef struct als_synth_spec {
  int64_t m;               /* users (rows)                                    */
  int64_t n;               /* items (columns)                                 */
  int32_t planted_rank;    /* rank k of the planted factors U (m x k), V (n x k) */
  int32_t integer_ratings; /* 1: round to nearest integer before clipping     */
  double factor_sigma;     /* planted factor entries ~ N(0, factor_sigma^2)   */
  double noise_sigma;      /* additive rating noise ~ N(0, noise_sigma^2)     */
  double mu;               /* rating offset: r = mu + u.v + eps               */
  double rating_min, rating_max;
  int32_t degree_law;      /* ALS_DEGREE_LOGNORMAL or ALS_DEGREE_POWERLAW      */
  int32_t threads;         /* 0: all hardware threads                         */
  double degree_p1;        /* lognormal: sigma of log-degree; powerlaw: exponent */
  int64_t degree_min, degree_max; /* clip range (degree_max is also capped at n) */
  double item_zipf_s;      /* item popularity weight (rank+1)^-s              */
  int64_t target_nnz;      /* degrees are scaled so the total hits this (0: unscaled) */
  uint64_t seed;
} als_synth_spec;

/* Per-user degrees; returns 0 on success. total_out receives the sum. */
int als_synth_degrees(const als_synth_spec *spec, int64_t *deg_out, int64_t *total_out);

/* Fill a CSR whose row_ptr was built from als_synth_degrees (prefix sum).
 * Column indices come out sorted ascending within each row. */
int als_synth_fill(const als_synth_spec *spec, const int64_t *row_ptr, int32_t *col, float *val);

/* Hash split of a CSR into train and test parts: entry e (global position)
 * goes to test when uniform(seed, e) < test_fraction.
 * Pass 1 (train_col == NULL): writes per-row train and test counts.
 * Pass 2: fills train/test CSRs whose row pointers are the prefix sums. */
int als_split(int64_t m, const int64_t *row_ptr, const int32_t *col, const float *val,
              double test_fraction, uint64_t seed,
              int64_t *train_cnt, int64_t *test_cnt,
              const int64_t *train_ptr, int32_t *train_col, float *train_val,
              const int64_t *test_ptr, int32_t *test_col, float *test_val, int32_t threads);

/* CSR (m x n) -> CSC, i.e. the CSR of the transpose. Row indices within each
 * column come out ascending. col_ptr has n+1 entries. */
int als_csr_transpose(int64_t m, int64_t n, const int64_t *row_ptr, const int32_t *col,
                      const float *val, int64_t *col_ptr, int32_t *row_idx, float *val_t,
                      int32_t threads);

/* Seeded N(0, sigma^2) factor matrix (rows x f, row-major) for the initial
 * source factors of an ALS run. */
int als_init_factors(int64_t rows, int32_t f, double sigma, uint64_t seed, float *out,
                     int32_t threads);

/* Raw binary CSR files as read by the reference's loadCSRSparseMatrixBin
 * (als/src/cuda/als.cu:914-933): int32 row pointers (m+1), int32 column
 * indices (nnz), float32 values (nnz). Returns 0, or -1 when a file is missing
 * or short (the reference prints and returns without reading). */
int als_load_csr_bin(const char *data_file, const char *row_file, const char *col_file,
                     float *data, int32_t *row, int32_t *col, int64_t m, int64_t nnz);
int als_save_csr_bin(const char *data_file, const char *row_file, const char *col_file,
                     const float *data, const int32_t *row, const int32_t *col, int64_t m,
                     int64_t nnz);

#ifdef __cplusplus
}
#endif
#endif /* ALS_DATA_H_ */
