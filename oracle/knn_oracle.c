/*
 * knn_oracle.c -- host FP64 brute-force L2 k-nearest-neighbour ORACLE.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the curplsh_b200 product links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py use it, as the checker
 * and as the timed CPU restatement of the reference's algorithm.
 *
 * What it restates (paths relative to the cuRPLSH source tree):
 *   - src/internal/norm.cu:191-202      computeL2Norm(squared=true): per-row
 *                                       sum of squares.
 *   - src/internal/search.cu:79-216     searchL2Distance(..., exact=true):
 *                                       squared L2 distance of every query to
 *                                       every base row, k smallest per query,
 *                                       ascending; N == 0 gives FLT_MAX / -1
 *                                       (search.cu:94-101).
 *   - src/internal/select.cu:189-224    ascending k-selection.  The reference
 *                                       compares keys only, so its tie order is
 *                                       unspecified; the oracle fixes it to
 *                                       (distance, index) lexicographic, the
 *                                       rule the GPU engine also implements.
 *   - include/index.h:40-53             k larger than the number of base rows
 *                                       is padded with index -1 (the reference
 *                                       asserts k <= N instead, search.cu:121).
 *
 * Arithmetic: distances are accumulated in FP64 as sum_i (q_i - x_i)^2
 * directly (no ||q||^2 + ||x||^2 - 2q.x cancellation), so the oracle is at
 * least as accurate as any FP32 evaluation.  oracle_ref_formula() evaluates
 * the reference's own FP32 formula for comparison.
 *
 * Parity pin: tests/test_oracle.py checks this file against the known-answer
 * patterns of the reference's own smoke programs (test/test_search.cpp:33-36,
 * test/test_norm.cpp:18-22), stored in tests/golden/.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_QBLOCK 8

typedef struct {
  double d;
  int64_t i;
} pair_t;

/* (d, i) lexicographic "a is worse than b" for a max-heap. */
static inline int pair_gt(pair_t a, pair_t b) {
  return (a.d > b.d) || (a.d == b.d && a.i > b.i);
}

static void heap_sift_down(pair_t* h, int n, int pos) {
  for (;;) {
    int l = 2 * pos + 1, r = l + 1, m = pos;
    if (l < n && pair_gt(h[l], h[m])) m = l;
    if (r < n && pair_gt(h[r], h[m])) m = r;
    if (m == pos) return;
    pair_t t = h[m];
    h[m] = h[pos];
    h[pos] = t;
    pos = m;
  }
}

static int cmp_pair(const void* a, const void* b) {
  const pair_t* x = (const pair_t*)a;
  const pair_t* y = (const pair_t*)b;
  if (x->d < y->d) return -1;
  if (x->d > y->d) return 1;
  return (x->i > y->i) - (x->i < y->i);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Squared L2 norm of each row, FP64 (norm.cu:191-202, squared=true). */
void oracle_l2_norms(const float* x, int64_t n, int32_t d, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    const float* row = x + r * (int64_t)d;
    double s = 0.0;
    for (int32_t c = 0; c < d; ++c) s += (double)row[c] * (double)row[c];
    out[r] = s;
  }
}

/*
 * Exact kNN.  out_idx / out_dist are [nq x k] row-major, ascending by
 * (distance, index).  Slots beyond n are (-1, FLT_MAX), the values
 * search.cu:94-101 writes when n == 0.  threads <= 0 uses all OpenMP threads.
 * Returns 0, or -1 on bad arguments / allocation failure.
 */
int oracle_knn(const float* base, int64_t n, const float* queries, int64_t nq,
               int32_t d, int32_t k, int64_t* out_idx, double* out_dist,
               int threads) {
  if (d <= 0 || k <= 0 || nq < 0 || n < 0) return -1;
  if (n == 0) {
    for (int64_t t = 0; t < nq * (int64_t)k; ++t) {
      out_idx[t] = -1;
      out_dist[t] = (double)FLT_MAX;
    }
    return 0;
  }
  int kk = (int64_t)k < n ? k : (int)n;
  int err = 0;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#else
  threads = 1;
#endif
  int64_t nblocks = (nq + ORACLE_QBLOCK - 1) / ORACLE_QBLOCK;
#pragma omp parallel num_threads(threads)
  {
    pair_t* heaps = (pair_t*)malloc(sizeof(pair_t) * (size_t)kk * ORACLE_QBLOCK);
    double* qd = (double*)malloc(sizeof(double) * (size_t)d * ORACLE_QBLOCK);
    if (!heaps || !qd) {
#pragma omp atomic write
      err = 1;
    }
#pragma omp for schedule(dynamic, 1)
    for (int64_t b = 0; b < nblocks; ++b) {
      if (!heaps || !qd) continue;
      int64_t q0 = b * ORACLE_QBLOCK;
      int nb = (int)((nq - q0) < ORACLE_QBLOCK ? (nq - q0) : ORACLE_QBLOCK);
      for (int j = 0; j < nb; ++j)
        for (int32_t c = 0; c < d; ++c)
          qd[j * d + c] = (double)queries[(q0 + j) * (int64_t)d + c];
      int fill = 0;
      for (int64_t r = 0; r < n; ++r) {
        const float* row = base + r * (int64_t)d;
        double dist[ORACLE_QBLOCK];
        for (int j = 0; j < nb; ++j) {
          const double* q = qd + j * d;
          double s = 0.0;
          for (int32_t c = 0; c < d; ++c) {
            double t = q[c] - (double)row[c];
            s += t * t;
          }
          dist[j] = s;
        }
        if (fill < kk) {
          for (int j = 0; j < nb; ++j) {
            pair_t* h = heaps + (size_t)j * kk;
            h[fill].d = dist[j];
            h[fill].i = r;
          }
          ++fill;
          if (fill == kk)
            for (int j = 0; j < nb; ++j)
              for (int p = kk / 2 - 1; p >= 0; --p)
                heap_sift_down(heaps + (size_t)j * kk, kk, p);
        } else {
          for (int j = 0; j < nb; ++j) {
            pair_t* h = heaps + (size_t)j * kk;
            pair_t cand = {dist[j], r};
            if (pair_gt(h[0], cand)) {
              h[0] = cand;
              heap_sift_down(h, kk, 0);
            }
          }
        }
      }
      for (int j = 0; j < nb; ++j) {
        pair_t* h = heaps + (size_t)j * kk;
        qsort(h, (size_t)kk, sizeof(pair_t), cmp_pair);
        int64_t q = q0 + j;
        for (int t = 0; t < k; ++t) {
          if (t < kk) {
            out_idx[q * k + t] = h[t].i;
            out_dist[q * k + t] = h[t].d;
          } else {
            out_idx[q * k + t] = -1;
            out_dist[q * k + t] = (double)FLT_MAX;
          }
        }
      }
    }
    free(heaps);
    free(qd);
  }
  return err ? -1 : 0;
}

/*
 * The reference's own FP32 distance for given (query, base) pairs:
 *   ||q||^2 + (||x||^2 + (-2 q.x))   with every term in FP32,
 * the evaluation order of search.cu:176-197 (SGEMM alpha=-2, then
 * select.cu:208 adds ||x||^2, then broadcast.cu:36 adds ||q||^2).  The dot
 * product is accumulated sequentially here; cuBLAS may order it differently,
 * so this is a model of the reference's rounding, not a bit-exact replay.
 */
void oracle_ref_formula(const float* base, const float* queries, int32_t d,
                        const int64_t* qi, const int64_t* bi, int64_t npairs,
                        float* out) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npairs; ++p) {
    const float* q = queries + qi[p] * (int64_t)d;
    const float* x = base + bi[p] * (int64_t)d;
    float qn = 0.f, xn = 0.f, dot = 0.f;
    for (int32_t c = 0; c < d; ++c) {
      qn += q[c] * q[c];
      xn += x[c] * x[c];
      dot += q[c] * x[c];
    }
    out[p] = qn + (xn + (-2.0f * dot));
  }
}
