/*
 * hml_oracle.c -- CPU oracle for the skinny SGEMM/SGEMV path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only the tests, the smoke check and the benchmark's CPU
 * baseline leg do, and only as the checker.
 *
 * Contents
 *   oracle_sgemm_rm_f32   restatement of the reference CPU verification loop
 *                         hmlSgemmCpu (apps/gemm/hml_sgemm_main.cu:260-292):
 *                         row-major NN, FP32 accumulator, i-j-e loop order,
 *                         one thread.  Compiled without FMA contraction so it
 *                         rounds exactly like the reference build.
 *   oracle_sgemv_rm_f32   restatement of hmlSgemvCpu
 *                         (apps/gemv/hml_sgemv_main.cu:254-283).
 *   oracle_csum           restatement of hmlComputeCsum
 *                         (apps/gemm/hml_sgemm_main.cu:294-305) and of
 *                         hmlComputeYsum (apps/gemv/hml_sgemv_main.cu:285-292,
 *                         the N == 1 case): a double sum of all outputs.
 *   oracle_dgemm_strided  FP64 GEMM over arbitrary element strides (covers
 *                         column-major, row-major and both transposes), with
 *                         an optional |A||B| output for componentwise error
 *                         bounds.  Multithreaded with pthreads.  This is new
 *                         code: the reference has no FP64 path.
 *
 * Parity pin: the FP32 restatements are compared bit for bit against the
 * reference's own loops compiled from its sources (oracle/Makefile builds
 * them into oracle/_ref) and against the committed fixtures that those loops
 * produced (tests/golden/).
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* C = alpha * A * B + beta * C, all row-major, A is M x K, B is K x N.
 * Follows apps/gemm/hml_sgemm_main.cu:276-285: for each row i and column j
 * a float sum over e in increasing order, then alpha * sum + beta * C. */
void oracle_sgemm_rm_f32(float *C, const float *A, const float *B, int M,
                         int N, int K, float alpha, float beta) {
  for (int i = 0; i < M; ++i, A += K, C += N) {
    for (int j = 0; j < N; ++j) {
      const float *colB = B + j;
      float sum = 0.0f;
      for (int e = 0; e < K; ++e) {
        sum += A[e] * colB[(size_t)e * N];
      }
      C[j] = alpha * sum + beta * C[j];
    }
  }
}

/* y = alpha * A * x + beta * y, A row-major M x N.
 * Follows apps/gemv/hml_sgemv_main.cu:268-276. */
void oracle_sgemv_rm_f32(float *y, const float *A, const float *x, int M,
                         int N, float alpha, float beta) {
  for (int i = 0; i < M; ++i, A += N) {
    float ax = 0.0f;
    for (int j = 0; j < N; ++j) ax += A[j] * x[j];
    y[i] = alpha * ax + beta * y[i];
  }
}

/* Double checksum of an M x N float array, row-major order of summation
 * (apps/gemm/hml_sgemm_main.cu:294-305). */
double oracle_csum(const float *C, int M, int N) {
  double s = 0.0;
  for (int i = 0; i < M; i++)
    for (int j = 0; j < N; j++) s += (double)C[(size_t)i * N + j];
  return s;
}

/* ------------------------------------------------------------------------ */
/* FP64 GEMM over element strides.
 *   A(m,k) = A[m*sam + k*sak]   B(k,n) = B[k*sbk + n*sbn]
 *   C(m,n) = C[m*scm + n*scn]   (read only when beta != 0 and C != NULL)
 *   D(m,n) = D[m + n*M]         (dense column-major double output)
 *   absD(m,n) = sum_k |A(m,k)| |B(k,n)|  (optional)
 * D = alpha * sum_k A(m,k) B(k,n) + beta * C(m,n), every product and sum in
 * double.  Strides are in elements and may be any non-negative value.    */
typedef struct {
  int M, N, K;
  double alpha, beta;
  const float *A, *B, *C;
  int64_t sam, sak, sbk, sbn, scm, scn;
  double *D, *absD;
  int n0, n1; /* column range for this worker */
} dgemm_job;

static void *dgemm_worker(void *p) {
  dgemm_job *j = (dgemm_job *)p;
  const int M = j->M, K = j->K;
  double *acc = (double *)malloc(sizeof(double) * (size_t)M * 2);
  double *aacc = acc + M;
  for (int n = j->n0; n < j->n1; ++n) {
    for (int m = 0; m < M; ++m) acc[m] = aacc[m] = 0.0;
    if (j->sam == 1) {
      /* unit stride along m: axpy form, vectorises */
      for (int k = 0; k < K; ++k) {
        const double b = (double)j->B[(int64_t)k * j->sbk + (int64_t)n * j->sbn];
        const double ab = b < 0 ? -b : b;
        const float *a = j->A + (int64_t)k * j->sak;
        if (j->absD) {
          for (int m = 0; m < M; ++m) {
            double av = (double)a[m];
            acc[m] += av * b;
            aacc[m] += (av < 0 ? -av : av) * ab;
          }
        } else {
          for (int m = 0; m < M; ++m) acc[m] += (double)a[m] * b;
        }
      }
    } else {
      /* dot form */
      for (int m = 0; m < M; ++m) {
        const float *a = j->A + (int64_t)m * j->sam;
        double s = 0.0, sa = 0.0;
        for (int k = 0; k < K; ++k) {
          double av = (double)a[(int64_t)k * j->sak];
          double bv = (double)j->B[(int64_t)k * j->sbk + (int64_t)n * j->sbn];
          s += av * bv;
          sa += (av < 0 ? -av : av) * (bv < 0 ? -bv : bv);
        }
        acc[m] = s;
        aacc[m] = sa;
      }
    }
    for (int m = 0; m < M; ++m) {
      double c = 0.0;
      if (j->beta != 0.0 && j->C)
        c = (double)j->C[(int64_t)m * j->scm + (int64_t)n * j->scn];
      j->D[(int64_t)m + (int64_t)n * M] = j->alpha * acc[m] + j->beta * c;
      if (j->absD) {
        double aa = j->alpha < 0 ? -j->alpha : j->alpha;
        double ab = j->beta < 0 ? -j->beta : j->beta;
        j->absD[(int64_t)m + (int64_t)n * M] =
            aa * aacc[m] + ab * (c < 0 ? -c : c);
      }
    }
  }
  free(acc);
  return NULL;
}

int oracle_dgemm_strided(int M, int N, int K, double alpha, const float *A,
                         int64_t sam, int64_t sak, const float *B, int64_t sbk,
                         int64_t sbn, double beta, const float *C, int64_t scm,
                         int64_t scn, double *D, double *absD, int threads) {
  if (M < 0 || N < 0 || K < 0) return 1;
  if (M == 0 || N == 0) return 0;
  if (threads < 1) threads = 1;
  if (threads > N) threads = N;
  if (threads > 256) threads = 256;
  pthread_t tid[256];
  dgemm_job jobs[256];
  for (int t = 0; t < threads; ++t) {
    dgemm_job *j = &jobs[t];
    j->M = M; j->N = N; j->K = K;
    j->alpha = alpha; j->beta = beta;
    j->A = A; j->B = B; j->C = C;
    j->sam = sam; j->sak = sak; j->sbk = sbk; j->sbn = sbn;
    j->scm = scm; j->scn = scn;
    j->D = D; j->absD = absD;
    j->n0 = (int)((int64_t)N * t / threads);
    j->n1 = (int)((int64_t)N * (t + 1) / threads);
  }
  for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, dgemm_worker, &jobs[t]);
  dgemm_worker(&jobs[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
  return 0;
}

/* Multithreaded row-major FP32 GEMM with the reference loop's per-output
 * summation order (same result as oracle_sgemm_rm_f32, bit for bit); used to
 * time a larger CPU baseline sample on several cores. */
typedef struct {
  float *C; const float *A, *B; int M, N, K; float alpha, beta; int i0, i1;
} sgemm_job;

static void *sgemm_worker(void *p) {
  sgemm_job *j = (sgemm_job *)p;
  oracle_sgemm_rm_f32(j->C + (size_t)j->i0 * j->N, j->A + (size_t)j->i0 * j->K,
                      j->B, j->i1 - j->i0, j->N, j->K, j->alpha, j->beta);
  return NULL;
}

int oracle_sgemm_rm_f32_mt(float *C, const float *A, const float *B, int M,
                           int N, int K, float alpha, float beta, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads > M) threads = M > 0 ? M : 1;
  pthread_t tid[256];
  sgemm_job jobs[256];
  for (int t = 0; t < threads; ++t) {
    sgemm_job *j = &jobs[t];
    j->C = C; j->A = A; j->B = B; j->M = M; j->N = N; j->K = K;
    j->alpha = alpha; j->beta = beta;
    j->i0 = (int)((int64_t)M * t / threads);
    j->i1 = (int)((int64_t)M * (t + 1) / threads);
  }
  for (int t = 1; t < threads; ++t) pthread_create(&tid[t], NULL, sgemm_worker, &jobs[t]);
  sgemm_worker(&jobs[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tid[t], NULL);
  return 0;
}

/* k-means assignment with the arithmetic of the reference's GPU kernel
 * hmlKmeansAssignCtrdSmem (include/hml_kmeans_kernel_template.h:19-90):
 * dist = sum over d, in order, of delta * delta with delta = x - c, each step
 * one fused multiply-add (what nvcc makes of `dist += delta * delta`), from
 * 0; the first k whose dist is below the running minimum (from FLT_MAX)
 * wins.  A point none of whose distances is below FLT_MAX (NaN or infinite
 * ones) gets 0 here; the reference kernel leaves its minK unset for such a
 * point (:30, :74), so its output there is whatever the register held.
 * points [n][d], centroids [k][d], row-major. */
void oracle_kmeans_assign(const float *points, int64_t n, int d, const float *ctrds, int k,
                          uint32_t *out) {
  for (int64_t p = 0; p < n; ++p) {
    const float *x = points + p * d;
    float min_dist = FLT_MAX;
    uint32_t min_k = 0;
    for (int c = 0; c < k; ++c) {
      const float *cc = ctrds + (int64_t)c * d;
      float dist = 0.0f;
      for (int j = 0; j < d; ++j) {
        const float delta = x[j] - cc[j];
        dist = fmaf(delta, delta, dist);
      }
      if (dist < min_dist) {
        min_dist = dist;
        min_k = (uint32_t)c;
      }
    }
    out[p] = min_k;
  }
}
