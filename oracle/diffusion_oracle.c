/*
 * ORACLE — test infrastructure only (see diffusion_oracle.h). Plain-C
 * restatement of scl-core's diffusion path; each function cites the
 * reference lines it follows. Compiled with -ffp-contract=off: the only fused
 * multiply-adds are the explicit fma()/fmaf() calls, placed where the
 * reference multiplies-and-accumulates through Highway MulAdd or a contracted
 * `y += a*x` (GCC contracts those at -O3 in the reference's C++20 build).
 */
#include "diffusion_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MIN_PROB 1e-15           /* diffusion.hpp:41 config::MIN_PROB */
#define MIN_BANDWIDTH 1e-10      /* kernel.hpp:28 config::MIN_BANDWIDTH */
#define DEFAULT_BANDWIDTH 1.0    /* kernel.hpp:27 config::DEFAULT_BANDWIDTH */

/* ===================================================================== */
/* Row sums — diffusion.hpp:452-484: sequential `sum += v` in Real.        */
/* ===================================================================== */
void oracle_row_sums_f32(int64_t n, const int64_t* indptr, const float* values, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    float s = 0.0f;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) s += values[p];
    out[i] = s;
  }
}

void oracle_row_sums_f64(int64_t n, const int64_t* indptr, const double* values, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) s += values[p];
    out[i] = s;
  }
}

/* ===================================================================== */
/* Transition matrix — diffusion.hpp:492-603.                              */
/*   row:  inv = d > 1e-15 ? 1/d : 0;           v *= inv          (565-600) */
/*   sym:  a_i = d > 1e-15 ? 1/sqrt(d) : 0;     v *= a_i * a_j    (508-564) */
/* ===================================================================== */
void oracle_transition_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                           float* values, int symmetric, int degree_fp64) {
  if (!degree_fp64) {
    float* d = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    oracle_row_sums_f32(n, indptr, values, d);
    if (symmetric) {
      float* a = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
      for (int64_t i = 0; i < n; ++i) a[i] = (d[i] > (float)MIN_PROB) ? 1.0f / sqrtf(d[i]) : 0.0f;
      for (int64_t i = 0; i < n; ++i) {
        const float ai = a[i];
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
          const float s = ai * a[indices[p]];
          values[p] = values[p] * s;
        }
      }
      free(a);
    } else {
      for (int64_t i = 0; i < n; ++i) {
        const float inv = (d[i] > (float)MIN_PROB) ? 1.0f / d[i] : 0.0f;
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) values[p] = values[p] * inv;
      }
    }
    free(d);
    return;
  }
  /* FP64 degrees: sequential double sums, double scale, one rounding. */
  double* d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) s += (double)values[p];
    d[i] = s;
  }
  if (symmetric) {
    double* a = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) a[i] = (d[i] > MIN_PROB) ? 1.0 / sqrt(d[i]) : 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double ai = a[i];
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const double s = ai * a[indices[p]];
        values[p] = (float)((double)values[p] * s);
      }
    }
    free(a);
  } else {
    for (int64_t i = 0; i < n; ++i) {
      const double inv = (d[i] > MIN_PROB) ? 1.0 / d[i] : 0.0;
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p)
        values[p] = (float)((double)values[p] * inv);
    }
  }
  free(d);
}

void oracle_transition_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                           double* values, int symmetric) {
  double* d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  oracle_row_sums_f64(n, indptr, values, d);
  if (symmetric) {
    double* a = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) a[i] = (d[i] > MIN_PROB) ? 1.0 / sqrt(d[i]) : 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double ai = a[i];
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const double s = ai * a[indices[p]];
        values[p] = values[p] * s;
      }
    }
    free(a);
  } else {
    for (int64_t i = 0; i < n; ++i) {
      const double inv = (d[i] > MIN_PROB) ? 1.0 / d[i] : 0.0;
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) values[p] = values[p] * inv;
    }
  }
  free(d);
}

/* ===================================================================== */
/* SpMM — diffusion.hpp:227-278 + axpy_simd 100-134.                       */
/* Y[i,:] = 0; for each stored (j, v) of row i in order: Y[i,c] = fma(v, X[j,c], Y[i,c]) */
/* ===================================================================== */
void oracle_spmm_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                     const float* values, const float* X, float* Y, int64_t F) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    float* yi = Y + i * F;
    for (int64_t c = 0; c < F; ++c) yi[c] = 0.0f;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const float v = values[p];
      const float* xj = X + indices[p] * F;
      for (int64_t c = 0; c < F; ++c) yi[c] = fmaf(v, xj[c], yi[c]);
    }
  }
}

void oracle_spmm_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                     const double* values, const double* X, double* Y, int64_t F) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    double* yi = Y + i * F;
    for (int64_t c = 0; c < F; ++c) yi[c] = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const double v = values[p];
      const double* xj = X + indices[p] * F;
      for (int64_t c = 0; c < F; ++c) yi[c] = fma(v, xj[c], yi[c]);
    }
  }
}

/* diffusion.hpp:638-664: X_new = P X; X <- X_new, steps times. */
void oracle_diffuse_matrix_f32(int64_t n, const int64_t* indptr, const int64_t* indices,
                               const float* values, float* X, int64_t F, int64_t steps) {
  float* tmp = (float*)malloc(sizeof(float) * (size_t)(n * F > 0 ? n * F : 1));
  for (int64_t s = 0; s < steps; ++s) {
    oracle_spmm_f32(n, indptr, indices, values, X, tmp, F);
    memcpy(X, tmp, sizeof(float) * (size_t)(n * F));
  }
  free(tmp);
}

void oracle_diffuse_matrix_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                               const double* values, double* X, int64_t F, int64_t steps) {
  double* tmp = (double*)malloc(sizeof(double) * (size_t)(n * F > 0 ? n * F : 1));
  for (int64_t s = 0; s < steps; ++s) {
    oracle_spmm_f64(n, indptr, indices, values, X, tmp, F);
    memcpy(X, tmp, sizeof(double) * (size_t)(n * F));
  }
  free(tmp);
}

/* ===================================================================== */
/* Low-precision storage (new in this project).                            */
/* ===================================================================== */
static uint32_t f32_bits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static float bits_f32(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* bfloat16 = top 16 bits of binary32, round to nearest even. */
uint16_t oracle_f32_to_bf16(float x) {
  uint32_t u = f32_bits(x);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x0040u); /* quiet NaN */
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}

float oracle_bf16_to_f32(uint16_t h) { return bits_f32(((uint32_t)h) << 16); }

/* IEEE binary16: 1 sign, 5 exponent (bias 15), 10 fraction bits; RNE. */
uint16_t oracle_f32_to_f16(float x) {
  const uint32_t u = f32_bits(x);
  const uint16_t sign = (uint16_t)((u >> 16) & 0x8000u);
  const uint32_t absu = u & 0x7fffffffu;
  if (absu > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);           /* NaN */
  if (absu >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);          /* >= 65520 rounds to inf */
  const int32_t e = (int32_t)(absu >> 23) - 127;                        /* unbiased exponent */
  uint32_t mant = (absu & 0x7fffffu) | 0x800000u;                       /* 24-bit significand */
  if (absu < 0x33000001u) return sign;                                 /* < 2^-25 (+tie) -> 0 */
  if (e < -14) {
    /* subnormal half: value = mant * 2^(e-23); half unit = 2^-24 */
    const int shift = (-14 - e) + 13;                                   /* bits to drop */
    const uint32_t keep = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1);
    uint32_t r = keep + ((rem > half || (rem == half && (keep & 1u))) ? 1u : 0u);
    return (uint16_t)(sign | r);
  }
  /* normal: drop 13 fraction bits with RNE; carry may bump the exponent. */
  uint32_t he = (uint32_t)(e + 15);
  uint32_t keep = (mant >> 13);
  const uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (keep & 1u))) keep += 1u;
  if (keep == 0x800u) { keep = 0x400u; he += 1u; }
  if (he >= 31u) return (uint16_t)(sign | 0x7c00u);
  return (uint16_t)(sign | (he << 10) | (keep & 0x3ffu));
}

float oracle_f16_to_f32(uint16_t h) {
  const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
  const uint32_t e = ((uint32_t)h >> 10) & 0x1fu;
  const uint32_t m = (uint32_t)h & 0x3ffu;
  if (e == 0) {
    const float v = (float)m * 5.9604644775390625e-08f; /* m * 2^-24, exact */
    return sign ? -v : v;
  }
  if (e == 31) return bits_f32(sign | 0x7f800000u | (m << 13));
  return bits_f32(sign | ((e + 112u) << 23) | (m << 13));
}

static float lowp_round(float x, int kind) {
  if (kind == ORACLE_BF16) return oracle_bf16_to_f32(oracle_f32_to_bf16(x));
  if (kind == ORACLE_F16) return oracle_f16_to_f32(oracle_f32_to_f16(x));
  return x;
}

void oracle_diffuse_lowp(int64_t n, const int64_t* indptr, const int64_t* indices,
                         const float* values_f32, const float* X0_f32, float* Y_out,
                         int64_t F, int64_t steps, int kind, int final_f32) {
  const int64_t nnz = indptr[n];
  float* v = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
  float* a = (float*)malloc(sizeof(float) * (size_t)(n * F > 0 ? n * F : 1));
  float* b = (float*)malloc(sizeof(float) * (size_t)(n * F > 0 ? n * F : 1));
  for (int64_t p = 0; p < nnz; ++p) v[p] = lowp_round(values_f32[p], kind);
  for (int64_t q = 0; q < n * F; ++q) a[q] = lowp_round(X0_f32[q], kind);
  for (int64_t s = 0; s < steps; ++s) {
    oracle_spmm_f32(n, indptr, indices, v, a, b, F);
    const int last = (s == steps - 1);
    if (!(last && final_f32))
      for (int64_t q = 0; q < n * F; ++q) b[q] = lowp_round(b[q], kind);
    float* t = a; a = b; b = t;
  }
  memcpy(Y_out, a, sizeof(float) * (size_t)(n * F));
  free(v); free(a); free(b);
}

/* Interleaved-chain form of the 16-bit storage diffusion. The B200 kernel for
 * bf16/f16 storage gathers Q entries per load instruction (Q = 32 lanes /
 * lanes per row): chain q (0 <= q < Q) is the sequential fma over the row's
 * entries q, q+Q, q+2Q, ... in stored order, and the chains are summed
 * pairwise over the bits of q from the lowest: Q=2 -> c0+c1,
 * Q=4 -> (c0+c1)+(c2+c3). Q=1 is oracle_diffuse_lowp. Same rounding of the
 * stored values and iterates as oracle_diffuse_lowp. */
static void spmm_f32_chains(int64_t n, const int64_t* indptr, const int64_t* indices,
                            const float* v, const float* X, float* Y, int64_t F, int Q) {
  float c[32];
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t col = 0; col < F; ++col) {
      for (int q = 0; q < Q; ++q) c[q] = 0.0f;
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const int q = (int)((p - indptr[i]) % Q);
        c[q] = fmaf(v[p], X[indices[p] * F + col], c[q]);
      }
      for (int w = 1; w < Q; w <<= 1)
        for (int q = 0; q < Q; q += 2 * w) c[q] = c[q] + c[q + w];
      Y[i * F + col] = c[0];
    }
  }
}

void oracle_diffuse_lowp_chains(int64_t n, const int64_t* indptr, const int64_t* indices,
                                const float* values_f32, const float* X0_f32, float* Y_out,
                                int64_t F, int64_t steps, int kind, int final_f32, int chains) {
  const int64_t nnz = indptr[n];
  float* v = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
  float* a = (float*)malloc(sizeof(float) * (size_t)(n * F > 0 ? n * F : 1));
  float* b = (float*)malloc(sizeof(float) * (size_t)(n * F > 0 ? n * F : 1));
  for (int64_t p = 0; p < nnz; ++p) v[p] = lowp_round(values_f32[p], kind);
  for (int64_t q = 0; q < n * F; ++q) a[q] = lowp_round(X0_f32[q], kind);
  for (int64_t s = 0; s < steps; ++s) {
    spmm_f32_chains(n, indptr, indices, v, a, b, F, chains);
    const int last = (s == steps - 1);
    if (!(last && final_f32))
      for (int64_t q = 0; q < n * F; ++q) b[q] = lowp_round(b[q], kind);
    float* t = a; a = b; b = t;
  }
  memcpy(Y_out, a, sizeof(float) * (size_t)(n * F));
  free(v); free(a); free(b);
}

/* ===================================================================== */
/* Graph build: Gaussian weights (kernel.hpp:403-453 sigma = max of the     */
/* first k stored distances, floored at MIN_BANDWIDTH; w = exp(-(d/s)^2)).  */
/* ===================================================================== */
void oracle_gauss_weights_f64(int64_t n, int64_t k, const int64_t* knn_idx,
                              const double* knn_dist, double* sigma, double* w) {
  for (int64_t i = 0; i < n; ++i) {
    double mx = 0.0;
    int any = 0;
    for (int64_t m = 0; m < k; ++m) {
      if (knn_idx[i * k + m] < 0) continue;
      any = 1;
      const double d = knn_dist[i * k + m];
      mx = (mx < d) ? d : mx;
    }
    const double s = any ? ((mx < MIN_BANDWIDTH) ? MIN_BANDWIDTH : mx) : DEFAULT_BANDWIDTH;
    sigma[i] = s;
    for (int64_t m = 0; m < k; ++m) {
      if (knn_idx[i * k + m] < 0) { w[i * k + m] = 0.0; continue; }
      const double q = knn_dist[i * k + m] / s;
      w[i * k + m] = exp(-(q * q));
    }
  }
}

void oracle_gauss_weights_f32(int64_t n, int64_t k, const int64_t* knn_idx,
                              const float* knn_dist, float* sigma, float* w) {
  for (int64_t i = 0; i < n; ++i) {
    float mx = 0.0f;
    int any = 0;
    for (int64_t m = 0; m < k; ++m) {
      if (knn_idx[i * k + m] < 0) continue;
      any = 1;
      const float d = knn_dist[i * k + m];
      mx = (mx < d) ? d : mx;
    }
    const float s = any ? ((mx < (float)MIN_BANDWIDTH) ? (float)MIN_BANDWIDTH : mx) : (float)DEFAULT_BANDWIDTH;
    sigma[i] = s;
    for (int64_t m = 0; m < k; ++m) {
      if (knn_idx[i * k + m] < 0) { w[i * k + m] = 0.0f; continue; }
      const float q = knn_dist[i * k + m] / s;
      w[i * k + m] = expf(-(q * q));
    }
  }
}

/* ===================================================================== */
/* (W + W^T)/2 union. Transposed lists are built stably (source rows in     */
/* increasing order), out-lists sorted by column, then merged per row.      */
/* ===================================================================== */
typedef struct { int64_t col; int64_t pos; } ColPos;

static int cmp_colpos(const void* a, const void* b) {
  const ColPos* x = (const ColPos*)a;
  const ColPos* y = (const ColPos*)b;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos ? 1 : 0);
}

#define DEFINE_SYMMETRIZE(SUFFIX, T)                                                         \
  int64_t oracle_symmetrize_##SUFFIX(int64_t n, int64_t k, const int64_t* knn_idx,           \
                                     const T* w, int64_t* indptr, int64_t* indices,           \
                                     T* values) {                                             \
    /* in-lists: for every valid (i, j=idx[i,m]) an entry (row j, col i, w) */                \
    int64_t* in_ptr = (int64_t*)calloc((size_t)(n + 1), sizeof(int64_t));                     \
    for (int64_t q = 0; q < n * k; ++q)                                                       \
      if (knn_idx[q] >= 0) in_ptr[knn_idx[q] + 1]++;                                          \
    for (int64_t i = 0; i < n; ++i) in_ptr[i + 1] += in_ptr[i];                               \
    const int64_t n_in = in_ptr[n];                                                           \
    int64_t* in_col = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_in > 0 ? n_in : 1));      \
    T* in_w = (T*)malloc(sizeof(T) * (size_t)(n_in > 0 ? n_in : 1));                          \
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));               \
    for (int64_t i = 0; i < n; ++i) cur[i] = in_ptr[i];                                       \
    for (int64_t i = 0; i < n; ++i)                                                           \
      for (int64_t m = 0; m < k; ++m) {                                                       \
        const int64_t j = knn_idx[i * k + m];                                                 \
        if (j < 0) continue;                                                                  \
        in_col[cur[j]] = i;                                                                   \
        in_w[cur[j]] = w[i * k + m];                                                          \
        cur[j]++;                                                                             \
      }                                                                                       \
    ColPos* outl = (ColPos*)malloc(sizeof(ColPos) * (size_t)(k > 0 ? k : 1));                 \
    int64_t nnz = 0;                                                                          \
    if (indptr) indptr[0] = 0;                                                                \
    for (int64_t i = 0; i < n; ++i) {                                                         \
      int64_t no = 0;                                                                         \
      for (int64_t m = 0; m < k; ++m)                                                         \
        if (knn_idx[i * k + m] >= 0) {                                                        \
          outl[no].col = knn_idx[i * k + m];                                                  \
          outl[no].pos = i * k + m;                                                           \
          no++;                                                                               \
        }                                                                                     \
      qsort(outl, (size_t)no, sizeof(ColPos), cmp_colpos);                                    \
      int64_t a = 0, b = in_ptr[i];                                                           \
      const int64_t be = in_ptr[i + 1];                                                       \
      while (a < no || b < be) {                                                              \
        int64_t c;                                                                            \
        if (b >= be || (a < no && outl[a].col <= in_col[b])) c = outl[a].col;                 \
        else c = in_col[b];                                                                   \
        T so = (T)0, si = (T)0;                                                               \
        while (a < no && outl[a].col == c) { so += w[outl[a].pos]; a++; }                     \
        while (b < be && in_col[b] == c) { si += in_w[b]; b++; }                              \
        if (indices) {                                                                        \
          indices[nnz] = c;                                                                   \
          values[nnz] = (T)0.5 * (so + si);                                                   \
        }                                                                                     \
        nnz++;                                                                                \
      }                                                                                       \
      if (indptr) indptr[i + 1] = nnz;                                                        \
    }                                                                                         \
    free(outl); free(cur); free(in_w); free(in_col); free(in_ptr);                            \
    return nnz;                                                                               \
  }

DEFINE_SYMMETRIZE(f64, double)
DEFINE_SYMMETRIZE(f32, float)

/* ===================================================================== */
/* FP64 adjoint of L = sum((X_T - Y)^2), X_{s+1} = P X_s, P = normalise(W). */
/*   G_T = 2 (X_T - Y);  G_s = P^T G_{s+1};  gP_ij = sum_s G_{s+1}[i].X_s[j] */
/*   row:  dW_ij = (gP_ij - u_i) / d_i,          u_i = sum_c gP_ic P_ic       */
/*   sym:  dW_ij = gP_ij a_i a_j - (u_i + v_i) / (2 d_i),                     */
/*         v_i = sum_r gP_ri P_ri (column sums), a = d^-1/2                   */
/* ===================================================================== */
double oracle_adjoint_f64(int64_t n, const int64_t* indptr, const int64_t* indices,
                          const double* W, int symmetric, const double* X0, const double* Y,
                          int64_t F, int64_t steps, double* dX0, double* dW) {
  const int64_t nnz = indptr[n];
  const size_t nf = (size_t)(n * F);
  double* P = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  double* d = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  memcpy(P, W, sizeof(double) * (size_t)nnz);
  oracle_row_sums_f64(n, indptr, W, d);
  oracle_transition_f64(n, indptr, indices, P, symmetric);

  double* Xs = (double*)malloc(sizeof(double) * nf * (size_t)(steps + 1));
  memcpy(Xs, X0, sizeof(double) * nf);
  for (int64_t s = 0; s < steps; ++s)
    oracle_spmm_f64(n, indptr, indices, P, Xs + (size_t)s * nf, Xs + (size_t)(s + 1) * nf, F);

  const double* XT = Xs + (size_t)steps * nf;
  double loss = 0.0;
  double* G = (double*)malloc(sizeof(double) * nf);
  double* Gn = (double*)malloc(sizeof(double) * nf);
  for (size_t q = 0; q < nf; ++q) {
    const double r = XT[q] - Y[q];
    loss += r * r;
    G[q] = 2.0 * r;
  }
  double* gP = (double*)calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
  for (int64_t s = steps - 1; s >= 0; --s) {
    const double* X = Xs + (size_t)s * nf;
    memset(Gn, 0, sizeof(double) * nf);
    for (int64_t i = 0; i < n; ++i) {
      const double* gi = G + i * F;
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
        const int64_t j = indices[p];
        const double* xj = X + j * F;
        double dot = 0.0;
        for (int64_t c = 0; c < F; ++c) dot += gi[c] * xj[c];
        gP[p] += dot;
        double* gj = Gn + j * F;
        for (int64_t c = 0; c < F; ++c) gj[c] += P[p] * gi[c];
      }
    }
    double* t = G; G = Gn; Gn = t;
  }
  memcpy(dX0, G, sizeof(double) * nf);

  double* u = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double* v = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  for (int64_t i = 0; i < n; ++i)
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      u[i] += gP[p] * P[p];
      v[indices[p]] += gP[p] * P[p];
    }
  for (int64_t i = 0; i < n; ++i) {
    if (!(d[i] > MIN_PROB)) {
      for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) dW[p] = 0.0;
      continue;
    }
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      if (symmetric) {
        const int64_t j = indices[p];
        const double ai = 1.0 / sqrt(d[i]);
        const double aj = (d[j] > MIN_PROB) ? 1.0 / sqrt(d[j]) : 0.0;
        dW[p] = gP[p] * ai * aj - (u[i] + v[i]) / (2.0 * d[i]);
      } else {
        dW[p] = (gP[p] - u[i]) / d[i];
      }
    }
  }
  free(u); free(v); free(gP); free(G); free(Gn); free(Xs); free(P); free(d);
  return loss;
}

/* (P x)_i in the walks' order: 32 partial fma chains over the entries  */
/* l, l+32, ... of the row, combined by the xor butterfly 16, 8, 4, 2, 1 */
/* (every lane of a warp ends with the same value; lane 0's is used).   */
static float warp_dot_f32(const int64_t* indptr, const int64_t* indices, const float* values, const float* x,
                          int64_t i) {
  float part[32], nxt[32];
  for (int l = 0; l < 32; ++l) {
    float s = 0.0f;
    for (int64_t p = indptr[i] + l; p < indptr[i + 1]; p += 32) s = fmaf(values[p], x[indices[p]], s);
    part[l] = s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int l = 0; l < 32; ++l) nxt[l] = part[l] + part[l ^ o];
    memcpy(part, nxt, sizeof(part));
  }
  return part[0];
}

static double warp_dot_f64(const int64_t* indptr, const int64_t* indices, const double* values, const double* x,
                           int64_t i) {
  double part[32], nxt[32];
  for (int l = 0; l < 32; ++l) {
    double s = 0.0;
    for (int64_t p = indptr[i] + l; p < indptr[i + 1]; p += 32) s = fma(values[p], x[indices[p]], s);
    part[l] = s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int l = 0; l < 32; ++l) nxt[l] = part[l] + part[l ^ o];
    memcpy(part, nxt, sizeof(part));
  }
  return part[0];
}

/* ===================================================================== */
/* Vector walks — diffusion.hpp:833-900 (random walk with restart),       */
/* 961-1007 (heat-kernel signature), 1157-1194 (lazy random walk), on    */
/* spmv_parallel (169-221). Each (P x)_i is formed in the warp order of  */
/* warp_dot_*; the step's combination is rounded as                      */
/*   lazy / heat kernel: y = fma(c_x, x, c_p * (P x))                     */
/*   restart:            y = fma(alpha, (P x), (1 - alpha) * r)           */
/* The restart walk's convergence sum is sum |y - x| (differences in the */
/* value type, summed in double in row order) and stops when it is below */
/* tol; buffers swap after every step that has not converged, so the    */
/* caller's array ends with the last iterate written into it.           */
/* ===================================================================== */
void oracle_walk_linear_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values, float* x,
                            int64_t steps, float cx, float cp) {
  float* y = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  for (int64_t st = 0; st < steps; ++st) {
    for (int64_t i = 0; i < n; ++i) {
      const float s = warp_dot_f32(indptr, indices, values, x, i);
      y[i] = fmaf(cx, x[i], cp * s);
    }
    memcpy(x, y, sizeof(float) * (size_t)n);
  }
  free(y);
}

void oracle_walk_linear_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values, double* x,
                            int64_t steps, double cx, double cp) {
  double* y = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int64_t st = 0; st < steps; ++st) {
    for (int64_t i = 0; i < n; ++i) {
      const double s = warp_dot_f64(indptr, indices, values, x, i);
      y[i] = fma(cx, x[i], cp * s);
    }
    memcpy(x, y, sizeof(double) * (size_t)n);
  }
  free(y);
}

int64_t oracle_walk_restart_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values,
                                const float* r, float* scores, float alpha, int64_t max_iter, float tol) {
  float* tmp = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  float* cur = scores;
  float* nxt = tmp;
  const float beta = 1.0f - alpha;
  int64_t it = 0;
  for (; it < max_iter; ++it) {
    double l1 = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const float s = warp_dot_f32(indptr, indices, values, cur, i);
      const float y = fmaf(alpha, s, beta * r[i]);
      const float d = y - cur[i];
      l1 += (double)(d >= 0.0f ? d : -d);
      nxt[i] = y;
    }
    if (l1 < (double)tol) {
      memcpy(cur, nxt, sizeof(float) * (size_t)n);
      ++it;
      break;
    }
    float* t = cur;
    cur = nxt;
    nxt = t;
  }
  free(tmp);
  return it;
}

int64_t oracle_walk_restart_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values,
                                const double* r, double* scores, double alpha, int64_t max_iter, double tol) {
  double* tmp = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* cur = scores;
  double* nxt = tmp;
  const double beta = 1.0 - alpha;
  int64_t it = 0;
  for (; it < max_iter; ++it) {
    double l1 = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double s = warp_dot_f64(indptr, indices, values, cur, i);
      const double y = fma(alpha, s, beta * r[i]);
      const double d = y - cur[i];
      l1 += (d >= 0.0 ? d : -d);
      nxt[i] = y;
    }
    if (l1 < tol) {
      memcpy(cur, nxt, sizeof(double) * (size_t)n);
      ++it;
      break;
    }
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  free(tmp);
  return it;
}

/* ===================================================================== */
/* Diffusion pseudotime — diffusion.hpp:670-772 (one root). p starts as   */
/* the root's indicator; each step p_new = P p (sequential fma chains),  */
/* then rows with visited < 0.99 and p_new > 1e-15 add                    */
/* new = p_new * (1 - visited) to visited (capped at 1) and              */
/* fma(step, new, hitting) to the hitting time; stop when the largest    */
/* 1 - visited is below tol. Visited rows (> 0.5) get hitting / visited  */
/* scaled by 1 / (largest such value), the others 1.                     */
/* ===================================================================== */
#define ORACLE_DPT_BODY(T, FMA)                                                                       \
  T* p = (T*)calloc((size_t)(n > 0 ? n : 1), sizeof(T));                                              \
  T* q = (T*)calloc((size_t)(n > 0 ? n : 1), sizeof(T));                                              \
  T* hit = (T*)calloc((size_t)(n > 0 ? n : 1), sizeof(T));                                            \
  T* vis = (T*)calloc((size_t)(n > 0 ? n : 1), sizeof(T));                                            \
  p[root] = (T)1;                                                                                     \
  vis[root] = (T)1;                                                                                   \
  for (int64_t it = 1; it <= max_iter; ++it) {                                                        \
    T mu = (T)0;                                                                                      \
    for (int64_t i = 0; i < n; ++i) {                                                                 \
      T s = (T)0;                                                                                     \
      for (int64_t k = indptr[i]; k < indptr[i + 1]; ++k) s = FMA(values[k], p[indices[k]], s);       \
      q[i] = s;                                                                                       \
      if (vis[i] < (T)0.99 && s > (T)1e-15) {                                                         \
        const T np = s * ((T)1 - vis[i]);                                                             \
        hit[i] = FMA((T)it, np, hit[i]);                                                              \
        T v = vis[i] + np;                                                                            \
        vis[i] = v < (T)1 ? v : (T)1;                                                                 \
      }                                                                                               \
      const T u = (T)1 - vis[i];                                                                      \
      mu = u > mu ? u : mu;                                                                           \
    }                                                                                                 \
    if (mu < tol) break;                                                                              \
    T* t = p;                                                                                         \
    p = q;                                                                                            \
    q = t;                                                                                            \
  }                                                                                                   \
  T mt = (T)0;                                                                                        \
  for (int64_t i = 0; i < n; ++i)                                                                     \
    if (vis[i] > (T)0.5) {                                                                            \
      hit[i] = hit[i] / vis[i];                                                                       \
      mt = hit[i] > mt ? hit[i] : mt;                                                                 \
    }                                                                                                 \
  const T inv = mt > (T)0 ? (T)1 / mt : (T)1;                                                         \
  for (int64_t i = 0; i < n; ++i) out[i] = vis[i] > (T)0.5 ? hit[i] * inv : (T)1;                     \
  free(p);                                                                                            \
  free(q);                                                                                            \
  free(hit);                                                                                          \
  free(vis);

void oracle_dpt_f32(int64_t n, const int64_t* indptr, const int64_t* indices, const float* values, int64_t root,
                    int64_t max_iter, float tol, float* out) {
  ORACLE_DPT_BODY(float, fmaf)
}

void oracle_dpt_f64(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values, int64_t root,
                    int64_t max_iter, double tol, double* out) {
  ORACLE_DPT_BODY(double, fma)
}

/* ===================================================================== */
/* General SpMM — scl/kernel/algebra.hpp:546-600 (scl_algebra_spmm):      */
/* Y <- beta Y (beta 0: zero, beta 1: untouched), then unless alpha is 0, */
/* for every stored entry in order w = a * alpha and, when w != 0,        */
/* y_row = fma(w, x_row, y_row).                                          */
/* ===================================================================== */
void oracle_algebra_spmm_f32(int64_t m, const int64_t* indptr, const int64_t* indices, const float* values,
                             const float* X, int64_t K, float* Y, float alpha, float beta) {
  for (int64_t i = 0; i < m * K; ++i) Y[i] = (beta == 0.0f) ? 0.0f : (beta == 1.0f ? Y[i] : Y[i] * beta);
  if (alpha == 0.0f) return;
  for (int64_t i = 0; i < m; ++i)
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const float w = values[p] * alpha;
      if (w == 0.0f) continue;
      const float* x = X + indices[p] * K;
      for (int64_t c = 0; c < K; ++c) Y[i * K + c] = fmaf(w, x[c], Y[i * K + c]);
    }
}

void oracle_algebra_spmm_f64(int64_t m, const int64_t* indptr, const int64_t* indices, const double* values,
                             const double* X, int64_t K, double* Y, double alpha, double beta) {
  for (int64_t i = 0; i < m * K; ++i) Y[i] = (beta == 0.0) ? 0.0 : (beta == 1.0 ? Y[i] : Y[i] * beta);
  if (alpha == 0.0) return;
  for (int64_t i = 0; i < m; ++i)
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
      const double w = values[p] * alpha;
      if (w == 0.0) continue;
      const double* x = X + indices[p] * K;
      for (int64_t c = 0; c < K; ++c) Y[i * K + c] = fma(w, x[c], Y[i * K + c]);
    }
}

/* ===================================================================== */
/* Brute-force kNN — scl/kernel/neighbors.hpp:319-478 (knn) on a dense   */
/* n x d block (a sparse row's missing entries are zeros, whose products */
/* leave an fma chain unchanged). For every query i, candidates j != i   */
/* in increasing j: skipped when (sqrt(norm_i) - sqrt(norm_j))^2 is not  */
/* below the current k-th distance; dot = fma chain over the features in */
/* order; dist_sq = fma(-2, dot, norm_i + norm_j) clamped at 0 (the same */
/* value as (norm_i + norm_j) - 2 * dot, 2 * dot being exact); a max-heap */
/* of k (dist_sq, j) takes the candidate while short (sift up, stopping  */
/* at a parent that is not smaller), else when strictly below the top    */
/* (replace the top, sift down to the larger child). The heap is then    */
/* sorted as the reference does (min-heap build, extract to the back,    */
/* reverse) and written as sqrt(dist_sq); missing slots (inf, -1).       */
/* ===================================================================== */
#define ORACLE_KNN_SWAP(a, b)   \
  do {                          \
    T td_ = hd[a];              \
    int64_t tj_ = hj[a];        \
    hd[a] = hd[b];              \
    hj[a] = hj[b];              \
    hd[b] = td_;                \
    hj[b] = tj_;                \
  } while (0)

#define ORACLE_KNN_BODY(T, FMA, SQRT, INF, MAXV)                                                      \
  T* hd = (T*)malloc(sizeof(T) * (size_t)(k > 0 ? k : 1));                                            \
  int64_t* hj = (int64_t*)malloc(sizeof(int64_t) * (size_t)(k > 0 ? k : 1));                          \
  for (int64_t i = 0; i < n; ++i) {                                                                   \
    int64_t cnt = 0;                                                                                  \
    T maxd = MAXV;                                                                                    \
    const T si = SQRT(norms[i]);                                                                      \
    for (int64_t j = 0; j < n; ++j) {                                                                 \
      if (j == i) continue;                                                                           \
      const T nd = si - SQRT(norms[j]);                                                               \
      if (nd * nd >= maxd) continue;                                                                  \
      T dot = (T)0;                                                                                   \
      for (int64_t f = 0; f < d; ++f) dot = FMA(X[i * d + f], X[j * d + f], dot);                     \
      T ds = contract ? FMA((T)-2, dot, norms[i] + norms[j]) : (norms[i] + norms[j]) - (T)2 * dot;    \
      if (ds < (T)0) ds = (T)0;                                                                       \
      if (cnt < k) {                                                                                  \
        int64_t pos = cnt;                                                                            \
        hd[pos] = ds;                                                                                 \
        hj[pos] = j;                                                                                  \
        while (pos > 0) {                                                                             \
          const int64_t par = (pos - 1) / 2;                                                          \
          if (hd[pos] <= hd[par]) break;                                                              \
          ORACLE_KNN_SWAP(pos, par);                                                                  \
          pos = par;                                                                                  \
        }                                                                                             \
        ++cnt;                                                                                        \
        if (cnt == k) maxd = hd[0];                                                                   \
      } else if (ds < hd[0]) {                                                                        \
        hd[0] = ds;                                                                                   \
        hj[0] = j;                                                                                    \
        int64_t pos = 0;                                                                              \
        for (;;) {                                                                                    \
          int64_t lg = pos;                                                                           \
          const int64_t l = 2 * pos + 1, r = 2 * pos + 2;                                             \
          if (l < cnt && hd[l] > hd[lg]) lg = l;                                                      \
          if (r < cnt && hd[r] > hd[lg]) lg = r;                                                      \
          if (lg == pos) break;                                                                       \
          ORACLE_KNN_SWAP(pos, lg);                                                                   \
          pos = lg;                                                                                   \
        }                                                                                             \
        maxd = hd[0];                                                                                 \
      }                                                                                               \
    }                                                                                                 \
    for (int64_t m = cnt / 2; cnt >= 2 && m > 0; --m) oracle_knn_sort_sift_##T(hd, hj, m - 1, cnt);   \
    for (int64_t m = cnt; m > 1; --m) {                                                               \
      ORACLE_KNN_SWAP(0, m - 1);                                                                      \
      oracle_knn_sort_sift_##T(hd, hj, 0, m - 1);                                                     \
    }                                                                                                 \
    for (int64_t m = 0; m < cnt / 2; ++m) ORACLE_KNN_SWAP(m, cnt - 1 - m);                            \
    for (int64_t m = 0; m < k; ++m) {                                                                 \
      out_dist[i * k + m] = m < cnt ? SQRT(hd[m]) : INF;                                              \
      out_idx[i * k + m] = m < cnt ? hj[m] : -1;                                                      \
    }                                                                                                 \
  }                                                                                                   \
  free(hd);                                                                                           \
  free(hj);

/* min-heap sift used by the final heap sort */
#define ORACLE_KNN_SORT_SIFT(T)                                                                       \
  static void oracle_knn_sort_sift_##T(T* hd, int64_t* hj, int64_t pos, int64_t size) {              \
    for (;;) {                                                                                        \
      int64_t sm = pos;                                                                               \
      const int64_t l = 2 * pos + 1, r = 2 * pos + 2;                                                 \
      if (l < size && hd[l] < hd[sm]) sm = l;                                                         \
      if (r < size && hd[r] < hd[sm]) sm = r;                                                         \
      if (sm == pos) break;                                                                           \
      ORACLE_KNN_SWAP(pos, sm);                                                                       \
      pos = sm;                                                                                       \
    }                                                                                                 \
  }
#define T float
ORACLE_KNN_SORT_SIFT(float)
#undef T
#define T double
ORACLE_KNN_SORT_SIFT(double)
#undef T

void oracle_knn_dense_f32(int64_t n, int64_t d, const float* X, const float* norms, int64_t k, int contract,
                          int64_t* out_idx, float* out_dist) {
#define T float
  ORACLE_KNN_BODY(float, fmaf, sqrtf, INFINITY, FLT_MAX)
#undef T
}

void oracle_knn_dense_f64(int64_t n, int64_t d, const double* X, const double* norms, int64_t k, int contract,
                          int64_t* out_idx, double* out_dist) {
#define T double
  ORACLE_KNN_BODY(double, fma, sqrt, (double)INFINITY, DBL_MAX)
#undef T
}
