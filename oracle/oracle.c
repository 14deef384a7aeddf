/* oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatements of the reference's contraction semantics, used as the
 * checker by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * and reference arms. Nothing in the library (tensoralgebra-rs_b200/) links,
 * loads or calls this file; the product path has no CPU fallback.
 *
 * Two independent implementations of
 *     D = op_D(alpha * op_A(A) * op_B(B) + beta * op_C(C))
 * over strided f32 / f64 / c32 / c64 operands with index labels:
 *
 *  1. oracle_label_contract: brute force over every label assignment, reading
 *     the raw layouts directly, restating the reference's independent oracle
 *     crates/tprims-testkit/src/oracle.rs:92-204 (a label repeated in one
 *     operand selects its diagonal; a label absent from D is summed; beta == 0
 *     reads no C; op_D conjugates the final value). It accumulates in x87
 *     extended precision (64-bit significand), so its f64 results serve as the
 *     "FP64 oracle" against which relative errors of 1e-12 are measurable, and
 *     it can write its result as double for f32 inputs.
 *
 *  2. oracle_packed_contract: the reference's packed block-scatter driver:
 *     lowering (crates/tprims-contract/src/api/validate.rs:47-308), role
 *     ordering and folding and scatter vectors (plan/analysis.rs:197-321,
 *     kernel pack/scatter.rs:70), blocking kc = 384 (4-byte reals) / 256
 *     (8-byte reals) with 512 KiB / 3 MiB panel budgets (kernel
 *     abi/types.rs:356-388), the five-loop nest with packed A / B panels
 *     (driver/static_grid.rs:126-216, driver/tile.rs:142-356,
 *     pack/pack.rs:152-270), the real and planar micro-kernels
 *     (kernels/reference/scalar.rs:31-106) and the KC-slabbed write-back, where
 *     the first slab applies beta * op_C(C) and later slabs accumulate into D
 *     with op_C = op_D (pack/writeback.rs:54-97, 311-486; driver/tile.rs:312-350).
 *     Parallel over the static output grid with OpenMP. This is the timed CPU
 *     baseline (the reference itself is Rust and cannot be built here).
 *
 * Return codes: 0 ok, 1 invalid labels/extents, 2 unsupported (output-only
 * label), 3 allocation failure.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  const void* data; /* origin: the element of index (0, .., 0) */
  int rank;
  const int64_t* ext;
  const int64_t* str;
  const int64_t* lab;
  int conj;
} or_operand;

enum { OR_F32 = 0, OR_F64 = 1, OR_C32 = 2, OR_C64 = 3 };

static int is_cplx(int t) { return t == OR_C32 || t == OR_C64; }

static void load_ld(int t, const void* base, int64_t off, long double* re, long double* im) {
  switch (t) {
    case OR_F32: *re = ((const float*)base)[off]; *im = 0; break;
    case OR_F64: *re = ((const double*)base)[off]; *im = 0; break;
    case OR_C32: *re = ((const float*)base)[2 * off]; *im = ((const float*)base)[2 * off + 1]; break;
    default: *re = ((const double*)base)[2 * off]; *im = ((const double*)base)[2 * off + 1]; break;
  }
}

static void store_ld(int t, int out_f64, void* base, int64_t off, long double re, long double im) {
  if (out_f64) {
    if (is_cplx(t)) {
      ((double*)base)[2 * off] = (double)re;
      ((double*)base)[2 * off + 1] = (double)im;
    } else {
      ((double*)base)[off] = (double)re;
    }
    return;
  }
  switch (t) {
    case OR_F32: ((float*)base)[off] = (float)re; break;
    case OR_F64: ((double*)base)[off] = (double)re; break;
    case OR_C32: ((float*)base)[2 * off] = (float)re; ((float*)base)[2 * off + 1] = (float)im; break;
    default: ((double*)base)[2 * off] = (double)re; ((double*)base)[2 * off + 1] = (double)im; break;
  }
}

/* ------------------------------------------------------------ label oracle */

typedef struct {
  int64_t label, extent;
} lab_ext;

static int add_labels(lab_ext* tab, int* n, const or_operand* o) {
  for (int i = 0; i < o->rank; ++i) {
    int found = -1;
    for (int j = 0; j < *n; ++j)
      if (tab[j].label == o->lab[i]) found = j;
    if (found >= 0) {
      if (tab[found].extent != o->ext[i]) return 1;
    } else {
      tab[*n].label = o->lab[i];
      tab[*n].extent = o->ext[i];
      ++*n;
    }
  }
  return 0;
}

static int64_t offset_of(const or_operand* o, const int64_t* labels, const int64_t* vals, int nl) {
  int64_t off = 0;
  for (int i = 0; i < o->rank; ++i) {
    int64_t v = 0;
    for (int j = 0; j < nl; ++j)
      if (labels[j] == o->lab[i]) v = vals[j];
    off += v * o->str[i];
  }
  return off;
}

int oracle_label_contract(int dtype, int out_f64, const double* alpha, const or_operand* A, const or_operand* B,
                          const double* beta, const or_operand* C, const or_operand* D) {
  lab_ext tab[64];
  int n = 0;
  if (A->rank + B->rank + (C ? C->rank : 0) + D->rank > 64) return 1;
  if (add_labels(tab, &n, A) || add_labels(tab, &n, B) || (C && add_labels(tab, &n, C)) || add_labels(tab, &n, D))
    return 1;
  int64_t out_l[64], sum_l[64], out_e[64], sum_e[64];
  int no = 0, ns = 0;
  for (int i = 0; i < n; ++i) {
    int in_d = 0;
    for (int j = 0; j < D->rank; ++j)
      if (D->lab[j] == tab[i].label) in_d = 1;
    if (in_d) {
      out_l[no] = tab[i].label;
      out_e[no++] = tab[i].extent;
    } else {
      sum_l[ns] = tab[i].label;
      sum_e[ns++] = tab[i].extent;
    }
  }
  int64_t out_total = 1, sum_total = 1;
  for (int i = 0; i < no; ++i) out_total *= out_e[i];
  for (int i = 0; i < ns; ++i) sum_total *= sum_e[i];
  const int beta_zero = beta[0] == 0 && beta[1] == 0;
  const long double ar = alpha[0], ai = is_cplx(dtype) ? alpha[1] : 0;
  const long double br = beta[0], bi = is_cplx(dtype) ? beta[1] : 0;

#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t o = 0; o < out_total; ++o) {
    int64_t all_l[128], all_v[128];
    int64_t rem = o;
    for (int i = 0; i < no; ++i) {
      all_l[i] = out_l[i];
      all_v[i] = rem % out_e[i];
      rem /= out_e[i];
    }
    for (int i = 0; i < ns; ++i) {
      all_l[no + i] = sum_l[i];
      all_v[no + i] = 0;
    }
    long double acc_r = 0, acc_i = 0;
    for (int64_t s = 0; s < sum_total; ++s) {
      int64_t r2 = s;
      for (int i = 0; i < ns; ++i) {
        all_v[no + i] = r2 % sum_e[i];
        r2 /= sum_e[i];
      }
      long double xr, xi, yr, yi;
      load_ld(dtype, A->data, offset_of(A, all_l, all_v, no + ns), &xr, &xi);
      load_ld(dtype, B->data, offset_of(B, all_l, all_v, no + ns), &yr, &yi);
      if (A->conj) xi = -xi;
      if (B->conj) yi = -yi;
      acc_r += xr * yr - xi * yi;
      acc_i += xr * yi + xi * yr;
    }
    long double vr = ar * acc_r - ai * acc_i, vi = ar * acc_i + ai * acc_r;
    if (!beta_zero && C) {
      long double cr, ci;
      load_ld(dtype, C->data, offset_of(C, all_l, all_v, no), &cr, &ci);
      if (C->conj) ci = -ci;
      vr += br * cr - bi * ci;
      vi += br * ci + bi * cr;
    }
    if (D->conj) vi = -vi;
    if (!is_cplx(dtype)) vi = 0;
    store_ld(dtype, out_f64, (void*)D->data, offset_of(D, all_l, all_v, no), vr, vi);
  }
  return 0;
}

/* ---------------------------------------------------------- packed driver */

typedef struct {
  int64_t extent, s[4]; /* strides in A, B, C, D */
} pk_axis;

typedef struct {
  int64_t label, extent, s[4];
  int in[4];
} pk_label;

typedef struct {
  int64_t *v;
  int64_t n;
} i64vec;

/* Collapse repeated labels (strides add), then merge into the table. */
static int pk_merge(pk_label* tab, int* n, const or_operand* o, int slot) {
  for (int i = 0; i < o->rank; ++i) {
    int j;
    for (j = 0; j < *n; ++j)
      if (tab[j].label == o->lab[i]) break;
    if (j == *n) {
      memset(&tab[j], 0, sizeof(pk_label));
      tab[j].label = o->lab[i];
      tab[j].extent = o->ext[i];
      ++*n;
    } else if (tab[j].extent != o->ext[i]) {
      return 1;
    }
    if (tab[j].in[slot]) tab[j].s[slot] += o->str[i]; /* repeated within this operand: diagonal */
    else tab[j].s[slot] = o->str[i];
    tab[j].in[slot] = 1;
  }
  return 0;
}

static uint64_t uabs64(int64_t x) { return x < 0 ? (uint64_t)(-x) : (uint64_t)x; }

/* Stable insertion sort by (|s[k1]|, |s[k2]|), then fold. */
static int pk_role(pk_axis* ax, int n, int k1, int k2) {
  for (int i = 1; i < n; ++i) {
    pk_axis x = ax[i];
    int j = i - 1;
    while (j >= 0 && (uabs64(ax[j].s[k1]) > uabs64(x.s[k1]) ||
                      (uabs64(ax[j].s[k1]) == uabs64(x.s[k1]) && uabs64(ax[j].s[k2]) > uabs64(x.s[k2])))) {
      ax[j + 1] = ax[j];
      --j;
    }
    ax[j + 1] = x;
  }
  int m = 0;
  for (int i = 0; i < n; ++i) {
    if (m > 0) {
      pk_axis* p = &ax[m - 1];
      if (ax[i].s[0] == p->s[0] * p->extent && ax[i].s[1] == p->s[1] * p->extent &&
          ax[i].s[2] == p->s[2] * p->extent && ax[i].s[3] == p->s[3] * p->extent) {
        p->extent *= ax[i].extent;
        continue;
      }
    }
    ax[m++] = ax[i];
  }
  return m;
}

static i64vec pk_scatter(const pk_axis* ax, int n, int slot) {
  i64vec r;
  int64_t total = 1;
  for (int i = 0; i < n; ++i) total *= ax[i].extent;
  r.n = total < 0 ? 0 : total;
  r.v = (int64_t*)malloc(sizeof(int64_t) * (size_t)(r.n > 0 ? r.n : 1));
  int64_t ctr[64] = {0};
  int64_t off = 0;
  for (int64_t i = 0; i < r.n; ++i) {
    r.v[i] = off;
    for (int d = 0; d < n; ++d) {
      off += ax[d].s[slot];
      if (++ctr[d] < ax[d].extent) break;
      off -= ax[d].s[slot] * ax[d].extent;
      ctr[d] = 0;
    }
  }
  return r;
}

/* One real type R and complexity: the loop nest is written once per (R, CPLX)
   through this macro-free generic body using double/float switches. */
typedef struct {
  int dtype, cplx, real_bytes;
  int mr, nr; /* register tile of the micro-kernel */
  int64_t M, N, K, H;
  i64vec a_m, a_k, b_k, b_n, c_m, c_n, d_m, d_n, h_a, h_b, h_c, h_d;
  int conj_a, conj_b, conj_c, conj_d;
} pk_plan;

/* Register tiles: the reference's default x86 families (f64 24x8 and f32 48x8
   AVX-512, crates/tprims-kernel/tests/snapshots/x86_64_manifest.txt) when this
   file is built with AVX-512, a scalar 8x6 tile otherwise and for the planar
   complex kernels. */
#define PK_MR_MAX 48
#define PK_NR_MAX 8
#ifdef __AVX512F__
#include <immintrin.h>
#endif

static double rd(const pk_plan* p, const void* base, int64_t off, int part) {
  switch (p->dtype) {
    case OR_F32: return part ? 0.0 : ((const float*)base)[off];
    case OR_F64: return part ? 0.0 : ((const double*)base)[off];
    case OR_C32: return ((const float*)base)[2 * off + part];
    default: return ((const double*)base)[2 * off + part];
  }
}
static void wr(const pk_plan* p, void* base, int64_t off, double re, double im) {
  switch (p->dtype) {
    case OR_F32: ((float*)base)[off] = (float)re; break;
    case OR_F64: ((double*)base)[off] = re; break;
    case OR_C32: ((float*)base)[2 * off] = (float)re; ((float*)base)[2 * off + 1] = (float)im; break;
    default: ((double*)base)[2 * off] = re; ((double*)base)[2 * off + 1] = im; break;
  }
}

/* The micro-kernel on packed panels: overwrite the mr x nr tile `ab`
   (column-major, j * mr + i; planar complex adds the imaginary plane at
   mr * nr) with the panel product. For f32 the accumulation runs in float, as
   the reference's f32 kernels do; planar complex follows planar_ukr's four
   real products (kernels/reference/scalar.rs:64-106). */
#ifdef __AVX512F__
static void ukr_f64_avx512(int kc, const double* a, const double* b, double* ab) {
  __m512d c[3][8];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 8; ++j) c[i][j] = _mm512_setzero_pd();
  for (int p = 0; p < kc; ++p) {
    const __m512d a0 = _mm512_loadu_pd(a + 24 * p), a1 = _mm512_loadu_pd(a + 24 * p + 8),
                  a2 = _mm512_loadu_pd(a + 24 * p + 16);
    for (int j = 0; j < 8; ++j) {
      const __m512d bj = _mm512_set1_pd(b[8 * p + j]);
      c[0][j] = _mm512_fmadd_pd(a0, bj, c[0][j]);
      c[1][j] = _mm512_fmadd_pd(a1, bj, c[1][j]);
      c[2][j] = _mm512_fmadd_pd(a2, bj, c[2][j]);
    }
  }
  for (int j = 0; j < 8; ++j)
    for (int i = 0; i < 3; ++i) _mm512_storeu_pd(ab + 24 * j + 8 * i, c[i][j]);
}
static void ukr_f32_avx512(int kc, const float* a, const float* b, float* ab) {
  __m512 c[3][8];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 8; ++j) c[i][j] = _mm512_setzero_ps();
  for (int p = 0; p < kc; ++p) {
    const __m512 a0 = _mm512_loadu_ps(a + 48 * p), a1 = _mm512_loadu_ps(a + 48 * p + 16),
                 a2 = _mm512_loadu_ps(a + 48 * p + 32);
    for (int j = 0; j < 8; ++j) {
      const __m512 bj = _mm512_set1_ps(b[8 * p + j]);
      c[0][j] = _mm512_fmadd_ps(a0, bj, c[0][j]);
      c[1][j] = _mm512_fmadd_ps(a1, bj, c[1][j]);
      c[2][j] = _mm512_fmadd_ps(a2, bj, c[2][j]);
    }
  }
  for (int j = 0; j < 8; ++j)
    for (int i = 0; i < 3; ++i) _mm512_storeu_ps(ab + 48 * j + 16 * i, c[i][j]);
}
#endif

static void ukr_f64(int kc, const double* a, const double* b, double* ab, int cplx, int mr, int nr) {
#ifdef __AVX512F__
  if (!cplx && mr == 24 && nr == 8) {
    ukr_f64_avx512(kc, a, b, ab);
    return;
  }
#endif
  if (!cplx) {
    double acc[PK_NR_MAX][PK_MR_MAX];
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) acc[j][i] = 0;
    for (int p = 0; p < kc; ++p)
      for (int j = 0; j < nr; ++j) {
        const double bv = b[p * nr + j];
        for (int i = 0; i < mr; ++i) acc[j][i] += a[p * mr + i] * bv;
      }
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) ab[j * mr + i] = acc[j][i];
  } else {
    double re[PK_NR_MAX][PK_MR_MAX], im[PK_NR_MAX][PK_MR_MAX];
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) re[j][i] = im[j][i] = 0;
    for (int p = 0; p < kc; ++p) {
      const double *ar = a + p * 2 * mr, *ai = ar + mr, *br = b + p * 2 * nr, *bi = br + nr;
      for (int j = 0; j < nr; ++j)
        for (int i = 0; i < mr; ++i) {
          re[j][i] += ar[i] * br[j];
          re[j][i] += -(ai[i] * bi[j]);
          im[j][i] += ar[i] * bi[j];
          im[j][i] += ai[i] * br[j];
        }
    }
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) {
        ab[j * mr + i] = re[j][i];
        ab[mr * nr + j * mr + i] = im[j][i];
      }
  }
}
static void ukr_f32(int kc, const float* a, const float* b, float* ab, int cplx, int mr, int nr) {
#ifdef __AVX512F__
  if (!cplx && mr == 48 && nr == 8) {
    ukr_f32_avx512(kc, a, b, ab);
    return;
  }
#endif
  if (!cplx) {
    float acc[PK_NR_MAX][PK_MR_MAX];
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) acc[j][i] = 0;
    for (int p = 0; p < kc; ++p)
      for (int j = 0; j < nr; ++j) {
        const float bv = b[p * nr + j];
        for (int i = 0; i < mr; ++i) acc[j][i] += a[p * mr + i] * bv;
      }
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) ab[j * mr + i] = acc[j][i];
  } else {
    float re[PK_NR_MAX][PK_MR_MAX], im[PK_NR_MAX][PK_MR_MAX];
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) re[j][i] = im[j][i] = 0;
    for (int p = 0; p < kc; ++p) {
      const float *ar = a + p * 2 * mr, *ai = ar + mr, *br = b + p * 2 * nr, *bi = br + nr;
      for (int j = 0; j < nr; ++j)
        for (int i = 0; i < mr; ++i) {
          re[j][i] += ar[i] * br[j];
          re[j][i] += -(ai[i] * bi[j]);
          im[j][i] += ar[i] * bi[j];
          im[j][i] += ai[i] * br[j];
        }
    }
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) {
        ab[j * mr + i] = re[j][i];
        ab[mr * nr + j * mr + i] = im[j][i];
      }
  }
}

static void cmul(double ar, double ai, double br, double bi, double* r, double* i) {
  *r = ar * br - ai * bi;
  *i = ar * bi + ai * br;
}

/* Write one MR x NR tile: first slab D = op_D(alpha*ab + beta*op_C(C)), later
   slabs D = op_D(alpha*ab + op_D(D)). */
static void pk_writeback(const pk_plan* p, const void* ab, int mrem, int nrem, int64_t i0, int64_t j0, int64_t h,
                         const double* alpha, const double* beta, int first, int beta_zero, const void* C, void* D) {
  const int cp = p->cplx;
  for (int j = 0; j < nrem; ++j)
    for (int i = 0; i < mrem; ++i) {
      double tr, ti = 0;
      if (p->real_bytes == 4) {
        tr = ((const float*)ab)[j * p->mr + i];
        if (cp) ti = ((const float*)ab)[p->mr * p->nr + j * p->mr + i];
      } else {
        tr = ((const double*)ab)[j * p->mr + i];
        if (cp) ti = ((const double*)ab)[p->mr * p->nr + j * p->mr + i];
      }
      const int64_t doff = p->h_d.v[h] + p->d_m.v[i0 + i] + p->d_n.v[j0 + j];
      double vr, vi;
      if (first) {
        if (beta_zero && alpha[0] == 1 && alpha[1] == 0 && !p->conj_d) {
          vr = tr;
          vi = ti;
        } else {
          cmul(tr, ti, alpha[0], cp ? alpha[1] : 0, &vr, &vi);
          if (!beta_zero) {
            const int64_t coff = p->h_c.v[h] + p->c_m.v[i0 + i] + p->c_n.v[j0 + j];
            double cr = rd(p, C, coff, 0), ci = cp ? rd(p, C, coff, 1) : 0, xr, xi;
            if (p->conj_c) ci = -ci;
            cmul(cr, ci, beta[0], cp ? beta[1] : 0, &xr, &xi);
            vr += xr;
            vi += xi;
          }
          if (p->conj_d) vi = -vi;
        }
      } else {
        double dr = rd(p, D, doff, 0), di = cp ? rd(p, D, doff, 1) : 0;
        if (p->conj_d) di = -di;
        if (!cp && alpha[0] == 1) {
          vr = tr + dr;
          vi = 0;
        } else {
          cmul(tr, ti, alpha[0], cp ? alpha[1] : 0, &vr, &vi);
          vr += dr;
          vi += di;
        }
        if (p->conj_d) vi = -vi;
      }
      /* f32 arithmetic for f32 storage: round the intermediate like the
         reference's f32 write-back does. */
      if (p->real_bytes == 4) {
        vr = (float)vr;
        vi = (float)vi;
      }
      wr(p, D, doff, vr, vi);
    }
}

static void pk_free(pk_plan* p) {
  i64vec* v[12] = {&p->a_m, &p->a_k, &p->b_k, &p->b_n, &p->c_m, &p->c_n,
                   &p->d_m, &p->d_n, &p->h_a, &p->h_b, &p->h_c, &p->h_d};
  for (int i = 0; i < 12; ++i) free(v[i]->v);
}

int oracle_packed_contract(int dtype, const double* alpha, const or_operand* A, const or_operand* B,
                           const double* beta, const or_operand* C, const or_operand* D, int nthreads) {
  pk_label tab[128];
  int n = 0;
  const int beta_zero = beta[0] == 0 && (!is_cplx(dtype) || beta[1] == 0);
  if (pk_merge(tab, &n, A, 0) || pk_merge(tab, &n, B, 1)) return 1;
  /* With no separate C, C mirrors D. */
  if (pk_merge(tab, &n, (C && !beta_zero) ? C : D, 2) || pk_merge(tab, &n, D, 3)) return 1;
  pk_axis am[64], an[64], ak[64], ah[64];
  int nm = 0, nn = 0, nk = 0, nh = 0;
  for (int i = 0; i < n; ++i) {
    pk_axis x = {tab[i].extent, {tab[i].s[0], tab[i].s[1], tab[i].s[2], tab[i].s[3]}};
    const int ia = tab[i].in[0], ib = tab[i].in[1], id = tab[i].in[3];
    if (id && !ia && !ib) return 2;
    if (x.extent == 1) continue;
    if (ia && ib && id) ah[nh++] = x;
    else if (ia && id) am[nm++] = x;
    else if (ib && id) an[nn++] = x;
    else ak[nk++] = x;
  }
  nm = pk_role(am, nm, 3, 0);
  nn = pk_role(an, nn, 3, 1);
  nk = pk_role(ak, nk, 0, 1);
  nh = pk_role(ah, nh, 3, 0);
  pk_plan p;
  memset(&p, 0, sizeof(p));
  p.dtype = dtype;
  p.cplx = is_cplx(dtype);
  p.real_bytes = (dtype == OR_F32 || dtype == OR_C32) ? 4 : 8;
  p.mr = 8;
  p.nr = 6;
#ifdef __AVX512F__
  if (dtype == OR_F64) {
    p.mr = 24;
    p.nr = 8;
  } else if (dtype == OR_F32) {
    p.mr = 48;
    p.nr = 8;
  }
#endif
  p.a_m = pk_scatter(am, nm, 0);
  p.a_k = pk_scatter(ak, nk, 0);
  p.b_k = pk_scatter(ak, nk, 1);
  p.b_n = pk_scatter(an, nn, 1);
  p.c_m = pk_scatter(am, nm, 2);
  p.c_n = pk_scatter(an, nn, 2);
  p.d_m = pk_scatter(am, nm, 3);
  p.d_n = pk_scatter(an, nn, 3);
  p.h_a = pk_scatter(ah, nh, 0);
  p.h_b = pk_scatter(ah, nh, 1);
  p.h_c = pk_scatter(ah, nh, 2);
  p.h_d = pk_scatter(ah, nh, 3);
  p.M = p.d_m.n;
  p.N = p.d_n.n;
  p.K = p.a_k.n;
  p.H = p.h_d.n;
  p.conj_a = p.cplx && A->conj;
  p.conj_b = p.cplx && B->conj;
  p.conj_c = p.cplx && C && C->conj;
  p.conj_d = p.cplx && D->conj;
  const int cp = p.cplx;
  const void* Cd = (C && !beta_zero) ? C->data : NULL;
  void* Dd = (void*)D->data;
  if (p.M == 0 || p.N == 0 || p.H == 0) {
    pk_free(&p);
    return 0;
  }
  const int alpha_zero = alpha[0] == 0 && (!cp || alpha[1] == 0);
  if (p.K == 0 || alpha_zero) { /* output-only pass */
    for (int64_t h = 0; h < p.H; ++h)
      for (int64_t j = 0; j < p.N; ++j)
        for (int64_t i = 0; i < p.M; ++i) {
          double vr = 0, vi = 0;
          if (!beta_zero) {
            const int64_t coff = p.h_c.v[h] + p.c_m.v[i] + p.c_n.v[j];
            double cr = rd(&p, Cd, coff, 0), ci = cp ? rd(&p, Cd, coff, 1) : 0;
            if (p.conj_c) ci = -ci;
            cmul(cr, ci, beta[0], cp ? beta[1] : 0, &vr, &vi);
          }
          if (p.conj_d) vi = -vi;
          wr(&p, Dd, p.h_d.v[h] + p.d_m.v[i] + p.d_n.v[j], vr, vi);
        }
    pk_free(&p);
    return 0;
  }

  const int planes = cp ? 2 : 1;
  const int64_t kc = p.real_bytes == 4 ? 384 : 256;
  int64_t mc = (512 * 1024) / (kc * planes * p.real_bytes);
  int64_t nc = (3 * 1024 * 1024) / (kc * planes * p.real_bytes);
  const int MR = p.mr, NR = p.nr;
  mc = mc / MR * MR;
  nc = nc / NR * NR;
  if (mc < MR) mc = MR;
  if (nc < NR) nc = NR;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const size_t rb = (size_t)p.real_bytes;
  char* bpanel = (char*)malloc((size_t)(nc + NR) * kc * planes * rb);
  if (!bpanel) {
    pk_free(&p);
    return 3;
  }
  for (int64_t h = 0; h < p.H; ++h) {
    const int64_t ha = p.h_a.v[h], hb = p.h_b.v[h];
    for (int64_t jc = 0; jc < p.N; jc += nc) {
      const int64_t ncur = (p.N - jc < nc) ? p.N - jc : nc;
      const int64_t nsl = (ncur + NR - 1) / NR;
      for (int64_t pc = 0; pc < p.K; pc += kc) {
        const int64_t kcur = (p.K - pc < kc) ? p.K - pc : kc;
        /* pack B: slivers of NR columns, per k: NR reals (x planes) */
#pragma omp parallel for schedule(static)
        for (int64_t s = 0; s < nsl; ++s) {
          for (int64_t q = 0; q < kcur; ++q)
            for (int j = 0; j < NR; ++j) {
              const int64_t col = jc + s * NR + j;
              double vr = 0, vi = 0;
              if (col < p.N) {
                const int64_t off = hb + p.b_k.v[pc + q] + p.b_n.v[col];
                vr = rd(&p, B->data, off, 0);
                vi = cp ? rd(&p, B->data, off, 1) : 0;
                if (p.conj_b) vi = -vi;
              }
              const size_t idx = (size_t)(s * kcur + q) * planes * NR;
              if (rb == 4) {
                ((float*)bpanel)[idx + j] = (float)vr;
                if (cp) ((float*)bpanel)[idx + NR + j] = (float)vi;
              } else {
                ((double*)bpanel)[idx + j] = vr;
                if (cp) ((double*)bpanel)[idx + NR + j] = vi;
              }
            }
        }
        /* the static grid: row blocks (MC) x column groups of slivers */
        const int64_t nic = (p.M + mc - 1) / mc;
        int threads = 1;
#ifdef _OPENMP
        threads = omp_get_max_threads();
#endif
        int64_t groups = threads / nic;
        if (groups < 1) groups = 1;
        if (groups > nsl) groups = nsl;
        const int first = pc == 0;
#pragma omp parallel
        {
          char* apanel = (char*)malloc((size_t)(mc + MR) * kc * planes * rb);
          double abbuf[2 * PK_MR_MAX * PK_NR_MAX];
#pragma omp for schedule(static) collapse(2)
          for (int64_t ib = 0; ib < nic; ++ib)
            for (int64_t gi = 0; gi < groups; ++gi) {
              const int64_t ic = ib * mc;
              const int64_t mcur = (p.M - ic < mc) ? p.M - ic : mc;
              const int64_t msl = (mcur + MR - 1) / MR;
              for (int64_t s = 0; s < msl; ++s)
                for (int64_t q = 0; q < kcur; ++q)
                  for (int i = 0; i < MR; ++i) {
                    const int64_t row = ic + s * MR + i;
                    double vr = 0, vi = 0;
                    if (row < p.M) {
                      const int64_t off = ha + p.a_m.v[row] + p.a_k.v[pc + q];
                      vr = rd(&p, A->data, off, 0);
                      vi = cp ? rd(&p, A->data, off, 1) : 0;
                      if (p.conj_a) vi = -vi;
                    }
                    const size_t idx = (size_t)(s * kcur + q) * planes * MR;
                    if (rb == 4) {
                      ((float*)apanel)[idx + i] = (float)vr;
                      if (cp) ((float*)apanel)[idx + MR + i] = (float)vi;
                    } else {
                      ((double*)apanel)[idx + i] = vr;
                      if (cp) ((double*)apanel)[idx + MR + i] = vi;
                    }
                  }
              const int64_t s0 = nsl * gi / groups, s1 = nsl * (gi + 1) / groups;
              for (int64_t jr = s0; jr < s1; ++jr)
                for (int64_t ir = 0; ir < msl; ++ir) {
                  const size_t aoff = (size_t)ir * kcur * planes * MR, boff = (size_t)jr * kcur * planes * NR;
                  if (rb == 4)
                    ukr_f32((int)kcur, (float*)apanel + aoff, (float*)bpanel + boff, (float*)abbuf, cp, MR, NR);
                  else
                    ukr_f64((int)kcur, (double*)apanel + aoff, (double*)bpanel + boff, abbuf, cp, MR, NR);
                  const int64_t i0 = ic + ir * MR, j0 = jc + jr * NR;
                  const int mrem = (int)((p.M - i0 < MR) ? p.M - i0 : MR);
                  const int nrem = (int)((p.N - j0 < NR) ? p.N - j0 : NR);
                  pk_writeback(&p, abbuf, mrem, nrem, i0, j0, h, alpha, beta, first, beta_zero, Cd, Dd);
                }
            }
          free(apanel);
        }
      }
    }
  }
  free(bpanel);
  pk_free(&p);
  return 0;
}

/* Checksum helper for size-independent checks: sum over the output layout of
   re + 2*im in extended precision, and the sum of squares. */
void oracle_layout_sums(int dtype, const or_operand* X, double* out_sum, double* out_sumsq) {
  int64_t total = 1;
  for (int i = 0; i < X->rank; ++i) total *= X->ext[i];
  long double s = 0, q = 0;
  int64_t idx[64] = {0};
  for (int64_t t = 0; t < total; ++t) {
    int64_t off = 0;
    for (int i = 0; i < X->rank; ++i) off += idx[i] * X->str[i];
    long double re, im;
    load_ld(dtype, X->data, off, &re, &im);
    s += re + 2 * im;
    q += re * re + im * im;
    for (int i = 0; i < X->rank; ++i) {
      if (++idx[i] < X->ext[i]) break;
      idx[i] = 0;
    }
  }
  *out_sum = (double)s;
  *out_sumsq = (double)q;
}
