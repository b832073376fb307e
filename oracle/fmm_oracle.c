/*
 * fmm_oracle.c — CPU restatement of fockl/FMMA's `exact`, `fmm`, `tree` and
 * `nrnmm` solvers.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library:
 * only tests, the smoke check and the benchmark's CPU-baseline leg load it.
 * The product path (fmma_b200/, pyfmma/, include/) never calls it.
 *
 * It restates the reference algorithm on the reference's dense uniform grid,
 * with the same loop orders, so that on the same inputs it agrees with the
 * compiled reference (oracle/_ref) to the last bits.  Each function cites the
 * reference lines it follows (paths relative to the reference project).
 * Parity pin: tests/test_oracle.py compares it with the compiled reference
 * and with the committed golden vectors in tests/golden/.
 *
 * Build: `make -C oracle` (gcc -O3 -fopenmp, no FMA contraction, like the
 * reference's x86-64 build).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/fmma_b200.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_MAXD 3

/* ---- kernels ------------------------------------------------------------
 * Same formulas as the CUDA functors (fmma_b200/csrc/kernels.cuh).  The
 * reference default 1/|x-y| is include/fmma/fmma.hpp:55-63 (no guard).    */
static double orc_kernel(int kid, double p0, int d, const double* x, const double* y) {
  double r2 = 0.0, s = 0.0;
  switch (kid) {
    case FMMA_KERNEL_INV_R:
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; }
      return 1.0 / sqrt(r2);
    case FMMA_KERNEL_INV_R_SAFE:
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; }
      return r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0;
    case FMMA_KERNEL_INV_DIFF: {
      double t = x[0] - y[0];
      return t != 0.0 ? 1.0 / t : 0.0;
    }
    case FMMA_KERNEL_LOG_R:
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; }
      return r2 > 0.0 ? 0.5 * log(r2) : 0.0;
    case FMMA_KERNEL_GAUSSIAN:
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; }
      return exp(-r2 / p0);
    case FMMA_KERNEL_MULTIQUADRIC:
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; }
      return sqrt(r2 + p0);
    case FMMA_KERNEL_SUM_OVER_R2:  /* test/src/fmma/fmm.cpp:82-91 */
      for (int k = 0; k < d; ++k) { double t = x[k] - y[k]; r2 += t * t; s += t; }
      return s / r2;
    case FMMA_KERNEL_SUM2_OVER_R2: /* test/src/fmma/fmm.cpp:151-160 */
      for (int k = 0; k < d; ++k) {
        double t = x[k] - y[k], u = x[k] + y[k];
        r2 += t * t; s += u * u;
      }
      return s / r2;
    default:
      return 0.0;
  }
}

/* ---- Chebyshev polynomials (src/math.cpp:14-50) ------------------------- */
static double orc_cheb(int n, double x) { return cos(n * acos(x)); }

static double orc_scheb(int n, double x, double y) {
  double a = 1.0 / n;
  for (int k = 1; k < n; ++k) a += 2.0 / n * orc_cheb(k, x) * orc_cheb(k, y);
  return a;
}

/* exported for the Chebyshev closed-form tests (test/src/math/common.cpp) */
double orc_chebyshev(int n, double x) { return orc_cheb(n, x); }
double orc_schebyshev(int n, double x, double y) { return orc_scheb(n, x, y); }

/* ---- exact (src/fmma.cpp:80-101) ----------------------------------------
 * ans_i = sum_j w_j f(t_i, s_j), j ascending; w == NULL means w = 1
 * (src/fmma.cpp:55-70).                                                     */
void orc_exact(int d, int kid, double p0, int64_t nt, const double* tgt,
               int64_t ns, const double* src, const double* w, double* ans) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nt; ++i) {
    double a = 0.0;
    for (int64_t j = 0; j < ns; ++j) {
      double f = orc_kernel(kid, p0, d, tgt + i * d, src + j * d);
      a += w ? w[j] * f : f;
    }
    ans[i] = a;
  }
}

/* exact over a subset of targets (sampled oracle for large configs) */
void orc_exact_rows(int d, int kid, double p0, int64_t nrows, const int64_t* rows,
                    const double* tgt, int64_t ns, const double* src,
                    const double* w, double* ans) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t r = 0; r < nrows; ++r) {
    const double* x = tgt + rows[r] * d;
    double a = 0.0;
    for (int64_t j = 0; j < ns; ++j) {
      double f = orc_kernel(kid, p0, d, x, src + j * d);
      a += w ? w[j] * f : f;
    }
    ans[r] = a;
  }
}

/* ---- grid helpers ------------------------------------------------------- */

/* Default depth (src/fmm.cpp:23-28). */
int orc_default_depth(int64_t nt, int d) {
  int D = (int)(log((double)nt) / d) + 1;
  return D <= 0 ? 1 : D;
}

/* Cube enclosing targets then sources (src/fmm_core.cpp:125-173). */
void orc_origin_len(int d, int64_t nt, const double* tgt, int64_t ns,
                    const double* src, double* origin, double* Len) {
  double mn[ORC_MAXD] = {0, 0, 0}, mx[ORC_MAXD] = {0, 0, 0};
  if (nt > 0) {
    for (int k = 0; k < d; ++k) mn[k] = mx[k] = tgt[k];
  } else if (ns > 0) {
    for (int k = 0; k < d; ++k) mn[k] = mx[k] = src[k];
  }
  for (int64_t i = 0; i < nt; ++i)
    for (int k = 0; k < d; ++k) {
      double v = tgt[i * d + k];
      if (v < mn[k]) mn[k] = v;  /* std::min(a,b) keeps a unless b < a */
      if (mx[k] < v) mx[k] = v;
    }
  for (int64_t i = 0; i < ns; ++i)
    for (int k = 0; k < d; ++k) {
      double v = src[i * d + k];
      if (v < mn[k]) mn[k] = v;
      if (mx[k] < v) mx[k] = v;
    }
  double L = 0.0;
  for (int k = 0; k < d; ++k) if (L < mx[k] - mn[k]) L = mx[k] - mn[k];
  for (int k = 0; k < d; ++k) origin[k] = (mx[k] + mn[k]) / 2 - L / 2;
  *Len = L;
}

/* Leaf coordinate of one point, and its local coordinate in [-1,1]
 * (src/fmm_core.cpp:261-264, src/fmm_core.cpp:595-596). */
static void orc_bin(int d, const double* x, const double* origin, double len, int N,
                    int* ib, double* rel) {
  for (int k = 0; k < d; ++k) {
    double q = (x[k] - origin[k]) / len;
    int t = (int)q;
    if (t > N - 1) t = N - 1;
    ib[k] = t;
    if (rel) {
      double r = 2.0 * (q - t) - 1.0;
      if (r > 1.0) r = 1.0;
      if (r < -1.0) r = -1.0;
      rel[k] = r;
    }
  }
}

static int64_t orc_rowmajor(int d, const int* ib, int N) {  /* fmm_core.cpp:204-212 */
  int64_t a = 0;
  for (int k = 0; k < d; ++k) a = a * N + ib[k];
  return a;
}

static void orc_unrow(int d, int64_t ind, int N, int* ib) {  /* fmm_core.cpp:183-193 */
  for (int k = 0; k < d; ++k) { ib[d - 1 - k] = (int)(ind % N); ind /= N; }
}

/* Row-major leaf index of every point at `depth` (binning of P2M and of the
 * P2P/L2P target lookup).  Exported for the tree bit-exactness test. */
void orc_bin_points(int d, int depth, int64_t n, const double* x,
                    const double* origin, double Len, int64_t* box) {
  int N = 1 << (depth - 1);
  double len = Len / N;
  for (int64_t i = 0; i < n; ++i) {
    int ib[ORC_MAXD];
    orc_bin(d, x + i * d, origin, len, N, ib, NULL);
    box[i] = orc_rowmajor(d, ib, N);
  }
}

/* Far (M2L) interaction list of one box (src/fmm_core.cpp:15-63):
 * children of the parent's in-grid neighbours, minus the 3^d near boxes,
 * in row-major order with the last dimension fastest.  Returns the count. */
int orc_far_list(int d, const int* b, int N, int64_t* out) {
  int lo[ORC_MAXD], hi[ORC_MAXD], shape[ORC_MAXD];
  int64_t size = 1;
  for (int k = 0; k < d; ++k) {
    int p = b[k] / 2;
    lo[k] = (p > 0 ? p - 1 : p) * 2;
    hi[k] = (p + 1 < N / 2 ? p + 1 : p) * 2 + 1;
    shape[k] = hi[k] - lo[k] + 1;
    size *= shape[k];
  }
  int cnt = 0;
  for (int64_t s = 0; s < size; ++s) {
    int64_t sc = s;
    int pos[ORC_MAXD], dist = 0;
    for (int k = d - 1; k >= 0; --k) {
      pos[k] = lo[k] + (int)(sc % shape[k]);
      sc /= shape[k];
      int a = abs(pos[k] - b[k]);
      if (a > dist) dist = a;
    }
    if (dist <= 1) continue;
    out[cnt++] = orc_rowmajor(d, pos, N);
  }
  return cnt;
}

/* Near (P2P) list of one leaf: clamped 3^d block including the box itself
 * (src/fmm_core.cpp:79-115). */
int orc_near_list(int d, const int* b, int N, int64_t* out) {
  int lo[ORC_MAXD], shape[ORC_MAXD];
  int64_t size = 1;
  for (int k = 0; k < d; ++k) {
    lo[k] = b[k] > 0 ? b[k] - 1 : b[k];
    int h = b[k] + 1 < N ? b[k] + 1 : b[k];
    shape[k] = h - lo[k] + 1;
    size *= shape[k];
  }
  int cnt = 0;
  for (int64_t s = 0; s < size; ++s) {
    int64_t sc = s;
    int pos[ORC_MAXD];
    for (int k = d - 1; k >= 0; --k) { pos[k] = lo[k] + (int)(sc % shape[k]); sc /= shape[k]; }
    out[cnt++] = orc_rowmajor(d, pos, N);
  }
  return cnt;
}

int orc_far_list_rowmajor(int d, int64_t box, int N, int64_t* out) {
  int b[ORC_MAXD];
  orc_unrow(d, box, N, b);
  return orc_far_list(d, b, N, out);
}

int orc_near_list_rowmajor(int d, int64_t box, int N, int64_t* out) {
  int b[ORC_MAXD];
  orc_unrow(d, box, N, b);
  return orc_near_list(d, b, N, out);
}

/* ---- fmm (src/fmm.cpp:15-144 with the stages of src/fmm_core.cpp) -------- */

typedef struct {
  int d, n, P, kid, trans_sym;
  double p0;
  double node[32];            /* Chebyshev nodes, descending (fmm_core.cpp:240-243) */
  double node_all[4096][ORC_MAXD]; /* P tensor nodes, last dim fastest (:244-253) */
} orc_setup;

static void orc_nodes(orc_setup* S) {
  int n = S->n;
  for (int k = 0; k < n; ++k) S->node[k] = cos((2.0 * k + 1.0) / (2 * n) * M_PI);
  for (int k = 0; k < S->P; ++k) {
    int kc = k;
    for (int q = 0; q < S->d; ++q) {
      S->node_all[k][S->d - 1 - q] = S->node[kc % n];
      kc /= n;
    }
  }
}

/* P2M at the leaf grid N (src/fmm_core.cpp:224-283): serial binning into
 * per-box lists in increasing source order, then per-box accumulation. */
static void orc_p2m(const orc_setup* S, int64_t ns, const double* src, const double* w,
                    int N, const double* origin, double len,
                    int64_t* box_start, int64_t* box_items, double* Wm) {
  int d = S->d, P = S->P;
  int64_t nbox = 1;
  for (int k = 0; k < d; ++k) nbox *= N;
  double* rel = (double*)malloc(sizeof(double) * (size_t)(ns > 0 ? ns : 1) * d);
  int64_t* sbox = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ns > 0 ? ns : 1));
  memset(box_start, 0, sizeof(int64_t) * (size_t)(nbox + 1));
  for (int64_t s = 0; s < ns; ++s) {
    int ib[ORC_MAXD];
    orc_bin(d, src + s * d, origin, len, N, ib, rel + s * d);
    sbox[s] = orc_rowmajor(d, ib, N);
    box_start[sbox[s] + 1]++;
  }
  for (int64_t b = 0; b < nbox; ++b) box_start[b + 1] += box_start[b];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)nbox);
  memcpy(fill, box_start, sizeof(int64_t) * (size_t)nbox);
  for (int64_t s = 0; s < ns; ++s) box_items[fill[sbox[s]]++] = s;
  free(fill);

  memset(Wm, 0, sizeof(double) * (size_t)(nbox * P));
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t b = 0; b < nbox; ++b) {
    for (int64_t it = box_start[b]; it < box_start[b + 1]; ++it) {
      int64_t s = box_items[it];
      for (int k = 0; k < P; ++k) {
        double v = 1.0;
        for (int q = 0; q < d; ++q) v *= orc_scheb(S->n, S->node_all[k][q], rel[s * d + q]);
        Wm[b * P + k] += (w ? w[s] : 1.0) * v;
      }
    }
  }
  free(rel);
  free(sbox);
}

/* M2M from grid N to N/2 (src/fmm_core.cpp:295-363). */
static void orc_m2m(const orc_setup* S, int N, const double* Win, double* Wout) {
  int d = S->d, P = S->P, nch = 1 << d;
  int64_t nin = 1, nout = 1;
  for (int k = 0; k < d; ++k) { nin *= N; nout *= N / 2; }
  double* vals = (double*)malloc(sizeof(double) * (size_t)P * P * nch);
  for (int kin = 0; kin < P; ++kin)
    for (int kout = 0; kout < P; ++kout)
      for (int si = 0; si < nch; ++si) {
        double v = 1.0;
        int sc = si;
        for (int q = 0; q < d; ++q) {
          int shift = 2 * (sc % 2) - 1;
          sc /= 2;
          v *= orc_scheb(S->n, S->node_all[kout][d - 1 - q],
                         (S->node_all[kin][d - 1 - q] + shift) / 2);
        }
        vals[((size_t)kin * P + kout) * nch + si] = v;
      }
  memset(Wout, 0, sizeof(double) * (size_t)(nout * P));
  for (int64_t in = 0; in < nin; ++in) {
    int bi[ORC_MAXD], bo[ORC_MAXD];
    orc_unrow(d, in, N, bi);
    int si = 0;
    for (int k = 0; k < d; ++k) { bo[k] = bi[k] / 2; si = si * 2 + bi[k] % 2; }
    int64_t out = orc_rowmajor(d, bo, N / 2);
    for (int kout = 0; kout < P; ++kout)
      for (int kin = 0; kin < P; ++kin) {
        double t = Win[in * P + kin];
        t *= vals[((size_t)kin * P + kout) * nch + si];
        Wout[out * P + kout] += t;
      }
  }
  free(vals);
}

/* M2L on grid N (src/fmm_core.cpp:375-495): table mode when trans_sym == 1,
 * per-pair evaluation on absolute node coordinates otherwise.  Adds into Wl
 * (the driver zero-initialises it, src/fmm.cpp:73-83).                     */
static void orc_m2l(const orc_setup* S, int N, const double* origin, double Len,
                    const double* Wm, double* Wl) {
  int d = S->d, P = S->P;
  double len = Len / N;
  int64_t nbox = 1;
  for (int k = 0; k < d; ++k) nbox *= N;
  if (S->trans_sym == 1) {
    int size = 1;
    for (int k = 0; k < d; ++k) size *= 7;
    double* fns = (double*)calloc((size_t)size * P * P, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int si = 0; si < size; ++si) {
      int shift[ORC_MAXD], sc = si, dist = 0;
      for (int q = 0; q < d; ++q) {
        shift[d - 1 - q] = sc % 7 - 3;
        if (abs(shift[d - 1 - q]) > dist) dist = abs(shift[d - 1 - q]);
        sc /= 7;
      }
      if (dist <= 1) continue;
      double xl[ORC_MAXD], ym[ORC_MAXD];
      for (int kl = 0; kl < P; ++kl) {
        for (int q = 0; q < d; ++q) xl[q] = len * (S->node_all[kl][q] / 2);
        for (int km = 0; km < P; ++km) {
          for (int q = 0; q < d; ++q) ym[q] = len * ((double)shift[q] + S->node_all[km][q] / 2);
          fns[((size_t)si * P + kl) * P + km] = orc_kernel(S->kid, S->p0, d, xl, ym);
        }
      }
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t ind = 0; ind < nbox; ++ind) {
      int lb[ORC_MAXD], mb[ORC_MAXD];
      int64_t lst[216];
      orc_unrow(d, ind, N, lb);
      int cnt = orc_far_list(d, lb, N, lst);
      for (int i = 0; i < cnt; ++i) {
        orc_unrow(d, lst[i], N, mb);
        int si = 0;
        for (int q = 0; q < d; ++q) si = si * 7 + (mb[q] + 3 - lb[q]);
        const double* A = fns + (size_t)si * P * P;
        const double* x = Wm + lst[i] * P;
        double* y = Wl + ind * P;
        for (int m = 0; m < P; ++m) {   /* matvec, src/math.cpp:264-327 */
          double a = y[m];
          for (int c = 0; c < P; ++c) a += A[m * P + c] * x[c];
          y[m] = a;
        }
      }
    }
    free(fns);
  } else {
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t ind = 0; ind < nbox; ++ind) {
      int lb[ORC_MAXD], mb[ORC_MAXD];
      int64_t lst[216];
      orc_unrow(d, ind, N, lb);
      int cnt = orc_far_list(d, lb, N, lst);
      double* xl = (double*)malloc(sizeof(double) * (size_t)P * d);
      double* ym = (double*)malloc(sizeof(double) * (size_t)P * d);
      double* A = (double*)malloc(sizeof(double) * (size_t)P * P);
      for (int kl = 0; kl < P; ++kl)
        for (int q = 0; q < d; ++q)
          xl[kl * d + q] = len * ((double)lb[q] + (1.0 + S->node_all[kl][q]) / 2) + origin[q];
      for (int i = 0; i < cnt; ++i) {
        orc_unrow(d, lst[i], N, mb);
        for (int km = 0; km < P; ++km)
          for (int q = 0; q < d; ++q)
            ym[km * d + q] = len * ((double)mb[q] + (1.0 + S->node_all[km][q]) / 2) + origin[q];
        for (int kl = 0; kl < P; ++kl)
          for (int km = 0; km < P; ++km)
            A[kl * P + km] = orc_kernel(S->kid, S->p0, d, xl + kl * d, ym + km * d);
        const double* x = Wm + lst[i] * P;
        double* y = Wl + ind * P;
        for (int m = 0; m < P; ++m) {
          double a = y[m];
          for (int c = 0; c < P; ++c) a += A[m * P + c] * x[c];
          y[m] = a;
        }
      }
      free(xl); free(ym); free(A);
    }
  }
}

/* L2L from grid N/2 to grid N, adding into Wout (src/fmm_core.cpp:507-568). */
static void orc_l2l(const orc_setup* S, int N, const double* Win, double* Wout) {
  int d = S->d, P = S->P, nch = 1 << d;
  int64_t nout = 1;
  for (int k = 0; k < d; ++k) nout *= N;
  double* vals = (double*)malloc(sizeof(double) * (size_t)P * P * nch);
  for (int kin = 0; kin < P; ++kin)
    for (int kout = 0; kout < P; ++kout)
      for (int si = 0; si < nch; ++si) {
        double v = 1.0;
        int sc = si;
        for (int q = 0; q < d; ++q) {
          int shift = 2 * (sc % 2) - 1;
          sc /= 2;
          v *= orc_scheb(S->n, (S->node_all[kout][d - 1 - q] + shift) / 2,
                         S->node_all[kin][d - 1 - q]);
        }
        vals[((size_t)kin * P + kout) * nch + si] = v;
      }
  for (int64_t out = 0; out < nout; ++out) {
    int bo[ORC_MAXD], bi[ORC_MAXD];
    orc_unrow(d, out, N, bo);
    int si = 0;
    for (int k = 0; k < d; ++k) { bi[k] = bo[k] / 2; si = si * 2 + bo[k] % 2; }
    int64_t in = orc_rowmajor(d, bi, N / 2);
    for (int kout = 0; kout < P; ++kout)
      for (int kin = 0; kin < P; ++kin) {
        double t = Win[in * P + kin];
        t *= vals[((size_t)kin * P + kout) * nch + si];
        Wout[out * P + kout] += t;
      }
  }
  free(vals);
}

/* L2P (src/fmm_core.cpp:580-615): sets ans then adds the interpolant. */
static void orc_l2p(const orc_setup* S, int64_t nt, const double* tgt, const double* origin,
                    double Len, int N, const double* Wl, double* ans) {
  int d = S->d, P = S->P;
  double len = Len / N;
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < nt; ++t) {
    int ib[ORC_MAXD];
    double rel[ORC_MAXD];
    orc_bin(d, tgt + t * d, origin, len, N, ib, rel);
    int64_t b = orc_rowmajor(d, ib, N);
    double dot = 0.0;
    for (int k = 0; k < P; ++k) {
      double v = 1.0;
      for (int q = 0; q < d; ++q) v *= orc_scheb(S->n, rel[q], S->node_all[k][q]);
      dot += Wl[b * P + k] * v;
    }
    ans[t] = 0.0;
    ans[t] += dot;
  }
}

/* fmm driver (src/fmm.cpp:15-144).  Returns the depth used (sticky default
 * resolved here), or -1 on an unsupported size.  ans must hold nt values and
 * is zeroed first (the reference relies on a freshly constructed vector). */
int orc_fmm(int d, int kid, double p0, int poly_ord, int depth, int trans_sym,
            int64_t nt, const double* tgt, int64_t ns, const double* src,
            const double* w, double* ans) {
  if (depth <= 0) depth = orc_default_depth(nt > 0 ? nt : 1, d);
  for (int64_t i = 0; i < nt; ++i) ans[i] = 0.0;
  if (nt == 0 || ns == 0) return depth;
  orc_setup* S = (orc_setup*)malloc(sizeof(orc_setup));
  S->d = d; S->n = poly_ord + 1; S->kid = kid; S->p0 = p0; S->trans_sym = trans_sym;
  S->P = 1;
  for (int k = 0; k < d; ++k) S->P *= S->n;
  if (S->n > 32 || S->P > 4096 || (int64_t)d * (depth - 1) > 30) { free(S); return -1; }
  orc_nodes(S);
  int P = S->P;

  double origin[ORC_MAXD], Len;
  orc_origin_len(d, nt, tgt, ns, src, origin, &Len);

  int L = depth;
  double** Wm = (double**)calloc((size_t)L, sizeof(double*));
  double** Wl = (double**)calloc((size_t)L, sizeof(double*));
  int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * (size_t)L);
  for (int l = 0; l < L; ++l) {
    int64_t c = 1;
    for (int k = 0; k < d; ++k) c *= (int64_t)1 << l;
    nb[l] = c;
  }
  int NL = 1 << (L - 1);
  int64_t* box_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nb[L - 1] + 1));
  int64_t* box_items = (int64_t*)malloc(sizeof(int64_t) * (size_t)ns);
  Wm[L - 1] = (double*)malloc(sizeof(double) * (size_t)(nb[L - 1] * P));
  orc_p2m(S, ns, src, w, NL, origin, Len / NL, box_start, box_items, Wm[L - 1]);

  /* M2M chain: levels L-2 .. 2 (src/fmm.cpp:62-70) */
  int tmpN = NL;
  for (int q = 0; q + 3 < L; ++q) {
    int l = L - q - 1;
    Wm[l - 1] = (double*)malloc(sizeof(double) * (size_t)(nb[l - 1] * P));
    orc_m2m(S, tmpN, Wm[l], Wm[l - 1]);
    tmpN /= 2;
  }
  for (int l = 2; l < L; ++l) Wl[l] = (double*)calloc((size_t)(nb[l] * P), sizeof(double));
  for (int l = 2; l < L; ++l) orc_m2l(S, 1 << l, origin, Len, Wm[l], Wl[l]);
  for (int l = 2; l + 1 < L; ++l) orc_l2l(S, 1 << (l + 1), Wl[l], Wl[l + 1]);
  if (L - 1 >= 2) orc_l2p(S, nt, tgt, origin, Len, NL, Wl[L - 1], ans);

  /* P2P (src/fmm.cpp:121-141) */
  double len = Len / NL;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < nt; ++t) {
    int ib[ORC_MAXD];
    int64_t lst[27];
    orc_bin(d, tgt + t * d, origin, len, NL, ib, NULL);
    int cnt = orc_near_list(d, ib, NL, lst);
    double a = ans[t];
    for (int i = 0; i < cnt; ++i)
      for (int64_t it = box_start[lst[i]]; it < box_start[lst[i] + 1]; ++it) {
        int64_t s = box_items[it];
        a += (w ? w[s] : 1.0) * orc_kernel(kid, p0, d, tgt + t * d, src + s * d);
      }
    ans[t] = a;
  }

  for (int l = 0; l < L; ++l) { free(Wm[l]); free(Wl[l]); }
  free(Wm); free(Wl); free(nb); free(box_start); free(box_items); free(S);
  return depth;
}

/* ---- tree (src/tree.cpp:12-100): P2M, M2M, M2P per level, P2P -------------
 * M2P (src/fmm_core.cpp:624-661): at every level l >= 2 each target adds
 * f(x_t, y_k) Wm[s][k] over the Chebyshev nodes y_k of every box s on its
 * far list at that level, the levels in increasing order; then the near
 * field of the leaf grid as in fmm. */
int orc_tree(int d, int kid, double p0, int poly_ord, int depth,
             int64_t nt, const double* tgt, int64_t ns, const double* src,
             const double* w, double* ans) {
  if (depth <= 0) depth = orc_default_depth(nt > 0 ? nt : 1, d);
  for (int64_t i = 0; i < nt; ++i) ans[i] = 0.0;
  if (nt == 0 || ns == 0) return depth;
  orc_setup* S = (orc_setup*)malloc(sizeof(orc_setup));
  S->d = d; S->n = poly_ord + 1; S->kid = kid; S->p0 = p0; S->trans_sym = 0;
  S->P = 1;
  for (int k = 0; k < d; ++k) S->P *= S->n;
  if (S->n > 32 || S->P > 4096 || (int64_t)d * (depth - 1) > 30) { free(S); return -1; }
  orc_nodes(S);
  int P = S->P;

  double origin[ORC_MAXD], Len;
  orc_origin_len(d, nt, tgt, ns, src, origin, &Len);

  int L = depth;
  double** Wm = (double**)calloc((size_t)L, sizeof(double*));
  int64_t* nb = (int64_t*)malloc(sizeof(int64_t) * (size_t)L);
  for (int l = 0; l < L; ++l) {
    int64_t c = 1;
    for (int k = 0; k < d; ++k) c *= (int64_t)1 << l;
    nb[l] = c;
  }
  int NL = 1 << (L - 1);
  int64_t* box_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nb[L - 1] + 1));
  int64_t* box_items = (int64_t*)malloc(sizeof(int64_t) * (size_t)ns);
  Wm[L - 1] = (double*)malloc(sizeof(double) * (size_t)(nb[L - 1] * P));
  orc_p2m(S, ns, src, w, NL, origin, Len / NL, box_start, box_items, Wm[L - 1]);
  int tmpN = NL;
  for (int q = 0; q + 3 < L; ++q) {
    int l = L - q - 1;
    Wm[l - 1] = (double*)malloc(sizeof(double) * (size_t)(nb[l - 1] * P));
    orc_m2m(S, tmpN, Wm[l], Wm[l - 1]);
    tmpN /= 2;
  }

  /* M2P, levels 2 .. L-1 */
  for (int l = 2; l < L; ++l) {
    const int N = 1 << l;
    const double len = Len / N;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < nt; ++t) {
      int ib[ORC_MAXD], is[ORC_MAXD];
      int64_t lst[189];
      orc_bin(d, tgt + t * d, origin, len, N, ib, NULL);
      int cnt = orc_far_list(d, ib, N, lst);
      double a = ans[t];
      for (int i = 0; i < cnt; ++i) {
        orc_unrow(d, lst[i], N, is);
        double corner[ORC_MAXD];
        for (int q = 0; q < d; ++q) corner[q] = len * is[q] + origin[q];
        for (int k = 0; k < P; ++k) {
          double y[ORC_MAXD];
          for (int q = 0; q < d; ++q) y[q] = (S->node_all[k][q] + 1.0) / 2.0 * len + corner[q];
          a += orc_kernel(kid, p0, d, tgt + t * d, y) * Wm[l][lst[i] * P + k];
        }
      }
      ans[t] = a;
    }
  }

  /* P2P (src/tree.cpp:80-96) */
  double len = Len / NL;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < nt; ++t) {
    int ib[ORC_MAXD];
    int64_t lst[27];
    orc_bin(d, tgt + t * d, origin, len, NL, ib, NULL);
    int cnt = orc_near_list(d, ib, NL, lst);
    double a = ans[t];
    for (int i = 0; i < cnt; ++i)
      for (int64_t it = box_start[lst[i]]; it < box_start[lst[i] + 1]; ++it) {
        int64_t s = box_items[it];
        a += (w ? w[s] : 1.0) * orc_kernel(kid, p0, d, tgt + t * d, src + s * d);
      }
    ans[t] = a;
  }

  for (int l = 0; l < L; ++l) free(Wm[l]);
  free(Wm); free(nb); free(box_start); free(box_items); free(S);
  return depth;
}

/* ---- nrnmm (src/nrnmm.cpp:13-102): one grid of nrn^d boxes ---------------
 * P2M on the grid (src/fmm_core.cpp:224-283); then every target visits the
 * boxes in row-major order: the sources of a box within one step of its own
 * box in every dimension directly, every other box through its Chebyshev
 * nodes weighted by Wm (node positions (x_k + 1) / 2 * len + (len * i +
 * origin), src/nrnmm.cpp:72-74 and :88-90).  nrn <= 0 selects the default
 * (int)(sqrt(3) * ns^(1/(2d))) + 1 (src/nrnmm.cpp:20-22), returned. */
int orc_default_nrn(int64_t ns, int d) {
  return (int)(sqrt(3.0) * pow((double)ns, 1.0 / (2.0 * d))) + 1;
}

int orc_nrnmm(int d, int kid, double p0, int poly_ord, int nrn,
              int64_t nt, const double* tgt, int64_t ns, const double* src,
              const double* w, double* ans) {
  if (nrn <= 0) nrn = orc_default_nrn(ns, d);
  for (int64_t i = 0; i < nt; ++i) ans[i] = 0.0;
  if (nt == 0 || ns == 0) return nrn;
  orc_setup* S = (orc_setup*)malloc(sizeof(orc_setup));
  S->d = d; S->n = poly_ord + 1; S->kid = kid; S->p0 = p0; S->trans_sym = 0;
  S->P = 1;
  for (int k = 0; k < d; ++k) S->P *= S->n;
  int64_t nbox = 1;
  for (int k = 0; k < d; ++k) nbox *= nrn;
  if (S->n > 32 || S->P > 4096 || nbox > ((int64_t)1 << 26)) { free(S); return -1; }
  orc_nodes(S);
  const int P = S->P;
  double origin[ORC_MAXD], Len;
  orc_origin_len(d, nt, tgt, ns, src, origin, &Len);
  const double len = Len / nrn;
  int64_t* box_start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nbox + 1));
  int64_t* box_items = (int64_t*)malloc(sizeof(int64_t) * (size_t)ns);
  double* Wm = (double*)malloc(sizeof(double) * (size_t)(nbox * P));
  orc_p2m(S, ns, src, w, nrn, origin, len, box_start, box_items, Wm);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t t = 0; t < nt; ++t) {
    const double* x = tgt + t * d;
    int ib[ORC_MAXD], is[ORC_MAXD];
    orc_bin(d, x, origin, len, nrn, ib, NULL);
    double a = 0.0;
    for (int64_t s = 0; s < nbox; ++s) {
      orc_unrow(d, s, nrn, is);
      int dist = 0;
      double corner[ORC_MAXD];
      for (int q = 0; q < d; ++q) {
        corner[q] = len * is[q] + origin[q];
        int e = abs(is[q] - ib[q]);
        if (e > dist) dist = e;
      }
      if (dist <= 1) {
        for (int64_t it = box_start[s]; it < box_start[s + 1]; ++it) {
          int64_t j = box_items[it];
          a += (w ? w[j] : 1.0) * orc_kernel(kid, p0, d, x, src + j * d);
        }
      } else {
        for (int k = 0; k < P; ++k) {
          double y[ORC_MAXD];
          for (int q = 0; q < d; ++q) y[q] = (S->node_all[k][q] + 1.0) / 2.0 * len + corner[q];
          a += orc_kernel(kid, p0, d, x, y) * Wm[s * P + k];
        }
      }
    }
    ans[t] = a;
  }
  free(box_start); free(box_items); free(Wm); free(S);
  return nrn;
}

/* ---- global Chebyshev approximation (src/chebyshev_approx.cpp:36-97) -------
 * The reference's collocation system Mat[i][j] = prod_q T_{j_q}(x_{i_q})
 * (T_k(x) = cos(k acos x), src/math.cpp:14-26; flat indices with dimension
 * 0 fastest) is solved here by Gaussian elimination with partial pivoting,
 * the deterministic exact solution that the reference's GCR iteration (from
 * a random start, stopping at a squared residual of 1e-6) approaches. */
static int orc_cheb_size(int dim, int nth) {
  int s = 1;
  for (int q = 0; q < dim; ++q) s *= nth + 1;
  return s;
}

int orc_cheb_fit(int dim, int nth, const double* values, double* coef) {
  const int n = nth + 1, N = orc_cheb_size(dim, nth);
  if (N > 4096) return -1;
  double* M = (double*)malloc(sizeof(double) * (size_t)N * (N + 1));
  double node[64];
  if (n > 64) { free(M); return -1; }
  for (int k = 0; k < n; ++k) node[k] = cos((2.0 * k + 1.0) / (2 * nth + 2) * M_PI);
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < N; ++j) {
      int ic = i, jc = j;
      double v = 1.0;
      for (int q = 0; q < dim; ++q) {
        v *= orc_cheb(jc % n, node[ic % n]);
        ic /= n;
        jc /= n;
      }
      M[(size_t)i * (N + 1) + j] = v;
    }
    M[(size_t)i * (N + 1) + N] = values[i];
  }
  for (int c = 0; c < N; ++c) {
    int piv = c;
    for (int r = c + 1; r < N; ++r)
      if (fabs(M[(size_t)r * (N + 1) + c]) > fabs(M[(size_t)piv * (N + 1) + c])) piv = r;
    if (piv != c)
      for (int k = 0; k <= N; ++k) {
        double t = M[(size_t)c * (N + 1) + k];
        M[(size_t)c * (N + 1) + k] = M[(size_t)piv * (N + 1) + k];
        M[(size_t)piv * (N + 1) + k] = t;
      }
    const double d = M[(size_t)c * (N + 1) + c];
    for (int r = c + 1; r < N; ++r) {
      const double f = M[(size_t)r * (N + 1) + c] / d;
      if (f == 0.0) continue;
      for (int k = c; k <= N; ++k) M[(size_t)r * (N + 1) + k] -= f * M[(size_t)c * (N + 1) + k];
    }
  }
  for (int c = N - 1; c >= 0; --c) {
    double s = M[(size_t)c * (N + 1) + N];
    for (int k = c + 1; k < N; ++k) s -= M[(size_t)c * (N + 1) + k] * coef[k];
    coef[c] = s / M[(size_t)c * (N + 1) + c];
  }
  free(M);
  return N;
}

/* predict (src/chebyshev_approx.cpp:88-101): sum_i coef[i] prod_q T_{i_q}(x_q),
 * in the reference's loop order.  Points outside [-1, 1] give NaN (the
 * reference exits). */
void orc_cheb_eval(int dim, int nth, const double* coef, int64_t npts, const double* pts, double* out) {
  const int n = nth + 1, N = orc_cheb_size(dim, nth);
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npts; ++p) {
    double ans = 0.0;
    for (int i = 0; i < N; ++i) {
      int ic = i;
      double v = 1.0;
      for (int q = 0; q < dim; ++q) {
        v *= orc_cheb(ic % n, pts[p * dim + q]);
        ic /= n;
      }
      ans += coef[i] * v;
    }
    out[p] = ans;
  }
}
