/*
 * bpx_oracle.c -- CPU oracle for the bedpostx per-voxel path.  TEST INFRASTRUCTURE ONLY.
 *
 * FP64 restatement of xfibres_gpu's per-voxel arithmetic, written from the reference's
 * semantics (file:line cited at each function).  Used by tests/ as the checker and by
 * bench.py as the timed CPU baseline; the product library never links it.
 *
 * Where the reference's GPU and CPU paths differ, this file follows the GPU path
 * (xfibres_gpu is the path being replaced); each such place says so.
 */
#include "bpx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_PI_GPU 0.636619772 /* CUDA/diffmodels_utils.h:13 */
#define FSMALL 0.001           /* CUDA/diffmodels_utils.h:16 */
#define UPPERDIFF 0.005        /* CUDA/runmcmc_kernels.cu:24 */
#define MAXFLOAT_PROP 1e10     /* CUDA/runmcmc_kernels.cu:23 */
#define MAXP 16
#define MAXK BPX_MAX_FIBRES

int bpx_nparams_fit_c(const bpx_options* o);

/* ------------------------------------------------------------------------------------------ */
/* Philox-4x32-10 (Salmon et al., SC11): 10 rounds of two 32x32->64 multiplies, Weyl key bumps. */
/* ------------------------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* 24-bit uniforms, exact in float and double: (0,1] and [0,1). */
static double u01_open0(uint32_t x) { return (double)((x >> 8) + 1u) * (1.0 / 16777216.0); }
static double u01_open1(uint32_t x) { return (double)(x >> 8) * (1.0 / 16777216.0); }

void orc_rng_slot(uint64_t seed, uint64_t vox, uint32_t iter, uint32_t slot, double* normal,
                  double* log_u) {
  uint32_t ctr[4] = {iter, slot, (uint32_t)vox, (uint32_t)(vox >> 32)};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t r[4];
  orc_philox4x32_10(ctr, key, r);
  /* Box-Muller from r0, r1; acceptance uniform from r2 */
  double u0 = u01_open0(r[0]), u1 = u01_open1(r[1]);
  *normal = sqrt(-2.0 * log(u0)) * cos(6.283185307179586 * u1);
  *log_u = log(u01_open0(r[2]));
}

/* log of the modified Bessel function I0, polynomial approximations of Abramowitz & Stegun
 * 9.8.1/9.8.2 as used by fibre.h:31-51 and CUDA/runmcmc_kernels.cu:126-145. */
double orc_logI0(double x) {
  double b = fabs(x);
  if (b < 3.75) {
    double a = x / 3.75;
    a *= a;
    double y = 1.0 + a * (3.5156229 + a * (3.0899424 + a * (1.2067492 + a * (0.2659732 + a * (0.0360768 + a * 0.0045813)))));
    return log(y);
  }
  double a = 3.75 / b;
  double p = 0.39894228 + a * (0.01328592 + a * (0.00225319 + a * (-0.00157565 + a * (0.00916281 + a * (-0.02057706 + a * (0.02635537 + a * (-0.01647633 + a * 0.00392377)))))));
  return b + log(p / sqrt(b));
}

/* ------------------------------------------------------------------------------------------ */
/* small dense linear algebra                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* symmetric eigen-decomposition by cyclic Jacobi rotations; eigenvalues descending, vectors in
 * columns of V (n <= 8).  Each eigenvector is signed so that its largest-magnitude component is
 * positive. */
static void jacobi_eig(int n, const double* Ain, double* w, double* V) {
  double A[64];
  memcpy(A, Ain, sizeof(double) * n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (fabs(apq) < 1e-300) continue;
        double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
    }
  }
  int idx[8];
  for (int i = 0; i < n; ++i) idx[i] = i;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (A[idx[j] * n + idx[j]] > A[idx[i] * n + idx[i]]) {
        int t = idx[i];
        idx[i] = idx[j];
        idx[j] = t;
      }
  double Vs[64];
  for (int c = 0; c < n; ++c) {
    w[c] = A[idx[c] * n + idx[c]];
    int big = 0;
    for (int r = 1; r < n; ++r)
      if (fabs(V[r * n + idx[c]]) > fabs(V[big * n + idx[c]])) big = r;
    double sg = V[big * n + idx[c]] < 0 ? -1.0 : 1.0;
    for (int r = 0; r < n; ++r) Vs[r * n + c] = sg * V[r * n + idx[c]];
  }
  memcpy(V, Vs, sizeof(double) * n * n);
}

/* Moore-Penrose pseudo-inverse of A [m][n] (n <= 8) through the eigen-decomposition of A^T A:
 * pinv = (A^T A)^+ A^T.  P is [n][m]. */
static void pinv_tall(int m, int n, const double* A, double* P) {
  double G[64], w[8], V[64];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0;
      for (int r = 0; r < m; ++r) s += A[r * n + i] * A[r * n + j];
      G[i * n + j] = s;
    }
  jacobi_eig(n, G, w, V);
  double tol = w[0] * 1e-14 * (m > n ? m : n);
  double Gi[64];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0;
      for (int c = 0; c < n; ++c)
        if (w[c] > tol) s += V[i * n + c] * V[j * n + c] / w[c];
      Gi[i * n + j] = s;
    }
  for (int i = 0; i < n; ++i)
    for (int r = 0; r < m; ++r) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += Gi[i * n + j] * A[r * n + j];
      P[i * m + r] = s;
    }
}

/* Solve A x = b by LU with partial pivoting (the newmat GeneralSolvI scheme that
 * CUDA/solver_mult_inverse.cu:14-166 restates).  Returns 0 if singular. */
static int lu_solve(int n, const double* Ain, const double* b, double* x) {
  double A[MAXP * MAXP], y[MAXP];
  int piv[MAXP];
  memcpy(A, Ain, sizeof(double) * n * n);
  memcpy(y, b, sizeof(double) * n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i * n + k]) > fabs(A[p * n + k])) p = i;
    piv[k] = p;
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        double t = A[k * n + j];
        A[k * n + j] = A[p * n + j];
        A[p * n + j] = t;
      }
      double t = y[k];
      y[k] = y[p];
      y[p] = t;
    }
    double d = A[k * n + k];
    if (d == 0.0) continue;
    for (int i = k + 1; i < n; ++i) {
      double mlt = A[i * n + k] / d;
      A[i * n + k] = mlt;
      for (int j = k + 1; j < n; ++j) A[i * n + j] -= mlt * A[k * n + j];
      y[i] -= mlt * y[k];
    }
  }
  (void)piv;
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * x[j];
    if (A[i * n + i] == 0.0) return 0;
    x[i] = s / A[i * n + i];
  }
  return 1;
}

/* ------------------------------------------------------------------------------------------ */
/* transforms (CUDA/diffmodels_utils.h:13-41, diffmodels.h)                                    */
/* ------------------------------------------------------------------------------------------ */
static double x2f(double x) { return fabs(TWO_PI_GPU * atan(x)); }
static double f2x(double f) { return tan(f / TWO_PI_GPU); }
static double beta2f(double b) {
  double s = sin(b);
  return s * s;
}
static double f2beta(double f) { return asin(sqrt(f)); }
static int sgn(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
static double pm1(double x) { return x > 0 ? 1.0 : -1.0; }

/* Spherical angles of a 3-vector, polar angle th in [0,pi] and azimuth ph in (-pi,pi]
 * (the convention of FSL miscmaths cart2sph, called at diffmodels.cc:452 and
 * CUDA/diffmodels.cu:70; that library is not in the reference tree). */
static void cart2sph(const double* v, double* th, double* ph) {
  double x = v[0], y = v[1], z = v[2];
  double mag = sqrt(x * x + y * y + z * z);
  if (mag == 0) {
    *ph = M_PI / 2;
    *th = M_PI / 2;
    return;
  }
  if (x == 0 && y >= 0)
    *ph = M_PI / 2;
  else if (x == 0 && y < 0)
    *ph = -M_PI / 2;
  else if (x > 0)
    *ph = atan(y / x);
  else if (y > 0)
    *ph = atan(y / x) + M_PI;
  else
    *ph = atan(y / x) - M_PI;
  double r = sqrt(x * x + y * y);
  if (z == 0)
    *th = M_PI / 2;
  else if (z > 0)
    *th = atan(r / z);
  else
    *th = atan(r / z) + M_PI;
}

static void sph2vec(double th, double ph, double* v) {
  v[0] = sin(th) * cos(ph);
  v[1] = sin(th) * sin(ph);
  v[2] = cos(th);
}

/* ------------------------------------------------------------------------------------------ */
/* DTI log-linear fit (diffmodels.cc:17-46, diffmodels.h:148-163, diffmodels.cc:239-266)      */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  double s0, md, fa, l1, l2, l3, v1[3], v2[3], v3[3], sse;
} dti_t;

static void dti_fit(int ndir, const float* Y, const float* bvecs, const float* bvals,
                    const double* iA /* pinv(Amat) [7][ndir] */, const double* Amat, dti_t* o) {
  double logS[1024], D[7];
  double ymax = 0, ysum = 0;
  for (int i = 0; i < ndir; ++i) {
    logS[i] = Y[i] > 0 ? log((double)Y[i]) : 0.0;
    if (fabs(Y[i]) > ymax) ymax = fabs(Y[i]);
    ysum += Y[i];
  }
  double ymean = ysum / ndir;
  for (int r = 0; r < 7; ++r) {
    double s = 0;
    for (int i = 0; i < ndir; ++i) s += iA[r * ndir + i] * logS[i];
    D[r] = -s;
  }
  double s0 = D[6] > -23 ? exp(-D[6]) : ymax;
  for (int i = 0; i < ndir; ++i) {
    if (s0 < ymean) s0 = ymax;
    logS[i] = (Y[i] / s0) > 0.01 ? log((double)Y[i]) : log(0.01 * s0);
  }
  for (int r = 0; r < 7; ++r) {
    double s = 0;
    for (int i = 0; i < ndir; ++i) s += iA[r * ndir + i] * logS[i];
    D[r] = -s;
  }
  double sse = 0;
  for (int i = 0; i < ndir; ++i) {
    double s = logS[i];
    for (int r = 0; r < 7; ++r) s += Amat[i * 7 + r] * D[r];
    sse += s * s;
  }
  s0 = exp(-D[6]);
  if (s0 < ymean) s0 = ymean;
  double T[9] = {D[0], D[1], D[2], D[1], D[3], D[4], D[2], D[4], D[5]};
  double w[3], V[9];
  jacobi_eig(3, T, w, V);
  o->s0 = s0;
  o->sse = sse;
  o->l1 = w[0];
  o->l2 = w[1];
  o->l3 = w[2];
  o->md = (w[0] + w[1] + w[2]) / 3.0;
  for (int r = 0; r < 3; ++r) {
    o->v1[r] = V[r * 3 + 0];
    o->v2[r] = V[r * 3 + 1];
    o->v3[r] = V[r * 3 + 2];
  }
  double numer = 1.5 * ((o->l1 - o->md) * (o->l1 - o->md) + (o->l2 - o->md) * (o->l2 - o->md) +
                        (o->l3 - o->md) * (o->l3 - o->md));
  double denom = o->l1 * o->l1 + o->l2 * o->l2 + o->l3 * o->l3;
  double fa = denom > 0 ? numer / denom : 0;
  o->fa = fa > 0 ? sqrt(fa) : 0;
}

static void form_amat(int ndir, const float* bvecs, const float* bvals, double* Amat) {
  for (int i = 0; i < ndir; ++i) {
    double gx = bvecs[i], gy = bvecs[ndir + i], gz = bvecs[2 * ndir + i], b = bvals[i];
    double* a = Amat + i * 7;
    a[0] = b * gx * gx;
    a[1] = 2 * b * gx * gy;
    a[2] = 2 * b * gx * gz;
    a[3] = b * gy * gy;
    a[4] = 2 * b * gy * gz;
    a[5] = b * gz * gz;
    a[6] = 1;
  }
}

int orc_dti(int ndir, const float* y, const float* bvecs, const float* bvals, double* out) {
  if (ndir < 7 || ndir > 1024) return -1;
  double* A = (double*)malloc(sizeof(double) * ndir * 7);
  double* iA = (double*)malloc(sizeof(double) * ndir * 7);
  form_amat(ndir, bvecs, bvals, A);
  pinv_tall(ndir, 7, A, iA);
  dti_t d;
  dti_fit(ndir, y, bvecs, bvals, iA, A, &d);
  out[0] = d.s0;
  out[1] = d.md;
  out[2] = d.fa;
  out[3] = d.l1;
  out[4] = d.l2;
  out[5] = d.l3;
  for (int r = 0; r < 3; ++r) {
    out[6 + r] = d.v1[r];
    out[9 + r] = d.v2[r];
    out[12 + r] = d.v3[r];
  }
  out[15] = d.sse;
  free(A);
  free(iA);
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* LM models (GPU versions: CUDA/PVM_single.cu, CUDA/PVM_single_c.cu, CUDA/PVM_multi.cu)       */
/* ------------------------------------------------------------------------------------------ */
enum { KIND_SINGLE = 0, KIND_SINGLE_C = 1, KIND_MULTI = 2 };

typedef struct {
  int kind, nfib, f0, np, ndir, gbo;
  double R, invR;
  const float *y, *gx, *gy, *gz, *b;
} lmctx;

typedef struct {
  double fs[MAXK], v[MAXK][3], sumf, d, a, bb, sth[MAXK], cth[MAXK], sph[MAXK], cph[MAXK];
  double deriv[MAXK][MAXK]; /* single_c: d f_j / d beta_k */
} lmpre;

static void lm_pre(const lmctx* c, const double* p, lmpre* q) {
  int K = c->nfib, o = (c->kind == KIND_MULTI) ? 3 : 2;
  for (int k = 0; k < K; ++k) {
    double th = p[o + 3 * k + 1], ph = p[o + 3 * k + 2];
    q->sth[k] = sin(th);
    q->cth[k] = cos(th);
    q->sph[k] = sin(ph);
    q->cph[k] = cos(ph);
    q->v[k][0] = q->sth[k] * q->cph[k];
    q->v[k][1] = q->sth[k] * q->sph[k];
    q->v[k][2] = q->cth[k];
  }
  q->sumf = 0;
  if (c->kind == KIND_SINGLE) {
    q->d = fabs(p[1]);
    for (int k = 0; k < K; ++k) {
      q->fs[k] = x2f(p[2 + 3 * k]);
      q->sumf += q->fs[k];
    }
  } else if (c->kind == KIND_SINGLE_C) {
    q->d = p[1] * p[1];
    for (int k = 0; k < K; ++k) {
      double pf = 1.0;
      for (int j = 0; j < k; ++j) pf -= q->fs[j];
      q->fs[k] = beta2f(p[2 + 3 * k]) * pf;
      q->sumf += q->fs[k];
    }
    /* fractions_deriv_PVM_single_c (CUDA/PVM_single_c.cu:104-139) */
    for (int k = 0; k < K; ++k) {
      for (int j = 0; j < K; ++j) q->deriv[j][k] = 0;
      double s2k = sin(2 * p[2 + 3 * k]);
      for (int j = 0; j < K; ++j) {
        if (j == k) {
          double fsum = 1;
          for (int n = 0; n <= j - 1; ++n) fsum -= q->fs[n];
          q->deriv[j][k] = s2k * fsum;
        } else if (j > k) {
          double sp = sin(p[2 + 3 * j]);
          double fsum = 0;
          for (int n = 0; n <= j - 1; ++n) fsum += q->deriv[n][k];
          q->deriv[j][k] = -(sp * sp) * fsum;
        }
      }
    }
  } else {
    q->a = fabs(p[1]);
    q->bb = fabs(p[2]);
    for (int k = 0; k < K; ++k) {
      q->fs[k] = x2f(p[3 + 3 * k]);
      q->sumf += q->fs[k];
    }
  }
}

/* Per-measurement prediction and Jacobian rows.  Jg is the row used for the gradient, Jh the
 * row used for the Hessian (they differ only in PVM_multi's S0 entry, CUDA/PVM_multi.cu:376
 * vs :452).  Returns the predicted signal. */
static double lm_point(const lmctx* c, const double* p, const lmpre* q, int m, double* Jg,
                       double* Jh) {
  int K = c->nfib, np = c->np;
  double gx = c->gx[m], gy = c->gy[m], gz = c->gz[m], b = c->b[m];
  double dp[MAXK], an[MAXK];
  for (int k = 0; k < K; ++k) dp[k] = gx * q->v[k][0] + gy * q->v[k][1] + gz * q->v[k][2];
  if (c->kind == KIND_SINGLE || c->kind == KIND_SINGLE_C) {
    double d = q->d, iso = exp(-b * d), sig = 0;
    for (int k = 0; k < K; ++k) {
      an[k] = exp(-b * d * dp[k] * dp[k]);
      sig += q->fs[k] * an[k];
    }
    if (!Jg) {
      if (c->f0) {
        double f0v;
        if (c->kind == KIND_SINGLE)
          f0v = x2f(p[np - 1]);
        else
          f0v = beta2f(p[np - 1]) * (1.0 - q->sumf);
        return p[0] * ((f0v + (1 - q->sumf - f0v) * iso) + sig);
      }
      return p[0] * ((1 - q->sumf) * iso + sig);
    }
    for (int i = 0; i < np; ++i) Jg[i] = 0;
    int o = 2;
    if (c->kind == KIND_SINGLE) {
      for (int k = 0; k < K; ++k) {
        int kk = o + 3 * k;
        Jg[1] += pm1(p[1]) * p[0] * q->fs[k] * (-b * dp[k] * dp[k] * an[k]);
        Jg[kk] = p[0] * (an[k] - iso) * TWO_PI_GPU * sgn(p[kk]) / (1 + p[kk] * p[kk]);
      }
    } else {
      double lam = p[1];
      for (int k = 0; k < K; ++k) {
        int kk = o + 3 * k;
        Jg[1] += p[0] * q->fs[k] * (-2 * b * lam * dp[k] * dp[k] * exp(-b * lam * lam * dp[k] * dp[k]));
        double s = 0;
        for (int j = 0; j < K; ++j)
          if (q->deriv[j][k] != 0) s += p[0] * (an[j] - iso) * q->deriv[j][k];
        Jg[kk] = s;
      }
    }
    for (int k = 0; k < K; ++k) {
      int kk = o + 3 * k;
      double dp1 = q->cth[k] * (gx * q->cph[k] + gy * q->sph[k]) - gz * q->sth[k];
      double dp2 = q->sth[k] * (-gx * q->sph[k] + gy * q->cph[k]);
      Jg[kk + 1] = p[0] * q->fs[k] * (-2 * b * d * dp[k] * dp1 * an[k]);
      Jg[kk + 2] = p[0] * q->fs[k] * (-2 * b * d * dp[k] * dp2 * an[k]);
    }
    if (c->f0) {
      double f0v;
      if (c->kind == KIND_SINGLE) {
        f0v = x2f(p[np - 1]);
        Jg[np - 1] = p[0] * (1 - iso) * TWO_PI_GPU * sgn(p[np - 1]) / (1 + p[np - 1] * p[np - 1]);
      } else {
        double pfs = 1.0 - q->sumf;
        f0v = beta2f(p[np - 1]) * pfs;
        Jg[np - 1] = p[0] * (1 - iso) * sin(2 * p[np - 1]) * pfs;
      }
      sig = p[0] * ((f0v + (1 - q->sumf - f0v) * iso) + sig);
      if (c->kind == KIND_SINGLE)
        Jg[1] += pm1(p[1]) * p[0] * (1 - q->sumf - f0v) * (-b * iso);
      else
        Jg[1] += p[0] * (1 - q->sumf - f0v) * (-2 * b * p[1] * exp(-b * p[1] * p[1]));
    } else {
      sig = p[0] * ((1 - q->sumf) * iso + sig);
      if (c->kind == KIND_SINGLE)
        Jg[1] += pm1(p[1]) * p[0] * (1 - q->sumf) * (-b * iso);
      else
        Jg[1] += p[0] * (1 - q->sumf) * (-2 * b * p[1] * exp(-b * p[1] * p[1]));
    }
    Jg[0] = sig / p[0];
    if (Jh)
      for (int i = 0; i < np; ++i) Jh[i] = Jg[i];
    return sig;
  }
  /* PVM_multi */
  double a = q->a, bb = q->bb, R = c->R, invR = c->invR;
  double iso = exp(-a * log(1 + b * bb)), sig = 0;
  double an_a[MAXK], an_b[MAXK], an_th[MAXK], an_ph[MAXK];
  for (int k = 0; k < K; ++k) {
    double x2 = dp[k] * dp[k];
    double dp1 = q->cth[k] * (gx * q->cph[k] + gy * q->sph[k]) - gz * q->sth[k];
    double dpp = q->sth[k] * (-gx * q->sph[k] + gy * q->cph[k]);
    if (c->gbo == 1) {
      an[k] = exp(-b * a * bb * x2);
      an_a[k] = -b * bb * x2 * an[k];
      an_b[k] = -b * a * x2 * an[k];
      an_th[k] = -2 * b * a * bb * dp[k] * dp1 * an[k];
      an_ph[k] = -2 * b * a * bb * dp[k] * dpp * an[k];
    } else if (c->gbo == 2) {
      double e = exp(-b * 3 * a * bb * invR * ((1 - R) * x2 + R));
      an[k] = e;
      double da = b * 3 * bb * invR * ((1 - R) * x2 + R);
      an_a[k] = -da * exp(-da * a);
      double db = b * 3 * a * invR * ((1 - R) * x2 + R);
      an_b[k] = -db * exp(-db * bb);
      /* CUDA/PVM_multi.cu:82-84,99-101: the zeppelin angle derivatives lack the factor dp */
      an_th[k] = -(2 * b * 3 * a * bb * invR * (1 - R) * dp1) * e;
      an_ph[k] = -(2 * b * 3 * a * bb * invR * (1 - R) * dpp) * e;
    } else {
      double l = log(1 + b * bb * x2);
      an[k] = exp(-a * l);
      an_a[k] = -l * an[k];
      an_b[k] = -a * b * x2 / (1 + b * x2 * bb) * an[k];
      an_th[k] = -a * bb * b / (1 + b * x2 * bb) * an[k] * 2 * dp[k] * dp1;
      an_ph[k] = -a * bb * b / (1 + b * x2 * bb) * an[k] * 2 * dp[k] * dpp;
    }
    sig += q->fs[k] * an[k];
  }
  double S0 = fabs(p[0]);
  double f0v = c->f0 ? x2f(p[np - 1]) : 0.0;
  double wiso = c->f0 ? (1 - q->sumf - f0v) : (1 - q->sumf);
  if (!Jg) {
    if (c->f0) return S0 * (f0v + (wiso * iso + sig));
    return S0 * (wiso * iso + sig);
  }
  for (int i = 0; i < np; ++i) Jg[i] = 0;
  double iso_a = -log(1 + b * bb) * iso;
  double iso_b = -a * b / (1 + b * bb) * iso;
  for (int k = 0; k < K; ++k) {
    int kk = 3 + 3 * k;
    Jg[1] += pm1(p[1]) * S0 * q->fs[k] * an_a[k];
    Jg[2] += pm1(p[2]) * S0 * q->fs[k] * an_b[k];
    Jg[kk] = S0 * (an[k] - iso) * TWO_PI_GPU * sgn(p[kk]) / (1 + p[kk] * p[kk]);
    Jg[kk + 1] = S0 * q->fs[k] * an_th[k];
    Jg[kk + 2] = S0 * q->fs[k] * an_ph[k];
  }
  if (c->f0) {
    Jg[np - 1] = S0 * (1 - iso) * TWO_PI_GPU * sgn(p[np - 1]) / (1 + p[np - 1] * p[np - 1]);
    sig = S0 * ((f0v + wiso * iso) + sig);
  } else {
    sig = S0 * (wiso * iso + sig);
  }
  Jg[1] += pm1(p[1]) * S0 * wiso * iso_a;
  Jg[2] += pm1(p[2]) * S0 * wiso * iso_b;
  if (Jh) {
    for (int i = 0; i < np; ++i) Jh[i] = Jg[i];
    Jh[0] = sig / p[0];
  }
  Jg[0] = pm1(p[0]) * sig / p[0];
  return sig;
}

static double lm_cf(const lmctx* c, const double* p) {
  lmpre q;
  lm_pre(c, p, &q);
  double cf = 0;
  for (int m = 0; m < c->ndir; ++m) {
    double e = lm_point(c, p, &q, m, NULL, NULL) - c->y[m];
    cf += e * e;
  }
  return cf;
}

static void lm_gradhess(const lmctx* c, const double* p, double* g, double* H) {
  lmpre q;
  lm_pre(c, p, &q);
  int np = c->np;
  double Jg[MAXP], Jh[MAXP];
  for (int i = 0; i < np; ++i) g[i] = 0;
  for (int i = 0; i < np * np; ++i) H[i] = 0;
  for (int m = 0; m < c->ndir; ++m) {
    double sig = lm_point(c, p, &q, m, Jg, Jh);
    double diff = sig - c->y[m];
    for (int i = 0; i < np; ++i) {
      g[i] += 2 * Jg[i] * diff;
      for (int j = i; j < np; ++j) H[i * np + j] += 2 * Jh[i] * Jh[j];
    }
  }
  for (int i = 0; i < np; ++i)
    for (int j = i + 1; j < np; ++j) H[j * np + i] = H[i * np + j];
}

/* levenberg_marquardt_*_gpu (CUDA/levenberg_marquardt.cu:17-122): lambda0 0.1, x/÷10,
 * cftol 1e-8, ltol 1e20, at most 200 successful iterations.  *capped (if given) is set when the
 * run stopped at that cap instead of at the cost tolerance or the lambda limit. */
static int lm_run(const lmctx* c, double* p, int* capped) {
  int np = c->np, niter = 0, maxiter = 200, success = 1, iters = 0;
  double lambda = 0.1, cftol = 1e-8, ltol = 1e20;
  double pcf = lm_cf(c, p), ncf;
  double g[MAXP], H[MAXP * MAXP], Hd[MAXP * MAXP], st[MAXP], step[MAXP];
  int stopped = 0;
  while (!(success && niter++ >= maxiter)) {
    ++iters;
    if (success) lm_gradhess(c, p, g, H);
    memcpy(Hd, H, sizeof(double) * np * np);
    for (int i = 0; i < np; ++i) Hd[i * np + i] += lambda;
    if (!lu_solve(np, Hd, g, st))
      for (int i = 0; i < np; ++i) st[i] = 0;
    for (int i = 0; i < np; ++i) step[i] = p[i] - st[i];
    ncf = lm_cf(c, step);
    int end = 0;
    if ((success = (ncf < pcf))) {
      memcpy(p, step, sizeof(double) * np);
      lambda /= 10.0;
      if (2.0 * fabs(pcf - ncf) <= cftol * (fabs(pcf) + fabs(ncf) + 2.0e-16)) end = 1;
      pcf = ncf;
    } else {
      lambda *= 10.0;
      if (lambda > ltol) end = 1;
    }
    if (end) {
      stopped = 1;
      break;
    }
  }
  if (capped) *capped = !stopped;
  return iters;
}

static void lm_ctx_init(lmctx* c, int kind, int nfib, int f0, int gbo, double R, int ndir,
                        const float* y, const float* bvecs, const float* bvals) {
  c->kind = kind;
  c->nfib = nfib;
  c->f0 = f0;
  c->np = 3 * nfib + 2 + (kind == KIND_MULTI ? 1 : 0) + (f0 ? 1 : 0);
  c->ndir = ndir;
  c->gbo = gbo;
  c->R = R;
  c->invR = 1.0 / (2.0 * R + 1);
  c->y = y;
  c->gx = bvecs;
  c->gy = bvecs + ndir;
  c->gz = bvecs + 2 * ndir;
  c->b = bvals;
}

double orc_lm_eval(int kind, int nfib, int f0, int gamma_ball_only, double R, int ndir,
                   const float* y, const float* bvecs, const float* bvals, const double* p,
                   double* grad, double* hess) {
  lmctx c;
  lm_ctx_init(&c, kind, nfib, f0, gamma_ball_only, R, ndir, y, bvecs, bvals);
  if (grad && hess) lm_gradhess(&c, p, grad, hess);
  return lm_cf(&c, p);
}

/* sort fibres by decreasing f: sort_PVM_* (CUDA/PVM_single.cu:86-104) -- adjacent swaps */
static void sort_fibres(int nfib, int o, double* p) {
  for (int i = 1; i < nfib; ++i)
    for (int j = 0; j < nfib - i; ++j)
      if (p[o + j * 3] < p[o + (j + 1) * 3])
        for (int t = 0; t < 3; ++t) {
          double tmp = p[o + j * 3 + t];
          p[o + j * 3 + t] = p[o + (j + 1) * 3 + t];
          p[o + (j + 1) * 3 + t] = tmp;
        }
}

/* finalise raw LM parameters into [S0, d, (dstd), (f,th,ph)*K, (f0)]
 * (CUDA/PVM_single.cu:451-466, CUDA/PVM_single_c.cu:582-607, CUDA/PVM_multi.cu:549-566) */
static void lm_finalise(const lmctx* c, double* p) {
  int K = c->nfib, np = c->np;
  if (c->kind == KIND_SINGLE) {
    p[1] = fabs(p[1]);
    for (int k = 0; k < K; ++k) p[2 + 3 * k] = x2f(p[2 + 3 * k]);
    if (c->f0) p[np - 1] = x2f(p[np - 1]);
    sort_fibres(K, 2, p);
    /* fix_fsum_PVM_single (CUDA/PVM_single.cu:68-84) */
    double sum = c->f0 ? p[np - 1] : 0;
    for (int i = 0; i < K; ++i) {
      sum += p[2 + 3 * i];
      if (sum >= 1) {
        for (int j = i; j < K; ++j) p[2 + 3 * j] = FSMALL;
        break;
      }
    }
  } else if (c->kind == KIND_SINGLE_C) {
    p[1] = p[1] * p[1];
    for (int k = 0; k < K; ++k) {
      double pf = 1.0;
      for (int j = 0; j < k; ++j) pf -= p[2 + 3 * j];
      p[2 + 3 * k] = beta2f(p[2 + 3 * k]) * pf;
    }
    if (c->f0) {
      double pf = 1.0;
      for (int j = 0; j < K; ++j) pf -= p[2 + 3 * j];
      p[np - 1] = beta2f(p[np - 1]) * pf;
    }
    sort_fibres(K, 2, p);
  } else {
    double aux = p[1];
    p[1] = fabs(aux * p[2]);
    p[2] = sqrt(fabs(aux * p[2] * p[2]));
    for (int k = 0; k < K; ++k) p[3 + 3 * k] = x2f(p[3 + 3 * k]);
    if (c->f0) p[np - 1] = x2f(p[np - 1]);
    sort_fibres(K, 3, p);
    /* fix_fsum_PVM_multi (CUDA/PVM_multi.cu:105-123) */
    double sum = c->f0 ? p[np - 1] : 0;
    for (int i = 0; i < K; ++i) {
      if (p[3 + 3 * i] == 0) p[3 + 3 * i] = FSMALL;
      sum += p[3 + 3 * i];
      if (sum >= 1) {
        for (int j = i; j < K; ++j) p[3 + 3 * j] = FSMALL;
        break;
      }
    }
  }
}

/* start values.  PVM_single: CUDA/diffmodels.cu:57-94; PVM_single_c: CUDA/diffmodels.cu:149-184
 * with fit_pvf (diffmodels.cc:561-603). */
static void start_single(int nfib, int f0, const dti_t* dt, double* p) {
  double th, ph;
  int np = 3 * nfib + 2 + (f0 ? 1 : 0);
  cart2sph(dt->v1, &th, &ph);
  p[0] = dt->s0;
  p[1] = dt->md > 0 ? dt->md * 2 : 0.001;
  p[2] = dt->fa < 1 ? f2x(dt->fa) : f2x(0.95);
  p[3] = th;
  p[4] = ph;
  double sumf = x2f(p[2]), tmpsumf;
  const double* vs[3] = {dt->v1, dt->v2, dt->v3};
  for (int ii = 2, i = 5; ii <= nfib; ii++, i += 3) {
    double denom = 2;
    do {
      p[i] = f2x(x2f(p[i - 3]) / denom);
      denom *= 2;
      tmpsumf = sumf + x2f(p[i]);
    } while (tmpsumf >= 1);
    sumf += x2f(p[i]);
    cart2sph(vs[ii - 1], &th, &ph);
    p[i + 1] = th;
    p[i + 2] = ph;
  }
  if (f0) p[np - 1] = f2x(FSMALL);
}

static void start_single_c(int nfib, int f0, const dti_t* dt, int ndir, const float* Y,
                           const float* bvecs, const float* bvals, double* x) {
  double th, ph;
  int np = 3 * nfib + 2 + (f0 ? 1 : 0);
  for (int i = 0; i < np; ++i) x[i] = 0;
  cart2sph(dt->v1, &th, &ph);
  x[0] = dt->s0;
  x[1] = sqrt(dt->l1 > 0 ? dt->l1 : 0.002);
  x[3] = th;
  x[4] = ph;
  const double* vs[3] = {dt->v1, dt->v2, dt->v3};
  for (int ii = 2, i = 5; ii <= nfib; ii++, i += 3) {
    cart2sph(vs[ii - 1], &th, &ph);
    x[i + 1] = th;
    x[i + 2] = ph;
  }
  /* fit_pvf: linear least squares for the fractions */
  double s0 = x[0], d = x[1] * x[1];
  double dir[MAXK][3];
  for (int k = 0; k < nfib; ++k) sph2vec(x[3 + 3 * k], x[4 + 3 * k], dir[k]);
  double* M = (double*)malloc(sizeof(double) * ndir * MAXK);
  double* P = (double*)malloc(sizeof(double) * ndir * MAXK);
  double* YI = (double*)malloc(sizeof(double) * ndir);
  for (int i = 0; i < ndir; ++i) {
    double gx = bvecs[i], gy = bvecs[ndir + i], gz = bvecs[2 * ndir + i], b = bvals[i];
    double iso = exp(-b * d);
    YI[i] = Y[i] - s0 * iso;
    for (int k = 0; k < nfib; ++k) {
      double dp = gx * dir[k][0] + gy * dir[k][1] + gz * dir[k][2];
      M[i * nfib + k] = s0 * (exp(-b * d * dp * dp) - iso);
    }
  }
  pinv_tall(ndir, nfib, M, P);
  double fs[MAXK], f0v = 0;
  for (int k = 0; k < nfib; ++k) {
    double s = 0;
    for (int i = 0; i < ndir; ++i) s += P[k * ndir + i] * YI[i];
    fs[k] = s;
  }
  if (f0) {
    f0v = FSMALL;
    fs[0] -= f0v;
  }
  for (int k = 0; k < nfib; ++k) fs[k] = fabs(fs[k]);
  double sumf = 0;
  for (int i = 0; i < nfib; ++i) {
    sumf += fs[i];
    if (sumf >= 1) {
      for (int j = i; j < nfib; ++j) fs[j] = FSMALL;
      break;
    }
  }
  for (int k = 0; k < nfib; ++k) {
    double pf = 1.0;
    for (int j = 0; j < k; ++j) pf -= fs[j];
    double tmpr = fs[k] / pf;
    if (tmpr > 1.0) tmpr = 1;
    x[2 + 3 * k] = f2beta(tmpr);
  }
  if (f0) {
    double pf = 1.0;
    for (int j = 0; j < nfib; ++j) pf -= fs[j];
    double tmpr = f0v / pf;
    if (tmpr > 1.0) tmpr = 1;
    x[np - 1] = f2beta(tmpr);
  }
  free(M);
  free(P);
  free(YI);
}

typedef struct {
  int ndir;
  double *A, *iA;
} dtiwork;

static void dti_for(const dtiwork* w, const float* y, const float* bvecs, const float* bvals,
                    int own_amat, dti_t* out) {
  if (own_amat) {
    double* A = (double*)malloc(sizeof(double) * w->ndir * 7);
    double* iA = (double*)malloc(sizeof(double) * w->ndir * 7);
    form_amat(w->ndir, bvecs, bvals, A);
    pinv_tall(w->ndir, 7, A, iA);
    dti_fit(w->ndir, y, bvecs, bvals, iA, A, out);
    free(A);
    free(iA);
  } else {
    dti_fit(w->ndir, y, bvecs, bvals, w->iA, w->A, out);
  }
}

int orc_lm_start(int kind, int nfib, int f0, int ndir, const float* y, const float* bvecs,
                 const float* bvals, double* p) {
  dtiwork w = {ndir, NULL, NULL};
  dti_t dt;
  dti_for(&w, y, bvecs, bvals, 1, &dt);
  if (kind == KIND_SINGLE)
    start_single(nfib, f0, &dt, p);
  else
    start_single_c(nfib, f0, &dt, ndir, y, bvecs, bvals, p);
  return 0;
}

/* orc_lm_start for every voxel of a volume [nvox][ndir] (OpenMP over voxels): p [nvox][np] */
int orc_lm_starts(int kind, int nfib, int f0, int nvox, int ndir, const float* data, const float* bvecs,
                  const float* bvals, double* p, int nthreads) {
  const int np = 3 * nfib + 2 + (f0 ? 1 : 0);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
  for (int v = 0; v < nvox; ++v)
    orc_lm_start(kind, nfib, f0, ndir, data + (size_t)v * ndir, bvecs, bvals, p + (size_t)v * np);
  return 0;
}

/* fit one model from start values; returns finalised params */
static int fit_model(int kind, int nfib, int f0, int gbo, double R, int ndir, const float* y,
                     const float* bvecs, const float* bvals, const double* start, double* out, int* capped) {
  lmctx c;
  lm_ctx_init(&c, kind, nfib, f0, gbo, R, ndir, y, bvecs, bvals);
  double p[MAXP];
  if (kind == KIND_MULTI) {
    /* fit_PVM_multi_kernel start (CUDA/PVM_multi.cu:514-530) from finalised PVM_single */
    p[0] = start[0];
    p[1] = 1.0;
    for (int i = 0, ii = 3; i < nfib; i++, ii += 3) {
      p[ii] = f2x(start[ii - 1]);
      p[ii + 1] = start[ii];
      p[ii + 2] = start[ii + 1];
    }
    p[2] = start[1];
    if (f0) p[c.np - 1] = f2x(start[c.np - 2]);
  } else {
    memcpy(p, start, sizeof(double) * c.np);
  }
  int it = lm_run(&c, p, capped);
  lm_finalise(&c, p);
  memcpy(out, p, sizeof(double) * c.np);
  return it;
}

int orc_lm_fit(int kind, int nfib, int f0, int gamma_ball_only, double R, int ndir,
               const float* y, const float* bvecs, const float* bvals, const double* start,
               double* final_params) {
  return fit_model(kind, nfib, f0, gamma_ball_only, R, ndir, y, bvecs, bvals, start,
                   final_params, NULL);
}

/* predicted signal from finalised params [S0, d, (dstd), (f,th,ph)*K, (f0)], as the
 * get_residuals_* kernels compute it (CUDA/PVM_single.cu:476-585, PVM_multi.cu:579-697) */
static double predict_final(int model, int nfib, int use_f0, const double* q, int has_f0_slot,
                            double R, double gx, double gy, double gz, double b) {
  int o = model >= 2 ? 3 : 2;
  int np = 3 * nfib + o + (has_f0_slot ? 1 : 0);
  double S0 = q[0], sumf = 0, val = 0, iso;
  if (model == 1) {
    double d = q[1];
    iso = exp(-b * d);
    for (int k = 0; k < nfib; ++k) {
      double v[3];
      sph2vec(q[o + 3 * k + 1], q[o + 3 * k + 2], v);
      double dp = gx * v[0] + gy * v[1] + gz * v[2];
      val += q[o + 3 * k] * exp(-b * d * dp * dp);
      sumf += q[o + 3 * k];
    }
  } else {
    double d = q[1], ds = q[2];
    double a = d * d / ds / ds, bb = ds * ds / d;
    double invR = 1.0 / (2.0 * R + 1);
    iso = exp(-a * log(1 + b * bb));
    for (int k = 0; k < nfib; ++k) {
      double v[3];
      sph2vec(q[o + 3 * k + 1], q[o + 3 * k + 2], v);
      double dp = gx * v[0] + gy * v[1] + gz * v[2], an;
      if (model == 3)
        an = exp(-b * 3 * a * bb * invR * ((1 - R) * dp * dp + R));
      else
        an = exp(-a * log(1 + b * bb * dp * dp));
      val += q[o + 3 * k] * an;
      sumf += q[o + 3 * k];
    }
    S0 = fabs(S0);
  }
  if (use_f0) {
    double f0 = q[np - 1];
    return S0 * (f0 + (1 - sumf - f0) * iso + val);
  }
  return S0 * ((1 - sumf) * iso + val);
}

void orc_prepare_data(int nvox, int ndir, float* data) {
  for (int v = 0; v < nvox; ++v) {
    float* y = data + (size_t)v * ndir;
    float mn = y[0], mx = y[0];
    for (int i = 1; i < ndir; ++i) {
      if (y[i] < mn) mn = y[i];
      if (y[i] > mx) mx = y[i];
    }
    if (mn <= 0 && mx > 0) {
      float minpos = mx;
      for (int i = 0; i < ndir; ++i)
        if (y[i] > 0 && y[i] < minpos) minpos = y[i];
      for (int i = 0; i < ndir; ++i)
        if (y[i] <= 0) y[i] = minpos;
    }
  }
}

/* one voxel of fit() (CUDA/xfibres_gpu.cu:173-348) and calculate_tau */
static void fit_voxel(const bpx_options* o, int ndir, const float* y, const float* bvecs,
                      const float* bvals, const dtiwork* w, int own_amat, double* params,
                      double* tau, uint32_t* status) {
  int K = o->nfibres, f0 = o->f0 ? 1 : 0, model = o->model;
  int np = bpx_nparams_fit_c(o);
  double R = o->R_prior_mean;
  int gbo = (model == 3) ? 2 : 0;
  dti_t dt;
  dti_for(w, y, bvecs, bvals, own_amat, &dt);
  double st[MAXP], out[MAXP];
  int refit = 0, capped = 0; /* capped: the LM run that produced the final parameters hit its cap */
  if (model == 1) {
    int kind = o->nonlin ? KIND_SINGLE : KIND_SINGLE_C;
    if (kind == KIND_SINGLE)
      start_single(K, f0, &dt, st);
    else
      start_single_c(K, f0, &dt, ndir, y, bvecs, bvals, st);
    fit_model(kind, K, f0, 0, R, ndir, y, bvecs, bvals, st, out, &capped);
    if (f0) {
      double md = out[1], mf = out[2], f0v = out[np - 1];
      if ((K > 0 && mf < 0.05) || md > 0.007 || f0v > 0.4) {
        double st2[MAXP], out2[MAXP];
        if (kind == KIND_SINGLE)
          start_single(K, 0, &dt, st2);
        else
          start_single_c(K, 0, &dt, ndir, y, bvecs, bvals, st2);
        fit_model(kind, K, 0, 0, R, ndir, y, bvecs, bvals, st2, out2, &capped);
        memcpy(out, out2, sizeof(double) * (np - 1));
        out[np - 1] = 0.001; /* mix_params, CUDA/xfibres_gpu.cu:571 */
        refit = 1;
      }
    }
  } else {
    double s1[MAXP];
    start_single(K, f0, &dt, st);
    fit_model(KIND_SINGLE, K, f0, 0, R, ndir, y, bvecs, bvals, st, s1, NULL);
    fit_model(KIND_MULTI, K, f0, gbo, R, ndir, y, bvecs, bvals, s1, out, &capped);
    if (f0) {
      double md = out[1], mf = out[3], f0v = out[np - 1];
      if ((K > 0 && mf < 0.05) || md > 0.007 || f0v > 0.4) {
        /* GPU re-fit path: PVM_single_c then PVM_multi (CUDA/xfibres_gpu.cu:331-333);
         * the CPU path re-fits PVM_multi from PVM_single (xfibres.cc:681-693) instead */
        double st2[MAXP], c1[MAXP], out2[MAXP];
        start_single_c(K, 0, &dt, ndir, y, bvecs, bvals, st2);
        fit_model(KIND_SINGLE_C, K, 0, 0, R, ndir, y, bvecs, bvals, st2, c1, NULL);
        fit_model(KIND_MULTI, K, 0, gbo, R, ndir, y, bvecs, bvals, c1, out2, &capped);
        memcpy(out, out2, sizeof(double) * (np - 1));
        out[np - 1] = 0.001;
        refit = 1;
      }
    }
  }
  memcpy(params, out, sizeof(double) * np);
  if (status && refit) *status |= BPX_VOX_F0_REFIT;
  if (status && capped) *status |= BPX_VOX_LM_ITERATION_CAP;
  if (o->rician && tau) {
    /* tau = 1/var(y - prediction), sample variance with n-1 (CUDA/diffmodels.cu:334-341) */
    int use_f0 = f0 && !refit;
    double mean = 0, ss = 0;
    double* r = (double*)malloc(sizeof(double) * ndir);
    for (int i = 0; i < ndir; ++i) {
      r[i] = y[i] - predict_final(model, K, use_f0, out, f0, R, bvecs[i], bvecs[ndir + i],
                                  bvecs[2 * ndir + i], bvals[i]);
      mean += r[i];
    }
    mean /= ndir;
    for (int i = 0; i < ndir; ++i) ss += (r[i] - mean) * (r[i] - mean);
    *tau = 1.0 / (ss / (ndir - 1));
    free(r);
  }
}

int bpx_nparams_fit_c(const bpx_options* o) {
  return 2 + 3 * o->nfibres + (o->model >= 2 ? 1 : 0) + (o->f0 ? 1 : 0);
}

static int check_opts(const bpx_options* o, int ndir) {
  if (o->model < 1 || o->model > 3) return -1;
  if (o->nfibres < 1 || o->nfibres > MAXK) return -1;
  if (ndir < 7 || ndir > 1024) return -1;
  return 0;
}

int orc_fit(const bpx_options* o, int nvox, int ndir, const float* data, const float* bvecs,
            const float* bvals, double* params, double* tau, uint32_t* status, int nthreads) {
  if (check_opts(o, ndir)) return -1;
  int np = bpx_nparams_fit_c(o);
  dtiwork w = {ndir, NULL, NULL};
  int per_vox = o->gradnonlin ? 1 : 0;
  if (!per_vox) {
    w.A = (double*)malloc(sizeof(double) * ndir * 7);
    w.iA = (double*)malloc(sizeof(double) * ndir * 7);
    form_amat(ndir, bvecs, bvals, w.A);
    pinv_tall(ndir, 7, w.A, w.iA);
  }
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int v = 0; v < nvox; ++v) {
    const float* bv = per_vox ? bvecs + (size_t)v * 3 * ndir : bvecs;
    const float* bl = per_vox ? bvals + (size_t)v * ndir : bvals;
    uint32_t st = 0;
    double t = 0;
    fit_voxel(o, ndir, data + (size_t)v * ndir, bv, bl, &w, per_vox, params + (size_t)v * np,
              &t, &st);
    if (tau) tau[v] = o->rician ? t : 0;
    if (status) status[v] = st;
  }
  free(w.A);
  free(w.iA);
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* MCMC (CUDA/runmcmc_kernels.cu:193-1474; CPU twin fibre.h:1191-1363, xfibres.cc:754-789)    */
/* ------------------------------------------------------------------------------------------ */
#define NSLOT (6 + 3 * MAXK)

typedef struct {
  const bpx_options* o;
  int ndir, K, model, rician, f0;
  const float *y, *gx, *gy, *gz, *b;
  double logy_sum;
} mcctx;

typedef struct {
  double S0, d, dstd, R, tau, f0, th[MAXK], ph[MAXK], f[MAXK];
  double S0_prior, d_prior, dstd_prior, R_prior, tau_prior, f0_prior;
  double th_prior[MAXK], ph_prior[MAXK], f_prior[MAXK], fib_prior[MAXK];
  double prior_en, lik_en, energy;
  double prop[NSLOT];
  int acc[NSLOT], rej[NSLOT];
  int lam_jump[MAXK];
  double *sig, *iso; /* sig [K][ndir], iso [ndir] */
  double *sig_new, *iso_new;
} chain_t;

/* compute_signal / compute_iso_signal (CUDA/runmcmc_kernels.cu:67-95) */
static double mc_signal(int model, double d, double dstd, double R, double b, double ang) {
  if (model == 1 || (dstd < 1e-5 && model == 2)) return exp(-d * b * ang);
  if (model == 2) {
    double sig2 = dstd * dstd, alpha = d * d / sig2;
    return exp(log(d / (d + b * ang * sig2)) * alpha);
  }
  double invR = 1.0 / (2.0 * R + 1.0);
  return exp(-b * 3 * d * invR * ((1 - R) * ang + R));
}
static double mc_iso(int model, double d, double dstd, double b) {
  if (model == 1 || dstd < 1e-5) return exp(-d * b);
  double sig2 = dstd * dstd, alpha = d * d / sig2;
  return exp(log(d / (d + b * sig2)) * alpha);
}

static double mc_ang(const mcctx* c, int m, double th, double ph) {
  double v[3];
  sph2vec(th, ph, v);
  double dp = c->gx[m] * v[0] + c->gy[m] * v[1] + c->gz[m] * v[2];
  return dp * dp;
}

/* compute_likelihood (CUDA/runmcmc_kernels.cu:147-191) with given signal arrays */
static double mc_lik(const mcctx* c, const chain_t* s, const double* sig, const double* iso) {
  double fsum = s->f0;
  for (int k = 0; k < c->K; ++k) fsum += s->f[k];
  double acc = 0;
  for (int m = 0; m < c->ndir; ++m) {
    double pred = 0;
    for (int k = 0; k < c->K; ++k) pred += s->f[k] * sig[k * c->ndir + m];
    pred = s->S0 * (pred + (1 - fsum) * iso[m] + s->f0);
    double y = c->y[m];
    if (!c->rician) {
      double diff = y - pred;
      acc += diff * diff;
    } else {
      acc += log(y) + (-0.5 * s->tau * (y * y + pred * pred) + orc_logI0(s->tau * pred * y));
    }
  }
  if (!c->rician) return (c->ndir / 2.0) * log(acc / 2.0);
  return -c->ndir * log(s->tau) - acc;
}

static double mc_prior_sum(const mcctx* c, const chain_t* s) {
  double p = s->d_prior + s->S0_prior + s->dstd_prior + s->R_prior + s->tau_prior + s->f0_prior;
  for (int k = 0; k < c->K; ++k) p += s->fib_prior[k];
  return p;
}

static double th_prior_of(double th) {
  if (th == 0) return 0;
  return -log(fabs(sin(th) / 2));
}

/* R prior (CUDA/runmcmc_kernels.cu:1058-1083).  Returns 1 if rejected. */
static int r_prior(const bpx_options* o, double R, double d, double* prior) {
  double upper_R = 2.0 * o->R_prior_mean, lower_R = o->R_prior_mean - 2.0 * o->R_prior_std;
  if (o->R_prior_mean > 0.5) upper_R = 1.0;
  if (lower_R < 0.0) lower_R = 1e-8;
  if (o->R_prior_fudge > 0.0 && d > UPPERDIFF / 2.0) {
    if (R < 1e-8 || R > upper_R) return 1;
    *prior = o->R_prior_fudge * log(R);
    return 0;
  }
  if (R <= lower_R || R > upper_R) return 1;
  double Rstd2 = (double)o->R_prior_std * o->R_prior_std;
  *prior = (R - o->R_prior_mean) * (R - o->R_prior_mean) / Rstd2;
  return 0;
}

/* init_Fibres_Multifibres_kernel (CUDA/runmcmc_kernels.cu:193-505) */
static void mc_init(const mcctx* c, chain_t* s, const double* prm, double tau) {
  const bpx_options* o = c->o;
  int K = c->K, model = c->model, np = bpx_nparams_fit_c(o);
  memset(s->acc, 0, sizeof(s->acc));
  memset(s->rej, 0, sizeof(s->rej));
  s->S0 = prm[0];
  s->d = prm[1];
  if (s->d < 0 || s->d > UPPERDIFF) s->d = 2e-3;
  s->R = 0;
  s->dstd = 0;
  if (model >= 2) {
    s->dstd = prm[2];
    double upper = model == 3 ? 0.004 : 0.01;
    if (s->dstd < 0 || s->dstd > upper) s->dstd = s->d / 10;
    s->R = model == 3 ? o->R_prior_mean : 0;
  }
  s->f0 = o->f0 ? prm[np - 1] : 0;
  s->tau = tau;
  int add = model >= 2 ? 1 : 0;
  for (int k = 0; k < K; ++k) {
    s->th[k] = prm[2 + 3 * k + 1 + add];
    s->ph[k] = prm[2 + 3 * k + 2 + add];
    s->f[k] = prm[2 + 3 * k + add];
    s->lam_jump[k] = (k == 0) ? (o->all_ard != 0) : (o->no_ard == 0);
    s->th_prior[k] = th_prior_of(s->th[k]);
    s->ph_prior[k] = 0;
    double fp = 0;
    if (!(s->f[k] <= 0 || s->f[k] >= 1)) {
      fp = s->lam_jump[k] ? log(s->f[k]) : 0;
      fp = o->fudge * fp;
    }
    s->f_prior[k] = fp;
    s->fib_prior[k] = s->th_prior[k] + s->ph_prior[k] + s->f_prior[k];
    s->prop[ORC_SLOT_TH(k)] = 0.2;
    s->prop[ORC_SLOT_PH(k)] = 0.2;
    s->prop[ORC_SLOT_F(k)] = 0.2;
  }
  for (int k = 0; k < K; ++k)
    for (int m = 0; m < c->ndir; ++m)
      s->sig[k * c->ndir + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
  for (int m = 0; m < c->ndir; ++m) s->iso[m] = mc_iso(model, s->d, s->dstd, c->b[m]);
  s->d_prior = 0;
  s->S0_prior = 0;
  s->dstd_prior = 0;
  s->R_prior = 0;
  s->tau_prior = 0;
  s->f0_prior = 0;
  if (s->d >= 0 && s->d <= UPPERDIFF && model == 3) s->d_prior = (1.0 - 3.0) * log(s->d) + 4000.0 * s->d;
  if (model >= 2) {
    double upper = model == 3 ? 0.004 : 0.01;
    if (s->dstd > 0 && s->dstd <= upper) s->dstd_prior = log(s->dstd);
    if (model == 3) {
      double pr = 0;
      if (!r_prior(o, s->R, s->d, &pr)) s->R_prior = pr;
    }
  }
  if (o->f0 && !(s->f0 <= 0 || s->f0 >= 1) && o->ardf0) s->f0_prior = log(s->f0);
  s->prior_en = mc_prior_sum(c, s);
  s->lik_en = mc_lik(c, s, s->sig, s->iso);
  s->energy = s->prior_en + s->lik_en;
  s->prop[ORC_SLOT_S0] = s->S0 / 10.0;
  s->prop[ORC_SLOT_D] = s->d / 10.0;
  s->prop[ORC_SLOT_DSTD] = s->dstd / 10.0;
  s->prop[ORC_SLOT_TAU] = s->tau / 2.0;
  s->prop[ORC_SLOT_F0] = 0.2;
  s->prop[ORC_SLOT_R] = s->R / 10.0;
}

/* test_energy + accept/reject bookkeeping.  Returns 1 if accepted. */
static int mc_decide(chain_t* s, int prior_reject, double new_prior, double new_lik,
                     double log_u) {
  if (prior_reject) return 0;
  double e_new = new_prior + new_lik;
  double de = s->energy - e_new;
  if (de > log_u) {
    s->energy = e_new;
    s->lik_en = new_lik;
    return 1;
  }
  return 0;
}

static void mc_iteration(const mcctx* c, chain_t* s, uint64_t vox, uint32_t it) {
  const bpx_options* o = c->o;
  int K = c->K, model = c->model, M = c->ndir;
  double n, lu;
  uint64_t seed = o->seed;
  int can_use_ard = !o->no_ard;
  /* f0 */
  if (o->f0) {
    orc_rng_slot(seed, vox, it, ORC_SLOT_F0, &n, &lu);
    double old = s->f0, oldp = s->f0_prior, oldpe = s->prior_en;
    s->f0 = old + n * s->prop[ORC_SLOT_F0];
    int rej = (s->f0 <= 0 || s->f0 >= 1);
    if (!rej) s->f0_prior = o->ardf0 ? log(s->f0) : 0;
    double fsum = s->f0;
    for (int k = 0; k < K; ++k) fsum += s->f[k];
    rej = rej || (fsum > 1);
    s->prior_en = mc_prior_sum(c, s);
    double lik = rej ? 0 : mc_lik(c, s, s->sig, s->iso);
    if (mc_decide(s, rej, s->prior_en, lik, lu))
      s->acc[ORC_SLOT_F0]++;
    else {
      s->f0 = old;
      s->f0_prior = oldp;
      s->prior_en = oldpe;
      s->rej[ORC_SLOT_F0]++;
    }
  }
  /* tau */
  if (c->rician) {
    orc_rng_slot(seed, vox, it, ORC_SLOT_TAU, &n, &lu);
    double old = s->tau, oldp = s->tau_prior, oldpe = s->prior_en;
    s->tau = old + n * s->prop[ORC_SLOT_TAU];
    int rej = s->tau <= 0;
    if (!rej) s->tau_prior = 0;
    s->prior_en = mc_prior_sum(c, s);
    double lik = rej ? 0 : mc_lik(c, s, s->sig, s->iso);
    if (mc_decide(s, rej, s->prior_en, lik, lu))
      s->acc[ORC_SLOT_TAU]++;
    else {
      s->tau = old;
      s->tau_prior = oldp;
      s->prior_en = oldpe;
      s->rej[ORC_SLOT_TAU]++;
    }
  }
  /* d */
  {
    orc_rng_slot(seed, vox, it, ORC_SLOT_D, &n, &lu);
    double old = s->d, oldp = s->d_prior, oldpe = s->prior_en;
    s->d = old + n * s->prop[ORC_SLOT_D];
    int rej = (s->d < 0 || s->d > UPPERDIFF);
    if (!rej) s->d_prior = model == 3 ? (1.0 - 3.0) * log(s->d) + 4000.0 * s->d : 0;
    s->prior_en = mc_prior_sum(c, s);
    double lik = 0;
    if (!rej) {
      for (int k = 0; k < K; ++k)
        for (int m = 0; m < M; ++m)
          s->sig_new[k * M + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
      for (int m = 0; m < M; ++m) s->iso_new[m] = mc_iso(model, s->d, s->dstd, c->b[m]);
      lik = mc_lik(c, s, s->sig_new, s->iso_new);
    }
    if (mc_decide(s, rej, s->prior_en, lik, lu)) {
      s->acc[ORC_SLOT_D]++;
      memcpy(s->sig, s->sig_new, sizeof(double) * K * M);
      memcpy(s->iso, s->iso_new, sizeof(double) * M);
    } else {
      s->d = old;
      s->d_prior = oldp;
      s->prior_en = oldpe;
      s->rej[ORC_SLOT_D]++;
    }
  }
  /* d_std */
  if (model >= 2) {
    orc_rng_slot(seed, vox, it, ORC_SLOT_DSTD, &n, &lu);
    double old = s->dstd, oldp = s->dstd_prior, oldpe = s->prior_en;
    s->dstd = old + n * s->prop[ORC_SLOT_DSTD];
    double upper = model == 3 ? 0.004 : 0.01;
    int rej = (s->dstd <= 0 || s->dstd > upper);
    if (!rej) s->dstd_prior = log(s->dstd);
    s->prior_en = mc_prior_sum(c, s);
    double lik = 0;
    if (!rej) {
      if (model == 2) {
        for (int k = 0; k < K; ++k)
          for (int m = 0; m < M; ++m)
            s->sig_new[k * M + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
      } else {
        memcpy(s->sig_new, s->sig, sizeof(double) * K * M);
      }
      for (int m = 0; m < M; ++m) s->iso_new[m] = mc_iso(model, s->d, s->dstd, c->b[m]);
      lik = mc_lik(c, s, s->sig_new, s->iso_new);
    }
    if (mc_decide(s, rej, s->prior_en, lik, lu)) {
      s->acc[ORC_SLOT_DSTD]++;
      memcpy(s->sig, s->sig_new, sizeof(double) * K * M);
      memcpy(s->iso, s->iso_new, sizeof(double) * M);
    } else {
      s->dstd = old;
      s->dstd_prior = oldp;
      s->prior_en = oldpe;
      s->rej[ORC_SLOT_DSTD]++;
    }
    /* R */
    if (model == 3) {
      orc_rng_slot(seed, vox, it, ORC_SLOT_R, &n, &lu);
      double oldR = s->R, oldRp = s->R_prior, oldpe2 = s->prior_en;
      s->R = oldR + n * s->prop[ORC_SLOT_R];
      double pr = s->R_prior;
      int rejR = r_prior(o, s->R, s->d, &pr);
      if (!rejR) s->R_prior = pr;
      s->prior_en = mc_prior_sum(c, s);
      double likR = 0;
      if (!rejR) {
        for (int k = 0; k < K; ++k)
          for (int m = 0; m < M; ++m)
            s->sig_new[k * M + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
        likR = mc_lik(c, s, s->sig_new, s->iso);
      }
      if (mc_decide(s, rejR, s->prior_en, likR, lu)) {
        s->acc[ORC_SLOT_R]++;
        memcpy(s->sig, s->sig_new, sizeof(double) * K * M);
      } else {
        s->R = oldR;
        s->R_prior = oldRp;
        s->prior_en = oldpe2;
        s->rej[ORC_SLOT_R]++;
      }
    }
  }
  /* S0 */
  {
    orc_rng_slot(seed, vox, it, ORC_SLOT_S0, &n, &lu);
    double old = s->S0, oldp = s->S0_prior, oldpe = s->prior_en;
    s->S0 = old + n * s->prop[ORC_SLOT_S0];
    int rej = s->S0 < 0;
    if (!rej) s->S0_prior = 0;
    s->prior_en = mc_prior_sum(c, s);
    double lik = rej ? 0 : mc_lik(c, s, s->sig, s->iso);
    if (mc_decide(s, rej, s->prior_en, lik, lu))
      s->acc[ORC_SLOT_S0]++;
    else {
      s->S0 = old;
      s->S0_prior = oldp;
      s->prior_en = oldpe;
      s->rej[ORC_SLOT_S0]++;
    }
  }
  /* fibres */
  for (int k = 0; k < K; ++k) {
    /* th */
    {
      orc_rng_slot(seed, vox, it, ORC_SLOT_TH(k), &n, &lu);
      double old = s->th[k], oldp = s->th_prior[k], oldfp = s->fib_prior[k], oldpe = s->prior_en;
      s->th[k] = old + n * s->prop[ORC_SLOT_TH(k)];
      s->th_prior[k] = th_prior_of(s->th[k]);
      s->fib_prior[k] = s->th_prior[k] + s->ph_prior[k] + s->f_prior[k];
      s->prior_en = mc_prior_sum(c, s);
      memcpy(s->sig_new, s->sig, sizeof(double) * K * M);
      for (int m = 0; m < M; ++m)
        s->sig_new[k * M + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
      double lik = mc_lik(c, s, s->sig_new, s->iso);
      if (mc_decide(s, 0, s->prior_en, lik, lu)) {
        s->acc[ORC_SLOT_TH(k)]++;
        memcpy(s->sig + k * M, s->sig_new + k * M, sizeof(double) * M);
      } else {
        s->th[k] = old;
        s->th_prior[k] = oldp;
        s->fib_prior[k] = oldfp;
        s->prior_en = oldpe;
        s->rej[ORC_SLOT_TH(k)]++;
      }
    }
    /* ph */
    {
      orc_rng_slot(seed, vox, it, ORC_SLOT_PH(k), &n, &lu);
      double old = s->ph[k], oldp = s->ph_prior[k], oldfp = s->fib_prior[k], oldpe = s->prior_en;
      s->ph[k] = old + n * s->prop[ORC_SLOT_PH(k)];
      s->ph_prior[k] = 0;
      s->fib_prior[k] = s->th_prior[k] + s->ph_prior[k] + s->f_prior[k];
      s->prior_en = mc_prior_sum(c, s);
      memcpy(s->sig_new, s->sig, sizeof(double) * K * M);
      for (int m = 0; m < M; ++m)
        s->sig_new[k * M + m] = mc_signal(model, s->d, s->dstd, s->R, c->b[m], mc_ang(c, m, s->th[k], s->ph[k]));
      double lik = mc_lik(c, s, s->sig_new, s->iso);
      if (mc_decide(s, 0, s->prior_en, lik, lu)) {
        s->acc[ORC_SLOT_PH(k)]++;
        memcpy(s->sig + k * M, s->sig_new + k * M, sizeof(double) * M);
      } else {
        s->ph[k] = old;
        s->ph_prior[k] = oldp;
        s->fib_prior[k] = oldfp;
        s->prior_en = oldpe;
        s->rej[ORC_SLOT_PH(k)]++;
      }
    }
    /* f */
    {
      orc_rng_slot(seed, vox, it, ORC_SLOT_F(k), &n, &lu);
      double old = s->f[k], oldp = s->f_prior[k], oldfp = s->fib_prior[k], oldpe = s->prior_en;
      s->f[k] = old + n * s->prop[ORC_SLOT_F(k)];
      int rej = (s->f[k] <= 0 || s->f[k] >= 1);
      if (!rej) {
        double fp;
        if (!can_use_ard)
          fp = 0;
        else
          fp = s->lam_jump[k] ? log(s->f[k]) : 0;
        s->f_prior[k] = o->fudge * fp;
      }
      s->fib_prior[k] = s->th_prior[k] + s->ph_prior[k] + s->f_prior[k];
      double fsum = s->f0;
      for (int j = 0; j < K; ++j) fsum += s->f[j];
      rej = rej || (fsum > 1);
      s->prior_en = mc_prior_sum(c, s);
      double lik = rej ? 0 : mc_lik(c, s, s->sig, s->iso);
      if (mc_decide(s, rej, s->prior_en, lik, lu))
        s->acc[ORC_SLOT_F(k)]++;
      else {
        s->f[k] = old;
        s->f_prior[k] = oldp;
        s->fib_prior[k] = oldfp;
        s->prior_en = oldpe;
        s->rej[ORC_SLOT_F(k)]++;
      }
    }
  }
}

/* update_proposals (CUDA/runmcmc_kernels.cu:1341-1395): sigma *= sqrt((acc+1)/(rej+1)) */
static void mc_update_props(const mcctx* c, chain_t* s) {
  int slots[NSLOT], n = 0;
  slots[n++] = ORC_SLOT_D;
  if (c->rician) slots[n++] = ORC_SLOT_TAU;
  if (c->f0) slots[n++] = ORC_SLOT_F0;
  if (c->model >= 2) slots[n++] = ORC_SLOT_DSTD;
  if (c->model == 3) slots[n++] = ORC_SLOT_R;
  slots[n++] = ORC_SLOT_S0;
  for (int k = 0; k < c->K; ++k) {
    slots[n++] = ORC_SLOT_TH(k);
    slots[n++] = ORC_SLOT_PH(k);
    slots[n++] = ORC_SLOT_F(k);
  }
  for (int i = 0; i < n; ++i) {
    int sl = slots[i];
    s->prop[sl] *= sqrt((double)(s->acc[sl] + 1) / (double)(s->rej[sl] + 1));
    if (s->prop[sl] > MAXFLOAT_PROP) s->prop[sl] = MAXFLOAT_PROP;
    s->acc[sl] = 0;
    s->rej[sl] = 0;
  }
}

static void mc_ctx_init(mcctx* c, const bpx_options* o, int ndir, const float* y,
                        const float* bvecs, const float* bvals) {
  c->o = o;
  c->ndir = ndir;
  c->K = o->nfibres;
  c->model = o->model;
  c->rician = o->rician ? 1 : 0;
  c->f0 = o->f0 ? 1 : 0;
  c->y = y;
  c->gx = bvecs;
  c->gy = bvecs + ndir;
  c->gz = bvecs + 2 * ndir;
  c->b = bvals;
}

int orc_mcmc(const bpx_options* o, int nvox, int ndir, const float* data, const float* bvecs,
             const float* bvals, const double* params, const double* tau, uint64_t voxel_offset,
             double* records, int nthreads) {
  if (check_opts(o, ndir)) return -1;
  int K = o->nfibres, np = bpx_nparams_fit_c(o);
  int ns = o->njumps / o->sampleevery;
  int nrec = 6 + 3 * K;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int v = 0; v < nvox; ++v) {
    const float* bv = o->gradnonlin ? bvecs + (size_t)v * 3 * ndir : bvecs;
    const float* bl = o->gradnonlin ? bvals + (size_t)v * ndir : bvals;
    mcctx c;
    mc_ctx_init(&c, o, ndir, data + (size_t)v * ndir, bv, bl);
    chain_t s;
    double* buf = (double*)malloc(sizeof(double) * 2 * (K + 1) * ndir);
    s.sig = buf;
    s.iso = buf + K * ndir;
    s.sig_new = buf + (K + 1) * ndir;
    s.iso_new = s.sig_new + K * ndir;
    mc_init(&c, &s, params + (size_t)v * np, tau ? tau[v] : 0.0);
    uint64_t gv = voxel_offset + (uint64_t)v;
    int total = o->nburn + o->njumps, sample = 0;
    for (int it = 0; it < total; ++it) {
      mc_iteration(&c, &s, gv, (uint32_t)it);
      if (it >= o->nburn && ((it - o->nburn + 1) % o->sampleevery) == 0 && sample < ns) {
        double vals[6 + 3 * MAXK];
        vals[0] = s.d;
        vals[1] = s.f0;
        vals[2] = s.tau;
        vals[3] = s.dstd;
        vals[4] = s.R;
        vals[5] = s.S0;
        for (int k = 0; k < K; ++k) {
          vals[6 + 3 * k] = s.th[k];
          vals[7 + 3 * k] = s.ph[k];
          vals[8 + 3 * k] = s.f[k];
        }
        for (int r = 0; r < nrec; ++r) records[((size_t)r * ns + sample) * nvox + v] = vals[r];
        ++sample;
      }
      if (((it + 1) % o->updateproposalevery) == 0) mc_update_props(&c, &s);
    }
    free(buf);
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* sample finishing (CUDA/samples.cu:134-347)                                                  */
/* ------------------------------------------------------------------------------------------ */
int orc_finish(const bpx_options* o, int nvox, const double* rec, double* th, double* ph,
               double* f, double* mean_d, double* mean_dstd, double* mean_R, double* mean_f0,
               double* mean_tau, double* mean_S0, double* mean_f, double* dyads) {
  int K = o->nfibres, ns = o->njumps / o->sampleevery;
#define REC(r, s, v) rec[((size_t)(r) * ns + (s)) * nvox + (v)]
  for (int v = 0; v < nvox; ++v) {
    double sums[6] = {0, 0, 0, 0, 0, 0}, sumf[MAXK] = {0, 0, 0}, dy[MAXK][9];
    memset(dy, 0, sizeof(dy));
    for (int s = 0; s < ns; ++s) {
      for (int r = 0; r < 6; ++r) sums[r] += REC(r, s, v);
      for (int k = 0; k < K; ++k) {
        double vv[3];
        sph2vec(REC(6 + 3 * k, s, v), REC(7 + 3 * k, s, v), vv);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) dy[k][a * 3 + b] += vv[a] * vv[b];
        sumf[k] += REC(8 + 3 * k, s, v);
      }
    }
    if (mean_d) mean_d[v] = sums[0] / ns;
    if (mean_f0) mean_f0[v] = sums[1] / ns;
    if (mean_tau) mean_tau[v] = sums[2] / ns;
    if (mean_dstd) mean_dstd[v] = sums[3] / ns;
    if (mean_R) mean_R[v] = sums[4] / ns;
    if (mean_S0) mean_S0[v] = sums[5] / ns;
    /* sort (sum f, index) ascending, output in reverse (CUDA/samples.cu:299-330) */
    int idx[MAXK];
    for (int k = 0; k < K; ++k) idx[k] = k;
    for (int i = 0; i < K; ++i)
      for (int j = i + 1; j < K; ++j) {
        int a = idx[i], b = idx[j];
        if (sumf[b] < sumf[a] || (sumf[b] == sumf[a] && b < a)) {
          idx[i] = b;
          idx[j] = a;
        }
      }
    for (int out = 0; out < K; ++out) {
      int src = idx[K - 1 - out];
      for (int s = 0; s < ns; ++s) {
        size_t o2 = ((size_t)out * ns + s) * nvox + v;
        if (th) th[o2] = REC(6 + 3 * src, s, v);
        if (ph) ph[o2] = REC(7 + 3 * src, s, v);
        if (f) f[o2] = REC(8 + 3 * src, s, v);
      }
      if (mean_f) mean_f[(size_t)out * nvox + v] = sumf[src] / ns;
      if (dyads) {
        double w[3], V[9];
        jacobi_eig(3, dy[src], w, V);
        for (int a = 0; a < 3; ++a) dyads[((size_t)out * 3 + a) * nvox + v] = V[a * 3 + 0];
      }
    }
  }
#undef REC
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* energies of given states                                                                    */
/* ------------------------------------------------------------------------------------------ */
int orc_energy(const bpx_options* o, int nvox, int ndir, const float* data, const float* bvecs,
               const float* bvals, const double* states, double* lik, double* prior) {
  if (check_opts(o, ndir)) return -1;
  int K = o->nfibres;
  for (int v = 0; v < nvox; ++v) {
    const double* st = states + (size_t)v * BPX_NSTATE;
    const float* bv = o->gradnonlin ? bvecs + (size_t)v * 3 * ndir : bvecs;
    const float* bl = o->gradnonlin ? bvals + (size_t)v * ndir : bvals;
    mcctx c;
    mc_ctx_init(&c, o, ndir, data + (size_t)v * ndir, bv, bl);
    chain_t s;
    memset(&s, 0, sizeof(s));
    double* buf = (double*)malloc(sizeof(double) * (K + 1) * ndir);
    s.sig = buf;
    s.iso = buf + K * ndir;
    s.S0 = st[0];
    s.d = st[1];
    s.dstd = st[2];
    s.R = st[3];
    s.tau = st[4];
    s.f0 = o->f0 ? st[5] : 0;
    for (int k = 0; k < K; ++k) {
      s.th[k] = st[6 + 3 * k];
      s.ph[k] = st[7 + 3 * k];
      s.f[k] = st[8 + 3 * k];
    }
    for (int k = 0; k < K; ++k)
      for (int m = 0; m < ndir; ++m)
        s.sig[k * ndir + m] = mc_signal(c.model, s.d, s.dstd, s.R, c.b[m], mc_ang(&c, m, s.th[k], s.ph[k]));
    for (int m = 0; m < ndir; ++m) s.iso[m] = mc_iso(c.model, s.d, s.dstd, c.b[m]);
    if (lik) lik[v] = mc_lik(&c, &s, s.sig, s.iso);
    if (prior) {
      /* the prior energy of the state, as init_Fibres_Multifibres_kernel composes it */
      double p = 0;
      if (c.model == 3 && s.d >= 0 && s.d <= UPPERDIFF) p += (1.0 - 3.0) * log(s.d) + 4000.0 * s.d;
      if (c.model >= 2) {
        double upper = c.model == 3 ? 0.004 : 0.01;
        if (s.dstd > 0 && s.dstd <= upper) p += log(s.dstd);
        if (c.model == 3) {
          double pr = 0;
          if (!r_prior(o, s.R, s.d, &pr)) p += pr;
        }
      }
      if (o->f0 && !(s.f0 <= 0 || s.f0 >= 1) && o->ardf0) p += log(s.f0);
      for (int k = 0; k < K; ++k) {
        int lj = (k == 0) ? (o->all_ard != 0) : (o->no_ard == 0);
        double fp = 0;
        if (!(s.f[k] <= 0 || s.f[k] >= 1)) fp = o->fudge * (lj ? log(s.f[k]) : 0);
        p += th_prior_of(s.th[k]) + fp;
      }
      prior[v] = p;
    }
    free(buf);
  }
  return 0;
}
