// bpx_fit.cu -- initial fits of the bedpostx path on the GPU.
//
// One warp fits one voxel.  Replaces, for every voxel at once:
//   * the host DTI start values  (CUDA/diffmodels.cu:57-94,149-184; DTI::linfit diffmodels.cc:17-46),
//   * PVM_single_c::fit_pvf      (diffmodels.cc:561-603),
//   * fit_PVM_single_kernel / fit_PVM_single_c_kernel / fit_PVM_multi_kernel
//     (CUDA/PVM_single.cu:387-473, CUDA/PVM_single_c.cu:516-616, CUDA/PVM_multi.cu:468-576)
//     with their LM driver (CUDA/levenberg_marquardt.cu:17-333),
//   * the f0 plausibility re-fit and mix_params (CUDA/xfibres_gpu.cu:207-339,552-576),
//   * calculate_tau with its residual kernels (CUDA/diffmodels.cu:259-347).
//
// Design: measurements are strided over the 32 lanes.  Scalar sums (cost, DTI moments) are
// combined with xor-butterfly shuffles so that every lane holds identical totals and takes
// identical LM decisions.  The Gauss-Newton normal equations J^T J, J^T r are contracted on the
// FP64 tensor cores (mma.sync m8n8k4 .f64) from Jacobian rows staged in a per-warp
// shared-memory tile, and kept there between LM steps; the damped system is solved in FP64
// with its rows spread over lanes.  Warps of a block take voxels from a shared counter.
//
// Precision: everything is FP64 -- parameters, model values, residuals, cost, gradient and the
// Gauss-Newton Hessian.  The reference's CPU fits are FP64, and on near-singular fits (a small
// third fibre) even rounding J^T J to FP32 sends the LM path of a tenth of the voxels elsewhere.
// The fits are a few percent of the path's arithmetic, so FP64 here costs little.
#include <cstdint>

#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {

enum Kind { kSingle = 0, kSingleC = 1, kMulti = 2 };

template <int KIND, int K, bool F0>
struct LmShape {
  static constexpr int P = 3 * K + 2 + (KIND == kMulti ? 1 : 0) + (F0 ? 1 : 0);
  static constexpr int O = (KIND == kMulti) ? 3 : 2;  // offset of the first fibre's f
  static constexpr int NH = P * (P + 1) / 2;
};

struct Meas {
  const float* y;
  const float* gx;
  const float* gy;
  const float* gz;
  const float* b;
  int M;
};

// ------------------------------------------------------------------------------------------
// Row-distributed FP64 solve of A x = r for an SPD matrix (A = J^T J + lambda I): lane i holds
// row i.  Gaussian elimination without pivoting (stable for SPD), then back substitution; every
// lane returns the whole solution.
// ------------------------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ void warp_solve(double (&row)[P], double rhs, double (&x)[P], int lane) {
  double inv_pivot = 0.0;  // lane k keeps 1 / (pivot k) for the back substitution
#pragma unroll
  for (int k = 0; k < P; ++k) {
    const double inv = 1.0 / __shfl_sync(0xffffffffu, row[k], k);
    const double rk = __shfl_sync(0xffffffffu, rhs, k);
    if (lane == k) inv_pivot = inv;
    const double m = row[k] * inv;
    const bool below = lane > k;
#pragma unroll
    for (int j = k + 1; j < P; ++j) {
      const double akj = __shfl_sync(0xffffffffu, row[j], k);
      if (below) row[j] -= m * akj;
    }
    if (below) rhs -= m * rk;
  }
#pragma unroll
  for (int i = P - 1; i >= 0; --i) {
    double s = rhs;
#pragma unroll
    for (int j = i + 1; j < P; ++j) s -= row[j] * x[j];
    x[i] = __shfl_sync(0xffffffffu, s * inv_pivot, i);
  }
}

// D += A B for one 8x8x4 FP64 tensor-core tile (mma.sync m8n8k4 .f64): lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Symmetric eigen-decomposition of a small matrix (n <= 3) by cyclic Jacobi, FP64; eigenvalues
// descending; each eigenvector signed so its largest-magnitude component is positive (the
// oracle uses the same convention, so both start the fits from the same angles).
template <int N>
__device__ void jacobi_eig(double (&A)[N][N], double (&w)[N], double (&V)[N][N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = 0;
#pragma unroll
    for (int p = 0; p < N; ++p)
#pragma unroll
      for (int q = p + 1; q < N; ++q) off += A[p][q] * A[p][q];
    if (off < 1e-300) break;
#pragma unroll
    for (int p = 0; p < N; ++p) {
#pragma unroll
      for (int q = p + 1; q < N; ++q) {
        const double apq = A[p][q];
        if (fabs(apq) < 1e-300) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
  // sort descending (selection on indices), canonical signs
  int idx[N];
#pragma unroll
  for (int i = 0; i < N; ++i) idx[i] = i;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = i + 1; j < N; ++j) {
      double ai = 0, aj = 0;
#pragma unroll
      for (int t = 0; t < N; ++t) {
        if (t == idx[i]) ai = A[t][t];
        if (t == idx[j]) aj = A[t][t];
      }
      if (aj > ai) {
        const int tmp = idx[i];
        idx[i] = idx[j];
        idx[j] = tmp;
      }
    }
  double Vs[N][N];
#pragma unroll
  for (int c = 0; c < N; ++c) {
    double col[N], wc = 0;
#pragma unroll
    for (int t = 0; t < N; ++t)
      if (t == idx[c]) {
        wc = A[t][t];
#pragma unroll
        for (int r = 0; r < N; ++r) col[r] = V[r][t];
      }
    int big = 0;
#pragma unroll
    for (int r = 1; r < N; ++r)
      if (fabs(col[r]) > fabs(col[big])) big = r;
    double sg = 1.0;
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (r == big && col[r] < 0) sg = -1.0;
    w[c] = wc;
#pragma unroll
    for (int r = 0; r < N; ++r) Vs[r][c] = sg * col[r];
  }
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) V[r][c] = Vs[r][c];
}

// spherical angles in the convention of FSL miscmaths cart2sph (called at CUDA/diffmodels.cu:70)
__device__ void cart2sph(const double (&v)[3], double& th, double& ph) {
  const double x = v[0], y = v[1], z = v[2];
  const double mag = sqrt(x * x + y * y + z * z);
  const double pi = 3.141592653589793;
  if (mag == 0) {
    th = pi / 2;
    ph = pi / 2;
    return;
  }
  double p;
  if (x == 0 && y >= 0)
    p = pi / 2;
  else if (x == 0 && y < 0)
    p = -pi / 2;
  else if (x > 0)
    p = atan(y / x);
  else if (y > 0)
    p = atan(y / x) + pi;
  else
    p = atan(y / x) - pi;
  const double r = sqrt(x * x + y * y);
  double t;
  if (z == 0)
    t = pi / 2;
  else if (z > 0)
    t = atan(r / z);
  else
    t = atan(r / z) + pi;
  th = t;
  ph = p;
}

struct Dti {
  double s0, md, fa, l1, v[3][3];  // v[i] = i-th eigenvector (descending eigenvalue)
};

// DTI::linfit (diffmodels.cc:17-46): two log-linear least-squares passes through the normal
// equations of the 7-column design matrix (form_Amat, diffmodels.h:148-163), then the
// eigen-system of the tensor (calc_tensor_parameters, diffmodels.cc:239-266).
__device__ void dti_fit(const Meas& ms, int lane, Dti& o) {
  double G[28];
  double r1[7];
#pragma unroll
  for (int i = 0; i < 28; ++i) G[i] = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i) r1[i] = 0;
  float ysum = 0.f, ymax = 0.f;
  for (int m = lane; m < ms.M; m += 32) {
    const double gx = ms.gx[m], gy = ms.gy[m], gz = ms.gz[m], b = ms.b[m];
    const double a[7] = {b * gx * gx, 2 * b * gx * gy, 2 * b * gx * gz, b * gy * gy, 2 * b * gy * gz, b * gz * gz, 1.0};
    const float y = ms.y[m];
    const double ls = y > 0 ? log((double)y) : 0.0;
    int e = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      r1[i] += a[i] * ls;
#pragma unroll
      for (int j = i; j < 7; ++j) G[e++] += a[i] * a[j];
    }
    ysum += y;
    ymax = fmaxf(ymax, fabsf(y));
  }
#pragma unroll
  for (int i = 0; i < 28; ++i) G[i] = group_sum<32>(G[i]);
#pragma unroll
  for (int i = 0; i < 7; ++i) r1[i] = group_sum<32>(r1[i]);
  ysum = group_sum<32>(ysum);
  ymax = group_max<32>(ymax);
  const double ymean = (double)ysum / ms.M;
  // distribute rows of G
  double row[7];
  {
    int e = 0;
    double full[7][7];
#pragma unroll
    for (int i = 0; i < 7; ++i)
#pragma unroll
      for (int j = i; j < 7; ++j) {
        full[i][j] = G[e];
        full[j][i] = G[e];
        ++e;
      }
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      row[j] = 0;
#pragma unroll
      for (int i = 0; i < 7; ++i)
        if (lane == i) row[j] = full[i][j];
    }
  }
  double rowc[7];
#pragma unroll
  for (int j = 0; j < 7; ++j) rowc[j] = row[j];
  double rhs = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i)
    if (lane == i) rhs = r1[i];
  double D[7];
  warp_solve<7>(rowc, rhs, D, lane);  // D = (A^T A)^-1 A^T logS ; Dvec = -D
  double s0 = (-D[6]) > -23 ? exp(D[6]) : (double)ymax;
  if (s0 < ymean) s0 = ymax;
  double r2[7];
#pragma unroll
  for (int i = 0; i < 7; ++i) r2[i] = 0;
  for (int m = lane; m < ms.M; m += 32) {
    const double gx = ms.gx[m], gy = ms.gy[m], gz = ms.gz[m], b = ms.b[m];
    const double a[7] = {b * gx * gx, 2 * b * gx * gy, 2 * b * gx * gz, b * gy * gy, 2 * b * gy * gz, b * gz * gz, 1.0};
    const double y = ms.y[m];
    const double ls = (y / s0) > 0.01 ? log(y) : log(0.01 * s0);
#pragma unroll
    for (int i = 0; i < 7; ++i) r2[i] += a[i] * ls;
  }
#pragma unroll
  for (int i = 0; i < 7; ++i) r2[i] = group_sum<32>(r2[i]);
  rhs = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i)
    if (lane == i) rhs = r2[i];
  warp_solve<7>(row, rhs, D, lane);
  // Dvec = -D
  s0 = exp(D[6]);
  if (s0 < ymean) s0 = ymean;
  double T[3][3] = {{-D[0], -D[1], -D[2]}, {-D[1], -D[3], -D[4]}, {-D[2], -D[4], -D[5]}};
  double w[3], V[3][3];
  jacobi_eig<3>(T, w, V);
  o.s0 = s0;
  o.l1 = w[0];
  o.md = (w[0] + w[1] + w[2]) / 3.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int r = 0; r < 3; ++r) o.v[i][r] = V[r][i];
  const double numer = 1.5 * ((w[0] - o.md) * (w[0] - o.md) + (w[1] - o.md) * (w[1] - o.md) + (w[2] - o.md) * (w[2] - o.md));
  const double denom = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  const double fa = denom > 0 ? numer / denom : 0;
  o.fa = fa > 0 ? sqrt(fa) : 0;
}

// ------------------------------------------------------------------------------------------
// model evaluation (FP64)
// ------------------------------------------------------------------------------------------
using Real = double;  // model-evaluation precision of the fits

template <int KIND, int K, bool F0>
struct Pre {
  Real fs[K], v[K][3], sth[K], cth[K], sph[K], cph[K], dfx[K];
  Real sumf, d, a, bb, S0, f0v, dfx0, sgn1, sgn2;
  Real deriv[K][K];
};

__device__ __forceinline__ Real x2fd(Real x) { return fabs(kTwoPiGpuD * atan(x)); }
__device__ __forceinline__ Real f2xd(Real f) { return tan(f / kTwoPiGpuD); }
__device__ __forceinline__ Real beta2fd(Real b) {
  const Real s = sin(b);
  return s * s;
}
__device__ __forceinline__ Real f2betad(Real f) { return asin(sqrt(f)); }
__device__ __forceinline__ Real sgnd(Real x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
__device__ __forceinline__ Real pm1d(Real x) { return x > 0 ? 1.0 : -1.0; }

template <int KIND, int K, bool F0>
__device__ __forceinline__ void precompute(const Real (&p)[LmShape<KIND, K, F0>::P], Pre<KIND, K, F0>& q) {
  constexpr int P = LmShape<KIND, K, F0>::P, O = LmShape<KIND, K, F0>::O;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    sincos(p[O + 3 * k + 1], &q.sth[k], &q.cth[k]);
    sincos(p[O + 3 * k + 2], &q.sph[k], &q.cph[k]);
    q.v[k][0] = q.sth[k] * q.cph[k];
    q.v[k][1] = q.sth[k] * q.sph[k];
    q.v[k][2] = q.cth[k];
  }
  q.sumf = 0.0;
  q.sgn1 = 1.0;
  q.sgn2 = 1.0;
  if (KIND == kSingle) {
    q.d = fabs(p[1]);
    q.S0 = p[0];
    q.sgn1 = pm1d(p[1]);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const Real x = p[O + 3 * k];
      q.fs[k] = x2fd(x);
      q.dfx[k] = kTwoPiGpuD * sgnd(x) / (1.0 + x * x);
      q.sumf += q.fs[k];
    }
    if (F0) {
      const Real x0 = p[P - 1];
      q.f0v = x2fd(x0);
      q.dfx0 = kTwoPiGpuD * sgnd(x0) / (1.0 + x0 * x0);
    }
  } else if (KIND == kSingleC) {
    q.d = p[1] * p[1];
    q.S0 = p[0];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      Real pf = 1.0;
#pragma unroll
      for (int j = 0; j < k; ++j) pf -= q.fs[j];
      q.fs[k] = beta2fd(p[O + 3 * k]) * pf;
      q.sumf += q.fs[k];
      q.dfx[k] = 0.0;
    }
    // fractions_deriv_PVM_single_c (CUDA/PVM_single_c.cu:104-139): d f_j / d beta_k
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const Real s2k = sin(2.0 * p[O + 3 * k]);
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (j == k) {
          Real fsum = 1.0;
#pragma unroll
          for (int n = 0; n < j; ++n) fsum -= q.fs[n];
          q.deriv[j][k] = s2k * fsum;
        } else if (j > k) {
          const Real sp = sin(p[O + 3 * j]);
          Real fsum = 0.0;
#pragma unroll
          for (int n = 0; n < j; ++n) fsum += q.deriv[n][k];
          q.deriv[j][k] = -(sp * sp) * fsum;
        } else {
          q.deriv[j][k] = 0.0;
        }
      }
    }
    if (F0) {
      const Real pfs = 1.0 - q.sumf;
      q.f0v = beta2fd(p[P - 1]) * pfs;
      q.dfx0 = sin(2.0 * p[P - 1]) * pfs;
    }
  } else {
    q.a = fabs(p[1]);
    q.bb = fabs(p[2]);
    q.S0 = fabs(p[0]);
    q.sgn1 = pm1d(p[1]);
    q.sgn2 = pm1d(p[2]);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const Real x = p[O + 3 * k];
      q.fs[k] = x2fd(x);
      q.dfx[k] = kTwoPiGpuD * sgnd(x) / (1.0 + x * x);
      q.sumf += q.fs[k];
    }
    if (F0) {
      const Real x0 = p[P - 1];
      q.f0v = x2fd(x0);
      q.dfx0 = kTwoPiGpuD * sgnd(x0) / (1.0 + x0 * x0);
    }
  }
  if (!F0) {
    q.f0v = 0.0;
    q.dfx0 = 0.0;
  }
}

// Predicted signal of one measurement; with WANTJ also the Jacobian row J (the one the
// reference uses for the gradient) and J0h, the S0 entry its Hessian uses (they differ only for
// PVM_multi, CUDA/PVM_multi.cu:376 vs :452).
template <int KIND, int K, bool F0, bool WANTJ>
__device__ __forceinline__ Real point(const Pre<KIND, K, F0>& q, const Real (&p)[LmShape<KIND, K, F0>::P], Real gx,
                                      Real gy, Real gz, Real b, int gbo, Real R, Real invR,
                                      Real (&J)[LmShape<KIND, K, F0>::P], Real& J0h) {
  constexpr int P = LmShape<KIND, K, F0>::P, O = LmShape<KIND, K, F0>::O;
  Real dp[K];
#pragma unroll
  for (int k = 0; k < K; ++k) dp[k] = gx * q.v[k][0] + gy * q.v[k][1] + gz * q.v[k][2];
  if (KIND == kSingle || KIND == kSingleC) {
    const Real d = q.d;
    const Real iso = exp(-b * d);
    Real an[K], sig = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      an[k] = exp(-b * d * dp[k] * dp[k]);
      sig += q.fs[k] * an[k];
    }
    const Real wiso = 1.0 - q.sumf - q.f0v;
    const Real full = q.S0 * ((q.f0v + wiso * iso) + sig);
    if (!WANTJ) return full;
#pragma unroll
    for (int i = 0; i < P; ++i) J[i] = 0.0;
    if (KIND == kSingle) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        J[1] += q.sgn1 * q.S0 * q.fs[k] * (-b * dp[k] * dp[k] * an[k]);
        J[O + 3 * k] = q.S0 * (an[k] - iso) * q.dfx[k];
      }
      J[1] += q.sgn1 * q.S0 * wiso * (-b * iso);
    } else {
      const Real lam = p[1];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        J[1] += q.S0 * q.fs[k] * (-2.0 * b * lam * dp[k] * dp[k] * an[k]);
        Real s = 0.0;
#pragma unroll
        for (int j = 0; j < K; ++j) s += q.S0 * (an[j] - iso) * q.deriv[j][k];
        J[O + 3 * k] = s;
      }
      J[1] += q.S0 * wiso * (-2.0 * b * lam * iso);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const Real dp1 = q.cth[k] * (gx * q.cph[k] + gy * q.sph[k]) - gz * q.sth[k];
      const Real dp2 = q.sth[k] * (-gx * q.sph[k] + gy * q.cph[k]);
      const Real c = q.S0 * q.fs[k] * (-2.0 * b * d * dp[k] * an[k]);
      J[O + 3 * k + 1] = c * dp1;
      J[O + 3 * k + 2] = c * dp2;
    }
    if (F0) J[P - 1] = q.S0 * (1.0 - iso) * q.dfx0;
    J[0] = full / p[0];
    J0h = J[0];
    return full;
  } else {
    const Real a = q.a, bb = q.bb;
    const Real liso = log1p(b * bb);
    const Real iso = exp(-a * liso);
    Real an[K], an_a[K], an_b[K], an_th[K], an_ph[K], sig = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const Real x2 = dp[k] * dp[k];
      const Real dp1 = q.cth[k] * (gx * q.cph[k] + gy * q.sph[k]) - gz * q.sth[k];
      const Real dpp = q.sth[k] * (-gx * q.sph[k] + gy * q.cph[k]);
      if (gbo == 2) {
        const Real arg = (1.0 - R) * x2 + R;
        const Real e = exp(-b * 3.0 * a * bb * invR * arg);
        an[k] = e;
        if (WANTJ) {
          const Real da = b * 3.0 * bb * invR * arg;
          an_a[k] = -da * exp(-da * a);
          const Real db = b * 3.0 * a * invR * arg;
          an_b[k] = -db * exp(-db * bb);
          // the zeppelin angle derivatives of CUDA/PVM_multi.cu:82-84,99-101 (no factor dp)
          an_th[k] = -(2.0 * b * 3.0 * a * bb * invR * (1.0 - R) * dp1) * e;
          an_ph[k] = -(2.0 * b * 3.0 * a * bb * invR * (1.0 - R) * dpp) * e;
        }
      } else {
        const Real l = log1p(b * bb * x2);
        an[k] = exp(-a * l);
        if (WANTJ) {
          const Real inv = 1.0 / (1.0 + b * x2 * bb);
          an_a[k] = -l * an[k];
          an_b[k] = -a * b * x2 * inv * an[k];
          const Real t = -a * bb * b * inv * an[k] * 2.0 * dp[k];
          an_th[k] = t * dp1;
          an_ph[k] = t * dpp;
        }
      }
      sig += q.fs[k] * an[k];
    }
    const Real wiso = 1.0 - q.sumf - q.f0v;
    const Real full = q.S0 * ((q.f0v + wiso * iso) + sig);
    if (!WANTJ) return full;
#pragma unroll
    for (int i = 0; i < P; ++i) J[i] = 0.0;
    const Real iso_a = -liso * iso;
    const Real iso_b = -a * b / (1.0 + b * bb) * iso;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      J[1] += q.sgn1 * q.S0 * q.fs[k] * an_a[k];
      J[2] += q.sgn2 * q.S0 * q.fs[k] * an_b[k];
      J[O + 3 * k] = q.S0 * (an[k] - iso) * q.dfx[k];
      J[O + 3 * k + 1] = q.S0 * q.fs[k] * an_th[k];
      J[O + 3 * k + 2] = q.S0 * q.fs[k] * an_ph[k];
    }
    J[1] += q.sgn1 * q.S0 * wiso * iso_a;
    J[2] += q.sgn2 * q.S0 * wiso * iso_b;
    if (F0) J[P - 1] = q.S0 * (1.0 - iso) * q.dfx0;
    J0h = full / p[0];
    J[0] = pm1d(p[0]) * J0h;  // (+-full) / p0 = +-(full / p0) exactly: one division
    return full;
  }
}

template <int KIND, int K, bool F0>
__device__ double cost(const Meas& ms, const Real (&p)[LmShape<KIND, K, F0>::P], int lane, int gbo, Real R,
                       Real invR) {
  constexpr int P = LmShape<KIND, K, F0>::P;
  Pre<KIND, K, F0> q;
  precompute<KIND, K, F0>(p, q);
  double acc = 0.0;
  Real Jd[P];
  Real j0;
  for (int m = lane; m < ms.M; m += 32) {
    const Real e = point<KIND, K, F0, false>(q, p, ms.gx[m], ms.gy[m], ms.gz[m], ms.b[m], gbo, R, invR, Jd, j0) -
                   (Real)ms.y[m];
    acc += e * e;
  }
  return group_sum<32>(acc);
}

// Gauss-Newton normal equations at p, left in the warp's staging area st as the 16x16 matrix
// N = [J | r]^T [J | r] (row stride kNormLd): N[i][j] for i,j < P is (J^T J)_ij with the Hessian's
// S0 column (J0h), N[i][P] is (J^T r)_i, r = S - y.  The rows of [J | r] are written to shared
// memory 32 measurements at a time (one per lane, stored column-major with stride kStageLd, which
// makes both the stores and the fragment loads bank-conflict free) and contracted on the FP64
// tensor cores in 8x8x4 tiles: the upper 8x8 block alone when P+1 <= 8, else the three blocks of
// the upper triangle.  Replaces the per-lane outer products and 32-lane butterflies of
// P(P+1)/2 + P partial sums (CUDA/PVM_multi.cu:371-465 computes the same sums serially).
constexpr int kStageLd = 36;                      // column stride (doubles) of the staged [J | r]
constexpr int kNormLd = 17;                       // row stride (doubles) of N
constexpr int kStageDoubles = 16 * kStageLd;      // per warp: 4.5 KB
static_assert(16 * kNormLd <= 8 * kStageLd, "N must not overlap staged columns 8..15");

template <int KIND, int K, bool F0>
__device__ void normal_eqs(const Meas& ms, const Real (&p)[LmShape<KIND, K, F0>::P], int lane, int gbo, Real R,
                           Real invR, double* st) {
  constexpr int P = LmShape<KIND, K, F0>::P;
  constexpr bool kWide = P + 1 > 8;
  Pre<KIND, K, F0> q;
  precompute<KIND, K, F0>(p, q);
  double n00[2] = {0.0, 0.0}, n01[2] = {0.0, 0.0}, n11[2] = {0.0, 0.0};
  const int fr = lane >> 2, fk = lane & 3;  // fragment row (parameter) and k (measurement) of this lane
  for (int m0 = 0; m0 < ms.M; m0 += 32) {
    const int m = m0 + lane;
    Real J[P], J0h = 0.0, diff = 0.0;
    if (m < ms.M) {
      const Real sig = point<KIND, K, F0, true>(q, p, ms.gx[m], ms.gy[m], ms.gz[m], ms.b[m], gbo, R, invR, J, J0h);
      diff = sig - (Real)ms.y[m];
    } else {
#pragma unroll
      for (int i = 0; i < P; ++i) J[i] = 0.0;
    }
    J[0] = J0h;
    __syncwarp();  // the previous chunk's fragment loads are done
#pragma unroll
    for (int c = 0; c < P; ++c) st[c * kStageLd + lane] = J[c];
    st[P * kStageLd + lane] = diff;
    __syncwarp();
#pragma unroll
    for (int k0 = 0; k0 < 32; k0 += 4) {
      const double lo = st[fr * kStageLd + k0 + fk];
      dmma_8x8x4(n00, lo, lo);
      if (kWide) {
        const double hi = st[(8 + fr) * kStageLd + k0 + fk];
        dmma_8x8x4(n01, lo, hi);
        dmma_8x8x4(n11, hi, hi);
      }
    }
  }
  __syncwarp();
  const int c0 = 2 * fk;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    st[fr * kNormLd + c0 + i] = n00[i];
    if (kWide) {
      st[fr * kNormLd + 8 + c0 + i] = n01[i];
      st[(8 + c0 + i) * kNormLd + fr] = n01[i];
      st[(8 + fr) * kNormLd + 8 + c0 + i] = n11[i];
    }
  }
  __syncwarp();
}

// LM driver (CUDA/levenberg_marquardt.cu:57-122): lambda0 = 0.1, x/÷ 10, converged when
// 2|dcf| <= 1e-8 (|cf_old|+|cf_new|+2e-16), stopped when lambda > 1e20 or after 200 successful
// iterations (the iteration counter advances only on success).  Gradient 2 J^T r and Hessian
// 2 J^T J come from normal_eqs after every successful step and stay in st between steps.
// Returns false when the run stopped at the iteration cap (warp-uniform).
template <int KIND, int K, bool F0>
__device__ bool lm_run(const Meas& ms, Real (&p)[LmShape<KIND, K, F0>::P], int lane, int gbo, Real R, Real invR,
                      double* st) {
  constexpr int P = LmShape<KIND, K, F0>::P;
  double lambda = 0.1;
  const double cftol = 1.0e-8, ltol = 1.0e20;
  double pcf = cost<KIND, K, F0>(ms, p, lane, gbo, R, invR);
  int niter = 0;
  bool success = true, stopped = false;
  double gsign = 1.0;  // PVM_multi's gradient S0 entry carries sign(S0) (CUDA/PVM_multi.cu:376)
  const int row = lane < P ? lane : 0;
  while (!(success && niter++ >= 200)) {
    if (success) {
      normal_eqs<KIND, K, F0>(ms, p, lane, gbo, R, invR, st);
      if (KIND == kMulti && lane == 0) gsign = pm1d(p[0]);
    }
    double A[P];
#pragma unroll
    for (int j = 0; j < P; ++j) A[j] = 2.0 * st[row * kNormLd + j] + ((lane == j) ? lambda : 0.0);
    const double grow = 2.0 * gsign * st[row * kNormLd + P];
    double x[P];
    warp_solve<P>(A, grow, x, lane);
    Real step[P];
#pragma unroll
    for (int i = 0; i < P; ++i) step[i] = p[i] - x[i];
    const double ncf = cost<KIND, K, F0>(ms, step, lane, gbo, R, invR);
    bool end = false;
    if ((success = (ncf < pcf))) {
#pragma unroll
      for (int i = 0; i < P; ++i) p[i] = step[i];
      lambda /= 10.0;
      if (2.0 * fabs(pcf - ncf) <= cftol * (fabs(pcf) + fabs(ncf) + 2.0e-16)) end = true;
      pcf = ncf;
    } else {
      lambda *= 10.0;
      if (lambda > ltol) end = true;
    }
    if (end) {
      stopped = true;
      break;
    }
  }
  return stopped;
}

// adjacent-swap sort of fibres by decreasing f (sort_PVM_*, CUDA/PVM_single.cu:86-104)
template <int K, int O, int P>
__device__ __forceinline__ void sort_fibres(Real (&p)[P]) {
#pragma unroll
  for (int i = 1; i < K; ++i)
#pragma unroll
    for (int j = 0; j < K - i; ++j)
      if (p[O + j * 3] < p[O + (j + 1) * 3]) {
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const Real tmp = p[O + j * 3 + t];
          p[O + j * 3 + t] = p[O + (j + 1) * 3 + t];
          p[O + (j + 1) * 3 + t] = tmp;
        }
      }
}

// finalise raw LM parameters (CUDA/PVM_single.cu:451-466, CUDA/PVM_single_c.cu:582-607,
// CUDA/PVM_multi.cu:549-566)
template <int KIND, int K, bool F0>
__device__ __forceinline__ void finalise(Real (&p)[LmShape<KIND, K, F0>::P]) {
  constexpr int P = LmShape<KIND, K, F0>::P, O = LmShape<KIND, K, F0>::O;
  const Real fsmall = 0.001;
  if (KIND == kSingle) {
    p[1] = fabs(p[1]);
#pragma unroll
    for (int k = 0; k < K; ++k) p[O + 3 * k] = x2fd(p[O + 3 * k]);
    if (F0) p[P - 1] = x2fd(p[P - 1]);
    sort_fibres<K, O, P>(p);
    Real sum = F0 ? p[P - 1] : 0.0;
    bool hit = false;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!hit) {
        sum += p[O + 3 * i];
        if (sum >= 1.0) hit = true;
      }
      if (hit) p[O + 3 * i] = fsmall;
    }
  } else if (KIND == kSingleC) {
    p[1] = p[1] * p[1];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      Real pf = 1.0;
#pragma unroll
      for (int j = 0; j < k; ++j) pf -= p[O + 3 * j];
      p[O + 3 * k] = beta2fd(p[O + 3 * k]) * pf;
    }
    if (F0) {
      Real pf = 1.0;
#pragma unroll
      for (int j = 0; j < K; ++j) pf -= p[O + 3 * j];
      p[P - 1] = beta2fd(p[P - 1]) * pf;
    }
    sort_fibres<K, O, P>(p);
  } else {
    const Real aux = p[1];
    p[1] = fabs(aux * p[2]);
    p[2] = sqrt(fabs(aux * p[2] * p[2]));
#pragma unroll
    for (int k = 0; k < K; ++k) p[O + 3 * k] = x2fd(p[O + 3 * k]);
    if (F0) p[P - 1] = x2fd(p[P - 1]);
    sort_fibres<K, O, P>(p);
    Real sum = F0 ? p[P - 1] : 0.0;
    bool hit = false;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!hit) {
        if (p[O + 3 * i] == 0.0) p[O + 3 * i] = fsmall;
        sum += p[O + 3 * i];
        if (sum >= 1.0) hit = true;
      }
      if (hit) p[O + 3 * i] = fsmall;
    }
  }
}

// PVM_single start values (CUDA/diffmodels.cu:67-91)
template <int K, bool F0>
__device__ void start_single(const Dti& dt, Real (&p)[LmShape<kSingle, K, F0>::P]) {
  constexpr int P = LmShape<kSingle, K, F0>::P;
  Real th, ph;
  cart2sph(dt.v[0], th, ph);
  p[0] = dt.s0;
  p[1] = dt.md > 0 ? dt.md * 2 : 0.001;
  p[2] = dt.fa < 1 ? f2xd(dt.fa) : f2xd(0.95);
  p[3] = th;
  p[4] = ph;
  Real sumf = x2fd(p[2]);
#pragma unroll
  for (int ii = 2; ii <= K; ++ii) {
    const int i = 5 + 3 * (ii - 2);
    Real denom = 2.0, tmpsumf;
    do {
      p[i] = f2xd(x2fd(p[i - 3]) / denom);
      denom *= 2.0;
      tmpsumf = sumf + x2fd(p[i]);
    } while (tmpsumf >= 1.0);
    sumf += x2fd(p[i]);
    cart2sph(dt.v[ii - 1], th, ph);
    p[i + 1] = th;
    p[i + 2] = ph;
  }
  if (F0) p[P - 1] = f2xd(0.001);
}

// PVM_single_c start values with fit_pvf (CUDA/diffmodels.cu:149-184, diffmodels.cc:561-603)
template <int K, bool F0>
__device__ void start_single_c(const Dti& dt, const Meas& ms, int lane, Real (&x)[LmShape<kSingleC, K, F0>::P]) {
  constexpr int P = LmShape<kSingleC, K, F0>::P;
  Real th, ph;
#pragma unroll
  for (int i = 0; i < P; ++i) x[i] = 0.0;
  cart2sph(dt.v[0], th, ph);
  x[0] = dt.s0;
  x[1] = sqrt(dt.l1 > 0 ? dt.l1 : 0.002);
  x[3] = th;
  x[4] = ph;
#pragma unroll
  for (int ii = 2; ii <= K; ++ii) {
    const int i = 5 + 3 * (ii - 2);
    cart2sph(dt.v[ii - 1], th, ph);
    x[i + 1] = th;
    x[i + 2] = ph;
  }
  // linear least squares for the fractions: pinv(M) * (Y - S0 iso)
  const double s0 = x[0], d = x[1] * x[1];
  double dir[K][3];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    dir[k][0] = sin(x[3 + 3 * k]) * cos(x[4 + 3 * k]);
    dir[k][1] = sin(x[3 + 3 * k]) * sin(x[4 + 3 * k]);
    dir[k][2] = cos(x[3 + 3 * k]);
  }
  double MtM[K][K], MtY[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    MtY[i] = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) MtM[i][j] = 0;
  }
  for (int m = lane; m < ms.M; m += 32) {
    const double gx = ms.gx[m], gy = ms.gy[m], gz = ms.gz[m], b = ms.b[m];
    const double iso = exp(-b * d);
    const double yi = ms.y[m] - s0 * iso;
    double row[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double dp = gx * dir[k][0] + gy * dir[k][1] + gz * dir[k][2];
      row[k] = s0 * (exp(-b * d * dp * dp) - iso);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      MtY[i] += row[i] * yi;
#pragma unroll
      for (int j = 0; j < K; ++j) MtM[i][j] += row[i] * row[j];
    }
  }
#pragma unroll
  for (int i = 0; i < K; ++i) {
    MtY[i] = group_sum<32>(MtY[i]);
#pragma unroll
    for (int j = 0; j < K; ++j) MtM[i][j] = group_sum<32>(MtM[i][j]);
  }
  double w[K], V[K][K];
  jacobi_eig<K>(MtM, w, V);
  const double tol = w[0] * 1e-14 * (ms.M > K ? ms.M : K);
  double fs[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    double s = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double gij = 0;
#pragma unroll
      for (int c = 0; c < K; ++c)
        if (w[c] > tol) gij += V[i][c] * V[j][c] / w[c];
      s += gij * MtY[j];
    }
    fs[i] = s;
  }
  double f0v = 0.0;
  if (F0) {
    f0v = 0.001;
    fs[0] -= f0v;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) fs[k] = fabs(fs[k]);
  {
    double sumf = 0.0;
    bool hit = false;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!hit) {
        sumf += fs[i];
        if (sumf >= 1.0) hit = true;
      }
      if (hit) fs[i] = 0.001;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double pf = 1.0;
#pragma unroll
    for (int j = 0; j < k; ++j) pf -= fs[j];
    double tmpr = fs[k] / pf;
    if (tmpr > 1.0) tmpr = 1.0;
    x[2 + 3 * k] = f2betad(tmpr);
  }
  if (F0) {
    double pf = 1.0;
#pragma unroll
    for (int j = 0; j < K; ++j) pf -= fs[j];
    double tmpr = f0v / pf;
    if (tmpr > 1.0) tmpr = 1.0;
    x[P - 1] = f2betad(tmpr);
  }
}

// fit_PVM_multi_kernel start from the finalised PVM_single / PVM_single_c parameters
// (CUDA/PVM_multi.cu:514-530)
template <int K, bool F0>
__device__ __forceinline__ void start_multi(const Real (&s)[LmShape<kSingle, K, F0>::P], Real (&p)[LmShape<kMulti, K, F0>::P]) {
  constexpr int P = LmShape<kMulti, K, F0>::P;
  p[0] = s[0];
  p[1] = 1.0;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const int ii = 3 + 3 * i;
    p[ii] = f2xd(s[ii - 1]);
    p[ii + 1] = s[ii];
    p[ii + 2] = s[ii + 1];
  }
  p[2] = s[1];
  if (F0) p[P - 1] = f2xd(s[P - 2]);
}

// predicted signal from finalised parameters (what get_residuals_*_kernel subtract)
template <int K>
__device__ __forceinline__ Real predict_final(int model, const Real* q, int o, bool use_f0, Real f0, Real R, Real gx,
                                              Real gy, Real gz, Real b) {
  Real sumf = 0.0, val = 0.0, iso, S0 = q[0];
  if (model == 1) {
    const Real d = q[1];
    iso = exp(-b * d);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      Real st, ct, sp, cp;
      sincos(q[o + 3 * k + 1], &st, &ct);
      sincos(q[o + 3 * k + 2], &sp, &cp);
      const Real dp = gx * st * cp + gy * st * sp + gz * ct;
      val += q[o + 3 * k] * exp(-b * d * dp * dp);
      sumf += q[o + 3 * k];
    }
  } else {
    const Real d = q[1], ds = q[2];
    const Real a = d * d / ds / ds, bb = ds * ds / d;
    const Real invR = 1.0 / (2.0 * R + 1.0);
    iso = exp(-a * log1p(b * bb));
#pragma unroll
    for (int k = 0; k < K; ++k) {
      Real st, ct, sp, cp;
      sincos(q[o + 3 * k + 1], &st, &ct);
      sincos(q[o + 3 * k + 2], &sp, &cp);
      const Real dp = gx * st * cp + gy * st * sp + gz * ct;
      Real an;
      if (model == 3)
        an = exp(-b * 3.0 * a * bb * invR * ((1.0 - R) * dp * dp + R));
      else
        an = exp(-a * log1p(b * bb * dp * dp));
      val += q[o + 3 * k] * an;
      sumf += q[o + 3 * k];
    }
    S0 = fabs(S0);
  }
  if (use_f0) return S0 * (f0 + (1.0 - sumf - f0) * iso + val);
  return S0 * ((1.0 - sumf) * iso + val);
}

// ------------------------------------------------------------------------------------------
// the fit as four kernels, one per stage, so each holds one or two LM instances and its warps
// run the same code (the single kernel with every stage was instruction-fetch bound):
//   A  non-finite check, DTI, the first LM fit (PVM_single or PVM_single_c, with f0 if asked)
//   B  PVM_multi from A's fit (models 2 and 3)
//   C  the f0 re-fit of the voxels the plausibility rule flags (CUDA/xfibres_gpu.cu:207-339)
//   D  tau = 1/var(residuals) and the FP32 outputs
// Between stages each voxel's FP64 parameters stay in scratch ([nvox][16] doubles) and its
// state in a flag word.  One warp per voxel; the warps of a block take voxels from a
// shared-memory counter.
// ------------------------------------------------------------------------------------------
// kFitCapped: the LM run that produced the voxel's current parameters stopped at its iteration cap
enum FitFlag : uint32_t { kFitBad = 1u, kFitRefit = 2u, kFitRefitted = 4u, kFitCapped = 8u };

struct VoxelMeas {
  Meas ms;
  __device__ VoxelMeas(const FitArgs& a, int v) {
    const int M = a.ndir;
    ms.y = a.data + (size_t)v * M;
    const float* bv = a.gradnonlin ? a.bvecs + (size_t)v * 3 * M : a.bvecs;
    ms.gx = bv;
    ms.gy = bv + M;
    ms.gz = bv + 2 * M;
    ms.b = a.gradnonlin ? a.bvals + (size_t)v * M : a.bvals;
    ms.M = M;
  }
};

template <int P>
__device__ __forceinline__ void store_res(double* res, const Real (&p)[P], int lane) {
  __syncwarp();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < P; ++i) res[i] = p[i];
  __syncwarp();
}

template <int P>
__device__ __forceinline__ void load_res(const double* res, Real (&p)[P]) {
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = res[i];
}

// the f0 plausibility rule (CUDA/xfibres_gpu.cu:207-222): f1 < 0.05, d > 0.007 or f0 > 0.4
template <int P>
__device__ __forceinline__ bool needs_refit(const Real (&p)[P], int of1) {
  return p[of1] < 0.05 || p[1] > 0.007 || p[P - 1] > 0.4;
}

template <int K, bool F0>
__device__ void stage_start(const FitArgs& a, int v, int lane, double* st) {
  const VoxelMeas vm(a, v);
  const Meas& ms = vm.ms;
  const Real R = a.R, invR = 1.0 / (2.0 * R + 1.0);
  double* res = a.scratch + (size_t)v * 16;
  bool bad = false;
  for (int m = lane; m < ms.M; m += 32) bad |= !isfinite(ms.y[m]);
  bad = __any_sync(0xffffffffu, bad);
  if (bad) {
    if (lane == 0) a.flags[v] = kFitBad;
    return;
  }
  Dti dt;
  dti_fit(ms, lane, dt);
  uint32_t flag = 0;
  if (a.model == 1 && !a.nonlin) {
    Real p[LmShape<kSingleC, K, F0>::P];
    start_single_c<K, F0>(dt, ms, lane, p);
    if (!lm_run<kSingleC, K, F0>(ms, p, lane, 0, R, invR, st)) flag = kFitCapped;
    finalise<kSingleC, K, F0>(p);
    if (F0 && needs_refit(p, 2)) flag |= kFitRefit;
    store_res(res, p, lane);
  } else {
    Real p[LmShape<kSingle, K, F0>::P];
    start_single<K, F0>(dt, p);
    if (!lm_run<kSingle, K, F0>(ms, p, lane, 0, R, invR, st)) flag = kFitCapped;
    finalise<kSingle, K, F0>(p);
    if (a.model == 1 && F0 && needs_refit(p, 2)) flag |= kFitRefit;
    store_res(res, p, lane);
  }
  if (lane == 0) a.flags[v] = flag;
}

template <int K, bool F0>
__device__ void stage_multi(const FitArgs& a, int v, int lane, double* st) {
  if (a.flags[v] & kFitBad) return;
  const VoxelMeas vm(a, v);
  const Real R = a.R, invR = 1.0 / (2.0 * R + 1.0);
  double* res = a.scratch + (size_t)v * 16;
  Real s[LmShape<kSingle, K, F0>::P];
  load_res(res, s);
  Real p[LmShape<kMulti, K, F0>::P];
  start_multi<K, F0>(s, p);
  const bool conv = lm_run<kMulti, K, F0>(vm.ms, p, lane, a.model == 3 ? 2 : 0, R, invR, st);
  finalise<kMulti, K, F0>(p);
  store_res(res, p, lane);
  if (lane == 0) {
    uint32_t fl = (a.flags[v] & ~kFitCapped) | (conv ? 0u : kFitCapped);
    if (F0 && needs_refit(p, 3)) fl |= kFitRefit;
    a.flags[v] = fl;
  }
}

// re-fit without f0 (f0 := 0.001): model 1 with the same start as A; models 2 and 3 through
// PVM_single_c then PVM_multi, as the GPU path does (CUDA/xfibres_gpu.cu:331-333)
template <int K>
__device__ void stage_refit(const FitArgs& a, int v, int lane, double* st) {
  if (!(a.flags[v] & kFitRefit)) return;
  const VoxelMeas vm(a, v);
  const Meas& ms = vm.ms;
  const Real R = a.R, invR = 1.0 / (2.0 * R + 1.0);
  double* res = a.scratch + (size_t)v * 16;
  Dti dt;
  dti_fit(ms, lane, dt);
  bool conv;
  if (a.model == 1) {
    constexpr int NPOUT = 2 + 3 * K + 1;
    if (a.nonlin) {
      Real p[LmShape<kSingle, K, false>::P];
      start_single<K, false>(dt, p);
      conv = lm_run<kSingle, K, false>(ms, p, lane, 0, R, invR, st);
      finalise<kSingle, K, false>(p);
      store_res(res, p, lane);
    } else {
      Real p[LmShape<kSingleC, K, false>::P];
      start_single_c<K, false>(dt, ms, lane, p);
      conv = lm_run<kSingleC, K, false>(ms, p, lane, 0, R, invR, st);
      finalise<kSingleC, K, false>(p);
      store_res(res, p, lane);
    }
    if (lane == 0) res[NPOUT - 1] = 0.001;
  } else {
    constexpr int NPM = LmShape<kMulti, K, true>::P;
    Real c[LmShape<kSingleC, K, false>::P];
    start_single_c<K, false>(dt, ms, lane, c);
    lm_run<kSingleC, K, false>(ms, c, lane, 0, R, invR, st);
    finalise<kSingleC, K, false>(c);
    Real p[LmShape<kMulti, K, false>::P];
    start_multi<K, false>(c, p);
    conv = lm_run<kMulti, K, false>(ms, p, lane, a.model == 3 ? 2 : 0, R, invR, st);
    finalise<kMulti, K, false>(p);
    store_res(res, p, lane);
    if (lane == 0) res[NPM - 1] = 0.001;
  }
  __syncwarp();
  if (lane == 0) a.flags[v] = kFitRefitted | (conv ? 0u : kFitCapped);
}

// tau = 1 / var(y - prediction) (sample variance, n-1) and the FP32 outputs
template <int K, bool F0>
__device__ void stage_finish(const FitArgs& a, int v, int lane, double*) {
  const uint32_t flag = a.flags[v];
  const int npo = a.np_out, M = a.ndir;
  float* out = a.params + (size_t)v * npo;
  if (flag & kFitBad) {
    if (lane < npo) out[lane] = 0.f;
    if (lane == 0) {
      if (a.tau) a.tau[v] = 0.f;
      if (a.status) a.status[v] = BPX_VOX_NONFINITE_DATA;
    }
    return;
  }
  const bool refit = (flag & kFitRefitted) != 0;
  const double* res = a.scratch + (size_t)v * 16;
  Real r[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = i < npo ? res[i] : 0.0;
  if (a.rician) {
    const VoxelMeas vm(a, v);
    const Meas& ms = vm.ms;
    const int o = a.model >= 2 ? 3 : 2;
    const bool use_f0 = F0 && !refit;
    const Real f0 = F0 ? res[npo - 1] : 0.0;
    double s1 = 0.0;
    for (int m = lane; m < M; m += 32)
      s1 += ms.y[m] - predict_final<K>(a.model, r, o, use_f0, f0, a.R, ms.gx[m], ms.gy[m], ms.gz[m], ms.b[m]);
    const double mean = group_sum<32>(s1) / M;
    double s2 = 0.0;
    for (int m = lane; m < M; m += 32) {
      const double e = ms.y[m] - predict_final<K>(a.model, r, o, use_f0, f0, a.R, ms.gx[m], ms.gy[m], ms.gz[m], ms.b[m]) -
                       mean;
      s2 += e * e;
    }
    s2 = group_sum<32>(s2);
    if (lane == 0 && a.tau) a.tau[v] = (float)(1.0 / (s2 / (M - 1)));
  } else if (lane == 0 && a.tau) {
    a.tau[v] = 0.f;
  }
  if (lane < npo) out[lane] = (float)res[lane];
  if (lane == 0 && a.status)
    a.status[v] = (refit ? BPX_VOX_F0_REFIT : 0u) | ((flag & kFitCapped) ? BPX_VOX_LM_ITERATION_CAP : 0u);
}

// Each block owns kFitVoxPerBlock consecutive voxels; its warps take the next one from a
// shared-memory counter as they finish, so a voxel whose fit runs 200 iterations holds up one
// warp instead of a fixed share of the block's voxels.
template <typename Stage>
__device__ __forceinline__ void run_stage(const FitArgs& a, Stage stage) {
  __shared__ double stage_buf[kFitThreads / 32][kStageDoubles];
  __shared__ int next;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* st = stage_buf[w];
  for (int i = lane; i < kStageDoubles; i += 32) st[i] = 0.0;
  const int v0 = blockIdx.x * kFitVoxPerBlock;
  const int v1 = min(v0 + kFitVoxPerBlock, a.nvox);
  if (threadIdx.x == 0) next = v0 + kFitThreads / 32;
  __syncthreads();
  int v = v0 + w;
  while (v < v1) {
    stage(a, v, lane, st);
    int nv = 0;
    if (lane == 0) nv = atomicAdd(&next, 1);
    v = __shfl_sync(0xffffffffu, nv, 0);
  }
}

template <int K, bool F0>
__global__ void __launch_bounds__(kFitThreads, kFitMinBlocks) fit_start_kernel(FitArgs a) {
  run_stage(a, [](const FitArgs& x, int v, int lane, double* st) { stage_start<K, F0>(x, v, lane, st); });
}
template <int K, bool F0>
__global__ void __launch_bounds__(kFitThreads, kFitMinBlocks) fit_multi_kernel(FitArgs a) {
  run_stage(a, [](const FitArgs& x, int v, int lane, double* st) { stage_multi<K, F0>(x, v, lane, st); });
}
template <int K>
__global__ void __launch_bounds__(kFitThreads, kFitMinBlocks) fit_refit_kernel(FitArgs a) {
  run_stage(a, [](const FitArgs& x, int v, int lane, double* st) { stage_refit<K>(x, v, lane, st); });
}
template <int K, bool F0>
__global__ void __launch_bounds__(kFitThreads, kFitMinBlocks) fit_finish_kernel(FitArgs a) {
  run_stage(a, [](const FitArgs& x, int v, int lane, double* st) { stage_finish<K, F0>(x, v, lane, st); });
}

// remove_NonPositive_entries (CUDA/xfibres_gpu.cu:350-367), one warp per voxel
__global__ void __launch_bounds__(kFitThreads) prepare_kernel(int nvox, int ndir, float* data) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int v = blockIdx.x * warps + (threadIdx.x >> 5); v < nvox; v += gridDim.x * warps) {
    float* y = data + (size_t)v * ndir;
    float mn = INFINITY, mx = -INFINITY;
    for (int m = lane; m < ndir; m += 32) {
      mn = fminf(mn, y[m]);
      mx = fmaxf(mx, y[m]);
    }
    mn = group_min<32>(mn);
    mx = group_max<32>(mx);
    if (mn <= 0.f && mx > 0.f) {
      float mp = INFINITY;
      for (int m = lane; m < ndir; m += 32)
        if (y[m] > 0.f) mp = fminf(mp, y[m]);
      mp = group_min<32>(mp);
      for (int m = lane; m < ndir; m += 32)
        if (y[m] <= 0.f) y[m] = mp;
    }
  }
}

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
template <int K, bool F0>
static cudaError_t launch_fit_kf(const FitArgs& a, cudaStream_t s) {
  const int grid = (a.nvox + kFitVoxPerBlock - 1) / kFitVoxPerBlock;
  fit_start_kernel<K, F0><<<grid, kFitThreads, 0, s>>>(a);
  if (a.model >= 2) fit_multi_kernel<K, F0><<<grid, kFitThreads, 0, s>>>(a);
  if (F0) fit_refit_kernel<K><<<grid, kFitThreads, 0, s>>>(a);
  fit_finish_kernel<K, F0><<<grid, kFitThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fit(const FitArgs& a, int nfib, bool f0, cudaStream_t s) {
  if (a.nvox == 0) return cudaSuccess;
  if (!a.scratch || !a.flags) return cudaErrorInvalidValue;
  switch (nfib * 2 + (f0 ? 1 : 0)) {
    case 2: return launch_fit_kf<1, false>(a, s);
    case 3: return launch_fit_kf<1, true>(a, s);
    case 4: return launch_fit_kf<2, false>(a, s);
    case 5: return launch_fit_kf<2, true>(a, s);
    case 6: return launch_fit_kf<3, false>(a, s);
    case 7: return launch_fit_kf<3, true>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_prepare(int nvox, int ndir, float* data, cudaStream_t s) {
  if (nvox == 0) return cudaSuccess;
  const int warps = kFitThreads / 32;
  int grid = (nvox + warps - 1) / warps;
  const int cap = sm_count() * 16;
  if (grid > cap) grid = cap;
  prepare_kernel<<<grid, kFitThreads, 0, s>>>(nvox, ndir, data);
  return cudaGetLastError();
}

}  // namespace bpx
