// Small-matrix math of the DiffPhD local step: 3x3 unsigned SVD, element
// projections and their directional derivatives, templated on precision.
//
// Conventions follow the reference projections
// (src/newton_solver_diff_phd/_src/solvers/diff_phd/projections.py):
//  * unsigned_svd (:88-167): Eigen's two-sided JacobiSVD for 3x3 -- sweep order
//    (1,0),(2,0),(2,1), threshold max(min_normal, 2 eps max|diag|) on the
//    max-abs-scaled matrix, sigma >= 0 with negative diagonal entries flipping
//    columns of U, descending sort that stops at the first zero maximum. U V^T is
//    therefore a reflection when det F < 0.
//  * volume_offset (:237-260), nh_prox_stretches (:278-305) with the pivoted
//    3x3 LDL^T of Eigen (:178-228), muscle_projection (:308-316).
//  * dsvd (:323-340) and the JVPs (:343-433) of the backward pass.
// All functions are plain per-thread code; a thread owns one element sample.
#pragma once

#include <cfloat>
#include <cmath>

#ifndef PD_HD
#define PD_HD __host__ __device__ __forceinline__
#endif

namespace pdb200 {

template <typename T>
struct Limits;
template <>
struct Limits<double> {
  static PD_HD double eps() { return DBL_EPSILON; }
  static PD_HD double min_normal() { return DBL_MIN; }
};
template <>
struct Limits<float> {
  static PD_HD float eps() { return FLT_EPSILON; }
  static PD_HD float min_normal() { return FLT_MIN; }
};

template <typename T>
struct V3 {
  T x, y, z;
  PD_HD T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  PD_HD T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

// Row-major 3x3 matrix; a[r][c].
template <typename T>
struct M3 {
  T a[3][3];
};

template <typename T>
PD_HD V3<T> v3(T x, T y, T z) {
  V3<T> r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
template <typename T>
PD_HD V3<T> operator+(V3<T> a, V3<T> b) { return v3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T>
PD_HD V3<T> operator-(V3<T> a, V3<T> b) { return v3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T>
PD_HD V3<T> operator*(T s, V3<T> a) { return v3<T>(s * a.x, s * a.y, s * a.z); }
template <typename T>
PD_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
PD_HD T length(V3<T> a) { return sqrt(dot(a, a)); }
template <typename T>
PD_HD V3<T> cross(V3<T> a, V3<T> b) {
  return v3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

template <typename T>
PD_HD M3<T> zero3() {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = T(0);
  return m;
}
template <typename T>
PD_HD M3<T> identity3() {
  M3<T> m = zero3<T>();
  m.a[0][0] = m.a[1][1] = m.a[2][2] = T(1);
  return m;
}
template <typename T>
PD_HD M3<T> operator+(const M3<T>& x, const M3<T>& y) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = x.a[i][j] + y.a[i][j];
  return m;
}
template <typename T>
PD_HD M3<T> operator-(const M3<T>& x, const M3<T>& y) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = x.a[i][j] - y.a[i][j];
  return m;
}
template <typename T>
PD_HD M3<T> operator*(T s, const M3<T>& x) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = s * x.a[i][j];
  return m;
}
template <typename T>
PD_HD M3<T> mul(const M3<T>& x, const M3<T>& y) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = x.a[i][0] * y.a[0][j] + x.a[i][1] * y.a[1][j] + x.a[i][2] * y.a[2][j];
  return m;
}
template <typename T>
PD_HD V3<T> mul(const M3<T>& x, V3<T> v) {
  return v3<T>(x.a[0][0] * v.x + x.a[0][1] * v.y + x.a[0][2] * v.z, x.a[1][0] * v.x + x.a[1][1] * v.y + x.a[1][2] * v.z,
               x.a[2][0] * v.x + x.a[2][1] * v.y + x.a[2][2] * v.z);
}
template <typename T>
PD_HD M3<T> transpose(const M3<T>& x) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = x.a[j][i];
  return m;
}
template <typename T>
PD_HD M3<T> outer(V3<T> u, V3<T> v) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) m.a[i][j] = u[i] * v[j];
  return m;
}
template <typename T>
PD_HD M3<T> diag3(V3<T> d) {
  M3<T> m = zero3<T>();
  m.a[0][0] = d.x;
  m.a[1][1] = d.y;
  m.a[2][2] = d.z;
  return m;
}
// U diag(d) V^T.
template <typename T>
PD_HD M3<T> udvt(const M3<T>& u, V3<T> d, const M3<T>& v) {
  M3<T> m;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      m.a[i][j] = u.a[i][0] * d.x * v.a[j][0] + u.a[i][1] * d.y * v.a[j][1] + u.a[i][2] * d.z * v.a[j][2];
  return m;
}
template <typename T>
PD_HD T determinant(const M3<T>& m) {
  return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) -
         m.a[0][1] * (m.a[1][0] * m.a[2][2] - m.a[1][2] * m.a[2][0]) +
         m.a[0][2] * (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]);
}
// Inverse by the adjugate over the determinant.
template <typename T>
PD_HD M3<T> inverse(const M3<T>& m) {
  const T inv = T(1) / determinant(m);
  M3<T> r;
  r.a[0][0] = (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) * inv;
  r.a[0][1] = (m.a[0][2] * m.a[2][1] - m.a[0][1] * m.a[2][2]) * inv;
  r.a[0][2] = (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]) * inv;
  r.a[1][0] = (m.a[1][2] * m.a[2][0] - m.a[1][0] * m.a[2][2]) * inv;
  r.a[1][1] = (m.a[0][0] * m.a[2][2] - m.a[0][2] * m.a[2][0]) * inv;
  r.a[1][2] = (m.a[0][2] * m.a[1][0] - m.a[0][0] * m.a[1][2]) * inv;
  r.a[2][0] = (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]) * inv;
  r.a[2][1] = (m.a[0][1] * m.a[2][0] - m.a[0][0] * m.a[2][1]) * inv;
  r.a[2][2] = (m.a[0][0] * m.a[1][1] - m.a[0][1] * m.a[1][0]) * inv;
  return r;
}

// ---------------------------------------------------------------------------
// Eigen-convention two-sided Jacobi SVD.

template <typename T>
PD_HD void rotate_rows(M3<T>& m, int p, int q, T c, T s) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const T x = m.a[p][j];
    const T y = m.a[q][j];
    m.a[p][j] = c * x + s * y;
    m.a[q][j] = -s * x + c * y;
  }
}
template <typename T>
PD_HD void rotate_columns(M3<T>& m, int p, int q, T c, T s) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T x = m.a[i][p];
    const T y = m.a[i][q];
    m.a[i][p] = c * x - s * y;
    m.a[i][q] = s * x + c * y;
  }
}
// 1 / sqrt(x) (a hardware-seeded reciprocal square root on the device).
template <typename T>
PD_HD T reciprocal_sqrt(T x) {
#ifdef __CUDA_ARCH__
  return rsqrt(x);
#else
  return T(1) / sqrt(x);
#endif
}

// Symmetric 2x2 Jacobi rotation (Eigen JacobiRotation::makeJacobi for reals):
// tau = (x - z) / 2|y|, t = 1 / (tau +- sqrt(tau^2 + 1)), c = 1 / sqrt(t^2 + 1),
// s = -sign(t) sign(y) |t| c. The reciprocal square root and the sign copy
// replace two of Eigen's divisions; results agree to rounding.
template <typename T>
PD_HD void make_jacobi(T x, T y, T z, T& c, T& s) {
  c = T(1);
  s = T(0);
  const T denominator = T(2) * fabs(y);
  if (denominator >= Limits<T>::min_normal()) {
    const T tau = (x - z) / denominator;
    const T w = sqrt(tau * tau + T(1));
    const T t = tau > T(0) ? T(1) / (tau + w) : T(1) / (tau - w);
    const T sign = t > T(0) ? T(1) : T(-1);
    const T n = reciprocal_sqrt(t * t + T(1));
    s = -sign * copysign(T(1), y) * fabs(t) * n;
    c = n;
  }
}

constexpr int kJacobiMaxSweeps = 64;

// Swap entries I and J of sigma and columns I and J of U and V.
template <typename T, int I, int J>
PD_HD void swap_columns(V3<T>& sigma, M3<T>& u, M3<T>& v) {
  const T value = sigma[I];
  sigma[I] = sigma[J];
  sigma[J] = value;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    T t = u.a[r][I];
    u.a[r][I] = u.a[r][J];
    u.a[r][J] = t;
    t = v.a[r][I];
    v.a[r][I] = v.a[r][J];
    v.a[r][J] = t;
  }
}

// F = U diag(sigma) V^T with sigma >= 0 sorted descending.
template <typename T>
PD_HD void unsigned_svd(const M3<T>& f, M3<T>& u, V3<T>& sigma, M3<T>& v) {
  T scale = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) scale = fmax(scale, fabs(f.a[i][j]));
  if (scale == T(0)) scale = T(1);
  M3<T> w;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) w.a[i][j] = f.a[i][j] / scale;
  u = identity3<T>();
  v = identity3<T>();
  T largest = fmax(fmax(fabs(w.a[0][0]), fabs(w.a[1][1])), fabs(w.a[2][2]));
  const T precision = T(2) * Limits<T>::eps();
  for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
    bool finished = true;
#pragma unroll
    for (int pair = 0; pair < 3; ++pair) {
      const int p = pair == 0 ? 1 : 2;
      const int q = pair == 2 ? 1 : 0;
      const T threshold = fmax(Limits<T>::min_normal(), precision * largest);
      if (fabs(w.a[p][q]) > threshold || fabs(w.a[q][p]) > threshold) {
        finished = false;
        const T t = w.a[p][p] + w.a[q][q];
        const T d = w.a[q][p] - w.a[p][q];
        T c1 = T(1);
        T s1 = T(0);
        if (fabs(d) >= Limits<T>::min_normal()) {
          const T ratio = t / d;
          const T inverse_root = reciprocal_sqrt(T(1) + ratio * ratio);
          s1 = inverse_root;
          c1 = ratio * inverse_root;
        }
        const T m00 = c1 * w.a[p][p] + s1 * w.a[q][p];
        const T m01 = c1 * w.a[p][q] + s1 * w.a[q][q];
        const T m11 = -s1 * w.a[p][q] + c1 * w.a[q][q];
        T cr, sr;
        make_jacobi(m00, m01, m11, cr, sr);
        const T cl = c1 * cr + s1 * sr;
        const T sl = s1 * cr - c1 * sr;
        rotate_rows(w, p, q, cl, sl);
        rotate_columns(u, p, q, cl, -sl);
        rotate_columns(w, p, q, cr, sr);
        rotate_columns(v, p, q, cr, sr);
        largest = fmax(largest, fmax(fabs(w.a[p][p]), fabs(w.a[q][q])));
      }
    }
    if (finished) break;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T value = w.a[i][i];
    sigma[i] = fabs(value) * scale;
    if (value < T(0)) {
#pragma unroll
      for (int r = 0; r < 3; ++r) u.a[r][i] = -u.a[r][i];
    }
  }
  // Descending selection sort that stops at the first zero maximum (Eigen),
  // written with compile-time column indices so U and V stay in registers.
  {
    int position = 0;
    if (sigma.y > sigma[position]) position = 1;
    if (sigma.z > sigma[position]) position = 2;
    if (sigma[position] != T(0)) {
      if (position == 1) {
        swap_columns<T, 0, 1>(sigma, u, v);
      } else if (position == 2) {
        swap_columns<T, 0, 2>(sigma, u, v);
      }
      if (sigma.z > sigma.y) {
        if (sigma.z != T(0)) swap_columns<T, 1, 2>(sigma, u, v);
      } else if (sigma.y == T(0)) {
        // The maximum of the remaining entries is zero: the sort stops.
      }
    }
  }
}

// Closest offset D with prod(sigma + D) = 1 (volume projection). `singular`
// reports min(sigma) < eps (the reference's "Singular F.").
template <typename T>
PD_HD V3<T> volume_offset(V3<T> sigma, bool& singular) {
  singular = sigma.z < Limits<T>::eps();
  const T product = sigma.x * sigma.y * sigma.z;
  const T root = cbrt(product);
  V3<T> d = v3<T>(sigma.x / root - sigma.x, sigma.y / root - sigma.y, sigma.z / root - sigma.z);
  for (int iteration = 0; iteration < 50; ++iteration) {
    const V3<T> s = sigma + d;
    const T constraint = s.x * s.y * s.z - T(1);
    const V3<T> gradient = v3<T>(s.y * s.z, s.x * s.z, s.x * s.y);
    const T factor = (dot(gradient, d) - constraint) / dot(gradient, gradient);
    const V3<T> following = factor * gradient;
    const T difference =
        fmax(fmax(fabs(following.x - d.x), fabs(following.y - d.y)), fabs(following.z - d.z));
    if (difference <= Limits<T>::eps()) break;
    d = following;
  }
  return d;
}

// Eigen dense LDLT of a symmetric 3x3 matrix (largest remaining diagonal as
// pivot, pseudo-inverse of D) followed by the solve.
template <typename T>
PD_HD V3<T> ldlt3_solve(M3<T> m, V3<T> b) {
  int perm[3] = {0, 1, 2};
  for (int k = 0; k < 3; ++k) {
    int biggest = k;
    for (int i = k + 1; i < 3; ++i)
      if (fabs(m.a[i][i]) > fabs(m.a[biggest][biggest])) biggest = i;
    if (biggest != k) {
      for (int j = 0; j < 3; ++j) {
        const T t = m.a[k][j];
        m.a[k][j] = m.a[biggest][j];
        m.a[biggest][j] = t;
      }
      for (int i = 0; i < 3; ++i) {
        const T t = m.a[i][k];
        m.a[i][k] = m.a[i][biggest];
        m.a[i][biggest] = t;
      }
      const int t = perm[k];
      perm[k] = perm[biggest];
      perm[biggest] = t;
    }
    for (int j = 0; j < k; ++j) m.a[k][k] = m.a[k][k] - m.a[k][j] * m.a[k][j] * m.a[j][j];
    for (int i = k + 1; i < 3; ++i) {
      for (int j = 0; j < k; ++j) m.a[i][k] = m.a[i][k] - m.a[i][j] * m.a[j][j] * m.a[k][j];
      if (m.a[k][k] != T(0)) m.a[i][k] = m.a[i][k] / m.a[k][k];
    }
  }
  T y[3] = {b[perm[0]], b[perm[1]], b[perm[2]]};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < i; ++j) y[i] = y[i] - m.a[i][j] * y[j];
  for (int i = 0; i < 3; ++i) y[i] = fabs(m.a[i][i]) > Limits<T>::min_normal() ? y[i] / m.a[i][i] : T(0);
  for (int r = 0; r < 3; ++r) {
    const int i = 2 - r;
    for (int j = i + 1; j < 3; ++j) y[i] = y[i] - m.a[j][i] * y[j];
  }
  V3<T> x;
  for (int i = 0; i < 3; ++i) x[perm[i]] = y[i];
  return x;
}

// Hessian of psi(sigma) + penalty/2 |sigma - sigma_F|^2 for the proximal Neo-Hookean map.
template <typename T>
PD_HD M3<T> nh_prox_hessian(V3<T> sigma, T mu, T lame, T penalty) {
  const T product = sigma.x * sigma.y * sigma.z;
  const T log_j = log(fmax(product, T(1.0e-12)));
  M3<T> h;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      h.a[i][j] = i == j ? mu + (mu + lame - lame * log_j) / (sigma[i] * sigma[i]) + penalty
                         : lame / (sigma[i] * sigma[j]);
  return h;
}

// Proximal Neo-Hookean singular values by damped Newton with a floor of 1e-4.
template <typename T>
PD_HD V3<T> nh_prox_stretches(V3<T> target, T mu, T lame, T penalty) {
  const T floor = T(1.0e-4);
  const T tolerance = T(1.0e-10);
  V3<T> sigma = v3<T>(fmax(target.x, floor), fmax(target.y, floor), fmax(target.z, floor));
  for (int iteration = 0; iteration < 32; ++iteration) {
    const T product = sigma.x * sigma.y * sigma.z;
    const T log_j = log(fmax(product, T(1.0e-12)));
    V3<T> gradient;
    for (int i = 0; i < 3; ++i)
      gradient[i] = mu * sigma[i] - mu / sigma[i] + lame * log_j / sigma[i] + penalty * (sigma[i] - target[i]);
    if (length(gradient) < tolerance) break;
    M3<T> hessian = nh_prox_hessian(sigma, mu, lame, penalty);
    for (int i = 0; i < 3; ++i) hessian.a[i][i] = hessian.a[i][i] + T(1.0e-9);
    const V3<T> delta = ldlt3_solve(hessian, gradient);
    T alpha = T(1);
    V3<T> trial = sigma - alpha * delta;
    for (int search = 0; search < 20; ++search) {
      if (fmin(fmin(trial.x, trial.y), trial.z) > floor * T(0.5)) break;
      alpha *= T(0.5);
      trial = sigma - alpha * delta;
    }
    const T step = fmax(fmax(fabs(trial.x - sigma.x), fabs(trial.y - sigma.y)), fabs(trial.z - sigma.z));
    sigma = v3<T>(fmax(trial.x, floor), fmax(trial.y, floor), fmax(trial.z, floor));
    if (step < tolerance) break;
  }
  return sigma;
}

// Fibre projection a F m / |F m| (zero for a collapsed fibre).
template <typename T>
PD_HD V3<T> muscle_projection(const M3<T>& f, V3<T> direction, T target_length) {
  const V3<T> fibre = mul(f, direction);
  const T len = length(fibre);
  if (len > Limits<T>::eps()) return (target_length / len) * fibre;
  return v3<T>(T(0), T(0), T(0));
}

// ---------------------------------------------------------------------------
// Directional derivatives (backward pass).

template <typename T>
PD_HD void dsvd(const M3<T>& u, V3<T> sigma, const M3<T>& v, const M3<T>& df, M3<T>& du, V3<T>& dsigma, M3<T>& dv) {
  const M3<T> dp = mul(mul(transpose(u), df), v);
  dsigma = v3<T>(dp.a[0][0], dp.a[1][1], dp.a[2][2]);
  M3<T> factor = zero3<T>();
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (sigma[i] - sigma[j] > T(10) * Limits<T>::eps()) {
        factor.a[i][j] = T(1) / (sigma[j] * sigma[j] - sigma[i] * sigma[i]);
        factor.a[j][i] = -factor.a[i][j];
      }
  M3<T> omega_u, omega_v;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      // (dp S + S dp^T) and (S dp + dp^T S) with S = diag(sigma).
      omega_u.a[i][j] = factor.a[i][j] * (dp.a[i][j] * sigma[j] + sigma[i] * dp.a[j][i]);
      omega_v.a[i][j] = factor.a[i][j] * (sigma[i] * dp.a[i][j] + dp.a[j][i] * sigma[j]);
    }
  du = mul(u, omega_u);
  dv = mul(v, omega_v);
}

// dR/dF of the polar rotation R = U V^T.
template <typename T>
PD_HD M3<T> corotated_jvp(const M3<T>& u, V3<T> sigma, const M3<T>& v, const M3<T>& df) {
  const M3<T> r = mul(u, transpose(v));
  const M3<T> s = udvt(v, sigma, v);
  const M3<T> lhs = mul(transpose(r), df) - mul(transpose(df), r);
  M3<T> a;
  a.a[0][0] = s.a[0][0] + s.a[1][1];
  a.a[0][1] = s.a[1][2];
  a.a[0][2] = -s.a[0][2];
  a.a[1][0] = s.a[1][2];
  a.a[1][1] = s.a[0][0] + s.a[2][2];
  a.a[1][2] = s.a[0][1];
  a.a[2][0] = -s.a[0][2];
  a.a[2][1] = s.a[0][1];
  a.a[2][2] = s.a[1][1] + s.a[2][2];
  const V3<T> xyz = mul(inverse(a), v3<T>(lhs.a[0][1], lhs.a[0][2], lhs.a[1][2]));
  M3<T> w;
  w.a[0][0] = T(0);
  w.a[0][1] = xyz.x;
  w.a[0][2] = xyz.y;
  w.a[1][0] = -xyz.x;
  w.a[1][1] = T(0);
  w.a[1][2] = xyz.z;
  w.a[2][0] = -xyz.y;
  w.a[2][1] = -xyz.z;
  w.a[2][2] = T(0);
  return mul(r, w);
}

// Solve a 4x4 system by Gaussian elimination with partial pivoting.
template <typename T>
PD_HD void solve4(T m[4][4], T b[4], T x[4]) {
  for (int k = 0; k < 4; ++k) {
    int pivot = k;
    for (int i = k + 1; i < 4; ++i)
      if (fabs(m[i][k]) > fabs(m[pivot][k])) pivot = i;
    if (pivot != k) {
      for (int j = 0; j < 4; ++j) {
        const T t = m[k][j];
        m[k][j] = m[pivot][j];
        m[pivot][j] = t;
      }
      const T t = b[k];
      b[k] = b[pivot];
      b[pivot] = t;
    }
    for (int i = k + 1; i < 4; ++i) {
      const T factor = m[i][k] / m[k][k];
      for (int j = k; j < 4; ++j) m[i][j] -= factor * m[k][j];
      b[i] -= factor * b[k];
    }
  }
  for (int i = 3; i >= 0; --i) {
    T value = b[i];
    for (int j = i + 1; j < 4; ++j) value -= m[i][j] * x[j];
    x[i] = value / m[i][i];
  }
}

// Derivative of the volume projection from the KKT system of the constraint.
template <typename T>
PD_HD M3<T> volume_jvp(const M3<T>& u, V3<T> sigma, const M3<T>& v, V3<T> offset, const M3<T>& df) {
  const V3<T> s = sigma + offset;
  const V3<T> gradient = v3<T>(s.y * s.z, s.x * s.z, s.x * s.y);
  M3<T> h;
  h.a[0][0] = T(0);
  h.a[0][1] = s.z;
  h.a[0][2] = s.y;
  h.a[1][0] = s.z;
  h.a[1][1] = T(0);
  h.a[1][2] = s.x;
  h.a[2][0] = s.y;
  h.a[2][1] = s.x;
  h.a[2][2] = T(0);
  M3<T> du, dv;
  V3<T> dsigma;
  dsvd(u, sigma, v, df, du, dsigma, dv);
  const T magnitude = length(offset) / length(gradient);
  T multiplier = magnitude;
  const V3<T> plus = offset - magnitude * gradient;
  const V3<T> minus = offset + magnitude * gradient;
  if (dot(plus, plus) < dot(minus, minus)) multiplier = -magnitude;
  T kkt[4][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) kkt[i][j] = multiplier * h.a[i][j];
    kkt[i][i] = kkt[i][i] + T(1);
    kkt[i][3] = gradient[i];
    kkt[3][i] = gradient[i];
  }
  kkt[3][3] = T(0);
  const V3<T> top = (-multiplier) * mul(h, dsigma);
  T rhs[4] = {top.x, top.y, top.z, -dot(gradient, dsigma)};
  T solution[4];
  solve4(kkt, rhs, solution);
  const V3<T> doffset = v3<T>(solution[0], solution[1], solution[2]);
  return df + udvt(du, offset, v) + udvt(u, doffset, v) + udvt(u, offset, dv);
}

// Implicit-function derivative of the proximal Neo-Hookean projection.
template <typename T>
PD_HD M3<T> nh_prox_jvp(const M3<T>& u, V3<T> sigma, const M3<T>& v, V3<T> stretches, const M3<T>& df, T mu, T lame,
                        T penalty) {
  M3<T> du, dv;
  V3<T> dsigma;
  dsvd(u, sigma, v, df, du, dsigma, dv);
  M3<T> hessian = nh_prox_hessian(stretches, mu, lame, penalty);
  for (int i = 0; i < 3; ++i) hessian.a[i][i] = hessian.a[i][i] + T(1.0e-9);
  const V3<T> dstretches = ldlt3_solve(hessian, penalty * dsigma);
  return udvt(du, stretches, v) + udvt(u, dstretches, v) + udvt(u, stretches, dv);
}

// Derivative of the fibre projection at a fixed target length.
template <typename T>
PD_HD V3<T> muscle_jvp(const M3<T>& f, V3<T> direction, T target_length, const M3<T>& df) {
  const V3<T> fibre = mul(f, direction);
  const T len = length(fibre);
  if (len > Limits<T>::eps()) {
    const V3<T> dfibre = mul(df, direction);
    const T dlen = dot((T(1) / len) * fibre, dfibre);
    const T ratio = target_length / len;
    return ratio * dfibre - (target_length / (len * len) * dlen) * fibre;
  }
  return v3<T>(T(0), T(0), T(0));
}

// True Neo-Hookean first Piola-Kirchhoff stress.
template <typename T>
PD_HD M3<T> neo_hookean_stress(const M3<T>& f, T mu, T lame) {
  const T log_j = log(fmax(determinant(f), T(1.0e-12)));
  const M3<T> inverse_transpose = transpose(inverse(f));
  return mu * (f - inverse_transpose) + (lame * log_j) * inverse_transpose;
}

}  // namespace pdb200
