// tl_math.cuh -- 3-vectors, 3x3 matrices and the element rotations used by
// the tet FEM kernels.  Row-major m[row][col].  Everything is templated on
// the scalar so the same code runs in FP64 and FP32.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include <type_traits>

#define TL_HD __host__ __device__ __forceinline__

namespace tl {

template <class T>
struct V3 {
  T x, y, z;
};

template <class T> TL_HD V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> TL_HD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> TL_HD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> TL_HD V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> TL_HD V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> TL_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> TL_HD V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T, class U> TL_HD V3<T> cvt(V3<U> a) { return {T(a.x), T(a.y), T(a.z)}; }

template <class T>
struct M3 {
  T m[3][3];
};

template <class T> TL_HD M3<T> zero3() {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = T(0);
  return r;
}
template <class T> TL_HD M3<T> eye3() {
  M3<T> r = zero3<T>();
  r.m[0][0] = r.m[1][1] = r.m[2][2] = T(1);
  return r;
}
template <class T> TL_HD V3<T> mul(const M3<T>& a, V3<T> v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
// a^T v
template <class T> TL_HD V3<T> mulT(const M3<T>& a, V3<T> v) {
  return {a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z, a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
          a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}
template <class T> TL_HD M3<T> mul(const M3<T>& a, const M3<T>& b) {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
  return r;
}
template <class T> TL_HD M3<T> transpose(const M3<T>& a) {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
  return r;
}
template <class T> TL_HD T det3(const M3<T>& a) {
  return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
         a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
         a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}
// Cofactor matrix: cof(A) = det(A) A^-T.
template <class T> TL_HD M3<T> cofactor(const M3<T>& a) {
  M3<T> c;
  c.m[0][0] = a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1];
  c.m[0][1] = a.m[1][2] * a.m[2][0] - a.m[1][0] * a.m[2][2];
  c.m[0][2] = a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0];
  c.m[1][0] = a.m[0][2] * a.m[2][1] - a.m[0][1] * a.m[2][2];
  c.m[1][1] = a.m[0][0] * a.m[2][2] - a.m[0][2] * a.m[2][0];
  c.m[1][2] = a.m[0][1] * a.m[2][0] - a.m[0][0] * a.m[2][1];
  c.m[2][0] = a.m[0][1] * a.m[1][2] - a.m[0][2] * a.m[1][1];
  c.m[2][1] = a.m[0][2] * a.m[1][0] - a.m[0][0] * a.m[1][2];
  c.m[2][2] = a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0];
  return c;
}
template <class T> TL_HD T trace3(const M3<T>& a) { return a.m[0][0] + a.m[1][1] + a.m[2][2]; }
template <class T> TL_HD T contract(const M3<T>& a, const M3<T>& b) {
  T s = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s += a.m[i][j] * b.m[i][j];
  return s;
}
// a b^T
template <class T> TL_HD M3<T> outer(V3<T> a, V3<T> b) {
  M3<T> r;
  r.m[0][0] = a.x * b.x; r.m[0][1] = a.x * b.y; r.m[0][2] = a.x * b.z;
  r.m[1][0] = a.y * b.x; r.m[1][1] = a.y * b.y; r.m[1][2] = a.y * b.z;
  r.m[2][0] = a.z * b.x; r.m[2][1] = a.z * b.y; r.m[2][2] = a.z * b.z;
  return r;
}
template <class T> TL_HD void addOuter(M3<T>& r, V3<T> a, V3<T> b) {
  r.m[0][0] += a.x * b.x; r.m[0][1] += a.x * b.y; r.m[0][2] += a.x * b.z;
  r.m[1][0] += a.y * b.x; r.m[1][1] += a.y * b.y; r.m[1][2] += a.y * b.z;
  r.m[2][0] += a.z * b.x; r.m[2][1] += a.z * b.y; r.m[2][2] += a.z * b.z;
}
template <class T> TL_HD V3<T> row(const M3<T>& a, int i) { return {a.m[i][0], a.m[i][1], a.m[i][2]}; }

// J - 1 from H = F - I without forming 1 + ... (neohookean.cc:41-47).
template <class T> TL_HD T volumeChange(const M3<T>& h) {
  const T tr = trace3(h);
  const T hh = h.m[0][0] * h.m[0][0] + h.m[1][1] * h.m[1][1] + h.m[2][2] * h.m[2][2] +
               T(2) * (h.m[0][1] * h.m[1][0] + h.m[0][2] * h.m[2][0] + h.m[1][2] * h.m[2][1]);  // tr(H H)
  return tr + T(0.5) * (tr * tr - hh) + det3(h);
}

// Polar rotation by the Newton iteration R <- (R + R^-T)/2 from R = F with
// at most 24 passes and a 1e-6 max-entry stop, identity for |det F| < 1e-12
// (reference material.cc:20-22, 168-197).  R^-T = cof(R)/det(R).
template <class T> TL_HD M3<T> polarRotation(const M3<T>& f) {
  if (fabs(det3(f)) < T(1.0e-12)) return eye3<T>();
  M3<T> r = f;
  for (int pass = 0; pass < 24; ++pass) {
    const M3<T> c = cofactor(r);
    const T inv = T(1) / (r.m[0][0] * c.m[0][0] + r.m[0][1] * c.m[0][1] + r.m[0][2] * c.m[0][2]);
    T largest = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T next = T(0.5) * (r.m[i][j] + inv * c.m[i][j]);
        largest = fmax(largest, fabs(next - r.m[i][j]));
        r.m[i][j] = next;
      }
    if (largest < T(1.0e-6)) break;
  }
  return r;
}

// Rotation of an inverted element (det F <= 0) as the reference computes it
// from Eigen::JacobiSVD (material.cc:29-63): with singular pairs sorted by
// decreasing value, R = U' V'^T where U' = [u1 u2 u1xu2], V' = [v1 v2 v1xv2].
// The singular vectors come from a cyclic Jacobi eigen solve of F^T F
// (Golub & Van Loan, "Matrix Computations", sec. 8.5) in FP64.
TL_HD void jacobiEigen3(double a[3][3], double v[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) v[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1.0e-30 * diag || off == 0.0) break;
    for (int p = 0; p < 2; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
}

template <class T> TL_HD M3<T> invertibleRotation(const M3<T>& fin) {
  M3<double> f;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) f.m[i][j] = double(fin.m[i][j]);
  const M3<double> ftf = mul(transpose(f), f);
  double a[3][3], v[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = ftf.m[i][j];
  jacobiEigen3(a, v);
  int o0 = 0, o1 = 1, o2 = 2, t;
  if (a[o1][o1] > a[o0][o0]) { t = o0; o0 = o1; o1 = t; }
  if (a[o2][o2] > a[o1][o1]) { t = o1; o1 = o2; o2 = t; }
  if (a[o1][o1] > a[o0][o0]) { t = o0; o0 = o1; o1 = t; }
  const V3<double> v1{v[0][o0], v[1][o0], v[2][o0]};
  const V3<double> v2{v[0][o1], v[1][o1], v[2][o1]};
  V3<double> u1 = mul(f, v1);
  const double n1 = sqrt(dot(u1, u1));
  if (!(n1 > 0.0)) return eye3<T>();
  u1 = (1.0 / n1) * u1;
  V3<double> u2 = mul(f, v2);
  u2 = u2 - dot(u1, u2) * u1;
  double n2 = sqrt(dot(u2, u2));
  if (!(n2 > 1.0e-300)) {
    const V3<double> axis = fabs(u1.x) < 0.9 ? V3<double>{1, 0, 0} : V3<double>{0, 1, 0};
    u2 = cross(u1, axis);
    n2 = sqrt(dot(u2, u2));
  }
  u2 = (1.0 / n2) * u2;
  const V3<double> u3 = cross(u1, u2), v3 = cross(v1, v2);
  const M3<double> turned = mul(transpose(M3<double>{{{u1.x, u1.y, u1.z}, {u2.x, u2.y, u2.z}, {u3.x, u3.y, u3.z}}}),
                                M3<double>{{{v1.x, v1.y, v1.z}, {v2.x, v2.y, v2.z}, {v3.x, v3.y, v3.z}}});
  M3<T> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = T(turned.m[i][j]);
  return r;
}

#ifdef __CUDACC__
// Out of line on the device: only inverted elements take this branch, and
// inlined it would hold its Jacobi arrays and registers in every element
// thread's frame.
static __device__ __noinline__ M3<double> invertibleRotationOutOfLine(M3<double> f) {
  return invertibleRotation(f);
}
#endif

// material.cc:24-27: polar unless the element is inverted and the caller
// asked for the invertible rotation.
template <class T> TL_HD M3<T> elementRotation(const M3<T>& f, bool invertible) {
  if (!invertible || det3(f) > T(0)) return polarRotation(f);
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same_v<T, double>) return invertibleRotationOutOfLine(f);
#endif
  return invertibleRotation(f);
}

// returnMap (plasticflow.cc:110-150) of one point, FP64 like the reference:
// the left stretch B = Fe Fe^T diagonalised by the cyclic Jacobi solve, log
// strains 0.5 log(lambda), deviator d, q = sqrt(3/2) 2 mu |d|; past the yield
// stress Fe <- V diag(exp(d (yield / q - 1))) V^T Fe.  False inside.
TL_HD bool henckyReturn(const M3<double>& fe, double shear, double yield, M3<double>& out,
                                    double& strain, double& trial) {
  double a[3][3], v[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      a[i][j] = fe.m[i][0] * fe.m[j][0] + fe.m[i][1] * fe.m[j][1] + fe.m[i][2] * fe.m[j][2];
  jacobiEigen3(a, v);
  if (!(fmin(a[0][0], fmin(a[1][1], a[2][2])) > 0.0)) return false;
  const double l[3] = {0.5 * log(a[0][0]), 0.5 * log(a[1][1]), 0.5 * log(a[2][2])};
  const double mean = (l[0] + l[1] + l[2]) / 3.0;
  const double d[3] = {l[0] - mean, l[1] - mean, l[2] - mean};
  const double size = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double stress = sqrt(1.5) * 2.0 * shear * size;
  if (!(stress > yield) || size <= 1.0e-15) return false;
  M3<double> c = zero3<double>();
#pragma unroll
  for (int k = 0; k < 3; ++k) addOuter(c, exp(d[k] * (yield / stress - 1.0)) * V3<double>{v[0][k], v[1][k], v[2][k]},
                                       V3<double>{v[0][k], v[1][k], v[2][k]});
  out = mul(c, fe);
  trial = stress;
  strain = (stress - yield) / (3.0 * shear);
  return true;
}

}  // namespace tl
