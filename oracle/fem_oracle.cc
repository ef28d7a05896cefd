// fem_oracle.cc -- CPU restatement of the Talus tet FEM step.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py, for comparison.  The product (talus_b200)
// never links or calls it.
//
// Every function names the reference lines it restates.  Paths are relative
// to the reference project (d-adel/talus).  Arithmetic is templated on the
// scalar type: float reproduces the reference's glm float arithmetic, double
// is the FP64 oracle.  Small 3-vector / 3x3 types are written here (glm is
// not available); matrices are column-major like glm (m.c[column][row]).
//
// Parity: pinned by known-answer tests restated from the reference's law
// tests; the glm::inverse and Eigen::JacobiSVD call sites are restated from
// their mathematics (adjugate / determinant; a cyclic Jacobi eigen solve of
// F^T F) and are "parity unpinned" against the real libraries.

#include "fem_oracle.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

// A caller-held solver state (DeformableSolverState, factor.h:205-210): the
// system factor (SystemFactor::Held, factor.cc:302-314), its FactorReference
// (factor.h:20-26) and SolverStats (factor.h:28-38).  The reference factors
// with Eigen's SimplicialLLT under an AMD ordering; this restatement factors
// the same FP64 matrix in its natural order inside its envelope (the row
// profile), so L differs while L L^T, and so the applied inverse, agree to
// rounding.
struct or_solver {
  uint32_t budget = 32u;              // Settings::factorBudget (solver.h:54)
  uint32_t nodes = 0u;
  bool analyzed = false, ready = false;
  uint64_t born = 0u, systemNonZeros = 0u;
  std::vector<uint32_t> first;         // envelope: first column of each row
  std::vector<size_t> start;           // row offsets into env
  std::vector<double> env;             // L, row by row, from first[i] to i
  std::vector<uint8_t> anchored;
  std::vector<double> refPosition;     // FactorReference::positions [3 nodes]
  double refCentroid[3] = {0.0, 0.0, 0.0};
  double refStep = 0.0, refInertia = 1.0, refDamping = 0.0;  // FactorReference step, inertia, damping key
  or_solver_stats stats{};
  float meanIterations = 0.0f;         // SolverStats::meanIterations is a float
};

namespace {

// ---------------------------------------------------------------- math ----

template <class R>
struct V3 {
  R x{0}, y{0}, z{0};
  V3() = default;
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  V3& operator*=(R s) { x *= s; y *= s; z *= s; return *this; }
};
template <class R> V3<R> operator+(V3<R> a, const V3<R>& b) { return a += b; }
template <class R> V3<R> operator-(V3<R> a, const V3<R>& b) { return a -= b; }
template <class R> V3<R> operator-(const V3<R>& a) { return V3<R>(-a.x, -a.y, -a.z); }
template <class R> V3<R> operator*(R s, V3<R> a) { return a *= s; }
template <class R> R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> V3<R> cross(const V3<R>& a, const V3<R>& b) {
  return V3<R>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <class R> R length(const V3<R>& a) { return std::sqrt(dot(a, a)); }

template <class R>
struct M3 {
  V3<R> c[3];
  M3() = default;
  explicit M3(R d) { c[0] = V3<R>(d, 0, 0); c[1] = V3<R>(0, d, 0); c[2] = V3<R>(0, 0, d); }
  M3(const V3<R>& a, const V3<R>& b, const V3<R>& d) { c[0] = a; c[1] = b; c[2] = d; }
  V3<R>& operator[](int i) { return c[i]; }
  const V3<R>& operator[](int i) const { return c[i]; }
};
template <class R> M3<R> operator+(const M3<R>& a, const M3<R>& b) { return M3<R>(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <class R> M3<R> operator-(const M3<R>& a, const M3<R>& b) { return M3<R>(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <class R> M3<R> operator*(R s, const M3<R>& a) { return M3<R>(s * a[0], s * a[1], s * a[2]); }
template <class R> V3<R> operator*(const M3<R>& m, const V3<R>& v) {
  return V3<R>(m[0].x * v.x + m[1].x * v.y + m[2].x * v.z,
               m[0].y * v.x + m[1].y * v.y + m[2].y * v.z,
               m[0].z * v.x + m[1].z * v.y + m[2].z * v.z);
}
template <class R> M3<R> operator*(const M3<R>& a, const M3<R>& b) { return M3<R>(a * b[0], a * b[1], a * b[2]); }
template <class R> M3<R> transpose(const M3<R>& m) {
  return M3<R>(V3<R>(m[0].x, m[1].x, m[2].x), V3<R>(m[0].y, m[1].y, m[2].y), V3<R>(m[0].z, m[1].z, m[2].z));
}
template <class R> R determinant(const M3<R>& m) { return dot(m[0], cross(m[1], m[2])); }
// glm::inverse restated as adjugate / determinant (parity unpinned).
template <class R> M3<R> inverse(const M3<R>& m) {
  const R inv = R(1) / determinant(m);
  return transpose(M3<R>(inv * cross(m[1], m[2]), inv * cross(m[2], m[0]), inv * cross(m[0], m[1])));
}
// a * b^T (glm::outerProduct).
template <class R> M3<R> outer(const V3<R>& a, const V3<R>& b) { return M3<R>(b.x * a, b.y * a, b.z * a); }
template <class R> R traceOf(const M3<R>& m) { return m[0].x + m[1].y + m[2].z; }
template <class R> M3<R> deviatorOf(const M3<R>& m) { return m - (traceOf(m) / R(3)) * M3<R>(R(1)); }
template <class R> R contract(const M3<R>& a, const M3<R>& b) { return dot(a[0], b[0]) + dot(a[1], b[1]) + dot(a[2], b[2]); }
// neohookean.cc:19-25
template <class R> M3<R> cofactorOf(const M3<R>& m) { return M3<R>(cross(m[1], m[2]), cross(m[2], m[0]), cross(m[0], m[1])); }
// neohookean.cc:41-47 (J - 1 without forming 1 + ...)
template <class R> R volumeChange(const M3<R>& offset) {
  const R trace = traceOf(offset);
  return trace + R(0.5) * (trace * trace - contract(offset, transpose(offset))) + determinant(offset);
}

template <class R> M3<R> loadRowMajor(const double* a) {
  M3<R> m;
  for (int row = 0; row < 3; ++row)
    for (int col = 0; col < 3; ++col) m[col][row] = R(a[3 * row + col]);
  return m;
}
template <class R> void storeRowMajor(const M3<R>& m, double* a) {
  for (int row = 0; row < 3; ++row)
    for (int col = 0; col < 3; ++col) a[3 * row + col] = double(m[col][row]);
}

// ------------------------------------------------------------ element ----

template <class R> struct Lame { R first{0}, second{0}; };

// material.cc:71-78
template <class R> Lame<R> lame(R youngs, R poisson) {
  const R nu = std::clamp(poisson, R(0), R(0.49));
  return {youngs * nu / ((R(1) + nu) * (R(1) - R(2) * nu)), youngs / (R(2) * (R(1) + nu))};
}

constexpr uint32_t POLAR_ITERATIONS = 24u;     // material.cc:20
constexpr double POLAR_TOLERANCE = 1.0e-6;     // material.cc:22

// material.cc:168-197
template <class R> M3<R> polarRotation(const M3<R>& gradient) {
  if (std::abs(determinant(gradient)) < R(1.0e-12)) return M3<R>(R(1));
  M3<R> rotation = gradient;
  for (uint32_t pass = 0; pass != POLAR_ITERATIONS; ++pass) {
    const M3<R> next = R(0.5) * (rotation + transpose(inverse(rotation)));
    const M3<R> change = next - rotation;
    rotation = next;
    R largest = 0;
    for (int col = 0; col < 3; ++col)
      for (int row = 0; row < 3; ++row) largest = std::max(largest, std::abs(change[col][row]));
    if (largest < R(POLAR_TOLERANCE)) break;
  }
  return rotation;
}

// Eigen::JacobiSVD (material.cc:29-63) restated: cyclic Jacobi eigen
// decomposition of the symmetric F^T F (Golub & Van Loan, "Matrix
// Computations", sec. 8.5), singular vectors u_i = F v_i / |F v_i| with
// Gram-Schmidt, then the reference's determinant fix-up of U and V, which
// makes the result U' V'^T with U' = [u1 u2 u1xu2], V' = [v1 v2 v1xv2].
inline void jacobiEigen(double a[3][3], double v[3][3]) {
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
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0);
        const double s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- A J
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {  // A <- J^T A
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {  // V <- V J
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
}

template <class R> M3<R> invertibleRotation(const M3<R>& gradient) {
  M3<double> f;
  for (int c = 0; c < 3; ++c) f[c] = V3<double>(double(gradient[c].x), double(gradient[c].y), double(gradient[c].z));
  const M3<double> ftf = transpose(f) * f;
  double a[3][3], v[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = ftf[j][i];
  jacobiEigen(a, v);
  int order[3] = {0, 1, 2};
  std::sort(order, order + 3, [&](int l, int r) { return a[l][l] > a[r][r]; });
  V3<double> v1(v[0][order[0]], v[1][order[0]], v[2][order[0]]);
  V3<double> v2(v[0][order[1]], v[1][order[1]], v[2][order[1]]);
  V3<double> u1 = f * v1;
  double n1 = length(u1);
  if (!(n1 > 0.0)) return M3<R>(R(1));
  u1 = (1.0 / n1) * u1;
  V3<double> u2 = f * v2;
  u2 -= dot(u1, u2) * u1;
  double n2 = length(u2);
  if (!(n2 > 1.0e-300)) {  // rank-1 gradient: any unit vector orthogonal to u1
    const V3<double> axis = std::abs(u1.x) < 0.9 ? V3<double>(1, 0, 0) : V3<double>(0, 1, 0);
    u2 = cross(u1, axis);
    n2 = length(u2);
  }
  u2 = (1.0 / n2) * u2;
  const M3<double> left(u1, u2, cross(u1, u2));
  const M3<double> right(v1, v2, cross(v1, v2));
  const M3<double> turned = left * transpose(right);
  M3<R> out;
  for (int c = 0; c < 3; ++c) out[c] = V3<R>(R(turned[c].x), R(turned[c].y), R(turned[c].z));
  return out;
}

// ------------------------------------------------- finite-strain flow ----
// plasticflow.cc:96-150 returnMap, FP64 like the reference.  The left stretch
// B = F_e F_e^T (leftStretch, plasticflow.cc:22-38) is diagonalised by the
// cyclic Jacobi solve above (Eigen::SelfAdjointEigenSolver in the reference;
// the spectral function V f(L) V^T built from it does not depend on the order
// or the signs of the eigenvectors).  Log strains 0.5 log(lambda_i), their
// deviator d, q = sqrt(3/2) 2 mu |d|; past the yield stress the deviator is
// scaled back by exp(d_i (yield / q - 1)) along the eigenvectors.
struct HenckyReturn {
  M3<double> elastic{1.0};
  double strain = 0.0, trial = 0.0;
  bool mapped = false;
};

// Log-strain deviator of F_e and the eigenvectors it is expressed in; false
// when B is not positive definite.
inline bool henckyDeviator(const M3<double>& fe, double dev[3], double vec[3][3], double& size) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = fe[0][i] * fe[0][j] + fe[1][i] * fe[1][j] + fe[2][i] * fe[2][j];
  jacobiEigen(a, vec);
  const double lo = std::min(a[0][0], std::min(a[1][1], a[2][2]));
  if (!(lo > 0.0)) return false;
  const double strain[3] = {0.5 * std::log(a[0][0]), 0.5 * std::log(a[1][1]), 0.5 * std::log(a[2][2])};
  const double mean = (strain[0] + strain[1] + strain[2]) / 3.0;
  for (int i = 0; i < 3; ++i) dev[i] = strain[i] - mean;
  size = std::sqrt(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]);
  return true;
}

// plasticflow.cc:96-108
inline double henckyVonMises(const M3<double>& fe, double shear) {
  double dev[3], vec[3][3], size = 0.0;
  if (!henckyDeviator(fe, dev, vec, size)) return 0.0;
  return std::sqrt(1.5) * 2.0 * shear * size;
}

// plasticflow.cc:110-150
inline HenckyReturn henckyReturn(const M3<double>& fe, double shear, double yieldStress) {
  HenckyReturn out;
  double dev[3], vec[3][3], size = 0.0;
  if (!henckyDeviator(fe, dev, vec, size)) return out;
  const double stress = std::sqrt(1.5) * 2.0 * shear * size;
  if (!(stress > yieldStress) || size <= 1.0e-15) return out;
  M3<double> correction(0.0);
  for (int k = 0; k < 3; ++k) {
    const double scale = std::exp(dev[k] * (yieldStress / stress - 1.0));
    const V3<double> v(vec[0][k], vec[1][k], vec[2][k]);
    correction = correction + scale * outer(v, v);
  }
  out.elastic = correction * fe;
  out.trial = stress;
  out.strain = (stress - yieldStress) / (3.0 * shear);
  out.mapped = true;
  return out;
}

inline double oneNorm(const M3<double>& m) {
  double total = 0.0;
  for (int c = 0; c < 3; ++c) total += std::abs(m[c].x) + std::abs(m[c].y) + std::abs(m[c].z);
  return total;
}

inline double frobenius(const M3<double>& m) {
  return std::sqrt(dot(m[0], m[0]) + dot(m[1], m[1]) + dot(m[2], m[2]));
}

struct FlowLimits {
  double crushStress = std::numeric_limits<double>::infinity(), crushLimit = 1.0;
  double plasticMax = std::numeric_limits<double>::infinity();
};

// plasticflow.cc:184-247 flowLattice at one point.  The elastic map F P
// returns with the yield stress blended toward the trial stress,
// (start + r q) / (1 + r), r = H / (3 mu).  A crushable material
// (finite crushStress, crushLimit < 1) squeezed below J = exp(-crushStress /
// K) compacts by min(-crush - log J, room), room = -log(det P crushLimit).
// The plastic map becomes F^-1 (grow F_e,returned); a plastic stretch Fp
// further than plasticMax from I (Frobenius) is pulled back to that distance
// at the same volume.  The hardening variable grows by the returned strain.
inline bool henckyFlow(const M3<double>& deformation, M3<double>& plastic, double& hardening, double shear,
                       double bulk, double yieldStress, double hardeningModulus, const FlowLimits& limits) {
  if (!(determinant(deformation) > 0.0)) return false;
  const M3<double> elastic = deformation * plastic;
  const double ratio = hardeningModulus / (3.0 * shear);
  const bool crushable = std::isfinite(limits.crushStress) && limits.crushLimit < 1.0;
  const double crush = limits.crushStress / bulk;
  const double start = yieldStress + hardeningModulus * hardening;
  const double room = crushable ? -std::log(determinant(plastic) * limits.crushLimit) : 0.0;
  const bool squeezed = crushable && room > 0.0 && determinant(elastic) < std::exp(-crush);
  const HenckyReturn trial = henckyReturn(elastic, shear, start);
  const double yieldNow = trial.mapped ? (start + ratio * trial.trial) / (1.0 + ratio) : start;
  const HenckyReturn mapped = trial.mapped ? henckyReturn(elastic, shear, yieldNow) : HenckyReturn{};
  const M3<double> after = mapped.mapped ? mapped.elastic : elastic;
  const double volume = determinant(after);
  const double compaction = squeezed && volume > 0.0 ? std::min(-crush - std::log(volume), room) : 0.0;
  if (!mapped.mapped && !(compaction > 0.0)) return false;
  const double grow = compaction > 0.0 ? std::exp(compaction / 3.0) : 1.0;
  M3<double> next = inverse(deformation) * (grow * after);
  const double kept = determinant(next);
  if (std::isfinite(limits.plasticMax) && kept > 0.0) {
    const M3<double> stretch = inverse(next) - M3<double>(1.0);
    const double size = frobenius(stretch);
    if (size > limits.plasticMax) {
      const M3<double> capped = M3<double>(1.0) + (limits.plasticMax / size) * stretch;
      const double cappedVolume = determinant(capped);
      if (!(cappedVolume > 1.0e-6)) return false;
      next = std::cbrt(kept * cappedVolume) * inverse(capped);
    }
  }
  if (!(oneNorm(next - plastic) > 1.0e-12)) return false;
  plastic = next;
  hardening += mapped.mapped ? mapped.strain : 0.0;
  return true;
}

// material.cc:24-27
template <class R> M3<R> elementRotation(const M3<R>& gradient, int mode) {
  if (mode == OR_ROTATION_POLAR || determinant(gradient) > R(0)) return polarRotation(gradient);
  return invertibleRotation(gradient);
}

// material.cc:199-207
template <class R> std::array<V3<R>, 4> shapeGradients(const M3<R>& restInverse) {
  const M3<R> rows = transpose(restInverse);
  return {-(rows[0] + rows[1] + rows[2]), rows[0], rows[1], rows[2]};
}

template <class R> struct TetStiffness {
  std::array<M3<R>, 16> block{};
  std::array<V3<R>, 4> gradient{};
  R first{0}, second{0};
};

// material.cc:80-90
template <class R> M3<R> stiffnessBlock(const V3<R>& a, const V3<R>& b, const Lame<R>& moduli, R volume) {
  return volume * (moduli.first * outer(a, b) + moduli.second * outer(b, a) + (moduli.second * dot(a, b)) * M3<R>(R(1)));
}

// material.cc:209-234
template <class R> TetStiffness<R> tetStiffness(const M3<R>& restInverse, R volume, const Lame<R>& moduli) {
  TetStiffness<R> k;
  k.gradient = shapeGradients(restInverse);
  k.first = moduli.first;
  k.second = moduli.second;
  for (int row = 0; row < 4; ++row)
    for (int col = 0; col < 4; ++col) k.block[row * 4 + col] = stiffnessBlock(k.gradient[row], k.gradient[col], moduli, volume);
  return k;
}


// material.cc:92-109
template <class R>
std::array<V3<R>, 4> corotatedOffsets(const std::array<V3<R>, 4>& d, const std::array<V3<R>, 4>& r, const M3<R>& rotation) {
  const M3<R> inv = transpose(rotation);
  const V3<R> dc = R(0.25) * (d[0] + d[1] + d[2] + d[3]);
  const V3<R> rc = R(0.25) * (r[0] + r[1] + r[2] + r[3]);
  return {inv * (d[0] - dc) - (r[0] - rc), inv * (d[1] - dc) - (r[1] - rc), inv * (d[2] - dc) - (r[2] - rc),
          inv * (d[3] - dc) - (r[3] - rc)};
}

template <class R> struct TetStrain { M3<R> rotation{R(1)}; std::array<V3<R>, 4> offsets{}; M3<R> strain{}; };

template <class R> M3<R> deformationOf(const std::array<V3<R>, 4>& d, const M3<R>& restInverse) {
  return M3<R>(d[1] - d[0], d[2] - d[0], d[3] - d[0]) * restInverse;
}

// material.cc:136-164
template <class R>
TetStrain<R> tetStrain(const std::array<V3<R>, 4>& d, const std::array<V3<R>, 4>& r, const M3<R>& restInverse,
                       const std::array<V3<R>, 4>& gradient, int mode) {
  TetStrain<R> m;
  m.rotation = elementRotation(deformationOf(d, restInverse), mode);
  m.offsets = corotatedOffsets(d, r, m.rotation);
  M3<R> displacement(R(0));
  for (int n = 0; n < 4; ++n) displacement = displacement + outer(m.offsets[n], gradient[n]);
  m.strain = R(0.5) * (displacement + transpose(displacement));
  return m;
}

template <class R> struct TrialState { M3<R> rotation{R(1)}; std::array<V3<R>, 4> force{}; R energy{0}; };

// material.cc:111-127, 236-265
template <class R>
TrialState<R> trial(const std::array<V3<R>, 4>& d, const std::array<V3<R>, 4>& r, const M3<R>& restInverse,
                    const TetStiffness<R>& k, int mode) {
  TrialState<R> s;
  const TetStrain<R> m = tetStrain(d, r, restInverse, k.gradient, mode);
  s.rotation = m.rotation;
  for (int row = 0; row < 4; ++row) {
    V3<R> sum;
    for (int col = 0; col < 4; ++col) sum += k.block[row * 4 + col] * m.offsets[col];
    s.energy += R(0.5) * dot(m.offsets[row], sum);
    s.force[row] = s.rotation * (-sum);
  }
  return s;
}

// material.cc:267-288
template <class R>
void applyStiffness(const std::array<V3<R>, 4>& direction, const M3<R>& rotation, const TetStiffness<R>& k,
                    std::array<V3<R>, 4>& result) {
  const M3<R> inv = transpose(rotation);
  std::array<V3<R>, 4> un;
  for (int n = 0; n < 4; ++n) un[n] = inv * direction[n];
  for (int row = 0; row < 4; ++row) {
    V3<R> sum;
    for (int col = 0; col < 4; ++col) sum += k.block[row * 4 + col] * un[col];
    result[row] = rotation * sum;
  }
}

// material.cc:290-304
template <class R> std::array<M3<R>, 4> stiffnessDiagonal(const TetStiffness<R>& k, const M3<R>& rotation) {
  std::array<M3<R>, 4> out;
  const M3<R> inv = transpose(rotation);
  for (int n = 0; n < 4; ++n) out[n] = rotation * k.block[n * 4 + n] * inv;
  return out;
}

template <class R> struct PlasticPoint { M3<R> strain{R(0)}; R equivalent{0}; };

template <class R> struct PointLaw { R bulk{0}, shear{0}, yield{0}, hardening{0}; };

template <class R> struct PointResponse {
  M3<R> stress{R(0)}, normal{R(0)};
  R theta{1}, thetaBar{0}, plasticWork{0}, excess{0};
  bool plastic = false;
  PlasticPoint<R> next{};
};

// material.cc:594-634
template <class R>
PointResponse<R> returnMap(const M3<R>& strain, const PlasticPoint<R>& committed, const PointLaw<R>& law, bool mapping) {
  PointResponse<R> r;
  r.next = committed;
  const M3<R> elastic = strain - committed.strain;
  const R pressure = law.bulk * traceOf(elastic);
  const M3<R> trialStress = (R(2) * law.shear) * deviatorOf(elastic);
  const R norm = std::sqrt(contract(trialStress, trialStress));
  const R equivalent = std::sqrt(R(1.5)) * norm;
  const R radius = law.yield + law.hardening * committed.equivalent;
  if (!mapping || !(equivalent > radius) || !(norm > R(0))) {
    r.stress = trialStress + pressure * M3<R>(R(1));
    return r;
  }
  const R gamma = (equivalent - radius) / (R(3) * law.shear + law.hardening);
  const M3<R> normal = (R(1) / norm) * trialStress;
  const R theta = R(1) - R(3) * law.shear * gamma / equivalent;
  r.stress = theta * trialStress + pressure * M3<R>(R(1));
  r.normal = normal;
  r.theta = theta;
  r.thetaBar = R(3) * law.shear / (R(3) * law.shear + law.hardening) - (R(1) - theta);
  r.plasticWork = (radius + law.hardening * gamma) * gamma;
  r.excess = (equivalent - radius) / radius;
  r.plastic = true;
  r.next.strain = committed.strain + (std::sqrt(R(1.5)) * gamma) * normal;
  r.next.equivalent = committed.equivalent + gamma;
  return r;
}

// material.cc:636-650
template <class R> M3<R> tangentOf(const PointResponse<R>& r, const PointLaw<R>& law, const M3<R>& strain) {
  M3<R> stress = (law.bulk * traceOf(strain)) * M3<R>(R(1)) + (R(2) * law.shear * r.theta) * deviatorOf(strain);
  if (r.plastic) stress = stress - (R(2) * law.shear * r.thetaBar * contract(r.normal, strain)) * r.normal;
  return stress;
}

// material.cc:652-672
template <class R> V3<R> pointForce(const M3<R>& deviator, R mean, const V3<R>& gradient, const V3<R>& centre) {
  return deviator * gradient + mean * centre;
}
template <class R> M3<R> unitStrain(int axis, const V3<R>& gradient, const V3<R>& centre) {
  V3<R> direction;
  direction[axis] = R(1);
  const M3<R> displacement = outer(direction, gradient);
  return deviatorOf(R(0.5) * (displacement + transpose(displacement))) + (centre[axis] / R(3)) * M3<R>(R(1));
}

template <class R> bool yieldsAt(R yieldStress) { return std::isfinite(yieldStress) && yieldStress > R(0); }

// material.cc:675-683
template <class R> PointLaw<R> pointLaw(const Lame<R>& m, R yieldStress, R hardening) {
  return {m.first + R(2) * m.second / R(3), m.second,
          yieldsAt(yieldStress) ? yieldStress : std::numeric_limits<R>::infinity(), std::max(hardening, R(0))};
}

template <class R> struct TetPointTrial {
  M3<R> rotation{R(1)};
  std::array<V3<R>, 4> force{};
  PlasticPoint<R> point{};
  TetStiffness<R> tangent{};
  R energy{0}, plasticWork{0};
  uint32_t yielding = 0, loading = 0;
};

// material.cc:978-1057
template <class R>
TetPointTrial<R> tetPointTrial(const std::array<V3<R>, 4>& d, const std::array<V3<R>, 4>& r, const M3<R>& restInverse,
                               R volume, const Lame<R>& moduli, R yieldStress, R hardening,
                               const PlasticPoint<R>& committed, R margin, int mode, bool mapping, bool tangent) {
  TetPointTrial<R> made;
  const std::array<V3<R>, 4> gradient = shapeGradients(restInverse);
  made.tangent.gradient = gradient;
  made.tangent.first = moduli.first;
  made.tangent.second = moduli.second;
  const TetStrain<R> measured = tetStrain(d, r, restInverse, gradient, mode);
  const PointLaw<R> law = pointLaw(moduli, yieldStress, hardening);
  const PointResponse<R> response = returnMap(measured.strain, committed, law, mapping);
  made.rotation = measured.rotation;
  made.point = response.next;
  made.energy = volume * R(0.5) * contract(response.stress, measured.strain - response.next.strain);
  made.plasticWork = volume * response.plasticWork;
  made.yielding = response.plastic ? 1u : 0u;
  const bool loading = response.plastic && response.excess > margin;
  made.loading = loading ? 1u : 0u;
  const PointResponse<R> linearized = loading || !response.plastic ? response : PointResponse<R>{};
  const M3<R> dev = deviatorOf(response.stress);
  const R mean = traceOf(response.stress) / R(3);
  for (int row = 0; row < 4; ++row) made.force[row] = -(made.rotation * (volume * pointForce(dev, mean, gradient[row], gradient[row])));
  if (!tangent) return made;
  for (int col = 0; col < 4; ++col) {
    for (int axis = 0; axis < 3; ++axis) {
      const M3<R> stress = tangentOf(linearized, law, unitStrain(axis, gradient[col], gradient[col]));
      const M3<R> tdev = deviatorOf(stress);
      const R tmean = traceOf(stress) / R(3);
      for (int row = 0; row < 4; ++row)
        made.tangent.block[row * 4 + col][axis] = volume * pointForce(tdev, tmean, gradient[row], gradient[row]);
    }
  }
  return made;
}

// Stable neo-Hookean law at one point of a tet.  Stress restated from the
// reference's FP32 hex law (material.cc:925-931, the cancellation-free form
// of neohookean.cc:183-184 P = mu (F - cof F) + (lambda + mu)(J - 1) cof F),
// energy from neohookean.cc:141-144.  The tangent is the exact differential
// dP = mu dF + ((lambda + mu)(J - 1) - mu) dcof + (lambda + mu)(cof : dF) cof;
// its diagonal node blocks reduce to the reference's node Hessian
// mu |g|^2 I + (lambda + mu) b b^T, b = cof g (neohookean.cc:186-192), because
// dcof[e_i g^T] g = 0.
template <class R> struct SnhTet {
  std::array<V3<R>, 4> force{};
  M3<R> gradient{R(1)};  // F = I + H
  R change{0};           // J - 1
  R energy{0};
};

template <class R>
SnhTet<R> snhTet(const std::array<V3<R>, 4>& d, const std::array<V3<R>, 4>& r, const M3<R>& restInverse, R volume,
                 const Lame<R>& moduli) {
  SnhTet<R> out;
  const std::array<V3<R>, 4> g = shapeGradients(restInverse);
  M3<R> offset(R(0));
  for (int n = 0; n < 4; ++n) offset = offset + outer(d[n] - r[n], g[n]);
  const R shear = moduli.second;
  const R shifted = moduli.first + moduli.second;
  const R change = volumeChange(offset);
  const M3<R> cofactor = cofactorOf(M3<R>(R(1)) + offset);
  const M3<R> stress = shear * (offset + transpose(offset) - traceOf(offset) * M3<R>(R(1)) - cofactorOf(offset)) +
                       (shifted * change) * cofactor;
  const R squared = contract(offset, offset);
  const R quadratic = change - traceOf(offset);
  out.energy = volume * (R(0.5) * shear * squared - shear * quadratic + R(0.5) * shifted * change * change);
  for (int n = 0; n < 4; ++n) out.force[n] = -(volume * (stress * g[n]));
  out.gradient = M3<R>(R(1)) + offset;
  out.change = change;
  return out;
}

// d cof(F) [dF]: column k of cof is F_{k+1} x F_{k+2} (neohookean.cc:19-25).
template <class R> M3<R> cofactorDifferential(const M3<R>& f, const M3<R>& df) {
  return M3<R>(cross(df[1], f[2]) + cross(f[1], df[2]), cross(df[2], f[0]) + cross(f[2], df[0]),
               cross(df[0], f[1]) + cross(f[0], df[1]));
}

// +K p for one tet: out_a = V dP(sum_b p_b g_b^T) g_a.
template <class R>
void snhApply(const std::array<V3<R>, 4>& p, const M3<R>& restInverse, R volume, const Lame<R>& m, const M3<R>& f,
              R change, std::array<V3<R>, 4>& out) {
  const std::array<V3<R>, 4> g = shapeGradients(restInverse);
  M3<R> df(R(0));
  for (int n = 0; n < 4; ++n) df = df + outer(p[n], g[n]);
  const M3<R> cof = cofactorOf(f);
  const R shifted = m.first + m.second;
  const M3<R> dp = m.second * df + (shifted * change - m.second) * cofactorDifferential(f, df) +
                   (shifted * contract(cof, df)) * cof;
  for (int n = 0; n < 4; ++n) out[n] = volume * (dp * g[n]);
}

// Diagonal node block, neohookean.cc:189-192 at one point of weight V.
template <class R> M3<R> snhDiagonal(const V3<R>& g, const M3<R>& f, R volume, const Lame<R>& m) {
  const V3<R> b = cofactorOf(f) * g;
  return volume * ((m.second * dot(g, g)) * M3<R>(R(1)) + (m.first + m.second) * outer(b, b));
}

// ------------------------------------------------------------- solver ----

// ----------------------------------------------------------- damping ----
// Stiffness damping (factor.cc:755-855, 183-272, 274-298; solver.cc:625-902):
// per element with weight tau > 0, D(p) = P_rigid^perp R K R^T P_rigid^perp p,
// where the projection removes the rigid motion fitted to the corners.

// factor.cc:183-272: symmetric 3x3 pseudo-inverse by cyclic Jacobi rotations,
// keeping the eigenvalues above `floor`.
inline M3<double> pseudoInverse(const M3<double>& held, double floor) {
  double reduced[3][3], basis[3][3];
  for (int row = 0; row < 3; ++row)
    for (int col = 0; col < 3; ++col) {
      reduced[row][col] = held[col][row];
      basis[row][col] = row == col ? 1.0 : 0.0;
    }
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, size = 0.0;
    for (int row = 0; row < 3; ++row) {
      size += reduced[row][row] * reduced[row][row];
      for (int col = row + 1; col < 3; ++col) off += reduced[row][col] * reduced[row][col];
    }
    if (!(off > 1.0e-30 * size)) break;
    for (const auto& pr : pairs) {
      const int p = pr[0], q = pr[1];
      if (reduced[p][q] == 0.0) continue;
      const double theta = (reduced[q][q] - reduced[p][p]) / (2.0 * reduced[p][q]);
      const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
      const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
      for (int k = 0; k < 3; ++k) {
        const double a = reduced[k][p], b = reduced[k][q];
        reduced[k][p] = c * a - sn * b;
        reduced[k][q] = sn * a + c * b;
      }
      for (int k = 0; k < 3; ++k) {
        const double a = reduced[p][k], b = reduced[q][k];
        reduced[p][k] = c * a - sn * b;
        reduced[q][k] = sn * a + c * b;
      }
      for (int k = 0; k < 3; ++k) {
        const double a = basis[k][p], b = basis[k][q];
        basis[k][p] = c * a - sn * b;
        basis[k][q] = sn * a + c * b;
      }
    }
  }
  M3<double> made(0.0);
  for (int axis = 0; axis < 3; ++axis) {
    const double value = reduced[axis][axis];
    if (!(value > floor)) continue;
    for (int row = 0; row < 3; ++row)
      for (int col = 0; col < 3; ++col) made[col][row] += basis[row][axis] * basis[col][axis] / value;
  }
  return made;
}

template <class R> struct RigidFit { std::array<V3<R>, 4> arms{}; M3<R> inverse{R(0)}; };

// factor.cc:780-817: arms from the centroid, inverse of the inertia tensor
// sum |a|^2 I - a a^T (pseudo-inverse when it is near singular), in FP64.
template <class R> RigidFit<R> rigidFit(const std::array<V3<R>, 4>& corners) {
  RigidFit<R> fit;
  V3<double> centre;
  for (const V3<R>& c : corners) centre += V3<double>(double(c.x), double(c.y), double(c.z));
  centre = (1.0 / 4.0) * centre;
  M3<double> inertia(0.0);
  for (int k = 0; k < 4; ++k) {
    const V3<double> d = V3<double>(double(corners[k].x), double(corners[k].y), double(corners[k].z)) - centre;
    fit.arms[k] = V3<R>(R(d.x), R(d.y), R(d.z));
    const V3<double> a(double(fit.arms[k].x), double(fit.arms[k].y), double(fit.arms[k].z));
    inertia = inertia + (dot(a, a) * M3<double>(1.0) - outer(a, a));
  }
  const double third = (inertia[0][0] + inertia[1][1] + inertia[2][2]) / 3.0;
  const M3<double> inv = determinant(inertia) > 1.0e-6 * third * third * third ? inverse(inertia)
                                                                                 : pseudoInverse(inertia, 1.0e-6 * third);
  for (int col = 0; col < 3; ++col) fit.inverse[col] = V3<R>(R(inv[col].x), R(inv[col].y), R(inv[col].z));
  return fit;
}

// factor.cc:819-841
template <class R> void removeRigid(const RigidFit<R>& fit, std::array<V3<R>, 4>& values) {
  V3<R> mean, moment;
  for (int k = 0; k < 4; ++k) {
    mean += values[k];
    moment += cross(fit.arms[k], values[k]);
  }
  mean = (R(1) / R(4)) * mean;
  const V3<R> spin = fit.inverse * moment;
  for (int k = 0; k < 4; ++k) values[k] -= mean + cross(spin, fit.arms[k]);
}

// factor.cc:843-853
template <class R>
void applyDamping(const RigidFit<R>& fit, const M3<R>& rotation, const TetStiffness<R>& k,
                  const std::array<V3<R>, 4>& direction, std::array<V3<R>, 4>& result) {
  std::array<V3<R>, 4> relative = direction;
  removeRigid(fit, relative);
  applyStiffness(relative, rotation, k, result);
  removeRigid(fit, result);
}

// factor.cc:274-298, 1041-1047: the diagonal corner blocks of D (columns from
// unit directions).
template <class R>
std::array<M3<R>, 4> dampingDiagonal(const RigidFit<R>& fit, const M3<R>& rotation, const TetStiffness<R>& k) {
  std::array<M3<R>, 4> out;
  std::array<V3<R>, 4> unit, column;
  for (int corner = 0; corner < 4; ++corner)
    for (int axis = 0; axis < 3; ++axis) {
      unit.fill(V3<R>());
      unit[corner][axis] = R(1);
      applyDamping(fit, rotation, k, unit, column);
      out[corner][axis] = column[corner];
    }
  return out;
}

// solver.cc:531-566
template <class R> struct IntegratorRule { R alphaMass{0}, alphaForce{0}, beta{0.25}, gamma{0.5}; };
template <class R> IntegratorRule<R> integratorRule(R spectral) {
  const R held = std::clamp(spectral, R(0), R(1));
  IntegratorRule<R> m;
  m.alphaMass = (R(2) * held - R(1)) / (held + R(1));
  m.alphaForce = held / (held + R(1));
  m.gamma = R(0.5) - m.alphaMass + m.alphaForce;
  m.beta = R(0.25) * (R(1) - m.alphaMass + m.alphaForce) * (R(1) - m.alphaMass + m.alphaForce);
  return m;
}
template <class R> struct EffectiveSystem { R inertia{1}, step{0}, mobility{1}; };
template <class R> EffectiveSystem<R> effectiveSystem(const IntegratorRule<R>& rule, R step) {
  return {R(1) - rule.alphaMass, std::sqrt((R(1) - rule.alphaForce) * rule.beta) * step, rule.beta};
}

constexpr uint32_t ANCHORED_READS = 3u;      // solver.cc:11
constexpr uint32_t INVERTED_SUBSTEPS = 4u;   // solver.cc:13
constexpr double LOADING_MARGIN = 1.0e-3;    // solver.cc:372
constexpr double PLASTIC_REDUCTION = 1.0e-2; // solver.cc:374
constexpr float PLASTIC_RESOLUTION = 8.0f;   // solver.cc:380

template <class R> struct Element {
  uint32_t nodes[4];
  M3<R> restInverse;
  R volume;
  Lame<R> moduli;
  R yieldStress, hardening;
  bool yields;
  R tau;  // stiffness damping weight (factor.cc:755-759)
  FlowLimits limits;  // finite-strain flow: crush and plastic cap
};

// ----------------------------------------------------- system factor ----

// L L^T x = b in place, with L in its envelope (the solve of applyFactor,
// factor.cc:690).
inline void envelopeSolve(const or_solver& f, std::vector<double>& b) {
  const size_t n = f.first.size();
  for (size_t i = 0; i < n; ++i) {
    const double* row = &f.env[f.start[i]] - f.first[i];
    double sum = b[i];
    for (size_t k = f.first[i]; k < i; ++k) sum -= row[k] * b[k];
    b[i] = sum / row[i];
  }
  for (size_t i = n; i-- > 0;) {
    const double* row = &f.env[f.start[i]] - f.first[i];
    b[i] /= row[i];
    for (size_t k = f.first[i]; k < i; ++k) b[k] -= row[k] * b[i];
  }
}

// factor.cc:669-704 applyFactor: turned into the factor's frame, packed to
// FP64, solved, unpacked in the arithmetic of the step, turned back, anchored
// nodes zero.
template <class R>
void applyFactor(const or_solver& f, const M3<R>& frame, std::vector<V3<R>>& vector) {
  const M3<R> inverse = transpose(frame);
  std::vector<double> packed(size_t(3) * f.nodes);
  for (uint32_t n = 0; n < f.nodes; ++n) {
    const V3<R> turned = inverse * vector[n];
    packed[3 * n] = double(turned.x);
    packed[3 * n + 1] = double(turned.y);
    packed[3 * n + 2] = double(turned.z);
  }
  envelopeSolve(f, packed);
  for (uint32_t n = 0; n < f.nodes; ++n) {
    const V3<R> raw(R(packed[3 * n]), R(packed[3 * n + 1]), R(packed[3 * n + 2]));
    vector[n] = f.anchored[n] != 0u ? V3<R>() : frame * raw;
  }
}

// factor.cc:638-667 bodyRotation: the polar rotation of the mass-weighted
// correlation of the positions now with those the factor was made at.
template <class R>
M3<R> bodyRotation(const std::vector<R>& mass, const std::vector<V3<R>>& position, const or_solver& f) {
  if (f.refPosition.size() != size_t(3) * position.size()) return M3<R>(R(1));
  V3<R> centre;
  R total = 0;
  for (size_t n = 0; n < position.size(); ++n) {
    total += mass[n];
    centre += mass[n] * position[n];
  }
  if (total > R(0)) centre = V3<R>(centre.x / total, centre.y / total, centre.z / total);
  const V3<R> before0(R(f.refCentroid[0]), R(f.refCentroid[1]), R(f.refCentroid[2]));
  M3<R> correlation(R(0));
  for (size_t n = 0; n < position.size(); ++n) {
    const V3<R> now = position[n] - centre;
    const V3<R> before = V3<R>(R(f.refPosition[3 * n]), R(f.refPosition[3 * n + 1]), R(f.refPosition[3 * n + 2])) - before0;
    correlation = correlation + mass[n] * outer(now, before);
  }
  return polarRotation(correlation);
}

template <class R> struct Solver {
  // inputs
  uint32_t V = 0, T = 0;
  std::vector<V3<R>> rest;
  std::vector<R> mass;
  std::vector<uint8_t> anchored;
  std::vector<V3<R>> prescribed;
  std::vector<Element<R>> elements;
  std::vector<TetStiffness<R>> store;    // ElementStiffness::tet (solver.cc:453-507)
  std::vector<TetStiffness<R>> working;  // Scratch::tetWorking
  bool consistent = false;               // scratch.stiffness == tetWorking
  int law = OR_LAW_COROTATED;
  // state
  std::vector<V3<R>> position, velocity, acceleration;
  std::vector<M3<R>> rotation;
  std::vector<PlasticPoint<R>> plastic;
  std::vector<RigidFit<R>> fits;         // Damping::fits at the last assemble
  bool damped = false;
  R dampScale{0};                        // Damping::scale = (1 - alpha_f) gamma h (solver.cc:3590)
  // finite-strain flow (OR_PLASTICITY_HENCKY): Dm^-1 as given, the plastic
  // map P = Fp^-1 and hardening variable per tet, and the corners of each
  // tet's plastic rest shape Dm' = Fp Dm (plasticRest, plasticflow.cc:263-300)
  bool hencky = false;
  std::vector<M3<double>> authored, flowMap;
  std::vector<double> hardeningOf;
  std::vector<std::array<V3<R>, 4>> plasticCorners;
  std::vector<M3<R>> snhGradient;        // SNH operator state: F per tet
  std::vector<R> snhChange;              // SNH operator state: J - 1 per tet
  // scratch (solver.cc:395-420)
  std::vector<V3<R>> force, right, residual, direction, applied, conditioned, increment, restart, shifted, weighted,
      carried, evaluated, total, lowestIterate, drive;
  std::vector<M3<R>> diagonal, preconditioner;
  or_report* report = nullptr;
  // a caller-held factor (the prepared SystemFactor of solver.cc:3808-3812)
  // and the frame it is applied in; block Jacobi while it is absent or empty
  const or_solver* factor = nullptr;
  M3<R> frame{R(1)};
  uint32_t factorApplications = 0;

  // solver.cc:1920-1952 condition
  void condition() {
    if (factor && factor->ready) {
      conditioned = residual;
      applyFactor(*factor, frame, conditioned);
      ++factorApplications;
      return;
    }
    for (uint32_t n = 0; n < V; ++n) conditioned[n] = preconditioner[n] * residual[n];
  }

  const TetStiffness<R>& stiffnessOf(uint32_t e) const { return consistent ? working[e] : store[e]; }

  std::array<V3<R>, 4> gather(const std::vector<V3<R>>& at, const Element<R>& el) const {
    return {at[el.nodes[0]], at[el.nodes[1]], at[el.nodes[2]], at[el.nodes[3]]};
  }

  // solver.cc:437-451 bindStiffness
  void bindStiffness(bool wantConsistent, bool anyYields) {
    if (!wantConsistent || !anyYields) {
      consistent = false;
      working.clear();
      return;
    }
    working = store;
    consistent = true;
  }

  struct Assembly { R energy{0}; uint32_t loading = 0, yielding = 0; };

  // solver.cc:1354-1572 assembleElastic (tets only), plus the SNH law
  Assembly assemble(R step, const std::vector<V3<R>>& at, bool keep, R margin, int mode, bool mapping = true) {
    std::fill(force.begin(), force.end(), V3<R>());
    std::fill(diagonal.begin(), diagonal.end(), M3<R>(R(0)));
    const R scale = step * step;
    Assembly out;
    for (uint32_t e = 0; e < T; ++e) {
      const Element<R>& el = elements[e];
      const std::array<V3<R>, 4> g = gather(at, el);
      // from the plastic rest shape the corotated offsets and K use Dm', V'
      const std::array<V3<R>, 4> r = hencky ? plasticCorners[e] : gather(rest, el);
      std::array<V3<R>, 4> f;
      std::array<M3<R>, 4> diag;
      if (law == OR_LAW_SNH) {
        const SnhTet<R> s = snhTet(g, r, el.restInverse, el.volume, el.moduli);
        snhGradient[e] = s.gradient;
        snhChange[e] = s.change;
        out.energy += s.energy;
        f = s.force;
        const std::array<V3<R>, 4> grad = shapeGradients(el.restInverse);
        for (int n = 0; n < 4; ++n) diag[n] = snhDiagonal(grad[n], s.gradient, el.volume, el.moduli);
      } else if (el.yields && !hencky) {
        const TetPointTrial<R> c = tetPointTrial(g, r, el.restInverse, el.volume, el.moduli, el.yieldStress,
                                                 el.hardening, plastic[e], margin, mode, mapping, consistent);
        rotation[e] = c.rotation;
        out.energy += c.energy;
        out.loading += c.loading;
        out.yielding += c.yielding;
        if (consistent) working[e] = c.tangent;
        if (keep) plastic[e] = c.point;
        diag = stiffnessDiagonal(stiffnessOf(e), c.rotation);
        f = c.force;
      } else {
        const TetStiffness<R>& k = stiffnessOf(e);
        const TrialState<R> c = trial(g, r, el.restInverse, k, mode);
        rotation[e] = c.rotation;
        out.energy += c.energy;
        diag = stiffnessDiagonal(k, c.rotation);
        f = c.force;
      }
      for (int n = 0; n < 4; ++n) {
        force[el.nodes[n]] += f[n];
        diagonal[el.nodes[n]][0] += scale * diag[n][0];
        diagonal[el.nodes[n]][1] += scale * diag[n][1];
        diagonal[el.nodes[n]][2] += scale * diag[n][2];
      }
    }
    if (damped) {  // fitDamping, blockDamping, addDampingDiagonal (solver.cc:645-681, 755-804, 806-830)
      for (uint32_t e = 0; e < T; ++e) {
        const Element<R>& el = elements[e];
        if (el.tau == R(0)) continue;
        fits[e] = rigidFit(gather(at, el));
        const std::array<M3<R>, 4> made = dampingDiagonal(fits[e], rotation[e], store[e]);
        const R weight = dampScale * el.tau;
        for (int n = 0; n < 4; ++n) diagonal[el.nodes[n]] = diagonal[el.nodes[n]] + weight * made[n];
      }
    }
    return out;
  }

  // addDamping (solver.cc:683-750): output += weight tau D(input) per element.
  void addDamping(R weight, const std::vector<V3<R>>& input, std::vector<V3<R>>& output) {
    std::array<V3<R>, 4> produced;
    for (uint32_t e = 0; e < T; ++e) {
      const Element<R>& el = elements[e];
      if (el.tau == R(0)) continue;
      applyDamping(fits[e], rotation[e], store[e], gather(input, el), produced);
      const R scaled = weight * el.tau;
      for (int n = 0; n < 4; ++n) output[el.nodes[n]] += scaled * produced[n];
    }
  }

  // solver.cc:904-1048 applySystem (tets, no damping, not stressed)
  void applySystem(R inertia, R step, const std::vector<V3<R>>& input, std::vector<V3<R>>& output) {
    for (uint32_t n = 0; n < V; ++n) output[n] = (inertia * mass[n]) * input[n];
    const R scale = step * step;
    std::array<V3<R>, 4> produced;
    for (uint32_t e = 0; e < T; ++e) {
      const Element<R>& el = elements[e];
      const std::array<V3<R>, 4> g = gather(input, el);
      if (law == OR_LAW_SNH) {
        snhApply(g, el.restInverse, el.volume, el.moduli, snhGradient[e], snhChange[e], produced);
      } else {
        applyStiffness(g, rotation[e], stiffnessOf(e), produced);
      }
      for (int n = 0; n < 4; ++n) output[el.nodes[n]] += scale * produced[n];
    }
    if (damped) addDamping(dampScale, input, output);  // solver.cc:1006-1007
    for (uint32_t n = 0; n < V; ++n)
      if (anchored[n]) output[n] = V3<R>();
    if (report) ++report->operator_applications;
  }

  // solver.cc:1574-1593
  void guardPreconditioner() {
    for (uint32_t n = 0; n < V; ++n) {
      if (anchored[n] || !(determinant(diagonal[n]) > R(0))) {
        preconditioner[n] = M3<R>(R(1));
        continue;
      }
      preconditioner[n] = inverse(diagonal[n]);
    }
  }

  // applications: the factor applications of this solve (CgResult::factorTiming, solver.cc:1926-1934)
  struct CgResult {
    uint32_t iterations = 0;
    R relativeResidual{0}, startResidual{0};
    bool capped = false;
    uint32_t applications = 0;
  };

  // solver.cc:1904-2089 conjugateGradient (block Jacobi or the factor, no free modes)
  CgResult conjugateGradient(R inertia, R step, uint32_t limit, R tolerance, std::vector<V3<R>>& solution) {
    CgResult result;
    const uint32_t applied0 = factorApplications;
    R reference = 0;
    for (uint32_t n = 0; n < V; ++n) reference += dot(right[n], right[n]);
    reference = std::sqrt(reference);
    applySystem(inertia, step, solution, applied);
    R squared = 0;
    for (uint32_t n = 0; n < V; ++n) residual[n] = anchored[n] ? V3<R>() : right[n] - applied[n];
    condition();
    for (uint32_t n = 0; n < V; ++n) {
      direction[n] = conditioned[n];
      squared += dot(residual[n], conditioned[n]);
    }
    const R referenceFloor = std::max(reference, std::numeric_limits<R>::min());
    const R target = tolerance * referenceFloor;
    R opening = 0;
    for (uint32_t n = 0; n < V; ++n) opening += dot(residual[n], residual[n]);
    result.startResidual = std::sqrt(opening) / referenceFloor;
    uint32_t taken = 0;
    for (uint32_t iteration = 0; iteration != limit; ++iteration) {
      R len = 0;
      for (uint32_t n = 0; n < V; ++n) len += dot(residual[n], residual[n]);
      if (std::sqrt(len) <= target) break;
      applySystem(inertia, step, direction, applied);
      R curvature = 0;
      for (uint32_t n = 0; n < V; ++n) curvature += dot(direction[n], applied[n]);
      if (!(curvature > R(0)) || !(squared > R(0))) break;
      const R stride = squared / curvature;
      for (uint32_t n = 0; n < V; ++n) {
        solution[n] += stride * direction[n];
        residual[n] -= stride * applied[n];
      }
      R next = 0;
      condition();
      for (uint32_t n = 0; n < V; ++n) next += dot(residual[n], conditioned[n]);
      const R blend = next / squared;
      squared = next;
      for (uint32_t n = 0; n < V; ++n) direction[n] = conditioned[n] + blend * direction[n];
      ++taken;
    }
    R rs = 0;
    for (uint32_t n = 0; n < V; ++n) rs += dot(residual[n], residual[n]);
    const R res = std::sqrt(rs);
    result.iterations = taken;
    result.relativeResidual = res / referenceFloor;
    result.capped = taken == limit && res > target;
    result.applications = factorApplications - applied0;
    return result;
  }

  // solver.cc:568-623
  bool predictorInverts(const IntegratorRule<R>& rule, R inner) {
    const R carryScale = (R(0.5) - rule.beta) * inner * inner;
    for (uint32_t n = 0; n < V; ++n) {
      const V3<R> s = position[n] + inner * velocity[n] + carryScale * acceleration[n];
      weighted[n] = (R(1) - rule.alphaForce) * s + rule.alphaForce * position[n];
    }
    for (uint32_t e = 0; e < T; ++e) {
      const std::array<V3<R>, 4> g = gather(weighted, elements[e]);
      if (determinant(deformationOf(g, elements[e].restInverse)) <= R(0)) return true;
    }
    return false;
  }

  // solver.cc:1260-1346 commitPlastic (tets)
  bool commitPlastic(int mode) {
    bool grew = false;
    for (uint32_t e = 0; e < T; ++e) {
      const Element<R>& el = elements[e];
      if (!el.yields || law == OR_LAW_SNH) continue;
      const TetPointTrial<R> c = tetPointTrial(gather(position, el), gather(rest, el), el.restInverse, el.volume,
                                               el.moduli, el.yieldStress, el.hardening, plastic[e], R(0), mode, true,
                                               false);
      grew = grew || c.point.equivalent > plastic[e].equivalent;
      plastic[e] = c.point;
    }
    return grew;
  }
};

// ------------------------------------------------- floating frame ----
// A body with no anchored node and RigidSplit != Off (floats, solver.cc:2964-2971)
// is stepped in a frame that moves with its centre of mass and turns with its
// rigid spin: the predictor, the drive of the fictitious forces, and the
// end-of-substep momentum and torque projection (solver.cc:3657-3690,
// 4265-4340).  The frame itself is FP64 like the reference's (floatingFrame,
// solver.cc:3046-3142; rigidAdvance, solver.cc:2983-3036) and stored in R.

constexpr double FLOATING_TOLERANCE = 1.0e-5;  // solver.cc:9
constexpr uint32_t RIGID_PARTS = 8u;           // solver.h:109

// solver.h:111-114 RigidMotion: angular momentum and accumulated turn
struct RigidMotion { V3<double> momentum; M3<double> turn{1.0}; };

// solver.cc:2973-2979 skew: skew(a) v = a x v
inline M3<double> skew(const V3<double>& a) {
  return M3<double>(V3<double>(0.0, a.z, -a.y), V3<double>(-a.z, 0.0, a.x), V3<double>(a.y, -a.x, 0.0));
}

// solver.cc:2983-2987 rigidRate: torque-free rigid body, inertia fixed in the world
inline RigidMotion rigidRate(const M3<double>& inverseInertia, const RigidMotion& at) {
  const V3<double> spin = inverseInertia * at.momentum;
  return RigidMotion{cross(at.momentum, spin), at.turn * skew(spin)};
}

// solver.cc:2989-3026 rigidAdvance: `count` classic Runge-Kutta steps over
// `span`, then three polar passes that pull the turn back to a rotation
inline RigidMotion rigidAdvance(const M3<double>& inverseInertia, RigidMotion motion, double span, uint32_t count) {
  const double part = span / double(count);
  const auto moved = [](const RigidMotion& from, const RigidMotion& rate, double by) {
    return RigidMotion{from.momentum + by * rate.momentum, from.turn + by * rate.turn};
  };
  for (uint32_t at = 0; at != count; ++at) {
    const RigidMotion first = rigidRate(inverseInertia, motion);
    const RigidMotion second = rigidRate(inverseInertia, moved(motion, first, 0.5 * part));
    const RigidMotion third = rigidRate(inverseInertia, moved(motion, second, 0.5 * part));
    const RigidMotion fourth = rigidRate(inverseInertia, moved(motion, third, part));
    motion.momentum += (part / 6.0) * (first.momentum + 2.0 * second.momentum + 2.0 * third.momentum + fourth.momentum);
    motion.turn = motion.turn + (part / 6.0) * (first.turn + 2.0 * second.turn + 2.0 * third.turn + fourth.turn);
  }
  for (uint32_t pass = 0; pass != 3u; ++pass) motion.turn = 0.5 * (motion.turn + transpose(inverse(motion.turn)));
  return motion;
}

// solver.cc:2944-2961 FloatingFrame
template <class R> struct FloatingFrame {
  V3<R> centre, velocity, acceleration, nextCentre, nextVelocity, nextAcceleration, momentum, torque, spin, spinRate,
      weightedSpin, weightedRate, endSpin, endRate;
  M3<R> turn{R(1)}, weightedTurn{R(1)};
};

template <class R> V3<R> narrow(const V3<double>& v) { return V3<R>(R(v.x), R(v.y), R(v.z)); }
template <class R> V3<double> widen(const V3<R>& v) { return V3<double>(double(v.x), double(v.y), double(v.z)); }
template <class R> M3<R> narrow(const M3<double>& m) { return M3<R>(narrow<R>(m[0]), narrow<R>(m[1]), narrow<R>(m[2])); }

// solver.cc:3031-3142 floatingFrame
template <class R>
FloatingFrame<R> floatingFrame(const std::vector<R>& nodeMass, const std::vector<V3<R>>& position,
                               const std::vector<V3<R>>& velocity, const std::vector<V3<R>>& acceleration,
                               const IntegratorRule<R>& rule, R inner, const V3<R>& gravity) {
  V3<double> centre, vel, acc;
  double total = 0.0;
  for (size_t n = 0; n < position.size(); ++n) {
    const double mass = double(nodeMass[n]);
    total += mass;
    centre += mass * widen(position[n]);
    vel += mass * widen(velocity[n]);
    acc += mass * widen(acceleration[n]);
  }
  const auto over = [](const V3<double>& v, double d) { return V3<double>(v.x / d, v.y / d, v.z / d); };
  centre = over(centre, total);
  vel = over(vel, total);
  acc = over(acc, total);
  M3<double> inertia(0.0);
  V3<double> momentum, torque;
  for (size_t n = 0; n < position.size(); ++n) {
    const double mass = double(nodeMass[n]);
    const V3<double> arm = widen(position[n]) - centre;
    inertia = inertia + mass * (dot(arm, arm) * M3<double>(1.0) - outer(arm, arm));
    momentum += mass * cross(arm, widen(velocity[n]) - vel);
    torque += mass * cross(arm, widen(acceleration[n]) - acc);
  }
  FloatingFrame<R> made;
  const double h = double(inner);
  const double alphaMass = double(rule.alphaMass), beta = double(rule.beta), gamma = double(rule.gamma);
  const V3<double> next = over(widen(gravity) - alphaMass * acc, 1.0 - alphaMass);
  made.centre = narrow<R>(centre);
  made.velocity = narrow<R>(vel);
  made.acceleration = narrow<R>(acc);
  made.nextAcceleration = narrow<R>(next);
  made.nextCentre = narrow<R>(centre + h * vel + (h * h) * ((0.5 - beta) * acc + beta * next));
  made.nextVelocity = narrow<R>(vel + h * ((1.0 - gamma) * acc + gamma * next));
  made.momentum = narrow<R>(momentum + (h * (1.0 - gamma - gamma * alphaMass / (1.0 - alphaMass))) * torque);
  made.torque = narrow<R>((-alphaMass / (1.0 - alphaMass)) * torque);
  const double det = determinant(inertia);
  const double scale = inertia[0][0] + inertia[1][1] + inertia[2][2];
  if (!(det > 1.0e-12 * scale * scale * scale) || dot(momentum, momentum) == 0.0) return made;
  const M3<double> inv = inverse(inertia);
  const double weighted = (1.0 - double(rule.alphaForce)) * h;
  const RigidMotion start{momentum, M3<double>(1.0)};
  const RigidMotion middle = rigidAdvance(inv, start, weighted, RIGID_PARTS);
  const RigidMotion end = rigidAdvance(inv, middle, h - weighted, RIGID_PARTS);
  const auto spinOf = [&](const RigidMotion& at) { return inv * at.momentum; };
  const auto rateOf = [&](const RigidMotion& at) { return inv * cross(at.momentum, inv * at.momentum); };
  made.spin = narrow<R>(spinOf(start));
  made.spinRate = narrow<R>(rateOf(start));
  made.weightedSpin = narrow<R>(spinOf(middle));
  made.weightedRate = narrow<R>(rateOf(middle));
  made.endSpin = narrow<R>(end.turn * spinOf(end));
  made.endRate = narrow<R>(end.turn * rateOf(end));
  made.turn = narrow<R>(end.turn);
  made.weightedTurn = narrow<R>(middle.turn);
  return made;
}

// factor.cc:21-30 preciseLame, 32-47 preciseTurned, 49-88 preciseTetBlocks:
// step^2 R K R^T in FP64, with Dm and V recomputed from the rest positions.
template <class R>
std::array<M3<double>, 16> preciseTetBlocks(const Solver<R>& s, const Element<R>& el, double youngs, double poisson,
                                            const M3<R>& rotation, R step) {
  const auto wide = [](const V3<R>& v) { return V3<double>(double(v.x), double(v.y), double(v.z)); };
  const V3<double> first = wide(s.rest[el.nodes[0]]);
  const M3<double> shape(wide(s.rest[el.nodes[1]]) - first, wide(s.rest[el.nodes[2]]) - first,
                         wide(s.rest[el.nodes[3]]) - first);
  const double volume = determinant(shape) / 6.0;
  const M3<double> rows = transpose(inverse(shape));
  const std::array<V3<double>, 4> gradient{-(rows[0] + rows[1] + rows[2]), rows[0], rows[1], rows[2]};
  const double nu = std::clamp(poisson, 0.0, 0.49);
  const double lambda = youngs * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = youngs / (2.0 * (1.0 + nu));
  M3<double> turn;
  for (int c = 0; c < 3; ++c) turn[c] = wide(rotation[c]);
  const M3<double> back = transpose(turn);
  const double scale = double(step) * double(step);
  std::array<M3<double>, 16> blocks;
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      const V3<double>& ga = gradient[a];
      const V3<double>& gb = gradient[b];
      const M3<double> k = volume * (lambda * outer(ga, gb) + mu * outer(gb, ga) + (mu * dot(ga, gb)) * M3<double>(1.0));
      blocks[4 * a + b] = scale * (turn * k * back);
    }
  return blocks;
}

// factor.cc:318-460 gather, 549-565 analyzeSystem, 567-618 refreshFactor: the
// system (1 - alpha_m) M + h^2 sum R K R^T at the committed rotations, anchored
// rows and columns replaced by the identity, factored; the reference
// positions and centroid are the state's.
template <class R>
void refreshFactor(or_solver& f, const Solver<R>& s, const std::vector<double>& youngs,
                   const std::vector<double>& poisson, R step, R inertia, R damping) {
  const uint32_t V = s.V;
  const size_t n = size_t(3) * V;
  if (f.analyzed && f.nodes != V) f.analyzed = false;
  if (!f.analyzed) {
    f.nodes = V;
    f.anchored = s.anchored;
    // stored entries of the full matrix: 9 per coupled pair of free nodes,
    // 3 on the diagonal of every node
    std::vector<std::vector<uint32_t>> pairs(V);
    for (const Element<R>& el : s.elements)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
          if (!s.anchored[el.nodes[a]] && !s.anchored[el.nodes[b]]) pairs[el.nodes[a]].push_back(el.nodes[b]);
    uint64_t stored = 0;
    for (uint32_t v = 0; v < V; ++v) {
      std::sort(pairs[v].begin(), pairs[v].end());
      pairs[v].erase(std::unique(pairs[v].begin(), pairs[v].end()), pairs[v].end());
      const bool diagonalHeld = std::binary_search(pairs[v].begin(), pairs[v].end(), v);
      stored += 9u * pairs[v].size() + (diagonalHeld ? 0u : 3u);
    }
    f.systemNonZeros = stored;
    f.first.assign(n, 0u);
    for (size_t i = 0; i < n; ++i) f.first[i] = uint32_t(i - i % 3);
    for (const Element<R>& el : s.elements)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          const uint32_t na = el.nodes[a], nb = el.nodes[b];
          if (s.anchored[na] || s.anchored[nb]) continue;
          for (int r = 0; r < 3; ++r) f.first[3 * na + r] = std::min(f.first[3 * na + r], 3u * nb);
        }
    f.start.assign(n + 1, 0u);
    for (size_t i = 0; i < n; ++i) f.start[i + 1] = f.start[i] + (i - f.first[i] + 1);
    f.analyzed = true;
  }
  f.env.assign(f.start[n], 0.0);
  auto at = [&](size_t i, size_t j) -> double& { return f.env[f.start[i] + (j - f.first[i])]; };
  for (uint32_t e = 0; e < s.T; ++e) {
    const Element<R>& el = s.elements[e];
    std::array<M3<double>, 16> blocks = preciseTetBlocks(s, el, youngs[e], poisson[e], s.rotation[e], step);
    // factor.cc:346-366, 386-389: the damping blocks weight * dampingBlocks(rigidFit(corners), R, K),
    // the fit at the state's positions, in the step's arithmetic (dampingBlocks, factor.cc:274-298)
    const R weight = damping * el.tau;
    if (weight != R(0)) {
      const RigidFit<R> fit = rigidFit(s.gather(s.position, el));
      std::array<V3<R>, 4> unit, column;
      for (int corner = 0; corner < 4; ++corner)
        for (int axis = 0; axis < 3; ++axis) {
          unit.fill(V3<R>());
          unit[corner][axis] = R(1);
          applyDamping(fit, s.rotation[e], s.store[e], unit, column);
          for (int row = 0; row < 4; ++row) {
            const V3<R> scaled = weight * column[row];
            blocks[4 * row + corner][axis] += V3<double>(double(scaled.x), double(scaled.y), double(scaled.z));
          }
        }
    }
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        const uint32_t na = el.nodes[a], nb = el.nodes[b];
        if (s.anchored[na] || s.anchored[nb]) continue;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c)
            if (3u * nb + c <= 3u * na + r) at(3 * na + r, 3 * nb + c) += blocks[4 * a + b][c][r];
      }
  }
  for (uint32_t v = 0; v < V; ++v) {
    const double diagonal = s.anchored[v] ? 1.0 : double(inertia * s.mass[v]);
    for (int k = 0; k < 3; ++k) at(3 * v + k, 3 * v + k) += diagonal;
  }
  // LL^T inside the envelope (SimplicialLLT::factorize fails on a pivot <= 0)
  f.ready = true;
  for (size_t i = 0; i < n && f.ready; ++i) {
    double* row = &f.env[f.start[i]] - f.first[i];
    for (size_t j = f.first[i]; j < i; ++j) {
      const double* other = &f.env[f.start[j]] - f.first[j];
      double sum = row[j];
      for (size_t k = std::max(f.first[i], f.first[j]); k < j; ++k) sum -= row[k] * other[k];
      row[j] = sum / other[j];
    }
    double d = row[i];
    for (size_t k = f.first[i]; k < i; ++k) d -= row[k] * row[k];
    if (!(d > 0.0)) f.ready = false;
    else row[i] = std::sqrt(d);
  }
  ++f.born;
  f.refStep = double(step);
  f.refInertia = double(inertia);
  f.refDamping = double(damping);
  f.refPosition.assign(n, 0.0);
  V3<R> centroid;
  R total = 0;
  for (uint32_t v = 0; v < V; ++v) {
    for (int k = 0; k < 3; ++k) f.refPosition[3 * v + k] = double(s.position[v][k]);
    total += s.mass[v];
    centroid += s.mass[v] * s.position[v];
  }
  if (total > R(0)) centroid = V3<R>(centroid.x / total, centroid.y / total, centroid.z / total);
  for (int k = 0; k < 3; ++k) f.refCentroid[k] = double(centroid[k]);
}

template <class R>
int stepImpl(const or_mesh* mesh, or_state* st, const or_material* materials, uint32_t lanes, const or_settings* settings,
             const double gravity[3], double dtIn, or_report* report, or_solver* solver) {
  const auto began = std::chrono::steady_clock::now();
  Solver<R> s;
  s.report = report;
  s.V = mesh->nodes;
  s.T = mesh->tets;
  s.law = int(settings->law);
  const uint32_t V = s.V, T = s.T;
  s.rest.resize(V);
  s.mass.resize(V);
  s.anchored.assign(mesh->anchored, mesh->anchored + V);
  s.prescribed.assign(V, V3<R>());
  s.position.resize(V);
  s.velocity.resize(V);
  s.acceleration.resize(V);
  bool anyAnchored = false;
  for (uint32_t n = 0; n < V; ++n) {
    s.rest[n] = V3<R>(R(mesh->rest[3 * n]), R(mesh->rest[3 * n + 1]), R(mesh->rest[3 * n + 2]));
    s.mass[n] = R(mesh->node_mass[n]);
    if (mesh->prescribed)
      s.prescribed[n] = V3<R>(R(mesh->prescribed[3 * n]), R(mesh->prescribed[3 * n + 1]), R(mesh->prescribed[3 * n + 2]));
    s.position[n] = V3<R>(R(st->position[3 * n]), R(st->position[3 * n + 1]), R(st->position[3 * n + 2]));
    s.velocity[n] = V3<R>(R(st->velocity[3 * n]), R(st->velocity[3 * n + 1]), R(st->velocity[3 * n + 2]));
    s.acceleration[n] = V3<R>(R(st->acceleration[3 * n]), R(st->acceleration[3 * n + 1]), R(st->acceleration[3 * n + 2]));
    anyAnchored = anyAnchored || s.anchored[n] != 0;
  }
  // floats (solver.cc:2964-2971): no anchored node and the rigid split on
  const bool floating = settings->rigid_split != 0u && V > 0u && !anyAnchored;
  s.elements.resize(T);
  s.store.resize(T);
  s.rotation.resize(T);
  s.plastic.resize(T);
  s.snhGradient.assign(T, M3<R>(R(1)));
  s.snhChange.assign(T, R(0));
  s.hencky = settings->plasticity == OR_PLASTICITY_HENCKY;
  if (s.hencky) {
    s.authored.resize(T);
    s.flowMap.resize(T);
    s.hardeningOf.resize(T);
    s.plasticCorners.resize(T);
  }
  bool anyYields = false;
  std::vector<double> factorYoungs(T), factorPoisson(T);  // the material of each tet, for the factor
  static const or_material DEFAULT = {1000.0, 0.0, 0.3, 0.0, std::numeric_limits<double>::infinity(), 0.0,
                                      std::numeric_limits<double>::infinity(), 1.0,
                                      std::numeric_limits<double>::infinity()};
  for (uint32_t e = 0; e < T; ++e) {
    Element<R>& el = s.elements[e];
    for (int k = 0; k < 4; ++k) el.nodes[k] = mesh->tet_nodes[4 * e + k];
    el.restInverse = loadRowMajor<R>(mesh->rest_inverse + 9 * e);
    el.volume = R(mesh->volume[e]);
    const or_material& m = mesh->lane[e] < lanes ? materials[mesh->lane[e]] : DEFAULT;  // material.cc:9-16
    el.tau = std::isfinite(m.stiffness_damping) && m.stiffness_damping > 0.0 ? R(m.stiffness_damping) : R(0);
    s.damped = s.damped || el.tau > R(0);
    const R youngs = mesh->element_youngs ? R(mesh->element_youngs[e]) : R(m.youngs_modulus);
    el.moduli = lame(youngs, R(m.poissons_ratio));
    factorYoungs[e] = double(youngs);
    factorPoisson[e] = double(R(m.poissons_ratio));
    el.yieldStress = R(m.yield_stress);
    el.hardening = R(m.hardening_modulus);
    el.yields = yieldsAt(el.yieldStress);
    el.limits = FlowLimits{m.crush_stress, m.crush_limit, m.plastic_max};
    anyYields = anyYields || el.yields;
    if (s.hencky) {
      const M3<double> given = loadRowMajor<double>(mesh->rest_inverse + 9 * e);
      const M3<double> p = loadRowMajor<double>(st->plastic + 10 * e);
      s.authored[e] = given;
      s.flowMap[e] = p;
      s.hardeningOf[e] = st->plastic[10 * e + 9];
      double rowMajor[9];
      storeRowMajor(given * p, rowMajor);  // Dm'^-1 = Dm^-1 P
      el.restInverse = loadRowMajor<R>(rowMajor);
      el.volume = R(mesh->volume[e] / determinant(p));  // V' = V det Fp
      storeRowMajor(inverse(given * p), rowMajor);
      const M3<R> shape = loadRowMajor<R>(rowMajor);
      s.plasticCorners[e] = {V3<R>(), shape[0], shape[1], shape[2]};
    }
    s.store[e] = tetStiffness(el.restInverse, el.volume, el.moduli);
    s.rotation[e] = loadRowMajor<R>(st->rotation + 9 * e);
    PlasticPoint<R> p;
    p.strain = loadRowMajor<R>(st->plastic + 10 * e);
    p.equivalent = R(st->plastic[10 * e + 9]);
    s.plastic[e] = p;
  }
  if (s.law == OR_LAW_SNH) anyYields = false;  // SNH runs elastic only
  // the finite-strain flow is written for the corotated law without damping
  if (s.hencky && (s.law == OR_LAW_SNH || s.damped)) return -3;
  const bool anyFlows = s.hencky && anyYields;
  if (s.hencky) anyYields = false;  // each step is elastic from the plastic rest
  // damping is defined with the corotated stiffness and committed rotation
  if (s.damped && s.law == OR_LAW_SNH) return -3;
  // a factor is restated for the small-strain path
  if (solver && s.hencky) return -3;
  if (s.damped) s.fits.assign(T, RigidFit<R>());
  auto sized = [&](std::vector<V3<R>>& v) { v.assign(V, V3<R>()); };
  sized(s.force); sized(s.right); sized(s.residual); sized(s.direction); sized(s.applied); sized(s.conditioned);
  sized(s.increment); sized(s.restart); sized(s.shifted); sized(s.weighted); sized(s.carried); sized(s.evaluated);
  sized(s.total); sized(s.lowestIterate); sized(s.drive);
  s.diagonal.assign(V, M3<R>(R(0)));
  s.preconditioner.assign(V, M3<R>(R(0)));

  const R dt = R(dtIn);
  const V3<R> g{R(gravity[0]), R(gravity[1]), R(gravity[2])};
  const uint32_t configured = std::max(settings->substeps, 1u);
  const IntegratorRule<R> rule = integratorRule(R(settings->spectral_radius));
  const bool newton = settings->plastic_passes > 1u && anyYields;
  const uint32_t plasticCap = settings->plastic_passes;
  s.bindStiffness(false, anyYields);
  // solver.cc:3560-3562, 3574-3583: a floating body solves to at most
  // FLOATING_TOLERANCE and is not tested for predictor inversion
  const R tolerance = floating ? std::min(R(settings->tolerance), R(FLOATING_TOLERANCE)) : R(settings->tolerance);
  const uint32_t substeps = !floating && s.predictorInverts(rule, dt / R(configured))
                                ? std::max(configured, INVERTED_SUBSTEPS)
                                : configured;
  const R inner = dt / R(substeps);
  const EffectiveSystem<R> effective = effectiveSystem(rule, inner);
  const R carryScale = (R(0.5) - rule.beta) * inner * inner;
  s.dampScale = (R(1) - rule.alphaForce) * rule.gamma * inner;
  std::vector<V3<R>> viscous(s.damped ? V : 0u), viscousVelocity(s.damped ? V : 0u);
  const int mode = floating ? OR_ROTATION_POLAR : OR_ROTATION_INVERTIBLE;  // solver.cc:3587-3588
  std::vector<V3<R>> relative(floating ? V : 0u), unconstrained(floating ? V : 0u);
  report->substeps += substeps;
  R elastic = 0;
  bool plasticGrowth = false;
  // solver.cc:3639-3655: the caller's factor is made again when it is empty
  // or was made for another step or inertia
  // dampingStep (solver.cc:3592): the damping scale when a material damps; the
  // reference compares the per-lane keys scale * tau, equal exactly when the scales are
  const R dampingStep = s.damped ? s.dampScale : R(0);
  if (solver && (!solver->ready || solver->refStep != double(effective.step) ||
                 solver->refInertia != double(effective.inertia) || solver->refDamping != double(dampingStep))) {
    refreshFactor(*solver, s, factorYoungs, factorPoisson, effective.step, effective.inertia, dampingStep);
    solver->stats.factor_age = 0u;
    ++solver->stats.refactor_count;
  }

  for (uint32_t pass = 0; pass != substeps; ++pass) {
    const FloatingFrame<R> body = floating
                                      ? floatingFrame(s.mass, s.position, s.velocity, s.acceleration, rule, inner, g)
                                      : FloatingFrame<R>{};
    if (floating) {
      // solver.cc:3662-3690: relative velocity and acceleration in the frame
      // that moves with the centre and turns with the spin; the drive holds
      // the centrifugal, Euler and Coriolis forces at the weighted time
      const V3<R> spin = body.spin, held = body.weightedSpin;
      const R lag = (R(1) - rule.alphaForce) * (R(1) - rule.gamma) * inner;
      for (uint32_t n = 0; n < V; ++n) {
        const V3<R> arm = s.position[n] - body.centre;
        const V3<R> moving = s.velocity[n] - body.velocity - cross(spin, arm);
        const V3<R> turning = s.acceleration[n] - body.acceleration - cross(body.spinRate, arm) -
                              cross(spin, cross(spin, arm)) - R(2) * cross(spin, moving);
        const R m = s.mass[n];
        relative[n] = moving;
        s.carried[n] = turning;
        s.shifted[n] = arm + inner * moving + carryScale * turning;
        s.weighted[n] = (R(1) - rule.alphaForce) * s.shifted[n] + rule.alphaForce * arm;
        s.drive[n] = -m * (cross(held, cross(held, s.weighted[n])) + cross(body.weightedRate, s.weighted[n]) +
                           R(2) * cross(held, moving + lag * turning));
        s.acceleration[n] = turning;
      }
    } else {
      // predictor, solver.cc:3691-3700 (anchored nodes move with their prescribed velocity)
      for (uint32_t n = 0; n < V; ++n) {
        s.carried[n] = s.acceleration[n];
        s.shifted[n] = s.position[n] + inner * s.velocity[n] + carryScale * s.acceleration[n];
        s.weighted[n] = (R(1) - rule.alphaForce) * s.shifted[n] + rule.alphaForce * s.position[n];
        s.drive[n] = s.mass[n] * g;
      }
    }
    auto assemble = [&](const std::vector<V3<R>>& at, R margin, bool mapping = true) {
      return s.assemble(effective.step, at, false, margin, mode, mapping);
    };
    // solver.cc:3746-3806 balance
    auto balance = [&](const std::vector<V3<R>>* taken) {
      if (s.damped) {  // viscous force of the lagged velocity (solver.cc:3747-3778)
        const R lag = (R(1) - rule.alphaForce) * inner;
        for (uint32_t n = 0; n < V; ++n) {
          if (s.anchored[n]) {
            viscousVelocity[n] = V3<R>();
            continue;
          }
          viscousVelocity[n] = (floating ? relative[n] : s.velocity[n]) + (lag * (R(1) - rule.gamma)) * s.carried[n];
          if (taken) viscousVelocity[n] += (lag * rule.gamma) * (*taken)[n];
        }
        std::fill(viscous.begin(), viscous.end(), V3<R>());
        s.addDamping(R(1), viscousVelocity, viscous);
      }
      for (uint32_t n = 0; n < V; ++n) {
        if (s.anchored[n]) {
          s.velocity[n] = s.prescribed[n];
          s.acceleration[n] = V3<R>();
          s.right[n] = V3<R>();
          continue;
        }
        const R m = s.mass[n];
        s.right[n] = s.force[n] + s.drive[n] - (rule.alphaMass * m) * s.carried[n];
        if (taken) s.right[n] -= (effective.inertia * m) * (*taken)[n];
        if (s.damped) s.right[n] -= viscous[n];
        s.diagonal[n][0].x += effective.inertia * m;
        s.diagonal[n][1].y += effective.inertia * m;
        s.diagonal[n][2].z += effective.inertia * m;
      }
      s.guardPreconditioner();
    };
    auto recordCg = [&](const typename Solver<R>::CgResult& r) {
      report->cg_iterations += r.iterations;
      report->cg_capped_solves += r.capped ? 1u : 0u;
      report->cg_worst_relative_residual = std::max(report->cg_worst_relative_residual, double(r.relativeResidual));
    };
    // solver.cc:3808-3821: the prepared factor, its frame and the budget of a
    // factored solve
    s.factor = solver && solver->ready ? solver : nullptr;
    s.frame = s.factor ? bodyRotation(s.mass, s.position, *solver) : M3<R>(R(1));
    const uint32_t budget = s.factor && solver->budget != 0u ? std::min(solver->budget, settings->cg_iterations)
                                                               : settings->cg_iterations;
    uint32_t passIterations = 0;  // primaryResult.iterations of the substep
    // solver.cc:3822-3910 solvePrimary: a capped factored solve that may
    // refresh makes the factor again at the latest rotations and solves
    // again from the same start with the full iteration cap
    auto solvePrimary = [&](std::vector<V3<R>>& solution, bool refreshes) {
      s.restart = solution;
      auto r = s.conjugateGradient(effective.inertia, effective.step, budget, tolerance, solution);
      if (r.capped && s.factor && refreshes) {
        or_solver_stats& fs = solver->stats;
        ++fs.refresh_requests;
        fs.refreshed_at_age = fs.substeps_since_refresh;
        fs.spent_before_refresh = r.iterations;
        fs.wasted_iterations += r.iterations;
        fs.refresh_requested = 1u;
        solution = s.restart;
        refreshFactor(*solver, s, factorYoungs, factorPoisson, effective.step, effective.inertia, dampingStep);
        ++fs.refactors;
        ++fs.retries;
        ++fs.refactor_count;
        ++fs.retry_count;
        fs.factor_age = 0u;
        fs.substeps_since_refresh = 0u;
        s.frame = M3<R>(R(1));
        s.factor = solver;
        r = s.conjugateGradient(effective.inertia, effective.step, settings->cg_iterations, tolerance, solution);
        fs.spent_after_refresh = r.iterations;
        if (r.capped) {
          ++fs.retries_failed;
          fs.fresh_retry_failed = 1u;
        }
      }
      passIterations += r.iterations;
      if (solver) solver->stats.factor_applications += r.applications;  // recordCg: the result's own
      recordCg(r);
      return r;
    };
    auto rightSquared = [&]() {
      double squared = 0.0;
      for (const V3<R>& r : s.right) squared += double(dot(r, r));
      return squared;
    };
    const R reach = effective.step * effective.step;

    if (!newton) {  // solver.cc:3914-3950
      const auto first = assemble(s.weighted, R(0));
      elastic = first.energy;
      report->yielding = first.yielding;
      balance(nullptr);
      solvePrimary(s.acceleration, true);
      for (uint32_t read = 1; read != ANCHORED_READS; ++read) {
        for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.acceleration[n];
        const auto again = assemble(s.evaluated, R(0));
        elastic = again.energy;
        report->yielding = again.yielding;
        balance(&s.acceleration);
        std::fill(s.increment.begin(), s.increment.end(), V3<R>());
        solvePrimary(s.increment, false);
        for (uint32_t n = 0; n < V; ++n)
          if (!s.anchored[n]) s.acceleration[n] += s.increment[n];
      }
    } else {  // solver.cc:3951-4250
      const R travel = rule.beta * inner * inner;
      uint32_t spent = 0;
      bool linearAllowed = true;
      for (;;) {
        std::fill(s.total.begin(), s.total.end(), V3<R>());
        double accepted = std::numeric_limits<double>::infinity();
        double opening = 0.0;
        double lowest = std::numeric_limits<double>::infinity();
        uint32_t loadingBefore = 0, solves = 0;
        bool converged = false, predictorUnloaded = false, handedOff = false;
        for (uint32_t attempt = 0; attempt != plasticCap; ++attempt) {
          if (attempt < 2u) s.bindStiffness(attempt != 0u, anyYields);
          for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.total[n];
          const auto assembled = assemble(s.evaluated, R(LOADING_MARGIN));
          elastic = assembled.energy;
          report->yielding = assembled.yielding;
          ++report->plastic_evaluations;
          balance(&s.total);
          const double squared = rightSquared();
          if (attempt != 0u) {
            const double ranked = std::isfinite(squared) ? squared : std::numeric_limits<double>::infinity();
            const bool lowestIsLast = attempt == 1u || ranked < lowest;
            if (lowestIsLast) {
              lowest = ranked;
              s.lowestIterate = s.total;
            }
          }
          if (attempt == 0u) predictorUnloaded = assembled.loading == 0u;
          if (attempt == 1u && linearAllowed && predictorUnloaded && std::isfinite(squared) && squared > accepted) {
            ++report->plastic_linear_reads;
            s.bindStiffness(false, anyYields);
            for (uint32_t read = 1; read != ANCHORED_READS; ++read) {
              for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.total[n];
              const auto reread = assemble(s.evaluated, R(LOADING_MARGIN));
              elastic = reread.energy;
              report->yielding = reread.yielding;
              ++report->plastic_evaluations;
              if (reread.loading != 0u) {
                handedOff = true;
                break;
              }
              balance(&s.total);
              std::fill(s.increment.begin(), s.increment.end(), V3<R>());
              const auto solved = solvePrimary(s.increment, false);
              spent += solved.iterations;
              ++solves;
              for (uint32_t n = 0; n < V; ++n)
                if (!s.anchored[n]) s.total[n] += s.increment[n];
            }
            converged = !handedOff;
            break;
          }
          if (attempt != 0u && !(squared <= accepted)) {
            for (uint32_t n = 0; n < V; ++n) {
              s.increment[n] *= R(0.5);
              s.total[n] -= s.increment[n];
            }
            ++report->plastic_backtracks;
            continue;
          }
          if (attempt != 0u && loadingBefore == 0u && assembled.loading == 0u) {
            converged = true;
            break;
          }
          opening = attempt == 0u ? squared : opening;
          accepted = squared;
          loadingBefore = assembled.loading;
          if (attempt == 0u) s.increment = s.acceleration;
          else std::fill(s.increment.begin(), s.increment.end(), V3<R>());
          const auto solved = solvePrimary(s.increment, attempt == 0u);
          spent += solved.iterations;
          ++solves;
          R moved = 0, extent = 0;
          for (uint32_t n = 0; n < V; ++n) {
            if (s.anchored[n]) {
              s.increment[n] = V3<R>();
              continue;
            }
            s.total[n] += s.increment[n];
            moved = std::max(moved, length(s.increment[n]));
            extent = std::max(extent, length(s.evaluated[n]));
          }
          if (solves > 1u && travel * moved <= R(PLASTIC_RESOLUTION) * R(std::numeric_limits<float>::epsilon()) * extent) {
            converged = true;
            break;
          }
        }
        report->plastic_solves += solves;
        if (handedOff) {
          ++report->plastic_handoffs;
          linearAllowed = false;
          continue;
        }
        if (!converged) {
          s.bindStiffness(false, anyYields);
          std::fill(s.total.begin(), s.total.end(), V3<R>());
          bool fellBack = true;
          for (uint32_t read = 0; read != ANCHORED_READS; ++read) {
            for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.total[n];
            const auto reread = assemble(s.evaluated, R(LOADING_MARGIN), read != 0u);
            elastic = reread.energy;
            report->yielding = reread.yielding;
            ++report->plastic_evaluations;
            if (reread.loading != 0u) {
              fellBack = false;
              break;
            }
            balance(&s.total);
            if (read == 0u) s.increment = s.acceleration;
            else std::fill(s.increment.begin(), s.increment.end(), V3<R>());
            const auto solved = solvePrimary(s.increment, read == 0u);
            spent += solved.iterations;
            ++report->plastic_solves;
            for (uint32_t n = 0; n < V; ++n)
              if (!s.anchored[n]) s.total[n] += s.increment[n];
          }
          if (fellBack) {
            for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.total[n];
            const auto reread = assemble(s.evaluated, R(LOADING_MARGIN));
            elastic = reread.energy;
            report->yielding = reread.yielding;
            ++report->plastic_evaluations;
            balance(&s.total);
            const double squared = rightSquared();
            fellBack = reread.loading == 0u && squared <= PLASTIC_REDUCTION * PLASTIC_REDUCTION * opening;
          }
          if (fellBack) {
            ++report->plastic_fallbacks;
            converged = true;
          } else {
            ++report->plastic_fallback_rejections;
            s.bindStiffness(true, anyYields);
            s.total = s.lowestIterate;
            for (uint32_t n = 0; n < V; ++n) s.evaluated[n] = s.weighted[n] + reach * s.total[n];
            const auto again = assemble(s.evaluated, R(LOADING_MARGIN));
            elastic = again.energy;
            report->yielding = again.yielding;
            ++report->plastic_evaluations;
            balance(&s.total);
            const double remaining = std::sqrt(lowest);
            if (remaining >= report->plastic_worst_residual) report->plastic_worst_residual = remaining;
          }
        }
        report->plastic_capped += converged ? 0u : 1u;
        s.acceleration = s.total;
        break;
      }
    }
    if (solver) {  // solver.cc:4258-4263
      ++solver->stats.substeps_since_refresh;
      solver->meanIterations = 0.9f * solver->meanIterations + 0.1f * float(passIterations);
    }
    const R spanned = rule.beta * inner * inner;
    if (floating) {
      // solver.cc:4265-4340: back from the frame.  The frame's end turn
      // carries the nodes' frame positions and velocities to the world, the
      // centre moves on its own generalized-alpha path, and with the
      // Projected split the body's angular momentum and torque are restored
      // to the frame's rigid values.
      V3<double> stray;
      double weight = 0.0;
      for (uint32_t n = 0; n < V; ++n) {
        weight += double(s.mass[n]);
        stray += double(s.mass[n]) * widen(s.acceleration[n]);
      }
      const V3<R> mean = narrow<R>(V3<double>(stray.x / weight, stray.y / weight, stray.z / weight));
      const V3<R> spin = body.endSpin;
      M3<double> inertia(0.0);
      V3<double> momentum, torque;
      for (uint32_t n = 0; n < V; ++n) {
        const V3<R> turned = s.acceleration[n] - mean;
        const V3<R> placed = body.turn * (s.shifted[n] + spanned * turned);
        const V3<R> moved = body.turn * (relative[n] + inner * ((R(1) - rule.gamma) * s.carried[n] + rule.gamma * turned));
        const V3<R> reached = body.nextCentre + placed;
        const V3<R> acc = body.nextAcceleration + cross(body.endRate, placed) + cross(spin, cross(spin, placed)) +
                          R(2) * cross(spin, moved) + body.turn * turned;
        unconstrained[n] = body.nextVelocity + cross(spin, placed) + moved;
        s.acceleration[n] = acc;
        s.shifted[n] = reached - spanned * acc;
        relative[n] = placed;
        const double m = double(s.mass[n]);
        const V3<double> arm = widen(placed);
        inertia = inertia + m * (dot(arm, arm) * M3<double>(1.0) - outer(arm, arm));
        momentum += m * cross(arm, widen(unconstrained[n] - body.nextVelocity));
        torque += m * cross(arm, widen(acc - body.nextAcceleration));
      }
      if (settings->rigid_split == 2u && determinant(inertia) > 0.0) {  // RigidSplit::Projected
        const M3<double> inv = inverse(inertia);
        const V3<R> restore = narrow<R>(inv * (widen(body.momentum) - momentum));
        const V3<R> settle = narrow<R>(inv * (widen(body.torque) - torque));
        for (uint32_t n = 0; n < V; ++n) {
          const V3<R> turning = cross(settle, relative[n]);
          unconstrained[n] += cross(restore, relative[n]);
          s.acceleration[n] += turning;
          s.shifted[n] -= spanned * turning;
        }
      }
      for (uint32_t n = 0; n < V; ++n) s.velocity[n] = unconstrained[n];
      for (uint32_t e = 0; e < T; ++e) s.rotation[e] = body.turn * s.rotation[e];
    } else {
      // solver.cc:4341-4358 velocity
      for (uint32_t n = 0; n < V; ++n) {
        if (s.anchored[n]) continue;
        s.velocity[n] = s.velocity[n] + inner * ((R(1) - rule.gamma) * s.carried[n] + rule.gamma * s.acceleration[n]);
      }
    }
    // solver.cc:5829-5849 position
    for (uint32_t n = 0; n < V; ++n) {
      if (s.anchored[n]) {
        s.velocity[n] = s.prescribed[n];
        s.acceleration[n] = V3<R>();
        s.position[n] = s.position[n] + inner * s.prescribed[n];
        continue;
      }
      s.position[n] = s.shifted[n] + spanned * s.acceleration[n];
    }
    // solver.cc:5860-5861
    if (!s.hencky) plasticGrowth = s.commitPlastic(mode) || plasticGrowth;
  }
  // strainstep.cc:822-825: flowLattice once per step, after the solve
  if (anyFlows) {
    uint32_t flowed = 0;
    for (uint32_t e = 0; e < T; ++e) {
      const Element<R>& el = s.elements[e];
      if (!el.yields) continue;
      std::array<V3<double>, 4> x;
      for (int k = 0; k < 4; ++k) {
        const V3<R>& p = s.position[el.nodes[k]];
        x[k] = V3<double>(double(p.x), double(p.y), double(p.z));
      }
      const double mu = double(el.moduli.second), bulk = double(el.moduli.first) + 2.0 * mu / 3.0;
      if (henckyFlow(deformationOf(x, s.authored[e]), s.flowMap[e], s.hardeningOf[e], mu, bulk,
                     double(el.yieldStress), double(el.hardening), el.limits))
        ++flowed;
    }
    report->yielding = flowed;
    plasticGrowth = plasticGrowth || flowed != 0u;
  }
  // solver.cc:5874-5882
  R kinetic = 0;
  for (uint32_t n = 0; n < V; ++n) kinetic += R(0.5) * s.mass[n] * dot(s.velocity[n], s.velocity[n]);
  report->kinetic_energy += double(kinetic);
  report->elastic_energy += double(elastic);
  report->plastic_growth |= plasticGrowth ? 1u : 0u;
  bool finite = true;
  for (uint32_t n = 0; n < V; ++n) {
    for (int k = 0; k < 3; ++k) {
      st->position[3 * n + k] = double(s.position[n][k]);
      st->velocity[3 * n + k] = double(s.velocity[n][k]);
      st->acceleration[3 * n + k] = double(s.acceleration[n][k]);
      finite = finite && std::isfinite(st->position[3 * n + k]);
    }
  }
  report->non_finite |= finite ? 0u : 1u;
  for (uint32_t e = 0; e < T; ++e) {
    storeRowMajor(s.rotation[e], st->rotation + 9 * e);
    if (s.hencky) {
      storeRowMajor(s.flowMap[e], st->plastic + 10 * e);
      st->plastic[10 * e + 9] = s.hardeningOf[e];
      continue;
    }
    storeRowMajor(s.plastic[e].strain, st->plastic + 10 * e);
    st->plastic[10 * e + 9] = double(s.plastic[e].equivalent);
  }
  report->seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - began).count();
  return 0;
}

template <class R> std::array<V3<R>, 4> corners(const double* a) {
  return {V3<R>(R(a[0]), R(a[1]), R(a[2])), V3<R>(R(a[3]), R(a[4]), R(a[5])), V3<R>(R(a[6]), R(a[7]), R(a[8])),
          V3<R>(R(a[9]), R(a[10]), R(a[11]))};
}
template <class R> void storeCorners(const std::array<V3<R>, 4>& f, double* out) {
  for (int n = 0; n < 4; ++n)
    for (int k = 0; k < 3; ++k) out[3 * n + k] = double(f[n][k]);
}
template <class R> void storeBlocks(const std::array<M3<R>, 16>& blocks, double* out) {
  for (int row = 0; row < 4; ++row)
    for (int col = 0; col < 4; ++col)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[(3 * row + i) * 12 + 3 * col + j] = double(blocks[row * 4 + col][j][i]);
}

template <class R>
int tetPointTrialImpl(const double* deformed, const double* rest, const double* rinv, double volume, const or_material* m,
                      const double* committed, double margin, int mode, int mapping, double* force, double* rotation,
                      double* plastic, double* tangent, double* scalars) {
  PlasticPoint<R> p;
  p.strain = loadRowMajor<R>(committed);
  p.equivalent = R(committed[9]);
  const auto t = tetPointTrial(corners<R>(deformed), corners<R>(rest), loadRowMajor<R>(rinv), R(volume),
                               lame(R(m->youngs_modulus), R(m->poissons_ratio)), R(m->yield_stress),
                               R(m->hardening_modulus), p, R(margin), mode, mapping != 0, tangent != nullptr);
  storeCorners(t.force, force);
  storeRowMajor(t.rotation, rotation);
  storeRowMajor(t.point.strain, plastic);
  plastic[9] = double(t.point.equivalent);
  if (tangent) storeBlocks(t.tangent.block, tangent);
  scalars[0] = double(t.energy);
  scalars[1] = double(t.plasticWork);
  scalars[2] = double(t.yielding);
  scalars[3] = double(t.loading);
  return 0;
}

template <class R>
int tetTrialImpl(const double* deformed, const double* rest, const double* rinv, double volume, const or_material* m,
                 int mode, double* force, double* rotation, double* energy) {
  const auto k = tetStiffness(loadRowMajor<R>(rinv), R(volume), lame(R(m->youngs_modulus), R(m->poissons_ratio)));
  const auto t = trial(corners<R>(deformed), corners<R>(rest), loadRowMajor<R>(rinv), k, mode);
  storeCorners(t.force, force);
  storeRowMajor(t.rotation, rotation);
  *energy = double(t.energy);
  return 0;
}

template <class R>
int snhImpl(const double* deformed, const double* rest, const double* rinv, double volume, const or_material* m,
            double* force, double* energy, double* hessian) {
  const M3<R> ri = loadRowMajor<R>(rinv);
  const Lame<R> moduli = lame(R(m->youngs_modulus), R(m->poissons_ratio));
  const auto s = snhTet(corners<R>(deformed), corners<R>(rest), ri, R(volume), moduli);
  storeCorners(s.force, force);
  *energy = double(s.energy);
  if (hessian) {  // column (3 b + i) = K e_{b,i}
    std::array<M3<R>, 16> blocks;
    for (int b = 0; b < 4; ++b)
      for (int i = 0; i < 3; ++i) {
        std::array<V3<R>, 4> unit{}, col{};
        unit[b][i] = R(1);
        snhApply(unit, ri, R(volume), moduli, s.gradient, s.change, col);
        for (int a = 0; a < 4; ++a) blocks[a * 4 + b][i] = col[a];
      }
    storeBlocks(blocks, hessian);
  }
  return 0;
}

// solver.cc:17-24
constexpr uint32_t KUHN[6][4] = {{0, 1, 3, 7}, {0, 3, 2, 7}, {0, 2, 6, 7}, {0, 6, 4, 7}, {0, 4, 5, 7}, {0, 5, 1, 7}};

}  // namespace

template <class R>
int dampingImpl(const double* at, const double* rotation, const double* rinv, double volume, const or_material* m,
                const double* direction, double* out) {
  const TetStiffness<R> k = tetStiffness(loadRowMajor<R>(rinv), R(volume), lame(R(m->youngs_modulus), R(m->poissons_ratio)));
  std::array<V3<R>, 4> result;
  applyDamping(rigidFit(corners<R>(at)), loadRowMajor<R>(rotation), k, corners<R>(direction), result);
  storeCorners(result, out);
  return 0;
}

extern "C" {

int or_grid_counts(const or_grid* grid, uint32_t* nodes, uint32_t* tets) {
  const uint64_t cx = grid->cells[0], cy = grid->cells[1], cz = grid->cells[2];
  if (cx == 0 || cy == 0 || cz == 0) return -1;
  *nodes = uint32_t((cx + 1) * (cy + 1) * (cz + 1));
  *tets = uint32_t(6 * cx * cy * cz);
  return 0;
}

// solver.cc:2185-2418 buildMesh, for a lattice whose every cell is solid with
// fill 1: nodes numbered by first use in x-fastest cell order, 6 Kuhn tets per
// cell with nodes 1 and 2 swapped when the rest determinant is negative,
// volume det/6, Dm^-1 = inverse(shape), lumped mass rho V / 4 per corner.
// Rest positions are rounded to float like the reference's glm::vec3.
int or_grid_build(const or_grid* grid, double* rest, double* node_mass, uint8_t* anchored, uint32_t* tet_nodes,
                  double* rest_inverse, double* volume, uint32_t* lane, uint32_t* grid_index) {
  uint32_t V = 0, T = 0;
  if (or_grid_counts(grid, &V, &T) != 0) return -1;
  const uint32_t cx = grid->cells[0], cy = grid->cells[1], cz = grid->cells[2];
  const uint32_t rx = cx + 1, ry = cy + 1;
  std::vector<uint32_t> nodeOf(size_t(rx) * ry * (cz + 1), UINT32_MAX);
  std::vector<std::array<uint32_t, 3>> at(V);
  uint32_t made = 0;
  for (uint32_t z = 0; z < cz; ++z)
    for (uint32_t y = 0; y < cy; ++y)
      for (uint32_t x = 0; x < cx; ++x)
        for (uint32_t c = 0; c < 8; ++c) {
          const uint32_t i = x + (c & 1u), j = y + ((c >> 1) & 1u), k = z + ((c >> 2) & 1u);
          const size_t sample = i + size_t(rx) * (j + size_t(ry) * k);
          if (nodeOf[sample] != UINT32_MAX) continue;
          nodeOf[sample] = made;
          at[made] = {i, j, k};
          if (grid_index) grid_index[made] = uint32_t(sample);
          ++made;
        }
  for (uint32_t n = 0; n < V; ++n) {
    for (int a = 0; a < 3; ++a) {
      // counter-based splitmix64 (Steele, Lea, Flood 2014) of draw 3 n + a
      uint64_t z = grid->seed + (uint64_t(3) * n + uint64_t(a) + 1u) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      const double u = double(z >> 11) * (1.0 / 9007199254740992.0);
      const double offset = (2.0 * u - 1.0) * grid->jitter * grid->voxel;
      rest[3 * n + a] = double(float(grid->origin[a] + grid->voxel * double(at[n][a]) + offset));
    }
    const uint32_t cells_on_axis = grid->cells[grid->anchor_axis < 3 ? grid->anchor_axis : 0];
    anchored[n] = grid->anchor_axis < 3 &&
                          at[n][grid->anchor_axis] == (grid->anchor_side == 0 ? 0u : cells_on_axis)
                      ? 1u
                      : 0u;
    node_mass[n] = 0.0;
  }
  uint32_t t = 0;
  for (uint32_t z = 0; z < cz; ++z)
    for (uint32_t y = 0; y < cy; ++y)
      for (uint32_t x = 0; x < cx; ++x) {
        uint32_t cornersOf[8];
        for (uint32_t c = 0; c < 8; ++c) {
          const uint32_t i = x + (c & 1u), j = y + ((c >> 1) & 1u), k = z + ((c >> 2) & 1u);
          cornersOf[c] = nodeOf[i + size_t(rx) * (j + size_t(ry) * k)];
        }
        for (const auto& pick : KUHN) {
          uint32_t nodes[4] = {cornersOf[pick[0]], cornersOf[pick[1]], cornersOf[pick[2]], cornersOf[pick[3]]};
          auto shapeOf = [&]() {
            const V3<double> x0(rest[3 * nodes[0]], rest[3 * nodes[0] + 1], rest[3 * nodes[0] + 2]);
            M3<double> m;
            for (int q = 1; q < 4; ++q)
              m[q - 1] = V3<double>(rest[3 * nodes[q]], rest[3 * nodes[q] + 1], rest[3 * nodes[q] + 2]) - x0;
            return m;
          };
          M3<double> shape = shapeOf();
          if (determinant(shape) < 0.0) {
            std::swap(nodes[1], nodes[2]);
            shape = shapeOf();
          }
          const double vol = determinant(shape) / 6.0;
          if (vol <= 0.0) continue;
          const M3<double> inv = inverse(shape);
          for (int q = 0; q < 4; ++q) tet_nodes[4 * t + q] = nodes[q];
          storeRowMajor(inv, rest_inverse + 9 * t);
          volume[t] = vol;
          lane[t] = 0;
          for (int q = 0; q < 4; ++q) node_mass[nodes[q]] += grid->density * vol * 0.25;
          ++t;
        }
      }
  return int(t == T ? 0 : -1);
}

int or_step_solver(int precision, const or_mesh* mesh, or_state* state, const or_material* materials, uint32_t lanes,
                   const or_settings* settings, const double gravity[3], double dt, or_report* report,
                   or_solver* solver) {
  if (!mesh || !state || !settings || !report) return -1;
  return precision == OR_F32 ? stepImpl<float>(mesh, state, materials, lanes, settings, gravity, dt, report, solver)
                             : stepImpl<double>(mesh, state, materials, lanes, settings, gravity, dt, report, solver);
}

int or_step(int precision, const or_mesh* mesh, or_state* state, const or_material* materials, uint32_t lanes,
            const or_settings* settings, const double gravity[3], double dt, or_report* report) {
  return or_step_solver(precision, mesh, state, materials, lanes, settings, gravity, dt, report, nullptr);
}

or_solver* or_solver_create(uint32_t factor_budget) {
  or_solver* s = new or_solver();
  s->budget = factor_budget;
  return s;
}

void or_solver_destroy(or_solver* solver) { delete solver; }

int or_solver_get_stats(const or_solver* solver, or_solver_stats* out) {
  if (!solver || !out) return -1;
  *out = solver->stats;
  out->mean_iterations = double(solver->meanIterations);
  out->rows = 3u * solver->nodes;
  out->ready = solver->ready ? 1u : 0u;
  out->system_nonzeros = solver->systemNonZeros;
  out->generation = solver->born;
  return 0;
}

int or_tet_point_trial(int precision, const double* deformed, const double* rest, const double* rest_inverse,
                       double volume, const or_material* material, const double* committed_plastic, double margin,
                       int rotation_mode, int return_mapping, double* force, double* rotation, double* plastic,
                       double* tangent, double* scalars) {
  return precision == OR_F32
             ? tetPointTrialImpl<float>(deformed, rest, rest_inverse, volume, material, committed_plastic, margin,
                                        rotation_mode, return_mapping, force, rotation, plastic, tangent, scalars)
             : tetPointTrialImpl<double>(deformed, rest, rest_inverse, volume, material, committed_plastic, margin,
                                         rotation_mode, return_mapping, force, rotation, plastic, tangent, scalars);
}

int or_tet_trial(int precision, const double* deformed, const double* rest, const double* rest_inverse, double volume,
                 const or_material* material, int rotation_mode, double* force, double* rotation, double* energy) {
  return precision == OR_F32 ? tetTrialImpl<float>(deformed, rest, rest_inverse, volume, material, rotation_mode, force,
                                                   rotation, energy)
                             : tetTrialImpl<double>(deformed, rest, rest_inverse, volume, material, rotation_mode,
                                                    force, rotation, energy);
}

int or_snh_tet(int precision, const double* deformed, const double* rest, const double* rest_inverse, double volume,
               const or_material* material, double* force, double* energy, double* hessian_blocks) {
  return precision == OR_F32
             ? snhImpl<float>(deformed, rest, rest_inverse, volume, material, force, energy, hessian_blocks)
             : snhImpl<double>(deformed, rest, rest_inverse, volume, material, force, energy, hessian_blocks);
}

int or_damping_apply(int precision, const double* corners, const double* rotation, const double* rest_inverse,
                     double volume, const or_material* material, const double* direction, double* out) {
  return precision == OR_F32 ? dampingImpl<float>(corners, rotation, rest_inverse, volume, material, direction, out)
                             : dampingImpl<double>(corners, rotation, rest_inverse, volume, material, direction, out);
}

int or_rotation(int precision, const double* gradient, int rotation_mode, double* out) {
  if (precision == OR_F32) storeRowMajor(elementRotation(loadRowMajor<float>(gradient), rotation_mode), out);
  else storeRowMajor(elementRotation(loadRowMajor<double>(gradient), rotation_mode), out);
  return 0;
}

int or_hencky_return(const double* elastic, double shear, double yield_stress, double* returned, double* strain,
                     double* trial) {
  const HenckyReturn r = henckyReturn(loadRowMajor<double>(elastic), shear, yield_stress);
  if (!r.mapped) return 0;
  storeRowMajor(r.elastic, returned);
  *strain = r.strain;
  *trial = r.trial;
  return 1;
}

double or_hencky_von_mises(const double* elastic, double shear) {
  return henckyVonMises(loadRowMajor<double>(elastic), shear);
}

int or_hencky_flow(const double* deformation, double* plastic, double* hardening, double shear, double bulk,
                   const or_material* material) {
  M3<double> p = loadRowMajor<double>(plastic);
  const FlowLimits limits{material->crush_stress, material->crush_limit, material->plastic_max};
  const bool changed = henckyFlow(loadRowMajor<double>(deformation), p, *hardening, shear, bulk, material->yield_stress,
                                  material->hardening_modulus, limits);
  storeRowMajor(p, plastic);
  return changed ? 1 : 0;
}

}  // extern "C"
