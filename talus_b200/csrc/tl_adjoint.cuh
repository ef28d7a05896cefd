// tl_adjoint.cuh -- kernels of the hand-written adjoint of the elastic step.
//
// One step (one substep of length h) of the forward maps (x, v, a) to
// (x', v', a') through
//   w  = x + (1 - alpha_f)(h v + c a),                c = (1/2 - beta) h^2
//   A  solves  R(A) = f(w + rho A) + M g - alpha_m M a - (1 - alpha_m) M A = 0
//              on free nodes (A = 0 on anchored ones), rho = h_eff^2
//   x' = x + h v + c a + beta h^2 A,  v' = v + h (1 - gamma) a + h gamma A,  a' = A
// (free nodes; anchored ones take x' = x + h v_p, v' = v_p, a' = 0).  With
// J = (1 - alpha_m) M + rho K, K = -df/dy symmetric (the exact neo-Hookean
// tangent), the implicit-function theorem gives the step's vector-Jacobian
// product for output cotangents (x', v', a')-bar:
//   solve  J lam = beta h^2 x'bar + h gamma v'bar + a'bar      (free nodes)
//   wbar = -K lam                                               (all nodes)
//   xbar = x'bar + wbar
//   vbar = h x'bar + v'bar + (1 - alpha_f) h wbar                (anchored: (1 - alpha_f) h wbar)
//   abar = c x'bar + h (1 - gamma) v'bar + (1 - alpha_f) c wbar - alpha_m M lam
//                                                               (anchored: (1 - alpha_f) c wbar)
//   Ebar_e += (df/dE_e)^T lam = sum_corners f_e,c . lam_c / E_e  (f_e is linear in E_e)
// K lam is formed by the element operator the PCG uses, evaluated at the
// converged point y = w + rho A, so rho K lam comes out directly.
#pragma once

namespace tl {

// Right side of the adjoint solve.
template <class S>
__global__ void __launch_bounds__(TILE)
    kAdjointRight(Sys<S> s, const Vec4<S>* xb, const Vec4<S>* vb, const Vec4<S>* ab) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  if (s.anch[n]) {
    s.right[n] = Vec4<S>{0, 0, 0, 0};
    return;
  }
  const BodyStepDev& st = s.step[b];
  const double h = st.inner;
  const V3<double> r = (st.beta * h * h) * cvt<double>(xyz(xb[n])) + (h * st.gamma) * cvt<double>(xyz(vb[n])) +
                       cvt<double>(xyz(ab[n]));
  s.right[n] = packc<S>(r);
}

// Per element: the products y_e = rho K_e lam_e of the matvec operator, and the
// Young's-modulus cotangent from the element forces of the same pass.
template <class S, int LAW>
__global__ void __launch_bounds__(TILE) kAdjointElement(Sys<S> s, const Vec4<S>* lam, double* ebar) {
  const uint32_t tile = blockIdx.x, b = s.elem_tile_body[tile];
  const uint32_t e = tile * TILE + threadIdx.x;
  if (e >= s.body[b].elem_end) return;
  const uint4 t = __ldg(&s.tet[e]);
  const uint32_t nodes[4] = {t.x, t.y, t.z, t.w};
  V3<S> p[4], y[4];
  double eb = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const Vec4<S> l = lam[nodes[c]];
    p[c] = xyz(l);
    const Vec4<S> f = s.fe[size_t(c) * s.Tp + e];
    eb += double(f.x) * double(l.x) + double(f.y) * double(l.y) + double(f.z) * double(l.z);
  }
  elementApply<S, LAW, false>(s, e, p, y);
#pragma unroll
  for (int c = 0; c < 4; ++c) s.ye[4 * e + c] = pack(y[c]);
  const MatDev m = s.mat[s.lane[e]];
  const double youngs = s.eyoung ? s.eyoung[e] : m.youngs;
  if (youngs != 0.0) ebar[e] += eb / youngs;
}

// Node gather of rho K lam in element order (the CSR of the assembly) and the
// cotangent update of (x, v, a) in place.
template <class S>
__global__ void __launch_bounds__(TILE)
    kAdjointNode(Sys<S> s, const Vec4<S>* lam, Vec4<S>* xb, Vec4<S>* vb, Vec4<S>* ab) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  const BodyStepDev& st = s.step[b];
  V3<double> q = {0, 0, 0};
  const uint32_t k0 = s.start[n], k1 = s.start[n + 1];
  for (uint32_t k = k0; k < k1; ++k) q = q + cvt<double>(xyz(s.ye[__ldg(&s.entry[k])]));
  const V3<double> wb = (-1.0 / st.scale) * q;
  const double h = st.inner, c = st.carry, keep = 1.0 - st.alpha_f;
  const V3<double> x1 = cvt<double>(xyz(xb[n]));
  if (s.anch[n]) {
    xb[n] = packc<S>(x1 + wb);
    vb[n] = packc<S>((keep * h) * wb);
    ab[n] = packc<S>((keep * c) * wb);
    return;
  }
  const V3<double> v1 = cvt<double>(xyz(vb[n]));  // a'bar reached lam through the right side
  const double mass = double(s.rest4[n].w);
  const V3<double> l = cvt<double>(xyz(lam[n]));
  xb[n] = packc<S>(x1 + wb);
  vb[n] = packc<S>(h * x1 + v1 + (keep * h) * wb);
  ab[n] = packc<S>(c * x1 + (h * (1.0 - st.gamma)) * v1 + (keep * c) * wb - (st.alpha_m * mass) * l);
}

// Internal node forces of the last element pass, gathered in element order.
template <class S>
__global__ void __launch_bounds__(TILE) kGatherForces(Sys<S> s, double* out) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  const uint32_t n = tile * TILE + threadIdx.x;
  if (n >= s.body[b].node_end) return;
  double f[3] = {0, 0, 0};
  for (uint32_t k = s.start[n], k1 = s.start[n + 1]; k < k1; ++k) {
    const Vec4<S> a = s.fe[cornerAt(__ldg(&s.entry[k]), s.Tp)];
    f[0] += double(a.x);
    f[1] += double(a.y);
    f[2] += double(a.z);
  }
  out[3 * size_t(n)] = f[0];
  out[3 * size_t(n) + 1] = f[1];
  out[3 * size_t(n) + 2] = f[2];
}

// Per-element E from the element's material lane (the start of an override).
template <class S>
__global__ void __launch_bounds__(TILE) kLaneYoungs(Sys<S> s, double* youngs) {
  const uint32_t e = blockIdx.x * TILE + threadIdx.x;
  if (e < s.Tp) youngs[e] = s.mat[s.lane[e]].youngs;
}

}  // namespace tl
