// tl_floating.cuh -- the floating-body frame of the tet FEM step.
//
// A body with no anchored node, stepped with the rigid split on (floats,
// solver.cc:2964-2971), is solved in a frame that moves with its centre of
// mass and turns with its rigid spin:
//   * floatingFrame (solver.cc:3031-3142): centre, mean velocity and
//     acceleration, inertia, angular momentum and torque about the centre;
//     the centre's generalized-alpha step; the torque-free spin advanced by
//     classic Runge-Kutta (rigidAdvance, solver.cc:2983-3036) to the weighted
//     time and to the end of the substep;
//   * the predictor and the drive of centrifugal, Euler and Coriolis forces
//     (solver.cc:3662-3690) are in kPredict, the drive enters the right side
//     in kNodeAssemble;
//   * back to the world at the substep end (solver.cc:4265-4340): the frame
//     acceleration loses its mean, the end turn carries arms and velocities
//     to the world, and with RigidSplit::Projected the body's angular
//     momentum and torque are restored to the frame's rigid values (kFrameEnd,
//     then kUpdate applies the corrections and the position).
// Every sum over nodes is FP64: per-tile partials in a fixed order, then the
// body's tiles in tile order (one block per body), like the PCG reductions.
// The frame itself is FP64 in both precisions.
#pragma once

#include "tl_kernels.cuh"

namespace tl {

__device__ __forceinline__ V3<double> ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double* p, V3<double> v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}

// Moments of inertia sum m (|r|^2 I - r r^T), stored (xx, yy, zz, xy, xz, yz).
__device__ __forceinline__ void addInertia(double* out, double m, V3<double> r) {
  const double rr = dot(r, r);
  out[0] += m * (rr - r.x * r.x);
  out[1] += m * (rr - r.y * r.y);
  out[2] += m * (rr - r.z * r.z);
  out[3] -= m * r.x * r.y;
  out[4] -= m * r.x * r.z;
  out[5] -= m * r.y * r.z;
}
__device__ __forceinline__ M3<double> inertiaOf(const double* k) {
  M3<double> i;
  i.m[0][0] = k[0];
  i.m[1][1] = k[1];
  i.m[2][2] = k[2];
  i.m[0][1] = i.m[1][0] = k[3];
  i.m[0][2] = i.m[2][0] = k[4];
  i.m[1][2] = i.m[2][1] = k[5];
  return i;
}

// Per node tile partial sums over the floating bodies' nodes.
//   which 0: m, m u, m v, m a                         (10 values)
//   which 1: inertia, angular momentum and torque about the centre, of the
//            velocities and accelerations relative to the mean ones (12)
//   which 2: m, m a of the solved frame acceleration   (4)
template <class S>
__global__ void __launch_bounds__(TILE) kFrameMoments(Sys<S> s, uint32_t pass, uint32_t which) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass) || !s.step[b].floating) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  double v[FRAME_PART];
#pragma unroll
  for (int k = 0; k < FRAME_PART; ++k) v[k] = 0.0;
  if (n < s.body[b].node_end) {
    const Vec4<S> rest = s.rest4[n];
    const double m = double(rest.w);
    const V3<double> u = cvt<double>(xyz(s.u[n])), vel = cvt<double>(xyz(s.v[n])), acc = cvt<double>(xyz(s.a[n]));
    if (which == 0u) {
      v[0] = m;
      v[1] = m * u.x;
      v[2] = m * u.y;
      v[3] = m * u.z;
      v[4] = m * vel.x;
      v[5] = m * vel.y;
      v[6] = m * vel.z;
      v[7] = m * acc.x;
      v[8] = m * acc.y;
      v[9] = m * acc.z;
    } else if (which == 1u) {
      const FrameDev& f = s.frame[b];
      const V3<double> arm = cvt<double>(xyz(rest)) - ld3(f.rest_centre) + (u - ld3(f.shift));
      addInertia(v, m, arm);
      const V3<double> h = m * cross(arm, vel - ld3(f.velocity));
      const V3<double> t = m * cross(arm, acc - ld3(f.acceleration));
      v[6] = h.x;
      v[7] = h.y;
      v[8] = h.z;
      v[9] = t.x;
      v[10] = t.y;
      v[11] = t.z;
    } else {
      v[0] = m;
      v[1] = m * acc.x;
      v[2] = m * acc.y;
      v[3] = m * acc.z;
    }
  }
  blockSum<FRAME_PART>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < FRAME_PART; ++k) s.fpart[size_t(tile) * FRAME_PART + k] = v[k];
}

// rigidRate (solver.cc:2983-2987): d(momentum) = m x w, d(turn) = turn skew(w),
// w = I^-1 m with the world inertia I fixed over the substep.
struct RigidMotionDev {
  V3<double> momentum;
  M3<double> turn;
};
__device__ inline RigidMotionDev rigidRateDev(const M3<double>& inv, const RigidMotionDev& at) {
  const V3<double> w = mul(inv, at.momentum);
  M3<double> k;  // skew(w): k v = w x v
  k.m[0][0] = 0.0;
  k.m[0][1] = -w.z;
  k.m[0][2] = w.y;
  k.m[1][0] = w.z;
  k.m[1][1] = 0.0;
  k.m[1][2] = -w.x;
  k.m[2][0] = -w.y;
  k.m[2][1] = w.x;
  k.m[2][2] = 0.0;
  return RigidMotionDev{cross(at.momentum, w), mul(at.turn, k)};
}
__device__ inline RigidMotionDev movedBy(const RigidMotionDev& from, const RigidMotionDev& rate, double by) {
  RigidMotionDev r;
  r.momentum = from.momentum + by * rate.momentum;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.turn.m[i][j] = from.turn.m[i][j] + by * rate.turn.m[i][j];
  return r;
}
// rigidAdvance (solver.cc:2989-3026): `count` Runge-Kutta steps over `span`,
// then three passes turn <- (turn + turn^-T) / 2.
__device__ inline RigidMotionDev rigidAdvanceDev(const M3<double>& inv, RigidMotionDev motion, double span,
                                                 uint32_t count) {
  const double part = span / double(count);
  for (uint32_t at = 0; at != count; ++at) {
    const RigidMotionDev first = rigidRateDev(inv, motion);
    const RigidMotionDev second = rigidRateDev(inv, movedBy(motion, first, 0.5 * part));
    const RigidMotionDev third = rigidRateDev(inv, movedBy(motion, second, 0.5 * part));
    const RigidMotionDev fourth = rigidRateDev(inv, movedBy(motion, third, part));
    const double w = part / 6.0;
    motion.momentum =
        motion.momentum + w * (first.momentum + 2.0 * second.momentum + 2.0 * third.momentum + fourth.momentum);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        motion.turn.m[i][j] += w * (first.turn.m[i][j] + 2.0 * second.turn.m[i][j] + 2.0 * third.turn.m[i][j] +
                                    fourth.turn.m[i][j]);
  }
  for (uint32_t pass = 0; pass != 3u; ++pass) {
    const M3<double> back = inverse3(motion.turn);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) motion.turn.m[i][j] = 0.5 * (motion.turn.m[i][j] + back.m[j][i]);
  }
  return motion;
}

constexpr uint32_t RIGID_PARTS = 8u;  // Runge-Kutta steps per span (solver.h:109)

// One block per body: the body's tile partials summed in tile order, then
// (thread 0) the frame quantities of stage `which`:
//   0: centre shift, mean velocity and acceleration;
//   1: the frame of the substep (floatingFrame, solver.cc:3095-3141);
//   2: the mean of the solved frame acceleration (solver.cc:4266-4276);
//   3: the Projected split's restore and settle spins (solver.cc:4318-4329),
//      zero otherwise or when the inertia is singular.
template <class S>
__global__ void __launch_bounds__(TILE) kFrameSolve(Sys<S> s, uint32_t pass, uint32_t which) {
  const uint32_t b = blockIdx.x;
  if (!bodyActive(s, b, pass) || !s.step[b].floating) return;
  const BodyDev bd = s.body[b];
  double sum[FRAME_PART];
#pragma unroll
  for (int k = 0; k < FRAME_PART; ++k) sum[k] = 0.0;
  for (uint32_t t = bd.node_tile_begin + threadIdx.x; t < bd.node_tile_end; t += TILE)
#pragma unroll
    for (int k = 0; k < FRAME_PART; ++k) sum[k] += __ldcg(s.fpart + size_t(t) * FRAME_PART + k);
  blockSum<FRAME_PART>(sum);
  if (threadIdx.x != 0) return;
  FrameDev& f = s.frame[b];
  const BodyStepDev& st = s.step[b];
  if (which == 0u) {
    const double total = sum[0];
    f.mass = total;
    st3(f.shift, V3<double>{sum[1] / total, sum[2] / total, sum[3] / total});
    st3(f.velocity, V3<double>{sum[4] / total, sum[5] / total, sum[6] / total});
    st3(f.acceleration, V3<double>{sum[7] / total, sum[8] / total, sum[9] / total});
    return;
  }
  if (which == 1u) {
    const M3<double> inertia = inertiaOf(sum);
    const V3<double> momentum = {sum[6], sum[7], sum[8]}, torque = {sum[9], sum[10], sum[11]};
    const double h = st.inner, am = st.alpha_m, beta = st.beta, gamma = st.gamma;
    const V3<double> acc = ld3(f.acceleration), vel = ld3(f.velocity);
    const V3<double> g = {st.gx, st.gy, st.gz};
    const V3<double> num = g - am * acc;
    const V3<double> next = {num.x / (1.0 - am), num.y / (1.0 - am), num.z / (1.0 - am)};
    st3(f.next_acceleration, next);
    st3(f.next_shift, ld3(f.shift) + h * vel + (h * h) * ((0.5 - beta) * acc + beta * next));
    st3(f.next_velocity, vel + h * ((1.0 - gamma) * acc + gamma * next));
    st3(f.momentum, momentum + (h * (1.0 - gamma - gamma * am / (1.0 - am))) * torque);
    st3(f.torque, (-am / (1.0 - am)) * torque);
    const V3<double> zero = {0.0, 0.0, 0.0};
    st3(f.spin, zero);
    st3(f.spin_rate, zero);
    st3(f.weighted_spin, zero);
    st3(f.weighted_rate, zero);
    st3(f.end_spin, zero);
    st3(f.end_rate, zero);
    for (int k = 0; k < 9; ++k) f.turn[k] = (k % 4) == 0 ? 1.0 : 0.0;
    const double det = det3(inertia);
    const double scale = trace3(inertia);
    if (!(det > 1.0e-12 * scale * scale * scale) || dot(momentum, momentum) == 0.0) return;
    const M3<double> inv = inverse3(inertia);
    const double weighted = (1.0 - st.alpha_f) * h;
    const RigidMotionDev start{momentum, eye3<double>()};
    const RigidMotionDev middle = rigidAdvanceDev(inv, start, weighted, RIGID_PARTS);
    const RigidMotionDev end = rigidAdvanceDev(inv, middle, h - weighted, RIGID_PARTS);
    auto spinOf = [&](const RigidMotionDev& at) { return mul(inv, at.momentum); };
    auto rateOf = [&](const RigidMotionDev& at) { return mul(inv, cross(at.momentum, mul(inv, at.momentum))); };
    st3(f.spin, spinOf(start));
    st3(f.spin_rate, rateOf(start));
    st3(f.weighted_spin, spinOf(middle));
    st3(f.weighted_rate, rateOf(middle));
    st3(f.end_spin, mul(end.turn, spinOf(end)));
    st3(f.end_rate, mul(end.turn, rateOf(end)));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) f.turn[3 * i + j] = end.turn.m[i][j];
    return;
  }
  if (which == 2u) {
    st3(f.mean, V3<double>{sum[1] / sum[0], sum[2] / sum[0], sum[3] / sum[0]});
    return;
  }
  const V3<double> zero = {0.0, 0.0, 0.0};
  st3(f.restore, zero);
  st3(f.settle, zero);
  const M3<double> inertia = inertiaOf(sum);
  if (!st.projected || !(det3(inertia) > 0.0)) return;
  const M3<double> inv = inverse3(inertia);
  st3(f.restore, mul(inv, ld3(f.momentum) - V3<double>{sum[6], sum[7], sum[8]}));
  st3(f.settle, mul(inv, ld3(f.torque) - V3<double>{sum[9], sum[10], sum[11]}));
}

// Back to the world (solver.cc:4278-4315) for every node of a floating body:
// the frame acceleration less its mean, turned by the end turn, gives the
// world arm (placed), velocity and acceleration; the partials of inertia,
// angular momentum and torque about the end centre feed kFrameSolve stage 3.
// Leaves v = unconstrained velocity, a = world acceleration, relv = placed
// arm, shifted = reached - beta h^2 a (as a displacement).
template <class S>
__global__ void __launch_bounds__(TILE) kFrameEnd(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.node_tile_body[tile];
  if (!bodyActive(s, b, pass) || !s.step[b].floating) return;
  const uint32_t n = tile * TILE + threadIdx.x;
  double v[FRAME_PART];
#pragma unroll
  for (int k = 0; k < FRAME_PART; ++k) v[k] = 0.0;
  if (n < s.body[b].node_end) {
    const FrameDev& f = s.frame[b];
    const BodyStepDev& st = s.step[b];
    M3<double> turn;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) turn.m[i][j] = f.turn[3 * i + j];
    const Vec4<S> rest = s.rest4[n];
    const V3<double> restArm = cvt<double>(xyz(rest)) - ld3(f.rest_centre);
    const double spanned = st.beta * st.inner * st.inner;
    const V3<double> turned = cvt<double>(xyz(s.a[n])) - ld3(f.mean);
    const V3<double> placed = mul(turn, restArm + cvt<double>(xyz(s.shifted[n])) + spanned * turned);
    const V3<double> moved = mul(turn, cvt<double>(xyz(s.relv[n])) +
                                           st.inner * ((1.0 - st.gamma) * cvt<double>(xyz(s.carried[n])) +
                                                       st.gamma * turned));
    const V3<double> spin = ld3(f.end_spin);
    const V3<double> acc = ld3(f.next_acceleration) + cross(ld3(f.end_rate), placed) + cross(spin, cross(spin, placed)) +
                           2.0 * cross(spin, moved) + mul(turn, turned);
    const V3<double> unconstrained = ld3(f.next_velocity) + cross(spin, placed) + moved;
    // reached - X = X0 + next shift + placed - X, kept as a displacement
    const V3<double> reached = ld3(f.next_shift) + (placed - restArm);
    s.v[n] = packc<S>(unconstrained);
    s.a[n] = packc<S>(acc);
    s.relv[n] = packc<S>(placed);
    s.shifted[n] = packc<S>(reached - spanned * acc);
    const double m = double(rest.w);
    addInertia(v, m, placed);
    const V3<double> h = m * cross(placed, unconstrained - ld3(f.next_velocity));
    const V3<double> t = m * cross(placed, acc - ld3(f.next_acceleration));
    v[6] = h.x;
    v[7] = h.y;
    v[8] = h.z;
    v[9] = t.x;
    v[10] = t.y;
    v[11] = t.z;
  }
  blockSum<FRAME_PART>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < FRAME_PART; ++k) s.fpart[size_t(tile) * FRAME_PART + k] = v[k];
}

// The committed rotations of a floating body's tets turn with the frame
// (solver.cc:4343-4345): R <- turn R.
template <class S>
__global__ void __launch_bounds__(TILE) kFrameTurn(Sys<S> s, uint32_t pass) {
  const uint32_t tile = blockIdx.x, b = s.elem_tile_body[tile];
  if (!bodyActive(s, b, pass) || !s.step[b].floating) return;
  const uint32_t e = tile * TILE + threadIdx.x;
  if (e >= s.body[b].elem_end) return;
  const FrameDev& f = s.frame[b];
  M3<double> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = double(s.op[size_t(3 * i + j) * s.Tp + e]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      s.op[size_t(3 * i + j) * s.Tp + e] =
          S(f.turn[3 * i] * r.m[0][j] + f.turn[3 * i + 1] * r.m[1][j] + f.turn[3 * i + 2] * r.m[2][j]);
}

}  // namespace tl
