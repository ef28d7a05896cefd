// talus_fem_adapter.hpp -- the C++ adapter a Talus build adds to call the
// B200 tet step with deformable::step's types.
//
// It compiles inside the Talus source tree: it includes the reference's
// talus/deformable/solver/solver.h for PreparedMesh, PreparedTet,
// PhysicalMaterial, DeformableState, Settings and StepReport (mesh.h:11-62,
// material.h:12-29, solver.h:51-311).  One device system is kept per
// PreparedMesh; the mesh is immutable and shared, as in bodyset.h:24.  Link
// with -ltalus_fem.
#pragma once

#include <talus/deformable/solver/solver.h>

#include "talus_fem.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <span>
#include <vector>

namespace talus::deformable::b200 {

// One PreparedMesh resident on the device, with the law its lanes select and
// the host staging of the element state in the C ABI's row-major layout.
struct DeviceBody {
  tl_ctx* ctx = nullptr;
  tl_system* system = nullptr;
  uint32_t law = TL_LAW_COROTATED;
  uint32_t nodes = 0u, tets = 0u;
  std::vector<float> rotation, plastic;  // [9 T] committed rotations, [10 T] plastic points
  bool factored = false;                 // the device holds a solver state's factor for this body
  DeviceBody() = default;
  DeviceBody(const DeviceBody&) = delete;
  DeviceBody& operator=(const DeviceBody&) = delete;
  ~DeviceBody() {
    if (system) tl_system_destroy(system);
    if (ctx) tl_ctx_destroy(ctx);
  }
};

// PhysicalMaterial::elasticModel (material.h:7-10, 22) of the lanes the tets
// use, as the step's law: Corotated is the reference tet law, NeoHookean the
// stable neo-Hookean law at one point per tet.  A tet whose lane is out of
// range takes the default material (material.cc:9-16), which is Corotated.
// The step applies one law to a body, so a body whose tets mix the two
// models is refused (TL_ERR_UNSUPPORTED).
inline int32_t lawOf(const talus::PreparedMesh& mesh, std::span<const talus::PhysicalMaterial> lanes, uint32_t& law) {
  bool corotated = false, neoHookean = false;
  for (const talus::PreparedTet& t : mesh.tets) {
    const bool snh = t.material < lanes.size() && lanes[t.material].elasticModel == talus::ElasticModel::NeoHookean;
    (snh ? neoHookean : corotated) = true;
  }
  if (corotated && neoHookean) return TL_ERR_UNSUPPORTED;
  law = neoHookean ? TL_LAW_SNH : TL_LAW_COROTATED;
  return TL_OK;
}

// buildMesh's PreparedMesh (tets only) and its material lanes uploaded once:
// the replacement for refreshStiffness and buildIncidence (solver.cc:453-507,
// 1065-1101) on every step.  glm matrices are column-major; the ABI is
// row-major.
inline int32_t upload(const talus::PreparedMesh& mesh, std::span<const talus::PhysicalMaterial> lanes,
                      DeviceBody& out, int32_t precision = TL_FP32_MIXED, int32_t device = 0) {
  const size_t V = mesh.restPositions.size(), T = mesh.tets.size();
  int32_t rc = lawOf(mesh, lanes, out.law);
  if (rc != TL_OK) return rc;
  std::vector<double> rest(3 * V), mass(V), rinv(9 * T), vol(T);
  std::vector<uint32_t> nodes(4 * T), lane(T);
  for (size_t n = 0; n < V; ++n) {
    for (int k = 0; k < 3; ++k) rest[3 * n + k] = mesh.restPositions[n][k];
    mass[n] = mesh.nodeMass[n];
  }
  for (size_t e = 0; e < T; ++e) {
    const talus::PreparedTet& t = mesh.tets[e];
    for (int k = 0; k < 4; ++k) nodes[4 * e + k] = t.nodes[k];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) rinv[9 * e + 3 * r + c] = t.restInverse[c][r];
    vol[e] = t.volume;
    lane[e] = t.material;
  }
  std::vector<tl_material> mats;
  for (const talus::PhysicalMaterial& m : lanes)
    mats.push_back({m.density, m.youngsModulus, m.poissonsRatio, m.stiffnessDamping, m.yieldStress,
                    m.hardeningModulus});
  const tl_mesh_desc d{uint32_t(V), uint32_t(T), rest.data(), mass.data(), mesh.anchored.data(), nodes.data(),
                       rinv.data(), vol.data(), lane.data(), mats.data(), uint32_t(mats.size()), nullptr, nullptr};
  rc = tl_ctx_create(device, &out.ctx);
  if (rc != TL_OK) return rc;
  rc = tl_system_create(out.ctx, &d, 1, precision, &out.system);
  if (rc != TL_OK) return rc;
  out.nodes = uint32_t(V);
  out.tets = uint32_t(T);
  // the finite-strain flow's crush and plastic cap (material.h:16-29), for
  // lanes that set them; read only in TL_PLASTICITY_HENCKY
  for (size_t l = 0; l < lanes.size(); ++l) {
    const talus::PhysicalMaterial& m = lanes[l];
    if (std::isinf(m.crushStress) && m.crushLimit >= 1.0f && std::isinf(m.plasticMax)) continue;
    rc = tl_system_set_flow_limits(out.system, 0, uint32_t(l), m.crushStress, m.crushLimit, m.plasticMax);
    if (rc != TL_OK) return rc;
  }
  return TL_OK;
}

inline tl_settings settingsOf(const Settings& s) {
  tl_settings t;
  tl_settings_default(&t);
  t.substeps = s.substeps;
  t.cg_iterations = s.cgIterations;
  t.plastic_passes = s.plasticPasses;
  t.tolerance = s.tolerance;
  t.spectral_radius = s.spectralRadius;
  t.rigid_split = uint32_t(s.rigidSplit);
  return t;
}

// The caller's plastic points (tet e in slot e, tetPoint solver.cc:1177-1190,
// for a mesh without hexes) in the ABI's row-major layout.
inline void packPlastic(const talus::DeformableState& state, size_t T, std::vector<float>& out) {
  out.assign(10 * T, 0.0f);
  for (size_t e = 0; e < T && e < state.plastic.size(); ++e) {
    const talus::PlasticPoint& p = state.plastic[e];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) out[10 * e + 3 * r + c] = p.strain[c][r];
    out[10 * e + 9] = p.equivalent;
  }
}

// Committed rotations and plastic points back into the caller's state.
inline void unpackElements(talus::DeformableState& state, size_t T, const std::vector<float>& rotation,
                           const std::vector<float>& plastic) {
  if (state.committed.size() < T) state.committed.resize(T);
  if (state.plastic.size() < T) state.plastic.resize(T);
  for (size_t e = 0; e < T; ++e) {
    for (int row = 0; row < 3; ++row)
      for (int c = 0; c < 3; ++c) {
        state.committed[e].rotation[c][row] = rotation[9 * e + 3 * row + c];
        state.plastic[e].strain[c][row] = plastic[10 * e + 3 * row + c];
      }
    state.plastic[e].equivalent = plastic[10 * e + 9];
  }
}

// One body's counters accumulated like the reference's (solver.cc:3612-3615,
// 5881-5882), with the per-substep lists appended (solver.cc:4253-4256).
inline void accumulate(StepReport& report, const tl_step_report& r, const tl_system* system, uint32_t body) {
  report.nodes += r.nodes;
  report.elements += r.elements;
  report.cgIterations += r.cg_iterations;
  report.cgCappedSolves += r.cg_capped_solves;
  report.plasticEvaluations += r.plastic_evaluations;
  report.plasticSolves += r.plastic_solves;
  report.plasticBacktracks += r.plastic_backtracks;
  report.plasticCapped += r.plastic_capped;
  report.plasticLinearReads += r.plastic_linear_reads;
  report.plasticHandoffs += r.plastic_handoffs;
  report.plasticFallbacks += r.plastic_fallbacks;
  report.plasticFallbackRejections += r.plastic_fallback_rejections;
  report.primaryCgOperatorApplications += r.operator_applications;
  report.cgWorstRelativeResidual = std::max(report.cgWorstRelativeResidual, float(r.cg_worst_relative_residual));
  report.plasticWorstResidual = std::max(report.plasticWorstResidual, float(r.plastic_worst_residual));
  report.elasticEnergy += float(r.elastic_energy);
  report.kineticEnergy += float(r.kinetic_energy);
  report.nonFinite = report.nonFinite || r.non_finite != 0;
  report.plasticGrowth = report.plasticGrowth || r.plastic_growth != 0;
  // device time of the element pass and the PCG (TL_FLAG_PROFILE) stand in
  // for the reference's wall-clock stage timers
  report.elasticSeconds += r.element_seconds;
  report.primaryCgSeconds += r.pcg_seconds;
  uint32_t iterations[16], count = 0u;
  double start[16], end[16];
  if (tl_step_substeps(system, body, iterations, start, end, 16, &count) == TL_OK) {
    for (uint32_t k = 0; k < count && k < 16u; ++k) {
      report.cgPerSubstep.push_back(iterations[k]);
      report.cgStartResidual.push_back(float(start[k]));
      report.cgEndResidual.push_back(float(end[k]));
      report.worstSubstep = std::max(report.worstSubstep, iterations[k]);
    }
  }
}

// deformable::step(mesh, state, materials, settings, gravity, dt, {}, {},
// nullptr, report) (solver.h:451-462) with the state in host memory, owned by
// the caller as in the reference (mesh.h:56-62):
//  * position, velocity and acceleration are read and written;
//  * the plastic points are read every step, so a caller that restores a
//    saved DeformableState steps from the plastic state it restored;
//  * the committed rotations are written (the step sets each before reading
//    it, assembleElastic solver.cc:1404-1547), sized to the tets if needed;
//  * the report is accumulated like the reference's.
inline int32_t step(DeviceBody& body, talus::DeformableState& state, const Settings& s, const glm::vec3& gravity,
                    float dt, StepReport& report) {
  tl_settings t = settingsOf(s);
  t.law = body.law;
  const size_t T = body.tets;
  body.rotation.assign(9 * T, 0.0f);
  packPlastic(state, T, body.plastic);
  const double g[3] = {gravity.x, gravity.y, gravity.z};
  tl_step_report r{};
  const int32_t rc = tl_step_host(body.system, 0, TL_DTYPE_F32, state.position.data(), state.velocity.data(),
                                  state.acceleration.data(), body.rotation.data(), body.plastic.data(), &t, g, dt, &r);
  if (rc != TL_OK && rc != TL_ERR_NONFINITE) return rc;
  unpackElements(state, T, body.rotation, body.plastic);
  accumulate(report, r, body.system, 0);
  return rc;
}

// deformable::step(mesh, state, materials, settings, gravity, dt, {}, {},
// solver, report) with a caller-held solver state (solver.h:451-462,
// factor.h:205-210).  The factor itself lives on the device with the body:
// the first call with a solver state turns it on (tl_system_use_factor with
// Settings::factorBudget), a call without one turns it off.  After each step
// the caller's SolverStats (factor.h:28-38) are those of the device state and
// the step's factor counters are added to the report (solver.cc:3606-3609,
// 3839-3899).  The reference's Eigen factor inside the caller's state is not
// built (the device factor takes its place).
inline int32_t step(DeviceBody& body, talus::DeformableState& state, const Settings& s, const glm::vec3& gravity,
                    float dt, DeformableSolverState* solver, StepReport& report) {
  if ((solver != nullptr) != body.factored) {
    const int32_t rc = tl_system_use_factor(body.system, solver ? 1u : 0u, s.factorBudget);
    if (rc != TL_OK) return rc;
    body.factored = solver != nullptr;
  }
  tl_factor_stats before{}, after{};
  if (solver) tl_system_factor_stats(body.system, &before);
  const int32_t rc = step(body, state, s, gravity, dt, report);
  if (!solver || (rc != TL_OK && rc != TL_ERR_NONFINITE)) return rc;
  tl_system_factor_stats(body.system, &after);
  SolverStats& st = solver->stats;
  st.factorAge = after.factor_age;
  st.refactorCount = after.refactor_count;
  st.retryCount = after.retry_count;
  st.substepsSinceRefresh = after.substeps_since_refresh;
  st.meanIterations = float(after.mean_iterations);
  st.refreshRequested = after.refresh_requested != 0u;
  st.freshRetryFailed = after.fresh_retry_failed != 0u;
  report.factorRows = before.rows;  // read before the step's refresh, as the reference reads them
  report.factorNonZeros = before.factor_nonzeros;
  report.systemNonZeros = before.system_nonzeros;
  report.refreshRequests += after.refresh_requests - before.refresh_requests;
  report.refactors += after.refactors - before.refactors;
  report.retries += after.retries - before.retries;
  report.retriesFailed += after.retries_failed - before.retries_failed;
  report.wastedIterations += after.wasted_iterations - before.wasted_iterations;
  report.factorApplications += after.factor_applications - before.factor_applications;
  if (after.refresh_requests != before.refresh_requests) {
    report.refreshedAtAge = after.refreshed_at_age;
    report.spentBeforeRefresh = after.spent_before_refresh;
    report.spentAfterRefresh = after.spent_after_refresh;
  }
  report.refactorSeconds += after.refactor_seconds - before.refactor_seconds;
  return rc;
}

// ----------------------------------------------------------------------------
// Every tet body of one World island stepped together.  The reference World
// hands each non-rigid island to a solver in its island loop
// (dynamics/pipeline/pipeline.cc:1002-1018 classifies, :1214-1241 solves); a
// tet owner would hold one Island per island and call step() there.  The
// island's bodies live in one resident batched system, so a World step costs
// one launch sequence for all of them, whatever their sizes: anchored or
// floating (a body with no anchored node takes the floating frame under the
// settings' rigidSplit), elastic or yielding (each yielding body runs its own
// plastic Newton control).  The states stay the caller's, as for step().
struct IslandBody {
  const talus::PreparedMesh* mesh = nullptr;
  std::span<const talus::PhysicalMaterial> lanes;
};

struct Island {
  tl_ctx* ctx = nullptr;
  tl_system* system = nullptr;
  uint32_t law = TL_LAW_COROTATED;
  std::vector<uint32_t> tets, plasticUsed;
  std::vector<float> rotation, plastic;
  std::vector<tl_step_report> reports;
  Island() = default;
  Island(const Island&) = delete;
  Island& operator=(const Island&) = delete;
  ~Island() {
    if (system) tl_system_destroy(system);
    if (ctx) tl_ctx_destroy(ctx);
  }
};

// Uploads the island's bodies once.  One law serves the island: its bodies'
// lanes must agree on elasticModel (else TL_ERR_UNSUPPORTED).
inline int32_t upload(std::span<const IslandBody> bodies, Island& out, int32_t precision = TL_FP32_MIXED,
                      int32_t device = 0) {
  if (bodies.empty()) return TL_ERR_ARG;
  struct Host {
    std::vector<double> rest, mass, rinv, vol;
    std::vector<uint32_t> nodes, lane;
    std::vector<tl_material> mats;
  };
  std::vector<Host> host(bodies.size());
  std::vector<tl_mesh_desc> descs(bodies.size());
  out.tets.assign(bodies.size(), 0u);
  out.plasticUsed.assign(bodies.size(), 0u);
  bool snh = false, corotated = false;
  for (size_t b = 0; b < bodies.size(); ++b) {
    const talus::PreparedMesh& mesh = *bodies[b].mesh;
    uint32_t law = TL_LAW_COROTATED;
    const int32_t rc = lawOf(mesh, bodies[b].lanes, law);
    if (rc != TL_OK) return rc;
    (law == TL_LAW_SNH ? snh : corotated) = true;
    const size_t V = mesh.restPositions.size(), T = mesh.tets.size();
    Host& h = host[b];
    h.rest.resize(3 * V);
    h.mass.resize(V);
    h.rinv.resize(9 * T);
    h.vol.resize(T);
    h.nodes.resize(4 * T);
    h.lane.resize(T);
    for (size_t n = 0; n < V; ++n) {
      for (int k = 0; k < 3; ++k) h.rest[3 * n + k] = mesh.restPositions[n][k];
      h.mass[n] = mesh.nodeMass[n];
    }
    for (size_t e = 0; e < T; ++e) {
      const talus::PreparedTet& t = mesh.tets[e];
      for (int k = 0; k < 4; ++k) h.nodes[4 * e + k] = t.nodes[k];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) h.rinv[9 * e + 3 * r + c] = t.restInverse[c][r];
      h.vol[e] = t.volume;
      h.lane[e] = t.material;
    }
    for (const talus::PhysicalMaterial& m : bodies[b].lanes) {
      h.mats.push_back({m.density, m.youngsModulus, m.poissonsRatio, m.stiffnessDamping, m.yieldStress,
                        m.hardeningModulus});
      if (std::isfinite(m.yieldStress) && m.yieldStress > 0.0f) out.plasticUsed[b] = 1u;
    }
    descs[b] = tl_mesh_desc{uint32_t(V), uint32_t(T), h.rest.data(), h.mass.data(), mesh.anchored.data(),
                            h.nodes.data(), h.rinv.data(), h.vol.data(), h.lane.data(), h.mats.data(),
                            uint32_t(h.mats.size()), nullptr, nullptr};
    out.tets[b] = uint32_t(T);
  }
  if (snh && corotated) return TL_ERR_UNSUPPORTED;
  out.law = snh ? TL_LAW_SNH : TL_LAW_COROTATED;
  int32_t rc = tl_ctx_create(device, &out.ctx);
  if (rc != TL_OK) return rc;
  rc = tl_system_create(out.ctx, descs.data(), uint32_t(descs.size()), precision, &out.system);
  if (rc != TL_OK) return rc;
  out.reports.assign(bodies.size(), tl_step_report{});
  return TL_OK;
}

// deformable::step for every body of the island, in one launch sequence.
// states[b] and reports[b] belong to body b of the upload.
inline int32_t step(Island& island, std::span<talus::DeformableState* const> states, const Settings& s,
                    const glm::vec3& gravity, float dt, std::span<StepReport> reports) {
  if (states.size() != island.tets.size() || reports.size() != island.tets.size()) return TL_ERR_ARG;
  tl_settings t = settingsOf(s);
  t.law = island.law;
  for (uint32_t b = 0; b < states.size(); ++b) {
    talus::DeformableState& st = *states[b];
    const bool crosses = island.law == TL_LAW_COROTATED && island.plasticUsed[b];
    if (crosses) packPlastic(st, island.tets[b], island.plastic);
    const int32_t rc = tl_state_set(island.system, b, TL_DTYPE_F32, st.position.data(), st.velocity.data(),
                                    st.acceleration.data(), nullptr, crosses ? island.plastic.data() : nullptr);
    if (rc != TL_OK) return rc;
  }
  std::fill(island.reports.begin(), island.reports.end(), tl_step_report{});
  const double g[3] = {gravity.x, gravity.y, gravity.z};
  const int32_t rc = tl_step(island.system, &t, g, dt, island.reports.data());
  if (rc != TL_OK && rc != TL_ERR_NONFINITE) return rc;
  for (uint32_t b = 0; b < states.size(); ++b) {
    talus::DeformableState& st = *states[b];
    const size_t T = island.tets[b];
    island.rotation.assign(9 * T, 0.0f);
    packPlastic(st, T, island.plastic);  // kept as it is unless the step used it
    const bool crosses = island.law == TL_LAW_COROTATED && island.plasticUsed[b];
    const int32_t got = tl_state_get(island.system, b, TL_DTYPE_F32, st.position.data(), st.velocity.data(),
                                     st.acceleration.data(), island.rotation.data(),
                                     crosses ? island.plastic.data() : nullptr);
    if (got != TL_OK) return got;
    unpackElements(st, T, island.rotation, island.plastic);
    accumulate(reports[b], island.reports[b], island.system, b);
  }
  return rc;
}

}  // namespace talus::deformable::b200
