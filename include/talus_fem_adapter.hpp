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

#include <cmath>
#include <cstdint>
#include <span>
#include <vector>

namespace talus::deformable::b200 {

struct DeviceBody {
  tl_ctx* ctx = nullptr;
  tl_system* system = nullptr;
  DeviceBody() = default;
  DeviceBody(const DeviceBody&) = delete;
  DeviceBody& operator=(const DeviceBody&) = delete;
  ~DeviceBody() {
    if (system) tl_system_destroy(system);
    if (ctx) tl_ctx_destroy(ctx);
  }
};

// buildMesh's PreparedMesh (tets only) and its material lanes uploaded once:
// the replacement for refreshStiffness and buildIncidence (solver.cc:453-507,
// 1065-1101) on every step.  glm matrices are column-major; the ABI is
// row-major.
inline int32_t upload(const talus::PreparedMesh& mesh, std::span<const talus::PhysicalMaterial> lanes,
                      DeviceBody& out, int32_t precision = TL_FP32_MIXED, int32_t device = 0) {
  const size_t V = mesh.restPositions.size(), T = mesh.tets.size();
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
  int32_t rc = tl_ctx_create(device, &out.ctx);
  if (rc != TL_OK) return rc;
  rc = tl_system_create(out.ctx, &d, 1, precision, &out.system);
  if (rc != TL_OK) return rc;
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

// deformable::step(mesh, state, materials, settings, gravity, dt, {}, {},
// nullptr, report) (solver.h:451-462) with the state in host memory.  The
// committed rotations are outputs of the step and the plastic points stay on
// the device (pass them through tl_state_get when the host needs them); the
// report is accumulated like the reference's (solver.cc:3612-3615).
inline int32_t step(DeviceBody& body, talus::DeformableState& state, const Settings& s, const glm::vec3& gravity,
                    float dt, StepReport& report) {
  const tl_settings t = settingsOf(s);
  const double g[3] = {gravity.x, gravity.y, gravity.z};
  tl_step_report r{};
  const int32_t rc = tl_step_host(body.system, 0, TL_DTYPE_F32, state.position.data(), state.velocity.data(),
                                  state.acceleration.data(), nullptr, nullptr, &t, g, dt, &r);
  report.cgIterations += r.cg_iterations;
  report.cgCappedSolves += r.cg_capped_solves;
  report.plasticEvaluations += r.plastic_evaluations;
  report.plasticBacktracks += r.plastic_backtracks;
  report.elasticEnergy += float(r.elastic_energy);
  report.kineticEnergy += float(r.kinetic_energy);
  report.nonFinite = report.nonFinite || r.non_finite != 0;
  return rc;
}

}  // namespace talus::deformable::b200
