// Host-side checks of what a caller hands the C ABI, run before anything is
// uploaded.  The reference steps only meshes its own buildMesh produced: that
// keeps tets of positive volume (solver.cc:2352-2356) and returns nullptr for
// an invalid lattice (solver.cc:2193-2198, 2405-2407).  A caller-built
// tl_mesh_desc gets the same guarantee here, so no kernel ever reads a
// non-finite rest shape, a non-positive volume or an out-of-range node.
#pragma once

#include "../../include/talus_fem.h"

#include <cmath>
#include <cstddef>
#include <cstdint>

namespace tl {

inline bool allFinite(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// nullptr when the descriptor can be stepped, else what is wrong with it.
inline const char* meshDescProblem(const tl_mesh_desc& d) {
  if (d.nodes == 0 || d.tets == 0 || !d.rest_positions || !d.node_mass || !d.anchored || !d.tet_nodes ||
      !d.rest_inverse || !d.volume || !d.material || (d.lanes && !d.materials))
    return "mesh descriptor has an empty or missing field";
  if (!allFinite(d.rest_positions, size_t(3) * d.nodes)) return "rest positions must be finite";
  for (uint32_t n = 0; n < d.nodes; ++n)
    if (!(d.node_mass[n] >= 0.0) || !std::isfinite(d.node_mass[n])) return "node masses must be finite and >= 0";
  if (!allFinite(d.rest_inverse, size_t(9) * d.tets)) return "rest inverses must be finite";
  for (uint32_t t = 0; t < d.tets; ++t) {
    if (!(d.volume[t] > 0.0) || !std::isfinite(d.volume[t])) return "tet volumes must be finite and positive";
    for (int k = 0; k < 4; ++k)
      if (d.tet_nodes[4 * size_t(t) + k] >= d.nodes) return "tet node index out of range";
    if (d.element_youngs && (!(d.element_youngs[t] > 0.0) || !std::isfinite(d.element_youngs[t])))
      return "Young's modulus must be positive";
  }
  if (d.prescribed_velocity)
    for (uint32_t n = 0; n < d.nodes; ++n)
      if (d.anchored[n] && !allFinite(d.prescribed_velocity + size_t(3) * n, 3))
        return "prescribed velocities must be finite";
  // PhysicalMaterial (material.h:12-29): E >= 0 (the default lane has E = 0,
  // material.cc:9-16), nu is clamped to [0, 0.49] by lame (material.cc:71-78),
  // an infinite or non-positive yield stress means no plasticity
  // (material.cc:747-749), hardening H >= 0.
  for (uint32_t l = 0; l < d.lanes; ++l) {
    const tl_material& m = d.materials[l];
    if (!(m.youngs_modulus >= 0.0) || !std::isfinite(m.youngs_modulus) || !std::isfinite(m.poissons_ratio))
      return "material lane needs a finite E >= 0 and a finite Poisson ratio";
    if (std::isfinite(m.yield_stress) && m.yield_stress > 0.0 &&
        (!(m.hardening_modulus >= 0.0) || !std::isfinite(m.hardening_modulus)))
      return "a yielding material lane needs a finite hardening modulus >= 0";
  }
  return nullptr;
}

// tl_step's own arguments: a finite positive step and finite gravity.
inline bool stepArgumentsValid(double dt, const double gravity[3]) {
  return dt > 0.0 && std::isfinite(dt) && allFinite(gravity, 3);
}

}  // namespace tl
