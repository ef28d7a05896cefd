"""include/talus_fem_adapter.hpp, the C++ adapter with deformable::step's
types, compiled and linked on the CPU.

The adapter includes the reference's talus/deformable/solver/solver.h,
which needs GLM and cannot be built here.  A stand-in header gives the
fields the adapter touches, with the reference's names and layouts
(mesh.h:11-62, material.h:7-29, solver.h:51-311; glm matrices
column-major).  The test program uploads one tet through the adapter and,
without a device, gets TL_ERR_NO_DEVICE back from tl_ctx_create: the
adapter compiles against those types, links against libtalus_fem.so and
reaches the C ABI.  A body whose lanes mix the two elastic models is refused
before any device work.  tests/test_gpu_adapter.py steps blocks through the
same adapter on the GPU against the oracle.
"""
import os
import shutil
import subprocess

import pytest

from talus_b200 import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STAND_IN = r"""
#pragma once
#include <cstdint>
#include <limits>
#include <vector>
namespace glm {
struct vec3 {
  float x = 0.0f, y = 0.0f, z = 0.0f;
  float& operator[](int i) { return (&x)[i]; }
  const float& operator[](int i) const { return (&x)[i]; }
};
struct uvec4 {
  uint32_t v[4] = {0u, 0u, 0u, 0u};
  uint32_t& operator[](int i) { return v[i]; }
  const uint32_t& operator[](int i) const { return v[i]; }
};
struct mat3 {  // column-major: m[column][row]
  vec3 c[3];
  vec3& operator[](int i) { return c[i]; }
  const vec3& operator[](int i) const { return c[i]; }
};
}  // namespace glm
namespace talus {
constexpr float kInf = std::numeric_limits<float>::infinity();
enum class ElasticModel : uint32_t { Corotated, NeoHookean };
struct PreparedTet { glm::uvec4 nodes; glm::mat3 restInverse; float volume = 0.0f; uint32_t material = 0u; };
struct PreparedMesh {
  std::vector<glm::vec3> restPositions;
  std::vector<float> nodeMass;
  std::vector<uint8_t> anchored;
  std::vector<PreparedTet> tets;
};
struct PlasticPoint { glm::mat3 strain; float equivalent = 0.0f; };
struct CommittedTet { glm::mat3 rotation; };
struct PhysicalMaterial {
  float friction = 0.5f, restitution = 0.0f, density = 1000.0f, strength = kInf, youngsModulus = 0.0f,
        poissonsRatio = 0.3f, stiffnessDamping = 0.0f, yieldStress = kInf, hardeningModulus = 0.0f;
  ElasticModel elasticModel = ElasticModel::Corotated;
  float hysteresis = 0.0f, dampingRatio = kInf, tearStrain = kInf, plasticMax = kInf, crushStress = kInf,
        crushLimit = 1.0f;
};
struct DeformableState {
  std::vector<glm::vec3> position, velocity, acceleration;
  std::vector<CommittedTet> committed;
  std::vector<PlasticPoint> plastic;
};
namespace deformable {
enum class RigidSplit { Off, Unprojected, Projected };
struct Settings {
  uint32_t substeps = 1u, cgIterations = 64u, plasticPasses = 40u, factorBudget = 32u;
  float tolerance = 1.0e-3f, spectralRadius = 0.5f;
  RigidSplit rigidSplit = RigidSplit::Projected;
};
struct StepReport {
  uint32_t nodes = 0u, elements = 0u, cgIterations = 0u, cgCappedSolves = 0u, plasticEvaluations = 0u,
           plasticSolves = 0u, plasticBacktracks = 0u, plasticCapped = 0u, plasticLinearReads = 0u,
           plasticHandoffs = 0u, plasticFallbacks = 0u, plasticFallbackRejections = 0u,
           primaryCgOperatorApplications = 0u;
  float cgWorstRelativeResidual = 0.0f, plasticWorstResidual = 0.0f;
  double elasticSeconds = 0.0, primaryCgSeconds = 0.0;
  float elasticEnergy = 0.0f, kineticEnergy = 0.0f;
  bool nonFinite = false, plasticGrowth = false;
  uint32_t worstSubstep = 0u;
  std::vector<uint32_t> cgPerSubstep;
  std::vector<float> cgStartResidual, cgEndResidual;
  uint32_t factorApplications = 0u, factorRows = 0u, refreshRequests = 0u, refreshedAtAge = 0u,
           spentBeforeRefresh = 0u, spentAfterRefresh = 0u, wastedIterations = 0u, refactors = 0u, retries = 0u,
           retriesFailed = 0u;
  uint64_t factorNonZeros = 0u, systemNonZeros = 0u;
  double refactorSeconds = 0.0;
};
struct SolverStats {
  uint32_t lastIterations = 0u;
  float lastResidual = 0.0f;
  uint32_t factorAge = 0u, refactorCount = 0u, retryCount = 0u, substepsSinceRefresh = 0u;
  float meanIterations = 0.0f;
  bool refreshRequested = false, freshRetryFailed = false;
};
struct DeformableSolverState { SolverStats stats; };
}  // namespace deformable
}  // namespace talus
"""

PROGRAM = r"""
#include "talus_fem_adapter.hpp"
#include <cstdio>
int main() {
  namespace d = talus::deformable;
  talus::PreparedMesh mesh;
  mesh.restPositions = {{0, 0, 0}, {0.1f, 0, 0}, {0, 0.1f, 0}, {0, 0, 0.1f}};
  mesh.nodeMass = {0.04f, 0.04f, 0.04f, 0.04f};
  mesh.anchored = {1, 1, 1, 0};
  talus::PreparedTet tet;
  for (int k = 0; k < 4; ++k) tet.nodes[k] = uint32_t(k);
  for (int c = 0; c < 3; ++c) tet.restInverse[c][c] = 10.0f;
  tet.volume = 1.0f / 6000.0f;
  mesh.tets = {tet};
  talus::PhysicalMaterial lanes[1];
  lanes[0].youngsModulus = 1.0e6f;
  lanes[0].plasticMax = 0.5f;
  {  // lanes mixing the elastic models: refused before any device work
    talus::PhysicalMaterial mixed[2];
    mixed[1].elasticModel = talus::ElasticModel::NeoHookean;
    talus::PreparedMesh two = mesh;
    two.tets.push_back(tet);
    two.tets[1].material = 1u;
    d::b200::DeviceBody refused;
    if (d::b200::upload(two, std::span<const talus::PhysicalMaterial>(mixed, 2), refused) != TL_ERR_UNSUPPORTED)
      return 4;
  }
  d::b200::DeviceBody body;
  const int32_t rc = d::b200::upload(mesh, std::span<const talus::PhysicalMaterial>(lanes, 1), body);
  if (rc == TL_OK) {  // with a device: one step through the adapter
    talus::DeformableState state;
    state.position = mesh.restPositions;
    state.velocity.assign(4, glm::vec3{});
    state.acceleration.assign(4, glm::vec3{});
    d::StepReport report;
    const int32_t s = d::b200::step(body, state, d::Settings{}, glm::vec3{0.0f, -9.81f, 0.0f}, 1.0f / 60.0f, report);
    std::printf("step %d cg %u\n", s, report.cgIterations);
    if (s != TL_OK) return 3;
    d::DeformableSolverState solver;  // the same step with a caller-held solver state
    const int32_t f = d::b200::step(body, state, d::Settings{}, glm::vec3{0.0f, -9.81f, 0.0f}, 1.0f / 60.0f,
                                    &solver, report);
    std::printf("factored %d refactors %u\n", f, solver.stats.refactorCount);
    return f == TL_OK && solver.stats.refactorCount == 1u ? 0 : 5;
  }
  std::printf("upload %d\n", rc);
  return rc == TL_ERR_NO_DEVICE ? 0 : 2;
}
"""


def test_adapter_compiles_links_and_reaches_the_abi(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    capi.lib()  # the library is built
    stub = tmp_path / "talus" / "deformable" / "solver"
    stub.mkdir(parents=True)
    (stub / "solver.h").write_text(STAND_IN)
    (tmp_path / "main.cc").write_text(PROGRAM)
    exe = tmp_path / "adapter"
    libdir = os.path.join(ROOT, "talus_b200")
    subprocess.run(["g++", "-std=c++20", "-Wall", "-Werror", f"-I{tmp_path}", f"-I{os.path.join(ROOT, 'include')}",
                    "-o", str(exe), str(tmp_path / "main.cc"), f"-L{libdir}", "-ltalus_fem", f"-Wl,-rpath,{libdir}"],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
