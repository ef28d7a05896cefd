"""The C++ adapter (include/talus_fem_adapter.hpp) on the GPU, against the oracle.

A C++ program built against the adapter and the stand-in of the reference
types (tests/test_adapter.py) steps a body through
talus::deformable::b200::step with the state in host memory, float like the
reference's DeformableState (mesh.h:56-62):

* positions after every step within a few float ulps of the FP64 oracle
  stepping the same float state: the oracle's state is rounded to float
  between its steps the way the caller's DeformableState is;
* the committed rotations and plastic points written back into the caller's
  DeformableState match the oracle's;
* StepReport's per-substep lists (cgPerSubstep, cgStartResidual,
  cgEndResidual, solver.h:299-301) are filled, one entry per substep;
* restoring a saved DeformableState (plastic points included) and stepping
  again reproduces the steps taken from it bit for bit;
* PhysicalMaterial::elasticModel = NeoHookean selects the neo-Hookean law;
* an Island steps anchored, floating and yielding bodies together.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from talus_b200 import _capi as capi
from tests.helpers import DT, GRAVITY, relative_error, to_oracle
from tests.test_adapter import ROOT, STAND_IN

pytestmark = pytest.mark.gpu

PROGRAM = r"""
#include "talus_fem_adapter.hpp"
#include <cstdio>
#include <cstring>
#include <fstream>
namespace d = talus::deformable;
template <class T> void get(std::ifstream& in, T* p, size_t n) { in.read(reinterpret_cast<char*>(p), sizeof(T) * n); }
template <class T> void put(std::ofstream& out, const T* p, size_t n) {
  out.write(reinterpret_cast<const char*>(p), sizeof(T) * n);
}
int main(int argc, char** argv) {
  std::ifstream in(argv[1], std::ios::binary);
  uint32_t V, T, steps, model;
  float mat[5];  // density, E, nu, yield, hardening
  get(in, &V, 1); get(in, &T, 1); get(in, &steps, 1); get(in, &model, 1); get(in, mat, 5);
  talus::PreparedMesh mesh;
  mesh.restPositions.resize(V); mesh.nodeMass.resize(V); mesh.anchored.resize(V); mesh.tets.resize(T);
  for (auto& p : mesh.restPositions) get(in, &p.x, 3);
  get(in, mesh.nodeMass.data(), V);
  get(in, mesh.anchored.data(), V);
  for (auto& t : mesh.tets) {
    get(in, t.nodes.v, 4);
    float rinv[9];
    get(in, rinv, 9);  // row-major
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) t.restInverse[c][r] = rinv[3 * r + c];
    get(in, &t.volume, 1);
  }
  talus::PhysicalMaterial lane;
  lane.density = mat[0]; lane.youngsModulus = mat[1]; lane.poissonsRatio = mat[2];
  lane.yieldStress = mat[3]; lane.hardeningModulus = mat[4];
  lane.elasticModel = model ? talus::ElasticModel::NeoHookean : talus::ElasticModel::Corotated;
  d::b200::DeviceBody body;
  int32_t rc = d::b200::upload(mesh, std::span<const talus::PhysicalMaterial>(&lane, 1), body, TL_FP64);
  if (rc != TL_OK) { std::printf("upload %d\n", rc); return 2; }
  talus::DeformableState state;
  state.position = mesh.restPositions;
  state.velocity.assign(V, glm::vec3{});
  state.acceleration.assign(V, glm::vec3{});
  d::StepReport report;
  std::ofstream out(argv[2], std::ios::binary);
  talus::DeformableState saved;
  const uint32_t half = steps / 2;
  for (uint32_t k = 0; k < steps; ++k) {
    if (k == half) saved = state;
    rc = d::b200::step(body, state, d::Settings{}, glm::vec3{0.0f, -9.81f, 0.0f}, 1.0f / 60.0f, report);
    if (rc != TL_OK) { std::printf("step %d\n", rc); return 3; }
    for (auto& p : state.position) put(out, &p.x, 3);
  }
  for (auto& c : state.committed) for (int col = 0; col < 3; ++col) put(out, &c.rotation[col].x, 3);
  for (auto& p : state.plastic) { for (int col = 0; col < 3; ++col) put(out, &p.strain[col].x, 3); put(out, &p.equivalent, 1); }
  const uint32_t n = uint32_t(report.cgPerSubstep.size());
  put(out, &n, 1);
  put(out, report.cgPerSubstep.data(), n);
  put(out, report.cgStartResidual.data(), n);
  put(out, report.cgEndResidual.data(), n);
  put(out, &report.cgIterations, 1);
  put(out, &report.worstSubstep, 1);
  // restore the saved state and take the second half again
  talus::DeformableState again = saved;
  d::StepReport other;
  for (uint32_t k = half; k < steps; ++k)
    if (d::b200::step(body, again, d::Settings{}, glm::vec3{0.0f, -9.81f, 0.0f}, 1.0f / 60.0f, other) != TL_OK) return 4;
  bool same = again.position.size() == state.position.size();
  for (size_t i = 0; same && i < state.position.size(); ++i)
    same = std::memcmp(&again.position[i], &state.position[i], sizeof(glm::vec3)) == 0;
  for (size_t i = 0; same && i < state.plastic.size(); ++i)
    same = std::memcmp(&again.plastic[i], &state.plastic[i], sizeof(talus::PlasticPoint)) == 0;
  const uint32_t flag = same ? 1u : 0u;
  put(out, &flag, 1);
  return 0;
}
"""


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    capi.lib()
    work = tmp_path_factory.mktemp("adapter")
    stub = work / "talus" / "deformable" / "solver"
    stub.mkdir(parents=True)
    (stub / "solver.h").write_text(STAND_IN)
    (work / "main.cc").write_text(PROGRAM)
    exe = work / "stepper"
    libdir = os.path.join(ROOT, "talus_b200")
    subprocess.run(["g++", "-std=c++20", "-O2", "-Wall", "-Werror", f"-I{work}", f"-I{os.path.join(ROOT, 'include')}",
                    "-o", str(exe), str(work / "main.cc"), f"-L{libdir}", "-ltalus_fem", f"-Wl,-rpath,{libdir}"],
                   check=True)
    return work, exe


def run_adapter(program, mesh, mat, steps, model):
    work, exe = program
    V, T = mesh.nodes, mesh.tets
    blob = struct.pack("<4I5f", V, T, steps, model, mat.density, mat.youngs_modulus, mat.poissons_ratio,
                       mat.yield_stress, mat.hardening_modulus)
    blob += mesh.rest_positions.astype(np.float32).tobytes() + mesh.node_mass.astype(np.float32).tobytes()
    blob += mesh.anchored.astype(np.uint8).tobytes()
    for e in range(T):
        blob += mesh.tet_nodes[e].astype(np.uint32).tobytes() + mesh.rest_inverse[e].astype(np.float32).tobytes()
        blob += np.float32(mesh.volume[e]).tobytes()
    (work / "in.bin").write_bytes(blob)
    out = subprocess.run([str(exe), str(work / "in.bin"), str(work / "out.bin")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    raw = (work / "out.bin").read_bytes()
    at = 0

    def take(dtype, count):
        nonlocal at
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=at)
        at += a.nbytes
        return a

    positions = take(np.float32, steps * V * 3).reshape(steps, V, 3).astype(np.float64)
    rotation = take(np.float32, T * 9).reshape(T, 3, 3).transpose(0, 2, 1)  # columns -> row-major
    plastic = take(np.float32, T * 10).reshape(T, 10)
    n = int(take(np.uint32, 1)[0])
    lists = (take(np.uint32, n), take(np.float32, n), take(np.float32, n))
    total, worst = int(take(np.uint32, 1)[0]), int(take(np.uint32, 1)[0])
    restored = int(take(np.uint32, 1)[0])
    return positions, rotation, plastic, lists, total, worst, restored


def as_float(state):
    """The caller's float DeformableState between two steps: what the adapter
    uploads is the previous step's result rounded to float."""
    for a in (state.position, state.velocity, state.acceleration, state.plastic):
        a[...] = a.astype(np.float32).astype(np.float64)


def float_close(x, ref, rest, ulps=32):
    """|x - ref| within `ulps` float ulps of the body's largest coordinate."""
    return float(np.abs(x - ref).max()) <= ulps * np.finfo(np.float32).eps * float(np.abs(rest).max())


def oracle_run(mesh, mat, steps, law):
    om = to_oracle(mesh)
    st = po.State.rest(om)
    record, reports = [], []
    omat = po.material(mat.density, mat.youngs_modulus, mat.poissons_ratio, 0.0, mat.yield_stress,
                       mat.hardening_modulus)
    for _ in range(steps):
        reports.append(po.step(po.F64, om, st, [omat], po.Settings(law=law), GRAVITY, DT).as_dict())
        as_float(st)
        record.append(st.position.copy())
    return record, st, reports


def test_plastic_cantilever_through_the_adapter(program):
    mesh = tb.box_mesh((8, 2, 2), voxel=0.1, jitter=0.01, seed=21, anchor_axis=0)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, yield_stress=2e4,
                              hardening_modulus=1e4)
    steps = 8
    positions, rotation, plastic, (per, start, end), total, worst, restored = run_adapter(program, mesh, mat, steps, 0)
    record, ostate, reports = oracle_run(mesh, mat, steps, po.LAW_COROTATED)
    for k in range(steps):
        assert float_close(positions[k], record[k], mesh.rest_positions), k
    assert (ostate.plastic[:, 9] > 0).any()
    assert np.abs(plastic[:, 9] - ostate.plastic[:, 9]).max() <= 1e-4 * ostate.plastic[:, 9].max()
    assert np.abs(plastic[:, :9] - ostate.plastic[:, :9]).max() <= 1e-4 * np.abs(ostate.plastic[:, :9]).max()
    assert np.abs(rotation - ostate.rotation).max() <= 1e-4
    assert len(per) == steps and int(per.sum()) == total and worst == int(per.max())
    assert (start > 0).all() and (end >= 0).all()
    assert restored == 1


def test_neo_hookean_lanes_select_the_neo_hookean_law(program):
    mesh = tb.box_mesh((4, 4, 4), voxel=0.1, jitter=0.01, seed=22)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e5, poissons_ratio=0.3)
    steps = 6
    positions, _, _, (per, _, _), _, _, restored = run_adapter(program, mesh, mat, steps, 1)
    snh, _, _ = oracle_run(mesh, mat, steps, po.LAW_SNH)
    corotated, _, _ = oracle_run(mesh, mat, steps, po.LAW_COROTATED)
    assert float_close(positions[-1], snh[-1], mesh.rest_positions)
    assert relative_error(corotated[-1], snh[-1], mesh.rest_positions) > 1e-5  # the laws do differ here
    assert len(per) == steps and restored == 1


ISLAND_PROGRAM = r"""
#include "talus_fem_adapter.hpp"
#include <cstdio>
#include <fstream>
namespace d = talus::deformable;
template <class T> void get(std::ifstream& in, T* p, size_t n) { in.read(reinterpret_cast<char*>(p), sizeof(T) * n); }
template <class T> void put(std::ofstream& out, const T* p, size_t n) {
  out.write(reinterpret_cast<const char*>(p), sizeof(T) * n);
}
int main(int argc, char** argv) {
  std::ifstream in(argv[1], std::ios::binary);
  uint32_t count, steps;
  get(in, &count, 1); get(in, &steps, 1);
  std::vector<talus::PreparedMesh> meshes(count);
  std::vector<talus::PhysicalMaterial> lanes(count);
  std::vector<talus::DeformableState> states(count);
  for (uint32_t b = 0; b < count; ++b) {
    uint32_t V, T;
    float mat[5];
    get(in, &V, 1); get(in, &T, 1); get(in, mat, 5);
    talus::PreparedMesh& mesh = meshes[b];
    mesh.restPositions.resize(V); mesh.nodeMass.resize(V); mesh.anchored.resize(V); mesh.tets.resize(T);
    for (auto& p : mesh.restPositions) get(in, &p.x, 3);
    get(in, mesh.nodeMass.data(), V);
    get(in, mesh.anchored.data(), V);
    for (auto& t : mesh.tets) {
      get(in, t.nodes.v, 4);
      float rinv[9];
      get(in, rinv, 9);
      for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) t.restInverse[c][r] = rinv[3 * r + c];
      get(in, &t.volume, 1);
    }
    lanes[b].density = mat[0]; lanes[b].youngsModulus = mat[1]; lanes[b].poissonsRatio = mat[2];
    lanes[b].yieldStress = mat[3]; lanes[b].hardeningModulus = mat[4];
    states[b].position.resize(V); states[b].velocity.resize(V); states[b].acceleration.resize(V);
    for (auto& p : states[b].position) get(in, &p.x, 3);
    for (auto& p : states[b].velocity) get(in, &p.x, 3);
  }
  std::vector<d::b200::IslandBody> bodies(count);
  for (uint32_t b = 0; b < count; ++b) bodies[b] = {&meshes[b], std::span<const talus::PhysicalMaterial>(&lanes[b], 1)};
  d::b200::Island island;
  int32_t rc = d::b200::upload(std::span<const d::b200::IslandBody>(bodies), island, TL_FP64);
  if (rc != TL_OK) { std::printf("upload %d\n", rc); return 2; }
  std::vector<talus::DeformableState*> ptrs(count);
  for (uint32_t b = 0; b < count; ++b) ptrs[b] = &states[b];
  std::vector<d::StepReport> reports(count);
  std::ofstream out(argv[2], std::ios::binary);
  for (uint32_t k = 0; k < steps; ++k) {
    rc = d::b200::step(island, std::span<talus::DeformableState* const>(ptrs), d::Settings{},
                       glm::vec3{0.0f, -9.81f, 0.0f}, 1.0f / 60.0f, std::span<d::StepReport>(reports));
    if (rc != TL_OK) { std::printf("step %d\n", rc); return 3; }
  }
  for (uint32_t b = 0; b < count; ++b) {
    for (auto& p : states[b].position) put(out, &p.x, 3);
    for (auto& p : states[b].plastic) put(out, &p.equivalent, 1);
    const uint32_t n = uint32_t(reports[b].cgPerSubstep.size());
    put(out, &n, 1);
    put(out, &reports[b].plasticEvaluations, 1);
  }
  return 0;
}
"""


def test_island_of_anchored_floating_and_yielding_bodies(program):
    """Every tet body of an island in one batched step through
    talus::deformable::b200::Island: a yielding cantilever, a spinning free
    block (floating frame, Projected split) and an elastic block, each
    within a few float ulps of its own FP64 oracle run on the same float
    state."""
    work, _ = program
    (work / "island.cc").write_text(ISLAND_PROGRAM)
    exe = work / "island"
    libdir = os.path.join(ROOT, "talus_b200")
    subprocess.run(["g++", "-std=c++20", "-O2", "-Wall", "-Werror", f"-I{work}", f"-I{os.path.join(ROOT, 'include')}",
                    "-o", str(exe), str(work / "island.cc"), f"-L{libdir}", "-ltalus_fem", f"-Wl,-rpath,{libdir}"],
                   check=True)
    cantilever = tb.box_mesh((6, 2, 2), voxel=0.1, jitter=0.01, seed=23, anchor_axis=0)
    free = tb.box_mesh((3, 3, 4), voxel=0.1, jitter=0.01, seed=24, anchor_axis=3)
    block = tb.box_mesh((4, 3, 3), voxel=0.1, jitter=0.01, seed=25)
    meshes = (cantilever, free, block)
    mats = [tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3, yield_stress=2e4,
                                hardening_modulus=1e4),
            tb.PhysicalMaterial(density=1000.0, youngs_modulus=5e5, poissons_ratio=0.3),
            tb.PhysicalMaterial(density=1000.0, youngs_modulus=2e6, poissons_ratio=0.35)]
    starts = []
    for mesh in meshes:
        st = tb.rest_state(mesh)
        if mesh is free:
            centre = (mesh.node_mass[:, None] * mesh.rest_positions).sum(0) / mesh.node_mass.sum()
            st.velocity[...] = np.cross([0.5, 2.0, 0.0], mesh.rest_positions - centre) + np.array([0.2, 0.5, 0.0])
        starts.append(st)
    steps = 6
    blob = struct.pack("<2I", 3, steps)
    for mesh, mat, st in zip(meshes, mats, starts):
        blob += struct.pack("<2I5f", mesh.nodes, mesh.tets, mat.density, mat.youngs_modulus, mat.poissons_ratio,
                            mat.yield_stress, mat.hardening_modulus)
        blob += mesh.rest_positions.astype(np.float32).tobytes() + mesh.node_mass.astype(np.float32).tobytes()
        blob += mesh.anchored.astype(np.uint8).tobytes()
        for e in range(mesh.tets):
            blob += mesh.tet_nodes[e].astype(np.uint32).tobytes() + mesh.rest_inverse[e].astype(np.float32).tobytes()
            blob += np.float32(mesh.volume[e]).tobytes()
        blob += st.position.astype(np.float32).tobytes() + st.velocity.astype(np.float32).tobytes()
    (work / "island.bin").write_bytes(blob)
    out = subprocess.run([str(exe), str(work / "island.bin"), str(work / "island.out")], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    raw = (work / "island.out").read_bytes()
    at = 0
    for mesh, mat, st in zip(meshes, mats, starts):
        pos = np.frombuffer(raw, np.float32, mesh.nodes * 3, at).reshape(-1, 3).astype(np.float64)
        at += pos.size * 4
        eq = np.frombuffer(raw, np.float32, mesh.tets, at)
        at += eq.size * 4
        n, evals = np.frombuffer(raw, np.uint32, 2, at)
        at += 8
        om = to_oracle(mesh)
        ostate = po.State(st.position.copy(), st.velocity.copy(), st.acceleration.copy(), st.rotation.copy(),
                          st.plastic.copy())
        omat = po.material(mat.density, mat.youngs_modulus, mat.poissons_ratio, 0.0, mat.yield_stress,
                           mat.hardening_modulus)
        as_float(ostate)  # the program starts from the float state it was given
        oevals = 0
        for _ in range(steps):
            oevals += po.step(po.F64, om, ostate, [omat], po.Settings(), GRAVITY, DT).plastic_evaluations
            as_float(ostate)
        assert float_close(pos, ostate.position, mesh.rest_positions)
        # the float host state rounds every step, which can move a Newton stopping decision by one
        assert n == steps and abs(int(evals) - oevals) <= max(2, oevals // 5)
        if np.isfinite(mat.yield_stress):
            assert (ostate.plastic[:, 9] > 0).any()
            assert np.abs(eq - ostate.plastic[:, 9]).max() <= 1e-4 * ostate.plastic[:, 9].max()


def test_solver_state_through_the_adapter(tmp_path):
    """deformable::step with a caller-held DeformableSolverState*: the adapter
    turns the device factor on and writes SolverStats back (one refresh for
    the first factored step)."""
    from tests.test_adapter import PROGRAM as SMALL
    if shutil.which("g++") is None:
        pytest.skip("g++ missing")
    capi.lib()
    stub = tmp_path / "talus" / "deformable" / "solver"
    stub.mkdir(parents=True)
    (stub / "solver.h").write_text(STAND_IN)
    (tmp_path / "main.cc").write_text(SMALL)
    exe = tmp_path / "adapter"
    libdir = os.path.join(ROOT, "talus_b200")
    subprocess.run(["g++", "-std=c++20", "-Wall", "-Werror", f"-I{tmp_path}", f"-I{os.path.join(ROOT, 'include')}",
                    "-o", str(exe), str(tmp_path / "main.cc"), f"-L{libdir}", "-ltalus_fem", f"-Wl,-rpath,{libdir}"],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "factored 0 refactors 1" in out.stdout, out.stdout
