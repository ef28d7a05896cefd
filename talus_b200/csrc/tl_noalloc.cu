// tl_noalloc.cu -- tl_step_noalloc: one tet FEM step of one small body that
// allocates nothing.
//
// Who needs this: callers that may not allocate device memory at all -- the
// frame loop of a game or robotics engine that works inside a fixed GPU memory
// budget decided at start-up, or a host program that hands out GPU memory only
// through its own pool and forbids libraries to call cudaMalloc behind its
// back.  Such callers cannot use tl_system_create, which allocates the device
// buffers of a resident system.
//
// How: every device buffer of the step lives in one file-scope
// `static __device__` array, tl_noalloc_arena, of a fixed size
// (TL_NOALLOC_ARENA_BYTES; every GPU that loads the library holds it until the
// process exits).  Host-side staging uses static host arrays.  The host code
// never calls cudaMalloc, cudaFree, cudaMallocHost or the C++ heap.  In host
// code the array's name is only a host-side stand-in for it: its device
// address comes from cudaGetSymbolAddress, called once per device (with that
// device current) by the first call on it, which also loads every kernel the
// step launches.  That first call should therefore be made before any stream
// capture begins.
//
// Every call shares the one arena and the static host arrays: calls are
// serialised by a host mutex, and the arena keeps the previous call's
// contents, so everything that must start at zero is cleared at the start of
// each call.  Work from two processes or two devices does not share it, but
// two calls whose GPU work overlaps (for example from two host threads
// bypassing the mutex through separate library copies) would race.
//
// Scope: FP64 arithmetic, one body, at most TL_NOALLOC_MAX_NODES nodes,
// TL_NOALLOC_MAX_TETS tets and TL_NOALLOC_MAX_LANES material lanes, the
// reference's step without its plastic Newton loop (plastic_passes <= 1 or no
// yielding material) and without stiffness damping; larger inputs are refused
// with TL_ERR_TOO_LARGE, the Newton and damping cases with TL_ERR_UNSUPPORTED.
// It runs the same kernels as tl_step (kElement, kNodeAssemble, kPcg, ...),
// issues its copies and launches on the legacy default stream (stream 0),
// synchronises that stream, and returns after the step has finished.

#include "../../include/talus_fem.h"
#include "tl_kernels.cuh"
#include "tl_validate.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>

using namespace tl;

namespace {

constexpr uint32_t NA_VP = TL_NOALLOC_MAX_NODES;  // multiples of TILE
constexpr uint32_t NA_TP = TL_NOALLOC_MAX_TETS;
constexpr uint32_t NA_LANES = TL_NOALLOC_MAX_LANES + 1;  // + the default lane (material.cc:9-16)
constexpr uint32_t NA_NODE_TILES = NA_VP / TILE, NA_ELEM_TILES = NA_TP / TILE;
static_assert(NA_VP % TILE == 0 && NA_TP % TILE == 0, "capacities are whole tiles");

static __device__ __align__(256) unsigned char tl_noalloc_arena[TL_NOALLOC_ARENA_BYTES];

using S = double;

// Bump allocator over the arena: the same order of takes at set-up and at
// every call gives every buffer a fixed place.
struct Carve {
  unsigned char* base;
  size_t used = 0;
  template <class T> T* take(size_t n) {
    used = (used + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += n * sizeof(T);
    return p;
  }
};

struct Layout {
  BodyDev* body;
  BodyStepDev* step;
  MatDev* mat;
  uint32_t *nodeTileBody, *elemTileBody, *start, *entry, *lane, *loading, *yielding, *counter;
  Vec4<S> *rest4, *pres, *u, *v, *a, *carried, *shifted, *weighted, *total, *incr, *right, *pre0, *pre1, *r, *z, *p,
      *ap, *fe, *de, *ye, *plast, *onorm;
  OpRec<S>* orec;
  uint8_t* anch;
  uint4* tet;
  double *dm, *vold, *eyoung, *op, *de2, *part, *npart, *epart;
  BodyAccDev* acc;
  CgBodyDev* cg;
  CgReportDev* cgrep;
  GridSyncDev* sync;
  size_t bytes;
};

Layout carve(unsigned char* base) {
  Carve c{base};
  Layout l;
  l.body = c.take<BodyDev>(1);
  l.step = c.take<BodyStepDev>(1);
  l.mat = c.take<MatDev>(NA_LANES);
  l.nodeTileBody = c.take<uint32_t>(NA_NODE_TILES);
  l.elemTileBody = c.take<uint32_t>(NA_ELEM_TILES);
  Vec4<S>** node[] = {&l.rest4, &l.pres, &l.u, &l.v, &l.a, &l.carried, &l.shifted, &l.weighted, &l.total,
                      &l.incr, &l.right, &l.pre0, &l.pre1, &l.r, &l.z, &l.p, &l.ap};
  for (Vec4<S>** q : node) *q = c.take<Vec4<S>>(NA_VP);
  l.anch = c.take<uint8_t>(NA_VP);
  l.start = c.take<uint32_t>(NA_VP + 1);
  l.entry = c.take<uint32_t>(size_t(4) * NA_TP);
  l.tet = c.take<uint4>(NA_TP);
  l.dm = c.take<double>(size_t(9) * NA_TP);
  l.vold = c.take<double>(NA_TP);
  l.eyoung = c.take<double>(NA_TP);
  l.lane = c.take<uint32_t>(NA_TP);
  l.op = c.take<double>(size_t(9) * NA_TP);
  l.orec = c.take<OpRec<S>>(NA_TP);
  l.onorm = c.take<Vec4<S>>(size_t(2) * NA_TP);
  l.plast = c.take<Vec4<S>>(size_t(2) * NA_TP);
  l.fe = c.take<Vec4<S>>(size_t(4) * NA_TP);
  l.de = c.take<Vec4<S>>(size_t(4) * NA_TP);
  l.de2 = c.take<double>(size_t(4) * NA_TP);
  l.ye = c.take<Vec4<S>>(size_t(4) * NA_TP);
  l.part = c.take<double>(size_t(4) * NA_NODE_TILES);
  l.npart = c.take<double>(size_t(2) * NA_NODE_TILES);
  l.epart = c.take<double>(NA_ELEM_TILES);
  l.loading = c.take<uint32_t>(1);
  l.yielding = c.take<uint32_t>(1);
  l.counter = c.take<uint32_t>(1);
  l.acc = c.take<BodyAccDev>(1);
  l.cg = c.take<CgBodyDev>(1);
  l.cgrep = c.take<CgReportDev>(1);
  l.sync = c.take<GridSyncDev>(1);
  l.bytes = c.used;
  return l;
}

// Per-device set-up: the arena's device address and the PCG grid sizes.
struct DeviceSetup {
  bool ready = false;
  unsigned char* arena = nullptr;
  int pcgGrid[2] = {0, 0};
};
constexpr int NA_MAX_DEVICES = 64;
DeviceSetup g_setup[NA_MAX_DEVICES];
std::mutex g_mutex;

// Static host staging (the arena's host-side twin).
Vec4<S> h_rest4[NA_VP], h_pres[NA_VP], h_node[3][NA_VP];
uint8_t h_anch[NA_VP];
uint32_t h_start[NA_VP + 1], h_cursor[NA_VP], h_entry[4 * NA_TP], h_lane[NA_TP], h_tileBody[NA_ELEM_TILES];
uint4 h_tet[NA_TP];
double h_dm[9 * NA_TP], h_vol[NA_TP], h_eyoung[NA_TP], h_op[9 * NA_TP];
Vec4<S> h_plast[2 * NA_TP];
MatDev h_mat[NA_LANES];
BodyDev h_body;
BodyStepDev h_step;
BodyAccDev h_acc;
CgReportDev h_rep;
GridSyncDev h_sync;
uint32_t h_count;

int32_t setupDevice(int32_t device, DeviceSetup*& out) {
  if (device < 0 || device >= NA_MAX_DEVICES) return TL_ERR_ARG;
  DeviceSetup& d = g_setup[device];
  if (!d.ready) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, tl_noalloc_arena) != cudaSuccess || ptr == nullptr) return TL_ERR_CUDA;
    if (carve(nullptr).bytes > TL_NOALLOC_ARENA_BYTES) return TL_ERR_TOO_LARGE;  // layout exceeds the arena
    int sms = 0, perSm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return TL_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kPcg<S, 0>, TILE, 0) != cudaSuccess || perSm < 1)
      return TL_ERR_CUDA;
    d.pcgGrid[0] = std::min(perSm * sms, int(std::max(NA_NODE_TILES, NA_ELEM_TILES)));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kPcg<S, 1>, TILE, 0) != cudaSuccess || perSm < 1)
      return TL_ERR_CUDA;
    d.pcgGrid[1] = std::min(perSm * sms, int(std::max(NA_NODE_TILES, NA_ELEM_TILES)));
    // Every kernel a step can launch is loaded here, by the first call, so
    // later calls load no module code (CUDA may load kernels lazily, on their
    // first launch).
    const void* kernels[] = {(const void*)kInversionCheck<S>, (const void*)kPcgPrepare<S>, (const void*)kPcg<S, 0>,
                             (const void*)kPcg<S, 1>,          (const void*)kPredict<S>,     (const void*)kElement<S, 0>,
                             (const void*)kElement<S, 1>,      (const void*)kNodeAssemble<S>, (const void*)kAddIncrement<S>,
                             (const void*)kUpdate<S>,          (const void*)kStepEnd<S>,     (const void*)kFinalize};
    for (const void* k : kernels) {
      cudaFuncAttributes attr;
      if (cudaFuncGetAttributes(&attr, k) != cudaSuccess) return TL_ERR_CUDA;
    }
    // the element pass's shared-memory stage is above the default 48 KB
    for (const void* k : {(const void*)kElement<S, 0>, (const void*)kElement<S, 1>})
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(elementStageBytes<S>())) !=
          cudaSuccess)
        return TL_ERR_CUDA;
    d.arena = static_cast<unsigned char*>(ptr);
    d.ready = true;
  }
  out = &d;
  return TL_OK;
}

Sys<S> viewOf(const Layout& l, uint32_t Vp, uint32_t Tp, bool perElementYoungs) {
  Sys<S> s;
  std::memset(&s, 0, sizeof(s));
  s.bodies = 1;
  s.Vp = Vp;
  s.Tp = Tp;
  s.node_tiles = Vp / TILE;
  s.elem_tiles = Tp / TILE;
  s.body = l.body;
  s.step = l.step;
  s.mat = l.mat;
  s.node_tile_body = l.nodeTileBody;
  s.elem_tile_body = l.elemTileBody;
  s.rest4 = l.rest4;
  s.anch = l.anch;
  s.pres = l.pres;
  s.u = l.u;
  s.v = l.v;
  s.a = l.a;
  s.carried = l.carried;
  s.shifted = l.shifted;
  s.weighted = l.weighted;
  s.total = l.total;
  s.incr = l.incr;
  s.right = l.right;
  s.pre0 = l.pre0;
  s.pre1 = l.pre1;
  s.r = l.r;
  s.z = l.z;
  s.p = l.p;
  s.ap = l.ap;
  s.start = l.start;
  s.entry = l.entry;
  s.tet = l.tet;
  s.dm = l.dm;
  s.dms = l.dm;
  s.vold = l.vold;
  s.vols = l.vold;
  s.lane = l.lane;
  s.eyoung = perElementYoungs ? l.eyoung : nullptr;
  s.op = l.op;
  s.orec = l.orec;
  s.sell_val = nullptr;
  s.sell_diag = nullptr;
  s.onorm = l.onorm;
  s.plast = l.plast;
  s.fe = l.fe;
  s.de = l.de;
  s.de2 = l.de2;
  s.ye = l.ye;
  s.part = l.part;
  s.npart = l.npart;
  s.epart = l.epart;
  s.loading = l.loading;
  s.yielding = l.yielding;
  s.acc = l.acc;
  s.cg = l.cg;
  s.cgrep = l.cgrep;
  s.counter = l.counter;
  s.sync = l.sync;
  return s;
}

template <class H> double at(const void* p, size_t i) { return double(static_cast<const H*>(p)[i]); }
template <class H> void put(void* p, size_t i, double v) { static_cast<H*>(p)[i] = H(v); }

#define NA_CUDA(call)                                \
  do {                                               \
    if ((call) != cudaSuccess) return TL_ERR_CUDA;   \
  } while (0)

int32_t stepLocked(int32_t device, const tl_mesh_desc& d, int32_t dtype, void* position, void* velocity,
                   void* acceleration, void* rotation, void* plastic, const tl_settings& set, const double gvec[3],
                   double dt, tl_step_report* report) {
  // ---- validation (no allocation below this point, ever)
  if (d.nodes == 0 || d.tets == 0 || !position || !velocity || !acceleration) return TL_ERR_ARG;
  if (d.nodes > TL_NOALLOC_MAX_NODES || d.tets > TL_NOALLOC_MAX_TETS || d.lanes > TL_NOALLOC_MAX_LANES)
    return TL_ERR_TOO_LARGE;
  if (meshDescProblem(d) || set.law > 1u || !stepArgumentsValid(dt, gvec)) return TL_ERR_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device >= count) return TL_ERR_NO_DEVICE;
  NA_CUDA(cudaSetDevice(device));
  DeviceSetup* dev = nullptr;
  const int32_t rc = setupDevice(device, dev);
  if (rc != TL_OK) return rc;
  const Layout l = carve(dev->arena);
  const uint32_t Vp = ((d.nodes + TILE - 1) / TILE) * TILE, Tp = ((d.tets + TILE - 1) / TILE) * TILE;
  const int law = int(set.law);
  // ---- materials (material.cc:71-78, 747-749) and the default lane
  bool anyYields = false, anyAnchored = false;
  bool laneDamps[NA_LANES];
  for (uint32_t k = 0; k <= d.lanes; ++k) {
    const tl_material m = k < d.lanes ? d.materials[k]
                                      : tl_material{1000.0, 0.0, 0.3, 0.0, std::numeric_limits<double>::infinity(), 0.0};
    // stiffnessDamping counts when finite and positive (factor.cc:755-759), the rule tl_system_create applies
    laneDamps[k] = std::isfinite(m.stiffness_damping) && m.stiffness_damping > 0.0;
    const double nu = std::clamp(m.poissons_ratio, 0.0, 0.49);
    h_mat[k] = MatDev{nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), 1.0 / (2.0 * (1.0 + nu)), m.youngs_modulus, m.yield_stress,
                      m.hardening_modulus, (std::isfinite(m.yield_stress) && m.yield_stress > 0.0) ? 1u : 0u, 0u};
  }
  // ---- nodes: rest + mass, anchors, prescribed velocity, state as displacement
  for (uint32_t n = 0; n < Vp; ++n) {
    const bool real = n < d.nodes;
    h_rest4[n] = real ? Vec4<S>{d.rest_positions[3 * n], d.rest_positions[3 * n + 1], d.rest_positions[3 * n + 2],
                                d.node_mass[n]}
                      : Vec4<S>{0, 0, 0, 0};
    h_anch[n] = real ? (d.anchored[n] ? 1u : 0u) : 1u;
    anyAnchored = anyAnchored || (real && d.anchored[n]);
    h_pres[n] = (real && d.prescribed_velocity && d.anchored[n])
                    ? Vec4<S>{d.prescribed_velocity[3 * n], d.prescribed_velocity[3 * n + 1],
                              d.prescribed_velocity[3 * n + 2], 0}
                    : Vec4<S>{0, 0, 0, 0};
    for (int q = 0; q < 3; ++q) {
      const void* src = q == 0 ? position : (q == 1 ? velocity : acceleration);
      Vec4<S> w = {0, 0, 0, 0};
      if (real) {
        for (int k = 0; k < 3; ++k) {
          double x = dtype == TL_DTYPE_F64 ? at<double>(src, 3 * n + k) : at<float>(src, 3 * n + k);
          if (q == 0) x -= d.rest_positions[3 * n + k];
          (&w.x)[k] = x;
        }
      }
      h_node[q][n] = w;
    }
  }
  if (!anyAnchored && set.rigid_split != TL_RIGID_SPLIT_OFF) return TL_ERR_UNSUPPORTED;
  // ---- elements and the node -> (element, corner) CSR in element order
  std::fill(h_start, h_start + Vp + 1, 0u);
  for (uint32_t e = 0; e < Tp; ++e) {
    const bool real = e < d.tets;
    uint32_t q[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4 && real; ++k) {
      q[k] = d.tet_nodes[4 * size_t(e) + k];
      if (q[k] >= d.nodes) return TL_ERR_ARG;
      ++h_start[q[k] + 1];
    }
    h_tet[e] = make_uint4(q[0], q[1], q[2], q[3]);
    for (int k = 0; k < 9; ++k) h_dm[size_t(k) * Tp + e] = real ? d.rest_inverse[9 * size_t(e) + k] : 0.0;
    h_vol[e] = real ? d.volume[e] : 0.0;
    const uint32_t ln = real && d.material[e] < d.lanes ? d.material[e] : d.lanes;
    h_lane[e] = ln;
    // the damping fit planes are an allocation this entry point does not make
    if (real && laneDamps[ln]) return TL_ERR_UNSUPPORTED;
    h_eyoung[e] = (real && d.element_youngs) ? d.element_youngs[e] : h_mat[ln].youngs;
    anyYields = anyYields || (real && h_mat[ln].yields);
    for (int k = 0; k < 9; ++k)
      h_op[size_t(k) * Tp + e] = (real && rotation) ? (dtype == TL_DTYPE_F64 ? at<double>(rotation, 9 * size_t(e) + k)
                                                                             : at<float>(rotation, 9 * size_t(e) + k))
                                                    : ((k % 4) == 0 ? 1.0 : 0.0);
    Vec4<S> p0 = {0, 0, 0, 0}, p1 = {0, 0, 0, 0};
    if (real && plastic) {
      double g[10];
      for (int k = 0; k < 10; ++k)
        g[k] = dtype == TL_DTYPE_F64 ? at<double>(plastic, 10 * size_t(e) + k) : at<float>(plastic, 10 * size_t(e) + k);
      p0 = {g[0], g[4], g[8], 0.5 * (g[1] + g[3])};
      p1 = {0.5 * (g[2] + g[6]), 0.5 * (g[5] + g[7]), g[9], 0};
    }
    h_plast[e] = p0;
    h_plast[Tp + e] = p1;
  }
  if (law == TL_LAW_SNH) anyYields = false;
  if (anyYields && set.plastic_passes > 1u) return TL_ERR_UNSUPPORTED;  // the Newton loop runs in tl_step
  for (uint32_t n = 0; n < Vp; ++n) h_start[n + 1] += h_start[n];
  std::copy(h_start, h_start + Vp, h_cursor);
  for (uint32_t e = 0; e < d.tets; ++e) {
    const uint32_t q[4] = {h_tet[e].x, h_tet[e].y, h_tet[e].z, h_tet[e].w};
    for (int k = 0; k < 4; ++k) h_entry[h_cursor[q[k]]++] = 4 * e + uint32_t(k);
  }
  for (uint32_t t = 0; t < NA_ELEM_TILES; ++t) h_tileBody[t] = 0u;
  h_body = BodyDev{0u, d.nodes, 0u, Vp / TILE, 0u, d.tets, 0u, Tp / TILE};
  // ---- integrator constants (solver.cc:538-566) and the inversion test (solver.cc:3574-3583)
  const double held = std::clamp(set.spectral_radius, 0.0, 1.0);
  const double am = (2.0 * held - 1.0) / (held + 1.0), af = held / (held + 1.0);
  const double gamma = 0.5 - am + af, beta = 0.25 * (1.0 - am + af) * (1.0 - am + af);
  const uint32_t configured = std::max(set.substeps, 1u);
  std::memset(&h_step, 0, sizeof(h_step));
  h_step.substeps = configured;
  h_step.limit = set.cg_iterations;
  h_step.alpha_f = af;
  h_step.alpha_m = am;
  h_step.beta = beta;
  h_step.gamma = gamma;
  h_step.gx = gvec[0];
  h_step.gy = gvec[1];
  h_step.gz = gvec[2];
  h_step.tolerance = set.tolerance;
  h_step.check_inner = dt / double(configured);
  h_step.check_carry = (0.5 - beta) * h_step.check_inner * h_step.check_inner;
  // ---- upload (plain copies into the arena) and clear what must start at zero
  cudaStream_t st = 0;
  NA_CUDA(cudaMemcpyAsync(l.body, &h_body, sizeof(h_body), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.step, &h_step, sizeof(h_step), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.mat, h_mat, sizeof(MatDev) * (d.lanes + 1), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.nodeTileBody, h_tileBody, sizeof(uint32_t) * NA_NODE_TILES, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.elemTileBody, h_tileBody, sizeof(uint32_t) * NA_ELEM_TILES, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.rest4, h_rest4, sizeof(Vec4<S>) * Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.pres, h_pres, sizeof(Vec4<S>) * Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.anch, h_anch, Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.u, h_node[0], sizeof(Vec4<S>) * Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.v, h_node[1], sizeof(Vec4<S>) * Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.a, h_node[2], sizeof(Vec4<S>) * Vp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.start, h_start, sizeof(uint32_t) * (Vp + 1), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.entry, h_entry, sizeof(uint32_t) * 4 * d.tets, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.tet, h_tet, sizeof(uint4) * Tp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.dm, h_dm, sizeof(double) * 9 * Tp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.vold, h_vol, sizeof(double) * Tp, cudaMemcpyHostToDevice, st));
  if (d.element_youngs)
    NA_CUDA(cudaMemcpyAsync(l.eyoung, h_eyoung, sizeof(double) * Tp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.lane, h_lane, sizeof(uint32_t) * Tp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.op, h_op, sizeof(double) * 9 * Tp, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(l.plast, h_plast, sizeof(Vec4<S>) * 2 * Tp, cudaMemcpyHostToDevice, st));
  std::memset(&h_acc, 0, sizeof(h_acc));
  h_acc.min_j_key = ~0ull;
  NA_CUDA(cudaMemcpyAsync(l.acc, &h_acc, sizeof(h_acc), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemsetAsync(l.cgrep, 0, sizeof(CgReportDev), st));
  NA_CUDA(cudaMemsetAsync(l.cg, 0, sizeof(CgBodyDev), st));
  NA_CUDA(cudaMemsetAsync(l.counter, 0, sizeof(uint32_t), st));
  NA_CUDA(cudaMemsetAsync(l.sync, 0, sizeof(GridSyncDev), st));
  NA_CUDA(cudaMemsetAsync(l.loading, 0, sizeof(uint32_t), st));
  NA_CUDA(cudaMemsetAsync(l.yielding, 0, sizeof(uint32_t), st));
  NA_CUDA(cudaMemsetAsync(l.orec, 0, sizeof(OpRec<S>) * Tp, st));
  NA_CUDA(cudaMemsetAsync(l.onorm, 0, sizeof(Vec4<S>) * 2 * Tp, st));
  const Sys<S> s = viewOf(l, Vp, Tp, d.element_youngs != nullptr);
  const uint32_t nodeTiles = Vp / TILE, elemTiles = Tp / TILE;
  uint32_t launches = 0;
  // ---- predictor inversion test -> substeps
  kInversionCheck<S><<<elemTiles, TILE, 0, st>>>(s);
  ++launches;
  NA_CUDA(cudaGetLastError());
  NA_CUDA(cudaMemcpyAsync(&h_acc, l.acc, sizeof(h_acc), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  h_step.substeps = h_acc.inverts ? std::max(configured, 4u) : configured;  // INVERTED_SUBSTEPS (solver.cc:13)
  h_step.inner = dt / double(h_step.substeps);
  h_step.carry = (0.5 - beta) * h_step.inner * h_step.inner;
  h_step.inertia = 1.0 - am;
  h_step.hstep = std::sqrt((1.0 - af) * beta) * h_step.inner;
  h_step.scale = h_step.hstep * h_step.hstep;
  NA_CUDA(cudaMemcpyAsync(l.step, &h_step, sizeof(h_step), cudaMemcpyHostToDevice, st));
  auto pcg = [&](Vec4<S>* X, uint32_t pass, bool x0zero) -> int32_t {
    kPcgPrepare<S><<<1, TILE, 0, st>>>(s, pass);
    Sys<S> sv = s;
    uint32_t ps = pass, xz = x0zero ? 1u : 0u, tg = 0u;
    void* args[] = {&sv, &X, &ps, &xz, &tg};
    const void* fn = law == TL_LAW_SNH ? (const void*)kPcg<S, 1> : (const void*)kPcg<S, 0>;
    launches += 2;
    return cudaLaunchCooperativeKernel(fn, dim3(dev->pcgGrid[law == TL_LAW_SNH ? 1 : 0]), dim3(TILE), args, 0, st) ==
                   cudaSuccess
               ? TL_OK
               : TL_ERR_CUDA;
  };
  auto element = [&](const Vec4<S>* base, const Vec4<S>* dir, uint32_t pass, uint32_t mode) -> int32_t {
    if (!(mode & EM_COMMIT)) {
      if (cudaMemsetAsync(l.loading, 0, sizeof(uint32_t), st) != cudaSuccess ||
          cudaMemsetAsync(l.yielding, 0, sizeof(uint32_t), st) != cudaSuccess)
        return TL_ERR_CUDA;
    }
    if (anyYields) mode |= EM_YIELDING;
    if (law == TL_LAW_SNH) kElement<S, 1><<<elemTiles, TILE, elementStageBytes<S>(), st>>>(s, base, dir, pass, mode, 0.0);
    else kElement<S, 0><<<elemTiles, TILE, elementStageBytes<S>(), st>>>(s, base, dir, pass, mode, 0.0);
    ++launches;
    return cudaGetLastError() == cudaSuccess ? TL_OK : TL_ERR_CUDA;
  };
  // ---- substeps: predictor, the three anchored reads (solver.cc:3914-3950), update, plastic commit
  for (uint32_t pass = 0; pass < h_step.substeps; ++pass) {
    kPredict<S><<<nodeTiles, TILE, 0, st>>>(s, pass);
    if (element(l.weighted, nullptr, pass, EM_MAPPING) != TL_OK) return TL_ERR_CUDA;
    kNodeAssemble<S><<<nodeTiles, TILE, 0, st>>>(s, nullptr, pass);
    launches += 2;
    if (pcg(l.a, pass, false) != TL_OK) return TL_ERR_CUDA;
    for (uint32_t read = 1; read != 3u; ++read) {
      if (element(l.weighted, l.a, pass, EM_MAPPING) != TL_OK) return TL_ERR_CUDA;
      kNodeAssemble<S><<<nodeTiles, TILE, 0, st>>>(s, l.a, pass);
      ++launches;
      if (pcg(l.incr, pass, true) != TL_OK) return TL_ERR_CUDA;
      kAddIncrement<S><<<nodeTiles, TILE, 0, st>>>(s, l.a, pass);
      ++launches;
    }
    kUpdate<S><<<nodeTiles, TILE, 0, st>>>(s, pass);
    ++launches;
    if (anyYields && element(l.u, nullptr, pass, EM_MAPPING | EM_COMMIT) != TL_OK) return TL_ERR_CUDA;
  }
  kStepEnd<S><<<nodeTiles, TILE, 0, st>>>(s);
  kFinalize<<<1, TILE, 0, st>>>(l.body, l.epart, l.npart, l.acc, 0);
  kFinalize<<<1, TILE, 0, st>>>(l.body, l.epart, l.npart, l.acc, 2);
  launches += 3;
  NA_CUDA(cudaGetLastError());
  NA_CUDA(cudaMemcpyAsync(&h_acc, l.acc, sizeof(h_acc), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&h_rep, l.cgrep, sizeof(h_rep), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&h_sync, l.sync, sizeof(h_sync), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(&h_count, l.yielding, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(h_node[0], l.u, sizeof(Vec4<S>) * d.nodes, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(h_node[1], l.v, sizeof(Vec4<S>) * d.nodes, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaMemcpyAsync(h_node[2], l.a, sizeof(Vec4<S>) * d.nodes, cudaMemcpyDeviceToHost, st));
  if (rotation) NA_CUDA(cudaMemcpyAsync(h_op, l.op, sizeof(double) * 9 * Tp, cudaMemcpyDeviceToHost, st));
  if (plastic) NA_CUDA(cudaMemcpyAsync(h_plast, l.plast, sizeof(Vec4<S>) * 2 * Tp, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
  if (h_sync.error != 0) return TL_ERR_TIMEOUT;
  // ---- state back to the caller
  for (uint32_t n = 0; n < d.nodes; ++n)
    for (int q = 0; q < 3; ++q) {
      void* dst = q == 0 ? position : (q == 1 ? velocity : acceleration);
      for (int k = 0; k < 3; ++k) {
        double x = (&h_node[q][n].x)[k];
        if (q == 0) x += d.rest_positions[3 * n + k];
        if (dtype == TL_DTYPE_F64) put<double>(dst, 3 * n + k, x);
        else put<float>(dst, 3 * n + k, x);
      }
    }
  for (uint32_t e = 0; e < d.tets; ++e) {
    if (rotation)
      for (int k = 0; k < 9; ++k) {
        if (dtype == TL_DTYPE_F64) put<double>(rotation, 9 * size_t(e) + k, h_op[size_t(k) * Tp + e]);
        else put<float>(rotation, 9 * size_t(e) + k, h_op[size_t(k) * Tp + e]);
      }
    if (plastic) {
      const Vec4<S> a0 = h_plast[e], a1 = h_plast[Tp + e];
      const double g[10] = {a0.x, a0.w, a1.x, a0.w, a0.y, a1.y, a1.x, a1.y, a0.z, a1.z};
      for (int k = 0; k < 10; ++k) {
        if (dtype == TL_DTYPE_F64) put<double>(plastic, 10 * size_t(e) + k, g[k]);
        else put<float>(plastic, 10 * size_t(e) + k, g[k]);
      }
    }
  }
  if (report) {
    report->nodes += d.nodes;
    report->elements += d.tets;
    report->substeps += h_step.substeps;
    report->cg_iterations += h_rep.iterations;
    report->cg_capped_solves += h_rep.capped;
    report->operator_applications += h_rep.applications;
    report->cg_solves += h_rep.solves;
    report->cg_worst_relative_residual = std::max(report->cg_worst_relative_residual, h_rep.worst_rel);
    report->yielding = h_count;
    report->plastic_growth |= h_acc.grew;
    report->non_finite |= h_acc.nonfinite;
    report->elastic_energy += h_acc.energy;
    report->kinetic_energy += h_acc.kinetic;
    report->min_volume_ratio = fromMinKey(h_acc.min_j_key);
    report->kernel_launches += launches;
  }
  return h_acc.nonfinite ? TL_ERR_NONFINITE : TL_OK;
}

}  // namespace

extern "C" int32_t tl_step_noalloc(int32_t device, const tl_mesh_desc* mesh, int32_t dtype, void* position,
                                   void* velocity, void* acceleration, void* rotation, void* plastic,
                                   const tl_settings* settings, const double gravity[3], double dt,
                                   tl_step_report* report) {
  if (!mesh || !settings || !gravity || (dtype != TL_DTYPE_F32 && dtype != TL_DTYPE_F64)) return TL_ERR_ARG;
  std::lock_guard<std::mutex> hold(g_mutex);
  return stepLocked(device, *mesh, dtype, position, velocity, acceleration, rotation, plastic, *settings, gravity,
                    dt, report);
}
