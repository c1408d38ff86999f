// Host side of the activechi4 B200 engine: device memory arena, tiling,
// CUDA-graph construction (with a device-decided conditional for the list
// rebuild) and the C ABI declared in include/activechi4.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/activechi4.h"
#include "acg_kernels.cuh"

using namespace acg;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(ACG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)

constexpr double TAU_T = 0.20;  // MDcode/time_evolve.c:477
constexpr int GRAPH_STEPS = 32;
constexpr int BENCH_MAX_GRAPH = 256;  // acg_bench_steps: one graph for up to this many steps

struct Layout {
  int nsys = 0, nslots = 0, ncells = 0, nact = 0, maxnb = 0, ngroups = 0, ngtiles = 0, nboxtiles = 0, box_nmax = 0;
  int nact_max = 0;  // most active particles of one system
  int nboxcap = 0;   // whole-box tiles at one cell per block (the most any partition needs)
  int box_m3max = 0;  // most list sub-cells of a whole-box system (0: none uses them)
  int box_cell_nmax = 0;  // most particles of a whole-box system listed from its cells
  int nsub = 0;           // sub-cell starts of all whole-box systems with list sub-cells
  std::vector<SysDesc> desc;
  size_t bytes = 0;
};

double sigma_of(int tsum) { return tsum == 0 ? 1.00 : (tsum == 1 ? 0.80 : 0.88); }

int resolve(const acg_params &p, SysDesc &d) {
  if (p.n < 2) return fail(ACG_ERR_INVALID, "n must be >= 2");
  memset(&d, 0, sizeof(d));
  d.n = p.n;
  d.nact = p.nact < 0 ? (int)((double)p.n * 0.1) : p.nact;
  if (d.nact > d.n) return fail(ACG_ERR_INVALID, "nact > n");
  double L = p.L > 0 ? p.L : std::pow((double)p.n / p.density, 0.33333333);
  if (!(L > 0) || !std::isfinite(L)) return fail(ACG_ERR_INVALID, "bad box length");
  const double cell_cut = 2.5 * 1.00 + p.skin;  // Cell_cut (MDcode/global.h:29)
  // Ncell = (int)Lpp / Cell_cut with the cast on Lpp (MDcode/Parallel.c:72)
  int nc = (int)((double)(int)L / cell_cut);
  if (nc < 2)
    return fail(ACG_ERR_INVALID, "box too small: need at least 2 cells of size >= 2.5+skin per side");
  double cs = L / (double)nc;
  d.nc = nc;
  d.ncell = nc * nc * nc;
  d.L = L;
  d.invL = 1.0 / L;
  d.inv_cell = L / cs;  // InvCellSize (MDcode/Parallel.c:78)
  d.cell_cut = cell_cut;
  // DENSITY: read from the parameter file where L follows from it, else N / L^3
  d.density = p.L > 0 ? (double)p.n / (L * L * L) : p.density;
  d.P = p.P;
  d.L0 = L;
  d.T = p.T;
  d.f0 = p.f0;
  d.dt = p.dt;
  d.half_dt = p.dt * 0.5;
  d.skin2 = p.skin * p.skin;
  d.rebuild_factor = p.rebuild_factor;
  d.dof = 3.0 * (double)p.n - 3.0;  // DOF (MDcode/global.h:35)
  for (int i = 0; i < NHC_M; i++) d.q[i] = p.T * TAU_T * TAU_T;
  d.q[0] = d.dof * p.T * TAU_T * TAU_T;
  for (int i = 0; i < NHC_M; i++) d.q_baro[i] = p.T * TAU_P * TAU_P;
  d.w_eps = d.dof * p.T * TAU_P * TAU_P;
  for (int t = 0; t < 3; t++) {
    double rl = p.list_mode == 0 ? cell_cut : 2.5 * sigma_of(t) + p.skin;
    d.lcut2[t] = rl * rl;
  }
  d.tau_p = p.tau_p_steps;
  d.thermostat = p.thermostat;
  d.shuffle = p.shuffle;
  d.drift_every = p.drift_every;
  d.list_mode = p.list_mode;
  d.precision = p.precision;
  d.seed = p.seed;
  if (p.dt <= 0 || p.skin <= 0 || p.rebuild_factor <= 0)
    return fail(ACG_ERR_INVALID, "dt, skin and rebuild_factor must be positive");
  if (p.thermostat < 0 || p.thermostat > 6) return fail(ACG_ERR_INVALID, "thermostat must be 0 to 6");
  if (p.thermostat && !(p.T > 0)) return fail(ACG_ERR_INVALID, "thermostat needs T > 0");
  if (p.shuffle < 0 || p.shuffle > 2) return fail(ACG_ERR_INVALID, "shuffle must be 0, 1 or 2");
  if (p.shuffle && p.tau_p_steps <= 0) return fail(ACG_ERR_INVALID, "shuffle needs tau_p_steps > 0");
  if (p.drift_every < 0) return fail(ACG_ERR_INVALID, "drift_every must be >= 0");
  return ACG_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int plan(const acg_params *params, int nsys, Layout &lay, int nsm) {
  if (!params || nsys < 1) return fail(ACG_ERR_INVALID, "need at least one system");
  lay = Layout();
  lay.nsys = nsys;
  lay.desc.resize(nsys);
  double dens_max = 0;
  for (int r = 0; r < nsys; r++) {
    int rc = resolve(params[r], lay.desc[r]);
    if (rc) return fail(rc, "system " + std::to_string(r) + ": " + g_err);
    if (params[r].precision != params[0].precision)
      return fail(ACG_ERR_INVALID, "all systems of an engine share one precision");
    SysDesc &d = lay.desc[r];
    d.poff = lay.nslots;
    d.coff = lay.ncells;
    d.aoff = lay.nact;
    d.box = d.nc >= 2 && d.nc <= MAX_BOX_NC && d.n <= MAX_BOX_N;
    d.ng = d.nc >= 3 && !d.box && d.n > PARTICLE_MAX ? (d.nc + 1) / 2 : 0;
    d.goff = lay.ngroups;
    lay.ngroups += d.ng * d.ng * d.ng;
    // force blocks per cell group: a small box has few groups, each split over
    // up to GSPLIT_MAX blocks (contiguous runs of its centre particles) so that
    // about GSPLIT_BLOCKS blocks share the pair work; depends on the system
    // alone, so its results do not depend on the engine it is in
    d.gsplit = d.ng > 0 ? std::max(1, std::min(GSPLIT_MAX, GSPLIT_BLOCKS / (d.ng * d.ng * d.ng))) : 1;
    d.gtile0 = lay.ngtiles;
    lay.ngtiles += d.ng * d.ng * d.ng * d.gsplit;
    if (d.box) lay.box_nmax = std::max(lay.box_nmax, d.n);
    // list sub-cells of a whole box: side >= 1.45 and >= half the widest list
    // cut, so a partner is at most two sub-cells away on each axis; at least 5
    // per side (each of the 5 x 5 x 5 neighbours once), else the cell path
    d.msub = 0;
    if (d.box) {
      double rl = 0;
      for (int t = 0; t < 3; t++) rl = std::max(rl, std::sqrt(d.lcut2[t]));
      const double h = std::max(1.45, 0.5 * rl * (1.0 + 1e-9));
      const int m = (int)(d.L / h);
      if (m >= 5 && m * m * m <= MAX_SUB3) {
        d.msub = m;
        // list bricks of 2 x 2 x 2 sub-cells, or 2 x 2 x 1 where that would
        // hold more than BRICK2_MAX particles (a brick's particles past 32
        // are listed one warp each)
        const double hs = d.L / m;
        d.bz = 8.0 * hs * hs * hs * d.n / (d.L * d.L * d.L) > BRICK2_MAX ? 1 : 2;
        lay.box_m3max = std::max(lay.box_m3max, m * m * m);
        d.soff = lay.nsub;
        lay.nsub += m * m * m + 1;
      }
      if (!d.msub) lay.box_cell_nmax = std::max(lay.box_cell_nmax, d.n);
    }
    lay.nslots += (int)align_up((size_t)d.n, 32);
    lay.ncells += d.ncell;
    lay.nact += d.nact;
    lay.nact_max = std::max(lay.nact_max, d.nact);
    dens_max = std::max(dens_max, (double)d.n / (d.L * d.L * d.L));
  }
  // whole-box partition: about two blocks per SM over all whole-box cells,
  // 1 to BOX_CELLS cells per block (the per-system sums do not depend on it)
  {
    long long cells = 0;
    for (int r = 0; r < nsys; r++)
      if (lay.desc[r].box) cells += lay.desc[r].ncell;
    const int cpb = (int)std::max(1LL, std::min((long long)BOX_CELLS, cells / (2LL * std::max(nsm, 1))));
    for (int r = 0; r < nsys; r++) {
      SysDesc &d = lay.desc[r];
      // 2 cells per side: one cell (of up to ~100 particles) per block
      d.cpb = d.nc == 2 ? 1 : cpb;
      d.xoff = lay.nboxtiles;
      if (d.box) {
        lay.nboxtiles += (d.ncell + d.cpb - 1) / d.cpb;
        lay.nboxcap += d.ncell;
      }
    }
  }
  // neighbour-row capacity: 1.45x the ideal-gas count within the widest list
  // cut plus margin; rare denser particles fall back to the cell scan
  const double rl = 2.5 + params[0].skin;
  double expect = dens_max * 4.0 / 3.0 * M_PI * rl * rl * rl;
  lay.maxnb = (int)align_up((size_t)(1.45 * expect + 16.0), 32);
  lay.maxnb = std::max(lay.maxnb, 64);
  if (params[0].nb_capacity > 0) lay.maxnb = (int)align_up((size_t)params[0].nb_capacity, 32);
  const size_t S = (size_t)lay.nslots, Cn = (size_t)lay.ncells;
  size_t b = 0;
  auto add = [&](size_t n) { b += align_up(n, 256); };
  add(sizeof(SysDesc) * nsys);
  add(sizeof(SysState) * nsys);
  add(32 * S);                    // pos
  for (int k = 0; k < 12; k++) add(8 * S);
  for (int k = 0; k < 4; k++) add(4 * S);  // id act cellof nbn
  add(4 * S * (size_t)lay.maxnb); // nbl
  add(4 * (size_t)std::max(lay.nact, 1));
  add(32 * S);                    // pos_s
  for (int k = 0; k < 9; k++) add(8 * S);
  for (int k = 0; k < 5; k++) add(4 * S);  // id_s act_s cell_tmp perm_u perm
  for (int k = 0; k < 4; k++) add(4 * Cn);
  add(8 * (S / BLOCK_A + nsys + 1));      // tiles_a
  add(8 * (S / 4 + nsys + 1));            // tiles_b (>= 4 particles per block)
  add(8 * (S / PART_L + Cn + nsys + 1));  // tiles_lc (one a cell), then tiles_l
  add(8 * (Cn / CELLS_PER_TILE + nsys + 1));
  const size_t Gn = (size_t)lay.ngroups, Gt = (size_t)lay.ngtiles;
  add(8 * (Gt + 1));                      // tiles_g
  add(4 * (Gn + 1));                      // gstart
  add(8 * ((size_t)lay.nboxcap + 1));     // tiles_x
  add(32 * (Gt + lay.nboxcap + S / 4 + nsys + 1));  // part_b
  add(32 * S);                            // pacc
  add(64);                                // counters
  add(sizeof(ObsDesc) * nsys);            // observables
  add(8 * (S / BLOCK_A + nsys + 1) * OBS_EMAX * OBS_NV);  // part_o
  add(72 * S);                            // stage_d
  add(8 * S);                             // stage_i
  add(24 * S);                            // stage_f
  add(16 * S);                            // xsub
  add(4 * ((size_t)lay.nsub + 1));        // ssub
  add(4 * (2 * (size_t)nsys + 2));        // rbs
  add(4 * 2 * (size_t)MT_WORDS * nsys);   // mt
  lay.bytes = b;
  return ACG_OK;
}

}  // namespace

namespace acg {
// lets other translation units of the library report through acg_last_error
int set_last_error(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace acg

struct acg_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  Layout lay;
  void *arena = nullptr;
  View v{};
  SysDesc *d_desc = nullptr;
  int tpp = 4, block = 128, gtpp = 2, btpp = 2;  // btpp: whole-box kernels
  int ntiles_a = 0, ntiles_b = 0, ntiles_l = 0, ntiles_c = 0, ntiles_g = 0, ntiles_x = 0, ntiles_lc = 0;
  int2 *d_tiles_b = nullptr;
  int2 *d_tiles_x = nullptr;
  std::vector<int> dirty;  // systems whose forces/lists must be recomputed
  // the host's copy of each system's step counter and ramp steps left (the
  // device's st.step / st.ramp_left), to schedule drift removals between
  // graph launches
  std::vector<long long> hstep, hramp;
  bool any_dirty = false;
  bool any_gauss = false;  // a system runs the Gaussian isokinetic integrator (thermostat 3)
  bool any_npt = false;    // a system runs the Berendsen barostat (thermostat 4)
  bool any_box = false;    // a system's box length changes on the device (thermostats 4 and 5)
  bool any_brown = false;  // a system runs active Brownian dynamics (thermostat 6)
  bool desc_live = false;  // the descriptors on the device are the current ones
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  int gsteps = 0;
  cudaGraphExec_t gexec1 = nullptr;
  cudaGraph_t graph1 = nullptr;
  // device-loop graphs of acg_step: two copies of the LOOP_STEPS-step body
  // used in turn (a launch never waits for the other copy) and a 1-step body
  // for the remainder; counts[0..2] are their block counters
  cudaGraphExec_t wexec[3] = {nullptr, nullptr, nullptr};
  cudaGraph_t wgraph[3] = {nullptr, nullptr, nullptr};
  long long *counts = nullptr;
  int wturn = 0;
  bool no_while = false;  // the device loop could not be built: launch per 32 steps
  void *flush = nullptr;  // bench-only L2 flush buffer
  size_t flush_bytes = 0;
  std::map<int, std::pair<cudaGraph_t, cudaGraphExec_t>> bench;  // acg_bench_steps: graphs by step count
  std::vector<std::vector<long long>> obs_events;  // per system: steps with observable events (sorted)
  std::vector<std::vector<void *>> obs_bufs;  // per system: device buffers of the observables
  std::vector<std::vector<long long>> obs_offsets;  // per system: offset (steps) of each time bin
};

namespace {

using ForceFn = void (*)(View, int, int);
using GroupFn = void (*)(View, int);

GroupFn group_fn(int gtpp, int prec) {
  switch (gtpp) {
    case 1: return prec ? (GroupFn)k_force_groups<1, 1> : (GroupFn)k_force_groups<1, 0>;
    case 2: return prec ? (GroupFn)k_force_groups<2, 1> : (GroupFn)k_force_groups<2, 0>;
    case 4: return prec ? (GroupFn)k_force_groups<4, 1> : (GroupFn)k_force_groups<4, 0>;
  }
  return nullptr;
}
// group force kernel: 24 bytes per staged particle and one dummy slot
size_t group_smem(int gcap) { return 3 * ((size_t)gcap + 1) * sizeof(double); }
size_t list_smem(int gcap) { return ((size_t)gcap + 3 * MAX_UNION) * sizeof(float4); }
size_t list_cells_smem(int lccap) { return (size_t)lccap * sizeof(float4); }

GroupFn box_fn(int gtpp, int prec) {
  switch (gtpp) {
    case 1: return prec ? (GroupFn)k_force_box<1, 1> : (GroupFn)k_force_box<1, 0>;
    case 2: return prec ? (GroupFn)k_force_box<2, 1> : (GroupFn)k_force_box<2, 0>;
    case 4: return prec ? (GroupFn)k_force_box<4, 1> : (GroupFn)k_force_box<4, 0>;
  }
  return nullptr;
}
// whole-box staging: int4 fixed point (FP32) or three doubles (FP64) per particle
size_t box_smem(int nmax, int prec) { return (size_t)nmax * 3 * (prec ? sizeof(int) : sizeof(double)); }
// whole-box list build: the staged system padded per cell (cell path); the
// sub-cell path reads the sorted system from memory.  The sub-cell sort: two
// 16-bit arrays of n and the sub-cell starts and counters.
size_t box_list_smem_cells(int nmax) { return ((size_t)nmax + 3 * MAX_BOX_CELLS) * sizeof(float4); }
size_t box_list_smem(int cell_nmax) { return cell_nmax > 0 ? box_list_smem_cells(cell_nmax) : 0; }
// reference-order shuffle: one system's directions staged as bytes
size_t shuffle_smem(const Layout &lay) { return align_up((size_t)std::max(1, std::min(lay.nact_max, SHUF_SMEM_NACT)), 16); }
size_t sort_sub_smem(int nmax, int m3max) { return (size_t)nmax * 2 * sizeof(uint16_t) + (2 * (size_t)m3max + 1) * sizeof(int); }

ForceFn force_fn(int tpp, int prec) {
#define F(T)                                                                     \
  case T:                                                                        \
    return prec ? (ForceFn)k_force_kick<T, 1> : (ForceFn)k_force_kick<T, 0>;
  switch (tpp) {
    F(1) F(2) F(4) F(8) F(16) F(32)
  }
#undef F
  return nullptr;
}

// whole-box tiles: d.cpb cells of one system per block, the blocks of the
// largest systems first (the partition does not change any result: the
// per-system sums are taken per particle, in slot order)
int build_tiles_x(acg_engine *e) {
  std::vector<int2> h_x;
  int nt = 0;
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    d.xoff = nt;
    if (!d.box) continue;
    const int k = (d.ncell + d.cpb - 1) / d.cpb;
    for (int b = 0; b < k; b++) h_x.push_back(make_int2(r, b));
    nt += k;
  }
  if (nt > e->lay.nboxcap) return fail(ACG_ERR_INVALID, "internal: more whole-box tiles than the layout holds");
  std::stable_sort(h_x.begin(), h_x.end(), [&](int2 a, int2 b) { return e->lay.desc[a.x].n > e->lay.desc[b.x].n; });
  e->lay.nboxtiles = nt;
  e->ntiles_x = nt;
  e->v.ntiles_x = nt;
  if (!h_x.empty())
    CK(cudaMemcpyAsync(e->d_tiles_x, h_x.data(), h_x.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream));
  return ACG_OK;
}

// constant-pressure systems change L, invL and density on the device (k_npt_box);
// the host copy of the descriptors takes them back before it is uploaded again
int sync_box(acg_engine *e) {
  if (!e->any_box || !e->desc_live) return ACG_OK;
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    if (d.thermostat != 4 && d.thermostat != 5) continue;
    SysDesc dd;
    CK(cudaMemcpyAsync(&dd, e->d_desc + r, sizeof(SysDesc), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    d.L = dd.L;
    d.invL = dd.invL;
    d.density = dd.density;
  }
  return ACG_OK;
}

// force tiles: one block per cell group for systems with >= 3 cells per
// side (partials [0, ntiles_g)), block/tpp particles per block for the others
// (partials [ntiles_g, ntiles_g + ntiles_b))
int build_tiles_b(acg_engine *e) {
  int rc0 = sync_box(e);
  if (rc0) return rc0;
  const int pb = e->block / e->tpp;
  std::vector<int2> tb;
  int ng_total = 0;
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    if (d.ng > 0) {
      d.tile0_b = d.gtile0;
      d.ntile_b = d.ng * d.ng * d.ng * d.gsplit;
    }
  }
  ng_total = e->lay.ngtiles;
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    if (d.box) {
      d.tile0_b = ng_total + d.xoff;
      d.ntile_b = (d.ncell + d.cpb - 1) / d.cpb;
    }
  }
  ng_total += e->lay.nboxtiles;
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    if (d.ng > 0 || d.box) continue;
    d.tile0_b = ng_total + (int)tb.size();
    for (int s = 0; s < d.n; s += pb) tb.push_back(make_int2(r, s));
    d.ntile_b = ng_total + (int)tb.size() - d.tile0_b;
  }
  e->ntiles_b = (int)tb.size();
  const size_t cap = e->lay.nslots / 4 + e->lay.nsys + 1;
  if (tb.size() > cap) return fail(ACG_ERR_INVALID, "launch shape needs >= 4 particles per block");
  if (!tb.empty())
    CK(cudaMemcpyAsync(e->d_tiles_b, tb.data(), tb.size() * sizeof(int2), cudaMemcpyHostToDevice,
                       e->stream));
  CK(cudaMemcpyAsync(e->d_desc, e->lay.desc.data(), sizeof(SysDesc) * e->lay.nsys,
                     cudaMemcpyHostToDevice, e->stream));
  e->v.ntiles_b = e->ntiles_b;
  e->desc_live = true;
  return ACG_OK;
}

void drop_graphs(acg_engine *e) {
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->gexec1) cudaGraphExecDestroy(e->gexec1);
  if (e->graph1) cudaGraphDestroy(e->graph1);
  e->gexec = e->gexec1 = nullptr;
  e->graph = e->graph1 = nullptr;
  e->gsteps = 0;
  for (auto &b : e->bench) {
    cudaGraphExecDestroy(b.second.second);
    cudaGraphDestroy(b.second.first);
  }
  e->bench.clear();
  for (int k = 0; k < 3; k++) {
    if (e->wexec[k]) cudaGraphExecDestroy(e->wexec[k]);
    if (e->wgraph[k]) cudaGraphDestroy(e->wgraph[k]);
    e->wexec[k] = nullptr;
    e->wgraph[k] = nullptr;
  }
}

// what decides the node structure of an engine's device-loop graph: graphs of
// the same shape differ only in node parameters (pointers, grids, shared
// memory) and can be updated in place instead of instantiated anew
std::string graph_shape(const acg_engine *e, int K) {
  char b[160];
  snprintf(b, sizeof(b), "K%d g%d x%d b%d l%d%d p%d t%d/%d/%d/%d i%d%d%d", K, e->ntiles_g > 0, e->ntiles_x > 0,
           e->ntiles_b > 0, e->ntiles_l > 0, e->ntiles_lc > 0, e->lay.desc[0].precision, e->tpp, e->gtpp, e->btpp, e->block,
           e->any_gauss, e->any_npt, e->any_brown);
  return b;
}

// Destroying a graph with conditional nodes waits until the whole device is
// idle, which would stall every other engine's work each time one engine is
// destroyed (a served run ending).  Destroyed engines therefore hand their
// graphs to this list; acg_release_retired (or the list growing past
// RETIRE_MAX) destroys them when the caller chooses.
struct Retired {
  int device;
  cudaGraphExec_t exec;
  cudaGraph_t graph;
  cudaStream_t stream;
  std::string shape;  // device-loop graphs: reusable by an engine of the same shape
};
std::mutex g_retire_mu;
std::vector<Retired> g_retired;
constexpr size_t RETIRE_MAX = 256;

void release_retired_locked() {
  int cur = 0;
  cudaGetDevice(&cur);
  for (auto &r : g_retired) {
    cudaSetDevice(r.device);
    if (r.exec) cudaGraphExecDestroy(r.exec);
    if (r.graph) cudaGraphDestroy(r.graph);
    if (r.stream) cudaStreamDestroy(r.stream);
  }
  g_retired.clear();
  cudaSetDevice(cur);
}

void retire_graphs(acg_engine *e) {
  std::lock_guard<std::mutex> lk(g_retire_mu);
  g_retired.push_back({e->device, e->gexec, e->graph, nullptr, ""});
  g_retired.push_back({e->device, e->gexec1, e->graph1, nullptr, ""});
  for (auto &b : e->bench) g_retired.push_back({e->device, b.second.second, b.second.first, nullptr, ""});
  e->bench.clear();
  e->gexec = e->gexec1 = nullptr;
  e->graph = e->graph1 = nullptr;
  for (int k = 0; k < 3; k++) {
    if (e->wexec[k]) g_retired.push_back({e->device, e->wexec[k], e->wgraph[k], nullptr, graph_shape(e, k < 2 ? GRAPH_STEPS : 1)});
    e->wexec[k] = nullptr;
    e->wgraph[k] = nullptr;
  }
  if (g_retired.size() > RETIRE_MAX) release_retired_locked();
}

// ---- launches --------------------------------------------------------------
int launch_rebuild(acg_engine *e) {
  View v = e->v;
  cudaStream_t s = e->stream;
  k_cells_count<<<e->ntiles_a, BLOCK_R, 0, s>>>(v);
  k_cells_scan<<<e->lay.nsys, BLOCK_SCAN, 0, s>>>(v);
  k_cells_scatter<<<e->ntiles_a, BLOCK_R, 0, s>>>(v);
  k_cells_order<<<e->ntiles_c, 32 * CELLS_PER_TILE, 0, s>>>(v);
  k_permute<<<e->ntiles_a, BLOCK_R, 0, s>>>(v);
  if (e->lay.box_m3max) k_sort_sub<<<e->lay.nsys, BLOCK_SORT, sort_sub_smem(e->lay.box_nmax, e->lay.box_m3max), s>>>(v);
  // the list build reads the compacted rebuild list whenever it runs
  if (e->ntiles_x) k_rebuild_compact<<<1, BLOCK_COMPACT, 0, s>>>(v);
  if (e->ntiles_g) k_build_list_groups<<<e->ntiles_g, BLOCK_G, list_smem(v.gcap), s>>>(v);
  if (e->ntiles_x) k_build_list_box<<<e->ntiles_x * LIST_SPLIT, BLOCK_X, box_list_smem(e->lay.box_cell_nmax), s>>>(v);
  if (e->ntiles_lc) k_build_list_cells<<<e->ntiles_lc, BLOCK_LC, list_cells_smem(v.lccap), s>>>(v);
  if (e->ntiles_l) k_build_list<<<e->ntiles_l, BLOCK_L, 0, s>>>(v);
  CK(cudaGetLastError());
  return ACG_OK;
}

int launch_force(acg_engine *e, int mode) {
  const int prec = e->lay.desc[0].precision;
  if (e->ntiles_g) group_fn(e->gtpp, prec)<<<e->ntiles_g, BLOCK_G, group_smem(e->v.gcap), e->stream>>>(e->v, mode);
  if (e->ntiles_x)
    box_fn(e->btpp, prec)<<<e->ntiles_x, BLOCK_X, box_smem(e->lay.box_nmax, prec), e->stream>>>(e->v, mode);
  if (e->ntiles_b)
    force_fn(e->tpp, prec)<<<e->ntiles_b, e->block, 0, e->stream>>>(e->v, mode, e->ntiles_g + e->ntiles_x);
  CK(cudaGetLastError());
  return ACG_OK;
}

// the Gaussian isokinetic kernels: the second half kick and the next first
// half (with_sum, after a step's forces) or the next first half only
void launch_gauss(acg_engine *e, bool with_sum) {
  if (!e->any_gauss) return;
  if (with_sum) k_gauss_sum<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  k_gauss_apply<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
}

// ---- drift removal between graph launches ----------------------------------
// The step graphs hold no drift removal (fixDrift after every drift_every-th
// step, MDcode/main.c:261): the host keeps a copy of each system's step
// counter and ramp steps left, launches graphs up to a step after which a
// removal is due, then the removal kernels (they act on the systems whose
// kick flagged st.drift), then the rest.
// Steps from now up to and including the first one after which some system
// removes its drift (step index % drift_every == 0, not a ramp step); 0 =
// none within `limit`.
long long steps_to_drift(const Layout &lay, const std::vector<long long> &hstep,
                         const std::vector<long long> &hramp, long long limit) {
  long long best = 0;
  for (int r = 0; r < lay.nsys; r++) {
    const long long de = lay.desc[r].drift_every;
    if (de <= 0) continue;
    const long long s0 = hstep[r];
    const long long off = hramp[r] + ((s0 + de - 1) / de * de - s0);
    if (off < limit && (best == 0 || off + 1 < best)) best = off + 1;
  }
  return best;
}

void advance_steps(std::vector<long long> &hstep, std::vector<long long> &hramp, long long k) {
  for (size_t r = 0; r < hstep.size(); r++) {
    const long long ramp = std::min(hramp[r], k);
    hramp[r] -= ramp;
    hstep[r] += k - ramp;
  }
}

// k steps cut where drift removals are due: (steps, removal after them)
std::vector<std::pair<long long, bool>> drift_pieces(const acg_engine *e, std::vector<long long> &hstep,
                                                     std::vector<long long> &hramp, long long k) {
  std::vector<std::pair<long long, bool>> out;
  while (k > 0) {
    const long long m = steps_to_drift(e->lay, hstep, hramp, k);
    const long long n = m ? m : k;
    out.push_back({n, m != 0});
    advance_steps(hstep, hramp, n);
    k -= n;
  }
  return out;
}

int launch_drift(acg_engine *e) {
  k_drift_sum<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  k_drift_apply<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  launch_gauss(e, false);
  CK(cudaGetLastError());
  return ACG_OK;
}

// before the kick: the Berendsen barostat's box update and the Brownian
// random forces and predictor, then the forces of those systems (mode 3)
int launch_pre(acg_engine *e) {
  if (!e->any_npt && !e->any_brown) return ACG_OK;
  if (e->any_npt) k_npt_box<<<1, 32, 0, e->stream>>>(e->v);
  if (e->any_brown) {
    k_brown_noise<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
    k_brown_predict<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  }
  CK(cudaGetLastError());
  return launch_force(e, 3);
}

int launch_step_eager(acg_engine *e) {
  int rc0 = launch_pre(e);
  if (rc0) return rc0;
  k_kick_drift<<<e->ntiles_a + 3 * e->lay.nsys, BLOCK_A, 0, e->stream>>>(e->v, 0, 0);
  k_shuffle_ref<<<3 * e->lay.nsys, BLOCK_SHUF, shuffle_smem(e->lay), e->stream>>>(e->v, -1);
  CK(cudaGetLastError());
  int rc = launch_rebuild(e);
  if (rc) return rc;
  rc = launch_force(e, 0);
  if (rc) return rc;
  launch_gauss(e, true);
  k_drift_sum<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  k_drift_apply<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  launch_gauss(e, false);
  k_observe<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  CK(cudaGetLastError());
  return ACG_OK;
}

// forces (and lists) for every system flagged dirty
int prime(acg_engine *e) {
  if (!e->any_dirty) return ACG_OK;
  for (int r = 0; r < e->lay.nsys; r++) {
    if (!e->dirty[r]) continue;
    int one = 1;
    CK(cudaMemcpyAsync(&e->v.st[r].prime, &one, sizeof(int), cudaMemcpyHostToDevice, e->stream));
    e->dirty[r] = 0;
  }
  k_flag_rebuild<<<1, 256, 0, e->stream>>>(e->v, 0);
  CK(cudaGetLastError());
  int rc = launch_rebuild(e);
  if (rc) return rc;
  rc = launch_force(e, 1);
  if (rc) return rc;
  launch_gauss(e, false);
  CK(cudaGetLastError());
  e->any_dirty = false;
  return ACG_OK;
}

// ---- graphs ----------------------------------------------------------------
int add_kernel(cudaGraph_t g, const cudaGraphNode_t *dep, size_t ndep, cudaGraphNode_t *out,
               void *fn, int grid, int block, void **args, size_t smem = 0) {
  cudaKernelNodeParams p = {};
  p.func = fn;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(block);
  p.sharedMemBytes = (unsigned)smem;
  p.kernelParams = args;
  CK(cudaGraphAddKernelNode(out, g, dep, ndep, &p));
  return ACG_OK;
}

// K timesteps appended to graph g after node *prev (none when null); *prev
// becomes the last node.  The conditional handles belong to g.
int add_steps(acg_engine *e, cudaGraph_t g, int K, cudaGraphNode_t *prev_io) {
  View v = e->v;
  const int prec = e->lay.desc[0].precision;
  cudaGraphNode_t prev = *prev_io;
  ForceFn ff = force_fn(e->tpp, prec);
  GroupFn gf = group_fn(e->gtpp, prec);
  GroupFn xf = box_fn(e->btpp, prec);
  int mode0 = 0, use_cond = 1, tbase = e->ntiles_g + e->ntiles_x;
  for (int s = 0; s < K; s++) {
    // per step: kick/drift, then one device-decided switch (any of the list
    // rebuild, the reference-order direction shuffle and the observable
    // events, or nothing), the force kernels (drift removals are launched by
    // the host between graphs)
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 7, cudaGraphCondAssignDefault));
    cudaGraphNode_t na, nc, nb;
    int rc;
    if (e->any_npt || e->any_brown) {
      // Berendsen barostat box update; Brownian random forces and predictor;
      // then the forces of those systems (mode 3)
      void *va0[] = {&v};
      if (e->any_npt) {
        rc = add_kernel(g, prev ? &prev : nullptr, prev ? 1 : 0, &nb, (void *)k_npt_box, 1, 32, va0);
        if (rc) return rc;
        prev = nb;
      }
      if (e->any_brown) {
        rc = add_kernel(g, prev ? &prev : nullptr, prev ? 1 : 0, &nb, (void *)k_brown_noise, e->ntiles_a, BLOCK_A,
                        va0);
        if (rc) return rc;
        prev = nb;
        rc = add_kernel(g, &prev, 1, &nb, (void *)k_brown_predict, e->ntiles_a, BLOCK_A, va0);
        if (rc) return rc;
        prev = nb;
      }
      int mode3 = 3;
      if (e->ntiles_g) {
        void *ga[] = {&v, &mode3};
        rc = add_kernel(g, &prev, 1, &nb, (void *)gf, e->ntiles_g, BLOCK_G, ga, group_smem(v.gcap));
        if (rc) return rc;
        prev = nb;
      }
      if (e->ntiles_x) {
        void *xa[] = {&v, &mode3};
        rc = add_kernel(g, &prev, 1, &nb, (void *)xf, e->ntiles_x, BLOCK_X, xa, box_smem(e->lay.box_nmax, prec));
        if (rc) return rc;
        prev = nb;
      }
      if (e->ntiles_b) {
        void *ba[] = {&v, &mode3, &tbase};
        rc = add_kernel(g, &prev, 1, &nb, (void *)ff, e->ntiles_b, e->block, ba);
        if (rc) return rc;
        prev = nb;
      }
    }
    void *aa[] = {&v, &use_cond, &h};
    rc = add_kernel(g, prev ? &prev : nullptr, prev ? 1 : 0, &na, (void *)k_kick_drift,
                    e->ntiles_a + 3 * e->lay.nsys, BLOCK_A, aa);
    if (rc) return rc;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeSwitch;
    cp.conditional.size = 7;
    CK(cudaGraphAddNode(&nc, g, &na, 1, &cp));
    void *va[] = {&v};
    struct {
      void *fn;
      int grid, block;
      size_t smem;
    } rb[] = {{(void *)k_cells_count, e->ntiles_a, BLOCK_R, 0},
              {(void *)k_cells_scan, e->lay.nsys, BLOCK_SCAN, 0},
              {(void *)k_cells_scatter, e->ntiles_a, BLOCK_R, 0},
              {(void *)k_cells_order, e->ntiles_c, 32 * CELLS_PER_TILE, 0},
              {(void *)k_permute, e->ntiles_a, BLOCK_R, 0},
              {(void *)k_sort_sub, e->lay.box_m3max ? e->lay.nsys : 0, BLOCK_SORT,
               sort_sub_smem(e->lay.box_nmax, e->lay.box_m3max)},
              {(void *)k_rebuild_compact, e->ntiles_x ? 1 : 0, BLOCK_COMPACT, 0},
              {(void *)k_build_list_groups, e->ntiles_g, BLOCK_G, list_smem(v.gcap)},
              {(void *)k_build_list_box, e->ntiles_x * LIST_SPLIT, BLOCK_X, box_list_smem(e->lay.box_cell_nmax)},
              {(void *)k_build_list_cells, e->ntiles_lc, BLOCK_LC, list_cells_smem(v.lccap)},
              {(void *)k_build_list, e->ntiles_l, BLOCK_L, 0}};
    int all = -1;
    void *sa[] = {&v, &all};
    for (int c = 0; c < 7; c++) {
      const int bits = c + 1;
      cudaGraph_t body = cp.conditional.phGraph_out[c];
      cudaGraphNode_t bp = nullptr;
      if (bits & 1) {  // the rebuild chain
        for (auto &k : rb) {
          if (k.grid == 0) continue;
          cudaGraphNode_t nn;
          rc = add_kernel(body, bp ? &bp : nullptr, bp ? 1 : 0, &nn, k.fn, k.grid, k.block, va, k.smem);
          if (rc) return rc;
          bp = nn;
        }
      }
      if (bits & 2) {  // the shuffle, independent of the rebuild chain
        cudaGraphNode_t nk;
        rc = add_kernel(body, nullptr, 0, &nk, (void *)k_shuffle_ref, 3 * e->lay.nsys, BLOCK_SHUF, sa,
                        shuffle_smem(e->lay));
        if (rc) return rc;
      }
      if (bits & 4) {  // observables, after the rebuild chain (which reorders the slots)
        cudaGraphNode_t nk;
        rc = add_kernel(body, bp ? &bp : nullptr, bp ? 1 : 0, &nk, (void *)k_observe, e->ntiles_a, BLOCK_A, va);
        if (rc) return rc;
      }
    }
    const cudaGraphNode_t *dep = &nc;
    size_t ndep = 1;
    cudaGraphNode_t last = nullptr;
    if (e->ntiles_g) {
      void *ga[] = {&v, &mode0};
      rc = add_kernel(g, dep, ndep, &nb, (void *)gf, e->ntiles_g, BLOCK_G, ga, group_smem(v.gcap));
      if (rc) return rc;
      last = nb;
      dep = &last;
      ndep = 1;
    }
    if (e->ntiles_x) {
      void *xa[] = {&v, &mode0};
      rc = add_kernel(g, dep, ndep, &nb, (void *)xf, e->ntiles_x, BLOCK_X, xa, box_smem(e->lay.box_nmax, prec));
      if (rc) return rc;
      last = nb;
      dep = &last;
      ndep = 1;
    }
    if (e->ntiles_b) {
      void *ba[] = {&v, &mode0, &tbase};
      rc = add_kernel(g, dep, ndep, &nb, (void *)ff, e->ntiles_b, e->block, ba);
      if (rc) return rc;
      last = nb;
      dep = &last;
      ndep = 1;
    }
    if (e->any_gauss) {  // Gaussian isokinetic: second half kick, next first half
      rc = add_kernel(g, dep, ndep, &nb, (void *)k_gauss_sum, e->ntiles_a, BLOCK_A, va);
      if (rc) return rc;
      last = nb;
      dep = &last;
      ndep = 1;
      rc = add_kernel(g, dep, ndep, &nb, (void *)k_gauss_apply, e->ntiles_a, BLOCK_A, va);
      if (rc) return rc;
      last = nb;
    }
    prev = last;
  }
  *prev_io = prev;
  return ACG_OK;
}

int build_graph(acg_engine *e, int K, cudaGraph_t *gout, cudaGraphExec_t *xout) {
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphNode_t prev = nullptr;
  int rc = add_steps(e, g, K, &prev);
  if (rc) return rc;
  cudaGraphExec_t x;
  CK(cudaGraphInstantiate(&x, g, 0));
  *gout = g;
  *xout = x;
  return ACG_OK;
}

// A graph that runs K-step blocks in a device-side loop: a WHILE conditional
// node whose body holds K steps and a control kernel that counts the blocks
// left in *count (set before each launch) and ends the loop at zero.  One
// launch runs any number of blocks, so the host never re-launches a graph
// that is still running (which blocks the calling thread until it ends).
int build_while_graph(acg_engine *e, int K, long long *count, cudaGraph_t *gout, cudaGraphExec_t *xout) {
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hw;
  CK(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = hw;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t nw;
  if (cudaGraphAddNode(&nw, g, nullptr, 0, &wp) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return ACG_ERR_CUDA;
  }
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  cudaGraphNode_t prev = nullptr;
  int rc = add_steps(e, body, K, &prev);
  if (rc) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return rc;
  }
  cudaGraphNode_t nl;
  void *la[] = {&count, &hw};
  rc = add_kernel(body, &prev, 1, &nl, (void *)k_loop_ctl, 1, 32, la);
  if (rc) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return rc;
  }
  // an executable graph of the same shape left by a destroyed engine is
  // updated with this graph's parameters (instantiating a new one can wait
  // for all work queued on the device)
  cudaGraphExec_t x = nullptr;
  {
    const std::string shape = graph_shape(e, K);
    std::lock_guard<std::mutex> lk(g_retire_mu);
    for (size_t i = 0; i < g_retired.size(); i++) {
      Retired &r = g_retired[i];
      if (!r.exec || r.device != e->device || r.shape != shape) continue;
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(r.exec, g, &info) == cudaSuccess) {
        x = r.exec;
        if (r.graph) cudaGraphDestroy(r.graph);
        g_retired.erase(g_retired.begin() + i);
      } else {
        cudaGetLastError();
      }
      break;
    }
  }
  if (!x && cudaGraphInstantiate(&x, g, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return ACG_ERR_CUDA;
  }
  *gout = g;
  *xout = x;
  return ACG_OK;
}

int check_sys(acg_engine *e, int sys) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (sys < 0 || sys >= e->lay.nsys) return fail(ACG_ERR_INVALID, "system index out of range");
  return ACG_OK;
}

}  // namespace

// ============================================================================
extern "C" {

const char *acg_last_error(void) { return g_err.c_str(); }
const char *acg_version(void) { return "activechi4-b200 0.1 (sm_100a)"; }

int acg_params_default(acg_params *p, int n) {
  if (!p) return fail(ACG_ERR_INVALID, "null params");
  memset(p, 0, sizeof(*p));
  p->n = n;
  p->nact = -1;
  p->L = 0.0;
  p->density = 1.2;
  p->T = 0.45;
  p->f0 = 1.0;
  p->tau_p_steps = 200;     // TAU_per (MDcode/global.h:58)
  p->dt = 0.005;            // time_step (MDcode/global.h:32)
  p->skin = 0.35 * 1.00;    // skin (MDcode/global.h:28)
  p->rebuild_factor = 3.0;  // MDcode/time_evolve.c:508
  p->list_mode = 0;
  p->thermostat = 1;
  p->shuffle = 1;
  p->precision = ACG_PREC_FP64;
  p->seed = 12345;
  p->drift_every = 100000;  // fixDrift cadence of run() (MDcode/main.c:261)
  return ACG_OK;
}

int acg_footprint(const acg_params *params, int nsys, size_t *bytes) {
  Layout lay;
  // the most whole-box blocks any device would get (one cell per block)
  int rc = plan(params, nsys, lay, 1 << 20);
  if (rc) return rc;
  if (bytes) *bytes = lay.bytes;
  return ACG_OK;
}

int acg_create(const acg_params *params, int nsys, int device, acg_engine **out) {
  if (!out) return fail(ACG_ERR_INVALID, "null out");
  *out = nullptr;
  acg_engine *e = new acg_engine();
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || nsm < 1) {
    cudaGetLastError();
    nsm = 148;
  }
  int rc = plan(params, nsys, e->lay, nsm);
  if (rc) {
    delete e;
    return rc;
  }
  e->device = device;
  for (int r = 0; r < nsys; r++) {
    e->any_gauss |= e->lay.desc[r].thermostat == 3;
    e->any_npt |= e->lay.desc[r].thermostat == 4;
    e->any_box |= e->lay.desc[r].thermostat == 4 || e->lay.desc[r].thermostat == 5;
    e->any_brown |= e->lay.desc[r].thermostat == 6;
  }
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) {
    delete e;
    return fail(ACG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));
  }
  ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  // stream-ordered: allocating and freeing an engine's memory does not wait
  // for the work of other engines on the device (a served run's start and end
  // do not stall the runs in flight)
  if (ce == cudaSuccess) ce = cudaMallocAsync(&e->arena, e->lay.bytes, e->stream);
  if (ce == cudaSuccess) ce = cudaMallocAsync((void **)&e->counts, 4 * sizeof(long long), e->stream);
  if (ce != cudaSuccess) {
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return fail(ce == cudaErrorMemoryAllocation ? ACG_ERR_NOMEM : ACG_ERR_CUDA,
                std::string("device allocation: ") + cudaGetErrorString(ce));
  }
  const Layout &L = e->lay;
  const size_t S = L.nslots, Cn = L.ncells;
  char *p = (char *)e->arena;
  auto take = [&](size_t n) {
    void *q = p;
    p += align_up(n, 256);
    return q;
  };
  View &v = e->v;
  e->d_desc = (SysDesc *)take(sizeof(SysDesc) * nsys);
  v.desc = e->d_desc;
  v.st = (SysState *)take(sizeof(SysState) * nsys);
  v.pos = (double4 *)take(32 * S);
  double **dd[] = {&v.ux, &v.uy, &v.uz, &v.vx, &v.vy, &v.vz, &v.fx, &v.fy, &v.fz, &v.ox, &v.oy, &v.oz};
  for (auto q : dd) *q = (double *)take(8 * S);
  v.id = (int *)take(4 * S);
  v.act = (int *)take(4 * S);
  v.cellof = (int *)take(4 * S);
  v.nbn = (int *)take(4 * S);
  v.nbl = (int *)take(4 * S * (size_t)L.maxnb);
  v.kdir = (char4 *)take(4 * (size_t)std::max(L.nact, 1));
  v.pos_s = (double4 *)take(32 * S);
  double **ds[] = {&v.ux_s, &v.uy_s, &v.uz_s, &v.vx_s, &v.vy_s, &v.vz_s, &v.fx_s, &v.fy_s, &v.fz_s};
  for (auto q : ds) *q = (double *)take(8 * S);
  v.id_s = (int *)take(4 * S);
  v.act_s = (int *)take(4 * S);
  v.cell_tmp = (int *)take(4 * S);
  v.perm_u = (int *)take(4 * S);
  v.perm = (int *)take(4 * S);
  v.ccount_b = (int *)take(4 * Cn);
  v.cfill = (int *)take(4 * Cn);
  v.cstart = (int *)take(4 * Cn);
  v.ccount = (int *)take(4 * Cn);
  int2 *ta = (int2 *)take(8 * (S / BLOCK_A + nsys + 1));
  e->d_tiles_b = (int2 *)take(8 * (S / 4 + nsys + 1));
  int2 *tl = (int2 *)take(8 * (S / PART_L + Cn + nsys + 1));
  int2 *tc = (int2 *)take(8 * (Cn / CELLS_PER_TILE + nsys + 1));
  const size_t Gn = (size_t)L.ngroups, Gt = (size_t)L.ngtiles;
  int2 *tg = (int2 *)take(8 * (Gt + 1));
  v.gstart = (int *)take(4 * (Gn + 1));
  const size_t Xn = (size_t)L.nboxcap;
  int2 *tx = (int2 *)take(8 * (Xn + 1));
  v.part_b = (double4 *)take(32 * (Gt + Xn + S / 4 + nsys + 1));
  v.pacc = (double4 *)take(32 * S);
  v.counter_a = (unsigned int *)take(64);
  v.obs = (ObsDesc *)take(sizeof(ObsDesc) * nsys);
  v.part_o = (double *)take(8 * (S / BLOCK_A + nsys + 1) * OBS_EMAX * OBS_NV);
  v.stage_d = (double *)take(72 * S);
  v.stage_i = (int *)take(8 * S);
  v.stage_f = (double *)take(24 * S);
  v.xsub = (float4 *)take(16 * S);
  v.ssub = (int *)take(4 * ((size_t)L.nsub + 1));
  v.rbs = (int *)take(4 * (2 * (size_t)nsys + 2));
  v.mt = (unsigned int *)take(4 * 2 * (size_t)MT_WORDS * nsys);
  v.tiles_a = ta;
  v.tiles_b = e->d_tiles_b;
  v.tiles_l = tl;
  v.tiles_c = tc;
  v.tiles_g = tg;
  v.tiles_x = tx;
  v.nsys = nsys;
  v.maxnb = L.maxnb;
  {
    // whole-box lists: one warp per particle while the sub-cell systems hold
    // few particles in all (a lone small system: latency), else one lane per
    // particle over bricks (a batch: fewer instructions)
    long long nsub_particles = 0;
    for (int r = 0; r < nsys; r++)
      if (L.desc[r].box && L.desc[r].msub >= 5) nsub_particles += L.desc[r].n;
    v.box_warp = nsub_particles <= BOX_WARP_MAX;
  }

  std::vector<int2> h_a, h_l, h_c, h_g, h_lc;
  for (int r = 0; r < nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    d.tile0_a = (int)h_a.size();
    for (int s = 0; s < d.n; s += BLOCK_A) h_a.push_back(make_int2(r, s));
    d.ntile_a = (int)h_a.size() - d.tile0_a;
    for (int s = 0; s < d.ncell; s += CELLS_PER_TILE) h_c.push_back(make_int2(r, s));
    if (d.ng > 0)
      for (int g = 0; g < d.ng * d.ng * d.ng * d.gsplit; g++) h_g.push_back(make_int2(r, g));
    else if (d.box)
      continue;  // whole-box tiles: build_tiles_x
    else if (d.nc >= 3)
      for (int c = 0; c < d.ncell; c++) h_lc.push_back(make_int2(r, c));
    else
      for (int s = 0; s < d.n; s += PART_L) h_l.push_back(make_int2(r, s));
  }
  // cell groups with the most cells first (2x2x2, then the thinner groups at
  // odd box edges), so the blocks of a second wave are the short ones; every
  // block writes its partial sums at its group's index, so the order of the
  // sums does not depend on the launch order
  auto group_cells = [&](int2 t) {
    const SysDesc &d = e->lay.desc[t.x];
    int c = 1;
    for (int k = 0, q = t.y / d.gsplit; k < 3; k++, q /= d.ng) c *= std::min(2 * (q % d.ng) + 2, d.nc) - 2 * (q % d.ng);
    return c;
  };
  std::stable_sort(h_g.begin(), h_g.end(), [&](int2 a, int2 b) { return group_cells(a) > group_cells(b); });
  e->d_tiles_x = tx;
  e->ntiles_a = (int)h_a.size();
  e->ntiles_l = (int)h_l.size();
  e->ntiles_lc = (int)h_lc.size();
  v.tiles_lc = tl;
  v.tiles_l = tl + h_lc.size();
  v.ntiles_lc = e->ntiles_lc;
  e->ntiles_c = (int)h_c.size();
  e->ntiles_g = (int)h_g.size();
  v.ntiles_a = e->ntiles_a;
  v.ntiles_l = e->ntiles_l;
  v.ntiles_c = e->ntiles_c;
  v.ntiles_g = e->ntiles_g;
  // staged-particle capacity of a cell group: 1.08x the mean union (4^3 cells)
  // of the densest system plus margin; a group above it uses the cell scan
  {
    double mean_u = 0;
    for (int r = 0; r < nsys; r++)
      if (L.desc[r].ng > 0) mean_u = std::max(mean_u, 64.0 * L.desc[r].n / (double)L.desc[r].ncell);
    v.gcap = (int)align_up((size_t)(1.08 * mean_u + 128.0), 32);
    v.gcap = std::min(v.gcap, 8192);
    // staged candidates of a cell's 27 neighbours (list build by cells):
    // 1.5x the mean of the densest such system plus margin; a cell above it
    // leaves its particles to the force kernel's cell scan
    double mean_c = 0;
    for (int r = 0; r < nsys; r++) {
      const SysDesc &dr = L.desc[r];
      if (!dr.box && dr.ng == 0 && dr.nc >= 3) mean_c = std::max(mean_c, 27.0 * dr.n / (double)dr.ncell);
    }
    v.lccap = (int)std::min<size_t>(align_up((size_t)(1.5 * mean_c + 128.0), 32), 8192);
  }
  // the shared-memory limit is a property of the kernel function, shared by
  // every engine of the process: only ever raise it
  auto raise_smem = [](const void *fn, size_t need) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return false;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= need) return true;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need) == cudaSuccess;
  };
  bool attr_ok = true;
  for (int gt : {1, 2, 4})
    for (int pr : {0, 1}) attr_ok = attr_ok && raise_smem((const void *)group_fn(gt, pr), group_smem(v.gcap));
  attr_ok = attr_ok && raise_smem((const void *)k_build_list_groups, list_smem(v.gcap));
  attr_ok = attr_ok && raise_smem((const void *)k_build_list_cells, list_cells_smem(v.lccap));
  if (L.box_nmax > 0) {
    if (box_list_smem(L.box_cell_nmax) > 227 * 1024 || box_smem(L.box_nmax, 0) > 227 * 1024) {
      acg_destroy(e);
      return fail(ACG_ERR_INVALID, "whole-box system too large for shared memory");
    }
    for (int gt : {1, 2, 4})
      for (int pr : {0, 1}) attr_ok = attr_ok && raise_smem((const void *)box_fn(gt, pr), box_smem(L.box_nmax, pr));
    attr_ok = attr_ok && raise_smem((const void *)k_build_list_box, box_list_smem(L.box_cell_nmax));
    attr_ok = attr_ok && raise_smem((const void *)k_sort_sub, sort_sub_smem(L.box_nmax, L.box_m3max));
  }
  // threads per particle of the whole-box kernels: fixed (not derived from the
  // batch), so an FP64 system sums its pairs in the same order alone and batched
  e->btpp = 2;
  if (!attr_ok) {
    acg_destroy(e);
    return fail(ACG_ERR_CUDA, "cudaFuncSetAttribute (group kernels' shared memory) failed");
  }
  auto cleanup_fail = [&](int code) {
    acg_destroy(e);
    return code;
  };
  if (cudaMemsetAsync(e->arena, 0, L.bytes, e->stream) != cudaSuccess ||
      cudaMemcpyAsync(ta, h_a.data(), h_a.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(tc, h_c.data(), h_c.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream) !=
          cudaSuccess ||
      (!h_g.empty() &&
       cudaMemcpyAsync(tg, h_g.data(), h_g.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream) !=
           cudaSuccess) ||
      (!h_lc.empty() &&
       cudaMemcpyAsync(tl, h_lc.data(), h_lc.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream) !=
           cudaSuccess) ||
      (!h_l.empty() &&
       cudaMemcpyAsync(tl + h_lc.size(), h_l.data(), h_l.size() * sizeof(int2), cudaMemcpyHostToDevice,
                       e->stream) != cudaSuccess) ||
      build_tiles_x(e) != ACG_OK)
    return cleanup_fail(fail(ACG_ERR_CUDA, "initial upload failed"));
  std::vector<SysState> st(nsys);
  memset(st.data(), 0, sizeof(SysState) * nsys);
  for (auto &s : st) {
    s.s1 = s.s2 = 1.0;
  }
  if (cudaMemcpyAsync(v.st, st.data(), sizeof(SysState) * nsys, cudaMemcpyHostToDevice, e->stream) !=
      cudaSuccess)
    return cleanup_fail(fail(ACG_ERR_CUDA, "state upload failed"));
  {
    // each system's direction-shuffle stream (state buffer 0 current)
    std::vector<unsigned int> mt(2 * (size_t)MT_WORDS * nsys, 0u);
    for (int r = 0; r < nsys; r++) mt_seed(mt.data() + 2 * (size_t)MT_WORDS * r, L.desc[r].seed);
    if (cudaMemcpyAsync(v.mt, mt.data(), mt.size() * sizeof(unsigned int), cudaMemcpyHostToDevice, e->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
      return cleanup_fail(fail(ACG_ERR_CUDA, "shuffle stream upload failed"));
  }
  rc = build_tiles_b(e);
  if (rc) return cleanup_fail(rc);
  e->dirty.assign(nsys, 1);
  e->hstep.assign(nsys, 0);
  e->hramp.assign(nsys, 0);
  e->obs_bufs.assign(nsys, {});
  e->obs_offsets.assign(nsys, {});
  e->obs_events.assign(nsys, {});
  e->any_dirty = true;
  if (cudaStreamSynchronize(e->stream) != cudaSuccess)
    return cleanup_fail(fail(ACG_ERR_CUDA, "set-up synchronisation failed"));
  *out = e;
  return ACG_OK;
}

int acg_destroy(acg_engine *e) {
  if (!e) return ACG_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  for (auto &bs : e->obs_bufs)
    for (void *b : bs) cudaFreeAsync(b, e->stream);
  if (e->flush) cudaFree(e->flush);
  if (e->arena) cudaFreeAsync(e->arena, e->stream);
  if (e->counts) cudaFreeAsync(e->counts, e->stream);
  if (e->stream) {
    cudaStreamSynchronize(e->stream);
    cudaStreamDestroy(e->stream);
  }
  retire_graphs(e);  // destroyed by acg_release_retired, or reused
  delete e;
  return ACG_OK;
}

int acg_release_retired(void) {
  std::lock_guard<std::mutex> lk(g_retire_mu);
  release_retired_locked();
  return ACG_OK;
}

int acg_num_systems(acg_engine *e) { return e ? e->lay.nsys : 0; }

int acg_system_size(acg_engine *e, int sys, int *n, int *nact) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (n) *n = e->lay.desc[sys].n;
  if (nact) *nact = e->lay.desc[sys].nact;
  return ACG_OK;
}

void *acg_stream(acg_engine *e) { return e ? (void *)e->stream : nullptr; }

int acg_set_priority(acg_engine *e, int level) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  // level 0 = the default (least urgent); each level up moves one step
  // towards `greatest` (numerically lower), clamped to the device's range
  const int prio = std::max(greatest, least - std::max(level, 0));
  cudaStream_t s = nullptr;
  CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio));
  // work and stream-ordered memory of the old stream finish before the new
  // stream runs anything
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, e->stream));
  CK(cudaStreamWaitEvent(s, ev, 0));
  CK(cudaEventDestroy(ev));
  CK(cudaStreamDestroy(e->stream));
  e->stream = s;
  return ACG_OK;
}

int acg_set_state(acg_engine *e, int sys, const double *x, const double *xu, const double *p,
                  const int *type, const int *act_tag) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!x || !p || !type || !act_tag) return fail(ACG_ERR_INVALID, "x, p, type and act_tag are required");
  const SysDesc &d = e->lay.desc[sys];
  const size_t n = d.n;
  for (size_t i = 0; i < n; i++) {
    if (type[i] != 0 && type[i] != 1) return fail(ACG_ERR_INVALID, "type must be 0 or 1");
    if (act_tag[i] < -1 || act_tag[i] >= d.nact) return fail(ACG_ERR_INVALID, "act_tag out of range");
    for (int c = 0; c < 3; c++)
      if (!(x[3 * i + c] >= 0.0 && x[3 * i + c] < 1.0))
        return fail(ACG_ERR_INVALID, "x must be wrapped reduced coordinates in [0,1)");
  }
  CK(cudaSetDevice(e->device));
  double *sd = e->v.stage_d + 9 * (size_t)d.poff;
  int *si = e->v.stage_i + 2 * (size_t)d.poff;
  CK(cudaMemcpyAsync(sd, x, 24 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(sd + 3 * n, xu ? xu : x, 24 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(sd + 6 * n, p, 24 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(si, type, 4 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(si + n, act_tag, 4 * n, cudaMemcpyHostToDevice, e->stream));
  k_load<<<std::max(1, std::min((int)((n + 255) / 256), 1024)), 256, 0, e->stream>>>(e->v, sys);
  CK(cudaGetLastError());
  double one = 1.0;
  long long zero_ll = 0;
  CK(cudaMemcpyAsync(&e->v.st[sys].s1, &one, sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(&e->v.st[sys].s2, &one, sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(&e->v.st[sys].ramp_left, &zero_ll, sizeof(long long), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));  // host buffers may be freed on return
  e->hramp[sys] = 0;
  e->dirty[sys] = 1;
  e->any_dirty = true;
  return ACG_OK;
}

int acg_get_state(acg_engine *e, int sys, double *x, double *xu, double *p, double *F) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  const SysDesc &d = e->lay.desc[sys];
  const size_t n = d.n;
  k_unload<<<std::max(1, std::min((int)((n + 255) / 256), 1024)), 256, 0, e->stream>>>(e->v, sys);
  CK(cudaGetLastError());
  double *sd = e->v.stage_d + 9 * (size_t)d.poff;
  double *sf = e->v.stage_f + 3 * (size_t)d.poff;
  if (x) CK(cudaMemcpyAsync(x, sd, 24 * n, cudaMemcpyDeviceToHost, e->stream));
  if (xu) CK(cudaMemcpyAsync(xu, sd + 3 * n, 24 * n, cudaMemcpyDeviceToHost, e->stream));
  if (p) CK(cudaMemcpyAsync(p, sd + 6 * n, 24 * n, cudaMemcpyDeviceToHost, e->stream));
  if (F) CK(cudaMemcpyAsync(F, sf, 24 * n, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_directions(acg_engine *e, int sys, const int *k) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  const SysDesc &d = e->lay.desc[sys];
  if (d.nact == 0) return ACG_OK;
  if (!k) return fail(ACG_ERR_INVALID, "null directions");
  std::vector<char4> h(d.nact);
  for (int a = 0; a < d.nact; a++) {
    int kx = k[a], ky = k[d.nact + a], kz = k[2 * d.nact + a];
    if (std::abs(kx) > 1 || std::abs(ky) > 1 || std::abs(kz) > 1)
      return fail(ACG_ERR_INVALID, "direction components must be -1, 0 or +1");
    h[a] = make_char4((signed char)kx, (signed char)ky, (signed char)kz, 0);
  }
  CK(cudaSetDevice(e->device));
  CK(cudaMemcpyAsync(e->v.kdir + d.aoff, h.data(), 4 * (size_t)d.nact, cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_get_directions(acg_engine *e, int sys, int *k) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  const SysDesc &d = e->lay.desc[sys];
  if (d.nact == 0) return ACG_OK;
  std::vector<char4> h(d.nact);
  CK(cudaSetDevice(e->device));
  CK(cudaMemcpyAsync(h.data(), e->v.kdir + d.aoff, 4 * (size_t)d.nact, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  for (int a = 0; a < d.nact; a++) {
    k[a] = h[a].x;
    k[d.nact + a] = h[a].y;
    k[2 * d.nact + a] = h[a].z;
  }
  return ACG_OK;
}

int acg_shuffle_directions(acg_engine *e, int sys) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (e->lay.desc[sys].nact == 0) return ACG_OK;
  CK(cudaSetDevice(e->device));
  if (e->lay.desc[sys].shuffle == 2) {
    k_shuffle_now<<<3, 256, 0, e->stream>>>(e->v, sys);
  } else {
    k_shuffle_ref<<<3, BLOCK_SHUF, shuffle_smem(e->lay), e->stream>>>(e->v, sys);
    k_mt_flip<<<1, 32, 0, e->stream>>>(e->v, sys);
  }
  CK(cudaGetLastError());
  return ACG_OK;
}

int acg_seed_shuffle(acg_engine *e, int sys, uint64_t seed) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  CK(cudaSetDevice(e->device));
  SysState st;
  CK(cudaMemcpyAsync(&st, e->v.st + sys, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  std::vector<unsigned int> mt(MT_WORDS);
  mt_seed(mt.data(), seed);
  CK(cudaMemcpyAsync(e->v.mt + ((size_t)2 * sys + st.mt_cur) * MT_WORDS, mt.data(), MT_WORDS * sizeof(unsigned int),
                     cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_fix_drift(acg_engine *e, int sys) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  k_flag_drift<<<1, 32, 0, e->stream>>>(e->v, sys);
  k_drift_sum<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  k_drift_apply<<<e->ntiles_a, BLOCK_A, 0, e->stream>>>(e->v);
  launch_gauss(e, false);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_adjust_temperature(acg_engine *e, int sys, double T, double *inst_T) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!(T > 0) || !std::isfinite(T)) return fail(ACG_ERR_INVALID, "T must be positive");
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  k_rescale<<<1, 1024, 0, e->stream>>>(e->v, sys, T);
  launch_gauss(e, false);
  CK(cudaGetLastError());
  double ke = 0;
  CK(cudaMemcpyAsync(&ke, &e->v.st[sys].ke_end, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  if (inst_T) *inst_T = 2.0 * ke / e->lay.desc[sys].dof;
  return ACG_OK;
}

int acg_start_ramp(acg_engine *e, int sys, double T_start, double T_end, double rate, int64_t *steps) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!(T_start > 0) || !(T_end > 0) || !(rate > 0) || !std::isfinite(T_start) || !std::isfinite(T_end))
    return fail(ACG_ERR_INVALID, "ramp temperatures and rate must be positive");
  const SysDesc &d = e->lay.desc[sys];
  if (d.thermostat == 3 || d.thermostat >= 5)
    return fail(ACG_ERR_INVALID,
                "temperature ramps are refused for Gaussian isokinetic, Nose-Hoover NPT and Brownian systems");
  double T0 = 0;
  rc = acg_adjust_temperature(e, sys, T_start, &T0);
  if (rc) return rc;
  // the reference's loop: while (T < final) { rescale to T; step; T += dt*rate }
  // (heating, MDcode/initialise.c:179-186) or while (T > final) ... T -= dt*rate
  // (cooling, :191-197), T starting at the temperature reached by the rescale
  const double dT = d.dt * rate;
  const bool heat = T_end > T_start;
  long long K = 0;
  for (double T = T0; heat ? T < T_end : T > T_end; T = heat ? T + dT : T - dT) {
    if (++K > 100000000LL) return fail(ACG_ERR_INVALID, "ramp longer than 1e8 steps");
  }
  CK(cudaSetDevice(e->device));
  // the ramps rebuild the lists at their start (update_cell_list,
  // MDcode/initialise.c:174,192); the positions, hence the forces, stay
  k_flag_rebuild_one<<<1, 256, 0, e->stream>>>(e->v, sys);
  CK(cudaGetLastError());
  rc = launch_rebuild(e);
  if (rc) return rc;
  k_ramp_begin<<<1, 32, 0, e->stream>>>(e->v, sys, T0, heat ? dT : -dT, T_end, K);
  e->hramp[sys] = K;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  if (steps) *steps = K;
  return ACG_OK;
}

int acg_extend_ramp(acg_engine *e, int sys, int64_t total_steps) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  CK(cudaSetDevice(e->device));
  k_ramp_extend<<<1, 32, 0, e->stream>>>(e->v, sys, (long long)total_steps);
  if (e->hramp[sys] > 0 && (long long)total_steps > e->hramp[sys]) e->hramp[sys] = total_steps;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_lattice(acg_engine *e, int sys, const int *site, const int *type, const double *p, const int *act_tag) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!site || !type || !p || !act_tag) return fail(ACG_ERR_INVALID, "site, type, p and act_tag are required");
  const SysDesc &d = e->lay.desc[sys];
  const size_t n = d.n;
  int troot = 1;
  while ((long long)troot * troot * troot < (long long)n) troot++;  // MDcode/initialise.c:35-37
  const long long nsite = (long long)troot * troot * troot;
  std::vector<char> used((size_t)nsite, 0);
  for (size_t i = 0; i < n; i++) {
    if (site[i] < 0 || site[i] >= nsite || used[site[i]])
      return fail(ACG_ERR_INVALID, "site must hold distinct grid sites in [0, troot^3)");
    used[site[i]] = 1;
    if (type[i] != 0 && type[i] != 1) return fail(ACG_ERR_INVALID, "type must be 0 or 1");
    if (act_tag[i] < -1 || act_tag[i] >= d.nact) return fail(ACG_ERR_INVALID, "act_tag out of range");
  }
  CK(cudaSetDevice(e->device));
  double *sd = e->v.stage_d + 9 * (size_t)d.poff;
  int *si = e->v.stage_i + 2 * (size_t)d.poff;
  CK(cudaMemcpyAsync(sd + 6 * n, p, 24 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(si, type, 4 * n, cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(si + n, site, 4 * n, cudaMemcpyHostToDevice, e->stream));
  const int grid = std::max(1, std::min((int)((n + 255) / 256), 1024));
  k_lattice<<<grid, 256, 0, e->stream>>>(e->v, sys, troot);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(si + n, act_tag, 4 * n, cudaMemcpyHostToDevice, e->stream));
  k_load<<<grid, 256, 0, e->stream>>>(e->v, sys);
  CK(cudaGetLastError());
  double one = 1.0;
  long long zero_ll = 0;
  CK(cudaMemcpyAsync(&e->v.st[sys].s1, &one, sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(&e->v.st[sys].s2, &one, sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(&e->v.st[sys].ramp_left, &zero_ll, sizeof(long long), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->hramp[sys] = 0;
  e->dirty[sys] = 1;
  e->any_dirty = true;
  return ACG_OK;
}

int acg_set_nhc(acg_engine *e, int sys, const double *eta3, const double *p_eta3) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!eta3 || !p_eta3) return fail(ACG_ERR_INVALID, "null chain");
  CK(cudaSetDevice(e->device));
  SysState *s = e->v.st + sys;
  CK(cudaMemcpyAsync(s->eta_end, eta3, 3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(s->p_eta_end, p_eta3, 3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  if (e->dirty[sys]) {
    // the prime pass computes the first half once forces and KE are known
    CK(cudaStreamSynchronize(e->stream));
    return ACG_OK;
  }
  k_prehalf<<<1, 1, 0, e->stream>>>(e->v, sys);
  launch_gauss(e, false);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_barostat(acg_engine *e, int sys, const double *eta_baro3, const double *p_eta_baro3, double p_eps) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!eta_baro3 || !p_eta_baro3 || !std::isfinite(p_eps)) return fail(ACG_ERR_INVALID, "bad barostat state");
  if (e->lay.desc[sys].thermostat != 5) return fail(ACG_ERR_INVALID, "the system is not Nose-Hoover NPT (thermostat 5)");
  CK(cudaSetDevice(e->device));
  SysState *s = e->v.st + sys;
  CK(cudaMemcpyAsync(s->eta_baro_end, eta_baro3, 3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(s->p_eta_baro_end, p_eta_baro3, 3 * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(&s->p_eps_end, &p_eps, sizeof(double), cudaMemcpyHostToDevice, e->stream));
  if (!e->dirty[sys]) {
    k_prehalf<<<1, 1, 0, e->stream>>>(e->v, sys);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_temperature(acg_engine *e, int sys, double T) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!(T > 0)) return fail(ACG_ERR_INVALID, "T must be positive");
  CK(cudaSetDevice(e->device));
  rc = sync_box(e);
  if (rc) return rc;
  SysDesc &d = e->lay.desc[sys];
  d.T = T;
  for (int i = 0; i < NHC_M; i++) d.q[i] = T * TAU_T * TAU_T;
  d.q[0] = d.dof * T * TAU_T * TAU_T;
  for (int i = 0; i < NHC_M; i++) d.q_baro[i] = T * TAU_P * TAU_P;
  d.w_eps = d.dof * T * TAU_P * TAU_P;
  CK(cudaMemcpyAsync(e->d_desc + sys, &d, sizeof(SysDesc), cudaMemcpyHostToDevice, e->stream));
  if (!e->dirty[sys]) {
    k_prehalf<<<1, 1, 0, e->stream>>>(e->v, sys);
    launch_gauss(e, false);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_rebuild(acg_engine *e) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  k_flag_rebuild<<<1, 256, 0, e->stream>>>(e->v, 1);
  CK(cudaGetLastError());
  rc = launch_rebuild(e);
  if (rc) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_compute_forces(acg_engine *e) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  k_flag_rebuild<<<1, 256, 0, e->stream>>>(e->v, 1);
  CK(cudaGetLastError());
  rc = launch_rebuild(e);
  if (rc) return rc;
  rc = launch_force(e, 2);
  if (rc) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

// nsteps steps in graph launches (no drift removal due inside them)
int step_graphs(acg_engine *e, int nsteps) {
  int rc;
  if (!e->no_while) {
    // device loop: one launch for the GRAPH_STEPS-step blocks, one for the rest
    const long long q = nsteps / GRAPH_STEPS, r = nsteps % GRAPH_STEPS;
    const int need[3] = {q > 0 && e->wturn == 0, q > 0 && e->wturn == 1, r > 0};
    for (int k = 0; k < 3 && !e->no_while; k++)
      if (need[k] && !e->wexec[k] &&
          build_while_graph(e, k < 2 ? GRAPH_STEPS : 1, e->counts + k, &e->wgraph[k], &e->wexec[k]) != ACG_OK)
        e->no_while = true;
    if (!e->no_while) {
      if (q > 0) {
        k_set_count<<<1, 32, 0, e->stream>>>(e->counts + e->wturn, q);
        CK(cudaGetLastError());
        CK(cudaGraphLaunch(e->wexec[e->wturn], e->stream));
        e->wturn ^= 1;
      }
      if (r > 0) {
        k_set_count<<<1, 32, 0, e->stream>>>(e->counts + 2, r);
        CK(cudaGetLastError());
        CK(cudaGraphLaunch(e->wexec[2], e->stream));
      }
      return ACG_OK;
    }
  }
  if (nsteps >= GRAPH_STEPS && !e->gexec) {
    rc = build_graph(e, GRAPH_STEPS, &e->graph, &e->gexec);
    if (rc) return rc;
    e->gsteps = GRAPH_STEPS;
  }
  if (nsteps % GRAPH_STEPS && !e->gexec1) {
    rc = build_graph(e, 1, &e->graph1, &e->gexec1);
    if (rc) return rc;
  }
  int left = nsteps;
  while (left >= GRAPH_STEPS) {
    CK(cudaGraphLaunch(e->gexec, e->stream));
    left -= GRAPH_STEPS;
  }
  while (left-- > 0) CK(cudaGraphLaunch(e->gexec1, e->stream));
  return ACG_OK;
}

int acg_step(acg_engine *e, int nsteps) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (nsteps < 0) return fail(ACG_ERR_INVALID, "nsteps < 0");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  for (const auto &pc : drift_pieces(e, e->hstep, e->hramp, nsteps)) {
    rc = step_graphs(e, (int)pc.first);
    if (rc) return rc;
    if (pc.second) {
      rc = launch_drift(e);
      if (rc) return rc;
    }
  }
  return ACG_OK;
}

int acg_prepare(acg_engine *e) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  if (e->no_while) return ACG_OK;
  for (int k = 0; k < 3 && !e->no_while; k++)
    if (!e->wexec[k] &&
        build_while_graph(e, k < 2 ? GRAPH_STEPS : 1, e->counts + k, &e->wgraph[k], &e->wexec[k]) != ACG_OK)
      e->no_while = true;
  return ACG_OK;
}

int acg_step_eager(acg_engine *e, int nsteps) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  for (int s = 0; s < nsteps; s++) {
    rc = launch_step_eager(e);  // its drift kernels act on the kick's st.drift flags
    if (rc) return rc;
  }
  advance_steps(e->hstep, e->hramp, nsteps);
  return ACG_OK;
}

int acg_sync(acg_engine *e) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  CK(cudaSetDevice(e->device));
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_poll(acg_engine *e, int *done) {
  if (!e || !done) return fail(ACG_ERR_INVALID, "bad arguments");
  CK(cudaSetDevice(e->device));
  cudaError_t q = cudaStreamQuery(e->stream);
  if (q == cudaSuccess) {
    *done = 1;
    return ACG_OK;
  }
  if (q == cudaErrorNotReady) {
    *done = 0;
    return ACG_OK;
  }
  return fail(ACG_ERR_CUDA, std::string("cudaStreamQuery: ") + cudaGetErrorString(q));
}

int acg_get_thermo(acg_engine *e, int sys, acg_thermo *out) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!out) return fail(ACG_ERR_INVALID, "null out");
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  SysState s;
  CK(cudaMemcpyAsync(&s, e->v.st + sys, sizeof(s), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  const SysDesc &d = e->lay.desc[sys];
  memset(out, 0, sizeof(*out));
  out->pe = s.pe;
  out->ke = s.ke_end;
  out->virial = s.virial;
  out->vir_act = s.vir_act;
  out->inst_T = 2.0 * s.ke_end / d.dof;
  out->maxD = s.maxD_last;
  for (int i = 0; i < NHC_M; i++) {
    out->eta[i] = s.eta_end[i];
    out->p_eta[i] = s.p_eta_end[i];
    out->q[i] = d.q[i];
  }
  // Heff (MDcode/print.c:85-87)
  double h = s.ke_end + s.pe + s.eta_end[0] * d.T * d.dof;
  for (int i = 0; i < NHC_M; i++) h += s.p_eta_end[i] * s.p_eta_end[i] / (2.0 * d.q[i]);
  for (int i = 1; i < NHC_M; i++) h += d.T * s.eta_end[i];
  out->heff = h;
  out->step = s.step;
  out->rebuilds = s.rebuilds;
  out->overflow = s.overflow;
  out->L = d.L;
  out->eps = s.eps_end;
  out->p_eps = s.p_eps_end;
  for (int i = 0; i < NHC_M; i++) {
    out->eta_baro[i] = s.eta_baro_end[i];
    out->p_eta_baro[i] = s.p_eta_baro_end[i];
  }
  if (d.thermostat == 5) out->L = d.L0 * std::exp(s.eps_end);
  if (d.thermostat == 4) {
    double Ld = 0;
    CK(cudaMemcpyAsync(&Ld, &e->d_desc[sys].L, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    out->L = Ld;
    out->pressure = s.pressure;
  }
  if (s.status == 2) {
    out->status = ACG_ERR_BOX;
    return fail(ACG_ERR_BOX, "system " + std::to_string(sys) + ": the box left its cell grid (L = " +
                                 std::to_string(out->L) + ")");
  }
  out->status = s.status ? ACG_ERR_NONFINITE : 0;
  if (s.status) return fail(ACG_ERR_NONFINITE, "system " + std::to_string(sys) + ": non-finite kinetic energy");
  return ACG_OK;
}

int acg_get_cells(acg_engine *e, int sys, int *dims, int *ncell, int *counts, int *members) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  const SysDesc &d = e->lay.desc[sys];
  if (dims) dims[0] = dims[1] = dims[2] = d.nc;
  if (ncell) *ncell = d.ncell;
  if (counts)
    CK(cudaMemcpyAsync(counts, e->v.ccount + d.coff, 4 * (size_t)d.ncell, cudaMemcpyDeviceToHost, e->stream));
  if (members) {
    // slots are in cell order after the rebuild: the member list is the id
    // array of the system's slots
    CK(cudaMemcpyAsync(members, e->v.id + d.poff, 4 * (size_t)d.n, cudaMemcpyDeviceToHost, e->stream));
  }
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_launch(acg_engine *e, int tpp, int block) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (!force_fn(tpp, 0)) return fail(ACG_ERR_INVALID, "tpp must be 1, 2, 4, 8, 16 or 32");
  if (block < 32 || block > 512 || block % 32 || block / tpp < 4)
    return fail(ACG_ERR_INVALID, "block must be a multiple of 32 in [32,512] with >= 4 particles");
  CK(cudaSetDevice(e->device));
  CK(cudaStreamSynchronize(e->stream));
  e->tpp = tpp;
  e->block = block;
  drop_graphs(e);
  int rc = build_tiles_b(e);
  if (rc) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_set_group_tpp(acg_engine *e, int gtpp) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (!group_fn(gtpp, 0)) return fail(ACG_ERR_INVALID, "group threads per particle must be 1, 2 or 4");
  CK(cudaSetDevice(e->device));
  CK(cudaStreamSynchronize(e->stream));
  e->gtpp = gtpp;
  e->btpp = gtpp;
  drop_graphs(e);
  return ACG_OK;
}

int acg_set_box_cells(acg_engine *e, int cells) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (cells < 1 || cells > BOX_CELLS) return fail(ACG_ERR_INVALID, "cells per whole-box block must be in [1, 8]");
  CK(cudaSetDevice(e->device));
  CK(cudaStreamSynchronize(e->stream));
  for (int r = 0; r < e->lay.nsys; r++) {
    SysDesc &d = e->lay.desc[r];
    if (d.box && d.nc > 2) d.cpb = cells;
  }
  int rc = build_tiles_x(e);
  if (rc) return rc;
  drop_graphs(e);
  rc = build_tiles_b(e);  // partial-sum slots and the descriptors
  if (rc) return rc;
  CK(cudaStreamSynchronize(e->stream));
  return ACG_OK;
}

int acg_get_box_cells(acg_engine *e, int *cells) {
  if (!e || !cells) return fail(ACG_ERR_INVALID, "bad arguments");
  *cells = 0;
  for (int r = 0; r < e->lay.nsys; r++)
    if (e->lay.desc[r].box && e->lay.desc[r].nc > 2) *cells = e->lay.desc[r].cpb;
  return ACG_OK;
}

int acg_get_launch(acg_engine *e, int *tpp, int *block) {
  if (!e) return fail(ACG_ERR_INVALID, "null engine");
  if (tpp) *tpp = e->tpp;
  if (block) *block = e->block;
  return ACG_OK;
}

int acg_time_stage(acg_engine *e, int stage, int reps, double *ms) {
  if (!e || reps < 1 || !ms) return fail(ACG_ERR_INVALID, "bad arguments");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  // stage 1 evaluates forces only (mode 2) and stage 2 rebuilds at the
  // current positions, so neither changes the trajectory; stage 0 drifts the
  // particles and is meant for a scratch engine.
  CK(cudaEventRecord(a, e->stream));
  for (int i = 0; i < reps; i++) {
    if (stage == 0) {
      k_kick_drift<<<e->ntiles_a + 3 * e->lay.nsys, BLOCK_A, 0, e->stream>>>(e->v, 0, 0);
    } else if (stage == 1) {
      rc = launch_force(e, 2);
    } else {
      k_flag_rebuild<<<1, 256, 0, e->stream>>>(e->v, 1);
      rc = launch_rebuild(e);
    }
    if (rc) return rc;
  }
  CK(cudaEventRecord(b, e->stream));
  CK(cudaEventSynchronize(b));
  float t = 0;
  CK(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = (double)t / reps;
  return ACG_OK;
}

// The log-time schedule of prepareSavingArray (MDcode/main.c:62-119) turned
// into device events: origins every run/num_origins steps; from each origin
// the offsets 1, then *factor truncated (+1 when that does not advance), below
// max_interval (the analysis pairs offsets below half the run,
// Analysis/overlap.c:28) and inside the run.  An origin snapshot occupies one of
// max_live slots from its step to its last offset; an origin for which no slot
// is free is left out.
int acg_obs_configure(acg_engine *e, int sys, const acg_obs_config *c) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  if (!c || c->run_length < 2 || c->num_origins < 1 || !(c->factor > 1.0) || !(c->a > 0) || c->nq < 0 ||
      c->nq > 256 || (c->nq > 0 && !c->qvec) || c->max_live_origins < 1 || c->max_live_origins > 4095)
    return fail(ACG_ERR_INVALID, "bad observable configuration");
  CK(cudaSetDevice(e->device));
  rc = prime(e);
  if (rc) return rc;
  SysState st;
  CK(cudaMemcpyAsync(&st, e->v.st + sys, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  const long long base = st.step, run = c->run_length;
  const long long lin = run / c->num_origins;
  const long long maxint = c->max_interval > 0 ? c->max_interval : run / 2;
  std::vector<long long> offs;
  for (unsigned long long off = 1; (long long)off < maxint && (long long)off < run;) {
    offs.push_back((long long)off);
    if ((unsigned long long)(off * c->factor) == off)
      off++;
    else
      off = (unsigned long long)((double)off * c->factor);
  }
  if (offs.empty() || offs.size() > 200000) return fail(ACG_ERR_INVALID, "schedule has no usable offsets");
  struct Ev {
    long long step;
    int kind, slot, bin;
  };
  std::vector<Ev> ev;
  std::vector<long long> busy(c->max_live_origins, -1);
  for (long long k = 0; k < c->num_origins && lin > 0; k++) {
    const long long t0 = k * lin;
    long long last = t0;
    for (long long o : offs)
      if (t0 + o < run) last = t0 + o;
    int slot = -1;
    for (int q = 0; q < c->max_live_origins; q++)
      if (busy[q] < t0) {
        slot = q;
        break;
      }
    if (slot < 0) continue;
    busy[slot] = last;
    ev.push_back({base + t0, 1, slot, 0});
    for (size_t m = 0; m < offs.size(); m++)
      if (t0 + offs[m] < run) ev.push_back({base + t0 + offs[m], 0, slot, (int)m});
  }
  std::sort(ev.begin(), ev.end(), [](const Ev &a, const Ev &b) {
    return a.step != b.step ? a.step < b.step : a.kind < b.kind;  // measure before snapshot
  });
  for (size_t i = 0, j; i < ev.size(); i = j) {
    for (j = i; j < ev.size() && ev[j].step == ev[i].step; j++) {
    }
    if (j - i > (size_t)OBS_EMAX) return fail(ACG_ERR_INVALID, "more than 16 observable events in one step");
  }
  const SysDesc &d = e->lay.desc[sys];
  std::vector<long long> h_step(ev.size());
  std::vector<int> h_info(ev.size());
  for (size_t i = 0; i < ev.size(); i++) {
    h_step[i] = ev[i].step;
    h_info[i] = ev[i].kind | (ev[i].slot << 1) | (ev[i].bin << 13);
  }
  for (void *b : e->obs_bufs[sys]) cudaFreeAsync(b, e->stream);
  e->obs_bufs[sys].clear();
  auto dalloc = [&](size_t bytes, void **p) {
    cudaError_t ce = cudaMallocAsync(p, bytes > 0 ? bytes : 8, e->stream);
    if (ce == cudaSuccess) e->obs_bufs[sys].push_back(*p);
    return ce;
  };
  void *p_step = nullptr, *p_info = nullptr, *p_snap = nullptr, *p_acc = nullptr, *p_q = nullptr;
  if (dalloc(8 * ev.size(), &p_step) != cudaSuccess || dalloc(4 * ev.size(), &p_info) != cudaSuccess ||
      dalloc((size_t)c->max_live_origins * d.n * 3 * sizeof(double), &p_snap) != cudaSuccess ||
      dalloc(offs.size() * 8 * sizeof(double), &p_acc) != cudaSuccess || dalloc(12 * (size_t)c->nq, &p_q) != cudaSuccess)
    return fail(ACG_ERR_NOMEM, "observable buffers: device allocation failed");
  CK(cudaMemcpyAsync(p_step, h_step.data(), 8 * ev.size(), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemcpyAsync(p_info, h_info.data(), 4 * ev.size(), cudaMemcpyHostToDevice, e->stream));
  CK(cudaMemsetAsync(p_acc, 0, offs.size() * 8 * sizeof(double), e->stream));
  if (c->nq) CK(cudaMemcpyAsync(p_q, c->qvec, 12 * (size_t)c->nq, cudaMemcpyHostToDevice, e->stream));
  ObsDesc od = {};
  od.ev_step = (const long long *)p_step;
  od.ev_info = (const int *)p_info;
  od.snap = (double *)p_snap;
  od.acc = (double *)p_acc;
  od.qvec = (const int *)p_q;
  od.n_events = (int)ev.size();
  od.nbins = (int)offs.size();
  od.nq = c->nq;
  od.nslots = c->max_live_origins;
  od.a2 = c->a * c->a;
  CK(cudaMemcpyAsync(e->v.obs + sys, &od, sizeof(od), cudaMemcpyHostToDevice, e->stream));
  int zero = 0;
  CK(cudaMemcpyAsync(&e->v.st[sys].obs_cur, &zero, sizeof(int), cudaMemcpyHostToDevice, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  e->obs_offsets[sys] = offs;
  e->obs_events[sys].assign(h_step.begin(), h_step.end());
  e->obs_events[sys].erase(std::unique(e->obs_events[sys].begin(), e->obs_events[sys].end()), e->obs_events[sys].end());
  return ACG_OK;
}

int acg_obs_sums(acg_engine *e, int sys, int *nbins, int64_t *offset, double *sums) {
  int rc = check_sys(e, sys);
  if (rc) return rc;
  const auto &offs = e->obs_offsets[sys];
  if (nbins) *nbins = (int)offs.size();
  if (offs.empty()) return ACG_OK;
  if (offset)
    for (size_t m = 0; m < offs.size(); m++) offset[m] = offs[m];
  if (sums) {
    CK(cudaSetDevice(e->device));
    ObsDesc od;
    CK(cudaMemcpyAsync(&od, e->v.obs + sys, sizeof(od), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    std::vector<double> a(offs.size() * 8);
    CK(cudaMemcpyAsync(a.data(), od.acc, a.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    for (size_t m = 0; m < offs.size(); m++)
      for (int k = 0; k < 7; k++) sums[7 * m + k] = a[8 * m + k];
  }
  return ACG_OK;
}

int acg_bench_steps(acg_engine *e, int64_t nsteps, size_t flush_bytes, double *ms, int64_t *launches) {
  if (!e || nsteps < 1 || !ms) return fail(ACG_ERR_INVALID, "bad arguments");
  CK(cudaSetDevice(e->device));
  int rc = prime(e);
  if (rc) return rc;
  // exactly nsteps steps: one graph of nsteps steps when that is short, else
  // graphs of GRAPH_STEPS steps and one of the remainder
  std::vector<int> plan;
  if (nsteps <= BENCH_MAX_GRAPH) {
    plan.push_back((int)nsteps);
  } else {
    for (int64_t k = 0; k < nsteps / GRAPH_STEPS; k++) plan.push_back(GRAPH_STEPS);
    if (nsteps % GRAPH_STEPS) plan.push_back((int)(nsteps % GRAPH_STEPS));
  }
  // each timed region in pieces cut where drift removals are due (launched
  // between the pieces, inside the region)
  std::vector<std::vector<std::pair<long long, bool>>> pieces;
  {
    std::vector<long long> hs = e->hstep, hr = e->hramp;
    for (int K : plan) pieces.push_back(drift_pieces(e, hs, hr, K));
  }
  for (const auto &reg : pieces)
    for (const auto &pc : reg) {
      const int K = (int)pc.first;
      if (e->bench.count(K)) continue;
      cudaGraph_t g;
      cudaGraphExec_t x;
      rc = build_graph(e, K, &g, &x);
      if (rc) return rc;
      e->bench[K] = {g, x};
    }
  if (flush_bytes > e->flush_bytes) {
    if (e->flush) cudaFree(e->flush);
    e->flush = nullptr;
    e->flush_bytes = 0;
    CK(cudaMalloc(&e->flush, flush_bytes));
    e->flush_bytes = flush_bytes;
  }
  const int nsys = e->lay.nsys;
  std::vector<SysState> st0(nsys), st1(nsys);
  CK(cudaMemcpyAsync(st0.data(), e->v.st, sizeof(SysState) * nsys, cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  for (int r = 0; r < nsys; r++)
    if (st0[r].step != e->hstep[r] || st0[r].ramp_left != e->hramp[r])
      return fail(ACG_ERR_STATE, "system " + std::to_string(r) + ": the host's step counter disagrees with the device's");
  const size_t nl = plan.size();
  std::vector<cudaEvent_t> ev(2 * nl);
  for (auto &x : ev) CK(cudaEventCreate(&x));
  long long ndrift = 0;
  for (size_t c = 0; c < nl; c++) {
    if (flush_bytes) CK(cudaMemsetAsync(e->flush, (int)(c & 0xff), flush_bytes, e->stream));
    CK(cudaEventRecord(ev[2 * c], e->stream));
    for (const auto &pc : pieces[c]) {
      CK(cudaGraphLaunch(e->bench[(int)pc.first].second, e->stream));
      if (pc.second) {
        rc = launch_drift(e);
        if (rc) return rc;
        ndrift++;
      }
    }
    CK(cudaEventRecord(ev[2 * c + 1], e->stream));
  }
  advance_steps(e->hstep, e->hramp, nsteps);
  CK(cudaStreamSynchronize(e->stream));
  double tot = 0;
  for (size_t c = 0; c < nl; c++) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, ev[2 * c], ev[2 * c + 1]));
    tot += t;
  }
  for (auto &x : ev) cudaEventDestroy(x);
  CK(cudaMemcpy(st1.data(), e->v.st, sizeof(SysState) * nsys, cudaMemcpyDeviceToHost));
  *ms = tot;
  if (!launches) return ACG_OK;
  // kernels launched in the timed region: every step the kick/drift kernel
  // and each force kernel in use; a step whose switch takes the rebuild the
  // rebuild kernels with a non-empty grid, the shuffle the shuffle kernel,
  // observable events the observable kernel (the node lists of add_steps);
  // each drift removal its two kernels (and a Gaussian one).  A Gaussian
  // isokinetic system adds two kernels per step; the Berendsen barostat the
  // box update, Brownian dynamics the random forces and the predictor, and
  // either a second force pass every step.
  const long long nforce = (e->ntiles_g > 0) + (e->ntiles_x > 0) + (e->ntiles_b > 0);
  const long long per_step = 1 + nforce + 2 * e->any_gauss + e->any_npt + 2 * e->any_brown +
                             (e->any_npt || e->any_brown) * nforce;
  const long long per_rebuild = 5 + (e->lay.box_m3max > 0) + 2 * (e->ntiles_x > 0) + (e->ntiles_g > 0) +
                                (e->ntiles_l > 0) + (e->ntiles_lc > 0);
  long long steps_with_rebuild = 0, shuffles = 0, obs_steps = 0;
  for (int r = 0; r < nsys; r++) steps_with_rebuild = std::max(steps_with_rebuild, st1[r].rebuilds - st0[r].rebuilds);
  for (long long k = 0; k < nsteps; k++) {
    bool shuf = false, obs = false;
    for (int r = 0; r < nsys && !(shuf && obs); r++) {
      const SysDesc &d = e->lay.desc[r];
      const long long step = st0[r].step + k;
      if (d.shuffle == 1 && d.nact > 0 && d.tau_p > 0 && step % d.tau_p == 0) shuf = true;
      const auto &evs = e->obs_events[r];
      if (!obs && std::binary_search(evs.begin(), evs.end(), step)) obs = true;
    }
    shuffles += shuf;
    obs_steps += obs;
  }
  *launches = per_step * nsteps + per_rebuild * steps_with_rebuild + shuffles + obs_steps + (2 + e->any_gauss) * ndrift;
  return ACG_OK;
}

int acg_measure_fp64_peak(int device, double *tflops) {
  if (!tflops) return fail(ACG_ERR_INVALID, "null out");
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double *out = nullptr;
  CK(cudaMalloc(&out, sizeof(double) * blocks * threads));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  k_fp64_fma<<<blocks, threads>>>(out, iters, 1.0000001);
  CK(cudaEventRecord(a));
  for (int r = 0; r < 5; r++) k_fp64_fma<<<blocks, threads>>>(out, iters, 1.0000001);
  CK(cudaEventRecord(b));
  CK(cudaEventSynchronize(b));
  float t = 0;
  CK(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const double flops = 5.0 * blocks * threads * (double)iters * 8 * 2;
  *tflops = flops / (t * 1e-3) / 1e12;
  return ACG_OK;
}

}  // extern "C"
