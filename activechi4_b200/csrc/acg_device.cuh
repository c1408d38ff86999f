// Device-side data layout, constants and helpers of the activechi4 B200 engine.
//
// Layout in HBM (all systems of a batch concatenated; one system = batch of 1):
//   particle slots  [poff_r, poff_r + n_r) per system r, poff_r a multiple of 32.
//     Between rebuilds the slots are in cell order (counting sort by cell,
//     ascending original index inside a cell), so neighbour gathers hit L1/L2.
//     pos  : double4 {x, y, z, type}   reduced coordinates in [0,1) + type as a
//            double, 32 B aligned -> one sector per neighbour gather
//     ux/uy/uz, vx/vy/vz, fx/fy/fz, ox/oy/oz : FP64 SoA (unfolded position,
//            momentum, force, unfolded position at the last rebuild)
//     id   : original particle index inside its system
//     act  : -1 or index into the system's direction array
//     cellof: cell of the slot at the last rebuild
//     nbn / nbl : full neighbour lists, `maxnb` entries per particle: 16-bit
//            staged indices per cell group (transposed) for boxes with >= 3
//            cells per side, int32 slot rows for 2-cell boxes
//   cells           [coff_r, coff_r + ncell_r): cstart (slot offset inside the
//                   system), ccount
//   directions      [aoff_r, aoff_r + nact_r): char4 {kx, ky, kz, 0}
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace acg {

constexpr int NHC_M = 3;
constexpr int BLOCK_A = 256;    // kick+drift: one thread per particle
constexpr int BLOCK_L = 256;    // list build: one warp per particle
constexpr int PART_L = BLOCK_L / 32;
constexpr int BLOCK_LC = 256;   // list build by cells: one block per cell
constexpr int BLOCK_R = 256;    // per-slot rebuild kernels (tiles of BLOCK_A)
constexpr int CELLS_PER_TILE = 8;
constexpr int BLOCK_SCAN = 512;
constexpr int BLOCK_G = 256;      // threads of the group kernels
constexpr int MAX_UNION = 64;     // 4 x 4 x 4 union cells of a 2 x 2 x 2 group
constexpr int BLOCK_X = 256;      // threads of the whole-box kernels
constexpr int BOX_CELLS = 8;      // most cells per whole-box block
constexpr int LIST_SPLIT = 4;     // blocks sharing a whole-box tile in the list build
// expected particles of a 2 x 2 x 2 list brick at most (else 2 x 2 x 1).
// Measured on the batched workload (256 FP32 replicas at density 1.2, where
// a 2 x 2 x 2 brick expects 29-51): 28 405 us a step, 48 and 64 650-660 us
// (the many particles past a brick's 32 lanes, listed one warp each, cost
// more than the lanes the smaller bricks leave idle)
#ifndef ACG_BRICK2_MAX
#define ACG_BRICK2_MAX 28.0
#endif
constexpr double BRICK2_MAX = ACG_BRICK2_MAX;
constexpr int BOX_WARP_MAX = 16384;  // whole-box particles up to which lists are built one warp per particle
constexpr int GSPLIT_MAX = 8;     // most force blocks per cell group (small boxes)
// measured on B200 (FP32, T = 0.45, step latency of one system alone):
// N = 4505 43-47 us per step on the per-particle kernels against 53 us on
// split cell groups, N = 11154 54 us against 59 us; N = 30000 68 us either way.
// With the per-particle lists built by cells: N = 30000 forces 43 us against
// 28 us on cell groups, a rebuild 101 us against 160 us, so the groups stay
// ahead at T = 0.45 (a rebuild every ~8 steps); N = 88250 134 against 103 us
// per step
#ifndef ACG_GSPLIT_BLOCKS
#define ACG_GSPLIT_BLOCKS 296
#endif
#ifndef ACG_PARTICLE_MAX
#define ACG_PARTICLE_MAX 20000
#endif
constexpr int GSPLIT_BLOCKS = ACG_GSPLIT_BLOCKS;  // cell-group force blocks aimed at per system (2 per SM)
// systems of up to this many particles take the per-particle kernels (lists
// of global slots, no staging, one warp per particle in the list build) even
// where cell groups would apply
constexpr int PARTICLE_MAX = ACG_PARTICLE_MAX;
constexpr int BLOCK_SORT = 1024;   // threads of the per-system sub-cell sort
constexpr int BLOCK_COMPACT = 1024; // threads of the rebuild-list compaction (one block)
constexpr int MAX_BOX_NC = 4;     // whole-box mode for 2..4 cells per side
constexpr int MAX_BOX_CELLS = MAX_BOX_NC * MAX_BOX_NC * MAX_BOX_NC;
constexpr int MAX_BOX_N = 8192;   // whole-box staging limit (FP64: 192 KB of shared memory)
constexpr int MAX_SUB3 = 1000;    // list sub-cells of a whole box (side >= 1.45 and L < 15: <= 10^3)
constexpr int MT_N = 624;         // MT19937 state words
constexpr int MT_WORDS = 625;     // one stored state: 624 words + the next word's index
constexpr int BLOCK_SHUF = 256;   // threads of the reference-order direction shuffle
constexpr int SHUF_SMEM_NACT = 32768;  // directions staged in shared memory up to this many

// A cell group: up to 2 x 2 x 2 cells (clipped at the box edge) and the union
// of their neighbour cells, up to 4 x 4 x 4, in which union cell (ux,uy,uz)
// is box cell lo+u wrapped, with the periodic image shift of that wrap.
struct GroupGeom {
  int lo[3], nu[3];
  double org[3];  // group centre, reduced units
};

__device__ __forceinline__ void group_geom(int g, int nc, int ng, GroupGeom &G) {
  const int gc[3] = {g % ng, (g / ng) % ng, g / (ng * ng)};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int c0 = 2 * gc[k], c1 = min(c0 + 2, nc);
    G.lo[k] = c0 - 1;
    G.nu[k] = (c1 - c0) + 2;
    G.org[k] = 0.5 * (double)(c0 + c1) / (double)nc;
  }
}

// KA pair constants (MDcode/cell_list+forces.c:19-20, MDcode/global.h:26,39-40)
constexpr double KA_C0 = 0.0162665594880;
constexpr double KA_C2 = -0.001949973872640;
constexpr double KA_RC2 = 6.25;  // (r/sigma)^2 cut
constexpr double TAU_P = 2.0;    // barostat time (tau_P, MDcode/global.h:42)

struct SysDesc {
  int n, nact, poff, aoff;
  int coff, ncell, nc, ng;     // ng: cell groups per side (0: no group path)
  int tile0_b, ntile_b, tau_p, thermostat;
  int shuffle, list_mode, precision, goff;  // goff: offset of the system's groups
  int tile0_a, ntile_a, box, xoff;            // kick/drift tiles; box: whole-box kernels (2..4 cells per side), xoff: first box tile
  int cpb, msub, bz, soff;                    // cpb: cells per whole-box block; msub: list sub-cells per side, bz: their list bricks' depth, soff: first sub-cell start
  int drift_every, gsplit, gtile0, pad2;      // drift_every: remove the mean momentum after every such step (0: never);
                                              // gsplit: force blocks per cell group, gtile0: first group force tile
  double L, invL, inv_cell;  // inv_cell: cells per unit reduced length (InvCellSize)
  double T, f0, dt, half_dt, skin2, rebuild_factor, dof;
  double q[NHC_M];
  double lcut2[3];           // list cut^2 (absolute units) for type sums 0 (AA), 1 (AB), 2 (BB)
  unsigned long long seed;
  // constant pressure (thermostat 4): L, invL and density above change on the
  // device before every step (k_npt_box); invL is the inverse of the length
  // before the last change, as the reference's drift uses it
  double density, P, cell_cut;
  // Nose-Hoover NPT (thermostat 5): L = L0 exp(eps); barostat mass w_eps =
  // DOF T tau_baro^2 and chain masses q_baro = T tau_baro^2
  // (InitialiseNoseHooverNPT, MDcode/time_evolve.c:614-652)
  double L0, w_eps, q_baro[NHC_M];
};

struct SysState {
  double eta_end[NHC_M], p_eta_end[NHC_M];  // chain at the step boundary
  double eta_cur[NHC_M], p_eta_cur[NHC_M];  // chain after the next step's first half
  double s1, s2;             // pending velocity scales (next first-half, last second-half)
  double ke_end;             // 0.5 sum p^2 at the boundary
  double pe, virial, vir_act;
  double maxD_last;
  unsigned long long maxd_bits;  // running max of |xu - xold|^2 (as bits) for this step
  long long step;
  long long rebuilds;
  int rebuild;               // rebuild this step
  int force_rebuild;         // host request
  int prime;                 // host request: recompute forces + thermostat pre-half
  int status;                // 1 = non-finite kinetic energy seen
  unsigned int counter_b;    // last-block counter of the force kernel
  int overflow;
  int obs_lo, obs_hi, obs_cur;  // observable events due this step, next event
  unsigned int counter_o;       // last-block counter of the observable kernel
  int shuf;                  // this step re-randomises the directions (reference order, MT19937)
  int mt_cur;                // which of the two stored MT19937 states is current
  int drift;                 // this step ends with the mean momentum removed (fixDrift)
  unsigned int counter_d;    // last-block counter of the drift kernels
  double drift_m[3];         // mean momentum of the last drift removal
  double ramp_T, ramp_dT;    // temperature ramp: this step's target and its change per step
  double ramp_end;           // the ramp's final temperature (target of the padding steps)
  long long ramp_left;       // ramp steps still to run (NVE with a velocity rescale before each)
  long long ramp_real;       // of these, steps of the ramp itself; the rest hold ramp_end
  // Gaussian isokinetic integrator (thermostat 3): the next first half kick
  // is p = s1 (p + g1 F); ga = this step's second half kick p = ga0 (p + ga1 F);
  // gmode = work due in the Gaussian kernels after the forces (1: the second
  // half kick and the next first half, 2: the next first half only)
  double g1;
  double ga[2];
  int gmode;
  unsigned int counter_g;    // last-block counter of the Gaussian kernels
  double pressure;           // constant pressure: pressure at the last box update
  // Nose-Hoover NPT (thermostat 5): barostat chain, p_eps and eps at the step
  // boundary and after the next step's first half; u2 = the half kicks'
  // p = p f1 + f2 F dt/2 factors of the current step
  double eta_baro_end[NHC_M], p_eta_baro_end[NHC_M], eta_baro_cur[NHC_M], p_eta_baro_cur[NHC_M];
  double p_eps_end, p_eps_cur, eps_end, eps_cur;
  double u2[2];
  double brown_m[3];         // active Brownian (thermostat 6): mean random force of this step
};

// In-place observables of one system (set by acg_obs_configure): events of the
// log-time schedule sorted by step; kind 0 = measure against an origin slot
// into a time bin, 1 = store the origin snapshot into a slot.
constexpr int OBS_EMAX = 16;  // events handled in one step
constexpr int OBS_NV = 5;     // per-event sums: overlap, r^2, sum d^4, r^4, Fs
struct ObsDesc {
  const long long *ev_step;
  const int *ev_info;   // kind | slot << 1 | bin << 13
  double *snap;         // [slot][particle id][3] unfolded reduced positions
  double *acc;          // [bin][8]: sum Q, sum Q^2, msd, msd_d4, msd_r4, Fs, count, -
  const int *qvec;      // [nq][3] integer wave vectors (q = 2 pi n / L)
  int n_events, nbins, nq, nslots;
  double a2;            // overlap cut squared (absolute units)
};

struct View {
  const SysDesc *desc;
  SysState *st;
  double4 *pos;
  double *ux, *uy, *uz, *vx, *vy, *vz, *fx, *fy, *fz, *ox, *oy, *oz;
  int *id, *act, *cellof, *nbn, *nbl;
  char4 *kdir;
  double4 *pos_s;
  double *ux_s, *uy_s, *uz_s, *vx_s, *vy_s, *vz_s, *fx_s, *fy_s, *fz_s;
  int *id_s, *act_s;
  int *cell_tmp, *perm_u, *perm;
  float4 *xsub;     // whole-box systems with list sub-cells: the system in sub-cell order {x, y, z, list code}
  int *ssub;        // their sub-cell starts [msub^3 + 1] per system
  int *rbs;         // this step's rebuilding systems with list sub-cells: count, bricks, then (system, first brick)
  unsigned int *mt; // [nsys][2][MT_WORDS]: two stored MT19937 states per system (current, next)
  int *ccount_b, *cfill, *cstart, *ccount;
  const int2 *tiles_a, *tiles_b, *tiles_l, *tiles_c, *tiles_g, *tiles_x;
  const int2 *tiles_lc;  // (system, cell): list build by cells (per-particle systems, >= 3 cells per side)
  int ntiles_lc, lccap;  // lccap: staged candidates of a cell's 27 neighbours (shared memory)
  int *gstart;      // per group: first centre particle (prefix over the system's groups)
  double4 *part_b;
  double4 *pacc;    // whole-box systems: per-particle pe, virial, KE, active virial
  unsigned int *counter_a;
  ObsDesc *obs;      // [nsys]
  double *part_o;    // [tiles_a][OBS_EMAX][OBS_NV]
  double *stage_d;  // [9n] x, xu, p interleaved per system (original order)
  int *stage_i;     // [2n] type, act
  double *stage_f;  // [3n] forces
  int ntiles_a, ntiles_b, ntiles_l, ntiles_c, ntiles_g, ntiles_x, nsys, maxnb;
  int box_warp;     // whole-box lists built one warp per particle (few such particles), else per brick
  int gcap;         // staged-particle capacity of a cell group (shared memory)
};

// minimum image in reduced units.  For |d| < 1.5 (all differences of wrapped
// coordinates) d - rint(d) performs exactly the reference's operations
// (MDcode/cell_list+forces.c:177-182): d-1 for d > 0.5, d+1 for d < -0.5, d
// unchanged otherwise, including d = +-0.5 (round-half-even gives 0).
__device__ __forceinline__ double min_image(double d) { return d - rint(d); }

// applypbc1 (MDcode/time_evolve.c:15-26) for a displacement far below one box:
// the while loops run at most once.  A coordinate still outside [0,1) (only
// possible for non-finite or absurd velocities) is folded with floor so that
// no loop can run unbounded.
__device__ __forceinline__ double wrap_unit(double x) {
  if (x >= 1.0) {
    x = __dadd_rn(x, -1.0);
    if (x >= 1.0) x = x - floor(x);
  } else if (x < 0.0) {
    x = __dadd_rn(x, 1.0);
    if (x < 0.0) x = x - floor(x);
  }
  return x;
}

__device__ __forceinline__ int cell_coord(double x, double inv, int nc) {
  double f = floor(__dmul_rn(x, inv));
  int c = (int)f;  // NaN converts to 0
  c = c < 0 ? 0 : c;
  return c >= nc ? nc - 1 : c;
}

// per-dimension neighbour-cell offsets without repeats: {-1,0,1} when there
// are >= 3 cells on a side, {0,1} for 2, {0} for 1
__device__ __forceinline__ int stencil_lo(int nc) { return nc >= 3 ? -1 : 0; }
__device__ __forceinline__ int stencil_hi(int nc) { return nc >= 2 ? 1 : 0; }
__device__ __forceinline__ int wrap_cell(int c, int nc) {
  c += nc;
  return c >= nc ? (c >= 2 * nc ? c - 2 * nc : c - nc) : c;
}

// U4Propagator (MDcode/time_evolve.c:578-609): one chain sweep jStart..jEnd,
// `ksum` = sum p^2 for the j == 0 link.
__device__ inline void nhc_u4(double *p_eta, const double *q, double T, double dof, double t,
                              int j0, int j1, double ksum) {
  int dj = j0 > j1 ? -1 : 1;
  int j = j0;
  double gj;
  do {
    if (j == 0)
      gj = ksum - dof * T;
    else
      gj = (p_eta[j - 1] * p_eta[j - 1]) / q[j - 1] - T;
    if (j == NHC_M - 1) {
      p_eta[j] = p_eta[j] + t * gj;
    } else {
      double x = t * p_eta[j + 1] / q[j + 1];
      double e = exp(-x);
      p_eta[j] = p_eta[j] * e + t * gj * (1.0 - e) / x;
    }
    j += dj;
  } while (j - dj != j1);
}

// U4(t/2..) U3 U4 half of the NHC Trotter split (MDcode/time_evolve.c:499-501)
// applied to chain (eta, p_eta) with sum p^2 = ksum; returns the velocity
// scale of U3.
__device__ inline double nhc_half(double *eta, double *p_eta, const double *q, double T,
                                  double dof, double dt, double ksum) {
  const double t4 = dt * 0.25, t3 = dt * 0.50;
  nhc_u4(p_eta, q, T, dof, t4, NHC_M - 1, 0, ksum);
  double s = exp(-t3 * p_eta[0] / q[0]);
  for (int i = 0; i < NHC_M; i++) eta[i] = eta[i] + t3 * p_eta[i] / q[i];
  double s2k = (s * s) * ksum;
  nhc_u4(p_eta, q, T, dof, t4, 0, NHC_M - 1, s2k);
  return s;
}

// Nose-Hoover NPT chains (MDcode/time_evolve.c:700-822).  U4PropagatorNPT:
// the particle chain as nhc_u4, then the barostat chain the same way with
// G_0 = p_eps^2 / w_eps - T.
__device__ inline void baro_u4(double *p_eta_b, const double *q_b, double T, double t, int j0, int j1,
                               double p_eps, double w_eps) {
  int dj = j0 > j1 ? -1 : 1;
  int j = j0;
  double gj;
  do {
    if (j == 0)
      gj = p_eps * p_eps / w_eps - T;
    else
      gj = (p_eta_b[j - 1] * p_eta_b[j - 1]) / q_b[j - 1] - T;
    if (j == NHC_M - 1) {
      p_eta_b[j] = p_eta_b[j] + t * gj;
    } else {
      double x = t * p_eta_b[j + 1] / q_b[j + 1];
      double e = exp(-x);
      p_eta_b[j] = p_eta_b[j] * e + t * gj * (1.0 - e) / x;
    }
    j += dj;
  } while (j - dj != j1);
}

// U4 U3 U4 of the NPT split (:660-662, :690-692) on the particle chain
// (eta, p_eta), the barostat chain (eta_b, p_eta_b) and p_eps, with sum p^2 =
// ksum before U3; returns the particles' U3 velocity scale.
__device__ inline double npt_half(double *eta, double *p_eta, double *eta_b, double *p_eta_b, double &p_eps,
                                  const double *q, const double *q_b, double w_eps, double T, double dof,
                                  double dt, double ksum) {
  const double t4 = dt * 0.25, t3 = dt * 0.50;
  nhc_u4(p_eta, q, T, dof, t4, NHC_M - 1, 0, ksum);
  baro_u4(p_eta_b, q_b, T, t4, NHC_M - 1, 0, p_eps, w_eps);
  const double s = exp(-t3 * p_eta[0] / q[0]);
  for (int i = 0; i < NHC_M; i++) {
    eta[i] = eta[i] + t3 * p_eta[i] / q[i];
    eta_b[i] += t3 * p_eta_b[i] / q_b[i];
  }
  p_eps = p_eps * exp(-t3 * p_eta_b[0] / q_b[0]);
  const double s2k = (s * s) * ksum;
  nhc_u4(p_eta, q, T, dof, t4, 0, NHC_M - 1, s2k);
  baro_u4(p_eta_b, q_b, T, t4, 0, NHC_M - 1, p_eps, w_eps);
  return s;
}

// U2PrimePropagatorNPT (:737-755): p_eps += 3 (PV - P L^3) dt/2 with PV =
// alpha sum p^2 / 3 + virial, alpha = 1 + 3/DOF
__device__ inline void npt_u2prime(double &p_eps, double ksum, double virial, double P, double L, double dof,
                                   double half_dt) {
  const double alpha = 1.0 + 3.0 / dof;
  const double PV = alpha * (ksum) / (3.00) + virial;
  p_eps += 3.00 * (PV - P * L * L * L) * half_dt;
}

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC'11): ten rounds of two
// 32x32->64 multiplies on a 128-bit counter under a 64-bit key bumped by the
// Weyl constants after every round
struct Philox4 {
  unsigned int x, y, z, w;
};
__host__ __device__ inline Philox4 philox4x32(Philox4 c, unsigned int k0, unsigned int k1) {
  for (int r = 0; r < 10; r++) {
    const unsigned long long p0 = 0xD2511F53ull * (unsigned long long)c.x;
    const unsigned long long p1 = 0xCD9E8D57ull * (unsigned long long)c.z;
    const unsigned int hi0 = (unsigned int)(p0 >> 32), lo0 = (unsigned int)p0;
    const unsigned int hi1 = (unsigned int)(p1 >> 32), lo1 = (unsigned int)p1;
    c = Philox4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// uniform in (0, 1) from 53 bits of two words
__host__ __device__ inline double u53(unsigned int a, unsigned int b) {
  const unsigned long long m = ((((unsigned long long)a) << 32) | b) >> 11;
  return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
}

// three standard normals of particle `id` at step `step` of stream `seed`
// (Box-Muller on two Philox draws: counters {id, step lo, step hi, 0 | 1})
__device__ inline void normals3(unsigned long long seed, long long step, int id, double g[3]) {
  const unsigned int k0 = (unsigned int)seed, k1 = (unsigned int)(seed >> 32);
  const unsigned int s0 = (unsigned int)(unsigned long long)step, s1 = (unsigned int)((unsigned long long)step >> 32);
  const Philox4 a = philox4x32(Philox4{(unsigned int)id, s0, s1, 0u}, k0, k1);
  const Philox4 b = philox4x32(Philox4{(unsigned int)id, s0, s1, 1u}, k0, k1);
  const double r1 = sqrt(-2.0 * log(u53(a.x, a.y))), t1 = 6.283185307179586 * u53(a.z, a.w);
  const double r2 = sqrt(-2.0 * log(u53(b.x, b.y))), t2 = 6.283185307179586 * u53(b.z, b.w);
  g[0] = r1 * cos(t1);
  g[1] = r1 * sin(t1);
  g[2] = r2 * cos(t2);
}

// MT19937 (Matsumoto & Nishimura 1998): seeding by their 2002 initialisation
// (GSL's gsl_rng_set for mt19937, seed 0 taken as 4357), tempering of one word
__host__ __device__ inline void mt_seed(unsigned int *mt, unsigned long long seed) {
  if (seed == 0) seed = 4357;
  mt[0] = (unsigned int)(seed & 0xffffffffull);
  for (int i = 1; i < MT_N; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (unsigned int)i;
  mt[MT_N] = MT_N;  // next word index: the first draw twists
}
__device__ __forceinline__ unsigned int mt_temper(unsigned int y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  return y ^ (y >> 18);
}

// keyed bijection of 32-bit integers (4-round Feistel network): distinct
// inputs give distinct keys, which makes rank-by-key an exact permutation
__device__ __forceinline__ uint32_t feistel32(uint32_t v, uint64_t key) {
  uint32_t L = v >> 16, R = v & 0xffffu;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    uint32_t k = (uint32_t)(key >> (16 * r)) * 0x9E3779B1u + (uint32_t)r * 0x7F4A7C15u;
    uint32_t f = (R ^ k) * 0x85EBCA6Bu;
    f ^= f >> 13;
    f *= 0xC2B2AE35u;
    f ^= f >> 16;
    uint32_t nl = R, nr = (L ^ f) & 0xffffu;
    L = nl;
    R = nr;
  }
  return (L << 16) | R;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace acg
