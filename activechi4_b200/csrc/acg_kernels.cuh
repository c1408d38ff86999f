// Kernels of one MD timestep (all systems of a batch in one launch each).
//
// Step s, for every system r (MDcode/time_evolve.c:495-526 restated):
//   k_kick_drift   v = (v*s2)*s1 + F*dt/2 ; x,xu += v*dt/L ; wrap ; max|xu-xold|^2
//                  (U3 of the previous step's second half, U3+U2 of this step's
//                  first half, U1).  Extra blocks re-randomise the direction
//                  arrays when the step is a shuffle step.  The last block to
//                  finish decides, per system, whether the lists are rebuilt
//                  and sets the CUDA-graph conditional that guards the rebuild.
//   rebuild (conditional):
//     k_cells_count    cell of every slot + per-cell counts
//     k_cells_scan     per-system exclusive scan -> cell starts
//     k_cells_scatter  slot -> position in its cell (unordered)
//     k_cells_order    per cell: order members by original index (stable
//                      counting sort, so InCell order is reproduced exactly)
//     k_permute        gather all per-particle arrays into cell order (scratch)
//     k_build_list_groups full neighbour lists, one block per group of 2x2x2
//                      cells with the union of their neighbour cells staged in
//                      shared memory (FP32 test, ballot compaction; 16-bit
//                      staged indices) and copy-back of the scratch arrays;
//                      k_build_list: int32 lists per particle for 2-cell boxes
//   k_force_groups pair forces from the 16-bit lists against the staged union
//                  (one thread per particle; k_force_kick: TPP threads per
//                  particle from int32 lists for 2-cell boxes), active force,
//                  second kick v += F dt/2, block
//                  sums of pe/virial/KE; the last block of each system finishes
//                  the sums in a fixed order and runs the thermostat chain
//                  (U4 U3 U4) for the end of this step and the first half of
//                  the next one.
#pragma once
#include "acg_device.cuh"

namespace acg {

// ---------------------------------------------------------------------------
// block reductions (fixed order => deterministic)
template <int NWARP>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NWARP; i++) t += sh[i];
  return t;  // valid in thread 0
}

__device__ __forceinline__ double block_sum_dyn(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; i++) t += sh[i];
  return t;
}

// ---------------------------------------------------------------------------
// direction shuffle: new k = +1 for the `count(+1)` smallest keyed ranks
__device__ inline int kcomp(char4 k, int c) { return c == 0 ? k.x : (c == 1 ? k.y : k.z); }
__device__ inline void kset(char4 *p, int c, int v) {
  signed char *b = reinterpret_cast<signed char *>(p);
  b[c] = (signed char)v;
}

__device__ void shuffle_component(const View &v, int r, int comp, long long step) {
  __shared__ unsigned int hist[256];
  __shared__ unsigned int s_cnt, s_prefix, s_mask, s_want;
  const SysDesc &d = v.desc[r];
  const int nact = d.nact;
  char4 *kd = v.kdir + d.aoff;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  unsigned int c = 0;
  for (int a = threadIdx.x; a < nact; a += blockDim.x) c += kcomp(kd[a], comp) > 0;
  atomicAdd(&s_cnt, c);
  __syncthreads();
  const unsigned int plus = s_cnt;
  if (plus == 0 || plus == (unsigned)nact) return;  // nothing to permute
  const uint64_t key = splitmix64(d.seed ^ splitmix64((uint64_t)step * 3ull + (uint64_t)comp));
  unsigned int prefix = 0, mask = 0, want = plus;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (int a = threadIdx.x; a < nact; a += blockDim.x) {
      uint32_t kk = feistel32((uint32_t)a, key);
      if ((kk & mask) == prefix) atomicAdd(&hist[(kk >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int cum = 0, sel = 255;
      for (unsigned int b = 0; b < 256; b++) {
        if (cum + hist[b] > want) {
          sel = b;
          break;
        }
        cum += hist[b];
      }
      s_want = want - cum;
      s_prefix = prefix | (sel << shift);
      s_mask = mask | (255u << shift);
    }
    __syncthreads();
    prefix = s_prefix;
    mask = s_mask;
    want = s_want;
    __syncthreads();
  }
  // exactly `plus` keys are below the key of rank `plus`
  for (int a = threadIdx.x; a < nact; a += blockDim.x)
    kset(&kd[a], comp, feistel32((uint32_t)a, key) < prefix ? 1 : -1);
}

// ---------------------------------------------------------------------------
// ShuffleActDirec (MDcode/active.c:45-85) in the reference's own order: for
// each component in turn (x, y, z) and i = 0 .. Nact-1, swap k[i] with k[j],
// j = (int)(Nact * u), u = the next MT19937 word / 2^32 (gsl_ran_flat(0, 1)
// through uniform(), MDcode/initialise.c:19-21).  All three components draw
// from one stream, so with the same seed the directions equal the reference
// program's bit for bit.
//
// One block per (system, component): every block regenerates the stream from
// the stored state (twisting 624 words per round in four dependency phases)
// and its one thread 0 applies the swaps of its component's draws to the
// component staged in shared memory; the swaps depend on one another and
// stay sequential.  The z block stores the state after all 3 Nact draws into
// the other buffer; the step's last force block makes it current.

// one twist of the 624-word state by all threads of the block: word i needs
// words i+1 (old) and i+397 (wrapping to i-227, already new for i >= 227),
// so [0,227), [227,454), [454,623) and 623 are computed one after another
__device__ __forceinline__ void mt_twist(unsigned int *mt) {
  const int lo[4] = {0, 227, 454, 623}, hi[4] = {227, 454, 623, 624};
#pragma unroll
  for (int ph = 0; ph < 4; ph++) {
    const int i = lo[ph] + (int)threadIdx.x;
    unsigned int w = 0;
    const bool act = i < hi[ph];
    if (act) {
      const unsigned int y = (mt[i] & 0x80000000u) | (mt[i + 1 < MT_N ? i + 1 : 0] & 0x7fffffffu);
      w = mt[i + 397 < MT_N ? i + 397 : i + 397 - MT_N] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    __syncthreads();
    if (act) mt[i] = w;
    __syncthreads();
  }
}

// one component of one system (blockDim.x == BLOCK_SHUF); state read from
// mt_in, the final state (after 3 nact draws) written to mt_out by comp 2
__device__ void shuffle_ref_component(const View &v, int r, int comp, const unsigned int *mt_in,
                                      unsigned int *mt_out) {
  __shared__ unsigned int s_mt[MT_N];
  __shared__ int s_j[MT_N];
  extern __shared__ signed char s_k[];
  const SysDesc &d = v.desc[r];
  const int nact = d.nact;
  char4 *kd = v.kdir + d.aoff;
  signed char *kg = reinterpret_cast<signed char *>(kd) + comp;  // component bytes, stride 4
  const bool staged = nact <= SHUF_SMEM_NACT;
  for (int a = threadIdx.x; a < MT_N; a += blockDim.x) s_mt[a] = mt_in[a];
  if (staged)
    for (int a = threadIdx.x; a < nact; a += blockDim.x) s_k[a] = kg[4 * (size_t)a];
  int idx = (int)mt_in[MT_N];
  __syncthreads();
  const long long beg = (long long)comp * nact, end = beg + nact;
  long long pos = 0;  // draws taken so far
  const double fn = (double)nact;
  while (pos < end) {
    if (idx >= MT_N) {
      mt_twist(s_mt);
      idx = 0;
    }
    const long long take = min((long long)(MT_N - idx), end - pos);
    const long long lo = max(pos, beg), hi = pos + take;
    if (lo < hi) {
      const int w0 = idx + (int)(lo - pos), cnt = (int)(hi - lo);
      for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        // (double)Nact * uniform(0,1); the word / 2^32 is exact
        const double u = (double)mt_temper(s_mt[w0 + t]) * (1.0 / 4294967296.0);
        s_j[t] = (int)__dmul_rn(fn, u);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int i = (int)(lo - beg);
        if (staged) {
          for (int t = 0; t < cnt; t++, i++) {
            const int j = s_j[t];
            const signed char a = s_k[i];
            s_k[i] = s_k[j];
            s_k[j] = a;
          }
        } else {
          for (int t = 0; t < cnt; t++, i++) {
            const size_t ii = 4 * (size_t)i, jj = 4 * (size_t)s_j[t];
            const signed char a = kg[ii];
            kg[ii] = kg[jj];
            kg[jj] = a;
          }
        }
      }
      __syncthreads();
    }
    pos += take;
    idx += (int)take;
  }
  if (staged)
    for (int a = threadIdx.x; a < nact; a += blockDim.x) kg[4 * (size_t)a] = s_k[a];
  if (comp == 2) {
    for (int a = threadIdx.x; a < MT_N; a += blockDim.x) mt_out[a] = s_mt[a];
    if (threadIdx.x == 0) mt_out[MT_N] = (unsigned int)idx;
  }
}

// blocks 3 r + c: component c of system r (only >= 0: system `only`, blocks 0..2)
__global__ void __launch_bounds__(BLOCK_SHUF) k_shuffle_ref(View v, int only) {
  const int r = only >= 0 ? only : (int)blockIdx.x / 3, comp = (int)blockIdx.x % 3;
  const SysDesc &d = v.desc[r];
  const SysState &st = v.st[r];
  if (d.nact == 0 || (only < 0 && !st.shuf)) return;
  unsigned int *mt = v.mt + (size_t)r * 2 * MT_WORDS;
  shuffle_ref_component(v, r, comp, mt + (size_t)st.mt_cur * MT_WORDS, mt + (size_t)(st.mt_cur ^ 1) * MT_WORDS);
}

// the stored state after a shuffle outside the step becomes current
__global__ void k_mt_flip(View v, int r) {
  if (threadIdx.x == 0 && v.desc[r].nact > 0) v.st[r].mt_cur ^= 1;
}

// ---------------------------------------------------------------------------
// systems whose step starts with a force pass of their own (force mode 3):
// the Berendsen barostat's box change (thermostat 4) and the active Brownian
// predictor (thermostat 6); none during a ramp
__device__ __forceinline__ bool pre_due(const SysDesc &d, const SysState &st) {
  return (d.thermostat == 4 || d.thermostat == 6) && st.ramp_left == 0;
}

// active Brownian constants with D0 = 1 (MDcode/global.h:50, initialise.c:
// 287-291): D0ByT = D0/T, TByD0 = T/D0, expFactor = exp(-dt TByD0); the
// displacement dx = D0ByT ((1 - e) p + c f) with c = D0ByT (TByD0 dt - (1 - e))
struct BrownConst {
  double d0t, e, ome, c, cp;
  __device__ __forceinline__ explicit BrownConst(const SysDesc &d) {
    d0t = 1.0 / d.T;
    const double t0 = d.T / 1.0;
    e = exp(-d.dt * t0);
    ome = 1.0 - e;
    c = d0t * (t0 * d.dt - ome);
    cp = d0t * ome;
  }
  __device__ __forceinline__ double dx(double p, double f) const {
    return __dmul_rn(d0t, __dadd_rn(__dmul_rn(ome, p), __dmul_rn(c, f)));
  }
};

// the system's Brownian scratch in the upload staging area (free while it
// steps): random force, position before the predictor, force before it
__device__ __forceinline__ double *brown_scratch(const View &v, const SysDesc &d) {
  return v.stage_d + 9 * (size_t)d.poff;
}

// advance_time_ActiveBrown_PC's corrector for one particle (MDcode/
// time_evolve.c:915-946): back to the position before the predictor, the
// mean of the two forces plus the random force, x and x_u moved, p updated;
// returns |x_u - x_old|^2 (reduced units) for the rebuild test
__device__ __forceinline__ double brown_correct_one(const View &v, const SysDesc &d, int i) {
  const BrownConst B(d);
  const int n = d.n, loc = i - d.poff;
  const double *s = brown_scratch(v, d);
  const double il = d.invL;
  const double fr[3] = {s[3 * loc], s[3 * loc + 1], s[3 * loc + 2]};
  const double ro[3] = {s[3 * n + 3 * loc], s[3 * n + 3 * loc + 1], s[3 * n + 3 * loc + 2]};
  const double fo[3] = {s[6 * n + 3 * loc], s[6 * n + 3 * loc + 1], s[6 * n + 3 * loc + 2]};
  const double F[3] = {v.fx[i], v.fy[i], v.fz[i]};
  double *pv[3] = {v.vx + i, v.vy + i, v.vz + i};
  double *uv[3] = {v.ux + i, v.uy + i, v.uz + i};
  const double *ov[3] = {v.ox + i, v.oy + i, v.oz + i};
  double4 pos = v.pos[i];
  double xo[3], e2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double f = __dadd_rn(fr[k], __dmul_rn(0.5, __dadd_rn(F[k], fo[k])));
    const double p = *pv[k];
    const double dd = B.dx(p, f);
    const double step = __dmul_rn(dd, il);
    xo[k] = wrap_unit(__dadd_rn(ro[k], step));
    const double u = __dadd_rn(*uv[k], step);
    *uv[k] = u;
    *pv[k] = __dadd_rn(__dmul_rn(B.e, p), __dmul_rn(B.cp, f));
    const double ex = __dadd_rn(u, -*ov[k]);
    e2 = __dadd_rn(e2, __dmul_rn(ex, ex));
  }
  pos.x = xo[0];
  pos.y = xo[1];
  pos.z = xo[2];
  v.pos[i] = pos;
  return e2;
}

// U3 U2 (pending thermostat scales and the half kick) and U1 for one
// particle, in the reference's order of roundings; returns |x_u - x_old|^2
// (reduced units) for the rebuild test
__device__ __forceinline__ double kick_drift_one(const View &v, const SysDesc &d, const SysState &st, int i) {
  const double hdt = d.half_dt, dt = d.dt, il = d.invL;
  const double s1 = st.s1, s2 = st.s2;
  double px, py, pz;
  if (d.thermostat == 5 && st.ramp_left == 0) {
    // Nose-Hoover NPT: U3 scale, then U2PropagatorNPT p f1 + f2 F dt/2
    // (MDcode/time_evolve.c:721-735)
    const double f1 = st.u2[0], f2 = st.u2[1];
    px = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(v.vx[i], s2), s1), f1), __dmul_rn(__dmul_rn(f2, v.fx[i]), hdt));
    py = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(v.vy[i], s2), s1), f1), __dmul_rn(__dmul_rn(f2, v.fy[i]), hdt));
    pz = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(v.vz[i], s2), s1), f1), __dmul_rn(__dmul_rn(f2, v.fz[i]), hdt));
  } else if (d.thermostat == 3) {
    const double g1 = st.g1;
    // Gaussian isokinetic half kick p = factor1 (p + factor2 F)
    // (MDcode/time_evolve.c:388-394)
    px = __dmul_rn(s1, __dadd_rn(__dmul_rn(v.vx[i], s2), __dmul_rn(g1, v.fx[i])));
    py = __dmul_rn(s1, __dadd_rn(__dmul_rn(v.vy[i], s2), __dmul_rn(g1, v.fy[i])));
    pz = __dmul_rn(s1, __dadd_rn(__dmul_rn(v.vz[i], s2), __dmul_rn(g1, v.fz[i])));
  } else {
    // v_b * s1 + F dt/2
    px = __dadd_rn(__dmul_rn(__dmul_rn(v.vx[i], s2), s1), __dmul_rn(v.fx[i], hdt));
    py = __dadd_rn(__dmul_rn(__dmul_rn(v.vy[i], s2), s1), __dmul_rn(v.fy[i], hdt));
    pz = __dadd_rn(__dmul_rn(__dmul_rn(v.vz[i], s2), s1), __dmul_rn(v.fz[i], hdt));
  }
  double ddx = __dmul_rn(__dmul_rn(px, dt), il);
  double ddy = __dmul_rn(__dmul_rn(py, dt), il);
  double ddz = __dmul_rn(__dmul_rn(pz, dt), il);
  double4 p = v.pos[i];
  double ux = __dadd_rn(v.ux[i], ddx), uy = __dadd_rn(v.uy[i], ddy), uz = __dadd_rn(v.uz[i], ddz);
  p.x = wrap_unit(__dadd_rn(p.x, ddx));
  p.y = wrap_unit(__dadd_rn(p.y, ddy));
  p.z = wrap_unit(__dadd_rn(p.z, ddz));
  double ex = __dadd_rn(ux, -v.ox[i]), ey = __dadd_rn(uy, -v.oy[i]), ez = __dadd_rn(uz, -v.oz[i]);
  v.vx[i] = px;
  v.vy[i] = py;
  v.vz[i] = pz;
  v.ux[i] = ux;
  v.uy[i] = uy;
  v.uz[i] = uz;
  v.pos[i] = p;
  return __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
}

// rebuild decision of one system from its max squared displacement (reduced)
__device__ __forceinline__ int rebuild_decision(const SysDesc &d, SysState &st, double maxd_red) {
  const double m = __dmul_rn(__dmul_rn(maxd_red, d.L), d.L);
  st.maxD_last = m;
  const int rb = (__dmul_rn(d.rebuild_factor, m) > d.skin2) || st.force_rebuild;
  st.rebuild = rb;
  st.force_rebuild = 0;
  return rb;
}

// observable events of one system due at the end of its current step
// (frame = loop index step); returns whether there are any
__device__ __forceinline__ int obs_due(const ObsDesc &o, SysState &st) {
  if (o.n_events == 0) {
    st.obs_lo = st.obs_hi = 0;
    return 0;
  }
  const long long step = st.step;
  int c = st.obs_cur;
  while (c < o.n_events && o.ev_step[c] < step) c++;
  const int lo = c;
  while (c < o.n_events && o.ev_step[c] == step && c - lo < OBS_EMAX) c++;
  st.obs_lo = lo;
  st.obs_hi = c;
  st.obs_cur = c;
  return c > lo;
}

// ---------------------------------------------------------------------------
// per-step events of one system decided before its forces: the direction
// shuffle every tau_p steps (MDcode/main.c:245-247) and the mean-momentum
// removal after every drift_every-th step (MDcode/main.c:261); neither runs
// during a temperature ramp (the reference's ramps, MDcode/initialise.c:166-201,
// only step)
__device__ __forceinline__ bool shuffle_due(const SysDesc &d, const SysState &st, int mode) {
  return d.shuffle == mode && d.nact > 0 && d.tau_p > 0 && st.ramp_left == 0 && (st.step % d.tau_p) == 0;
}

// stage 1: kick + drift (+ uniform-shuffle blocks) + rebuild decision
// The last block sets the step's graph branch h_pre, a switch before the
// forces over the work due in some system: bit 0 list rebuild, bit 1
// reference-order shuffle, bit 2 observable events (the positions of the step
// are final after the drift); value = bits - 1, or 7 for none.  The drift
// removal after the step (st.drift) is scheduled by the host between graph
// launches, or run by the kernel-by-kernel step.
__global__ void __launch_bounds__(BLOCK_A) k_kick_drift(View v, int use_cond, cudaGraphConditionalHandle h_pre) {
  __shared__ double sm[BLOCK_A / 32];
  __shared__ int s_last;
  const int b = blockIdx.x;
  double mymax = 0.0;
  int r = -1;
  if (b < v.ntiles_a) {
    int2 t = v.tiles_a[b];
    r = t.x;
    const SysDesc &d = v.desc[r];
    int loc = t.y + threadIdx.x;
    if (loc < d.n) {
      if (d.thermostat == 6 && v.st[r].ramp_left == 0)
        mymax = brown_correct_one(v, d, d.poff + loc);
      else
        mymax = kick_drift_one(v, d, v.st[r], d.poff + loc);
    }
    // per-system block max (a tile never straddles systems)
    for (int o = 16; o > 0; o >>= 1) mymax = fmax(mymax, __shfl_down_sync(0xffffffffu, mymax, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mymax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = sm[0];
      for (int w = 1; w < BLOCK_A / 32; w++) m = fmax(m, sm[w]);
      if (m > 0.0)
        atomicMax(&v.st[r].maxd_bits, (unsigned long long)__double_as_longlong(m));
    }
  } else {
    int q = b - v.ntiles_a;
    int rs = q / 3, comp = q % 3;
    if (shuffle_due(v.desc[rs], v.st[rs], 2)) shuffle_component(v, rs, comp, v.st[rs].step);
  }
  // the last block to finish takes the per-system rebuild decisions
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(v.counter_a, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  int any = 0, any_obs = 0, any_shuf = 0;
  for (int s = threadIdx.x; s < v.nsys; s += blockDim.x) {
    const SysDesc &d = v.desc[s];
    SysState &st = v.st[s];
    unsigned long long bits = atomicExch(&st.maxd_bits, 0ull);
    any |= rebuild_decision(d, st, __longlong_as_double((long long)bits));
    st.shuf = shuffle_due(d, st, 1);
    any_shuf |= st.shuf;
    st.drift = d.drift_every > 0 && st.ramp_left == 0 && (st.step % d.drift_every) == 0;
    // observable events due at the end of this step (none during a ramp)
    int ob = 0;
    if (st.ramp_left == 0) {
      ob = obs_due(v.obs[s], st);
    } else {
      st.obs_lo = st.obs_hi = 0;
    }
    any_obs |= ob;
  }
  any = __syncthreads_or(any);
  any_obs = __syncthreads_or(any_obs);
  any_shuf = __syncthreads_or(any_shuf);
  if (threadIdx.x == 0) {
    *v.counter_a = 0;
    if (use_cond) {
      const unsigned bits = (any ? 1u : 0u) | (any_shuf ? 2u : 0u) | (any_obs ? 4u : 0u);
      cudaGraphSetConditional(h_pre, bits ? bits - 1u : 7u);
    }
  }
}

// one particle's part of observable event `info`: store its origin snapshot
// (kind 1) or its overlap, |dr|^2, sum dx^4, |dr|^4 and sum_q cos(q.dr)
// against the origin (kind 0)
__device__ __forceinline__ void obs_particle(const ObsDesc &o, int n, int info, int id, double ux, double uy,
                                             double uz, double L, double val[OBS_NV]) {
  const int kind = info & 1, slot = (info >> 1) & 4095;
  double *sn = o.snap + ((size_t)slot * n + id) * 3;
  if (kind == 1) {
    sn[0] = ux;
    sn[1] = uy;
    sn[2] = uz;
    return;
  }
  const double dx = ux - sn[0], dy = uy - sn[1], dz = uz - sn[2];
  double mx = dx, my = dy, mz = dz;  // Analysis/overlap.c:67-78
  if (mz >= 0.5) mz -= 1.0; else if (mz < -0.5) mz += 1.0;
  if (my >= 0.5) my -= 1.0; else if (my < -0.5) my += 1.0;
  if (mx >= 0.5) mx -= 1.0; else if (mx < -0.5) mx += 1.0;
  const double r2q = L * L * (mx * mx + my * my + mz * mz);
  val[0] = r2q < o.a2 ? 1.0 : 0.0;
  const double r2 = L * L * (dx * dx + dy * dy + dz * dz);
  val[1] = r2;
  val[2] = L * L * L * L * (dx * dx * dx * dx + dy * dy * dy * dy + dz * dz * dz * dz);
  val[3] = r2 * r2;
  double fs = 0.0;
  for (int q = 0; q < o.nq; q++)
    fs += cos(6.283185307179586 * ((double)o.qvec[3 * q] * dx + (double)o.qvec[3 * q + 1] * dy +
                                   (double)o.qvec[3 * q + 2] * dz));
  val[4] = fs;
}

// add one event's sums over the system to its time bin
__device__ __forceinline__ void obs_accumulate(const ObsDesc &o, int n, int info, const double sum[OBS_NV]) {
  const int bin = info >> 13;
  const double tot = (double)n;  // TotPart (Analysis/overlap.c:25)
  const double Q = sum[0] / tot;
  double *acc = o.acc + (size_t)bin * 8;
  acc[0] += Q;  // c[time_index] (Analysis/overlap.c:90-93)
  acc[1] += Q * Q;
  acc[2] += sum[1] / tot;  // msd[0..2] (Analysis/msd_pos.c:88-91)
  acc[3] += sum[2] / tot;
  acc[4] += sum[3] / tot;
  acc[5] += o.nq > 0 ? sum[4] / (tot * o.nq) : 0.0;
  acc[6] += 1.0;
}

// In-place observables at the scheduled steps (replaces writing data_coor.out
// at the log times, MDcode/main.c:252-257, and the offline Analysis/overlap.c,
// msd_pos.c, Fsqt.c sums over (origin, later frame) pairs).  Per particle and
// due event: store the origin snapshot, or accumulate the overlap
// Theta(a^2 - |dr_minimg|^2) (Analysis/overlap.c:61-83), |dr|^2, sum dx^4,
// |dr|^4 (Analysis/msd_pos.c:64-76) and sum_q cos(q.dr) over the wave vectors.
__global__ void __launch_bounds__(BLOCK_A) k_observe(View v) {
  __shared__ double red[OBS_EMAX * OBS_NV][BLOCK_A / 32];
  __shared__ int s_last;
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  const int lo = st.obs_lo, hi = st.obs_hi;
  if (hi <= lo) return;
  const SysDesc &d = v.desc[r];
  const ObsDesc &o = v.obs[r];
  const int loc = t.y + threadIdx.x;
  const bool valid = loc < d.n;
  const int i = d.poff + (valid ? loc : 0);
  const int id = valid ? v.id[i] : 0;
  const double ux = valid ? v.ux[i] : 0.0, uy = valid ? v.uy[i] : 0.0, uz = valid ? v.uz[i] : 0.0;
  const double L = d.L;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int e = lo; e < hi; e++) {
    const int info = o.ev_info[e];
    const int kind = info & 1;
    double val[OBS_NV] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid) obs_particle(o, d.n, info, id, ux, uy, uz, L, val);
    if (kind == 0) {
#pragma unroll
      for (int k = 0; k < OBS_NV; k++) {
        double x = val[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (l == 0) red[(e - lo) * OBS_NV + k][w] = x;
      }
    }
  }
  __syncthreads();
  double *part = v.part_o + (size_t)blockIdx.x * OBS_EMAX * OBS_NV;
  for (int k = threadIdx.x; k < (hi - lo) * OBS_NV; k += blockDim.x) {
    if (o.ev_info[lo + k / OBS_NV] & 1) continue;
    double x = 0.0;
    for (int ww = 0; ww < BLOCK_A / 32; ww++) x += red[k][ww];
    part[k] = x;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st.counter_o, 1u) == (unsigned)(d.ntile_a - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < hi - lo) {
    const int e = lo + threadIdx.x;
    const int info = o.ev_info[e];
    if ((info & 1) == 0) {
      double sum[OBS_NV] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int b = 0; b < d.ntile_a; b++) {
        const double *pb = v.part_o + ((size_t)(d.tile0_a + b) * OBS_EMAX + threadIdx.x) * OBS_NV;
        for (int k = 0; k < OBS_NV; k++) sum[k] += __ldcg(pb + k);
      }
      obs_accumulate(o, d.n, info, sum);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) st.counter_o = 0;
}

// host request: rebuild the systems flagged `prime` (all < 0: rebuild all)
__global__ void k_flag_rebuild(View v, int all) {
  for (int s = threadIdx.x; s < v.nsys; s += blockDim.x) {
    SysState &st = v.st[s];
    st.rebuild = all ? 1 : st.prime;
  }
}

// host request: rebuild system r only (at its current positions)
__global__ void k_flag_rebuild_one(View v, int r) {
  for (int s = threadIdx.x; s < v.nsys; s += blockDim.x) v.st[s].rebuild = s == r;
}

// ---------------------------------------------------------------------------
// rebuild stage (runs only for systems with st.rebuild set)
__global__ void __launch_bounds__(BLOCK_R) k_cells_count(View v) {
  int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  int loc = t.y + threadIdx.x;
  if (loc >= d.n) return;
  const int i = d.poff + loc;
  double4 p = v.pos[i];
  // cell = floor(x*Inv) + floor(y*Inv)*Nc + floor(z*Inv)*Nc*Nc
  // (MDcode/cell_list+forces.c:73-74), clamped to the grid
  int cx = cell_coord(p.x, d.inv_cell, d.nc), cy = cell_coord(p.y, d.inv_cell, d.nc),
      cz = cell_coord(p.z, d.inv_cell, d.nc);
  int c = cx + cy * d.nc + cz * d.nc * d.nc;
  v.cell_tmp[i] = c;
  atomicAdd(&v.ccount_b[d.coff + c], 1);
}

__global__ void __launch_bounds__(BLOCK_SCAN) k_cells_scan(View v) {
  __shared__ int sh[BLOCK_SCAN];
  const int r = blockIdx.x;
  SysState &st = v.st[r];
  if (!st.rebuild) return;
  const SysDesc &d = v.desc[r];
  const int nc = d.ncell, B = blockDim.x;
  const int chunk = (nc + B - 1) / B;
  const int beg = min(threadIdx.x * chunk, nc), end = min(beg + chunk, nc);
  int sum = 0;
  for (int c = beg; c < end; c++) sum += v.ccount_b[d.coff + c];
  sh[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < B; o <<= 1) {  // inclusive Hillis-Steele scan
    int x = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += x;
    __syncthreads();
  }
  int run = sh[threadIdx.x] - sum;
  for (int c = beg; c < end; c++) {
    int k = v.ccount_b[d.coff + c];
    v.cstart[d.coff + c] = run;
    v.ccount[d.coff + c] = k;
    v.ccount_b[d.coff + c] = 0;
    v.cfill[d.coff + c] = 0;
    run += k;
  }
  if (threadIdx.x == 0) {
    st.rebuilds += 1;
    st.overflow = 0;
  }
  if (d.ng > 0) {
    // first centre particle of every cell group (groups in index order):
    // per-thread chunks of groups, then the same block scan
    __syncthreads();
    const int ng = d.ng, nc_ = d.nc, ngr = ng * ng * ng;
    const int gch = (ngr + B - 1) / B;
    const int g0 = min(threadIdx.x * gch, ngr), g1 = min(g0 + gch, ngr);
    int gsum = 0;
    for (int g = g0; g < g1; g++) {
      const int gx = g % ng, gy = (g / ng) % ng, gz = g / (ng * ng);
      for (int cz = 2 * gz; cz < min(2 * gz + 2, nc_); cz++)
        for (int cy = 2 * gy; cy < min(2 * gy + 2, nc_); cy++)
          for (int cx = 2 * gx; cx < min(2 * gx + 2, nc_); cx++)
            gsum += v.ccount[d.coff + cx + cy * nc_ + cz * nc_ * nc_];
    }
    sh[threadIdx.x] = gsum;
    __syncthreads();
    for (int o = 1; o < B; o <<= 1) {
      int x = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += x;
      __syncthreads();
    }
    int grun = sh[threadIdx.x] - gsum;
    for (int g = g0; g < g1; g++) {
      v.gstart[d.goff + g] = grun;
      const int gx = g % ng, gy = (g / ng) % ng, gz = g / (ng * ng);
      for (int cz = 2 * gz; cz < min(2 * gz + 2, nc_); cz++)
        for (int cy = 2 * gy; cy < min(2 * gy + 2, nc_); cy++)
          for (int cx = 2 * gx; cx < min(2 * gx + 2, nc_); cx++)
            grun += v.ccount[d.coff + cx + cy * nc_ + cz * nc_ * nc_];
    }
  }
}

__global__ void __launch_bounds__(BLOCK_R) k_cells_scatter(View v) {
  int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  int loc = t.y + threadIdx.x;
  if (loc >= d.n) return;
  const int i = d.poff + loc;
  int c = v.cell_tmp[i];
  int k = atomicAdd(&v.cfill[d.coff + c], 1);
  v.perm_u[d.poff + v.cstart[d.coff + c] + k] = i;
}

// one warp per cell: order the members by original particle index.  Each
// lane holds one member; ranks are counted over register shuffles.
__global__ void __launch_bounds__(32 * CELLS_PER_TILE) k_cells_order(View v) {
  int2 t = v.tiles_c[blockIdx.x];
  const int r = t.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  const int c = t.y + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= d.ncell) return;
  const int m = v.ccount[d.coff + c];
  const int base = d.poff + v.cstart[d.coff + c];
  for (int a0 = 0; a0 < m; a0 += 32) {
    const int a = a0 + lane;
    int sa = -1, ida = 0x7fffffff;
    if (a < m) {
      sa = v.perm_u[base + a];
      ida = v.id[sa];
    }
    int rank = 0;
    for (int b0 = 0; b0 < m; b0 += 32) {
      const int b = b0 + lane;
      const int idb = b < m ? v.id[v.perm_u[base + b]] : 0x7fffffff;
#pragma unroll 8
      for (int q = 0; q < 32; q++) rank += __shfl_sync(0xffffffffu, idb, q) < ida;
    }
    if (a < m) {
      v.perm[base + rank] = sa;
      v.cellof[base + rank] = c;
    }
  }
}

__global__ void __launch_bounds__(BLOCK_R) k_permute(View v) {
  int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  int loc = t.y + threadIdx.x;
  if (loc >= d.n) return;
  const int i = d.poff + loc;
  const int o = v.perm[i];
  v.pos_s[i] = v.pos[o];
  v.ux_s[i] = v.ux[o];
  v.uy_s[i] = v.uy[o];
  v.uz_s[i] = v.uz[o];
  v.vx_s[i] = v.vx[o];
  v.vy_s[i] = v.vy[o];
  v.vz_s[i] = v.vz[o];
  v.fx_s[i] = v.fx[o];
  v.fy_s[i] = v.fy[o];
  v.fz_s[i] = v.fz[o];
  v.id_s[i] = v.id[o];
  v.act_s[i] = v.act[o];
}

__device__ __forceinline__ double lcut2_of(const SysDesc &d, int tsum) {
  return tsum == 0 ? d.lcut2[0] : (tsum == 1 ? d.lcut2[1] : d.lcut2[2]);
}

__device__ __forceinline__ void copy_back(const View &v, int i) {
  v.pos[i] = v.pos_s[i];
  v.ux[i] = v.ux_s[i];
  v.uy[i] = v.uy_s[i];
  v.uz[i] = v.uz_s[i];
  v.ox[i] = v.ux_s[i];
  v.oy[i] = v.uy_s[i];
  v.oz[i] = v.uz_s[i];
  v.vx[i] = v.vx_s[i];
  v.vy[i] = v.vy_s[i];
  v.vz[i] = v.vz_s[i];
  v.fx[i] = v.fx_s[i];
  v.fy[i] = v.fy_s[i];
  v.fz[i] = v.fz_s[i];
  v.id[i] = v.id_s[i];
  v.act[i] = v.act_s[i];
}

// Neighbour lists for boxes with 2 cells per side (one warp per particle, FP64
// minimum image per pair: the stencil's shifted frame is ambiguous there).
// the union cell holding staged index q: the last u with pre[u] <= q (pre is a
// non-decreasing prefix over n cells in shared memory)
__device__ __forceinline__ int union_of(const int *pre, int n, int q) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= q) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Lists of the per-particle kernels by cells (>= 3 cells per side): one
// block per cell stages its 27 neighbour cells' particles once (float4 of the
// FP32 reduced coordinates and slot | type << 30, cells in (oz, oy, ox) order,
// slots ascending), then each warp lists one centre particle at a time, the
// lanes testing 32 staged candidates a step and a ballot appending the
// accepted ones in staged order.  Same test, same order and so the same lists
// as k_build_list, which reads every candidate of every particle from global
// memory (27 cells x ~30 candidates x 32 bytes a particle).  A cell whose
// neighbourhood exceeds lccap staged candidates leaves its particles to the
// force kernel's cell scan.
__global__ void __launch_bounds__(BLOCK_LC) k_build_list_cells(View v) {
  extern __shared__ float4 cstg[];
  __shared__ int s_pre[28], s_start[27];
  const int2 t = v.tiles_lc[blockIdx.x];
  const int r = t.x, c = t.y;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  const int nc = d.nc;
  const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (warp == 0) {
    int m = 0;
    if (lane < 27) {
      const int ox = lane % 3 - 1, oy = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
      const int c2 = wrap_cell(cx + ox, nc) + wrap_cell(cy + oy, nc) * nc + wrap_cell(cz + oz, nc) * nc * nc;
      s_start[lane] = d.poff + v.cstart[d.coff + c2];
      m = v.ccount[d.coff + c2];
    }
    int x = m;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane < 27) s_pre[lane + 1] = x;
    if (lane == 0) s_pre[0] = 0;
  }
  __syncthreads();
  const int Q = s_pre[27];
  const int i0 = s_start[13], mc = s_pre[14] - s_pre[13];  // the centre cell (offset 0, 0, 0)
  const int maxnb = v.maxnb;
  if (Q <= v.lccap) {
    // staged index q over the 27 cells' runs, four loads in flight a thread
    for (int q0 = threadIdx.x; q0 < Q; q0 += 4 * blockDim.x) {
      double4 p[4];
      int jj[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int q = q0 + e * blockDim.x;
        jj[e] = -1;
        if (q < Q) {
          const int u = union_of(s_pre, 27, q);
          jj[e] = s_start[u] + (q - s_pre[u]);
          p[e] = v.pos_s[jj[e]];
        }
      }
#pragma unroll
      for (int e = 0; e < 4; e++)
        if (jj[e] >= 0)
          cstg[q0 + e * blockDim.x] =
              make_float4((float)p[e].x, (float)p[e].y, (float)p[e].z, __int_as_float(jj[e] | ((int)p[e].w << 30)));
    }
    __syncthreads();
    const float L2f = (float)(d.L * d.L);
    float lc[3];
    for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * (1.0 + 1e-5));
    for (int w = warp; w < mc; w += nwarps) {
      const int i = i0 + w;
      const float4 fi = cstg[s_pre[13] + w];
      const int ti = __float_as_int(fi.w) >> 30;
      // cut for a partner of type 0 / 1 (the sum of the two types indexes lc)
      const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
      int *row = v.nbl + (size_t)i * maxnb;
      int cnt = 0;
      for (int q0 = 0; q0 < Q; q0 += 32) {
        const int q = q0 + lane;
        bool ok = false;
        int j = 0;
        if (q < Q) {
          const float4 fj = cstg[q];
          const int code = __float_as_int(fj.w);
          j = code & 0x3fffffff;
          float dx = fi.x - fj.x, dy = fi.y - fj.y, dz = fi.z - fj.z;
          dx -= rintf(dx);
          dy -= rintf(dy);
          dz -= rintf(dz);
          const float dr2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) * L2f;
          ok = dr2 < ((code >> 30) ? c1 : c0) && j != i;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        if (ok) {
          const int pos = cnt + __popc(mask & ((1u << lane) - 1u));
          if (pos < maxnb) row[pos] = j;
        }
        cnt += __popc(mask);
      }
      if (lane == 0) {
        if (cnt > maxnb) {
          v.nbn[i] = -1;  // served from the cell list by the force kernel
          atomicAdd(&v.st[r].overflow, 1);
        } else {
          v.nbn[i] = cnt;
        }
      }
    }
  } else {
    for (int w = threadIdx.x; w < mc; w += blockDim.x) {
      v.nbn[i0 + w] = -1;
      atomicAdd(&v.st[r].overflow, 1);
    }
  }
  for (int w = threadIdx.x; w < mc; w += blockDim.x) copy_back(v, i0 + w);
}

__global__ void __launch_bounds__(BLOCK_L) k_build_list(View v) {
  int2 t = v.tiles_l[blockIdx.x];
  const int r = t.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  const int loc = t.y + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (loc >= d.n) return;
  const int i = d.poff + loc;
  const double4 pi = v.pos_s[i];
  const int ti = (int)pi.w;
  const int nc = d.nc, c = v.cellof[i];
  const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
  const int lo = stencil_lo(nc), w = stencil_hi(nc) - lo + 1, ncell = w * w * w;
  const int maxnb = v.maxnb;
  int *row = v.nbl + (size_t)i * maxnb;
  // the neighbour cells' runs, one cell per lane (27 lanes at most), read at
  // once; cell q in (oz, oy, ox) order is then broadcast from lane q
  int my_s0 = 0, my_m = 0;
  if (lane < ncell) {
    const int ox = lane % w + lo, oy = (lane / w) % w + lo, oz = lane / (w * w) + lo;
    const int c2 = wrap_cell(cx + ox, nc) + wrap_cell(cy + oy, nc) * nc + wrap_cell(cz + oz, nc) * nc * nc;
    my_s0 = d.poff + v.cstart[d.coff + c2];
    my_m = v.ccount[d.coff + c2];
  }
  // the test in FP32 on reduced coordinates with the cut widened by 1e-5
  // (the lists may hold a few pairs just outside the cut; the force loop tests
  // every entry): separation error ~1e-7 L against a margin of 1e-5 x 2.85
  const float L2f = (float)(d.L * d.L);
  float lc[3];
  for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * (1.0 + 1e-5));
  const float xi = (float)pi.x, yi = (float)pi.y, zi = (float)pi.z;
  int cnt = 0;
  // one cell ahead: the next cell's first 32 candidates load while this
  // cell's are tested
  int s0 = __shfl_sync(0xffffffffu, my_s0, 0), m = __shfl_sync(0xffffffffu, my_m, 0);
  double4 cur = lane < m ? v.pos_s[s0 + lane] : make_double4(0, 0, 0, 0);
  for (int q = 0; q < ncell; q++) {
    const int qn = q + 1 < ncell ? q + 1 : q;
    const int s0n = __shfl_sync(0xffffffffu, my_s0, qn), mn = __shfl_sync(0xffffffffu, my_m, qn);
    const double4 nxt = (q + 1 < ncell && lane < mn) ? v.pos_s[s0n + lane] : make_double4(0, 0, 0, 0);
    for (int k0 = 0; k0 < m; k0 += 32) {
      const int k = k0 + lane;
      const int j = s0 + k;
      bool ok = false;
      if (k < m && j != i) {
        const double4 pj = k0 == 0 ? cur : v.pos_s[j];
        float dx = xi - (float)pj.x, dy = yi - (float)pj.y, dz = zi - (float)pj.z;
        dx -= rintf(dx);
        dy -= rintf(dy);
        dz -= rintf(dz);
        const float dr2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) * L2f;
        ok = dr2 < lc[ti + (int)pj.w];
      }
      const unsigned int mask = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const int pos = cnt + __popc(mask & ((1u << lane) - 1u));
        if (pos < maxnb) row[pos] = j;
      }
      cnt += __popc(mask);
    }
    cur = nxt;
    s0 = s0n;
    m = mn;
  }
  if (lane == 0) {
    if (cnt > maxnb) {
      v.nbn[i] = -1;  // served from the cell list by the force kernel
      atomicAdd(&v.st[r].overflow, 1);
    } else {
      v.nbn[i] = cnt;
    }
    copy_back(v, i);
  }
}

// ---------------------------------------------------------------------------
// pair term (MDcode/cell_list+forces.c:174-203).  dr2/sigma^2 and 1/dr2 use
// the precomputed 1/sigma^2 instead of the reference's two divisions; the
// results agree to rounding.
struct PairAcc {
  double fx, fy, fz, pe, vir;
};

__device__ __forceinline__ void pair_fp64(PairAcc &a, const double4 &pi, int ti, const double4 &pj,
                                          double L, double L2) {
  const int tp = ti + (int)pj.w;
  double dx = min_image(pi.x - pj.x), dy = min_image(pi.y - pj.y), dz = min_image(pi.z - pj.z);
  double dr2 = (dx * dx + dy * dy + dz * dz) * L2;
  // 1/sigma^2, 4 eps, 8 eps/sigma^2 for AA / AB / BB
  const double is2 = tp == 0 ? 1.0 : (tp == 1 ? 1.5625 : 1.0 / (0.88 * 0.88));
  double rs2 = dr2 * is2;
  if (rs2 < KA_RC2) {
    const double e4 = tp == 0 ? 4.0 : (tp == 1 ? 6.0 : 2.0);
    double s2 = 1.0 / rs2;
    double s6 = s2 * s2 * s2;
    a.pe += e4 * ((s6 * (s6 - 1.0)) + KA_C0 + KA_C2 * rs2);
    double g = (2.0 * e4 * is2) * (6.0 * s6 * (s6 - 0.5) * s2 - KA_C2);
    double gl = g * L;
    a.fx += gl * dx;
    a.fy += gl * dy;
    a.fz += gl * dz;
    a.vir += g * dr2;
  }
}

__device__ __forceinline__ void pair_fp32(PairAcc &a, const double4 &pi, int ti, const double4 &pj,
                                          double L, double) {
  const int tp = ti + (int)pj.w;
  // the separation is formed in FP64 (positions stay FP64), the pair math in FP32
  const float Lf = (float)L;
  float dx = (float)min_image(pi.x - pj.x) * Lf, dy = (float)min_image(pi.y - pj.y) * Lf,
        dz = (float)min_image(pi.z - pj.z) * Lf;
  float dr2 = dx * dx + dy * dy + dz * dz;
  const float is2 = tp == 0 ? 1.0f : (tp == 1 ? 1.5625f : (float)(1.0 / (0.88 * 0.88)));
  float rs2 = dr2 * is2;
  if (rs2 < (float)KA_RC2) {
    const float e4 = tp == 0 ? 4.0f : (tp == 1 ? 6.0f : 2.0f);
    float s2 = __frcp_rn(rs2);
    float s6 = s2 * s2 * s2;
    a.pe += (double)(e4 * ((s6 * (s6 - 1.0f)) + (float)KA_C0 + (float)KA_C2 * rs2));
    float g = (2.0f * e4 * is2) * (6.0f * s6 * (s6 - 0.5f) * s2 - (float)KA_C2);
    a.fx += (double)(g * dx);
    a.fy += (double)(g * dy);
    a.fz += (double)(g * dz);
    a.vir += (double)(g * dr2);
  }
}

// finish one system after its last force block: fixed-order sums, then the
// thermostat chain (runs in a single block)
__device__ __noinline__ void finalize_sums(const SysDesc &d, SysState &st, int mode, double pe, double vir, double ke, double va);

__device__ void finalize_system(const View &v, int r, int mode) {
  __shared__ double sh[32];
  const SysDesc &d = v.desc[r];
  SysState &st = v.st[r];
  double pe = 0.0, vir = 0.0, ke = 0.0, va = 0.0;
  const bool per_particle = d.box;
  const int nparts = per_particle ? d.n : d.ntile_b;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    const double2 *pp = per_particle ? reinterpret_cast<const double2 *>(&v.pacc[d.poff + k])
                                     : reinterpret_cast<const double2 *>(&v.part_b[d.tile0_b + k]);
    const double2 p0 = __ldcg(pp), p1 = __ldcg(pp + 1);
    pe += p0.x;
    vir += p0.y;
    ke += p1.x;
    va += p1.y;
  }
  pe = block_sum_dyn(pe, sh);
  vir = block_sum_dyn(vir, sh);
  ke = block_sum_dyn(ke, sh);
  va = block_sum_dyn(va, sh);
  if (threadIdx.x != 0) return;
  finalize_sums(d, st, mode, pe, vir, ke, va);
}

// thermostat and scalars of one system from its sums (one thread): pe and
// virial halved (every pair is counted from both sides), then for a step the
// chain's second half on the new KE and its first half of the next step
// the velocity scale of the next step's first half from sum p^2 = kb of the
// velocities at the step boundary: the thermostat chain's U4 U3 U4
// (MDcode/time_evolve.c:499-501), a ramp step's rescale to the ramp target
// (adjustInitialTemp, MDcode/initialise.c:141-151, with inst_T of
// calculate_temp, :153-164), or none (NVE)
__device__ __noinline__ void next_first_half(const SysDesc &d, SysState &st, double kb) {
  if (st.ramp_left > 0) {
    const double inst = 2.0 * (kb * 0.5) / d.dof;
    st.s1 = sqrt(st.ramp_T / inst);
  } else if (d.thermostat == 1) {
    double eta[NHC_M], pet[NHC_M];
    for (int k = 0; k < NHC_M; k++) {
      eta[k] = st.eta_end[k];
      pet[k] = st.p_eta_end[k];
    }
    double s1 = nhc_half(eta, pet, d.q, d.T, d.dof, d.dt, kb);
    for (int k = 0; k < NHC_M; k++) {
      st.eta_cur[k] = eta[k];
      st.p_eta_cur[k] = pet[k];
    }
    st.s1 = s1;
  } else if (d.thermostat == 5) {
    // Nose-Hoover NPT first half (MDcode/time_evolve.c:660-665): U4 U3 U4 on
    // both chains and p_eps from the boundary state, U2Prime with sum p^2 after
    // U3 and the last forces' virial at the boundary length L0 exp(eps), the
    // U2 factors, then U1's box change eps += dt p_eps / w_eps, L = L0 exp(eps)
    // (:680-683); the drift keeps inv_L of the boundary length
    // (UpdateBoxForNPT ran at the end of the previous step)
    SysDesc &dm = const_cast<SysDesc &>(d);
    double eta[NHC_M], pet[NHC_M], etab[NHC_M], petb[NHC_M];
    for (int k = 0; k < NHC_M; k++) {
      eta[k] = st.eta_end[k];
      pet[k] = st.p_eta_end[k];
      etab[k] = st.eta_baro_end[k];
      petb[k] = st.p_eta_baro_end[k];
    }
    double p_eps = st.p_eps_end;
    const double s1 = npt_half(eta, pet, etab, petb, p_eps, d.q, d.q_baro, d.w_eps, d.T, d.dof, d.dt, kb);
    const double Lb = d.L0 * exp(st.eps_end);
    npt_u2prime(p_eps, (s1 * s1) * kb, st.virial, d.P, Lb, d.dof, d.half_dt);
    const double alpha = 1.0 + 3.0 / d.dof;
    const double x = d.half_dt * alpha * p_eps / d.w_eps;
    const double f1 = exp(-x);
    st.u2[0] = f1;
    st.u2[1] = (1.0 - f1) / x;
    const double eps = st.eps_end + d.dt * p_eps / d.w_eps;
    const double Ln = d.L0 * exp(eps);
    for (int k = 0; k < NHC_M; k++) {
      st.eta_cur[k] = eta[k];
      st.p_eta_cur[k] = pet[k];
      st.eta_baro_cur[k] = etab[k];
      st.p_eta_baro_cur[k] = petb[k];
    }
    st.p_eps_cur = p_eps;
    st.eps_cur = eps;
    st.s1 = s1;
    dm.invL = 1.0 / Lb;
    dm.L = Ln;
    dm.density = (double)d.n / (Ln * Ln * Ln);
    if (!(Ln > 0.0) || (int)((double)(int)Ln / d.cell_cut) != d.nc) st.status = 2;
  } else if (d.thermostat == 3) {
    // Gaussian isokinetic: the factors need sums of p.F and F^2 over the
    // system; k_gauss_apply computes them (no half kick until it has run)
    st.s1 = 1.0;
    st.g1 = 0.0;
    st.gmode = 2;
  } else {
    st.s1 = 1.0;
  }
}

__device__ __noinline__ void finalize_sums(const SysDesc &d, SysState &st, int mode, double pe, double vir, double ke, double va) {
  st.pe = 0.5 * pe;
  st.virial = (0.5 * vir) / 3.0;
  st.vir_act = va;
  if (mode >= 2) {  // force evaluation only (calculate_forces)
    __threadfence();
    st.counter_b = 0;
    return;
  }
  double kb;
  if (mode == 0 && st.ramp_left > 0) {
    // a ramp step (advance_time_NVEFrog inside coldstart / breakxal): NVE, the
    // step counter and its schedules stay where they are; the next ramp step
    // rescales to the next target (T +- time_step * rate)
    st.s2 = 1.0;
    kb = ke;
    st.ramp_left -= 1;
    st.ramp_real -= 1;
    if (st.ramp_left > 0) st.ramp_T = st.ramp_real > 0 ? __dadd_rn(st.ramp_T, st.ramp_dT) : st.ramp_end;
  } else if (mode == 0 && (d.thermostat == 2 || d.thermostat == 4)) {
    // advance_time_NVT_Berendsen (MDcode/time_evolve.c:173-256): after the
    // NVE step the momenta are scaled by chi = sqrt(1 + (T/inst_T - 1) dt /
    // tau_T); the step's KE and inst_T are reported before the scaling, as
    // the reference's globals hold them
    const double inst = 2.0 * (ke * 0.5) / d.dof;
    st.s2 = sqrt(1.00 + (d.T / inst - 1.00) * d.dt / 0.20);
    kb = ke;
    st.step += 1;
    if (st.shuf) {
      st.mt_cur ^= 1;
      st.shuf = 0;
    }
  } else if (mode == 0 && d.thermostat == 5) {
    // AdvanceTimeNPTNoseHoover's second half (MDcode/time_evolve.c:685-692):
    // U2 ran in the force pass; U2Prime with its sum p^2 and the new virial at
    // this step's length, then U4 U3 U4 on both chains and p_eps
    double eta[NHC_M], pet[NHC_M], etab[NHC_M], petb[NHC_M];
    for (int k = 0; k < NHC_M; k++) {
      eta[k] = st.eta_cur[k];
      pet[k] = st.p_eta_cur[k];
      etab[k] = st.eta_baro_cur[k];
      petb[k] = st.p_eta_baro_cur[k];
    }
    double p_eps = st.p_eps_cur;
    npt_u2prime(p_eps, ke, st.virial, d.P, d.L0 * exp(st.eps_cur), d.dof, d.half_dt);
    const double s2 = npt_half(eta, pet, etab, petb, p_eps, d.q, d.q_baro, d.w_eps, d.T, d.dof, d.dt, ke);
    for (int k = 0; k < NHC_M; k++) {
      st.eta_end[k] = eta[k];
      st.p_eta_end[k] = pet[k];
      st.eta_baro_end[k] = etab[k];
      st.p_eta_baro_end[k] = petb[k];
    }
    st.p_eps_end = p_eps;
    st.eps_end = st.eps_cur;
    st.s2 = s2;
    kb = (s2 * s2) * ke;
    st.step += 1;
    if (st.shuf) {
      st.mt_cur ^= 1;
      st.shuf = 0;
    }
  } else if (mode == 0 && d.thermostat == 3) {
    // AdvanceTimeNVTGaussOSM (MDcode/time_evolve.c:351-470): the second half
    // kick and the next first half need sums over the new forces; the
    // Gaussian kernels after this pass apply them (gmode 1)
    st.s2 = 1.0;
    kb = ke;
    st.step += 1;
    if (st.shuf) {
      st.mt_cur ^= 1;
      st.shuf = 0;
    }
  } else if (mode == 0) {
    if (d.thermostat == 1) {
      double eta[NHC_M], pet[NHC_M];
      for (int k = 0; k < NHC_M; k++) {
        eta[k] = st.eta_cur[k];
        pet[k] = st.p_eta_cur[k];
      }
      double s2 = nhc_half(eta, pet, d.q, d.T, d.dof, d.dt, ke);
      for (int k = 0; k < NHC_M; k++) {
        st.eta_end[k] = eta[k];
        st.p_eta_end[k] = pet[k];
      }
      st.s2 = s2;
      kb = (s2 * s2) * ke;
    } else {
      st.s2 = 1.0;
      kb = ke;
    }
    st.step += 1;
    if (st.shuf) {  // the shuffle's new MT19937 state becomes current
      st.mt_cur ^= 1;
      st.shuf = 0;
    }
  } else {
    st.s2 = 1.0;  // velocities were materialised by the prime pass
    kb = ke;
  }
  st.ke_end = kb * 0.5;
  next_first_half(d, st, kb);
  if (mode == 0 && d.thermostat == 3 && st.gmode == 2) st.gmode = 1;
  if (!(ke == ke) || ke > 1.0e300) st.status = 1;
  st.prime = 0;
  __threadfence();
  st.counter_b = 0;
}

// ---------------------------------------------------------------------------
// fixDrift (MDcode/initialise.c:104-138) after the step, on the momenta at the
// step boundary p = v * s2: P = sum p / N, p -= P; then the next step's first
// half from the new sum p^2 (the reference's next U4 sums the corrected p).
// Two passes over the flagged systems: the mean, then the removal.
__global__ void __launch_bounds__(BLOCK_A) k_drift_sum(View v) {
  __shared__ double sh[BLOCK_A / 32];
  __shared__ int s_last;
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  if (!st.drift) return;
  const SysDesc &d = v.desc[r];
  const int loc = t.y + threadIdx.x;
  const double s2 = st.s2;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (loc < d.n) {
    const int i = d.poff + loc;
    px = __dmul_rn(v.vx[i], s2);
    py = __dmul_rn(v.vy[i], s2);
    pz = __dmul_rn(v.vz[i], s2);
  }
  px = block_sum<BLOCK_A / 32>(px, sh);
  py = block_sum<BLOCK_A / 32>(py, sh);
  pz = block_sum<BLOCK_A / 32>(pz, sh);
  double *part = v.part_o + (size_t)blockIdx.x * OBS_EMAX * OBS_NV;
  if (threadIdx.x == 0) {
    part[0] = px;
    part[1] = py;
    part[2] = pz;
    __threadfence();
    s_last = atomicAdd(&st.counter_d, 1u) == (unsigned)(d.ntile_a - 1);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double P[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < d.ntile_a; b++) {
    const double *pb = v.part_o + (size_t)(d.tile0_a + b) * OBS_EMAX * OBS_NV;
    for (int k = 0; k < 3; k++) P[k] += __ldcg(pb + k);
  }
  for (int k = 0; k < 3; k++) st.drift_m[k] = P[k] / (double)d.n;
  __threadfence();
  st.counter_d = 0;
}

__global__ void __launch_bounds__(BLOCK_A) k_drift_apply(View v) {
  __shared__ double sh[BLOCK_A / 32];
  __shared__ int s_last;
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  if (!st.drift) return;
  const SysDesc &d = v.desc[r];
  const int loc = t.y + threadIdx.x;
  const double s2 = st.s2, mx = st.drift_m[0], my = st.drift_m[1], mz = st.drift_m[2];
  double k2 = 0.0;
  if (loc < d.n) {
    const int i = d.poff + loc;
    const double px = __dadd_rn(__dmul_rn(v.vx[i], s2), -mx);
    const double py = __dadd_rn(__dmul_rn(v.vy[i], s2), -my);
    const double pz = __dadd_rn(__dmul_rn(v.vz[i], s2), -mz);
    v.vx[i] = px;
    v.vy[i] = py;
    v.vz[i] = pz;
    k2 = px * px + py * py + pz * pz;
  }
  k2 = block_sum<BLOCK_A / 32>(k2, sh);
  double *part = v.part_o + (size_t)blockIdx.x * OBS_EMAX * OBS_NV;
  if (threadIdx.x == 0) {
    part[3] = k2;
    __threadfence();
    s_last = atomicAdd(&st.counter_d, 1u) == (unsigned)(d.ntile_a - 1);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double kb = 0.0;
  for (int b = 0; b < d.ntile_a; b++) kb += __ldcg(v.part_o + (size_t)(d.tile0_a + b) * OBS_EMAX * OBS_NV + 3);
  st.s2 = 1.0;
  st.ke_end = kb * 0.5;
  next_first_half(d, st, kb);
  st.drift = 0;
  __threadfence();
  st.counter_d = 0;
}

// ---------------------------------------------------------------------------
// Gaussian isokinetic thermostat (AdvanceTimeNVTGaussOSM, MDcode/time_evolve.c:
// 351-470).  Each half kick p = factor1 (p + factor2 F) takes its factors from
// X1 = sum p.F, X2 = sum F^2 and K0 = sum p^2 over the system:
// alpha = sqrt(X2/K0), zeta0 = -X1/K0, beta = exp(-alpha dt/2),
// gamma = (zeta0 - alpha)/(zeta0 + alpha), factor1 = (1 - gamma)/(beta -
// gamma/beta), factor2 = (1 + gamma - beta - gamma/beta)/((1 - gamma) alpha).
// With F = 0 or p = 0 these are 0/0; the limit (p unchanged) is used there.
__device__ __forceinline__ void gauss_factors(double x1, double x2, double k0, double dt, double &f1,
                                              double &f2) {
  if (!(x2 > 0.0) || !(k0 > 0.0)) {
    f1 = 1.0;
    f2 = 0.0;
    return;
  }
  const double alpha = sqrt(x2 / k0);
  const double zeta0 = -x1 / k0;
  const double beta = exp(-alpha * dt * 0.5);
  const double gamma = (zeta0 - alpha) / (zeta0 + alpha);
  f1 = (1.0 - gamma) / (beta - gamma / beta);
  f2 = (1.0 + gamma - beta - gamma / beta) / ((1.0 - gamma) * alpha);
}

// block sums of one tile's X1, X2, K0 into the tile's partial slot; returns
// (in every thread) whether this block is the system's last (counter_g)
__device__ __forceinline__ bool gauss_block_sums(const View &v, const SysDesc &d, SysState &st, double x1,
                                                 double x2, double k0) {
  __shared__ double sh[BLOCK_A / 32];
  __shared__ int s_last;
  x1 = block_sum<BLOCK_A / 32>(x1, sh);
  x2 = block_sum<BLOCK_A / 32>(x2, sh);
  k0 = block_sum<BLOCK_A / 32>(k0, sh);
  double *part = v.part_o + (size_t)blockIdx.x * OBS_EMAX * OBS_NV;
  if (threadIdx.x == 0) {
    part[0] = x1;
    part[1] = x2;
    part[2] = k0;
    __threadfence();
    s_last = atomicAdd(&st.counter_g, 1u) == (unsigned)(d.ntile_a - 1);
  }
  __syncthreads();
  return s_last != 0;
}

// the system's X1, X2, K0 from the tile partials, in tile order
__device__ __forceinline__ void gauss_totals(const View &v, const SysDesc &d, double &x1, double &x2,
                                             double &k0) {
  __threadfence();
  x1 = x2 = k0 = 0.0;
  for (int b = 0; b < d.ntile_a; b++) {
    const double *pb = v.part_o + (size_t)(d.tile0_a + b) * OBS_EMAX * OBS_NV;
    x1 += __ldcg(pb);
    x2 += __ldcg(pb + 1);
    k0 += __ldcg(pb + 2);
  }
}

// after a step's forces (gmode 1): the sums over the momenta after the first
// half kick and drift and the new forces give the second half kick's factors
__global__ void __launch_bounds__(BLOCK_A) k_gauss_sum(View v) {
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  if (st.gmode != 1) return;
  const SysDesc &d = v.desc[r];
  const int loc = t.y + threadIdx.x;
  double x1 = 0.0, x2 = 0.0, k0 = 0.0;
  if (loc < d.n) {
    const int i = d.poff + loc;
    const double px = v.vx[i], py = v.vy[i], pz = v.vz[i];
    const double fx = v.fx[i], fy = v.fy[i], fz = v.fz[i];
    x1 = px * fx + py * fy + pz * fz;
    x2 = fx * fx + fy * fy + fz * fz;
    k0 = px * px + py * py + pz * pz;
  }
  if (!gauss_block_sums(v, d, st, x1, x2, k0) || threadIdx.x != 0) return;
  gauss_totals(v, d, x1, x2, k0);
  gauss_factors(x1, x2, k0, d.dt, st.ga[0], st.ga[1]);
  __threadfence();
  st.counter_g = 0;
}

// the second half kick (gmode 1) or none (gmode 2: after a host change of the
// momenta, a drift removal or a rescale), then the sums over the momenta at the
// step boundary give the next step's first half kick factors (s1, g1); KE at
// the boundary as the reference reports it (0.5 sum p^2)
__global__ void __launch_bounds__(BLOCK_A) k_gauss_apply(View v) {
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  const int gm = st.gmode;
  if (gm == 0) return;
  const SysDesc &d = v.desc[r];
  const int loc = t.y + threadIdx.x;
  double x1 = 0.0, x2 = 0.0, k0 = 0.0;
  if (loc < d.n) {
    const int i = d.poff + loc;
    double px = v.vx[i], py = v.vy[i], pz = v.vz[i];
    const double fx = v.fx[i], fy = v.fy[i], fz = v.fz[i];
    if (gm == 1) {
      const double f1 = st.ga[0], f2 = st.ga[1];
      px = __dmul_rn(f1, __dadd_rn(px, __dmul_rn(f2, fx)));
      py = __dmul_rn(f1, __dadd_rn(py, __dmul_rn(f2, fy)));
      pz = __dmul_rn(f1, __dadd_rn(pz, __dmul_rn(f2, fz)));
      v.vx[i] = px;
      v.vy[i] = py;
      v.vz[i] = pz;
    }
    x1 = px * fx + py * fy + pz * fz;
    x2 = fx * fx + fy * fy + fz * fz;
    k0 = px * px + py * py + pz * pz;
  }
  if (!gauss_block_sums(v, d, st, x1, x2, k0) || threadIdx.x != 0) return;
  gauss_totals(v, d, x1, x2, k0);
  gauss_factors(x1, x2, k0, d.dt, st.s1, st.g1);
  st.s2 = 1.0;
  st.ke_end = k0 * 0.5;
  if (!(k0 == k0) || k0 > 1.0e300) st.status = 1;
  st.gmode = 0;
  __threadfence();
  st.counter_g = 0;
}

// ---------------------------------------------------------------------------
// active Brownian dynamics, predictor-corrector (thermostat 6,
// advance_time_ActiveBrown_PC, MDcode/time_evolve.c:855-974).  Random forces
// SqrtVariance N(0,1) per component with SqrtVariance = sqrt(2 T^2 / (dt D0))
// (initialise.c:287), the reference's GSL draws replaced by a counter-based
// stream (Philox4x32-10 keyed by the system's seed, counter = particle id and
// step), minus their mean; k_brown_predict moves the particles to the
// predicted positions, force mode 3 evaluates the forces there, and the
// corrector runs in k_kick_drift.
__global__ void __launch_bounds__(BLOCK_A) k_brown_noise(View v) {
  __shared__ double sh[BLOCK_A / 32];
  __shared__ int s_last;
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  const SysDesc &d = v.desc[r];
  SysState &st = v.st[r];
  if (d.thermostat != 6 || st.ramp_left != 0) return;
  const int loc = t.y + threadIdx.x;
  double g[3] = {0.0, 0.0, 0.0};
  if (loc < d.n) {
    const int i = d.poff + loc;
    normals3(d.seed ^ 0x5DEECE66DULL, st.step, v.id[i], g);
    const double sv = sqrt(2.0 * d.T * d.T / (d.dt * 1.0));
    double *s = brown_scratch(v, d);
    for (int k = 0; k < 3; k++) {
      g[k] = sv * g[k];
      s[3 * loc + k] = g[k];
    }
  }
  double *part = v.part_o + (size_t)blockIdx.x * OBS_EMAX * OBS_NV;
  for (int k = 0; k < 3; k++) {
    const double b = block_sum<BLOCK_A / 32>(g[k], sh);
    if (threadIdx.x == 0) part[k] = b;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&st.counter_g, 1u) == (unsigned)(d.ntile_a - 1);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double m[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < d.ntile_a; b++) {
    const double *pb = v.part_o + (size_t)(d.tile0_a + b) * OBS_EMAX * OBS_NV;
    for (int k = 0; k < 3; k++) m[k] += __ldcg(pb + k);
  }
  for (int k = 0; k < 3; k++) st.brown_m[k] = m[k] / (double)d.n;
  __threadfence();
  st.counter_g = 0;
}

// the random forces minus their mean; position and force before the predictor
// kept; predicted positions x + D0ByT ((1 - e) p + c (F_random + F)) / L
// (MDcode/time_evolve.c:885-912, x_u untouched)
__global__ void __launch_bounds__(BLOCK_A) k_brown_predict(View v) {
  const int2 t = v.tiles_a[blockIdx.x];
  const int r = t.x;
  const SysDesc &d = v.desc[r];
  const SysState &st = v.st[r];
  if (d.thermostat != 6 || st.ramp_left != 0) return;
  const int loc = t.y + threadIdx.x;
  if (loc >= d.n) return;
  const int i = d.poff + loc, n = d.n;
  const BrownConst B(d);
  double *s = brown_scratch(v, d);
  double4 pos = v.pos[i];
  const double F[3] = {v.fx[i], v.fy[i], v.fz[i]};
  const double P[3] = {v.vx[i], v.vy[i], v.vz[i]};
  double x[3] = {pos.x, pos.y, pos.z};
  for (int k = 0; k < 3; k++) {
    const double fr = __dadd_rn(s[3 * loc + k], -st.brown_m[k]);
    s[3 * loc + k] = fr;
    s[3 * n + 3 * loc + k] = x[k];
    s[6 * n + 3 * loc + k] = F[k];
    const double dd = B.dx(P[k], __dadd_rn(fr, F[k]));
    x[k] = wrap_unit(__dadd_rn(x[k], __dmul_rn(dd, d.invL)));
  }
  pos.x = x[0];
  pos.y = x[1];
  pos.z = x[2];
  v.pos[i] = pos;
}

// ---------------------------------------------------------------------------
// Berendsen NPT (thermostat 4, advance_time_NPT, MDcode/time_evolve.c:258-348):
// at the start of each step (not during a ramp) the box is rescaled and the
// forces recomputed at the new length (force mode 3) before the kick.
__device__ __forceinline__ bool npt_due(const SysDesc &d, const SysState &st) {
  return d.thermostat == 4 && st.ramp_left == 0;
}

// one thread per system: the pressure from the last forces' virial and
// calculate_temp's inst_T of the momenta at the step boundary (v * s2, sum
// p^2 = s2^2 * 2 ke_end), chi_P = (1 + dt (pressure - P) / tau_P)^0.33333333;
// UpdateBoxForNPT (:823-850) sets DENSITY and inv_L from the length before the
// change, then L *= chi_P (:266-269).  The cell grid stays; a length whose
// reference cell count differs sets status 2.
__global__ void k_npt_box(View v) {
  for (int r = threadIdx.x; r < v.nsys; r += blockDim.x) {
    SysDesc &d = const_cast<SysDesc &>(v.desc[r]);
    SysState &st = v.st[r];
    if (!npt_due(d, st)) continue;
    const double keb = (st.s2 * st.s2) * st.ke_end;
    const double inst = 2.0 * keb / d.dof;
    const double L = d.L;
    const double pressure = d.density * inst + st.virial / (L * L * L);
    const double chi = pow(1.0 + d.dt * (pressure - d.P) / TAU_P, 0.33333333);
    d.density = (double)d.n / (L * L * L);
    d.invL = 1.00 / L;
    const double Ln = chi * L;
    d.L = Ln;
    st.pressure = pressure;
    if (!(Ln > 0.0) || (int)((double)(int)Ln / d.cell_cut) != d.nc) st.status = 2;
  }
}

// host request: remove the mean momentum of system r now (with k_drift_sum and
// k_drift_apply after it)
__global__ void k_flag_drift(View v, int r) {
  if (threadIdx.x == 0) v.st[r].drift = 1;
}

// adjustInitialTemp (MDcode/initialise.c:141-151) for system r, one block:
// the momenta at the step boundary (v * s2) are scaled by sqrt(T / inst_T)
// with inst_T from their sum p^2 (calculate_temp); the new sum sets ke_end and
// the next step's first half.  Ramp (ramp_left > 0, set by k_ramp_begin after
// this): the first ramp step's rescale.
__global__ void __launch_bounds__(1024) k_rescale(View v, int r, double T) {
  __shared__ double sh[32];
  __shared__ double s_xi;
  const SysDesc &d = v.desc[r];
  SysState &st = v.st[r];
  const double s2 = st.s2;
  double k2 = 0.0;
  for (int k = threadIdx.x; k < d.n; k += blockDim.x) {
    const int i = d.poff + k;
    const double px = __dmul_rn(v.vx[i], s2), py = __dmul_rn(v.vy[i], s2), pz = __dmul_rn(v.vz[i], s2);
    v.vx[i] = px;
    v.vy[i] = py;
    v.vz[i] = pz;
    k2 += px * px + py * py + pz * pz;
  }
  k2 = block_sum_dyn(k2, sh);
  if (threadIdx.x == 0) {
    const double inst = 2.0 * (k2 * 0.5) / d.dof;
    s_xi = sqrt(T / inst);
  }
  __syncthreads();
  const double xi = s_xi;
  double k3 = 0.0;
  for (int k = threadIdx.x; k < d.n; k += blockDim.x) {
    const int i = d.poff + k;
    const double px = __dmul_rn(v.vx[i], xi), py = __dmul_rn(v.vy[i], xi), pz = __dmul_rn(v.vz[i], xi);
    v.vx[i] = px;
    v.vy[i] = py;
    v.vz[i] = pz;
    k3 += px * px + py * py + pz * pz;
  }
  k3 = block_sum_dyn(k3, sh);
  if (threadIdx.x == 0) {
    st.s2 = 1.0;
    st.ke_end = k3 * 0.5;
    next_first_half(d, st, k3);
  }
}

// arm a temperature ramp of K steps on system r starting at target T0 (the
// momenta already rescaled to it by k_rescale), changing by dT per step
__global__ void k_ramp_begin(View v, int r, double T0, double dT, double T_end, long long K) {
  if (threadIdx.x != 0) return;
  const SysDesc &d = v.desc[r];
  SysState &st = v.st[r];
  st.ramp_T = T0;
  st.ramp_dT = dT;
  st.ramp_end = T_end;
  st.ramp_left = K;
  st.ramp_real = K;
  next_first_half(d, st, 2.0 * st.ke_end);
}

// lengthen system r's armed ramp to `total` steps; the steps after the ramp
// itself rescale to its final temperature (lets systems whose ramps differ in
// length finish together inside one engine)
__global__ void k_ramp_extend(View v, int r, long long total) {
  if (threadIdx.x != 0) return;
  SysState &st = v.st[r];
  if (st.ramp_left > 0 && total > st.ramp_left) {
    if (st.ramp_real <= 0) st.ramp_T = st.ramp_end;
    st.ramp_left = total;
  }
}

// GetFccGrid (MDcode/initialise.c:34-101) placement of system r's particles on
// the reference's near-cubic grid: particle k goes to grid site site[k] of
// troot^3 sites (troot = the smallest integer with troot^3 >= N), with the
// reference's arithmetic (the y and z coordinates use floating divisions);
// types and momenta come from the host.  Reads the staged upload of
// acg_set_lattice and writes the staged x = xu for k_load.
__global__ void k_lattice(View v, int r, int troot) {
  const SysDesc &d = v.desc[r];
  double *s = v.stage_d + 9 * (size_t)d.poff;
  const int *site = v.stage_i + 2 * (size_t)d.poff + (size_t)d.n;  // act tags follow at k_load time
  const double dr = 1.0 / (double)troot;  // LENGTH / troot_n
  const int t2 = troot * troot;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < d.n; k += gridDim.x * blockDim.x) {
    const int i = site[k];
    const double X = dr * (double)((i % t2) % troot);
    const double Y = dr * (double)(i % t2) / (double)troot;
    const double Z = dr * (double)(i / (double)t2);
    s[3 * k] = X;
    s[3 * k + 1] = Y;
    s[3 * k + 2] = Z;
    s[3 * (size_t)d.n + 3 * k] = X;
    s[3 * (size_t)d.n + 3 * k + 1] = Y;
    s[3 * (size_t)d.n + 3 * k + 2] = Z;
  }
}

// 1/x for x in the pair range (0.3 < x < 7): the hardware estimate
// (rcp.approx.ftz.f64) refined by two Newton-Raphson steps y += y (1 - x y),
// each squaring the relative error, to within an ulp of the rounded quotient
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// 1/x in FP32 from the hardware estimate (a Newton step on it changed the
// measured force error by nothing: the FP32 rounding of r^2 dominates)
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct PairAccF {
  float fx, fy, fz, pe, vir;
};

// the sums of one list chunk (at most two FP32 terms in each of fa, fb) moved
// into the FP64 sums: the per-particle force is a sum of large terms of both
// signs, whose FP32 rounding would otherwise grow with the list; and the FP64
// sum of these chunk values is exact in practice, so it does not depend on how
// the chunks are split over threads
__device__ __forceinline__ void flush_chunk(PairAccF &fa, PairAccF &fb, PairAcc &a) {
  a.fx += (double)(fa.fx + fb.fx);
  a.fy += (double)(fa.fy + fb.fy);
  a.fz += (double)(fa.fz + fb.fz);
  a.pe += (double)(fa.pe + fb.pe);
  a.vir += (double)(fa.vir + fb.vir);
  fa = PairAccF{0.f, 0.f, 0.f, 0.f, 0.f};
  fb = PairAccF{0.f, 0.f, 0.f, 0.f, 0.f};
}

// FP32 pair constants of particle i against a partner of type 0 and of type 1:
// 1/sigma^2, 4 eps and 8 eps/sigma^2 (MDcode/cell_list+forces.c:19-20)
struct PairParamsF {
  float is2[2], e4[2], ge[2];
  __device__ __forceinline__ explicit PairParamsF(int ti) {
#pragma unroll
    for (int tj = 0; tj < 2; tj++) {
      const int tp = ti + tj;
      is2[tj] = tp == 0 ? 1.0f : (tp == 1 ? 1.5625f : (float)(1.0 / (0.88 * 0.88)));
      e4[tj] = tp == 0 ? 4.0f : (tp == 1 ? 6.0f : 2.0f);
      ge[tj] = 2.0f * e4[tj] * is2[tj];
    }
  }
  // for separations counted in units of u: 1/sigma^2 u^2 and 8 eps/sigma^2 u,
  // so forces come out in absolute units and the virial in units of 1/u
  __device__ __forceinline__ PairParamsF(int ti, float u) : PairParamsF(ti) {
#pragma unroll
    for (int tj = 0; tj < 2; tj++) {
      is2[tj] *= u * u;
      ge[tj] *= u;
    }
  }
};

// FP32 pair term: U = 4 eps (s^12 - s^6) + C0 + C2 (r/sigma)^2 and its radial
// force factor, written as s6 (s6 - 1) and s6 (6 s6 - 3) s2
__device__ __forceinline__ void pair_f32(PairAccF &a, float dx, float dy, float dz, const PairParamsF &P,
                                         bool tj) {
  const float is2 = tj ? P.is2[1] : P.is2[0];
  const float dr2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rs2 = dr2 * is2;
  // evaluated for every entry and masked (no divergent branch): beyond the cut
  // the factors are zero and each sum gains exactly nothing
  const bool in = rs2 < (float)KA_RC2;
  const float e4 = in ? (tj ? P.e4[1] : P.e4[0]) : 0.0f, ge = in ? (tj ? P.ge[1] : P.ge[0]) : 0.0f;
  const float s2 = rcp_approx(rs2);
  const float s6 = s2 * s2 * s2;
  a.pe = fmaf(e4, fmaf(s6, s6, -s6) + fmaf((float)KA_C2, rs2, (float)KA_C0), a.pe);
  const float g = ge * fmaf(s6 * fmaf(6.0f, s6, -3.0f), s2, -(float)KA_C2);
  a.fx = fmaf(g, dx, a.fx);
  a.fy = fmaf(g, dy, a.fy);
  a.fz = fmaf(g, dz, a.fz);
  a.vir = fmaf(g, dr2, a.vir);
}

// stage 2: forces + second kick.  mode 0 = step; 1 = prime (forces at the
// current positions for systems flagged `prime`, pending velocity scale
// applied, thermostat first half recomputed); 2 = forces only, velocities and
// thermostat untouched (calculate_forces)
template <int TPP, int PREC>
__global__ void __launch_bounds__(512) k_force_kick(View v, int mode, int tile_base) {
  __shared__ double sh[32];
  __shared__ int s_last;
  const int2 t = v.tiles_b[blockIdx.x];
  const int r = t.x;
  SysState &st = v.st[r];
  if (mode == 1 && !st.prime) return;
  const SysDesc &d = v.desc[r];
  if (mode == 3 && !pre_due(d, st)) return;
  const int grp = threadIdx.x / TPP, lane = threadIdx.x % TPP;
  const int loc = t.y + grp;
  const bool valid = loc < d.n;
  const int i = d.poff + (valid ? loc : 0);
  const double L = d.L, L2 = d.L * d.L;
  PairAcc a = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (valid) {
    const double4 pi = v.pos[i];
    const int ti = (int)pi.w;
    const PairParamsF PF(ti);
    const int nn = v.nbn[i];
    if (nn >= 0) {
      // four list entries per lane per iteration (one 16-byte load; rows are
      // 16-byte aligned and padded to maxnb, entries past nn are not used)
      const int4 *row4 = reinterpret_cast<const int4 *>(v.nbl + (size_t)i * v.maxnb);
      const int nb4 = (nn + 3) >> 2;
      // each chunk's slots are loaded one iteration ahead, so the positions it
      // gathers wait for one L2 round trip, not two
      int4 jn = lane < nb4 ? __ldg(row4 + lane) : make_int4(0, 0, 0, 0);
      for (int b = lane; b < nb4; b += TPP) {
        const int4 jj = jn;
        if (b + TPP < nb4) jn = __ldg(row4 + b + TPP);
        const int k0 = 4 * b;
        const bool v1 = k0 + 1 < nn, v2 = k0 + 2 < nn, v3 = k0 + 3 < nn;
        const double4 p0 = v.pos[jj.x];
        const double4 p1 = v1 ? v.pos[jj.y] : pi;
        const double4 p2 = v2 ? v.pos[jj.z] : pi;
        const double4 p3 = v3 ? v.pos[jj.w] : pi;
        if (PREC == 0) {
          pair_fp64(a, pi, ti, p0, L, L2);
          if (v1) pair_fp64(a, pi, ti, p1, L, L2);
          if (v2) pair_fp64(a, pi, ti, p2, L, L2);
          if (v3) pair_fp64(a, pi, ti, p3, L, L2);
        } else {
          // separations from the FP64 minimum image, the pair terms in FP32
          // summed per chunk of four and moved into the FP64 sums (as the
          // cell-group and whole-box kernels do); an unused entry (past nn)
          // is the particle itself at separation zero, masked by the cut test
          const float Lf = (float)L;
          PairAccF fa = {0.f, 0.f, 0.f, 0.f, 0.f}, fb = {0.f, 0.f, 0.f, 0.f, 0.f};
          const double4 pj[4] = {p0, p1, p2, p3};
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const float dx = (float)min_image(pi.x - pj[e].x) * Lf;
            const float dy = (float)min_image(pi.y - pj[e].y) * Lf;
            const float dz = (float)min_image(pi.z - pj[e].z) * Lf;
            const float dr2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            // separation zero (the particle itself in an unused entry) gains nothing
            if (dr2 > 0.0f) pair_f32(e & 1 ? fb : fa, dx, dy, dz, PF, (int)pj[e].w != 0);
          }
          flush_chunk(fa, fb, a);
        }
      }
    } else {
      // neighbour-list overflow: scan the cells around the cell of the last
      // rebuild (every pair within the cut is there since displacements stay
      // below the skin)
      const int nc = d.nc, c = v.cellof[i];
      const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
      const int lo = stencil_lo(nc), hi = stencil_hi(nc);
      for (int oz = lo; oz <= hi; oz++)
        for (int oy = lo; oy <= hi; oy++)
          for (int ox = lo; ox <= hi; ox++) {
            int c2 = wrap_cell(cx + ox, nc) + wrap_cell(cy + oy, nc) * nc + wrap_cell(cz + oz, nc) * nc * nc;
            const int s0 = d.poff + v.cstart[d.coff + c2], m = v.ccount[d.coff + c2];
            for (int k = lane; k < m; k += TPP) {
              const int j = s0 + k;
              if (j == i) continue;
              const double4 pj = v.pos[j];
              if (PREC == 0)
                pair_fp64(a, pi, ti, pj, L, L2);
              else
                pair_fp32(a, pi, ti, pj, L, L2);
            }
          }
    }
  }
#pragma unroll
  for (int o = TPP / 2; o > 0; o >>= 1) {
    a.fx += __shfl_xor_sync(0xffffffffu, a.fx, o);
    a.fy += __shfl_xor_sync(0xffffffffu, a.fy, o);
    a.fz += __shfl_xor_sync(0xffffffffu, a.fz, o);
    a.pe += __shfl_xor_sync(0xffffffffu, a.pe, o);
    a.vir += __shfl_xor_sync(0xffffffffu, a.vir, o);
  }
  double ke = 0.0, va = 0.0, pe = 0.0, vir = 0.0;
  if (valid && lane == 0) {
    double fx = a.fx, fy = a.fy, fz = a.fz;
    const int ai = v.act[i];
    if (ai >= 0) {  // active force (MDcode/cell_list+forces.c:207-218)
      const char4 k = v.kdir[d.aoff + ai];
      const double kx = (double)k.x, ky = (double)k.y, kz = (double)k.z;
      fx += d.f0 * kx;
      fy += d.f0 * ky;
      fz += d.f0 * kz;
      va = d.f0 * (kx * v.ux[i] + ky * v.uy[i] + kz * v.uz[i]);
    }
    v.fx[i] = fx;
    v.fy[i] = fy;
    v.fz[i] = fz;
    double px, py, pz;
    if (mode >= 2) {
      px = py = pz = 0.0;
    } else if (mode == 0 && (d.thermostat == 3 || (d.thermostat == 6 && st.ramp_left == 0))) {
      // Gaussian: the kick waits for k_gauss_sum; Brownian: no kick
      px = v.vx[i];
      py = v.vy[i];
      pz = v.vz[i];
    } else if (mode == 0 && d.thermostat == 5 && st.ramp_left == 0) {  // U2PropagatorNPT
      const double f1 = st.u2[0], f2 = st.u2[1];
      px = __dadd_rn(__dmul_rn(v.vx[i], f1), __dmul_rn(__dmul_rn(f2, fx), d.half_dt));
      py = __dadd_rn(__dmul_rn(v.vy[i], f1), __dmul_rn(__dmul_rn(f2, fy), d.half_dt));
      pz = __dadd_rn(__dmul_rn(v.vz[i], f1), __dmul_rn(__dmul_rn(f2, fz), d.half_dt));
    } else if (mode == 0) {  // U2 (MDcode/time_evolve.c:558-567)
      px = __dadd_rn(v.vx[i], __dmul_rn(fx, d.half_dt));
      py = __dadd_rn(v.vy[i], __dmul_rn(fy, d.half_dt));
      pz = __dadd_rn(v.vz[i], __dmul_rn(fz, d.half_dt));
    } else {
      const double s2 = st.s2;
      px = __dmul_rn(v.vx[i], s2);
      py = __dmul_rn(v.vy[i], s2);
      pz = __dmul_rn(v.vz[i], s2);
    }
    if (mode < 2) {
      v.vx[i] = px;
      v.vy[i] = py;
      v.vz[i] = pz;
    }
    ke = px * px + py * py + pz * pz;
    pe = a.pe;
    vir = a.vir;
  }
  pe = block_sum_dyn(pe, sh);
  vir = block_sum_dyn(vir, sh);
  ke = block_sum_dyn(ke, sh);
  va = block_sum_dyn(va, sh);
  if (threadIdx.x == 0) {
    v.part_b[tile_base + blockIdx.x] = make_double4(pe, vir, ke, va);
    __threadfence();
    s_last = atomicAdd(&st.counter_b, 1u) == (unsigned)(d.ntile_b - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  finalize_system(v, r, mode);
}

// ---------------------------------------------------------------------------
// Cell-group kernels (boxes with >= 3 cells per side).  One block per group
// of up to 2 x 2 x 2 cells.  The union of the group cells' neighbour cells
// (up to 4 x 4 x 4) is staged in shared memory in the group's frame: each
// union cell is shifted by its periodic image, so every pair within the cut
// has its minimum image without a per-pair test (cells are at least as wide
// as the list cut and there are >= 3 per side).  Neighbour lists hold 16-bit
// staged indices (bit 15: the neighbour's type), stored per group transposed
// (entry k of centre particle t at k*M + t) so a warp's loads are contiguous.
struct GroupStage {
  int nU, nC, Q, M;
  int ustart[MAX_UNION];     // first slot of each union cell
  int upre[MAX_UNION + 1];   // staged offset of each union cell
  int ushift[MAX_UNION];     // periodic image shifts, 2 bits per dimension
  double ucen[3][MAX_UNION]; // centre of each union cell's box cell, reduced units
  int cu[8];                 // union index of each centre cell
  int cpre[9];               // centre offset of each centre cell
};


__device__ void group_prologue(const View &v, const SysDesc &d, const GroupGeom &G, GroupStage &S) {
  const int nc = d.nc;
  const int nux = G.nu[0], nuy = G.nu[1], nuz = G.nu[2];
  const int nU = nux * nuy * nuz;
  __shared__ int cnt_u[MAX_UNION];
  if (threadIdx.x < nU) {
    const int t = threadIdx.x;
    const int u[3] = {t % nux, (t / nux) % nuy, t / (nux * nuy)};
    int c = 0, mul = 1, sh = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int ci = G.lo[k] + u[k];
      const int s = ci < 0 ? -1 : (ci >= nc ? 1 : 0);
      const int cw = wrap_cell(ci, nc);
      c += cw * mul;
      mul *= nc;
      sh |= (s + 1) << (2 * k);
      S.ucen[k][t] = ((double)cw + 0.5) / (double)nc;
    }
    S.ustart[t] = d.poff + v.cstart[d.coff + c];
    cnt_u[t] = v.ccount[d.coff + c];
    S.ushift[t] = sh;
  }
  __syncthreads();
  // inclusive scan of the (<= 64) union-cell counts over the first two warps
  // (every thread of the block reaches every barrier below)
  __shared__ int wtot;
  int x = 0;
  if (threadIdx.x < 64) {
    const int l = threadIdx.x & 31;
    x = threadIdx.x < nU ? cnt_u[threadIdx.x] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (threadIdx.x == 31) wtot = x;
  }
  __syncthreads();
  if (threadIdx.x < 64) {
    const int incl = x + (threadIdx.x >= 32 ? wtot : 0);
    if (threadIdx.x < nU) S.upre[threadIdx.x + 1] = incl;
    if (threadIdx.x == 0) S.upre[0] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    S.Q = S.upre[nU];
    S.nU = nU;
    int k = 0, m = 0;
    for (int uz = 1; uz <= nuz - 2; uz++)
      for (int uy = 1; uy <= nuy - 2; uy++)
        for (int ux = 1; ux <= nux - 2; ux++) {
          const int t = ux + uy * nux + uz * nux * nuy;
          S.cu[k] = t;
          S.cpre[k] = m;
          m += cnt_u[t];
          k++;
        }
    S.cpre[k] = m;
    S.nC = k;
    S.M = m;
  }
  __syncthreads();
}

__device__ __forceinline__ double shift_of(int code, int k) { return (double)(((code >> (2 * k)) & 3) - 1); }

// staged coordinate of a particle of union cell u along dimension k: the
// image of its wrapped coordinate nearest to its cell's centre (a particle that
// crossed the box edge since the rebuild keeps a continuous coordinate; it has
// moved far less than half a box), plus the union cell's image shift, relative
// to the group centre, in absolute units
__device__ __forceinline__ double staged_coord(const GroupStage &S, const GroupGeom &G, int u, int k,
                                               double x, double L) {
  const double img = x + rint(S.ucen[k][u] - x);
  return ((img + shift_of(S.ushift[u], k)) - G.org[k]) * L;
}

// centre particle t -> (centre cell k, slot, staged index)
__device__ __forceinline__ void group_centre(const GroupStage &S, int t, int &k, int &slot, int &qself) {
  k = 0;
  while (S.cpre[k + 1] <= t) k++;
  const int w = t - S.cpre[k];
  slot = S.ustart[S.cu[k]] + w;
  qself = S.upre[S.cu[k]] + w;
}

__device__ __forceinline__ uint16_t *group_list(const View &v, const SysDesc &d, int g) {
  return reinterpret_cast<uint16_t *>(v.nbl) + 2 * (size_t)d.poff * v.maxnb +
         (size_t)v.gstart[d.goff + g] * v.maxnb;
}

// list entry k of centre particle t, chunks of four entries per particle
// (entry k at ((k/4)*M + t)*4 + k%4): the force kernel reads four entries with
// one 8-byte load and a warp's loads are contiguous
__device__ __forceinline__ size_t group_entry(int k, int t, int M) {
  return ((size_t)(k >> 2) * M + t) * 4 + (k & 3);
}

// 16-bit list entries of one particle, packed four to a chunk in a 64-bit
// shift register (the newest entry enters at the top, so after four the
// first is in the low bits); whole chunks are stored as uint2 at
// chunk * stride + row
// the next index of a block-shared counter for the calling warp (lane 0 takes
// it, the warp shares it)
__device__ __forceinline__ int warp_next(int &counter) {
  int o = 0;
  if ((threadIdx.x & 31) == 0) o = atomicAdd(&counter, 1);
  return __shfl_sync(0xffffffffu, o, 0);
}

struct ListWriter {
  unsigned lo = 0u, hi = 0u;
  int n = 0;
  __device__ __forceinline__ void add(unsigned code, uint2 *lst, size_t stride, int row, int maxnb) {
    lo = __funnelshift_r(lo, hi, 16);
    hi = (hi >> 16) | (code << 16);
    n++;
    if ((n & 3) == 0 && n <= maxnb) lst[(size_t)((n >> 2) - 1) * stride + row] = make_uint2(lo, hi);
  }
  // the last, partial chunk: its k pending entries sit in the top 16k bits
  __device__ __forceinline__ void finish(uint2 *lst, size_t stride, int row, int maxnb, unsigned pad = 0u) {
    const int k = n & 3;
    if (k && n <= maxnb) {
      unsigned long long p = (((unsigned long long)hi << 32) | lo) >> (16 * (4 - k));
      for (int e = k; e < 4; e++) p |= (unsigned long long)pad << (16 * e);
      lst[(size_t)(n >> 2) * stride + row] = make_uint2((unsigned)p, (unsigned)(p >> 32));
    }
  }
};

// Lists of a cell group: the neighbour cells in (dz, dy, dx) order, each
// cell's particles in staged order.  Each union cell's staged run is padded
// to a multiple of four with far-away dummies; the staged .w holds the list
// code (unpadded staged index | type << 15).  The last chunk of four entries
// is padded with the force kernel's far-away slot (index gcap).  The force
// tiles split a small system's groups into gsplit contiguous runs of centre
// particles; each run's block stages the union and builds the lists of its
// run with one warp per particle (the lanes test 32 candidates at a time and
// a ballot appends the accepted ones: a short chain per particle, for the
// latency of a few blocks).  An unsplit group (a large system, whose blocks
// fill the GPU) takes one lane per particle, which issues fewer instructions
// in all.
// one centre particle's list built by the whole warp (staged index ps, union
// cell cu, list row t): the lanes test 32 staged candidates at a time over the
// 27 neighbour cells in (dz, dy, dx) order and a ballot appends the accepted
// ones in staged order; the last chunk is padded with `pad`.  Returns the
// entry count (entries past maxnb are not stored).
__device__ __forceinline__ int warp_list_particle(const float4 *stg, const int *pre4, int nux, int nuy, int cu,
                                                  int ps, const float lc[3], uint16_t *lst, int t, int M, int maxnb,
                                                  unsigned pad) {
  const int lane = threadIdx.x & 31;
  const int ux = cu % nux, uy = (cu / nux) % nuy, uz = cu / (nux * nuy);
  const float4 fi = stg[ps];
  const int ti = __float_as_int(fi.w) >> 15;
  // cut for a partner of type 0 / 1 (the sum of the two types indexes lc)
  const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
  int n = 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int u2 = (ux + dx) + (uy + dy) * nux + (uz + dz) * nux * nuy;
        const int q1 = pre4[u2 + 1];
        for (int qb = pre4[u2]; qb < q1; qb += 32) {
          const int q = qb + lane;
          bool ok = false;
          int code = 0;
          if (q < q1) {
            const float4 fj = stg[q];
            const float ex = fi.x - fj.x, ey = fi.y - fj.y, ez = fi.z - fj.z;
            const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            code = __float_as_int(fj.w);
            ok = r2 < ((code >> 15) ? c1 : c0) && q != ps;
          }
          const unsigned bal = __ballot_sync(0xffffffffu, ok);
          if (ok) {
            const int k = n + __popc(bal & ((1u << lane) - 1u));
            if (k < maxnb) lst[group_entry(k, t, M)] = (uint16_t)(code & 0xffff);
          }
          n += __popc(bal);
        }
      }
  if (n <= maxnb && lane < ((4 - (n & 3)) & 3)) lst[group_entry(n + lane, t, M)] = (uint16_t)pad;
  return n;
}

__global__ void __launch_bounds__(BLOCK_G) k_build_list_groups(View v) {
  extern __shared__ float4 stg[];
  __shared__ GroupStage S;
  __shared__ int pre4[MAX_UNION + 1];
  __shared__ int s_over;  // next overflow particle to hand out
  const int2 tile = v.tiles_g[blockIdx.x];
  const int r = tile.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  const int g = tile.y / d.gsplit, part = tile.y - g * d.gsplit;
  GroupGeom G;
  group_geom(g, d.nc, d.ng, G);
  group_prologue(v, d, G, S);
  const int Q = S.Q, M = S.M, nux = G.nu[0], nuy = G.nu[1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int maxnb = v.maxnb;
  const int run = (M + d.gsplit - 1) / d.gsplit, t_lo = part * run, t_hi = min(M, t_lo + run);
  if (Q <= v.gcap) {
    if (threadIdx.x == 0) {
      int m = 0;
      for (int u = 0; u < S.nU; u++) {
        pre4[u] = m;
        m += (S.upre[u + 1] - S.upre[u] + 3) & ~3;
      }
      pre4[S.nU] = m;
      s_over = 0;
    }
    __syncthreads();
    const double L = d.L;
    // padded staged index q over the whole union, two loads in flight per
    // thread; each union cell's run is padded to a multiple of four
    const int P4 = pre4[S.nU];
    for (int q0 = threadIdx.x; q0 < P4; q0 += 2 * blockDim.x) {
      double4 p[2];
      int uu[2], kk[2];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int q = q0 + e * blockDim.x;
        uu[e] = -1;
        kk[e] = 0;
        if (q < P4) {
          const int u = union_of(pre4, S.nU, q);
          const int k = q - pre4[u];
          uu[e] = u;
          kk[e] = k;
          if (k < S.upre[u + 1] - S.upre[u]) p[e] = v.pos_s[S.ustart[u] + k];
        }
      }
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int u = uu[e], k = kk[e], q = q0 + e * blockDim.x;
        if (u < 0) continue;
        float4 f;
        if (k < S.upre[u + 1] - S.upre[u]) {
          f.x = (float)staged_coord(S, G, u, 0, p[e].x, L);
          f.y = (float)staged_coord(S, G, u, 1, p[e].y, L);
          f.z = (float)staged_coord(S, G, u, 2, p[e].z, L);
          f.w = __int_as_float((S.upre[u] + k) | ((int)p[e].w << 15));
        } else {
          f = make_float4(1e18f, 1e18f, 1e18f, __int_as_float(0));
        }
        stg[q] = f;
      }
    }
    __syncthreads();
    if (d.gsplit > 1) {
      float lc[3];
      for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * (1.0 + 1e-5));
      uint16_t *lst = group_list(v, d, g);
      for (int t = t_lo + warp; t < t_hi; t += nwarps) {
        int kc, i, qs;
        group_centre(S, t, kc, i, qs);
        const int cu = S.cu[kc];
        const int n = warp_list_particle(stg, pre4, nux, nuy, cu, pre4[cu] + (t - S.cpre[kc]), lc, lst, t, M, maxnb,
                                         (unsigned)v.gcap);
        if (lane == 0) {
          if (n > maxnb) {
            v.nbn[i] = -1;
            atomicAdd(&v.st[r].overflow, 1);
          } else {
            v.nbn[i] = n;
          }
        }
      }
    } else {
      // an unsplit group (many groups per system): one warp per centre cell,
      // one lane per particle, every lane testing the same staged candidate
      // (a shared-memory broadcast); each lane packs its entries into a 64-bit
      // register and stores whole 4-entry chunks (the same lists: cells in
      // (dz, dy, dx) order, staged order inside a cell)
      float lc[3];
      for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * (1.0 + 1e-5));
      const bool one_cut = lc[0] == lc[1] && lc[1] == lc[2];
      uint2 *lst = reinterpret_cast<uint2 *>(group_list(v, d, g));
      // the first 32 particles of each centre cell; a cell's further
      // particles (a dense cell) are listed below, one warp each, so that no
      // warp sweeps the 27 cells twice while the others wait at the barrier
      for (int kc = warp; kc < S.nC; kc += nwarps) {
        const int cu = S.cu[kc];
        const int m = S.cpre[kc + 1] - S.cpre[kc];
        const int ux = cu % nux, uy = (cu / nux) % nuy, uz = cu / (nux * nuy);
        {
          const int w = lane;
          const bool valid = w < m;
          const int t = S.cpre[kc] + w, ps = pre4[cu] + w;
          const float4 fi = valid ? stg[ps] : make_float4(-1e18f, -1e18f, -1e18f, __int_as_float(0));
          const int ti = __float_as_int(fi.w) >> 15;
          // cut for a partner of type 0 / 1 (the sum of the two types indexes lc)
          const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
          ListWriter lw;
          for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dx = -1; dx <= 1; dx++) {
                const int u2 = (ux + dx) + (uy + dy) * nux + (uz + dz) * nux * nuy;
                const int q1 = pre4[u2 + 1];
                for (int q = pre4[u2]; q < q1; q += 4) {
                  int code[4];
                  bool ok[4];
#pragma unroll
                  for (int e = 0; e < 4; e++) {
                    const float4 fj = stg[q + e];
                    const float ex = fi.x - fj.x, ey = fi.y - fj.y, ez = fi.z - fj.z;
                    const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                    code[e] = __float_as_int(fj.w);
                    const float cut = one_cut ? c0 : ((code[e] >> 15) ? c1 : c0);
                    ok[e] = valid && r2 < cut && q + e != ps;
                  }
#pragma unroll
                  for (int e = 0; e < 4; e++)
                    if (ok[e]) lw.add((unsigned)code[e] & 0xffffu, lst, M, t, maxnb);
                }
              }
          if (valid) {
            lw.finish(lst, M, t, maxnb, (unsigned)v.gcap);
            const int n = lw.n;
            const int i = S.ustart[cu] + w;
            if (n > maxnb) {
              v.nbn[i] = -1;
              atomicAdd(&v.st[r].overflow, 1);
            } else {
              v.nbn[i] = n;
            }
          }
        }
      }
      int nover = 0;
      for (int k = 0; k < S.nC; k++) nover += max(0, S.cpre[k + 1] - S.cpre[k] - 32);
      uint16_t *lst16 = group_list(v, d, g);
      // handed out as warps come free (a particle's list does not depend on
      // which warp builds it)
      for (int o = warp_next(s_over); o < nover; o = warp_next(s_over)) {
        int k = 0, oo = o;
        for (;;) {
          const int ex = max(0, S.cpre[k + 1] - S.cpre[k] - 32);
          if (oo < ex) break;
          oo -= ex;
          k++;
        }
        const int w = 32 + oo, cu = S.cu[k], t = S.cpre[k] + w;
        const int n = warp_list_particle(stg, pre4, nux, nuy, cu, pre4[cu] + w, lc, lst16, t, M, maxnb,
                                         (unsigned)v.gcap);
        if (lane == 0) {
          const int i = S.ustart[cu] + w;
          if (n > maxnb) {
            v.nbn[i] = -1;
            atomicAdd(&v.st[r].overflow, 1);
          } else {
            v.nbn[i] = n;
          }
        }
      }
    }
  } else {
    // the union does not fit in shared memory: the force kernel scans cells
    for (int t = t_lo + threadIdx.x; t < t_hi; t += blockDim.x) {
      int kc, i, qs;
      group_centre(S, t, kc, i, qs);
      v.nbn[i] = -1;
      atomicAdd(&v.st[r].overflow, 1);
    }
  }
  // no barrier: the copy reads and writes no shared memory and no list, so a
  // warp done with its lists starts it while the others finish theirs
  for (int t = t_lo + threadIdx.x; t < t_hi; t += blockDim.x) {
    int kc, i, qs;
    group_centre(S, t, kc, i, qs);
    copy_back(v, i);
  }
}

// FP64 pair constants of particle i against a partner of type 0 and of type 1:
// 1/sigma^2, 4 eps and 8 eps/sigma^2 (MDcode/cell_list+forces.c:19-20)
struct PairParamsD {
  double is2[2], e4[2], ge[2];
  __device__ __forceinline__ explicit PairParamsD(int ti) {
#pragma unroll
    for (int tj = 0; tj < 2; tj++) {
      const int tp = ti + tj;
      is2[tj] = tp == 0 ? 1.0 : (tp == 1 ? 1.5625 : 1.0 / (0.88 * 0.88));
      e4[tj] = tp == 0 ? 4.0 : (tp == 1 ? 6.0 : 2.0);
      ge[tj] = 2.0 * e4[tj] * is2[tj];
    }
  }
};

// FP64 pair term on a separation already in the minimum image (absolute
// units): U = 4 eps (s^12 - s^6) + C0 + C2 (r/sigma)^2 and the radial force
// factor 8 eps/sigma^2 (s6 (6 s6 - 3) s2 - C2), s2 = sigma^2/r^2
// (MDcode/cell_list+forces.c:174-203), written in fused multiply-adds
__device__ __forceinline__ void pair_f64(PairAcc &a, double dx, double dy, double dz, const PairParamsD &P,
                                         bool tj) {
  const double is2 = tj ? P.is2[1] : P.is2[0];
  const double dr2 = fma(dx, dx, fma(dy, dy, dz * dz));
  const double rs2 = dr2 * is2;
  // evaluated for every entry and masked, as the FP32 term: beyond the cut
  // (s2 <= 0.16, every product finite) the factors are zero and each sum
  // gains an exact zero, so the sums are those of a branch on the cut; with
  // no branch the four pairs of a list chunk interleave
  const bool in = rs2 < KA_RC2;
  const double e4 = in ? (tj ? P.e4[1] : P.e4[0]) : 0.0, ge = in ? (tj ? P.ge[1] : P.ge[0]) : 0.0;
  const double s2 = rcp_nr(rs2);
  const double s6 = s2 * s2 * s2;
  a.pe = fma(e4, fma(s6, s6, -s6) + fma(KA_C2, rs2, KA_C0), a.pe);
  const double g = ge * fma(s6 * fma(6.0, s6, -3.0), s2, -KA_C2);
  a.fx = fma(g, dx, a.fx);
  a.fy = fma(g, dy, a.fy);
  a.fz = fma(g, dz, a.fz);
  a.vir = fma(g, dr2, a.vir);
}

// launch-bounds occupancy targets of the cell-group force kernel (blocks per
// SM).  FP64: 2, no spills (the masked pair term interleaves the four pairs of
// a chunk; at 4 blocks, 64 registers, it spilled: N = 2.56e5 force 143 -> 129
// us, N = 1e5 unchanged at 60 us); FP32: 4
#ifndef ACG_FORCE_MINB64
#define ACG_FORCE_MINB64 2
#endif
#ifndef ACG_FORCE_MINB32
#define ACG_FORCE_MINB32 4
#endif

// per-particle end of the force pass: active force (MDcode/cell_list+forces.c:
// 207-218), forces stored, then the second half kick U2 (mode 0,
// MDcode/time_evolve.c:558-567) or the pending thermostat scale (mode 1),
// and the block's pe / virial / KE / active-virial partial sums
__device__ __forceinline__ void particle_epilogue(const View &v, const SysDesc &d, const SysState &st, int i,
                                                  int mode, const PairAcc &a, double &pe, double &vir,
                                                  double &ke, double &va) {
  const int ai = v.act[i];
  double fx = a.fx, fy = a.fy, fz = a.fz;
  if (ai >= 0) {
    const char4 kk = v.kdir[d.aoff + ai];
    const double kx = (double)kk.x, ky = (double)kk.y, kz = (double)kk.z;
    fx += d.f0 * kx;
    fy += d.f0 * ky;
    fz += d.f0 * kz;
    va += d.f0 * (kx * v.ux[i] + ky * v.uy[i] + kz * v.uz[i]);
  }
  v.fx[i] = fx;
  v.fy[i] = fy;
  v.fz[i] = fz;
  if (mode < 2) {
    // p = a v + b F: the second half kick U2 (a = 1, b = dt/2,
    // MDcode/time_evolve.c:558-567), U2PropagatorNPT (a = f1, b = f2 dt/2,
    // :721-735), none (Gaussian isokinetic: after k_gauss_sum; Brownian), or
    // the pending thermostat scale (mode 1: a = s2, b = 0)
    // (the force term is left out where b = 0, so a non-finite force of a
    // system that holds no state yet does not reach its momenta)
    double a = 1.0, b = d.half_dt;
    if (mode == 1) {
      a = st.s2;
      b = 0.0;
    } else if (d.thermostat == 3 || d.thermostat == 6) {
      b = 0.0;
    } else if (d.thermostat == 5 && st.ramp_left == 0) {
      a = st.u2[0];
      b = st.u2[1] * d.half_dt;
    }
    double px = __dmul_rn(v.vx[i], a), py = __dmul_rn(v.vy[i], a), pz = __dmul_rn(v.vz[i], a);
    if (b != 0.0) {
      px = __dadd_rn(px, __dmul_rn(fx, b));
      py = __dadd_rn(py, __dmul_rn(fy, b));
      pz = __dadd_rn(pz, __dmul_rn(fz, b));
    }
    v.vx[i] = px;
    v.vy[i] = py;
    v.vz[i] = pz;
    ke += px * px + py * py + pz * pz;
  }
  pe += a.pe;
  vir += a.vir;
}

// block sums stored at the block's partial slot of the system; the last block
// of the system to finish (a counter, no waiting) finalises it
__device__ __forceinline__ void end_force_block(const View &v, int r, int slot, int mode, double pe, double vir,
                                                double ke, double va) {
  __shared__ double sh[32];
  __shared__ int s_last;
  const SysDesc &d = v.desc[r];
  SysState &st = v.st[r];
  pe = block_sum_dyn(pe, sh);
  vir = block_sum_dyn(vir, sh);
  ke = block_sum_dyn(ke, sh);
  va = block_sum_dyn(va, sh);
  if (threadIdx.x == 0) {
    v.part_b[d.tile0_b + slot] = make_double4(pe, vir, ke, va);
    __threadfence();
    s_last = atomicAdd(&st.counter_b, 1u) == (unsigned)(d.ntile_b - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  finalize_system(v, r, mode);
}

template <int TPP, int PREC>
__global__ void __launch_bounds__(BLOCK_G, PREC ? ACG_FORCE_MINB32 : ACG_FORCE_MINB64) k_force_groups(View v, int mode) {
  // FP64: three double arrays; FP32: float4 {hi x, y, z, lo x} + float2
  // {lo y, lo z} (hi = the coordinate rounded to float, lo = the remainder),
  // 24 bytes per staged particle either way
  extern __shared__ __align__(16) unsigned char gsm_raw[];
  double *gsm = reinterpret_cast<double *>(gsm_raw);
  // one slot past the union (index gcap) holds a far-away dummy that pads
  // the last list chunk of every particle, so chunks need no length tests
  const int gs = v.gcap + 1;
  double *sx = gsm, *sy = gsm + gs, *sz = gsm + 2 * gs;
  float4 *shi = reinterpret_cast<float4 *>(gsm_raw);
  float2 *slo = reinterpret_cast<float2 *>(gsm_raw + 16 * (size_t)gs);
  __shared__ GroupStage S;
  const int2 tile = v.tiles_g[blockIdx.x];
  const int r = tile.x;
  const SysState &st = v.st[r];
  if (mode == 1 && !st.prime) return;
  const SysDesc &d = v.desc[r];
  if (mode == 3 && !pre_due(d, st)) return;
  // tile.y = group * gsplit + part: this block takes the part-th contiguous
  // run of the group's centre particles
  const int g = tile.y / d.gsplit, part = tile.y - g * d.gsplit;
  GroupGeom G;
  group_geom(g, d.nc, d.ng, G);
  group_prologue(v, d, G, S);
  const int Q = S.Q, M = S.M;
  const bool staged = Q <= v.gcap;
  const double L = d.L;
  if (staged) {
    if (threadIdx.x == 0) {
      if (PREC == 0) {
        sx[v.gcap] = 1e18;
        sy[v.gcap] = 1e18;
        sz[v.gcap] = 1e18;
      } else {
        shi[v.gcap] = make_float4(1e18f, 1e18f, 1e18f, 0.0f);
        slo[v.gcap] = make_float2(0.0f, 0.0f);
      }
    }
    // staged index q over the whole union, SG loads in flight per thread
    // (the union's cells are runs of consecutive slots; every block of the
    // grid stages at once at the start, so nothing else hides the latency)
    constexpr int SG = 4;
    for (int q0 = threadIdx.x; q0 < Q; q0 += SG * blockDim.x) {
      double4 p[SG];
      int uu[SG];
#pragma unroll
      for (int e = 0; e < SG; e++) {
        const int q = q0 + e * blockDim.x;
        uu[e] = -1;
        if (q < Q) {
          const int u = union_of(S.upre, S.nU, q);
          uu[e] = u;
          p[e] = v.pos[S.ustart[u] + (q - S.upre[u])];
        }
      }
#pragma unroll
      for (int e = 0; e < SG; e++) {
        const int u = uu[e], q = q0 + e * blockDim.x;
        if (u < 0) continue;
        const double cx = staged_coord(S, G, u, 0, p[e].x, L);
        const double cy = staged_coord(S, G, u, 1, p[e].y, L);
        const double cz = staged_coord(S, G, u, 2, p[e].z, L);
        if (PREC == 0) {
          sx[q] = cx;
          sy[q] = cy;
          sz[q] = cz;
        } else {
          const float hx = (float)cx, hy = (float)cy, hz = (float)cz;
          shi[q] = make_float4(hx, hy, hz, (float)(cx - (double)hx));
          slo[q] = make_float2((float)(cy - (double)hy), (float)(cz - (double)hz));
        }
      }
    }
  }
  __syncthreads();
  const uint16_t *lst = staged ? group_list(v, d, g) : nullptr;
  double pe = 0.0, vir = 0.0, ke = 0.0, va = 0.0;
  const int lane = threadIdx.x % TPP, nper = blockDim.x / TPP;
  const int run = (M + d.gsplit - 1) / d.gsplit, t_lo = part * run, t_hi = min(M, t_lo + run);
  // rounds over the centre particles: TPP threads per particle, all threads of
  // a round take part in the shuffle reduction
  for (int t0 = t_lo; t0 < t_hi; t0 += nper) {
    const int t = t0 + threadIdx.x / TPP;
    const bool valid = t < t_hi;
    int kc = 0, i = 0, qs = 0;
    if (valid) group_centre(S, t, kc, i, qs);
    const double4 pi = valid ? v.pos[i] : make_double4(0, 0, 0, 0);
    const int ti = (int)pi.w;
    const int nn = valid ? v.nbn[i] : 0;
    PairAcc a = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (PREC == 1 && valid && staged && nn >= 0) {
      const float4 hi = shi[qs];
      const float2 li = slo[qs];
      const PairParamsF P(ti);
      const int nch = (nn + 3) >> 2;
      const uint2 *lp = reinterpret_cast<const uint2 *>(lst) + t;
      PairAccF fa = {0.f, 0.f, 0.f, 0.f, 0.f}, fb = {0.f, 0.f, 0.f, 0.f, 0.f};
      uint2 w = lane < nch ? __ldg(lp + (size_t)lane * M) : make_uint2(0u, 0u);
      for (int c = lane; c < nch; c += TPP) {
        const uint2 wn = c + TPP < nch ? __ldg(lp + (size_t)(c + TPP) * M) : make_uint2(0u, 0u);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int code = ((e < 2 ? w.x : w.y) >> (16 * (e & 1))) & 0xffff;
          const int q = code & 0x7fff;
          const float4 hj = shi[q];
          const float2 lj = slo[q];
          const float dx = (hi.x - hj.x) + (hi.w - hj.w);
          const float dy = (hi.y - hj.y) + (li.x - lj.x);
          const float dz = (hi.z - hj.z) + (li.y - lj.y);
          pair_f32(e & 1 ? fb : fa, dx, dy, dz, P, code >> 15);
        }
        flush_chunk(fa, fb, a);
        w = wn;
      }
    } else if (PREC == 0 && valid && staged && nn >= 0) {
      const double xi = sx[qs], yi = sy[qs], zi = sz[qs];
      const PairParamsD P(ti);
      const int nch = (nn + 3) >> 2;
      const uint2 *lp = reinterpret_cast<const uint2 *>(lst) + t;
      // list chunks are loaded two iterations ahead (an L2 round trip is
      // longer than one chunk's arithmetic); two accumulators break the
      // dependency chains of consecutive pairs
      PairAcc b = {0.0, 0.0, 0.0, 0.0, 0.0};
      uint2 w = lane < nch ? __ldg(lp + (size_t)lane * M) : make_uint2(0u, 0u);
      uint2 wn = lane + TPP < nch ? __ldg(lp + (size_t)(lane + TPP) * M) : make_uint2(0u, 0u);
      for (int c = lane; c < nch; c += TPP) {
        const uint2 wnn = c + 2 * TPP < nch ? __ldg(lp + (size_t)(c + 2 * TPP) * M) : make_uint2(0u, 0u);
        const int e0 = w.x & 0xffff, e1 = w.x >> 16, e2 = w.y & 0xffff, e3 = w.y >> 16;
        {
          const int q = e0 & 0x7fff;
          pair_f64(a, xi - sx[q], yi - sy[q], zi - sz[q], P, e0 >> 15);
        }
        {
          const int q = e1 & 0x7fff;
          pair_f64(b, xi - sx[q], yi - sy[q], zi - sz[q], P, e1 >> 15);
        }
        {
          const int q = e2 & 0x7fff;
          pair_f64(a, xi - sx[q], yi - sy[q], zi - sz[q], P, e2 >> 15);
        }
        {
          const int q = e3 & 0x7fff;
          pair_f64(b, xi - sx[q], yi - sy[q], zi - sz[q], P, e3 >> 15);
        }
        w = wn;
        wn = wnn;
      }
      a.fx += b.fx;
      a.fy += b.fy;
      a.fz += b.fz;
      a.pe += b.pe;
      a.vir += b.vir;
    } else if (valid) {
      // list overflow or oversized union: scan the neighbour cells directly
      const int nc = d.nc, c = v.cellof[i];
      const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
      const double L2 = L * L;
      for (int oz = -1; oz <= 1; oz++)
        for (int oy = -1; oy <= 1; oy++)
          for (int ox = -1; ox <= 1; ox++) {
            const int c2 = wrap_cell(cx + ox, nc) + wrap_cell(cy + oy, nc) * nc + wrap_cell(cz + oz, nc) * nc * nc;
            const int s0 = d.poff + v.cstart[d.coff + c2], m = v.ccount[d.coff + c2];
            for (int k = lane; k < m; k += TPP) {
              const int j = s0 + k;
              if (j == i) continue;
              const double4 pj = v.pos[j];
              if (PREC == 0)
                pair_fp64(a, pi, ti, pj, L, L2);
              else
                pair_fp32(a, pi, ti, pj, L, L2);
            }
          }
    }
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
      a.fx += __shfl_xor_sync(0xffffffffu, a.fx, o);
      a.fy += __shfl_xor_sync(0xffffffffu, a.fy, o);
      a.fz += __shfl_xor_sync(0xffffffffu, a.fz, o);
      a.pe += __shfl_xor_sync(0xffffffffu, a.pe, o);
      a.vir += __shfl_xor_sync(0xffffffffu, a.vir, o);
    }
    if (!valid || lane != 0) continue;
    particle_epilogue(v, d, st, i, mode, a, pe, vir, ke, va);
  }
  end_force_block(v, r, tile.y, mode, pe, vir, ke, va);
}

// ---------------------------------------------------------------------------
// whole-box kernels: systems with 2 to 4 cells per side (N up to ~3.5k at
// density 1.2).  A 2x2x2 cell group of such a box would stage the whole box
// (and, at 3 cells per side, part of it twice) for each of its 8 groups; here
// every block stages the system once and handles d.cpb cells of it (1 to
// BOX_CELLS, chosen per engine for about two blocks per SM).
// List entries are system-local slot indices (| type << 15); entry k of slot
// s sits in chunk k/4 at uint2 index (k/4)*N + s.

__device__ __forceinline__ uint16_t *box_list(const View &v, const SysDesc &d) {
  return reinterpret_cast<uint16_t *>(v.nbl) + 2 * (size_t)d.poff * v.maxnb;
}

// 32-bit fixed point of a reduced coordinate (x * 2^32, two's-complement
// wrap): the difference of two is the minimum-image separation, exactly
__device__ __forceinline__ int fixed32(double x) {
  return (int)(unsigned)(unsigned long long)__double2ll_rz(x * 4294967296.0);
}

// per-system cell starts (system-local slots) and the per-cell runs padded to
// a multiple of four, for <= 64 cells
__device__ __forceinline__ void box_cells(const View &v, const SysDesc &d, int *cst, int *pre4) {
  const int nce = d.ncell;
  __shared__ int wtot;
  int x = 0;
  if (threadIdx.x < MAX_BOX_CELLS) {
    const int t = threadIdx.x, l = t & 31;
    if (t < nce) {
      cst[t] = v.cstart[d.coff + t];
      x = (v.ccount[d.coff + t] + 3) & ~3;
    }
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (t == 31) wtot = x;
  }
  __syncthreads();
  if (threadIdx.x < MAX_BOX_CELLS) {
    const int incl = x + (threadIdx.x >= 32 ? wtot : 0);
    if (threadIdx.x < nce) pre4[threadIdx.x + 1] = incl;
    if (threadIdx.x == 0) {
      pre4[0] = 0;
      cst[nce] = d.n;
    }
  }
  __syncthreads();
}

// lists of the particles of cell c of a whole box (one warp; lanes are the
// particles of the cell, in rounds of 32) against the staged system: the 27
// neighbour cells with their periodic image shifts (at 2 cells per side a cell
// appears under two shifts, of which at most one can be in range since L > 2 x
// the list cut), candidates in slot order within each cell
__device__ __forceinline__ void box_list_cell(const View &v, const SysDesc &d, int r, const float4 *xstg,
                                              const int *cst, const int *pre4, int c, int lane, int round0,
                                              int rstep) {
  const int nc = d.nc, n = d.n;
  const double iL2 = 1.0 / (d.L * d.L);
  float lc[3];
  for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * iL2 * (1.0 + 1e-5));
  const bool one_cut = lc[0] == lc[1] && lc[1] == lc[2];
  uint2 *lst = reinterpret_cast<uint2 *>(box_list(v, d));
  const int maxnb = v.maxnb;
  {

    const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
    const int m = cst[c + 1] - cst[c];
    for (int w0 = 32 * round0; w0 < m; w0 += 32 * rstep) {
      const int w = w0 + lane;
      const bool valid = w < m;
      const int sl = cst[c] + w, ps = pre4[c] + w;
      // a lane past the cell's particles gets NaN coordinates: it passes no test
      const float nan = __int_as_float(0x7fc00000);
      const float4 fi = valid ? xstg[ps] : make_float4(nan, nan, nan, __int_as_float(0));
      const int ti = __float_as_int(fi.w) >> 15;
      const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
      ListWriter lw;
      if (nc == 2) {
        // two cells per side: every cell neighbours every other under two
        // images, so test each particle once with the minimum image instead
        // of 27 images of 8 cells
        const int q1 = pre4[d.ncell];
        for (int q = 0; q < q1; q += 4) {
          int code[4];
          bool ok[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const float4 fj = xstg[q + e];
            float ex = fi.x - fj.x, ey = fi.y - fj.y, ez = fi.z - fj.z;
            ex -= rintf(ex);
            ey -= rintf(ey);
            ez -= rintf(ez);
            const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            code[e] = __float_as_int(fj.w);
            const float cut = one_cut ? c0 : ((code[e] >> 15) ? c1 : c0);
            ok[e] = valid && r2 < cut && q + e != ps;
          }
#pragma unroll
          for (int e = 0; e < 4; e++)
            if (ok[e]) lw.add((unsigned)code[e] & 0xffffu, lst, n, sl, maxnb);
        }
      }
      for (int dz = -1; dz <= 1 && nc > 2; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            const int ax = cx + dx, ay = cy + dy, az = cz + dz;
            const int sx = ax < 0 ? -1 : (ax >= nc ? 1 : 0), sy = ay < 0 ? -1 : (ay >= nc ? 1 : 0),
                      sz = az < 0 ? -1 : (az >= nc ? 1 : 0);
            const int c2 = (ax - sx * nc) + (ay - sy * nc) * nc + (az - sz * nc) * nc * nc;
            // candidate image x_j + s: compare x_i - s with x_j
            const float xi = fi.x - (float)sx, yi = fi.y - (float)sy, zi = fi.z - (float)sz;
            const int q1 = pre4[c2 + 1];
            for (int q = pre4[c2]; q < q1; q += 4) {
              int code[4];
              bool ok[4];
#pragma unroll
              for (int e = 0; e < 4; e++) {
                const float4 fj = xstg[q + e];
                const float ex = xi - fj.x, ey = yi - fj.y, ez = zi - fj.z;
                const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                code[e] = __float_as_int(fj.w);
                const float cut = one_cut ? c0 : ((code[e] >> 15) ? c1 : c0);
                ok[e] = valid && r2 < cut && q + e != ps;
              }
#pragma unroll
              for (int e = 0; e < 4; e++)
                if (ok[e]) lw.add((unsigned)code[e] & 0xffffu, lst, n, sl, maxnb);
            }
          }
      if (valid) {
        lw.finish(lst, n, sl, maxnb);
        const int nn = lw.n;
        const int i = d.poff + sl;
        if (nn > maxnb) {
          v.nbn[i] = -1;
          atomicAdd(&v.st[r].overflow, 1);
        } else {
          v.nbn[i] = nn;
        }
      }
    }
  }
}

// the system in cell order (after the permutation) as float4 {reduced x, y, z,
// list code}, each cell's run padded to a multiple of four with NaN dummies
__device__ __forceinline__ void box_stage_list(const View &v, const SysDesc &d, float4 *xstg, const int *cst,
                                               const int *pre4) {
  const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int c = threadIdx.x >> 5; c < d.ncell; c += nwarps) {
    const int s0 = cst[c], m = cst[c + 1] - s0, p0 = pre4[c], m4 = pre4[c + 1] - p0;
    for (int k = lane; k < m4; k += 32) {
      float4 f;
      if (k < m) {
        const double4 p = v.pos_s[d.poff + s0 + k];
        f = make_float4((float)p.x, (float)p.y, (float)p.z, __int_as_float((s0 + k) | ((int)p.w << 15)));
      } else {
        // padding: NaN coordinates fail every distance test
        const float nan = __int_as_float(0x7fc00000);
        f = make_float4(nan, nan, nan, __int_as_float(0));
      }
      xstg[p0 + k] = f;
    }
  }
}

// lists of up to 8 particles of cell c of a whole box (particles w0.. of the
// cell), four lanes per particle: the four lanes of a particle test four
// consecutive staged candidates at a time and a ballot ranks the partners
// found, so the entries keep the staged order (the 27 neighbour cells with
// their periodic image shifts, slot order within a cell; at 2 cells per side
// every particle of the box once under the minimum image).  The lists are the
// ones one lane per particle would write, in a quarter of the serial chain.
__device__ __forceinline__ void box_list_group(const View &v, const SysDesc &d, int r, const float4 *xstg,
                                               const int *cst, const int *pre4, int c, int w0, int lane) {
  const int nc = d.nc, n = d.n;
  const double iL2 = 1.0 / (d.L * d.L);
  float lc[3];
  for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * iL2 * (1.0 + 1e-5));
  uint16_t *lst = box_list(v, d);
  const int maxnb = v.maxnb;
  const int sub = lane & 3, grp = lane >> 2;
  const int m = cst[c + 1] - cst[c];
  const int w = w0 + grp;
  const bool valid = w < m;
  const int sl = cst[c] + w, ps = pre4[c] + w;
  // a lane past the cell's particles gets NaN coordinates: it passes no test
  const float nan = __int_as_float(0x7fc00000);
  const float4 fi = valid ? xstg[ps] : make_float4(nan, nan, nan, __int_as_float(0));
  const int ti = __float_as_int(fi.w) >> 15;
  const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
  const unsigned below = (1u << sub) - 1u;
  int cnt = 0;
  // one staged candidate per lane; the run [q0, q1) is a multiple of four long
  auto scan = [&](int q0, int q1, float xi, float yi, float zi, bool wrap) {
    for (int q = q0 + sub; q < q1; q += 4) {
      const float4 fj = xstg[q];
      float ex = xi - fj.x, ey = yi - fj.y, ez = zi - fj.z;
      if (wrap) {
        ex -= rintf(ex);
        ey -= rintf(ey);
        ez -= rintf(ez);
      }
      const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
      const int code = __float_as_int(fj.w);
      const bool ok = valid && r2 < ((code >> 15) ? c1 : c0) && q != ps;
      const unsigned gm = (__ballot_sync(0xffffffffu, ok) >> (4 * grp)) & 15u;
      if (ok) {
        const int k = cnt + __popc(gm & below);
        if (k < maxnb) lst[((size_t)(k >> 2) * n + sl) * 4 + (k & 3)] = (uint16_t)(code & 0xffff);
      }
      cnt += __popc(gm);
    }
  };
  if (nc == 2) {
    // two cells per side: every cell neighbours every other under two
    // images, so each particle is tested once with the minimum image
    scan(0, pre4[d.ncell], fi.x, fi.y, fi.z, true);
  } else {
    const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int ax = cx + dx, ay = cy + dy, az = cz + dz;
          const int sx = ax < 0 ? -1 : (ax >= nc ? 1 : 0), sy = ay < 0 ? -1 : (ay >= nc ? 1 : 0),
                    sz = az < 0 ? -1 : (az >= nc ? 1 : 0);
          const int c2 = (ax - sx * nc) + (ay - sy * nc) * nc + (az - sz * nc) * nc * nc;
          // candidate image x_j + s: compare x_i - s with x_j
          scan(pre4[c2], pre4[c2 + 1], fi.x - (float)sx, fi.y - (float)sy, fi.z - (float)sz, false);
        }
  }
  if (valid && sub == 0) {
    const int i = d.poff + sl;
    if (cnt > maxnb) {
      v.nbn[i] = -1;
      atomicAdd(&v.st[r].overflow, 1);
    } else {
      v.nbn[i] = cnt;
    }
  }
}

// Lists of a whole box from list sub-cells (d.msub per side, side >= half the
// widest list cut): a partner is at most two sub-cells away on each axis, so the
// candidates of a particle are the 5 x 5 x 5 sub-cells around its own, rows of
// sub-cells that are contiguous in sub-cell order (a row that crosses the box
// edge is two runs with their image shifts) -- about a quarter of the volume of
// the 27 reference cells of a small box.
//
// k_sort_sub puts each rebuilding system in sub-cell order (in memory); the
// warps of the list blocks take one particle each (engines with few such
// particles) or bricks of 2 x 2 x d.bz sub-cells, one lane per particle.
__device__ __forceinline__ int subcell_of(double x, int m) { return min(max((int)(x * (double)m), 0), m - 1); }

// lists of the particles of brick B (2 x 2 x d.bz sub-cells), one lane per
// particle in rounds of 32: every lane tests the same candidate (a broadcast
// load of the sorted system) from the union of the brick's sub-cells' 5 x 5 x 5
// neighbourhoods,
// rows of up to 6 sub-cells contiguous in sub-cell order.  Where the union is
// wider than the box (5 sub-cells per side) a sub-cell comes under two image
// shifts, of which at most one can be in range (L > 2 x the list cut).
__device__ __forceinline__ void box_list_particle(const View &v, const SysDesc &d, int r, const float4 *xs,
                                                  const int *sst, int ps, int lane);

__device__ __forceinline__ void box_list_brick(const View &v, const SysDesc &d, int r, const float4 *xs,
                                               const int *sst, int B, int lane) {
  const int m = d.msub, bz = d.bz, n = d.n;
  const int nbx = (m + 1) >> 1;
  const int Bx = B % nbx, By = (B / nbx) % nbx, Bz = B / (nbx * nbx);
  const int x0 = 2 * Bx, x1 = min(x0 + 2, m), y0 = 2 * By, y1 = min(y0 + 2, m), z0 = bz * Bz,
            z1 = min(z0 + bz, m);
  const double iL2 = 1.0 / (d.L * d.L);
  float lc[3];
  for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * iL2 * (1.0 + 1e-5));
  uint2 *lst = reinterpret_cast<uint2 *>(box_list(v, d));
  const int maxnb = v.maxnb;
  const float nan = __int_as_float(0x7fc00000);
  int total = 0;
  for (int z = z0; z < z1; z++)
    for (int y = y0; y < y1; y++) {
      const int row = m * (y + m * z);
      total += sst[row + x1] - sst[row + x0];
    }
  // the brick's first 32 particles, one lane each; the others (a dense
  // brick) one warp each below, so the warp does not sweep the brick's
  // neighbourhood a second time for a few lanes
  {
    // this lane's particle: entry k of the brick's runs (z, y) of x0..x1-1
    int k = lane, ps = -1;
    for (int z = z0; z < z1; z++)
      for (int y = y0; y < y1; y++) {
        const int row = m * (y + m * z);
        const int q0 = sst[row + x0], len = sst[row + x1] - q0;
        if (ps < 0) {
          if (k < len) ps = q0 + k;
          else k -= len;
        }
      }
    const bool valid = ps >= 0;
    // a lane past the brick's particles gets NaN coordinates: it passes no test
    const float4 fi = valid ? xs[ps] : make_float4(nan, nan, nan, __int_as_float(0));
    const int codei = __float_as_int(fi.w);
    const int sl = codei & 0x7fff, ti = codei >> 15;
    const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
    ListWriter lw;
    auto run = [&](int q0, int q1, float xi, float yi, float zi) {
      for (int q = q0; q < q1; q += 4) {
        int code[4];
        bool ok[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int qe = q + e;
          const float4 fj = qe < q1 ? __ldg(xs + qe) : make_float4(nan, nan, nan, __int_as_float(0));
          const float ex = xi - fj.x, ey = yi - fj.y, ez = zi - fj.z;
          const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
          code[e] = __float_as_int(fj.w);
          ok[e] = r2 < ((code[e] >> 15) ? c1 : c0) && qe != ps;
        }
#pragma unroll
        for (int e = 0; e < 4; e++)
          if (ok[e]) lw.add((unsigned)code[e] & 0xffffu, lst, n, sl, maxnb);
      }
    };
    for (int zz = z0 - 2; zz < z1 + 2; zz++) {
      const int sz = zz < 0 ? -1 : (zz >= m ? 1 : 0), az = zz - sz * m;
      for (int yy = y0 - 2; yy < y1 + 2; yy++) {
        const int sy = yy < 0 ? -1 : (yy >= m ? 1 : 0), ay = yy - sy * m;
        const int row = m * (ay + m * az);
        // candidate image x_j + s: compare x_i - s with x_j
        const float yi = fi.y - (float)sy, zi = fi.z - (float)sz;
        int xa = x0 - 2;
        const int xb = x1 + 2;
        if (xa < 0) {
          run(sst[row + m + xa], sst[row + m], fi.x + 1.0f, yi, zi);
          xa = 0;
        }
        if (xb > m) {
          run(sst[row + xa], sst[row + m], fi.x, yi, zi);
          run(sst[row], sst[row + xb - m], fi.x - 1.0f, yi, zi);
        } else {
          run(sst[row + xa], sst[row + xb], fi.x, yi, zi);
        }
      }
    }
    if (valid) {
      lw.finish(lst, n, sl, maxnb);
      const int i = d.poff + sl;
      if (lw.n > maxnb) {
        v.nbn[i] = -1;
        atomicAdd(&v.st[r].overflow, 1);
      } else {
        v.nbn[i] = lw.n;
      }
    }
  }
  // the same lists (the sub-cells within two of the particle's own, rows in
  // (z, y) order, increasing unwrapped x): the brick's neighbourhood holds
  // them, and candidates farther than two sub-cells are beyond every cut
  for (int k1 = 32; k1 < total; k1++) {
    int k = k1, ps = -1;
    for (int z = z0; z < z1; z++)
      for (int y = y0; y < y1; y++) {
        const int row = m * (y + m * z);
        const int q0 = sst[row + x0], len = sst[row + x1] - q0;
        if (ps < 0) {
          if (k < len) ps = q0 + k;
          else k -= len;
        }
      }
    box_list_particle(v, d, r, xs, sst, ps, lane);
  }
}

// One warp per particle of a whole-box system with list sub-cells: the
// particle at position ps of the sub-cell order scans the sub-cells within two
// of its own (5 x 5 x 5 with m >= 5 per side: each once), rows in (z, y)
// order and each row's x range in increasing unwrapped x (periodic images
// split it into runs), 32 candidates per ballot; the accepted ones are
// appended in that order.  List entries are system-local slots | type << 15,
// in 4-entry chunks at uint2 index chunk * n + slot.
__device__ __forceinline__ void box_list_particle(const View &v, const SysDesc &d, int r, const float4 *xs,
                                                  const int *sst, int ps, int lane) {
  const int m = d.msub, n = d.n;
  // the particle's sub-cell: the last c with sst[c] <= ps
  int lo = 0, hi = m * m * m - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sst[mid] <= ps) lo = mid;
    else hi = mid - 1;
  }
  const int sx = lo % m, sy = (lo / m) % m, sz = lo / (m * m);
  const double iL2 = 1.0 / (d.L * d.L);
  float lc[3];
  for (int k = 0; k < 3; k++) lc[k] = (float)(lcut2_of(d, k) * iL2 * (1.0 + 1e-5));
  uint16_t *lst = reinterpret_cast<uint16_t *>(box_list(v, d));
  const int maxnb = v.maxnb;
  const float4 fi = xs[ps];
  const int codei = __float_as_int(fi.w);
  const int sl = codei & 0x7fff, ti = codei >> 15;
  const float c0 = ti == 0 ? lc[0] : lc[1], c1 = ti == 0 ? lc[1] : lc[2];
  int cnt = 0;
  auto run = [&](int q0, int q1, float xi, float yi, float zi) {
    for (int qb = q0; qb < q1; qb += 32) {
      const int q = qb + lane;
      bool ok = false;
      int code = 0;
      if (q < q1) {
        const float4 fj = __ldg(xs + q);
        const float ex = xi - fj.x, ey = yi - fj.y, ez = zi - fj.z;
        const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
        code = __float_as_int(fj.w);
        ok = r2 < ((code >> 15) ? c1 : c0) && q != ps;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const int k = cnt + __popc(bal & ((1u << lane) - 1u));
        if (k < maxnb) lst[(((size_t)(k >> 2) * n + sl) << 2) + (k & 3)] = (uint16_t)(code & 0xffff);
      }
      cnt += __popc(bal);
    }
  };
  for (int zz = sz - 2; zz <= sz + 2; zz++) {
    const int wz = zz < 0 ? -1 : (zz >= m ? 1 : 0), az = zz - wz * m;
    for (int yy = sy - 2; yy <= sy + 2; yy++) {
      const int wy = yy < 0 ? -1 : (yy >= m ? 1 : 0), ay = yy - wy * m;
      const int row = m * (ay + m * az);
      // candidate image x_j + w: compare x_i - w with x_j
      const float yi = fi.y - (float)wy, zi = fi.z - (float)wz;
      int xa = sx - 2;
      const int xb = sx + 3;
      if (xa < 0) {
        run(sst[row + m + xa], sst[row + m], fi.x + 1.0f, yi, zi);
        xa = 0;
      }
      if (xb > m) {
        run(sst[row + xa], sst[row + m], fi.x, yi, zi);
        run(sst[row], sst[row + xb - m], fi.x - 1.0f, yi, zi);
      } else {
        run(sst[row + xa], sst[row + xb], fi.x, yi, zi);
      }
    }
  }
  // the rest of the last chunk written as 0 (the force loop stops at the count)
  if (cnt <= maxnb && lane < ((4 - (cnt & 3)) & 3))
    lst[(((size_t)((cnt + lane) >> 2) * n + sl) << 2) + ((cnt + lane) & 3)] = 0;
  if (lane == 0) {
    const int i = d.poff + sl;
    if (cnt > maxnb) {
      v.nbn[i] = -1;
      atomicAdd(&v.st[r].overflow, 1);
    } else {
      v.nbn[i] = cnt;
    }
  }
}

// one block per whole-box system with list sub-cells (rebuilding systems
// only): the system in sub-cell order into xsub (reduced x, y, z as float, the
// list code slot | type << 15) with the sub-cell starts in ssub.  A counting
// sort in shared memory; members of a sub-cell end in slot order, so the order
// does not depend on the atomics.
__global__ void __launch_bounds__(BLOCK_SORT) k_sort_sub(View v) {
  extern __shared__ int ssm[];
  const int r = blockIdx.x;
  if (!v.st[r].rebuild) return;
  const SysDesc &d = v.desc[r];
  if (!d.box || d.msub < 5) return;
  const int n = d.n, m = d.msub, M3 = m * m * m;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int *fill = ssm;                                             // [M3]
  int *sst = fill + M3;                                        // [M3 + 1]
  uint16_t *key = reinterpret_cast<uint16_t *>(sst + M3 + 1);  // sub-cell of slot s
  uint16_t *ord = key + n;                                     // slot at sorted position (unordered in a sub-cell)
  const double4 *pp = v.pos_s + d.poff;
  float4 *xs = v.xsub + d.poff;
  for (int k = threadIdx.x; k < M3; k += blockDim.x) fill[k] = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    const double4 p = pp[s];
    const int k = subcell_of(p.x, m) + m * (subcell_of(p.y, m) + m * subcell_of(p.z, m));
    key[s] = (uint16_t)k;
    atomicAdd(&fill[k], 1);
  }
  __syncthreads();
  {
    // exclusive scan of the counts: a run of sub-cells per thread, then warps
    __shared__ int wsum[32];
    const int per = (M3 + blockDim.x - 1) / blockDim.x;
    const int k0 = min((int)threadIdx.x * per, M3), k1 = min(k0 + per, M3);
    int loc = 0;
    for (int k = k0; k < k1; k++) loc += fill[k];
    int incl = loc;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; w++) before += wsum[w];
    int run = before + incl - loc;
    for (int k = k0; k < k1; k++) {
      const int c = fill[k];
      sst[k] = run;
      fill[k] = 0;
      run += c;
    }
    if (threadIdx.x == blockDim.x - 1) sst[M3] = run;
    __syncthreads();
  }
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    const int k = key[s];
    ord[sst[k] + atomicAdd(&fill[k], 1)] = (uint16_t)s;
  }
  __syncthreads();
  // final place of a member: its sub-cell's start + the members of lower slot
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int s = ord[q], k = key[s];
    const int q0 = sst[k], q1 = sst[k + 1];
    int rank = 0;
    for (int t = q0; t < q1; t++) rank += ord[t] < s;
    const double4 p = pp[s];
    xs[q0 + rank] = make_float4((float)p.x, (float)p.y, (float)p.z, __int_as_float(s | ((int)p.w << 15)));
  }
  int *gst = v.ssub + d.soff;
  for (int k = threadIdx.x; k <= M3; k += blockDim.x) gst[k] = sst[k];
}


// list bricks of a whole-box system with list sub-cells
__device__ __forceinline__ int bricks_of(const SysDesc &d) {
  const int nbx = (d.msub + 1) >> 1;
  return nbx * nbx * ((d.msub + d.bz - 1) / d.bz);
}

// one block: the whole-box systems with list sub-cells that rebuild this step,
// in system order, with the running count of their work items (particles
// with box_warp, else bricks), so the list build can spread them evenly over
// its warps: rbs[0] systems, rbs[1] items, then (system, first item) pairs
__global__ void __launch_bounds__(BLOCK_COMPACT) k_rebuild_compact(View v) {
  __shared__ int wk[32], wb[32];
  __shared__ int base_k, base_b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) base_k = base_b = 0;
  __syncthreads();
  for (int r0 = 0; r0 < v.nsys; r0 += blockDim.x) {
    const int r = r0 + threadIdx.x;
    int f = 0, nb = 0;
    if (r < v.nsys) {
      const SysDesc &d = v.desc[r];
      if (v.st[r].rebuild && d.box && d.msub >= 5) {
        f = 1;
        nb = v.box_warp ? d.n : bricks_of(d);
      }
    }
    // block-wide exclusive scans of the flags and brick counts
    int kf = f, kb = nb;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, kf, o), z = __shfl_up_sync(0xffffffffu, kb, o);
      if (lane >= o) {
        kf += y;
        kb += z;
      }
    }
    if (lane == 31) {
      wk[warp] = kf;
      wb[warp] = kb;
    }
    __syncthreads();
    int bk = base_k, bb = base_b;
    for (int w = 0; w < warp; w++) {
      bk += wk[w];
      bb += wb[w];
    }
    if (f) {
      const int k = bk + kf - 1;
      v.rbs[2 + 2 * k] = r;
      v.rbs[3 + 2 * k] = bb + kb - nb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < nw; w++) {
        base_k += wk[w];
        base_b += wb[w];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    v.rbs[0] = base_k;
    v.rbs[1] = base_b;
  }
}

// lists of whole boxes, each tile shared by LIST_SPLIT blocks: the bricks of
// all systems with list sub-cells that rebuild go round all warps of the grid
// (k_rebuild_compact lists them), so the few systems that rebuild in a step
// spread evenly over the SMs; a system without list sub-cells has the work
// items (cell, 8 particles) of each tile go round the tile's LIST_SPLIT x 8
// warps, each block staging the system once.
__global__ void __launch_bounds__(BLOCK_X) k_build_list_box(View v) {
  extern __shared__ float4 xstg[];
  __shared__ int cst[MAX_BOX_CELLS + 1], pre4[MAX_BOX_CELLS + 1];
  const int2 tile = v.tiles_x[blockIdx.x / LIST_SPLIT];
  const int part = blockIdx.x % LIST_SPLIT;
  const int r = tile.x, b = tile.y;
  const SysDesc &d = v.desc[r];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5, warp = threadIdx.x >> 5;
  if (v.st[r].rebuild) {
    // the tile's own work: lists of a system without list sub-cells, and the
    // copy-back of the tile's slots
    const int nce = d.ncell;
    box_cells(v, d, cst, pre4);
    const int ca = b * d.cpb, cb = min(nce, ca + d.cpb);
    if (d.msub < 5) {
      const int W = LIST_SPLIT * nw, gw = part * nw + warp;
      box_stage_list(v, d, xstg, cst, pre4);
      __syncthreads();
      int item = 0;
      for (int c = ca; c < cb; c++) {
        const int groups = (cst[c + 1] - cst[c] + 7) >> 3;
        // warp gw takes the cell's groups g with (item + g) % W == gw
        for (int g = (gw - item % W + W) % W; g < groups; g += W)
          box_list_group(v, d, r, xstg, cst, pre4, c, 8 * g, lane);
        item += groups;
      }
    }
    const int stride = LIST_SPLIT * blockDim.x;
    for (int sl = cst[ca] + part * blockDim.x + threadIdx.x; sl < cst[cb]; sl += stride) copy_back(v, d.poff + sl);
  }
  // the work items of all rebuilding systems with list sub-cells, spread over
  // the warps of the whole grid: global warp w takes items w, w + W, ...
  // (one particle each for few particles in all, else a brick each: per
  // particle the chains are shorter, per brick the instructions fewer)
  const int K = v.rbs[0], T = v.rbs[1], Wg = gridDim.x * nw;
  for (int it = blockIdx.x * nw + warp; it < T; it += Wg) {
    int lo = 0, hi = K - 1;  // the last system whose first brick is <= it
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (v.rbs[3 + 2 * mid] <= it) lo = mid;
      else hi = mid - 1;
    }
    const int rs = v.rbs[2 + 2 * lo];
    const SysDesc &ds = v.desc[rs];
    if (v.box_warp)
      box_list_particle(v, ds, rs, v.xsub + ds.poff, v.ssub + ds.soff, it - v.rbs[3 + 2 * lo], lane);
    else
      box_list_brick(v, ds, rs, v.xsub + ds.poff, v.ssub + ds.soff, it - v.rbs[3 + 2 * lo], lane);
  }
}

// the system's current positions staged for the pair loop: FP32 as three
// arrays of 32-bit fixed point (a partner's type comes with its list entry),
// FP64 as three arrays of reduced coordinates
template <int PREC>
__device__ __forceinline__ void box_stage_force(const View &v, const SysDesc &d, unsigned char *xsm) {
  const int n = d.n;
  int *qx = reinterpret_cast<int *>(xsm), *qy = qx + n, *qz = qy + n;
  double *sx = reinterpret_cast<double *>(xsm), *sy = sx + n, *sz = sy + n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double4 p = v.pos[d.poff + k];
    if (PREC == 1) {
      qx[k] = fixed32(p.x);
      qy[k] = fixed32(p.y);
      qz[k] = fixed32(p.z);
    } else {
      sx[k] = p.x;
      sy[k] = p.y;
      sz[k] = p.z;
    }
  }
}

// pair sums of system-local slot sl (particle i) from its list, TPP threads
// per particle (summed across the TPP lanes on return; every thread of the
// warp takes part)
template <int TPP, int PREC>
__device__ __forceinline__ PairAcc box_pairs(const View &v, const SysDesc &d, const unsigned char *xsm, bool valid,
                                             int sl, int i, int lane) {
  const int n = d.n;
  const int *qx = reinterpret_cast<const int *>(xsm), *qy = qx + n, *qz = qy + n;
  const double *sx = reinterpret_cast<const double *>(xsm), *sy = sx + n, *sz = sy + n;
  const uint2 *lst = reinterpret_cast<const uint2 *>(box_list(v, d));
  const double L = d.L;
  const float scale = (float)(L * (1.0 / 4294967296.0));
  const int nn = valid ? v.nbn[i] : 0;
  {
    PairAcc a = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid && nn >= 0) {
      const int nch = (nn + 3) >> 2;
      const uint2 *lp = lst + sl;
      uint2 w = lane < nch ? __ldg(lp + (size_t)lane * n) : make_uint2(0u, 0u);
      if (PREC == 1) {
        // separations in fixed-point units (L / 2^32), folded into the constants
        const unsigned xi = qx[sl], yi = qy[sl], zi = qz[sl];
        const PairParamsF P((int)v.pos[i].w, scale);
        PairAccF fa = {0.f, 0.f, 0.f, 0.f, 0.f}, fb = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = lane; c < nch; c += TPP) {
          const uint2 wn = c + TPP < nch ? __ldg(lp + (size_t)(c + TPP) * n) : make_uint2(0u, 0u);
          const int k0 = 4 * c;
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int code = ((e < 2 ? w.x : w.y) >> (16 * (e & 1))) & 0xffff;
            if (e == 0 || k0 + e < nn) {
              const int j = code & 0x7fff;
              const float dx = (float)(int)(xi - (unsigned)qx[j]);
              const float dy = (float)(int)(yi - (unsigned)qy[j]);
              const float dz = (float)(int)(zi - (unsigned)qz[j]);
              pair_f32(e & 1 ? fb : fa, dx, dy, dz, P, code >> 15);
            }
          }
          flush_chunk(fa, fb, a);
          w = wn;
        }
        a.vir *= (double)scale;
      } else {
        const double xi = sx[sl], yi = sy[sl], zi = sz[sl];
        const PairParamsD P((int)v.pos[i].w);
        PairAcc bb = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = lane; c < nch; c += TPP) {
          const uint2 wn = c + TPP < nch ? __ldg(lp + (size_t)(c + TPP) * n) : make_uint2(0u, 0u);
          const int k0 = 4 * c;
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int code = ((e < 2 ? w.x : w.y) >> (16 * (e & 1))) & 0xffff;
            if (e == 0 || k0 + e < nn) {
              const int q = code & 0x7fff;
              pair_f64(e & 1 ? bb : a, min_image(xi - sx[q]) * L, min_image(yi - sy[q]) * L,
                       min_image(zi - sz[q]) * L, P, code >> 15);
            }
          }
          w = wn;
        }
        a.fx += bb.fx;
        a.fy += bb.fy;
        a.fz += bb.fz;
        a.pe += bb.pe;
        a.vir += bb.vir;
      }
    } else if (valid) {
      // list overflow: all particles of the 27 neighbour images (each pair once)
      const double4 pi = v.pos[i];
      const int ti = (int)pi.w;
      const double L2 = L * L;
      for (int k = lane; k < n; k += TPP) {
        if (k == sl) continue;
        const double4 pj = v.pos[d.poff + k];
        if (PREC == 0)
          pair_fp64(a, pi, ti, pj, L, L2);
        else
          pair_fp32(a, pi, ti, pj, L, L2);
      }
    }
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
      a.fx += __shfl_xor_sync(0xffffffffu, a.fx, o);
      a.fy += __shfl_xor_sync(0xffffffffu, a.fy, o);
      a.fz += __shfl_xor_sync(0xffffffffu, a.fz, o);
      a.pe += __shfl_xor_sync(0xffffffffu, a.pe, o);
      a.vir += __shfl_xor_sync(0xffffffffu, a.vir, o);
    }
    return a;
  }
}

// pair forces of a whole box from its lists.  FP32: staged 32-bit fixed-point
// reduced coordinates, separation = wrapped integer difference x L/2^32 (one
// rounding); FP64: staged reduced coordinates, minimum image d - rint(d).
template <int TPP, int PREC>
__global__ void __launch_bounds__(BLOCK_X, 4) k_force_box(View v, int mode) {
  extern __shared__ __align__(16) unsigned char xsm[];
  const int2 tile = v.tiles_x[blockIdx.x];
  const int r = tile.x, b = tile.y;
  const SysState &st = v.st[r];
  if (mode == 1 && !st.prime) return;
  const SysDesc &d = v.desc[r];
  if (mode == 3 && !pre_due(d, st)) return;
  const int n = d.n, nce = d.ncell;
  box_stage_force<PREC>(v, d, xsm);
  const int ca = b * d.cpb, cb = min(nce, ca + d.cpb);
  const int s_lo = v.cstart[d.coff + ca], s_hi = cb < nce ? v.cstart[d.coff + cb] : n;
  __syncthreads();
  double pe = 0.0, vir = 0.0, ke = 0.0, va = 0.0;
  const int lane = threadIdx.x % TPP, nper = blockDim.x / TPP;
  for (int t0 = s_lo; t0 < s_hi; t0 += nper) {
    const int sl = t0 + threadIdx.x / TPP;
    const bool valid = sl < s_hi;
    const int i = d.poff + (valid ? sl : s_lo);
    PairAcc a = box_pairs<TPP, PREC>(v, d, xsm, valid, sl, i, lane);
    if (!valid || lane != 0) continue;
    // per-particle sums, added up in slot order by the finaliser, so the
    // system's totals do not depend on how its cells are split into blocks
    double pei = 0.0, viri = 0.0, kei = 0.0, vai = 0.0;
    particle_epilogue(v, d, st, i, mode, a, pei, viri, kei, vai);
    v.pacc[i] = make_double4(pei, viri, kei, vai);
  }
  end_force_block(v, r, b, mode, pe, vir, ke, va);
}

// ---------------------------------------------------------------------------
// device-side step loop control (a graph's WHILE node): one block of steps done
__global__ void k_loop_ctl(long long *count, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0) {
    const long long c = *count - 1;
    *count = c;
    cudaGraphSetConditional(h, c > 0 ? 1u : 0u);
  }
}

__global__ void k_set_count(long long *count, long long n) {
  if (threadIdx.x == 0) *count = n;
}

// ---------------------------------------------------------------------------
// state upload / download (caller order <-> slots)
__global__ void k_load(View v, int r) {
  const SysDesc &d = v.desc[r];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < d.n; k += gridDim.x * blockDim.x) {
    const int i = d.poff + k;
    const double *s = v.stage_d + 9 * (size_t)d.poff;
    const int *si = v.stage_i + 2 * (size_t)d.poff;
    v.pos[i] = make_double4(s[3 * k], s[3 * k + 1], s[3 * k + 2], (double)si[k]);
    const double *u = s + 3 * (size_t)d.n, *p = s + 6 * (size_t)d.n;
    v.ux[i] = u[3 * k];
    v.uy[i] = u[3 * k + 1];
    v.uz[i] = u[3 * k + 2];
    v.ox[i] = u[3 * k];
    v.oy[i] = u[3 * k + 1];
    v.oz[i] = u[3 * k + 2];
    v.vx[i] = p[3 * k];
    v.vy[i] = p[3 * k + 1];
    v.vz[i] = p[3 * k + 2];
    v.fx[i] = v.fy[i] = v.fz[i] = 0.0;
    v.id[i] = k;
    v.act[i] = si[d.n + k];
    v.nbn[i] = 0;
    v.cellof[i] = 0;
  }
}

__global__ void k_unload(View v, int r) {
  const SysDesc &d = v.desc[r];
  const double s2 = v.st[r].s2;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < d.n; k += gridDim.x * blockDim.x) {
    const int i = d.poff + k;
    const int o = v.id[i];
    double *s = v.stage_d + 9 * (size_t)d.poff;
    double *u = s + 3 * (size_t)d.n, *p = s + 6 * (size_t)d.n;
    double *f = v.stage_f + 3 * (size_t)d.poff;
    const double4 q = v.pos[i];
    s[3 * o] = q.x;
    s[3 * o + 1] = q.y;
    s[3 * o + 2] = q.z;
    u[3 * o] = v.ux[i];
    u[3 * o + 1] = v.uy[i];
    u[3 * o + 2] = v.uz[i];
    p[3 * o] = __dmul_rn(v.vx[i], s2);
    p[3 * o + 1] = __dmul_rn(v.vy[i], s2);
    p[3 * o + 2] = __dmul_rn(v.vz[i], s2);
    f[3 * o] = v.fx[i];
    f[3 * o + 1] = v.fy[i];
    f[3 * o + 2] = v.fz[i];
    v.stage_i[2 * (size_t)d.poff + k] = o;  // slot order -> original index (cells)
  }
}

// recompute the next step's first thermostat half after a host change of the
// chain or temperature (single thread per system)
__global__ void k_prehalf(View v, int r) {
  if (threadIdx.x == 0) next_first_half(v.desc[r], v.st[r], 2.0 * v.st[r].ke_end);
}

__global__ void k_shuffle_now(View v, int r) { shuffle_component(v, r, blockIdx.x, v.st[r].step); }

// FP64 pipe probe: 8 independent FMA chains per thread
__global__ void k_fp64_fma(double *out, int iters, double m) {
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, 1e-9);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace acg
