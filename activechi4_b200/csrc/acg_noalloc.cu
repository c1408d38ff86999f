// Allocation-free force evaluation: acg_forces_noalloc (include/activechi4.h).
//
// Some callers cannot call cudaMalloc: code that runs inside a framework that
// owns all device memory through its own pool, hosts that forbid allocation
// after start-up (real-time or latency-bounded loops), and plug-ins that only
// receive device pointers from their host.  For them this entry point
// evaluates the pair + active forces of one system from device arrays the
// caller owns, keeping every intermediate (cell of each particle, cell counts,
// starts and fill cursors, cell-ordered particle indices, per-block partial
// sums, the last-block counter) in one fixed file-scope device array,
// acg_noalloc_scratch, instead of allocating.  Every GPU that loads the
// library holds that array (ACG_NOALLOC_SCRATCH_BYTES) until the process
// exits.
//
// All calls share the array and it keeps the last call's contents; whatever
// must start at zero is cleared at the start of each call.  Calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/activechi4.h"
#include "acg_device.cuh"

namespace acg {
int set_last_error(int code, const std::string &msg);  // acg_engine.cu: the text acg_last_error returns
}

namespace {

constexpr int NA_BLOCK = 128;
constexpr int NA_TPP = 4;
constexpr int NA_PB = NA_BLOCK / NA_TPP;  // particles per force block
constexpr int NA_MAX_BLOCKS = (ACG_NOALLOC_MAX_N + NA_PB - 1) / NA_PB;

// scratch layout (bytes): cell_of[N] order[N] ccount[C] cstart[C] cfill[C]
// partials[B][4] counter
constexpr size_t OFF_CELL = 0;
constexpr size_t OFF_ORDER = OFF_CELL + 4ull * ACG_NOALLOC_MAX_N;
constexpr size_t OFF_COUNT = OFF_ORDER + 4ull * ACG_NOALLOC_MAX_N;
constexpr size_t OFF_START = OFF_COUNT + 4ull * ACG_NOALLOC_MAX_CELLS;
constexpr size_t OFF_FILL = OFF_START + 4ull * ACG_NOALLOC_MAX_CELLS;
constexpr size_t OFF_PART = (OFF_FILL + 4ull * ACG_NOALLOC_MAX_CELLS + 255) / 256 * 256;
constexpr size_t OFF_CTR = OFF_PART + 32ull * NA_MAX_BLOCKS;
constexpr size_t SCRATCH_BYTES = (OFF_CTR + 256 + 255) / 256 * 256;
static_assert(SCRATCH_BYTES <= ACG_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

}  // namespace

static __device__ __align__(256) unsigned char acg_noalloc_scratch[ACG_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex na_mu;
void *na_ptr[256];  // device address of the scratch array, per device

int na_fail(int code, const std::string &m) { return acg::set_last_error(code, m); }

struct NaArgs {
  const double *x, *xu;
  const int *type, *act, *k;
  double *F, *out;
  unsigned char *scr;
  int n, nact, nc;
  double L, inv_cell, f0;
};

__device__ __forceinline__ int *na_i(const NaArgs &a, size_t off) { return (int *)(a.scr + off); }

__global__ void k_na_clear(NaArgs a) {
  const int ncell = a.nc * a.nc * a.nc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    na_i(a, OFF_COUNT)[c] = 0;
    na_i(a, OFF_FILL)[c] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *(unsigned int *)(a.scr + OFF_CTR) = 0u;
}

__global__ void k_na_count(NaArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int cx = acg::cell_coord(a.x[3 * i], a.inv_cell, a.nc);
  const int cy = acg::cell_coord(a.x[3 * i + 1], a.inv_cell, a.nc);
  const int cz = acg::cell_coord(a.x[3 * i + 2], a.inv_cell, a.nc);
  const int c = cx + cy * a.nc + cz * a.nc * a.nc;
  na_i(a, OFF_CELL)[i] = c;
  atomicAdd(&na_i(a, OFF_COUNT)[c], 1);
}

__global__ void k_na_scan(NaArgs a) {
  __shared__ int sh[1024];
  const int ncell = a.nc * a.nc * a.nc, B = blockDim.x;
  const int chunk = (ncell + B - 1) / B;
  const int beg = min((int)threadIdx.x * chunk, ncell), end = min(beg + chunk, ncell);
  int sum = 0;
  for (int c = beg; c < end; c++) sum += na_i(a, OFF_COUNT)[c];
  sh[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < B; o <<= 1) {
    int v = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  int run = sh[threadIdx.x] - sum;
  for (int c = beg; c < end; c++) {
    na_i(a, OFF_START)[c] = run;
    run += na_i(a, OFF_COUNT)[c];
  }
}

__global__ void k_na_scatter(NaArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int c = na_i(a, OFF_CELL)[i];
  const int slot = na_i(a, OFF_START)[c] + atomicAdd(&na_i(a, OFF_FILL)[c], 1);
  na_i(a, OFF_ORDER)[slot] = i;
}

// KA pair term, as MDcode/cell_list+forces.c:174-203 (each pair seen from
// both sides, so energy and virial are halved at the end)
__device__ __forceinline__ void na_pair(double xi, double yi, double zi, int ti, const NaArgs &a, int j,
                                        double &fx, double &fy, double &fz, double &pe, double &vir) {
  const double L = a.L;
  const double dx = acg::min_image(xi - a.x[3 * j]), dy = acg::min_image(yi - a.x[3 * j + 1]),
               dz = acg::min_image(zi - a.x[3 * j + 2]);
  const double dr2 = (dx * dx + dy * dy + dz * dz) * L * L;
  const int tp = ti + a.type[j];
  const double is2 = tp == 0 ? 1.0 : (tp == 1 ? 1.5625 : 1.0 / (0.88 * 0.88));
  const double rs2 = dr2 * is2;
  if (rs2 < acg::KA_RC2) {
    const double e4 = tp == 0 ? 4.0 : (tp == 1 ? 6.0 : 2.0);
    const double s2 = 1.0 / rs2, s6 = s2 * s2 * s2;
    pe += e4 * ((s6 * (s6 - 1.0)) + acg::KA_C0 + acg::KA_C2 * rs2);
    const double g = (2.0 * e4 * is2) * (6.0 * s6 * (s6 - 0.5) * s2 - acg::KA_C2);
    fx += g * L * dx;
    fy += g * L * dy;
    fz += g * L * dz;
    vir += g * dr2;
  }
}

__global__ void __launch_bounds__(NA_BLOCK) k_na_force(NaArgs a) {
  __shared__ double sh[4][NA_BLOCK / 32];
  __shared__ int s_last;
  const int grp = threadIdx.x / NA_TPP, lane = threadIdx.x % NA_TPP;
  const int i = blockIdx.x * NA_PB + grp;
  const bool valid = i < a.n;
  double fx = 0, fy = 0, fz = 0, pe = 0, vir = 0;
  if (valid) {
    const double xi = a.x[3 * i], yi = a.x[3 * i + 1], zi = a.x[3 * i + 2];
    const int ti = a.type[i];
    const int nc = a.nc, c = na_i(a, OFF_CELL)[i];
    const int cx = c % nc, cy = (c / nc) % nc, cz = c / (nc * nc);
    const int lo = acg::stencil_lo(nc), hi = acg::stencil_hi(nc);
    for (int oz = lo; oz <= hi; oz++)
      for (int oy = lo; oy <= hi; oy++)
        for (int ox = lo; ox <= hi; ox++) {
          const int c2 = acg::wrap_cell(cx + ox, nc) + acg::wrap_cell(cy + oy, nc) * nc +
                         acg::wrap_cell(cz + oz, nc) * nc * nc;
          const int s0 = na_i(a, OFF_START)[c2], m = na_i(a, OFF_COUNT)[c2];
          for (int q = lane; q < m; q += NA_TPP) {
            const int j = na_i(a, OFF_ORDER)[s0 + q];
            if (j != i) na_pair(xi, yi, zi, ti, a, j, fx, fy, fz, pe, vir);
          }
        }
  }
#pragma unroll
  for (int o = NA_TPP / 2; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    pe += __shfl_xor_sync(0xffffffffu, pe, o);
    vir += __shfl_xor_sync(0xffffffffu, vir, o);
  }
  double va = 0.0;
  if (valid && lane == 0) {
    const int t = a.act[i];
    if (t >= 0 && t < a.nact) {  // active force (MDcode/cell_list+forces.c:207-218)
      const double kx = (double)a.k[t], ky = (double)a.k[a.nact + t], kz = (double)a.k[2 * a.nact + t];
      const double *u = a.xu ? a.xu : a.x;
      fx += a.f0 * kx;
      fy += a.f0 * ky;
      fz += a.f0 * kz;
      va = a.f0 * (kx * u[3 * i] + ky * u[3 * i + 1] + kz * u[3 * i + 2]);
    }
    a.F[3 * i] = fx;
    a.F[3 * i + 1] = fy;
    a.F[3 * i + 2] = fz;
  }
  if (lane != 0 || !valid) pe = vir = 0.0;
  double v3[3] = {pe, vir, va};
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int q = 0; q < 3; q++) {
    double s = v3[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (l == 0) sh[q][w] = s;
  }
  __syncthreads();
  double *part = (double *)(a.scr + OFF_PART);
  if (threadIdx.x == 0) {
    double t[3] = {0, 0, 0};
    for (int q = 0; q < 3; q++)
      for (int ww = 0; ww < NA_BLOCK / 32; ww++) t[q] += sh[q][ww];
    part[4 * blockIdx.x] = t[0];
    part[4 * blockIdx.x + 1] = t[1];
    part[4 * blockIdx.x + 2] = t[2];
    __threadfence();
    s_last = atomicAdd((unsigned int *)(a.scr + OFF_CTR), 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double t[3] = {0, 0, 0};
  for (unsigned int b = 0; b < gridDim.x; b++)
    for (int q = 0; q < 3; q++) t[q] += __ldcg(&part[4 * b + q]);
  a.out[0] = 0.5 * t[0];
  a.out[1] = (0.5 * t[1]) / 3.0;
  a.out[2] = t[2];
  *(unsigned int *)(a.scr + OFF_CTR) = 0u;
}

}  // namespace

extern "C" int acg_forces_noalloc(const double *x, const double *xu, const int *type, const int *act_tag,
                                  const int *k, int n, int nact, double L, double f0, double *F,
                                  double *scalars, void *stream) {
  if (!x || !type || !act_tag || !F || !scalars || (nact > 0 && !k))
    return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: null device pointer");
  if (n < 2 || n > ACG_NOALLOC_MAX_N)
    return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: n must be in [2, " +
                                        std::to_string(ACG_NOALLOC_MAX_N) + "], got " + std::to_string(n));
  if (nact < 0 || nact > n) return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: nact must be in [0, n]");
  if (!(L > 0) || L > 1e6) return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: bad box length");
  // cell geometry of MDcode/Parallel.c:72-78 (cells no smaller than 2.85)
  const int nc = (int)((double)(int)L / 2.85);
  if (nc < 2) return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: box smaller than 2 cells of 2.85 per side");
  if ((long long)nc * nc * nc > ACG_NOALLOC_MAX_CELLS)
    return na_fail(ACG_ERR_INVALID, "acg_forces_noalloc: " + std::to_string((long long)nc * nc * nc) +
                                        " cells exceed ACG_NOALLOC_MAX_CELLS (" +
                                        std::to_string(ACG_NOALLOC_MAX_CELLS) + ")");
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess || dev < 0 || dev >= 256)
    return na_fail(ACG_ERR_CUDA, std::string("acg_forces_noalloc: cudaGetDevice: ") + cudaGetErrorString(ce));
  void *scr = nullptr;
  {
    // once per device, with that device current: the host-side name of the
    // array is not a device address; ask the runtime for the address
    std::lock_guard<std::mutex> lk(na_mu);
    if (!na_ptr[dev]) {
      void *p = nullptr;
      ce = cudaGetSymbolAddress(&p, acg_noalloc_scratch);
      if (ce != cudaSuccess || !p)
        return na_fail(ACG_ERR_CUDA,
                       std::string("acg_forces_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
      na_ptr[dev] = p;
    }
    scr = na_ptr[dev];
  }
  NaArgs a;
  a.x = x;
  a.xu = xu;
  a.type = type;
  a.act = act_tag;
  a.k = k;
  a.F = F;
  a.out = scalars;
  a.scr = (unsigned char *)scr;
  a.n = n;
  a.nact = nact;
  a.nc = nc;
  a.L = L;
  a.inv_cell = L / (L / (double)nc);
  a.f0 = f0;
  cudaStream_t s = (cudaStream_t)stream;
  const int ncell = nc * nc * nc;
  k_na_clear<<<(ncell + 255) / 256, 256, 0, s>>>(a);
  k_na_count<<<(n + 255) / 256, 256, 0, s>>>(a);
  k_na_scan<<<1, 1024, 0, s>>>(a);
  k_na_scatter<<<(n + 255) / 256, 256, 0, s>>>(a);
  k_na_force<<<(n + NA_PB - 1) / NA_PB, NA_BLOCK, 0, s>>>(a);
  ce = cudaGetLastError();
  if (ce != cudaSuccess)
    return na_fail(ACG_ERR_CUDA, std::string("acg_forces_noalloc: launch: ") + cudaGetErrorString(ce));
  return ACG_OK;
}
