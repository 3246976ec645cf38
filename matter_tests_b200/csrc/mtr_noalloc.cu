// mtr_noalloc.cu — mtr_p2g_noalloc: the particle-to-grid transfer of one
// particle set onto a caller-described grid, without allocating any memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// transfer particles to a grid.  A host loop being captured into a CUDA graph
// cannot allocate (allocation is not a capturable stream operation); a solver
// embedded in a framework that owns all device memory through its own pool
// (PyTorch's caching allocator, a game or VFX engine) may not allocate behind
// that pool's back; a real-time or fixed-budget caller must not pay for, or
// risk the failure of, an allocation inside its step.  Such callers pass
// device pointers they already own for the inputs and outputs, and this entry
// point keeps every intermediate (the cell-key sort, the tile ranges and the
// grid accumulators) in one file-scope device array of fixed size.
//
// Limits: at most MTR_NOALLOC_MAX_PARTICLES particles and
// MTR_NOALLOC_MAX_NODES grid nodes per call; larger requests are rejected
// with MTR_ERR_TOO_LARGE before anything is launched.  The array costs ~10 MB of device memory on every GPU
// that loads the library, until the process exits.
//
// Sharing: every call on a device uses the same array.  Each call clears
// what must start at zero (accumulators, tile ranges) at its start, so
// back-to-back calls are independent when they are ordered on the device;
// calls that overlap on the GPU (different streams without ordering, or
// several host threads) race on the array and give wrong results.
//
// Set-up: the first call on each device looks up the array's device address
// (cudaGetSymbolAddress) with that device current and raises the shared
// memory limit of the kernel; make that first call outside any stream
// capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/matter_gpu.h"
#include "mtr_kernels.cuh"

using namespace mtr;

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kMaxP = MTR_NOALLOC_MAX_PARTICLES;
constexpr size_t kMaxNodes = MTR_NOALLOC_MAX_NODES;
constexpr size_t kMaxTiles = MTR_NOALLOC_MAX_NODES;  // a tile holds at least one node
constexpr size_t kSortBlocks = (kMaxP + kSortTile - 1) / kSortTile;

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// scratch layout (byte offsets)
constexpr size_t kOffHeader = 0;
constexpr size_t kOffParams = kOffHeader + align256(sizeof(StepHeader));
constexpr size_t kOffKeys0 = kOffParams + align256(sizeof(DevParams));
constexpr size_t kOffKeysA = kOffKeys0 + align256(kMaxP * 4);
constexpr size_t kOffValsA = kOffKeysA + align256(kMaxP * 4);
constexpr size_t kOffKeysB = kOffValsA + align256(kMaxP * 4);
constexpr size_t kOffValsB = kOffKeysB + align256(kMaxP * 4);
constexpr size_t kOffHist = kOffValsB + align256(kMaxP * 4);
constexpr size_t kOffDtot = kOffHist + align256(256 * kSortBlocks * 4);
constexpr size_t kOffTileB = kOffDtot + align256(256 * 4);
constexpr size_t kOffTileE = kOffTileB + align256(kMaxTiles * 4);
constexpr size_t kOffAcc = kOffTileE + align256(kMaxTiles * 4);
constexpr size_t kScratchBytes = kOffAcc + align256(4 * kMaxNodes * sizeof(double));  // mass + momentum[3]

}  // namespace

// The scratch array.  In host code this name is a host-side stand-in, not a
// device address: host code must use the address returned by
// cudaGetSymbolAddress (scratch_for_current_device below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// The P2G variant: as k_p2g_w, but mass and momentum only (no stress, no
// friction channel), accumulating into the scratch grid.
template <int D, int DEG>
__global__ void __launch_bounds__(kChunk) k_p2g_noalloc(StepArgs A, const uint32_t* __restrict__ perm) {
  using TL = Tiling<D>;
  constexpr int PN = TL::PN, NODES = TL::NODES, TB = TL::TB;
  constexpr int NCH = 1 + D;
  const StepHeader* H = A.H;
  const uint32_t t = blockIdx.x;
  if (t >= H->ntiles) return;
  const uint32_t pb = A.tile_begin[t], pe = A.tile_end[t];
  if (pb >= pe) return;
  const DevParams& P = *A.P;
  extern __shared__ double smem[];
  double(*patch)[NODES] = reinterpret_cast<double(*)[NODES]>(smem);
  double(*crd)[PN] = reinterpret_cast<double(*)[PN]>(smem + NCH * NODES);
  MStage<D>* st = reinterpret_cast<MStage<D>*>(smem + NCH * NODES + 3 * PN);
  int tc[3];
  tile_coords<D>(H, t, tc);
  const int n0[3] = {tc[0] * TB - 1, tc[1] * TB - 1, D == 3 ? tc[2] * TB - 1 : 0};
  for (int i = threadIdx.x; i < NCH * NODES; i += blockDim.x) (&patch[0][0])[i] = 0.0;
  for (int i = threadIdx.x; i < D * PN; i += blockDim.x) {
    const int a = i / PN, o = i % PN;
    const int g = n0[a] + o;
    const double* ax = a == 0 ? A.gx : (a == 1 ? A.gy : A.gz);
    crd[a][o] = (g >= 0 && g < (int)H->N[a]) ? ax[g] : 0.0;
  }
  __syncthreads();
  const uint32_t Np = A.Np;
  const double ioh = P.one_over_dx, apicD = P.apicDinverse;
  const bool apic = P.flip_ratio < 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int LPP = D == 3 ? 16 : 4;
  const int q = lane % LPP;
  const int iy = D == 3 ? (q >> 2) : q;
  const int iz = D == 3 ? (q & 3) : 0;
  const int kbeg = warp * 32 + (lane / LPP) * LPP, kend = kbeg + LPP;
  for (uint32_t c0 = pb; c0 < pe; c0 += kChunk) {
    {
      const uint32_t s = c0 + threadIdx.x;
      MStage<D>& S = st[threadIdx.x];
      int packed = -1;
      if (s < pe) {
        const uint32_t j = perm[s];
        double xp[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < D; ++a) {
          xp[a] = A.in.x[(size_t)a * Np + j];
          S.x[a] = xp[a];
          S.v[a] = A.in.v[(size_t)a * Np + j];
        }
#pragma unroll
        for (int r = 0; r < D * D; ++r) S.B[r] = apic ? A.in.B[(size_t)r * Np + j] : 0.0;
        int lb[3];
        if (local_base<D>(H, xp, ioh, n0, true, lb)) {
#pragma unroll
          for (int a = 0; a < D; ++a)
#pragma unroll
            for (int o = 0; o < 4; ++o) S.w[a * 4 + o] = bspline_N<DEG>((xp[a] - crd[a][lb[a] + o]) * ioh);
          packed = lb[0] | (lb[1] << 4) | (lb[2] << 8);
        } else {
          atomicOr(&A.H->status, MTR_STATUS_STENCIL_OOB);
        }
      }
      S.lb = packed;
    }
    __syncthreads();
    {
      double acc[4][NCH];
#pragma unroll
      for (int h = 0; h < 4; ++h)
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) acc[h][ch] = 0.0;
      int cur = -1;
      auto flush = [&]() {
        const int lbx = cur & 15, lby = (cur >> 4) & 15, lbz = cur >> 8;
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int node = D == 3 ? ((lbx + h) * PN + (lby + iy)) * PN + (lbz + iz) : (lbx + h) * PN + (lby + iy);
#pragma unroll
          for (int ch = 0; ch < NCH; ++ch) {
            if (acc[h][ch] != 0.0) atomicAdd(&patch[ch][node], acc[h][ch]);
            acc[h][ch] = 0.0;
          }
        }
      };
      for (int k = kbeg; k < kend; ++k) {
        const MStage<D>& S = st[k];
        const int lbp = S.lb;
        if (lbp < 0) continue;
        if (lbp != cur) {
          if (cur >= 0) flush();
          cur = lbp;
        }
        const int lbx = lbp & 15, lby = (lbp >> 4) & 15, lbz = lbp >> 8;
        const double wyz = D == 3 ? S.w[4 + iy] * S.w[8 + iz] : S.w[4 + iy];
        const double pdy = crd[1][lby + iy] - S.x[1];
        const double pdz = D == 3 ? crd[2][lbz + iz] - S.x[D - 1] : 0.0;
        double Tm[D], Sm[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          if (apic) {
            double byz = S.B[a * D + 1] * pdy;
            if constexpr (D == 3) byz += S.B[a * D + 2] * pdz;
            Tm[a] = S.v[a] + apicD * byz;
            Sm[a] = apicD * S.B[a * D];
          } else {
            Tm[a] = S.v[a];
            Sm[a] = 0.0;
          }
        }
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const double weight = S.w[h] * wyz;
          if (!(weight > 1e-25)) continue;
          const double pdx = crd[0][lbx + h] - S.x[0];
          acc[h][0] += weight;
#pragma unroll
          for (int a = 0; a < D; ++a) acc[h][1 + a] += weight * (Tm[a] + Sm[a] * pdx);
        }
      }
      if (cur >= 0) flush();
    }
    __syncthreads();
  }
  const uint32_t cap = A.cap_nodes;
  for (int n = threadIdx.x; n < NODES; n += blockDim.x) {
    int li, lj, lk;
    if constexpr (D == 3) {
      lk = n % PN;
      lj = (n / PN) % PN;
      li = n / (PN * PN);
    } else {
      lk = 0;
      lj = n % PN;
      li = n / PN;
    }
    const int gi = n0[0] + li, gj = n0[1] + lj, gk = n0[2] + lk;
    if (gi < 0 || gj < 0 || gk < 0 || gi >= (int)H->N[0] || gj >= (int)H->N[1] || gk >= (int)H->N[2]) continue;
    const uint32_t l = node_index(H, gi, gj, gk);
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      const double val = patch[ch][n];
      if (val != 0.0) atomicAdd(&A.acc[(size_t)ch * cap + l], val);
    }
  }
}

// Cell keys of the first sort pass.  A particle whose cell lies outside the
// caller's grid (or whose position is not finite) gets the sentinel key
// ntiles * 64, one past every real tile: it sorts behind all real particles,
// no tile range names it, and it is reported through the status word.  The
// test is written on the same expression cell_key floors, so a particle kept
// here has a tile index below ntiles.
template <int D>
__global__ void __launch_bounds__(256) k_noalloc_keys(StepCommon A) {
  const StepHeader* H = A.H;
  const double ioh = A.P->one_over_dx;
  const uint32_t sentinel = H->ntiles * 64u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.Np; i += gridDim.x * blockDim.x) {
    double x[3] = {0.0, 0.0, 0.0};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      x[a] = A.xin[(size_t)a * A.Np + i];
      const double u = (x[a] - H->org[a]) * ioh;
      if (!(u >= 0.0 && u < (double)H->N[a])) inside = false;
    }
    if (inside) {
      A.keys0[i] = cell_key<D>(H, ioh, x);
    } else {
      A.keys0[i] = sentinel;
      atomicOr(&A.H->status, MTR_STATUS_STENCIL_OOB);
      atomicMin(&A.H->first_bad, i);
    }
  }
}

template <int D>
constexpr size_t noalloc_smem_bytes() {
  return sizeof(double) * ((1 + D) * Tiling<D>::NODES + 3 * Tiling<D>::PN) + sizeof(MStage<D>) * kChunk;
}

// Writes the grid description and the few constants the kernels read into
// the scratch header and parameter block (passed by value: no host copy).
__global__ void k_noalloc_setup(StepHeader* H, DevParams* P, const double* gx, const double* gy, const double* gz,
                                uint32_t nx, uint32_t ny, uint32_t nz, uint32_t tx, uint32_t ty, uint32_t tz,
                                double one_over_dx, double apicD, double flip_ratio, double particle_mass, uint32_t Np,
                                int dim) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  H->done = 0;
  H->abort = 0;
  H->frame = 0;
  H->stop_frame = 0xffffffffu;
  H->step = 0;
  H->stop_step = 0xffffffffu;
  H->status = 0;
  H->first_bad = 0xffffffffu;
  H->org[0] = gx[0];
  H->org[1] = gy[0];
  H->org[2] = dim == 3 ? gz[0] : 0.0;
  H->N[0] = nx;
  H->N[1] = ny;
  H->N[2] = nz;
  H->G = nx * ny * nz;
  H->T[0] = tx;
  H->T[1] = ty;
  H->T[2] = tz;
  H->ntiles = tx * ty * tz;
  P->one_over_dx = one_over_dx;
  P->apicDinverse = apicD;
  P->flip_ratio = flip_ratio;
  P->particle_mass = particle_mass;
  P->Np = Np;
  P->use_mibf = 0;
  P->dim = dim;
}

// p2g.cpp:84-98: v = momentum / (sum of weights), mass *= particle mass.
template <int D>
__global__ void k_noalloc_finalize(const double* __restrict__ acc, uint32_t cap, uint32_t G, double particle_mass,
                                   double* grid_mass, double* grid_v, const StepHeader* __restrict__ H,
                                   uint32_t* status) {
  if (status && blockIdx.x == 0 && threadIdx.x == 0) *status = H->status;
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < G; l += gridDim.x * blockDim.x) {
    const double m = acc[l];
#pragma unroll
    for (int a = 0; a < D; ++a) grid_v[(size_t)a * G + l] = (m > 0) ? acc[(size_t)(1 + a) * cap + l] / m : 0.0;
    grid_mass[l] = m * particle_mass;
  }
}

template <int D, int DEG>
bool set_attr() {
  return cudaFuncSetAttribute(k_p2g_noalloc<D, DEG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)noalloc_smem_bytes<D>()) == cudaSuccess;
}

// Once per device, with that device current: the device address of the
// scratch array.  Returns nullptr on failure.
unsigned char* scratch_for_current_device(int* rc_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *rc_out = MTR_ERR_NO_DEVICE;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      *rc_out = MTR_ERR_CUDA;
      return nullptr;
    }
    if (!(set_attr<2, 2>() && set_attr<2, 3>() && set_attr<3, 2>() && set_attr<3, 3>())) {
      *rc_out = MTR_ERR_CUDA;  // the device stays unset: the next call tries again
      return nullptr;
    }
    g_scratch_ptr[dev] = ptr;
  }
  *rc_out = MTR_OK;
  return static_cast<unsigned char*>(g_scratch_ptr[dev]);
}

template <int D, int DEG>
int run_noalloc(unsigned char* base, const mtr_params& p, const double* x, const double* v, const double* B,
                uint32_t Np, const double* gx, const double* gy, const double* gz, const uint32_t dims[3],
                double* grid_mass, double* grid_v, uint32_t* status, cudaStream_t st) {
  constexpr int TB = Tiling<D>::TB;
  StepHeader* H = reinterpret_cast<StepHeader*>(base + kOffHeader);
  DevParams* P = reinterpret_cast<DevParams*>(base + kOffParams);
  const uint32_t nx = dims[0], ny = dims[1], nz = D == 3 ? dims[2] : 1;
  const uint32_t tx = (nx + TB - 1) / TB, ty = (ny + TB - 1) / TB, tz = D == 3 ? (nz + TB - 1) / TB : 1;
  const uint64_t G = (uint64_t)nx * ny * nz, ntiles = (uint64_t)tx * ty * tz;
  const double apicD = p.spline_deg == 3 ? 3.0 / (p.dx * p.dx) : 4.0 / (p.dx * p.dx);
  StepArgs A{};
  A.P = P;
  A.H = H;
  A.Np = Np;
  A.gx = const_cast<double*>(gx);
  A.gy = const_cast<double*>(gy);
  A.gz = const_cast<double*>(gz ? gz : gy);
  A.cap_nodes = (uint32_t)kMaxNodes;
  A.cap_tiles = (uint32_t)ntiles;  // k_tile_ranges skips the sentinel tile (index ntiles)
  A.acc = reinterpret_cast<double*>(base + kOffAcc);
  A.keys0 = reinterpret_cast<uint32_t*>(base + kOffKeys0);
  A.keysA = reinterpret_cast<uint32_t*>(base + kOffKeysA);
  A.valsA = reinterpret_cast<uint32_t*>(base + kOffValsA);
  A.keysB = reinterpret_cast<uint32_t*>(base + kOffKeysB);
  A.valsB = reinterpret_cast<uint32_t*>(base + kOffValsB);
  A.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
  A.dtot = reinterpret_cast<uint32_t*>(base + kOffDtot);
  A.sort_blocks = (int)((Np + kSortTile - 1) / kSortTile);
  A.tile_begin = reinterpret_cast<uint32_t*>(base + kOffTileB);
  A.tile_end = reinterpret_cast<uint32_t*>(base + kOffTileE);
  A.in.x = const_cast<double*>(x);
  A.xin = x;
  A.in.v = const_cast<double*>(v);
  A.in.B = const_cast<double*>(B);
  // what must start at zero: the accumulators and the tile ranges of this grid
  // (memsets first, so that a failure leaves nothing of this call queued)
  if (cudaMemsetAsync(A.acc, 0, sizeof(double) * 4 * kMaxNodes, st) != cudaSuccess) return MTR_ERR_CUDA;
  if (cudaMemsetAsync(A.tile_begin, 0, sizeof(uint32_t) * ntiles, st) != cudaSuccess) return MTR_ERR_CUDA;
  if (cudaMemsetAsync(A.tile_end, 0, sizeof(uint32_t) * ntiles, st) != cudaSuccess) return MTR_ERR_CUDA;
  k_noalloc_setup<<<1, 32, 0, st>>>(H, P, gx, gy, gz, nx, ny, nz, tx, ty, tz, 1.0 / p.dx, apicD, p.flip_ratio,
                                    p.particle_mass, Np, D);
  k_noalloc_keys<D><<<(uint32_t)std::min<uint64_t>((Np + 255) / 256, 148 * 8), 256, 0, st>>>(A);
  // enough digits for every real key (below ntiles * 64) and the sentinel (ntiles * 64)
  uint64_t keybits = 1;
  while ((1ull << keybits) < ntiles * 64ull + 1ull) ++keybits;
  const int passes = (int)((keybits + 7) / 8);
  const uint32_t* skeys = nullptr;
  const uint32_t* perm = nullptr;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = 8 * pass;
    const uint32_t* ksrc = pass == 0 ? A.keys0 : ((pass & 1) ? A.keysB : A.keysA);
    const uint32_t* vsrc = pass == 0 ? nullptr : ((pass & 1) ? A.valsB : A.valsA);
    uint32_t* kdst = (pass & 1) ? A.keysA : A.keysB;
    uint32_t* vdst = (pass & 1) ? A.valsA : A.valsB;
    k_sort_hist<D, false><<<A.sort_blocks, kSortThreads, 0, st>>>(A, ksrc, shift);
    k_sort_scan<<<256, 256, 0, st>>>(A);
    k_sort_scatter<<<A.sort_blocks, kSortThreads, 0, st>>>(A, ksrc, vsrc, kdst, vdst, shift);
    skeys = kdst;
    perm = vdst;
  }
  k_tile_ranges<<<(Np + 255) / 256, 256, 0, st>>>(A, skeys);
  k_p2g_noalloc<D, DEG><<<(uint32_t)ntiles, kChunk, noalloc_smem_bytes<D>(), st>>>(A, perm);
  k_noalloc_finalize<D><<<(uint32_t)std::min<uint64_t>((G + 255) / 256, 148 * 8), 256, 0, st>>>(
      A.acc, (uint32_t)kMaxNodes, (uint32_t)G, p.particle_mass, grid_mass, grid_v, H, status);
  return cudaGetLastError() == cudaSuccess ? MTR_OK : MTR_ERR_CUDA;
}

}  // namespace

extern "C" int mtr_p2g_noalloc(const mtr_params* params, const double* x, const double* v, const double* B,
                               uint32_t Np, const double* gx, const double* gy, const double* gz,
                               const uint32_t dims[3], double* grid_mass, double* grid_v, uint32_t* status,
                               void* stream) {
  // an error left by earlier, unrelated work of this thread is not this call's failure
  (void)cudaGetLastError();
  if (!params || !x || !v || !gx || !gy || !dims || !grid_mass || !grid_v || Np == 0) return MTR_ERR_INVALID;
  const mtr_params& p = *params;
  if ((p.dim != 2 && p.dim != 3) || (p.spline_deg != 2 && p.spline_deg != 3) || !(p.dx > 0)) return MTR_ERR_INVALID;
  if (p.dim == 3 && !gz) return MTR_ERR_INVALID;
  if (p.flip_ratio < 0 && !B) return MTR_ERR_INVALID;
  const uint64_t G = (uint64_t)dims[0] * dims[1] * (p.dim == 3 ? dims[2] : 1);
  if (dims[0] < 4 || dims[1] < 4 || (p.dim == 3 && dims[2] < 4)) return MTR_ERR_INVALID;
  if (Np > MTR_NOALLOC_MAX_PARTICLES || G > MTR_NOALLOC_MAX_NODES) return MTR_ERR_TOO_LARGE;
  int rc = MTR_OK;
  unsigned char* base = scratch_for_current_device(&rc);
  if (!base) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (p.dim == 3)
    return p.spline_deg == 3 ? run_noalloc<3, 3>(base, p, x, v, B, Np, gx, gy, gz, dims, grid_mass, grid_v, status, st)
                             : run_noalloc<3, 2>(base, p, x, v, B, Np, gx, gy, gz, dims, grid_mass, grid_v, status, st);
  return p.spline_deg == 3 ? run_noalloc<2, 3>(base, p, x, v, B, Np, gx, gy, gz, dims, grid_mass, grid_v, status, st)
                           : run_noalloc<2, 2>(base, p, x, v, B, Np, gx, gy, gz, dims, grid_mass, grid_v, status, st);
}
