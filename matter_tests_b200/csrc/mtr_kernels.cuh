// mtr_kernels.cuh — the sm_100a kernels of one explicit MPM step
// (Simulation::advanceStep, simulation.cpp:219-273).
//
// Step pipeline (all on one stream, no host round trip, CUDA-graph capturable):
//   k_bbox        per-block min/max x, max |v|^2 and sum v    update_dt.cpp, remesh.cpp
//   k_header      dt, gravity ramp, remesh + arange axes      update_dt.cpp:5-66, remesh.cpp:38-311
//   k_sort_*      stable LSD radix sort by blocked cell key   (new: locality for P2G)
//   k_tile_ranges particle range of every 4^3 (2D: 8^2) tile
//   k_p2g_w       tile block -> shared grid patch -> one global atomic per node and channel
//                 (mass, momentum with APIC, force tau.grad w, MIBF friction)
//                                                              p2g.cpp:6-100, explicit_euler_update.cpp:15-77
//   k_grid        normalise, v += -dt V0 f/m + dt g, boundary collision, flip, FP64 balances
//                                                              p2g.cpp:84-98, explicit_euler_update.cpp:83-132
//   USL:  k_g2p_t gather pic/B/flip/grad v, F update, return mapping, tau, x/v update, coalesced stores
//                                                              g2p.cpp, deformation_update.cpp, plasticity.cpp,
//                                                              position_update.cpp
//   MUSL: k_g2p_musl_w (gather + v blend + re-scatter), k_musl_norm, k_defgrad_t
//                                                              musl.cpp:6-96
//   k_tail        plate motion, clock, frame and end test     object_plate.hpp:136-162, simulation.cpp:176-200
//
// Particle state is SoA, one array per component (x + a*Np), double buffered:
// the step reads the `in` set through the sort permutation and writes the
// `out` set in sorted order, so the particle order follows the cell order and
// every later read of the same data is nearly coalesced.
//
// Precision.  Every kernel that touches particle or grid state is templated
// on the storage type R.  R = double is the reference's FP64 arithmetic,
// operation for operation.  R = float is the mixed-precision form: particle
// v, F, B, stress and plastic scalars, the grid mass, momentum, force,
// friction and flip channels, the spline weights, the P2G and MUSL sums and
// the G2P gathers are FP32.  FP64 stays on the positions, the clock, the grid
// axes and node velocities, the deformation update, the SVD, the Hencky
// log/exp, the return mapping with its projections, and the mass and
// momentum balances.  F is stored as F - I in FP32, so its rounding is
// relative to the strain (about 1e-3) rather than to 1; the gathers work on
// FP32 deviations from a per-tile reference velocity, so the FP32 sums that
// form grad v do not cancel a common velocity.
#pragma once
#include <type_traits>

#include "mtr_boundary.cuh"
#include "mtr_device.cuh"
#include "mtr_plasticity.cuh"

namespace mtr {

template <typename R>
struct PBufT {
  double* x;     // [D][Np] positions, FP64 on both paths
  R* v;          // [D][Np]
  R* F;          // [D*D][Np], entry (r,c) at (r*D + c); FP32 path: F - I
  R* B;          // [D*D][Np]
  R* sc;         // [6][Np] MTR_SCALAR_* order
  R* tau;        // [Sym<D>::n][Np] Kirchhoff stress carried to the next P2G
  uint32_t* id;  // original particle index
};
using PBuf = PBufT<double>;

// What every kernel of a step shares, whatever the storage type.
struct StepCommon {
  const DevParams* P;
  StepHeader* H;
  BBoxPartial* partials;
  int npartials;
  uint32_t Np;
  double *gx, *gy, *gz;
  uint32_t cap_axis[3];
  uint32_t cap_nodes;
  uint32_t cap_tiles;
  const double* xin;  // positions of the step's input buffer (sort keys)
  uint32_t* keys0;    // cell key of each particle in input order
  uint32_t *keysA, *valsA, *keysB, *valsB;
  uint32_t* hist;  // [256][sort_blocks]
  uint32_t* dtot;  // [256]
  int sort_blocks;
  uint32_t* tile_begin;
  uint32_t* tile_end;
  const uint32_t* skeys;  // sorted keys and permutation after the last radix pass
  const uint32_t* perm;
  int out_parity;         // particle buffer this step writes
};

template <typename R>
struct StepArgsT : StepCommon {
  R* acc;         // [NCH][cap_nodes] P2G accumulators: mass, mom[D], force[D], friction
  double* nv;     // [D][cap_nodes] node velocity after the update (FP64 on both paths)
  R* nflip;       // [D][cap_nodes]
  R* nmass;       // [cap_nodes]
  R* nfric;       // [cap_nodes]
  double* v2;     // [D][cap_nodes] MUSL re-projection accumulator (FP64 on both paths)
  PBufT<R> in, out;
  R* pic;   // optional [D][Np] in output order
  R* flip;  // optional [D][Np]
};
using StepArgs = StepArgsT<double>;

template <typename R>
constexpr bool kFP64 = std::is_same<R, double>::value;

constexpr uint32_t kMaxAxisNodes = 1u << 22;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

template <int D>
struct Tiling {
  static constexpr int TB = D == 3 ? 4 : 8;     // cells per tile edge
  static constexpr int SH = D == 3 ? 2 : 3;     // log2(TB)
  static constexpr int PN = TB + 3;             // patch nodes per edge (stencil -1..+2)
  static constexpr int NODES = D == 3 ? PN * PN * PN : PN * PN;
  static constexpr int NCH = 2 + 2 * D;         // mass, mom[D], force[D], friction
};

constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

__device__ __forceinline__ bool step_inactive(const StepHeader* H) {
  return H->done || H->abort || H->frame >= H->stop_frame || H->step >= H->stop_step;
}

__device__ __forceinline__ uint32_t node_index(const StepHeader* H, int i, int j, int k) {
  return ((uint32_t)i * H->N[1] + (uint32_t)j) * H->N[2] + (uint32_t)k;
}

// sum over the block of a per-thread value, added once to *dst (all threads call)
__device__ __forceinline__ void block_add(double v, double* dst) {
  __shared__ double red[32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w];
    if (s != 0.0) atomicAdd(dst, s);
  }
}

// plastic particles of the block, one global atomic per block
__device__ __forceinline__ void block_count(unsigned n, unsigned long long* dst) {
  __shared__ unsigned cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  n = __reduce_add_sync(0xffffffffu, n);
  if ((threadIdx.x & 31) == 0 && n) atomicAdd(&cnt, n);
  __syncthreads();
  if (threadIdx.x == 0 && cnt) atomicAdd(dst, (unsigned long long)cnt);
}

// ---------------------------------------------------------------------------
// 1. bbox / vmax / sum v partials
// ---------------------------------------------------------------------------
template <int D, typename R>
__device__ __forceinline__ void bbox_body(const StepArgsT<R>& A, const uint32_t bid, const uint32_t nblk) {
  if (step_inactive(A.H)) return;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300}, v2 = 0.0, vs[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
  for (uint32_t i = bid * blockDim.x + threadIdx.x; i < A.Np; i += nblk * blockDim.x) {
    double vv[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      double xa = A.in.x[(size_t)a * A.Np + i];
      mn[a] = fmin(mn[a], xa);
      mx[a] = fmax(mx[a], xa);
      vv[a] = A.in.v[(size_t)a * A.Np + i];
      vs[a] += vv[a];
    }
    double s = __dadd_rn(__dmul_rn(vv[0], vv[0]), __dmul_rn(vv[1], vv[1]));
    if constexpr (D == 3) s = __dadd_rn(s, __dmul_rn(vv[2], vv[2]));
    v2 = fmax(v2, s);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int a = 0; a < D; ++a) {
      mn[a] = fmin(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
      mx[a] = fmax(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
      vs[a] += __shfl_xor_sync(0xffffffffu, vs[a], off);
    }
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, off));
  }
  __shared__ BBoxPartial wp[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      wp[warp].mn[a] = mn[a];
      wp[warp].mx[a] = mx[a];
      wp[warp].vsum[a] = vs[a];
    }
    wp[warp].v2 = v2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    BBoxPartial r = wp[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        r.mn[a] = fmin(r.mn[a], wp[w].mn[a]);
        r.mx[a] = fmax(r.mx[a], wp[w].mx[a]);
        r.vsum[a] += wp[w].vsum[a];
      }
      r.v2 = fmax(r.v2, wp[w].v2);
    }
    A.partials[bid] = r;
  }
}

template <int D, typename R>
__global__ void __launch_bounds__(256) k_bbox(StepArgsT<R> A) {
  bbox_body<D, R>(A, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// 2. step header: dt (update_dt.cpp:5-66) and grid (remesh.cpp:38-311)
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void header_body(const StepCommon& A) {
  StepHeader* H = A.H;
  const DevParams& P = *A.P;
  if (step_inactive(H)) return;
  // the block (blockDim.x a multiple of 32, at most 256) reduces the bbox
  // partials; warp 0 then does the rest
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300}, v2 = 0.0, vs[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < A.npartials; b += blockDim.x) {
    const BBoxPartial& q = A.partials[b];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = fmin(mn[a], q.mn[a]);
      mx[a] = fmax(mx[a], q.mx[a]);
      vs[a] += q.vsum[a];
    }
    v2 = fmax(v2, q.v2);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = fmin(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
      mx[a] = fmax(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
      vs[a] += __shfl_xor_sync(0xffffffffu, vs[a], off);
    }
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, off));
  }
  if (nw > 1) {
    __shared__ BBoxPartial wred[8];
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        wred[wid].mn[a] = mn[a];
        wred[wid].mx[a] = mx[a];
        wred[wid].vsum[a] = vs[a];
      }
      wred[wid].v2 = v2;
    }
    __syncthreads();
    if (wid != 0) return;
    for (int w = 1; w < nw; ++w) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mn[a] = fmin(mn[a], wred[w].mn[a]);
        mx[a] = fmax(mx[a], wred[w].mx[a]);
        vs[a] += wred[w].vsum[a];
      }
      v2 = fmax(v2, wred[w].v2);
    }
  }
  __shared__ double s_low[3], s_high[3], s_stop[3];
  __shared__ int s_ok;
  if (lane == 0) {
    // balances of this step (read back by mtr_balance)
    H->grid_mass = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      H->grid_mom[a] = 0.0;
      H->part_mom[a] = P.particle_mass * vs[a];
    }
    // updateDt
    const double max_speed = sqrt(v2);
    double dt;
    if (fabs(max_speed) > 1e-10) {
      double dt_cfl = P.cfl * P.dx / max_speed;
      dt = dmin(dt_cfl, P.dt_max);
    } else {
      dt = P.dt_max;
    }
    dt = dmin(dt, __dsub_rn(__dmul_rn(P.frame_dt, (double)(H->frame + 1)), H->time));
    dt = dmin(dt, __dsub_rn(P.final_time, H->time));
    H->dt = dt;
    if (P.gravity_special) {
#pragma unroll
      for (int a = 0; a < D; ++a)
        H->gravity[a] = (H->time < P.gravity_time) ? P.gravity_final[a] * H->time / P.gravity_time : P.gravity_final[a];
    }
    // remesh
    const double dx = P.dx;
    if (P.pbc) {  // remeshFixed(4), remesh.cpp:14-36: the same fixed grid every step
      const double e1 = 5.0, e2 = 6.0;  // 1 + extra_nodes, 2 + extra_nodes
#pragma unroll
      for (int a = 0; a < D; ++a) {
        s_low[a] = a == 1 ? -dx : __dmul_rn(-dx, e1);
        s_stop[a] = __dadd_rn(P.L[a], __dmul_rn(e2, dx));
      }
    } else if (H->step == 0) {  // remeshFixedInit(2,2,2)
      if (P.grid_ref[0] < 1e10) {
#pragma unroll
        for (int a = 0; a < D; ++a) {
          if (P.grid_ref[a] < mn[a])
            mn[a] = P.grid_ref[a];
          else if (P.grid_ref[a] > mx[a])
            mx[a] = P.grid_ref[a];
        }
      }
#pragma unroll
      for (int a = 0; a < D; ++a) {
        H->max_init[a] = mx[a];
        H->min_init[a] = mn[a];
        H->low_init[a] = __dsub_rn(mn[a], __dmul_rn(dx, 2.0));
        H->high_init[a] = __dadd_rn(mx[a], __dmul_rn(dx, 2.0));
        s_low[a] = H->low_init[a];
        s_high[a] = H->high_init[a];
      }
    } else {  // remeshFixedCont
      // explicit roundings: each product and difference is rounded on its own,
      // as in the host code this restates (no fused multiply-add)
      const double tiny = __dmul_rn(1e-8, dx);
      for (int a = 0; a < D; ++a) {
        double hi, lo;
        if (mx[a] < H->max_init[a]) {
          unsigned int f = (unsigned int)floor(dmax(0.0, __dsub_rn(__ddiv_rn(__dsub_rn(H->max_init[a], mx[a]), dx), tiny)));
          hi = __dsub_rn(H->high_init[a], __dmul_rn((double)f, dx));
        } else {
          unsigned int f = (unsigned int)floor(dmax(0.0, __dsub_rn(__ddiv_rn(__dsub_rn(mx[a], H->max_init[a]), dx), tiny)));
          hi = __dadd_rn(H->high_init[a], __dmul_rn((double)f, dx));
        }
        if (mn[a] > H->min_init[a]) {
          unsigned int f = (unsigned int)floor(dmax(0.0, __dsub_rn(__ddiv_rn(__dsub_rn(mn[a], H->min_init[a]), dx), tiny)));
          lo = __dadd_rn(H->low_init[a], __dmul_rn((double)f, dx));
        } else {
          unsigned int f = (unsigned int)floor(dmax(0.0, __dsub_rn(__ddiv_rn(__dsub_rn(H->min_init[a], mn[a]), dx), tiny)));
          lo = __dsub_rn(H->low_init[a], __dmul_rn((double)f, dx));
        }
        s_low[a] = lo;
        s_high[a] = hi;
      }
    }
    if (!P.pbc) {
#pragma unroll
      for (int a = 0; a < D; ++a) s_stop[a] = __dadd_rn(s_high[a], dx);
    }
    s_ok = 1;
  }
  __syncwarp();
  // arange (tools.hpp:291-296): one lane per axis accumulates value += step
  if (lane < D) {
    const double dx = P.dx;
    double* ax = lane == 0 ? A.gx : (lane == 1 ? A.gy : A.gz);
    const uint32_t cap = A.cap_axis[lane];
    const double stop = s_stop[lane];
    uint32_t n = 0;
    // counted exactly up to kMaxAxisNodes so the host can size the regrowth in
    // one go; the bound also ends the loop for non-finite extents
    for (double value = s_low[lane]; value < stop && n < kMaxAxisNodes; value = __dadd_rn(value, dx)) {
      if (n < cap) ax[n] = value;
      ++n;
    }
    H->N[lane] = n;
    H->org[lane] = s_low[lane];
    if (n > cap || n < 4 || n >= kMaxAxisNodes) atomicExch(&s_ok, 0);
  }
  __syncwarp();
  if (lane == 0) {
    if (D == 2) {
      H->N[2] = 1;
      H->org[2] = 0.0;
    }
    constexpr int TB = Tiling<D>::TB;
    uint64_t G = (uint64_t)H->N[0] * H->N[1] * H->N[2];
    H->T[0] = (H->N[0] + TB - 1) / TB;
    H->T[1] = (H->N[1] + TB - 1) / TB;
    H->T[2] = D == 3 ? (H->N[2] + TB - 1) / TB : 1;
    uint64_t nt = (uint64_t)H->T[0] * H->T[1] * H->T[2];
    if (!s_ok || G > A.cap_nodes || nt > A.cap_tiles) {
      H->abort = 1;
      atomicOr(&H->status, MTR_STATUS_GRID_OVERFLOW);
    }
    H->G = (uint32_t)G;
    H->ntiles = (uint32_t)nt;
  }
}

template <int D>
__global__ void __launch_bounds__(256) k_header(StepCommon A) {
  header_body<D>(A);
}

// ---------------------------------------------------------------------------
// 3. stable LSD radix sort of (blocked cell key, input position)
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ uint32_t cell_key(const StepHeader* H, double ioh, const double (&x)[3]) {
  constexpr int SH = Tiling<D>::SH, TB = Tiling<D>::TB;
  int c[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) c[a] = (int)floor((x[a] - H->org[a]) * ioh);
  uint32_t t, in;
  if constexpr (D == 3) {
    t = ((uint32_t)(c[0] >> SH) * H->T[1] + (uint32_t)(c[1] >> SH)) * H->T[2] + (uint32_t)(c[2] >> SH);
    in = ((uint32_t)(c[0] & (TB - 1)) * TB + (uint32_t)(c[1] & (TB - 1))) * TB + (uint32_t)(c[2] & (TB - 1));
  } else {
    t = (uint32_t)(c[0] >> SH) * H->T[1] + (uint32_t)(c[1] >> SH);
    in = (uint32_t)(c[0] & (TB - 1)) * TB + (uint32_t)(c[1] & (TB - 1));
  }
  return t * 64u + in;
}

// Per-block digit histogram.  The first pass computes the keys from x.
template <int D, bool FIRST>
__device__ __forceinline__ void sort_hist_body(const StepCommon& A, const uint32_t* __restrict__ keys,
                                                            int shift, const uint32_t bid, const uint32_t nblk) {
  if (step_inactive(A.H)) return;
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = bid * kSortTile;
  const double ioh = A.P->one_over_dx;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    uint32_t i = base + r * kSortThreads + threadIdx.x;
    if (i < A.Np) {
      uint32_t k;
      if (FIRST) {
        double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < D; ++a) x[a] = A.xin[(size_t)a * A.Np + i];
        k = cell_key<D>(A.H, ioh, x);
        A.keys0[i] = k;
      } else {
        k = keys[i];
      }
      atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
  }
  __syncthreads();
  A.hist[threadIdx.x * A.sort_blocks + bid] = h[threadIdx.x];
}

template <int D, bool FIRST>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(StepCommon A, const uint32_t* __restrict__ keys,
                                                            int shift) {
  sort_hist_body<D, FIRST>(A, keys, shift, blockIdx.x, gridDim.x);
}

// Exclusive scan of each digit's row over the blocks; row totals to dtot.
static __device__ __forceinline__ void sort_scan_body(const StepCommon& A, const uint32_t bid, const uint32_t nblk) {
  if (step_inactive(A.H)) return;
  const int dgt = bid;
  uint32_t* row = A.hist + (size_t)dgt * A.sort_blocks;
  __shared__ uint32_t ws[8];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < A.sort_blocks; b0 += 256) {
    int b = b0 + threadIdx.x;
    uint32_t v = b < A.sort_blocks ? row[b] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
      if ((threadIdx.x & 31) >= off) incl += t;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += ws[w];
    uint32_t total = 0;
    for (int w = 0; w < 8; ++w) total += ws[w];
    if (b < A.sort_blocks) row[b] = carry + wpre + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) A.dtot[dgt] = carry;
}

static __global__ void __launch_bounds__(256) k_sort_scan(StepCommon A) {
  sort_scan_body(A, blockIdx.x, gridDim.x);
}

// The same scan with one warp per digit, kScanDigitsPerBlock digits per
// 256-thread block: the batched form, where most scenes have few sort blocks
// and a block per digit and scene would leave the blocks nearly idle.
constexpr int kScanDigitsPerBlock = 8;
static __device__ __forceinline__ void sort_scan_warp_body(const StepCommon& A, const uint32_t bid) {
  if (step_inactive(A.H)) return;
  const int lane = threadIdx.x & 31;
  const int dgt = (int)bid * kScanDigitsPerBlock + (int)(threadIdx.x >> 5);
  if (dgt >= 256) return;  // no block-wide barrier below
  uint32_t* row = A.hist + (size_t)dgt * A.sort_blocks;
  uint32_t carry = 0;
  for (int b0 = 0; b0 < A.sort_blocks; b0 += 32) {
    const int b = b0 + lane;
    const uint32_t v = b < A.sort_blocks ? row[b] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += t;
    }
    if (b < A.sort_blocks) row[b] = carry + incl - v;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) A.dtot[dgt] = carry;
}

// Stable scatter.  Elements are ranked round by round (256 at a time, in
// index order) with warp match + per-warp digit counts, which keeps equal
// digits in input order.
static __device__ __forceinline__ void sort_scatter_body(const StepCommon& A, const uint32_t* __restrict__ ksrc,
                                                               const uint32_t* __restrict__ vsrc, uint32_t* kdst,
                                                               uint32_t* vdst, int shift, const uint32_t bid, const uint32_t nblk) {
  if (step_inactive(A.H)) return;
  __shared__ uint32_t goff[256];
  __shared__ uint32_t run[256];
  __shared__ uint32_t wcnt[kSortThreads / 32][256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  {  // digit base = exclusive prefix of digit totals, plus this block's row offset
    uint32_t v = A.dtot[tid];
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += t;
    }
    __shared__ uint32_t ws[8];
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += ws[w];
    goff[tid] = wpre + incl - v + A.hist[(size_t)tid * A.sort_blocks + bid];
    run[tid] = 0;
  }
  const uint32_t base = bid * kSortTile;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < kSortItems; ++r) {
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    const uint32_t i = base + r * kSortThreads + tid;
    const bool valid = i < A.Np;
    uint32_t k = 0, val = 0, dgt = 256;
    if (valid) {
      k = ksrc[i];
      val = vsrc ? vsrc[i] : i;
      dgt = (k >> shift) & 255u;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, dgt);
    const uint32_t rank = __popc(peers & lt_mask);
    if (valid && rank == 0) wcnt[warp][dgt] = __popc(peers);
    __syncthreads();
    {  // exclusive prefix over warps per digit, on top of earlier rounds
      uint32_t acc = run[tid];
#pragma unroll
      for (int w = 0; w < kSortThreads / 32; ++w) {
        uint32_t c = wcnt[w][tid];
        wcnt[w][tid] = acc;
        acc += c;
      }
      run[tid] = acc;
    }
    __syncthreads();
    if (valid) {
      const uint32_t pos = goff[dgt] + wcnt[warp][dgt] + rank;
      kdst[pos] = k;
      vdst[pos] = val;
    }
    __syncthreads();
  }
}

static __global__ void __launch_bounds__(kSortThreads) k_sort_scatter(StepCommon A, const uint32_t* __restrict__ ksrc,
                                                               const uint32_t* __restrict__ vsrc, uint32_t* kdst,
                                                               uint32_t* vdst, int shift) {
  sort_scatter_body(A, ksrc, vsrc, kdst, vdst, shift, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// 4. tile ranges over the sorted keys
// ---------------------------------------------------------------------------
static __device__ __forceinline__ void tile_ranges_body(const StepCommon& A, const uint32_t* __restrict__ skeys, const uint32_t bid, const uint32_t nblk) {
  if (step_inactive(A.H)) return;
  for (uint32_t s = bid * blockDim.x + threadIdx.x; s < A.Np; s += nblk * blockDim.x) {
    const uint32_t t = skeys[s] >> 6;
    if (t >= A.cap_tiles) continue;
    if (s == 0 || (skeys[s - 1] >> 6) != t) A.tile_begin[t] = s;
    if (s == A.Np - 1 || (skeys[s + 1] >> 6) != t) A.tile_end[t] = s + 1;
  }
}

static __global__ void __launch_bounds__(256) k_tile_ranges(StepCommon A, const uint32_t* __restrict__ skeys) {
  tile_ranges_body(A, skeys, blockIdx.x, gridDim.x);
}

template <int D>
__device__ __forceinline__ void tile_coords(const StepHeader* H, uint32_t t, int (&tc)[3]) {
  if constexpr (D == 3) {
    tc[2] = (int)(t % H->T[2]);
    uint32_t r = t / H->T[2];
    tc[1] = (int)(r % H->T[1]);
    tc[0] = (int)(r / H->T[1]);
  } else {
    tc[2] = 0;
    tc[1] = (int)(t % H->T[1]);
    tc[0] = (int)(t / H->T[1]);
  }
}

// Sets the patch origin n0 of tile t and copies the grid coordinates its
// stencils can reach into crd.
template <int D>
__device__ __forceinline__ void load_tile_setup(const StepCommon& A, const StepHeader* H, uint32_t t, int (&n0)[3],
                                                double (*crd)[Tiling<D>::PN]) {
  constexpr int PN = Tiling<D>::PN, TB = Tiling<D>::TB;
  int tc[3];
  tile_coords<D>(H, t, tc);
  n0[0] = tc[0] * TB - 1;
  n0[1] = tc[1] * TB - 1;
  n0[2] = D == 3 ? tc[2] * TB - 1 : 0;
  for (int i = threadIdx.x; i < D * PN; i += blockDim.x) {
    const int a = i / PN, o = i % PN;
    const int g = n0[a] + o;
    const double* ax = a == 0 ? A.gx : (a == 1 ? A.gy : A.gz);
    crd[a][o] = (g >= 0 && g < (int)H->N[a]) ? ax[g] : 0.0;
  }
}

// local stencil base of a particle in its tile patch; false if outside
template <int D>
__device__ __forceinline__ bool local_base(const StepHeader* H, const double (&xp)[3], double ioh, const int (&n0)[3],
                                           bool clamp, int (&lb)[3]) {
  constexpr int PN = Tiling<D>::PN;
  bool ok = true;
  lb[0] = lb[1] = lb[2] = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    int b = (int)floor((xp[a] - H->org[a]) * ioh) - 1;
    if (clamp) b = b < 0 ? 0 : b;
    lb[a] = b - n0[a];
    if (b < 0 || lb[a] < 0 || lb[a] > PN - 4 || b + 3 >= (int)H->N[a]) ok = false;
  }
  return ok;
}

// global node of patch entry n, or false outside the grid
template <int D>
__device__ __forceinline__ bool patch_node(const StepHeader* H, const int (&n0)[3], int n, uint32_t& l) {
  constexpr int PN = Tiling<D>::PN;
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
  if (gi < 0 || gj < 0 || gk < 0 || gi >= (int)H->N[0] || gj >= (int)H->N[1] || gk >= (int)H->N[2]) return false;
  l = node_index(H, gi, gj, gk);
  return true;
}

// ---------------------------------------------------------------------------
// 5. P2G + stress force, warp-cooperative, one block per tile.
//
// A tile block walks its sorted particles in chunks of blockDim.x (64, 128 or
// 256 threads, chosen per scene at run time by measurement).  Phase 1, one
// thread per particle, loads the particle and stages its stencil weights and
// gradients in shared memory.  Phase 2: lane groups (3D: 16 lanes, 2D: 4 lanes)
// take consecutive staged particles; a lane owns one stencil column of the
// particle's cell (3D: (iy, iz) and its 4 ix nodes, 2D: iy and its 4 ix
// nodes), accumulates every channel in registers while consecutive particles
// share a cell, and adds them to the shared patch once per cell.  Sorted
// particles share cells in runs of about ppc, so this issues ~ppc times fewer
// shared atomics than one atomic per particle and node, with no two lanes of
// a group on one address.  The patch is flushed with one global atomic per
// node and channel.
// ---------------------------------------------------------------------------
constexpr int kChunk = 128;  // default block size of the tile kernels
// Largest block of the tile kernels.  The scatter kernels stage one particle
// per thread, so their shared memory grows with the block; k_g2p_t stays at
// kChunk threads at most (its register bound below is per 128-thread block).
constexpr int kMaxTileThreads = 256;

// Minimum resident blocks of 128 threads per SM requested for the tile kernels
// that run the return mapping; it bounds their registers per thread.  Four
// blocks of 128 threads (128 registers, some spilled to L1) measured 15-25%
// faster for k_defgrad_t than the unbounded two blocks (240 registers) on the
// 3D collapse; three blocks measured best for k_g2p_t on the 3D Cam-Clay incline.
// The FP32-storage form holds fewer live values and gains from a tighter bound:
// six blocks of 128 threads (80 registers) measured 6% faster for its
// k_defgrad_t on the 3D collapse than four.  The FP64 form keeps four: six
// measured 2% faster (0.295 -> 0.287 ms at step 300 of the 1M collapse) but
// spilled to DRAM, writing 378 MB per launch instead of 150 MB (ncu).
#ifndef MTR_DEFGRAD_MIN_BLOCKS
#define MTR_DEFGRAD_MIN_BLOCKS 4
#endif
#ifndef MTR_DEFGRAD_MIN_BLOCKS_F32
#define MTR_DEFGRAD_MIN_BLOCKS_F32 6
#endif
// The return mapping takes its SVD from the symmetric eigenproblem of F F^T
// (svd_sym); 0 selects the two-sided Jacobi iteration with the reference's
// ordering and sign conventions instead.
#ifndef MTR_SYM_SVD
#define MTR_SYM_SVD 1
#endif
#ifndef MTR_G2P_MIN_BLOCKS
#define MTR_G2P_MIN_BLOCKS 3
#endif
// the same register bound for blocks of up to kMaxTileThreads threads (R is
// the storage type of the kernel the bound is written on)
#define MTR_DEFGRAD_BOUNDS \
  kMaxTileThreads, ((sizeof(R) == 4 ? MTR_DEFGRAD_MIN_BLOCKS_F32 : MTR_DEFGRAD_MIN_BLOCKS) * kChunk / kMaxTileThreads)

// FP64 stage: the position is kept and node offsets are formed in phase 2.
template <int D, typename R = double>
struct PStage {
  double x[D], v[D], B[D * D], tau[Sym<D>::n], w[D * 4], dw[D * 4];
  double mui;
  int lb;  // packed local stencil base (4 bits per axis); -1 marks an empty slot
  int pad;
};

// FP32 stage: node offsets x_i - x_p are formed in FP64 in phase 1 and
// stored rounded, so phase 2 runs in FP32 only.
template <int D>
struct PStage<D, float> {
  float pd[D * 4], v[D], B[D * D], tau[Sym<D>::n], w[D * 4], dw[D * 4];
  float mui;
  int lb;
};

template <int D, typename R>
__device__ __forceinline__ R stage_pd(const PStage<D, R>& S, const double (*crd)[Tiling<D>::PN], int a, int lba,
                                      int o) {
  if constexpr (kFP64<R>)
    return crd[a][lba + o] - S.x[a];
  else
    return S.pd[a * 4 + o];
}

// Particles staged per chunk by a scatter block of `threads` threads:
// threads / DIV.  A smaller chunk needs less shared memory per block (more
// resident blocks per SM) at the price of more chunk barriers and shorter
// register runs per lane group.  Measured on the 1M 3D collapse and the 1.2M
// incline (ms per launch at each kernel's best block shape): P2G with half
// chunks FP64 0.461 -> 0.449, mixed 0.252 -> 0.245, at 256 threads FP64
// 0.682 -> 0.471; the MUSL scatter slower with them (mixed 0.252 -> 0.309),
// so it keeps full chunks.
// The scatters stage B already multiplied by D^-1 (apicDinverse) and P2G the
// stress already multiplied by 1/dx, so phase 2 (run by every lane of a
// particle's group) does not repeat those products.
// The scatters' test of the reference's weight threshold as a select (a
// zero weight adds nothing) instead of a branch around each node's sums; the
// branch split the unrolled node loop.  Measured (ms per launch at the best
// shape): FP64 P2G 0.391 -> 0.370 on the 1M collapse and 0.511 -> 0.471 on the
// 1.2M incline, mixed P2G 0.244 -> 0.237, FP64 MUSL 0.397 -> 0.375.
#ifndef MTR_SCATTER_SELECT
#define MTR_SCATTER_SELECT 1
#endif
#ifndef MTR_SCATTER_PRESCALE
#define MTR_SCATTER_PRESCALE 1
#endif
// With half chunks, every P2G thread takes part in staging: two threads per
// staged particle (otherwise half the block waits at the barrier after the
// staging, the kernel's top stall): FP64 P2G 0.369 -> 0.356 ms on the 1M
// collapse and 0.473 -> 0.452 on the 1.2M incline, mixed 0.238 -> 0.232.
#ifndef MTR_P2G_PAIR_STAGE
#define MTR_P2G_PAIR_STAGE 1
#endif
#ifndef MTR_P2G_CHUNK_DIV
#define MTR_P2G_CHUNK_DIV 2
#endif
// Largest block of the MUSL scatter and the resident blocks of that size its
// register bound asks for.  Capped at 128 threads with five resident blocks
// (at most 102 registers; the FP64 form had 124): FP64 MUSL 0.413 -> 0.399 ms,
// mixed 0.297 -> 0.265 on the 1M collapse at step 300 (256-thread blocks,
// which the bound rules out, never measured fastest for this kernel).
#ifndef MTR_MUSL_MAX_THREADS
#define MTR_MUSL_MAX_THREADS 128
#endif
#ifndef MTR_MUSL_MIN_BLOCKS
#define MTR_MUSL_MIN_BLOCKS 5
#endif
#ifndef MTR_MUSL_CHUNK_DIV
#define MTR_MUSL_CHUNK_DIV 1
#endif
template <typename S, int DIV>
constexpr size_t stage_bytes(int threads) {
  return sizeof(S) * (size_t)(threads / DIV);
}

template <int D, typename R>
constexpr size_t p2g_crd_bytes() {
  return align16(sizeof(double) * 3 * Tiling<D>::PN);
}
// The patch's last channel (MIBF friction) is allocated only under MIBF: a
// block without it needs 2.7 KB (FP64, 3D) less shared memory, which lets
// five FP64 P2G blocks of 128 threads share an SM instead of four.
template <int D, typename R>
__host__ __device__ constexpr size_t p2g_patch_bytes(bool mibf) {
  return align16(sizeof(R) * (Tiling<D>::NCH - (mibf ? 0 : 1)) * Tiling<D>::NODES);
}
template <int D, typename R>
constexpr size_t p2g_smem_bytes(int threads, bool mibf = true) {
  return p2g_crd_bytes<D, R>() + p2g_patch_bytes<D, R>(mibf) + stage_bytes<PStage<D, R>, MTR_P2G_CHUNK_DIV>(threads);
}

template <int D, int DEG, typename R, int XS = 1>
__device__ __forceinline__ void p2g_w_body(const StepArgsT<R>& A, const uint32_t* __restrict__ perm, const uint32_t bid, const uint32_t nblk) {
  using TL = Tiling<D>;
  constexpr int PN = TL::PN, NODES = TL::NODES, NCH = TL::NCH, TB = TL::TB;
  constexpr int NS = Sym<D>::n;
  const StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const uint32_t t = bid;
  if (t >= H->ntiles) return;
  const uint32_t pb = A.tile_begin[t], pe = A.tile_end[t];
  if (pb >= pe) return;
  const DevParams& P = *A.P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double(*crd)[PN] = reinterpret_cast<double(*)[PN]>(smem_raw);
  R(*patch)[NODES] = reinterpret_cast<R(*)[NODES]>(smem_raw + p2g_crd_bytes<D, R>());
  const bool mibf = P.use_mibf;
  const int nch = mibf ? NCH : NCH - 1;  // channels the patch holds
  PStage<D, R>* st =
      reinterpret_cast<PStage<D, R>*>(smem_raw + p2g_crd_bytes<D, R>() + p2g_patch_bytes<D, R>(mibf));
  int tc[3];
  tile_coords<D>(H, t, tc);
  const int n0[3] = {tc[0] * TB - 1, tc[1] * TB - 1, D == 3 ? tc[2] * TB - 1 : 0};
  for (int i = threadIdx.x; i < nch * NODES; i += blockDim.x) (&patch[0][0])[i] = R(0.0);
  for (int i = threadIdx.x; i < D * PN; i += blockDim.x) {
    const int a = i / PN, o = i % PN;
    const int g = n0[a] + o;
    const double* ax = a == 0 ? A.gx : (a == 1 ? A.gy : A.gz);
    crd[a][o] = (g >= 0 && g < (int)H->N[a]) ? ax[g] : 0.0;
  }
  __syncthreads();
  const uint32_t Np = A.Np;
  const double ioh = P.one_over_dx;
  const R iohR = (R)ioh, apicD = (R)P.apicDinverse;
  const bool apic = P.flip_ratio < 0;
  const int lane = threadIdx.x & 31;
  // XS lanes share a stencil column, each owning HN = 4 / XS of its x nodes
  constexpr int COLS = D == 3 ? 16 : 4, LPP = COLS * XS, HN = 4 / XS;
  const int q = lane % LPP;
  const int iy = D == 3 ? ((q % COLS) >> 2) : q % COLS;
  const int iz = D == 3 ? ((q % COLS) & 3) : 0;
  const int h0 = (q / COLS) * HN;
  // group g takes the consecutive staged particles [g*LPP, (g+1)*LPP) of the
  // warp's 32, so groups work on different cells and their flushes rarely
  // meet on one patch node (interleaving them made both groups flush the same
  // cell at once, which measured slower despite fewer bank conflicts)
  // (with a chunk of blockDim / MTR_P2G_CHUNK_DIV particles, a group takes
  // LPP / MTR_P2G_CHUNK_DIV of them)
  static_assert(LPP % MTR_P2G_CHUNK_DIV == 0, "chunk divisor must divide the lanes per particle");
  constexpr int PPG = LPP / MTR_P2G_CHUNK_DIV;
  const int chunk = (int)blockDim.x / MTR_P2G_CHUNK_DIV;
  const int kbeg = ((int)threadIdx.x / LPP) * PPG, kend = kbeg + PPG;
  for (uint32_t c0 = pb; c0 < pe; c0 += chunk) {
    if constexpr (MTR_P2G_PAIR_STAGE && MTR_P2G_CHUNK_DIV == 2) {
      // phase 1, two threads per staged particle: thread t < chunk loads the
      // position, velocity and B and evaluates the weights; thread t + chunk
      // loads the stress and mu(I) and evaluates the weight derivatives
      const int role = (int)threadIdx.x >= chunk ? 1 : 0;
      const int slot = (int)threadIdx.x - role * chunk;
      const uint32_t s = c0 + (uint32_t)slot;
      PStage<D, R>& S = st[slot];
      int packed = -1;
      if (s < pe) {
        const uint32_t j = perm[s];
        double xp[3] = {0.0, 0.0, 0.0};
        int lb[3] = {0, 0, 0};
        bool oob = false;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          xp[a] = A.in.x[(size_t)a * Np + j];
          int b = (int)floor((xp[a] - H->org[a]) * ioh) - 1;
          b = b < 0 ? 0 : b;  // p2g.cpp:21-24 clamps at zero
          lb[a] = b - n0[a];
          if (lb[a] < 0 || lb[a] > PN - 4 || b + 3 >= (int)H->N[a]) oob = true;
        }
        if (role == 0) {
#pragma unroll
          for (int a = 0; a < D; ++a) {
            if constexpr (kFP64<R>) S.x[a] = xp[a];
            S.v[a] = A.in.v[(size_t)a * Np + j];
          }
#pragma unroll
          for (int q = 0; q < D * D; ++q)
            S.B[q] = apic ? (MTR_SCATTER_PRESCALE ? apicD * A.in.B[(size_t)q * Np + j] : A.in.B[(size_t)q * Np + j])
                          : R(0.0);
          if (oob) {
            raise_status(A.H, MTR_STATUS_STENCIL_OOB, A.in.id[j]);
          } else {
#pragma unroll
            for (int a = 0; a < D; ++a) {
#pragma unroll
              for (int o = 0; o < 4; ++o) {
                const double c = crd[a][lb[a] + o];
                S.w[a * 4 + o] = bspline_N<DEG>((R)((xp[a] - c) * ioh));
                if constexpr (!kFP64<R>) S.pd[a * 4 + o] = (R)(c - xp[a]);
              }
            }
            packed = lb[0] | (lb[1] << 4) | (lb[2] << 8);
          }
        } else {
#pragma unroll
          for (int q = 0; q < NS; ++q)
            S.tau[q] = MTR_SCATTER_PRESCALE ? iohR * A.in.tau[(size_t)q * Np + j] : A.in.tau[(size_t)q * Np + j];
          S.mui = mibf ? (R)((double)A.in.sc[(size_t)MTR_SCALAR_MUI * Np + j] - P.mui0) : R(0.0);
          if (!oob) {
#pragma unroll
            for (int a = 0; a < D; ++a) {
#pragma unroll
              for (int o = 0; o < 4; ++o) {
                const double c = crd[a][lb[a] + o];
                S.dw[a * 4 + o] = bspline_dN<DEG>((R)((xp[a] - c) * ioh));
              }
            }
          }
        }
      }
      if (role == 0) S.lb = packed;
    } else if ((int)threadIdx.x < chunk) {  // phase 1: stage one particle per thread
      const uint32_t s = c0 + threadIdx.x;
      PStage<D, R>& S = st[threadIdx.x];
      int packed = -1;
      if (s < pe) {
        const uint32_t j = perm[s];
        double xp[3] = {0.0, 0.0, 0.0};
        int lb[3] = {0, 0, 0};
        bool oob = false;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          xp[a] = A.in.x[(size_t)a * Np + j];
          if constexpr (kFP64<R>) S.x[a] = xp[a];
          S.v[a] = A.in.v[(size_t)a * Np + j];
          int b = (int)floor((xp[a] - H->org[a]) * ioh) - 1;
          b = b < 0 ? 0 : b;  // p2g.cpp:21-24 clamps at zero
          lb[a] = b - n0[a];
          if (lb[a] < 0 || lb[a] > PN - 4 || b + 3 >= (int)H->N[a]) oob = true;
        }
#pragma unroll
        for (int q = 0; q < D * D; ++q)
          S.B[q] = apic ? (MTR_SCATTER_PRESCALE ? apicD * A.in.B[(size_t)q * Np + j] : A.in.B[(size_t)q * Np + j])
                        : R(0.0);
#pragma unroll
        for (int q = 0; q < NS; ++q)
          S.tau[q] = MTR_SCATTER_PRESCALE ? iohR * A.in.tau[(size_t)q * Np + j] : A.in.tau[(size_t)q * Np + j];
        // MIBF friction is accumulated as the deviation from its initial value
        // mui0, so a uniform field reproduces mui0 exactly at every node
        S.mui = mibf ? (R)((double)A.in.sc[(size_t)MTR_SCALAR_MUI * Np + j] - P.mui0) : R(0.0);
        if (oob) {
          raise_status(A.H, MTR_STATUS_STENCIL_OOB, A.in.id[j]);
        } else {
#pragma unroll
          for (int a = 0; a < D; ++a) {
#pragma unroll
            for (int o = 0; o < 4; ++o) {
              const double c = crd[a][lb[a] + o];
              const R u = (R)((xp[a] - c) * ioh);
              S.w[a * 4 + o] = bspline_N<DEG>(u);
              S.dw[a * 4 + o] = bspline_dN<DEG>(u);
              if constexpr (!kFP64<R>) S.pd[a * 4 + o] = (R)(c - xp[a]);
            }
          }
          packed = lb[0] | (lb[1] << 4) | (lb[2] << 8);
        }
      }
      S.lb = packed;
    }
    __syncthreads();
    {  // phase 2: a lane owns one (iy, iz) stencil column and HN of its ix nodes
      R acc[HN][NCH];
#pragma unroll
      for (int h = 0; h < HN; ++h)
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) acc[h][ch] = R(0.0);
      int cur = -1;
      auto flush = [&]() {
        const int lbx = cur & 15, lby = (cur >> 4) & 15, lbz = cur >> 8;
#pragma unroll
        for (int hh = 0; hh < HN; ++hh) {
          const int h = h0 + hh;
          const int node = D == 3 ? ((lbx + h) * PN + (lby + iy)) * PN + (lbz + iz) : (lbx + h) * PN + (lby + iy);
#pragma unroll
          for (int ch = 0; ch < NCH; ++ch) {  // the friction accumulator stays zero without MIBF
            if (acc[hh][ch] != R(0.0)) atomicAdd(&patch[ch][node], acc[hh][ch]);
            acc[hh][ch] = R(0.0);
          }
        }
      };
      for (int k = kbeg; k < kend; ++k) {
        const PStage<D, R>& S = st[k];
        const int lbp = S.lb;
        if (lbp < 0) continue;
        if (lbp != cur) {
          if (cur >= 0) flush();
          cur = lbp;
        }
        const int lbx = lbp & 15, lby = (lbp >> 4) & 15, lbz = lbp >> 8;
        // tensor-product factors of this lane's column
        const R wy = S.w[4 + iy], dwy = S.dw[4 + iy];
        R wyz, G0, G1, G2 = R(0.0);
        if constexpr (D == 3) {
          const R wz = S.w[8 + iz], dwz = S.dw[8 + iz];
          wyz = wy * wz;
          if constexpr (MTR_SCATTER_PRESCALE) {
            G0 = wyz;
            G1 = dwy * wz;
            G2 = wy * dwz;
          } else {
            G0 = wyz * iohR;
            G1 = dwy * wz * iohR;
            G2 = wy * dwz * iohR;
          }
        } else {
          wyz = wy;
          G0 = MTR_SCATTER_PRESCALE ? wy : wy * iohR;
          G1 = MTR_SCATTER_PRESCALE ? dwy : dwy * iohR;
        }
        // force f_a = tau_a . grad w = dwx * Pf_a + wx * Qf_a
        R Pf[D], Qf[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          Pf[a] = sym_at<D>(S.tau, a, 0) * G0;
          R q = sym_at<D>(S.tau, a, 1) * G1;
          if constexpr (D == 3) q += sym_at<D>(S.tau, a, 2) * G2;
          Qf[a] = q;
        }
        // momentum per weight: v_a + apicD B_a . (x_i - x_p) = Tm_a + Sm_a * pdx
        const R pdy = stage_pd<D, R>(S, crd, 1, lby, iy);
        const R pdz = D == 3 ? stage_pd<D, R>(S, crd, D - 1, lbz, iz) : R(0.0);
        R Tm[D], Sm[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          if (apic) {
            R byz = S.B[a * D + 1] * pdy;
            if constexpr (D == 3) byz += S.B[a * D + 2] * pdz;
            Tm[a] = S.v[a] + (MTR_SCATTER_PRESCALE ? byz : apicD * byz);
            Sm[a] = MTR_SCATTER_PRESCALE ? S.B[a * D] : apicD * S.B[a * D];
          } else {
            Tm[a] = S.v[a];
            Sm[a] = R(0.0);
          }
        }
        const R mui = S.mui;
#pragma unroll
        for (int hh = 0; hh < HN; ++hh) {
          const int h = h0 + hh;
          const R wx = S.w[h], dwx = S.dw[h];
          const R weight = wx * wyz;
          if constexpr (MTR_SCATTER_SELECT) {
            // p2g.cpp:35 skips weights <= 1e-25; a zero weight adds nothing
            const R ws = weight > R(1e-25) ? weight : R(0.0);
            const R pdx = stage_pd<D, R>(S, crd, 0, lbx, h);
            acc[hh][0] += ws;
#pragma unroll
            for (int a = 0; a < D; ++a) acc[hh][1 + a] += ws * (Tm[a] + Sm[a] * pdx);
            if (mibf) acc[hh][1 + 2 * D] += mui * ws;
          } else if (weight > R(1e-25)) {
            const R pdx = stage_pd<D, R>(S, crd, 0, lbx, h);
            acc[hh][0] += weight;
#pragma unroll
            for (int a = 0; a < D; ++a) acc[hh][1 + a] += weight * (Tm[a] + Sm[a] * pdx);
            if (mibf) acc[hh][1 + 2 * D] += mui * weight;
          }
#pragma unroll
          for (int a = 0; a < D; ++a) acc[hh][1 + D + a] += dwx * Pf[a] + wx * Qf[a];
        }
      }
      if (cur >= 0) flush();
    }
    __syncthreads();
  }
  const uint32_t cap = A.cap_nodes;
  for (int n = threadIdx.x; n < NODES; n += blockDim.x) {
    uint32_t l;
    if (!patch_node<D>(H, n0, n, l)) continue;
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      if (ch >= nch) break;  // no friction channel without MIBF
      const R val = patch[ch][n];
      if (val != R(0.0)) atomicAdd(&A.acc[(size_t)ch * cap + l], val);
    }
  }
}

template <int D, int DEG, typename R, int XS = 1>
__global__ void __launch_bounds__(kMaxTileThreads) k_p2g_w(StepArgsT<R> A, const uint32_t* __restrict__ perm) {
  p2g_w_body<D, DEG, R, XS>(A, perm, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// 5b. periodic copies (pbc.cpp:37-85): a particle within 4 dx of x = Lx (else
// of x = 0) also scatters mass, momentum and force from x - Lx (else x + Lx),
// with the same stencil and formulas as P2G (p2g.cpp:6-100,
// explicit_euler_update.cpp:15-77).  Few particles have a copy; each one is a
// thread with global atomics.
// ---------------------------------------------------------------------------
template <int D, int DEG, typename R>
__global__ void __launch_bounds__(256) k_p2g_periodic(StepArgsT<R> A) {
  const StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const DevParams& P = *A.P;
  constexpr int NS = Sym<D>::n, KN = D == 3 ? 4 : 1;
  const uint32_t Np = A.Np, cap = A.cap_nodes;
  const double ioh = P.one_over_dx, lim = 4.0 * P.dx, Lx = P.L[0], apicD = P.apicDinverse;
  const bool apic = P.flip_ratio < 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < Np; i += gridDim.x * blockDim.x) {
    double xp[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < D; ++a) xp[a] = A.in.x[(size_t)a * Np + i];
    double diff = Lx - xp[0];
    if (diff < lim && diff > 0) {
      xp[0] = -diff;
    } else {
      diff = xp[0];
      if (!(diff < lim && diff >= 0)) continue;
      xp[0] = Lx + diff;
    }
    double vp[3] = {0.0, 0.0, 0.0}, Bm[D][D], tau[NS];
#pragma unroll
    for (int a = 0; a < D; ++a) vp[a] = A.in.v[(size_t)a * Np + i];
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) Bm[r][c] = apic ? (double)A.in.B[(size_t)(r * D + c) * Np + i] : 0.0;
#pragma unroll
    for (int q = 0; q < NS; ++q) tau[q] = A.in.tau[(size_t)q * Np + i];
    int base[3] = {0, 0, 0};
    bool oob = false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      int b = (int)floor((xp[a] - H->org[a]) * ioh) - 1;
      b = b < 0 ? 0 : b;  // p2g.cpp:21-24 clamps at zero
      base[a] = b;
      if (b + 3 >= (int)H->N[a]) oob = true;
    }
    if (oob) {
      raise_status(A.H, MTR_STATUS_STENCIL_OOB, A.in.id[i]);
      continue;
    }
    double w[3][4], dw[3][4], crd[3][4];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const double* ax = a == 0 ? A.gx : (a == 1 ? A.gy : A.gz);
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        crd[a][o] = ax[base[a] + o];
        const double u = (xp[a] - crd[a][o]) * ioh;
        w[a][o] = bspline_N<DEG>(u);
        dw[a][o] = bspline_dN<DEG>(u);
      }
    }
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int kk = 0; kk < KN; ++kk) {
          const uint32_t l = node_index(H, base[0] + ii, base[1] + jj, D == 3 ? base[2] + kk : 0);
          const double wxy = w[0][ii] * w[1][jj];
          const double weight = D == 3 ? wxy * w[2][kk] : wxy;
          if (weight > 1e-25) {
            atomicAdd(&A.acc[l], (R)weight);
            const double pd[3] = {crd[0][ii] - xp[0], crd[1][jj] - xp[1], D == 3 ? crd[2][kk] - xp[2] : 0.0};
#pragma unroll
            for (int a = 0; a < D; ++a) {
              double bv = Bm[a][0] * pd[0];
#pragma unroll
              for (int c = 1; c < D; ++c) bv += Bm[a][c] * pd[c];
              atomicAdd(&A.acc[(size_t)(1 + a) * cap + l], (R)(weight * (vp[a] + apicD * bv)));
            }
          }
          double g[3];
          if constexpr (D == 3) {
            g[0] = dw[0][ii] * w[1][jj] * w[2][kk] * ioh;
            g[1] = w[0][ii] * dw[1][jj] * w[2][kk] * ioh;
            g[2] = w[0][ii] * w[1][jj] * dw[2][kk] * ioh;
          } else {
            g[0] = dw[0][ii] * w[1][jj] * ioh;
            g[1] = w[0][ii] * dw[1][jj] * ioh;
          }
#pragma unroll
          for (int a = 0; a < D; ++a) {
            double f = sym_at<D>(tau, a, 0) * g[0];
#pragma unroll
            for (int c = 1; c < D; ++c) f += sym_at<D>(tau, a, c) * g[c];
            if (f != 0.0) atomicAdd(&A.acc[(size_t)(1 + D + a) * cap + l], (R)f);
          }
        }
  }
}

// ---------------------------------------------------------------------------
// 6. grid update, one thread per node (arithmetic in FP64 on both paths)
// ---------------------------------------------------------------------------
template <int D, typename R>
__device__ __forceinline__ void grid_body(const StepArgsT<R>& A, const uint32_t bid, const uint32_t nblk) {
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const DevParams& P = *A.P;
  const uint32_t G = H->G, cap = A.cap_nodes;
  const double dt = H->dt;
  const double dtpv = dt * P.particle_volume;
  double dtg[3];
#pragma unroll
  for (int a = 0; a < D; ++a) dtg[a] = dt * H->gravity[a];
  __shared__ mtr_plate plates[MTR_MAXP];
  for (int i = threadIdx.x; i < P.nplates; i += blockDim.x) plates[i] = H->plates[i];
  __syncthreads();
  double sum_m = 0.0, sum_p[3] = {0.0, 0.0, 0.0};  // mass and momentum balance (simulation.cpp:292-333)
  for (uint32_t l = bid * blockDim.x + threadIdx.x; l < G; l += nblk * blockDim.x) {
    // every load of the node first, ahead of the branches on its mass: one
    // round of memory latency per node instead of several in a row
    const double mraw = A.acc[l];
    double pacc[3] = {0, 0, 0}, facc[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
      pacc[a] = A.acc[(size_t)(1 + a) * cap + l];
      facc[a] = A.acc[(size_t)(1 + D + a) * cap + l];
    }
    const double fracc = P.use_mibf ? (double)A.acc[(size_t)(1 + 2 * D) * cap + l] : 0.0;
    const uint32_t k = D == 3 ? l % H->N[2] : 0;
    const uint32_t r = D == 3 ? l / H->N[2] : l;
    const uint32_t jj = r % H->N[1], i = r / H->N[1];
    const double Xi0 = A.gx[i], Xi1 = A.gy[jj], Xi2 = D == 3 ? A.gz[k] : 0.0;
    double v[3] = {0, 0, 0}, vold[3] = {0, 0, 0};
    double fric = 0.0;
    sum_m += mraw;
    if (mraw > 0) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        sum_p[a] += pacc[a];
        v[a] = pacc[a] / mraw;
      }
    }
    if (P.use_mibf) fric = P.mui0 + fracc / mraw;
    const double mi = mraw * P.particle_mass;
    double fl[3] = {0, 0, 0};
    if (mi > 0) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        double inc = -dtpv * facc[a] / mi + dtg[a];
        vold[a] = v[a];
        v[a] = vold[a] + inc;
      }
      double Xi[3] = {Xi0, Xi1, Xi2};
      if (!boundary_collision<D>(P, plates, fric, Xi, dt, v)) raise_status(H, MTR_STATUS_BAD_BC, 0xffffffffu);
#pragma unroll
      for (int a = 0; a < D; ++a) fl[a] = v[a] - vold[a];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
      A.nv[(size_t)a * cap + l] = v[a];
      A.nflip[(size_t)a * cap + l] = (R)fl[a];
    }
    A.nmass[l] = (R)mi;
    if (P.use_mibf) A.nfric[l] = (R)fric;
#pragma unroll
    for (int ch = 0; ch < Tiling<D>::NCH; ++ch) A.acc[(size_t)ch * cap + l] = R(0.0);  // ready for the next step
  }
  block_add(sum_m * P.particle_mass, &H->grid_mass);
#pragma unroll
  for (int a = 0; a < D; ++a) block_add(sum_p[a] * P.particle_mass, &H->grid_mom[a]);
}

template <int D, typename R>
__global__ void __launch_bounds__(256) k_grid(StepArgsT<R> A) {
  grid_body<D, R>(A, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// particle I/O helpers (the deformation update and return mapping are FP64)
// ---------------------------------------------------------------------------
template <int D>
struct PLoad {
  double x[3], v[3], F[D][D];
  PScalars s;
  uint32_t id;
};

template <int D, typename R>
__device__ __forceinline__ void load_particle(const PBufT<R>& b, uint32_t Np, uint32_t j, PLoad<D>& p) {
#pragma unroll
  for (int a = 0; a < 3; ++a) p.x[a] = p.v[a] = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    p.x[a] = b.x[(size_t)a * Np + j];
    p.v[a] = b.v[(size_t)a * Np + j];
  }
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) {
      if constexpr (kFP64<R>)
        p.F[r][c] = b.F[(size_t)(r * D + c) * Np + j];
      else
        p.F[r][c] = (double)b.F[(size_t)(r * D + c) * Np + j] + (r == c ? 1.0 : 0.0);
    }
  p.s.eps_pl_dev = b.sc[(size_t)MTR_SCALAR_EPS_PL_DEV * Np + j];
  p.s.eps_pl_vol = b.sc[(size_t)MTR_SCALAR_EPS_PL_VOL * Np + j];
  p.s.eps_pl_vol_pradhana = b.sc[(size_t)MTR_SCALAR_EPS_PL_VOL_PRADHANA * Np + j];
  p.s.delta_gamma = 0.0;  // deformation_update.cpp:13 zeroes it every step
  p.s.viscosity = b.sc[(size_t)MTR_SCALAR_VISCOSITY * Np + j];
  p.s.muI = b.sc[(size_t)MTR_SCALAR_MUI * Np + j];
  p.id = b.id[j];
}

template <int D, typename R>
__device__ __forceinline__ void store_defgrad(const PBufT<R>& b, uint32_t Np, uint32_t s, const double (&F)[D][D],
                                              const PScalars& sc, const double* tau) {
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) {
      if constexpr (kFP64<R>)
        b.F[(size_t)(r * D + c) * Np + s] = F[r][c];
      else
        b.F[(size_t)(r * D + c) * Np + s] = (R)(F[r][c] - (r == c ? 1.0 : 0.0));
    }
  b.sc[(size_t)MTR_SCALAR_EPS_PL_DEV * Np + s] = (R)sc.eps_pl_dev;
  b.sc[(size_t)MTR_SCALAR_EPS_PL_VOL * Np + s] = (R)sc.eps_pl_vol;
  b.sc[(size_t)MTR_SCALAR_EPS_PL_VOL_PRADHANA * Np + s] = (R)sc.eps_pl_vol_pradhana;
  b.sc[(size_t)MTR_SCALAR_DELTA_GAMMA * Np + s] = (R)sc.delta_gamma;
  b.sc[(size_t)MTR_SCALAR_VISCOSITY * Np + s] = (R)sc.viscosity;
  b.sc[(size_t)MTR_SCALAR_MUI * Np + s] = (R)sc.muI;
#pragma unroll
  for (int q = 0; q < Sym<D>::n; ++q) b.tau[(size_t)q * Np + s] = (R)tau[q];
}

// the end of positionUpdate (position_update.cpp:26-41): periodic wrap in x,
// then the hard-coded teleport hook
__device__ __forceinline__ void wrap_and_teleport(const DevParams& P, double (&xn)[3]) {
  if (P.pbc) {
    if (xn[0] > P.L[0])
      xn[0] = xn[0] - P.L[0];
    else if (xn[0] < 0)
      xn[0] = P.L[0] + xn[0];
  }
  if (P.change_particle_positions && xn[0] > 0.8) {
    xn[0] = -0.1;
    xn[1] += 0.27;
  }
}

// velocity blend of position_update.cpp:14-24 / musl.cpp:15-22
__device__ __forceinline__ double blend_v(double fr, double v, double fl, double pic) {
  if (fr < -1) return pic;
  if (fr < 0) return (-fr) * (v + fl) + (1 - (-fr)) * pic;
  return fr * (v + fl) + (1 - fr) * pic;
}

// F_trial = F + dt * gradv * F (deformation_update.cpp:42-44), then the
// return mapping; writes F, scalars and tau into the out buffer at slot s.
template <int D, typename R, int PM>
__device__ __forceinline__ void defgrad_and_store(const StepArgsT<R>& A, uint32_t s, double dt, PLoad<D>& p,
                                                  const R (&gv)[D][D], uint32_t& flags, bool& plastic) {
  double T1[D][D], T2[D][D];
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) T1[r][c] = dt * (double)gv[r][c];
  mat_mul<D>(T1, p.F, T2);
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) p.F[r][c] = p.F[r][c] + T2[r][c];
  double tau[Sym<D>::n];
  plastic = return_map<D, PM, MTR_SYM_SVD != 0>(*A.P, dt, p.F, p.s, tau, flags);
  store_defgrad<D, R>(A.out, A.Np, s, p.F, p.s, tau);
}

// ---------------------------------------------------------------------------
// Tile-structured gathers.  A tile block first copies the node values its
// particles' stencils can reach (the PN^D patch of the tile) from the node
// arrays into shared memory, then every particle gathers from there.
// ---------------------------------------------------------------------------

// copies NF fields of D components each, src[f] = [D][cap] node arrays
template <int D, int NF, typename R>
__device__ __forceinline__ void load_node_patch(const StepCommon& A, const StepHeader* H, const int (&n0)[3],
                                                const R* const (&src)[NF], R* dst /*[NF*D][NODES]*/) {
  constexpr int NODES = Tiling<D>::NODES;
  const uint32_t cap = A.cap_nodes;
  for (int n = threadIdx.x; n < NODES; n += blockDim.x) {
    uint32_t l = 0;
    const bool in = patch_node<D>(H, n0, n, l);
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int a = 0; a < D; ++a) dst[(f * D + a) * NODES + n] = in ? src[f][(size_t)a * cap + l] : R(0.0);
  }
}

// Reference velocity of a tile: the FP64 node velocity at the patch node
// nearest the tile centre (zero outside the grid, and always zero on the FP64
// path, which gathers the node velocities themselves).
template <int D, typename R>
__device__ __forceinline__ void tile_vref(const StepCommon& A, const StepHeader* H, const int (&n0)[3],
                                          const double* src, double (&vref)[3]) {
  vref[0] = vref[1] = vref[2] = 0.0;
  if constexpr (!kFP64<R>) {
    constexpr int c = 1 + Tiling<D>::TB / 2;
    const int gi = n0[0] + c, gj = n0[1] + c, gk = D == 3 ? n0[2] + c : 0;
    if (gi < (int)H->N[0] && gj < (int)H->N[1] && gk < (int)H->N[2]) {
      const uint32_t l = node_index(H, gi, gj, gk);
#pragma unroll
      for (int a = 0; a < D; ++a) vref[a] = src[(size_t)a * A.cap_nodes + l];
    }
  }
}

// node velocity patch as deviations from vref, rounded to R
template <int D, typename R>
__device__ __forceinline__ void load_velocity_patch(const StepCommon& A, const StepHeader* H, const int (&n0)[3],
                                                    const double* src, const double (&vref)[3],
                                                    R* dst /*[D][NODES]*/) {
  constexpr int NODES = Tiling<D>::NODES;
  const uint32_t cap = A.cap_nodes;
  for (int n = threadIdx.x; n < NODES; n += blockDim.x) {
    uint32_t l = 0;
    const bool in = patch_node<D>(H, n0, n, l);
#pragma unroll
    for (int a = 0; a < D; ++a) {
      if constexpr (kFP64<R>)
        dst[a * NODES + n] = in ? src[(size_t)a * cap + l] : 0.0;
      else
        dst[a * NODES + n] = in ? (R)(src[(size_t)a * cap + l] - vref[a]) : R(0.0);
    }
  }
}

// G2P gather (g2p.cpp:24-77) and velocity gradient (deformation_update.cpp:17-40)
// from a shared node patch; lb = stencil base relative to the patch origin.
// Sums are factorised over the tensor-product stencil.  The offsets and the
// spline argument are formed in FP64 from the FP64 position, then rounded to
// R.  pv holds node velocities minus vref: B-spline weights sum to one and
// reproduce linears, so pic = vref + sum w dv, while B and grad v need the
// deviations only.
// The sums over the stencil's x layers ii0 .. ii1-1: ps = sum w v (deviations
// from vref on the mixed path), B, flip and grad v (unscaled).
template <int D, int DEG, bool GRADV, typename R>
__device__ __forceinline__ void gather_sums(const R* pv, const R* pf, const double (*crd)[Tiling<D>::PN],
                                            const int (&lb)[3], const double (&xp)[3], double ioh, R (&ps)[3],
                                            R (&Bp)[D][D], R (&flp)[3], R (&gv)[D][D], bool want_b, bool want_flip,
                                            int ii0, int ii1) {
  constexpr int PN = Tiling<D>::PN, NODES = Tiling<D>::NODES;
  R w[3][4], dw[3][4], pd[3][4];
#pragma unroll
  for (int a = 0; a < D; ++a)
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const double c = crd[a][lb[a] + o];
      const R u = (R)((xp[a] - c) * ioh);
      w[a][o] = bspline_N<DEG>(u);
      dw[a][o] = GRADV ? bspline_dN<DEG>(u) : R(0.0);
      pd[a][o] = (R)(c - xp[a]);
    }
#pragma unroll
  for (int a = 0; a < 3; ++a) ps[a] = flp[a] = R(0.0);
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int c = 0; c < D; ++c) Bp[r][c] = gv[r][c] = R(0.0);
  constexpr int KN = D == 3 ? 4 : 1;
  // the x layers of the stencil stay a loop: unrolling all 64 nodes made
  // the return-mapping kernels that call this too large for the instruction
  // cache
#pragma unroll 1
  for (int ii = ii0; ii < ii1; ++ii)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const R wxy = w[0][ii] * w[1][jj];
      const R gx_ = dw[0][ii] * w[1][jj], gy_ = w[0][ii] * dw[1][jj];
#pragma unroll
      for (int kk = 0; kk < KN; ++kk) {
        const int node = D == 3 ? ((lb[0] + ii) * PN + (lb[1] + jj)) * PN + (lb[2] + kk) : (lb[0] + ii) * PN + (lb[1] + jj);
        const R weight = D == 3 ? wxy * w[2][kk] : wxy;
        R vi[D];
#pragma unroll
        for (int a = 0; a < D; ++a) vi[a] = pv[a * NODES + node];
#pragma unroll
        for (int a = 0; a < D; ++a) ps[a] += vi[a] * weight;
        if (want_b) {
          R wpd[3] = {weight * pd[0][ii], weight * pd[1][jj], D == 3 ? weight * pd[2][kk] : R(0.0)};
#pragma unroll
          for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) Bp[r][c] += vi[r] * wpd[c];
        }
        if (want_flip) {
#pragma unroll
          for (int a = 0; a < D; ++a) flp[a] += pf[a * NODES + node] * weight;
        }
        if (GRADV) {
          R g[3];
          if constexpr (D == 3) {
            g[0] = gx_ * w[2][kk];
            g[1] = gy_ * w[2][kk];
            g[2] = wxy * dw[2][kk];
          } else {
            g[0] = gx_;
            g[1] = gy_;
          }
#pragma unroll
          for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) gv[r][c] += vi[r] * g[c];
        }
      }
    }
}

// pic = vref + ps (the FP64 path gathers the velocities themselves), grad v
// scaled by 1/dx
template <int D, bool GRADV, typename R>
__device__ __forceinline__ void gather_finish(const R (&ps)[3], const double (&vref)[3], double ioh, double (&pic)[3],
                                              R (&gv)[D][D]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if constexpr (kFP64<R>)
      pic[a] = ps[a];
    else
      pic[a] = vref[a] + (double)ps[a];
  }
  if (GRADV) {
    const R iohR = (R)ioh;
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) gv[r][c] *= iohR;
  }
}

template <int D, int DEG, bool GRADV, typename R>
__device__ __forceinline__ void gather_patch(const R* pv, const R* pf, const double (*crd)[Tiling<D>::PN],
                                             const int (&lb)[3], const double (&xp)[3], double ioh,
                                             const double (&vref)[3], double (&pic)[3], R (&Bp)[D][D], R (&flp)[3],
                                             R (&gv)[D][D], bool want_b, bool want_flip) {
  R ps[3];
  gather_sums<D, DEG, GRADV, R>(pv, pf, crd, lb, xp, ioh, ps, Bp, flp, gv, want_b, want_flip, 0, 4);
  gather_finish<D, GRADV, R>(ps, vref, ioh, pic, gv);
}

// ---------------------------------------------------------------------------
// 7a. USL: G2P + deformation update + return mapping + position update, one
// block per tile, node patch in shared memory.
// ---------------------------------------------------------------------------
template <int D, int DEG, typename R, int PM>
__device__ __forceinline__ void g2p_t_body(const StepArgsT<R>& A, const uint32_t* __restrict__ perm, const uint32_t bid, const uint32_t nblk) {
  using TL = Tiling<D>;
  constexpr int PN = TL::PN, NODES = TL::NODES;
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const uint32_t t = bid;
  if (t >= H->ntiles) return;
  const uint32_t pb = A.tile_begin[t], pe = A.tile_end[t];
  if (pb >= pe) return;
  const DevParams& P = *A.P;
  __shared__ R pv[2 * D * NODES];
  __shared__ double crd[3][PN];
  int n0[3];
  load_tile_setup<D>(A, H, t, n0, crd);
  double vref[3];
  tile_vref<D, R>(A, H, n0, A.nv, vref);
  load_velocity_patch<D, R>(A, H, n0, A.nv, vref, pv);
  const R* const src[1] = {A.nflip};
  load_node_patch<D, 1, R>(A, H, n0, src, pv + D * NODES);
  __syncthreads();
  const uint32_t Np = A.Np;
  const double dt = H->dt, fr = P.flip_ratio, ioh = P.one_over_dx;
  unsigned nplastic = 0;
  for (uint32_t s = pb + threadIdx.x; s < pe; s += blockDim.x) {
    const uint32_t j = perm[s];
    PLoad<D> p;
    load_particle<D, R>(A.in, Np, j, p);
    double pic[3];
    R flp[3], Bp[D][D], gv[D][D];
    int lb[3];
    if (local_base<D>(H, p.x, ioh, n0, false, lb)) {
      gather_patch<D, DEG, true, R>(pv, pv + D * NODES, crd, lb, p.x, ioh, vref, pic, Bp, flp, gv, fr < 0, fr >= -1);
    } else {
      raise_status(H, MTR_STATUS_STENCIL_OOB, p.id);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        pic[a] = 0.0;
        flp[a] = R(0.0);
      }
#pragma unroll
      for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) Bp[r][c] = gv[r][c] = R(0.0);
    }
    uint32_t f = 0;
    bool plastic = false;
    defgrad_and_store<D, R, PM>(A, s, dt, p, gv, f, plastic);
    if (f) raise_status(H, f, p.id);
    nplastic += plastic ? 1u : 0u;
    double xn[3], vn[3];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      xn[a] = p.x[a] + dt * pic[a];
      vn[a] = blend_v(fr, p.v[a], (double)flp[a], pic[a]);
    }
    wrap_and_teleport(P, xn);
#pragma unroll
    for (int a = 0; a < D; ++a) {
      A.out.x[(size_t)a * Np + s] = xn[a];
      A.out.v[(size_t)a * Np + s] = (R)vn[a];
    }
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) A.out.B[(size_t)(r * D + c) * Np + s] = (fr < 0) ? Bp[r][c] : R(0.0);
    A.out.id[s] = p.id;
    if (P.store_pic_flip) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        A.pic[(size_t)a * Np + s] = (R)pic[a];
        A.flip[(size_t)a * Np + s] = (fr >= -1) ? flp[a] : R(0.0);
      }
    }
  }
  block_count(nplastic, &H->plastic_count);
}

template <int D, int DEG, typename R, int PM = -1>
__global__ void __launch_bounds__(kChunk, MTR_G2P_MIN_BLOCKS) k_g2p_t(StepArgsT<R> A, const uint32_t* __restrict__ perm) {
  g2p_t_body<D, DEG, R, PM>(A, perm, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// 7b. MUSL (musl.cpp:6-96), one block per tile.  Phase 1 (thread per
// particle): gather pic/B/flip from the shared node patch, blend v, write
// x + dt pic, v, B; stage v_new, B_new and the re-scatter weights.  Phase 2
// (lane groups owning stencil columns, as in P2G): accumulate
// v_p + B D^-1 (x_i - x_p) per cell in registers, add once per cell to the
// shared re-projection patch, flush with one global atomic per node.
// ---------------------------------------------------------------------------
template <int D, typename R = double>
struct MStage {
  double x[D], v[D], B[D * D], w[D * 4];
  int lb;
  int pad;
};

template <int D>
struct MStage<D, float> {
  float pd[D * 4], v[D], B[D * D], w[D * 4];
  int lb;
};

template <int D, typename R>
__device__ __forceinline__ R stage_pd(const MStage<D, R>& S, const double (*crd)[Tiling<D>::PN], int a, int lba,
                                      int o) {
  if constexpr (kFP64<R>)
    return crd[a][lba + o] - S.x[a];
  else
    return S.pd[a * 4 + o];
}

template <int D, typename R>
constexpr size_t musl_crd_bytes() {
  return align16(sizeof(double) * 3 * Tiling<D>::PN);
}
template <int D, typename R>
constexpr size_t musl_patch_bytes() {
  return align16(sizeof(R) * 3 * D * Tiling<D>::NODES);
}
template <int D, typename R>
constexpr size_t musl_smem_bytes(int threads) {
  return musl_crd_bytes<D, R>() + musl_patch_bytes<D, R>() + stage_bytes<MStage<D, R>, MTR_MUSL_CHUNK_DIV>(threads);
}

template <int D, int DEG, typename R, int XS = 1>
__device__ __forceinline__ void g2p_musl_w_body(const StepArgsT<R>& A, const uint32_t* __restrict__ perm, const uint32_t bid, const uint32_t nblk) {
  using TL = Tiling<D>;
  constexpr int PN = TL::PN, NODES = TL::NODES;
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const uint32_t t = bid;
  if (t >= H->ntiles) return;
  const uint32_t pb = A.tile_begin[t], pe = A.tile_end[t];
  if (pb >= pe) return;
  const DevParams& P = *A.P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double(*crd)[PN] = reinterpret_cast<double(*)[PN]>(smem_raw);
  R* pv = reinterpret_cast<R*>(smem_raw + musl_crd_bytes<D, R>());  // [2D][NODES] node v, flip
  R(*vsum)[NODES] = reinterpret_cast<R(*)[NODES]>(pv + 2 * D * NODES);  // [D][NODES]
  MStage<D, R>* st = reinterpret_cast<MStage<D, R>*>(smem_raw + musl_crd_bytes<D, R>() + musl_patch_bytes<D, R>());
  int n0[3];
  load_tile_setup<D>(A, H, t, n0, crd);
  double vref[3];
  tile_vref<D, R>(A, H, n0, A.nv, vref);
  load_velocity_patch<D, R>(A, H, n0, A.nv, vref, pv);
  const R* const src[1] = {A.nflip};
  load_node_patch<D, 1, R>(A, H, n0, src, pv + D * NODES);
  for (int i = threadIdx.x; i < D * NODES; i += blockDim.x) (&vsum[0][0])[i] = R(0.0);
  __syncthreads();
  const uint32_t Np = A.Np;
  const double dt = H->dt, fr = P.flip_ratio, ioh = P.one_over_dx;
  const R apicD = (R)P.apicDinverse;
  const bool apic = fr < 0;
  const int lane = threadIdx.x & 31;
  constexpr int COLS = D == 3 ? 16 : 4, LPP = COLS * XS, HN = 4 / XS;  // as in k_p2g_w
  const int q = lane % LPP;
  const int iy = D == 3 ? ((q % COLS) >> 2) : q % COLS;
  const int iz = D == 3 ? ((q % COLS) & 3) : 0;
  const int h0 = (q / COLS) * HN;
  // a staged particle after its gather: velocity blend, position update,
  // outputs and the re-scatter stencil; returns the packed stencil base
  // (-1: none)
  auto finish = [&](MStage<D, R>& S, uint32_t s, uint32_t pid, const double (&xp)[3], const double (&vp)[3],
                    const double (&pic)[3], const R (&flp)[3], const R (&Bp)[D][D], bool ok) -> int {
    int packed = -1;
    double xn[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const double vn = blend_v(fr, vp[a], (double)flp[a], pic[a]);
      if constexpr (kFP64<R>) S.x[a] = xp[a];
      S.v[a] = (R)vn;
      xn[a] = xp[a] + dt * pic[a];  // positionUpdate: x + dt pic
      A.out.v[(size_t)a * Np + s] = (R)vn;
    }
    wrap_and_teleport(P, xn);
#pragma unroll
    for (int a = 0; a < D; ++a) A.out.x[(size_t)a * Np + s] = xn[a];
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const R b = apic ? Bp[r][c] : R(0.0);
        A.out.B[(size_t)(r * D + c) * Np + s] = b;
        S.B[r * D + c] = MTR_SCATTER_PRESCALE ? apicD * b : b;
      }
    A.out.id[s] = pid;
    if (P.store_pic_flip) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        A.pic[(size_t)a * Np + s] = (R)pic[a];
        A.flip[(size_t)a * Np + s] = (fr >= -1) ? flp[a] : R(0.0);
      }
    }
    // re-scatter stencil, base clamped at zero like P2G (musl.cpp:35-40)
    int lbs[3];
    if (ok && local_base<D>(H, xp, ioh, n0, true, lbs)) {
#pragma unroll
      for (int a = 0; a < D; ++a)
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          const double c = crd[a][lbs[a] + o];
          S.w[a * 4 + o] = bspline_N<DEG>((R)((xp[a] - c) * ioh));
          if constexpr (!kFP64<R>) S.pd[a * 4 + o] = (R)(c - xp[a]);
        }
      packed = lbs[0] | (lbs[1] << 4) | (lbs[2] << 8);
    } else if (ok) {
      raise_status(H, MTR_STATUS_STENCIL_OOB, pid);
    }
    return packed;
  };
  // consecutive particles per lane group, as in k_p2g_w
  static_assert(LPP % MTR_MUSL_CHUNK_DIV == 0, "chunk divisor must divide the lanes per particle");
  constexpr int PPG = LPP / MTR_MUSL_CHUNK_DIV;
  const int chunk = (int)blockDim.x / MTR_MUSL_CHUNK_DIV;
  const int kbeg = ((int)threadIdx.x / LPP) * PPG, kend = kbeg + PPG;
  for (uint32_t c0 = pb; c0 < pe; c0 += chunk) {
    if ((int)threadIdx.x < chunk) {  // phase 1
      const uint32_t s = c0 + threadIdx.x;
      MStage<D, R>& S = st[threadIdx.x];
      int packed = -1;
      if (s < pe) {
        const uint32_t j = perm[s];
        double xp[3] = {0, 0, 0}, vp[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < D; ++a) {
          xp[a] = A.in.x[(size_t)a * Np + j];
          vp[a] = A.in.v[(size_t)a * Np + j];
        }
        const uint32_t pid = A.in.id[j];
        double pic[3];
        R flp[3], Bp[D][D], gv[D][D];
        int lb[3];
        const bool ok = local_base<D>(H, xp, ioh, n0, false, lb);
        if (ok) {
          gather_patch<D, DEG, false, R>(pv, pv + D * NODES, crd, lb, xp, ioh, vref, pic, Bp, flp, gv, apic,
                                         fr >= -1);
        } else {
          raise_status(H, MTR_STATUS_STENCIL_OOB, pid);
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            pic[a] = 0.0;
            flp[a] = R(0.0);
          }
#pragma unroll
          for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) Bp[r][c] = R(0.0);
        }
        packed = finish(S, s, pid, xp, vp, pic, flp, Bp, ok);
      }
      S.lb = packed;
    }
    __syncthreads();
    {  // phase 2
      R acc[HN][D];
#pragma unroll
      for (int h = 0; h < HN; ++h)
#pragma unroll
        for (int a = 0; a < D; ++a) acc[h][a] = R(0.0);
      int cur = -1;
      auto flush = [&]() {
        const int lbx = cur & 15, lby = (cur >> 4) & 15, lbz = cur >> 8;
#pragma unroll
        for (int hh = 0; hh < HN; ++hh) {
          const int h = h0 + hh;
          const int node = D == 3 ? ((lbx + h) * PN + (lby + iy)) * PN + (lbz + iz) : (lbx + h) * PN + (lby + iy);
#pragma unroll
          for (int a = 0; a < D; ++a) {
            if (acc[hh][a] != R(0.0)) atomicAdd(&vsum[a][node], acc[hh][a]);
            acc[hh][a] = R(0.0);
          }
        }
      };
      for (int k = kbeg; k < kend; ++k) {
        const MStage<D, R>& S = st[k];
        const int lbp = S.lb;
        if (lbp < 0) continue;
        if (lbp != cur) {
          if (cur >= 0) flush();
          cur = lbp;
        }
        const int lbx = lbp & 15, lby = (lbp >> 4) & 15, lbz = lbp >> 8;
        const R wyz = D == 3 ? S.w[4 + iy] * S.w[8 + iz] : S.w[4 + iy];
        const R pdy = stage_pd<D, R>(S, crd, 1, lby, iy);
        const R pdz = D == 3 ? stage_pd<D, R>(S, crd, D - 1, lbz, iz) : R(0.0);
        R Tm[D], Sm[D];
#pragma unroll
        for (int a = 0; a < D; ++a) {
          if (apic) {
            R byz = S.B[a * D + 1] * pdy;
            if constexpr (D == 3) byz += S.B[a * D + 2] * pdz;
            Tm[a] = S.v[a] + (MTR_SCATTER_PRESCALE ? byz : apicD * byz);
            Sm[a] = MTR_SCATTER_PRESCALE ? S.B[a * D] : apicD * S.B[a * D];
          } else {
            Tm[a] = S.v[a];
            Sm[a] = R(0.0);
          }
        }
#pragma unroll
        for (int hh = 0; hh < HN; ++hh) {
          const int h = h0 + hh;
          const R weight = S.w[h] * wyz;
          if constexpr (MTR_SCATTER_SELECT) {
            const R ws = weight > R(1e-25) ? weight : R(0.0);  // musl.cpp:51 skips weights <= 1e-25
            const R pdx = stage_pd<D, R>(S, crd, 0, lbx, h);
#pragma unroll
            for (int a = 0; a < D; ++a) acc[hh][a] += ws * (Tm[a] + Sm[a] * pdx);
          } else {
            if (!(weight > R(1e-25))) continue;
            const R pdx = stage_pd<D, R>(S, crd, 0, lbx, h);
#pragma unroll
            for (int a = 0; a < D; ++a) acc[hh][a] += weight * (Tm[a] + Sm[a] * pdx);
          }
        }
      }
      if (cur >= 0) flush();
    }
    __syncthreads();
  }
  const uint32_t cap = A.cap_nodes;
  for (int n = threadIdx.x; n < NODES; n += blockDim.x) {
    uint32_t l;
    if (!patch_node<D>(H, n0, n, l)) continue;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const R val = vsum[a][n];
      if (val != R(0.0)) atomicAdd(&A.v2[(size_t)a * cap + l], (double)val);
    }
  }
}

template <int D, int DEG, typename R, int XS = 1>
__global__ void __launch_bounds__(MTR_MUSL_MAX_THREADS, MTR_MUSL_MIN_BLOCKS)
    k_g2p_musl_w(StepArgsT<R> A, const uint32_t* __restrict__ perm) {
  g2p_musl_w_body<D, DEG, R, XS>(A, perm, blockIdx.x, gridDim.x);
}

// musl.cpp:80-95: v2 /= (m_i / m_p) (zero where m_i == 0)
template <int D, typename R>
__device__ __forceinline__ void musl_norm_body(const StepArgsT<R>& A, const uint32_t bid, const uint32_t nblk) {
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const uint32_t G = H->G, cap = A.cap_nodes;
  const double mp = A.P->particle_mass;
  for (uint32_t l = bid * blockDim.x + threadIdx.x; l < G; l += nblk * blockDim.x) {
    const double mi = A.nmass[l];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      double* p = &A.v2[(size_t)a * cap + l];
      *p = (mi > 0) ? *p / (mi / mp) : 0.0;
    }
  }
}

template <int D, typename R>
__global__ void __launch_bounds__(256) k_musl_norm(StepArgsT<R> A) {
  musl_norm_body<D, R>(A, blockIdx.x, gridDim.x);
}

// MUSL: deformation update from the normalised re-projected velocity v2 and
// the old positions (deformation_update.cpp:6), then the return mapping.
template <int D, int DEG, typename R, int PM>
__device__ __forceinline__ void defgrad_t_body(const StepArgsT<R>& A, const uint32_t* __restrict__ perm, const uint32_t bid, const uint32_t nblk) {
  using TL = Tiling<D>;
  constexpr int PN = TL::PN, NODES = TL::NODES;
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const uint32_t t = bid;
  if (t >= H->ntiles) return;
  const uint32_t pb = A.tile_begin[t], pe = A.tile_end[t];
  if (pb >= pe) return;
  __shared__ R pv[D * NODES];
  __shared__ double crd[3][PN];
  int n0[3];
  load_tile_setup<D>(A, H, t, n0, crd);
  double vref[3];
  tile_vref<D, R>(A, H, n0, A.v2, vref);
  load_velocity_patch<D, R>(A, H, n0, A.v2, vref, pv);
  __syncthreads();
  const uint32_t Np = A.Np;
  const double dt = H->dt, ioh = A.P->one_over_dx;
  unsigned nplastic = 0;
  for (uint32_t s = pb + threadIdx.x; s < pe; s += blockDim.x) {
    const uint32_t j = perm[s];
    PLoad<D> p;
    load_particle<D, R>(A.in, Np, j, p);
    double pic[3];
    R flp[3], Bp[D][D], gv[D][D];
    int lb[3];
    if (local_base<D>(H, p.x, ioh, n0, false, lb)) {
      gather_patch<D, DEG, true, R>(pv, nullptr, crd, lb, p.x, ioh, vref, pic, Bp, flp, gv, false, false);
    } else {
      raise_status(H, MTR_STATUS_STENCIL_OOB, p.id);
#pragma unroll
      for (int r = 0; r < D; ++r)
#pragma unroll
        for (int c = 0; c < D; ++c) gv[r][c] = R(0.0);
    }
    uint32_t f = 0;
    bool plastic = false;
    defgrad_and_store<D, R, PM>(A, s, dt, p, gv, f, plastic);
    if (f) raise_status(H, f, p.id);
    nplastic += plastic ? 1u : 0u;
  }
  block_count(nplastic, &H->plastic_count);
}

template <int D, int DEG, typename R, int PM = -1>
__global__ void __launch_bounds__(MTR_DEFGRAD_BOUNDS) k_defgrad_t(StepArgsT<R> A, const uint32_t* __restrict__ perm) {
  defgrad_t_body<D, DEG, R, PM>(A, perm, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// 8. end of step: moveObjects and the clock of simulate()
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void tail_body(const StepCommon& A, int out_parity) {
  StepHeader* H = A.H;
  if (step_inactive(H)) return;
  const DevParams& P = *A.P;
  if (threadIdx.x != 0) return;
  const double dt = H->dt;
  for (int i = 0; i < P.nplates; ++i) {  // ObjectPlate::move, object_plate.hpp:136-162
    mtr_plate& o = H->plates[i];
    double factor = (H->time < o.load_factor * P.frame_dt) ? (1.0 / o.vmin_factor) : 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) o.v_object[a] = (a < D) ? o.v_object_original[a] * factor : 0.0;
    if (o.plate_type == MTR_PLATE_LEFT || o.plate_type == MTR_PLATE_RIGHT) {
      o.pos_object += dt * o.v_object[0];
      o.pos_upper += dt * o.v_object[1];
      o.pos_lower += dt * o.v_object[1];
    } else if (o.plate_type == MTR_PLATE_BOTTOM || o.plate_type == MTR_PLATE_TOP) {
      o.pos_object += dt * o.v_object[1];
      o.pos_upper += dt * o.v_object[0];
      o.pos_lower += dt * o.v_object[0];
    } else if (D == 3 && (o.plate_type == MTR_PLATE_BACK || o.plate_type == MTR_PLATE_FRONT)) {
      o.pos_object += dt * o.v_object[2];
    }
  }
  H->cur = out_parity;
  if (H->status & kExitMask) {  // simulation.cpp:176-177: return before time += dt
    H->done = 1;
    return;
  }
  H->time += dt;
  H->step += 1;
  if (__dsub_rn(__dmul_rn(P.frame_dt, (double)(H->frame + 1)), H->time) < 1e-15) H->frame += 1;
  if (fabs(__dsub_rn(P.final_time, H->time)) < 1e-15 || P.final_time < H->time || !(H->frame < P.end_frame)) H->done = 1;
}

template <int D>
__global__ void k_tail(StepCommon A, int out_parity) {
  tail_body<D>(A, out_parity);
}

// ---------------------------------------------------------------------------
// 9. batched steps: the scenes of one group (same dim, spline, precision and
// USL/MUSL) advance together, one launch per phase for all of them.  Each
// launch's blocks are laid out scene after scene; a block finds its scene in
// a per-launch-kind offset table and runs the same body as the single-scene
// kernel on that scene's arguments.  Both particle-buffer parities of every
// scene are in the table and the block picks the one its scene's header
// names, so one captured graph stays valid while scenes advance, stop or
// regrow independently.
// ---------------------------------------------------------------------------
enum BatchKind { kBK_BBOX = 0, kBK_SORT, kBK_SCAN, kBK_TILES, kBK_CLEAR, kBK_TILEK, kBK_NODES, kBK_ONE, kBK_KINDS };

template <typename R>
struct BatchView {
  const StepArgsT<R>* args;  // [2][n]: args[c * n + s] = scene s reading particle buffer c
  const uint32_t* off;       // [kBK_KINDS][n + 1]: first block of each scene, per launch kind
  int n;
};

// arguments of the scene that owns global block g, the block index b within
// the scene and the scene's block count nb; null past the last scene
template <typename R>
__device__ __forceinline__ const StepArgsT<R>* batch_locate_at(const BatchView<R>& B, int kind, uint32_t g,
                                                               uint32_t& b, uint32_t& nb) {
  const uint32_t* o = B.off + (size_t)kind * (B.n + 1);
  if (g >= o[B.n]) return nullptr;
  int lo = 0, hi = B.n - 1;  // last scene whose first block is <= g
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (o[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  b = g - o[lo];
  nb = o[lo + 1] - o[lo];
  const int cur = B.args[lo].H->cur;
  return B.args + (size_t)(cur & 1) * B.n + lo;
}

template <typename R>
__device__ __forceinline__ const StepArgsT<R>* batch_locate(const BatchView<R>& B, int kind, uint32_t& b,
                                                            uint32_t& nb) {
  return batch_locate_at(B, kind, blockIdx.x, b, nb);
}

// The tile kernels of a batch run one block per tile block of every scene;
// `body(A, b, nb)` runs this block's tile.
template <typename R, typename Body>
__device__ __forceinline__ void batch_tiles(const BatchView<R>& B, Body&& body) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_TILEK, b, nb);
  if (A) body(*A, b, nb);
}

template <int D, typename R>
__global__ void __launch_bounds__(256) kb_bbox(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_BBOX, b, nb);
  if (A) bbox_body<D, R>(*A, b, nb);
}

template <int D, typename R>
__global__ void __launch_bounds__(256) kb_header(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_ONE, b, nb);
  if (A) header_body<D>(*A);
}

// zeroes the tile ranges and (MUSL) the re-projection accumulator of an
// active scene (the single-scene step does this with memsets)
template <int D, typename R>
__global__ void __launch_bounds__(256) kb_clear(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_CLEAR, b, nb);
  if (!A || step_inactive(A->H)) return;
  const uint32_t stride = nb * blockDim.x;
  for (uint32_t i = b * blockDim.x + threadIdx.x; i < A->cap_tiles; i += stride) {
    A->tile_begin[i] = 0u;
    A->tile_end[i] = 0u;
  }
  if (A->P->use_musl) {
    const size_t n = (size_t)D * A->cap_nodes;
    for (size_t i = b * blockDim.x + threadIdx.x; i < n; i += stride) A->v2[i] = 0.0;
  }
}

template <int D, typename R>
__global__ void __launch_bounds__(kSortThreads) kb_sort_hist(BatchView<R> B, int pass) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_SORT, b, nb);
  if (!A) return;
  if (pass == 0)
    sort_hist_body<D, true>(*A, nullptr, 0, b, nb);
  else
    sort_hist_body<D, false>(*A, (pass & 1) ? A->keysB : A->keysA, 8 * pass, b, nb);
}

template <typename R>
__global__ void __launch_bounds__(256) kb_sort_scan(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_SCAN, b, nb);
  if (A) sort_scan_warp_body(*A, b);
}

template <typename R>
__global__ void __launch_bounds__(kSortThreads) kb_sort_scatter(BatchView<R> B, int pass) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_SORT, b, nb);
  if (!A) return;
  const uint32_t* ksrc = pass == 0 ? A->keys0 : ((pass & 1) ? A->keysB : A->keysA);
  const uint32_t* vsrc = pass == 0 ? nullptr : ((pass & 1) ? A->valsB : A->valsA);
  uint32_t* kdst = (pass & 1) ? A->keysA : A->keysB;
  uint32_t* vdst = (pass & 1) ? A->valsA : A->valsB;
  sort_scatter_body(*A, ksrc, vsrc, kdst, vdst, 8 * pass, b, nb);
}

template <typename R>
__global__ void __launch_bounds__(256) kb_tile_ranges(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_TILES, b, nb);
  if (A) tile_ranges_body(*A, A->skeys, b, nb);
}

template <int D, int DEG, typename R, int XS = 1>
__global__ void __launch_bounds__(kMaxTileThreads) kb_p2g_w(BatchView<R> B) {
  batch_tiles(B, [&](const StepArgsT<R>& A, uint32_t b, uint32_t nb) { p2g_w_body<D, DEG, R, XS>(A, A.perm, b, nb); });
}

template <int D, typename R>
__global__ void __launch_bounds__(256) kb_grid(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_NODES, b, nb);
  if (A) grid_body<D, R>(*A, b, nb);
}

template <int D, int DEG, typename R, int PM = -1>
__global__ void __launch_bounds__(kChunk, MTR_G2P_MIN_BLOCKS) kb_g2p_t(BatchView<R> B) {
  batch_tiles(B, [&](const StepArgsT<R>& A, uint32_t b, uint32_t nb) { g2p_t_body<D, DEG, R, PM>(A, A.perm, b, nb); });
}

template <int D, int DEG, typename R, int XS = 1>
__global__ void __launch_bounds__(MTR_MUSL_MAX_THREADS, MTR_MUSL_MIN_BLOCKS) kb_g2p_musl_w(BatchView<R> B) {
  batch_tiles(B, [&](const StepArgsT<R>& A, uint32_t b, uint32_t nb) {
    g2p_musl_w_body<D, DEG, R, XS>(A, A.perm, b, nb);
  });
}

template <int D, typename R>
__global__ void __launch_bounds__(256) kb_musl_norm(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_NODES, b, nb);
  if (A) musl_norm_body<D, R>(*A, b, nb);
}

template <int D, int DEG, typename R, int PM = -1>
__global__ void __launch_bounds__(MTR_DEFGRAD_BOUNDS) kb_defgrad_t(BatchView<R> B) {
  batch_tiles(B, [&](const StepArgsT<R>& A, uint32_t b, uint32_t nb) {
    defgrad_t_body<D, DEG, R, PM>(A, A.perm, b, nb);
  });
}

template <int D, typename R>
__global__ void __launch_bounds__(32) kb_tail(BatchView<R> B) {
  uint32_t b, nb;
  const StepArgsT<R>* A = batch_locate(B, kBK_ONE, b, nb);
  if (A) tail_body<D>(*A, A->out_parity);
}

// ---------------------------------------------------------------------------
// set-up and download
// ---------------------------------------------------------------------------
template <int D, typename R>
__global__ void k_init_state(StepCommon A, PBufT<R> b) {  // tau of the uploaded F, id = index
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.Np) return;
  PLoad<D> p;
  load_particle<D, R>(b, A.Np, i, p);
  double tau[Sym<D>::n];
  initial_tau<D>(*A.P, p.F, tau);
#pragma unroll
  for (int q = 0; q < Sym<D>::n; ++q) b.tau[(size_t)q * A.Np + i] = (R)tau[q];
  b.id[i] = i;
}

// AoS (host layout, column-major matrices) <-> SoA, in original particle order.
// kind 0: vector (D), 1: matrix (D*D, column-major AoS <-> (r*D+c) SoA),
// 2: scalars (6), 3: matrix stored as M - I (the FP32 deformation gradient).
// A null src stands for every particle's value being zero, or with eye set
// (matrices) the identity: absent inputs are filled here, not copied.
template <int D, typename R>
__global__ void k_aos_to_soa(uint32_t Np, const double* __restrict__ src, R* dst, int kind, bool eye = false) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Np) return;
  if (kind == 0) {
#pragma unroll
    for (int a = 0; a < D; ++a) dst[(size_t)a * Np + i] = src ? (R)src[(size_t)i * D + a] : (R)0;
  } else if (kind == 1 || kind == 3) {
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const double m = src ? src[(size_t)i * D * D + c * D + r] : (eye && r == c ? 1.0 : 0.0);
        dst[(size_t)(r * D + c) * Np + i] = (R)(kind == 3 ? m - (r == c ? 1.0 : 0.0) : m);
      }
  } else {
#pragma unroll
    for (int q = 0; q < MTR_NUM_SCALARS; ++q)
      dst[(size_t)q * Np + i] = src ? (R)src[(size_t)i * MTR_NUM_SCALARS + q] : (R)0;
  }
}

template <int D, typename R>
__global__ void k_soa_to_aos(uint32_t Np, const R* __restrict__ src, const uint32_t* __restrict__ id, double* dst,
                             int kind) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= Np) return;
  const uint32_t i = id[s];
  if (kind == 0) {
#pragma unroll
    for (int a = 0; a < D; ++a) dst[(size_t)i * D + a] = src[(size_t)a * Np + s];
  } else if (kind == 1 || kind == 3) {
#pragma unroll
    for (int r = 0; r < D; ++r)
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const double m = src[(size_t)(r * D + c) * Np + s];
        dst[(size_t)i * D * D + c * D + r] = kind == 3 ? m + (r == c ? 1.0 : 0.0) : m;
      }
  } else {
#pragma unroll
    for (int q = 0; q < MTR_NUM_SCALARS; ++q) dst[(size_t)i * MTR_NUM_SCALARS + q] = src[(size_t)q * Np + s];
  }
}

// ---------------------------------------------------------------------------
// Frame output (Simulation::saveParticleData, save_data.cpp:7-171): one row of
// FP64 columns per particle, in the original particle order, with the
// columns and their order of the reference's particle file:
//   x[D], v[D], p, q, Je,
//   eps_pl_vol, eps_pl_dev, delta_gamma   (kFrameCols & kFramePlastic)
//   muI                                    (kFrameCols & kFrameMuI)
//   viscosity                              (kFrameCols & kFrameViscosity)
// p = -tr(tau)/D, q = sqrt(c tau_dev : tau_dev) with c = 3/2 (use_mises_q) or
// 1/2, Je = det F (save_data.cpp:14-35).  tau is the particle's carried
// Kirchhoff stress, which the step computes from the final F exactly as
// HenckyPiola(F) F^T / NeoHookeanPiola(F) F^T.  The particle buffer read is
// the current one of the header (H->cur), so the kernel can be enqueued
// behind any number of steps.  The clock of the snapshot goes to clock[0..4]:
// time, dt, step, frame, done.
// ---------------------------------------------------------------------------
enum : unsigned { kFramePlastic = 1u, kFrameMuI = 2u, kFrameViscosity = 4u };

template <int D, typename R>
__global__ void __launch_bounds__(256) k_frame_rows(PBufT<R> b0, PBufT<R> b1, const StepHeader* __restrict__ H,
                                                    const DevParams* __restrict__ P, uint32_t Np, unsigned cols,
                                                    uint32_t ncols, double* __restrict__ rows,
                                                    double* __restrict__ clock) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) {
    clock[0] = H->time;
    clock[1] = H->dt;
    clock[2] = (double)H->step;
    clock[3] = (double)H->frame;
    clock[4] = (double)H->done;
  }
  if (s >= Np) return;
  const PBufT<R>& b = H->cur ? b1 : b0;
  constexpr int NS = Sym<D>::n;
  PLoad<D> p;
  load_particle<D, R>(b, Np, s, p);
  double tau[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) tau[q] = (double)b.tau[(size_t)q * Np + s];
  double tr = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) tr += tau[a];
  const double pressure = -tr / D;
  double dd = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const double t = sym_at<D>(tau, i, j) + (i == j ? pressure : 0.0);
      dd += t * t;
    }
  const double q = sqrt((P->use_mises_q ? 1.5 : 0.5) * dd);
  const double(&F)[D][D] = p.F;
  double Je;
  if constexpr (D == 3)
    Je = F[0][0] * (F[1][1] * F[2][2] - F[2][1] * F[1][2]) - F[1][0] * (F[0][1] * F[2][2] - F[2][1] * F[0][2]) +
         F[2][0] * (F[0][1] * F[1][2] - F[1][1] * F[0][2]);
  else
    Je = F[0][0] * F[1][1] - F[1][0] * F[0][1];
  double* row = rows + (size_t)p.id * ncols;
  int c = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) row[c++] = p.x[a];
#pragma unroll
  for (int a = 0; a < D; ++a) row[c++] = p.v[a];
  row[c++] = pressure;
  row[c++] = q;
  row[c++] = Je;
  if (cols & kFramePlastic) {
    row[c++] = p.s.eps_pl_vol;
    row[c++] = p.s.eps_pl_dev;
    row[c++] = (double)b.sc[(size_t)MTR_SCALAR_DELTA_GAMMA * Np + s];
  }
  if (cols & kFrameMuI) row[c++] = p.s.muI;
  if (cols & kFrameViscosity) row[c++] = p.s.viscosity;
}

// Gradient of a dense level set by second-order central differences,
// 0.5 (phi[i+1] - phi[i-1]) / h per axis, neighbours outside the lattice
// reading `background` (OpenVDB's Gradient with CD_2ND, tools/GridOperators.h,
// on a fully active grid).  Three floats per sample; unused axes are zero.
static __global__ void __launch_bounds__(256) k_levelset_grad(const float* __restrict__ phi, float* __restrict__ grad,
                                                       uint32_t n0, uint32_t n1, uint32_t n2, int dim,
                                                       float background, double half_inv_h) {
  const uint64_t total = (uint64_t)n0 * n1 * n2;
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < total; l += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(l % n2), j = (uint32_t)((l / n2) % n1), i = (uint32_t)(l / ((uint64_t)n1 * n2));
    const uint32_t n[3] = {n0, n1, n2}, c[3] = {i, j, k};
    const uint64_t step[3] = {(uint64_t)n1 * n2, n2, 1};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float g = 0.0f;
      if (a < dim) {
        const float plus = c[a] + 1 < n[a] ? phi[l + step[a]] : background;
        const float minus = c[a] >= 1 ? phi[l - step[a]] : background;
        g = (float)((double)__fsub_rn(plus, minus) * half_inv_h);
      }
      grad[l * 3 + a] = g;
    }
  }
}

// node array of type R -> FP64 (grid read-back of the FP32 path)
template <typename R>
__global__ void k_to_f64(uint64_t n, const R* __restrict__ src, double* dst) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

}  // namespace mtr
