// mtr_abi.cu — the C ABI of include/matter_gpu.h: context, transfers and the
// step loop of Simulation::simulate (simulation.cpp:73-213) driving the
// kernels of mtr_kernels.cuh on one CUDA stream.
//
// A step is ~16 kernel launches with no host synchronisation: dt, the grid
// extents and the clock live in a device-side StepHeader.  Steps are captured
// into CUDA graphs of kGraphSteps steps (two variants, one per starting
// particle buffer) and replayed; the host reads the header back once per
// mtr_step call.  If the grid outgrows its capacity the header kernel aborts
// the step before any state is touched, every later kernel of the batch skips,
// and the host regrows the grid buffers, re-captures the graphs and resumes.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/matter_gpu.h"
#include "mtr_kernels.cuh"

using namespace mtr;

namespace {

thread_local std::string g_last_error;

struct MtrError {
  int code;
  std::string msg;
};

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) throw MtrError{MTR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

constexpr int kGraphSteps = 16;

template <typename T>
T* dalloc(size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw MtrError{MTR_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<T*>(p);
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// blocks for `work` items at `per_block` each, at least 1 and at most `cap`
uint32_t cap_blocks(uint64_t work, uint32_t per_block, uint32_t cap) {
  const uint64_t b = (work + per_block - 1) / per_block;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, cap));
}

int nsym(int d) { return d == 3 ? 6 : 3; }

// Events recorded after launches on one stream (per-launch timing): an entry
// per launch, events reused from a pool.
struct EventMarks {
  bool on = false;
  std::vector<std::pair<const char*, cudaEvent_t>> list;
  std::vector<int> tag;  // caller's tag of each entry (the batch group)
  std::vector<cudaEvent_t> pool;
  size_t next = 0;
  void record(const char* name, cudaStream_t st, int t = 0) {
    if (!on) return;
    if (next == pool.size()) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      pool.push_back(e);
    }
    cudaEvent_t e = pool[next++];
    CK(cudaEventRecord(e, st));
    list.emplace_back(name, e);
    tag.push_back(t);
  }
  void reset() {
    list.clear();
    tag.clear();
    next = 0;
  }
  // milliseconds between entry i - 1 and entry i
  float since_previous(size_t i) const {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, list[i - 1].second, list[i].second));
    return ms;
  }
  ~EventMarks() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

// Block shapes of the tile kernels (threads per tile block), one per kernel
// slot: P2G, MUSL G2P + re-scatter, USL G2P, MUSL deformation update.
enum { kSlotP2G = 0, kSlotMUSL = 1, kSlotG2P = 2, kSlotDefgrad = 3, kTileSlots = 4 };
// mark names that end each slot's kernel in a step
const char* const kSlotMark[kTileSlots] = {"k_p2g", "k_g2p_musl", "k_g2p", "k_defgrad"};
// largest block of each slot (k_g2p_t is register-bounded per 128 threads)
const int kSlotMax[kTileSlots] = {kMaxTileThreads, MTR_MUSL_MAX_THREADS, kChunk, kMaxTileThreads};
const int kTileCandidates[3] = {64, 128, 256};

bool valid_tile_threads(const int* t) {
  for (int i = 0; i < kTileSlots; ++i)
    if (t[i] < 32 || t[i] > kSlotMax[i] || t[i] % 32 != 0) return false;
  return true;
}

// Lanes per particle of the two scatters (P2G, MUSL): the stencil columns of
// a particle's cell (16 in 3D, 4 in 2D) times the split of each column's 4 x
// nodes over 1 or 2 lanes; a warp then takes 32 / lanes particles at a time.
constexpr int kScatterSlots = 2;
int scatter_columns(int dim) { return dim == 3 ? 16 : 4; }
bool valid_tile_lanes(int dim, const int* lanes) {
  for (int i = 0; i < kScatterSlots; ++i)
    if (lanes[i] != scatter_columns(dim) && lanes[i] != 2 * scatter_columns(dim)) return false;
  return true;
}

}  // namespace

struct mtr_ctx {
  mtr_params prm{};
  DevParams hp{};
  int device = 0;
  int dim = 3, deg = 2;
  cudaStream_t stream = nullptr;
  DevParams* dP = nullptr;
  StepHeader* dH = nullptr;
  StepHeader* hH = nullptr;  // pinned mirror
  uint32_t Np = 0;
  bool uploaded = false;
  // storage type of particle and grid state: double (MTR_PREC_FP64) or float (MTR_PREC_MIXED)
  bool fp32 = false;
  size_t rsize = sizeof(double);
  // particle buffers (two sets, positions FP64, the rest of type R) and their backing allocations
  PBufT<void> buf[2]{};
  std::vector<void*> pallocs;
  void *pic = nullptr, *flip = nullptr;
  // grid (axes FP64, node channels of type R)
  uint32_t cap_axis[3] = {0, 0, 0};
  uint32_t cap_nodes = 0, cap_tiles = 0;
  double *gx = nullptr, *gy = nullptr, *gz = nullptr;
  void *acc = nullptr, *nflip = nullptr, *nmass = nullptr, *nfric = nullptr;
  double *nv = nullptr, *v2 = nullptr;  // node velocities: FP64 on both paths
  uint32_t *tile_begin = nullptr, *tile_end = nullptr;
  // sort
  uint32_t *keys0 = nullptr, *keysA = nullptr, *valsA = nullptr, *keysB = nullptr, *valsB = nullptr;
  uint32_t *hist = nullptr, *dtot = nullptr;
  int sort_blocks = 0, passes = 0;
  BBoxPartial* partials = nullptr;
  int npartials = 0;
  double* staging = nullptr;  // Np * dim * dim doubles
  // plates/objects
  std::vector<mtr_plate> plates;
  std::vector<mtr_object> objects;
  // graphs
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int host_parity = 0;
  int64_t launches_last = 0;
  int64_t uploads_reused = 0;  // uploads that refilled the buffers already there
  int launches_per_step = 0;
  bool use_graphs = true;
  uint32_t step_limit = 0xffffffffu;  // mtr_set_step_limit: no step beyond this step count
  int tile_threads[kTileSlots] = {kChunk, kChunk, kChunk, kChunk};
  int tile_split[kScatterSlots] = {1, 1};  // x-node split of the P2G and MUSL scatters (1 or 2)
  // a trial step runs every kernel of a step but the commit (k_tail): the
  // particle buffer it reads and the clock stay as they were
  bool trial = false;
  // per-launch timing (mtr_profile, mtr_autotune): an event after every launch of a step
  EventMarks marks;
  // frame output (mtr_frame_begin / mtr_frame_wait): rows built on the device
  // behind the steps, copied to pinned host memory on a copy stream while the
  // next steps run
  double* frame_dev = nullptr;
  double* frame_host = nullptr;
  size_t frame_cap = 0;  // doubles in each
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t frame_ready = nullptr, frame_copied = nullptr;
  bool frame_pending = false;
  uint32_t frame_n = 0;
  int frame_ncols = 0;
  // dense level sets (mtr_set_levelset)
  float* ls_phi[MTR_MAX_LEVELSETS] = {};
  float* ls_grad[MTR_MAX_LEVELSETS] = {};
};

namespace {

void set_error(const std::string& m) { g_last_error = m; }

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const MtrError& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return MTR_ERR_INVALID;
  } catch (...) {
    set_error("unknown error");
    return MTR_ERR_INVALID;
  }
}

// Grid buffers come from a stream-ordered memory pool per device that keeps
// up to kGridPoolKeep bytes of freed memory for reuse: a spreading scene
// regrows its grid several times, and a plain cudaFree + cudaMalloc of the
// grid took 15-50 ms of host time per regrowth (a batch waits for it).
constexpr uint64_t kGridPoolKeep = 2ull << 30;
std::mutex g_grid_pool_mutex;
cudaMemPool_t g_grid_pool[64] = {};

cudaMemPool_t grid_pool(int device) {
  std::lock_guard<std::mutex> lock(g_grid_pool_mutex);
  if (device < 0 || device >= 64) throw MtrError{MTR_ERR_INVALID, "device index out of range"};
  if (!g_grid_pool[device]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CK(cudaMemPoolCreate(&g_grid_pool[device], &props));
    uint64_t keep = kGridPoolKeep;
    CK(cudaMemPoolSetAttribute(g_grid_pool[device], cudaMemPoolAttrReleaseThreshold, &keep));
  }
  return g_grid_pool[device];
}

// Host copies of particle arrays.  A copy to or from pageable host memory
// (a numpy array, a std::vector) goes through two pinned chunks per device,
// alternately: the host copies one chunk while the DMA of the other runs.  A
// plain pageable cudaMemcpy of a few hundred MB, issued by a serving loop's
// worker thread, held up the batch's own launches and header copies on the
// main thread for its whole duration (ticks of 1 step took as long as the
// upload beside them); in chunks, the driver and the copy engine are free
// between chunks.  Pinned host memory (cudaMallocHost, registered) is copied
// directly.
constexpr size_t kStageChunk = 8u << 20;
struct HostStage {
  std::mutex m;
  char* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
};
HostStage g_stage[64];

bool is_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

HostStage& host_stage(int device) {
  if (device < 0 || device >= 64) throw MtrError{MTR_ERR_INVALID, "device index out of range"};
  HostStage& S = g_stage[device];
  if (!S.buf[0]) {  // called with S.m held
    for (int i = 0; i < 2; ++i) {
      if (cudaMallocHost((void**)&S.buf[i], kStageChunk) != cudaSuccess) {
        (void)cudaGetLastError();
        throw MtrError{MTR_ERR_OOM, "cudaMallocHost (copy staging)"};
      }
      CK(cudaEventCreateWithFlags(&S.done[i], cudaEventDisableTiming));
    }
  }
  return S;
}

// bytes host -> device on the context's stream; returns when the copy is done
void copy_to_device(mtr_ctx* c, void* dst, const void* host, size_t bytes) {
  if (is_pinned(host)) {
    CK(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return;
  }
  HostStage& S = g_stage[c->device < 64 && c->device >= 0 ? c->device : 0];
  std::lock_guard<std::mutex> lock(S.m);
  host_stage(c->device);
  int k = 0;
  for (size_t off = 0; off < bytes; off += kStageChunk, k ^= 1) {
    const size_t n = std::min(kStageChunk, bytes - off);
    CK(cudaEventSynchronize(S.done[k]));  // the chunk's previous DMA has finished
    std::memcpy(S.buf[k], (const char*)host + off, n);
    CK(cudaMemcpyAsync((char*)dst + off, S.buf[k], n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(S.done[k], c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
}

// bytes device -> host on the context's stream (work already queued on it
// comes first); returns when the data is in host memory
void copy_to_host(mtr_ctx* c, void* host, const void* src, size_t bytes) {
  if (is_pinned(host)) {
    CK(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return;
  }
  HostStage& S = g_stage[c->device < 64 && c->device >= 0 ? c->device : 0];
  std::lock_guard<std::mutex> lock(S.m);
  host_stage(c->device);
  const size_t nchunks = (bytes + kStageChunk - 1) / kStageChunk;
  auto issue = [&](size_t j) {
    const size_t off = j * kStageChunk, n = std::min(kStageChunk, bytes - off);
    CK(cudaMemcpyAsync(S.buf[j & 1], (const char*)src + off, n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(S.done[j & 1], c->stream));
  };
  if (nchunks > 0) issue(0);
  for (size_t j = 0; j < nchunks; ++j) {
    if (j + 1 < nchunks) issue(j + 1);  // the next chunk's DMA runs while this one is copied out
    CK(cudaEventSynchronize(S.done[j & 1]));
    const size_t off = j * kStageChunk, n = std::min(kStageChunk, bytes - off);
    std::memcpy((char*)host + off, S.buf[j & 1], n);
  }
}

// n elements of T from the grid pool, ordered on the context's stream
template <typename T>
T* galloc(mtr_ctx* c, size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMallocFromPoolAsync(&p, n * sizeof(T), grid_pool(c->device), c->stream);
  if (e != cudaSuccess) throw MtrError{MTR_ERR_OOM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e)};
  return static_cast<T*>(p);
}

void free_grid(mtr_ctx* c) {
  for (void* p : {(void*)c->gx, (void*)c->gy, (void*)c->gz, (void*)c->acc, (void*)c->nv,
                  (void*)c->nflip, (void*)c->nmass, (void*)c->nfric, (void*)c->v2, (void*)c->tile_begin,
                  (void*)c->tile_end})
    if (p) cudaFreeAsync(p, c->stream);
  c->gx = c->gy = c->gz = c->nv = c->v2 = nullptr;
  c->acc = c->nflip = c->nmass = c->nfric = nullptr;
  c->tile_begin = c->tile_end = nullptr;
}

void free_graphs(mtr_ctx* c) {
  for (auto& g : c->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

int tile_edge(int d) { return d == 3 ? 4 : 8; }

// Zeroes the grid channels a fresh grid starts from.
void clear_grid(mtr_ctx* c) {
  const int d = c->dim;
  const int nch = 2 + 2 * d;
  const size_t rs = c->rsize, nodes = c->cap_nodes;
  CK(cudaMemsetAsync(c->acc, 0, rs * nch * nodes, c->stream));
  CK(cudaMemsetAsync(c->nv, 0, sizeof(double) * d * nodes, c->stream));
  CK(cudaMemsetAsync(c->nflip, 0, rs * d * nodes, c->stream));
  CK(cudaMemsetAsync(c->nmass, 0, rs * nodes, c->stream));
  CK(cudaMemsetAsync(c->v2, 0, sizeof(double) * d * nodes, c->stream));
}

// (Re)allocates the grid for per-axis node capacities.
void alloc_grid(mtr_ctx* c, const uint32_t want[3]) {
  free_grid(c);
  const int d = c->dim, tb = tile_edge(d);
  uint64_t nodes = 1, tiles = 1;
  for (int a = 0; a < 3; ++a) {
    c->cap_axis[a] = (a < d) ? std::max<uint32_t>(want[a], 8u) : 1u;
    nodes *= c->cap_axis[a];
    tiles *= (a < d) ? (c->cap_axis[a] + tb - 1) / tb : 1;
  }
  if (nodes > 0xffffffffull / 8 || tiles * 64ull > 0xffffffffull)
    throw MtrError{MTR_ERR_OOM, "grid capacity exceeds the 32-bit node/key range"};
  c->cap_nodes = (uint32_t)nodes;
  c->cap_tiles = (uint32_t)tiles;
  const int nch = 2 + 2 * d;  // mass, momentum, force, friction
  const size_t rs = c->rsize;
  c->gx = galloc<double>(c, c->cap_axis[0]);
  c->gy = galloc<double>(c, c->cap_axis[1]);
  c->gz = galloc<double>(c, c->cap_axis[2]);
  c->acc = galloc<unsigned char>(c, rs * nch * nodes);
  c->nv = galloc<double>(c, (size_t)d * nodes);
  c->nflip = galloc<unsigned char>(c, rs * d * nodes);
  c->nmass = galloc<unsigned char>(c, rs * nodes);
  c->nfric = galloc<unsigned char>(c, rs * nodes);
  c->v2 = galloc<double>(c, (size_t)d * nodes);
  c->tile_begin = galloc<uint32_t>(c, tiles);
  c->tile_end = galloc<uint32_t>(c, tiles);
  clear_grid(c);
  uint64_t keybits = 1;
  while ((1ull << keybits) < tiles * 64ull) ++keybits;
  c->passes = (int)((keybits + 7) / 8);
}

void mark(mtr_ctx* c, const char* name) { c->marks.record(name, c->stream); }

template <typename K>
void scatter_attributes(K kernel, size_t smem) {
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

template <int D, int DEG, typename R>
void set_kernel_attributes_t() {
  scatter_attributes(k_p2g_w<D, DEG, R, 1>, p2g_smem_bytes<D, R>(kMaxTileThreads));
  scatter_attributes(k_p2g_w<D, DEG, R, 2>, p2g_smem_bytes<D, R>(kMaxTileThreads));
  scatter_attributes(k_g2p_musl_w<D, DEG, R, 1>, musl_smem_bytes<D, R>(MTR_MUSL_MAX_THREADS));
  scatter_attributes(k_g2p_musl_w<D, DEG, R, 2>, musl_smem_bytes<D, R>(MTR_MUSL_MAX_THREADS));
}

void set_kernel_attributes(bool fp32) {
  if (fp32) {
    set_kernel_attributes_t<2, 2, float>();
    set_kernel_attributes_t<2, 3, float>();
    set_kernel_attributes_t<3, 2, float>();
    set_kernel_attributes_t<3, 3, float>();
  } else {
    set_kernel_attributes_t<2, 2, double>();
    set_kernel_attributes_t<2, 3, double>();
    set_kernel_attributes_t<3, 2, double>();
    set_kernel_attributes_t<3, 3, double>();
  }
}

template <typename R>
PBufT<R> typed(const PBufT<void>& b) {
  return PBufT<R>{b.x, (R*)b.v, (R*)b.F, (R*)b.B, (R*)b.sc, (R*)b.tau, b.id};
}

template <typename R>
StepArgsT<R> make_args(mtr_ctx* c, int parity) {
  StepArgsT<R> A{};
  A.P = c->dP;
  A.H = c->dH;
  A.partials = c->partials;
  A.npartials = c->npartials;
  A.Np = c->Np;
  A.gx = c->gx;
  A.gy = c->gy;
  A.gz = c->gz;
  for (int a = 0; a < 3; ++a) A.cap_axis[a] = c->cap_axis[a];
  A.cap_nodes = c->cap_nodes;
  A.cap_tiles = c->cap_tiles;
  A.acc = (R*)c->acc;
  A.nv = c->nv;
  A.nflip = (R*)c->nflip;
  A.nmass = (R*)c->nmass;
  A.nfric = (R*)c->nfric;
  A.v2 = c->v2;
  A.xin = c->buf[parity].x;
  A.keys0 = c->keys0;
  A.keysA = c->keysA;
  A.valsA = c->valsA;
  A.keysB = c->keysB;
  A.valsB = c->valsB;
  A.hist = c->hist;
  A.dtot = c->dtot;
  A.sort_blocks = c->sort_blocks;
  A.tile_begin = c->tile_begin;
  A.tile_end = c->tile_end;
  A.skeys = (c->passes & 1) ? c->keysB : c->keysA;  // where the last radix pass writes
  A.perm = (c->passes & 1) ? c->valsB : c->valsA;
  A.out_parity = 1 - parity;
  A.in = typed<R>(c->buf[parity]);
  A.out = typed<R>(c->buf[1 - parity]);
  A.pic = (R*)c->pic;
  A.flip = (R*)c->flip;
  return A;
}

// Enqueues one step reading buffer `parity` and writing the other.  Returns
// the number of kernels launched.
// Plastic models whose return-mapping kernels are also compiled for that
// model alone (3D; the workloads' models): the model-specific kernel skips
// the other models' code and stays within the instruction cache.  Any other
// model runs the generic kernel, which reads the model at run time.
int rm_specialization(int dim, bool musl, int pm) {
  if (dim != 3) return -1;
  if (musl) return pm == MTR_PM_DPMUI ? pm : -1;
  return (pm == MTR_PM_DP || pm == MTR_PM_MCCVISC) ? pm : -1;
}

template <int D, int DEG, typename R>
void launch_defgrad(int spm, uint32_t blocks, int threads, cudaStream_t st, const StepArgsT<R>& A,
                    const uint32_t* perm) {
  if constexpr (D == 3) {
    if (spm == MTR_PM_DPMUI) {
      k_defgrad_t<D, DEG, R, MTR_PM_DPMUI><<<blocks, threads, 0, st>>>(A, perm);
      return;
    }
  }
  k_defgrad_t<D, DEG, R><<<blocks, threads, 0, st>>>(A, perm);
}

template <int D, int DEG, typename R>
void launch_g2p(int spm, uint32_t blocks, int threads, cudaStream_t st, const StepArgsT<R>& A,
                const uint32_t* perm) {
  if constexpr (D == 3) {
    if (spm == MTR_PM_DP) {
      k_g2p_t<D, DEG, R, MTR_PM_DP><<<blocks, threads, 0, st>>>(A, perm);
      return;
    }
    if (spm == MTR_PM_MCCVISC) {
      k_g2p_t<D, DEG, R, MTR_PM_MCCVISC><<<blocks, threads, 0, st>>>(A, perm);
      return;
    }
  }
  k_g2p_t<D, DEG, R><<<blocks, threads, 0, st>>>(A, perm);
}

template <int D, int DEG, typename R>
int enqueue_step_t(mtr_ctx* c, int parity) {
  cudaStream_t st = c->stream;
  StepArgsT<R> A = make_args<R>(c, parity);
  int n = 0;
  mark(c, "start");
  k_bbox<D, R><<<c->npartials, 256, 0, st>>>(A);
  ++n;
  mark(c, "k_bbox");
  k_header<D><<<1, 256, 0, st>>>(A);
  ++n;
  mark(c, "k_header");
  // sort
  const uint32_t* skeys = nullptr;
  const uint32_t* perm = nullptr;
  for (int pass = 0; pass < c->passes; ++pass) {
    const int shift = 8 * pass;
    const uint32_t* ksrc = pass == 0 ? c->keys0 : ((pass & 1) ? c->keysB : c->keysA);
    const uint32_t* vsrc = pass == 0 ? nullptr : ((pass & 1) ? c->valsB : c->valsA);
    uint32_t* kdst = (pass & 1) ? c->keysA : c->keysB;
    uint32_t* vdst = (pass & 1) ? c->valsA : c->valsB;
    if (pass == 0)
      k_sort_hist<D, true><<<c->sort_blocks, kSortThreads, 0, st>>>(A, nullptr, shift);
    else
      k_sort_hist<D, false><<<c->sort_blocks, kSortThreads, 0, st>>>(A, ksrc, shift);
    mark(c, pass == 0 ? "k_sort_hist(keys)" : "k_sort_hist");
    k_sort_scan<<<256, 256, 0, st>>>(A);
    mark(c, "k_sort_scan");
    k_sort_scatter<<<c->sort_blocks, kSortThreads, 0, st>>>(A, ksrc, vsrc, kdst, vdst, shift);
    mark(c, "k_sort_scatter");
    n += 3;
    skeys = kdst;
    perm = vdst;
  }
  CK(cudaMemsetAsync(c->tile_begin, 0, sizeof(uint32_t) * c->cap_tiles, st));
  CK(cudaMemsetAsync(c->tile_end, 0, sizeof(uint32_t) * c->cap_tiles, st));
  mark(c, "memset(tiles)");
  k_tile_ranges<<<std::min<uint32_t>((c->Np + 255) / 256, 148 * 8), 256, 0, st>>>(A, skeys);
  ++n;
  mark(c, "k_tile_ranges");
  const int* tt = c->tile_threads;
  {
    const size_t sm = p2g_smem_bytes<D, R>(tt[kSlotP2G], c->prm.use_mibf != 0);
    if (c->tile_split[kSlotP2G] == 2)
      k_p2g_w<D, DEG, R, 2><<<c->cap_tiles, tt[kSlotP2G], sm, st>>>(A, perm);
    else
      k_p2g_w<D, DEG, R, 1><<<c->cap_tiles, tt[kSlotP2G], sm, st>>>(A, perm);
  }
  ++n;
  mark(c, "k_p2g");
  if (c->prm.pbc) {
    k_p2g_periodic<D, DEG, R><<<cap_blocks(c->Np, 256, 148 * 8), 256, 0, st>>>(A);
    ++n;
    mark(c, "k_p2g_periodic");
  }
  const uint32_t gblocks = std::min<uint32_t>((c->cap_nodes + 255) / 256, 148 * 16);
  k_grid<D, R><<<gblocks, 256, 0, st>>>(A);
  ++n;
  mark(c, "k_grid");
  if (c->prm.use_musl) {
    CK(cudaMemsetAsync(c->v2, 0, sizeof(double) * D * c->cap_nodes, st));
    mark(c, "memset(v2)");
    const size_t sm = musl_smem_bytes<D, R>(tt[kSlotMUSL]);
    if (c->tile_split[kSlotMUSL] == 2)
      k_g2p_musl_w<D, DEG, R, 2><<<c->cap_tiles, tt[kSlotMUSL], sm, st>>>(A, perm);
    else
      k_g2p_musl_w<D, DEG, R, 1><<<c->cap_tiles, tt[kSlotMUSL], sm, st>>>(A, perm);
    mark(c, "k_g2p_musl");
    k_musl_norm<D, R><<<gblocks, 256, 0, st>>>(A);
    mark(c, "k_musl_norm");
    launch_defgrad<D, DEG, R>(rm_specialization(D, true, c->prm.plastic_model), c->cap_tiles, tt[kSlotDefgrad], st,
                              A, perm);
    mark(c, "k_defgrad");
    n += 3;
  } else {
    launch_g2p<D, DEG, R>(rm_specialization(D, false, c->prm.plastic_model), c->cap_tiles, tt[kSlotG2P], st, A,
                          perm);
    ++n;
    mark(c, "k_g2p");
  }
  if (!c->trial) {
    k_tail<D><<<1, 32, 0, st>>>(A, 1 - parity);
    ++n;
    mark(c, "k_tail");
  }
  CK(cudaGetLastError());
  return n;
}

template <typename R>
int enqueue_step_r(mtr_ctx* c, int parity) {
  if (c->dim == 3) return c->deg == 3 ? enqueue_step_t<3, 3, R>(c, parity) : enqueue_step_t<3, 2, R>(c, parity);
  return c->deg == 3 ? enqueue_step_t<2, 3, R>(c, parity) : enqueue_step_t<2, 2, R>(c, parity);
}

int enqueue_step(mtr_ctx* c, int parity) {
  return c->fp32 ? enqueue_step_r<float>(c, parity) : enqueue_step_r<double>(c, parity);
}

void build_graphs(mtr_ctx* c) {
  free_graphs(c);
  if (!c->use_graphs) return;
  for (int p0 = 0; p0 < 2; ++p0) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int n = 0;
    try {
      for (int s = 0; s < kGraphSteps; ++s) n += enqueue_step(c, (p0 + s) & 1);
    } catch (...) {
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&c->graph[p0], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw MtrError{MTR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
    c->launches_per_step = n / kGraphSteps;
  }
}

// Every MTR_OBJ_LEVELSET object must name a loaded slot before a step.
void check_levelsets(const mtr_ctx* c) {
  for (const mtr_object& o : c->objects)
    if (o.kind == MTR_OBJ_LEVELSET && !c->ls_phi[(int)o.prm[0]])
      throw MtrError{MTR_ERR_STATE, "level-set object whose slot has no mtr_set_levelset data"};
}

// Columns of the particle frame file (save_data.cpp:7-171) for these parameters.
unsigned frame_columns(const mtr_params& p, std::vector<const char*>* names) {
  static const char* const xs[3] = {"x", "y", "z"};
  static const char* const vs[3] = {"vx", "vy", "vz"};
  unsigned cols = 0;
  const int pm = p.plastic_model;
  if (pm != MTR_PM_NOPLASTICITY) cols |= kFramePlastic;
  if (((pm == MTR_PM_DPVISC || pm == MTR_PM_MCCVISC) && p.use_mibf) || pm == MTR_PM_DPMUI || pm == MTR_PM_MCCMUI)
    cols |= kFrameMuI;
  if (pm == MTR_PM_DPMUI || pm == MTR_PM_MCCMUI) cols |= kFrameViscosity;
  if (names) {
    names->clear();
    for (int a = 0; a < p.dim; ++a) names->push_back(xs[a]);
    for (int a = 0; a < p.dim; ++a) names->push_back(vs[a]);
    for (const char* n : {"p", "q", "Je"}) names->push_back(n);
    if (cols & kFramePlastic)
      for (const char* n : {"eps_pl_vol", "eps_pl_dev", "delta_gamma"}) names->push_back(n);
    if (cols & kFrameMuI) names->push_back("muI");
    if (cols & kFrameViscosity) names->push_back("viscosity");
  }
  return cols;
}

// The header kernel aborted a step because the grid outgrew its capacity
// (H.N holds the extents it needed): reallocates the grid with 50% headroom
// (a spreading flow outgrows 25% again within a few hundred steps, and every
// regrowth frees and allocates device memory and, in a batch, recaptures the
// batch) and clears the abort in the host copy of the header (the caller
// writes it back).
void regrow_grid(mtr_ctx* c, StepHeader& H) {
  uint32_t want[3];
  for (int a = 0; a < 3; ++a)
    want[a] = (a < c->dim) ? std::max<uint32_t>(c->cap_axis[a], (uint32_t)std::ceil(H.N[a] * 1.5 + 8.0)) : 1u;
  for (int a = 0; a < c->dim; ++a)
    if (H.N[a] >= kMaxAxisNodes || H.N[a] < 4)
      throw MtrError{MTR_ERR_OOM, "grid extent exploded or collapsed (non-finite particle positions?)"};
  free_graphs(c);
  alloc_grid(c, want);
  CK(cudaStreamSynchronize(c->stream));
  H.abort = 0;
  H.status &= ~MTR_STATUS_GRID_OVERFLOW;
}

void read_header(mtr_ctx* c) {
  CK(cudaMemcpyAsync(c->hH, c->dH, sizeof(StepHeader), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

void write_header(mtr_ctx* c) { CK(cudaMemcpyAsync(c->dH, c->hH, sizeof(StepHeader), cudaMemcpyHostToDevice, c->stream)); }

void upload_params(mtr_ctx* c) {
  c->hp.nplates = (int)c->plates.size();
  c->hp.nobjects = (int)c->objects.size();
  for (size_t i = 0; i < c->objects.size(); ++i) c->hp.objects[i] = c->objects[i];
  CK(cudaMemcpyAsync(c->dP, &c->hp, sizeof(DevParams), cudaMemcpyHostToDevice, c->stream));
}

void derive_constants(mtr_ctx* c) {  // simulation.cpp:94-136
  const mtr_params& p = c->prm;
  DevParams& h = c->hp;
  const int d = p.dim;
  h.dim = d;
  h.deg = p.spline_deg;
  h.plastic_model = p.plastic_model;
  h.elastic_model = p.elastic_model;
  h.hardening_law = p.hardening_law;
  h.use_pradhana = p.use_pradhana;
  h.use_mises_q = p.use_mises_q;
  h.use_mibf = p.use_mibf;
  h.use_musl = p.use_musl;
  h.gravity_special = p.gravity_special;
  h.change_particle_positions = p.change_particle_positions;
  h.end_frame = p.end_frame;
  h.flip_ratio = p.flip_ratio;
  h.cfl = p.cfl;
  h.dx = p.dx;
  h.one_over_dx = 1.0 / p.dx;
  h.apicDinverse = p.spline_deg == 3 ? 3.0 / (p.dx * p.dx) : 4.0 / (p.dx * p.dx);
  h.particle_mass = p.particle_mass;
  h.particle_volume = p.particle_volume;
  h.lambda = p.nu * p.E / ((1.0 + p.nu) * (1.0 - 2.0 * p.nu));
  h.mu = p.E / (2.0 * (1.0 + p.nu));
  h.K = h.lambda + 2.0 * h.mu / d;  // simulation.cpp:288-290
  h.wave_speed = std::sqrt(p.E / p.rho);
  h.dt_max = p.cfl_elastic * p.dx / h.wave_speed;
  h.frame_dt = 1.0 / p.fps;
  h.final_time = p.end_frame * h.frame_dt;
  if (p.use_mises_q) {
    h.q_prefac = std::sqrt(3.0) / std::sqrt(2.0);
    h.d_prefac = std::sqrt(2.0) / std::sqrt(3.0);
  } else {
    h.q_prefac = 1.0 / std::sqrt(2.0);
    h.d_prefac = std::sqrt(2.0);
  }
  h.e_mu_prefac = 2 * h.q_prefac * h.mu;
  h.f_mu_prefac = 2 * h.q_prefac / h.d_prefac * h.mu;
  h.rma_prefac = 2 * h.q_prefac * h.q_prefac;
  h.fac_Q = p.I_ref / (p.grain_diameter * std::sqrt(p.rho_s));
  for (int a = 0; a < 3; ++a) {
    h.gravity_final[a] = a < d ? p.gravity[a] : 0.0;
    h.grid_ref[a] = a < d ? p.grid_reference_point[a] : 0.0;
  }
  h.gravity_time = p.gravity_time;
  h.E = p.E;
  h.nu = p.nu;
  h.stress_tolerance = p.stress_tolerance;
  h.xi = p.xi;
  h.q_max = p.q_max;
  h.q_min = p.q_min;
  h.p_min = p.p_min;
  h.M = p.M;
  h.q_cohesion = p.q_cohesion;
  h.perzyna_exp = p.perzyna_exp;
  h.perzyna_visc = p.perzyna_visc;
  h.beta = p.beta;
  h.p0 = p.p0;
  h.mu_1 = p.mu_1;
  h.mu_2 = p.mu_2;
  h.mui0 = (p.plastic_model == MTR_PM_DPMUI || p.plastic_model == MTR_PM_MCCMUI) ? p.mu_1 : p.M;
  h.dgamma_tol = p.precision == MTR_PREC_MIXED ? 1e-9 : 0.0;
  h.svd_rel = p.precision == MTR_PREC_MIXED ? 1e-12 : 2.220446049250313e-16;
  h.pbc = p.pbc ? 1 : 0;
  for (int a = 0; a < 3; ++a) h.L[a] = p.L[a];
}

// The first step's grid extents, as remeshFixedInit(2,2,2) will compute them
// (remesh.cpp:38-182), to size the initial grid allocation.
void grid_extent(const mtr_params& p, uint32_t Np, const double* x, uint32_t want[3]) {
  const int d = p.dim;
  const double dx = p.dx;
  for (int a = 0; a < 3; ++a) want[a] = 1;
  if (p.pbc) {  // the fixed grid of remeshFixed(4): [-5 dx (y: -dx), L + 6 dx)
    for (int a = 0; a < d; ++a) want[a] = (uint32_t)std::ceil(p.L[a] / dx + 12.0) + 2;
    return;
  }
  for (int a = 0; a < d; ++a) {
    double mn = x[a], mx = x[a];
    for (uint32_t q = 1; q < Np; ++q) {
      double v = x[(size_t)q * d + a];
      mn = std::min(mn, v);
      mx = std::max(mx, v);
    }
    const double g = p.grid_reference_point[a];
    if (p.grid_reference_point[0] < 1e10) {
      mn = std::min(mn, g);
      mx = std::max(mx, g);
    }
    const double n = (mx - mn) / dx + 6.0;
    want[a] = (uint32_t)std::ceil(n * 1.25 + 8.0);
  }
}

void initial_grid_extent(mtr_ctx* c, const double* x, uint32_t want[3]) { grid_extent(c->prm, c->Np, x, want); }

// SoA device array of the current particle order -> AoS host array in the
// caller's order (kinds as k_soa_to_aos); f64 marks an FP64 array on either path.
void get_soa(mtr_ctx* c, double* host, const void* src, const uint32_t* id, int width, int kind, bool f64) {
  if (!host) return;
  const uint32_t Np = c->Np, blocks = (Np + 255) / 256;
  const int d = c->dim;
  if (f64 || !c->fp32) {
    if (d == 3)
      k_soa_to_aos<3, double><<<blocks, 256, 0, c->stream>>>(Np, (const double*)src, id, c->staging, kind);
    else
      k_soa_to_aos<2, double><<<blocks, 256, 0, c->stream>>>(Np, (const double*)src, id, c->staging, kind);
  } else {
    if (d == 3)
      k_soa_to_aos<3, float><<<blocks, 256, 0, c->stream>>>(Np, (const float*)src, id, c->staging, kind);
    else
      k_soa_to_aos<2, float><<<blocks, 256, 0, c->stream>>>(Np, (const float*)src, id, c->staging, kind);
  }
  CK(cudaGetLastError());
  copy_to_host(c, host, c->staging, sizeof(double) * Np * width);
}

// n node values of the context's storage type -> FP64 host array
void get_nodes(mtr_ctx* c, double* host, const void* src, size_t n) {
  if (!c->fp32) {
    CK(cudaMemcpy(host, src, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return;
  }
  std::vector<float> tmp(n);
  CK(cudaMemcpy(tmp.data(), src, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i) host[i] = tmp[i];
}

// ---------------------------------------------------------------------------
// Batches: scenes grouped by (dim, spline, precision, MUSL), one launch per
// step phase and group over a device table of the scenes' arguments.
// ---------------------------------------------------------------------------

}  // namespace

struct mtr_batch_group {
  int dim = 3, deg = 2, musl = 0;
  int spm = -1;  // plastic model the return-mapping kernel is compiled for (-1: any)
  bool fp32 = false;
  int passes = 1;
  std::vector<mtr_ctx*> members;
  void* dargs = nullptr;      // StepArgsT<R>[2][n]
  uint32_t* doff = nullptr;   // [kBK_KINDS][n + 1]
  uint32_t total[kBK_KINDS] = {};
  int tile_threads[kTileSlots] = {kChunk, kChunk, kChunk, kChunk};
  int tile_split[kScatterSlots] = {1, 1};
  uint64_t tuned_nodes = 0;  // members' grid nodes at the last tune (0: take the next step's as the baseline)
};

struct mtr_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<mtr_ctx*> members;
  std::vector<mtr_batch_group> groups;
  cudaGraphExec_t graph = nullptr;
  bool dirty = true;
  int64_t launches_last = 0;
  int launches_per_step = 0;
  bool trial = false;  // trial steps: no kb_tail (see mtr_ctx::trial)
  EventMarks marks;    // tagged with the group index
  // host-side bookkeeping of mtr_batch_step (mtr_batch_stats)
  int64_t regrowths = 0, rebuilds = 0;
  int64_t updates = 0;  // rebuilds that updated the instantiated graph in place
  // > 0 after mtr_batch_set_retune: mtr_batch_step re-tunes with this many
  // repetitions when a group's grids have grown past twice their size at the
  // last tune (the tuned shapes fit the state they were tuned on; spreading
  // scenes move the optimum)
  int retune_reps = 0;
  int64_t retunes = 0;
  double regrow_ms = 0.0, rebuild_ms = 0.0;
};

namespace {

void free_batch_graph(mtr_batch* b) {
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
}

// Frees the argument and offset tables.  The instantiated step graph is kept:
// rebuild_batch updates it in place from the next capture when the step's
// launch sequence is unchanged.
void free_batch_tables(mtr_batch* b) {
  for (auto& g : b->groups) {
    // stream-ordered frees: a plain cudaFree waits for the whole GPU, which
    // would stall other contexts' work (the serving loop rebuilds batches
    // while new scenes upload)
    if (g.dargs) cudaFreeAsync(g.dargs, b->stream);
    if (g.doff) cudaFreeAsync(g.doff, b->stream);
    g.dargs = nullptr;
    g.doff = nullptr;
  }
}

template <typename R>
void build_group_tables(mtr_batch* b, mtr_batch_group& g) {
  const int n = (int)g.members.size();
  g.passes = 1;
  for (mtr_ctx* c : g.members) g.passes = std::max(g.passes, c->passes);
  std::vector<StepArgsT<R>> args((size_t)2 * n);
  std::vector<uint32_t> off((size_t)kBK_KINDS * (n + 1), 0u);
  for (int s = 0; s < n; ++s) {
    mtr_ctx* c = g.members[s];
    if (c->passes != g.passes) free_graphs(c);  // its own graphs were captured with fewer passes
    c->passes = g.passes;                      // extra radix passes over zero digits keep the order
    for (int par = 0; par < 2; ++par) args[(size_t)par * n + s] = make_args<R>(c, par);
    const uint32_t cnt[kBK_KINDS] = {
        (uint32_t)c->npartials,
        (uint32_t)c->sort_blocks,
        (uint32_t)(256 / kScanDigitsPerBlock),
        cap_blocks(c->Np, 256, 148 * 8),
        cap_blocks(std::max<uint64_t>(c->cap_tiles, g.musl ? (uint64_t)g.dim * c->cap_nodes : 0), 256, 148 * 8),
        c->cap_tiles,
        cap_blocks(c->cap_nodes, 256, 148 * 16),
        1u};
    for (int k = 0; k < kBK_KINDS; ++k) off[(size_t)k * (n + 1) + s + 1] = off[(size_t)k * (n + 1) + s] + cnt[k];
  }
  for (int k = 0; k < kBK_KINDS; ++k) g.total[k] = off[(size_t)k * (n + 1) + n];
  CK(cudaMallocAsync(&g.dargs, sizeof(StepArgsT<R>) * args.size(), b->stream));
  CK(cudaMallocAsync((void**)&g.doff, sizeof(uint32_t) * off.size(), b->stream));
  CK(cudaMemcpyAsync(g.dargs, args.data(), sizeof(StepArgsT<R>) * args.size(), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(g.doff, off.data(), sizeof(uint32_t) * off.size(), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
}

// Launches a batched tile kernel: one block per tile block of every scene.
template <typename R>
void launch_tiles(void (*kernel)(BatchView<R>), uint32_t total, int threads, size_t smem, cudaStream_t st,
                  const BatchView<R>& B) {
  kernel<<<std::max<uint32_t>(1, total), threads, smem, st>>>(B);
}

template <int D, int DEG, typename R>
int enqueue_group_step_t(mtr_batch* b, mtr_batch_group& g, int gi) {
  cudaStream_t st = b->stream;
  BatchView<R> B{(const StepArgsT<R>*)g.dargs, g.doff, (int)g.members.size()};
  const int* tt = g.tile_threads;
  int n = 0;
  kb_bbox<D, R><<<g.total[kBK_BBOX], 256, 0, st>>>(B);
  kb_header<D, R><<<g.total[kBK_ONE], 256, 0, st>>>(B);
  kb_clear<D, R><<<g.total[kBK_CLEAR], 256, 0, st>>>(B);
  n += 3;
  for (int pass = 0; pass < g.passes; ++pass) {
    kb_sort_hist<D, R><<<g.total[kBK_SORT], kSortThreads, 0, st>>>(B, pass);
    kb_sort_scan<R><<<g.total[kBK_SCAN], 256, 0, st>>>(B);
    kb_sort_scatter<R><<<g.total[kBK_SORT], kSortThreads, 0, st>>>(B, pass);
    n += 3;
  }
  kb_tile_ranges<R><<<g.total[kBK_TILES], 256, 0, st>>>(B);
  b->marks.record("kb_tile_ranges", st, gi);
  const uint32_t tiles = g.total[kBK_TILEK];
  launch_tiles<R>(g.tile_split[kSlotP2G] == 2 ? kb_p2g_w<D, DEG, R, 2> : kb_p2g_w<D, DEG, R, 1>, tiles,
                  tt[kSlotP2G], p2g_smem_bytes<D, R>(tt[kSlotP2G]), st, B);
  b->marks.record(kSlotMark[kSlotP2G], st, gi);
  kb_grid<D, R><<<g.total[kBK_NODES], 256, 0, st>>>(B);
  b->marks.record("kb_grid", st, gi);
  n += 3;
  if (g.musl) {
    launch_tiles<R>(g.tile_split[kSlotMUSL] == 2 ? kb_g2p_musl_w<D, DEG, R, 2> : kb_g2p_musl_w<D, DEG, R, 1>,
                    tiles, tt[kSlotMUSL], musl_smem_bytes<D, R>(tt[kSlotMUSL]), st, B);
    b->marks.record(kSlotMark[kSlotMUSL], st, gi);
    kb_musl_norm<D, R><<<g.total[kBK_NODES], 256, 0, st>>>(B);
    b->marks.record("kb_musl_norm", st, gi);
    void (*kd)(BatchView<R>) = kb_defgrad_t<D, DEG, R>;
    if constexpr (D == 3) {
      if (g.spm == MTR_PM_DPMUI) kd = kb_defgrad_t<D, DEG, R, MTR_PM_DPMUI>;
    }
    launch_tiles<R>(kd, tiles, tt[kSlotDefgrad], 0, st, B);
    b->marks.record(kSlotMark[kSlotDefgrad], st, gi);
    n += 3;
  } else {
    void (*kg)(BatchView<R>) = kb_g2p_t<D, DEG, R>;
    if constexpr (D == 3) {
      if (g.spm == MTR_PM_DP) kg = kb_g2p_t<D, DEG, R, MTR_PM_DP>;
      if (g.spm == MTR_PM_MCCVISC) kg = kb_g2p_t<D, DEG, R, MTR_PM_MCCVISC>;
    }
    launch_tiles<R>(kg, tiles, tt[kSlotG2P], 0, st, B);
    b->marks.record(kSlotMark[kSlotG2P], st, gi);
    ++n;
  }
  if (!b->trial) {
    kb_tail<D, R><<<g.total[kBK_ONE], 32, 0, st>>>(B);
    ++n;
  }
  CK(cudaGetLastError());
  return n;
}

template <typename R>
int enqueue_group_step_r(mtr_batch* b, mtr_batch_group& g, int gi) {
  if (g.dim == 3)
    return g.deg == 3 ? enqueue_group_step_t<3, 3, R>(b, g, gi) : enqueue_group_step_t<3, 2, R>(b, g, gi);
  return g.deg == 3 ? enqueue_group_step_t<2, 3, R>(b, g, gi) : enqueue_group_step_t<2, 2, R>(b, g, gi);
}

int enqueue_batch_step(mtr_batch* b) {
  int n = 0;
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    mtr_batch_group& g = b->groups[gi];
    n += g.fp32 ? enqueue_group_step_r<float>(b, g, (int)gi) : enqueue_group_step_r<double>(b, g, (int)gi);
  }
  return n;
}

template <int D, int DEG, typename R>
void set_batch_attributes_t() {
  scatter_attributes(kb_p2g_w<D, DEG, R, 1>, p2g_smem_bytes<D, R>(kMaxTileThreads));
  scatter_attributes(kb_p2g_w<D, DEG, R, 2>, p2g_smem_bytes<D, R>(kMaxTileThreads));
  scatter_attributes(kb_g2p_musl_w<D, DEG, R, 1>, musl_smem_bytes<D, R>(MTR_MUSL_MAX_THREADS));
  scatter_attributes(kb_g2p_musl_w<D, DEG, R, 2>, musl_smem_bytes<D, R>(MTR_MUSL_MAX_THREADS));
}

void set_batch_attributes(const mtr_batch_group& g) {
  if (g.fp32) {
    if (g.dim == 3) g.deg == 3 ? set_batch_attributes_t<3, 3, float>() : set_batch_attributes_t<3, 2, float>();
    else g.deg == 3 ? set_batch_attributes_t<2, 3, float>() : set_batch_attributes_t<2, 2, float>();
  } else {
    if (g.dim == 3) g.deg == 3 ? set_batch_attributes_t<3, 3, double>() : set_batch_attributes_t<3, 2, double>();
    else g.deg == 3 ? set_batch_attributes_t<2, 3, double>() : set_batch_attributes_t<2, 2, double>();
  }
}

// Steps per captured batch graph.  One: a batch is rebuilt (tables, capture,
// instantiation) whenever its membership changes, which the serving loop does
// often, and the capture cost grows with the steps captured, while replaying
// a one-step graph n times costs n graph launches of a few microseconds.
constexpr int kBatchGraphSteps = 1;
// steps replayed between two reads of the members' headers in mtr_batch_step
constexpr uint32_t kBatchCheckSteps = 8;

// (re)builds the device tables of every group and captures kBatchGraphSteps steps
void rebuild_batch(mtr_batch* b) {
  free_batch_tables(b);
  for (auto& g : b->groups) {
    set_batch_attributes(g);
    if (g.fp32)
      build_group_tables<float>(b, g);
    else
      build_group_tables<double>(b, g);
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int n = 0;
  try {
    for (int s = 0; s < kBatchGraphSteps; ++s) n += enqueue_batch_step(b);
  } catch (...) {
    cudaStreamEndCapture(b->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  CK(cudaStreamEndCapture(b->stream, &graph));
  // A membership change or a regrown grid changes launch sizes and table
  // addresses but usually not the launch sequence: the instantiated graph is
  // then updated in place (much cheaper than instantiating it again).
  if (b->graph) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(b->graph, graph, &info) == cudaSuccess) {
      b->updates += 1;
    } else {
      (void)cudaGetLastError();
      free_batch_graph(b);
    }
  }
  cudaError_t e = cudaSuccess;
  if (!b->graph) e = cudaGraphInstantiate(&b->graph, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) throw MtrError{MTR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
  b->launches_per_step = n / kBatchGraphSteps;
  b->dirty = false;
}

// reads every member's step header on the batch stream
void read_batch_headers(mtr_batch* b) {
  for (mtr_ctx* c : b->members)
    CK(cudaMemcpyAsync(c->hH, c->dH, sizeof(StepHeader), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
}

void write_batch_headers(mtr_batch* b) {
  for (mtr_ctx* c : b->members)
    CK(cudaMemcpyAsync(c->dH, c->hH, sizeof(StepHeader), cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
}

// Block-shape tuning over kTuneRounds candidates: candidate k runs every tile
// kernel with kTileCandidates[k % 3] threads (capped at the slot's maximum)
// and the scatters with x split 1 + k / 3 (16 or 32 lanes per particle in 3D,
// 4 or 8 in 2D).  The candidates are interleaved: each repetition times every
// candidate once, so slow drifts of the state or the clock touch them all
// alike.  samples[slot][k] holds the times of the slot's kernel with
// candidate k; for the gathers, whose shape is the thread count alone,
// rounds k and k + 3 are the same candidate.  A candidate's time is the
// median of its samples and its noise the half-range of its samples relative
// to that median; a slot keeps its current shape unless another candidate is
// faster by more than 2% and by more than the noise of the two together, so
// timing noise does not trade an equal shape for a slower one.
constexpr int kTuneRounds = 6;

struct TuneTimes {
  std::vector<double> samples[kTileSlots][kTuneRounds];
  void add(const char* name, float ms, int k) {
    for (int sl = 0; sl < kTileSlots; ++sl)
      if (std::strcmp(name, kSlotMark[sl]) == 0) samples[sl][k].push_back((double)ms);
  }
  // (median, relative half-range) of one candidate of a slot; median < 0: not measured
  std::pair<double, double> stats(int sl, int k) const {
    std::vector<double> v = samples[sl][k];
    if (sl >= kScatterSlots) v.insert(v.end(), samples[sl][k + 3].begin(), samples[sl][k + 3].end());
    if (v.empty()) return {-1.0, 0.0};
    std::sort(v.begin(), v.end());
    const size_t n = v.size();
    const double med = n % 2 ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
    return {med, med > 0.0 ? 0.5 * (v.back() - v.front()) / med : 0.0};
  }
  void choose(int* threads, int* split) const {
    for (int sl = 0; sl < kTileSlots; ++sl) {
      const bool scatter = sl < kScatterSlots;
      const int nk = scatter ? kTuneRounds : 3;
      int cur = -1, arg = -1;
      double tcur = 0.0, ncur = 0.0, targ = 0.0, narg = 0.0;
      for (int k = 0; k < nk; ++k) {
        if (kTileCandidates[k % 3] > kSlotMax[sl]) continue;
        const auto st = stats(sl, k);
        if (st.first < 0.0) continue;
        if (kTileCandidates[k % 3] == threads[sl] && (!scatter || 1 + k / 3 == split[sl])) {
          cur = k;
          tcur = st.first;
          ncur = st.second;
        }
        if (arg < 0 || st.first < targ) {
          arg = k;
          targ = st.first;
          narg = st.second;
        }
      }
      if (arg < 0) continue;  // the slot's kernel does not run in this step
      const double margin = std::max(0.02, ncur + narg);
      if (cur >= 0 && tcur <= (1.0 + margin) * targ) continue;
      threads[sl] = kTileCandidates[arg % 3];
      if (scatter) split[sl] = 1 + arg / 3;
    }
  }
};

// the shapes of candidate k for every slot
void set_candidate(int* threads, int* split, int k) {
  for (int sl = 0; sl < kTileSlots; ++sl) threads[sl] = std::min(kTileCandidates[k % 3], kSlotMax[sl]);
  for (int sl = 0; sl < kScatterSlots; ++sl) split[sl] = 1 + k / 3;
}

// Restores flags changed for trial steps even when a step throws.
struct TrialScope {
  bool* trial;
  bool* marks_on;
  TrialScope(bool* t, bool* m) : trial(t), marks_on(m) {}
  ~TrialScope() {
    *trial = false;
    *marks_on = false;
  }
};

}  // namespace

extern "C" {

const char* mtr_last_error(void) { return g_last_error.c_str(); }

int mtr_ctx_create(const mtr_params* params, int device, mtr_ctx** out) {
  return guarded([&]() -> int {
    if (!params || !out) throw MtrError{MTR_ERR_INVALID, "null argument"};
    *out = nullptr;
    const mtr_params& p = *params;
    if (p.dim != 2 && p.dim != 3) throw MtrError{MTR_ERR_INVALID, "dim must be 2 or 3"};
    if (p.spline_deg != 2 && p.spline_deg != 3) throw MtrError{MTR_ERR_INVALID, "spline_deg must be 2 or 3"};
    if (p.precision != MTR_PREC_FP64 && p.precision != MTR_PREC_MIXED)
      throw MtrError{MTR_ERR_INVALID, "precision must be MTR_PREC_FP64 or MTR_PREC_MIXED"};
    if (p.pbc && (p.use_mibf || p.plastic_model == MTR_PM_SNOW))  // pbc.cpp copies x, v, F, B only
      throw MtrError{MTR_ERR_INVALID, "periodic boundaries do not combine with use_mibf or the Snow model"};
    if (p.pbc && !(p.L[0] > 0 && p.L[1] > 0 && (p.dim == 2 || p.L[2] > 0)))
      throw MtrError{MTR_ERR_INVALID, "periodic boundaries need L > 0"};
    if (p.plastic_model < 0 || p.plastic_model > MTR_PM_SNOW) throw MtrError{MTR_ERR_INVALID, "invalid plastic model"};
    if (p.elastic_model != MTR_EL_HENCKY && p.elastic_model != MTR_EL_NEOHOOKEAN)
      throw MtrError{MTR_ERR_INVALID, "invalid elastic model"};
    if (p.elastic_model != MTR_EL_HENCKY && p.plastic_model != MTR_PM_NOPLASTICITY)  // simulation.cpp:80-84
      throw MtrError{MTR_ERR_INVALID, "This plastic model is only compatible with Hencky's elasticity model"};
    if (!(p.dx > 0) || !(p.fps > 0) || !(p.rho > 0)) throw MtrError{MTR_ERR_INVALID, "dx, fps and rho must be > 0"};
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw MtrError{MTR_ERR_NO_DEVICE, "no CUDA device"};
    if (device < 0 || device >= ndev) throw MtrError{MTR_ERR_INVALID, "device index out of range"};
    mtr_ctx* c = new mtr_ctx();
    try {
      c->prm = p;
      c->device = device;
      c->dim = p.dim;
      c->deg = p.spline_deg;
      c->fp32 = p.precision == MTR_PREC_MIXED;
      c->rsize = c->fp32 ? sizeof(float) : sizeof(double);
      CK(cudaSetDevice(device));
      CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      set_kernel_attributes(c->fp32);
      derive_constants(c);
      c->dP = dalloc<DevParams>(1);
      c->dH = dalloc<StepHeader>(1);
      CK(cudaMallocHost((void**)&c->hH, sizeof(StepHeader)));
      std::memset(c->hH, 0, sizeof(StepHeader));
      upload_params(c);
      CK(cudaStreamSynchronize(c->stream));
    } catch (...) {
      mtr_ctx_destroy(c);
      throw;
    }
    *out = c;
    return MTR_OK;
  });
}

int mtr_upload(mtr_ctx* c, const double* x, const double* v, const double* F, const double* B,
               const double* scalars, uint32_t Np) {
  return guarded([&]() -> int {
    if (!c || !x || Np == 0) throw MtrError{MTR_ERR_INVALID, "null context/positions or Np == 0"};
    CK(cudaSetDevice(c->device));
    const int d = c->dim, dd = d * d, ns = nsym(d);
    // A new scene of the same particle count refills the buffers it already
    // has: their addresses, and with them the captured step graphs, stay valid
    // (freeing and allocating them again costs more than the copies).
    const bool reuse = c->uploaded && c->Np == Np && !c->pallocs.empty();
    c->uploaded = false;
    if (!reuse) {
      free_graphs(c);
      for (void* p : c->pallocs) dfree(p);
      c->pallocs.clear();
      for (void* p : {(void*)c->keys0, (void*)c->keysA, (void*)c->valsA, (void*)c->keysB, (void*)c->valsB,
                      (void*)c->hist, (void*)c->dtot, (void*)c->partials, (void*)c->staging})
        dfree(p);
      c->Np = Np;
      c->hp.Np = Np;
      const size_t rs = c->rsize;
      for (int s = 0; s < 2; ++s) {
        double* xb = dalloc<double>((size_t)Np * d);  // positions: FP64 on both paths
        unsigned char* blk = dalloc<unsigned char>(rs * Np * (d + 2 * dd + MTR_NUM_SCALARS + ns));
        c->pallocs.push_back(xb);
        c->pallocs.push_back(blk);
        c->buf[s].x = xb;
        c->buf[s].v = blk;
        c->buf[s].F = blk + rs * Np * d;
        c->buf[s].B = blk + rs * Np * (d + dd);
        c->buf[s].sc = blk + rs * Np * (d + 2 * dd);
        c->buf[s].tau = blk + rs * Np * (d + 2 * dd + MTR_NUM_SCALARS);
        c->buf[s].id = dalloc<uint32_t>(Np);
        c->pallocs.push_back(c->buf[s].id);
      }
      c->pic = dalloc<unsigned char>(rs * Np * d);
      c->flip = dalloc<unsigned char>(rs * Np * d);
      c->pallocs.push_back(c->pic);
      c->pallocs.push_back(c->flip);
      c->sort_blocks = (int)((Np + kSortTile - 1) / kSortTile);
      c->keys0 = dalloc<uint32_t>(Np);
      c->keysA = dalloc<uint32_t>(Np);
      c->valsA = dalloc<uint32_t>(Np);
      c->keysB = dalloc<uint32_t>(Np);
      c->valsB = dalloc<uint32_t>(Np);
      c->hist = dalloc<uint32_t>((size_t)256 * c->sort_blocks);
      c->dtot = dalloc<uint32_t>(256);
      c->npartials = (int)std::min<uint32_t>((Np + 255) / 256, 148 * 8);
      c->partials = dalloc<BBoxPartial>(c->npartials);
      c->staging = dalloc<double>((size_t)Np * std::max<int>(dd, (int)MTR_NUM_SCALARS));
    }
    c->uploads_reused += reuse ? 1 : 0;
    // state -> buffer 0 (AoS host layout -> SoA)
    const uint32_t blocks = (Np + 255) / 256;
    // an absent array is filled on the device (zeros, or identity with eye)
    auto put = [&](const double* host, void* dst, int width, int kind, bool eye) {
      const double* src = nullptr;
      if (host) {
        copy_to_device(c, c->staging, host, sizeof(double) * Np * width);
        src = c->staging;
      }
      if (kind == 0 && dst == c->buf[0].x) {  // positions stay FP64
        if (d == 3)
          k_aos_to_soa<3, double><<<blocks, 256, 0, c->stream>>>(Np, src, (double*)dst, kind, eye);
        else
          k_aos_to_soa<2, double><<<blocks, 256, 0, c->stream>>>(Np, src, (double*)dst, kind, eye);
      } else if (c->fp32) {
        if (d == 3)
          k_aos_to_soa<3, float><<<blocks, 256, 0, c->stream>>>(Np, src, (float*)dst, kind, eye);
        else
          k_aos_to_soa<2, float><<<blocks, 256, 0, c->stream>>>(Np, src, (float*)dst, kind, eye);
      } else {
        if (d == 3)
          k_aos_to_soa<3, double><<<blocks, 256, 0, c->stream>>>(Np, src, (double*)dst, kind, eye);
        else
          k_aos_to_soa<2, double><<<blocks, 256, 0, c->stream>>>(Np, src, (double*)dst, kind, eye);
      }
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(c->stream));
    };
    put(x, c->buf[0].x, d, 0, false);
    put(v, c->buf[0].v, d, 0, false);
    put(F, c->buf[0].F, dd, c->fp32 ? 3 : 1, true);  // FP32 keeps F - I
    put(B, c->buf[0].B, dd, 1, false);
    std::vector<double> sc;
    const double* scp = scalars;
    if (c->prm.use_mibf) {  // simulation.cpp:138-145
      sc.assign((size_t)Np * MTR_NUM_SCALARS, 0.0);
      if (scalars) std::memcpy(sc.data(), scalars, sizeof(double) * sc.size());
      const double m0 = (c->prm.plastic_model == MTR_PM_DPMUI || c->prm.plastic_model == MTR_PM_MCCMUI) ? c->prm.mu_1
                                                                                                     : c->prm.M;
      for (uint32_t p = 0; p < Np; ++p) sc[(size_t)p * MTR_NUM_SCALARS + MTR_SCALAR_MUI] = m0;
      scp = sc.data();
    }
    put(scp, c->buf[0].sc, MTR_NUM_SCALARS, 2, false);
    // initial grid: kept when the new scene's extent fits the grid there is
    uint32_t want[3];
    initial_grid_extent(c, x, want);
    bool fits = reuse && c->gx != nullptr;
    for (int a = 0; a < d; ++a) fits = fits && want[a] <= c->cap_axis[a];
    if (fits) {
      clear_grid(c);
    } else {
      free_graphs(c);  // captured with the old grid's addresses
      alloc_grid(c, want);
    }
    // header
    std::memset(c->hH, 0, sizeof(StepHeader));
    c->hH->first_bad = 0xffffffffu;
    c->hH->stop_frame = 0xffffffffu;
    c->hH->stop_step = 0xffffffffu;
    c->step_limit = 0xffffffffu;
    for (int a = 0; a < 3; ++a) c->hH->gravity[a] = a < d ? c->prm.gravity[a] : 0.0;
    c->hH->done = (0 < c->prm.end_frame) ? 0 : 1;
    for (size_t i = 0; i < c->plates.size(); ++i) c->hH->plates[i] = c->plates[i];
    write_header(c);
    upload_params(c);
    if (c->fp32) {
      StepArgsT<float> A = make_args<float>(c, 0);
      if (d == 3)
        k_init_state<3, float><<<blocks, 256, 0, c->stream>>>(A, A.in);
      else
        k_init_state<2, float><<<blocks, 256, 0, c->stream>>>(A, A.in);
    } else {
      StepArgsT<double> A = make_args<double>(c, 0);
      if (d == 3)
        k_init_state<3, double><<<blocks, 256, 0, c->stream>>>(A, A.in);
      else
        k_init_state<2, double><<<blocks, 256, 0, c->stream>>>(A, A.in);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    c->host_parity = 0;
    c->uploaded = true;
    return MTR_OK;
  });
}

int mtr_set_objects(mtr_ctx* c, const mtr_plate* plates, int n_plates, const mtr_object* objects, int n_objects) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    if (n_plates < 0 || n_plates > MTR_MAXP || n_objects < 0 || n_objects > MTR_MAXO)
      throw MtrError{MTR_ERR_INVALID, "too many plates or objects"};
    for (int i = 0; i < n_plates; ++i)
      if (plates[i].bc < 0 || plates[i].bc > 2 || plates[i].plate_type < 0 || plates[i].plate_type > 5)
        throw MtrError{MTR_ERR_INVALID, "invalid plate type or BC"};
    for (int i = 0; i < n_objects; ++i) {
      if (objects[i].bc < 0 || objects[i].bc > 2 || objects[i].kind < 0 || objects[i].kind > MTR_OBJ_LEVELSET)
        throw MtrError{MTR_ERR_INVALID, "invalid object kind or BC"};
      if (objects[i].kind == MTR_OBJ_LEVELSET) {
        const double sl = objects[i].prm[0];
        if (!(sl >= 0 && sl < MTR_MAX_LEVELSETS) || sl != std::floor(sl))
          throw MtrError{MTR_ERR_INVALID, "level-set object: prm[0] must be a slot 0..MTR_MAX_LEVELSETS-1"};
      }
    }
    CK(cudaSetDevice(c->device));
    c->plates.assign(plates, plates + n_plates);
    c->objects.assign(objects, objects + n_objects);
    if (c->dim == 2)
      for (auto& q : c->plates) q.v_object[2] = q.v_object_original[2] = 0.0;
    upload_params(c);
    if (c->uploaded) {
      read_header(c);
      for (int i = 0; i < n_plates; ++i) c->hH->plates[i] = c->plates[i];
      write_header(c);
    }
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
}

int mtr_step(mtr_ctx* c, int nsteps) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    if (!c->uploaded) throw MtrError{MTR_ERR_STATE, "mtr_step before mtr_upload"};
    check_levelsets(c);
    if (nsteps <= 0) return MTR_OK;
    CK(cudaSetDevice(c->device));
    read_header(c);
    if (c->hH->done) return (c->hH->status & kExitMask) ? MTR_ERR_DEVICE_STATUS : MTR_OK;
    if (c->hH->frame >= c->hH->stop_frame || c->hH->step >= c->hH->stop_step) return MTR_OK;
    c->host_parity = c->hH->cur;
    int64_t launches = 0;
    int remaining = nsteps;
    for (int guard = 0; guard < 64 && remaining > 0; ++guard) {
      const uint32_t step0 = c->hH->step;
      if (c->use_graphs && (!c->graph[0] || !c->graph[1])) build_graphs(c);
      int parity = c->host_parity;
      int todo = remaining;
      while (todo > 0) {
        if (c->use_graphs && todo >= kGraphSteps) {
          CK(cudaGraphLaunch(c->graph[parity], c->stream));
          launches += (int64_t)c->launches_per_step * kGraphSteps;
          todo -= kGraphSteps;  // kGraphSteps is even: parity unchanged
        } else {
          launches += enqueue_step(c, parity);
          parity ^= 1;
          todo -= 1;
        }
      }
      read_header(c);
      StepHeader& H = *c->hH;
      c->host_parity = H.cur;
      const int executed = (int)(H.step - step0) + ((H.status & kExitMask) && H.done ? 1 : 0);
      remaining -= executed;
      if (H.abort) {  // grid outgrew its capacity: regrow and resume
        regrow_grid(c, H);
        write_header(c);
        CK(cudaStreamSynchronize(c->stream));
        continue;
      }
      if (H.done || H.frame >= H.stop_frame || H.step >= H.stop_step) break;
    }
    c->launches_last = launches;
    if (c->hH->status & kExitMask) return MTR_ERR_DEVICE_STATUS;
    return MTR_OK;
  });
}

int mtr_run_frame(mtr_ctx* c, int* frame_done) {
  int rc = guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    c->hH->stop_frame = c->hH->frame + 1;
    write_header(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
  if (rc != MTR_OK) return rc;
  mtr_clock ck{};
  uint32_t f0 = 0;
  rc = mtr_get_clock(c, &ck);
  f0 = ck.frame;
  while (rc == MTR_OK) {
    const uint32_t s0 = ck.step;
    rc = mtr_step(c, 128);
    if (rc != MTR_OK) break;
    rc = mtr_get_clock(c, &ck);
    if (rc != MTR_OK || ck.done || ck.frame > f0 || ck.step == s0) break;  // ck.step == s0: step limit reached
  }
  int rc2 = guarded([&]() -> int {
    read_header(c);
    c->hH->stop_frame = 0xffffffffu;
    write_header(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
  if (frame_done) *frame_done = (rc == MTR_OK && ck.frame > f0) ? 1 : 0;
  return rc != MTR_OK ? rc : rc2;
}

int mtr_run(mtr_ctx* c) {
  mtr_clock ck{};
  int rc = mtr_get_clock(c, &ck);
  while (rc == MTR_OK && !ck.done) {
    const uint32_t s0 = ck.step;
    rc = mtr_step(c, 1024);
    if (rc != MTR_OK) return rc;
    rc = mtr_get_clock(c, &ck);
    if (rc == MTR_OK && ck.step == s0) break;  // step limit reached
  }
  return rc;
}

int mtr_set_step_limit(mtr_ctx* c, uint32_t last_step) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    c->step_limit = last_step;
    c->hH->stop_step = last_step;
    write_header(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
}

int mtr_download(mtr_ctx* c, double* x, double* v, double* F, double* B, double* scalars) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    const int d = c->dim, dd = d * d;
    const PBufT<void>& b = c->buf[c->hH->cur];
    get_soa(c, x, b.x, b.id, d, 0, true);
    get_soa(c, v, b.v, b.id, d, 0, false);
    get_soa(c, F, b.F, b.id, dd, c->fp32 ? 3 : 1, false);
    get_soa(c, B, b.B, b.id, dd, 1, false);
    get_soa(c, scalars, b.sc, b.id, MTR_NUM_SCALARS, 2, false);
    return MTR_OK;
  });
}

int mtr_download_pic_flip(mtr_ctx* c, double* pic, double* flip) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    if (!c->hp.store_pic_flip) throw MtrError{MTR_ERR_STATE, "pic/flip are kept only after mtr_keep_pic_flip(ctx, 1)"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    const PBufT<void>& b = c->buf[c->hH->cur];
    get_soa(c, pic, c->pic, b.id, c->dim, 0, false);
    get_soa(c, flip, c->flip, b.id, c->dim, 0, false);
    return MTR_OK;
  });
}

// Not in the header: switches the optional per-particle pic/flip output used
// by the parity tests (off by default; it costs 2*dim stores per particle).
int mtr_keep_pic_flip(mtr_ctx* c, int on) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    CK(cudaSetDevice(c->device));
    c->hp.store_pic_flip = on ? 1 : 0;
    upload_params(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
}

int mtr_get_grid(mtr_ctx* c, uint32_t dims[3], double* gx, double* gy, double* gz, double* mass, double* v,
                 double* flip) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded || !dims) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    const StepHeader& H = *c->hH;
    for (int a = 0; a < 3; ++a) dims[a] = H.N[a];
    const int d = c->dim;
    const uint32_t G = H.G;
    if (G > c->cap_nodes) throw MtrError{MTR_ERR_STATE, "no completed step"};
    if (gx) CK(cudaMemcpy(gx, c->gx, sizeof(double) * H.N[0], cudaMemcpyDeviceToHost));
    if (gy) CK(cudaMemcpy(gy, c->gy, sizeof(double) * H.N[1], cudaMemcpyDeviceToHost));
    if (gz && d == 3) CK(cudaMemcpy(gz, c->gz, sizeof(double) * H.N[2], cudaMemcpyDeviceToHost));
    if (mass) get_nodes(c, mass, c->nmass, G);
    std::vector<double> tmp((size_t)G);
    for (int w = 0; w < 2; ++w) {
      double* host = w == 0 ? v : flip;
      if (!host) continue;
      for (int a = 0; a < d; ++a) {
        if (w == 0) {  // node velocities are FP64 on both paths
          const double* src = (c->prm.use_musl ? c->v2 : c->nv) + (size_t)a * c->cap_nodes;
          CK(cudaMemcpy(tmp.data(), src, sizeof(double) * G, cudaMemcpyDeviceToHost));
        } else {
          get_nodes(c, tmp.data(), (const unsigned char*)c->nflip + c->rsize * a * c->cap_nodes, G);
        }
        for (uint32_t l = 0; l < G; ++l) host[(size_t)l * d + a] = tmp[l];
      }
    }
    return MTR_OK;
  });
}

int mtr_get_sort(mtr_ctx* c, uint32_t* keys_in_input_order, uint32_t* sorted_input_index, uint32_t* input_particle_id) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    const uint32_t Np = c->Np;
    const uint32_t* perm = (c->passes & 1) ? c->valsB : c->valsA;
    if (keys_in_input_order) CK(cudaMemcpy(keys_in_input_order, c->keys0, sizeof(uint32_t) * Np, cudaMemcpyDeviceToHost));
    if (sorted_input_index) CK(cudaMemcpy(sorted_input_index, perm, sizeof(uint32_t) * Np, cudaMemcpyDeviceToHost));
    if (input_particle_id)
      CK(cudaMemcpy(input_particle_id, c->buf[1 - c->hH->cur].id, sizeof(uint32_t) * Np, cudaMemcpyDeviceToHost));
    return MTR_OK;
  });
}

int mtr_get_plates(mtr_ctx* c, mtr_plate* plates, int n_plates) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    for (int i = 0; i < n_plates && i < (int)c->plates.size(); ++i) plates[i] = c->hH->plates[i];
    return MTR_OK;
  });
}

int mtr_get_clock(mtr_ctx* c, mtr_clock* ck) {
  return guarded([&]() -> int {
    if (!c || !ck) throw MtrError{MTR_ERR_INVALID, "null argument"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    ck->time = c->hH->time;
    ck->dt = c->hH->dt;
    ck->step = c->hH->step;
    ck->frame = c->hH->frame;
    ck->done = c->hH->done;
    ck->reserved = 0;
    return MTR_OK;
  });
}

int mtr_status(mtr_ctx* c, uint32_t* flags, uint32_t* first_bad) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    if (flags) *flags = c->hH->status;
    if (first_bad) *first_bad = c->hH->first_bad;
    return MTR_OK;
  });
}

int mtr_clear_status(mtr_ctx* c) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    c->hH->status = 0;
    c->hH->first_bad = 0xffffffffu;
    write_header(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
}

int mtr_sync(mtr_ctx* c, double timeout_seconds) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    CK(cudaSetDevice(c->device));
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, c->stream));
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      cudaError_t e = cudaEventQuery(ev);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) {
        cudaEventDestroy(ev);
        throw MtrError{MTR_ERR_CUDA, cudaGetErrorString(e)};
      }
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > timeout_seconds) {
        cudaEventDestroy(ev);
        throw MtrError{MTR_ERR_TIMEOUT, "device did not finish within the timeout"};
      }
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    cudaEventDestroy(ev);
    return MTR_OK;
  });
}

void* mtr_stream(mtr_ctx* c) { return c ? (void*)c->stream : nullptr; }

int64_t mtr_launch_count(mtr_ctx* c) { return c ? c->launches_last : 0; }

// Not in the header: graph replay on/off (on by default) for timing studies.
int mtr_use_graphs(mtr_ctx* c, int on) {
  if (!c) return MTR_ERR_INVALID;
  c->use_graphs = on != 0;
  cudaSetDevice(c->device);
  free_graphs(c);
  return MTR_OK;
}

int mtr_profile(mtr_ctx* c, int nsteps, double* slot_ms, const char** slot_names, int max_slots, int* nslots) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded || nsteps <= 0 || !nslots) throw MtrError{MTR_ERR_INVALID, "bad profile request"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    if (c->hH->done) throw MtrError{MTR_ERR_STATE, "simulation already finished"};
    int parity = c->hH->cur;
    std::vector<double> acc;
    std::vector<const char*> names;
    c->marks.on = true;
    int done_steps = 0;
    try {
      for (int s = 0; s < nsteps; ++s) {
        c->marks.reset();
        enqueue_step(c, parity);
        parity ^= 1;
        CK(cudaStreamSynchronize(c->stream));
        const auto& L = c->marks.list;
        if (acc.empty()) {
          acc.assign(L.size() - 1, 0.0);
          for (size_t i = 1; i < L.size(); ++i) names.push_back(L[i].first);
        }
        for (size_t i = 1; i < L.size() && i - 1 < acc.size(); ++i) acc[i - 1] += c->marks.since_previous(i);
        ++done_steps;
      }
    } catch (...) {
      c->marks.on = false;
      throw;
    }
    c->marks.on = false;
    read_header(c);
    if (c->hH->abort) throw MtrError{MTR_ERR_STATE, "grid regrowth during profiling; step first"};
    *nslots = (int)acc.size();
    for (int i = 0; i < (int)acc.size() && i < max_slots; ++i) {
      if (slot_ms) slot_ms[i] = acc[i] / done_steps;
      if (slot_names) slot_names[i] = names[i];
    }
    return MTR_OK;
  });
}

int mtr_set_levelset(mtr_ctx* c, int slot, const float* phi, const float* normals, const uint32_t dims[3],
                     const double origin[3], double spacing) {
  return guarded([&]() -> int {
    if (!c || !phi || !dims || !origin) throw MtrError{MTR_ERR_INVALID, "null argument"};
    if (slot < 0 || slot >= MTR_MAX_LEVELSETS) throw MtrError{MTR_ERR_INVALID, "slot out of range"};
    if (!(spacing > 0) || !std::isfinite(spacing)) throw MtrError{MTR_ERR_INVALID, "spacing must be positive"};
    if (dims[0] < 2 || dims[1] < 2 || (c->dim == 3 ? dims[2] < 2 : dims[2] != 1))
      throw MtrError{MTR_ERR_INVALID, "dims: at least 2 samples per axis (dims[2] = 1 in 2D)"};
    const uint64_t n = (uint64_t)dims[0] * dims[1] * dims[2];
    if (n > (1ull << 34)) throw MtrError{MTR_ERR_TOO_LARGE, "level set larger than 2^34 samples"};
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));  // no step may still read the old arrays
    dfree(c->ls_phi[slot]);
    dfree(c->ls_grad[slot]);
    c->ls_phi[slot] = c->ls_grad[slot] = nullptr;
    c->hp.ls[slot] = DevParams::LevelSet{};
    float* dphi = dalloc<float>(n);
    c->ls_phi[slot] = dphi;
    float* dgrad = dalloc<float>(3 * n);
    c->ls_grad[slot] = dgrad;
    CK(cudaMemcpyAsync(dphi, phi, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    const float background = (float)(3.0 * spacing);
    if (normals) {
      CK(cudaMemcpyAsync(dgrad, normals, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    } else {
      k_levelset_grad<<<cap_blocks(n, 256, 148 * 16), 256, 0, c->stream>>>(dphi, dgrad, dims[0], dims[1], dims[2],
                                                                        c->dim, background, 0.5 / spacing);
      CK(cudaGetLastError());
    }
    DevParams::LevelSet& L = c->hp.ls[slot];
    L.phi = dphi;
    L.grad = dgrad;
    for (int a = 0; a < 3; ++a) {
      L.n[a] = dims[a];
      L.org[a] = a < c->dim ? origin[a] : 0.0;
    }
    L.h = spacing;
    L.inv_h = 1.0 / spacing;
    L.background = (double)background;
    upload_params(c);
    CK(cudaStreamSynchronize(c->stream));
    return MTR_OK;
  });
}

int mtr_frame_columns(mtr_ctx* c, const char** names, int max_names) {
  if (!c) return MTR_ERR_INVALID;
  std::vector<const char*> n;
  frame_columns(c->prm, &n);
  for (int i = 0; names && i < (int)n.size() && i < max_names; ++i) names[i] = n[i];
  return (int)n.size();
}

int mtr_frame_begin(mtr_ctx* c) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    if (!c->copy_stream) {
      CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&c->frame_ready, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->frame_copied, cudaEventDisableTiming));
    }
    if (c->frame_pending) CK(cudaEventSynchronize(c->frame_copied));  // frame_dev is about to be rewritten
    c->frame_pending = false;
    std::vector<const char*> names;
    const unsigned cols = frame_columns(c->prm, &names);
    const int ncols = (int)names.size();
    const size_t need = (size_t)c->Np * ncols + 8;
    if (need > c->frame_cap) {
      dfree(c->frame_dev);
      if (c->frame_host) cudaFreeHost(c->frame_host);
      c->frame_dev = nullptr;
      c->frame_host = nullptr;
      c->frame_cap = 0;
      c->frame_dev = dalloc<double>(need);
      void* h = nullptr;
      if (cudaMallocHost(&h, sizeof(double) * need) != cudaSuccess) throw MtrError{MTR_ERR_OOM, "cudaMallocHost"};
      c->frame_host = (double*)h;
      c->frame_cap = need;
    }
    const uint32_t Np = c->Np, blocks = (Np + 255) / 256;
    double* clock = c->frame_dev + (size_t)Np * ncols;
    if (c->fp32) {
      auto launch = [&](auto dimc) {
        constexpr int D = decltype(dimc)::value;
        k_frame_rows<D, float><<<blocks, 256, 0, c->stream>>>(typed<float>(c->buf[0]), typed<float>(c->buf[1]), c->dH,
                                                               c->dP, Np, cols, (uint32_t)ncols, c->frame_dev, clock);
      };
      c->dim == 3 ? launch(std::integral_constant<int, 3>{}) : launch(std::integral_constant<int, 2>{});
    } else {
      auto launch = [&](auto dimc) {
        constexpr int D = decltype(dimc)::value;
        k_frame_rows<D, double><<<blocks, 256, 0, c->stream>>>(typed<double>(c->buf[0]), typed<double>(c->buf[1]),
                                                                c->dH, c->dP, Np, cols, (uint32_t)ncols, c->frame_dev,
                                                                clock);
      };
      c->dim == 3 ? launch(std::integral_constant<int, 3>{}) : launch(std::integral_constant<int, 2>{});
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->frame_ready, c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, c->frame_ready, 0));
    CK(cudaMemcpyAsync(c->frame_host, c->frame_dev, sizeof(double) * ((size_t)Np * ncols + 5), cudaMemcpyDeviceToHost,
                       c->copy_stream));
    CK(cudaEventRecord(c->frame_copied, c->copy_stream));
    c->frame_pending = true;
    c->frame_n = Np;
    c->frame_ncols = ncols;
    return MTR_OK;
  });
}

int mtr_frame_wait(mtr_ctx* c, double timeout_seconds, const double** rows, uint32_t* n, int* ncols,
                   mtr_clock* clock) {
  return guarded([&]() -> int {
    if (!c) throw MtrError{MTR_ERR_INVALID, "null context"};
    if (!c->frame_pending) throw MtrError{MTR_ERR_STATE, "no frame snapshot in flight (mtr_frame_begin first)"};
    CK(cudaSetDevice(c->device));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t e = cudaEventQuery(c->frame_copied);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) CK(e);
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_seconds)
        throw MtrError{MTR_ERR_TIMEOUT, "frame snapshot not copied within the timeout"};
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    c->frame_pending = false;
    const double* ck = c->frame_host + (size_t)c->frame_n * c->frame_ncols;
    if (rows) *rows = c->frame_host;
    if (n) *n = c->frame_n;
    if (ncols) *ncols = c->frame_ncols;
    if (clock) {
      clock->time = ck[0];
      clock->dt = ck[1];
      clock->step = (uint32_t)ck[2];
      clock->frame = (uint32_t)ck[3];
      clock->done = (int32_t)ck[4];
      clock->reserved = 0;
    }
    return MTR_OK;
  });
}

int mtr_get_grid_friction(mtr_ctx* c, double* friction) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded || !friction) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    if (!c->prm.use_mibf) throw MtrError{MTR_ERR_INVALID, "grid friction exists with use_mibf only"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    if (c->hH->G > c->cap_nodes) throw MtrError{MTR_ERR_STATE, "no completed step"};
    get_nodes(c, friction, c->nfric, c->hH->G);
    return MTR_OK;
  });
}

int mtr_set_tile_threads(mtr_ctx* c, const int* threads) {
  return guarded([&]() -> int {
    if (!c || !threads) throw MtrError{MTR_ERR_INVALID, "null argument"};
    if (!valid_tile_threads(threads)) throw MtrError{MTR_ERR_INVALID, "tile threads: multiples of 32, 32..256 (USL G2P: ..128)"};
    CK(cudaSetDevice(c->device));
    std::copy(threads, threads + kTileSlots, c->tile_threads);
    free_graphs(c);
    return MTR_OK;
  });
}

int mtr_get_tile_threads(mtr_ctx* c, int* threads) {
  if (!c || !threads) return MTR_ERR_INVALID;
  std::copy(c->tile_threads, c->tile_threads + kTileSlots, threads);
  return MTR_OK;
}

int mtr_set_tile_lanes(mtr_ctx* c, const int* lanes) {
  return guarded([&]() -> int {
    if (!c || !lanes) throw MtrError{MTR_ERR_INVALID, "null argument"};
    if (!valid_tile_lanes(c->dim, lanes)) throw MtrError{MTR_ERR_INVALID, "lanes per particle: 16 or 32 (3D), 4 or 8 (2D)"};
    CK(cudaSetDevice(c->device));
    for (int i = 0; i < kScatterSlots; ++i) c->tile_split[i] = lanes[i] / scatter_columns(c->dim);
    free_graphs(c);
    return MTR_OK;
  });
}

int mtr_get_tile_lanes(mtr_ctx* c, int* lanes) {
  if (!c || !lanes) return MTR_ERR_INVALID;
  for (int i = 0; i < kScatterSlots; ++i) lanes[i] = c->tile_split[i] * scatter_columns(c->dim);
  return MTR_OK;
}

int mtr_autotune(mtr_ctx* c, int reps, int* threads) {
  return guarded([&]() -> int {
    if (!c || reps <= 0) throw MtrError{MTR_ERR_INVALID, "null context or reps <= 0"};
    if (!c->uploaded) throw MtrError{MTR_ERR_STATE, "mtr_autotune before mtr_upload"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    StepHeader saved = *c->hH;
    const bool active = !saved.done && saved.frame < saved.stop_frame && saved.step < saved.stop_step;
    if (active) {
      const int parity = saved.cur;
      TrialScope scope(&c->trial, &c->marks.on);
      // an untimed trial first; it also meets a grid overflow the next step would meet
      bool ready = false;
      for (int attempt = 0; attempt < 8 && !ready; ++attempt) {
        c->trial = true;
        enqueue_step(c, parity);
        read_header(c);
        if (c->hH->abort) {
          regrow_grid(c, *c->hH);
          *c->hH = saved;
          write_header(c);
          CK(cudaStreamSynchronize(c->stream));
        } else {
          ready = true;
        }
      }
      if (!ready) throw MtrError{MTR_ERR_STATE, "grid kept growing during tuning"};
      TuneTimes tt;
      int chosen[kTileSlots], chosen_split[kScatterSlots];
      std::copy(c->tile_threads, c->tile_threads + kTileSlots, chosen);
      std::copy(c->tile_split, c->tile_split + kScatterSlots, chosen_split);
      c->marks.on = true;
      for (int r = 0; r < reps; ++r)
        for (int k = 0; k < kTuneRounds; ++k) {
          set_candidate(c->tile_threads, c->tile_split, k);
          c->marks.reset();
          enqueue_step(c, parity);
          CK(cudaStreamSynchronize(c->stream));
          const auto& L = c->marks.list;
          for (size_t i = 1; i < L.size(); ++i) tt.add(L[i].first, c->marks.since_previous(i), k);
        }
      tt.choose(chosen, chosen_split);
      std::copy(chosen, chosen + kTileSlots, c->tile_threads);
      std::copy(chosen_split, chosen_split + kScatterSlots, c->tile_split);
      *c->hH = saved;  // the trial steps leave no trace: clock, plates, counters as before
      write_header(c);
      CK(cudaStreamSynchronize(c->stream));
      free_graphs(c);
    }
    if (threads) std::copy(c->tile_threads, c->tile_threads + kTileSlots, threads);
    return MTR_OK;
  });
}

int mtr_active_nodes(mtr_ctx* c, uint64_t* active, uint64_t* total) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    std::vector<double> m(c->hH->G);
    get_nodes(c, m.data(), c->nmass, m.size());
    uint64_t a = 0;
    for (double v : m) a += v > 0;
    if (active) *active = a;
    if (total) *total = m.size();
    return MTR_OK;
  });
}

int mtr_balance(mtr_ctx* c, double* grid_mass, double* grid_momentum, double* particle_mass,
                double* particle_momentum) {
  return guarded([&]() -> int {
    if (!c || !c->uploaded) throw MtrError{MTR_ERR_STATE, "nothing uploaded"};
    CK(cudaSetDevice(c->device));
    read_header(c);
    const StepHeader& H = *c->hH;
    if (grid_mass) *grid_mass = H.grid_mass;
    if (particle_mass) *particle_mass = c->prm.particle_mass * (double)c->Np;
    for (int a = 0; a < c->dim; ++a) {
      if (grid_momentum) grid_momentum[a] = H.grid_mom[a];
      if (particle_momentum) particle_momentum[a] = H.part_mom[a];
    }
    return MTR_OK;
  });
}

int mtr_footprint(const mtr_params* params, uint32_t Np, const double* x, uint64_t* bytes) {
  return guarded([&]() -> int {
    if (!params || !x || !bytes || Np == 0) throw MtrError{MTR_ERR_INVALID, "null argument or Np == 0"};
    const mtr_params& p = *params;
    if ((p.dim != 2 && p.dim != 3) || !(p.dx > 0)) throw MtrError{MTR_ERR_INVALID, "dim must be 2 or 3, dx > 0"};
    const uint64_t d = p.dim, dd = d * d, ns = p.dim == 3 ? 6 : 3, n = Np;
    const uint64_t rs = p.precision == MTR_PREC_MIXED ? 4 : 8;
    const uint64_t sort_blocks = (n + kSortTile - 1) / kSortTile;
    uint64_t total = 2 * (8 * d * n + rs * n * (d + 2 * dd + MTR_NUM_SCALARS + ns) + 4 * n)  // particle buffers
                     + 2 * rs * d * n                                                      // pic, flip
                     + 5 * 4 * n + 4 * 256 * sort_blocks + 4 * 256                           // sort
                     + 8 * n * std::max<uint64_t>(dd, MTR_NUM_SCALARS);                       // staging
    uint32_t want[3];
    grid_extent(p, Np, x, want);
    const uint64_t tb = p.dim == 3 ? 4 : 8;
    uint64_t nodes = 1, tiles = 1, axes = 0;
    for (int a = 0; a < 3; ++a) {
      const uint64_t cap = a < p.dim ? std::max<uint32_t>(want[a], 8u) : 1u;
      nodes *= cap;
      tiles *= a < p.dim ? (cap + tb - 1) / tb : 1;
      axes += cap;
    }
    total += 8 * axes + rs * (2 + 2 * d) * nodes + 8 * d * nodes + rs * d * nodes + 2 * rs * nodes + 8 * d * nodes +
             8 * tiles;
    *bytes = total;
    return MTR_OK;
  });
}

}  // extern "C"

namespace {

// Checks a member list and (re)groups it into b: groups keep their order and
// block shapes when their key (dim, spline, precision, MUSL, return-mapping
// kernel) stays in use, new keys are appended with the shapes of their first
// member, and groups left without members are dropped.
void assign_members(mtr_batch* b, mtr_ctx* const* ctxs, int n) {
  if (!ctxs || n <= 0) throw MtrError{MTR_ERR_INVALID, "null argument or n <= 0"};
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || !ctxs[i]->uploaded) throw MtrError{MTR_ERR_STATE, "every member needs mtr_upload first"};
    check_levelsets(ctxs[i]);
    if (ctxs[i]->device != ctxs[0]->device) throw MtrError{MTR_ERR_INVALID, "members must share one device"};
    if (ctxs[i]->prm.pbc) throw MtrError{MTR_ERR_INVALID, "periodic scenes step on their own, not in a batch"};
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) throw MtrError{MTR_ERR_INVALID, "a context appears twice"};
  }
  if (!b->members.empty() && ctxs[0]->device != b->device)
    throw MtrError{MTR_ERR_INVALID, "members must share the batch's device"};
  b->members.clear();
  for (auto& g : b->groups) {
    g.members.clear();
    g.tuned_nodes = 0;  // a new membership: its grid size is the next baseline
  }
  for (int i = 0; i < n; ++i) {
    mtr_ctx* c = ctxs[i];
    CK(cudaStreamSynchronize(c->stream));  // nothing of the member may still run on its own stream
    b->members.push_back(c);
    mtr_batch_group* g = nullptr;
    const int musl = c->prm.use_musl ? 1 : 0;
    const int spm = rm_specialization(c->dim, musl != 0, c->prm.plastic_model);
    for (auto& q : b->groups)
      if (q.dim == c->dim && q.deg == c->deg && q.fp32 == c->fp32 && q.musl == musl && q.spm == spm) g = &q;
    if (!g) {
      b->groups.emplace_back();
      g = &b->groups.back();
      g->dim = c->dim;
      g->deg = c->deg;
      g->fp32 = c->fp32;
      g->musl = musl;
      g->spm = spm;
      std::copy(c->tile_threads, c->tile_threads + kTileSlots, g->tile_threads);
      std::copy(c->tile_split, c->tile_split + kScatterSlots, g->tile_split);
    }
    g->members.push_back(c);
  }
  for (size_t i = 0; i < b->groups.size();) {
    if (b->groups[i].members.empty()) {
      mtr_batch_group& g = b->groups[i];
      if (g.dargs) cudaFreeAsync(g.dargs, b->stream);
      if (g.doff) cudaFreeAsync(g.doff, b->stream);
      b->groups.erase(b->groups.begin() + (long)i);
    } else {
      ++i;
    }
  }
  b->dirty = true;
}

}  // namespace

extern "C" {

int mtr_batch_create(mtr_ctx* const* ctxs, int n, mtr_batch** out) {
  return guarded([&]() -> int {
    if (!ctxs || !out || n <= 0) throw MtrError{MTR_ERR_INVALID, "null argument or n <= 0"};
    *out = nullptr;
    mtr_batch* b = new mtr_batch();
    try {
      if (!ctxs[0]) throw MtrError{MTR_ERR_INVALID, "null member"};
      b->device = ctxs[0]->device;
      CK(cudaSetDevice(b->device));
      CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
      assign_members(b, ctxs, n);
    } catch (...) {
      mtr_batch_destroy(b);
      throw;
    }
    *out = b;
    return MTR_OK;
  });
}

int mtr_batch_set_members(mtr_batch* b, mtr_ctx* const* ctxs, int n) {
  return guarded([&]() -> int {
    if (!b) throw MtrError{MTR_ERR_INVALID, "null batch"};
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    assign_members(b, ctxs, n);
    return MTR_OK;
  });
}

int mtr_batch_step(mtr_batch* b, int nsteps) {
  return guarded([&]() -> int {
    if (!b) throw MtrError{MTR_ERR_INVALID, "null batch"};
    if (nsteps <= 0) return MTR_OK;
    CK(cudaSetDevice(b->device));
    read_batch_headers(b);
    for (mtr_ctx* c : b->members) {  // every member advances nsteps steps (or to its end)
      StepHeader& H = *c->hH;
      H.stop_step = (uint32_t)std::min<uint64_t>(std::min<uint64_t>((uint64_t)H.step + (uint64_t)nsteps, 0xfffffffeull),
                                                 c->step_limit);
    }
    write_batch_headers(b);
    int64_t launches = 0;
    int regrowths = 0;
    for (;;) {
      uint32_t remaining = 0;
      uint64_t steps_before = 0;
      for (mtr_ctx* c : b->members) {
        steps_before += c->hH->step;
        if (!c->hH->done && c->hH->step < c->hH->stop_step)
          remaining = std::max(remaining, c->hH->stop_step - c->hH->step);
      }
      if (remaining == 0) break;
      if (b->dirty || !b->graph) {
        const auto t0 = std::chrono::steady_clock::now();
        rebuild_batch(b);
        b->rebuilds += 1;
        b->rebuild_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      }
      // Replay in runs of at most kBatchCheckSteps steps and read the headers
      // after each: a member whose grid outgrew its capacity sits out the
      // rest of the run (its header aborts), and every step it missed costs
      // a replay of the whole batch later, so a short run bounds that waste.
      const uint32_t run = std::min<uint32_t>(remaining, kBatchCheckSteps);
      const uint32_t reps = (run + kBatchGraphSteps - 1) / kBatchGraphSteps;
      for (uint32_t r = 0; r < reps; ++r) {
        CK(cudaGraphLaunch(b->graph, b->stream));
        launches += (int64_t)b->launches_per_step * kBatchGraphSteps;
      }
      read_batch_headers(b);
      bool regrown = false;
      uint64_t steps_after = 0;
      for (mtr_ctx* c : b->members) {
        StepHeader& H = *c->hH;
        steps_after += H.step;
        if (!H.abort) continue;
        const auto t0 = std::chrono::steady_clock::now();
        regrow_grid(c, H);
        b->regrowths += 1;
        b->regrow_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        regrown = true;
      }
      if (regrown) {
        if (++regrowths > 4096) throw MtrError{MTR_ERR_STATE, "batch grids kept growing"};
        write_batch_headers(b);
        b->dirty = true;
      } else if (steps_after == steps_before) {
        break;  // no member can advance (ended, or held by a frame stop)
      }
      // Re-tuning (mtr_batch_set_retune) is checked after regrowths too: a
      // spreading scene regrows at most checks, and its grid doubles at one.
      if (b->retune_reps > 0) {
        bool retune = false;
        for (auto& g : b->groups) {
          uint64_t nodes = 0;
          for (mtr_ctx* c : g.members) nodes += c->hH->G;
          if (g.tuned_nodes == 0)
            g.tuned_nodes = nodes;
          else if (nodes > 2 * g.tuned_nodes)
            retune = true;
        }
        if (retune) {
          const int rc = mtr_batch_autotune(b, b->retune_reps);
          if (rc != MTR_OK) throw MtrError{rc, std::string("re-tuning the batch: ") + mtr_last_error()};
          b->retunes += 1;
        }
      }
    }
    for (mtr_ctx* c : b->members) {
      c->hH->stop_step = c->step_limit;
      c->host_parity = c->hH->cur;
    }
    write_batch_headers(b);
    b->launches_last = launches;
    return MTR_OK;
  });
}

int mtr_batch_groups(mtr_batch* b) { return b ? (int)b->groups.size() : MTR_ERR_INVALID; }

int mtr_batch_clocks(mtr_batch* b, mtr_clock* clocks, int n) {
  if (!b || !clocks || n < (int)b->members.size()) return MTR_ERR_INVALID;
  for (size_t i = 0; i < b->members.size(); ++i) {  // host mirrors, read at the end of mtr_batch_step
    const StepHeader& H = *b->members[i]->hH;
    clocks[i].time = H.time;
    clocks[i].dt = H.dt;
    clocks[i].step = H.step;
    clocks[i].frame = H.frame;
    clocks[i].done = H.done;
    clocks[i].reserved = 0;
  }
  return (int)b->members.size();
}

int mtr_batch_get_group(mtr_batch* b, int group, mtr_group_info* info) {
  if (!b || !info || group < 0 || group >= (int)b->groups.size()) return MTR_ERR_INVALID;
  const mtr_batch_group& g = b->groups[group];
  info->dim = g.dim;
  info->spline_deg = g.deg;
  info->fp32 = g.fp32 ? 1 : 0;
  info->musl = g.musl;
  info->plastic_model_kernel = g.spm;
  info->members = (int)g.members.size();
  std::copy(g.tile_threads, g.tile_threads + kTileSlots, info->tile_threads);
  for (int i = 0; i < kScatterSlots; ++i) info->tile_lanes[i] = g.tile_split[i] * scatter_columns(g.dim);
  return MTR_OK;
}

int mtr_batch_set_tile_lanes(mtr_batch* b, int group, const int* lanes) {
  return guarded([&]() -> int {
    if (!b || !lanes || group < 0 || group >= (int)b->groups.size()) throw MtrError{MTR_ERR_INVALID, "bad group"};
    mtr_batch_group& g = b->groups[group];
    if (!valid_tile_lanes(g.dim, lanes)) throw MtrError{MTR_ERR_INVALID, "lanes per particle: 16 or 32 (3D), 4 or 8 (2D)"};
    for (int i = 0; i < kScatterSlots; ++i) g.tile_split[i] = lanes[i] / scatter_columns(g.dim);
    b->dirty = true;
    return MTR_OK;
  });
}

int mtr_batch_set_tile_threads(mtr_batch* b, int group, const int* threads) {
  return guarded([&]() -> int {
    if (!b || !threads || group < 0 || group >= (int)b->groups.size()) throw MtrError{MTR_ERR_INVALID, "bad group"};
    if (!valid_tile_threads(threads)) throw MtrError{MTR_ERR_INVALID, "tile threads: multiples of 32, 32..256 (USL G2P: ..128)"};
    std::copy(threads, threads + kTileSlots, b->groups[group].tile_threads);
    b->dirty = true;
    return MTR_OK;
  });
}

int mtr_batch_autotune(mtr_batch* b, int reps) {
  return guarded([&]() -> int {
    if (!b || reps <= 0) throw MtrError{MTR_ERR_INVALID, "null batch or reps <= 0"};
    CK(cudaSetDevice(b->device));
    if (b->dirty || !b->graph) rebuild_batch(b);
    read_batch_headers(b);
    std::vector<StepHeader> saved;
    bool any = false;
    for (mtr_ctx* c : b->members) {
      saved.push_back(*c->hH);
      StepHeader& H = *c->hH;
      // one step of every member that still runs; the others stay inactive
      const bool run = !H.done && H.frame < H.stop_frame && H.step < c->step_limit;
      H.stop_step = run ? H.step + 1 : H.step;
      any = any || run;
    }
    std::vector<StepHeader> trial_headers;
    for (mtr_ctx* c : b->members) trial_headers.push_back(*c->hH);
    write_batch_headers(b);
    if (any) {
      TrialScope scope(&b->trial, &b->marks.on);
      bool ready = false;
      for (int attempt = 0; attempt < 8 && !ready; ++attempt) {
        b->trial = true;
        enqueue_batch_step(b);
        b->trial = false;
        read_batch_headers(b);
        bool regrown = false;
        for (size_t i = 0; i < b->members.size(); ++i) {
          mtr_ctx* c = b->members[i];
          if (!c->hH->abort) continue;
          regrow_grid(c, *c->hH);
          regrown = true;
        }
        if (regrown) {
          for (size_t i = 0; i < b->members.size(); ++i) *b->members[i]->hH = trial_headers[i];
          write_batch_headers(b);
          rebuild_batch(b);
        } else {
          ready = true;
        }
      }
      if (!ready) throw MtrError{MTR_ERR_STATE, "grid kept growing during tuning"};
      // the grid sizes the shapes are tuned on (the trial step computed them)
      for (auto& g : b->groups) {
        uint64_t nodes = 0;
        for (mtr_ctx* c : g.members) nodes += c->hH->G;
        g.tuned_nodes = nodes;
      }
      std::vector<TuneTimes> tt(b->groups.size());
      std::vector<std::vector<int>> chosen, chosen_split;
      for (auto& g : b->groups) {
        chosen.emplace_back(g.tile_threads, g.tile_threads + kTileSlots);
        chosen_split.emplace_back(g.tile_split, g.tile_split + kScatterSlots);
      }
      b->marks.on = true;
      b->trial = true;
      for (int r = 0; r < reps; ++r)
        for (int k = 0; k < kTuneRounds; ++k) {
          for (auto& g : b->groups) set_candidate(g.tile_threads, g.tile_split, k);
          b->marks.reset();
          b->marks.record("start", b->stream, -1);
          enqueue_batch_step(b);
          CK(cudaStreamSynchronize(b->stream));
          const auto& L = b->marks.list;
          for (size_t i = 1; i < L.size(); ++i)
            if (b->marks.tag[i] == b->marks.tag[i - 1]) tt[b->marks.tag[i]].add(L[i].first, b->marks.since_previous(i), k);
        }
      for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        tt[gi].choose(chosen[gi].data(), chosen_split[gi].data());
        std::copy(chosen[gi].begin(), chosen[gi].end(), b->groups[gi].tile_threads);
        std::copy(chosen_split[gi].begin(), chosen_split[gi].end(), b->groups[gi].tile_split);
      }
    }
    for (size_t i = 0; i < b->members.size(); ++i) *b->members[i]->hH = saved[i];
    write_batch_headers(b);
    b->dirty = true;
    return MTR_OK;
  });
}

int mtr_batch_set_retune(mtr_batch* b, int reps) {
  if (!b || reps < 0) return MTR_ERR_INVALID;
  b->retune_reps = reps;
  return MTR_OK;
}

int mtr_batch_retunes(mtr_batch* b) { return b ? (int)std::min<int64_t>(b->retunes, 0x7fffffff) : MTR_ERR_INVALID; }

int64_t mtr_batch_launch_count(mtr_batch* b) { return b ? b->launches_last : 0; }

int mtr_batch_graph_updates(mtr_batch* b) { return b ? (int)std::min<int64_t>(b->updates, 0x7fffffff) : MTR_ERR_INVALID; }

int mtr_batch_stats(mtr_batch* b, int64_t* regrowths, double* regrow_ms, int64_t* rebuilds, double* rebuild_ms) {
  if (!b) return MTR_ERR_INVALID;
  if (regrowths) *regrowths = b->regrowths;
  if (regrow_ms) *regrow_ms = b->regrow_ms;
  if (rebuilds) *rebuilds = b->rebuilds;
  if (rebuild_ms) *rebuild_ms = b->rebuild_ms;
  return MTR_OK;
}

void* mtr_batch_stream(mtr_batch* b) { return b ? (void*)b->stream : nullptr; }

void mtr_batch_destroy(mtr_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_batch_graph(b);
  free_batch_tables(b);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

void mtr_ctx_destroy(mtr_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
    cudaEventDestroy(c->frame_ready);
    cudaEventDestroy(c->frame_copied);
  }
  dfree(c->frame_dev);
  if (c->frame_host) cudaFreeHost(c->frame_host);
  for (int i = 0; i < MTR_MAX_LEVELSETS; ++i) {
    dfree(c->ls_phi[i]);
    dfree(c->ls_grad[i]);
  }
  free_graphs(c);
  free_grid(c);
  for (void* p : c->pallocs) dfree(p);
  for (void* p : {(void*)c->keys0, (void*)c->keysA, (void*)c->valsA, (void*)c->keysB, (void*)c->valsB,
                  (void*)c->hist, (void*)c->dtot, (void*)c->partials, (void*)c->staging, (void*)c->dP, (void*)c->dH})
    dfree(p);
  if (c->hH) cudaFreeHost(c->hH);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // extern "C"
