// api.cu -- the C ABI (include/nbx.h): handles, device memory, step
// sequencing and graph capture, introspection for parity checks.
#include "nbx.h"
#include "mlp.cuh"
#include "nbx_state.cuh"

#include <algorithm>
#include <cstddef>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

namespace nbx {
void launch_integrate(cudaStream_t s, const DevState &S, bool integrate,
                      bool collide);
void launch_collide(cudaStream_t s, DevState &S, ScanScratch &scan, SortScratch &sort,
                    const SideStream *side);
void launch_bounds(cudaStream_t s, const DevState &S);
void launch_build(cudaStream_t s, DevState &S, ScanScratch &scan,
                  SortScratch &sort, bool moments);
void launch_bfs_tree(cudaStream_t s, const DevState &S, ScanScratch &scan,
                     SortScratch &sort);
void launch_step_zero(cudaStream_t s, const DevState &S, ScanScratch &scan, SortScratch &sort,
                      bool grid);
void launch_forces(cudaStream_t s, const DevState &S, bool exact, int blocks,
                   const MlpDev *mlp, float band, int corr, bool noClamp, int threads,
                   bool pairs);
void render_vertices(cudaStream_t s, const float4 *pv, const float2 *mr, uint32_t n,
                     const RenderParams &P, float4 *v0, float4 *v1, uint32_t *tiles,
                     double4 *partial, unsigned long long *total, float *stats);
uint32_t render_vertex_blocks(uint32_t n);
void render_emit(cudaStream_t s, const float4 *v0, const uint32_t *off, uint32_t n,
                 const RenderParams &P, uint64_t *keys, uint32_t *vals);
void render_composite(cudaStream_t s, const float4 *v0, const float4 *v1,
                      const uint64_t *keys, const uint32_t *bodies, const uint32_t *count,
                      uint32_t maxEntries, uint32_t *first, uint32_t *last,
                      const RenderParams &P, float4 *image);
DevState launch_naive_gather(cudaStream_t s, const DevState &S);
void launch_naive_forces(cudaStream_t s, const DevState &S, bool exact);
void mlp_harvest(cudaStream_t s, const DevState &S, const uint32_t *targets,
                 uint32_t nt, float theta, float band, float eps, uint2 *items,
                 uint32_t cap, uint32_t *count, float *rows);
void mlp_pack(cudaStream_t s, const float *P, MlpDev *W);
void mlp_gradient(cudaStream_t s, const float *rows, const uint32_t *order,
                  uint32_t first, uint32_t batch, const float *P, float *partial,
                  float *lossPart, float *grad, float *loss);
void mlp_adam(cudaStream_t s, float *P, const float *grad, float *m, float *v,
              int step, float lr, MlpDev *W);
void mlp_eval(cudaStream_t s, const float *feat, uint32_t n, const float *P,
              const MlpDev *W, float *out, bool tensor);
int mlp_rows_per_block();
void launch_interaction_count(cudaStream_t s, const DevState &S,
                              unsigned long long *counts);
double fp32_fma_peak_tflops(cudaStream_t s);
void launch_query_forces(cudaStream_t s, const DevState &S, bool exact,
                         const float2 *query, uint32_t nq, float2 *out);
void launch_direct_fp64(cudaStream_t s, const float4 *pv, const float2 *mr,
                        uint32_t n, const uint32_t *targets, const uint2 *ranges,
                        uint32_t m, double eps, int plummer, double2 *partial,
                        double *ax, double *ay);
size_t direct_partial_elems(uint32_t m);
void launch_energy_momentum(cudaStream_t s, const float4 *pv, const float2 *mr,
                            uint32_t n, double *part, double *out);
} // namespace nbx

namespace nbx {
thread_local PhaseMarks *g_marks = nullptr;
}

using namespace nbx;

namespace {

// Unpacks body records; *maxMassBits receives the largest |mass| as float
// bits (non-negative floats order as their bit patterns; NaN orders last).
__global__ void k_unpack(const nbx_body *__restrict__ in, uint32_t n,
                         float4 *pv, float2 *acc, float2 *mr, uint32_t *id,
                         uint32_t *maxMassBits) {
  uint32_t mb = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const nbx_body b = in[i];
    pv[i] = make_float4(b.pos_x, b.pos_y, b.vel_x, b.vel_y);
    acc[i] = make_float2(b.acc_x, b.acc_y);
    mr[i] = make_float2(b.mass, b.radius);
    id[i] = b.id;
    // bit order = value order for non-negative floats; any negative mass
    // (sign bit set) lands above every non-negative one
    mb = max(mb, __float_as_uint(b.mass));
  }
  mb = __reduce_max_sync(0xffffffffu, mb);
  if ((threadIdx.x & 31) == 0 && mb) atomicMax(maxMassBits, mb);
}

// A bounded wait on a flag that nothing sets, shaped like the waits of the
// ordered resolution and the sort look-back (poll, back off, give up after
// kSpinLimit rounds and raise kStatusSpinLimit).
__global__ void k_expire_wait(const uint32_t *flag, uint32_t *status) {
  uint32_t idle = 0;
  for (;;) {
    if (ld_acquire_u32(flag) != 0u) return;
    if (++idle > kSpinLimit) {
      if (threadIdx.x == 0) atomicOr(status, kStatusSpinLimit);
      return;
    }
    __nanosleep(32);
  }
}

// NBS2 frame record in id order: {x, y, vx, vy} = the body's pv record.
__global__ void k_frame_scatter(const float4 *__restrict__ pv,
                                const uint32_t *__restrict__ id, uint32_t n,
                                float4 *__restrict__ frame) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    frame[id[i]] = pv[i];
}

// Body records; id_order scatters body i to instance_start + id.
__global__ void k_pack(const float4 *__restrict__ pv, const float2 *__restrict__ acc,
                       const float2 *__restrict__ mr, const uint32_t *__restrict__ id,
                       const uint16_t *__restrict__ segOf, const SegDev *seg,
                       uint32_t begin, uint32_t n, int idOrder, nbx_body *out) {
  for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const float4 p = pv[i];
    const float2 a = acc[i];
    const float2 m = mr[i];
    nbx_body b;
    b.pos_x = p.x;
    b.pos_y = p.y;
    b.vel_x = p.z;
    b.vel_y = p.w;
    b.acc_x = a.x;
    b.acc_y = a.y;
    b.mass = m.x;
    b.radius = m.y;
    b.id = id[i];
    const uint32_t dst = idOrder ? seg[segOf[i]].start + b.id : i;
    out[dst] = b;
  }
}

__global__ void k_check_ids(const uint32_t *__restrict__ id,
                            const uint16_t *__restrict__ segOf,
                            const SegDev *seg, uint32_t n, uint32_t *seen,
                            uint32_t *bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const SegDev &G = seg[segOf[i]];
    const uint32_t v = id[i];
    if (v >= G.count || atomicExch(&seen[G.start + v], 1u) != 0u) *bad = 1u;
  }
}

__global__ void k_fill_u16(uint16_t *p, uint32_t start, uint32_t count,
                           uint16_t v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += gridDim.x * blockDim.x)
    p[start + i] = v;
}

template <typename T> struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
};

} // namespace


// Device-path frame output: an id-order scatter on the handle's stream into
// one of two device frames, a copy into a pinned slot on a second stream
// (overlapping the following steps), and a writer thread that appends the
// slot to the file once its copy has completed.
struct FrameWriter {
  int device = 0;
  uint32_t n = 0;
  cudaStream_t copy = nullptr;
  float4 *dFrame[2] = {nullptr, nullptr};
  float *hSlot[2] = {nullptr, nullptr};
  cudaEvent_t scattered[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
  int next = 0;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<int, nbx_nbs2 *>> queue; // (slot, file), in call order
  bool busy[2] = {false, false};                // slot copied or being written
  bool stop = false;
  int err = NBX_OK;

  void run() {
    cudaSetDevice(device);
    for (;;) {
      std::pair<int, nbx_nbs2 *> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return; // stop with nothing pending
        job = queue.front();
      }
      const int sl = job.first;
      int rc = cudaEventSynchronize(copied[sl]) == cudaSuccess ? NBX_OK : NBX_ERR_CUDA;
      if (rc == NBX_OK) rc = nbx_nbs2_write_packed(job.second, hSlot[sl], n);
      {
        std::lock_guard<std::mutex> lk(mu);
        if (rc != NBX_OK && err == NBX_OK) err = rc;
        queue.pop_front();
        busy[sl] = false;
      }
      cv.notify_all();
    }
  }
};

struct nbx_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  nbx_params params{};
  uint32_t n = 0, nseg = 0;
  std::vector<uint32_t> segStart, segCount;
  std::vector<void *> allocs;
  DevState base{};       // buffer set A current
  int cur = 0;           // 0: state in set A (pv), 1: in set B (pv2)
  ScanScratch scan;
  SortScratch sort;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  uint32_t graphKernels = 0; // kernel nodes per captured step
  bool graphsValid = false;
  // timed step graphs: the same step with event-record nodes around the
  // force launch; each launch points them at the next pair of pool events
  cudaGraph_t graphTSrc[2] = {nullptr, nullptr};
  cudaGraphExec_t graphT[2] = {nullptr, nullptr};
  cudaGraphNode_t forceEvNode[2][2] = {};
  cudaEvent_t forceMark[2] = {nullptr, nullptr}; // placeholders at capture
  std::vector<cudaEvent_t> forceEv;               // 2 per timed step
  uint32_t timedSteps = 0;                        // steps of the last call
  bool timedValid = false;
  bool timedCapture = false;
  // step graphs of nbx_step_io: the force pass in kIoChunks target ranges
  // on their own streams, each range packed and copied to ioOut (pinned
  // host memory) as soon as its forces are done
  static constexpr int kIoChunks = 8;
  cudaGraphExec_t ioGraph[2] = {nullptr, nullptr};
  nbx_body *ioOut = nullptr;   // the host buffer the io graphs write
  bool ioCapture = false;
  cudaStream_t ioStream[kIoChunks] = {};
  SideStream side; // a step's independent branch (collide: chain entries)
  cudaEvent_t ioFork = nullptr;
  cudaEvent_t ioDone[kIoChunks] = {};
  bool uploaded = false;
  bool treeValid = false;   // a Barnes-Hut tree of the current state exists
  bool bfsValid = false;    // its breadth-first arrays (built on demand)
  bool momentsValid = false; // its cells' second moments were computed
  bool forceInput = false;  // S.xym holds the current state's bodies
  bool collideValid = false;
  bool idsChecked = false;     // ids verified to be per-instance permutations
  bool idsPermutation = false;
  nbx_body *dAoS = nullptr;     // device staging of body records
  nbx_body *hPinned = nullptr;  // pinned host staging
  // pinned words for the upload's small copies: [0] largest mass bits,
  // [1] coordinate limit bits, [4 + 3 s ..] instance s's collision cell
  uint32_t *hWord = nullptr;
  double2 *dPartial = nullptr;  // FP64 direct-sum partials
  uint32_t dPartialTargets = 0;
  double *dF64 = nullptr;       // small FP64 scratch
  uint32_t *dTargets = nullptr;
  std::string lastError;
  // learned correction
  float *mlpP = nullptr, *mlpM = nullptr, *mlpV = nullptr, *mlpGrad = nullptr;
  MlpDev *mlpW = nullptr;
  bool mlpLoaded = false;
  int mlpStep = 0;
  std::vector<void *> scratch; // grow-on-demand buffers (MLP data)
  // attractor (CudaSimulation.cuh:9-15 defaults): {x, y, mass, softening},
  // {active, 0, 0, 0}; mirrored into S.attr
  float attrHost[8] = {0.0f, 0.0f, 1e6f, 50.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float maxMass = INFINITY; // largest uploaded mass; +inf if any is negative
  FrameWriter *frames = nullptr; // created by the first nbx_nbs2_record
  // splat renderer buffers, grown on demand
  struct {
    uint32_t bodies = 0, entries = 0, tiles = 0;
    size_t pixels = 0;
    float4 *v0 = nullptr, *v1 = nullptr, *image = nullptr;
    uint32_t *count = nullptr, *off = nullptr, *first = nullptr, *last = nullptr;
    double4 *partial = nullptr;
    unsigned long long *total = nullptr;
    float *stats = nullptr;
    SortScratch sort;
  } rs;

  DevState state() const {
    DevState S = base;
    if (cur == 1) {
      std::swap(S.pv, S.pv2);
      std::swap(S.mr, S.mr2);
      std::swap(S.id, S.id2);
    }
    return S;
  }
};

namespace {

int fail(nbx_handle *h, int code, const std::string &msg) {
  if (h) h->lastError = msg;
  return code;
}

int cuda_fail(nbx_handle *h, cudaError_t e, const char *what) {
  if (h) {
    h->lastError = std::string(what) + ": " + cudaGetErrorString(e);
  }
  return e == cudaErrorMemoryAllocation ? NBX_ERR_NOMEM : NBX_ERR_CUDA;
}

#define NBX_CUDA(h, call)                                                    \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call);                 \
  } while (0)

template <typename T> cudaError_t dalloc(nbx_handle *h, T *&p, size_t count) {
  void *v = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&v, bytes);
  if (e != cudaSuccess) return e;
  h->allocs.push_back(v);
  p = static_cast<T *>(v);
  return cudaMemset(v, 0, bytes);
}

uint32_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

int allocate(nbx_handle *h) {
  DevState &S = h->base;
  const uint32_t n = h->n, ns = h->nseg;
  const nbx_params &P = h->params;
  S.n = n;
  S.nseg = ns;
  const double nf = P.node_factor > 0 ? P.node_factor : 8.0f;
  S.nodeCapacity = (uint32_t)std::min<double>(nf * n + 8.0 * ns + 8, 2.0e9);
  const double pf = P.pair_factor > 0 ? P.pair_factor : 32.0f;
  // chain entry indices carry two flag bits (collide.cu): below 2^30
  S.pairCapacity = (uint32_t)std::min<double>(pf * n + 64, (double)(1u << 30) - 64.0);
  S.nBuckets = next_pow2(2ull * std::max<uint32_t>(n, 1));
  const uint32_t nodes = S.nodeCapacity;
  const uint32_t sortCap = 2 * n + 64;
#define A(ptr, count) \
  if (cudaError_t e = dalloc(h, ptr, count)) return cuda_fail(h, e, "cudaMalloc " #ptr)
  A(S.seg, ns);
  A(S.segOf, n);
  A(S.pv, n);
  A(S.mr, n);
  A(S.id, n);
  A(S.pv2, n);
  A(S.mr2, n);
  A(S.id2, n);
  A(S.acc, n);
  A(S.xym, n);
  A(S.bounds, 4 * ns);
  A(S.status, 1);
  A(S.box, n);
  A(S.cellXY, n);
  A(S.slot, n);
  A(S.bucketCount, S.nBuckets + 1);
  A(S.bucketStart, S.nBuckets + 2);
  A(S.grid, n);
  A(S.gridBox, n);
  A(S.largeCount, ns);
  A(S.largeStartA, ns + 1);
  A(S.largeList, n);
  A(S.deg, n);
  A(S.pstart, n + 1);
  A(S.plist, S.pairCapacity);
  A(S.plistTmp, S.pairCapacity);
  A(S.twin, S.pairCapacity);
  A(S.stash, (size_t)n * 16);
  A(S.largePairs, n + 64);
  A(S.fillLarge, n);
  A(S.nLater, n);
  A(S.chain, S.pairCapacity);
  A(S.unitOrder, n);
  A(S.counters, 16);
  A(S.longRuns, n / 16 + 64);
  A(S.codes, n);
  A(S.perm, n);
  A(S.sortedCodes, n);
  A(S.splitCount, n);
  A(S.splitStart, n + 1);
  A(S.splitLo, n);
  A(S.groupStart, (size_t)ns * kLevelSlots);
  A(S.groupEnd, (size_t)ns * kLevelSlots);
  A(S.levelStart, (size_t)ns * (kLevelSlots + 1));
  A(S.comX, nodes);
  A(S.comY, nodes);
  A(S.mass, nodes);
  A(S.centerX, nodes);
  A(S.centerY, nodes);
  A(S.size, nodes);
  A(S.children, nodes);
  A(S.next, nodes);
  A(S.start, nodes);
  A(S.end, nodes);
  A(S.parent, nodes);
  A(S.sumX, nodes);
  A(S.sumY, nodes);
  A(S.moments, nodes);
  A(S.subtree, nodes);
  A(S.arrive, nodes);
  A(S.tN, nodes); // cudaMalloc: 256-byte aligned, so every record is 32
  A(S.tM, nodes);
  // scan / sort scratch
  SortScratch &so = h->sort;
  so.capacity = sortCap;
  so.maxTiles = (uint32_t)sort_tiles(sortCap);
  A(so.keys[0], sortCap);
  A(so.keys[1], sortCap);
  A(so.vals[0], sortCap);
  A(so.vals[1], sortCap);
  A(so.hist, 8 * 256);
  A(so.status, 8 * ((size_t)so.maxTiles * 256 + 256));
  A(so.tileCounter, 8);
  ScanScratch &sc = h->scan;
  sc.maxTiles = (uint32_t)scan_scratch_tiles(std::max<uint32_t>(S.nBuckets + 2, sortCap));
  A(sc.status, sc.maxTiles + 1);
  A(sc.slotStatus, (size_t)kScanSlots * sc.maxTiles);
  A(sc.tileCounter, kScanSlots);
  A(sc.tileCounter, 1);
  A(h->dAoS, n);
  A(h->dF64, 16 * 592);
  A(S.tC, nodes);
  A(h->mlpP, kMlpParams);
  A(h->mlpM, kMlpParams);
  A(h->mlpV, kMlpParams);
  A(h->mlpGrad, kMlpParams + 1);
  A(h->mlpW, 1);
  A(S.attr, 2);
#undef A
  NBX_CUDA(h, cudaMemcpy(S.attr, h->attrHost, sizeof(h->attrHost), cudaMemcpyHostToDevice));
  // bounds accumulators start empty
  std::vector<uint32_t> b(4 * ns);
  for (uint32_t s = 0; s < ns; ++s) {
    b[4 * s + 0] = 0xffffffffu;
    b[4 * s + 1] = 0u;
    b[4 * s + 2] = 0xffffffffu;
    b[4 * s + 3] = 0u;
  }
  NBX_CUDA(h, cudaMemcpy(S.bounds, b.data(), b.size() * 4, cudaMemcpyHostToDevice));
  // instance table and body -> instance map
  std::vector<SegDev> seg(ns);
  for (uint32_t s = 0; s < ns; ++s) {
    std::memset(&seg[s], 0, sizeof(SegDev));
    seg[s].start = h->segStart[s];
    seg[s].count = h->segCount[s];
    seg[s].cell = 1.0f;
    seg[s].invCell = 1.0f;
    seg[s].smallW = 0.999f;
  }
  NBX_CUDA(h, cudaMemcpy(S.seg, seg.data(), ns * sizeof(SegDev), cudaMemcpyHostToDevice));
  for (uint32_t s = 0; s < ns; ++s) {
    if (h->segCount[s] == 0) continue;
    k_fill_u16<<<256, 256, 0, h->stream>>>(S.segOf, h->segStart[s], h->segCount[s],
                                          (uint16_t)s);
  }
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  NBX_CUDA(h, cudaMallocHost(&h->hPinned, std::max<size_t>(n, 1) * sizeof(nbx_body)));
  NBX_CUDA(h, cudaMallocHost(&h->hWord, (4 + 3 * (size_t)ns) * sizeof(uint32_t)));
  return NBX_OK;
}

void sync_params(nbx_handle *h) {
  DevState &S = h->base;
  const nbx_params &P = h->params;
  S.dt = P.dt;
  S.tSq = P.theta * P.theta;
  S.eSq = P.epsilon * P.epsilon;
  S.leafCapacity = P.leaf_capacity;
  S.collisions = P.collisions;
}

// Whether the default force law (plain or with the quadrupole term) can
// leave out its FLT_MAX clamp: the factor
// m * fastInvSqrt(d^2) / (d^2 + eps^2) stays below FLT_MAX (fastInvSqrt <=
// ~2e19 for finite d^2) for a normal eps^2 and masses in
// [0, 1.6e19 * min(1, eps^2)); NaN or negative masses keep it.  Non-negative
// masses keep every centre of mass inside its bodies' box, and the build's
// per-instance coordinate check (SegDev::wide) keeps d^2 finite.
bool forces_unclamped(const nbx_handle *h) {
  const nbx_params &P = h->params;
  const float eSq = P.epsilon * P.epsilon;
  return !P.exact_math && P.use_mlp != 1 && eSq >= FLT_MIN &&
         h->maxMass < 1.6e19f * fminf(1.0f, eSq);
}

// Ranges of the force pass for nbx_step_io: whole warps, at most
// kIoChunks of them, none for fewer than 64K bodies (the copy is short).
uint32_t io_chunks(const nbx_handle *h) {
  const uint32_t c = h->n / 65536u;
  return c < 1u ? 1u : (c > (uint32_t)nbx_handle::kIoChunks ? (uint32_t)nbx_handle::kIoChunks : c);
}

// The force pass of an io step graph: each target range on its own stream
// (forked from s after the build, so the ranges run as one pool of blocks,
// dispatched in range order), writing its bodies' whole records; each
// range's records go to the host as soon as its launch ends, while the
// later ranges still compute.  s joins every range.
static_assert(sizeof(nbx_body) == 9 * sizeof(uint32_t), "the force pass writes 9-word records");
void enqueue_forces_io(nbx_handle *h, cudaStream_t s, const DevState &S) {
  const uint32_t n = S.n, chunks = io_chunks(h);
  const uint32_t per = ((n + chunks - 1) / chunks + 31u) & ~31u;
  cudaEventRecord(h->ioFork, s);
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t b = c * per, e = std::min(n, b + per);
    if (b >= e) break;
    cudaStream_t cs = h->ioStream[c];
    cudaStreamWaitEvent(cs, h->ioFork, 0);
    DevState R = S;
    R.forceBegin = b;
    R.forceEnd = e;
    R.recOut = reinterpret_cast<uint32_t *>(h->dAoS);
    launch_forces(cs, R, h->params.exact_math != 0, h->params.force_blocks,
                  h->mlpLoaded ? h->mlpW : nullptr, h->params.mlp_band, h->params.use_mlp,
                  forces_unclamped(h), h->params.force_block, h->params.leaf_pairs != 0);
    cudaMemcpyAsync(h->ioOut + b, h->dAoS + b, (size_t)(e - b) * sizeof(nbx_body),
                    cudaMemcpyDeviceToHost, cs);
    cudaEventRecord(h->ioDone[c], cs);
    cudaStreamWaitEvent(s, h->ioDone[c], 0);
  }
}

// One Simulation::step on stream s for state S; returns the state after the
// Morton gather's buffer swap.
DevState enqueue_step(nbx_handle *h, cudaStream_t s, DevState S) {
  launch_step_zero(s, S, h->scan, h->sort, S.collisions != 0);
  launch_integrate(s, S, true, S.collisions != 0);
  mark(s, "integrate");
  if (S.collisions) launch_collide(s, S, h->scan, h->sort, &h->side);
  if (h->params.force_law == 1) {
    S = launch_naive_gather(s, S);
    mark(s, "naive.gather");
    if (h->timedCapture) cudaEventRecordWithFlags(h->forceMark[0], s, cudaEventRecordExternal);
    launch_naive_forces(s, S, h->params.exact_math != 0);
    if (h->timedCapture) cudaEventRecordWithFlags(h->forceMark[1], s, cudaEventRecordExternal);
    mark(s, "forces");
    return S;
  }
  // second moments only where the force pass reads them
  launch_build(s, S, h->scan, h->sort, h->params.use_mlp != 0);
  if (h->ioCapture) {
    enqueue_forces_io(h, s, S);
    return S;
  }
  if (h->timedCapture) cudaEventRecordWithFlags(h->forceMark[0], s, cudaEventRecordExternal);
  launch_forces(s, S, h->params.exact_math != 0, h->params.force_blocks,
                h->mlpLoaded ? h->mlpW : nullptr, h->params.mlp_band,
                h->params.use_mlp, forces_unclamped(h), h->params.force_block,
                h->params.leaf_pairs != 0);
  if (h->timedCapture) cudaEventRecordWithFlags(h->forceMark[1], s, cudaEventRecordExternal);
  mark(s, "forces");
  return S;
}

void destroy_graphs(nbx_handle *h) {
  for (auto &g : h->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  h->graphsValid = false;
  for (int p = 0; p < 2; ++p) {
    if (h->graphT[p]) cudaGraphExecDestroy(h->graphT[p]);
    if (h->graphTSrc[p]) cudaGraphDestroy(h->graphTSrc[p]);
    h->graphT[p] = nullptr;
    h->graphTSrc[p] = nullptr;
  }
  h->timedValid = false;
  for (auto &g : h->ioGraph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  h->ioOut = nullptr;
}

// Flags after a whole step: the naive law builds no tree.
void after_step(nbx_handle *h) {
  h->treeValid = h->params.force_law == 0;
  h->bfsValid = false;
  h->momentsValid = h->params.use_mlp != 0; // what the step's build computed
  h->forceInput = true;
  h->collideValid = h->params.collisions != 0;
}

// Step graphs with the force launch bracketed by event-record nodes (kept
// with their source graphs, whose node handles re-point the events).
int capture_timed_graphs(nbx_handle *h) {
  for (int q = 0; q < 2; ++q)
    if (!h->forceMark[q]) NBX_CUDA(h, cudaEventCreate(&h->forceMark[q]));
  for (int p = 0; p < 2; ++p) {
    if (h->graphT[p]) cudaGraphExecDestroy(h->graphT[p]);
    if (h->graphTSrc[p]) cudaGraphDestroy(h->graphTSrc[p]);
    h->graphT[p] = nullptr;
    h->graphTSrc[p] = nullptr;
    const int saved = h->cur;
    h->cur = p;
    const DevState S = h->state();
    h->cur = saved;
    cudaGraph_t g = nullptr;
    NBX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->timedCapture = true;
    enqueue_step(h, h->stream, S);
    h->timedCapture = false;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    h->graphTSrc[p] = g;
    size_t count = 0;
    cudaGraphGetNodes(g, nullptr, &count);
    std::vector<cudaGraphNode_t> nodes(count);
    cudaGraphGetNodes(g, nodes.data(), &count);
    h->forceEvNode[p][0] = h->forceEvNode[p][1] = nullptr;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeEventRecord)
        continue;
      cudaEvent_t ev = nullptr;
      cudaGraphEventRecordNodeGetEvent(nd, &ev);
      for (int q = 0; q < 2; ++q)
        if (ev == h->forceMark[q]) h->forceEvNode[p][q] = nd;
    }
    if (!h->forceEvNode[p][0] || !h->forceEvNode[p][1])
      return fail(h, NBX_ERR_CUDA, "timed step graph lacks its event-record nodes");
    e = cudaGraphInstantiate(&h->graphT[p], g, 0);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
  }
  h->timedValid = true;
  return NBX_OK;
}

int capture_graphs(nbx_handle *h) {
  destroy_graphs(h);
  for (int p = 0; p < 2; ++p) {
    const int saved = h->cur;
    h->cur = p;
    const DevState S = h->state();
    h->cur = saved;
    cudaGraph_t g = nullptr;
    NBX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(h, h->stream, S);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    if (p == 0) {
      size_t count = 0;
      cudaGraphGetNodes(g, nullptr, &count);
      std::vector<cudaGraphNode_t> nodes(count);
      cudaGraphGetNodes(g, nodes.data(), &count);
      uint32_t kernels = 0;
      for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
          ++kernels;
      }
      h->graphKernels = kernels;
    }
    e = cudaGraphInstantiate(&h->graph[p], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
  }
  h->graphsValid = true;
  return NBX_OK;
}

// The two io step graphs writing to out (pinned host memory).
int capture_io_graphs(nbx_handle *h, nbx_body *out) {
  for (auto &g : h->ioGraph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  h->ioOut = nullptr;
  if (!h->ioFork) {
    NBX_CUDA(h, cudaEventCreateWithFlags(&h->ioFork, cudaEventDisableTiming));
    // earlier ranges on higher-priority streams: their blocks are
    // dispatched first, so the ranges finish (and copy) in order
    int least = 0, greatest = 0;
    NBX_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    for (int c = 0; c < nbx_handle::kIoChunks; ++c) {
      const int prio = std::min(greatest + c, least);
      NBX_CUDA(h, cudaStreamCreateWithPriority(&h->ioStream[c], cudaStreamNonBlocking, prio));
      NBX_CUDA(h, cudaEventCreateWithFlags(&h->ioDone[c], cudaEventDisableTiming));
    }
  }
  h->ioOut = out;
  for (int p = 0; p < 2; ++p) {
    const int saved = h->cur;
    h->cur = p;
    const DevState S = h->state();
    h->cur = saved;
    cudaGraph_t g = nullptr;
    NBX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->ioCapture = true;
    enqueue_step(h, h->stream, S);
    h->ioCapture = false;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) {
      h->ioOut = nullptr;
      return cuda_fail(h, e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&h->ioGraph[p], g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      h->ioOut = nullptr;
      return cuda_fail(h, e, "cudaGraphInstantiate");
    }
  }
  return NBX_OK;
}

int check_status(nbx_handle *h) {
  uint32_t bits = 0;
  NBX_CUDA(h, cudaMemcpyAsync(&bits, h->base.status, 4, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!bits) return NBX_OK;
  NBX_CUDA(h, cudaMemsetAsync(h->base.status, 0, 4, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  if (bits & kStatusSpinLimit) return fail(h, NBX_ERR_TIMEOUT, "a bounded device wait gave up");
  if (bits & (kStatusTreeCapacity | kStatusPairCapacity | kStatusLargeCapacity))
    return fail(h, NBX_ERR_CAPACITY, bits & kStatusTreeCapacity
                                         ? "tree node capacity exceeded"
                                         : "collision pair capacity exceeded");
  if (bits & kStatusNonFinite) return fail(h, NBX_ERR_NONFINITE, "non-finite body position");
  return fail(h, NBX_ERR_STATE, "device status bits set");
}

bool valid_params(const nbx_params *p) {
  return p && p->dt == p->dt && p->theta >= 0.0f && p->epsilon >= 0.0f &&
         p->leaf_capacity >= 1 && p->leaf_capacity <= 64 && p->use_mlp >= 0 &&
         p->use_mlp <= 2 && (p->force_law == 0 || p->force_law == 1) &&
         !(p->force_law == 1 && p->use_mlp != 0) &&
         (p->force_block == 0 || p->force_block == 128 || p->force_block == 256 ||
          p->force_block == 512) &&
         (p->leaf_pairs == 0 || p->leaf_pairs == 1);
}

} // namespace

// Reallocates p for count elements (contents are not kept).
template <typename T> static cudaError_t grow(T *&p, size_t count) {
  if (p) cudaFree(p);
  p = nullptr;
  return cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
}

extern "C" {

const char *nbx_version(void) { return "nbx 0.1 (sm_100a)"; }

int nbx_params_default(nbx_params *p) {
  if (!p) return NBX_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->dt = 0.05f;
  p->theta = 1.0f;
  p->epsilon = 1.0f;
  p->leaf_capacity = 16;
  p->collisions = 1;
  p->exact_math = 0;
  p->use_mlp = 0;
  p->node_factor = 8.0f;
  p->pair_factor = 32.0f;
  p->force_blocks = 0;
  p->device = -1;
  p->mlp_band = 0.5f;
  p->force_law = 0;
  p->force_block = 0;
  p->leaf_pairs = 1;
  return NBX_OK;
}

static int frames_flush(nbx_handle *h);
static void frames_destroy(nbx_handle *h);
static void render_free(nbx_handle *h);

int nbx_create(const nbx_params *p, uint32_t num, const uint32_t *sizes,
               nbx_handle **out) {
  if (!out || num == 0 || !sizes || num > 65535) return NBX_ERR_ARG;
  *out = nullptr;
  nbx_params P;
  nbx_params_default(&P);
  if (p) P = *p;
  if (!valid_params(&P)) return NBX_ERR_ARG;
  uint64_t total = 0;
  for (uint32_t s = 0; s < num; ++s) total += sizes[s];
  if (total >= (1ull << 30)) return NBX_ERR_ARG;
  nbx_handle *h = new (std::nothrow) nbx_handle();
  if (!h) return NBX_ERR_NOMEM;
  h->params = P;
  h->n = (uint32_t)total;
  h->nseg = num;
  uint32_t run = 0;
  for (uint32_t s = 0; s < num; ++s) {
    h->segStart.push_back(run);
    h->segCount.push_back(sizes[s]);
    run += sizes[s];
  }
  cudaError_t e = cudaSuccess;
  if (P.device >= 0) e = cudaSetDevice(P.device);
  if (e == cudaSuccess) e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->side.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->side.join, cudaEventDisableTiming);
  int rc = e == cudaSuccess ? allocate(h) : cuda_fail(h, e, "stream");
  if (rc != NBX_OK) {
    std::fprintf(stderr, "nbx_create: %s\n", h->lastError.c_str());
    nbx_destroy(h);
    return rc;
  }
  sync_params(h);
  *out = h;
  return NBX_OK;
}

int nbx_destroy(nbx_handle *h) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  frames_destroy(h);
  render_free(h);
  destroy_graphs(h);
  for (cudaEvent_t ev : h->forceEv) cudaEventDestroy(ev);
  for (cudaEvent_t ev : h->forceMark)
    if (ev) cudaEventDestroy(ev);
  if (h->ioFork) cudaEventDestroy(h->ioFork);
  for (int c = 0; c < nbx_handle::kIoChunks; ++c) {
    if (h->ioDone[c]) cudaEventDestroy(h->ioDone[c]);
    if (h->ioStream[c]) cudaStreamDestroy(h->ioStream[c]);
  }
  for (void *v : h->allocs) cudaFree(v);
  for (void *v : h->scratch) cudaFree(v);
  if (h->hPinned) cudaFreeHost(h->hPinned);
  if (h->hWord) cudaFreeHost(h->hWord);
  if (h->dPartial) cudaFree(h->dPartial);
  if (h->dTargets) cudaFree(h->dTargets);
  if (h->side.fork) cudaEventDestroy(h->side.fork);
  if (h->side.join) cudaEventDestroy(h->side.join);
  if (h->side.stream) cudaStreamDestroy(h->side.stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return NBX_OK;
}

int nbx_set_params(nbx_handle *h, const nbx_params *p) {
  if (!h || !valid_params(p)) return NBX_ERR_ARG;
  const bool sizes = p->node_factor != h->params.node_factor ||
                     p->pair_factor != h->params.pair_factor;
  if (sizes) return fail(h, NBX_ERR_ARG, "capacity factors are fixed at nbx_create");
  h->params = *p;
  sync_params(h);
  destroy_graphs(h);
  return NBX_OK;
}

int nbx_get_params(const nbx_handle *h, nbx_params *p) {
  if (!h || !p) return NBX_ERR_ARG;
  *p = h->params;
  return NBX_OK;
}

int nbx_upload_bodies(nbx_handle *h, const nbx_body *bodies, size_t n) {
  if (!h || (!bodies && n) || n != h->n) return h ? fail(h, NBX_ERR_ARG, "body count mismatch") : NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (n == 0) {
    h->uploaded = true;
    return NBX_OK;
  }
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, bodies) == cudaSuccess &&
                      attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  const void *src = bodies;
  if (!pinned) {
    std::memcpy(h->hPinned, bodies, n * sizeof(nbx_body));
    src = h->hPinned;
  }
  NBX_CUDA(h, cudaMemcpyAsync(h->dAoS, src, n * sizeof(nbx_body),
                              cudaMemcpyHostToDevice, h->stream));
  const DevState S = h->state();
  NBX_CUDA(h, cudaMemsetAsync(S.counters + 12, 0, sizeof(uint32_t), h->stream));
  k_unpack<<<std::min<uint32_t>((h->n + 255) / 256, 4096), 256, 0, h->stream>>>(
      h->dAoS, h->n, S.pv, S.acc, S.mr, S.id, S.counters + 12);
  NBX_CUDA(h, cudaGetLastError());
  NBX_CUDA(h, cudaMemcpyAsync(h->hWord, S.counters + 12, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, h->stream));
  // While the records cross PCIe: the collision cell per instance, 2 x
  // 1.01 x the median radius (CudaCollision.cu:201-215).  The cell only
  // sets how the broadphase partitions space: the candidate set (every
  // overlapping box pair) does not depend on it.  The median is over an
  // evenly strided sample of at most 4096 bodies per instance (the
  // reference takes all radii); deterministic for a given input.
  std::vector<float> cells(3 * (size_t)h->nseg); // {cell, invCell, smallW}
  std::vector<float> radii;
  for (uint32_t s = 0; s < h->nseg; ++s) {
    const uint32_t s0 = h->segStart[s], cnt = h->segCount[s];
    const uint32_t stride = cnt > 4096 ? cnt / 4096 : 1;
    radii.clear();
    for (uint32_t i = 0; i < cnt; i += stride) radii.push_back(bodies[s0 + i].radius);
    float cell = 1.0f;
    if (!radii.empty()) {
      const size_t mid = radii.size() / 2;
      std::nth_element(radii.begin(), radii.begin() + mid, radii.end());
      cell = 2.0f * radii[mid] * 1.01f;
    }
    if (!(cell > 0.0f) || !std::isfinite(cell)) cell = 1.0f;
    cells[3 * s] = cell;
    cells[3 * s + 1] = 1.0f / cell;
    cells[3 * s + 2] = cell * 0.999f;
  }
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  const uint32_t massBits = *h->hWord;
  // the force pass leaves out its FLT_MAX clamp when it cannot act; a
  // change of that choice needs new step graphs
  uint32_t coordLimitBits = 0;
  {
    const bool before = forces_unclamped(h);
    float mm = INFINITY; // a negative mass (or -0): keep the clamp
    if (!(massBits & 0x80000000u)) std::memcpy(&mm, &massBits, sizeof(mm));
    h->maxMass = mm;
    if (forces_unclamped(h) != before) destroy_graphs(h);
    // every node sum of x * m stays below 1e36 and every distance below
    // 1.2e19 (its square finite) while all |x|, |y| < this limit
    float lim = 4e18f;
    if (mm > 0.0f && std::isfinite(mm))
      lim = std::fmin(lim, 1e36f / (static_cast<float>(h->n) * mm));
    std::memcpy(&coordLimitBits, &lim, sizeof(lim));
  }
  // the three cell fields of every SegDev and the limit, ordered before
  // the next step on the stream; the pinned words are free again once the
  // synchronisation above has passed (the last upload's copies came before)
  h->hWord[1] = coordLimitBits;
  std::memcpy(h->hWord + 4, cells.data(), cells.size() * sizeof(float));
  static_assert(offsetof(SegDev, invCell) == offsetof(SegDev, cell) + 4 &&
                    offsetof(SegDev, smallW) == offsetof(SegDev, cell) + 8,
                "SegDev cell fields are contiguous");
  NBX_CUDA(h, cudaMemcpy2DAsync(reinterpret_cast<char *>(S.seg) + offsetof(SegDev, cell),
                                sizeof(SegDev), h->hWord + 4, 3 * sizeof(float),
                                3 * sizeof(float), h->nseg, cudaMemcpyHostToDevice,
                                h->stream));
  NBX_CUDA(h, cudaMemcpyAsync(S.counters + kCtrCoordLimit, h->hWord + 1,
                              sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
  h->idsChecked = false;
  h->uploaded = true;
  h->treeValid = false;
  h->forceInput = false;
  h->collideValid = false;
  return NBX_OK;
}

// ids must be a permutation of 0..size-1 in every instance for id-order
// output; checked on the device once per upload (steps only permute bodies).
static int ensure_id_permutation(nbx_handle *h) {
  if (!h->idsChecked) {
    const DevState S0 = h->state();
    uint32_t *seen = S0.splitCount, *bad = S0.counters + 8;
    NBX_CUDA(h, cudaMemsetAsync(seen, 0, 4ull * h->n, h->stream));
    NBX_CUDA(h, cudaMemsetAsync(bad, 0, 4, h->stream));
    k_check_ids<<<std::min<uint32_t>((h->n + 255) / 256, 4096), 256, 0, h->stream>>>(
        S0.id, S0.segOf, S0.seg, h->n, seen, bad);
    uint32_t b = 0;
    NBX_CUDA(h, cudaMemcpyAsync(&b, bad, 4, cudaMemcpyDeviceToHost, h->stream));
    NBX_CUDA(h, cudaStreamSynchronize(h->stream));
    h->idsPermutation = b == 0;
    h->idsChecked = true;
  }
  if (!h->idsPermutation)
    return fail(h, NBX_ERR_ARG, "ids are not a permutation of 0..size-1 per instance");
  return NBX_OK;
}

int nbx_download_bodies(nbx_handle *h, nbx_body *bodies, size_t n, int idOrder) {
  if (!h || (!bodies && n) || n != h->n) return h ? fail(h, NBX_ERR_ARG, "body count mismatch") : NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (idOrder) {
    const int rc = ensure_id_permutation(h);
    if (rc != NBX_OK) return rc;
  }
  if (n == 0) return NBX_OK;
  const DevState S = h->state();
  k_pack<<<std::min<uint32_t>((h->n + 255) / 256, 4096), 256, 0, h->stream>>>(
      S.pv, S.acc, S.mr, S.id, S.segOf, S.seg, 0u, h->n, idOrder, h->dAoS);
  NBX_CUDA(h, cudaGetLastError());
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, bodies) == cudaSuccess &&
                      attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  void *dst = pinned ? (void *)bodies : (void *)h->hPinned;
  NBX_CUDA(h, cudaMemcpyAsync(dst, h->dAoS, n * sizeof(nbx_body),
                              cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!pinned) std::memcpy(bodies, h->hPinned, n * sizeof(nbx_body));
  return check_status(h);
}

int nbx_step(nbx_handle *h, uint32_t steps) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  if (h->n == 0 || steps == 0) return NBX_OK;
  if (h->params.use_mlp == 1 && !h->mlpLoaded)
    return fail(h, NBX_ERR_STATE, "use_mlp = 1 without MLP parameters");
  if (!h->graphsValid) {
    int rc = capture_graphs(h);
    if (rc != NBX_OK) return rc;
  }
  for (uint32_t k = 0; k < steps; ++k) {
    NBX_CUDA(h, cudaGraphLaunch(h->graph[h->cur], h->stream));
    h->cur ^= 1;
  }
  after_step(h);
  return NBX_OK;
}

int nbx_step_io(nbx_handle *h, const nbx_body *in, nbx_body *out, size_t n) {
  if (!h || (!in && n) || (!out && n) || n != h->n)
    return h ? fail(h, NBX_ERR_ARG, "body count mismatch") : NBX_ERR_ARG;
  int rc = nbx_upload_bodies(h, in, n);
  if (rc != NBX_OK || n == 0) return rc;
  if (h->params.use_mlp == 1 && !h->mlpLoaded)
    return fail(h, NBX_ERR_STATE, "use_mlp = 1 without MLP parameters");
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, out) == cudaSuccess &&
                      attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (!pinned || h->params.force_law != 0) {
    // pageable memory cannot be a graph's copy target: step, then copy
    rc = nbx_step(h, 1);
    if (rc != NBX_OK) return rc;
    return nbx_download_bodies(h, out, n, 0);
  }
  if (!h->graphsValid) {
    rc = capture_graphs(h);
    if (rc != NBX_OK) return rc;
  }
  if (h->ioOut != out || !h->ioGraph[h->cur]) {
    rc = capture_io_graphs(h, out);
    if (rc != NBX_OK) return rc;
  }
  NBX_CUDA(h, cudaGraphLaunch(h->ioGraph[h->cur], h->stream));
  h->cur ^= 1;
  after_step(h);
  return check_status(h);
}

int nbx_step_timed(nbx_handle *h, uint32_t steps) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  h->timedSteps = 0;
  if (h->n == 0 || steps == 0) return NBX_OK;
  if (h->params.use_mlp == 1 && !h->mlpLoaded)
    return fail(h, NBX_ERR_STATE, "use_mlp = 1 without MLP parameters");
  if (!h->timedValid) {
    int rc = capture_timed_graphs(h);
    if (rc != NBX_OK) return rc;
  }
  while (h->forceEv.size() < 2 * (size_t)steps) {
    cudaEvent_t ev = nullptr;
    NBX_CUDA(h, cudaEventCreate(&ev));
    h->forceEv.push_back(ev);
  }
  for (uint32_t k = 0; k < steps; ++k) {
    const int p = h->cur;
    // affects this and later launches only; earlier launches keep theirs
    NBX_CUDA(h, cudaGraphExecEventRecordNodeSetEvent(h->graphT[p], h->forceEvNode[p][0],
                                                     h->forceEv[2 * k]));
    NBX_CUDA(h, cudaGraphExecEventRecordNodeSetEvent(h->graphT[p], h->forceEvNode[p][1],
                                                     h->forceEv[2 * k + 1]));
    NBX_CUDA(h, cudaGraphLaunch(h->graphT[p], h->stream));
    h->cur ^= 1;
  }
  h->timedSteps = steps;
  after_step(h);
  return NBX_OK;
}

int nbx_force_times(nbx_handle *h, float *ms, uint32_t count) {
  if (!h || (!ms && count)) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (count > h->timedSteps)
    return fail(h, NBX_ERR_ARG, "more force times requested than steps timed");
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  for (uint32_t k = 0; k < count; ++k)
    NBX_CUDA(h, cudaEventElapsedTime(&ms[k], h->forceEv[2 * k], h->forceEv[2 * k + 1]));
  return check_status(h);
}

// Waits for every recorded frame to be written; returns the first error.
static int frames_flush(nbx_handle *h) {
  FrameWriter *w = h->frames;
  if (!w) return NBX_OK;
  std::unique_lock<std::mutex> lk(w->mu);
  w->cv.wait(lk, [&] { return w->queue.empty(); });
  const int rc = w->err;
  w->err = NBX_OK;
  return rc;
}

static void frames_destroy(nbx_handle *h) {
  FrameWriter *w = h->frames;
  if (!w) return;
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->stop = true;
  }
  w->cv.notify_all();
  if (w->th.joinable()) w->th.join(); // drains the queue first
  for (int k = 0; k < 2; ++k) {
    if (w->dFrame[k]) cudaFree(w->dFrame[k]);
    if (w->hSlot[k]) cudaFreeHost(w->hSlot[k]);
    if (w->scattered[k]) cudaEventDestroy(w->scattered[k]);
    if (w->copied[k]) cudaEventDestroy(w->copied[k]);
  }
  if (w->copy) cudaStreamDestroy(w->copy);
  delete w;
  h->frames = nullptr;
}

int nbx_nbs2_record(nbx_handle *h, nbx_nbs2 *f) {
  if (!h || !f) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->nseg != 1) return fail(h, NBX_ERR_ARG, "NBS2 frames hold one simulation");
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  int rc = ensure_id_permutation(h);
  if (rc != NBX_OK) return rc;
  if (!h->frames) {
    FrameWriter *w = new (std::nothrow) FrameWriter();
    if (!w) return NBX_ERR_NOMEM;
    h->frames = w;
    w->device = h->device;
    w->n = h->n;
    NBX_CUDA(h, cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      NBX_CUDA(h, cudaMalloc(&w->dFrame[k], std::max<size_t>(w->n, 1) * sizeof(float4)));
      NBX_CUDA(h, cudaMallocHost(&w->hSlot[k], std::max<size_t>(w->n, 1) * sizeof(float4)));
      NBX_CUDA(h, cudaEventCreateWithFlags(&w->scattered[k], cudaEventDisableTiming));
      NBX_CUDA(h, cudaEventCreateWithFlags(&w->copied[k], cudaEventDisableTiming));
    }
    w->th = std::thread([w] { w->run(); });
  }
  FrameWriter *w = h->frames;
  const int sl = w->next;
  {
    // the slot's previous frame must be written before it is reused
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [&] { return !w->busy[sl]; });
    w->busy[sl] = true;
  }
  const DevState S = h->state();
  if (w->n) {
    k_frame_scatter<<<std::min<uint32_t>((w->n + 255) / 256, 4096), 256, 0, h->stream>>>(
        S.pv, S.id, w->n, w->dFrame[sl]);
    NBX_CUDA(h, cudaGetLastError());
  }
  NBX_CUDA(h, cudaEventRecord(w->scattered[sl], h->stream));
  NBX_CUDA(h, cudaStreamWaitEvent(w->copy, w->scattered[sl], 0));
  NBX_CUDA(h, cudaMemcpyAsync(w->hSlot[sl], w->dFrame[sl], (size_t)w->n * sizeof(float4),
                              cudaMemcpyDeviceToHost, w->copy));
  NBX_CUDA(h, cudaEventRecord(w->copied[sl], w->copy));
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->queue.emplace_back(sl, f);
  }
  w->cv.notify_all();
  w->next ^= 1;
  return NBX_OK;
}

int nbx_nbs2_flush(nbx_handle *h) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  const int rc = frames_flush(h);
  return rc == NBX_OK ? NBX_OK : fail(h, rc, "writing a recorded NBS2 frame failed");
}

static void render_free(nbx_handle *h) {
  auto &r = h->rs;
  void *ptrs[] = {r.v0, r.v1, r.image, r.count, r.off, r.first, r.last, r.partial,
                  r.total, r.stats, r.sort.keys[0], r.sort.keys[1], r.sort.vals[0],
                  r.sort.vals[1], r.sort.hist, r.sort.status, r.sort.tileCounter};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  r = {};
}

// Vertices and statistics of the current state for image P; on return the
// stats (3 floats) are on the device and the entry total is known.
static int render_prepare(nbx_handle *h, const RenderParams &P, unsigned long long *entries) {
  auto &r = h->rs;
  const uint32_t n = h->n;
  if (r.bodies < n || !r.v0) {
    NBX_CUDA(h, grow(r.v0, n));
    NBX_CUDA(h, grow(r.v1, n));
    NBX_CUDA(h, grow(r.count, n));
    NBX_CUDA(h, grow(r.off, n));
    NBX_CUDA(h, grow(r.partial, render_vertex_blocks(n)));
    if (!r.total) NBX_CUDA(h, cudaMalloc(&r.total, 2 * sizeof(unsigned long long)));
    if (!r.stats) NBX_CUDA(h, cudaMalloc(&r.stats, 4 * sizeof(float)));
    r.bodies = n;
  }
  const DevState S = h->state();
  render_vertices(h->stream, S.pv, S.mr, n, P, r.v0, r.v1, r.count, r.partial, r.total,
                  r.stats);
  NBX_CUDA(h, cudaGetLastError());
  NBX_CUDA(h, cudaMemcpyAsync(entries, r.total, sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

static int render_params(const nbx_camera *cam, const nbx_draw *d, uint32_t width,
                         uint32_t height, RenderParams &P) {
  if (!cam || !d || width == 0 || height == 0 || width > 16384 || height > 16384 ||
      (d->mode != 0 && d->mode != 1) || !(d->min_point_px > 0.0f) || !(d->speed_max > 0.0f))
    return NBX_ERR_ARG;
  P.camX = cam->center_x;
  P.camY = cam->center_y;
  P.scale = cam->scale;
  P.halfW = (float)width * 0.5f;
  P.halfH = (float)height * 0.5f;
  P.width = width;
  P.height = height;
  P.tilesX = (width + 15) / 16;
  P.tilesY = (height + 15) / 16;
  P.mode = d->mode;
  P.pointScale = d->point_scale;
  P.minPoint = d->min_point_px;
  P.brightness = d->brightness;
  P.speedMax = d->speed_max;
  return NBX_OK;
}

int nbx_draw_default(nbx_draw *d) {
  if (!d) return NBX_ERR_ARG;
  d->mode = 1; // glow
  d->point_scale = 1.0f;
  d->min_point_px = 1.5f;
  d->brightness = 0.6f;
  d->speed_max = 60.0f;
  return NBX_OK;
}

int nbx_body_stats(nbx_handle *h, float *stats) {
  if (!h || !stats) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  if (h->n == 0) {
    stats[0] = stats[1] = 0.0f;
    stats[2] = 1.0f;
    return NBX_OK;
  }
  const nbx_camera cam = {0.0f, 0.0f, 1.0f};
  nbx_draw d;
  nbx_draw_default(&d);
  RenderParams P{};
  render_params(&cam, &d, 1, 1, P);
  unsigned long long entries = 0;
  int rc = render_prepare(h, P, &entries);
  if (rc != NBX_OK) return rc;
  NBX_CUDA(h, cudaMemcpy(stats, h->rs.stats, 3 * sizeof(float), cudaMemcpyDeviceToHost));
  return NBX_OK;
}

int nbx_render(nbx_handle *h, const nbx_camera *cam, const nbx_draw *d, uint32_t width,
               uint32_t height, float *rgba, float *stats) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  RenderParams P{};
  if (render_params(cam, d, width, height, P) != NBX_OK)
    return fail(h, NBX_ERR_ARG, "bad camera, draw settings or image size");
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  auto &r = h->rs;
  const size_t pixels = (size_t)width * height;
  const uint32_t tiles = P.tilesX * P.tilesY;
  if (r.pixels < pixels || !r.image) {
    NBX_CUDA(h, grow(r.image, pixels));
    r.pixels = pixels;
  }
  if (r.tiles < tiles || !r.first) {
    NBX_CUDA(h, grow(r.first, tiles));
    NBX_CUDA(h, grow(r.last, tiles));
    r.tiles = tiles;
  }
  unsigned long long entries = 0;
  if (h->n > 0) {
    int rc = render_prepare(h, P, &entries);
    if (rc != NBX_OK) return rc;
  }
  if (entries > (1ull << 30))
    return fail(h, NBX_ERR_CAPACITY,
                "splats cover more than 2^30 (tile, body) pairs: zoom out or shrink the image");
  const uint32_t m = (uint32_t)entries;
  if (m > r.entries || !r.sort.keys[0]) {
    SortScratch &so = r.sort;
    const uint32_t cap = std::max<uint32_t>(m, 1024);
    NBX_CUDA(h, grow(so.keys[0], cap));
    NBX_CUDA(h, grow(so.keys[1], cap));
    NBX_CUDA(h, grow(so.vals[0], cap));
    NBX_CUDA(h, grow(so.vals[1], cap));
    if (!so.hist) NBX_CUDA(h, cudaMalloc(&so.hist, 8 * 256 * sizeof(uint32_t)));
    if (!so.tileCounter) NBX_CUDA(h, cudaMalloc(&so.tileCounter, 8 * sizeof(uint32_t)));
    so.capacity = cap;
    so.maxTiles = (uint32_t)sort_tiles(cap);
    NBX_CUDA(h, grow(so.status, 8 * ((size_t)so.maxTiles * 256 + 256)));
    r.entries = cap;
  }
  int bits = 8;
  while (bits < 32 && (1ull << bits) < tiles) bits += 8;
  cudaStream_t s = h->stream;
  int buf = 0;
  if (m > 0) {
    exclusive_scan_u32(s, r.count, r.off, h->n, nullptr, nullptr, h->scan, h->base.status);
    render_emit(s, r.v0, r.off, h->n, P, r.sort.keys[0], r.sort.vals[0]);
    NBX_CUDA(h, cudaMemcpyAsync(r.total + 1, &m, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    buf = radix_sort_u64(s, r.sort, m, reinterpret_cast<const uint32_t *>(r.total + 1), 0,
                         bits, false, false, h->base.status);
  }
  render_composite(s, r.v0, r.v1, r.sort.keys[buf], r.sort.vals[buf],
                   reinterpret_cast<const uint32_t *>(r.total + 1), m, r.first, r.last, P,
                   r.image);
  NBX_CUDA(h, cudaGetLastError());
  if (rgba)
    NBX_CUDA(h, cudaMemcpyAsync(rgba, r.image, pixels * sizeof(float4), cudaMemcpyDeviceToHost, s));
  float st[3] = {0.0f, 0.0f, 1.0f};
  if (h->n > 0)
    NBX_CUDA(h, cudaMemcpyAsync(st, r.stats, sizeof(st), cudaMemcpyDeviceToHost, s));
  NBX_CUDA(h, cudaStreamSynchronize(s));
  if (stats) std::memcpy(stats, st, sizeof(st));
  return check_status(h);
}

int nbx_set_attractor(nbx_handle *h, int active, float x, float y, float mass,
                      float softening) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  const float v[8] = {x, y, mass, softening, active ? 1.0f : 0.0f, 0.0f, 0.0f, 0.0f};
  std::memcpy(h->attrHost, v, sizeof(v));
  // stream-ordered: steps enqueued before see the old attractor, later
  // ones the new; the captured graphs read it from device memory
  NBX_CUDA(h, cudaMemcpyAsync(h->base.attr, h->attrHost, sizeof(v),
                              cudaMemcpyHostToDevice, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

int nbx_reset(nbx_handle *h, const nbx_body *bodies, size_t n) {
  if (!h || (!bodies && n) || n >= (1ull << 30)) return NBX_ERR_ARG;
  if (h->nseg != 1)
    return fail(h, NBX_ERR_ARG, "nbx_reset replaces the bodies of a single-instance handle");
  cudaSetDevice(h->device);
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  // pending frames are written first; the writer is rebuilt for the new size
  const int frc = frames_flush(h);
  frames_destroy(h);
  render_free(h);
  if (frc != NBX_OK) return fail(h, frc, "writing a recorded NBS2 frame failed");
  // keep the network parameters across the reallocation (optimizer
  // moments start again)
  std::vector<float> mlp;
  if (h->mlpLoaded) {
    mlp.resize(kMlpParams);
    NBX_CUDA(h, cudaMemcpy(mlp.data(), h->mlpP, kMlpParams * sizeof(float),
                           cudaMemcpyDeviceToHost));
  }
  destroy_graphs(h);
  for (void *v : h->allocs) cudaFree(v);
  h->allocs.clear();
  for (void *v : h->scratch) cudaFree(v);
  h->scratch.clear();
  if (h->hPinned) cudaFreeHost(h->hPinned);
  if (h->dPartial) cudaFree(h->dPartial);
  if (h->dTargets) cudaFree(h->dTargets);
  h->hPinned = nullptr;
  h->dPartial = nullptr;
  h->dTargets = nullptr;
  h->dPartialTargets = 0;
  h->base = DevState{};
  h->scan = ScanScratch{};
  h->sort = SortScratch{};
  h->cur = 0;
  h->n = (uint32_t)n;
  h->segStart.assign(1, 0u);
  h->segCount.assign(1, (uint32_t)n);
  h->uploaded = h->treeValid = h->forceInput = h->collideValid = false;
  h->idsChecked = h->idsPermutation = false;
  h->mlpLoaded = false;
  h->timedSteps = 0;
  int rc = allocate(h);
  if (rc != NBX_OK) return rc;
  sync_params(h);
  if (!mlp.empty() && (rc = nbx_mlp_set_params(h, mlp.data(), kMlpParams)) != NBX_OK)
    return rc;
  return nbx_upload_bodies(h, bodies, n);
}

int nbx_debug_expire_wait(nbx_handle *h) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  uint32_t *flag = h->base.counters + 13; // never set
  NBX_CUDA(h, cudaMemsetAsync(flag, 0, sizeof(uint32_t), h->stream));
  k_expire_wait<<<1, 32, 0, h->stream>>>(flag, h->base.status);
  NBX_CUDA(h, cudaGetLastError());
  return NBX_OK;
}

int nbx_sync(nbx_handle *h) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int nbx_phase(nbx_handle *h, int phase) {
  if (!h) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  if (h->n == 0) return NBX_OK;
  cudaStream_t s = h->stream;
  DevState S = h->state();
  switch (phase) {
  case NBX_PHASE_ITERATE:
    launch_integrate(s, S, true, false);
    break;
  case NBX_PHASE_COLLIDE:
    launch_step_zero(s, S, h->scan, h->sort, true);
    launch_integrate(s, S, false, true);
    launch_collide(s, S, h->scan, h->sort, &h->side);
    h->collideValid = true;
    break;
  case NBX_PHASE_BUILD:
    if (h->params.force_law == 1) { // no tree: the identity gather
      S = launch_naive_gather(s, S);
      h->cur ^= 1;
      h->treeValid = false;
      h->forceInput = true;
      break;
    }
    launch_step_zero(s, S, h->scan, h->sort, false);
    launch_build(s, S, h->scan, h->sort, true);
    h->momentsValid = true;
    h->cur ^= 1;
    h->treeValid = true;
    h->bfsValid = false;
    h->forceInput = true;
    break;
  case NBX_PHASE_FORCES:
    if (h->params.force_law == 1) {
      if (!h->forceInput) return fail(h, NBX_ERR_STATE, "no force input gathered");
      launch_naive_forces(s, S, h->params.exact_math != 0);
      break;
    }
    if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
    launch_forces(s, S, h->params.exact_math != 0, h->params.force_blocks,
                  h->mlpLoaded ? h->mlpW : nullptr, h->params.mlp_band,
                  h->params.use_mlp, forces_unclamped(h), h->params.force_block,
                h->params.leaf_pairs != 0);
    break;
  case NBX_PHASE_ATTRACT:
    if (h->params.force_law == 1) {
      S = launch_naive_gather(s, S);
      h->cur ^= 1;
      h->treeValid = false;
      h->forceInput = true;
      launch_naive_forces(s, S, h->params.exact_math != 0);
      break;
    }
    launch_step_zero(s, S, h->scan, h->sort, false);
    launch_build(s, S, h->scan, h->sort, true);
    h->momentsValid = true;
    h->cur ^= 1;
    h->treeValid = true;
    h->bfsValid = false;
    h->forceInput = true;
    launch_forces(s, S, h->params.exact_math != 0, h->params.force_blocks,
                  h->mlpLoaded ? h->mlpW : nullptr, h->params.mlp_band,
                  h->params.use_mlp, forces_unclamped(h), h->params.force_block,
                h->params.leaf_pairs != 0);
    break;
  case NBX_PHASE_STEP:
    enqueue_step(h, s, S);
    h->cur ^= 1;
    after_step(h);
    break;
  default:
    return fail(h, NBX_ERR_ARG, "unknown phase");
  }
  NBX_CUDA(h, cudaGetLastError());
  return nbx_sync(h);
}

int nbx_get_morton(nbx_handle *h, uint32_t inst, uint64_t *codes, uint32_t *perm,
                   size_t n) {
  if (!h || inst >= h->nseg || n != h->segCount[inst]) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
  const uint32_t s0 = h->segStart[inst];
  if (codes)
    NBX_CUDA(h, cudaMemcpyAsync(codes, h->base.codes + s0, n * 8, cudaMemcpyDeviceToHost, h->stream));
  std::vector<uint32_t> p(n);
  NBX_CUDA(h, cudaMemcpyAsync(p.data(), h->base.perm + s0, n * 4, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  if (perm)
    for (size_t i = 0; i < n; ++i) perm[i] = p[i] - s0;
  return NBX_OK;
}

static int read_seg(nbx_handle *h, uint32_t inst, SegDev &g) {
  NBX_CUDA(h, cudaMemcpyAsync(&g, h->base.seg + inst, sizeof(SegDev),
                              cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

} // extern "C"

// The breadth-first arrays of the last tree, built from its sorted codes
// the first time they are asked for (the step path builds only the
// traversal layout).
static int ensure_bfs_tree(nbx_handle *h) {
  if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
  if (h->bfsValid) return NBX_OK;
  launch_bfs_tree(h->stream, h->state(), h->scan, h->sort);
  NBX_CUDA(h, cudaGetLastError());
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  int rc = check_status(h);
  if (rc) return rc;
  h->bfsValid = true;
  return NBX_OK;
}

extern "C" {

int nbx_tree_size(nbx_handle *h, uint32_t inst, uint32_t *nodes, uint32_t *levels) {
  if (!h || inst >= h->nseg) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  int rc0 = ensure_bfs_tree(h);
  if (rc0) return rc0;
  SegDev g;
  int rc = read_seg(h, inst, g);
  if (rc) return rc;
  if (nodes) *nodes = g.nodeCount;
  if (levels) *levels = g.levelCount;
  return NBX_OK;
}

int nbx_get_tree(nbx_handle *h, uint32_t inst, float *comX, float *comY, float *mass,
                 float *cx, float *cy, float *size, int32_t *children, int32_t *next,
                 int32_t *start, int32_t *end, size_t capacity) {
  if (!h || inst >= h->nseg) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  int rc0 = ensure_bfs_tree(h);
  if (rc0) return rc0;
  SegDev g;
  int rc = read_seg(h, inst, g);
  if (rc) return rc;
  if (capacity < g.nodeCount) return fail(h, NBX_ERR_ARG, "capacity below node count");
  const size_t c = g.nodeCount, b = g.nodeBase;
  const DevState &S = h->base;
  struct {
    void *dst;
    const void *src;
  } arrays[] = {{comX, S.comX}, {comY, S.comY}, {mass, S.mass}, {cx, S.centerX},
                {cy, S.centerY}, {size, S.size}, {children, S.children},
                {next, S.next}, {start, S.start}, {end, S.end}};
  for (auto &a : arrays) {
    if (!a.dst || !c) continue;
    NBX_CUDA(h, cudaMemcpyAsync(a.dst, (const char *)a.src + b * 4, c * 4,
                                cudaMemcpyDeviceToHost, h->stream));
  }
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

int nbx_get_pairs(nbx_handle *h, int32_t *later, int32_t *earlier, int64_t cap,
                  int64_t *count) {
  if (!h || !count) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->collideValid) return fail(h, NBX_ERR_STATE, "no collide run");
  const DevState &S = h->base;
  const uint32_t n = h->n;
  uint32_t cnt[2];
  NBX_CUDA(h, cudaMemcpyAsync(cnt, S.counters, 8, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  const uint32_t total = cnt[0], units = cnt[1];
  if (total > S.pairCapacity) return fail(h, NBX_ERR_CAPACITY, "pair capacity exceeded");
  std::vector<uint32_t> pstart(n), plist(total), nl(n), order(units);
  NBX_CUDA(h, cudaMemcpyAsync(pstart.data(), S.pstart, 4ull * n, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaMemcpyAsync(plist.data(), S.plist, 4ull * total, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaMemcpyAsync(nl.data(), S.nLater, 4ull * n, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaMemcpyAsync(order.data(), S.unitOrder, 4ull * units, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  int64_t k = 0;
  for (uint32_t u = 0; u < units; ++u) {
    const uint32_t L = order[u];
    for (uint32_t j = 0; j < nl[L]; ++j, ++k) {
      if (k < cap) {
        later[k] = (int32_t)L;
        earlier[k] = (int32_t)plist[pstart[L] + j];
      }
    }
  }
  *count = k;
  return NBX_OK;
}

int nbx_collision_stats(nbx_handle *h, int64_t *pairs, uint32_t *depth) {
  if (!h || !pairs || !depth) return NBX_ERR_ARG;
  int64_t total = 0;
  int rc = nbx_get_pairs(h, nullptr, nullptr, 0, &total);
  if (rc) return rc;
  std::vector<int32_t> later((size_t)total), earlier((size_t)total);
  rc = nbx_get_pairs(h, later.data(), earlier.data(), total, &total);
  if (rc) return rc;
  // a pair waits for the last earlier pair of either body (the sequential
  // loop's order, Collision.cpp:341-348): longest chain of such waits
  std::vector<uint32_t> last(h->n, 0u);
  uint32_t deepest = 0;
  for (int64_t k = 0; k < total; ++k) {
    const uint32_t a = (uint32_t)later[k], b = (uint32_t)earlier[k];
    const uint32_t d = std::max(last[a], last[b]) + 1u;
    last[a] = last[b] = d;
    deepest = std::max(deepest, d);
  }
  *pairs = total;
  *depth = deepest;
  return NBX_OK;
}

} // extern "C"

namespace {
// FP64 direct sums for targets at the given current indices (checked by
// the caller) over the bodies of each target's own instance; kind as
// launch_direct_fp64.  Writes m values to ax (and to ay for forces).
int direct_sums(nbx_handle *h, const uint32_t *targets, uint32_t m, int kind,
                double *ax, double *ay) {
  if (h->dPartialTargets < m) {
    if (h->dPartial) cudaFree(h->dPartial);
    if (h->dTargets) cudaFree(h->dTargets);
    h->dPartial = nullptr;
    h->dTargets = nullptr;
    h->dPartialTargets = 0;
    NBX_CUDA(h, cudaMalloc(&h->dPartial, direct_partial_elems(m) * sizeof(double2) + 16 * m));
    // targets (u32), then 8-byte aligned source ranges (uint2)
    NBX_CUDA(h, cudaMalloc(&h->dTargets, 4ull * (m + 1) + 8ull * m));
    h->dPartialTargets = m;
  }
  double *dOut = reinterpret_cast<double *>(h->dPartial + direct_partial_elems(h->dPartialTargets));
  // each target's sources: the bodies of its own instance
  uint2 *dRanges = reinterpret_cast<uint2 *>(h->dTargets + ((h->dPartialTargets + 1) & ~1u));
  std::vector<uint32_t> staged(3ull * m);
  for (uint32_t k = 0; k < m; ++k) {
    const auto it = std::upper_bound(h->segStart.begin(), h->segStart.end(), targets[k]);
    const size_t sg = (size_t)(it - h->segStart.begin()) - 1;
    staged[k] = targets[k];
    staged[m + 2 * k] = h->segStart[sg];
    staged[m + 2 * k + 1] = h->segStart[sg] + h->segCount[sg];
  }
  NBX_CUDA(h, cudaMemcpyAsync(h->dTargets, staged.data(), 4ull * m, cudaMemcpyHostToDevice, h->stream));
  NBX_CUDA(h, cudaMemcpyAsync(dRanges, staged.data() + m, 8ull * m, cudaMemcpyHostToDevice, h->stream));
  const DevState S = h->state();
  launch_direct_fp64(h->stream, S.pv, S.mr, h->n, h->dTargets, dRanges, m,
                     h->params.epsilon, kind, h->dPartial, dOut, dOut + m);
  NBX_CUDA(h, cudaGetLastError());
  NBX_CUDA(h, cudaMemcpyAsync(ax, dOut, 8ull * m, cudaMemcpyDeviceToHost, h->stream));
  if (ay)
    NBX_CUDA(h, cudaMemcpyAsync(ay, dOut + m, 8ull * m, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

// Neumaier accumulation in FP64 (host side of the compensated sums).
struct HostKSum {
  double s = 0.0, c = 0.0;
  void add(double v) {
    const double t = s + v;
    if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};
} // namespace

extern "C" {

int nbx_direct_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m, double *ax,
                    double *ay) {
  if (!h || (m && (!targets || !ax || !ay))) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (m == 0) return NBX_OK;
  for (uint32_t k = 0; k < m; ++k)
    if (targets[k] >= h->n) return fail(h, NBX_ERR_ARG, "target index out of range");
  return direct_sums(h, targets, m, h->params.force_law == 1 ? 1 : 0, ax, ay);
}

int nbx_law_error_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                       double *stats) {
  if (!h || !stats || (m && !targets)) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->params.force_law != 0) return fail(h, NBX_ERR_STATE, "defined for the tree law");
  for (int k = 0; k < 4; ++k) stats[k] = 0.0;
  if (m == 0) return NBX_OK;
  for (uint32_t k = 0; k < m; ++k)
    if (targets[k] >= h->n) return fail(h, NBX_ERR_ARG, "target index out of range");
  std::vector<double> ex(m), ey(m), fx(m), fy(m);
  int rc = direct_sums(h, targets, m, 0, ex.data(), ey.data());
  if (rc) return rc;
  rc = direct_sums(h, targets, m, 4, fx.data(), fy.data());
  if (rc) return rc;
  std::vector<double> e(m);
  double mean = 0.0;
  for (uint32_t k = 0; k < m; ++k) {
    const double dx = fx[k] - ex[k], dy = fy[k] - ey[k];
    e[k] = std::sqrt(dx * dx + dy * dy) /
           std::max(std::sqrt(ex[k] * ex[k] + ey[k] * ey[k]), 1e-30);
    mean += e[k];
  }
  std::sort(e.begin(), e.end());
  stats[0] = e[m / 2];
  stats[1] = e[std::min<size_t>(m - 1, (size_t)(0.99 * m))];
  stats[2] = e.back();
  stats[3] = mean / m;
  return NBX_OK;
}

int nbx_potential_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m, double *phi,
                       double *u) {
  if (!h || !u || (targets && m && !phi)) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  const int kind = h->params.force_law == 1 ? 3 : 2;
  const DevState S = h->state();
  if (targets) {
    *u = 0.0;
    if (m == 0) return NBX_OK;
    for (uint32_t k = 0; k < m; ++k)
      if (targets[k] >= h->n) return fail(h, NBX_ERR_ARG, "target index out of range");
    int rc = direct_sums(h, targets, m, kind, phi, nullptr);
    if (rc) return rc;
    std::vector<float2> mr(h->n);
    NBX_CUDA(h, cudaMemcpyAsync(mr.data(), S.mr, 8ull * h->n, cudaMemcpyDeviceToHost, h->stream));
    NBX_CUDA(h, cudaStreamSynchronize(h->stream));
    HostKSum sum;
    for (uint32_t k = 0; k < m; ++k) sum.add((double)mr[targets[k]].x * phi[k]);
    *u = 0.5 * sum.value() * ((double)h->n / (double)m);
    return NBX_OK;
  }
  // every body a target, in batches that keep the partial sums small
  std::vector<float2> mr(h->n);
  NBX_CUDA(h, cudaMemcpyAsync(mr.data(), S.mr, 8ull * h->n, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  constexpr uint32_t kBatch = 1u << 16;
  std::vector<uint32_t> idx(std::min<size_t>(kBatch, h->n));
  std::vector<double> ph(idx.size());
  HostKSum sum;
  for (uint32_t b0 = 0; b0 < h->n; b0 += kBatch) {
    const uint32_t cnt = std::min<uint32_t>(kBatch, h->n - b0);
    for (uint32_t k = 0; k < cnt; ++k) idx[k] = b0 + k;
    int rc = direct_sums(h, idx.data(), cnt, kind, ph.data(), nullptr);
    if (rc) return rc;
    for (uint32_t k = 0; k < cnt; ++k) sum.add((double)mr[b0 + k].x * ph[k]);
  }
  *u = 0.5 * sum.value();
  return NBX_OK;
}

int nbx_force_error_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                         double *stats, double *err) {
  if (!h || !stats) return NBX_ERR_ARG;
  std::vector<double> ex(m), ey(m);
  int rc = nbx_direct_fp64(h, targets, m, ex.data(), ey.data());
  if (rc) return rc;
  const DevState S = h->state();
  std::vector<float2> acc(h->n);
  NBX_CUDA(h, cudaMemcpyAsync(acc.data(), S.acc, 8ull * h->n, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  std::vector<double> e(m);
  double mean = 0.0;
  for (uint32_t k = 0; k < m; ++k) {
    const float2 a = acc[targets[k]];
    const double dx = (double)a.x - ex[k], dy = (double)a.y - ey[k];
    const double ref = std::sqrt(ex[k] * ex[k] + ey[k] * ey[k]);
    e[k] = std::sqrt(dx * dx + dy * dy) / std::max(ref, 1e-30);
    mean += e[k];
    if (err) err[k] = e[k];
  }
  std::vector<double> s = e;
  std::sort(s.begin(), s.end());
  stats[0] = m ? s[m / 2] : 0.0;
  stats[1] = m ? s[std::min<size_t>(m - 1, (size_t)(0.99 * m))] : 0.0;
  stats[2] = m ? s.back() : 0.0;
  stats[3] = m ? mean / m : 0.0;
  return NBX_OK;
}

int nbx_energy_momentum_fp64(nbx_handle *h, double *out5) {
  if (!h || !out5) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  const DevState S = h->state();
  launch_energy_momentum(h->stream, S.pv, S.mr, h->n, h->dF64, h->dF64 + 10 * 592);
  NBX_CUDA(h, cudaGetLastError());
  NBX_CUDA(h, cudaMemcpyAsync(out5, h->dF64 + 10 * 592, 40, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

int nbx_status_bits(nbx_handle *h, uint32_t *bits) {
  if (!h || !bits) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  NBX_CUDA(h, cudaMemcpyAsync(bits, h->base.status, 4, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaMemsetAsync(h->base.status, 0, 4, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

int nbx_profile_step(nbx_handle *h, uint32_t max_marks, char *labels,
                     float *ms, uint32_t *count) {
  if (!h || !count || (max_marks && (!labels || !ms))) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  PhaseMarks marks;
  for (int k = 0; k < PhaseMarks::kMax; ++k) cudaEventCreate(&marks.ev[k]);
  cudaStream_t s = h->stream;
  g_marks = &marks;
  mark(s, "start");
  enqueue_step(h, s, h->state());
  g_marks = nullptr;
  h->cur ^= 1;
  after_step(h);
  cudaError_t e = cudaStreamSynchronize(s);
  const uint32_t segs = marks.count > 0 ? (uint32_t)marks.count - 1 : 0;
  *count = segs;
  for (uint32_t k = 0; k < segs && k < max_marks; ++k) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, marks.ev[k], marks.ev[k + 1]);
    ms[k] = t;
    std::snprintf(labels + 32 * k, 32, "%s", marks.label[k + 1]);
  }
  for (int k = 0; k < PhaseMarks::kMax; ++k) cudaEventDestroy(marks.ev[k]);
  if (e != cudaSuccess) return cuda_fail(h, e, "profile step");
  return check_status(h);
}

// ---------------------------------------------------------------- MLP
static int scratch_alloc(nbx_handle *h, void **p, size_t bytes) {
  NBX_CUDA(h, cudaMalloc(p, std::max<size_t>(bytes, 16)));
  h->scratch.push_back(*p);
  return NBX_OK;
}

static void scratch_free(nbx_handle *h, void *p) {
  for (auto it = h->scratch.begin(); it != h->scratch.end(); ++it)
    if (*it == p) {
      cudaFree(p);
      h->scratch.erase(it);
      return;
    }
}

int nbx_mlp_set_params(nbx_handle *h, const float *params, uint32_t n) {
  if (!h || !params || n != (uint32_t)kMlpParams) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  NBX_CUDA(h, cudaMemcpyAsync(h->mlpP, params, 4ull * n, cudaMemcpyHostToDevice, h->stream));
  NBX_CUDA(h, cudaMemsetAsync(h->mlpM, 0, 4ull * n, h->stream));
  NBX_CUDA(h, cudaMemsetAsync(h->mlpV, 0, 4ull * n, h->stream));
  mlp_pack(h->stream, h->mlpP, h->mlpW);
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  h->mlpLoaded = true;
  h->mlpStep = 0;
  destroy_graphs(h);
  return NBX_OK;
}

int nbx_mlp_get_params(nbx_handle *h, float *params, uint32_t n) {
  if (!h || !params || n != (uint32_t)kMlpParams) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  NBX_CUDA(h, cudaMemcpyAsync(params, h->mlpP, 4ull * n, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  return NBX_OK;
}

int nbx_mlp_init(nbx_handle *h, uint32_t seed) {
  if (!h) return NBX_ERR_ARG;
  std::vector<float> P(kMlpParams, 0.0f);
  std::mt19937 rng(seed);
  auto fill = [&](int off, int rows, int cols) {
    const float a = std::sqrt(6.0f / (float)(rows + cols));
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < rows * cols; ++i) P[off + i] = u(rng);
  };
  fill(kOffW1, 32, 9);
  fill(kOffW2, 32, 32);
  fill(kOffW3, 2, 32);
  for (int i = 0; i < 2 * 32; ++i) P[kOffW3 + i] *= 0.1f; // start near zero correction
  return nbx_mlp_set_params(h, P.data(), kMlpParams);
}

int nbx_mlp_harvest(nbx_handle *h, const uint32_t *targets, uint32_t nt,
                    float theta, float band, float *rows, uint32_t maxRows,
                    uint32_t *nRows) {
  if (!h || !nRows || (nt && !targets) || (maxRows && !rows)) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
  if (!h->momentsValid)
    return fail(h, NBX_ERR_STATE,
                "the last tree has no cell moments: build it with nbx_phase (BUILD or "
                "ATTRACT), or step with use_mlp != 0");
  for (uint32_t k = 0; k < nt; ++k)
    if (targets[k] >= h->n) return fail(h, NBX_ERR_ARG, "target index out of range");
  *nRows = 0;
  if (nt == 0 || maxRows == 0) return NBX_OK;
  void *dT = nullptr, *dItems = nullptr, *dRows = nullptr, *dCount = nullptr;
  int rc = scratch_alloc(h, &dT, 4ull * nt);
  if (!rc) rc = scratch_alloc(h, &dItems, 8ull * maxRows);
  if (!rc) rc = scratch_alloc(h, &dRows, 4ull * kMlpRow * maxRows);
  if (!rc) rc = scratch_alloc(h, &dCount, 16);
  if (!rc) {
    cudaMemcpyAsync(dT, targets, 4ull * nt, cudaMemcpyHostToDevice, h->stream);
    const DevState S = h->state();
    mlp_harvest(h->stream, S, (const uint32_t *)dT, nt, theta, band, h->params.epsilon,
                (uint2 *)dItems, maxRows, (uint32_t *)dCount, (float *)dRows);
    uint32_t cnt = 0;
    cudaMemcpyAsync(&cnt, dCount, 4, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      rc = cuda_fail(h, e, "harvest");
    } else {
      cnt = std::min(cnt, maxRows);
      e = cudaMemcpy(rows, dRows, 4ull * kMlpRow * cnt, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = cuda_fail(h, e, "harvest copy");
      *nRows = cnt;
    }
  }
  for (void *p : {dT, dItems, dRows, dCount})
    if (p) scratch_free(h, p);
  return rc;
}

int nbx_mlp_gradient(nbx_handle *h, const float *rows, uint32_t n, float *grad,
                     float *loss) {
  if (!h || !rows || !n || !grad) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->mlpLoaded) return fail(h, NBX_ERR_STATE, "no MLP parameters");
  const int blocks = (n + mlp_rows_per_block() - 1) / mlp_rows_per_block();
  void *dRows = nullptr, *dPart = nullptr, *dLoss = nullptr;
  int rc = scratch_alloc(h, &dRows, 4ull * kMlpRow * n);
  if (!rc) rc = scratch_alloc(h, &dPart, 4ull * kMlpParams * blocks);
  if (!rc) rc = scratch_alloc(h, &dLoss, 4ull * (blocks + 1));
  if (!rc) {
    cudaMemcpyAsync(dRows, rows, 4ull * kMlpRow * n, cudaMemcpyHostToDevice, h->stream);
    mlp_gradient(h->stream, (float *)dRows, nullptr, 0, n, h->mlpP, (float *)dPart,
                 (float *)dLoss, h->mlpGrad, h->mlpGrad + kMlpParams);
    float out[kMlpParams + 1];
    cudaMemcpyAsync(out, h->mlpGrad, sizeof out, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "mlp gradient");
    else {
      std::memcpy(grad, out, 4ull * kMlpParams);
      if (loss) *loss = out[kMlpParams] / (float)n;
    }
  }
  for (void *p : {dRows, dPart, dLoss})
    if (p) scratch_free(h, p);
  return rc;
}

int nbx_mlp_train(nbx_handle *h, const float *rows, uint32_t n, uint32_t epochs,
                  uint32_t batch, float lr, uint32_t seed, float *epochLoss) {
  if (!h || !rows || !n || !batch || batch > n) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->mlpLoaded) {
    int rc = nbx_mlp_init(h, seed);
    if (rc) return rc;
  }
  const uint32_t steps = n / batch;
  const int blocks = (batch + mlp_rows_per_block() - 1) / mlp_rows_per_block();
  void *dRows = nullptr, *dOrder = nullptr, *dPart = nullptr, *dLoss = nullptr,
       *dSteps = nullptr;
  int rc = scratch_alloc(h, &dRows, 4ull * kMlpRow * n);
  if (!rc) rc = scratch_alloc(h, &dOrder, 4ull * n);
  if (!rc) rc = scratch_alloc(h, &dPart, 4ull * kMlpParams * blocks);
  if (!rc) rc = scratch_alloc(h, &dLoss, 4ull * (blocks + 1));
  if (!rc) rc = scratch_alloc(h, &dSteps, 4ull * steps);
  if (!rc) {
    cudaMemcpyAsync(dRows, rows, 4ull * kMlpRow * n, cudaMemcpyHostToDevice, h->stream);
    std::vector<uint32_t> order(n);
    std::vector<float> stepLoss(steps);
    std::mt19937 rng(seed);
    for (uint32_t e = 0; e < epochs && !rc; ++e) {
      for (uint32_t i = 0; i < n; ++i) order[i] = i;
      std::shuffle(order.begin(), order.end(), rng);
      cudaMemcpyAsync(dOrder, order.data(), 4ull * n, cudaMemcpyHostToDevice, h->stream);
      for (uint32_t k = 0; k < steps; ++k) {
        mlp_gradient(h->stream, (float *)dRows, (uint32_t *)dOrder, k * batch, batch,
                     h->mlpP, (float *)dPart, (float *)dLoss, h->mlpGrad,
                     (float *)dSteps + k);
        mlp_adam(h->stream, h->mlpP, h->mlpGrad, h->mlpM, h->mlpV, ++h->mlpStep, lr,
                 h->mlpW);
      }
      cudaMemcpyAsync(stepLoss.data(), dSteps, 4ull * steps, cudaMemcpyDeviceToHost,
                      h->stream);
      cudaError_t ce = cudaStreamSynchronize(h->stream);
      if (ce != cudaSuccess) rc = cuda_fail(h, ce, "mlp train");
      if (epochLoss) {
        double s = 0.0;
        for (float v : stepLoss) s += v;
        epochLoss[e] = (float)(s / ((double)steps * batch));
      }
    }
  }
  for (void *p : {dRows, dOrder, dPart, dLoss, dSteps})
    if (p) scratch_free(h, p);
  destroy_graphs(h);
  return rc;
}

int nbx_mlp_eval(nbx_handle *h, const float *feat, uint32_t n, float *out,
                 int tensor) {
  if (!h || (n && (!feat || !out))) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->mlpLoaded) return fail(h, NBX_ERR_STATE, "no MLP parameters");
  if (!n) return NBX_OK;
  void *dF = nullptr, *dO = nullptr;
  int rc = scratch_alloc(h, &dF, 36ull * n);
  if (!rc) rc = scratch_alloc(h, &dO, 8ull * n);
  if (!rc) {
    cudaMemcpyAsync(dF, feat, 36ull * n, cudaMemcpyHostToDevice, h->stream);
    mlp_eval(h->stream, (float *)dF, n, h->mlpP, h->mlpW, (float *)dO, tensor != 0);
    cudaMemcpyAsync(out, dO, 8ull * n, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = cuda_fail(h, e, "mlp eval");
  }
  for (void *p : {dF, dO})
    if (p) scratch_free(h, p);
  return rc;
}

int nbx_accel_at(nbx_handle *h, const float *px, const float *py, uint32_t nq,
                 float *ax, float *ay) {
  if (!h || (nq && (!px || !py || !ax || !ay))) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
  if (nq == 0) return NBX_OK;
  std::vector<float2> q(nq), r(nq);
  for (uint32_t i = 0; i < nq; ++i) q[i] = make_float2(px[i], py[i]);
  void *buf = nullptr;
  int rc = scratch_alloc(h, &buf, 16ull * nq);
  if (rc) return rc;
  float2 *dq = (float2 *)buf, *dr = dq + nq;
  cudaMemcpyAsync(dq, q.data(), 8ull * nq, cudaMemcpyHostToDevice, h->stream);
  launch_query_forces(h->stream, h->state(), h->params.exact_math != 0, dq, nq, dr);
  cudaMemcpyAsync(r.data(), dr, 8ull * nq, cudaMemcpyDeviceToHost, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  scratch_free(h, buf);
  if (e != cudaSuccess) return cuda_fail(h, e, "accel_at");
  for (uint32_t i = 0; i < nq; ++i) {
    ax[i] = r[i].x;
    ay[i] = r[i].y;
  }
  return NBX_OK;
}

// ------------------------------------------------------------ autotuner
int nbx_autotune(nbx_handle *h, int allowLeaf, uint32_t steps, nbx_params *best,
                 float *bestMs) {
  if (!h || !best || steps == 0) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
  if (h->n == 0) {
    *best = h->params;
    if (bestMs) *bestMs = 0.0f;
    return NBX_OK;
  }
  // snapshot of the state: every trial starts from it, and it is restored
  const DevState S0 = h->state();
  const size_t n = h->n;
  void *sv = nullptr;
  int rc = scratch_alloc(h, &sv, n * (sizeof(float4) + sizeof(float2) * 2 + 4));
  if (rc) return rc;
  char *b = (char *)sv;
  float4 *pv = (float4 *)b;
  float2 *mr = (float2 *)(b + n * 16), *acc = (float2 *)(b + n * 24);
  uint32_t *id = (uint32_t *)(b + n * 32);
  const int cur0 = h->cur;
  auto save = [&]() {
    cudaMemcpyAsync(pv, S0.pv, n * 16, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(mr, S0.mr, n * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(acc, S0.acc, n * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(id, S0.id, n * 4, cudaMemcpyDeviceToDevice, h->stream);
  };
  auto restore = [&]() {
    h->cur = cur0;
    cudaMemcpyAsync(S0.pv, pv, n * 16, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(S0.mr, mr, n * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(S0.acc, acc, n * 8, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(S0.id, id, n * 4, cudaMemcpyDeviceToDevice, h->stream);
  };
  save();
  const nbx_params start = h->params;
  std::vector<int> leaves = {start.leaf_capacity};
  if (allowLeaf) leaves = {8, 12, 16, 24, 32};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  // block shape and leaf width apply to the default plain walk only
  const bool plain = !start.exact_math && start.use_mlp == 0;
  std::vector<int> blockShapes = {start.force_block};
  std::vector<int> leafWidths = {start.leaf_pairs};
  if (plain) {
    blockShapes = {128, 256, 512};
    leafWidths = {1, 0};
  }
  struct Trial {
    int leaf, threads, pairs, grid;
  };
  std::vector<Trial> trials;
  for (int leaf : leaves)
    for (int threads : blockShapes)
      for (int pairs : leafWidths) {
        // grids: one warp per 32 bodies, or a half, one or two full SMs'
        // worth of resident blocks per SM (the paired walk's launch bounds
        // hold 1536 threads per SM, the single-body walk's 2048)
        const int perSm = (pairs ? 1536 : 2048) / (threads > 0 ? threads : 256);
        for (int grid : {0, sms * perSm / 2, sms * perSm, sms * perSm * 2})
          trials.push_back({leaf, threads, pairs, grid});
      }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  nbx_params bestP = start;
  float bestT = 1e30f;
  {
    for (const Trial &tr : trials) {
      nbx_params p = start;
      p.leaf_capacity = tr.leaf;
      p.force_blocks = tr.grid;
      p.force_block = tr.threads;
      p.leaf_pairs = tr.pairs;
      h->params = p;
      sync_params(h);
      destroy_graphs(h);
      restore();
      if ((rc = nbx_step(h, 1)) != NBX_OK) break;
      cudaEventRecord(e0, h->stream);
      if ((rc = nbx_step(h, steps)) != NBX_OK) break;
      cudaEventRecord(e1, h->stream);
      if ((rc = nbx_sync(h)) != NBX_OK) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)steps;
      if (ms < bestT) {
        bestT = ms;
        bestP = p;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->params = rc ? start : bestP;
  sync_params(h);
  destroy_graphs(h);
  restore();
  cudaError_t e = cudaStreamSynchronize(h->stream);
  scratch_free(h, sv);
  if (e != cudaSuccess && !rc) rc = cuda_fail(h, e, "autotune");
  h->treeValid = false;
  h->forceInput = false;
  h->collideValid = false;
  *best = h->params;
  if (bestMs) *bestMs = bestT;
  return rc;
}

int nbx_get_stream(nbx_handle *h, void **stream) {
  if (!h || !stream) return NBX_ERR_ARG;
  *stream = (void *)h->stream;
  return NBX_OK;
}

int nbx_step_kernel_count(nbx_handle *h, uint32_t *kernels) {
  if (!h || !kernels) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->graphsValid) {
    if (!h->uploaded) return fail(h, NBX_ERR_STATE, "no bodies uploaded");
    int rc = capture_graphs(h);
    if (rc) return rc;
  }
  *kernels = h->graphKernels;
  return NBX_OK;
}

int nbx_interaction_count(nbx_handle *h, double *out5) {
  // out3 holds 5 entries: far, near, visits, warp iterations, tile loads
  if (!h || !out5) return NBX_ERR_ARG;
  cudaSetDevice(h->device);
  if (!h->treeValid) return fail(h, NBX_ERR_STATE, "no tree built");
  const DevState S = h->state();
  unsigned long long *d = reinterpret_cast<unsigned long long *>(h->dF64 + 15 * 592);
  launch_interaction_count(h->stream, S, d);
  NBX_CUDA(h, cudaGetLastError());
  unsigned long long c[5];
  NBX_CUDA(h, cudaMemcpyAsync(c, d, sizeof c, cudaMemcpyDeviceToHost, h->stream));
  NBX_CUDA(h, cudaStreamSynchronize(h->stream));
  for (int k = 0; k < 5; ++k) out5[k] = (double)c[k];
  return NBX_OK;
}

int nbx_fp32_peak_tflops(double *tflops) {
  if (!tflops) return NBX_ERR_ARG;
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    return NBX_ERR_CUDA;
  *tflops = fp32_fma_peak_tflops(s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return *tflops > 0 ? NBX_OK : NBX_ERR_CUDA;
}

const char *nbx_last_error(const nbx_handle *h) {
  return h ? h->lastError.c_str() : "null handle";
}

} // extern "C"
