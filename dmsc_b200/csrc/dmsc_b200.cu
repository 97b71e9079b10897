// dmsc_b200: host orchestration and C ABI (include/dmsc_b200.h).
//
// Replaces the reference CUDA binding and its host-side pipeline
// (dmsc/csrc/dmsc_gpu.cpp:18-180, dmsc/csrc/gpu/dmsc_cuda.hxx:64-477,
// dmsc/csrc/gpu/workspace.hxx:91-397): every stage runs on the device, the
// persistence sweeps and the arc-simplification replay included. The host
// reads back only sizes and round counters.
//
// Internal sides: side 0 = faces (maxima in the primal), side 1 = vertices
// (minima in the primal); the dual swaps roles at the boundary exactly as the
// reference does (dmsc_cpu.cpp:34-37, workspace.hxx:322-362).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cub/cub.cuh>
#include <cudaTypedefs.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/dmsc_b200.h"
#include "assemble.cuh"
#include "common.cuh"
#include "gradient.cuh"
#include "pairing.cuh"
#include "persistent.cuh"
#include "replay.cuh"
#include "pairs.cuh"
#include "walks.cuh"

using namespace dmsc;

namespace {


enum Slot {
  S_MASK, S_FLOW, S_SEG0, S_SEG1, S_SEG2, S_OFF0, S_OFF1, S_OFF2, S_TOT, S_TAB, S_BASES,
  S_CSAD, S_IMIN, S_ISAD, S_IMAX, S_MINBITS, S_MAXBITS, S_KMIN, S_KMAX, S_SVAL, S_SKEY2, S_IOTA,
  S_ASC, S_ARCF, S_ARCV, S_CANC, S_FLAG, S_FPOS, S_SURV, S_STATUS, S_NCANC, S_STATS, S_TIMELINE, S_ROUTE,
  S_BKEY, S_BIDX, S_BKEY2, S_BIDX2, S_PERF, S_PERV, S_EXF, S_EXV, S_NEX, S_SKEY32B, S_SKEYS, S_SURVIC,
  S_SIDE0,  // per-side slots start here, kSideSlots each
};
enum SideSlot {
  X_ROUT, X_SVT, X_SVL, X_SVR, X_DYING, X_GRP, X_LINK, X_MINE, X_ACT0, X_ACT1, X_CNT, X_PAIR, X_ALIVE,
  X_ALIVEI, X_TOOUTX, X_TOOUT, X_UF, X_CROOT, X_CKEY, X_CVAL, X_NODE,
  X_ALEN, X_ACL, X_AROOT, X_PLEN, X_SEND, X_APOS, X_EROWC, X_EROWO, X_Q0, X_Q1, X_QB, X_G12,
  X_GBASE, X_WX, X_WA, X_CENDS, kSideSlots
};

struct Buf {
  void* p = nullptr;
  size_t cap = 0;
};

// Device-side per-image bases (B + 1 entries each) of the last extract.
struct Bases {
  int* min;       // first minimum (vertex extremum) of each image
  int* sad;       // first saddle
  int* max;       // first maximum (face extremum)
  int* surv;      // first surviving saddle
  int* alive[2];  // first output rank of each side's surviving extrema
  int* erow[2];   // first e row of each side
};

struct Side {
  int M = 0;
  bool faces = true;
  bool arcs = false;    // some image takes this side's arcs
  bool groups = false;  // some image takes this side's labels
  bool arcs_primal = false, arcs_dual = false;      // by orientation
  bool groups_primal = false, groups_dual = false;
  int* ext_img = nullptr;
  const int2* key = nullptr;  // (value bits, global cell id) per extremum, list order
  int4* arc = nullptr;              // [nsad] per saddle (list order): arc ends and raw-arc cells
  int* rout = nullptr;              // [M] out rank of each extremum's thresholded root (-1: the void)
  int2* sv_t = nullptr;             // [nsurv] per survivor (output order): arc ends
  longlong2* sv_len = nullptr;      // raw-arc lengths
  int4* sv_rec = nullptr;           // out ranks of the ends' roots, persistence, out rank of the pair's root
  int* dying = nullptr;
  int2* pp = nullptr;               // [nsad] paired extremum (-1: none) and persistence bits
  uint8_t* alive = nullptr;
  int* to_out_excl = nullptr;
  int* to_out = nullptr;
  ReplayState R{};
  int C = 0;
  long long* arc_len = nullptr;
  long long* arc_cl = nullptr;
  int* arc_root = nullptr;
  long long* send = nullptr;
  long long* plen = nullptr;
  long long* gbase = nullptr;  // [B+1] geometry start of each image
  long long total = 0;
  int n_alive = 0;
  int n_erows = 0;
  int* erow_off = nullptr;
};

}  // namespace

constexpr int kStageMarks = 19;
constexpr int kInBands = 8;  // row bands of an image uploaded from a host source

struct dmsc_b200_context {
  int device = 0;
  std::vector<Buf> bufs;
  Buf cub_tmp;
  Buf cub_tmp_side;  // CUB scratch of the work queued on side_st
  long long* pinned = nullptr;  // host staging for readbacks and tables
  size_t pinned_cap = 0;
  std::string err;
  // state of the last extract
  bool valid = false;
  int B = 0;
  unsigned flags = 0;
  int nmin = 0, nsad = 0, nmax = 0, nsurv = 0;
  long long nidx = 0;
  Imgs I{};
  std::vector<int> hH, hW;
  std::vector<uint8_t> hdual;
  Bases bases{};
  const uint8_t* flow = nullptr;
  const float* img = nullptr;  // input of the last extract (read again by fetch_pair_pixels)
  int* crit_sad = nullptr;
  int* sad_img = nullptr;
  int* surv = nullptr;
  int2* surv_ic = nullptr;  // [nsurv] image and cell of each survivor (output order)
  unsigned* status = nullptr;
  Side side[2];
  std::vector<dmsc_b200_sizes> sizes;
  std::vector<long long> geom[2];  // per-image geometry lengths of each side
  // profiling: launch counter and stage boundary events
  long long launches = 0;
  bool profile = false;
  uint32_t* fifo_lut = nullptr;  // face-pairing FIFO table (device)
  int num_sms = 0;
  cudaEvent_t ev[kStageMarks] = {};
  // each side's geometry expansion, launched at the end of extract; the
  // writer in fetch reads its segment list (expanded: launched this call)
  EmitArgs emit[2] = {};
  bool expanded[2] = {false, false};
  cudaEvent_t sync_ev = nullptr;   // polled by wait_stream
  // host destinations of the fixed-size outputs for the next extract (copied
  // on copy_st as soon as each is produced; see dmsc_b200_set_host_outputs)
  int32_t* host_grad = nullptr;
  int32_t* host_peaks = nullptr;
  int32_t* host_basins = nullptr;
  dmsc_b200_outputs host_fetch{};  // host destinations of the next fetch's outputs
  bool host_fetch_set = false;
  bool copies_pending = false;
  cudaStream_t copy_st = nullptr;
  // the second side's persistence, cancellation and rank kernels run on
  // side_st, forked from and joined back to the call's stream
  cudaStream_t side_st = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaEvent_t copy_ev = nullptr;
  // pinned host source of the next extract's image (dmsc_b200_set_host_input),
  // uploaded in bands of rows on in_st; in_ev[k]: band k's rows have arrived
  const float* host_img = nullptr;
  cudaStream_t in_st = nullptr;
  cudaEvent_t in_ev[kInBands] = {};
  // readback area: pinned host memory mapped into the device address space;
  // a small kernel writes the values, so readbacks never queue behind bulk
  // device-to-host copies on the copy engines
  char* rb_h = nullptr;
  char* rb_d = nullptr;
  size_t rb_cap = 0;
  // host wait deadline (seconds) and test-only loop caps (0 = the bounds
  // that every input provably stays within)
  double wait_timeout_s = 600.0;
  // tuned launch shapes (dmsc_b200_set_tuning): gradient tile shape (index
  // into kGradTY / kGradNT), label tile threads (index into kLabelNT), and
  // the resident blocks per SM of the three persistent kernels (0 = all that fit)
  int grad_shape = 3;
  int label_shape = 1;
  int pair_per_sm = 0, replay_per_sm = 0, emit_per_sm = 0;
  int pair_shape = 0;    // pairing items per thread batch: 0 -> 2, 1 -> 4
  int replay_shape = 0;  // replay items per thread batch: 0 -> 1, 1 -> 2
  int emit_shape = 0;    // expansion chain tasks per thread batch: 0 -> 1, 1 -> 2
  int seg_cursors = 1;  // raw-arc cursors per lane of the segment writer
  bool label_smem_set = false;  // dynamic shared memory limit raised for the label kernels
  int cap_pair_rounds = 0, cap_replay_rounds = 0, cap_emit_levels = 0;
};



namespace dmsc {

__global__ void totals3_kernel(const int* o0, const int* s0, const int* o1, const int* s1, const int* o2,
                               const int* s2, long long n, long long* out) {
  out[0] = (long long)o0[n - 1] + s0[n - 1];
  out[1] = (long long)o1[n - 1] + s1[n - 1];
  out[2] = (long long)o2[n - 1] + s2[n - 1];
}

template <class T>
__global__ void last_plus_kernel(const T* excl, const T* val, int n, long long* out) {
  *out = n > 0 ? (long long)excl[n - 1] + (long long)val[n - 1] : 0;
}

__global__ void copy2_kernel(const int* a, long long* out) {
  out[0] = a[0];
  out[1] = a[1];
}

template <class T>
__global__ void last_kernel(const T* a, int n, long long* out) {
  *out = n > 0 ? (long long)a[n - 1] : 0;
}

__global__ void u8_last_plus_kernel(const int* excl, const uint8_t* v, int n, long long* out) {
  *out = n > 0 ? (long long)excl[n - 1] + v[n - 1] : 0;
}

// 32-bit words from device memory into the mapped readback area.
__global__ void copy_words_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

}  // namespace dmsc

namespace {

struct Fail {
  int code;
};

void set_err(dmsc_b200_context* c, const char* fmt, ...) {
  char b[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(b, sizeof b, fmt, ap);
  va_end(ap);
  c->err = b;
}

void ck(dmsc_b200_context* c, cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    set_err(c, "%s: %s", what, cudaGetErrorString(e));
    throw Fail{kErrCuda};
  }
}
#define CK(x) ck(ctx, (x), #x)
#define LAUNCH_CHECK(name) ck(ctx, cudaGetLastError(), name)
// every kernel launch of this library goes through LK so the context can
// report how many kernels one call issued (CUB scans/sorts count once each)
#define LK(...)      \
  do {                \
    __VA_ARGS__;      \
    ++ctx->launches;  \
  } while (0)

// A loop bound lowered to a test-only cap (cap <= 0: the bound itself).
int capped(long long bound, int cap) {
  const long long b = cap > 0 && cap < bound ? cap : bound;
  return (int)std::min<long long>(b, 2147483647LL);
}

template <class T>
T* get(dmsc_b200_context* ctx, int slot, size_t n) {
  size_t bytes = n * sizeof(T);
  if (bytes == 0) bytes = 16;
  if ((size_t)slot >= ctx->bufs.size()) ctx->bufs.resize(slot + 1);
  Buf& b = ctx->bufs[slot];
  if (b.cap < bytes) {
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    size_t nb = bytes + bytes / 4 + 256;
    CK(cudaMalloc(&b.p, nb));
    b.cap = nb;
  }
  return (T*)b.p;
}

template <class T>
T* sget(dmsc_b200_context* ctx, int side, int slot, size_t n) {
  return get<T>(ctx, S_SIDE0 + side * kSideSlots + slot, n);
}

void* cub_tmp(dmsc_b200_context* ctx, size_t bytes, cudaStream_t st) {
  Buf& b = (st && st == ctx->side_st) ? ctx->cub_tmp_side : ctx->cub_tmp;
  if (b.cap < bytes) {
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    size_t nb = bytes + bytes / 4 + 256;
    CK(cudaMalloc(&b.p, nb));
    b.cap = nb;
  }
  return b.p;
}

template <class In, class Out>
void excl_sum(dmsc_b200_context* ctx, const In* in, Out* out, int n, cudaStream_t st) {
  if (n <= 0) return;
  size_t bytes = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
  void* tmp = cub_tmp(ctx, bytes, st);
  CK(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, st));
  ++ctx->launches;
}

template <class In, class Out>
void incl_sum(dmsc_b200_context* ctx, const In* in, Out* out, int n, cudaStream_t st) {
  if (n <= 0) return;
  size_t bytes = 0;
  CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, n, st));
  void* tmp = cub_tmp(ctx, bytes, st);
  CK(cub::DeviceScan::InclusiveSum(tmp, bytes, in, out, n, st));
  ++ctx->launches;
}

template <class K>
void sort_pairs(dmsc_b200_context* ctx, const K* kin, K* kout, const int* vin, int* vout, int n, cudaStream_t st,
                int end_bit = (int)(8 * sizeof(K))) {
  if (n <= 0) return;
  size_t bytes = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, st));
  void* tmp = cub_tmp(ctx, bytes, st);
  CK(cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, n, 0, end_bit, st));
  ++ctx->launches;
}

// Records stage boundary `k` when profiling.
void mark(dmsc_b200_context* ctx, int k, cudaStream_t st) {
  if (ctx->profile) CK(cudaEventRecord(ctx->ev[k], st));
}

// Cooperative launch of a persistent kernel: as many blocks as can be
// co-resident, so grid-wide barriers are safe.
template <class T>
void coop_launch(dmsc_b200_context* ctx, void (*kernel)(T), T args, cudaStream_t st, const char* name,
                 int per_cap = 0) {
  int per = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, 0));
  if (per < 1) {
    set_err(ctx, "%s cannot be made resident", name);
    throw Fail{kErrInternal};
  }
  if (per_cap > 0 && per_cap < per) per = per_cap;
  void* a[] = {&args};
  CK(cudaLaunchCooperativeKernel((void*)kernel, dim3(per * ctx->num_sms), dim3(256), a, 0, st));
  ++ctx->launches;
}

// Waits until the stream has drained by polling an event: the host thread
// spins instead of sleeping in the driver, so the next launches follow the
// readback without an operating-system wake-up delay (the few host round
// trips of a call are on its critical path). Gives up after the context's
// wait deadline with DMSC_B200_ERR_CUDA; the work may still be running then,
// so the context must be destroyed, not reused.
void wait_stream(dmsc_b200_context* ctx, cudaStream_t st) {
  CK(cudaEventRecord(ctx->sync_ev, st));
  const auto t0 = std::chrono::steady_clock::now();
  for (unsigned k = 0;; ++k) {
    const cudaError_t e = cudaEventQuery(ctx->sync_ev);
    if (e == cudaSuccess) return;
    if (e != cudaErrorNotReady) CK(e);
    if ((k & 15u) == 15u &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > ctx->wait_timeout_s) {
      set_err(ctx, "device work did not finish within %.1f s", ctx->wait_timeout_s);
      throw Fail{kErrCuda};
    }
  }
}

// Device -> host copy of a finished output on the context's copy stream,
// ordered after the work enqueued on `st` so far.
void copy_out_async(dmsc_b200_context* ctx, void* host, const void* dev, size_t bytes, cudaStream_t st) {
  if (!host || !dev || !bytes) return;
  CK(cudaEventRecord(ctx->copy_ev, st));
  CK(cudaStreamWaitEvent(ctx->copy_st, ctx->copy_ev, 0));
  CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->copy_st));
  ctx->copies_pending = true;
}

// Makes `st` wait for every copy issued on the copy stream.
void join_copies(dmsc_b200_context* ctx, cudaStream_t st) {
  if (!ctx->copies_pending) return;
  CK(cudaEventRecord(ctx->copy_ev, ctx->copy_st));
  CK(cudaStreamWaitEvent(st, ctx->copy_ev, 0));
  ctx->copies_pending = false;
}

// After a failure: wait for the copies already issued, so no host buffer is
// written after the call returns, and forget the registered destinations.
void abandon_copies(dmsc_b200_context* ctx) {
  if (ctx->copy_st) cudaStreamSynchronize(ctx->copy_st);
  if (ctx->in_st) cudaStreamSynchronize(ctx->in_st);  // uploads from a host image source
  ctx->copies_pending = false;
  ctx->host_grad = ctx->host_peaks = ctx->host_basins = nullptr;
  ctx->host_fetch_set = false;
}

// Mapped readback area of at least `bytes` (grown only between readbacks).
void rb_reserve(dmsc_b200_context* ctx, size_t bytes) {
  if (ctx->rb_cap >= bytes) return;
  if (ctx->rb_h) CK(cudaFreeHost(ctx->rb_h));
  ctx->rb_h = ctx->rb_d = nullptr;
  ctx->rb_cap = 0;
  const size_t nb = ((bytes + bytes / 2 + 4096) + 255) & ~(size_t)255;
  CK(cudaHostAlloc((void**)&ctx->rb_h, nb, cudaHostAllocMapped));
  CK(cudaHostGetDevicePointer((void**)&ctx->rb_d, ctx->rb_h, 0));
  ctx->rb_cap = nb;
}

// Enqueues the copy of `bytes` (a multiple of 4) from device `src` to offset
// `off` of the readback area.
void rb_copy(dmsc_b200_context* ctx, cudaStream_t st, size_t off, const void* src, size_t bytes) {
  const int n = (int)(bytes / 4);
  if (n <= 0) return;
  LK(copy_words_kernel<<<grid_for(n, 256) < 64 ? grid_for(n, 256) : 64, 256, 0, st>>>(
      (const uint32_t*)src, (uint32_t*)(ctx->rb_d + off), n));
  LAUNCH_CHECK("copy_words_kernel");
}

// Host read of `k` device scalars (into rb, as long long) after the stream drains.
void readback(dmsc_b200_context* ctx, cudaStream_t st, const long long* dev, int k) {
  rb_reserve(ctx, k * sizeof(long long));
  rb_copy(ctx, st, 0, dev, k * sizeof(long long));
  wait_stream(ctx, st);
}
const long long* rb_ll(dmsc_b200_context* ctx) { return (const long long*)ctx->rb_h; }

// Error of a device status word (0: none).
void raise_status(dmsc_b200_context* ctx, unsigned h) {
  if (h & (kStatusWalkCap | kStatusRoundCap | kStatusChainCap | kStatusFindCap)) {
    set_err(ctx, "a bounded device loop reached its cap (status 0x%x)", h);
    throw Fail{kErrIterationCap};
  }
  if (h & kStatusCopyWait) {
    set_err(ctx, "a tensor copy into shared memory timed out (status 0x%x)", h);
    throw Fail{kErrCuda};
  }
  if (h & kStatusQueueOverflow) {
    set_err(ctx, "geometry work queue overflow (status 0x%x)", h);
    throw Fail{kErrOverflow};
  }
  if (h) {
    set_err(ctx, "device status 0x%x", h);
    throw Fail{kErrInternal};
  }
}

void check_status(dmsc_b200_context* ctx, cudaStream_t st) {
  rb_reserve(ctx, 64);
  rb_copy(ctx, st, 0, ctx->status, sizeof(unsigned));
  wait_stream(ctx, st);
  raise_status(ctx, *(const unsigned*)ctx->rb_h);
}



constexpr int TB = 256;

// Pinned host staging of at least `bytes`.
void* staging(dmsc_b200_context* ctx, size_t bytes) {
  if (ctx->pinned_cap < bytes) {
    if (ctx->pinned) CK(cudaFreeHost(ctx->pinned));
    ctx->pinned = nullptr;
    size_t nb = bytes + bytes / 2 + 1024;
    CK(cudaMallocHost(&ctx->pinned, nb));
    ctx->pinned_cap = nb;
  }
  return ctx->pinned;
}

// Sweep-ordered edges and the pairing arguments of one side (see pairing.cuh).
PairArgs pairing_args(dmsc_b200_context* ctx, int si, Side& S) {
  const int nsad = ctx->nsad, M = S.M;
  S.dying = sget<int>(ctx, si, X_DYING, nsad);  // list order
  PairArgs A;
  A.nsad = nsad;
  A.M = M;
  A.sval = get<float>(ctx, S_SVAL, nsad);
  A.sad_img = ctx->sad_img;
  A.g12 = sget<int2>(ctx, si, X_G12, nsad);
  A.dying = S.dying;
  A.link = sget<int>(ctx, si, X_LINK, M + 1);
  A.minedge = sget<unsigned long long>(ctx, si, X_MINE, M + 1);
  A.act0 = sget<int>(ctx, si, X_ACT0, nsad);
  A.act1 = sget<int>(ctx, si, X_ACT1, nsad);
  A.roots0 = sget<int>(ctx, si, X_GRP, M + 1);
  A.roots1 = sget<int>(ctx, si, X_UF, M + 1);
  A.cnt = sget<int>(ctx, si, X_CNT, 8);
  A.key = S.key;
  A.idx_base = ctx->I.idx_base;
  A.B = ctx->B;
  A.dual = ctx->I.dual;
  A.faces = S.faces;
  A.status = ctx->status;
  A.max_rounds = capped(M + 2, ctx->cap_pair_rounds);
  A.rounds = get<int>(ctx, S_STATS, 8) + 0 + si;
  A.timeline = get<unsigned long long>(ctx, S_TIMELINE, kTimelineSlots) + si * kTimeline;
  return A;
}

// Both sides' pairing rounds in one cooperative launch.
void run_pairing(dmsc_b200_context* ctx, cudaStream_t st) {
  PairArgs2 P;
  for (int si = 0; si < 2; ++si) P.s[si] = pairing_args(ctx, si, ctx->side[si]);
  if (ctx->nsad > 0)
    coop_launch(ctx, ctx->pair_shape ? pairing_persistent_kernel<4, 4> : pairing_persistent_kernel<2, 5>, P, st,
                "pairing_persistent_kernel", ctx->pair_per_sm);
}

// Persistence, cancellation, thresholded union-find and output ranks of one side.
void finish_pairing(dmsc_b200_context* ctx, int si, Side& S, cudaStream_t st) {
  const int nsad = ctx->nsad, M = S.M;
  // persistence, cancellation, alive flags
  S.pp = sget<int2>(ctx, si, X_PAIR, nsad);
  S.alive = sget<uint8_t>(ctx, si, X_ALIVE, M + 4);
  CK(cudaMemsetAsync(S.alive, 1, M + 4, st));
  uint8_t* canc = get<uint8_t>(ctx, S_CANC, nsad + 4);
  int* ncanc = get<int>(ctx, S_NCANC, 4) + si;
  CK(cudaMemsetAsync(ncanc, 0, sizeof(int), st));
  int2* cends = sget<int2>(ctx, si, X_CENDS, nsad);
  // the replay's cancellation list (keys and saddles) comes out of the same
  // pass when this side's arcs are simplified
  unsigned long long* ckey = S.arcs ? sget<unsigned long long>(ctx, si, X_CKEY, nsad) : nullptr;
  int* cval = S.arcs ? sget<int>(ctx, si, X_CVAL, nsad) : nullptr;
  ReplayNode* node = S.arcs ? sget<ReplayNode>(ctx, si, X_NODE, M + 1) : nullptr;
  if (nsad > 0) {
    LK(persistence_kernel<<<grid_for(nsad, TB), TB, 0, st>>>(
        nsad, !S.faces, ctx->I.dual, ctx->I.thr, ctx->sad_img, S.dying, get<float>(ctx, S_SVAL, nsad), S.key,
        S.pp, canc, (uint8_t)(S.faces ? 1 : 2), S.alive, ncanc, S.arc, cends, ctx->crit_sad, ckey,
        cval, node));
    LAUNCH_CHECK("persistence_kernel");
  }
  // thresholded union-find roots
  int* uf = sget<int>(ctx, si, X_UF, M + 1);
  int* croot = sget<int>(ctx, si, X_CROOT, M + 1);
  LK(iota_kernel<<<grid_for(M + 1, TB), TB, 0, st>>>(uf, M + 1));
  if (nsad > 0)
    LK(ut_union_kernel<<<grid_for(nsad, TB), TB, 0, st>>>(cends, ncanc, M, uf, M + 2, ctx->status));
  LK(ut_flatten_kernel<<<grid_for((M + 1 + kUtBatch - 1) / kUtBatch, TB), TB, 0, st>>>(M + 1, uf, M + 2,
                                                                                       ctx->status));
  LK(ut_mark_kernel<<<grid_for(M + 1, TB), TB, 0, st>>>(M, uf, S.alive, croot));
  LAUNCH_CHECK("thresholded union-find");
  // batch-wide output rank of alive extrema
  int* alive_i = sget<int>(ctx, si, X_ALIVEI, M + 1);
  S.to_out_excl = sget<int>(ctx, si, X_TOOUTX, M + 1);
  S.to_out = sget<int>(ctx, si, X_TOOUT, M + 1);
  if (M > 0) {
    LK(u8_to_int_kernel<<<grid_for(M, TB), TB, 0, st>>>(S.alive, M, alive_i));
    excl_sum(ctx, alive_i, S.to_out_excl, M, st);
    LK(to_out_kernel<<<grid_for(M, TB), TB, 0, st>>>(M, S.alive, S.to_out_excl, S.to_out));
    LAUNCH_CHECK("to_out_kernel");
  }
  S.rout = sget<int>(ctx, si, X_ROUT, M + 1);
  if (M > 0) LK(root_out_kernel<<<grid_for(M, TB), TB, 0, st>>>(M, uf, croot, S.to_out, S.rout));
  LAUNCH_CHECK("root_out_kernel");
}

// Replay inputs of one side (batch); returns the replay kernel's arguments,
// with n_cancel == nullptr when the side has no cancellation to replay.
ReplayArgs replay_prepare(dmsc_b200_context* ctx, int si, Side& S, cudaStream_t st) {
  const int nsad = ctx->nsad, M = S.M;
  // cancellations (keys, saddles, count) as the persistence pass listed them
  unsigned long long* ckey = sget<unsigned long long>(ctx, si, X_CKEY, nsad);
  int* cval = sget<int>(ctx, si, X_CVAL, nsad);
  int* cnt = sget<int>(ctx, si, X_CNT, 8);

  ReplayState& R = S.R;
  R.node = sget<ReplayNode>(ctx, si, X_NODE, M + 1);
  ReplayArgs A{};
  A.n_cancel = S.C > 0 ? get<int>(ctx, S_NCANC, 4) + si : nullptr;
  A.key = ckey;
  A.cj = cval;
  A.dying = S.dying;
  A.arc = S.arc;
  A.alive = S.alive;
  A.crit_sad = ctx->crit_sad;
  A.S = R;
  A.max_steps = nsad + 1;
  A.act0 = sget<int>(ctx, si, X_ACT0, nsad);
  A.act1 = sget<int>(ctx, si, X_ACT1, nsad);
  A.cnt = cnt;
  A.wx = sget<int>(ctx, si, X_WX, 2 * (size_t)nsad);
  A.wa = sget<long long>(ctx, si, X_WA, 2 * (size_t)nsad);
  A.status = ctx->status;
  A.max_rounds = capped(nsad + 2, ctx->cap_replay_rounds);
  A.rounds = get<int>(ctx, S_STATS, 8) + 2 + si;
  A.timeline = get<unsigned long long>(ctx, S_TIMELINE, kTimelineSlots) + (4 + si) * kTimeline;
  return A;
}

// Final arcs of one side's survivors after the replay: lengths, chain roots
// and the side's geometry total (device, into *total).
void replay_final(dmsc_b200_context* ctx, int si, Side& S, long long* total, cudaStream_t st) {
  const int nsurv = ctx->nsurv;
  S.arc_len = sget<long long>(ctx, si, X_ALEN, 2 * (size_t)nsurv);
  S.arc_cl = sget<long long>(ctx, si, X_ACL, 2 * (size_t)nsurv);
  S.arc_root = sget<int>(ctx, si, X_AROOT, 2 * (size_t)nsurv);
  S.plen = sget<long long>(ctx, si, X_PLEN, nsurv);
  S.send = sget<long long>(ctx, si, X_SEND, nsurv);
  LK(final_arcs_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, ctx->surv_ic, ctx->I.dual, S.arcs_primal,
                                                           S.arcs_dual, S.sv_t, S.sv_len, S.alive, S.R, ctx->nsad + 1,
                                                           S.arc_len, S.arc_cl, S.arc_root, S.plen, ctx->status));
  incl_sum(ctx, S.plen, S.send, nsurv, st);
  LK(last_kernel<long long><<<1, 1, 0, st>>>(S.send, nsurv, total));
  LAUNCH_CHECK("final arcs");
}

// The driver's tensor-map encoder (through the runtime, so the library needs
// no link against the driver library); null when unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The TMA-staged persistent gradient of one H x W image (tile TY x 32, NT
// threads); false when it does not apply (rows not 16-byte multiples, an
// unaligned buffer, no encoder), and the caller runs the batch kernel.
// With a host source (`host_img`, pinned) the image is uploaded into `img`
// in kInBands bands of rows on in_st, and each band of tile rows is launched
// as soon as the rows its value windows read have arrived; with a host
// gradient destination (`host_grad`), each band's gradient rows are copied
// back as soon as the band is done, so the upload overlaps the downloads.
template <int TY, int NT>
bool launch_gradient_tma(dmsc_b200_context* ctx, int H, int W, bool dual, const float* img, int4* grad,
                         int* const* seg, uint8_t* flow, cudaStream_t st, const float* host_img,
                         int32_t* host_grad) {
  if (W % 4 != 0 || (reinterpret_cast<uintptr_t>(img) & 15u) != 0) return false;
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
  const cuuint64_t strides[1] = {(cuuint64_t)W * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)kTmaCols, (cuuint32_t)(TY + 3)};
  const cuuint32_t estr[2] = {1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(img), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  auto kernel = dual ? gradient_tma_kernel<true, TY, NT> : gradient_tma_kernel<false, TY, NT>;
  constexpr int kSmem = grad_tma_smem_bytes<TY>();
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
  int per = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, NT, kSmem));
  const int ntx = (W + 1 + kTileX - 1) / kTileX, nty = (H + 1 + TY - 1) / TY;
  const long long ntiles = (long long)ntx * nty;
  const long long resident = (long long)std::max(1, per) * ctx->num_sms;
  auto launch = [&](long long t0, long long t1) {  // tiles [t0, t1): whole tile rows
    const int grid = (int)std::min<long long>(t1 - t0, resident);
    LK((kernel<<<grid, NT, kSmem, st>>>(map, H, W, ntx, (int)t0, (int)t1, grad, flow, seg[0], seg[1], seg[2],
                                        ctx->fifo_lut, ctx->status)));
    LAUNCH_CHECK("gradient_tma_kernel");
  };
  if (!host_img) {
    launch(0, ntiles);
    if (host_grad && grad) copy_out_async(ctx, host_grad, grad, 16 * (size_t)(H + 1) * (W + 1), st);
    return true;
  }
  // the device buffer's earlier users on st come first
  CK(cudaEventRecord(ctx->in_ev[0], st));
  CK(cudaStreamWaitEvent(ctx->in_st, ctx->in_ev[0], 0));
  float* dimg = const_cast<float*>(img);
  const int nb = std::min(kInBands, nty);
  long long rows_in = 0;
  for (int k = 0; k < nb; ++k) {
    const long long r0 = (long long)nty * k / nb, r1 = (long long)nty * (k + 1) / nb;  // tile rows
    // a tile's value window reads image rows y0 - 2 .. y0 + TY (y0 = its
    // first index row); rows outside the image read as zero fill
    const long long need = std::min<long long>(H, r1 * TY + 1);
    if (need > rows_in)
      CK(cudaMemcpyAsync(dimg + rows_in * W, host_img + rows_in * W, (size_t)(need - rows_in) * W * sizeof(float),
                         cudaMemcpyHostToDevice, ctx->in_st));
    rows_in = std::max(rows_in, need);
    CK(cudaEventRecord(ctx->in_ev[k], ctx->in_st));
    CK(cudaStreamWaitEvent(st, ctx->in_ev[k], 0));
    launch(r0 * ntx, r1 * ntx);
    if (host_grad && grad) {  // the band's index rows r0 TY .. min(H + 1, r1 TY) - 1
      const long long i0 = r0 * TY, i1 = std::min<long long>(H + 1, r1 * TY);
      if (i1 > i0)
        copy_out_async(ctx, host_grad + i0 * (W + 1) * 4, grad + i0 * (W + 1), 16 * (size_t)(i1 - i0) * (W + 1), st);
    }
  }
  return true;
}

// Gradient kernel of tile shape `shape` over `ntile` tiles of the batch (a
// TMA shape on a one-image batch runs the persistent kernel when it applies),
// with the image's upload from `host_img` (one image; nullptr: the image is
// on the device); true when it also issued the gradient's copy to
// `host_grad` (the persistent kernel copies it band by band), false when
// the caller copies it after the kernel.
bool launch_gradient(dmsc_b200_context* ctx, int shape, unsigned ntile, const Imgs& I, const float* img, int4* grad,
                     uint8_t* mask, int* const* seg, uint8_t* flow, cudaStream_t st, int B, int H0, int W0,
                     bool dual0, const float* host_img, int32_t* host_grad) {
  if (kGradTma[shape] && B == 1 && !mask) {
    const bool done = shape == 3 ? launch_gradient_tma<kGradTY[3], kGradNT[3]>(ctx, H0, W0, dual0, img, grad, seg,
                                                                                flow, st, host_img, host_grad)
                                 : launch_gradient_tma<kGradTY[4], kGradNT[4]>(ctx, H0, W0, dual0, img, grad, seg,
                                                                                flow, st, host_img, host_grad);
    if (done) return true;
  }
  if (host_img)  // the whole image first
    CK(cudaMemcpyAsync(const_cast<float*>(img), host_img, (size_t)H0 * W0 * sizeof(float), cudaMemcpyHostToDevice,
                       st));
  switch (kGradTY[shape]) {
    case kGradTY[0]:
      LK((gradient_batch_kernel<kGradTY[0], kGradNT[0]><<<ntile, kGradNT[0], 0, st>>>(I, img, grad, mask, seg[0], seg[1],
                                                                                      seg[2], ctx->fifo_lut, flow)));
      break;
    case kGradTY[1]:
      LK((gradient_batch_kernel<kGradTY[1], kGradNT[1]><<<ntile, kGradNT[1], 0, st>>>(I, img, grad, mask, seg[0], seg[1],
                                                                                      seg[2], ctx->fifo_lut, flow)));
      break;
    default:
      LK((gradient_batch_kernel<kGradTY[2], kGradNT[2]><<<ntile, kGradNT[2], 0, st>>>(I, img, grad, mask, seg[0], seg[1],
                                                                                      seg[2], ctx->fifo_lut, flow)));
      break;
  }
  LAUNCH_CHECK("gradient_batch_kernel");
  return false;
}

// Number of bits needed for values 0 .. n-1 (at least 1).
int bits_for(int n) {
  int b = 1;
  while ((1LL << b) < n) ++b;
  return b;
}

void emit_expand(dmsc_b200_context* ctx, int si, Side& S, cudaStream_t st);

int extract_batch_impl(dmsc_b200_context* ctx, int B, const float* img, const int* hH, const int* hW,
                       const float* hthr, const unsigned char* hdual, unsigned flags, int32_t* grad_out,
                       int32_t* peaks_out, int32_t* basins_out, dmsc_b200_sizes* sizes_out, cudaStream_t st) {
  ctx->valid = false;
  const float* host_img = ctx->host_img;  // the registration covers this call only
  ctx->host_img = nullptr;
  if (host_img && B != 1) {
    set_err(ctx, "a host image source takes one image");
    return kErrInvalidArgument;
  }
  if (!img || B <= 0 || !hH || !hW || !hthr || !hdual || !sizes_out) {
    set_err(ctx, "invalid argument");
    return kErrInvalidArgument;
  }
  const bool ret_grad = flags & DMSC_B200_RETURN_GRADIENT;
  const bool f_ridges = flags & DMSC_B200_TRACE_RIDGES, f_valleys = flags & DMSC_B200_TRACE_VALLEYS;
  const bool f_peaks = flags & DMSC_B200_TRACE_PEAKS, f_basins = flags & DMSC_B200_TRACE_BASINS;
  if ((ret_grad && !grad_out) || (f_peaks && !peaks_out) || (f_basins && !basins_out)) {
    set_err(ctx, "missing output buffer for a requested field");
    return kErrInvalidArgument;
  }
  if (ret_grad && ((uintptr_t)grad_out & 15u)) {  // written with 16-byte stores
    set_err(ctx, "grad_out must be 16-byte aligned");
    return kErrInvalidArgument;
  }
  // per-image tables (host): 32-bit cell ids per image (input_validation.hxx:24-26) and for the batch
  std::vector<int> tab(9 * (size_t)(B + 1), 0);
  int* tH = tab.data();
  int* tW = tH + (B + 1);
  int* idx_base = tW + (B + 1);
  int* px_base = idx_base + (B + 1);
  int* tile_base = px_base + (B + 1);
  int* seg_base = tile_base + (B + 1);
  int* peaks_off = seg_base + (B + 1);
  int* basins_off = peaks_off + (B + 1);
  int* ltile_base = basins_off + (B + 1);
  const int gshape = ctx->grad_shape;
  const int gTY = kGradTY[gshape];
  long long nidx = 0, npx = 0, ntile = 0, nseg = 0, npk = 0, nbs = 0, nltile = 0;
  bool any_primal = false, any_dual = false;
  for (int b = 0; b < B; ++b) {
    const long long H = hH[b], W = hW[b];
    if (H <= 0 || W <= 0) {
      set_err(ctx, "image %d has an empty dimension", b);
      return kErrInvalidArgument;
    }
    if (H + 1 > 2147483647LL / 4 / (W + 1)) {
      set_err(ctx, "Input is too large for 32-bit cell IDs: %lldx%lld", H, W);
      return kErrTooLarge;
    }
    tH[b] = (int)H;
    tW[b] = (int)W;
    idx_base[b] = (int)nidx;
    px_base[b] = (int)npx;
    tile_base[b] = (int)ntile;
    seg_base[b] = (int)nseg;
    peaks_off[b] = (int)npk;
    basins_off[b] = (int)nbs;
    ltile_base[b] = (int)nltile;
    nltile += ((W + kLT) / kLT) * ((H + kLT) / kLT);
    const long long ntx = (W + 1 + kTileX - 1) / kTileX, nty = (H + 1 + gTY - 1) / gTY;
    nidx += (H + 1) * (W + 1);
    npx += H * W;
    ntile += ntx * nty;
    nseg += (H + 1) * ntx;
    npk += hdual[b] ? H * W : (H + 1) * (W + 1);
    nbs += hdual[b] ? (H + 1) * (W + 1) : H * W;
    (hdual[b] ? any_dual : any_primal) = true;
    if (4 * nidx > 2147483647LL || npx > 2147483647LL || npk > 2147483647LL || nbs > 2147483647LL) {
      set_err(ctx, "batch too large for 32-bit cell ids; split it");
      return kErrTooLarge;
    }
  }
  idx_base[B] = (int)nidx;
  px_base[B] = (int)npx;
  tile_base[B] = (int)ntile;
  seg_base[B] = (int)nseg;
  peaks_off[B] = (int)npk;
  basins_off[B] = (int)nbs;
  ltile_base[B] = (int)nltile;
  CK(cudaSetDevice(ctx->device));
  ctx->B = B;
  ctx->flags = flags;
  ctx->nidx = nidx;
  ctx->hH.assign(hH, hH + B);
  ctx->hW.assign(hW, hW + B);
  ctx->hdual.assign(hdual, hdual + B);
  ctx->status = get<unsigned>(ctx, S_STATUS, 4);
  ctx->launches = 0;
  join_copies(ctx, st);  // host copies of an earlier call still reading its outputs
  mark(ctx, 0, st);
  CK(cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), st));
  CK(cudaMemsetAsync(get<int>(ctx, S_STATS, 8), 0, 8 * sizeof(int), st));
  CK(cudaMemsetAsync(get<unsigned long long>(ctx, S_TIMELINE, kTimelineSlots), 0,
                     kTimelineSlots * sizeof(unsigned long long), st));
  {  // upload the tables: 9 int arrays, then thr (float) and dual (u8)
    size_t ib = tab.size() * sizeof(int), fb = (size_t)B * sizeof(float);
    size_t total = ib + fb + B + 16;
    char* h = (char*)staging(ctx, total);
    memcpy(h, tab.data(), ib);
    memcpy(h + ib, hthr, fb);
    memcpy(h + ib + fb, hdual, B);
    char* d = get<char>(ctx, S_TAB, total);
    CK(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, st));
    int* di = (int*)d;
    ctx->I.B = B;
    ctx->I.H = di;
    ctx->I.W = di + (B + 1);
    ctx->I.idx_base = di + 2 * (B + 1);
    ctx->I.px_base = di + 3 * (B + 1);
    ctx->I.tile_base = di + 4 * (B + 1);
    ctx->I.seg_base = di + 5 * (B + 1);
    ctx->I.ltile_base = di + 8 * (B + 1);
    ctx->I.thr = (const float*)(d + ib);
    ctx->I.dual = (const uint8_t*)(d + ib + fb);
  }
  const int* d_peaks_off = ctx->I.H + 6 * (B + 1);
  const int* d_basins_off = ctx->I.H + 7 * (B + 1);
  const Imgs I = ctx->I;
  const long long ncells = 4 * nidx;

  // ---- K1 gradient + criticality (all images, one grid) ----
  // the 16 B/index gradient is written only when returned; every later stage
  // works from the flow codes, which also carry the criticality bits
  int* grad = ret_grad ? grad_out : nullptr;
  uint8_t* flow = get<uint8_t>(ctx, S_FLOW, nidx);
  ctx->flow = flow;
  ctx->img = img;
  int* seg[3] = {get<int>(ctx, S_SEG0, nseg), get<int>(ctx, S_SEG1, nseg), get<int>(ctx, S_SEG2, nseg)};
  int* off[3] = {get<int>(ctx, S_OFF0, nseg), get<int>(ctx, S_OFF1, nseg), get<int>(ctx, S_OFF2, nseg)};
  mark(ctx, 15, st);  // the gradient stage times the kernel alone
  const bool grad_copied = launch_gradient(ctx, gshape, (unsigned)ntile, I, img, (int4*)grad, nullptr, seg, flow, st,
                                           B, hH[0], hW[0], hdual[0] != 0, host_img,
                                           ret_grad ? ctx->host_grad : nullptr);
  mark(ctx, 1, st);
  if (ret_grad && !grad_copied) copy_out_async(ctx, ctx->host_grad, grad, 16 * (size_t)nidx, st);
  for (int k = 0; k < 3; ++k) excl_sum(ctx, seg[k], off[k], (int)nseg, st);
  long long* tot = get<long long>(ctx, S_TOT, 8);
  LK(totals3_kernel<<<1, 1, 0, st>>>(off[0], seg[0], off[1], seg[1], off[2], seg[2], nseg, tot));
  LAUNCH_CHECK("totals3_kernel");
  readback(ctx, st, tot, 3);
  const int nmin = (int)rb_ll(ctx)[0], nsad = (int)rb_ll(ctx)[1], nmax = (int)rb_ll(ctx)[2];
  ctx->nmin = nmin;
  ctx->nsad = nsad;
  ctx->nmax = nmax;

  // ---- K2 ordered compaction ----
  int* csad = get<int>(ctx, S_CSAD, nsad);
  int* imin = get<int>(ctx, S_IMIN, nmin);
  int* isad = get<int>(ctx, S_ISAD, nsad);
  int* imax = get<int>(ctx, S_IMAX, nmax);
  uint32_t* bmin = get<uint32_t>(ctx, S_MINBITS, nseg);  // per-segment bit masks of the extrema
  uint32_t* bmax = get<uint32_t>(ctx, S_MAXBITS, nseg);
  int2* kmin = get<int2>(ctx, S_KMIN, nmin);  // (value bits, cell): the extremum lists
  int2* kmax = get<int2>(ctx, S_KMAX, nmax);
  float* sval = get<float>(ctx, S_SVAL, nsad);
  ctx->crit_sad = csad;
  ctx->sad_img = isad;
  // the pairing's starting state (side 0: faces / maxima, side 1: vertices /
  // minima), set up by the compaction and the saddle walks
  PairStart ps;
  ps.nsad = nsad;
  ps.sval = sval;
  for (int si = 0; si < 2; ++si) {
    const int M = si ? nmin : nmax;
    ps.M[si] = M;
    ps.minedge[si] = sget<unsigned long long>(ctx, si, X_MINE, M + 1);
    ps.link[si] = sget<int>(ctx, si, X_LINK, M + 1);
    ps.cnt[si] = sget<int>(ctx, si, X_CNT, 8);
    ps.g12[si] = sget<int2>(ctx, si, X_G12, nsad);
    ps.dying[si] = sget<int>(ctx, si, X_DYING, nsad);
  }
  LK(compact_kernel<<<grid_for(nseg, 8 * kCompactSegs), 256, 0, st>>>(
      I, img, nseg, flow, off[0], off[1], off[2], csad, imin, isad, imax, bmin, bmax, kmin, kmax, sval, ps));
  LAUNCH_CHECK("compact_kernel");
  // per-image bases of the critical lists (B + 1 entries each)
  int* bases = get<int>(ctx, S_BASES, 9 * (size_t)(B + 1));
  Bases& BS = ctx->bases;
  BS.min = bases;
  BS.sad = bases + (B + 1);
  BS.max = bases + 2 * (B + 1);
  BS.surv = bases + 3 * (B + 1);
  BS.alive[0] = bases + 4 * (B + 1);
  BS.alive[1] = bases + 5 * (B + 1);
  BS.erow[0] = bases + 6 * (B + 1);
  BS.erow[1] = bases + 7 * (B + 1);
  LK(image_base_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, I.seg_base, (int)nseg, off[0], nmin, BS.min));
  LK(image_base_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, I.seg_base, (int)nseg, off[1], nsad, BS.sad));
  LK(image_base_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, I.seg_base, (int)nseg, off[2], nmax, BS.max));
  LAUNCH_CHECK("image_base_kernel");
  mark(ctx, 2, st);

  // ---- K4 saddle walks ----
  // per saddle and side: arc ends and raw-arc lengths (cells)
  int4* arc_f = get<int4>(ctx, S_ARCF, nsad);
  int4* arc_v = get<int4>(ctx, S_ARCV, nsad);
  if (nsad > 0) {
    LK(saddle_walk_kernel<<<grid_for(nsad, TB), TB, 0, st>>>(I, flow, nsad, csad, isad, off[2], bmax, off[0], bmin,
                                                             arc_f, arc_v, ncells, ps, ctx->status));
    LAUNCH_CHECK("saddle_walk_kernel");
  }

  // ---- sides ----
  Side& F = ctx->side[0];
  Side& V = ctx->side[1];
  F = Side();
  V = Side();
  F.faces = true;
  V.faces = false;
  F.M = nmax;
  V.M = nmin;
  F.ext_img = imax;
  V.ext_img = imin;
  F.key = kmax;
  V.key = kmin;
  F.arc = arc_f;
  V.arc = arc_v;
  // faces: ridges/peaks in the primal, valleys/basins in the dual (workspace.hxx:322-362)
  F.arcs_primal = f_ridges;
  F.arcs_dual = f_valleys;
  V.arcs_primal = f_valleys;
  V.arcs_dual = f_ridges;
  F.groups_primal = f_peaks;
  F.groups_dual = f_basins;
  V.groups_primal = f_basins;
  V.groups_dual = f_peaks;
  for (Side* S : {&F, &V}) {
    S->arcs = (S->arcs_primal && any_primal) || (S->arcs_dual && any_dual);
    S->groups = (S->groups_primal && any_primal) || (S->groups_dual && any_dual);
  }

  uint8_t* canc = get<uint8_t>(ctx, S_CANC, nsad + 4);
  mark(ctx, 4, st);
  CK(cudaMemsetAsync(canc, 0, nsad + 4, st));
  run_pairing(ctx, st);
  mark(ctx, 5, st);
  // the two sides' persistence, thresholded union-find and ranks are
  // independent (disjoint buffers; their cancellation bits are ORed into the
  // shared byte map with atomics): the vertex side runs on side_st
  CK(cudaEventRecord(ctx->fork_ev, st));
  CK(cudaStreamWaitEvent(ctx->side_st, ctx->fork_ev, 0));
  finish_pairing(ctx, 0, F, st);
  finish_pairing(ctx, 1, V, ctx->side_st);
  CK(cudaEventRecord(ctx->join_ev, ctx->side_st));
  CK(cudaStreamWaitEvent(st, ctx->join_ev, 0));
  mark(ctx, 6, st);

  // ---- surviving saddles in minima-sweep (vertex side) order ----
  int* flag = get<int>(ctx, S_FLAG, nsad);
  int* fpos = get<int>(ctx, S_FPOS, nsad);
  ctx->surv = get<int>(ctx, S_SURV, nsad);
  ctx->nsurv = 0;
  if (nsad > 0) {
    LK(survivor_flag_kernel<<<grid_for(nsad, TB), TB, 0, st>>>(nsad, canc, flag));
    excl_sum(ctx, flag, fpos, nsad, st);
    LK(last_plus_kernel<int><<<1, 1, 0, st>>>(fpos, flag, nsad, tot));
    LK(copy2_kernel<<<1, 1, 0, st>>>(get<int>(ctx, S_NCANC, 4), tot + 1));
    LAUNCH_CHECK("survivors");
    // the status word rides along: a capped pairing or union-find loop ends
    // the call here, before the replay
    rb_reserve(ctx, 4 * sizeof(long long));
    rb_copy(ctx, st, 0, tot, 3 * sizeof(long long));
    rb_copy(ctx, st, 3 * sizeof(long long), ctx->status, sizeof(unsigned));
    wait_stream(ctx, st);
    raise_status(ctx, *(const unsigned*)(ctx->rb_h + 3 * sizeof(long long)));
    ctx->nsurv = (int)rb_ll(ctx)[0];
    F.C = (int)rb_ll(ctx)[1];
    V.C = (int)rb_ll(ctx)[2];
  }
  const int nsurv = ctx->nsurv;
  LK(image_base_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, BS.sad, nsad, fpos, nsurv, BS.surv));
  LAUNCH_CHECK("survivor bases");
  // the survivor order and records run on side_st, overlapping the replay
  // and the labels (neither reads them); the final arcs wait for them
  cudaStream_t ss = ctx->side_st;
  CK(cudaEventRecord(ctx->fork_ev, st));
  mark(ctx, 7, st);

  // ---- replay (both sides in one cooperative launch) ----
  {
    ReplayArgs2 RA{};
    bool any = false;
    for (int si = 0; si < 2; ++si) {
      Side& S = ctx->side[si];
      RA.s[si].status = ctx->status;
      if (S.arcs && nsad > 0) {
        RA.s[si] = replay_prepare(ctx, si, S, st);
        any = any || RA.s[si].n_cancel != nullptr;
      }
    }
    if (any)
      coop_launch(ctx, ctx->replay_shape ? replay_persistent_kernel<2, 3> : replay_persistent_kernel<1, 4>, RA, st,
                  "replay_persistent_kernel", ctx->replay_per_sm);
    mark(ctx, 8, st);
  }

  // the survivors' side-stream work is enqueued after the replay's launch,
  // so the device starts the replay while the host sets up the sort
  CK(cudaStreamWaitEvent(ss, ctx->fork_ev, 0));
  if (nsurv > 0) {
    // the survivors (list order) sorted by (image, s_val) with the list index
    // as the stable tie-break, then each image's range in its vertex-side
    // sweep direction (reversed for a dual image)
    int* sidx = get<int>(ctx, S_IOTA, nsurv);
    int* sorted = get<int>(ctx, S_ASC, nsurv);
    if (B > 1) {
      unsigned long long* k = get<unsigned long long>(ctx, S_SKEY2, nsurv);
      LK(survivor_gather_kernel<unsigned long long><<<grid_for(nsad, TB), TB, 0, ss>>>(
          nsad, flag, fpos, get<float>(ctx, S_SVAL, nsad), ctx->sad_img, k, sidx));
      sort_pairs(ctx, k, get<unsigned long long>(ctx, S_SKEYS, nsurv), sidx, sorted, nsurv, ss, 32 + bits_for(B));
    } else {
      uint32_t* k = get<uint32_t>(ctx, S_SKEY32B, nsurv);
      LK(survivor_gather_kernel<uint32_t><<<grid_for(nsad, TB), TB, 0, ss>>>(
          nsad, flag, fpos, get<float>(ctx, S_SVAL, nsad), ctx->sad_img, k, sidx));
      sort_pairs(ctx, k, get<uint32_t>(ctx, S_SKEYS, nsurv), sidx, sorted, nsurv, ss, 32);
    }
    // the survivors in output order, with their records gathered once
    ctx->surv_ic = get<int2>(ctx, S_SURVIC, nsurv);
    LK(survivor_order_kernel<<<grid_for(nsurv, TB), TB, 0, ss>>>(nsurv, sorted, ctx->sad_img, ctx->crit_sad, I.dual,
                                                               BS.surv, ctx->surv, ctx->surv_ic));
    LAUNCH_CHECK("survivor order");
    for (int si = 0; si < 2; ++si) {
      Side& S = ctx->side[si];
      S.sv_t = sget<int2>(ctx, si, X_SVT, nsurv);
      S.sv_len = sget<longlong2>(ctx, si, X_SVL, nsurv);
      S.sv_rec = sget<int4>(ctx, si, X_SVR, nsurv);
      LK(surv_side_kernel<<<grid_for(nsurv, TB), TB, 0, ss>>>(nsurv, ctx->surv, S.arc, S.pp,
                                                            S.rout, S.sv_t, S.sv_len, S.sv_rec));
    }
    LAUNCH_CHECK("survivor records");
  }
  CK(cudaEventRecord(ctx->join_ev, ss));

  // ---- labels (region id = rank among the image's alive extrema) ----
  LabelOut OF{}, OV{};
  LabelSide LF{}, LV{};
  for (int si = 0; si < 2; ++si) {
    Side& S = ctx->side[si];
    // alive bases first (needed by the labels and the outputs)
    long long* at = get<long long>(ctx, S_TOT, 8) + 4 + si;
    if (S.M > 0)
      LK(u8_last_plus_kernel<<<1, 1, 0, st>>>(S.to_out_excl, S.alive, S.M, at));
    else
      CK(cudaMemsetAsync(at, 0, sizeof(long long), st));
    LK(image_base_dev_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, S.faces ? BS.max : BS.min, S.M, S.to_out_excl,
                                                                   at, BS.alive[si]));
    LAUNCH_CHECK("alive bases");
    if (!S.groups) continue;
    LabelOut& O = S.faces ? OF : OV;
    if (S.faces) {
      O.primal = f_peaks ? peaks_out : nullptr;
      O.dual = f_basins ? basins_out : nullptr;
      O.primal_off = d_peaks_off;
      O.dual_off = d_basins_off;
    } else {
      O.primal = f_basins ? basins_out : nullptr;
      O.dual = f_peaks ? peaks_out : nullptr;
      O.primal_off = d_basins_off;
      O.dual_off = d_peaks_off;
    }
    LabelSide& L = S.faces ? LF : LV;
    L.off = S.faces ? off[2] : off[0];
    L.rout = S.rout;
    L.abase = BS.alive[si];
    L.perim = get<int>(ctx, S.faces ? S_PERF : S_PERV, (size_t)nltile * kPerim);
  }
  int* nex = get<int>(ctx, S_NEX, 2);
  CK(cudaMemsetAsync(nex, 0, 2 * sizeof(int), st));
  mark(ctx, 16, st);  // the labels stage times the label kernels alone
  if (F.groups || V.groups) {
    int2* exf = F.groups ? get<int2>(ctx, S_EXF, nidx) : nullptr;
    int2* exv = V.groups ? get<int2>(ctx, S_EXV, nidx) : nullptr;
    constexpr int kLSm = (int)sizeof(LabelSmem);
    if (!ctx->label_smem_set) {  // more than the 48 KB of static shared memory
      CK(cudaFuncSetAttribute(label_tile_kernel<kLabelNT[0]>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLSm));
      CK(cudaFuncSetAttribute(label_tile_kernel<kLabelNT[1]>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLSm));
      ctx->label_smem_set = true;
    }
    if (ctx->label_shape == 1)
      LK((label_tile_kernel<kLabelNT[1]><<<(unsigned)nltile, kLabelNT[1], kLSm, st>>>(I, flow, LF, LV, OF, OV, exf,
                                                                                    exv, nex, ctx->status)));
    else
      LK((label_tile_kernel<kLabelNT[0]><<<(unsigned)nltile, kLabelNT[0], kLSm, st>>>(I, flow, LF, LV, OF, OV, exf,
                                                                                    exv, nex, ctx->status)));
    LAUNCH_CHECK("label_tile_kernel");
    int per = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, label_exit_kernel<true>, 256, 0));
    const unsigned eg = (unsigned)std::max(1, per) * ctx->num_sms;
    if (F.groups) LK(label_exit_kernel<true><<<eg, 256, 0, st>>>(I, exf, nex + 0, LF.perim, OF, (int)nltile + 2, ctx->status));
    if (V.groups) LK(label_exit_kernel<false><<<eg, 256, 0, st>>>(I, exv, nex + 1, LV.perim, OV, (int)nltile + 2, ctx->status));
    LAUNCH_CHECK("label_exit_kernel");
  }
  mark(ctx, 10, st);
  if (f_peaks) copy_out_async(ctx, ctx->host_peaks, peaks_out, 4 * (size_t)npk, st);
  if (f_basins) copy_out_async(ctx, ctx->host_basins, basins_out, 4 * (size_t)nbs, st);
  ctx->host_grad = ctx->host_peaks = ctx->host_basins = nullptr;  // one extract only

  // ---- final arc lengths (after the survivor records on side_st) ----
  CK(cudaStreamWaitEvent(st, ctx->join_ev, 0));
  {
    // geometry totals stay on the device (read back with the sizes)
    long long* tot = get<long long>(ctx, S_TOT, 8);
    CK(cudaMemsetAsync(tot, 0, 2 * sizeof(long long), st));
    for (int si = 0; si < 2; ++si) {
      Side& S = ctx->side[si];
      S.gbase = sget<long long>(ctx, si, X_GBASE, B + 1);
      S.total = 0;
      if (S.arcs && nsad > 0) {
        if (nsurv > 0) replay_final(ctx, si, S, tot + si, st);
        LK(geom_base_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, BS.surv, nsurv, S.send, S.plen, tot + si,
                                                                  S.gbase));
        LAUNCH_CHECK("geom_base_kernel");
      } else {
        CK(cudaMemsetAsync(S.gbase, 0, (B + 1) * sizeof(long long), st));
      }
    }
    mark(ctx, 9, st);
  }

  // ---- e rows ----
  for (int si = 0; si < 2; ++si) {
    Side& S = ctx->side[si];
    int* ec = sget<int>(ctx, si, X_EROWC, nsurv);
    S.erow_off = sget<int>(ctx, si, X_EROWO, nsurv);
    long long* et = get<long long>(ctx, S_TOT, 8) + 6 + si;
    if (nsurv > 0) {
      LK(erow_count_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, S.faces, BS.surv, B, S.sv_rec, ec));
      excl_sum(ctx, ec, S.erow_off, nsurv, st);
      LK(last_plus_kernel<int><<<1, 1, 0, st>>>(S.erow_off, ec, nsurv, et));
    } else {
      CK(cudaMemsetAsync(et, 0, sizeof(long long), st));
    }
    LK(image_base_dev_kernel<<<grid_for(B + 1LL, TB), TB, 0, st>>>(B, BS.surv, nsurv, S.erow_off, et, BS.erow[si]));
    LAUNCH_CHECK("e rows");
  }

  // ---- per-image sizes: one read of the bases ----
  {
    // int bases, then (8-byte aligned) the two geometry bases, then the status word
    size_t ib = (9 * (size_t)(B + 1) * sizeof(int) + 7) & ~(size_t)7, lb = 2 * (size_t)(B + 1) * sizeof(long long);
    rb_reserve(ctx, ib + lb + 64);
    rb_copy(ctx, st, 0, bases, 9 * (size_t)(B + 1) * sizeof(int));
    rb_copy(ctx, st, ib, F.gbase, (B + 1) * sizeof(long long));
    rb_copy(ctx, st, ib + (B + 1) * sizeof(long long), V.gbase, (B + 1) * sizeof(long long));
    rb_copy(ctx, st, ib + lb, ctx->status, sizeof(unsigned));
    wait_stream(ctx, st);
    mark(ctx, 11, st);
    const char* h = ctx->rb_h;
    raise_status(ctx, *(const unsigned*)(h + ib + lb));
    const int* hb = (const int*)h;
    const int* hsurv = hb + 3 * (B + 1);
    const int* hal[2] = {hb + 4 * (B + 1), hb + 5 * (B + 1)};
    const int* her[2] = {hb + 6 * (B + 1), hb + 7 * (B + 1)};
    const long long* hg[2] = {(const long long*)(h + ib), (const long long*)(h + ib) + (B + 1)};
    for (int si = 0; si < 2; ++si) {
      ctx->side[si].total = hg[si][B];
      if (hg[si][B] > 2147483647LL) {
        set_err(ctx, "arc geometry of %lld cells exceeds int32 offsets", hg[si][B]);
        throw Fail{kErrOverflow};
      }
    }
    ctx->sizes.assign(B, dmsc_b200_sizes{});
    ctx->geom[0].assign(B, 0);
    ctx->geom[1].assign(B, 0);
    for (int b = 0; b < B; ++b) {
      const bool dual = hdual[b];
      const int PX = dual ? 1 : 0, PN = dual ? 0 : 1;  // public max / min side
      const long long ns = hsurv[b + 1] - hsurv[b];
      const long long H = hH[b], W = hW[b];
      for (int si = 0; si < 2; ++si) ctx->geom[si][b] = hg[si][b + 1] - hg[si][b];
      dmsc_b200_sizes z{};
      z.max_pts = hal[PX][b + 1] - hal[PX][b];
      z.min_pts = hal[PN][b + 1] - hal[PN][b];
      z.sad_pts = ns;
      z.e_max_rows = her[PX][b + 1] - her[PX][b];
      z.e_min_rows = her[PN][b + 1] - her[PN][b];
      z.p_max = z.p_min = z.ppairs_max = z.ppairs_min = ns;
      z.grad_indices = ret_grad ? 4 * (H + 1) * (W + 1) : 0;
      z.peaks_h = f_peaks ? (dual ? H : H + 1) : 0;
      z.peaks_w = f_peaks ? (dual ? W : W + 1) : 0;
      z.basins_h = f_basins ? (dual ? H + 1 : H) : 0;
      z.basins_w = f_basins ? (dual ? W + 1 : W) : 0;
      z.ridges = f_ridges ? ctx->geom[PX][b] : 0;
      z.ridge_offsets = f_ridges ? ns + 1 : 0;
      z.ridge_arc_offsets = f_ridges ? ns : 0;
      z.valleys = f_valleys ? ctx->geom[PN][b] : 0;
      z.valley_offsets = f_valleys ? ns + 1 : 0;
      z.valley_arc_offsets = f_valleys ? ns : 0;
      ctx->sizes[b] = z;
      sizes_out[b] = z;
    }
  }
  // the geometry's chain expansion needs no output buffer: it runs now,
  // while the caller allocates the outputs of the fetch
  mark(ctx, 17, st);
  for (int si = 0; si < 2; ++si) emit_expand(ctx, si, ctx->side[si], st);
  mark(ctx, 18, st);
  ctx->valid = true;
  return kOk;
}

// Geometry of one side, first half (end of extract, before the caller has
// allocated the outputs): the arcs' image-local positions and the
// breadth-first chain expansion into the segment list. The writer runs in
// fetch (emit_write); the device runs this while the host allocates.
void emit_expand(dmsc_b200_context* ctx, int si, Side& S, cudaStream_t st) {
  const int nsurv = ctx->nsurv;
  ctx->expanded[si] = false;
  if (!S.arcs || S.total <= 0 || nsurv <= 0) return;
  long long* arc_pos = sget<long long>(ctx, si, X_APOS, 2 * (size_t)nsurv);
  LK(arc_pos_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, S.arc_len, S.send, ctx->surv_ic, S.gbase, arc_pos));
  LAUNCH_CHECK("arc_pos_kernel");
  const long long cap = S.total;
  EmitArgs& A = ctx->emit[si];
  A = EmitArgs{};
  EmitCtx& E = A.E;
  E.flow = ctx->flow;
  E.I = ctx->I;
  E.faces = S.faces;
  E.S = S.R;
  E.q_cap = cap;
  E.max_steps = ctx->nsad + 1;
  E.status = ctx->status;
  A.nsurv = nsurv;
  E.nvirt = 2 * nsurv;
  E.surv_ic = ctx->surv_ic;
  E.sv_t = S.sv_t;
  E.sv_len = S.sv_len;
  E.arc_pos = arc_pos;
  A.arc_cl = S.arc_cl;
  A.arc_root = S.arc_root;
  A.q0 = sget<int4>(ctx, si, X_Q0, cap);
  A.q1 = sget<int4>(ctx, si, X_Q1, cap);
  A.cnt = sget<int>(ctx, si, X_CNT, 8);
  E.base_q = sget<int4>(ctx, si, X_QB, cap);
  E.base_cap = cap;
  A.max_levels = capped(ctx->nsad + 4, ctx->cap_emit_levels);
  A.levels = get<int>(ctx, S_STATS, 8) + 4 + si;
  A.timeline = get<unsigned long long>(ctx, S_TIMELINE, kTimelineSlots) + (2 + si) * kTimeline;
  coop_launch(ctx, ctx->emit_shape ? emit_persistent_kernel<2, 3> : emit_persistent_kernel<1, 5>, A, st,
              "emit_persistent_kernel", ctx->emit_per_sm);
  ctx->expanded[si] = true;
}

// Geometry of one side, second half (fetch): the CSR offsets and the writer
// of every raw-arc segment into the caller's arrays (`dst_off[b]`: image b's
// start in its destination).
void emit_write(dmsc_b200_context* ctx, int si, Side& S, int32_t* flat_primal, int32_t* flat_dual, const int* dst_off,
                Route OFF, Route AOFF, cudaStream_t st) {
  const int nsurv = ctx->nsurv, B = ctx->B;
  LK(arc_offsets_kernel<<<grid_for(nsurv + (long long)B, TB), TB, 0, st>>>(nsurv, B, ctx->bases.surv, ctx->I.dual,
                                                                           S.arc_len, S.send, S.gbase, OFF, AOFF));
  LAUNCH_CHECK("arc_offsets_kernel");
  if (!ctx->expanded[si] || (!flat_primal && !flat_dual)) return;
  EmitArgs& A = ctx->emit[si];
  EmitCtx E = A.E;
  E.out_primal = flat_primal;
  E.out_dual = flat_dual;
  E.dst_off = dst_off;
  int per = 0;
  if (ctx->seg_cursors == 1) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, emit_segments_kernel<1>, 256, 0));
    LK(emit_segments_kernel<1><<<dim3(per * ctx->num_sms * 4), 256, 0, st>>>(E, A.cnt + 3));
  } else {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, emit_segments_kernel<2>, 256, 0));
    LK(emit_segments_kernel<2><<<dim3(per * ctx->num_sms * 4), 256, 0, st>>>(E, A.cnt + 3));
  }
  LAUNCH_CHECK("emit_segments_kernel");
}

int fetch_batch_impl(dmsc_b200_context* ctx, const dmsc_b200_outputs* o, cudaStream_t st) {
  if (!ctx->valid || !o) {
    set_err(ctx, "fetch without a successful extract");
    return kErrInvalidArgument;
  }
  CK(cudaSetDevice(ctx->device));
  mark(ctx, 12, st);
  const int B = ctx->B, nsurv = ctx->nsurv;
  const Imgs I = ctx->I;
  // per-image offsets of every output, and their per-side routes
  enum { R_PTS0, R_PTS1, R_E0, R_E1, R_G0, R_G1, R_OFF0, R_OFF1, R_AOFF0, R_AOFF1, R_N };
  std::vector<int> route((size_t)R_N * B);
  {
    long long mx = 0, mn = 0, ex = 0, en = 0, rg = 0, vl = 0, ro = 0, vo = 0, ra = 0, va = 0;
    for (int b = 0; b < B; ++b) {
      const dmsc_b200_sizes& z = ctx->sizes[b];
      const bool d = ctx->hdual[b];
      // side 0 (faces) is the public max side in the primal, min side in the dual
      route[R_PTS0 * B + b] = (int)(d ? mn : mx);
      route[R_PTS1 * B + b] = (int)(d ? mx : mn);
      route[R_E0 * B + b] = (int)(2 * (d ? en : ex));
      route[R_E1 * B + b] = (int)(2 * (d ? ex : en));
      route[R_G0 * B + b] = (int)(d ? vl : rg);
      route[R_G1 * B + b] = (int)(d ? rg : vl);
      route[R_OFF0 * B + b] = (int)(d ? vo : ro);
      route[R_OFF1 * B + b] = (int)(d ? ro : vo);
      route[R_AOFF0 * B + b] = (int)(d ? va : ra);
      route[R_AOFF1 * B + b] = (int)(d ? ra : va);
      mx += z.max_pts;
      mn += z.min_pts;
      ex += z.e_max_rows;
      en += z.e_min_rows;
      rg += z.ridges;
      vl += z.valleys;
      ro += z.ridge_offsets;
      vo += z.valley_offsets;
      ra += z.ridge_arc_offsets;
      va += z.valley_arc_offsets;
    }
    size_t bytes = route.size() * sizeof(int);
    void* h = staging(ctx, bytes);
    memcpy(h, route.data(), bytes);
    int* d = get<int>(ctx, S_ROUTE, route.size());
    CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
  }
  const int* rt = (const int*)ctx->bufs[S_ROUTE].p;
  auto rt_of = [&](int k) { return rt + (size_t)k * B; };
  // extrema lists
  for (int si = 0; si < 2; ++si) {
    Side& S = ctx->side[si];
    Route R{S.faces ? o->max_pts : o->min_pts, S.faces ? o->min_pts : o->max_pts, rt_of(si == 0 ? R_PTS0 : R_PTS1)};
    if (S.M > 0)
      LK(points_kernel<<<grid_for(S.M, TB), TB, 0, st>>>(S.M, S.alive, S.to_out_excl, ctx->bases.alive[si], S.key,
                                                         S.ext_img, I, R));
  }
  if (nsurv > 0 && o->sad_pts)
    LK(sad_pts_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, ctx->surv_ic, ctx->bases.surv, I, o->sad_pts,
                                                          ctx->bases.surv));
  LAUNCH_CHECK("point lists");
  // per-saddle scalars and e rows
  if (nsurv > 0) {
    for (int si = 0; si < 2; ++si) {
      Side& S = ctx->side[si];
      RouteF P{S.faces ? o->p_max : o->p_min, S.faces ? o->p_min : o->p_max, ctx->bases.surv};
      Route PP{S.faces ? o->ppairs_max : o->ppairs_min, S.faces ? o->ppairs_min : o->ppairs_max, ctx->bases.surv};
      Route E{S.faces ? o->e_max : o->e_min, S.faces ? o->e_min : o->e_max, rt_of(si == 0 ? R_E0 : R_E1)};
      LK(side_outputs_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, S.faces, ctx->bases.surv, I, S.sv_rec,
                                                                 ctx->bases.alive[si], S.erow_off,
                                                                 ctx->bases.erow[si], P, PP, E));
    }
    LAUNCH_CHECK("side_outputs_kernel");
  }
  mark(ctx, 13, st);
  // per-field totals over the batch (elements)
  long long tot_n[15] = {0};
  for (int b = 0; b < B; ++b) {
    const dmsc_b200_sizes& z = ctx->sizes[b];
    const long long v[15] = {z.max_pts, z.min_pts, z.sad_pts, 2 * z.e_max_rows, 2 * z.e_min_rows, z.p_max, z.p_min,
                             z.ppairs_max, z.ppairs_min, z.ridges, z.ridge_offsets, z.ridge_arc_offsets, z.valleys,
                             z.valley_offsets, z.valley_arc_offsets};
    for (int k = 0; k < 15; ++k) tot_n[k] += v[k];
  }
  const dmsc_b200_outputs& HO = ctx->host_fetch;
  void* const dev_f[15] = {o->max_pts, o->min_pts, o->sad_pts, o->e_max, o->e_min, o->p_max, o->p_min,
                           o->ppairs_max, o->ppairs_min, o->ridges, o->ridge_offsets, o->ridge_arc_offsets,
                           o->valleys, o->valley_offsets, o->valley_arc_offsets};
  void* const host_f[15] = {HO.max_pts, HO.min_pts, HO.sad_pts, HO.e_max, HO.e_min, HO.p_max, HO.p_min,
                            HO.ppairs_max, HO.ppairs_min, HO.ridges, HO.ridge_offsets, HO.ridge_arc_offsets,
                            HO.valleys, HO.valley_offsets, HO.valley_arc_offsets};
  if (ctx->host_fetch_set)  // lists and per-saddle outputs are final: copy them while the geometry is built
    for (int k = 0; k < 9; ++k) copy_out_async(ctx, host_f[k], dev_f[k], 4 * (size_t)tot_n[k], st);
  // arc geometry
  for (int si = 0; si < 2; ++si) {
    Side& S = ctx->side[si];
    if (!S.arcs) continue;
    // faces: ridges in the primal, valleys in the dual
    int32_t* gp = S.faces ? o->ridges : o->valleys;
    int32_t* gd = S.faces ? o->valleys : o->ridges;
    Route OFF{S.faces ? o->ridge_offsets : o->valley_offsets, S.faces ? o->valley_offsets : o->ridge_offsets,
              rt_of(si == 0 ? R_OFF0 : R_OFF1)};
    Route AOFF{S.faces ? o->ridge_arc_offsets : o->valley_arc_offsets,
               S.faces ? o->valley_arc_offsets : o->ridge_arc_offsets, rt_of(si == 0 ? R_AOFF0 : R_AOFF1)};
    if (!S.arcs_primal) {
      gp = nullptr;
      OFF.primal = nullptr;
      AOFF.primal = nullptr;
    }
    if (!S.arcs_dual) {
      gd = nullptr;
      OFF.dual = nullptr;
      AOFF.dual = nullptr;
    }
    emit_write(ctx, si, S, gp, gd, rt_of(si == 0 ? R_G0 : R_G1), OFF, AOFF, st);
  }
  mark(ctx, 14, st);
  if (ctx->host_fetch_set)
    for (int k = 9; k < 15; ++k) copy_out_async(ctx, host_f[k], dev_f[k], 4 * (size_t)tot_n[k], st);
  ctx->host_fetch_set = false;  // one fetch only
  check_status(ctx, st);
  join_copies(ctx, st);  // the caller's stream passes here only once the host copies are done
  return kOk;
}

// Pixel pairs of the surviving saddles of the last extract (pairs.cuh).
int fetch_pair_pixels_impl(dmsc_b200_context* ctx, int32_t* plus_max, int32_t* minus_max, int32_t* plus_min,
                           int32_t* minus_min, cudaStream_t st) {
  if (!ctx->valid) {
    set_err(ctx, "fetch_pair_pixels without a successful extract");
    return kErrInvalidArgument;
  }
  CK(cudaSetDevice(ctx->device));
  const int nsurv = ctx->nsurv;
  if (nsurv == 0) return kOk;
  for (int si = 0; si < 2; ++si) {
    Side& S = ctx->side[si];
    // faces: the max side in the primal, the min side in the dual
    Route PLUS{S.faces ? plus_max : plus_min, S.faces ? plus_min : plus_max, ctx->bases.surv};
    Route MINUS{S.faces ? minus_max : minus_min, S.faces ? minus_min : minus_max, ctx->bases.surv};
    LK(pair_pixels_kernel<<<grid_for(nsurv, TB), TB, 0, st>>>(nsurv, S.faces, ctx->bases.surv, ctx->I, ctx->img,
                                                              ctx->surv, ctx->crit_sad, S.pp, S.key, PLUS,
                                                              MINUS));
  }
  LAUNCH_CHECK("pair_pixels_kernel");
  return kOk;
}

// grad_img[0, npx) = deterministic scatter of +-grad[i] onto (plus[i], minus[i]).
int scatter_pair_grads_impl(dmsc_b200_context* ctx, const int32_t* plus, const int32_t* minus, const float* grad,
                            long long n, float* grad_img, long long npx, cudaStream_t st) {
  if (n < 0 || npx < 0 || (n > 0 && (!plus || !minus || !grad)) || (npx > 0 && !grad_img)) {
    set_err(ctx, "invalid argument");
    return kErrInvalidArgument;
  }
  if (npx >= 2147483647LL || 2 * n >= 2147483647LL) {
    set_err(ctx, "scatter of %lld pairs onto %lld pixels exceeds int32 indexing", n, npx);
    return kErrTooLarge;
  }
  CK(cudaSetDevice(ctx->device));
  if (npx > 0) CK(cudaMemsetAsync(grad_img, 0, npx * sizeof(float), st));
  if (n == 0 || npx == 0) return kOk;
  const int m = (int)(2 * n);
  int* key = get<int>(ctx, S_BKEY, m);
  int* idx = get<int>(ctx, S_BIDX, m);
  int* key2 = get<int>(ctx, S_BKEY2, m);
  int* idx2 = get<int>(ctx, S_BIDX2, m);
  LK(pair_entries_kernel<<<grid_for(m, TB), TB, 0, st>>>(n, plus, minus, (int)npx, key, idx));
  LAUNCH_CHECK("pair_entries_kernel");
  sort_pairs(ctx, key, key2, idx, idx2, m, st, bits_for((int)npx + 1));
  LK(pair_segments_kernel<<<grid_for(m, TB), TB, 0, st>>>(m, key2, idx2, grad, (int)npx, grad_img));
  LAUNCH_CHECK("pair_segments_kernel");
  return kOk;
}

}  // namespace


extern "C" {

int dmsc_b200_create(dmsc_b200_context** out, int device) {
  if (!out) return kErrInvalidArgument;
  *out = nullptr;
  auto* c = new (std::nothrow) dmsc_b200_context();
  if (!c) return kErrInternal;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaMallocHost(&c->pinned, 64 * sizeof(long long)) != cudaSuccess) {
    delete c;
    return kErrCuda;
  }
  c->pinned_cap = 64 * sizeof(long long);
  if (cudaEventCreateWithFlags(&c->sync_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy_st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->side_st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->in_st, cudaStreamNonBlocking) != cudaSuccess) {
    dmsc_b200_destroy(c);
    return kErrCuda;
  }
  for (int k = 0; k < kInBands; ++k)
    if (cudaEventCreateWithFlags(&c->in_ev[k], cudaEventDisableTiming) != cudaSuccess) {
      dmsc_b200_destroy(c);
      return kErrCuda;
    }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  {
    std::vector<uint32_t> lut(kGradTable);
    gradient_tables(lut.data());
    // the copy from pageable memory may return before the table has reached
    // the device and orders only the legacy default stream: wait for it once
    // here, so calls on any (non-blocking) stream see the whole table
    if (cudaMalloc(&c->fifo_lut, kGradTable * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemcpy(c->fifo_lut, lut.data(), kGradTable * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
      dmsc_b200_destroy(c);
      return kErrCuda;
    }
  }
  *out = c;
  return kOk;
}

void dmsc_b200_destroy(dmsc_b200_context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  for (auto& b : c->bufs)
    if (b.p) cudaFree(b.p);
  if (c->cub_tmp.p) cudaFree(c->cub_tmp.p);
  if (c->cub_tmp_side.p) cudaFree(c->cub_tmp_side.p);
  if (c->side_st) {
    cudaStreamSynchronize(c->side_st);
    cudaStreamDestroy(c->side_st);
  }
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  if (c->fifo_lut) cudaFree(c->fifo_lut);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->rb_h) cudaFreeHost(c->rb_h);
  if (c->sync_ev) cudaEventDestroy(c->sync_ev);
  if (c->copy_st) {
    cudaStreamSynchronize(c->copy_st);
    cudaStreamDestroy(c->copy_st);
  }
  if (c->copy_ev) cudaEventDestroy(c->copy_ev);
  if (c->in_st) {
    cudaStreamSynchronize(c->in_st);
    cudaStreamDestroy(c->in_st);
  }
  for (int k = 0; k < kInBands; ++k)
    if (c->in_ev[k]) cudaEventDestroy(c->in_ev[k]);
  for (int k = 0; k < kStageMarks; ++k)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  delete c;
}

int dmsc_b200_extract(dmsc_b200_context* ctx, const float* image, int H, int W, float thr, unsigned flags,
                      int32_t* grad_out, int32_t* peaks_out, int32_t* basins_out, dmsc_b200_sizes* sizes,
                      void* stream) {
  if (!ctx) return kErrInvalidArgument;
  ctx->err.clear();
  try {
    const unsigned char dual = (flags & DMSC_B200_DUAL) ? 1 : 0;
    return extract_batch_impl(ctx, 1, image, &H, &W, &thr, &dual, flags, grad_out, peaks_out, basins_out, sizes,
                              (cudaStream_t)stream);
  } catch (const Fail& f) {
    ctx->valid = false;
    abandon_copies(ctx);
    return f.code;
  }
}

int dmsc_b200_fetch(dmsc_b200_context* ctx, const dmsc_b200_outputs* out, void* stream) {
  if (!ctx) return kErrInvalidArgument;
  ctx->err.clear();
  try {
    return fetch_batch_impl(ctx, out, (cudaStream_t)stream);
  } catch (const Fail& f) {
    abandon_copies(ctx);
    return f.code;
  }
}

int dmsc_b200_set_host_fetch_outputs(dmsc_b200_context* ctx, const dmsc_b200_outputs* host) {
  if (!ctx) return kErrInvalidArgument;
  ctx->host_fetch_set = host != nullptr;
  if (host) ctx->host_fetch = *host;
  return kOk;
}

int dmsc_b200_set_host_input(dmsc_b200_context* ctx, const float* host_image) {
  if (!ctx) return kErrInvalidArgument;
  ctx->host_img = host_image;
  return kOk;
}

int dmsc_b200_set_host_outputs(dmsc_b200_context* ctx, int32_t* grad_host, int32_t* peaks_host,
                               int32_t* basins_host) {
  if (!ctx) return kErrInvalidArgument;
  ctx->host_grad = grad_host;
  ctx->host_peaks = peaks_host;
  ctx->host_basins = basins_host;
  return kOk;
}

int dmsc_b200_extract_batch(dmsc_b200_context* ctx, const float* images, int B, const int* H, const int* W,
                            const float* thresholds, const unsigned char* is_dual, unsigned flags, int32_t* grad_out,
                            int32_t* peaks_out, int32_t* basins_out, dmsc_b200_sizes* sizes, void* stream) {
  if (!ctx) return kErrInvalidArgument;
  ctx->err.clear();
  if (ctx->host_img) {  // a host image source covers one single-image extract only
    ctx->host_img = nullptr;
    set_err(ctx, "dmsc_b200_set_host_input applies to dmsc_b200_extract only");
    return kErrInvalidArgument;
  }
  try {
    return extract_batch_impl(ctx, B, images, H, W, thresholds, is_dual, flags, grad_out, peaks_out, basins_out,
                              sizes, (cudaStream_t)stream);
  } catch (const Fail& f) {
    ctx->valid = false;
    abandon_copies(ctx);
    return f.code;
  }
}

int dmsc_b200_fetch_pair_pixels(dmsc_b200_context* ctx, int32_t* plus_max, int32_t* minus_max, int32_t* plus_min,
                                int32_t* minus_min, void* stream) {
  if (!ctx) return kErrInvalidArgument;
  ctx->err.clear();
  try {
    return fetch_pair_pixels_impl(ctx, plus_max, minus_max, plus_min, minus_min, (cudaStream_t)stream);
  } catch (const Fail& f) {
    return f.code;
  }
}

int dmsc_b200_scatter_pair_grads(dmsc_b200_context* ctx, const int32_t* plus, const int32_t* minus, const float* grad,
                                 int64_t n, float* grad_img, int64_t npx, void* stream) {
  if (!ctx) return kErrInvalidArgument;
  ctx->err.clear();
  try {
    return scatter_pair_grads_impl(ctx, plus, minus, grad, n, grad_img, npx, (cudaStream_t)stream);
  } catch (const Fail& f) {
    return f.code;
  }
}

const char* dmsc_b200_error_string(int code) {
  switch (code) {
    case kOk: return "ok";
    case kErrInvalidArgument: return "invalid argument";
    case kErrTooLarge: return "input is too large for 32-bit cell ids";
    case kErrCuda: return "CUDA runtime error";
    case kErrIterationCap: return "bounded device loop reached its cap";
    case kErrOverflow: return "output or work queue overflow";
    default: return "internal error";
  }
}

const char* dmsc_b200_last_error(const dmsc_b200_context* ctx) { return ctx ? ctx->err.c_str() : ""; }

int dmsc_b200_set_profiling(dmsc_b200_context* ctx, int enable) {
  if (!ctx) return kErrInvalidArgument;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return kErrCuda;
  if (enable && !ctx->ev[0]) {
    for (int k = 0; k < kStageMarks; ++k)
      if (cudaEventCreate(&ctx->ev[k]) != cudaSuccess) return kErrCuda;
  }
  ctx->profile = enable != 0;
  return kOk;
}

int dmsc_b200_stage_times(dmsc_b200_context* ctx, float* ms, int n) {
  if (!ctx || !ms || !ctx->profile) return -1;
  // extract stages are marks 0, 15, 1, 2, 4..8, 16, 10, 9, 11 in stream
  // order (15: just before the gradient kernel, 16: just before the label
  // kernels; the labels run before the final arcs; mark 3 is not recorded),
  // fetch stages 12..14; the geometry stage adds the expansion at the end of
  // extract (marks 17, 18) to the writer in fetch (13, 14)
  static const int from[] = {0, 15, 1, 2, 4, 5, 6, 7, 10, 8, 16, 9, 12, 13};
  static const int to[] = {15, 1, 2, 4, 5, 6, 7, 8, 9, 16, 10, 11, 13, 14};
  const int ns = (int)(sizeof(from) / sizeof(from[0]));
  if (cudaEventSynchronize(ctx->ev[14]) != cudaSuccess) return -1;
  for (int k = 0; k < ns && k < n; ++k) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ctx->ev[from[k]], ctx->ev[to[k]]) != cudaSuccess) t = -1.f;
    if (k == ns - 1 && t >= 0.f) {
      float e = 0.f;
      if (cudaEventElapsedTime(&e, ctx->ev[17], ctx->ev[18]) == cudaSuccess) t += e;
    }
    ms[k] = t;
  }
  return ns;
}

long long dmsc_b200_launch_count(const dmsc_b200_context* ctx) { return ctx ? ctx->launches : -1; }

int dmsc_b200_pairing_timeline(dmsc_b200_context* ctx, long long* out, int n) {
  if (!ctx || !out || ctx->bufs.size() <= (size_t)S_TIMELINE || !ctx->bufs[S_TIMELINE].p) return -1;
  int k = n < kTimelineSlots ? n : kTimelineSlots;
  if (cudaSetDevice(ctx->device) != cudaSuccess ||
      cudaMemcpy(out, ctx->bufs[S_TIMELINE].p, k * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return k;
}

int dmsc_b200_loop_counts(dmsc_b200_context* ctx, int* out, int n) {
  if (!ctx || !out || ctx->bufs.size() <= (size_t)S_STATS || !ctx->bufs[S_STATS].p) return -1;
  int h[6] = {0};
  if (cudaSetDevice(ctx->device) != cudaSuccess ||
      cudaMemcpy(h, ctx->bufs[S_STATS].p, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  for (int k = 0; k < 6 && k < n; ++k) out[k] = h[k];
  return 6;
}

int dmsc_b200_set_loop_caps(dmsc_b200_context* ctx, int pair_rounds, int replay_rounds, int emit_levels) {
  if (!ctx || pair_rounds < 0 || replay_rounds < 0 || emit_levels < 0) return kErrInvalidArgument;
  ctx->cap_pair_rounds = pair_rounds;
  ctx->cap_replay_rounds = replay_rounds;
  ctx->cap_emit_levels = emit_levels;
  return kOk;
}

int dmsc_b200_set_tuning(dmsc_b200_context* ctx, const dmsc_b200_tuning* t) {
  if (!ctx || !t || t->grad_shape < 0 || t->grad_shape >= kGradShapes || t->label_shape < 0 ||
      t->label_shape >= kLabelShapes || t->pair_blocks_per_sm < 0 || t->replay_blocks_per_sm < 0 ||
      t->emit_blocks_per_sm < 0 || t->seg_cursors < 1 || t->seg_cursors > kSegCursorShapes || t->pair_shape < 0 ||
      t->pair_shape >= kPairShapes || t->replay_shape < 0 || t->replay_shape >= kReplayShapes ||
      t->emit_shape < 0 || t->emit_shape >= kEmitShapes)
    return kErrInvalidArgument;
  ctx->emit_shape = t->emit_shape;
  ctx->pair_shape = t->pair_shape;
  ctx->replay_shape = t->replay_shape;
  ctx->seg_cursors = t->seg_cursors;
  ctx->grad_shape = t->grad_shape;
  ctx->label_shape = t->label_shape;
  ctx->pair_per_sm = t->pair_blocks_per_sm;
  ctx->replay_per_sm = t->replay_blocks_per_sm;
  ctx->emit_per_sm = t->emit_blocks_per_sm;
  return kOk;
}

int dmsc_b200_get_tuning(const dmsc_b200_context* ctx, dmsc_b200_tuning* t) {
  if (!ctx || !t) return kErrInvalidArgument;
  t->grad_shape = ctx->grad_shape;
  t->label_shape = ctx->label_shape;
  t->pair_blocks_per_sm = ctx->pair_per_sm;
  t->replay_blocks_per_sm = ctx->replay_per_sm;
  t->emit_blocks_per_sm = ctx->emit_per_sm;
  t->seg_cursors = ctx->seg_cursors;
  t->pair_shape = ctx->pair_shape;
  t->replay_shape = ctx->replay_shape;
  t->emit_shape = ctx->emit_shape;
  return kOk;
}

int dmsc_b200_tuning_limits(dmsc_b200_context* ctx, int* out, int n) {
  if (!ctx || !out) return -1;
  int v[9] = {kGradShapes, kLabelShapes, 0, 0, 0, kSegCursorShapes, kPairShapes, kReplayShapes, kEmitShapes};
  if (cudaSetDevice(ctx->device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &v[2], ctx->pair_shape ? pairing_persistent_kernel<4, 4> : pairing_persistent_kernel<2, 5>, 256, 0) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &v[3], ctx->replay_shape ? replay_persistent_kernel<2, 3> : replay_persistent_kernel<1, 4>, 256, 0) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &v[4], ctx->emit_shape ? emit_persistent_kernel<2, 3> : emit_persistent_kernel<1, 5>, 256, 0) !=
          cudaSuccess)
    return -1;
  for (int k = 0; k < 9 && k < n; ++k) out[k] = v[k];
  return 9;
}

int dmsc_b200_set_wait_timeout(dmsc_b200_context* ctx, double seconds) {
  if (!ctx || !(seconds > 0.0)) return kErrInvalidArgument;
  ctx->wait_timeout_s = seconds;
  return kOk;
}

}  // extern "C"
