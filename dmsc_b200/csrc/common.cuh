// Shared device helpers for the dmsc_b200 kernels (sm_100a).
//
// Cell encoding follows the reference cell complex (dmsc/csrc/cell_complex.hxx:13-51):
//   cell id = type + 4 * (y * Nx + x),  Nx = W + 1
//   type 0 vertex (pixel), 1 H-edge, 2 V-edge, 3 face (pixel corner).
// The "index" of a cell is y * Nx + x; every index holds 4 slots in the
// gradient array (16 bytes), which is the layout of the grad_indices output.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dmsc {

// Error codes shared with the C-ABI (include/dmsc_b200.h).
enum : int {
  kOk = 0,
  kErrInvalidArgument = 1,
  kErrTooLarge = 2,
  kErrCuda = 3,
  kErrIterationCap = 4,
  kErrOverflow = 5,
  kErrInternal = 6,
};

// Bits of the device-side status word.
enum : unsigned {
  kStatusWalkCap = 1u,      // a V-path walk exceeded its step bound
  kStatusRoundCap = 2u,     // a round loop exceeded its bound
  kStatusChainCap = 4u,     // a replay chain walk exceeded its bound
  kStatusQueueOverflow = 8u,
  kStatusBadIndex = 16u,
  kStatusFindCap = 32u,     // a union-find root search or union retry loop exceeded its bound
  kStatusCopyWait = 64u,    // a bulk copy into shared memory did not complete within its time bound
};

__host__ __device__ __forceinline__ int cell_id(int t, int y, int x, int Nx) { return t + 4 * (y * Nx + x); }
__host__ __device__ __forceinline__ int cell_type(int id) { return id & 3; }
__host__ __device__ __forceinline__ int cell_index(int id) { return id >> 2; }

// std::tie(v1, id1) < std::tie(v2, id2) with IEEE '<' (cpu/cell_compare.hxx:10-12):
// -0 == +0 and NaN compare as ties, broken by id.
__device__ __forceinline__ bool tie_lt(float v1, int id1, float v2, int id2) {
  return (v1 < v2) || (!(v2 < v1) && id1 < id2);
}
// value_less<IS_DUAL> / value_greater<IS_DUAL> (cpu/cell_compare.hxx:9-21).
template <bool DUAL>
__device__ __forceinline__ bool value_less(float v1, int id1, float v2, int id2) {
  return DUAL ? tie_lt(v2, id2, v1, id1) : tie_lt(v1, id1, v2, id2);
}
template <bool DUAL>
__device__ __forceinline__ bool value_greater(float v1, int id1, float v2, int id2) {
  return value_less<!DUAL>(v1, id1, v2, id2);
}

// Monotone float -> uint32 key: ascending key order == ascending IEEE order,
// with -0 mapped onto +0 and every NaN onto one key (ties, as std::tie sees them).
__device__ __forceinline__ uint32_t orderable_key(float f) {
  if (f != f) return 0xFFFFFFFFu;
  if (f == 0.0f) f = 0.0f;
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Flow codes: one byte per index, the V-path successor of the vertex in
// bits 0-2 and of the face in bits 4-6: 0 = none (critical or no cell),
// 1 = left (x-1), 2 = right (x+1), 3 = up (y-1), 4 = down (y+1). Bits 3 and
// 7 mark the index's H and V edge critical, so the byte also gives the
// index's criticality: vertex (bits 0-2 zero, for a pixel), H edge, V edge,
// face (bits 4-6 zero).
// The gradient kernel writes them; every V-path walk uses them (17 MB at
// 4096^2, resident in L2) instead of reading the 16 B/index gradient.
enum : unsigned { kFlowNone = 0, kFlowLeft = 1, kFlowRight = 2, kFlowUp = 3, kFlowDown = 4 };

__device__ __forceinline__ int flow_step(unsigned code, int Nx) {
  return code == kFlowLeft ? -1 : code == kFlowRight ? 1 : code == kFlowUp ? -Nx : Nx;
}

// Face code of the face at index `idx` paired with edge cell `e`: the other
// coface of the edge (cpu/arcs_topology.hxx:19-39).
__device__ __forceinline__ unsigned face_flow(int e, int idx) {
  if (e < 0) return kFlowNone;
  int eidx = e >> 2;
  if ((e & 3) == 1) return eidx == idx ? kFlowDown : kFlowUp;  // H(fy,fx) -> F(fy+1,fx); H(fy-1,fx) -> F(fy-1,fx)
  return eidx == idx ? kFlowRight : kFlowLeft;                 // V(fy,fx) -> F(fy,fx+1); V(fy,fx-1) -> F(fy,fx-1)
}

// a - b with the NaN results of the x86 SSE subtraction the reference CPU
// path executes: a NaN operand propagates (first operand first, quieted) and
// an invalid operation (inf - inf) yields the default NaN 0xFFC00000. Non-NaN
// results are the IEEE difference, identical on both.
__device__ __forceinline__ float sub_like_host(float a, float b) {
  float r = a - b;
  if (r == r) return r;
  if (a != a) return __uint_as_float(__float_as_uint(a) | 0x00400000u);
  if (b != b) return __uint_as_float(__float_as_uint(b) | 0x00400000u);
  return __uint_as_float(0xFFC00000u);
}

__device__ __forceinline__ void set_status(unsigned* status, unsigned bit) { atomicOr(status, bit); }

// Per-image tables of a batch. The images' index grids ((H+1) x (W+1) each)
// are concatenated into one global index space, so a global cell id is
// type + 4 * (idx_base[b] + y * (W+1) + x); every per-image quantity is
// looked up from the image id b. Bases are exclusive prefix sums with B+1
// entries. Cell ids stay int32: the batch's total index count is < 2^29.
struct Imgs {
  int B;
  const int* H;
  const int* W;
  const int* idx_base;   // indices
  const int* px_base;    // pixels
  const int* tile_base;  // 32 x 64 gradient index tiles
  const int* seg_base;   // 32-index row segments
  const int* ltile_base;  // 64 x 64 label tiles
  const uint8_t* dual;
  const float* thr;
};

// The persistence pairing's starting state, written by the kernels that
// produce its inputs instead of a pass of its own: the ordered compaction
// sets every group's union-find link (itself) and smallest outgoing key
// (none) as it lists the extrema, plus the void slots and the round
// counters; the saddle walks then run the first round's saddle phase as they
// find each arc's end (see pairing.cuh). Side 0 is the face side (maxima),
// side 1 the vertex side (minima).
struct PairStart {
  int nsad;
  int M[2];                        // extrema of each side; the void is group M
  unsigned long long* minedge[2];  // [M + 1] smallest sweep key of each group's outgoing saddles
  int* link[2];                    // [M + 1] group union-find
  int* cnt[2];                     // [6] rotating active-saddle and live-root counters
  int2* g12[2];                    // [nsad] groups of each saddle's two ends
  int* dying[2];                   // [nsad] decision of each saddle
  const float* sval;               // [nsad] saddle values
};

// Largest b with base[b] <= g (the image holding global item g).
__device__ __forceinline__ int find_image(const int* __restrict__ base, int B, long long g) {
  int lo = 0, hi = B - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Block-aggregated reservation of consecutive slots on two counters at once
// (n0 slots on c0 and n1 on c1 per thread): one global atomic per counter and
// block, the warp totals scanned by warp 0, one set of barriers for both. A
// counter that receives no slots from the block is not touched. Every thread
// of the block must call it (blockDim.x a multiple of 32, at most 1024). p0
// and p1 receive this thread's first slots.
__device__ __forceinline__ void block_reserve2(int* c0, int n0, int* c1, int n1, int& p0, int& p1) {
  __shared__ int wsum2[2][32], bbase2[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x0 = n0, x1 = n1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y0 = __shfl_up_sync(0xffffffffu, x0, o), y1 = __shfl_up_sync(0xffffffffu, x1, o);
    if (lane >= o) {
      x0 += y0;
      x1 += y1;
    }
  }
  if (lane == 31) {
    wsum2[0][warp] = x0;
    wsum2[1][warp] = x1;
  }
  __syncthreads();
  if (warp == 0) {
    const int s0 = lane < nw ? wsum2[0][lane] : 0, s1 = lane < nw ? wsum2[1][lane] : 0;
    int i0 = s0, i1 = s1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y0 = __shfl_up_sync(0xffffffffu, i0, o), y1 = __shfl_up_sync(0xffffffffu, i1, o);
      if (lane >= o) {
        i0 += y0;
        i1 += y1;
      }
    }
    if (lane < nw) {
      wsum2[0][lane] = i0 - s0;
      wsum2[1][lane] = i1 - s1;
    }
    if (lane == 31) {  // block totals
      bbase2[0] = i0 ? atomicAdd(c0, i0) : 0;
      bbase2[1] = i1 ? atomicAdd(c1, i1) : 0;
    }
  }
  __syncthreads();
  p0 = bbase2[0] + wsum2[0][warp] + x0 - n0;
  p1 = bbase2[1] + wsum2[1][warp] + x1 - n1;
  __syncthreads();
}

// Block-aggregated append: one global atomic per block. Every thread of the
// block must call it (with blockDim.x a multiple of 32, at most 1024).
// Returns the slot of this thread's item, or -1 when `take` is false.
__device__ __forceinline__ int block_append(int* counter, bool take) {
  __shared__ int wbase[32], bbase;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, take);
  if (lane == 0) wbase[warp] = __popc(b);
  __syncthreads();
  if (warp == 0) {
    const int s = lane < nw ? wbase[lane] : 0;
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < nw) wbase[lane] = incl - s;
    if (lane == 31) bbase = incl ? atomicAdd(counter, incl) : 0;  // block total
  }
  __syncthreads();
  const int r = take ? bbase + wbase[warp] + __popc(b & ((1u << lane) - 1u)) : -1;
  __syncthreads();
  return r;
}

inline unsigned grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return (unsigned)g;
}

}  // namespace dmsc
