// Gradient and critical cells without any device allocation.
//
// Some callers cannot allocate device memory at call time: code running while
// a stream is being captured into a CUDA graph (cudaMalloc is not allowed in a
// capture), real-time or embedded hosts whose memory is fixed at start-up, and
// plugins whose host framework owns every allocation and hands out only the
// input and output buffers. For them, dmsc_b200_critical_cells_static()
// computes the discrete gradient and the ascending critical-cell lists of one
// image using only the caller's buffers and the fixed scratch array below.
//
// The scratch is one file-scope __device__ array, so every GPU that loads the
// library holds it until the process exits. All calls share it: calls that
// overlap on the GPU (on different streams, or from several host threads)
// race on it, so callers must serialise them. Host code never dereferences the
// array's name (on the host it is only a stand-in symbol); its device address
// is looked up once per device with cudaGetSymbolAddress, with that device
// current. The first call on a device does this set-up (and uploads the face
// pairing table to a second static array), so that first call should come
// before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/dmsc_b200.h"
#include "common.cuh"
#include "gradient.cuh"

namespace {

using namespace dmsc;

// 8 MiB: per image, 2 bytes per index (criticality mask and flow codes) plus
// 6 ints per 32-index row segment (three counts, three offsets), each of the
// eight parts rounded up to 256 bytes: about 2.75 bytes per index, so square
// images up to 1743 x 1743 fit (1744 x 1744 needs 8,394,240 bytes). The
// scratch check also keeps the segment count far below INT_MAX, which the
// single-block scan relies on.
constexpr size_t kStaticScratchBytes = 8u << 20;
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
__device__ uint32_t g_static_fifo_lut[kGradTable];

constexpr int kMaxDevices = 64;
struct DeviceStatic {
  bool ready = false;
  unsigned char* scratch = nullptr;
  uint32_t* lut = nullptr;
};
std::mutex g_static_mutex;
DeviceStatic g_static[kMaxDevices];

// Device addresses of the static arrays on the current device (set up once).
int static_setup(int device, DeviceStatic** out) {
  if (device < 0 || device >= kMaxDevices) return DMSC_B200_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(g_static_mutex);
  DeviceStatic& d = g_static[device];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return DMSC_B200_ERR_CUDA;
    d.scratch = (unsigned char*)p;
    if (cudaGetSymbolAddress(&p, g_static_fifo_lut) != cudaSuccess || !p) return DMSC_B200_ERR_CUDA;
    d.lut = (uint32_t*)p;
    std::vector<uint32_t> lut(kGradTable);
    gradient_tables(lut.data());
    if (cudaMemcpyToSymbol(g_static_fifo_lut, lut.data(), kGradTable * sizeof(uint32_t)) != cudaSuccess)
      return DMSC_B200_ERR_CUDA;
    // A copy from pageable host memory may return before the table has
    // reached the device, and it is ordered on the legacy default stream
    // only; the caller's stream (possibly non-blocking) is not ordered after
    // it. Waiting here, once per device, makes the table visible to every
    // later launch on any stream.
    if (cudaDeviceSynchronize() != cudaSuccess) return DMSC_B200_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return DMSC_B200_OK;
}

// Exclusive scans of the three segment-count arrays in one block (segments
// are few: one per 32 indices of a row).
__global__ void __launch_bounds__(1024) static_scan3_kernel(const int* __restrict__ c0, const int* __restrict__ c1,
                                                           const int* __restrict__ c2, int n, int* __restrict__ o0,
                                                           int* __restrict__ o1, int* __restrict__ o2,
                                                           int32_t* __restrict__ totals) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int* in[3] = {c0, c1, c2};
  int* out[3] = {o0, o1, o2};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int a = 0; a < 3; ++a) {
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
      int i = base + threadIdx.x;
      int v = i < n ? in[a][i] : 0, x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      if (warp == 0) {
        int w = wsum[lane], z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          int y = __shfl_up_sync(0xffffffffu, z, o);
          if (lane >= o) z += y;
        }
        wsum[lane] = z - w;
      }
      __syncthreads();
      if (i < n) out[a][i] = carry + wsum[warp] + x - v;
      __syncthreads();
      if (threadIdx.x == 1023) carry += wsum[31] + x;
      __syncthreads();
    }
    if (threadIdx.x == 0) totals[a] = carry;
    __syncthreads();
  }
}

// Ordered compaction of the critical cells into the three ascending lists
// (cpu/critical_points.hxx:14-65); the list-only variant of compact_kernel.
__global__ void __launch_bounds__(256) static_lists_kernel(int W, int nsegx, long long nseg,
                                                           const uint8_t* __restrict__ crit_mask,
                                                           const int* __restrict__ off_min,
                                                           const int* __restrict__ off_sad,
                                                           const int* __restrict__ off_max, int32_t* __restrict__ mins,
                                                           int32_t* __restrict__ sads, int32_t* __restrict__ maxs) {
  const int lane = threadIdx.x & 31;
  long long seg = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (seg >= nseg) return;
  const int Nx = W + 1;
  int iy = (int)(seg / nsegx), sx = (int)(seg - (long long)iy * nsegx);
  int ix = sx * kTileX + lane;
  unsigned m = 0;
  size_t idx = (size_t)iy * Nx + ix;
  if (ix <= W) m = crit_mask[idx];
  unsigned lt = (1u << lane) - 1u;
  unsigned bmin = __ballot_sync(0xffffffffu, m & 1u);
  unsigned bmax = __ballot_sync(0xffffffffu, m & 8u);
  int ns = ((m >> 1) & 1u) + ((m >> 2) & 1u);
  int incl = ns;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (m & 1u) mins[off_min[seg] + __popc(bmin & lt)] = (int)(4 * idx);
  if (m & 8u) maxs[off_max[seg] + __popc(bmax & lt)] = (int)(4 * idx + 3);
  int p = off_sad[seg] + incl - ns;
  if (m & 2u) sads[p++] = (int)(4 * idx + 1);
  if (m & 4u) sads[p] = (int)(4 * idx + 2);
}

}  // namespace

extern "C" int dmsc_b200_critical_cells_static(const float* image, int H, int W, unsigned flags, int32_t* grad_out,
                                               int32_t* mins_out, int32_t* saddles_out, int32_t* maxes_out,
                                               int32_t* counts_out, void* stream) {
  if (!image || !grad_out || !mins_out || !saddles_out || !maxes_out || !counts_out || H <= 0 || W <= 0)
    return DMSC_B200_ERR_INVALID_ARGUMENT;
  if ((uintptr_t)grad_out & 15u) return DMSC_B200_ERR_INVALID_ARGUMENT;  // written with 16-byte stores
  if ((long long)H + 1 > 2147483647LL / 4 / ((long long)W + 1)) return DMSC_B200_ERR_TOO_LARGE;
  const long long nidx = (long long)(H + 1) * (W + 1);
  const int nsegx = (W + 1 + kTileX - 1) / kTileX;
  const long long nseg = (long long)(H + 1) * nsegx;
  // scratch layout: mask [nidx] | flow [nidx] | 6 x nseg ints, 256-byte aligned parts
  auto up = [](long long b) { return (b + 255) & ~255LL; };
  const long long need = up(nidx) + up(nidx) + 6 * up(nseg * 4);
  if (need > (long long)kStaticScratchBytes) return DMSC_B200_ERR_TOO_LARGE;  // before any launch
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return DMSC_B200_ERR_CUDA;
  DeviceStatic* d = nullptr;
  int rc = static_setup(device, &d);
  if (rc != DMSC_B200_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* p = d->scratch;
  uint8_t* mask = p;
  p += up(nidx);
  uint8_t* flow = p;
  p += up(nidx);
  int* seg[3];
  int* off[3];
  for (int k = 0; k < 3; ++k) {
    seg[k] = (int*)p;
    p += up(nseg * 4);
  }
  for (int k = 0; k < 3; ++k) {
    off[k] = (int*)p;
    p += up(nseg * 4);
  }
  constexpr int TY = kGradTY[1], NT = kGradNT[1];
  dim3 g1(nsegx, (H + 1 + TY - 1) / TY);
  if (flags & DMSC_B200_DUAL)
    gradient_kernel<true, TY, NT><<<g1, NT, 0, st>>>(image, H, W, (int4*)grad_out, mask, seg[0], seg[1], seg[2],
                                                     d->lut, flow);
  else
    gradient_kernel<false, TY, NT><<<g1, NT, 0, st>>>(image, H, W, (int4*)grad_out, mask, seg[0], seg[1], seg[2],
                                                      d->lut, flow);
  static_scan3_kernel<<<1, 1024, 0, st>>>(seg[0], seg[1], seg[2], (int)nseg, off[0], off[1], off[2], counts_out);
  static_lists_kernel<<<(unsigned)((nseg + 7) / 8), 256, 0, st>>>(W, nsegx, nseg, mask, off[0], off[1], off[2],
                                                                  mins_out, saddles_out, maxes_out);
  return cudaGetLastError() == cudaSuccess ? DMSC_B200_OK : DMSC_B200_ERR_CUDA;
}
