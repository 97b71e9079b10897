// V-path walks: saddle arc targets/lengths and basin/peak labels.
//
// Reference semantics: cpu/arcs_topology.hxx:67-172 (targets and lengths of the
// two face walks and up-to-two vertex walks of each saddle),
// cpu/arcs_geometry.hxx:74-81, 124-131 (arc k = k-th valid start cell) and
// cpu/cell_groups.hxx:96-229 (label = region of the thresholded union-find root
// of the critical cell a cell's V-path reaches). A cell's label depends only on
// its path's endpoint, so the reference's opportunistic label cache is not
// needed for identical results.
#pragma once

#include "common.cuh"

namespace dmsc {

// The j-th valid start cell of saddle `s_cell` on the face side (both cofaces
// are always valid).
__device__ __forceinline__ int face_start(int s_cell, int j, int Nx) {
  int idx = s_cell >> 2;
  if (j == 0) return 3 + 4 * idx;
  return (cell_type(s_cell) == 1) ? 3 + 4 * (idx + Nx) : 3 + 4 * (idx + 1);
}

// The j-th valid start cell on the vertex side, or -1. `s_cell` may be a
// global cell id of a batch whose image starts at index `ibase`.
__device__ __forceinline__ int vertex_start(int s_cell, int j, int H, int W, int Nx, int ibase = 0) {
  int idx = s_cell >> 2, t = cell_type(s_cell);
  int lidx = idx - ibase;
  int ey = lidx / Nx, ex = lidx - ey * Nx;
  int v[2], n = 0;
  if (t == 1) {
    if (ex - 1 >= 0) v[n++] = 4 * (idx - 1);
    if (ex < W) v[n++] = 4 * idx;
  } else {
    if (ey - 1 >= 0) v[n++] = 4 * (idx - Nx);
    if (ey < H) v[n++] = 4 * idx;
  }
  return j < n ? v[j] : -1;
}

// Walks from index `idx` along the flow codes (nibble shift 0 = vertices,
// 4 = faces) to the index of the critical cell; counts the steps.
template <int SHIFT>
__device__ __forceinline__ int flow_walk(const uint8_t* __restrict__ flow, int idx, int Nx, long long cap,
                                         long long* steps, unsigned* status) {
  long long n = 0;
  unsigned c;
  while ((c = (__ldg(flow + idx) >> SHIFT) & 0xFu) != kFlowNone) {
    idx += flow_step(c, Nx);
    if (++n > cap) {
      set_status(status, kStatusWalkCap);
      break;
    }
  }
  *steps = n;
  return idx;
}

// K4: per saddle, both face walks and the vertex walks. Writes per arc
// (2 per saddle and side): dense target index (or -1) and step count.
__global__ void __launch_bounds__(256) saddle_walk_kernel(Imgs I, const uint8_t* __restrict__ flow, int nsad,
                                                          const int* __restrict__ crit_sad,
                                                          const int* __restrict__ sad_img,
                                                          const int* __restrict__ max_rank,
                                                          const int* __restrict__ min_rank, int* __restrict__ tf,
                                                          int* __restrict__ lf, int* __restrict__ tv,
                                                          int* __restrict__ lv, long long cap, unsigned* status) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsad) return;
  const int b = sad_img[s];
  const int H = I.H[b], W = I.W[b], Nx = W + 1;
  int sc = crit_sad[s];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    long long steps;
    int end = flow_walk<4>(flow, face_start(sc, j, Nx) >> 2, Nx, cap, &steps, status);
    tf[2 * s + j] = max_rank[end];
    lf[2 * s + j] = (int)steps;
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int start = vertex_start(sc, j, H, W, Nx, I.idx_base[b]);
    long long steps = 0;
    if (start >= 0) {
      int end = flow_walk<0>(flow, start >> 2, Nx, cap, &steps, status);
      tv[2 * s + j] = min_rank[end];
    } else {
      tv[2 * s + j] = -1;
    }
    lv[2 * s + j] = (int)steps;
  }
}

// Label of every extremum, stored at its index in `map` (which held the
// extremum's dense rank): the rank among its image's surviving extrema of its
// thresholded union-find root, or -1 when the root is the void
// (cpu/cell_groups.hxx:128-146, 168-173). `alive_base[b]` is the first output
// rank of image b's extrema.
__global__ void label_map_kernel(int M, const int* __restrict__ crit, const int* __restrict__ ext_img,
                                 const int* __restrict__ ut_root, const int* __restrict__ region,
                                 const int* __restrict__ alive_base, int* __restrict__ map) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  int u = ut_root[r];
  map[crit[r] >> 2] = u < 0 ? -1 : region[u] - alive_base[ext_img[r]];
}

// Where the labels of one side go: image b's block of the output array picked
// by its orientation (faces are peaks in the primal, basins in the dual).
struct LabelOut {
  int* primal;            // output for primal images (nullptr: not requested)
  int* dual;              // output for dual images
  const int* primal_off;  // [B] block offset of image b in `primal`
  const int* dual_off;
};

// K9: labels. One thread per face index (FACES) or per pixel (vertices) of
// the batch: walk to the critical cell and read its label from the map.
template <bool FACES>
__global__ void __launch_bounds__(256) label_kernel(Imgs I, const uint8_t* __restrict__ flow, long long n,
                                                    const int* __restrict__ label_map, LabelOut O, long long cap,
                                                    unsigned* status) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = find_image(FACES ? I.idx_base : I.px_base, I.B, i);
  const bool d = I.dual[b];
  int* out = d ? O.dual : O.primal;
  if (!out) return;
  const int W = I.W[b], Nx = W + 1;
  long long local;
  int idx;
  if (FACES) {
    local = i - I.idx_base[b];
    idx = (int)i;
  } else {
    local = i - I.px_base[b];
    int y = (int)(local / W), x = (int)(local - (long long)y * W);
    idx = I.idx_base[b] + y * Nx + x;
  }
  long long steps;
  int end = flow_walk<FACES ? 4 : 0>(flow, idx, Nx, cap, &steps, status);
  out[(d ? O.dual_off : O.primal_off)[b] + local] = steps <= cap ? __ldg(label_map + end) : -1;
}

}  // namespace dmsc
