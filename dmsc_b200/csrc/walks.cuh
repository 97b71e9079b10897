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

// The j-th valid start cell on the vertex side, or -1.
__device__ __forceinline__ int vertex_start(int s_cell, int j, int H, int W, int Nx) {
  int idx = s_cell >> 2, t = cell_type(s_cell);
  int ey = idx / Nx, ex = idx - ey * Nx;
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

// K4: per saddle, both face walks and the vertex walks. Writes per arc
// (2 per saddle and side): dense target index (or -1) and step count.
__global__ void __launch_bounds__(256) saddle_walk_kernel(const int* __restrict__ grad, int H, int W, int nsad,
                                                          const int* __restrict__ crit_sad,
                                                          const int* __restrict__ max_rank,
                                                          const int* __restrict__ min_rank, int* __restrict__ tf,
                                                          int* __restrict__ lf, int* __restrict__ tv,
                                                          int* __restrict__ lv, long long cap, unsigned* status) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsad) return;
  const int Nx = W + 1;
  int sc = crit_sad[s];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int curr = face_start(sc, j, Nx);
    long long steps = 0;
    int e;
    while ((e = __ldg(grad + curr)) != -1) {
      curr = next_face(e, curr, Nx);
      if (++steps > cap) {
        set_status(status, kStatusWalkCap);
        break;
      }
    }
    tf[2 * s + j] = max_rank[curr >> 2];
    lf[2 * s + j] = (int)steps;
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int curr = vertex_start(sc, j, H, W, Nx);
    long long steps = 0;
    if (curr >= 0) {
      int e;
      while (curr != -1 && (e = __ldg(grad + curr)) != -1) {
        curr = next_vertex(e, curr, H, W, Nx);
        if (++steps > cap) {
          set_status(status, kStatusWalkCap);
          break;
        }
      }
      tv[2 * s + j] = curr >= 0 ? min_rank[curr >> 2] : -1;
    } else {
      tv[2 * s + j] = -1;
    }
    lv[2 * s + j] = (int)steps;
  }
}

// K9: labels. One thread per face index (FACES) or per pixel (vertices):
// walk to the critical cell, map it through the flattened thresholded
// union-find root to the rank of the surviving extremum.
template <bool FACES>
__global__ void __launch_bounds__(256) label_kernel(const int* __restrict__ grad, int H, int W,
                                                    const int* __restrict__ rank_map, const int* __restrict__ ut_root,
                                                    const int* __restrict__ region, int* __restrict__ out, long long cap,
                                                    unsigned* status) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nx = W + 1;
  long long n = FACES ? (long long)(H + 1) * Nx : (long long)H * W;
  if (i >= n) return;
  int curr;
  if (FACES) {
    curr = (int)(4 * i + 3);
  } else {
    int y = (int)(i / W), x = (int)(i - (long long)y * W);
    curr = 4 * (y * Nx + x);
  }
  long long steps = 0;
  int e;
  while (curr != -1 && (e = __ldg(grad + curr)) != -1) {
    curr = FACES ? next_face(e, curr, Nx) : next_vertex(e, curr, H, W, Nx);
    if (++steps > cap) {
      set_status(status, kStatusWalkCap);
      curr = -1;
      break;
    }
  }
  int lab = -1;
  if (curr != -1) {
    int r = ut_root[rank_map[curr >> 2]];
    if (r != -1) lab = region[r];
  }
  out[i] = lab;
}

}  // namespace dmsc
