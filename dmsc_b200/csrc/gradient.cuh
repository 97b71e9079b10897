// Discrete gradient (steepest lower-star pairing) and ordered critical-cell
// compaction.
//
// Reference semantics: cpu/gradient.hxx:19-196 (compute_gradient),
// cpu/critical_points.hxx:14-65 (extract_critical_points, canonical order =
// ascending cell id), cpu/gradient.hxx:198-231 (fast_crit_map and values).
//
// Layout. The gradient array holds 4 int32 slots per index (y, x) of the
// (H+1) x (W+1) index grid, i.e. 16 bytes per index; it is the grad_indices
// output. One CTA owns a 32 x 8 tile of indices and writes it with one int4
// store per index, so every warp writes 512 contiguous bytes. The cells at a
// tile's indices are owned (have their highest vertex) in the pixels of the
// tile plus one halo row above and one halo column to the left, so the CTA
// evaluates the lower star of (8+1) x (32+1) pixels from a (8+3) x (32+3)
// value tile in shared memory. Slots of invalid cells stay -1.
//
// The same pass writes one criticality byte per index (bit t = slot t is an
// unpaired valid cell) and per-(row, 32-column segment) counts of minima,
// saddles and maxima; a scan over the segments in row-major order gives every
// critical cell its position in the ascending-cell-id lists.
#pragma once

#include "common.cuh"

namespace dmsc {

constexpr int kTileX = 32;  // indices per tile row (one warp)
constexpr int kTileY = 8;   // tile rows (one warp each)
constexpr int kValX = kTileX + 3;
constexpr int kValY = kTileY + 3;

template <bool DUAL>
struct PixelTile {
  const float (*v)[kValX];
  int oy, ox, W;  // tile value origin = (y0 - 2, x0 - 2)
  __device__ __forceinline__ float val(int y, int x) const { return v[y - oy][x - ox]; }
  // v_greater (cpu/cell_compare.hxx:23-31): pixels ordered by (value, y*W+x)
  __device__ __forceinline__ bool gt(int ay, int ax, int by, int bx) const {
    return value_greater<DUAL>(val(ay, ax), ay * W + ax, val(by, bx), by * W + bx);
  }
};

// get_highest_vertex_yx scan over a face's candidates in the reference order
// (cpu/cell_compare.hxx:33-63); returns true when pixel (py, px) wins.
template <bool DUAL>
__device__ __forceinline__ bool face_top_is(const PixelTile<DUAL>& T, int fy, int fx, int H, int W, int py,
                                            int px) {
  int by = -1, bx = -1;
  int cy[4] = {fy - 1, fy - 1, fy, fy};
  int cx[4] = {fx - 1, fx, fx - 1, fx};
  bool ok[4] = {fy >= 1 && fx >= 1, fy >= 1 && fx < W, fy < H && fx >= 1, fy < H && fx < W};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!ok[k]) continue;
    if (by < 0 || T.gt(cy[k], cx[k], by, bx)) {
      by = cy[k];
      bx = cx[k];
    }
  }
  return by == py && bx == px;
}

// Lower star of pixel (y, x) and its pairing (cpu/gradient.hxx:48-192).
// Edge slots: e0 = H(y,x), e1 = H(y,x+1), e2 = V(y,x), e3 = V(y+1,x).
// Face slots: f0 = F(y,x), f1 = F(y,x+1), f2 = F(y+1,x), f3 = F(y+1,x+1).
// The owned cells' gradient values are written into the shared index tile.
template <bool DUAL>
__device__ __forceinline__ void lower_star(const PixelTile<DUAL>& T, int y, int x, int H, int W, int Nx, int ty0,
                                           int tx0, int (*tile)[kTileX][4]) {
  // --- lower-star membership, with the reference's candidate scan order ---
  unsigned eL = 0, fL = 0;
  if (x - 1 < 0 || T.gt(y, x, y, x - 1)) eL |= 1u;
  if (!(x + 1 < W && T.gt(y, x + 1, y, x))) eL |= 2u;
  if (y - 1 < 0 || T.gt(y, x, y - 1, x)) eL |= 4u;
  if (!(y + 1 < H && T.gt(y + 1, x, y, x))) eL |= 8u;
  if (face_top_is<DUAL>(T, y, x, H, W, y, x)) fL |= 1u;
  if (face_top_is<DUAL>(T, y, x + 1, H, W, y, x)) fL |= 2u;
  if (face_top_is<DUAL>(T, y + 1, x, H, W, y, x)) fL |= 4u;
  if (face_top_is<DUAL>(T, y + 1, x + 1, H, W, y, x)) fL |= 8u;

  // --- vertex pairing: the lower-star edge whose other vertex is lowest ---
  int ov_y[4] = {y, y, y - 1, y + 1};
  int ov_x[4] = {x - 1, x + 1, x, x};
  bool ov_ok[4] = {x - 1 >= 0, x + 1 < W, y - 1 >= 0, y + 1 < H};
  int best = -1, bo_y = 0, bo_x = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!((eL >> k) & 1u) || !ov_ok[k]) continue;
    if (best == -1 || T.gt(bo_y, bo_x, ov_y[k], ov_x[k])) {
      best = k;
      bo_y = ov_y[k];
      bo_x = ov_x[k];
    }
  }
  // pairing state: epair[k] = -1 none, 4 vertex, 0..3 face slot; fpair[f] = edge slot or -1
  int epair[4] = {-1, -1, -1, -1};
  int fpair[4] = {-1, -1, -1, -1};
  unsigned epaired = 0, fpaired = 0;
  if (best >= 0) {
    epair[best] = 4;
    epaired |= 1u << best;
  }

  // --- face pairing by FIFO (cpu/gradient.hxx:115-191) ---
  // face f's lower-star-candidate edges in the reference visiting order
  const int fe_a[4] = {0, 1, 0, 1};
  const int fe_b[4] = {2, 2, 3, 3};
  // faces bounding edge slot k, in check_and_push order
  const int ef_a[4] = {0, 1, 0, 2};
  const int ef_b[4] = {2, 3, 1, 3};
  unsigned long long q = 0;  // queue of face slots, 4 bits per entry
  int head = 0, tail = 0;
#pragma unroll
  for (int f = 0; f < 4; ++f)
    if ((fL >> f) & 1u) {
      q |= (unsigned long long)f << (4 * tail);
      tail++;
    }
  while (head < tail) {
    int f = (int)((q >> (4 * head)) & 0xFull);
    head++;
    if ((fpaired >> f) & 1u) continue;
    int unp_e = -1, unp_n = 0;
    int ea = fe_a[f], eb = fe_b[f];
    if (((eL >> ea) & 1u) && !((epaired >> ea) & 1u)) {
      unp_n++;
      unp_e = ea;
    }
    if (((eL >> eb) & 1u) && !((epaired >> eb) & 1u)) {
      unp_n++;
      unp_e = eb;
    }
    if (unp_n != 1) continue;
    fpair[f] = unp_e;
    fpaired |= 1u << f;
    epair[unp_e] = f;
    epaired |= 1u << unp_e;
    int cand[2] = {ef_a[unp_e], ef_b[unp_e]};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      int nf = cand[c];
      if (nf == f || !((fL >> nf) & 1u) || ((fpaired >> nf) & 1u)) continue;
      bool already = false;
      for (int qi = head; qi < tail; ++qi)
        if ((int)((q >> (4 * qi)) & 0xFull) == nf) already = true;
      if (!already && tail < 16) {
        q |= (unsigned long long)nf << (4 * tail);
        tail++;
      }
    }
  }

  // --- write owned cells into the index tile ---
  const int e_iy[4] = {y, y, y, y + 1};
  const int e_ix[4] = {x, x + 1, x, x};
  const int e_t[4] = {1, 1, 2, 2};
  const int f_iy[4] = {y, y, y + 1, y + 1};
  const int f_ix[4] = {x, x + 1, x, x + 1};
  auto put = [&](int iy, int ix, int t, int v) {
    int r = iy - ty0, c = ix - tx0;
    if (r >= 0 && r < kTileY && c >= 0 && c < kTileX) tile[r][c][t] = v;
  };
  put(y, x, 0, best >= 0 ? cell_id(e_t[best], e_iy[best], e_ix[best], Nx) : -1);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!((eL >> k) & 1u)) continue;
    int v = -1;
    if (epair[k] == 4)
      v = cell_id(0, y, x, Nx);
    else if (epair[k] >= 0)
      v = cell_id(3, f_iy[epair[k]], f_ix[epair[k]], Nx);
    put(e_iy[k], e_ix[k], e_t[k], v);
  }
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (!((fL >> f) & 1u)) continue;
    int k = fpair[f];
    put(f_iy[f], f_ix[f], 3, k >= 0 ? cell_id(e_t[k], e_iy[k], e_ix[k], Nx) : -1);
  }
}

// K1: gradient over one 32 x 8 index tile per CTA (256 threads).
template <bool DUAL>
__global__ void __launch_bounds__(256) gradient_kernel(const float* __restrict__ img, int H, int W,
                                                       int4* __restrict__ grad, uint8_t* __restrict__ crit_mask,
                                                       int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                                       int* __restrict__ seg_max) {
  __shared__ float sv[kValY][kValX];
  __shared__ int tile[kTileY][kTileX][4];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY;
  const int Nx = W + 1;

  for (int i = tid; i < kValY * kValX; i += 256) {
    int r = i / kValX, c = i - r * kValX;
    int gy = y0 - 2 + r, gx = x0 - 2 + c;
    sv[r][c] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? __ldg(img + (size_t)gy * W + gx) : 0.0f;
  }
  for (int i = tid; i < kTileY * kTileX; i += 256) {
    int r = i / kTileX, c = i - r * kTileX;
    tile[r][c][0] = tile[r][c][1] = tile[r][c][2] = tile[r][c][3] = -1;
  }
  __syncthreads();

  PixelTile<DUAL> T{sv, y0 - 2, x0 - 2, W};
  for (int i = tid; i < (kTileY + 1) * (kTileX + 1); i += 256) {
    int r = i / (kTileX + 1), c = i - r * (kTileX + 1);
    int y = y0 - 1 + r, x = x0 - 1 + c;
    if (y < 0 || y >= H || x < 0 || x >= W) continue;
    lower_star<DUAL>(T, y, x, H, W, Nx, y0, x0, tile);
  }
  __syncthreads();

  // one warp per tile row: coalesced int4 stores, criticality mask and counts
  const int warp = tid >> 5, lane = tid & 31;
  const int iy = y0 + warp, ix = x0 + lane;
  if (iy > H) return;
  bool in = ix <= W;
  int4 v = make_int4(tile[warp][lane][0], tile[warp][lane][1], tile[warp][lane][2], tile[warp][lane][3]);
  unsigned m = 0;
  if (in) {
    size_t idx = (size_t)iy * Nx + ix;
    grad[idx] = v;
    if (v.x == -1 && iy < H && ix < W) m |= 1u;
    if (v.y == -1 && iy < H) m |= 2u;
    if (v.z == -1 && ix < W) m |= 4u;
    if (v.w == -1) m |= 8u;
    crit_mask[idx] = (uint8_t)m;
  }
  unsigned bmin = __ballot_sync(0xffffffffu, m & 1u);
  unsigned bs1 = __ballot_sync(0xffffffffu, m & 2u);
  unsigned bs2 = __ballot_sync(0xffffffffu, m & 4u);
  unsigned bmax = __ballot_sync(0xffffffffu, m & 8u);
  if (lane == 0) {
    int seg = iy * gridDim.x + blockIdx.x;
    seg_min[seg] = __popc(bmin);
    seg_sad[seg] = __popc(bs1) + __popc(bs2);
    seg_max[seg] = __popc(bmax);
  }
}

// cell_value (cpu/cell_compare.hxx:82-87): value of the highest (dual: lowest)
// vertex, chosen by (value, pixel id) with the reference scan order; the chosen
// pixel's own value is returned, so -0.0 survives.
template <bool DUAL>
__device__ __forceinline__ float cell_value_g(const float* __restrict__ img, int t, int y, int x, int H, int W) {
  int cy[4], cx[4], n = 0;
  if (t == 0) {
    cy[n] = y;
    cx[n++] = x;
  } else if (t == 1) {
    if (x - 1 >= 0) {
      cy[n] = y;
      cx[n++] = x - 1;
    }
    if (x < W) {
      cy[n] = y;
      cx[n++] = x;
    }
  } else if (t == 2) {
    if (y - 1 >= 0) {
      cy[n] = y - 1;
      cx[n++] = x;
    }
    if (y < H) {
      cy[n] = y;
      cx[n++] = x;
    }
  } else {
    if (y - 1 >= 0 && x - 1 >= 0) {
      cy[n] = y - 1;
      cx[n++] = x - 1;
    }
    if (y - 1 >= 0 && x < W) {
      cy[n] = y - 1;
      cx[n++] = x;
    }
    if (y < H && x - 1 >= 0) {
      cy[n] = y;
      cx[n++] = x - 1;
    }
    if (y < H && x < W) {
      cy[n] = y;
      cx[n++] = x;
    }
  }
  int b = cy[0] * W + cx[0];
  float bv = __ldg(img + b);
  for (int k = 1; k < n; ++k) {
    int id = cy[k] * W + cx[k];
    float v = __ldg(img + id);
    if (value_greater<DUAL>(v, id, bv, b)) {
      b = id;
      bv = v;
    }
  }
  return bv;
}

// K2: ordered compaction. One warp per (row, 32-column) segment; segment
// offsets are exclusive scans of the per-segment counts. Writes the three
// ascending-cell-id lists, the index -> dense-rank maps of the extrema, the
// extremum values and the saddle values with their radix-sort keys.
template <bool DUAL>
__global__ void __launch_bounds__(256) compact_kernel(
    const float* __restrict__ img, int H, int W, int nsegx, long long nseg, const uint8_t* __restrict__ crit_mask,
    const int* __restrict__ off_min, const int* __restrict__ off_sad, const int* __restrict__ off_max,
    int* __restrict__ crit_min, int* __restrict__ crit_sad, int* __restrict__ crit_max, int* __restrict__ min_rank,
    int* __restrict__ max_rank, float* __restrict__ min_val, float* __restrict__ max_val, float* __restrict__ sad_val,
    uint32_t* __restrict__ sad_key) {
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
  int excl = incl - ns;
  if (m & 1u) {
    int p = off_min[seg] + __popc(bmin & lt);
    crit_min[p] = (int)(4 * idx);
    min_rank[idx] = p;
    min_val[p] = __ldg(img + (size_t)iy * W + ix);
  }
  if (m & 8u) {
    int p = off_max[seg] + __popc(bmax & lt);
    crit_max[p] = (int)(4 * idx + 3);
    max_rank[idx] = p;
    max_val[p] = cell_value_g<DUAL>(img, 3, iy, ix, H, W);
  }
  int p = off_sad[seg] + excl;
  if (m & 2u) {
    crit_sad[p] = (int)(4 * idx + 1);
    float v = cell_value_g<DUAL>(img, 1, iy, ix, H, W);
    sad_val[p] = v;
    sad_key[p] = orderable_key(v);
    p++;
  }
  if (m & 4u) {
    crit_sad[p] = (int)(4 * idx + 2);
    float v = cell_value_g<DUAL>(img, 2, iy, ix, H, W);
    sad_val[p] = v;
    sad_key[p] = orderable_key(v);
  }
}

}  // namespace dmsc
