// Persistence pairs as pixel pairs, and the deterministic backward scatter.
//
// A persistence value is the float32 difference of two input pixels: the
// value pixel of the saddle and the value pixel of the extremum that dies at
// it (cpu/persistence.hxx:82-104, 139-161), where a cell's value pixel is its
// highest vertex in the primal, its lowest in the dual, chosen under the
// (value, pixel id) order (cpu/cell_compare.hxx:33-87). On a field without
// ties the pairing is locally constant, so d p / d img is +1 on one pixel and
// -1 on the other; the backward pass scatters dL/dp onto those pixels.
#pragma once

#include "assemble.cuh"
#include "common.cuh"

namespace dmsc {

// Image-local value pixel of cell (t, y, x) (the pixel cell_value reads).
template <bool DUAL>
__device__ __forceinline__ int cell_pixel_g(const float* __restrict__ img, int t, int y, int x, int H, int W) {
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
  return b;
}

// Value pixel of global cell `cell` of image b.
__device__ __forceinline__ int value_pixel(const float* __restrict__ img_all, const Imgs& I, int b, int cell) {
  const int H = I.H[b], W = I.W[b], Nx = W + 1;
  const int lidx = (cell >> 2) - I.idx_base[b];
  const int y = lidx / Nx, x = lidx - y * Nx;
  const float* img = img_all + I.px_base[b];
  return I.dual[b] ? cell_pixel_g<true>(img, cell & 3, y, x, H, W) : cell_pixel_g<false>(img, cell & 3, y, x, H, W);
}

// Per surviving saddle of one side, in the order of that side's p output
// (survivor order; the face side visits each image's survivors reversed),
// the image-local pixels entering its persistence with sign + and -
// (-1, -1 for a cycle, whose persistence is the constant -1). The sign
// follows persistence_kernel: p = saddle - extremum on the vertex side in the
// primal and on the face side in the dual, extremum - saddle otherwise.
__global__ void pair_pixels_kernel(int nsurv, bool faces, const int* __restrict__ surv_base, Imgs I,
                                   const float* __restrict__ img_all, const int* __restrict__ surv_sad,
                                   const int* __restrict__ crit_sad, const int2* __restrict__ pp,
                                   const int2* __restrict__ ext_key, Route PLUS, Route MINUS) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsurv) return;
  int b;
  int i = visit(q, faces, surv_base, I.B, &b);
  const bool d = I.dual[b];
  const int li = i - surv_base[b];
  const int s = surv_sad[i];
  const int e = pp[s].x;
  int plus = -1, minus = -1;
  if (e >= 0) {
    const int sp = value_pixel(img_all, I, b, crit_sad[s]);
    const int ep = value_pixel(img_all, I, b, ext_key[e].y);
    const bool saddle_plus = (!faces) != d;
    plus = saddle_plus ? sp : ep;
    minus = saddle_plus ? ep : sp;
  }
  if (int* p = PLUS.at(d, b)) p[li] = plus;
  if (int* m = MINUS.at(d, b)) m[li] = minus;
}

// ---------------------------------------------------------------------------
// backward: grad_img[pix] = sum of +-dL/dp over the pair ends at pix, summed
// in a fixed order (no float atomics), so repeated runs give identical bits.

// Entry k of 2n: pair k >> 1, + end for even k, - end for odd k. Key = pixel
// (npx for an absent end, which sorts last).
__global__ void pair_entries_kernel(long long n, const int* __restrict__ plus, const int* __restrict__ minus,
                                    int npx, int* __restrict__ key, int* __restrict__ idx) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 2 * n) return;
  const long long i = k >> 1;
  int p = (k & 1) ? minus[i] : plus[i];
  key[k] = (p >= 0 && p < npx) ? p : npx;
  idx[k] = (int)k;
}

// One thread per sorted entry that starts a run of equal keys: sums the run
// in ascending entry order (the radix sort is stable) and writes the pixel.
__global__ void pair_segments_kernel(long long m, const int* __restrict__ key, const int* __restrict__ idx,
                                     const float* __restrict__ grad_p, int npx, float* __restrict__ grad_img) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int pix = key[k];
  if (pix >= npx || (k > 0 && key[k - 1] == pix)) return;
  float acc = 0.0f;
  for (long long j = k; j < m && key[j] == pix; ++j) {
    const int e = idx[j];
    const float g = grad_p[e >> 1];
    acc = (e & 1) ? acc - g : acc + g;
  }
  grad_img[pix] = acc;
}

}  // namespace dmsc
