// Output assembly on the device (cpu/workspace.hxx:86-365).
//
// Surviving extrema keep their ascending-cell-id order; surviving saddles are
// listed in minima-sweep order; e_min rows follow the minima sweep and e_max
// rows the maxima sweep, which is the reverse of the minima sweep for the
// same saddles (cpu/arcs_topology.hxx:142).
#pragma once

#include "common.cuh"

namespace dmsc {

__global__ void u8_to_int_kernel(const uint8_t* __restrict__ a, int n, int* __restrict__ b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// pts[to_out[x]] = cell[x] for alive x.
__global__ void compact_alive_kernel(int n, const uint8_t* __restrict__ alive, const int* __restrict__ to_out_excl,
                                     const int* __restrict__ cell, int* __restrict__ pts, int* __restrict__ to_out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  if (alive[x]) {
    to_out[x] = to_out_excl[x];
    if (pts) pts[to_out_excl[x]] = cell[x];
  } else {
    to_out[x] = -1;
  }
}

// flag[j] = 1 when the saddle at minima-sweep position j survives both sides.
__global__ void survivor_flag_kernel(int nsad, const int* __restrict__ sweep_min, const uint8_t* __restrict__ cancelled,
                                     int* __restrict__ flag) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nsad) return;
  flag[j] = cancelled[sweep_min[j]] == 0;
}

__global__ void survivor_list_kernel(int nsad, const int* __restrict__ sweep_min, const int* __restrict__ flag,
                                     const int* __restrict__ pos, int* __restrict__ surv_sad) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nsad) return;
  if (flag[j]) surv_sad[pos[j]] = sweep_min[j];
}

// Per survivor, in iteration order (minima: i; maxima: nsurv-1-i): number of
// e rows (0..2) (cpu/workspace.hxx:175-195, 197-219).
__device__ __forceinline__ int erow_ends(int s, const int* __restrict__ t, const int* __restrict__ ut,
                                         const int* __restrict__ to_out, int* o1, int* o2) {
  int c1 = t[2 * s], c2 = t[2 * s + 1];
  int r1 = c1 >= 0 ? ut[c1] : -1;
  int r2 = c2 >= 0 ? ut[c2] : -1;
  int n = 0;
  if (r1 != -1 && to_out[r1] != -1) {
    *o1 = to_out[r1];
    n = 1;
  }
  if (r1 != r2 && r2 != -1 && to_out[r2] != -1) {
    if (n == 0)
      *o1 = to_out[r2];
    else
      *o2 = to_out[r2];
    n++;
  }
  return n;
}

__global__ void erow_count_kernel(int nsurv, bool reversed, const int* __restrict__ surv_sad,
                                  const int* __restrict__ t, const int* __restrict__ ut,
                                  const int* __restrict__ to_out, int* __restrict__ cnt) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsurv) return;
  int i = reversed ? nsurv - 1 - q : q;
  int a, b;
  cnt[q] = erow_ends(surv_sad[i], t, ut, to_out, &a, &b);
}

// Per-survivor scalar outputs and e rows of one side.
__global__ void side_outputs_kernel(int nsurv, bool reversed, const int* __restrict__ surv_sad,
                                    const int* __restrict__ t, const int* __restrict__ ut,
                                    const int* __restrict__ to_out, const float* __restrict__ pers,
                                    const int* __restrict__ pair_dense, const int* __restrict__ row_off,
                                    float* __restrict__ p_out, int* __restrict__ pp_out, int* __restrict__ e_out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsurv) return;
  int i = reversed ? nsurv - 1 - q : q;
  int s = surv_sad[i];
  if (p_out) p_out[i] = pers[s];
  if (pp_out) {
    int pd = pair_dense[s];
    int r = pd >= 0 ? ut[pd] : -1;
    pp_out[i] = r >= 0 ? to_out[r] : -1;
  }
  if (e_out) {
    int a = 0, b = 0;
    int n = erow_ends(s, t, ut, to_out, &a, &b);
    int o = row_off[q];
    if (n >= 1) {
      e_out[2 * o] = i;
      e_out[2 * o + 1] = a;
    }
    if (n == 2) {
      e_out[2 * o + 2] = i;
      e_out[2 * o + 3] = b;
    }
  }
}

__global__ void sad_pts_kernel(int nsurv, const int* __restrict__ surv_sad, const int* __restrict__ crit_sad,
                               int* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsurv) out[i] = crit_sad[surv_sad[i]];
}

// CSR offsets of one side's arcs (cpu/workspace.hxx:247-287):
// offsets[i+1] = end of survivor i, arc_offsets[i] = end of its first arc.
__global__ void arc_offsets_kernel(int nsurv, const long long* __restrict__ arc_len,
                                   const long long* __restrict__ saddle_end_incl, int* __restrict__ offsets,
                                   int* __restrict__ arc_offsets) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nsurv) return;
  if (i == 0) offsets[0] = 0;
  if (i < nsurv) {
    long long end = saddle_end_incl[i];
    long long start = end - arc_len[2 * i] - arc_len[2 * i + 1];
    offsets[i + 1] = (int)end;
    arc_offsets[i] = (int)(start + arc_len[2 * i]);
  }
}

__global__ void arc_pos_kernel(int nsurv, const long long* __restrict__ arc_len,
                               const long long* __restrict__ saddle_end_incl, long long* __restrict__ arc_pos) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv) return;
  long long start = saddle_end_incl[i] - arc_len[2 * i] - arc_len[2 * i + 1];
  arc_pos[2 * i] = start;
  arc_pos[2 * i + 1] = start + arc_len[2 * i];
}

__global__ void pair_len_kernel(int nsurv, const long long* __restrict__ arc_len, long long* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsurv) out[i] = arc_len[2 * i] + arc_len[2 * i + 1];
}

}  // namespace dmsc
