// Persistence pairing and cancellation on the device.
//
// Reference semantics: cpu/persistence.hxx:16-182. Each side is a sequential
// union-find sweep over the saddles in sweep order (ascending (s_val, cell id)
// for minima in the primal, the reverse for maxima; flipped in the dual)
// with the elder rule: at a saddle joining two components the one whose
// oldest extremum is younger dies, and the void (-1, one-sided saddles) is
// older than every extremum.
//
// Parallel form (exact). Groups start as single extrema plus the void; a
// group is named by its oldest member. Every round, each group takes the
// first (lowest sweep index) saddle leaving it; a group whose partner group
// has an older oldest member dies at that saddle, which pairs the saddle with
// the group's oldest member, and joins the partner. Saddles whose ends fall
// in one group are cycles (pair -1, persistence -1). Why this equals the
// sweep: a group is always connected, by the time any of its outgoing saddles
// is swept, to its oldest member, so at its first outgoing saddle the dying
// side is exactly known; the globally first remaining saddle is always
// decided, so every round makes progress.
//
// The thresholded union-find (the reference's uf_min / uf_max) ends with one
// component per connected set of cancelled saddles; its root is the unique
// member not killed by a cancelled saddle, or the void.
#pragma once

#include <cuda/atomic>

#include "common.cuh"

namespace dmsc {

constexpr uint32_t kNoEdge = 0xFFFFFFFFu;
constexpr int kUndecided = -2;

// older(a, b) for extremum dense indices of one image; `void_id` is older
// than all. Older = smaller (value, cell) under value_less on the vertex side
// in the primal and the face side in the dual, larger otherwise.
// `key[x]` = (value bits, cell) of extremum x, one 8-byte record per extremum.
__device__ __forceinline__ bool older(int a, int b, int void_id, const int2* __restrict__ key, bool older_less) {
  if (a == void_id) return b != void_id;
  if (b == void_id) return false;
  const int2 ka = key[a], kb = key[b];
  const float va = __int_as_float(ka.x), vb = __int_as_float(kb.x);
  return older_less ? tie_lt(va, ka.y, vb, kb.y) : tie_lt(vb, kb.y, va, ka.y);
}

__global__ void iota_kernel(int* __restrict__ a, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// Sweep-ordered edge list of one side for a batch. `asc` lists every image's
// saddles in ascending (s_val, cell id), images in order; the face side sweeps
// each image descending in the primal and ascending in the dual, the vertex
// side the reverse (cpu/arcs_topology.hxx:99-102, 142). Edge q is saddle
// sweep[q] with ends (t[2s], t[2s+1]); an image's edges stay contiguous.
__global__ void sweep_edges_kernel(int nsad, const int* __restrict__ asc, const int* __restrict__ sad_img,
                                   const int* __restrict__ sad_base, const uint8_t* __restrict__ dual, bool faces,
                                   const int* __restrict__ t, int* __restrict__ sweep, int* __restrict__ rank,
                                   int* __restrict__ c1, int* __restrict__ c2) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nsad) return;
  int s = asc[p];
  int b = sad_img[s];
  int base = sad_base[b], n = sad_base[b + 1] - base;
  bool rev = faces ? !dual[b] : dual[b];
  int q = rev ? base + n - 1 - (p - base) : p;
  sweep[q] = s;
  rank[s] = q;  // sweep position of the saddle with list index s
  c1[q] = t[2 * s];
  c2[q] = t[2 * s + 1];
}

// The pairing works on saddles in list order (ascending cell id, so the
// saddles a block handles touch extrema close to each other); its results go
// back to sweep order for the later stages: dying[q] and the deciding groups
// g12[q] of sweep position q.
__global__ void pair_to_sweep_kernel(int nsad, const int* __restrict__ sweep, const int* __restrict__ dying_l,
                                     const int2* __restrict__ g12_l, int* __restrict__ dying,
                                     int2* __restrict__ g12) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsad) return;
  const int s = sweep[q];
  dying[q] = dying_l[s];
  g12[q] = g12_l[s];
}

// Persistence of each decided saddle and cancellation (persistence.hxx:82-104,
// 139-161), with the saddle's image's orientation and threshold; `sbit` marks
// the side in `cancelled`.
__global__ void __launch_bounds__(256) persistence_kernel(int nsad, bool min_side, const uint8_t* __restrict__ dual,
                                                          const float* __restrict__ thr,
                                                          const int* __restrict__ sad_img,
                                                          const int* __restrict__ sweep,
                                                          const int* __restrict__ dying,
                                                          const float* __restrict__ sad_val,
                                                          const float* __restrict__ ext_val,
                                                          int* __restrict__ pair_dense, float* __restrict__ pers,
                                                          uint8_t* __restrict__ cancelled, uint8_t sbit,
                                                          uint8_t* __restrict__ alive, int* __restrict__ n_cancel,
                                                          const int* __restrict__ c1, const int* __restrict__ c2,
                                                          const int2* __restrict__ g12, int void_id,
                                                          int* __restrict__ cparent) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  bool canc = false;
  if (j < nsad) {
    int s = sweep[j], d = dying[j];
    if (d < 0) {
      pair_dense[s] = -1;
      pers[s] = -1.0f;
    } else {
      const int b = sad_img[s];
      const bool du = dual[b];
      float sv = sad_val[s], ev = ext_val[d];
      float p;
      if (min_side)
        p = du ? sub_like_host(ev, sv) : sub_like_host(sv, ev);
      else
        p = du ? sub_like_host(sv, ev) : sub_like_host(ev, sv);
      pair_dense[s] = d;
      pers[s] = p;
      if (p <= thr[b]) {
        canc = true;
        atomicOr((unsigned*)(cancelled + (s & ~3)), (unsigned)sbit << (8 * (s & 3)));
        alive[d] = 0;
        // the dying group hangs under the saddle's other end (g12: the two
        // ends' groups when the saddle was decided; d is one of them)
        const int other = g12[j].x == d ? c2[j] : c1[j];
        cparent[d] = other < 0 ? void_id : other;
      }
    }
  }
  block_append(n_cancel, canc);  // cancellation count (the replay runs only where it is not 0)
}

// Thresholded union-find (the reference's uf_min / uf_max, persistence.hxx:
// 90-104, 147-161): its components are those of the cancelled saddles, and
// the reference's unite_from_root always hangs the dying end's root under the
// surviving end's, so a component's root is its one member not killed by a
// cancelled saddle, or the void. Here a cancelled death at saddle e hangs the
// dying group's oldest member d under e's surviving end (persistence_kernel,
// `cparent`); d and e's dying end lie in one component already, because every
// earlier merge into d's group was cancelled too (swept earlier, so its saddle
// value is not above e's, and its dying extremum is not older than d, so its
// float persistence is not larger). Each extremum dies at most once, so
// `cparent` is a forest whose roots are the surviving members; the root of x
// is found with path halving (pointers only move to ancestors), capped at
// `cap` steps (kStatusFindCap, then the node reached).
__device__ __forceinline__ int uf_root(int* p, int x, int cap, unsigned* status) {
  for (int k = 0;; ++k) {
    int px = p[x];
    if (px == x) return x;
    if (k >= cap) {
      set_status(status, kStatusFindCap);
      return x;
    }
    int ppx = p[px];
    if (ppx != px) p[x] = ppx;  // path halving; benign race
    x = ppx;
  }
}

// ut[x] = the surviving member of x's component, -1 for the void's.
__global__ void ut_root_kernel(int n_ext, int* __restrict__ cparent, int* __restrict__ ut, int cap,
                               unsigned* status) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_ext) return;
  const int r = uf_root(cparent, x, cap, status);
  ut[x] = r == n_ext ? -1 : r;
}

}  // namespace dmsc
