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
#include "replay.cuh"

namespace dmsc {

constexpr unsigned long long kNoEdge = ~0ull;

// Sweep key of saddle e (list index) on one side: the side sweeps its image's
// saddles in ascending (s_val, cell id) order, or exactly the reverse (desc;
// cpu/arcs_topology.hxx:99-102, 142). List indices ascend with the cell id
// inside an image, so (orderable(s_val), e) orders the ascending sweep and
// (~orderable(s_val), 0x7FFFFFFF - e) the descending one; both stay below
// kNoEdge, and keys of one image never meet another image's.
__device__ __forceinline__ unsigned long long sweep_key(float v, int e, bool desc) {
  const uint32_t o = orderable_key(v);
  return desc ? ((unsigned long long)(~o) << 32) | (uint32_t)(0x7FFFFFFF - e)
              : ((unsigned long long)o << 32) | (uint32_t)e;
}
__device__ __forceinline__ int sweep_key_saddle(unsigned long long k, bool desc) {
  const int lo = (int)(uint32_t)k;
  return desc ? 0x7FFFFFFF - lo : lo;
}
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

// K4: per saddle, both face walks and the vertex walks. Writes per saddle and
// side one record {target 0, target 1, cells 0, cells 1}: each arc's dense
// target index (or -1) and its raw arc's cell count; then runs the pairing's round-0 saddle phase for both sides (all
// groups are still single extrema, so the ends are the groups): a saddle
// whose two ends coincide is a cycle, the others record their ends' groups
// and reduce their sweep key into both groups' minimum, and each block adds
// the saddles that stay active to the side's round-1 counter.
__global__ void __launch_bounds__(256) saddle_walk_kernel(Imgs I, const uint8_t* __restrict__ flow, int nsad,
                                                          const int* __restrict__ crit_sad,
                                                          const int* __restrict__ sad_img,
                                                          const int* __restrict__ off_max,
                                                          const uint32_t* __restrict__ max_bits,
                                                          const int* __restrict__ off_min,
                                                          const uint32_t* __restrict__ min_bits,
                                                          int4* __restrict__ arc_f, int4* __restrict__ arc_v,
                                                          long long cap, PairStart ps, unsigned* status) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  int keep[2] = {0, 0};
  if (s < nsad) {
    const int b = sad_img[s];
    const int H = I.H[b], W = I.W[b], Nx = W + 1;
    const int sc = crit_sad[s];
    int te[2][2], len[2][2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      long long steps;
      const int end = flow_walk<4>(flow, face_start(sc, j, Nx) >> 2, Nx, cap, &steps, status);
      const int target = seg_rank(I, b, end, Nx, off_max, max_bits);
      te[0][j] = target;
      len[0][j] = target >= 0 ? (int)steps + 1 : 0;  // cells of the raw arc, start and end included
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int start = vertex_start(sc, j, H, W, Nx, I.idx_base[b]);
      long long steps = 0;
      int target = -1;
      if (start >= 0) {
        const int end = flow_walk<0>(flow, start >> 2, Nx, cap, &steps, status);
        target = seg_rank(I, b, end, Nx, off_min, min_bits);
      }
      te[1][j] = target;
      len[1][j] = target >= 0 ? (int)steps + 1 : 0;  // an arc that leaves the image is empty
    }
    // a raw arc has fewer cells than the batch (cell ids are int32)
    arc_f[s] = make_int4(te[0][0], te[0][1], len[0][0], len[0][1]);
    arc_v[s] = make_int4(te[1][0], te[1][1], len[1][0], len[1][1]);
    // round 0 of the pairing: descending sweep on the face side in the
    // primal and the vertex side in the dual
    const bool d = I.dual[b];
    const float v = ps.sval[s];
#pragma unroll
    for (int sd = 0; sd < 2; ++sd) {
      const int M = ps.M[sd];
      const int ga = te[sd][0] < 0 ? M : te[sd][0], gb = te[sd][1] < 0 ? M : te[sd][1];
      if (ga == gb) {
        ps.dying[sd][s] = -1;
        continue;
      }
      ps.dying[sd][s] = kUndecided;
      ps.g12[sd][s] = make_int2(ga, gb);
      const unsigned long long k = sweep_key(v, s, sd == 0 ? !d : d);
      atomicMin(ps.minedge[sd] + ga, k);  // result unused: a reduction
      atomicMin(ps.minedge[sd] + gb, k);
      keep[sd] = 1;
    }
  }
  const int c0 = __syncthreads_count(keep[0]), c1 = __syncthreads_count(keep[1]);
  if (threadIdx.x == 0) {
    if (c0) atomicAdd(ps.cnt[0] + 1, c0);
    if (c1) atomicAdd(ps.cnt[1] + 1, c1);
  }
}

__global__ void iota_kernel(int* __restrict__ a, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// Persistence of each decided saddle and cancellation (persistence.hxx:82-104,
// 139-161), with the saddle's image's orientation and threshold: pp[s] =
// (paired extremum or -1, persistence bits; -1 for a cycle); `sbit` marks the
// side in `cancelled`.
__global__ void __launch_bounds__(256) persistence_kernel(int nsad, bool min_side, const uint8_t* __restrict__ dual,
                                                          const float* __restrict__ thr,
                                                          const int* __restrict__ sad_img,
                                                          const int* __restrict__ dying,
                                                          const float* __restrict__ sad_val,
                                                          const int2* __restrict__ ext_key,
                                                          int2* __restrict__ pp,
                                                          uint8_t* __restrict__ cancelled, uint8_t sbit,
                                                          uint8_t* __restrict__ alive, int* __restrict__ n_cancel,
                                                          const int4* __restrict__ arc,
                                                          int2* __restrict__ canc_ends,
                                                          const int* __restrict__ crit_sad,
                                                          unsigned long long* __restrict__ ckey,
                                                          int* __restrict__ cval, ReplayNode* __restrict__ node) {
  // saddles in list order: every per-saddle access is sequential
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  bool canc = false;
  int d = -1;
  float p = -1.0f;
  if (s < nsad) {
    d = dying[s];
    if (d < 0) {
      d = -1;
    } else {
      const int b = sad_img[s];
      const bool du = dual[b];
      float sv = sad_val[s], ev = __int_as_float(ext_key[d].x);
      if (min_side)
        p = du ? sub_like_host(ev, sv) : sub_like_host(sv, ev);
      else
        p = du ? sub_like_host(sv, ev) : sub_like_host(ev, sv);
      if (p <= thr[b]) {
        canc = true;
        atomicOr((unsigned*)(cancelled + (s & ~3)), (unsigned)sbit << (8 * (s & 3)));
        alive[d] = 0;
      }
    }
    pp[s] = make_int2(d, __float_as_int(p));
  }
  // cancelled edges' ends, compacted for the thresholded union-find, and (when
  // the side's arcs are simplified) the same cancellations with their replay
  // keys (CancelEvent::operator<, cpu/persistence_struct.hxx:16-21):
  // (persistence, saddle cell); a saddle is cancelled at most once per side,
  // so the pair is unique and the target cell never breaks a tie
  const int slot = block_append(n_cancel, canc);
  if (canc) {
    const int4 a = arc[s];
    canc_ends[slot] = make_int2(a.x, a.y);
    if (ckey) {
      const unsigned long long key = ((unsigned long long)orderable_key(p) << 32) | (unsigned)crit_sad[s];
      ckey[slot] = key;
      cval[slot] = s;
      // the killed extremum's replay record: its cancellation key, undecided
      // (the other records are never read, see replay.cuh)
      node[d].ctime = key;
      node[d].status = kPending;
    }
  }
}


// Thresholded union-find (the reference's uf_min / uf_max, persistence.hxx:
// 90-104, 147-161): lock-free union of the ends of every cancelled saddle
// (link the larger root under the smaller), over the compact list of
// cancelled edges written by persistence_kernel. Every link points to a
// smaller index, so a root search takes at most n steps and every failed CAS
// means another thread linked one of the two roots (at most n - 1 links
// exist); both loops are capped at `cap` anyway, and a cap sets
// kStatusFindCap and returns the node reached (a valid index). One edge per
// thread: advancing 4 edges' searches in lockstep measured slower here (the
// forest is deep while the unions run, and a thread waits for its longest).
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

__global__ void __launch_bounds__(256) ut_union_kernel(const int2* __restrict__ ends, const int* __restrict__ count,
                                                       int void_id, int* __restrict__ p, int cap,
                                                       unsigned* status) {
  const int n = *count;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int2 e = ends[q];
    int a = e.x < 0 ? void_id : e.x;
    int b = e.y < 0 ? void_id : e.y;
    for (int tries = 0;; ++tries) {
      if (tries >= cap) {
        set_status(status, kStatusFindCap);
        break;
      }
      a = uf_root(p, a, cap, status);
      b = uf_root(p, b, cap, status);
      if (a == b) break;
      if (a > b) {
        int t = a;
        a = b;
        b = t;
      }
      if (atomicCAS(p + b, b, a) == b) break;
    }
  }
}

constexpr int kUtBatch = 4;

// Every node's root, kUtBatch nodes per thread with their pointer chains
// followed in lockstep (a written root is an ancestor for every reader).
__global__ void ut_flatten_kernel(int n, int* __restrict__ p, int cap, unsigned* status) {
  const long long nt = (long long)gridDim.x * blockDim.x;
  const long long x0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int r[kUtBatch];
  unsigned live = 0;
#pragma unroll
  for (int u = 0; u < kUtBatch; ++u) {
    const long long x = x0 + nt * u;
    r[u] = (int)x;
    if (x < n) live |= 1u << u;
  }
  const unsigned own = live;
  for (int k = 0; live; ++k) {
    if (k >= cap) {
      set_status(status, kStatusFindCap);
      break;
    }
    int pr[kUtBatch];
#pragma unroll
    for (int u = 0; u < kUtBatch; ++u) pr[u] = ((live >> u) & 1u) ? p[r[u]] : r[u];
#pragma unroll
    for (int u = 0; u < kUtBatch; ++u) {
      if (pr[u] == r[u]) live &= ~(1u << u);
      r[u] = pr[u];
    }
  }
#pragma unroll
  for (int u = 0; u < kUtBatch; ++u)
    if ((own >> u) & 1u) p[x0 + nt * u] = r[u];
}

// Component root = its alive member, or -1 for the void's component.
__global__ void ut_mark_kernel(int n_ext, const int* __restrict__ p, const uint8_t* __restrict__ alive,
                               int* __restrict__ comp_root) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x > n_ext) return;
  if (x == n_ext)
    comp_root[p[x]] = -1;
  else if (alive[x])
    comp_root[p[x]] = x;
}

// Out rank of each extremum's thresholded root: the component's alive
// member (comp_root of its flattened union-find root; -1 for the void's
// component), which always has an out rank.
__global__ void root_out_kernel(int n_ext, const int* __restrict__ p, const int* __restrict__ comp_root,
                                const int* __restrict__ to_out, int* __restrict__ rout) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_ext) return;
  const int u = comp_root[p[x]];
  rout[x] = u >= 0 ? to_out[u] : -1;
}

}  // namespace dmsc
