// Output assembly on the device (cpu/workspace.hxx:86-365), for a batch.
//
// Per image: surviving extrema keep their ascending-cell-id order; surviving
// saddles are listed in minima-sweep order; e_min rows follow the minima sweep
// and e_max rows the maxima sweep, which is the reverse of the minima sweep
// for the same saddles (cpu/arcs_topology.hxx:142). Internal side 0 is the
// faces, side 1 the vertices; in the primal the faces are the maxima, in the
// dual the minima (workspace.hxx:322-362), so every side's per-image output
// goes to the array that image's orientation selects, at an offset the host
// computed from the per-image sizes. All written ids are image-local.
#pragma once

#include "common.cuh"

namespace dmsc {

// Destination of one side's per-image output: the array picked by the
// image's orientation, at the image's offset in it.
struct Route {
  int* primal;
  int* dual;
  const int* off;  // [B]
  __device__ __forceinline__ int* at(bool d, int b) const {
    int* p = d ? dual : primal;
    return p ? p + off[b] : nullptr;
  }
};
struct RouteF {
  float* primal;
  float* dual;
  const int* off;
  __device__ __forceinline__ float* at(bool d, int b) const {
    float* p = d ? dual : primal;
    return p ? p + off[b] : nullptr;
  }
};

__global__ void u8_to_int_kernel(const uint8_t* __restrict__ a, int n, int* __restrict__ b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// to_out[x] = batch-wide output rank of alive extremum x (-1 otherwise).
__global__ void to_out_kernel(int n, const uint8_t* __restrict__ alive, const int* __restrict__ to_out_excl,
                              int* __restrict__ to_out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < n) to_out[x] = alive[x] ? to_out_excl[x] : -1;
}

// Surviving extrema, image-local cell ids, into the routed point lists.
__global__ void points_kernel(int n, const uint8_t* __restrict__ alive, const int* __restrict__ to_out_excl,
                              const int* __restrict__ alive_base, const int2* __restrict__ key,
                              const int* __restrict__ ext_img, Imgs I, Route R) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n || !alive[x]) return;
  int b = ext_img[x];
  int* dst = R.at(I.dual[b], b);
  if (dst) dst[to_out_excl[x] - alive_base[b]] = key[x].y - 4 * I.idx_base[b];
}

// flag[s] = 1 when saddle s (list order) survives both sides.
__global__ void survivor_flag_kernel(int nsad, const uint8_t* __restrict__ cancelled, int* __restrict__ flag) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsad) return;
  flag[s] = cancelled[s] == 0;
}

// The survivors in list order with their sort keys ((image, s_val) order:
// the image id above the orderable value, so one sort orders every image;
// a 32-bit key of the value alone for one image).
template <class K>
__global__ void survivor_gather_kernel(int nsad, const int* __restrict__ flag, const int* __restrict__ pos,
                                       const float* __restrict__ sval, const int* __restrict__ sad_img,
                                       K* __restrict__ key_out, int* __restrict__ idx_out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsad || !flag[s]) return;
  const uint32_t o = orderable_key(sval[s]);
  key_out[pos[s]] = sizeof(K) > 4 ? (K)(((unsigned long long)sad_img[s] << 32) | o) : (K)o;
  idx_out[pos[s]] = s;
}

// Surviving saddles in the vertex side's sweep order (arcs_topology.hxx:99-102):
// `sorted` lists them by ascending (image, s_val, cell id); an image whose
// vertex side sweeps descending (dual) takes its range reversed. Also
// gathers each survivor's image and cell in output order (`ic`), so the
// later per-survivor kernels read them in order.
__global__ void survivor_order_kernel(int n, const int* __restrict__ sorted, const int* __restrict__ sad_img,
                                      const int* __restrict__ crit_sad, const uint8_t* __restrict__ dual,
                                      const int* __restrict__ surv_base, int* __restrict__ surv,
                                      int2* __restrict__ ic) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int s = sorted[p], b = sad_img[s];
  int q = p;
  if (dual[b]) {
    const int base = surv_base[b], cnt = surv_base[b + 1] - base;
    q = base + cnt - 1 - (p - base);
  }
  surv[q] = s;
  ic[q] = make_int2(b, crit_sad[s]);
}

// Per-survivor records of one side gathered once in output (sweep) order, so
// the later per-survivor kernels read them in order instead of gathering
// from the list-ordered saddle arrays again: its arc ends, raw-arc lengths
// and the record of its outputs (out ranks of its ends' thresholded roots,
// persistence, out rank of its pair's root; -1 for the void).
__global__ void surv_side_kernel(int nsurv, const int* __restrict__ surv, const int4* __restrict__ arc,
                                 const int2* __restrict__ pp, const int* __restrict__ rout, int2* __restrict__ sv_t,
                                 longlong2* __restrict__ sv_len, int4* __restrict__ sv_rec) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv) return;
  const int s = surv[i];
  const int4 a = arc[s];
  const int2 pr = pp[s];
  sv_t[i] = make_int2(a.x, a.y);
  sv_len[i] = make_longlong2(a.z, a.w);
  sv_rec[i] = make_int4(a.x >= 0 ? rout[a.x] : -1, a.y >= 0 ? rout[a.y] : -1, pr.y, pr.x >= 0 ? rout[pr.x] : -1);
}

// Per-image first positions (B + 1 entries, the last one the total):
// base[b] = excl[first[b]] where first[] are the image's first items.
__global__ void image_base_kernel(int B, const int* __restrict__ first, int n_items, const int* __restrict__ excl,
                                  int total, int* __restrict__ base) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > B) return;
  int f = b < B ? first[b] : n_items;
  base[b] = f < n_items ? excl[f] : total;
}

// The same with the total read from the device.
__global__ void image_base_dev_kernel(int B, const int* __restrict__ first, int n_items, const int* __restrict__ excl,
                                      const long long* __restrict__ total, int* __restrict__ base) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > B) return;
  int f = b < B ? first[b] : n_items;
  base[b] = f < n_items ? excl[f] : (int)*total;
}

// The survivor of output position q when an image's survivors are visited in
// reverse (maxima sweep) or forward (minima sweep) order.
__device__ __forceinline__ int visit(int q, bool reversed, const int* __restrict__ surv_base, int B, int* b_out) {
  int b = find_image(surv_base, B, q);
  *b_out = b;
  if (!reversed) return q;
  int base = surv_base[b], n = surv_base[b + 1] - base;
  return base + n - 1 - (q - base);
}

// e rows of one survivor (cpu/workspace.hxx:175-195, 197-219) from the out
// ranks of its ends' roots (-1: the void; a thresholded root is always an
// alive extremum, so it always has an out rank): up to two ends.
__device__ __forceinline__ int erow_ends(int r1, int r2, int* o1, int* o2) {
  int n = 0;
  if (r1 != -1) {
    *o1 = r1;
    n = 1;
  }
  if (r1 != r2 && r2 != -1) {
    if (n == 0)
      *o1 = r2;
    else
      *o2 = r2;
    n++;
  }
  return n;
}

__global__ void erow_count_kernel(int nsurv, bool reversed, const int* __restrict__ surv_base, int B,
                                  const int4* __restrict__ sv_rec, int* __restrict__ cnt) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsurv) return;
  int b;
  const int i = visit(q, reversed, surv_base, B, &b);
  const int4 r = sv_rec[i];
  int a, c;
  cnt[q] = erow_ends(r.x, r.y, &a, &c);
}

// Per-survivor scalars and e rows of one side. `row_off` is the batch-wide
// exclusive scan of the row counts in visiting order; `row_base[b]` its value
// at image b's first survivor.
__global__ void side_outputs_kernel(int nsurv, bool reversed, const int* __restrict__ surv_base, Imgs I,
                                    const int4* __restrict__ sv_rec, const int* __restrict__ alive_base,
                                    const int* __restrict__ row_off, const int* __restrict__ row_base, RouteF P,
                                    Route PP, Route E) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsurv) return;
  int b;
  int i = visit(q, reversed, surv_base, I.B, &b);
  const bool d = I.dual[b];
  const int li = i - surv_base[b];
  const int4 r = sv_rec[i];
  if (float* p = P.at(d, b)) p[li] = __int_as_float(r.z);
  if (int* pp = PP.at(d, b)) pp[li] = r.w >= 0 ? r.w - alive_base[b] : -1;
  if (int* e = E.at(d, b)) {
    int a = 0, c = 0;
    int n = erow_ends(r.x, r.y, &a, &c);
    int o = row_off[q] - row_base[b];
    if (n >= 1) {
      e[2 * o] = li;
      e[2 * o + 1] = a - alive_base[b];
    }
    if (n == 2) {
      e[2 * o + 2] = li;
      e[2 * o + 3] = c - alive_base[b];
    }
  }
}

__global__ void sad_pts_kernel(int nsurv, const int2* __restrict__ surv_ic, const int* __restrict__ surv_base, Imgs I,
                               int* __restrict__ out, const int* __restrict__ out_off) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv) return;
  const int2 ic = surv_ic[i];
  const int b = ic.x;
  out[out_off[b] + (i - surv_base[b])] = ic.y - 4 * I.idx_base[b];
}

// Geometry start of every image on one side (B + 1 entries).
__global__ void geom_base_kernel(int B, const int* __restrict__ surv_base, int nsurv,
                                 const long long* __restrict__ saddle_end_incl, const long long* __restrict__ plen,
                                 const long long* __restrict__ total, long long* __restrict__ gbase) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > B) return;
  int f = b < B ? surv_base[b] : nsurv;
  gbase[b] = f < nsurv ? saddle_end_incl[f] - plen[f] : *total;
}

// Image-local output position of every arc (its start inside its image's
// geometry of this side), for the geometry expansion and writer.
__global__ void arc_pos_kernel(int nsurv, const long long* __restrict__ arc_len,
                               const long long* __restrict__ saddle_end_incl, const int2* __restrict__ surv_ic,
                               const long long* __restrict__ gbase, long long* __restrict__ arc_pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv) return;
  const longlong2 al = *reinterpret_cast<const longlong2*>(arc_len + 2 * i);
  const long long start = saddle_end_incl[i] - gbase[surv_ic[i].x] - al.x - al.y;
  *reinterpret_cast<longlong2*>(arc_pos + 2 * i) = make_longlong2(start, start + al.x);
}

// CSR offsets of one side's arcs, per image (cpu/workspace.hxx:247-287):
// offsets[0] = 0, offsets[k+1] = end of survivor k, arc_offsets[k] = end of
// its first arc, image-local. `off_off[b]` / `arc_off[b]` place image b's
// block (n_b + 1 and n_b entries) in the routed arrays.
__global__ void arc_offsets_kernel(int nsurv, int B, const int* __restrict__ surv_base, const uint8_t* __restrict__ dual,
                                   const long long* __restrict__ arc_len,
                                   const long long* __restrict__ saddle_end_incl, const long long* __restrict__ gbase,
                                   Route OFF, Route AOFF) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv + B) return;
  if (i >= nsurv) {  // one leading zero per image
    int b = i - nsurv;
    if (int* o = OFF.at(dual[b], b)) o[0] = 0;
    return;
  }
  int b = find_image(surv_base, B, i);
  const bool d = dual[b];
  const longlong2 al = *reinterpret_cast<const longlong2*>(arc_len + 2 * i);
  long long end = saddle_end_incl[i] - gbase[b];
  long long start = end - al.x - al.y;
  int li = i - surv_base[b];
  if (int* o = OFF.at(d, b)) o[li + 1] = (int)end;
  if (int* a = AOFF.at(d, b)) a[li] = (int)(start + al.x);
}

}  // namespace dmsc
