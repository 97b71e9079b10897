// Discrete gradient (steepest lower-star pairing) and ordered critical-cell
// compaction.
//
// Reference semantics: cpu/gradient.hxx:19-196 (compute_gradient),
// cpu/critical_points.hxx:14-65 (extract_critical_points, canonical order =
// ascending cell id), cpu/gradient.hxx:198-231 (fast_crit_map and values).
//
// Layout. The gradient array holds 4 int32 slots per index (y, x) of the
// (H+1) x (W+1) index grid, i.e. 16 bytes per index; it is the grad_indices
// output. One CTA owns a 32 x 64 tile of indices and writes it with one int4
// store per index, so every warp writes 512 contiguous bytes per row. The
// cells at a tile's indices are owned (have their highest vertex) in the
// pixels of the tile plus one halo row above and one halo column to the left,
// so the CTA evaluates the lower star of (64+1) x (32+1) pixels from a (64+3) x (32+3)
// value tile in shared memory, one 32-bit pairing word per pixel, and every
// index then gathers its four slots from the words of their owners. Slots of
// invalid cells are -1.
//
// The same pass writes one criticality byte per index (bit t = slot t is an
// unpaired valid cell) and per-(row, 32-column segment) counts of minima,
// saddles and maxima; a scan over the segments in row-major order gives every
// critical cell its position in the ascending-cell-id lists.
#pragma once

#include "common.cuh"

namespace dmsc {

constexpr int kTileX = 32;  // indices per tile row (one warp)
constexpr int kTileY = 64;  // tile rows
constexpr int kValX = kTileX + 3;
constexpr int kValY = kTileY + 3;

// Face-edge pairing FIFO of one lower star (cpu/gradient.hxx:115-191) as a
// pure function of eL (lower-star edge slots), fL (lower-star face slots) and
// `best` (edge slot paired with the vertex, -1 for none). Result: 4 bits per
// edge slot (4 = vertex, 0..3 = face slot, 15 = unpaired) in the low half and
// 4 bits per face slot (edge slot or 15) in the high half. Edge slots
// e0 = H(y,x), e1 = H(y,x+1), e2 = V(y,x), e3 = V(y+1,x); face slots
// f0 = F(y,x), f1 = F(y,x+1), f2 = F(y+1,x), f3 = F(y+1,x+1). Face f's
// candidate edges in the reference visiting order are (f & 1, 2 + (f >> 1));
// edge e bounds faces (e, e+2) for e < 2 and (2(e-2), 2(e-2)+1) otherwise.
inline uint32_t face_fifo_entry(unsigned eL, unsigned fL, int best) {
  unsigned epk = 0xFFFFu, fpk = 0xFFFFu, epaired = 0, fpaired = 0;
  if (best >= 0) {
    epk = (epk & ~(0xFu << (4 * best))) | (4u << (4 * best));
    epaired = 1u << best;
  }
  int q[16], head = 0, tail = 0;
  for (int f = 0; f < 4; ++f)
    if ((fL >> f) & 1u) q[tail++] = f;
  while (head < tail) {
    const int f = q[head++];
    if ((fpaired >> f) & 1u) continue;
    const int ea = f & 1, eb = 2 + (f >> 1);
    const bool ua = ((eL >> ea) & 1u) && !((epaired >> ea) & 1u);
    const bool ub = ((eL >> eb) & 1u) && !((epaired >> eb) & 1u);
    if (ua == ub) continue;  // zero or two unpaired lower-star edges
    const int e = ua ? ea : eb;
    fpk = (fpk & ~(0xFu << (4 * f))) | ((unsigned)e << (4 * f));
    fpaired |= 1u << f;
    epk = (epk & ~(0xFu << (4 * e))) | ((unsigned)f << (4 * e));
    epaired |= 1u << e;
    const int nb[2] = {e < 2 ? e : 2 * (e - 2), e < 2 ? e + 2 : 2 * (e - 2) + 1};
    for (int k = 0; k < 2; ++k) {
      const int nf = nb[k];
      if (nf == f || !((fL >> nf) & 1u) || ((fpaired >> nf) & 1u)) continue;
      bool already = false;
      for (int qi = head; qi < tail; ++qi)
        if (q[qi] == nf) already = true;
      if (!already && tail < 16) q[tail++] = nf;
    }
  }
  return (fpk << 16) | epk;
}

// Nibble value of a slot whose cell is not in this pixel's lower star (the
// cell belongs to a neighbour, or does not exist).
constexpr unsigned kNotMine = 14u;
// Word of a pixel outside the image: it owns no cell.
constexpr uint32_t kNoPixel = 0xEEEEEEEEu;

// All 16 x 16 x 5 entries, indexed ((eL << 4) | fL) * 5 + best + 1: the
// pairing word of a pixel. Nibbles 0-3 describe edge slots 0-3 (4 = paired
// with the vertex, 0..3 = paired with that face slot, 15 = critical, 14 = not
// in the lower star), nibbles 4-7 face slots 0-3 (0..3 = paired with that
// edge slot, 15 = critical, 14 = not in the lower star).
inline void face_fifo_table(uint32_t* out) {
  for (unsigned eL = 0; eL < 16; ++eL)
    for (unsigned fL = 0; fL < 16; ++fL)
      for (int b = -1; b < 4; ++b) {
        uint32_t w = face_fifo_entry(eL, fL, b);
        for (int k = 0; k < 4; ++k) {
          if (!((eL >> k) & 1u)) w = (w & ~(0xFu << (4 * k))) | (kNotMine << (4 * k));
          if (!((fL >> k) & 1u)) w = (w & ~(0xFu << (16 + 4 * k))) | (kNotMine << (16 + 4 * k));
        }
        out[((eL << 4) | fL) * 5 + (b + 1)] = w;
      }
}
constexpr int kFifoTable = 16 * 16 * 5;

// 16 warps; each thread evaluates about 4 of the (kTileY + 1) x (kTileX + 1)
// lower stars of a tile and each warp writes kTileY / 16 of its rows, so one
// CTA's global loads (all issued before their first use) are amortised over
// 2048 indices.
constexpr int kGradThreads = 512;
constexpr int kGradWarps = kGradThreads / 32;

// v_greater (cpu/cell_compare.hxx:23-31) orders pixels by (value, y*W+x),
// flipped in the dual. gt(a, b) when a's linear id is known to be larger (a "after" b) or smaller:
// the (value, id) tie rule then reduces to one float compare.
//   primal: after -> !(a < b), before -> (b < a); dual: after -> (a < b), before -> !(b < a)
template <bool DUAL>
__device__ __forceinline__ bool gt_after(float a, float b) {
  return DUAL ? (a < b) : !(a < b);
}
template <bool DUAL>
__device__ __forceinline__ bool gt_before(float a, float b) {
  return DUAL ? !(b < a) : (b < a);
}

// Lower star of pixel (y, x) and its pairing (cpu/gradient.hxx:48-192), all in
// registers. The highest-vertex scans keep the reference's candidate order
// (cpu/cell_compare.hxx:33-63), so ties and non-finite values resolve the same
// way. Edge slots: e0 = H(y,x), e1 = H(y,x+1), e2 = V(y,x), e3 = V(y+1,x);
// face slots: f0 = F(y,x), f1 = F(y,x+1), f2 = F(y+1,x), f3 = F(y+1,x+1).
// Returns the pixel's pairing word (face_fifo_table).
template <bool DUAL, bool INTERIOR = false>
__device__ __forceinline__ uint32_t lower_star(const float (*sv)[kValX], int y, int x, int H, int W, int ty0, int tx0,
                                               const uint32_t* __restrict__ fifo_lut) {
  // 3x3 neighbourhood; r, c index the value tile (origin y0-2, x0-2)
  const int r = y - (ty0 - 2), c = x - (tx0 - 2);
  // INTERIOR: every neighbour of the pixel is in the image
  const bool lv = INTERIOR || x >= 1, rv = INTERIOR || x + 1 < W, uv = INTERIOR || y >= 1, dv = INTERIOR || y + 1 < H;
  // row-major linear order of the 3x3 neighbourhood: UL < U < UR < L < P < R < DL < D < DR
  const float P = sv[r][c];
  const float L = sv[r][c - 1], R = sv[r][c + 1];
  const float U = sv[r - 1][c], D = sv[r + 1][c];
  const float UL = sv[r - 1][c - 1], UR = sv[r - 1][c + 1];
  const float DL = sv[r + 1][c - 1], DR = sv[r + 1][c + 1];
#define GT_A(a, b) gt_after<DUAL>(a, b)   /* a after b */
#define GT_B(a, b) gt_before<DUAL>(a, b)  /* a before b */

  const bool p_gt_l = lv && GT_A(P, L);
  const bool r_gt_p = rv && GT_A(R, P);
  const bool p_gt_u = uv && GT_A(P, U);
  const bool d_gt_p = dv && GT_A(D, P);

  unsigned eL = 0, fL = 0;
  if (!lv || p_gt_l) eL |= 1u;
  if (!r_gt_p) eL |= 2u;
  if (!uv || p_gt_u) eL |= 4u;
  if (!d_gt_p) eL |= 8u;
  {  // f0 = F(y,x): scan UL, U, L, then P (each later candidate is after the earlier ones)
    bool p_top;
    if (uv && lv) {
      // best of UL, U, L
      int b = GT_A(U, UL) ? 1 : 0;  // 0 = UL, 1 = U
      float bv = b ? U : UL;
      if (GT_A(L, bv)) {
        bv = L;
      }
      p_top = GT_A(P, bv);
    } else if (uv) {
      p_top = GT_A(P, U);
    } else if (lv) {
      p_top = GT_A(P, L);
    } else {
      p_top = true;
    }
    if (p_top) fL |= 1u;
  }
  {  // f1 = F(y,x+1): scan U, UR, P, R
    bool p_best;
    if (uv) {
      float bv = (rv && GT_A(UR, U)) ? UR : U;  // U, UR both before P
      p_best = GT_A(P, bv);
    } else {
      p_best = true;
    }
    if (p_best && !r_gt_p) fL |= 2u;
  }
  {  // f2 = F(y+1,x): scan L, P, DL, D
    bool p_best = !lv || p_gt_l;
    if (p_best && dv && lv && GT_A(DL, P)) p_best = false;
    if (p_best && d_gt_p) p_best = false;
    if (p_best) fL |= 4u;
  }
  {  // f3 = F(y+1,x+1): scan P, R, D, DR
    bool p_best = !r_gt_p && !d_gt_p && !(dv && rv && GT_A(DR, P));
    if (p_best) fL |= 8u;
  }

  // vertex pairing: the lower-star edge whose other vertex is lowest
  // (candidates visited L, R, U, D; "bo greater than the new one" decides)
  int best = -1;
  float bo = 0.0f;
  if ((eL & 1u) && lv) {
    best = 0;
    bo = L;
  }
  if ((eL & 2u) && rv && (best < 0 || GT_B(bo, R))) {  // L before R
    best = 1;
    bo = R;
  }
  if ((eL & 4u) && uv && (best < 0 || GT_A(bo, U))) {  // L, R after U
    best = 2;
    bo = U;
  }
  if ((eL & 8u) && dv && (best < 0 || GT_B(bo, D))) {  // L, R, U before D
    best = 3;
    bo = D;
  }
#undef GT_A
#undef GT_B

  // face pairing: the FIFO of cpu/gradient.hxx:115-191 depends only on the
  // lower-star masks and the vertex-paired edge, so its result is looked up
  // (face_fifo_table() builds the 1280 entries with the same procedure).
  return __ldg(fifo_lut + (((eL << 4) | fL) * 5 + (best + 1)));
}

// Pairing words of the (kTileY + 1) x (kTileX + 1) pixels whose lower stars
// hold the cells of one 32 x kTileY index tile (origin pixel (y0 - 1, x0 - 1)).
// INTERIOR: the tile's value window lies inside the image, so no bound is tested.
template <bool DUAL, bool INTERIOR>
__device__ __forceinline__ void gradient_tile(const float* __restrict__ img, int H, int W, int y0, int x0, int tid,
                                              float (*sv)[kValX], uint32_t (*word)[kTileX + 1],
                                              const uint32_t* __restrict__ fifo_lut) {
  constexpr int kValN = kValY * kValX;
  constexpr int kLoads = (kValN + kGradThreads - 1) / kGradThreads;
  float v[kLoads];
#pragma unroll
  for (int k = 0; k < kLoads; ++k) {  // every load in flight before the first shared store
    const int i = tid + k * kGradThreads;
    const int r = i / kValX, c = i - r * kValX;
    const int gy = y0 - 2 + r, gx = x0 - 2 + c;
    v[k] = (i < kValN && (INTERIOR || (gy >= 0 && gy < H && gx >= 0 && gx < W))) ? __ldg(img + (size_t)gy * W + gx)
                                                                                  : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < kLoads; ++k) {
    const int i = tid + k * kGradThreads;
    if (i < kValN) (&sv[0][0])[i] = v[k];
  }
  __syncthreads();
  constexpr int kWordN = (kTileY + 1) * (kTileX + 1);
  for (int p = tid; p < kWordN; p += kGradThreads) {
    const int r = p / (kTileX + 1), c = p - r * (kTileX + 1);
    const int y = y0 - 1 + r, x = x0 - 1 + c;
    uint32_t w = kNoPixel;
    if (INTERIOR || (y >= 0 && y < H && x >= 0 && x < W)) w = lower_star<DUAL, INTERIOR>(sv, y, x, H, W, y0, x0, fifo_lut);
    word[r][c] = w;
  }
  __syncthreads();
}

// Cell of edge slot k / face slot f of the pixel at index `b`.
__device__ __forceinline__ int slot_edge_cell(int k, int b, int Nx) {
  return (1 + (k >> 1)) + 4 * (b + (k == 3 ? Nx : 0) + (k == 1 ? 1 : 0));
}
__device__ __forceinline__ int slot_face_cell(int f, int b, int Nx) { return 3 + 4 * (b + (f >> 1) * Nx + (f & 1)); }

// Write-out of tile row `warp` by one warp. Index (iy, ix) gathers its four
// slots from the pairing words of the pixels owning them: its vertex and
// (when owned there) its H edge, V edge and face from pixel (iy, ix), else
// the H edge from (iy, ix-1), the V edge from (iy-1, ix) and the face from
// (iy, ix-1), (iy-1, ix) or (iy-1, ix-1). Coalesced int4 gradient stores at
// global index base `gbase` (skipped when `grad` is null: the later stages
// read only the mask and flow codes), criticality mask, flow codes and the
// row segment's counts (segment id `seg`).
template <bool INTERIOR>
__device__ __forceinline__ void gradient_store_row(const uint32_t (*word)[kTileX + 1], int warp, int lane, int H,
                                                   int W, int iy, int ix, long long gbase, int seg,
                                                   int4* __restrict__ grad, uint8_t* __restrict__ crit_mask,
                                                   uint8_t* __restrict__ flow, int* __restrict__ seg_min,
                                                   int* __restrict__ seg_sad, int* __restrict__ seg_max) {
  const int Nx = W + 1;
  const bool in = INTERIOR || ix <= W;
  unsigned m = 0;
  if (in) {
    const uint32_t wP = word[warp + 1][lane + 1], wL = word[warp + 1][lane];
    const uint32_t wU = word[warp][lane + 1], wUL = word[warp][lane];
    const int b = iy * Nx + ix;  // image-local index: the cell ids written are local
    // vertex: the edge slot of its own pixel marked 4
    const unsigned e = wP & 0xFFFFu;
    const int vk = ((e & 0xFu) == 4u) ? 0 : (((e >> 4) & 0xFu) == 4u) ? 1 : (((e >> 8) & 0xFu) == 4u) ? 2
                 : (((e >> 12) & 0xFu) == 4u) ? 3 : -1;
    const int s0 = vk >= 0 ? slot_edge_cell(vk, b, Nx) : -1;
    // H edge (iy, ix): slot 0 of (iy, ix) or slot 1 of (iy, ix-1)
    const unsigned h0 = wP & 0xFu;
    const bool hown = h0 != kNotMine;
    const unsigned hn = hown ? h0 : ((wL >> 4) & 0xFu);
    const int hb = hown ? b : b - 1;
    const int s1 = hn == 4u ? 4 * hb : (hn < 4u ? slot_face_cell((int)hn, hb, Nx) : -1);
    // V edge (iy, ix): slot 2 of (iy, ix) or slot 3 of (iy-1, ix)
    const unsigned v0 = (wP >> 8) & 0xFu;
    const bool vown = v0 != kNotMine;
    const unsigned vn = vown ? v0 : ((wU >> 12) & 0xFu);
    const int vb = vown ? b : b - Nx;
    const int s2 = vn == 4u ? 4 * vb : (vn < 4u ? slot_face_cell((int)vn, vb, Nx) : -1);
    // face (iy, ix): face slot 0 of (iy, ix), 1 of (iy, ix-1), 2 of (iy-1, ix), 3 of (iy-1, ix-1)
    const unsigned f0 = (wP >> 16) & 0xFu, f1 = (wL >> 20) & 0xFu, f2 = (wU >> 24) & 0xFu, f3 = wUL >> 28;
    const unsigned fn = f0 != kNotMine ? f0 : f1 != kNotMine ? f1 : f2 != kNotMine ? f2 : f3;
    const int fb = f0 != kNotMine ? b : f1 != kNotMine ? b - 1 : f2 != kNotMine ? b - Nx : b - Nx - 1;
    const int s3 = fn < 4u ? slot_edge_cell((int)fn, fb, Nx) : -1;
    const size_t gidx = (size_t)(gbase + b);
    if (grad) grad[gidx] = make_int4(s0, s1, s2, s3);  // null when the gradient is not returned
    if (vk < 0 && (INTERIOR || (iy < H && ix < W))) m |= 1u;
    if (hn == 15u) m |= 2u;
    if (vn == 15u) m |= 4u;
    if (fn == 15u) m |= 8u;
    crit_mask[gidx] = (uint8_t)m;
    flow[gidx] = (uint8_t)((unsigned)(vk + 1) | (face_flow(s3, b) << 4));
  }
  unsigned bmin = __ballot_sync(0xffffffffu, m & 1u);
  unsigned bs1 = __ballot_sync(0xffffffffu, m & 2u);
  unsigned bs2 = __ballot_sync(0xffffffffu, m & 4u);
  unsigned bmax = __ballot_sync(0xffffffffu, m & 8u);
  if (lane == 0) {
    seg_min[seg] = __popc(bmin);
    seg_sad[seg] = __popc(bs1) + __popc(bs2);
    seg_max[seg] = __popc(bmax);
  }
}

// K1 (one image): gradient over one 32 x 64 index tile per CTA.
template <bool DUAL>
__global__ void __launch_bounds__(kGradThreads) gradient_kernel(const float* __restrict__ img, int H, int W,
                                                               int4* __restrict__ grad,
                                                               uint8_t* __restrict__ crit_mask,
                                                               int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                                               int* __restrict__ seg_max,
                                                               const uint32_t* __restrict__ fifo_lut,
                                                               uint8_t* __restrict__ flow) {
  __shared__ float sv[kValY][kValX];
  __shared__ uint32_t word[kTileY + 1][kTileX + 1];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY;
  gradient_tile<DUAL, false>(img, H, W, y0, x0, tid, sv, word, fifo_lut);
  const int warp = tid >> 5, lane = tid & 31;
  for (int rr = warp; rr < kTileY; rr += kGradWarps) {
    const int iy = y0 + rr, ix = x0 + lane;
    if (iy > H) break;  // uniform per warp
    gradient_store_row<false>(word, rr, lane, H, W, iy, ix, 0, iy * gridDim.x + blockIdx.x, grad, crit_mask, flow,
                              seg_min, seg_sad, seg_max);
  }
}

// K1 (batch): the tiles of every image of a batch in one 1-D grid; each CTA
// finds its image from the tile bases.
static __global__ void __launch_bounds__(kGradThreads) gradient_batch_kernel(Imgs I, const float* __restrict__ img_all,
                                                                     int4* __restrict__ grad,
                                                                     uint8_t* __restrict__ crit_mask,
                                                                     int* __restrict__ seg_min,
                                                                     int* __restrict__ seg_sad,
                                                                     int* __restrict__ seg_max,
                                                                     const uint32_t* __restrict__ fifo_lut,
                                                                     uint8_t* __restrict__ flow) {
  __shared__ float sv[kValY][kValX];
  __shared__ uint32_t word[kTileY + 1][kTileX + 1];
  const int tid = threadIdx.x;
  const int b = find_image(I.tile_base, I.B, blockIdx.x);
  const int H = I.H[b], W = I.W[b];
  const int ntx = (W + 1 + kTileX - 1) / kTileX;
  const int t = blockIdx.x - I.tile_base[b];
  const int ty = t / ntx, tx = t - ty * ntx;
  const int x0 = tx * kTileX, y0 = ty * kTileY;
  const float* img = img_all + I.px_base[b];
  // tiles whose value window [y0-2, y0+kTileY] x [x0-2, x0+kTileX] lies inside
  // the image (almost all of them) run without bound tests
  const bool interior = y0 >= 2 && x0 >= 2 && y0 + kTileY <= H - 1 && x0 + kTileX <= W - 1;
  if (I.dual[b]) {
    if (interior)
      gradient_tile<true, true>(img, H, W, y0, x0, tid, sv, word, fifo_lut);
    else
      gradient_tile<true, false>(img, H, W, y0, x0, tid, sv, word, fifo_lut);
  } else {
    if (interior)
      gradient_tile<false, true>(img, H, W, y0, x0, tid, sv, word, fifo_lut);
    else
      gradient_tile<false, false>(img, H, W, y0, x0, tid, sv, word, fifo_lut);
  }
  const int warp = tid >> 5, lane = tid & 31;
  const long long gbase = I.idx_base[b];
  const int sbase = I.seg_base[b];
  for (int rr = warp; rr < kTileY; rr += kGradWarps) {
    const int iy = y0 + rr, ix = x0 + lane;
    if (iy > H) break;  // uniform per warp
    if (interior)
      gradient_store_row<true>(word, rr, lane, H, W, iy, ix, gbase, sbase + iy * ntx + tx, grad, crit_mask, flow,
                               seg_min, seg_sad, seg_max);
    else
      gradient_store_row<false>(word, rr, lane, H, W, iy, ix, gbase, sbase + iy * ntx + tx, grad, crit_mask, flow,
                                seg_min, seg_sad, seg_max);
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

// K2: ordered compaction. One warp per (row, 32-column) segment of an image;
// segment offsets are exclusive scans of the per-segment counts over the
// whole batch (images in order, rows in order), so each image's lists are a
// contiguous slice in ascending cell-id order. Writes the three lists as
// global cell ids, each critical cell's image, the per-segment bit masks of
// the minima and maxima (an extremum's list rank is its segment's offset plus
// the extrema before it in the mask), the extremum values (also as (value,
// cell) records for the elder comparisons of the pairing) and the saddle
// values with their sort keys (image id above the orderable value, so one
// sort orders every image).
static __global__ void __launch_bounds__(256) compact_kernel(
    Imgs I, const float* __restrict__ img_all, long long nseg, const uint8_t* __restrict__ crit_mask,
    const int* __restrict__ off_min, const int* __restrict__ off_sad, const int* __restrict__ off_max,
    int* __restrict__ crit_min, int* __restrict__ crit_sad, int* __restrict__ crit_max, int* __restrict__ min_img,
    int* __restrict__ sad_img, int* __restrict__ max_img, uint32_t* __restrict__ min_bits,
    uint32_t* __restrict__ max_bits,
    float* __restrict__ min_val, float* __restrict__ max_val, int2* __restrict__ min_key, int2* __restrict__ max_key,
    float* __restrict__ sad_val,
    unsigned long long* __restrict__ sad_key, uint32_t* __restrict__ sad_key32) {
  const int lane = threadIdx.x & 31;
  long long seg = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (seg >= nseg) return;
  const int b = find_image(I.seg_base, I.B, seg);
  const int H = I.H[b], W = I.W[b], Nx = W + 1;
  const bool dual = I.dual[b];
  const int nsegx = (W + 1 + kTileX - 1) / kTileX;
  const long long lseg = seg - I.seg_base[b];
  int iy = (int)(lseg / nsegx), sx = (int)(lseg - (long long)iy * nsegx);
  int ix = sx * kTileX + lane;
  unsigned m = 0;
  const long long gidx = (long long)I.idx_base[b] + (long long)iy * Nx + ix;
  const float* img = img_all + I.px_base[b];
  if (ix <= W) m = crit_mask[gidx];
  unsigned lt = (1u << lane) - 1u;
  unsigned bmin = __ballot_sync(0xffffffffu, m & 1u);
  unsigned bmax = __ballot_sync(0xffffffffu, m & 8u);
  if (lane == 0) {
    min_bits[seg] = bmin;
    max_bits[seg] = bmax;
  }
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
    crit_min[p] = (int)(4 * gidx);
    min_img[p] = b;
    const float v = __ldg(img + (size_t)iy * W + ix);
    min_val[p] = v;
    min_key[p] = make_int2(__float_as_int(v), (int)(4 * gidx));
  }
  if (m & 8u) {
    int p = off_max[seg] + __popc(bmax & lt);
    crit_max[p] = (int)(4 * gidx + 3);
    max_img[p] = b;
    const float v = dual ? cell_value_g<true>(img, 3, iy, ix, H, W) : cell_value_g<false>(img, 3, iy, ix, H, W);
    max_val[p] = v;
    max_key[p] = make_int2(__float_as_int(v), (int)(4 * gidx + 3));
  }
  int p = off_sad[seg] + excl;
#pragma unroll
  for (int t = 1; t <= 2; ++t) {
    if (!(m & (1u << t))) continue;
    crit_sad[p] = (int)(4 * gidx + t);
    sad_img[p] = b;
    float v = dual ? cell_value_g<true>(img, t, iy, ix, H, W) : cell_value_g<false>(img, t, iy, ix, H, W);
    sad_val[p] = v;
    if (sad_key32)  // one image: the image id is 0, a 32-bit key suffices
      sad_key32[p] = orderable_key(v);
    else
      sad_key[p] = ((unsigned long long)b << 32) | orderable_key(v);
    p++;
  }
}

}  // namespace dmsc
