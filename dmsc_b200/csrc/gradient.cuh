// Discrete gradient (steepest lower-star pairing) and ordered critical-cell
// compaction.
//
// Reference semantics: cpu/gradient.hxx:19-196 (compute_gradient),
// cpu/critical_points.hxx:14-65 (extract_critical_points, canonical order =
// ascending cell id), cpu/gradient.hxx:198-231 (fast_crit_map and values).
//
// Layout. The gradient array holds 4 int32 slots per index (y, x) of the
// (H+1) x (W+1) index grid, i.e. 16 bytes per index; it is the grad_indices
// output. One CTA owns a 32-column x TY-row tile of indices and writes it with
// one int4 store per index, so every warp writes 512 contiguous bytes per row.
// The cells at a tile's indices have their highest vertex in the tile's
// pixels or in one halo row above / one halo column to the left, so the CTA
// stages a (TY + 3) x 35 value window in shared memory and evaluates
// (TY + 1) x 33 lower stars, one 32-bit pairing word per pixel:
//   * the 32 main columns with one lane per column, each warp sliding down a
//     run of consecutive rows with the 3 x 3 neighbourhood in registers
//     (three new shared loads per pixel);
//   * the halo column with one lane per row (32 lower stars per pass), so it
//     costs 1/32 of a pass per row instead of a second pass.
// Every index then gathers its four slots from the words of the pixels that
// own them: (iy, ix), (iy, ix-1), (iy-1, ix) and (iy-1, ix-1). Slots of
// invalid cells are -1.
//
// The same pass writes one criticality byte per index (bit t = slot t is an
// unpaired valid cell), the flow codes (common.cuh) and per-(row, 32-column
// segment) counts of minima, saddles and maxima; a scan over the segments in
// row-major order gives every critical cell its position in the
// ascending-cell-id lists.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace dmsc {

constexpr int kTileX = 32;  // indices per tile row (one warp) and per row segment

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

// Pairing word of a pixel: 3-bit fields that describe every cell it owns
// (the cells of its lower star) by the partner of that cell, relative to the
// cell itself, so an index can combine the fields of its four possible owners
// with ORs (a cell has exactly one owner; the others hold 0 there):
//   bits 0-2   vertex: 0 = unpaired (or no pixel), 1..4 = paired with e0..e3,
//              which is also the vertex's flow code (left, right, up, down);
//   bits 3-14  edges e0..e3, 3 bits each: 0 = not owned, 1 = unpaired,
//              2 = paired with its vertex at the lower coordinate (left end
//              of an H edge, upper end of a V edge), 3 = with its vertex at
//              the higher coordinate, 4 = with its coface at the lower
//              coordinate (the face above an H edge, left of a V edge),
//              5 = with its coface at the higher coordinate;
//   bits 15-26 faces f0..f3, 3 bits each: 0 = not owned, 1 = unpaired,
//              2..5 = paired with its left, right, upper, lower edge, i.e.
//              its flow code + 1.
// A pixel outside the image has word 0.
constexpr int kWE0 = 3, kWE1 = 6, kWE2 = 9, kWE3 = 12, kWF0 = 15, kWF1 = 18, kWF2 = 21, kWF3 = 24;

// All 16 x 16 x 5 pairing words, indexed ((eL << 4) | fL) * 5 + best + 1,
// built with face_fifo_entry (the reference's FIFO procedure).
inline void face_fifo_table(uint32_t* out) {
  // edge slot k paired with the pixel (its vertex): P is the right end of
  // e0 = H(y,x), the left end of e1 = H(y,x+1), the lower end of e2 = V(y,x)
  // and the upper end of e3 = V(y+1,x)
  static const unsigned kEdgeVertex[4] = {3, 2, 3, 2};
  // edge slot k paired with face slot f: lower (4) or higher (5) coface
  static const unsigned kEdgeFace[4][4] = {{4, 0, 5, 0}, {0, 4, 0, 5}, {4, 5, 0, 0}, {0, 0, 4, 5}};
  // face slot f paired with edge slot k: flow code of the face + 1
  // (f0 = F(y,x): e0 = its lower edge (down), e2 = its right edge; f1 =
  // F(y,x+1): e1 lower, e2 left; f2 = F(y+1,x): e0 upper, e3 right; f3 =
  // F(y+1,x+1): e1 upper, e3 left)
  static const unsigned kFaceEdge[4][4] = {
      {kFlowDown + 1, 0, kFlowRight + 1, 0},
      {0, kFlowDown + 1, kFlowLeft + 1, 0},
      {kFlowUp + 1, 0, 0, kFlowRight + 1},
      {0, kFlowUp + 1, 0, kFlowLeft + 1}};
  for (unsigned eL = 0; eL < 16; ++eL)
    for (unsigned fL = 0; fL < 16; ++fL)
      for (int b = -1; b < 4; ++b) {
        const uint32_t pk = face_fifo_entry(eL, fL, b);
        uint32_t w = (uint32_t)(b + 1);
        for (int k = 0; k < 4; ++k) {
          if (!((eL >> k) & 1u)) continue;
          const unsigned n = (pk >> (4 * k)) & 0xFu;
          const unsigned code = n == 15u ? 1u : n == 4u ? kEdgeVertex[k] : kEdgeFace[k][n];
          w |= code << (3 + 3 * k);
        }
        for (int f = 0; f < 4; ++f) {
          if (!((fL >> f) & 1u)) continue;
          const unsigned n = (pk >> (16 + 4 * f)) & 0xFu;
          const unsigned code = n == 15u ? 1u : kFaceEdge[f][n];
          w |= code << (15 + 3 * f);
        }
        out[((eL << 4) | fL) * 5 + (b + 1)] = w;
      }
}
constexpr int kFifoTable = 16 * 16 * 5;

// Pixels whose eight neighbours all exist (every pixel of an interior tile):
// the word is a function of 14 comparisons, P against its eight neighbours
// and the six pairs of its edge neighbours (L, R, U, D) that decide which
// lower edge pairs with the vertex, so one lookup in a 2^14-entry table
// replaces the scan. Entry bits: 0 L, 1 R, 2 U, 3 D, 4 UL, 5 UR, 6 DL, 7 DR
// (P above that neighbour), 8 L above R, 9 L above U, 10 R above U, 11 L
// above D, 12 R above D, 13 U above D (each under the (value, id) order, the
// flipped one in the dual). The table follows the general path's rules
// (star_word below) and is appended to the FIFO table.
constexpr int kStarTable = 1 << 14;
constexpr int kGradTable = kFifoTable + kStarTable;
inline void gradient_tables(uint32_t* out) {
  face_fifo_table(out);
  for (unsigned idx = 0; idx < (unsigned)kStarTable; ++idx) {
    auto bit = [&](int k) { return (idx >> k) & 1u; };
    const unsigned eL = bit(0) | bit(1) << 1 | bit(2) << 2 | bit(3) << 3;
    const unsigned fL = (bit(0) & bit(2) & bit(4)) | (bit(1) & bit(2) & bit(5)) << 1 | (bit(0) & bit(3) & bit(6)) << 2 |
                        (bit(1) & bit(3) & bit(7)) << 3;
    int best = -1, bo = -1;  // bo: 0 L, 1 R, 2 U
    if (bit(0)) {
      best = 0;
      bo = 0;
    }
    if (bit(1) && (best < 0 || bit(8))) {
      best = 1;
      bo = 1;
    }
    if (bit(2) && (best < 0 || (bo == 0 ? bit(9) : bit(10)))) {
      best = 2;
      bo = 2;
    }
    if (bit(3) && (best < 0 || (bo == 0 ? bit(11) : bo == 1 ? bit(12) : bit(13)))) best = 3;
    out[kFifoTable + idx] = out[((eL << 4) | fL) * 5 + best + 1];
  }
}

// v_greater (cpu/cell_compare.hxx:23-31) orders pixels by (value, y*W+x),
// flipped in the dual. gt(a, b) when a's linear id is known to be larger (a
// "after" b) or smaller: the (value, id) tie rule then reduces to one float
// compare.
//   primal: after -> !(a < b), before -> (b < a); dual: after -> (a < b), before -> !(b < a)
template <bool DUAL>
__host__ __device__ __forceinline__ bool gt_after(float a, float b) {
  return DUAL ? (a < b) : !(a < b);
}
template <bool DUAL>
__host__ __device__ __forceinline__ bool gt_before(float a, float b) {
  return DUAL ? !(b < a) : (b < a);
}

// Pairing word of pixel P from its 3 x 3 neighbourhood (cpu/gradient.hxx:48-192).
// A cell is in P's lower star when P is its highest vertex; under the
// (value, id) order, a strict total order on every field whose values are
// numbers or all NaN, that is P being above each of the cell's other
// vertices, so eight comparisons of P with its neighbours decide the eight
// cells. The vertex pairs with the lower-star edge whose other vertex is
// lowest, scanned L, R, U, D as the reference does; the face FIFO depends
// only on (eL, fL, best) and is looked up. lv/rv/uv/dv: the neighbour exists.
template <bool DUAL, bool INTERIOR>
__host__ __device__ __forceinline__ uint32_t star_word(float UL, float U, float UR, float L, float P, float R, float DL, float D,
                                              float DR, bool lv, bool rv, bool uv, bool dv,
                                              const uint32_t* __restrict__ lut) {
  if (INTERIOR) {  // all neighbours exist: the 14-comparison table (gradient_tables)
    const unsigned idx = (unsigned)gt_after<DUAL>(P, L) | (unsigned)gt_before<DUAL>(P, R) << 1 |
                         (unsigned)gt_after<DUAL>(P, U) << 2 | (unsigned)gt_before<DUAL>(P, D) << 3 |
                         (unsigned)gt_after<DUAL>(P, UL) << 4 | (unsigned)gt_after<DUAL>(P, UR) << 5 |
                         (unsigned)gt_before<DUAL>(P, DL) << 6 | (unsigned)gt_before<DUAL>(P, DR) << 7 |
                         (unsigned)gt_before<DUAL>(L, R) << 8 | (unsigned)gt_after<DUAL>(L, U) << 9 |
                         (unsigned)gt_after<DUAL>(R, U) << 10 | (unsigned)gt_before<DUAL>(L, D) << 11 |
                         (unsigned)gt_before<DUAL>(R, D) << 12 | (unsigned)gt_before<DUAL>(U, D) << 13;
#ifdef __CUDA_ARCH__
    return __ldg(lut + kFifoTable + idx);
#else
    return lut[kFifoTable + idx];
#endif
  }
  const bool gL = gt_after<DUAL>(P, L), gU = gt_after<DUAL>(P, U);
  const bool gUL = gt_after<DUAL>(P, UL), gUR = gt_after<DUAL>(P, UR);  // UR = (y-1, x+1) precedes P too
  const bool gR = gt_before<DUAL>(P, R), gD = gt_before<DUAL>(P, D);
  const bool gDL = gt_before<DUAL>(P, DL), gDR = gt_before<DUAL>(P, DR);
  const bool e0 = !lv || gL, e1 = !rv || gR, e2 = !uv || gU, e3 = !dv || gD;
  const bool f0 = e0 && e2 && (!(lv && uv) || gUL);
  const bool f1 = e1 && e2 && (!(rv && uv) || gUR);
  const bool f2 = e0 && e3 && (!(lv && dv) || gDL);
  const bool f3 = e1 && e3 && (!(rv && dv) || gDR);
  int best = -1;
  float bo = 0.0f;
  if (lv && gL) {
    best = 0;
    bo = L;
  }
  if (rv && gR && (best < 0 || gt_before<DUAL>(bo, R))) {  // L before R
    best = 1;
    bo = R;
  }
  if (uv && gU && (best < 0 || gt_after<DUAL>(bo, U))) {  // L, R after U
    best = 2;
    bo = U;
  }
  if (dv && gD && (best < 0 || gt_before<DUAL>(bo, D))) {  // L, R, U before D
    best = 3;
  }
  const unsigned eL = (unsigned)e0 | (unsigned)e1 << 1 | (unsigned)e2 << 2 | (unsigned)e3 << 3;
  const unsigned fL = (unsigned)f0 | (unsigned)f1 << 1 | (unsigned)f2 << 2 | (unsigned)f3 << 3;
#ifdef __CUDA_ARCH__
  return __ldg(lut + (((eL << 4) | fL) * 5 + (best + 1)));
#else
  return lut[((eL << 4) | fL) * 5 + (best + 1)];
#endif
}

// Partner offsets of the gather (4 * index + offset = partner cell), per
// image width; codes as in the pairing word:
//   [0 + v]   vertex paired with e0..e3: H(y,x), H(y,x+1), V(y,x), V(y+1,x)
//   [8 + c]   H edge H(y,x): left vertex, right vertex, face above, face below
//   [16 + c]  V edge V(y,x): upper vertex, lower vertex, face left, face right
//   [24 + c]  face F(y,x): left edge V(y,x-1), right V(y,x), upper H(y-1,x), lower H(y,x)
__host__ __device__ __forceinline__ int gather_offset(int k, int Nx) {
  switch (k) {
    case 1: return 1;
    case 2: return 5;
    case 3: return 2;
    case 4: return 4 * Nx + 2;
    case 8 + 2: return -4;
    case 8 + 3: return 0;
    case 8 + 4: return 3;
    case 8 + 5: return 4 * Nx + 3;
    case 16 + 2: return -4 * Nx;
    case 16 + 3: return 0;
    case 16 + 4: return 3;
    case 16 + 5: return 7;
    case 24 + 2: return -2;
    case 24 + 3: return 2;
    case 24 + 4: return 1 - 4 * Nx;
    case 24 + 5: return 1;
    default: return 0;
  }
}

// Slots, criticality bits and flow code of the index b4 / 4 from the words of
// the four pixels that may own its cells: P = (iy, ix), L = (iy, ix-1),
// U = (iy-1, ix), UL = (iy-1, ix-1). `vin`: the index's vertex is a pixel.
__host__ __device__ __forceinline__ void gather_index(uint32_t wP, uint32_t wL, uint32_t wU, uint32_t wUL, int b4,
                                                      const int* off, bool vin, int4& g, unsigned& m,
                                                      unsigned& fl) {
  const unsigned v = wP & 7u;
  const unsigned hc = ((wP >> kWE0) | (wL >> kWE1)) & 7u;
  const unsigned vc = ((wP >> kWE2) | (wU >> kWE3)) & 7u;
  const unsigned fc = ((wP >> kWF0) | (wL >> kWF1) | (wU >> kWF2) | (wUL >> kWF3)) & 7u;
  g = make_int4(v ? b4 + off[v] : -1, hc >= 2u ? b4 + off[8 + hc] : -1, vc >= 2u ? b4 + off[16 + vc] : -1,
                fc >= 2u ? b4 + off[24 + fc] : -1);
  m = (unsigned)(v == 0u && vin) | (unsigned)(hc == 1u) << 1 | (unsigned)(vc == 1u) << 2 | (unsigned)(fc == 1u) << 3;
  // every index has its face, so fc >= 1; bits 3 and 7: the H and V edge are critical
  fl = v | (unsigned)(hc == 1u) << 3 | ((fc - 1u) << 4) | (unsigned)(vc == 1u) << 7;
}

template <int TY>
struct GradSmem {
  float v[TY + 3][35];         // pixel rows y0-2 .. y0+TY, columns x0-2 .. x0+32
  uint32_t w[TY + 1][33];      // words of pixel rows y0-1 .. y0+TY-1, columns x0-1 .. x0+31
  int off[32];                 // gather offsets of the tile's image
};

// One 32 x TY index tile at index origin (y0, x0) of an H x W image:
// gradient, criticality, flow codes and row-segment counts. INTERIOR: the
// value window [y0-2, y0+TY] x [x0-2, x0+32] lies inside the image, so no
// bound is tested. `gbase`: global index of the image's index (0, 0);
// `sbase`: its first row segment; `ntx`: its row segments per row. The tile
// runs in three parts: the value window is staged in shared memory; the
// pairing words of its pixels are computed from the window
// (gradient_words: value of window row r, column c = pixel (y0 - 2 + r,
// x0 - 2 + c) at V[r][c + VOFF]); every index gathers its slots from the
// words (gradient_gather).
template <bool DUAL, bool INTERIOR, int TY, int NT, int VC, int VOFF>
__device__ __forceinline__ void gradient_words(const float (*V)[VC], uint32_t (*Wd)[33], int H, int W, int y0, int x0,
                                               const uint32_t* __restrict__ lut) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {  // main columns: lane -> column x0 + lane (word column lane + 1), a run of rows per warp
    constexpr int kRun = (TY + 1 + NW - 1) / NW;
    const int ra = warp * kRun, rb = min(TY + 1, ra + kRun);
    const int x = x0 + lane, c = lane + 2;  // value column of the pixel
    const bool xin = INTERIOR || x < W;
    const bool lv = INTERIOR || x >= 1, rv = INTERIOR || x + 1 < W;
    if (ra < rb) {
      float u0 = V[ra][c - 1 + VOFF], u1 = V[ra][c + VOFF], u2 = V[ra][c + 1 + VOFF];
      float p0 = V[ra + 1][c - 1 + VOFF], p1 = V[ra + 1][c + VOFF], p2 = V[ra + 1][c + 1 + VOFF];
      for (int r = ra; r < rb; ++r) {
        const float d0 = V[r + 2][c - 1 + VOFF], d1 = V[r + 2][c + VOFF], d2 = V[r + 2][c + 1 + VOFF];
        const int y = y0 - 1 + r;
        uint32_t w = 0;
        if (INTERIOR || (xin && y >= 0 && y < H))
          w = star_word<DUAL, INTERIOR>(u0, u1, u2, p0, p1, p2, d0, d1, d2, lv, rv, INTERIOR || y >= 1,
                                        INTERIOR || y + 1 < H, lut);
        Wd[r][lane + 1] = w;
        u0 = p0;
        u1 = p1;
        u2 = p2;
        p0 = d0;
        p1 = d1;
        p2 = d2;
      }
    }
  }
  {  // halo column x0 - 1 (word column 0, value column 1): lane -> row
    constexpr int kHaloPasses = (TY + 1 + 31) / 32;
    if (warp < kHaloPasses) {
      const int r = warp * 32 + lane;
      if (r <= TY) {
        const int y = y0 - 1 + r, x = x0 - 1;
        uint32_t w = 0;
        if (INTERIOR || (x >= 0 && x < W && y >= 0 && y < H))
          w = star_word<DUAL, INTERIOR>(V[r][VOFF], V[r][1 + VOFF], V[r][2 + VOFF], V[r + 1][VOFF],
                                        V[r + 1][1 + VOFF], V[r + 1][2 + VOFF], V[r + 2][VOFF], V[r + 2][1 + VOFF],
                                        V[r + 2][2 + VOFF], INTERIOR || x >= 1, INTERIOR || x + 1 < W,
                                        INTERIOR || y >= 1, INTERIOR || y + 1 < H, lut);
        Wd[r][0] = w;
      }
    }
  }
}

template <bool INTERIOR, int TY, int NT>
__device__ __forceinline__ void gradient_gather(const uint32_t (*Wd)[33], const int* off, int H, int W, int y0, int x0,
                                                long long gbase, int sbase, int ntx, int tx, int4* __restrict__ grad,
                                                uint8_t* __restrict__ crit_mask, uint8_t* __restrict__ flow,
                                                int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                                int* __restrict__ seg_max) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int Nx = W + 1;
  // ---- gather and stores: one index row per warp step ----
  const int ix = x0 + lane;
  const bool xok = INTERIOR || ix <= W;
  for (int rr = warp; rr < TY; rr += NW) {
    const int iy = y0 + rr;
    if (!INTERIOR && iy > H) break;  // uniform per warp
    unsigned m = 0;
    if (xok) {
      const uint32_t wP = Wd[rr + 1][lane + 1], wL = Wd[rr + 1][lane];
      const uint32_t wU = Wd[rr][lane + 1], wUL = Wd[rr][lane];
      const int b = iy * Nx + ix;  // image-local index: the cell ids written are local
      const size_t gidx = (size_t)(gbase + b);
      int4 g;
      unsigned fl;
      gather_index(wP, wL, wU, wUL, 4 * b, off, INTERIOR || (iy < H && ix < W), g, m, fl);
      if (grad) grad[gidx] = g;  // null when the gradient is not returned
      if (crit_mask) crit_mask[gidx] = (uint8_t)m;  // null: the flow byte carries the same bits
      flow[gidx] = (uint8_t)fl;
    }
    // the segment's counts (at most 32, 64 and 32) packed in one warp sum
    const unsigned cnt = __reduce_add_sync(
        0xffffffffu, (m & 1u) | (((m >> 1) & 1u) + ((m >> 2) & 1u)) << 8 | ((m >> 3) & 1u) << 16);
    if (lane == 0) {
      const int seg = sbase + iy * ntx + tx;
      seg_min[seg] = (int)(cnt & 0xFFu);
      seg_sad[seg] = (int)((cnt >> 8) & 0xFFu);
      seg_max[seg] = (int)(cnt >> 16);
    }
  }
}


template <bool DUAL, bool INTERIOR, int TY, int NT>
__device__ __forceinline__ void gradient_tile(GradSmem<TY>& S, const float* __restrict__ img, int H, int W, int y0,
                                              int x0, long long gbase, int sbase, int ntx, int tx,
                                              const uint32_t* __restrict__ lut, int4* __restrict__ grad,
                                              uint8_t* __restrict__ crit_mask, uint8_t* __restrict__ flow,
                                              int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                              int* __restrict__ seg_max) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int Nx = W + 1;
  if (threadIdx.x < 32) S.off[lane] = gather_offset(lane, Nx);
  // ---- value window: rows by warp, 32 + 3 columns per row ----
  for (int r = warp; r < TY + 3; r += NW) {
    const int gy = y0 - 2 + r;
    const float* row = img + (size_t)(INTERIOR ? gy : max(0, min(gy, H - 1))) * W;
    const bool yin = INTERIOR || (gy >= 0 && gy < H);
    const int gx = x0 - 2 + lane, gx2 = x0 + 30 + lane;
    const float a = (INTERIOR || (yin && gx >= 0 && gx < W)) ? __ldg(row + gx) : 0.0f;
    float b = 0.0f;
    if (lane < 3 && (INTERIOR || (yin && gx2 < W))) b = __ldg(row + gx2);
    S.v[r][lane] = a;
    if (lane < 3) S.v[r][32 + lane] = b;
  }
  __syncthreads();
  gradient_words<DUAL, INTERIOR, TY, NT, 35, 0>(S.v, S.w, H, W, y0, x0, lut);
  __syncthreads();
  gradient_gather<INTERIOR, TY, NT>(S.w, S.off, H, W, y0, x0, gbase, sbase, ntx, tx, grad, crit_mask, flow, seg_min,
                                    seg_sad, seg_max);
}

// Tile shapes of the gradient kernels (index rows, threads): the tuner in
// the host code picks one per call from these instantiations. Shapes 0-2 run
// gradient_batch_kernel; shapes 3 and 4 run gradient_tma_kernel (one image
// whose rows are 16-byte multiples in a 16-byte aligned buffer; otherwise
// the batch kernel with the same tile).
constexpr int kGradShapes = 5;
constexpr int kGradTY[kGradShapes] = {31, 63, 127, 63, 127};
constexpr int kGradNT[kGradShapes] = {256, 256, 512, 256, 512};
constexpr bool kGradTma[kGradShapes] = {false, false, false, true, true};

// ---------------------------------------------------------------------------
// Persistent gradient with the value windows staged by the tensor-memory
// accelerator: each CTA walks its tiles (tile blockIdx.x, then + gridDim.x,
// ...) and, while it computes one tile, the next tile's window is already
// being copied into the other half of a double buffer
// (cp.async.bulk.tensor.2d with an mbarrier; no multicast, and the tensor
// map covers this call's own image only). The copy box starts on a 16-byte
// boundary: 40 columns x0-4 .. x0+35 and TY + 3 rows y0-2 .. y0+TY; parts of
// the box outside the image read as zeros (the bounded path never uses them).
// ---------------------------------------------------------------------------
constexpr int kTmaCols = 40;

template <int TY>
struct alignas(128) GradTmaWindow {  // one copy destination, on a 128-byte boundary
  float v[TY + 3][kTmaCols];
};
template <int TY>
struct alignas(128) GradTmaSmem {
  GradTmaWindow<TY> win[2];
  uint32_t w[TY + 1][33];
  int off[32];
  unsigned long long bar[2];
};
// dynamic shared memory of the kernel: the struct plus room to align it
template <int TY>
constexpr int grad_tma_smem_bytes() {
  return (int)sizeof(GradTmaSmem<TY>) + 128;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// orders this CTA's earlier generic-proxy reads of shared memory before the
// next bulk copy into it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ unsigned long long grad_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for phase `parity` of a copy barrier: false after `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity,
                                                  unsigned long long limit_ns) {
  const unsigned long long t0 = grad_ns();
  while (!mbar_try_wait(bar, parity))
    if (grad_ns() - t0 > limit_ns) return false;
  return true;
}

template <bool DUAL, int TY, int NT>
__global__ void __launch_bounds__(NT) gradient_tma_kernel(const __grid_constant__ CUtensorMap map, int H, int W,
                                                          int ntx, int tile0, int ntiles, int4* __restrict__ grad,
                                                          uint8_t* __restrict__ flow, int* __restrict__ seg_min,
                                                          int* __restrict__ seg_sad, int* __restrict__ seg_max,
                                                          const uint32_t* __restrict__ lut, unsigned* status) {
  extern __shared__ __align__(128) unsigned char grad_tma_smem[];
  // the copy destinations must sit on 128-byte boundaries: align the base
  const uint32_t base = smem_u32(grad_tma_smem);
  GradTmaSmem<TY>& S = *reinterpret_cast<GradTmaSmem<TY>*>(grad_tma_smem + (((base + 127u) & ~127u) - base));
  constexpr uint32_t kBytes = (uint32_t)(TY + 3) * kTmaCols * sizeof(float);
  constexpr unsigned long long kLimitNs = 1000000000ull;  // a copy takes microseconds
  const int Nx = W + 1;
  if (threadIdx.x < 32) S.off[threadIdx.x] = gather_offset(threadIdx.x, Nx);
  if (threadIdx.x == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int t = tile0 + blockIdx.x;  // tiles tile0 .. ntiles - 1 (a band of tile rows, or all)
  if (threadIdx.x == 0 && t < ntiles) {
    const int ty = t / ntx, tx = t - ty * ntx;
    mbar_arrive_expect_tx(&S.bar[0], kBytes);
    tma_load_2d(&S.win[0].v[0][0], &map, tx * kTileX - 4, ty * TY - 2, &S.bar[0]);
  }
  for (int k = 0; t < ntiles; ++k, t += gridDim.x) {
    const int b = k & 1;
    const int tn = t + gridDim.x;
    // the other buffer was last read before the barrier that ended the
    // previous tile: the next tile's copy goes there now
    if (threadIdx.x == 0 && tn < ntiles) {
      const int ty = tn / ntx, tx = tn - ty * ntx;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&S.bar[b ^ 1], kBytes);
      tma_load_2d(&S.win[b ^ 1].v[0][0], &map, tx * kTileX - 4, ty * TY - 2, &S.bar[b ^ 1]);
    }
    const bool ok = mbar_wait_bounded(&S.bar[b], (uint32_t)(k >> 1) & 1u, kLimitNs);
    if (__syncthreads_or(!ok)) {
      // report, wait (bounded) for this CTA's copies still in flight, leave
      if (threadIdx.x == 0) {
        set_status(status, kStatusCopyWait);
        mbar_wait_bounded(&S.bar[b], (uint32_t)(k >> 1) & 1u, kLimitNs);
        if (tn < ntiles) mbar_wait_bounded(&S.bar[b ^ 1], (uint32_t)((k + 1) >> 1) & 1u, kLimitNs);
      }
      return;
    }
    const int ty = t / ntx, tx = t - ty * ntx, y0 = ty * TY, x0 = tx * kTileX;
    const bool interior = y0 >= 2 && x0 >= 2 && y0 + TY <= H - 1 && x0 + kTileX <= W - 1;
    if (interior)
      gradient_words<DUAL, true, TY, NT, kTmaCols, 2>(S.win[b].v, S.w, H, W, y0, x0, lut);
    else
      gradient_words<DUAL, false, TY, NT, kTmaCols, 2>(S.win[b].v, S.w, H, W, y0, x0, lut);
    __syncthreads();
    if (interior)
      gradient_gather<true, TY, NT>(S.w, S.off, H, W, y0, x0, 0, 0, ntx, tx, grad, nullptr, flow, seg_min, seg_sad,
                                    seg_max);
    else
      gradient_gather<false, TY, NT>(S.w, S.off, H, W, y0, x0, 0, 0, ntx, tx, grad, nullptr, flow, seg_min, seg_sad,
                                     seg_max);
    __syncthreads();
  }
}

// K1 (one image): a 2-D grid of tiles, (ntx, nty).
template <bool DUAL, int TY, int NT>
__global__ void __launch_bounds__(NT) gradient_kernel(const float* __restrict__ img, int H, int W,
                                                      int4* __restrict__ grad, uint8_t* __restrict__ crit_mask,
                                                      int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                                      int* __restrict__ seg_max, const uint32_t* __restrict__ lut,
                                                      uint8_t* __restrict__ flow) {
  __shared__ GradSmem<TY> S;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * TY;
  const bool interior = y0 >= 2 && x0 >= 2 && y0 + TY <= H - 1 && x0 + kTileX <= W - 1;
  if (interior)
    gradient_tile<DUAL, true, TY, NT>(S, img, H, W, y0, x0, 0, 0, gridDim.x, blockIdx.x, lut, grad, crit_mask, flow,
                                      seg_min, seg_sad, seg_max);
  else
    gradient_tile<DUAL, false, TY, NT>(S, img, H, W, y0, x0, 0, 0, gridDim.x, blockIdx.x, lut, grad, crit_mask, flow,
                                       seg_min, seg_sad, seg_max);
}

// K1 (batch): the tiles of every image of a batch in one 1-D grid; each CTA
// finds its image from the tile bases (tiles of TY index rows).
template <int TY, int NT>
__global__ void __launch_bounds__(NT) gradient_batch_kernel(Imgs I, const float* __restrict__ img_all,
                                                            int4* __restrict__ grad, uint8_t* __restrict__ crit_mask,
                                                            int* __restrict__ seg_min, int* __restrict__ seg_sad,
                                                            int* __restrict__ seg_max,
                                                            const uint32_t* __restrict__ lut,
                                                            uint8_t* __restrict__ flow) {
  __shared__ GradSmem<TY> S;
  const int b = find_image(I.tile_base, I.B, blockIdx.x);
  const int H = I.H[b], W = I.W[b];
  const int ntx = (W + 1 + kTileX - 1) / kTileX;
  const int t = blockIdx.x - I.tile_base[b];
  const int ty = t / ntx, tx = t - ty * ntx;
  const int x0 = tx * kTileX, y0 = ty * TY;
  const float* img = img_all + I.px_base[b];
  const long long gbase = I.idx_base[b];
  const int sbase = I.seg_base[b];
  // tiles whose value window lies inside the image (almost all) run without bound tests
  const bool interior = y0 >= 2 && x0 >= 2 && y0 + TY <= H - 1 && x0 + kTileX <= W - 1;
  if (I.dual[b]) {
    if (interior)
      gradient_tile<true, true, TY, NT>(S, img, H, W, y0, x0, gbase, sbase, ntx, tx, lut, grad, crit_mask, flow,
                                        seg_min, seg_sad, seg_max);
    else
      gradient_tile<true, false, TY, NT>(S, img, H, W, y0, x0, gbase, sbase, ntx, tx, lut, grad, crit_mask, flow,
                                         seg_min, seg_sad, seg_max);
  } else {
    if (interior)
      gradient_tile<false, true, TY, NT>(S, img, H, W, y0, x0, gbase, sbase, ntx, tx, lut, grad, crit_mask, flow,
                                         seg_min, seg_sad, seg_max);
    else
      gradient_tile<false, false, TY, NT>(S, img, H, W, y0, x0, gbase, sbase, ntx, tx, lut, grad, crit_mask, flow,
                                          seg_min, seg_sad, seg_max);
  }
}

// cell_value (cpu/cell_compare.hxx:82-87): value of the highest (dual: lowest)
// vertex, chosen by (value, pixel id) in the reference's scan order (each
// candidate replaces the current choice when value_greater); the chosen
// pixel's own value is returned, so -0.0 survives. `pick` adds one candidate.
template <bool DUAL>
__device__ __forceinline__ void pick(bool& have, float& bv, int& bi, bool valid, float v, int id) {
  if (valid && (!have || value_greater<DUAL>(v, id, bv, bi))) {
    have = true;
    bv = v;
    bi = id;
  }
}

// Values of the four cells of index (y, x) for a whole warp of consecutive
// columns: every lane loads its pixel and the one above it, takes its left
// neighbours' from the lane to its left (lane 0 loads them), and evaluates
// the candidates of cpu/cell_compare.hxx:82-87 in the reference's order
// (vertex (y-1, x-1), (y-1, x), (y, x-1), (y, x) among those in the image).
// Every lane of the warp must call it.
struct CellValues {
  float v, h, e, f;  // vertex, H edge (t = 1), V edge (t = 2), face (t = 3)
};

// The four pixel values an index's cells need: its own (y, x), the one above
// and their left neighbours (0 outside the image).
struct CellPixels {
  float a, u, aL, uL;
};

// The loads of the cell values: every lane loads its pixel and the one above
// it; lane 0 also loads its left neighbours (the other lanes take theirs from
// the lane to their left in cell_values_of).
__device__ __forceinline__ CellPixels warp_cell_loads(const float* __restrict__ img, int y, int x, int H, int W,
                                                      int lane) {
  const bool in_x = x < W, in_xl = x >= 1 && x - 1 < W, up = y >= 1, here = y < H;
  CellPixels c;
  c.a = (here && in_x) ? __ldg(img + (size_t)y * W + x) : 0.f;
  c.u = (up && in_x) ? __ldg(img + (size_t)(y - 1) * W + x) : 0.f;
  c.aL = (lane == 0 && here && in_xl) ? __ldg(img + (size_t)y * W + x - 1) : 0.f;
  c.uL = (lane == 0 && up && in_xl) ? __ldg(img + (size_t)(y - 1) * W + x - 1) : 0.f;
  return c;
}

template <bool DUAL>
__device__ __forceinline__ CellValues cell_values_of(CellPixels px, int y, int x, int H, int W, int lane) {
  const bool in_x = x < W, up = y >= 1, here = y < H;
  const float a = px.a, u = px.u;
  float aL = __shfl_up_sync(0xffffffffu, a, 1), uL = __shfl_up_sync(0xffffffffu, u, 1);
  if (lane == 0) {
    aL = px.aL;
    uL = px.uL;
  }
  const int id = y * W + x, idu = id - W;
  CellValues c;
  c.v = a;
  {
    bool hv = false;
    float bv = 0.f;
    int bi = 0;
    pick<DUAL>(hv, bv, bi, here && x >= 1, aL, id - 1);
    pick<DUAL>(hv, bv, bi, here && in_x, a, id);
    c.h = bv;
  }
  {
    bool hv = false;
    float bv = 0.f;
    int bi = 0;
    pick<DUAL>(hv, bv, bi, up && in_x, u, idu);
    pick<DUAL>(hv, bv, bi, here && in_x, a, id);
    c.e = bv;
  }
  {
    bool hv = false;
    float bv = 0.f;
    int bi = 0;
    pick<DUAL>(hv, bv, bi, up && x >= 1, uL, idu - 1);
    pick<DUAL>(hv, bv, bi, up && in_x, u, idu);
    pick<DUAL>(hv, bv, bi, here && x >= 1, aL, id - 1);
    pick<DUAL>(hv, bv, bi, here && in_x, a, id);
    c.f = bv;
  }
  return c;
}

// Criticality bits of an index (bit t: slot t is an unpaired valid cell) from
// its flow byte; `vin`: the index's vertex is a pixel.
__host__ __device__ __forceinline__ unsigned crit_bits(unsigned fl, bool vin) {
  return (unsigned)((fl & 7u) == 0u && vin) | ((fl >> 2) & 2u) | ((fl >> 5) & 4u) | (unsigned)(((fl >> 4) & 7u) == 0u) << 3;
}

// K2: ordered compaction. One warp per (row, 32-column) segment of an image,
// kCompactSegs consecutive segments per warp with every load of all of them
// (flow bytes, pixel values, list offsets) issued before any is used, so a
// warp waits on one round of loads instead of three per segment; segment
// offsets are exclusive scans of the per-segment counts over the whole batch
// (images in order, rows in order), so each image's lists are a contiguous
// slice in ascending cell-id order. Writes the saddle list as global cell
// ids with each saddle's image and value; each extremum's image and its
// (value bits, global cell id) record (the extremum lists, read by the
// elder comparisons of the pairing, the persistence pass and the outputs);
// the per-segment bit masks of the minima and maxima (an extremum's list
// rank is its segment's offset plus the extrema before it in the mask); and
// the pairing's starting state of the groups (PairStart).
constexpr int kCompactSegs = 2;

static __global__ void __launch_bounds__(256) compact_kernel(
    Imgs I, const float* __restrict__ img_all, long long nseg, const uint8_t* __restrict__ flow,
    const int* __restrict__ off_min, const int* __restrict__ off_sad, const int* __restrict__ off_max,
    int* __restrict__ crit_sad, int* __restrict__ min_img, int* __restrict__ sad_img, int* __restrict__ max_img,
    uint32_t* __restrict__ min_bits, uint32_t* __restrict__ max_bits, int2* __restrict__ min_key,
    int2* __restrict__ max_key, float* __restrict__ sad_val, PairStart ps) {
  constexpr int K = kCompactSegs;
  const int lane = threadIdx.x & 31;
  const long long seg0 = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * K;
  if (seg0 >= nseg) return;
  if (seg0 == 0 && lane == 0) {  // the pairing's void groups and round counters
#pragma unroll
    for (int sd = 0; sd < 2; ++sd) {
      ps.minedge[sd][ps.M[sd]] = ~0ull;
      ps.link[sd][ps.M[sd]] = ps.M[sd];
      int* c = ps.cnt[sd];
      c[0] = ps.nsad;  // round 0 takes every saddle
      c[1] = 0;        // the saddles still active after it (counted by the walks)
      c[2] = 0;
      c[3] = ps.M[sd] + 1;
      c[4] = 0;
      c[5] = 0;
    }
  }
  const unsigned lt = (1u << lane) - 1u;
  int b[K], iy[K], ix[K], o_min[K], o_sad[K], o_max[K];
  unsigned fl[K];
  CellPixels px[K];
  // every load of the warp's segments first
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const long long seg = seg0 + k;
    b[k] = 0;
    iy[k] = ix[k] = 0;
    fl[k] = 0;
    o_min[k] = o_sad[k] = o_max[k] = 0;
    px[k] = CellPixels{0.f, 0.f, 0.f, 0.f};
    if (seg >= nseg) continue;  // warp-uniform
    b[k] = find_image(I.seg_base, I.B, seg);
    const int H = I.H[b[k]], W = I.W[b[k]], Nx = W + 1;
    const int nsegx = (W + 1 + kTileX - 1) / kTileX;
    const int lseg = (int)(seg - I.seg_base[b[k]]);  // an image has fewer than 2^31 / 4 indices
    iy[k] = lseg / nsegx;
    ix[k] = (lseg - iy[k] * nsegx) * kTileX + lane;
    if (ix[k] <= W) fl[k] = flow[(long long)I.idx_base[b[k]] + (long long)iy[k] * Nx + ix[k]];
    px[k] = warp_cell_loads(img_all + I.px_base[b[k]], iy[k], ix[k], H, W, lane);
    o_min[k] = off_min[seg];
    o_sad[k] = off_sad[seg];
    o_max[k] = off_max[seg];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const long long seg = seg0 + k;
    if (seg >= nseg) break;  // warp-uniform
    const int bk = b[k], H = I.H[bk], W = I.W[bk], Nx = W + 1;
    const long long gidx = (long long)I.idx_base[bk] + (long long)iy[k] * Nx + ix[k];
    const unsigned m = ix[k] <= W ? crit_bits(fl[k], iy[k] < H && ix[k] < W) : 0u;
    const unsigned bmin = __ballot_sync(0xffffffffu, m & 1u);
    const unsigned bmax = __ballot_sync(0xffffffffu, m & 8u);
    const unsigned bh = __ballot_sync(0xffffffffu, m & 2u), bv = __ballot_sync(0xffffffffu, m & 4u);
    if (lane == 0) {
      min_bits[seg] = bmin;
      max_bits[seg] = bmax;
    }
    if ((bmin | bmax | bh | bv) == 0u) continue;  // the whole warp together
    const CellValues cv = I.dual[bk] ? cell_values_of<true>(px[k], iy[k], ix[k], H, W, lane)
                                     : cell_values_of<false>(px[k], iy[k], ix[k], H, W, lane);
    // saddles before this lane's: both edge kinds of the lanes below it
    int p = o_sad[k] + __popc(bh & lt) + __popc(bv & lt);
    if (m & 1u) {
      const int q = o_min[k] + __popc(bmin & lt);
      min_img[q] = bk;
      min_key[q] = make_int2(__float_as_int(cv.v), (int)(4 * gidx));
      ps.minedge[1][q] = ~0ull;  // a single-extremum group without outgoing saddles yet
      ps.link[1][q] = q;
    }
    if (m & 8u) {
      const int q = o_max[k] + __popc(bmax & lt);
      max_img[q] = bk;
      max_key[q] = make_int2(__float_as_int(cv.f), (int)(4 * gidx + 3));
      ps.minedge[0][q] = ~0ull;
      ps.link[0][q] = q;
    }
#pragma unroll
    for (int t = 1; t <= 2; ++t) {
      if (!(m & (1u << t))) continue;
      const float v = t == 1 ? cv.h : cv.e;
      crit_sad[p] = (int)(4 * gidx + t);
      sad_img[p] = bk;
      sad_val[p] = v;
      p++;
    }
  }
}

}  // namespace dmsc
