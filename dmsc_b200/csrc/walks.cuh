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

// Dense rank in its critical list of the extremum at global index g of image
// b: its 32-index row segment's first rank (the compaction's exclusive scan)
// plus the extrema before it in the segment's bit mask.
__device__ __forceinline__ int seg_rank(const Imgs& I, int b, int g, int Nx, const int* __restrict__ off,
                                        const uint32_t* __restrict__ bits) {
  const int l = g - I.idx_base[b];
  const int y = l / Nx, x = l - y * Nx;
  const int seg = I.seg_base[b] + y * ((Nx + 31) >> 5) + (x >> 5);
  return __ldg(off + seg) + __popc(__ldg(bits + seg) & ((1u << (x & 31)) - 1u));
}

// K4: per saddle, both face walks and the vertex walks. Writes per arc
// (2 per saddle and side): dense target index (or -1) and step count.
__global__ void __launch_bounds__(256) saddle_walk_kernel(Imgs I, const uint8_t* __restrict__ flow, int nsad,
                                                          const int* __restrict__ crit_sad,
                                                          const int* __restrict__ sad_img,
                                                          const int* __restrict__ off_max,
                                                          const uint32_t* __restrict__ max_bits,
                                                          const int* __restrict__ off_min,
                                                          const uint32_t* __restrict__ min_bits, int* __restrict__ tf,
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
    tf[2 * s + j] = seg_rank(I, b, end, Nx, off_max, max_bits);
    lf[2 * s + j] = (int)steps;
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int start = vertex_start(sc, j, H, W, Nx, I.idx_base[b]);
    long long steps = 0;
    if (start >= 0) {
      int end = flow_walk<0>(flow, start >> 2, Nx, cap, &steps, status);
      tv[2 * s + j] = seg_rank(I, b, end, Nx, off_min, min_bits);
    } else {
      tv[2 * s + j] = -1;
    }
    lv[2 * s + j] = (int)steps;
  }
}

// Label of every extremum (batch-wide rank r): the rank among its image's
// surviving extrema of its thresholded union-find root, or -1 when the root is
// the void (cpu/cell_groups.hxx:128-146, 168-173). `alive_base[b]` is the
// first output rank of image b's extrema.
__global__ void label_map_kernel(int M, const int* __restrict__ ext_img, const int* __restrict__ ut_root,
                                 const int* __restrict__ region, const int* __restrict__ alive_base,
                                 int* __restrict__ lab) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  int u = ut_root[r];
  lab[r] = u < 0 ? -1 : region[u] - alive_base[ext_img[r]];
}

// Where the labels of one side go: image b's block of the output array picked
// by its orientation (faces are peaks in the primal, basins in the dual).
struct LabelOut {
  int* primal;            // output for primal images (nullptr: not requested)
  int* dual;              // output for dual images
  const int* primal_off;  // [B] block offset of image b in `primal`
  const int* dual_off;
};

// ---------------------------------------------------------------------------
// K9 (tiled): labels of both sides through 64 x 64 index tiles. A tile's flow
// codes are staged in shared memory, so every step of a V-path inside the
// tile is a shared-memory read. A path that leaves the tile continues from
// the first cell outside it, which lies on the border of the neighbouring
// tile: label_tile_kernel writes, for every border cell of every tile, its
// label or the border-map entry of the cell its path next enters, and lists
// the cells whose paths leave their tile; label_exit_kernel then crosses each
// further tile of such a path with one lookup in that border map.
constexpr int kLT = 64;
constexpr int kLTN = kLT * kLT;
constexpr int kPerim = 4 * kLT;  // border slots per tile: top row, bottom row, left column, right column

struct LabelTile {
  int b, H, W, Nx, y0, x0;
  long long base;  // global index of the tile's first cell
};

__device__ __forceinline__ LabelTile label_tile_of(const Imgs& I, int t) {
  LabelTile g;
  g.b = find_image(I.ltile_base, I.B, t);
  g.H = I.H[g.b];
  g.W = I.W[g.b];
  g.Nx = g.W + 1;
  const int ntx = (g.W + kLT) / kLT;  // ceil((W + 1) / 64)
  const int tt = t - I.ltile_base[g.b];
  const int ty = tt / ntx, tx = tt - ty * ntx;
  g.y0 = ty * kLT;
  g.x0 = tx * kLT;
  g.base = (long long)I.idx_base[g.b] + (long long)g.y0 * g.Nx + g.x0;
  return g;
}

// Flow bytes of the tile; cells beyond the image read as critical (never reached).
__device__ __forceinline__ void load_flow_tile(const uint8_t* __restrict__ flow, const LabelTile& g,
                                               uint8_t (*fl)[kLT], int tid, int nthreads) {
  for (int i = tid; i < kLTN; i += nthreads) {
    const int r = i / kLT, c = i % kLT;
    const bool in = g.y0 + r <= g.H && g.x0 + c <= g.W;
    fl[r][c] = in ? __ldg(flow + g.base + (long long)r * g.Nx + c) : (uint8_t)0;
  }
}

__device__ __forceinline__ int perim_slot(int r, int c) {
  return r == 0 ? c : r == kLT - 1 ? kLT + c : c == 0 ? 2 * kLT + r : 3 * kLT + r;
}

// Per tile: for each row and each of its two 32-cell segments, the bit mask
// of the critical faces (maxima of the face side) and critical vertices, and
// the segment's first rank in the batch-wide critical lists (the exclusive
// scans of the compaction), so a critical cell's list rank is
// off + popc(bits below it) and needs no index-sized map.
struct TileRanks {
  uint32_t fbits[kLT][2], vbits[kLT][2];
  int foff[kLT][2], voff[kLT][2];
};

__device__ __forceinline__ void tile_ranks(const uint8_t (*fl)[kLT], const LabelTile& g, const Imgs& I,
                                           const int* __restrict__ off_f, const int* __restrict__ off_v,
                                           TileRanks& R) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nsegx = (g.W + 32) / 32;  // 32-index row segments of the compaction: ceil((W + 1) / 32)
  for (int rs = warp; rs < 2 * kLT; rs += nw) {
    const int r = rs >> 1, sg = rs & 1;
    const int y = g.y0 + r, x = g.x0 + sg * 32 + lane;
    const unsigned code = fl[r][sg * 32 + lane];
    const unsigned fb = __ballot_sync(0xffffffffu, y <= g.H && x <= g.W && (code >> 4) == kFlowNone);
    const unsigned vb = __ballot_sync(0xffffffffu, y < g.H && x < g.W && (code & 0xFu) == kFlowNone);
    if (lane == 0) {
      R.fbits[r][sg] = fb;
      R.vbits[r][sg] = vb;
      const bool seg_in = y <= g.H && g.x0 + sg * 32 <= g.W;
      const long long sid = (long long)I.seg_base[g.b] + (long long)y * nsegx + (g.x0 >> 5) + sg;
      R.foff[r][sg] = (seg_in && off_f) ? __ldg(off_f + sid) : 0;
      R.voff[r][sg] = (seg_in && off_v) ? __ldg(off_v + sid) : 0;
    }
  }
}

// Label of the critical cell at tile-local id j (FACES: a face of the face
// side, else a vertex): lab[rank].
template <bool FACES>
__device__ __forceinline__ int tile_label(const TileRanks& R, int j, const int* __restrict__ lab) {
  const int r = j / kLT, c = j % kLT, sg = c >> 5;
  const uint32_t below = (1u << (c & 31)) - 1u;
  const int rank = FACES ? R.foff[r][sg] + __popc(R.fbits[r][sg] & below)
                         : R.voff[r][sg] + __popc(R.vbits[r][sg] & below);
  return __ldg(lab + rank);
}

// In-tile resolution of a tile's cells for both sides. st[side][i] starts as
// the cell's successor decoded once from its flow code: kDone | i for a
// critical cell, kDone | kExit | i when the successor lies outside the tile,
// else the successor's tile-local id. Pointer jumping in place
// (st[i] = st[st[i]] for the cells not yet done; every value read is still a
// position on the cell's path) doubles the distance covered per round, so a
// path of n steps inside the tile resolves in about log2(n) rounds; then
// st[i] = kDone | [kExit] | (the critical cell reached, or the path's last
// cell in the tile).
constexpr unsigned kDone = 0x8000u, kExit = 0x4000u, kCell = 0x0FFFu;

template <int SHIFT>
__device__ __forceinline__ uint16_t tile_succ(const uint8_t (*fl)[kLT], int r, int c) {
  const unsigned code = ((unsigned)fl[r][c] >> SHIFT) & 0xFu;
  const unsigned i = (unsigned)(r * kLT + c);
  if (code == kFlowNone) return (uint16_t)(kDone | i);
  const int nr = r + (code == kFlowUp ? -1 : code == kFlowDown ? 1 : 0);
  const int nc = c + (code == kFlowLeft ? -1 : code == kFlowRight ? 1 : 0);
  if ((unsigned)nr >= (unsigned)kLT || (unsigned)nc >= (unsigned)kLT) return (uint16_t)(kDone | kExit | i);
  return (uint16_t)(nr * kLT + nc);
}

constexpr int kLabelThreads = 1024;
constexpr int kTileCells = kLTN / kLabelThreads;  // 4 cells per thread: rows tid/64 + 16k

// st[0] faces, st[1] vertices, for the sides whose flags are set.
__device__ __forceinline__ void tile_resolve(const uint8_t (*fl)[kLT], uint16_t (*st)[kLTN], bool do_f, bool do_v,
                                             unsigned* status) {
  const int c = threadIdx.x % kLT, rb = threadIdx.x / kLT;
  unsigned pending = 0;  // bit 2k + side
#pragma unroll
  for (int k = 0; k < kTileCells; ++k) {
    const int r = rb + 16 * k, i = r * kLT + c;
    if (do_f) {
      const uint16_t v = tile_succ<4>(fl, r, c);
      st[0][i] = v;
      if (!(v & kDone)) pending |= 1u << (2 * k);
    }
    if (do_v) {
      const uint16_t v = tile_succ<0>(fl, r, c);
      st[1][i] = v;
      if (!(v & kDone)) pending |= 2u << (2 * k);
    }
  }
  int round = 0;
  for (; round < 16; ++round) {
    if (!__syncthreads_or(pending != 0)) break;
#pragma unroll
    for (int k = 0; k < kTileCells; ++k) {
      const int i = (rb + 16 * k) * kLT + c;
#pragma unroll
      for (int sd = 0; sd < 2; ++sd) {
        if (!((pending >> (2 * k + sd)) & 1u)) continue;
        const unsigned w = st[sd][st[sd][i] & kCell];
        st[sd][i] = (uint16_t)w;
        if (w & kDone) pending &= ~(1u << (2 * k + sd));
      }
    }
  }
  if (round == 16 && pending) set_status(status, kStatusWalkCap);
  __syncthreads();
}

// Border map entry or label of a resolved state: (label << 1) | 1 for a
// critical cell in the tile, else (border-map index of the next tile's entry
// cell) << 1. Tile `tile` of an image with `ntx` tiles per row.
template <bool FACES>
__device__ __forceinline__ int state_entry(unsigned w, const uint8_t (*fl)[kLT], const TileRanks& R,
                                           const int* __restrict__ lab, int tile, int ntx) {
  const int j = (int)(w & kCell);
  if (!(w & kExit)) return (int)(((unsigned)tile_label<FACES>(R, j, lab) << 1) | 1u);
  const int r = j / kLT, c = j % kLT;
  const unsigned code = ((unsigned)fl[r][c] >> (FACES ? 4 : 0)) & 0xFu;
  int nt, nr = r, nc = c;
  if (code == kFlowLeft) {
    nt = tile - 1;
    nc = kLT - 1;
  } else if (code == kFlowRight) {
    nt = tile + 1;
    nc = 0;
  } else if (code == kFlowUp) {
    nt = tile - ntx;
    nr = kLT - 1;
  } else {
    nt = tile + ntx;
    nr = 0;
  }
  return (int)(((long long)nt * kPerim + perim_slot(nr, nc)) << 1);
}

// Follows border-map entries to a label.
__device__ __forceinline__ int entry_label(int e, const int* __restrict__ perim, int cap, unsigned* status) {
  for (int h = 0; h <= cap; ++h) {
    if (e & 1) return e >> 1;
    e = __ldg(perim + (e >> 1));
  }
  set_status(status, kStatusWalkCap);
  return -1;
}

struct LabelSide {
  const int* off;  // segment offsets of this side's critical list (exclusive scan)
  const int* lab;  // label per critical extremum (batch-wide rank)
  int* perim;      // border map (nullptr: side not labelled)
};

__device__ __forceinline__ int label_ntx(const LabelTile& g) { return (g.W + kLT) / kLT; }

// Labels of every cell of a tile: face labels over the (H+1) x (W+1) indices,
// vertex labels over the H x W pixels (cpu/cell_groups.hxx:151-228). A cell
// whose path ends inside the tile gets its label here; the tile's border
// cells also get their border-map entries; a cell whose path leaves the tile
// is appended to its side's exit list (global index, entry) and finished by
// label_exit_kernel once every tile's border map is written.
__global__ void __launch_bounds__(kLabelThreads, 2) label_tile_kernel(Imgs I, const uint8_t* __restrict__ flow,
                                                                   LabelSide F, LabelSide V, LabelOut OF, LabelOut OV,
                                                                   int2* __restrict__ exits_f, int2* __restrict__ exits_v,
                                                                   int* __restrict__ n_exits, unsigned* status) {
  __shared__ uint8_t fl[kLT][kLT];
  __shared__ uint16_t st[2][kLTN];
  __shared__ TileRanks R;
  const LabelTile g = label_tile_of(I, blockIdx.x);
  const bool d = I.dual[g.b];
  int* of = d ? OF.dual : OF.primal;
  int* ov = d ? OV.dual : OV.primal;
  if (of) of += (d ? OF.dual_off : OF.primal_off)[g.b];
  if (ov) ov += (d ? OV.dual_off : OV.primal_off)[g.b];
  load_flow_tile(flow, g, fl, threadIdx.x, blockDim.x);
  __syncthreads();
  tile_ranks(fl, g, I, F.off, V.off, R);
  tile_resolve(fl, st, F.perim != nullptr, V.perim != nullptr, status);
  const int c = threadIdx.x % kLT, rb = threadIdx.x / kLT;
  const int ntx = label_ntx(g);
  const bool border_c = c == 0 || c == kLT - 1;
  // cells of this thread whose path leaves the tile, on a side whose labels
  // this image outputs: bit 2k (faces) and 2k + 1 (vertices); all of them are
  // reserved in the exit lists at once
  unsigned xm = 0;
#pragma unroll
  for (int k = 0; k < kTileCells; ++k) {
    const int r = rb + 16 * k, i = r * kLT + c;
    const int y = g.y0 + r, x = g.x0 + c;
    if (F.perim && of && y <= g.H && x <= g.W && (st[0][i] & kExit)) xm |= 1u << (2 * k);
    if (V.perim && ov && y < g.H && x < g.W && (st[1][i] & kExit)) xm |= 2u << (2 * k);
  }
  int pf, pv;
  block_reserve2(n_exits + 0, __popc(xm & 0x55u), n_exits + 1, __popc(xm & 0xAAu), pf, pv);
#pragma unroll 1
  for (int k = 0; k < kTileCells; ++k) {
    const int r = rb + 16 * k, i = r * kLT + c;
    const int y = g.y0 + r, x = g.x0 + c;
    const long long gidx = g.base + (long long)r * g.Nx + c;
    const bool border = border_c || r == 0 || r == kLT - 1;
    const long long po = (long long)blockIdx.x * kPerim + perim_slot(r, c);
    if (F.perim && y <= g.H && x <= g.W) {
      // odd: (label << 1) | 1 of a path ending in the tile; even: exit entry
      const int ef = state_entry<true>(st[0][i], fl, R, F.lab, blockIdx.x, ntx);
      if (border) F.perim[po] = ef;
      if (of && (ef & 1)) of[(long long)y * g.Nx + x] = ef >> 1;
      if ((xm >> (2 * k)) & 1u) exits_f[pf++] = make_int2((int)gidx, ef);
    }
    if (V.perim && y < g.H && x < g.W) {
      const int ev = state_entry<false>(st[1][i], fl, R, V.lab, blockIdx.x, ntx);
      if (border) V.perim[po] = ev;
      if (ov && (ev & 1)) ov[(long long)y * g.W + x] = ev >> 1;
      if ((xm >> (2 * k + 1)) & 1u) exits_v[pv++] = make_int2((int)gidx, ev);
    }
  }
}

// Cells whose paths leave their tile: follow the border map to the label.
template <bool FACES>
__global__ void __launch_bounds__(256) label_exit_kernel(Imgs I, const int2* __restrict__ exits,
                                                         const int* __restrict__ n_exits, const int* __restrict__ perim,
                                                         LabelOut O, int cap, unsigned* status) {
  const int n = *n_exits;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int2 e = exits[q];
    const int b = find_image(I.idx_base, I.B, e.x);
    const bool d = I.dual[b];
    int* out = d ? O.dual : O.primal;
    const int W = I.W[b], Nx = W + 1;
    const int lidx = e.x - I.idx_base[b];
    const int y = lidx / Nx, x = lidx - y * Nx;
    out += (d ? O.dual_off : O.primal_off)[b];
    out[FACES ? lidx : y * W + x] = entry_label(e.y, perim, cap, status);
  }
}

}  // namespace dmsc
