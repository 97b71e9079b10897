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
  while ((c = (__ldg(flow + idx) >> SHIFT) & 7u) != kFlowNone) {
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
                                                          long long* __restrict__ lf, int* __restrict__ tv,
                                                          long long* __restrict__ lv, long long cap, unsigned* status) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsad) return;
  const int b = sad_img[s];
  const int H = I.H[b], W = I.W[b], Nx = W + 1;
  int sc = crit_sad[s];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    long long steps;
    int end = flow_walk<4>(flow, face_start(sc, j, Nx) >> 2, Nx, cap, &steps, status);
    const int target = seg_rank(I, b, end, Nx, off_max, max_bits);
    tf[2 * s + j] = target;
    lf[2 * s + j] = target >= 0 ? steps + 1 : 0;  // cells of the raw arc, start and end included
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int start = vertex_start(sc, j, H, W, Nx, I.idx_base[b]);
    long long steps = 0;
    int target = -1;
    if (start >= 0) {
      int end = flow_walk<0>(flow, start >> 2, Nx, cap, &steps, status);
      target = seg_rank(I, b, end, Nx, off_min, min_bits);
    }
    tv[2 * s + j] = target;
    lv[2 * s + j] = target >= 0 ? steps + 1 : 0;  // an arc that leaves the image is empty
  }
}

// Label of every extremum (batch-wide rank r): the rank among its image's
// surviving extrema of its thresholded union-find root, or -1 when the root is
// the void (cpu/cell_groups.hxx:128-146, 168-173). `alive_base[b]` is the
// first output rank of image b's extrema.
__global__ void label_map_kernel(int M, const int* __restrict__ ext_img, const int* __restrict__ rout,
                                 const int* __restrict__ alive_base, int* __restrict__ lab) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  const int o = rout[r];  // batch-wide out rank of the root (-1: the void)
  lab[r] = o < 0 ? -1 : o - alive_base[ext_img[r]];
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
    const unsigned fb = __ballot_sync(0xffffffffu, y <= g.H && x <= g.W && ((code >> 4) & 7u) == kFlowNone);
    const unsigned vb = __ballot_sync(0xffffffffu, y < g.H && x < g.W && (code & 7u) == kFlowNone);
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

// In-tile resolution. Every (side, cell) of the tile has a 16-bit successor
// and a 32-bit state. A terminal cell (critical, or whose successor lies
// outside the tile) has successor kTerm | itself and a final state from the
// start: the entry (label << 1) | 1 of its extremum (label -1 encodes as all
// ones), or (border-map index of the cell its path enters next, in the
// neighbouring tile) << 1. Every other cell walks its successors for up to
// kWalk steps (paths are short: means of 3.2 steps for faces and 1.5 for
// vertices on the bench field) and takes the state of the terminal cell it
// reaches; a cell still walking after kWalk steps becomes pending (kPend | the
// cell reached), and pending cells then jump their pointers,
// state = state of the pointed-to cell, without block barriers: any state
// read belongs to a cell further along the same path (written by any thread,
// at any time), so a pointer only moves toward the path's end and gets there
// in at most the path's length of jumps. Border-map indices and labels stay
// below 2^30, so the top two bits tell a pending state apart.
constexpr uint32_t kPend = 0x40000000u, kCellMask = 0x0FFFu;
constexpr unsigned kTerm = 0x8000u;
constexpr int kWalk = 8;
__device__ __forceinline__ bool st_pending(uint32_t v) { return (v >> 30) == 1u; }

// Threads per label tile (the tuner picks one): each thread owns column
// tid % 64 of rows tid / 64 + (NT / 64) k, k < 4096 / NT.
constexpr int kLabelShapes = 2;
constexpr int kLabelNT[kLabelShapes] = {1024, 512};

// Successor of the cell at tile position (r, c) (FACES: face side; the cell
// is in the image) and, for a terminal cell, its final state.
template <bool FACES>
__device__ __forceinline__ uint16_t tile_step(const uint8_t (*fl)[kLT], const TileRanks& R,
                                              const int* __restrict__ lab, int r, int c, int tile, int ntx,
                                              uint32_t* final_state) {
  const unsigned code = ((unsigned)fl[r][c] >> (FACES ? 4 : 0)) & 7u;
  const int i = r * kLT + c;
  if (code == kFlowNone) {
    *final_state = ((uint32_t)tile_label<FACES>(R, i, lab) << 1) | 1u;
    return (uint16_t)(kTerm | i);
  }
  int nr = r, nc = c, nt = tile;
  if (code == kFlowLeft) {
    if (--nc < 0) {
      nt = tile - 1;
      nc = kLT - 1;
    }
  } else if (code == kFlowRight) {
    if (++nc == kLT) {
      nt = tile + 1;
      nc = 0;
    }
  } else if (code == kFlowUp) {
    if (--nr < 0) {
      nt = tile - ntx;
      nr = kLT - 1;
    }
  } else {
    if (++nr == kLT) {
      nt = tile + ntx;
      nr = 0;
    }
  }
  if (nt != tile) {
    *final_state = (uint32_t)(((long long)nt * kPerim + perim_slot(nr, nc)) << 1);
    return (uint16_t)(kTerm | i);
  }
  return (uint16_t)(nr * kLT + nc);
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
// Shared memory of a label tile (55 KB: dynamic shared memory).
struct LabelSmem {
  uint32_t st[2][kLTN];
  uint16_t succ[2][kLTN];
  uint8_t fl[kLT][kLT];
  TileRanks R;
};

template <int NT>
__global__ void __launch_bounds__(NT, 2048 / NT) label_tile_kernel(Imgs I, const uint8_t* __restrict__ flow,
                                                                   LabelSide F, LabelSide V, LabelOut OF, LabelOut OV,
                                                                   int2* __restrict__ exits_f, int2* __restrict__ exits_v,
                                                                   int* __restrict__ n_exits, unsigned* status) {
  extern __shared__ __align__(16) unsigned char label_smem[];
  LabelSmem& SM = *reinterpret_cast<LabelSmem*>(label_smem);
  uint8_t (*fl)[kLT] = SM.fl;
  uint16_t (*succ)[kLTN] = SM.succ;
  uint32_t (*st)[kLTN] = SM.st;
  TileRanks& R = SM.R;
  constexpr int kTileCells = kLTN / NT, kStep = NT / kLT;
  const LabelTile g = label_tile_of(I, blockIdx.x);
  const bool d = I.dual[g.b];
  int* of = d ? OF.dual : OF.primal;
  int* ov = d ? OV.dual : OV.primal;
  if (of) of += (d ? OF.dual_off : OF.primal_off)[g.b];
  if (ov) ov += (d ? OV.dual_off : OV.primal_off)[g.b];
  load_flow_tile(flow, g, fl, threadIdx.x, blockDim.x);
  __syncthreads();
  tile_ranks(fl, g, I, F.off, V.off, R);
  __syncthreads();
  const int c = threadIdx.x % kLT, rb = threadIdx.x / kLT;
  const int ntx = label_ntx(g);
  const bool do_f = F.perim != nullptr, do_v = V.perim != nullptr;
  // successors; terminal cells get their final state (cells outside the
  // image are terminal and never reached)
#pragma unroll
  for (int k = 0; k < kTileCells; ++k) {
    const int r = rb + kStep * k, i = r * kLT + c;
    const int y = g.y0 + r, x = g.x0 + c;
    uint32_t a = 1u, b = 1u;
    uint16_t sa = (uint16_t)(kTerm | i), sb = sa;
    if (do_f && y <= g.H && x <= g.W) sa = tile_step<true>(fl, R, F.lab, r, c, blockIdx.x, ntx, &a);
    if (do_v && y < g.H && x < g.W) sb = tile_step<false>(fl, R, V.lab, r, c, blockIdx.x, ntx, &b);
    succ[0][i] = sa;
    succ[1][i] = sb;
    if (sa & kTerm) st[0][i] = a;
    if (sb & kTerm) st[1][i] = b;
  }
  __syncthreads();
  // short walks to the terminal cell; bit 2k + side of `pend`: still walking
  unsigned pend = 0;
#pragma unroll
  for (int q = 0; q < 2 * kTileCells; ++q) {
    const int sd = q & 1, i = (rb + kStep * (q >> 1)) * kLT + c;
    unsigned cur = succ[sd][i];
    if (cur & kTerm) continue;
    unsigned nx = succ[sd][cur];
#pragma unroll 1
    for (int w = 1; w < kWalk && !(nx & kTerm); ++w) {
      cur = nx;
      nx = succ[sd][cur];
    }
    if (nx & kTerm) {
      st[sd][i] = st[sd][cur];  // cur is terminal: its state is final
    } else {
      st[sd][i] = kPend | cur;
      pend |= 1u << q;
    }
  }
  __syncthreads();
  {  // barrier-free pointer jumping of this thread's pending cells (only this
     // thread writes its cells' states; other threads read them at any time)
    volatile uint32_t* vs = &st[0][0];
    for (int it = 0; pend; ++it) {
      if (it >= kLTN) {  // a path is at most kLTN cells long inside a tile
        set_status(status, kStatusWalkCap);
        break;
      }
#pragma unroll
      for (int q = 0; q < 2 * kTileCells; ++q) {
        if (!((pend >> q) & 1u)) continue;
        const int side = (q & 1) * kLTN, i = side + (rb + kStep * (q >> 1)) * kLT + c;
        const uint32_t w = vs[side + (vs[i] & kCellMask)];
        vs[i] = w;
        if (!st_pending(w)) pend &= ~(1u << q);
      }
    }
  }
  // this thread's own states are final now (read back from shared memory)
  const bool border_c = c == 0 || c == kLT - 1;
  // cells of this thread whose path leaves the tile, on a side whose labels
  // this image outputs: bit 2k (faces) and 2k + 1 (vertices); all of them are
  // reserved in the exit lists at once
  unsigned xm = 0;
#pragma unroll
  for (int k = 0; k < kTileCells; ++k) {
    const int y = g.y0 + rb + kStep * k, x = g.x0 + c;
    const int i = (rb + kStep * k) * kLT + c;
    if (do_f && of && y <= g.H && x <= g.W && !(st[0][i] & 1u)) xm |= 1u << (2 * k);
    if (do_v && ov && y < g.H && x < g.W && !(st[1][i] & 1u)) xm |= 2u << (2 * k);
  }
  int pf, pv;
  block_reserve2(n_exits + 0, __popc(xm & 0x55555555u), n_exits + 1, __popc(xm & 0xAAAAAAAAu), pf, pv);
#pragma unroll
  for (int k = 0; k < kTileCells; ++k) {
    const int r = rb + kStep * k;
    const int y = g.y0 + r, x = g.x0 + c;
    const long long gidx = g.base + (long long)r * g.Nx + c;
    const bool border = border_c || r == 0 || r == kLT - 1;
    const long long po = (long long)blockIdx.x * kPerim + perim_slot(r, c);
    if (do_f && y <= g.H && x <= g.W) {
      // odd: (label << 1) | 1 of a path ending in the tile; even: exit entry
      const int ef = (int)st[0][r * kLT + c];
      if (border) F.perim[po] = ef;
      if (of && (ef & 1)) of[(long long)y * g.Nx + x] = ef >> 1;
      if ((xm >> (2 * k)) & 1u) exits_f[pf++] = make_int2((int)gidx, ef);
    }
    if (do_v && y < g.H && x < g.W) {
      const int ev = (int)st[1][r * kLT + c];
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
