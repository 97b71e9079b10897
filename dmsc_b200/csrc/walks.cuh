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

// Successor set-up of one (row, 32-cell segment) item of a tile for both
// sides, one lane per cell: a critical cell (terminal) takes the state
// (label << 1) | 1 of its extremum, lab[rank], where rank is the segment's
// first rank in the batch-wide critical list (the compaction's exclusive
// scan) plus the critical cells before it in the segment (a ballot); a cell
// whose successor lies in another tile (terminal) takes the border-map entry
// of that cell; any other cell gets its successor's tile-local id. Cells
// outside the image are terminal and never reached. `labf` / `labv`: the
// labels loaded for this lane's critical cells (issued for a group of a
// warp's items before any is used).
__device__ __forceinline__ void tile_cell_setup(const uint8_t (*fl)[kLT], const LabelTile& g, int tile, int ntx,
                                                int r, int c, bool do_f, bool do_v, bool critf, bool critv,
                                                int labf, int labv, uint16_t (*succ)[kLTN], uint32_t (*st)[kLTN]) {
  const int i = r * kLT + c;
  const unsigned code = fl[r][c];
  const int y = g.y0 + r, x = g.x0 + c;
#pragma unroll
  for (int sd = 0; sd < 2; ++sd) {
    const bool in = sd == 0 ? (do_f && y <= g.H && x <= g.W) : (do_v && y < g.H && x < g.W);
    const unsigned k = sd == 0 ? (code >> 4) & 7u : code & 7u;
    uint16_t sc = (uint16_t)(kTerm | i);
    uint32_t state = 1u;
    if (in) {
      if (sd == 0 ? critf : critv) {
        state = ((uint32_t)(sd == 0 ? labf : labv) << 1) | 1u;
      } else {
        const int dc = (k == kFlowRight) - (k == kFlowLeft), dr = (k == kFlowDown) - (k == kFlowUp);
        const int nr = r + dr, nc = c + dc;
        if ((unsigned)nr < (unsigned)kLT && (unsigned)nc < (unsigned)kLT) {
          sc = (uint16_t)(nr * kLT + nc);
        } else {  // enters the neighbouring tile at its border cell (nr, nc) mod 64
          const int nt = tile + dc + dr * ntx;
          state = (uint32_t)(((long long)nt * kPerim + perim_slot(nr & (kLT - 1), nc & (kLT - 1))) << 1);
        }
      }
    }
    succ[sd][i] = sc;
    if (sc & kTerm) st[sd][i] = state;
  }
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
  const int* off;    // segment offsets of this side's critical list (exclusive scan)
  const int* rout;   // per critical extremum (batch-wide rank): out rank of its thresholded root, -1 for the void
  const int* abase;  // [B + 1] first out rank of each image's alive extrema
  int* perim;        // border map (nullptr: side not labelled)
};

// Label of an extremum from its root's batch-wide out rank: the root's rank
// among its image's surviving extrema, -1 for the void
// (cpu/cell_groups.hxx:128-146, 168-173).
__device__ __forceinline__ int region_label(int rout, int abase) { return rout < 0 ? -1 : rout - abase; }

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
  constexpr int kTileCells = kLTN / NT, kStep = NT / kLT;
  constexpr int NW = NT / 32, kItems = 2 * kLT / NW;  // (row, segment) items per warp
  const LabelTile g = label_tile_of(I, blockIdx.x);
  const bool d = I.dual[g.b];
  int* of = d ? OF.dual : OF.primal;
  int* ov = d ? OV.dual : OV.primal;
  if (of) of += (d ? OF.dual_off : OF.primal_off)[g.b];
  if (ov) ov += (d ? OV.dual_off : OV.primal_off)[g.b];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ntx = label_ntx(g);
  const bool do_f = F.perim != nullptr, do_v = V.perim != nullptr;
  // the first ranks of this warp's items: lane k loads item k's (issued
  // before the flow tile is waited for)
  int offf = 0, offv = 0;
  const int abf = do_f ? __ldg(F.abase + g.b) : 0, abv = do_v ? __ldg(V.abase + g.b) : 0;
  if (lane < kItems) {
    const int rs = warp + NW * lane, r = rs >> 1, sg = rs & 1;
    const int y = g.y0 + r;
    if (y <= g.H && g.x0 + sg * 32 <= g.W) {
      const int nsegx = (g.W + 32) / 32;  // 32-index row segments of the compaction: ceil((W + 1) / 32)
      const long long sid = (long long)I.seg_base[g.b] + (long long)y * nsegx + (g.x0 >> 5) + sg;
      if (do_f && F.off) offf = __ldg(F.off + sid);
      if (do_v && V.off) offv = __ldg(V.off + sid);
    }
  }
  load_flow_tile(flow, g, fl, threadIdx.x, blockDim.x);
  __syncthreads();
  {  // successors and terminal states, one warp per (row, segment) item, in
     // groups of 4 items whose label loads are issued together
    const unsigned lt = (1u << lane) - 1u;
    constexpr int kGroup = kItems < 4 ? kItems : 4;
#pragma unroll
    for (int k0 = 0; k0 < kItems; k0 += kGroup) {
      int labf[kGroup], labv[kGroup];
      unsigned cf = 0, cv = 0;  // bit k: this lane's cell of item k0 + k is critical
#pragma unroll
      for (int k = 0; k < kGroup; ++k) {  // ranks and label loads of the critical cells
        const int rs = warp + NW * (k0 + k), r = rs >> 1, c = (rs & 1) * 32 + lane;
        const int y = g.y0 + r, x = g.x0 + c;
        const unsigned code = fl[r][c];
        const bool fcrit = do_f && y <= g.H && x <= g.W && ((code >> 4) & 7u) == kFlowNone;
        const bool vcrit = do_v && y < g.H && x < g.W && (code & 7u) == kFlowNone;
        const unsigned fb = __ballot_sync(0xffffffffu, fcrit), vb = __ballot_sync(0xffffffffu, vcrit);
        const int of0 = __shfl_sync(0xffffffffu, offf, k0 + k), ov0 = __shfl_sync(0xffffffffu, offv, k0 + k);
        labf[k] = fcrit ? region_label(__ldg(F.rout + of0 + __popc(fb & lt)), abf) : 0;
        labv[k] = vcrit ? region_label(__ldg(V.rout + ov0 + __popc(vb & lt)), abv) : 0;
        cf |= (unsigned)fcrit << k;
        cv |= (unsigned)vcrit << k;
      }
#pragma unroll
      for (int k = 0; k < kGroup; ++k) {
        const int rs = warp + NW * (k0 + k);
        tile_cell_setup(fl, g, blockIdx.x, ntx, rs >> 1, (rs & 1) * 32 + lane, do_f, do_v, (cf >> k) & 1u,
                        (cv >> k) & 1u, labf[k], labv[k], succ, st);
      }
    }
  }
  __syncthreads();
  const int c = threadIdx.x % kLT, rb = threadIdx.x / kLT;
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
  // this thread's own states are final now (read back from shared memory):
  // labels of paths that end in the tile, border-map entries of the border
  // cells, and a bit per cell whose path leaves the tile on a side whose
  // labels this image outputs (bit 2k: faces, 2k + 1: vertices); those are
  // reserved in the exit lists at once and written afterwards
  const bool border_c = c == 0 || c == kLT - 1;
  const int x = g.x0 + c;
  const bool fx = do_f && x <= g.W, vx = do_v && x < g.W;
  unsigned xm = 0;
  {
    int* ofr = of ? of + (g.y0 + rb) * g.Nx + x : nullptr;  // image-local outputs stay below 2^31
    int* ovr = ov ? ov + (g.y0 + rb) * g.W + x : nullptr;
#pragma unroll
    for (int k = 0; k < kTileCells; ++k) {
      const int r = rb + kStep * k, y = g.y0 + r, i = r * kLT + c;
      const bool border = border_c || r == 0 || r == kLT - 1;
      if (fx && y <= g.H) {
        // odd: (label << 1) | 1 of a path ending in the tile; even: exit entry
        const uint32_t ef = st[0][i];
        if (border) F.perim[blockIdx.x * kPerim + perim_slot(r, c)] = (int)ef;
        if (ofr) {
          if (ef & 1u)
            ofr[k * kStep * g.Nx] = (int)ef >> 1;
          else
            xm |= 1u << (2 * k);
        }
      }
      if (vx && y < g.H) {
        const uint32_t ev = st[1][i];
        if (border) V.perim[blockIdx.x * kPerim + perim_slot(r, c)] = (int)ev;
        if (ovr) {
          if (ev & 1u)
            ovr[k * kStep * g.W] = (int)ev >> 1;
          else
            xm |= 2u << (2 * k);
        }
      }
    }
  }
  int pf, pv;
  block_reserve2(n_exits + 0, __popc(xm & 0x55555555u), n_exits + 1, __popc(xm & 0xAAAAAAAAu), pf, pv);
  while (xm) {  // the few cells whose paths leave the tile
    const int q = __ffs(xm) - 1, k = q >> 1, sd = q & 1;
    xm &= xm - 1u;
    const int r = rb + kStep * k;
    const int gidx = (int)(g.base + (long long)r * g.Nx + c);  // global indices stay below 2^29
    const int e = (int)st[sd][r * kLT + c];
    if (sd == 0)
      exits_f[pf++] = make_int2(gidx, e);
    else
      exits_v[pv++] = make_int2(gidx, e);
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
