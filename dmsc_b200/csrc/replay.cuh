// Arc simplification: replay of the cancellations and emission of the
// simplified arc geometry.
//
// Reference semantics: cpu/arcs_simplification.hxx:310-504. The cancellations
// of one side are replayed in (persistence, saddle cell, target cell) order on
// a union-find whose roots are extrema. For a cancellation of saddle s killing
// extremum d, with arc targets T0 and T1: R0 = Find(T0), R1 = Find(T1); if
// R0 == d != R1 then d is linked under R1 (symmetric for R1 == d); otherwise
// the cancellation is skipped. Every link carries a path: the geometry from d
// back along the dying side's arc through s and on to the other root.
//
// Parallel form (exact). Links never move once made and link times increase
// along every parent chain, so the root of x just before replay step t is the
// first node on x's parent chain that is not linked before t. Each unresolved
// cancellation walks its two chains; it can decide as soon as every node it
// passes has been decided, and decisions are final, so rounds of such walks
// reproduce the sequential replay (including skips, which arise only from
// ties in persistence). Path lengths are summed along the same walks.
//
// Geometry. A link's path W(d) is
//   reverse(chain(T_dying -> d)) + reverse(arc_dying) + arc_other + chain(T_other -> R)
// where chain(x -> R) concatenates W along x's parent chain up to R, and every
// surviving saddle's final arc is arc + chain(T -> root). These are expanded
// breadth-first as chain tasks that each cover a known output range (a chain
// task writes every W along its chain at once: their raw-arc segments and
// their own chains as the next level's tasks); raw arcs are re-walked from
// their start cells when written.
#pragma once

#include "common.cuh"
#include "walks.cuh"

namespace dmsc {

constexpr unsigned long long kNever = ~0ull;  // replay key of a node that is never cancelled
enum : int { kPending = 0, kLinked = 1, kRootForever = 2 };
// A replay status word is kind | tag << 2; a decision made in replay round r
// carries tag r + 1 (the initial kRootForever of never-cancelled nodes has
// tag 0). Walks in round r use only decisions with tag <= r: those were
// written before the grid barrier that opened round r, which orders them, so
// plain (L2) loads see them complete and no acquire/release is needed.
__device__ __forceinline__ int status_kind(int st) { return st & 3; }
__device__ __forceinline__ int status_word(int kind, int round) { return kind | ((round + 1) << 2); }

// A replay node in one 64-byte line: everything a chain walk reads, in the
// first 32-byte sector as two 16-byte halves, (ctime, wlen) and (status,
// parent, side, saddle cell); in the second, what the emission needs to expand
// W(node) without touching the saddle's arrays: the two chain lengths, the
// saddle's arc ends on the dying and the other side and their raw-arc
// lengths (written at link time).
struct alignas(64) ReplayNode {
  unsigned long long ctime;  // replay key of the cancellation killing the node, kNever if none
  long long wlen;            // length of W(node)
  int status;                // kPending / kLinked / kRootForever, with the deciding round's tag
  int parent;                // link target (-1 = void) when kLinked
  int side;                  // side_word: dying side of the node's cancellation and what W(node) expands to
  int scell;                 // global cell id of the saddle of the node's cancellation
  long long cl_dy;           // chain length T_dying -> node at link time
  long long cl_ot;           // chain length T_other -> parent at link time
  int t_dy, t_ot;            // the saddle's arc ends on the dying and the other side
  int len_dy, len_ot;        // their raw-arc lengths (cells; a side's geometry stays below 2^31)
};
static_assert(sizeof(ReplayNode) == 64, "one 64-byte line per node");

struct ReplayState {
  ReplayNode* node;  // [M + 1]
};

// The halves of a node's record: through L2 inside the replay (other blocks
// write records during the launch), plain loads after it.
__device__ __forceinline__ longlong2 node_keylen_cg(const ReplayNode* n, int x) {
  return __ldcg(reinterpret_cast<const longlong2*>(&n[x].ctime));
}
__device__ __forceinline__ longlong2 node_keylen(const ReplayNode* n, int x) {
  return *reinterpret_cast<const longlong2*>(&n[x].ctime);
}
__device__ __forceinline__ int4 node_words(const ReplayNode* n, int x) {
  return *reinterpret_cast<const int4*>(&n[x].status);
}

// Node records are written only for the nodes a cancellation kills: the
// persistence pass sets their key and kPending, and the replay their decision
// when it is made. Every reader first checks the side's alive flags: an alive
// extremum (no cancellation kills it) is a root forever and its record is
// never read, so no pass initialises the records of the others.
// Side word of a linked node: the dying side k (bit 0), the number of
// non-empty chains of W(node) (bits 1-2) and of its raw-arc segments (bits
// 3-4), so counting a chain's expansion reads one word per node.
__device__ __forceinline__ int side_word(int k, int n_chain, int n_base) { return k | (n_chain << 1) | (n_base << 3); }
__device__ __forceinline__ int side_of(int w) { return w & 1; }
__device__ __forceinline__ int chains_of(int w) { return (w >> 1) & 3; }
__device__ __forceinline__ int bases_of(int w) { return (w >> 3) & 3; }

// Root of x just before the replay step with key t, with the summed path
// length; returns false when a node on the way is still undecided. Replay
// steps are compared by their (persistence, saddle cell) keys, which are
// unique, so no ranks are needed.
__device__ __forceinline__ bool walk_root(const ReplayState& S, const uint8_t* __restrict__ alive, int x,
                                          unsigned long long t, int* root, long long* acc, int max_steps,
                                          unsigned* status) {
  long long a = 0;
  int steps = 0;
  while (x >= 0 && !alive[x]) {
    const longlong2 kl = node_keylen(S.node, x);
    const int4 w = node_words(S.node, x);
    if ((unsigned long long)kl.x >= t) break;
    const int st = status_kind(w.x);
    if (st == kPending) return false;
    if (st == kRootForever) break;
    a += kl.y;
    x = w.y;
    if (++steps > max_steps) {
      set_status(status, kStatusChainCap);
      break;
    }
  }
  *root = x;
  *acc = a;
  return true;
}

// Final arcs of the surviving saddles: length and the chain root of each
// (survivor i in output order, arcs 0 and 1), and the survivor's total path
// length, from the survivors' gathered records (image, arc ends, raw-arc
// lengths). Images whose output does not take this side's arcs
// (`arcs_primal` / `arcs_dual` by orientation) get empty arcs.
__global__ void final_arcs_kernel(int nsurv, const int2* __restrict__ surv_ic, const uint8_t* __restrict__ dual,
                                  bool arcs_primal, bool arcs_dual, const int2* __restrict__ sv_t,
                                  const longlong2* __restrict__ sv_len, const uint8_t* __restrict__ alive,
                                  ReplayState S, int max_steps, long long* __restrict__ arc_len,
                                  long long* __restrict__ arc_cl, int* __restrict__ arc_root,
                                  long long* __restrict__ plen, unsigned* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsurv) return;
  const int2 tt = sv_t[i];
  const longlong2 bl = sv_len[i];
  const bool take = dual[surv_ic[i].x] ? arcs_dual : arcs_primal;
  long long len[2] = {0, 0}, cl[2] = {0, 0};
  int root[2] = {-1, -1};
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int T = j ? tt.y : tt.x;
    if (T < 0 || !take) continue;
    // an extremum that no cancellation kills (alive) is its own final root;
    // only the others walk their parent chains
    int R = T;
    long long a = 0;
    if (!alive[T]) walk_root(S, alive, T, kNever, &R, &a, max_steps, status);
    len[j] = (j ? bl.y : bl.x) + a;
    cl[j] = a;
    root[j] = R;
  }
  *reinterpret_cast<longlong2*>(arc_len + 2 * i) = make_longlong2(len[0], len[1]);
  *reinterpret_cast<longlong2*>(arc_cl + 2 * i) = make_longlong2(cl[0], cl[1]);
  *reinterpret_cast<int2*>(arc_root + 2 * i) = make_int2(root[0], root[1]);
  plen[i] = len[0] + len[1];
}

// ---------------------------------------------------------------------------
// geometry emission
// ---------------------------------------------------------------------------
enum : int { kTaskChain = 2 };
// chain task = {kind | dir << 2, start node, stop node (-1 = void), pos}
__device__ __forceinline__ int4 make_task(int kind, int rev, int a, int b, long long pos) {
  return make_int4(kind | (rev << 2), a, b, (int)pos);
}

struct EmitCtx {
  const uint8_t* flow;
  Imgs I;
  bool faces;
  ReplayState S;
  int* out_primal;  // destination of primal images' arcs of this side
  int* out_dual;    // destination of dual images' arcs
  const int* dst_off;  // [B] start of each image's geometry in its destination (positions are image-local)
  long long q_cap;
  int4* base_q;  // raw-arc segments of the chain expansion
  long long base_cap;
  // the survivors' own raw arcs (segment items 0 .. 2 nsurv - 1 of the
  // writer, read from the survivor records instead of a task list)
  int nvirt;                 // 2 nsurv
  const int2* surv_ic;       // [nsurv] image and cell of each survivor (output order)
  const int2* sv_t;          // [nsurv] this side's arc ends
  const longlong2* sv_len;   // [nsurv] this side's raw-arc lengths
  const long long* arc_pos;  // [2 nsurv] image-local output position of each arc
  int max_steps;
  unsigned* status;
};

// A raw-arc segment task of the chain expansion: {reversed | arc << 1,
// saddle cell, cells, output position}: the writer finds the arc's start
// cell from the saddle's cell with no further load.
__device__ __forceinline__ int arc_start_of_cell(const EmitCtx& E, int sc, int j, int b) {
  const int W = E.I.W[b], Nx = W + 1;
  const int cell = E.faces ? face_start(sc, j, Nx) : vertex_start(sc, j, E.I.H[b], W, Nx, E.I.idx_base[b]);
  return cell >> 2;
}
__device__ __forceinline__ int4 make_saddle_seg(int scell, int j, int rev, long long len, long long pos) {
  return make_int4(rev | (j << 1), scell, (int)len, (int)pos);
}

// A raw arc being written by one lane: the V-path from its start cell, `len`
// cells (cpu/arcs_geometry.hxx:83-111, 133-161), following the flow codes.
// dst is the next output slot, step its stride (-1 for a reversed arc), rem
// the cells left and idx the current index.
struct SegCursor {
  int* dst;
  int step;
  int rem;
  int idx, ibase, Nx;
};

// Starts segment item q: q < nvirt is raw arc (q / 2, q % 2) of a survivor,
// forward at its arc's output position; the others are the chain
// expansion's tasks. rem = 0 when it writes nothing (no arc, or its image's
// output does not take this side's arcs).
__device__ __forceinline__ void seg_start(const EmitCtx& E, long long q, SegCursor& c) {
  c.rem = 0;
  int b, idx, len, pos;
  bool rev;
  if (q < E.nvirt) {
    const int i = (int)(q >> 1), j = (int)(q & 1);
    const int2 tt = E.sv_t[i];
    const longlong2 bl = E.sv_len[i];
    len = (int)(j ? bl.y : bl.x);
    if ((j ? tt.y : tt.x) < 0 || len <= 0) return;
    const int2 ic = E.surv_ic[i];
    b = ic.x;
    idx = arc_start_of_cell(E, ic.y, j, b);
    pos = (int)E.arc_pos[q];
    rev = false;
  } else {
    const int4 t = E.base_q[q - E.nvirt];
    const int j = (t.x >> 1) & 1;
    len = t.z;
    b = find_image(E.I.idx_base, E.I.B, t.y >> 2);
    idx = arc_start_of_cell(E, t.y, j, b);
    pos = t.w;
    rev = t.x & 1;
  }
  int* out = E.I.dual[b] ? E.out_dual : E.out_primal;
  if (!out || len <= 0) return;
  c.Nx = E.I.W[b] + 1;
  c.ibase = E.I.idx_base[b];
  c.idx = idx;
  c.dst = out + E.dst_off[b] + (rev ? (long long)pos + len - 1 : (long long)pos);
  c.step = rev ? -1 : 1;
  c.rem = len;
}

}  // namespace dmsc
