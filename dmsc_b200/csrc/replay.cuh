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
// parent, side, csad); the two chain lengths the emission adds in the second.
struct alignas(64) ReplayNode {
  unsigned long long ctime;  // replay key of the cancellation killing the node, kNever if none
  long long wlen;            // length of W(node)
  int status;                // kPending / kLinked / kRootForever, with the deciding round's tag
  int parent;                // link target (-1 = void) when kLinked
  int side;                  // side_word: dying side of the node's cancellation and what W(node) expands to
  int csad;                  // saddle of the node's cancellation
  long long cl_dy;           // chain length T_dying -> node at link time
  long long cl_ot;           // chain length T_other -> parent at link time
  long long pad[2];
};

struct ReplayState {
  ReplayNode* node;  // [M + 1]
};

// The halves of a node's record: through L2 inside the replay (other blocks
// write records during the launch), plain loads after it.
__device__ __forceinline__ longlong2 node_keylen_cg(const ReplayNode* n, int x) {
  return __ldcg(reinterpret_cast<const longlong2*>(&n[x].ctime));
}
__device__ __forceinline__ int4 node_words_cg(const ReplayNode* n, int x) {
  return __ldcg(reinterpret_cast<const int4*>(&n[x].status));
}
__device__ __forceinline__ longlong2 node_keylen(const ReplayNode* n, int x) {
  return *reinterpret_cast<const longlong2*>(&n[x].ctime);
}
__device__ __forceinline__ int4 node_words(const ReplayNode* n, int x) {
  return *reinterpret_cast<const int4*>(&n[x].status);
}

// Every node a root that is never cancelled, with tag 0 (a cancellation's
// own key and kPending are set when the replay starts).
__global__ void replay_node_init_kernel(ReplayNode* __restrict__ n, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  *reinterpret_cast<longlong2*>(&n[i].ctime) = make_longlong2((long long)kNever, 0);
  *reinterpret_cast<int4*>(&n[i].status) = make_int4(kRootForever, -1, 0, 0);
}

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
__device__ __forceinline__ bool walk_root(const ReplayState& S, int x, unsigned long long t, int* root,
                                          long long* acc, int max_steps, unsigned* status) {
  long long a = 0;
  int steps = 0;
  while (x >= 0) {
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

// The same walk resumed from (*x, *acc) and left there: returns false, with
// *x the first undecided node and *acc the length summed before it, when the
// walk has to wait; the prefix already walked is final (decisions never
// change), so a later round continues from that node.
__device__ __forceinline__ bool walk_resume(const ReplayState& S, int* x_io, unsigned long long t, long long* acc_io,
                                            int max_steps, unsigned* status, int round) {
  int x = *x_io;
  long long a = *acc_io;
  int steps = 0;
  bool done = true;
  while (true) {
    if (x < 0) break;
    const longlong2 kl = node_keylen_cg(S.node, x);  // one sector: both halves issued together
    const int4 w = node_words_cg(S.node, x);
    if ((unsigned long long)kl.x >= t) break;
    const int st = w.x;
    if (status_kind(st) == kPending || (st >> 2) > round) {  // undecided, or decided in this round
      done = false;
      break;
    }
    if (status_kind(st) == kRootForever) break;
    a += kl.y;
    x = w.y;
    if (++steps > max_steps) {
      set_status(status, kStatusChainCap);
      break;
    }
  }
  *x_io = x;
  *acc_io = a;
  return done;
}

// Cancellations of one side, compacted in any order with their sort keys
// (CancelEvent::operator<, cpu/persistence_struct.hxx:16-21): (persistence,
// saddle cell); a saddle is cancelled at most once per side, so the pair is
// unique and the target cell never breaks a tie.
__global__ void __launch_bounds__(256) cancel_collect_kernel(int nsad, const int* __restrict__ dying,
                                                             const float* __restrict__ pers,
                                                             const float* __restrict__ thr,
                                                             const int* __restrict__ sad_img,
                                                             const int* __restrict__ crit_sad,
                                                             unsigned long long* __restrict__ keys,
                                                             int* __restrict__ vals, int* __restrict__ count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;  // saddles in list order
  bool take = false;
  unsigned long long key = 0;
  if (s < nsad && dying[s] >= 0) {
    float p = pers[s];
    if (p <= thr[sad_img[s]]) {
      take = true;
      key = ((unsigned long long)orderable_key(p) << 32) | (unsigned)crit_sad[s];
    }
  }
  int pos = block_append(count, take);
  if (take) {
    keys[pos] = key;
    vals[pos] = s;
  }
}

// Final arcs of the surviving saddles: length and the chain root of each
// (survivor i in output order, arc j). `surv_sad[i]` = dense saddle index.
// Images whose output does not take this side's arcs (`arcs_primal` /
// `arcs_dual` by orientation) get empty arcs.
__global__ void final_arcs_kernel(int nsurv, const int* __restrict__ surv_sad, const int* __restrict__ sad_img,
                                  const uint8_t* __restrict__ dual, bool arcs_primal, bool arcs_dual,
                                  const int* __restrict__ t, const long long* __restrict__ blen, ReplayState S,
                                  int max_steps, long long* __restrict__ arc_len, long long* __restrict__ arc_cl,
                                  int* __restrict__ arc_root, unsigned* status) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * nsurv) return;
  int i = q >> 1, j = q & 1;
  int s = surv_sad[i];
  int T = t[2 * s + j];
  if (T < 0 || !(dual[sad_img[s]] ? arcs_dual : arcs_primal)) {
    arc_len[q] = 0;
    arc_cl[q] = 0;
    arc_root[q] = -1;
    return;
  }
  int R;
  long long a;
  walk_root(S, T, kNever, &R, &a, max_steps, status);
  arc_len[q] = blen[2 * s + j] + a;
  arc_cl[q] = a;
  arc_root[q] = R;
}

// ---------------------------------------------------------------------------
// geometry emission
// ---------------------------------------------------------------------------
enum : int { kTaskBase = 0, kTaskChain = 2 };
// task = {kind | dir << 2, a, b, pos}; base: a = saddle, b = arc;
// chain: a = start node, b = stop node (-1 = void).
__device__ __forceinline__ int4 make_task(int kind, int rev, int a, int b, long long pos) {
  return make_int4(kind | (rev << 2), a, b, (int)pos);
}

struct EmitCtx {
  const uint8_t* flow;
  const int* crit_sad;
  Imgs I;
  const int* sad_img;
  bool faces;
  const int* t;            // per arc target
  const long long* blen;   // per arc length
  ReplayState S;
  int* out_primal;  // destination of primal images' arcs of this side
  int* out_dual;    // destination of dual images' arcs
  int4* q_out;
  int* n_out;
  long long q_cap;
  int4* base_q;  // raw-arc segments, written after the expansion
  int* n_base;
  long long base_cap;
  int max_steps;
  unsigned* status;
};

// A raw arc (s, j) being written by one lane: the V-path from its start cell,
// `len` cells (cpu/arcs_geometry.hxx:83-111, 133-161), following the flow
// codes. dst is the next output slot, step its stride (-1 for a reversed
// arc), rem the cells left and idx the current index.
struct SegCursor {
  int* dst;
  int step;
  long long rem;
  int idx, ibase, Nx;
};

// Starts raw arc (s, j) at output position pos; rem = 0 when it writes
// nothing (no arc, or its image's output does not take this side's arcs).
__device__ __forceinline__ void seg_start(const EmitCtx& E, int s, int j, int rev, long long pos, SegCursor& c) {
  c.rem = 0;
  const long long len = E.blen[2 * s + j];
  if (len <= 0) return;
  const int b = E.sad_img[s];
  int* out = E.I.dual[b] ? E.out_dual : E.out_primal;
  if (!out) return;
  const int W = E.I.W[b];
  c.Nx = W + 1;
  c.ibase = E.I.idx_base[b];
  const int sc = E.crit_sad[s];
  const int cell = E.faces ? face_start(sc, j, c.Nx) : vertex_start(sc, j, E.I.H[b], W, c.Nx, c.ibase);
  c.idx = cell >> 2;
  c.dst = out + (rev ? pos + len - 1 : pos);
  c.step = rev ? -1 : 1;
  c.rem = len;
}

// Writes the cursor's cell (image-local id: faces are type 3, vertices type 0)
// and moves to the next one.
__device__ __forceinline__ void seg_step(const EmitCtx& E, SegCursor& c) {
  *c.dst = (E.faces ? 3 : 0) + 4 * (c.idx - c.ibase);
  c.dst += c.step;
  if (--c.rem > 0) c.idx += flow_step((__ldg(E.flow + c.idx) >> (E.faces ? 4 : 0)) & 7u, c.Nx);
}

// Expands W(d): queues its two chains at slot p and its two raw-arc segments
// at base slot pb, advancing both.
__device__ __forceinline__ void emit_w(const EmitCtx& E, int d, int rev, long long pos, int& p, int& pb) {
  const int4 nw = node_words(E.S.node, d);
  int k = side_of(nw.z), o = 1 - k, s = nw.w;
  int Tk = E.t[2 * s + k], To = E.t[2 * s + o];
  const longlong2 cl = *reinterpret_cast<const longlong2*>(&E.S.node[d].cl_dy);
  long long la = cl.x, lb = E.blen[2 * s + k], lc = E.blen[2 * s + o], ld = cl.y;
  int R = nw.y;
  if (!rev) {
    // reverse(chain(Tk -> d)) + reverse(arc k) + arc o + chain(To -> R)
    if (la > 0) E.q_out[p++] = make_task(kTaskChain, 1, Tk, d, pos);
    if (lb > 0) E.base_q[pb++] = make_task(kTaskBase, 1, s, k, pos + la);
    if (lc > 0) E.base_q[pb++] = make_task(kTaskBase, 0, s, o, pos + la + lb);
    if (ld > 0) E.q_out[p++] = make_task(kTaskChain, 0, To, R, pos + la + lb + lc);
  } else {
    if (ld > 0) E.q_out[p++] = make_task(kTaskChain, 1, To, R, pos);
    if (lc > 0) E.base_q[pb++] = make_task(kTaskBase, 1, s, o, pos + ld);
    if (lb > 0) E.base_q[pb++] = make_task(kTaskBase, 0, s, k, pos + ld + lc);
    if (la > 0) E.q_out[p++] = make_task(kTaskChain, 0, Tk, d, pos + ld + lc + lb);
  }
}

// A chain task expanded in one step: chain(x -> stop) is the concatenation
// of W(z) for the nodes z on x's parent chain up to stop; every W(z) is
// expanded in place (its raw-arc segments and its own two chains), so the
// breadth-first expansion needs one level per chain depth instead of two.
// Counts of the chain tasks and raw-arc segments the expansion writes, and
// the chain's total length.
// Returns false (with zero counts) when the chain exceeds its step cap; the
// task is then dropped and the status reports the cap.
__device__ __forceinline__ bool chain_expand_counts(const EmitCtx& E, int x, int stop, int* n_chain, int* n_base,
                                                    long long* total) {
  long long tot = 0;
  int nc = 0, nb = 0, k = 0, z = x;
  *n_chain = 0;
  *n_base = 0;
  *total = 0;
  while (z != stop && z >= 0) {
    const longlong2 kl = node_keylen(E.S.node, z);
    const int4 w = node_words(E.S.node, z);
    tot += kl.y;
    nc += chains_of(w.z);  // counts stored at link time
    nb += bases_of(w.z);
    z = w.y;
    if (++k > E.max_steps) {
      set_status(E.status, kStatusChainCap);
      return false;
    }
  }
  *n_chain = nc;
  *n_base = nb;
  *total = tot;
  return true;
}

// Writes the expansion counted by chain_expand_counts at slots p and pb.
__device__ void chain_expand(const EmitCtx& E, int x, int stop, int rev, long long pos, long long total, int p,
                             int pb) {
  long long off = 0;
  int k = 0;
  for (int z = x; z != stop && z >= 0; z = E.S.node[z].parent) {
    if (++k > E.max_steps) break;
    const long long w = E.S.node[z].wlen;
    emit_w(E, z, rev, rev ? pos + total - off - w : pos + off, p, pb);
    off += w;
  }
}

}  // namespace dmsc
