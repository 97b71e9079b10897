// Persistent cooperative kernels: the round loops of the pairing, the replay
// and the geometry expansion run entirely on the device, separated by
// grid-wide barriers, with no host round trip per round.
//
// Counters rotate over three slots: round r reads its input count from
// cnt[r % 3], appends its output to cnt[(r + 1) % 3] and clears
// cnt[(r + 2) % 3], which was last read at the top of round r - 1 (before the
// barrier that ended that round). Every loop is capped; hitting a cap sets a
// status bit the host turns into an error, and every thread leaves the loop at
// the same round because the loop condition reads the same counters.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "pairing.cuh"
#include "replay.cuh"

namespace dmsc {

namespace cg = cooperative_groups;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
constexpr int kTimeline = 64;  // timestamps kept per loop (round starts)

// Root of x in the pairing's group forest. A group links only under an
// older group (ages strictly decrease along links), so a search visits at
// most M + 1 nodes; the loop is capped at `cap` anyway and a cap sets
// kStatusFindCap and returns the node reached (a valid group).
__device__ __forceinline__ int find_halving(int* link, int x, int cap, unsigned* status) {
  for (int k = 0;; ++k) {
    int p = link[x];
    if (p == x) return x;
    if (k >= cap) {
      set_status(status, kStatusFindCap);
      return x;
    }
    int pp = link[p];
    if (pp != p) link[x] = pp;  // path halving: replaces a pointer with an ancestor
    x = pp;
  }
}



// Chunked processing with two output lists: each block takes contiguous
// chunks of items (up to kChunkPer per thread, fewer when there are few
// items, so small rounds still spread over the whole grid; no barrier between
// a thread's items); kept items are gathered in shared memory with shared
// atomics and written out once per chunk with one global reservation per
// list, so a block meets at a barrier a few times per chunk instead of after
// every item.
constexpr int kChunkPer = 8;
constexpr int kChunk = 256 * kChunkPer;  // blocks of 256 threads

struct ChunkLists {
  int n[2];
  int base[2];
  int buf[2][kChunk];
};

__device__ __forceinline__ long long chunk_size(long long n, int blocks) {
  const long long lanes = (long long)blocks * 256;
  return 256LL * max(1LL, min((long long)kChunkPer, (n + lanes - 1) / lanes));
}

// Round loops whose active set has shrunk below kSoloItems finish in block 0
// alone: the other blocks leave (all decide alike, from the same counters
// read after the grid barrier that ended the previous round), and block 0
// separates the remaining phases with block barriers instead of grid
// barriers, which cost several microseconds each.
constexpr long long kSoloItems = 4096;

__device__ __forceinline__ void chunk_start(ChunkLists& L) {
  if (threadIdx.x < 2) L.n[threadIdx.x] = 0;
  __syncthreads();
}

__device__ __forceinline__ void chunk_keep(ChunkLists& L, int side, int v) { L.buf[side][atomicAdd(&L.n[side], 1)] = v; }

__device__ __forceinline__ void chunk_flush(ChunkLists& L, int* cnt0, int* out0, int* cnt1, int* out1) {
  const int t = threadIdx.x;
  __syncthreads();
  if (t < 2 && L.n[t] > 0) L.base[t] = atomicAdd(t == 0 ? cnt0 : cnt1, L.n[t]);
  __syncthreads();
  for (int k = t; k < L.n[0]; k += 256) out0[L.base[0] + k] = L.buf[0][k];
  for (int k = t; k < L.n[1]; k += 256) out1[L.base[1] + k] = L.buf[1][k];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// pairing rounds (see pairing.cuh for the algorithm)
// ---------------------------------------------------------------------------
struct PairArgs {
  int nsad, M;  // void group = M
  // saddles are indexed in list order (ascending cell id); `rank` gives a
  // saddle's sweep position, which orders the saddles (the atomicMin key),
  // and `sweep` maps a sweep position back to the saddle
  const int* t;       // [2 nsad] extremum ends of each saddle (-1: void)
  const int* rank;    // [nsad]
  const int* sweep;   // [nsad]
  int2* g12;          // [nsad] groups of the two ends, as of the saddle's last active round
  int* dying;
  int* link;          // [M+1] group union-find
  unsigned* minedge;  // [M+1]
  int* act0;          // active saddles (ping-pong)
  int* act1;
  int* roots0;        // live group roots (ping-pong), [M+1] each
  int* roots1;
  int* cnt;           // [0..2] rotating active counts, [3..5] rotating root counts
  const int2* key;       // [M] (value bits, cell) of each extremum
  const int* idx_base;   // [B + 1] first global index of each image
  int B;
  const uint8_t* dual;   // [B] orientation of each image
  bool faces;            // face side (maxima in the primal) or vertex side
  unsigned* status;
  int max_rounds;
  int* rounds;                   // receives the number of rounds (statistics)
  unsigned long long* timeline;  // [kTimeline] round start times (ns), optional
};

// Both sides' persistence pairing in one cooperative launch; each round
// processes both sides' active saddles and live roots, so the two sides share
// their grid barriers. Per round and side: (A) every active saddle finds its
// ends' groups, cycles are decided, the rest reduce their sweep index into
// both groups' minimum (no returned value needed) and stay active; (B1) every
// live root with an outgoing saddle decides whether it dies there, and a
// root that dies links itself under the other group's root at once (phase B1
// reads no link, and the next reader is the next round's phase A, behind the
// round's barrier); the others stay live; roots without outgoing saddles
// leave the list for good. Round 0 skips the lookups: all groups are single
// extrema. A side whose active list is empty just idles.
struct PairArgs2 {
  PairArgs s[2];
};

__device__ __forceinline__ void pair_phase_a(const PairArgs& A, int r, long long i, int n, bool& keep, int& e) {
  keep = false;
  e = -1;
  if (i < 0 || i >= n) return;
  const int* in = (r & 1) ? A.act1 : A.act0;
  const int M = A.M;
  e = in[i];
  if (r == 0 || A.dying[e] == kUndecided) {
    int ga, gb;
    if (r == 0) {
      const int2 ab = *reinterpret_cast<const int2*>(A.t + 2 * e);
      ga = ab.x < 0 ? M : ab.x;
      gb = ab.y < 0 ? M : ab.y;
    } else {  // the ends' groups of the previous round, followed to their roots
      const int2 g = A.g12[e];
      ga = find_halving(A.link, g.x, M + 2, A.status);
      gb = find_halving(A.link, g.y, M + 2, A.status);
    }
    if (ga == gb) {
      A.dying[e] = -1;
    } else {
      A.g12[e] = make_int2(ga, gb);
      const unsigned rk = (unsigned)A.rank[e];
      atomicMin(A.minedge + ga, rk);  // result unused: a reduction
      atomicMin(A.minedge + gb, rk);
      keep = true;
    }
  }
}

__device__ __forceinline__ void pair_phase_b1(const PairArgs& A, int r, long long k, int nr, bool& live, int& g) {
  live = false;
  g = -1;
  if (k < 0 || k >= nr) return;
  const int* rin = (r & 1) ? A.roots1 : A.roots0;
  const int M = A.M;
  int h = -1;
  g = rin[k];
  unsigned me = A.minedge[g];
  if (me != kNoEdge) {
    A.minedge[g] = kNoEdge;
    const int e = A.sweep[me];  // the saddle at that sweep position
    const int2 gg = A.g12[e];  // roots as of phase A
    const int ga = gg.x, gb = gg.y;
    h = (ga == g) ? gb : ga;
    // g is an extremum of one image (the void never dies); older = value_less
    // order on the vertex side in the primal and the face side in the dual
    // (its image from its cell, in the record the comparison reads anyway)
    const bool du = g < M && A.dual[find_image(A.idx_base, A.B, A.key[g].y >> 2)];
    if (older(h, g, M, A.key, A.faces ? du : !du)) {
      A.dying[e] = g;
      A.link[g] = h;
    } else {
      live = true;
    }
  }
}

__global__ void __launch_bounds__(256, 6) pairing_persistent_kernel(PairArgs2 P) {
  __shared__ ChunkLists L;
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  for (int sd = 0; sd < 2; ++sd) {
    const PairArgs& A = P.s[sd];
    for (long long i = tid; i <= A.M; i += nth) {
      A.link[i] = (int)i;
      A.minedge[i] = kNoEdge;
      A.roots0[i] = (int)i;
    }
    for (long long i = tid; i < A.nsad; i += nth) {
      A.act0[i] = (int)i;
      A.dying[i] = kUndecided;
    }
    if (tid == 0) {
      A.cnt[0] = A.nsad;
      A.cnt[1] = 0;
      A.cnt[2] = 0;
      A.cnt[3] = A.M + 1;
      A.cnt[4] = 0;
      A.cnt[5] = 0;
    }
  }
  grid.sync();
  bool done0 = false, done1 = false, solo = false;
  for (int r = 0;; ++r) {
    const int n0 = *(volatile int*)(P.s[0].cnt + r % 3), n1 = *(volatile int*)(P.s[1].cnt + r % 3);
    // a side whose active list is empty is finished: its roots are not visited
    const int nr0 = n0 ? *(volatile int*)(P.s[0].cnt + 3 + r % 3) : 0;
    const int nr1 = n1 ? *(volatile int*)(P.s[1].cnt + 3 + r % 3) : 0;
    if (tid == 0) {
      for (int sd = 0; sd < 2; ++sd) {
        const PairArgs& A = P.s[sd];
        const int n = sd ? n1 : n0;
        bool& done = sd ? done1 : done0;
        if (A.timeline && r < kTimeline && !done) A.timeline[r] = global_ns();
        if (n == 0 && !done && A.rounds) *A.rounds = r;
        done = done || n == 0;
      }
    }
    if (n0 == 0 && n1 == 0) break;
    if (!solo && (long long)n0 + n1 + nr0 + nr1 <= kSoloItems) {
      solo = true;
      if (blockIdx.x != 0) break;
    }
    if (r >= max(P.s[0].max_rounds, P.s[1].max_rounds)) {
      // every thread leaves here in the same round (the counters it read are
      // the same); saddles still undecided become cycles, so the kernels
      // that run before the host sees the status read valid extremum indices
      if (tid == 0) set_status(P.s[0].status, kStatusRoundCap);
      const long long t0 = solo ? threadIdx.x : tid, nt = solo ? blockDim.x : nth;
      for (int sd = 0; sd < 2; ++sd)
        for (long long i = t0; i < P.s[sd].nsad; i += nt)
          if (P.s[sd].dying[i] == kUndecided) P.s[sd].dying[i] = -1;
      break;
    }
    const int bid = solo ? 0 : (int)blockIdx.x, nblk = solo ? 1 : (int)gridDim.x;
    if (tid == 0) {
      for (int sd = 0; sd < 2; ++sd) {
        P.s[sd].cnt[(r + 2) % 3] = 0;
        P.s[sd].cnt[3 + (r + 2) % 3] = 0;
      }
    }
    // phase A over both sides' active saddles
    {
      const long long n = (long long)n0 + n1, chunk = chunk_size(n, nblk);
      for (long long c0 = (long long)bid * chunk; c0 < n; c0 += (long long)nblk * chunk) {
        chunk_start(L);
        for (long long i = c0 + threadIdx.x; i < min(n, c0 + chunk); i += 256) {
          bool keep;
          int v;
          if (i < n0) {
            pair_phase_a(P.s[0], r, i, n0, keep, v);
            if (keep) chunk_keep(L, 0, v);
          } else {
            pair_phase_a(P.s[1], r, i - n0, n1, keep, v);
            if (keep) chunk_keep(L, 1, v);
          }
        }
        chunk_flush(L, P.s[0].cnt + (r + 1) % 3, (r & 1) ? P.s[0].act0 : P.s[0].act1, P.s[1].cnt + (r + 1) % 3,
                    (r & 1) ? P.s[1].act0 : P.s[1].act1);
      }
    }
    if (solo)
      __syncthreads();
    else
      grid.sync();
    // phase B1: live roots decide on their first outgoing saddle
    {
      const long long n = (long long)nr0 + nr1, chunk = chunk_size(n, nblk);
      for (long long c0 = (long long)bid * chunk; c0 < n; c0 += (long long)nblk * chunk) {
        chunk_start(L);
        for (long long k = c0 + threadIdx.x; k < min(n, c0 + chunk); k += 256) {
          bool live;
          int g;
          if (k < nr0) {
            pair_phase_b1(P.s[0], r, k, nr0, live, g);
            if (live) chunk_keep(L, 0, g);
          } else {
            pair_phase_b1(P.s[1], r, k - nr0, nr1, live, g);
            if (live) chunk_keep(L, 1, g);
          }
        }
        chunk_flush(L, P.s[0].cnt + 3 + (r + 1) % 3, (r & 1) ? P.s[0].roots0 : P.s[0].roots1,
                    P.s[1].cnt + 3 + (r + 1) % 3, (r & 1) ? P.s[1].roots0 : P.s[1].roots1);
      }
    }
    if (solo)
      __syncthreads();
    else
      grid.sync();
  }
}

// ---------------------------------------------------------------------------
// replay rounds (see replay.cuh)
// ---------------------------------------------------------------------------
struct ReplayArgs {
  const int* n_cancel;               // device count of cancellations
  const unsigned long long* key;     // [C] replay key of each cancellation
  const int* cj;                     // [C] saddle (list index) of each cancellation
  const int* dying;  // [nsad] in saddle list order
  const int* t;      // [2 nsad] extremum ends of each saddle, list order
  const long long* blen;
  ReplayState S;
  int max_steps;
  int* act0;
  int* act1;
  int* cnt;  // [0..2]
  int* wx;         // [2C] position of each cancellation's two walks
  long long* wa;   // [2C] path length summed so far by each walk
  unsigned* status;
  int max_rounds;
  int* rounds;
  unsigned long long* timeline;  // [kTimeline] round start times (ns), optional
};

// Rounds of cancellation resolution (replay.cuh) for both sides in one
// cooperative launch (a side with n_cancel == nullptr takes no part). The
// cancellations are in collection order; their keys order the replay.
struct ReplayArgs2 {
  ReplayArgs s[2];
};

__device__ __forceinline__ bool replay_step(const ReplayArgs& A, int r, int round) {
  const unsigned long long t = A.key[r];
  const int s = A.cj[r], d = A.dying[s];
  // both walks resume where the previous round left them
  int R0 = A.wx[2 * r], R1 = A.wx[2 * r + 1];
  long long a0 = A.wa[2 * r], a1 = A.wa[2 * r + 1];
  const bool ok0 = walk_resume(A.S, &R0, t, &a0, A.max_steps, A.status, round);
  const bool ok1 = walk_resume(A.S, &R1, t, &a1, A.max_steps, A.status, round);
  if (!(ok0 && ok1)) {  // still waiting on an earlier cancellation
    A.wx[2 * r] = R0;
    A.wx[2 * r + 1] = R1;
    A.wa[2 * r] = a0;
    A.wa[2 * r + 1] = a1;
    return true;
  }
  int k = -1;
  if (R0 == d && R0 != R1)
    k = 0;
  else if (R1 == d && R0 != R1)
    k = 1;
  if (k >= 0) {
    const long long b0 = A.blen[2 * s], b1 = A.blen[2 * s + 1];
    *reinterpret_cast<longlong2*>(&A.S.node[d].cl_dy) = make_longlong2(k == 0 ? a0 : a1, k == 0 ? a1 : a0);
    A.S.node[d].wlen = b0 + b1 + a0 + a1;
    // status, parent, the dying side with what W(d) expands to (its non-empty
    // chains and raw-arc segments), and the saddle, in one store; a walk of
    // this round uses no field of a record whose status carries this round's
    // tag, so the order of these stores does not matter
    *reinterpret_cast<int4*>(&A.S.node[d].status) =
        make_int4(status_word(kLinked, round), k == 0 ? R1 : R0,
                  side_word(k, (a0 > 0) + (a1 > 0), (b0 > 0) + (b1 > 0)), s);
  } else {
    A.S.node[d].status = status_word(kRootForever, round);
  }
  return false;
}

__global__ void __launch_bounds__(256, 5) replay_persistent_kernel(ReplayArgs2 P) {
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  for (int sd = 0; sd < 2; ++sd) {
    const ReplayArgs& A = P.s[sd];
    if (!A.n_cancel) continue;
    const int C = *A.n_cancel;
    for (long long r = tid; r < C; r += nth) {
      A.act0[r] = (int)r;
      const int s = A.cj[r];
      int d = A.dying[s];
      A.S.node[d].ctime = A.key[r];
      A.S.node[d].status = kPending;
      A.wx[2 * r] = A.t[2 * s];
      A.wx[2 * r + 1] = A.t[2 * s + 1];
      A.wa[2 * r] = 0;
      A.wa[2 * r + 1] = 0;
    }
    if (tid == 0) {
      A.cnt[0] = C;
      A.cnt[1] = 0;
      A.cnt[2] = 0;
    }
  }
  grid.sync();
  bool done0 = false, done1 = false, solo = false;
  for (int rd = 0;; ++rd) {
    const int na = P.s[0].n_cancel ? *(volatile int*)(P.s[0].cnt + rd % 3) : 0;
    const int nb = P.s[1].n_cancel ? *(volatile int*)(P.s[1].cnt + rd % 3) : 0;
    if (tid == 0) {
      if (P.s[0].n_cancel && !done0) {
        if (P.s[0].timeline && rd < kTimeline) P.s[0].timeline[rd] = global_ns();
        if (na == 0 && P.s[0].rounds) *P.s[0].rounds = rd;
      }
      if (P.s[1].n_cancel && !done1) {
        if (P.s[1].timeline && rd < kTimeline) P.s[1].timeline[rd] = global_ns();
        if (nb == 0 && P.s[1].rounds) *P.s[1].rounds = rd;
      }
    }
    done0 = done0 || na == 0;
    done1 = done1 || nb == 0;
    if (na == 0 && nb == 0) break;
    if (!solo && (long long)na + nb <= kSoloItems) {  // block 0 finishes alone (see kSoloItems)
      solo = true;
      if (blockIdx.x != 0) break;
    }
    const long long t0 = solo ? threadIdx.x : tid, nt = solo ? blockDim.x : nth;
    if (rd >= max(P.s[0].max_rounds, P.s[1].max_rounds)) {
      if (tid == 0) set_status(P.s[0].n_cancel ? P.s[0].status : P.s[1].status, kStatusRoundCap);
      // the cancellations still pending are dropped (their dying nodes
      // become roots), so the chain walks of the kernels that run before the
      // host sees the status meet decided nodes only
      for (long long i = t0; i < (long long)na + nb; i += nt) {
        const ReplayArgs& A = i < na ? P.s[0] : P.s[1];
        const long long k = i < na ? i : i - na;
        const int r = ((rd & 1) ? A.act1 : A.act0)[k];
        A.S.node[A.dying[A.cj[r]]].status = kRootForever;
      }
      break;
    }
    if (tid == 0)
      for (int sd = 0; sd < 2; ++sd)
        if (P.s[sd].n_cancel) P.s[sd].cnt[(rd + 2) % 3] = 0;
    // grid-stride over both sides' pending cancellations (a cancellation
    // decided earlier in the same round is visible to later walks)
    for (long long base = 0; base < (long long)na + nb; base += nt) {
      const long long i = base + t0;
      bool k0 = false, k1 = false;
      int r0 = -1, r1 = -1;
      if (i < na) {
        r0 = ((rd & 1) ? P.s[0].act1 : P.s[0].act0)[i];
        k0 = replay_step(P.s[0], r0, rd);
      } else if (i < (long long)na + nb) {
        r1 = ((rd & 1) ? P.s[1].act1 : P.s[1].act0)[i - na];
        k1 = replay_step(P.s[1], r1, rd);
      }
      // every thread of the block takes part in the reservation (a side
      // without cancellations reserves nothing and its counter is not touched)
      int p0, p1;
      block_reserve2(P.s[0].cnt + (rd + 1) % 3, k0 ? 1 : 0, P.s[1].cnt + (rd + 1) % 3, k1 ? 1 : 0, p0, p1);
      if (k0) ((rd & 1) ? P.s[0].act0 : P.s[0].act1)[p0] = r0;
      if (k1) ((rd & 1) ? P.s[1].act0 : P.s[1].act1)[p1] = r1;
    }
    if (solo)
      __syncthreads();
    else
      grid.sync();
  }
}

// ---------------------------------------------------------------------------
// geometry expansion levels (see replay.cuh)
// ---------------------------------------------------------------------------
struct EmitArgs {
  EmitCtx E;
  int nsurv;
  const int* surv_sad;
  const long long* arc_pos;
  const long long* arc_cl;
  const int* arc_root;
  int4* q0;
  int4* q1;
  int* cnt;  // [0..2] rotating level counts, [3] raw-arc segment count
  int max_levels;
  int* levels;                   // receives the number of levels (statistics)
  unsigned long long* timeline;  // [kTimeline] level start times (ns), optional
};

// Geometry of one side: breadth-first expansion of the chain and W tasks
// (replay.cuh), collecting the raw-arc segments with their output positions,
// then one parallel pass that walks and writes every segment.
__global__ void __launch_bounds__(256) emit_persistent_kernel(EmitArgs A) {
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  if (tid == 0) {
    A.cnt[0] = 0;
    A.cnt[1] = 0;
    A.cnt[2] = 0;
    A.cnt[3] = 0;
  }
  grid.sync();
  EmitCtx E = A.E;
  E.n_base = A.cnt + 3;
  // level 0: each surviving arc's own raw arc, then its chain
  for (long long base = 0; base < 2LL * A.nsurv; base += nth) {
    long long q = base + tid;
    bool push = false, seg = false;
    int4 task = make_int4(0, 0, 0, 0), btask = make_int4(0, 0, 0, 0);
    if (q < 2LL * A.nsurv) {
      int i = (int)(q >> 1), j = (int)(q & 1);
      int s = A.surv_sad[i];
      // images whose output takes none of this side's arcs emit nothing
      const int b = E.sad_img[s];
      const bool takes = (E.I.dual[b] ? E.out_dual : E.out_primal) != nullptr;
      if (takes && E.t[2 * s + j] >= 0) {
        long long pos = A.arc_pos[q];
        seg = E.blen[2 * s + j] > 0;
        btask = make_task(kTaskBase, 0, s, j, pos);
        if (A.arc_cl[q] > 0) {
          push = true;
          task = make_task(kTaskChain, 0, E.t[2 * s + j], A.arc_root[q], pos + E.blen[2 * s + j]);
        }
      }
    }
    int p, pb;
    block_reserve2(A.cnt, push ? 1 : 0, E.n_base, seg ? 1 : 0, p, pb);
    if (push) {
      if (p < E.q_cap)
        A.q0[p] = task;
      else
        set_status(E.status, kStatusQueueOverflow);
    }
    if (seg) {
      if (pb < E.base_cap)
        E.base_q[pb] = btask;
      else
        set_status(E.status, kStatusQueueOverflow);
    }
  }
  grid.sync();
  bool solo = false;
  for (int lv = 0;; ++lv) {
    int n = *(volatile int*)(A.cnt + lv % 3);
    if (tid == 0 && A.timeline && lv < kTimeline - 2) A.timeline[lv] = global_ns();
    if (n == 0) {
      if (tid == 0 && A.levels) *A.levels = lv;
      break;
    }
    if (lv >= A.max_levels || n > E.q_cap) {
      if (tid == 0) set_status(E.status, lv >= A.max_levels ? kStatusRoundCap : kStatusQueueOverflow);
      break;
    }
    // a level of at most one task per thread of a block finishes the
    // expansion in block 0 alone (each task is one thread's work either way)
    if (!solo && n <= 256) {
      solo = true;
      if (blockIdx.x != 0) break;
    }
    const long long t0 = solo ? threadIdx.x : tid, nt = solo ? blockDim.x : nth;
    const int4* in = (lv & 1) ? A.q1 : A.q0;
    E.q_out = (lv & 1) ? A.q0 : A.q1;
    E.n_out = A.cnt + (lv + 1) % 3;
    if (tid == 0) A.cnt[(lv + 2) % 3] = 0;
    for (long long base = 0; base < n; base += nt) {
      long long i = base + t0;
      int4 t = make_int4(-1, 0, 0, 0);
      int kind = -1, rev = 0, need = 0, nb = 0;
      long long total = 0;
      if (i < n) {  // every queued task is a chain task
        t = in[i];
        kind = t.x & 3;
        rev = (t.x >> 2) & 1;
        if (kind == kTaskChain && !chain_expand_counts(E, t.y, t.z, &need, &nb, &total)) kind = -1;
      }
      int p, pb;
      block_reserve2(E.n_out, need, E.n_base, nb, p, pb);
      if (p + (long long)need > E.q_cap || pb + (long long)nb > E.base_cap) {
        set_status(E.status, kStatusQueueOverflow);
        kind = -1;
      }
      if (kind == kTaskChain) chain_expand(E, t.y, t.z, rev, t.w, total, p, pb);
    }
    if (solo)
      __syncthreads();
    else
      grid.sync();
  }
}

// Every raw-arc segment collected by emit_persistent_kernel. Segment
// lengths are very uneven, so a lane that finishes its segment takes the next
// one instead of idling until the warp's longest is done: each warp owns
// ranges of kSegRange consecutive segments (grid-stride over the ranges) and,
// every kSegSteps cells, hands the next unstarted segments of its range to its
// idle cursors by ballot (warp-local, no atomics). Each lane drives NC
// cursors whose flow-code loads are issued together, so a lane waits on NC
// independent dependent-load chains at once instead of one.
constexpr int kSegRange = 256;
constexpr int kSegSteps = 8;
constexpr int kSegCursorShapes = 2;  // NC = 1 or 2 (tuned)

template <int NC>
__global__ void __launch_bounds__(256) emit_segments_kernel(EmitCtx E, const int* __restrict__ count) {
  const long long nb = min((long long)*count, E.base_cap);
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const int shift = E.faces ? 4 : 0, type = E.faces ? 3 : 0;
  for (long long r0 = warp * kSegRange; r0 < nb; r0 += nwarps * kSegRange) {
    const long long r1 = min(nb, r0 + kSegRange);
    long long next = r0;  // first segment of the range not yet handed out (same in every lane)
    SegCursor c[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) c[q].rem = 0;
    while (true) {
      bool busy = false;
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        const unsigned idle = __ballot_sync(0xffffffffu, c[q].rem <= 0);
        if (c[q].rem <= 0) {
          const long long my = next + __popc(idle & lt);
          if (my < r1) {
            const int4 t = E.base_q[my];
            seg_start(E, t.y, t.z, (t.x >> 2) & 1, t.w, c[q]);
          }
        }
        next += __popc(idle);
        busy = busy || c[q].rem > 0;
      }
      if (next >= r1 && __ballot_sync(0xffffffffu, busy) == 0) break;
#pragma unroll 1
      for (int k = 0; k < kSegSteps; ++k) {
        unsigned f[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {  // all loads first: independent chains overlap
          f[q] = 0;
          if (c[q].rem > 1) f[q] = __ldg(E.flow + c[q].idx);
        }
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          if (c[q].rem <= 0) continue;
          *c[q].dst = type + 4 * (c[q].idx - c[q].ibase);
          c[q].dst += c[q].step;
          if (--c[q].rem > 0) c[q].idx += flow_step((f[q] >> shift) & 7u, c[q].Nx);
        }
      }
    }
  }
}

}  // namespace dmsc
