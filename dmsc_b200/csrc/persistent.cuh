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
// The timeline buffer holds 6 loops' round start times, then each round's
// item count at the same position + kTimelineCounts, then the pairing's
// phase-B start times (faces, vertices) at kTimelinePhaseB.
constexpr int kTimelineCounts = 6 * kTimeline;
constexpr int kTimelinePhaseB = 12 * kTimeline;
constexpr int kTimelineSlots = 14 * kTimeline;

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

// Round loops whose active set has shrunk below a threshold finish in block 0
// alone: the other blocks leave (all decide alike, from the same counters
// read after the grid barrier that ended the previous round), and block 0
// separates the remaining phases with block barriers instead of grid
// barriers, which cost several microseconds each. The pairing's items are
// short (a few dependent loads each), so block 0 takes over while each of
// its threads still has several; a replay item walks whole parent chains, so
// the replay goes solo only at one item per thread.
constexpr long long kPairSoloItems = 2048;
constexpr long long kReplaySoloItems = 256;

__device__ __forceinline__ void chunk_start(ChunkLists& L) {
  if (threadIdx.x < 2) L.n[threadIdx.x] = 0;
  __syncthreads();
}

__device__ __forceinline__ void chunk_keep(ChunkLists& L, int side, int v) { L.buf[side][atomicAdd(&L.n[side], 1)] = v; }
// the same, counting only (no list is written)
__device__ __forceinline__ void chunk_count(ChunkLists& L, int side) { atomicAdd(&L.n[side], 1); }
__device__ __forceinline__ void chunk_flush_count(ChunkLists& L, int* cnt0, int* cnt1) {
  __syncthreads();
  if (threadIdx.x < 2 && L.n[threadIdx.x] > 0) atomicAdd(threadIdx.x == 0 ? cnt0 : cnt1, L.n[threadIdx.x]);
  __syncthreads();
}

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
  // saddles are indexed in list order (ascending cell id); a saddle's sweep
  // key (sweep_key) orders the saddles of its image in this side's sweep
  // and is the atomicMin key, so no sorted copy of the saddles is needed
  const float* sval;  // [nsad] saddle values
  const int* sad_img; // [nsad] image of each saddle
  int2* g12;          // [nsad] groups of the two ends, as of the saddle's last active round
  int* dying;
  int* link;                    // [M+1] group union-find
  unsigned long long* minedge;  // [M+1] smallest sweep key of the group's active saddles
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
// ends' groups, cycles are decided, the rest reduce their sweep key into
// both groups' minimum (no returned value needed) and stay active; (B) every
// live root with an outgoing saddle decides whether it dies there, and a
// root that dies links itself under the other group's root at once (phase B
// reads no link, and the next reader is the next round's phase A, behind the
// round's barrier); the others stay live; roots without outgoing saddles
// leave for good. Round 0's phase A runs in the saddle walks (all groups are
// single extrema then, so it needs no lookups), which also leave the round
// counters; the groups' union-find and minima are set up by the compaction
// (PairStart). Rounds 0 and 1 scan every saddle and group instead of reading
// lists (see the round loop). A side with no active saddle just idles.
struct PairArgs2 {
  PairArgs s[2];
};

// Items a thread advances together in each phase (U): every load of a stage
// is issued for all of them before any is used, so a thread waits on U
// independent chains of dependent loads at once instead of one after the
// other (the stores and atomics between items would otherwise keep the
// compiler from overlapping them). Two shapes (tuned): U = 2 with 5 resident
// blocks per SM (48 registers) and U = 4 with 4 (64 registers).
constexpr int kPairShapes = 2;

// Per-side fields picked by a flag (the parameter struct is only indexed
// with constants, so it stays in the constant bank).
#define PSIDE(f) (s1 ? P.s[1].f : P.s[0].f)

// Phase A for the thread's items i0 + 256 u (u < U) below cend: side 0's
// items come first (i < n0). In a scan the items are the saddles themselves
// (the decided ones are skipped), else the active list; the saddles that stay
// active are appended to the next list (`lists`) or only counted.
template <int U>
__device__ __forceinline__ void pair_batch_a(const PairArgs2& P, int r, long long i0, long long cend, int n0,
                                             bool scan, bool lists, ChunkLists& L) {
  int e[U], ga[U], gb[U];
  float sv[U];
  unsigned act = 0, s1m = 0, du = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long i = i0 + 256LL * u;
    e[u] = 0;
    if (i < cend) {
      const bool s1 = i >= n0;
      const long long j = s1 ? i - n0 : i;
      act |= 1u << u;
      s1m |= (unsigned)s1 << u;
      e[u] = scan ? (int)j : ((r & 1) ? PSIDE(act1) : PSIDE(act0))[j];
    }
  }
  // the saddle's state, ends and key value, all issued together
  int dy[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    dy[u] = kUndecided;
    ga[u] = gb[u] = 0;
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    dy[u] = PSIDE(dying)[e[u]];
    const int2 g = PSIDE(g12)[e[u]];  // the ends' groups of the previous round
    ga[u] = g.x;
    gb[u] = g.y;
  }
#pragma unroll
  for (int u = 0; u < U; ++u)
    if (dy[u] != kUndecided) act &= ~(1u << u);
  {
    // the groups' current roots: path-halving finds of all 2U ends in lockstep
    unsigned live = 0;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if ((act >> u) & 1u) live |= 3u << (2 * u);
    for (int it = 0; live; ++it) {
      if (it > P.s[0].M + P.s[1].M + 2) {  // ages strictly decrease along links: never reached
        set_status(P.s[0].status, kStatusFindCap);
        break;
      }
      int pa[2 * U], pp[2 * U];
#pragma unroll
      for (int c = 0; c < 2 * U; ++c) {
        const bool s1 = (s1m >> (c >> 1)) & 1u;
        const int x = (c & 1) ? gb[c >> 1] : ga[c >> 1];
        pa[c] = ((live >> c) & 1u) ? PSIDE(link)[x] : x;
      }
#pragma unroll
      for (int c = 0; c < 2 * U; ++c) {
        const bool s1 = (s1m >> (c >> 1)) & 1u;
        const int x = (c & 1) ? gb[c >> 1] : ga[c >> 1];
        if (pa[c] == x) live &= ~(1u << c);
        pp[c] = ((live >> c) & 1u) ? PSIDE(link)[pa[c]] : pa[c];
      }
#pragma unroll
      for (int c = 0; c < 2 * U; ++c) {
        if (!((live >> c) & 1u)) continue;
        const bool s1 = (s1m >> (c >> 1)) & 1u;
        int& x = (c & 1) ? gb[c >> 1] : ga[c >> 1];
        if (pp[c] == pa[c]) {  // pa is the root
          live &= ~(1u << c);
        } else {
          PSIDE(link)[x] = pp[c];  // path halving: replaces a pointer with an ancestor
        }
        x = pp[c];
      }
    }
  }
  // key values (loaded after the finds: fewer registers live across them)
#pragma unroll
  for (int u = 0; u < U; ++u) {
    sv[u] = 0.f;
    if (!((act >> u) & 1u) || ga[u] == gb[u]) continue;
    const bool s1 = (s1m >> u) & 1u;
    sv[u] = PSIDE(sval)[e[u]];
    const bool d = P.s[0].dual[P.s[0].B > 1 ? P.s[0].sad_img[e[u]] : 0];
    du |= (unsigned)(s1 ? d : !d) << u;  // descending sweep: faces in the primal, vertices in the dual
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    if (ga[u] == gb[u]) {
      PSIDE(dying)[e[u]] = -1;
      continue;
    }
    PSIDE(g12)[e[u]] = make_int2(ga[u], gb[u]);
    const unsigned long long k = sweep_key(sv[u], e[u], (du >> u) & 1u);
    atomicMin(PSIDE(minedge) + ga[u], k);  // result unused: a reduction
    atomicMin(PSIDE(minedge) + gb[u], k);
    if (lists)
      chunk_keep(L, s1, e[u]);
    else
      chunk_count(L, s1);
  }
}

// Phase B for the thread's live roots k0 + 256 u (u < U) below cend (side 0's
// first, k < nr0; in a scan every group, in index order, and the groups
// without an outgoing saddle are skipped): each root with an outgoing saddle
// decides there and a dying root links itself under the other group's root;
// the void never dies; roots without outgoing saddles leave for good. The
// roots that stay live are listed when `lists` is set.
template <int U>
__device__ __forceinline__ void pair_batch_b(const PairArgs2& P, int r, long long k0, long long cend, int nr0,
                                             bool scan, bool lists, ChunkLists& L) {
  int g[U];
  unsigned act = 0, s1m = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long k = k0 + 256LL * u;
    g[u] = 0;
    if (k < cend) {
      const bool s1 = k >= nr0;
      const long long j = s1 ? k - nr0 : k;
      act |= 1u << u;
      s1m |= (unsigned)s1 << u;
      g[u] = scan ? (int)j : ((r & 1) ? PSIDE(roots1) : PSIDE(roots0))[j];
    }
  }
  unsigned long long me[U];
  int2 kg[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    me[u] = kNoEdge;
    kg[u] = make_int2(0, 0);
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    me[u] = PSIDE(minedge)[g[u]];
    if (g[u] < PSIDE(M)) kg[u] = PSIDE(key)[g[u]];
  }
  int e[U];
  unsigned older_less = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    e[u] = 0;
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    if (me[u] == kNoEdge) {  // no outgoing saddle: leaves the list for good
      act &= ~(1u << u);
      continue;
    }
    PSIDE(minedge)[g[u]] = kNoEdge;
    if (g[u] == PSIDE(M)) {  // the void is older than every group: it never dies
      if (lists) chunk_keep(L, s1, g[u]);
      act &= ~(1u << u);
      continue;
    }
    // g is an extremum of one image; its image (from its cell) gives the
    // sweep direction of the key and the age order: value_less on the vertex
    // side in the primal and the face side in the dual
    const bool d = P.s[0].dual[find_image(P.s[0].idx_base, P.s[0].B, kg[u].y >> 2)];
    e[u] = sweep_key_saddle(me[u], s1 ? d : !d);
    older_less |= (unsigned)(s1 ? !d : d) << u;
  }
  int h[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    h[u] = 0;
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    const int2 gg = PSIDE(g12)[e[u]];  // roots as of phase A
    h[u] = gg.x == g[u] ? gg.y : gg.x;
  }
  int2 kh[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    kh[u] = make_int2(0, 0);
    const bool s1 = (s1m >> u) & 1u;
    if (((act >> u) & 1u) && h[u] < PSIDE(M)) kh[u] = PSIDE(key)[h[u]];
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    // older(h, g): the void is older than any extremum; else (value, cell)
    // under the side's order
    bool dies = h[u] == PSIDE(M);
    if (!dies) {
      const float vh = __int_as_float(kh[u].x), vg = __int_as_float(kg[u].x);
      dies = ((older_less >> u) & 1u) ? tie_lt(vh, kh[u].y, vg, kg[u].y) : tie_lt(vg, kg[u].y, vh, kh[u].y);
    }
    if (dies) {
      PSIDE(dying)[e[u]] = g[u];
      PSIDE(link)[g[u]] = h[u];
    } else if (lists) {
      chunk_keep(L, s1, g[u]);
    }
  }
}
#undef PSIDE

template <int U, int MINB>
__global__ void __launch_bounds__(256, MINB) pairing_persistent_kernel(PairArgs2 P) {
  __shared__ ChunkLists L;
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  bool done0 = false, done1 = false, solo = false;
  // Round 0 takes every group and keeps no list (nearly all stay live; its
  // saddle phase ran in the saddle walks, which also counted the saddles
  // that stay active); round 1 scans every saddle (skipping the decided ones) and every
  // group (skipping those without an outgoing saddle) and writes the lists
  // that the later rounds read. Scanning all items in later rounds too, while
  // many are active, measured slower (1.58 against 1.28 ms at 4096^2: the
  // decided items still cost their loads).
  bool scan = true;
  for (int r = 0;; ++r) {
    const int n0 = *(volatile int*)(P.s[0].cnt + r % 3), n1 = *(volatile int*)(P.s[1].cnt + r % 3);
    // a side whose active list is empty is finished: its roots are not visited
    const int nr0 = n0 && !scan ? *(volatile int*)(P.s[0].cnt + 3 + r % 3) : 0;
    const int nr1 = n1 && !scan ? *(volatile int*)(P.s[1].cnt + 3 + r % 3) : 0;
    const bool lists = !scan || r >= 1;
    if (tid == 0) {
      for (int sd = 0; sd < 2; ++sd) {
        const PairArgs& A = P.s[sd];
        const int n = sd ? n1 : n0;
        bool& done = sd ? done1 : done0;
        if (A.timeline && r < kTimeline && !done) {
          A.timeline[r] = global_ns();
          A.timeline[kTimelineCounts + r] = n;
        }
        if (n == 0 && !done && A.rounds) *A.rounds = r;
        done = done || n == 0;
      }
    }
    if (n0 == 0 && n1 == 0) break;
    if (!solo && !scan && (long long)n0 + n1 + nr0 + nr1 <= kPairSoloItems) {
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
    // phase A over both sides' active saddles (or every saddle in a scan);
    // round 0's ran in the saddle walks
    if (r > 0) {
      const int na0 = scan ? P.s[0].nsad : n0, na1 = scan ? P.s[1].nsad : n1;
      const long long n = (long long)na0 + na1, chunk = chunk_size(n, nblk);
      for (long long c0 = (long long)bid * chunk; c0 < n; c0 += (long long)nblk * chunk) {
        chunk_start(L);
        const long long cend = min(n, c0 + chunk);
        for (long long i0 = c0 + threadIdx.x; i0 < cend; i0 += 256LL * U)
          pair_batch_a<U>(P, r, i0, cend, na0, scan, lists, L);
        if (lists)
          chunk_flush(L, P.s[0].cnt + (r + 1) % 3, (r & 1) ? P.s[0].act0 : P.s[0].act1, P.s[1].cnt + (r + 1) % 3,
                      (r & 1) ? P.s[1].act0 : P.s[1].act1);
        else
          chunk_flush_count(L, P.s[0].cnt + (r + 1) % 3, P.s[1].cnt + (r + 1) % 3);
      }
      if (solo)
        __syncthreads();
      else
        grid.sync();
    }
    if (tid == 0 && r < kTimeline)  // side sd's phase-B starts: block 12 + sd
      for (int sd = 0; sd < 2; ++sd)
        if (P.s[sd].timeline) P.s[sd].timeline[kTimelinePhaseB + r] = global_ns();
    // phase B: live roots (or every group in a scan) decide on their first
    // outgoing saddle
    {
      const int nb0 = scan ? P.s[0].M + 1 : nr0, nb1 = scan ? P.s[1].M + 1 : nr1;
      const long long n = (long long)nb0 + nb1, chunk = chunk_size(n, nblk);
      for (long long c0 = (long long)bid * chunk; c0 < n; c0 += (long long)nblk * chunk) {
        if (lists) chunk_start(L);
        const long long cend = min(n, c0 + chunk);
        for (long long k0 = c0 + threadIdx.x; k0 < cend; k0 += 256LL * U)
          pair_batch_b<U>(P, r, k0, cend, nb0, scan, lists, L);
        if (lists)
          chunk_flush(L, P.s[0].cnt + 3 + (r + 1) % 3, (r & 1) ? P.s[0].roots0 : P.s[0].roots1,
                      P.s[1].cnt + 3 + (r + 1) % 3, (r & 1) ? P.s[1].roots0 : P.s[1].roots1);
      }
    }
    scan = scan && !lists;
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
  const int4* arc;   // [nsad] {end 0, end 1, raw-arc cells 0, raw-arc cells 1} of each saddle, list order
  const uint8_t* alive;  // [M] extrema that no cancellation kills (their records are never read)
  const int* crit_sad;   // [nsad] global cell id of each saddle
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

// One batch of a thread's pending cancellations, the items i0 + nt u (u < U)
// below na + nb (side 0's first): both walks of every item resume where the
// previous round left them and advance in lockstep (2U independent chains of
// node loads at once); an item whose walks meet an undecided node keeps its
// walk positions and stays pending, the others decide (link or skip). The
// batch's pending items are appended to the next round's lists with one block
// reservation.
#define RSIDE(f) (s1 ? P.s[1].f : P.s[0].f)
template <int U>
__device__ __forceinline__ void replay_batch(const ReplayArgs2& P, int rd, long long i0, long long nt, int na, int nb) {
  int r[U];
  unsigned act = 0, s1m = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long i = i0 + nt * u;
    r[u] = 0;
    if (i < (long long)na + nb) {
      const bool s1 = i >= na;
      act |= 1u << u;
      s1m |= (unsigned)s1 << u;
      const long long j = s1 ? i - na : i;
      r[u] = rd == 0 ? (int)j : ((rd & 1) ? RSIDE(act1) : RSIDE(act0))[j];
    }
  }
  unsigned long long tk[U];
  int sd[U], x[2 * U];
  long long a[2 * U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    tk[u] = 0;
    sd[u] = 0;
    x[2 * u] = x[2 * u + 1] = -1;
    a[2 * u] = a[2 * u + 1] = 0;
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    tk[u] = RSIDE(key)[r[u]];
    sd[u] = RSIDE(cj)[r[u]];
    if (rd > 0) {  // resume where the previous round left the walks
      const int2 w = *reinterpret_cast<const int2*>(RSIDE(wx) + 2 * r[u]);
      const longlong2 aa = *reinterpret_cast<const longlong2*>(RSIDE(wa) + 2 * r[u]);
      x[2 * u] = w.x;
      x[2 * u + 1] = w.y;
      a[2 * u] = aa.x;
      a[2 * u + 1] = aa.y;
    }
  }
  if (rd == 0) {  // the walks start at the saddle's arc ends
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!((act >> u) & 1u)) continue;
      const bool s1 = (s1m >> u) & 1u;
      const int4 w = RSIDE(arc)[sd[u]];
      x[2 * u] = w.x;
      x[2 * u + 1] = w.y;
    }
  }
  int d[U];  // the dying node (issued before the walks, used after them)
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const bool s1 = (s1m >> u) & 1u;
    d[u] = ((act >> u) & 1u) ? RSIDE(dying)[sd[u]] : 0;
  }
  // the walks, resumed where the previous round left them and advanced in
  // lockstep (the root as of the step's key, with the length summed on the
  // way): bit c of `live` is a walk still
  // moving, bit c of `wait` one that met an undecided node
  unsigned live = 0, wait = 0;
#pragma unroll
  for (int c = 0; c < 2 * U; ++c)
    if (((act >> (c >> 1)) & 1u) && x[c] >= 0) live |= 1u << c;
  // a chain is at most its side's node count long (a side without arcs takes
  // no part and has no bound of its own)
  const int cap = max(P.s[0].max_steps, P.s[1].max_steps);
  for (int steps = 0; live; ++steps) {
    if (steps > cap) {
      set_status(P.s[0].status, kStatusChainCap);
      break;
    }
    longlong2 kl[2 * U];
    int2 w[2 * U];  // status, parent
    bool al[2 * U];
#pragma unroll
    for (int c = 0; c < 2 * U; ++c) {
      const bool s1 = (s1m >> (c >> 1)) & 1u;
      if ((live >> c) & 1u) {  // the alive flag and the record's sector, issued together
        al[c] = RSIDE(alive)[x[c]];
        kl[c] = node_keylen_cg(RSIDE(S.node), x[c]);
        w[c] = __ldcg(reinterpret_cast<const int2*>(&RSIDE(S.node)[x[c]].status));
      }
    }
#pragma unroll
    for (int c = 0; c < 2 * U; ++c) {
      if (!((live >> c) & 1u)) continue;
      // never cancelled (its record is not written), or not linked before
      // this step: the root
      if (al[c] || (unsigned long long)kl[c].x >= tk[c >> 1]) {
        live &= ~(1u << c);
        continue;
      }
      const int st = w[c].x;
      if (status_kind(st) == kPending || (st >> 2) > rd) {  // undecided, or decided in this round
        live &= ~(1u << c);
        wait |= 1u << c;
        continue;
      }
      if (status_kind(st) == kRootForever) {
        live &= ~(1u << c);
        continue;
      }
      a[c] += kl[c].y;
      x[c] = w[c].y;
      if (x[c] < 0) live &= ~(1u << c);
    }
  }
  unsigned keep = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!((act >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    if ((wait >> (2 * u)) & 3u) {  // still waiting on an earlier cancellation
      keep |= 1u << u;
      *reinterpret_cast<int2*>(RSIDE(wx) + 2 * r[u]) = make_int2(x[2 * u], x[2 * u + 1]);
      *reinterpret_cast<longlong2*>(RSIDE(wa) + 2 * r[u]) = make_longlong2(a[2 * u], a[2 * u + 1]);
      continue;
    }
    const int R0 = x[2 * u], R1 = x[2 * u + 1], dd = d[u], s = sd[u];
    const long long a0 = a[2 * u], a1 = a[2 * u + 1];
    int k = -1;
    if (R0 == dd && R0 != R1)
      k = 0;
    else if (R1 == dd && R0 != R1)
      k = 1;
    ReplayNode* node = RSIDE(S.node);
    if (k >= 0) {
      const int4 ar = RSIDE(arc)[s];
      const int2 tt = make_int2(ar.x, ar.y);
      const longlong2 bl = make_longlong2(ar.z, ar.w);
      *reinterpret_cast<longlong2*>(&node[dd].cl_dy) = make_longlong2(k == 0 ? a0 : a1, k == 0 ? a1 : a0);
      *reinterpret_cast<int4*>(&node[dd].t_dy) =
          make_int4(k == 0 ? tt.x : tt.y, k == 0 ? tt.y : tt.x, (int)(k == 0 ? bl.x : bl.y),
                    (int)(k == 0 ? bl.y : bl.x));
      node[dd].wlen = bl.x + bl.y + a0 + a1;
      // status, parent, the dying side with what W(d) expands to (its
      // non-empty chains and raw-arc segments), and the saddle, in one store;
      // a walk of this round uses no field of a record whose status carries
      // this round's tag, so the order of these stores does not matter
      *reinterpret_cast<int4*>(&node[dd].status) =
          make_int4(status_word(kLinked, rd), k == 0 ? R1 : R0,
                    side_word(k, (a0 > 0) + (a1 > 0), (bl.x > 0) + (bl.y > 0)), RSIDE(crit_sad)[s]);
    } else {
      node[dd].status = status_word(kRootForever, rd);
    }
  }
  // every thread of the block takes part in the reservation (a side without
  // cancellations reserves nothing and its counter is not touched)
  const int n0 = __popc(keep & ~s1m), n1 = __popc(keep & s1m);
  int p0, p1;
  block_reserve2(P.s[0].cnt + (rd + 1) % 3, n0, P.s[1].cnt + (rd + 1) % 3, n1, p0, p1);
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!((keep >> u) & 1u)) continue;
    const bool s1 = (s1m >> u) & 1u;
    ((rd & 1) ? RSIDE(act0) : RSIDE(act1))[s1 ? p1++ : p0++] = r[u];
  }
}
#undef RSIDE

// Replay shapes (tuned): U = 1 with 4 resident blocks per SM, U = 2 with 3.
constexpr int kReplayShapes = 2;

template <int U, int MINB>
__global__ void __launch_bounds__(256, MINB) replay_persistent_kernel(ReplayArgs2 P) {
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  for (int sd = 0; sd < 2; ++sd) {
    const ReplayArgs& A = P.s[sd];
    if (!A.n_cancel) continue;
    const int C = *A.n_cancel;
    // the killed nodes' records hold their keys (written by the persistence
    // pass); round 0 takes every cancellation with its walks starting at the
    // saddle's arc ends (no list or walk state yet)
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
        if (P.s[0].timeline && rd < kTimeline) {
          P.s[0].timeline[rd] = global_ns();
          P.s[0].timeline[kTimelineCounts + rd] = na;
        }
        if (na == 0 && P.s[0].rounds) *P.s[0].rounds = rd;
      }
      if (P.s[1].n_cancel && !done1) {
        if (P.s[1].timeline && rd < kTimeline) {
          P.s[1].timeline[rd] = global_ns();
          P.s[1].timeline[kTimelineCounts + rd] = nb;
        }
        if (nb == 0 && P.s[1].rounds) *P.s[1].rounds = rd;
      }
    }
    done0 = done0 || na == 0;
    done1 = done1 || nb == 0;
    if (na == 0 && nb == 0) break;
    if (!solo && (long long)na + nb <= kReplaySoloItems) {  // block 0 finishes alone
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
        const int r = rd == 0 ? (int)k : ((rd & 1) ? A.act1 : A.act0)[k];
        A.S.node[A.dying[A.cj[r]]].status = kRootForever;
      }
      break;
    }
    if (tid == 0)
      for (int sd = 0; sd < 2; ++sd)
        if (P.s[sd].n_cancel) P.s[sd].cnt[(rd + 2) % 3] = 0;
    // grid-stride over both sides' pending cancellations, U per thread at a
    // time (a cancellation decided earlier in the same round is visible to
    // later walks)
    for (long long base = 0; base < (long long)na + nb; base += nt * U) replay_batch<U>(P, rd, base + t0, nt, na, nb);
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
  const long long* arc_cl;
  const int* arc_root;
  int4* q0;
  int4* q1;
  int* cnt;  // [0..2] rotating level counts, [3] raw-arc segment count
  int max_levels;
  int* levels;                   // receives the number of levels (statistics)
  unsigned long long* timeline;  // [kTimeline] level start times (ns), optional
};

// One batch of a thread's chain tasks at one expansion level, in[i0 + nt u]
// (u < U) below n: the U chains are counted in lockstep (one node-record load
// per chain and step), the batch reserves its chain tasks and raw-arc
// segments with one block reservation, and the U chains are expanded in
// lockstep: per step, every chain issues its node's loads, then the loads of
// the node's saddle (arc ends and raw-arc lengths), then writes W(node)
// (chain_expand / emit_w, replay.cuh).
template <int U>
__device__ __forceinline__ void emit_batch(const EmitCtx& E, int4* __restrict__ q_out, int* n_out, int* n_base,
                                           const int4* __restrict__ in, long long i0, long long nt, long long n) {
  int x[U], stop[U], z[U], nc[U], nb[U];
  long long pos[U], tot[U];
  unsigned act = 0, rev = 0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long i = i0 + nt * u;
    x[u] = stop[u] = -1;
    pos[u] = 0;
    if (i < n) {  // every queued task is a chain task
      const int4 t = in[i];
      if ((t.x & 3) == kTaskChain) {
        act |= 1u << u;
        rev |= (unsigned)((t.x >> 2) & 1) << u;
        x[u] = t.y;
        stop[u] = t.z;
        pos[u] = t.w;
      }
    }
    z[u] = x[u];
    nc[u] = nb[u] = 0;
    tot[u] = 0;
  }
  // counts and total length of each chain (chain_expand_counts)
  unsigned live = 0;
#pragma unroll
  for (int u = 0; u < U; ++u)
    if (((act >> u) & 1u) && z[u] != stop[u] && z[u] >= 0) live |= 1u << u;
  for (int k = 0; live; ++k) {
    if (k > E.max_steps) {  // a chain is at most the side's node count long
      set_status(E.status, kStatusChainCap);
      act &= ~live;  // the capped tasks are dropped
      break;
    }
    longlong2 kl[U];
    int4 w[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if ((live >> u) & 1u) {
        kl[u] = node_keylen(E.S.node, z[u]);
        w[u] = node_words(E.S.node, z[u]);
      }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if ((live >> u) & 1u) {
        tot[u] += kl[u].y;
        nc[u] += chains_of(w[u].z);  // counts stored at link time
        nb[u] += bases_of(w[u].z);
        z[u] = w[u].y;
        if (z[u] == stop[u] || z[u] < 0) live &= ~(1u << u);
      }
  }
  int need = 0, nbase = 0;
#pragma unroll
  for (int u = 0; u < U; ++u)
    if ((act >> u) & 1u) {
      need += nc[u];
      nbase += nb[u];
    }
  int p, pb;
  block_reserve2(n_out, need, n_base, nbase, p, pb);
  if (p + (long long)need > E.q_cap || pb + (long long)nbase > E.base_cap) {
    set_status(E.status, kStatusQueueOverflow);
    return;
  }
  // expansion: the slots of chain u follow those of the chains before it
  int pc[U], pbc[U];
  long long off[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    pc[u] = p;
    pbc[u] = pb;
    if ((act >> u) & 1u) {
      p += nc[u];
      pb += nb[u];
    }
    z[u] = x[u];
    off[u] = 0;
  }
  live = 0;
#pragma unroll
  for (int u = 0; u < U; ++u)
    if (((act >> u) & 1u) && z[u] != stop[u] && z[u] >= 0) live |= 1u << u;
  while (live) {
    int4 w[U], te[U];  // (status, parent, side, saddle), (arc ends, raw-arc lengths)
    long long wl[U];
    longlong2 cl[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if ((live >> u) & 1u) {  // the node's two sectors, issued together
        const ReplayNode* nd = E.S.node + z[u];
        w[u] = node_words(E.S.node, z[u]);
        wl[u] = nd->wlen;
        cl[u] = *reinterpret_cast<const longlong2*>(&nd->cl_dy);
        te[u] = *reinterpret_cast<const int4*>(&nd->t_dy);
      }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!((live >> u) & 1u)) continue;
      // W(z) = reverse(chain(Tk -> z)) + reverse(arc k) + arc o + chain(To -> R)
      const int d = z[u], k = side_of(w[u].z), s = w[u].w, R = w[u].y;  // s: the saddle's cell
      const int Tk = te[u].x, To = te[u].y;
      const long long la = cl[u].x, lb = te[u].z, lc = te[u].w, ld = cl[u].y;
      const bool rv = (rev >> u) & 1u;
      const long long at = rv ? pos[u] + tot[u] - off[u] - wl[u] : pos[u] + off[u];
      int& q = pc[u];
      int& qb = pbc[u];
      if (!rv) {
        if (la > 0) q_out[q++] = make_task(kTaskChain, 1, Tk, d, at);
        if (lb > 0) E.base_q[qb++] = make_saddle_seg(s, k, 1, lb, at + la);
        if (lc > 0) E.base_q[qb++] = make_saddle_seg(s, 1 - k, 0, lc, at + la + lb);
        if (ld > 0) q_out[q++] = make_task(kTaskChain, 0, To, R, at + la + lb + lc);
      } else {
        if (ld > 0) q_out[q++] = make_task(kTaskChain, 1, To, R, at);
        if (lc > 0) E.base_q[qb++] = make_saddle_seg(s, 1 - k, 1, lc, at + ld);
        if (lb > 0) E.base_q[qb++] = make_saddle_seg(s, k, 0, lb, at + ld + lc);
        if (la > 0) q_out[q++] = make_task(kTaskChain, 0, Tk, d, at + ld + lc + lb);
      }
      off[u] += wl[u];
      z[u] = w[u].y;
      if (z[u] == stop[u] || z[u] < 0) live &= ~(1u << u);
    }
  }
}
// Expansion shapes (tuned): U = 1 with 5 resident blocks per SM, U = 2 with 3.
constexpr int kEmitShapes = 2;

// Geometry of one side: breadth-first expansion of the chain and W tasks
// (replay.cuh), collecting the raw-arc segments with their output positions,
// then one parallel pass that walks and writes every segment.
template <int U, int MINB>
__global__ void __launch_bounds__(256, MINB) emit_persistent_kernel(EmitArgs A) {
  cg::grid_group grid = cg::this_grid();
  const long long tid = grid.thread_rank(), nth = grid.size();
  if (tid == 0) {
    A.cnt[0] = 0;
    A.cnt[1] = 0;
    A.cnt[2] = 0;
    A.cnt[3] = 0;
  }
  grid.sync();
  const EmitCtx& E = A.E;
  int* const n_base = A.cnt + 3;
  // level 0: the chain of each surviving arc (its own raw arc is a segment
  // item of the writer, read from the survivor records). A block takes
  // kLevel0Arcs arcs per thread at a time: it counts their chains, reserves
  // queue slots once for all of them and then writes the tasks, so the
  // blocks queue on the shared counter once per 4096 arcs instead of once
  // per 256 (each reservation waits on the atomic's return).
  constexpr int kLevel0Arcs = 16;
  const long long narcs = 2LL * A.nsurv, span = (long long)blockDim.x * kLevel0Arcs;
  for (long long base = (long long)blockIdx.x * span; base < narcs; base += (long long)gridDim.x * span) {
    // a chain exists only on arcs that the image's output takes (arc_cl = 0 otherwise)
    int mine = 0;
#pragma unroll
    for (int k = 0; k < kLevel0Arcs; ++k) {
      const long long q = base + (long long)k * blockDim.x + threadIdx.x;
      mine += q < narcs && A.arc_cl[q] > 0;
    }
    // most arcs have no chain (at threshold 0 nearly all): a block reserves
    // queue slots only when one of its threads has a task
    if (!__syncthreads_or(mine > 0)) continue;
    int p, pb;
    block_reserve2(A.cnt, mine, n_base, 0, p, pb);
    if (mine == 0) continue;
    for (int k = 0; k < kLevel0Arcs; ++k) {
      const long long q = base + (long long)k * blockDim.x + threadIdx.x;
      if (q >= narcs || A.arc_cl[q] <= 0) continue;
      const int i = (int)(q >> 1), j = (int)(q & 1);
      const int2 tt = E.sv_t[i];
      const longlong2 bl = E.sv_len[i];
      if (p < E.q_cap)
        A.q0[p] = make_task(kTaskChain, 0, j ? tt.y : tt.x, A.arc_root[q], E.arc_pos[q] + (j ? bl.y : bl.x));
      else
        set_status(E.status, kStatusQueueOverflow);
      ++p;
    }
  }
  grid.sync();
  bool solo = false;
  for (int lv = 0;; ++lv) {
    int n = *(volatile int*)(A.cnt + lv % 3);
    if (tid == 0 && A.timeline && lv < kTimeline - 2) {
      A.timeline[lv] = global_ns();
      A.timeline[kTimelineCounts + lv] = n;
    }
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
    int4* q_out = (lv & 1) ? A.q0 : A.q1;
    int* n_out = A.cnt + (lv + 1) % 3;
    if (tid == 0) A.cnt[(lv + 2) % 3] = 0;
    for (long long base = 0; base < n; base += nt * U) emit_batch<U>(E, q_out, n_out, n_base, in, base + t0, nt, n);
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
constexpr int kSegRange = 128;
constexpr int kSegSteps = 4;
constexpr int kSegCursorShapes = 2;  // NC = 1 or 2 (tuned)

template <int NC>
__global__ void __launch_bounds__(256) emit_segments_kernel(EmitCtx E, const int* __restrict__ count) {
  const long long nb = E.nvirt + min((long long)*count, E.base_cap);
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
            seg_start(E, my, c[q]);
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
