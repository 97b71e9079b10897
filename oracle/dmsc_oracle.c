/*
 * dmsc_oracle.c -- CPU restatement of the reference `compute_dmsc` path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity oracle: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker. The product path (dmsc_b200) never calls it.
 *
 * It restates, stage by stage and in plain sequential C, the reference CPU
 * pipeline `extract_single_dmsc_cpu_t` (dmsc/csrc/dmsc_cpu.cpp:29-51) so that
 * every output can be compared bit for bit with the CUDA path. It is pinned
 * against the compiled reference (oracle/build_ref.py) and the reference's own
 * fixtures by tests/test_oracle.py.
 *
 * Conventions (dmsc/csrc/cell_complex.hxx:13-51): cell id = type + 4*(y*Nx+x),
 * Nx = W+1; type 0 vertex (pixel), 1 H-edge, 2 V-edge, 3 face (pixel corner).
 * The "dual" flag flips every value comparison (cpu/cell_compare.hxx:9-21).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* growable int / float buffers                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
  int32_t* a;
  int64_t n, cap;
} ivec;

static void iv_push(ivec* v, int32_t x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 64;
    v->a = (int32_t*)realloc(v->a, (size_t)v->cap * sizeof(int32_t));
  }
  v->a[v->n++] = x;
}

static void* xcalloc(int64_t n, size_t sz) {
  void* p = calloc((size_t)(n > 0 ? n : 1), sz);
  if (!p) {
    fprintf(stderr, "dmsc_oracle: out of memory (%lld x %zu)\n", (long long)n, sz);
    abort();
  }
  return p;
}
static void* xmalloc(int64_t n, size_t sz) { return xcalloc(n, sz); }

/* ------------------------------------------------------------------------ */
/* cell complex and ordering                                                 */
/* ------------------------------------------------------------------------ */
static inline int cid(int t, int y, int x, int Nx) { return t + 4 * (y * Nx + x); }
static inline int ctype(int id) { return id % 4; }
static inline int cy(int id, int Nx) { return (id / 4) / Nx; }
static inline int cx(int id, int Nx) { return (id / 4) % Nx; }
static inline int valid_v(int y, int x, int H, int W) { return y >= 0 && y < H && x >= 0 && x < W; }
static inline int valid_eh(int y, int x, int H, int W) { return y >= 0 && y < H && x >= 0 && x <= W; }
static inline int valid_ev(int y, int x, int H, int W) { return y >= 0 && y <= H && x >= 0 && x < W; }
static inline int valid_f(int y, int x, int H, int W) { return y >= 0 && y <= H && x >= 0 && x <= W; }

/* std::tie(v1,id1) < std::tie(v2,id2) with IEEE '<' (cpu/cell_compare.hxx:10-12) */
static inline int tie_lt(float v1, int id1, float v2, int id2) {
  return (v1 < v2) || (!(v2 < v1) && id1 < id2);
}
/* value_less<IS_DUAL> (cpu/cell_compare.hxx:9-16) */
static inline int value_less(int dual, float v1, int id1, float v2, int id2) {
  return dual ? tie_lt(v2, id2, v1, id1) : tie_lt(v1, id1, v2, id2);
}
/* value_greater<IS_DUAL> = value_less<!IS_DUAL> (cpu/cell_compare.hxx:18-21) */
static inline int value_greater(int dual, float v1, int id1, float v2, int id2) {
  return value_less(!dual, v1, id1, v2, id2);
}

typedef struct {
  int H, W, Nx, dual;
  const float* d;
} field_t;

/* v_greater: pixels compared by (value, y*W+x) (cpu/cell_compare.hxx:23-31) */
static inline int v_greater(const field_t* F, int y1, int x1, int y2, int x2) {
  int i1 = y1 * F->W + x1, i2 = y2 * F->W + x2;
  return value_greater(F->dual, F->d[i1], i1, F->d[i2], i2);
}

/* get_highest_vertex_yx (cpu/cell_compare.hxx:33-63): same visiting order. */
static void highest_vertex(const field_t* F, int type, int y, int x, int* by, int* bx) {
  int H = F->H, W = F->W;
  int best_y = -1, best_x = -1;
#define CHK(vy, vx)                                                   \
  do {                                                                \
    if (best_y == -1 || v_greater(F, (vy), (vx), best_y, best_x)) {   \
      best_y = (vy);                                                  \
      best_x = (vx);                                                  \
    }                                                                 \
  } while (0)
  if (type == 0) {
    CHK(y, x);
  } else if (type == 1) {
    if (x - 1 >= 0) CHK(y, x - 1);
    if (x < W) CHK(y, x);
  } else if (type == 2) {
    if (y - 1 >= 0) CHK(y - 1, x);
    if (y < H) CHK(y, x);
  } else {
    if (y - 1 >= 0 && x - 1 >= 0) CHK(y - 1, x - 1);
    if (y - 1 >= 0 && x < W) CHK(y - 1, x);
    if (y < H && x - 1 >= 0) CHK(y, x - 1);
    if (y < H && x < W) CHK(y, x);
  }
#undef CHK
  *by = best_y;
  *bx = best_x;
}

/* cell_value: value of the highest (dual: lowest) vertex (cpu/cell_compare.hxx:82-87) */
static float cell_value(const field_t* F, int type, int y, int x) {
  int by, bx;
  highest_vertex(F, type, y, x, &by, &bx);
  return F->d[by * F->W + bx];
}

static inline int is_highest(const field_t* F, int type, int y, int x, int vy, int vx) {
  int by, bx;
  highest_vertex(F, type, y, x, &by, &bx);
  return by == vy && bx == vx;
}

/* ------------------------------------------------------------------------ */
/* stage 1: discrete gradient (cpu/gradient.hxx:19-196)                     */
/* ------------------------------------------------------------------------ */
static void compute_gradient(const field_t* F, int32_t* pw) {
  int H = F->H, W = F->W, Nx = F->Nx;
  int64_t ncells = 4LL * (H + 1) * (W + 1);
  for (int64_t i = 0; i < ncells; ++i) pw[i] = -1;
  int Le[4], Lf[4], fe[4], queue[32];
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      int ne = 0, nf = 0;
      /* lower-star edges and faces, same order as gradient.hxx:55-74 */
      if (is_highest(F, 1, y, x, y, x)) Le[ne++] = cid(1, y, x, Nx);
      if (is_highest(F, 1, y, x + 1, y, x)) Le[ne++] = cid(1, y, x + 1, Nx);
      if (is_highest(F, 2, y, x, y, x)) Le[ne++] = cid(2, y, x, Nx);
      if (is_highest(F, 2, y + 1, x, y, x)) Le[ne++] = cid(2, y + 1, x, Nx);
      if (is_highest(F, 3, y, x, y, x)) Lf[nf++] = cid(3, y, x, Nx);
      if (is_highest(F, 3, y, x + 1, y, x)) Lf[nf++] = cid(3, y, x + 1, Nx);
      if (is_highest(F, 3, y + 1, x, y, x)) Lf[nf++] = cid(3, y + 1, x, Nx);
      if (is_highest(F, 3, y + 1, x + 1, y, x)) Lf[nf++] = cid(3, y + 1, x + 1, Nx);

      /* vertex-edge pairing: edge whose other vertex is lowest (gradient.hxx:76-112) */
      int best_e = -1, bo_y = -1, bo_x = -1;
      for (int i = 0; i < ne; ++i) {
        int e = Le[i], ey = cy(e, Nx), ex = cx(e, Nx);
        int oy = -1, ox = -1;
        if (ctype(e) == 1) {
          if (ex - 1 == x && ex < W) {
            oy = ey;
            ox = ex;
          } else if (ex == x && ex - 1 >= 0) {
            oy = ey;
            ox = ex - 1;
          }
        } else {
          if (ey - 1 == y && ey < H) {
            oy = ey;
            ox = ex;
          } else if (ey == y && ey - 1 >= 0) {
            oy = ey - 1;
            ox = ex;
          }
        }
        if (oy != -1) {
          if (best_e == -1 || v_greater(F, bo_y, bo_x, oy, ox)) {
            best_e = e;
            bo_y = oy;
            bo_x = ox;
          }
        }
      }
      if (best_e != -1) {
        int v = cid(0, y, x, Nx);
        pw[v] = best_e;
        pw[best_e] = v;
      }

      /* face-edge pairing by FIFO (gradient.hxx:115-191) */
      int qn = 0, head = 0;
      for (int i = 0; i < nf; ++i) queue[qn++] = Lf[i];
      while (head < qn) {
        int f = queue[head++];
        if (pw[f] != -1) continue;
        int fy = cy(f, Nx), fx = cx(f, Nx), nfe = 0;
        if (valid_eh(fy - 1, fx, H, W)) fe[nfe++] = cid(1, fy - 1, fx, Nx);
        if (valid_eh(fy, fx, H, W)) fe[nfe++] = cid(1, fy, fx, Nx);
        if (valid_ev(fy, fx - 1, H, W)) fe[nfe++] = cid(2, fy, fx - 1, Nx);
        if (valid_ev(fy, fx, H, W)) fe[nfe++] = cid(2, fy, fx, Nx);
        int unp_e = -1, unp_n = 0;
        for (int k = 0; k < nfe; ++k) {
          int e = fe[k], inL = 0;
          for (int j = 0; j < ne; ++j)
            if (Le[j] == e) {
              inL = 1;
              break;
            }
          if (inL && pw[e] == -1) {
            unp_n++;
            unp_e = e;
          }
        }
        if (unp_n == 1) {
          pw[f] = unp_e;
          pw[unp_e] = f;
          int ey = cy(unp_e, Nx), ex = cx(unp_e, Nx);
          int cand[2], nc = 0;
          if (ctype(unp_e) == 1) {
            if (valid_f(ey, ex, H, W)) cand[nc++] = cid(3, ey, ex, Nx);
            if (valid_f(ey + 1, ex, H, W)) cand[nc++] = cid(3, ey + 1, ex, Nx);
          } else {
            if (valid_f(ey, ex, H, W)) cand[nc++] = cid(3, ey, ex, Nx);
            if (valid_f(ey, ex + 1, H, W)) cand[nc++] = cid(3, ey, ex + 1, Nx);
          }
          for (int c = 0; c < nc; ++c) {
            int nfc = cand[c];
            if (nfc == f) continue;
            int inF = 0;
            for (int j = 0; j < nf; ++j)
              if (Lf[j] == nfc) {
                inF = 1;
                break;
              }
            if (!inF || pw[nfc] != -1) continue;
            int already = 0;
            for (int q = head; q < qn; ++q)
              if (queue[q] == nfc) {
                already = 1;
                break;
              }
            if (!already) queue[qn++] = nfc;
          }
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* V-path walks (cpu/arcs_topology.hxx:19-65)                                */
/* ------------------------------------------------------------------------ */
static inline int next_face(const int32_t* pw, int curr, int H, int W, int Nx) {
  int e = pw[curr], ey = cy(e, Nx), ex = cx(e, Nx), f1 = -1, f2 = -1;
  if (ctype(e) == 1) {
    if (valid_f(ey, ex, H, W)) f1 = cid(3, ey, ex, Nx);
    if (valid_f(ey + 1, ex, H, W)) f2 = cid(3, ey + 1, ex, Nx);
  } else {
    if (valid_f(ey, ex, H, W)) f1 = cid(3, ey, ex, Nx);
    if (valid_f(ey, ex + 1, H, W)) f2 = cid(3, ey, ex + 1, Nx);
  }
  return (f1 == curr) ? f2 : f1;
}

static inline int next_vertex(const int32_t* pw, int curr, int H, int W, int Nx) {
  int e = pw[curr], ey = cy(e, Nx), ex = cx(e, Nx), v1 = -1, v2 = -1;
  if (ctype(e) == 1) {
    if (ex - 1 >= 0) v1 = cid(0, ey, ex - 1, Nx);
    if (ex < W) v2 = cid(0, ey, ex, Nx);
  } else {
    if (ey - 1 >= 0) v1 = cid(0, ey - 1, ex, Nx);
    if (ey < H) v2 = cid(0, ey, ex, Nx);
  }
  return (v1 == curr) ? v2 : v1;
}

static void trace_face(const int32_t* pw, int start, int H, int W, int Nx, int* target, int* steps) {
  int curr = start, n = 0;
  while (curr != -1 && pw[curr] != -1) {
    n++;
    curr = next_face(pw, curr, H, W, Nx);
  }
  *target = curr;
  *steps = n;
}

static void trace_vertex(const int32_t* pw, int start, int H, int W, int Nx, int* target, int* steps) {
  int curr = start, n = 0;
  while (curr != -1 && pw[curr] != -1) {
    n++;
    curr = next_vertex(pw, curr, H, W, Nx);
  }
  *target = curr;
  *steps = n;
}

/* ------------------------------------------------------------------------ */
/* sorting helper: merge sort of int keys by a comparator with context       */
/* ------------------------------------------------------------------------ */
typedef int (*less_fn)(const void* ctx, int a, int b);

static void msort_rec(int* a, int* tmp, int n, less_fn lt, const void* ctx) {
  if (n < 2) return;
  int h = n / 2;
  msort_rec(a, tmp, h, lt, ctx);
  msort_rec(a + h, tmp, n - h, lt, ctx);
  int i = 0, j = h, k = 0;
  while (i < h && j < n) tmp[k++] = lt(ctx, a[j], a[i]) ? a[j++] : a[i++];
  while (i < h) tmp[k++] = a[i++];
  while (j < n) tmp[k++] = a[j++];
  memcpy(a, tmp, (size_t)n * sizeof(int));
}

static void msort(int* a, int n, less_fn lt, const void* ctx) {
  int* tmp = (int*)xmalloc(n, sizeof(int));
  msort_rec(a, tmp, n, lt, ctx);
  free(tmp);
}

/* ------------------------------------------------------------------------ */
/* data structures (the reference cpu/ *_struct.hxx headers)                    */
/* ------------------------------------------------------------------------ */
typedef struct { /* SadEvent, cpu/arcs_topology_struct.hxx:8-15 */
  int saddle_id, c1, c2;
  float s_val;
  int pair_id;
  float persistence;
} sad_event;

typedef struct { /* Arc, cpu/arcs_geometry_struct.hxx:10-14 */
  int target, offset, length;
} arc_t;

typedef struct { /* SaddleNode, cpu/arcs_geometry_struct.hxx:17-21 */
  int alive;
  arc_t max_arcs[2], min_arcs[2];
} saddle_node;

typedef struct { /* CancelEvent, cpu/persistence_struct.hxx:9-22 */
  int saddle_id, s_idx, target_id, t_idx;
  float persistence;
} cancel_event;

/* UnionFind with void root -1 (union_find.hxx:6-49) */
static int uf_find(int32_t* parent, int i) {
  if (i == -1) return -1;
  int root = i;
  while (root != -1 && parent[root] != root) root = parent[root];
  int curr = i;
  while (curr != root && curr != -1) {
    int nxt = parent[curr];
    parent[curr] = root;
    curr = nxt;
  }
  return root;
}
static inline void uf_unite_from_root(int32_t* parent, int ri, int rj) {
  if (ri != rj && ri != -1) parent[ri] = rj;
}

/* DAG of path references (cpu/arcs_simplification.hxx:23-34) */
typedef struct {
  int left, right;
  uint8_t lfwd, rfwd;
  int total_len;
} dag_node;
typedef struct {
  int id;
  uint8_t fwd;
} path_ref;

typedef struct {
  dag_node* nodes;
  int64_t n, cap; /* cap = the reference's fixed allocation size */
  int N2;
  const int* base_len;
  int overflow;
  int len_overflow; /* a merged path longer than INT32_MAX cells */
} dag_t;

/* MergePaths (cpu/arcs_simplification.hxx:378-392) */
static path_ref merge_paths(dag_t* g, path_ref p1, path_ref p2) {
  if (p1.id == -1) return p2;
  if (p2.id == -1) return p1;
  if (g->n >= g->cap) {
    g->overflow = 1;
    path_ref r = {-1, 1};
    return r;
  }
  int l1 = (p1.id < g->N2) ? g->base_len[p1.id] : g->nodes[p1.id - g->N2].total_len;
  int l2 = (p2.id < g->N2) ? g->base_len[p2.id] : g->nodes[p2.id - g->N2].total_len;
  /* the reference sums these lengths in int (arcs_simplification.hxx:385);
     a sum past INT32_MAX makes its offsets negative and the call fail */
  if ((int64_t)l1 + l2 > 2147483647LL || l1 < 0 || l2 < 0) g->len_overflow = 1;
  dag_node nd = {p1.id, p2.id, p1.fwd, p2.fwd, (int)(((int64_t)l1 + l2) & 0x7fffffff)};
  g->nodes[g->n] = nd;
  path_ref r = {(int)(g->n + g->N2), 1};
  g->n++;
  return r;
}

static inline int path_len(const dag_t* g, path_ref p) {
  if (p.id == -1) return 0;
  return (p.id < g->N2) ? g->base_len[p.id] : g->nodes[p.id - g->N2].total_len;
}

/* Find with weight compression (cpu/arcs_simplification.hxx:394-407), iterative. */
static int w_find(dag_t* g, int32_t* parent, path_ref* weight, int i) {
  if (i == -1) return -1;
  /* collect the chain i -> ... -> root, then fold weights from the top down,
     which is the order the recursive reference applies its merges */
  int n = 0, cap = 64;
  int* chain = (int*)malloc(cap * sizeof(int));
  int c = i;
  while (c != -1 && parent[c] != c) {
    if (n == cap) {
      cap *= 2;
      chain = (int*)realloc(chain, cap * sizeof(int));
    }
    chain[n++] = c;
    c = parent[c];
  }
  int root = c;
  for (int k = n - 1; k >= 0; --k) {
    int node = chain[k];
    int p = parent[node];
    if (p != -1 && weight[p].id != -1) weight[node] = merge_paths(g, weight[node], weight[p]);
    parent[node] = root;
  }
  free(chain);
  return root;
}

/* Iterative DFS flatten (cpu/arcs_simplification.hxx:194-234). */
static void write_geom(const dag_t* g, path_ref path, int32_t* out, int64_t start, const int32_t* old_flat,
                       const int* base_off) {
  if (path.id == -1) return;
  int64_t cap = 256, sp = 0;
  path_ref* st = (path_ref*)malloc(cap * sizeof(path_ref));
  st[sp++] = path;
  int64_t w = start;
  while (sp > 0) {
    path_ref cur = st[--sp];
    if (cur.id < g->N2) {
      int len = g->base_len[cur.id], off = base_off[cur.id];
      if (cur.fwd)
        for (int k = 0; k < len; ++k) out[w++] = old_flat[off + k];
      else
        for (int k = 0; k < len; ++k) out[w++] = old_flat[off + len - 1 - k];
    } else {
      const dag_node* nd = &g->nodes[cur.id - g->N2];
      if (sp + 2 > cap) {
        cap *= 2;
        st = (path_ref*)realloc(st, cap * sizeof(path_ref));
      }
      if (cur.fwd) {
        path_ref r = {nd->right, nd->rfwd}, l = {nd->left, nd->lfwd};
        st[sp++] = r;
        st[sp++] = l;
      } else {
        path_ref l = {nd->left, (uint8_t)!nd->lfwd}, r = {nd->right, (uint8_t)!nd->rfwd};
        st[sp++] = l;
        st[sp++] = r;
      }
    }
  }
  free(st);
}

/* ------------------------------------------------------------------------ */
/* result object                                                             */
/* ------------------------------------------------------------------------ */
#define NF_OUT 19
#define NF_DBG 23
#define NF_ALL (NF_OUT + NF_DBG)

typedef struct {
  void* data;
  int64_t dims[2];
  int ndim;
  int is_float;
} field_out;

typedef struct {
  field_out f[NF_ALL];
  int status; /* 0 ok, 1 dag overflow, 2 invalid input, 3 sentinel saddle, 4 int32 geometry overflow */
  char msg[256];
} oracle_result;

static void set_i(oracle_result* r, int k, int32_t* p, int64_t d0) {
  r->f[k].data = p;
  r->f[k].dims[0] = d0;
  r->f[k].dims[1] = 0;
  r->f[k].ndim = 1;
  r->f[k].is_float = 0;
}
static void set_i2(oracle_result* r, int k, int32_t* p, int64_t d0, int64_t d1) {
  r->f[k].data = p;
  r->f[k].dims[0] = d0;
  r->f[k].dims[1] = d1;
  r->f[k].ndim = 2;
  r->f[k].is_float = 0;
}
static void set_f(oracle_result* r, int k, float* p, int64_t d0) {
  r->f[k].data = p;
  r->f[k].dims[0] = d0;
  r->f[k].dims[1] = 0;
  r->f[k].ndim = 1;
  r->f[k].is_float = 1;
}
static int32_t* idup(const int32_t* src, int64_t n) {
  int32_t* p = (int32_t*)xmalloc(n, sizeof(int32_t));
  if (n > 0) memcpy(p, src, (size_t)n * sizeof(int32_t));
  return p;
}

/* sort contexts */
typedef struct {
  int dual;
  const float* sval;
  const int32_t* sid;
} sad_ctx;
static int sad_greater(const void* c, int a, int b) {
  const sad_ctx* s = (const sad_ctx*)c;
  return value_greater(s->dual, s->sval[a], s->sid[a], s->sval[b], s->sid[b]);
}
static int cancel_less(const void* c, int a, int b) { /* CancelEvent::operator< */
  const cancel_event* ev = (const cancel_event*)c;
  const cancel_event *x = &ev[a], *y = &ev[b];
  if (x->persistence != y->persistence) return x->persistence < y->persistence;
  if (x->saddle_id != y->saddle_id) return x->saddle_id < y->saddle_id;
  return x->target_id < y->target_id;
}

/* ------------------------------------------------------------------------ */
/* the pipeline                                                              */
/* ------------------------------------------------------------------------ */
enum {
  FL_DUAL = 1,
  FL_GRAD = 2,
  FL_RIDGES = 4,  /* trace_max_arcs (API: trace_ridges) */
  FL_VALLEYS = 8, /* trace_min_arcs (API: trace_valleys) */
  FL_PEAKS = 16,  /* trace_max_groups (API: trace_peaks) */
  FL_BASINS = 32  /* trace_min_groups (API: trace_basins) */
};

void* dmsc_oracle_run(const float* img, int H, int W, float thr, int flags) {
  oracle_result* R = (oracle_result*)xcalloc(1, sizeof(oracle_result));
  if (H <= 0 || W <= 0 || (int64_t)(H + 1) > (int64_t)2147483647 / 4 / (W + 1)) {
    R->status = 2;
    snprintf(R->msg, sizeof R->msg, "invalid size %dx%d", H, W);
    return R;
  }
  int dual = (flags & FL_DUAL) != 0;
  int ret_grad = (flags & FL_GRAD) != 0;
  int t_max_arcs = (flags & FL_RIDGES) != 0, t_min_arcs = (flags & FL_VALLEYS) != 0;
  int t_max_grp = (flags & FL_PEAKS) != 0, t_min_grp = (flags & FL_BASINS) != 0;
  if (dual) { /* dmsc_cpu.cpp:34-37 */
    int t = t_max_arcs;
    t_max_arcs = t_min_arcs;
    t_min_arcs = t;
    t = t_max_grp;
    t_max_grp = t_min_grp;
    t_min_grp = t;
  }
  field_t F = {H, W, W + 1, dual, img};
  int Nx = W + 1;
  int64_t ncells = 4LL * (H + 1) * (W + 1);

  /* gradient + critical points + helpers (cpu/gradient.hxx:263-272) */
  int32_t* pw = (int32_t*)xmalloc(ncells, sizeof(int32_t));
  compute_gradient(&F, pw);

  ivec mins = {0}, sads = {0}, maxs = {0}; /* cpu/critical_points.hxx:14-65, ascending ids */
  for (int64_t id = 0; id < ncells; ++id) {
    if (pw[id] != -1) continue;
    int t = (int)(id % 4), y = cy((int)id, Nx), x = cx((int)id, Nx);
    if (t == 0) {
      if (valid_v(y, x, H, W)) iv_push(&mins, (int32_t)id);
    } else if (t == 1) {
      if (valid_eh(y, x, H, W)) iv_push(&sads, (int32_t)id);
    } else if (t == 2) {
      if (valid_ev(y, x, H, W)) iv_push(&sads, (int32_t)id);
    } else {
      if (valid_f(y, x, H, W)) iv_push(&maxs, (int32_t)id);
    }
  }
  int nmin = (int)mins.n, nsad = (int)sads.n, nmax = (int)maxs.n;

  int32_t* fcm = (int32_t*)xmalloc(ncells, sizeof(int32_t)); /* fast_crit_map, gradient.hxx:198-231 */
  for (int64_t i = 0; i < ncells; ++i) fcm[i] = -1;
  float* max_vals = (float*)xmalloc(nmax, sizeof(float));
  float* min_vals = (float*)xmalloc(nmin, sizeof(float));
  for (int i = 0; i < nmax; ++i) {
    fcm[maxs.a[i]] = i;
    max_vals[i] = cell_value(&F, 3, cy(maxs.a[i], Nx), cx(maxs.a[i], Nx));
  }
  for (int i = 0; i < nmin; ++i) {
    fcm[mins.a[i]] = i;
    min_vals[i] = cell_value(&F, 0, cy(mins.a[i], Nx), cx(mins.a[i], Nx));
  }
  for (int i = 0; i < nsad; ++i) fcm[sads.a[i]] = i;

  /* trace_from_saddles (cpu/arcs_topology.hxx:67-172) */
  float* sval = (float*)xmalloc(nsad, sizeof(float));
  int* order = (int*)xmalloc(nsad, sizeof(int));
  for (int j = 0; j < nsad; ++j) {
    int s = sads.a[j];
    sval[j] = cell_value(&F, ctype(s), cy(s, Nx), cx(s, Nx));
    order[j] = j;
  }
  sad_ctx sc = {dual, sval, sads.a};
  msort(order, nsad, sad_greater, &sc);
  sad_event* smax = (sad_event*)xcalloc(nsad, sizeof(sad_event));
  sad_event* smin = (sad_event*)xcalloc(nsad, sizeof(sad_event));
  int* max_len = (int*)xcalloc(2LL * nsad, sizeof(int));
  int* min_len = (int*)xcalloc(2LL * nsad, sizeof(int));
  for (int j = 0; j < nsad; ++j) {
    /* maxima side, face walks */
    int k = order[j], s = sads.a[k], ey = cy(s, Nx), ex = cx(s, Nx), t = ctype(s);
    int f1 = -1, f2 = -1;
    if (t == 1) {
      if (valid_f(ey, ex, H, W)) f1 = cid(3, ey, ex, Nx);
      if (valid_f(ey + 1, ex, H, W)) f2 = cid(3, ey + 1, ex, Nx);
    } else {
      if (valid_f(ey, ex, H, W)) f1 = cid(3, ey, ex, Nx);
      if (valid_f(ey, ex + 1, H, W)) f2 = cid(3, ey, ex + 1, Nx);
    }
    int t1 = -1, l1 = 0, t2 = -1, l2 = 0;
    if (f1 != -1) trace_face(pw, f1, H, W, Nx, &t1, &l1);
    if (f2 != -1) trace_face(pw, f2, H, W, Nx, &t2, &l2);
    sad_event ev = {-999, -1, -1, 0.0f, -1, 0.0f};
    if (t1 != -1 && t2 != -1) {
      ev.saddle_id = s;
      ev.c1 = fcm[t1];
      ev.c2 = fcm[t2];
      ev.s_val = sval[k];
      max_len[2 * k] = l1;
      max_len[2 * k + 1] = l2;
    } else if (t1 != -1 || t2 != -1) {
      ev.saddle_id = s;
      ev.c1 = fcm[t1 != -1 ? t1 : t2];
      ev.s_val = sval[k];
      max_len[2 * k] = (t1 != -1) ? l1 : l2;
    }
    smax[j] = ev;
  }
  for (int j = 0; j < nsad; ++j) {
    /* minima side, vertex walks, reverse order (arcs_topology.hxx:142) */
    int k = order[nsad - j - 1], s = sads.a[k], ey = cy(s, Nx), ex = cx(s, Nx), t = ctype(s);
    int v1 = -1, v2 = -1;
    if (t == 1) {
      if (ex - 1 >= 0) v1 = cid(0, ey, ex - 1, Nx);
      if (ex < W) v2 = cid(0, ey, ex, Nx);
    } else {
      if (ey - 1 >= 0) v1 = cid(0, ey - 1, ex, Nx);
      if (ey < H) v2 = cid(0, ey, ex, Nx);
    }
    int t1 = -1, l1 = 0, t2 = -1, l2 = 0;
    if (v1 != -1) trace_vertex(pw, v1, H, W, Nx, &t1, &l1);
    if (v2 != -1) trace_vertex(pw, v2, H, W, Nx, &t2, &l2);
    sad_event ev = {-999, -1, -1, 0.0f, -1, 0.0f};
    if (t1 != -1 && t2 != -1) {
      ev.saddle_id = s;
      ev.c1 = fcm[t1];
      ev.c2 = fcm[t2];
      ev.s_val = sval[k];
      min_len[2 * k] = l1;
      min_len[2 * k + 1] = l2;
    } else if (t1 != -1 || t2 != -1) {
      ev.saddle_id = s;
      ev.c1 = fcm[t1 != -1 ? t1 : t2];
      ev.s_val = sval[k];
      min_len[2 * k] = (t1 != -1) ? l1 : l2;
    }
    smin[j] = ev;
  }

  /* raw arc geometry (cpu/arcs_geometry.hxx:14-169) */
  int any_arcs = t_max_arcs || t_min_arcs;
  saddle_node* nodes = (saddle_node*)xcalloc(nsad, sizeof(saddle_node));
  int32_t *flat_max = NULL, *flat_min = NULL;
  int64_t flat_max_n = 0, flat_min_n = 0;
  if (any_arcs && nsad > 0) {
    int64_t* moff = (int64_t*)xcalloc(2LL * nsad + 1, sizeof(int64_t));
    int64_t* noff = (int64_t*)xcalloc(2LL * nsad + 1, sizeof(int64_t));
    for (int i = 0; i < 2 * nsad; ++i) {
      moff[i + 1] = t_max_arcs ? moff[i] + max_len[i] + 1 : 0;
      noff[i + 1] = t_min_arcs ? noff[i] + min_len[i] + 1 : 0;
    }
    flat_max_n = moff[2 * nsad];
    flat_min_n = noff[2 * nsad];
    flat_max = (int32_t*)xmalloc(flat_max_n, sizeof(int32_t));
    flat_min = (int32_t*)xmalloc(flat_min_n, sizeof(int32_t));
    for (int i = 0; i < nsad; ++i) {
      nodes[i].alive = 1;
      int s = sads.a[i], ey = cy(s, Nx), ex = cx(s, Nx), t = ctype(s);
      arc_t none = {-1, 0, 0};
      nodes[i].max_arcs[0] = nodes[i].max_arcs[1] = none;
      nodes[i].min_arcs[0] = nodes[i].min_arcs[1] = none;
      if (t_max_arcs) {
        int st[2], ns = 0;
        if (t == 1) {
          if (valid_f(ey, ex, H, W)) st[ns++] = cid(3, ey, ex, Nx);
          if (valid_f(ey + 1, ex, H, W)) st[ns++] = cid(3, ey + 1, ex, Nx);
        } else {
          if (valid_f(ey, ex, H, W)) st[ns++] = cid(3, ey, ex, Nx);
          if (valid_f(ey, ex + 1, H, W)) st[ns++] = cid(3, ey, ex + 1, Nx);
        }
        for (int a = 0; a < ns; ++a) {
          int curr = st[a], cnt = 0;
          int64_t base = moff[2 * i + a];
          while (curr != -1) {
            if (ctype(curr) == 3) flat_max[base + cnt++] = curr;
            if (pw[curr] == -1) break;
            curr = next_face(pw, curr, H, W, Nx);
          }
          arc_t A = {(curr != -1) ? fcm[curr] : -1, (int)base, cnt};
          nodes[i].max_arcs[a] = A;
        }
      }
      if (t_min_arcs) {
        int st[2], ns = 0;
        if (t == 1) {
          if (ex - 1 >= 0) st[ns++] = cid(0, ey, ex - 1, Nx);
          if (ex < W) st[ns++] = cid(0, ey, ex, Nx);
        } else {
          if (ey - 1 >= 0) st[ns++] = cid(0, ey - 1, ex, Nx);
          if (ey < H) st[ns++] = cid(0, ey, ex, Nx);
        }
        for (int a = 0; a < ns; ++a) {
          int curr = st[a], cnt = 0;
          int64_t base = noff[2 * i + a];
          while (curr != -1) {
            if (ctype(curr) == 0) flat_min[base + cnt++] = curr;
            if (pw[curr] == -1) break;
            curr = next_vertex(pw, curr, H, W, Nx);
          }
          arc_t A = {(curr != -1) ? fcm[curr] : -1, (int)base, cnt};
          nodes[i].min_arcs[a] = A;
        }
      }
    }
    free(moff);
    free(noff);
  }

  /* persistence pairing and cancellation (cpu/persistence.hxx:16-182) */
  uint8_t* min_alive = (uint8_t*)xmalloc(nmin, 1);
  uint8_t* max_alive = (uint8_t*)xmalloc(nmax, 1);
  memset(min_alive, 1, (size_t)(nmin > 0 ? nmin : 1));
  memset(max_alive, 1, (size_t)(nmax > 0 ? nmax : 1));
  int32_t* uf_min = (int32_t*)xmalloc(nmin, sizeof(int32_t));
  int32_t* uf_max = (int32_t*)xmalloc(nmax, sizeof(int32_t));
  int32_t* g_min = (int32_t*)xmalloc(nmin, sizeof(int32_t));
  int32_t* g_max = (int32_t*)xmalloc(nmax, sizeof(int32_t));
  for (int i = 0; i < nmin; ++i) uf_min[i] = g_min[i] = i;
  for (int i = 0; i < nmax; ++i) uf_max[i] = g_max[i] = i;
  cancel_event* min_c = (cancel_event*)xcalloc(nsad, sizeof(cancel_event));
  cancel_event* max_c = (cancel_event*)xcalloc(nsad, sizeof(cancel_event));
  int n_min_c = 0, n_max_c = 0;
  int32_t* removed = (int32_t*)xmalloc(2LL * nsad, sizeof(int32_t));
  int n_removed = 0;
  /* debug: per-saddle (crit_saddles order) pairing records */
  int32_t* dbg_pair_min = (int32_t*)xmalloc(nsad, sizeof(int32_t));
  int32_t* dbg_pair_max = (int32_t*)xmalloc(nsad, sizeof(int32_t));
  float* dbg_pers_min = (float*)xmalloc(nsad, sizeof(float));
  float* dbg_pers_max = (float*)xmalloc(nsad, sizeof(float));

  for (int j = 0; j < nsad; ++j) { /* minima sweep (persistence.hxx:55-105) */
    sad_event* ev = &smin[j];
    if (ev->saddle_id < 0) {
      R->status = 3;
      snprintf(R->msg, sizeof R->msg, "saddle with no valid descending walk");
      ev->pair_id = -1;
      ev->persistence = -1.0f;
      continue;
    }
    int r1 = uf_find(g_min, ev->c1), r2 = uf_find(g_min, ev->c2);
    if (r1 == r2) {
      ev->pair_id = -1;
      ev->persistence = -1.0f;
      continue;
    }
    int surv = -1, dying;
    if (r1 == -1)
      dying = r2;
    else if (r2 == -1)
      dying = r1;
    else if (value_greater(dual, min_vals[r1], mins.a[r1], min_vals[r2], mins.a[r2])) {
      surv = r2;
      dying = r1;
    } else {
      surv = r1;
      dying = r2;
    }
    ev->persistence = dual ? min_vals[dying] - ev->s_val : ev->s_val - min_vals[dying];
    ev->pair_id = mins.a[dying];
    uf_unite_from_root(g_min, dying, surv);
    if (ev->persistence <= thr) {
      removed[n_removed++] = ev->saddle_id;
      min_alive[dying] = 0;
      int d = uf_find(uf_min, ev->c1), sv = uf_find(uf_min, ev->c2);
      if (dying == r2) {
        int t = d;
        d = sv;
        sv = t;
      }
      uf_unite_from_root(uf_min, d, sv);
      if (t_min_arcs) {
        cancel_event c = {ev->saddle_id, fcm[ev->saddle_id], mins.a[d], d, ev->persistence};
        min_c[n_min_c++] = c;
      }
    }
  }
  for (int j = 0; j < nsad; ++j) { /* maxima sweep (persistence.hxx:107-162) */
    sad_event* ev = &smax[j];
    if (ev->saddle_id < 0) {
      R->status = 3;
      snprintf(R->msg, sizeof R->msg, "saddle with no valid ascending walk");
      ev->pair_id = -1;
      ev->persistence = -1.0f;
      continue;
    }
    int r1 = uf_find(g_max, ev->c1), r2 = uf_find(g_max, ev->c2);
    if (r1 == r2) {
      ev->pair_id = -1;
      ev->persistence = -1.0f;
      continue;
    }
    int surv = -1, dying;
    if (r1 == -1)
      dying = r2;
    else if (r2 == -1)
      dying = r1;
    else if (value_less(dual, max_vals[r1], maxs.a[r1], max_vals[r2], maxs.a[r2])) {
      surv = r2;
      dying = r1;
    } else {
      surv = r1;
      dying = r2;
    }
    ev->persistence = dual ? ev->s_val - max_vals[dying] : max_vals[dying] - ev->s_val;
    ev->pair_id = maxs.a[dying];
    uf_unite_from_root(g_max, dying, surv);
    if (ev->persistence <= thr) {
      removed[n_removed++] = ev->saddle_id;
      max_alive[dying] = 0;
      int d = uf_find(uf_max, ev->c1), sv = uf_find(uf_max, ev->c2);
      if (dying == r2) {
        int t = d;
        d = sv;
        sv = t;
      }
      uf_unite_from_root(uf_max, d, sv);
      if (t_max_arcs) {
        cancel_event c = {ev->saddle_id, fcm[ev->saddle_id], maxs.a[d], d, ev->persistence};
        max_c[n_max_c++] = c;
      }
    }
  }
  for (int j = 0; j < nsad; ++j) {
    if (smin[j].saddle_id >= 0) {
      int k = fcm[smin[j].saddle_id];
      dbg_pair_min[k] = smin[j].pair_id;
      dbg_pers_min[k] = smin[j].persistence;
    }
    if (smax[j].saddle_id >= 0) {
      int k = fcm[smax[j].saddle_id];
      dbg_pair_max[k] = smax[j].pair_id;
      dbg_pers_max[k] = smax[j].persistence;
    }
  }
  /* debug: sweep-order events (saddle dense idx, c1, c2) per side */
  int32_t* dbg_ev_min = (int32_t*)xmalloc(3LL * nsad, sizeof(int32_t));
  int32_t* dbg_ev_max = (int32_t*)xmalloc(3LL * nsad, sizeof(int32_t));
  for (int j = 0; j < nsad; ++j) {
    dbg_ev_min[3 * j] = smin[j].saddle_id >= 0 ? fcm[smin[j].saddle_id] : -1;
    dbg_ev_min[3 * j + 1] = smin[j].c1;
    dbg_ev_min[3 * j + 2] = smin[j].c2;
    dbg_ev_max[3 * j] = smax[j].saddle_id >= 0 ? fcm[smax[j].saddle_id] : -1;
    dbg_ev_max[3 * j + 1] = smax[j].c1;
    dbg_ev_max[3 * j + 2] = smax[j].c2;
  }
  int32_t* dbg_arcs = (int32_t*)xmalloc(8LL * nsad, sizeof(int32_t));
  for (int i = 0; i < nsad; ++i) {
    dbg_arcs[8 * i + 0] = nodes[i].max_arcs[0].target;
    dbg_arcs[8 * i + 1] = nodes[i].max_arcs[0].length;
    dbg_arcs[8 * i + 2] = nodes[i].max_arcs[1].target;
    dbg_arcs[8 * i + 3] = nodes[i].max_arcs[1].length;
    dbg_arcs[8 * i + 4] = nodes[i].min_arcs[0].target;
    dbg_arcs[8 * i + 5] = nodes[i].min_arcs[0].length;
    dbg_arcs[8 * i + 6] = nodes[i].min_arcs[1].target;
    dbg_arcs[8 * i + 7] = nodes[i].min_arcs[1].length;
  }
  /* erase cancelled saddles from both sorted lists (persistence.hxx:164-181) */
  for (int i = 0; i < n_removed; ++i) fcm[removed[i]] = -1;
  int nsurv = 0;
  for (int j = 0; j < nsad; ++j)
    if (fcm[smin[j].saddle_id] >= 0) smin[nsurv++] = smin[j];
  int nsurv2 = 0;
  for (int j = 0; j < nsad; ++j)
    if (fcm[smax[j].saddle_id] >= 0) smax[nsurv2++] = smax[j];

  /* arc simplification (cpu/arcs_simplification.hxx:310-504) */
  int32_t *new_flat_max = NULL, *new_flat_min = NULL;
  int32_t* dbg_rep_par_max = (int32_t*)xmalloc(nmax, sizeof(int32_t));
  int32_t* dbg_rep_par_min = (int32_t*)xmalloc(nmin, sizeof(int32_t));
  for (int i = 0; i < nmax; ++i) dbg_rep_par_max[i] = i;
  for (int i = 0; i < nmin; ++i) dbg_rep_par_min[i] = i;
  int32_t* dbg_cancel_max = NULL; /* sorted cancels: saddle_id, t_idx, applied */
  int32_t* dbg_cancel_min = NULL;
  if (any_arcs && nsad > 0) {
    int N2 = 2 * nsad;
    for (int side = 0; side < 2; ++side) { /* 0 = maxima (faces), 1 = minima (vertices) */
      int traced = side == 0 ? t_max_arcs : t_min_arcs;
      int next = side == 0 ? nmax : nmin;
      cancel_event* cl = side == 0 ? max_c : min_c;
      int ncl = side == 0 ? n_max_c : n_min_c;
      int* base_len = (int*)xcalloc(N2, sizeof(int));
      int* base_off = (int*)xcalloc(N2, sizeof(int));
      int* init_t = (int*)xmalloc(N2, sizeof(int));
      for (int i = 0; i < N2; ++i) init_t[i] = -1;
      uint8_t* s_alive = (uint8_t*)xmalloc(nsad, 1);
      memset(s_alive, 1, (size_t)nsad);
      int32_t* parent = (int32_t*)xmalloc(next, sizeof(int32_t));
      path_ref* weight = (path_ref*)xmalloc(next, sizeof(path_ref));
      for (int i = 0; i < next; ++i) {
        parent[i] = i;
        weight[i].id = -1;
        weight[i].fwd = 1;
      }
      for (int i = 0; i < nsad && traced; ++i) {
        const arc_t* A = side == 0 ? nodes[i].max_arcs : nodes[i].min_arcs;
        for (int a = 0; a < 2; ++a) {
          init_t[2 * i + a] = A[a].target;
          base_len[2 * i + a] = A[a].length;
          base_off[2 * i + a] = A[a].offset;
        }
      }
      int64_t cap = 5LL * ncl;
      if (cap < (1LL << 18)) cap = 1LL << 18;
      dag_t g = {(dag_node*)xmalloc(cap, sizeof(dag_node)), 0, cap, N2, base_len, 0, 0};
      int32_t* dbgc = (int32_t*)xmalloc(3LL * ncl, sizeof(int32_t));
      if (traced) {
        int* co = (int*)xmalloc(ncl, sizeof(int));
        for (int i = 0; i < ncl; ++i) co[i] = i;
        msort(co, ncl, cancel_less, cl);
        for (int q = 0; q < ncl; ++q) {
          const cancel_event* c = &cl[co[q]];
          dbgc[3 * q] = c->saddle_id;
          dbgc[3 * q + 1] = c->t_idx;
          dbgc[3 * q + 2] = 0;
          int s = c->s_idx;
          if (!s_alive[s]) continue;
          int dead = c->t_idx;
          if (dead < 0 || dead >= next) continue;
          int T0 = init_t[2 * s], T1 = init_t[2 * s + 1];
          int R0 = w_find(&g, parent, weight, T0);
          int R1 = w_find(&g, parent, weight, T1);
          path_ref none = {-1, 1};
          path_ref w0 = (T0 == -1) ? none : weight[T0];
          path_ref w1 = (T1 == -1) ? none : weight[T1];
          path_ref b0 = {2 * s, 1}, b1 = {2 * s + 1, 1};
          path_ref full0 = merge_paths(&g, b0, w0);
          path_ref full1 = merge_paths(&g, b1, w1);
          int merged = 0;
          if (R0 == dead && R0 != R1) {
            parent[R0] = R1;
            path_ref r0 = {full0.id, (uint8_t)!full0.fwd};
            weight[R0] = merge_paths(&g, r0, full1);
            merged = 1;
          } else if (R1 == dead && R0 != R1) {
            parent[R1] = R0;
            path_ref r1 = {full1.id, (uint8_t)!full1.fwd};
            weight[R1] = merge_paths(&g, r1, full0);
            merged = 1;
          }
          if (merged) {
            s_alive[s] = 0;
            dbgc[3 * q + 2] = 1;
            if (side == 0)
              dbg_rep_par_max[dead] = parent[dead];
            else
              dbg_rep_par_min[dead] = parent[dead];
          }
        }
        for (int i = 0; i < next; ++i) w_find(&g, parent, weight, i);
        free(co);
      }
      if (side == 0)
        dbg_cancel_max = dbgc;
      else
        dbg_cancel_min = dbgc;

      /* assemble_simplified_geometry (arcs_simplification.hxx:37-308) */
      int* fin_len = (int*)xcalloc(N2, sizeof(int));
      int64_t* fin_off = (int64_t*)xcalloc(N2 + 1, sizeof(int64_t));
      path_ref* fin_path = (path_ref*)xmalloc(N2, sizeof(path_ref));
      for (int i = 0; i < N2; ++i) {
        fin_path[i].id = -1;
        fin_path[i].fwd = 1;
      }
      for (int i = 0; i < nsad; ++i) {
        if (fcm[sads.a[i]] == -1) continue;
        for (int a = 0; a < 2; ++a) {
          int T = init_t[2 * i + a];
          if (T != -1) {
            path_ref b = {2 * i + a, 1};
            fin_path[2 * i + a] = merge_paths(&g, b, weight[T]);
            fin_len[2 * i + a] = path_len(&g, fin_path[2 * i + a]);
          }
        }
      }
      for (int i = 0; i < N2; ++i) fin_off[i + 1] = fin_off[i] + fin_len[i];
      int64_t total = fin_off[N2];
      const int geom_failed = g.len_overflow || total > 2147483647LL;
      if (geom_failed) {
        /* the reference's int32 prefix sums go negative here
           (arcs_simplification.hxx:114, 140, 150-155) and it fails with
           "Trying to create tensor with negative dimension"; stop the same
           way, before allocating the arena */
        R->status = 4;
        snprintf(R->msg, sizeof R->msg, "arc geometry of %lld cells exceeds int32 offsets",
                 (long long)(g.len_overflow ? -1 : total));
        for (int i = 0; i < N2; ++i) {
          fin_len[i] = 0;
          fin_off[i + 1] = 0;
        }
        total = 0;
      }
      int32_t* out = (int32_t*)xmalloc(total, sizeof(int32_t));
      const int32_t* old = side == 0 ? flat_max : flat_min;
      /* per-side alive is combined below, after both sides ran */
      if (side == 0) {
        new_flat_max = out;
        flat_max_n = total;
      } else {
        new_flat_min = out;
        flat_min_n = total;
      }
      /* stash for the combined pass */
      for (int i = 0; i < nsad; ++i) {
        arc_t* A = side == 0 ? nodes[i].max_arcs : nodes[i].min_arcs;
        /* encode alive per side in spare bits of .alive: bit 1 = max side dead, bit 2 = min side dead */
        if (!s_alive[i]) nodes[i].alive |= (side == 0 ? 2 : 4);
        (void)A;
      }
      /* write geometry for saddles that will be globally alive: we need the
         other side's flag, so record what to write and defer */
      for (int i = 0; i < nsad; ++i) {
        arc_t* A = side == 0 ? nodes[i].max_arcs : nodes[i].min_arcs;
        for (int a = 0; a < 2; ++a) {
          int T = init_t[2 * i + a];
          if (T != -1) {
            /* tentative: becomes final if the saddle stays globally alive */
            A[a].target = parent[T];
            A[a].offset = (int)fin_off[2 * i + a];
            A[a].length = fin_len[2 * i + a];
            if (!geom_failed) write_geom(&g, fin_path[2 * i + a], out, fin_off[2 * i + a], old, base_off);
          }
        }
      }
      if (g.overflow) {
        R->status = 1;
        snprintf(R->msg, sizeof R->msg,
                 "The cancellation tree is too deep to merge path geometries."
                 "Please increase MAX_DAG_ALLOC_PER_PAIR in the C++ backend. ");
      }
      free(fin_len);
      free(fin_off);
      free(fin_path);
      free(g.nodes);
      free(base_len);
      free(base_off);
      free(init_t);
      free(s_alive);
      free(parent);
      free(weight);
    }
    /* Flat_Arena_Assembly alive combination (arcs_simplification.hxx:238-250) */
    for (int i = 0; i < nsad; ++i) {
      int alive = !(nodes[i].alive & 6);
      nodes[i].alive = alive;
      if (!alive) {
        nodes[i].max_arcs[0].length = nodes[i].max_arcs[1].length = 0;
        nodes[i].min_arcs[0].length = nodes[i].min_arcs[1].length = 0;
      }
    }
  }

  /* cell groups (cpu/cell_groups.hxx:96-229); labels are path-endpoint
     determined, so a plain walk reproduces the cached walk's result */
  int32_t *face_grp = NULL, *vert_grp = NULL;
  {
    for (int i = 0; i < nmax; ++i) uf_find(uf_max, i);
    for (int i = 0; i < nmin; ++i) uf_find(uf_min, i);
    int32_t* reg_max = (int32_t*)xmalloc(nmax, sizeof(int32_t));
    int32_t* reg_min = (int32_t*)xmalloc(nmin, sizeof(int32_t));
    int rc = 0;
    for (int i = 0; i < nmax; ++i) reg_max[i] = max_alive[i] ? rc++ : -1;
    rc = 0;
    for (int i = 0; i < nmin; ++i) reg_min[i] = min_alive[i] ? rc++ : -1;
    if (t_max_grp) {
      face_grp = (int32_t*)xmalloc((int64_t)(H + 1) * (W + 1), sizeof(int32_t));
      for (int y = 0; y <= H; ++y)
        for (int x = 0; x <= W; ++x) {
          int tgt, st;
          trace_face(pw, cid(3, y, x, Nx), H, W, Nx, &tgt, &st);
          int val = -1;
          if (tgt != -1 && fcm[tgt] != -1) {
            int root = uf_max[fcm[tgt]];
            if (root != -1) val = reg_max[root];
          }
          face_grp[(int64_t)y * Nx + x] = val;
        }
    }
    if (t_min_grp) {
      vert_grp = (int32_t*)xmalloc((int64_t)H * W, sizeof(int32_t));
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          int tgt, st;
          trace_vertex(pw, cid(0, y, x, Nx), H, W, Nx, &tgt, &st);
          int val = -1;
          if (tgt != -1 && fcm[tgt] != -1) {
            int root = uf_min[fcm[tgt]];
            if (root != -1) val = reg_min[root];
          }
          vert_grp[(int64_t)y * W + x] = val;
        }
    }
    free(reg_max);
    free(reg_min);
  }

  /* output assembly (cpu/workspace.hxx:86-365) */
  int32_t* max_to_out = (int32_t*)xmalloc(nmax, sizeof(int32_t));
  int32_t* min_to_out = (int32_t*)xmalloc(nmin, sizeof(int32_t));
  int32_t* sad_to_out = (int32_t*)xmalloc(nsad, sizeof(int32_t));
  int32_t* out_max = (int32_t*)xmalloc(nmax, sizeof(int32_t));
  int32_t* out_min = (int32_t*)xmalloc(nmin, sizeof(int32_t));
  int32_t* out_sad = (int32_t*)xmalloc(nsurv, sizeof(int32_t));
  float* out_p_max = (float*)xmalloc(nsurv, sizeof(float));
  float* out_p_min = (float*)xmalloc(nsurv, sizeof(float));
  int32_t* out_pp_max = (int32_t*)xmalloc(nsurv, sizeof(int32_t));
  int32_t* out_pp_min = (int32_t*)xmalloc(nsurv, sizeof(int32_t));
  int32_t* out_e_max = (int32_t*)xmalloc(4LL * nsurv, sizeof(int32_t));
  int32_t* out_e_min = (int32_t*)xmalloc(4LL * nsurv, sizeof(int32_t));
  int max_count = 0, min_count = 0;
  for (int i = 0; i < nmax; ++i) {
    max_to_out[i] = -1;
    if (max_alive[i]) {
      max_to_out[i] = max_count;
      out_max[max_count++] = maxs.a[i];
    }
  }
  for (int i = 0; i < nmin; ++i) {
    min_to_out[i] = -1;
    if (min_alive[i]) {
      min_to_out[i] = min_count;
      out_min[min_count++] = mins.a[i];
    }
  }
  for (int i = 0; i < nsad; ++i) sad_to_out[i] = -1;
  for (int i = 0; i < nsurv; ++i) {
    sad_event* ev = &smin[i];
    int dense = fcm[ev->saddle_id];
    sad_to_out[dense] = i;
    out_sad[i] = ev->saddle_id;
    ev->saddle_id = i;
    ev->pair_id = (ev->pair_id != -1) ? fcm[ev->pair_id] : -1;
  }
  for (int i = 0; i < nsurv; ++i) {
    sad_event* ev = &smax[i];
    ev->saddle_id = fcm[ev->saddle_id];
    ev->pair_id = (ev->pair_id != -1) ? fcm[ev->pair_id] : -1;
  }
  int e_min_n = 0, e_max_n = 0;
  for (int i = 0; i < nsurv; ++i) {
    const sad_event* ev = &smin[i];
    int s = ev->saddle_id;
    out_p_min[s] = ev->persistence;
    out_pp_min[s] = (ev->pair_id != -1) ? min_to_out[uf_find(uf_min, ev->pair_id)] : -1;
    int r1 = (ev->c1 != -1) ? uf_find(uf_min, ev->c1) : -1;
    int r2 = (ev->c2 != -1) ? uf_find(uf_min, ev->c2) : -1;
    if (r1 != -1 && min_to_out[r1] != -1) {
      out_e_min[2 * e_min_n] = s;
      out_e_min[2 * e_min_n + 1] = min_to_out[r1];
      e_min_n++;
    }
    if (r1 != r2 && r2 != -1 && min_to_out[r2] != -1) {
      out_e_min[2 * e_min_n] = s;
      out_e_min[2 * e_min_n + 1] = min_to_out[r2];
      e_min_n++;
    }
  }
  for (int i = 0; i < nsurv; ++i) {
    const sad_event* ev = &smax[i];
    int s = sad_to_out[ev->saddle_id];
    out_p_max[s] = ev->persistence;
    out_pp_max[s] = (ev->pair_id != -1) ? max_to_out[uf_find(uf_max, ev->pair_id)] : -1;
    int r1 = (ev->c1 != -1) ? uf_find(uf_max, ev->c1) : -1;
    int r2 = (ev->c2 != -1) ? uf_find(uf_max, ev->c2) : -1;
    if (r1 != -1 && max_to_out[r1] != -1) {
      out_e_max[2 * e_max_n] = s;
      out_e_max[2 * e_max_n + 1] = max_to_out[r1];
      e_max_n++;
    }
    if (r1 != r2 && r2 != -1 && max_to_out[r2] != -1) {
      out_e_max[2 * e_max_n] = s;
      out_e_max[2 * e_max_n + 1] = max_to_out[r2];
      e_max_n++;
    }
  }
  /* ridge / valley CSR over surviving saddles in sorted-min order (workspace.hxx:220-288) */
  int32_t *rf = NULL, *rf_off = NULL, *af_off = NULL, *rv = NULL, *rv_off = NULL, *av_off = NULL;
  int64_t n_rf = 0, n_rv = 0;
  int n_arcs = 0;
  if (any_arcs) {
    for (int i = 0; i < nsurv; ++i) {
      int s_idx = fcm[out_sad[smin[i].saddle_id]];
      const saddle_node* nd = &nodes[s_idx];
      if (!nd->alive) continue;
      if (t_max_arcs) n_rf += nd->max_arcs[0].length + nd->max_arcs[1].length;
      if (t_min_arcs) n_rv += nd->min_arcs[0].length + nd->min_arcs[1].length;
      n_arcs++;
    }
    rf = (int32_t*)xmalloc(n_rf, sizeof(int32_t));
    rf_off = (int32_t*)xmalloc(n_arcs + 1, sizeof(int32_t));
    af_off = (int32_t*)xmalloc(n_arcs, sizeof(int32_t));
    rv = (int32_t*)xmalloc(n_rv, sizeof(int32_t));
    rv_off = (int32_t*)xmalloc(n_arcs + 1, sizeof(int32_t));
    av_off = (int32_t*)xmalloc(n_arcs, sizeof(int32_t));
    rf_off[0] = rv_off[0] = 0;
    int64_t fi = 0, vi = 0;
    int rfi = 1, rvi = 1, afi = 0, avi = 0;
    for (int i = 0; i < nsurv; ++i) {
      int s_idx = fcm[out_sad[smin[i].saddle_id]];
      const saddle_node* nd = &nodes[s_idx];
      if (!nd->alive) continue;
      if (t_max_arcs) {
        for (int k = 0; k < 2; ++k) {
          int len = nd->max_arcs[k].length;
          if (len > 0) memcpy(rf + fi, new_flat_max + nd->max_arcs[k].offset, (size_t)len * sizeof(int32_t));
          fi += len;
          if (k == 0) af_off[afi++] = (int32_t)fi;
        }
        rf_off[rfi++] = (int32_t)fi;
      }
      if (t_min_arcs) {
        for (int k = 0; k < 2; ++k) {
          int len = nd->min_arcs[k].length;
          if (len > 0) memcpy(rv + vi, new_flat_min + nd->min_arcs[k].offset, (size_t)len * sizeof(int32_t));
          vi += len;
          if (k == 0) av_off[avi++] = (int32_t)vi;
        }
        rv_off[rvi++] = (int32_t)vi;
      }
    }
  }

  /* bind, with the primal / dual permutation (workspace.hxx:291-362) */
  int32_t* shp = (int32_t*)xmalloc(2, sizeof(int32_t));
  shp[0] = H;
  shp[1] = W;
  set_i(R, 0, shp, 2);
  int32_t* pmax = idup(out_max, max_count);
  int32_t* pmin = idup(out_min, min_count);
  set_i(R, 3, idup(out_sad, nsurv), nsurv);
  int32_t* emax = idup(out_e_max, 2LL * e_max_n);
  int32_t* emin = idup(out_e_min, 2LL * e_min_n);
  int32_t* grad = ret_grad ? idup(pw, ncells) : (int32_t*)xmalloc(0, 4);
  set_i(R, 10, grad, ret_grad ? ncells : 0);
  int32_t* t_rf = t_max_arcs ? idup(rf, n_rf) : (int32_t*)xmalloc(0, 4);
  int32_t* t_rf_off = t_max_arcs ? idup(rf_off, n_arcs + 1) : (int32_t*)xmalloc(0, 4);
  int32_t* t_af_off = t_max_arcs ? idup(af_off, n_arcs) : (int32_t*)xmalloc(0, 4);
  int64_t n_t_rf = t_max_arcs ? n_rf : 0, n_t_rf_off = t_max_arcs ? n_arcs + 1 : 0,
          n_t_af_off = t_max_arcs ? n_arcs : 0;
  int32_t* t_rv = t_min_arcs ? idup(rv, n_rv) : (int32_t*)xmalloc(0, 4);
  int32_t* t_rv_off = t_min_arcs ? idup(rv_off, n_arcs + 1) : (int32_t*)xmalloc(0, 4);
  int32_t* t_av_off = t_min_arcs ? idup(av_off, n_arcs) : (int32_t*)xmalloc(0, 4);
  int64_t n_t_rv = t_min_arcs ? n_rv : 0, n_t_rv_off = t_min_arcs ? n_arcs + 1 : 0,
          n_t_av_off = t_min_arcs ? n_arcs : 0;
  int64_t fg0 = t_max_grp ? H + 1 : 0, fg1 = t_max_grp ? W + 1 : 0;
  int64_t vg0 = t_min_grp ? H : 0, vg1 = t_min_grp ? W : 0;
  if (!face_grp) face_grp = (int32_t*)xmalloc(0, 4);
  if (!vert_grp) vert_grp = (int32_t*)xmalloc(0, 4);
  float* pmx = (float*)xmalloc(nsurv, sizeof(float));
  float* pmn = (float*)xmalloc(nsurv, sizeof(float));
  memcpy(pmx, out_p_max, (size_t)nsurv * sizeof(float));
  memcpy(pmn, out_p_min, (size_t)nsurv * sizeof(float));
  int32_t* ppx = idup(out_pp_max, nsurv);
  int32_t* ppn = idup(out_pp_min, nsurv);
  if (!dual) {
    set_i(R, 1, pmax, max_count);
    set_i(R, 2, pmin, min_count);
    set_i2(R, 4, emax, e_max_n, 2);
    set_i2(R, 5, emin, e_min_n, 2);
    set_f(R, 6, pmx, nsurv);
    set_f(R, 7, pmn, nsurv);
    set_i(R, 8, ppx, nsurv);
    set_i(R, 9, ppn, nsurv);
    set_i2(R, 11, face_grp, fg0, fg1);
    set_i(R, 12, t_rf, n_t_rf);
    set_i(R, 13, t_rf_off, n_t_rf_off);
    set_i(R, 14, t_af_off, n_t_af_off);
    set_i2(R, 15, vert_grp, vg0, vg1);
    set_i(R, 16, t_rv, n_t_rv);
    set_i(R, 17, t_rv_off, n_t_rv_off);
    set_i(R, 18, t_av_off, n_t_av_off);
  } else {
    set_i(R, 1, pmin, min_count);
    set_i(R, 2, pmax, max_count);
    set_i2(R, 4, emin, e_min_n, 2);
    set_i2(R, 5, emax, e_max_n, 2);
    set_f(R, 6, pmn, nsurv);
    set_f(R, 7, pmx, nsurv);
    set_i(R, 8, ppn, nsurv);
    set_i(R, 9, ppx, nsurv);
    set_i2(R, 11, vert_grp, vg0, vg1);
    set_i(R, 12, t_rv, n_t_rv);
    set_i(R, 13, t_rv_off, n_t_rv_off);
    set_i(R, 14, t_av_off, n_t_av_off);
    set_i2(R, 15, face_grp, fg0, fg1);
    set_i(R, 16, t_rf, n_t_rf);
    set_i(R, 17, t_rf_off, n_t_rf_off);
    set_i(R, 18, t_af_off, n_t_af_off);
  }

  /* debug fields (internal "max" = faces, "min" = vertices, before the dual swap) */
  set_i(R, 19, idup(pw, ncells), ncells);
  set_i(R, 20, idup(mins.a, nmin), nmin);
  set_i(R, 21, idup(sads.a, nsad), nsad);
  set_i(R, 22, idup(maxs.a, nmax), nmax);
  {
    float* sv = (float*)xmalloc(nsad, sizeof(float));
    memcpy(sv, sval, (size_t)nsad * sizeof(float));
    set_f(R, 23, sv, nsad);
  }
  set_i(R, 24, idup(order, nsad), nsad); /* sort by value_greater */
  set_i(R, 25, dbg_pair_min, nsad);
  set_f(R, 26, dbg_pers_min, nsad);
  set_i(R, 27, dbg_pair_max, nsad);
  set_f(R, 28, dbg_pers_max, nsad);
  {
    int32_t* a = (int32_t*)xmalloc(nmin, sizeof(int32_t));
    for (int i = 0; i < nmin; ++i) a[i] = min_alive[i];
    set_i(R, 29, a, nmin);
    int32_t* b = (int32_t*)xmalloc(nmax, sizeof(int32_t));
    for (int i = 0; i < nmax; ++i) b[i] = max_alive[i];
    set_i(R, 30, b, nmax);
  }
  set_i(R, 31, idup(uf_min, nmin), nmin); /* flattened thresholded roots */
  set_i(R, 32, idup(uf_max, nmax), nmax);
  set_i(R, 33, dbg_rep_par_min, nmin); /* replay parents at link time */
  set_i(R, 34, dbg_rep_par_max, nmax);
  set_i2(R, 35, dbg_ev_min, nsad, 3);
  set_i2(R, 36, dbg_ev_max, nsad, 3);
  set_i2(R, 37, dbg_arcs, nsad, 8);
  set_i2(R, 38, dbg_cancel_min ? dbg_cancel_min : (int32_t*)xmalloc(0, 4), dbg_cancel_min ? n_min_c : 0, 3);
  set_i2(R, 39, dbg_cancel_max ? dbg_cancel_max : (int32_t*)xmalloc(0, 4), dbg_cancel_max ? n_max_c : 0, 3);
  {
    float* mv = (float*)xmalloc(nmin, sizeof(float));
    memcpy(mv, min_vals, (size_t)nmin * sizeof(float));
    set_f(R, 40, mv, nmin);
    float* xv = (float*)xmalloc(nmax, sizeof(float));
    memcpy(xv, max_vals, (size_t)nmax * sizeof(float));
    set_f(R, 41, xv, nmax);
  }

  free(pw);
  free(mins.a);
  free(sads.a);
  free(maxs.a);
  free(fcm);
  free(max_vals);
  free(min_vals);
  free(sval);
  free(order);
  free(smax);
  free(smin);
  free(max_len);
  free(min_len);
  free(nodes);
  free(flat_max);
  free(flat_min);
  free(new_flat_max);
  free(new_flat_min);
  free(min_alive);
  free(max_alive);
  free(uf_min);
  free(uf_max);
  free(g_min);
  free(g_max);
  free(min_c);
  free(max_c);
  free(removed);
  free(max_to_out);
  free(min_to_out);
  free(sad_to_out);
  free(out_max);
  free(out_min);
  free(out_sad);
  free(out_p_max);
  free(out_p_min);
  free(out_pp_max);
  free(out_pp_min);
  free(out_e_max);
  free(out_e_min);
  free(rf);
  free(rf_off);
  free(af_off);
  free(rv);
  free(rv_off);
  free(av_off);
  return R;
}

/* ------------------------------------------------------------------------ */
/* ctypes accessors                                                          */
/* ------------------------------------------------------------------------ */
int dmsc_oracle_status(void* h, char* msg, int msg_len) {
  oracle_result* R = (oracle_result*)h;
  if (msg && msg_len > 0) snprintf(msg, (size_t)msg_len, "%s", R->msg);
  return R->status;
}

int dmsc_oracle_num_fields(void) { return NF_ALL; }

int dmsc_oracle_field(void* h, int k, void** data, int64_t* d0, int64_t* d1, int* ndim, int* is_float) {
  oracle_result* R = (oracle_result*)h;
  if (k < 0 || k >= NF_ALL) return -1;
  *data = R->f[k].data;
  *d0 = R->f[k].dims[0];
  *d1 = R->f[k].dims[1];
  *ndim = R->f[k].ndim;
  *is_float = R->f[k].is_float;
  return 0;
}

void dmsc_oracle_free(void* h) {
  oracle_result* R = (oracle_result*)h;
  if (!R) return;
  for (int k = 0; k < NF_ALL; ++k) free(R->f[k].data);
  free(R);
}
