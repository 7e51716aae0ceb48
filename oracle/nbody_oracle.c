/*
 * nbody_oracle.c -- CPU restatement of the reference's Simulation::step path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the thing measured or
 * shipped).  See nbody_oracle.h for the contract and the pinning story.
 * Built with -O2 -ffp-contract=off -fno-fast-math: each float expression
 * below is evaluated exactly as written, one rounding per operation.
 */
#include "nbody_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Body::update -- src/Body.h:20-23: vel += acc*dt; pos += vel*dt.     */
void orc_integrate(size_t n, orc_body *b, float dt) {
  for (size_t i = 0; i < n; ++i) {
    b[i].vx = b[i].vx + b[i].ax * dt;
    b[i].vy = b[i].vy + b[i].ay * dt;
    b[i].px = b[i].px + b[i].vx * dt;
    b[i].py = b[i].py + b[i].vy * dt;
  }
}

/* ------------------------------------------------------------------ */
/* Quad::newContaining -- src/QuadTree.cpp:30-51.  std::min(a, b) returns
 * (b < a) ? b : a, so a NaN coordinate never replaces the running value. */
void orc_root_square(size_t n, const float *x, const float *y, float out[3]) {
  float minX = FLT_MAX, minY = FLT_MAX, maxX = -FLT_MAX, maxY = -FLT_MAX;
  for (size_t i = 0; i < n; ++i) {
    if (x[i] < minX) minX = x[i];
    if (y[i] < minY) minY = y[i];
    if (maxX < x[i]) maxX = x[i];
    if (maxY < y[i]) maxY = y[i];
  }
  out[0] = (minX + maxX) * 0.5f;
  out[1] = (minY + maxY) * 0.5f;
  const float w = maxX - minX, h = maxY - minY;
  out[2] = (w < h) ? h : w; /* std::max(w, h) */
}

/* ------------------------------------------------------------------ */
/* spreadBits / quantise / mortonCode -- src/cuda/TreeKernels.cuh:37-66. */
static uint64_t spread_bits(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

static uint32_t quantise(float v, double lo, double scale) {
  const double q = floor(((double)v - lo) * scale);
  if (!(q > 0.0)) return 0u; /* also NaN */
  if (q >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)q;
}

void orc_morton(size_t n, const float *x, const float *y, const float root[3],
                uint64_t *codes) {
  /* mortonKernel's origin and scale, CudaQuadTree.cu:41-44. */
  const double x0 = (double)root[0] - 0.5 * (double)root[2];
  const double y0 = (double)root[1] - 0.5 * (double)root[2];
  const double scale = root[2] > 0.0f ? 4294967296.0 / (double)root[2] : 0.0;
  for (size_t i = 0; i < n; ++i) {
    codes[i] = (spread_bits(quantise(y[i], y0, scale)) << 1) |
               spread_bits(quantise(x[i], x0, scale));
  }
}

/* ------------------------------------------------------------------ */
/* Stable merge sort of indices by 64-bit code. */
static void merge_perm(const uint64_t *codes, uint32_t *a, uint32_t *tmp,
                       size_t n) {
  for (size_t width = 1; width < n; width *= 2) {
    for (size_t lo = 0; lo < n; lo += 2 * width) {
      size_t mid = lo + width < n ? lo + width : n;
      size_t hi = lo + 2 * width < n ? lo + 2 * width : n;
      size_t i = lo, j = mid, k = lo;
      while (i < mid && j < hi) {
        /* take from the right only if strictly smaller: stable */
        if (codes[a[j]] < codes[a[i]]) tmp[k++] = a[j++];
        else tmp[k++] = a[i++];
      }
      while (i < mid) tmp[k++] = a[i++];
      while (j < hi) tmp[k++] = a[j++];
    }
    memcpy(a, tmp, n * sizeof(uint32_t));
  }
}

void orc_stable_perm(size_t n, const uint64_t *codes, uint32_t *perm) {
  for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  if (n < 2) return;
  uint32_t *tmp = (uint32_t *)malloc(n * sizeof(uint32_t));
  merge_perm(codes, perm, tmp, n);
  free(tmp);
}

/* ------------------------------------------------------------------ */
/* Morton tree: TreeKernels.cuh:68-177 driven as buildHostLoop,
 * CudaQuadTree.cu:452-498 (kMaxDepth = 32, TreeKernels.cuh:29). */
static int digit_at(uint64_t code, int depth) {
  return (int)((code >> (62 - 2 * depth)) & 3u);
}

static int first_with_digit(const uint64_t *codes, int lo, int hi, int depth,
                            int q) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (digit_at(codes[mid], depth) < q) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

static void init_node(orc_tree *t, int node, float cx, float cy, float size,
                      int next, int start, int end) {
  t->comX[node] = 0.0f;
  t->comY[node] = 0.0f;
  t->mass[node] = 0.0f;
  t->centerX[node] = cx;
  t->centerY[node] = cy;
  t->size[node] = size;
  t->children[node] = 0;
  t->next[node] = next;
  t->start[node] = start;
  t->end[node] = end;
}

static void split_node(orc_tree *t, int node, int children, int depth,
                       const uint64_t *codes) {
  const int start = t->start[node], end = t->end[node];
  int bound[5];
  bound[0] = start;
  bound[4] = end;
  for (int q = 1; q < 4; ++q)
    bound[q] = first_with_digit(codes, bound[q - 1], end, depth, q);
  const float childSize = t->size[node] * 0.5f;
  const float cx = t->centerX[node], cy = t->centerY[node];
  const int parentNext = t->next[node];
  t->children[node] = children;
  for (int q = 0; q < 4; ++q) {
    const float ccx = cx + ((float)(q & 1) - 0.5f) * childSize;
    const float ccy = cy + ((float)(q >> 1) - 0.5f) * childSize;
    const int next = q < 3 ? children + q + 1 : parentNext;
    init_node(t, children + q, ccx, ccy, childSize, next, bound[q],
              bound[q + 1]);
  }
}

int orc_build_tree(size_t n, const uint64_t *codes, const float *x,
                   const float *y, const float *m, const float root[3],
                   int leafCapacity, orc_tree *t) {
  const int kMaxDepth = 32;
  t->nodeCount = 0;
  t->levelCount = 0;
  if (n == 0) return 0;
  init_node(t, 0, root[0], root[1], root[2], 0, 0, (int)n);
  int levelBegin[34], levelEnd[34];
  int lb = 0, le = 1, depth = 0, levels = 0;
  for (; lb < le; ++depth) {
    levelBegin[levels] = lb;
    levelEnd[levels] = le;
    ++levels;
    int count = le;
    for (int k = lb; k < le; ++k) {
      if (t->end[k] - t->start[k] > leafCapacity && depth < kMaxDepth) {
        if ((long long)count + 4 > t->capacity) return -1;
        split_node(t, k, count, depth, codes);
        count += 4;
      }
    }
    if (count == le) break; /* no splits: host loop stops here */
    lb = le;
    le = count;
  }
  t->nodeCount = le;
  t->levelCount = levels;
  /* sumNode deepest level first, then finishNode (TreeKernels.cuh:150-177) */
  for (int L = levels - 1; L >= 0; --L) {
    for (int k = levelBegin[L]; k < levelEnd[L]; ++k) {
      float px = 0.0f, py = 0.0f, mm = 0.0f;
      const int c = t->children[k];
      if (c == 0) {
        for (int i = t->start[k]; i < t->end[k]; ++i) {
          px = px + x[i] * m[i];
          py = py + y[i] * m[i];
          mm = mm + m[i];
        }
      } else {
        px = ((t->comX[c] + t->comX[c + 1]) + t->comX[c + 2]) + t->comX[c + 3];
        py = ((t->comY[c] + t->comY[c + 1]) + t->comY[c + 2]) + t->comY[c + 3];
        mm = ((t->mass[c] + t->mass[c + 1]) + t->mass[c + 2]) + t->mass[c + 3];
      }
      t->comX[k] = px;
      t->comY[k] = py;
      t->mass[k] = mm;
    }
  }
  for (int k = 0; k < le; ++k) {
    const float mm = fmaxf(t->mass[k], FLT_MIN);
    t->comX[k] = t->comX[k] / mm;
    t->comY[k] = t->comY[k] / mm;
  }
  return 0;
}

/* QuadTree.cpp:11-26 / TreeKernels.cuh:180-195. */
static float fast_inv_sqrt(float x) {
  const float xhalf = 0.5f * x;
  uint32_t i;
  memcpy(&i, &x, sizeof i);
  i = 0x5f3759dfu - (i >> 1);
  memcpy(&x, &i, sizeof x);
  return x * (1.5f - (xhalf * x) * x);
}

/* accelerationAt -- TreeKernels.cuh:197-245. */
static void acceleration_at(float x, float y, const float *bx, const float *by,
                            const float *bm, const orc_tree *t, float tSq,
                            float eSq, float *outX, float *outY) {
  float accX = 0.0f, accY = 0.0f;
  int node = 0;
  for (;;) {
    const float dx = t->comX[node] - x;
    const float dy = t->comY[node] - y;
    const float dSq = dx * dx + dy * dy;
    const float size = t->size[node];
    if (size * size < dSq * tSq) {
      const float mm = t->mass[node];
      if (mm > 0.0f) {
        const float factor =
            fminf((mm * fast_inv_sqrt(dSq)) * (1.0f / (dSq + eSq)), FLT_MAX);
        accX = accX + dx * factor;
        accY = accY + dy * factor;
      }
    } else if (t->children[node] == 0) {
      for (int i = t->start[node]; i < t->end[node]; ++i) {
        const float ex = bx[i] - x;
        const float ey = by[i] - y;
        const float bSq = ex * ex + ey * ey;
        const float factor =
            fminf((bm[i] * fast_inv_sqrt(bSq)) * (1.0f / (bSq + eSq)), FLT_MAX);
        accX = accX + ex * factor;
        accY = accY + ey * factor;
      }
    } else {
      node = t->children[node];
      continue;
    }
    node = t->next[node];
    if (node == 0) break;
  }
  *outX = accX;
  *outY = accY;
}

void orc_tree_forces(size_t n, const float *x, const float *y, const float *m,
                     const orc_tree *t, float theta, float epsilon, float *ax,
                     float *ay) {
  const float tSq = theta * theta, eSq = epsilon * epsilon;
  if (t->nodeCount == 0) return;
  for (size_t i = 0; i < n; ++i)
    acceleration_at(x[i], y[i], x, y, m, t, tSq, eSq, &ax[i], &ay[i]);
}

void orc_interaction_counts(size_t nt, const uint32_t *targets, const float *x,
                            const float *y, const orc_tree *t, float theta,
                            double out[3]) {
  const float tSq = theta * theta;
  double far = 0, near = 0, visits = 0;
  for (size_t k = 0; k < nt && t->nodeCount > 0; ++k) {
    const float px = x[targets[k]], py = y[targets[k]];
    int node = 0;
    for (;;) {
      const float dx = t->comX[node] - px, dy = t->comY[node] - py;
      const float dSq = dx * dx + dy * dy;
      visits += 1;
      if (t->size[node] * t->size[node] < dSq * tSq) {
        if (t->mass[node] > 0.0f) far += 1;
      } else if (t->children[node] == 0) {
        near += t->end[node] - t->start[node];
      } else {
        node = t->children[node];
        continue;
      }
      node = t->next[node];
      if (node == 0) break;
    }
  }
  out[0] = far;
  out[1] = near;
  out[2] = visits;
}

/* ------------------------------------------------------------------ */
/* QuadTree.cpp's partition tree (QuadTree.cpp:154-389, Partition.h).   */
typedef struct qnode {
  int children, next;
  float px, py, mass;
  float cx, cy, size;
  size_t start, end;
} qnode;

static size_t partition_by(orc_body *b, size_t begin, size_t end, int axis,
                           float c) {
  /* Partition.h:7-18 (predicate: coordinate < c) */
#define PRED(B) ((axis) ? ((B).py < c) : ((B).px < c))
  if (begin == end) return begin;
  size_t l = begin, r = end - 1;
  for (;;) {
    while (l <= r && PRED(b[l])) ++l;
    while (l < r && !PRED(b[r])) --r;
    if (l >= r) return l;
    orc_body tmp = b[l];
    b[l] = b[r];
    b[r] = tmp;
    ++l;
    --r;
  }
#undef PRED
}

int orc_quadtree_forces(size_t n, orc_body *b, float theta, float epsilon,
                        int leafCapacity) {
  if (n == 0) return 0;
  const float tSq = theta * theta, eSq = epsilon * epsilon;
  size_t cap = 16, count = 1;
  qnode *nodes = (qnode *)malloc(cap * sizeof(qnode));
  int *parents = NULL;
  size_t nparents = 0, capParents = 0;
  /* Quad::newContaining */
  {
    float *xs = (float *)malloc(n * sizeof(float));
    float *ys = (float *)malloc(n * sizeof(float));
    for (size_t i = 0; i < n; ++i) {
      xs[i] = b[i].px;
      ys[i] = b[i].py;
    }
    float root[3];
    orc_root_square(n, xs, ys, root);
    free(xs);
    free(ys);
    qnode r = {0, 0, 0.0f, 0.0f, 0.0f, root[0], root[1], root[2], 0, n};
    nodes[0] = r;
  }
  size_t levelBegin = 0, levelEnd = 0;
  int guard = 0;
  for (;;) {
    levelBegin = levelEnd;
    levelEnd = count;
    if (levelBegin == levelEnd) break;
    if (++guard > 200) { /* the reference has no depth limit */
      free(nodes);
      free(parents);
      return -1;
    }
    size_t children = levelEnd;
    for (size_t k = levelBegin; k < levelEnd; ++k) {
      if (nodes[k].end - nodes[k].start > (size_t)leafCapacity) children += 4;
    }
    if (children > cap) {
      while (cap < children) cap *= 2;
      nodes = (qnode *)realloc(nodes, cap * sizeof(qnode));
    }
    size_t slot = levelEnd;
    for (size_t k = levelBegin; k < levelEnd; ++k) {
      qnode *nd = &nodes[k];
      if (nd->end - nd->start > (size_t)leafCapacity) {
        if (nparents == capParents) {
          capParents = capParents ? 2 * capParents : 1024;
          parents = (int *)realloc(parents, capParents * sizeof(int));
        }
        parents[nparents++] = (int)k;
        /* subdivide, QuadTree.cpp:55-91 */
        const size_t s = nd->start, e = nd->end;
        const float cx = nd->cx, cy = nd->cy;
        const size_t mid = partition_by(b, s, e, 1, cy);
        const size_t lb2 = partition_by(b, s, mid, 0, cx);
        const size_t rt = partition_by(b, mid, e, 0, cx);
        nd->children = (int)slot;
        const float half = nd->size * 0.5f;
        const size_t bounds[5] = {s, lb2, mid, rt, e};
        for (int q = 0; q < 4; ++q) {
          qnode c;
          c.children = 0;
          c.next = q < 3 ? (int)slot + q + 1 : nd->next;
          c.px = c.py = c.mass = 0.0f;
          c.size = half;
          c.cx = cx + ((float)(q & 1) - 0.5f) * half;
          c.cy = cy + ((float)(q >> 1) - 0.5f) * half;
          c.start = bounds[q];
          c.end = bounds[q + 1];
          nodes[slot + q] = c;
        }
        slot += 4;
      } else {
        /* accumulateLeaf, QuadTree.cpp:93-142 (4 independent sums) */
        float p0x = 0, p0y = 0, p1x = 0, p1y = 0, p2x = 0, p2y = 0, p3x = 0,
              p3y = 0, m0 = 0, m1 = 0, m2 = 0, m3 = 0;
        size_t i = nd->start;
        const size_t e = nd->end;
        for (; i + 3 < e; i += 4) {
          p0x = p0x + b[i].px * b[i].mass;
          p0y = p0y + b[i].py * b[i].mass;
          m0 = m0 + b[i].mass;
          p1x = p1x + b[i + 1].px * b[i + 1].mass;
          p1y = p1y + b[i + 1].py * b[i + 1].mass;
          m1 = m1 + b[i + 1].mass;
          p2x = p2x + b[i + 2].px * b[i + 2].mass;
          p2y = p2y + b[i + 2].py * b[i + 2].mass;
          m2 = m2 + b[i + 2].mass;
          p3x = p3x + b[i + 3].px * b[i + 3].mass;
          p3y = p3y + b[i + 3].py * b[i + 3].mass;
          m3 = m3 + b[i + 3].mass;
        }
        for (; i < e; ++i) {
          p0x = p0x + b[i].px * b[i].mass;
          p0y = p0y + b[i].py * b[i].mass;
          m0 = m0 + b[i].mass;
        }
        nd->px = ((p0x + p1x) + p2x) + p3x;
        nd->py = ((p0y + p1y) + p2y) + p3y;
        nd->mass = ((m0 + m1) + m2) + m3;
      }
    }
    count = slot;
  }
  /* propagate, QuadTree.cpp:237-262 */
  for (size_t k = nparents; k-- > 0;) {
    qnode *nd = &nodes[parents[k]];
    const int c = nd->children;
    nd->px = ((nodes[c].px + nodes[c + 1].px) + nodes[c + 2].px) + nodes[c + 3].px;
    nd->py = ((nodes[c].py + nodes[c + 1].py) + nodes[c + 2].py) + nodes[c + 3].py;
    nd->mass =
        ((nodes[c].mass + nodes[c + 1].mass) + nodes[c + 2].mass) + nodes[c + 3].mass;
  }
  for (size_t k = 0; k < count; ++k) {
    const float mm = fmaxf(nodes[k].mass, FLT_MIN);
    nodes[k].px = nodes[k].px / mm;
    nodes[k].py = nodes[k].py / mm;
  }
  /* QuadTree::acceleration, QuadTree.cpp:264-389 */
  for (size_t t = 0; t < n; ++t) {
    const float x = b[t].px, y = b[t].py;
    float ax = 0.0f, ay = 0.0f;
    int node = 0;
    for (;;) {
      const qnode *nd = &nodes[node];
      const float dx = nd->px - x, dy = nd->py - y;
      const float dSq = dx * dx + dy * dy;
      if (nd->size * nd->size < dSq * tSq) {
        if (nd->mass > 0.0f) {
          const float inv = fast_inv_sqrt(dSq);
          const float invSoft = 1.0f / (dSq + eSq);
          const float factor = fminf((nd->mass * inv) * invSoft, FLT_MAX);
          ax = ax + dx * factor;
          ay = ay + dy * factor;
        }
        if (nd->next == 0) break;
        node = nd->next;
      } else if (nd->children == 0) {
        float a0x = 0, a0y = 0, a1x = 0, a1y = 0, a2x = 0, a2y = 0, a3x = 0,
              a3y = 0;
        size_t i = nd->start;
        const size_t e = nd->end;
#define TERM(J, AX, AY)                                                       \
  do {                                                                        \
    const float ex = b[J].px - x, ey = b[J].py - y;                           \
    const float sq = ex * ex + ey * ey;                                       \
    const float inv = fast_inv_sqrt(sq);                                      \
    const float invSoft = 1.0f / (sq + eSq);                                  \
    const float f = fminf((b[J].mass * inv) * invSoft, FLT_MAX);              \
    AX = AX + ex * f;                                                         \
    AY = AY + ey * f;                                                         \
  } while (0)
        for (; i + 3 < e; i += 4) {
          TERM(i, a0x, a0y);
          TERM(i + 1, a1x, a1y);
          TERM(i + 2, a2x, a2y);
          TERM(i + 3, a3x, a3y);
        }
        for (; i < e; ++i) TERM(i, a0x, a0y);
#undef TERM
        ax = ax + (((a0x + a1x) + a2x) + a3x);
        ay = ay + (((a0y + a1y) + a2y) + a3y);
        if (nd->next == 0) break;
        node = nd->next;
      } else {
        node = nd->children;
      }
    }
    b[t].ax = ax;
    b[t].ay = ay;
  }
  free(nodes);
  free(parents);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Collision.cpp                                                         */
typedef struct box {
  float minX, maxX, minY, maxY;
  int index;
} box;

/* before(), Collision.cpp:88-90 */
static int before(const box *a, const box *b) {
  return a->minX < b->minX || (a->minX == b->minX && a->index < b->index);
}
/* overlaps(), Collision.cpp:95-98 */
static int overlaps(const box *earlier, const box *later) {
  return earlier->maxX >= later->minX && later->minY <= earlier->maxY &&
         earlier->minY <= later->maxY;
}

typedef struct pair {
  float laterMinX;
  int later;
  float earlierMinX;
  int earlier;
} pair;

/* pairLess, Collision.cpp:333-340 */
static int pair_cmp(const void *pa, const void *pb) {
  const pair *p = (const pair *)pa, *q = (const pair *)pb;
  int less, greater;
  if (p->later != q->later) {
    less = p->laterMinX < q->laterMinX ||
           (p->laterMinX == q->laterMinX && p->later < q->later);
    greater = q->laterMinX < p->laterMinX ||
              (q->laterMinX == p->laterMinX && q->later < p->later);
  } else {
    less = p->earlierMinX < q->earlierMinX ||
           (p->earlierMinX == q->earlierMinX && p->earlier < q->earlier);
    greater = q->earlierMinX < p->earlierMinX ||
              (q->earlierMinX == p->earlierMinX && q->earlier < p->earlier);
  }
  return less ? -1 : (greater ? 1 : 0);
}

static const box *g_sort_boxes;
static int box_order_cmp(const void *pa, const void *pb) {
  const box *a = &g_sort_boxes[*(const int *)pa];
  const box *b = &g_sort_boxes[*(const int *)pb];
  if (before(a, b)) return -1;
  if (before(b, a)) return 1;
  return 0;
}
static int float_cmp(const void *pa, const void *pb) {
  const float a = *(const float *)pa, b = *(const float *)pb;
  return (a < b) ? -1 : (b < a ? 1 : 0);
}

typedef struct pair_vec {
  pair *data;
  int64_t size, cap;
} pair_vec;

static int push_pair(pair_vec *v, const box *a, const box *b) {
  const box *earlier = before(a, b) ? a : b;
  const box *later = before(a, b) ? b : a;
  if (!overlaps(earlier, later)) return 0;
  if (v->size == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 4096;
    pair *d = (pair *)realloc(v->data, (size_t)v->cap * sizeof(pair));
    if (!d) return -1;
    v->data = d;
  }
  pair p = {later->minX, later->index, earlier->minX, earlier->index};
  v->data[v->size++] = p;
  return 0;
}

/* Every overlapping box pair (the set the grid broadphase of
 * Collision.cpp:176-334 finds), by an exact sweep in before() order.
 * Boxes much wider than the median are tested against every box. */
static int find_pairs(size_t n, const orc_body *b, pair_vec *out) {
  out->size = 0;
  if (n < 2) return 0;
  box *boxes = (box *)malloc(n * sizeof(box));
  float *widths = (float *)malloc(n * sizeof(float));
  int *order = (int *)malloc(n * sizeof(int));
  unsigned char *large = (unsigned char *)malloc(n);
  for (size_t i = 0; i < n; ++i) {
    /* pos -/+ Vec2::one() * radius, Collision.cpp:165-172 */
    const float r = b[i].radius;
    box bx = {b[i].px - r, b[i].px + r, b[i].py - r, b[i].py + r, (int)i};
    boxes[i] = bx;
    const float w = bx.maxX - bx.minX, h = bx.maxY - bx.minY;
    widths[i] = (w < h) ? h : w;
  }
  float *sortedW = (float *)malloc(n * sizeof(float));
  memcpy(sortedW, widths, n * sizeof(float));
  qsort(sortedW, n, sizeof(float), float_cmp);
  const float median = sortedW[n / 2];
  free(sortedW);
  const double bigW = 4.0 * (double)median + 1e-30;
  double maxSmall = 0.0;
  for (size_t i = 0; i < n; ++i) {
    /* NaN widths count as large so they are compared against all */
    large[i] = !((double)widths[i] <= bigW);
    if (!large[i] && (double)widths[i] > maxSmall) maxSmall = widths[i];
  }
  const double window = maxSmall * 1.001 + 1e-6;
  for (size_t i = 0; i < n; ++i) order[i] = (int)i;
  g_sort_boxes = boxes;
  qsort(order, n, sizeof(int), box_order_cmp);
  int rc = 0;
  /* small vs small: sweep in before() order */
  for (size_t k = 0; k < n && rc == 0; ++k) {
    const box *later = &boxes[order[k]];
    if (large[later->index]) continue;
    for (size_t e = k; e-- > 0;) {
      const box *earlier = &boxes[order[e]];
      if ((double)earlier->minX < (double)later->minX - window) break;
      if (large[earlier->index]) continue;
      if (push_pair(out, earlier, later)) { rc = -1; break; }
    }
  }
  /* large vs everything (large-large once) */
  for (size_t l = 0; l < n && rc == 0; ++l) {
    if (!large[l]) continue;
    for (size_t x = 0; x < n; ++x) {
      if (x == l) continue;
      if (large[x] && x < l) continue;
      if (push_pair(out, &boxes[l], &boxes[x])) { rc = -1; break; }
    }
  }
  free(boxes);
  free(widths);
  free(order);
  free(large);
  if (rc == 0 && out->size > 1)
    qsort(out->data, (size_t)out->size, sizeof(pair), pair_cmp);
  return rc;
}

int64_t orc_collision_pairs(size_t n, const orc_body *b, int32_t *later,
                            int32_t *earlier, int64_t cap) {
  pair_vec v = {NULL, 0, 0};
  if (find_pairs(n, b, &v)) {
    free(v.data);
    return INT64_MIN;
  }
  if (v.size > cap) {
    const int64_t need = v.size;
    free(v.data);
    return -need;
  }
  for (int64_t k = 0; k < v.size; ++k) {
    later[k] = v.data[k].later;
    earlier[k] = v.data[k].earlier;
  }
  const int64_t s = v.size;
  free(v.data);
  return s;
}

/* resolve(bodies, i, j), Collision.cpp:16-84 (i = later, j = earlier). */
static void resolve(orc_body *b, int i, int j) {
  float p1x = b[i].px, p1y = b[i].py, p2x = b[j].px, p2y = b[j].py;
  const float r1 = b[i].radius, r2 = b[j].radius;
  float dx = p2x - p1x, dy = p2y - p1y;
  const float r = r1 + r2;
  if (dx * dx + dy * dy > r * r) return;
  const float v1x = b[i].vx, v1y = b[i].vy, v2x = b[j].vx, v2y = b[j].vy;
  const float vx = v2x - v1x, vy = v2y - v1y;
  float dDotV = dx * vx + dy * vy;
  const float m1 = b[i].mass, m2 = b[j].mass;
  const float weight1 = m2 / (m1 + m2);
  const float weight2 = m1 / (m1 + m2);
  const int dNonZero = !(dx == 0.0f && dy == 0.0f);
  if (dDotV >= 0.0f && dNonZero) {
    const float s = r / sqrtf(dx * dx + dy * dy) - 1.0f;
    const float tx = dx * s, ty = dy * s;
    b[i].px = b[i].px - weight1 * tx;
    b[i].py = b[i].py - weight1 * ty;
    b[j].px = b[j].px + weight2 * tx;
    b[j].py = b[j].py + weight2 * ty;
    return;
  }
  const float vSqEarly = vx * vx + vy * vy;
  if (vSqEarly < 1e-12f) {
    float dirX = 1.0f, dirY = 0.0f;
    if (dNonZero) {
      const float inv = 1.0f / sqrtf(dx * dx + dy * dy);
      dirX = dx * inv;
      dirY = dy * inv;
    }
    const float tx = dirX * r, ty = dirY * r;
    b[i].px = b[i].px - weight1 * tx;
    b[i].py = b[i].py - weight1 * ty;
    b[j].px = b[j].px + weight2 * tx;
    b[j].py = b[j].py + weight2 * ty;
    return;
  }
  const float vSq = vx * vx + vy * vy;
  const float dSq = dx * dx + dy * dy;
  const float rSq = r * r;
  const float t =
      (dDotV + sqrtf(fmaxf(dDotV * dDotV - vSq * (dSq - rSq), 0.0f))) / vSq;
  b[i].px = b[i].px - v1x * t;
  b[i].py = b[i].py - v1y * t;
  b[j].px = b[j].px - v2x * t;
  b[j].py = b[j].py - v2y * t;
  p1x = b[i].px;
  p1y = b[i].py;
  p2x = b[j].px;
  p2y = b[j].py;
  dx = p2x - p1x;
  dy = p2y - p1y;
  dDotV = dx * vx + dy * vy;
  const float dSq2 = dx * dx + dy * dy;
  const float s = (1.5f * dDotV) / dSq2;
  const float tx = dx * s, ty = dy * s;
  const float n1x = v1x + tx * weight1, n1y = v1y + ty * weight1;
  const float n2x = v2x - tx * weight2, n2y = v2y - ty * weight2;
  b[i].vx = n1x;
  b[i].vy = n1y;
  b[j].vx = n2x;
  b[j].vy = n2y;
  b[i].px = b[i].px + n1x * t;
  b[i].py = b[i].py + n1y * t;
  b[j].px = b[j].px + n2x * t;
  b[j].py = b[j].py + n2y * t;
}

int64_t orc_collide(size_t n, orc_body *b) {
  if (n < 2) return 0;
  pair_vec v = {NULL, 0, 0};
  if (find_pairs(n, b, &v)) {
    free(v.data);
    return -1;
  }
  for (int64_t k = 0; k < v.size; ++k)
    resolve(b, v.data[k].later, v.data[k].earlier);
  const int64_t s = v.size;
  free(v.data);
  return s;
}

/* ------------------------------------------------------------------ */
int orc_step(size_t n, orc_body *b, float dt, float theta, float epsilon,
             int leafCapacity, int collisions) {
  orc_integrate(n, b, dt);
  if (collisions && orc_collide(n, b) < 0) return -1;
  if (n == 0) return 0;
  float *x = (float *)malloc(n * sizeof(float));
  float *y = (float *)malloc(n * sizeof(float));
  float *m = (float *)malloc(n * sizeof(float));
  float *ax = (float *)malloc(n * sizeof(float));
  float *ay = (float *)malloc(n * sizeof(float));
  uint64_t *codes = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint64_t *sorted = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint32_t *perm = (uint32_t *)malloc(n * sizeof(uint32_t));
  orc_body *tmp = (orc_body *)malloc(n * sizeof(orc_body));
  for (size_t i = 0; i < n; ++i) {
    x[i] = b[i].px;
    y[i] = b[i].py;
  }
  float root[3];
  orc_root_square(n, x, y, root);
  orc_morton(n, x, y, root, codes);
  orc_stable_perm(n, codes, perm);
  for (size_t i = 0; i < n; ++i) {
    tmp[i] = b[perm[i]];
    sorted[i] = codes[perm[i]];
  }
  memcpy(b, tmp, n * sizeof(orc_body));
  for (size_t i = 0; i < n; ++i) {
    x[i] = b[i].px;
    y[i] = b[i].py;
    m[i] = b[i].mass;
  }
  orc_tree t;
  const size_t cap = 8 * n + 8;
  float *fbuf = (float *)malloc(6 * cap * sizeof(float));
  int32_t *ibuf = (int32_t *)malloc(4 * cap * sizeof(int32_t));
  t.comX = fbuf;
  t.comY = fbuf + cap;
  t.mass = fbuf + 2 * cap;
  t.centerX = fbuf + 3 * cap;
  t.centerY = fbuf + 4 * cap;
  t.size = fbuf + 5 * cap;
  t.children = ibuf;
  t.next = ibuf + cap;
  t.start = ibuf + 2 * cap;
  t.end = ibuf + 3 * cap;
  t.capacity = (int32_t)cap;
  int rc = orc_build_tree(n, sorted, x, y, m, root, leafCapacity, &t);
  if (rc == 0) {
    orc_tree_forces(n, x, y, m, &t, theta, epsilon, ax, ay);
    for (size_t i = 0; i < n; ++i) {
      b[i].ax = ax[i];
      b[i].ay = ay[i];
    }
  }
  free(x);
  free(y);
  free(m);
  free(ax);
  free(ay);
  free(codes);
  free(sorted);
  free(perm);
  free(tmp);
  free(fbuf);
  free(ibuf);
  return rc;
}

/* ------------------------------------------------------------------ */
void orc_direct_fp64(size_t n, const float *x, const float *y, const float *m,
                     double epsilon, size_t nt, const uint32_t *targets,
                     double *ax, double *ay) {
  const double eSq = epsilon * epsilon;
  for (size_t k = 0; k < nt; ++k) {
    const size_t i = targets[k];
    double sx = 0.0, sy = 0.0;
    for (size_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double dx = (double)x[j] - (double)x[i];
      const double dy = (double)y[j] - (double)y[i];
      const double dSq = dx * dx + dy * dy;
      if (dSq == 0.0) continue; /* coincident: the tree law gives 0 */
      const double f = (double)m[j] / (sqrt(dSq) * (dSq + eSq));
      sx += dx * f;
      sy += dy * f;
    }
    ax[k] = sx;
    ay[k] = sy;
  }
}

static void neumaier(double *sum, double *c, double v) {
  const double t = *sum + v;
  if (fabs(*sum) >= fabs(v)) *c += (*sum - t) + v;
  else *c += (v - t) + *sum;
  *sum = t;
}

void orc_energy_momentum(size_t n, const orc_body *b, double out[5]) {
  double s[5] = {0, 0, 0, 0, 0}, c[5] = {0, 0, 0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    const double m = b[i].mass, vx = b[i].vx, vy = b[i].vy;
    const double x = b[i].px, y = b[i].py;
    neumaier(&s[0], &c[0], 0.5 * m * (vx * vx + vy * vy));
    neumaier(&s[1], &c[1], m * vx);
    neumaier(&s[2], &c[2], m * vy);
    neumaier(&s[3], &c[3], m * (x * vy - y * vx));
    neumaier(&s[4], &c[4], m);
  }
  for (int k = 0; k < 5; ++k) out[k] = s[k] + c[k];
}

double orc_potential_fp64(size_t n, const orc_body *b, double epsilon) {
  double s = 0.0, c = 0.0;
  const double halfPi = 1.5707963267948966;
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = i + 1; j < n; ++j) {
      const double dx = (double)b[j].px - b[i].px;
      const double dy = (double)b[j].py - b[i].py;
      const double r = sqrt(dx * dx + dy * dy);
      const double mm = (double)b[i].mass * (double)b[j].mass;
      neumaier(&s, &c, -(mm / epsilon) * (halfPi - atan(r / epsilon)));
    }
  }
  return s + c;
}

void orc_naive_forces(size_t n, const float *x, const float *y, const float *m,
                      float epsilon, float *ax, float *ay) {
  const float eSq = epsilon * epsilon;
  for (size_t i = 0; i < n; ++i) {
    float sx = 0.0f, sy = 0.0f;
    const float xi = x[i], yi = y[i];
    for (size_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const float dx = x[j] - xi, dy = y[j] - yi;
      const float dSq = dx * dx + dy * dy;
      const float invSoft = 1.0f / (dSq + eSq);
      const float invDist = 1.0f / sqrtf(dSq + eSq);
      const float factor = m[j] * invDist * invSoft;
      sx += dx * factor;
      sy += dy * factor;
    }
    ax[i] = sx;
    ay[i] = sy;
  }
}

int orc_naive_step(size_t n, orc_body *b, float dt, float epsilon, int collisions) {
  orc_integrate(n, b, dt);
  if (collisions && orc_collide(n, b) < 0) return -1;
  if (n == 0) return 0;
  float *x = (float *)malloc(5 * n * sizeof(float));
  if (!x) return -1;
  float *y = x + n, *m = x + 2 * n, *ax = x + 3 * n, *ay = x + 4 * n;
  for (size_t i = 0; i < n; ++i) {
    x[i] = b[i].px;
    y[i] = b[i].py;
    m[i] = b[i].mass;
  }
  orc_naive_forces(n, x, y, m, epsilon, ax, ay);
  for (size_t i = 0; i < n; ++i) {
    b[i].ax = ax[i];
    b[i].ay = ay[i];
  }
  free(x);
  return 0;
}

void orc_attractor(size_t n, const float *x, const float *y, float axp, float ayp,
                   float mass, float softening, float *ax, float *ay) {
  for (size_t i = 0; i < n; ++i) {
    const float dx = axp - x[i], dy = ayp - y[i];
    const float dSq = dx * dx + dy * dy;
    const float f = (mass * (1.0f / sqrtf(dSq + 1e-12f))) / (dSq + softening * softening);
    ax[i] = ax[i] + dx * f;
    ay[i] = ay[i] + dy * f;
  }
}

static float orc_mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }

static void orc_ramp(float t, float c[3]) {
  static const float slow[3] = {0.15f, 0.3f, 1.0f}, mid[3] = {0.2f, 0.95f, 1.0f},
                     fast[3] = {1.0f, 0.9f, 0.55f};
  t = fminf(fmaxf(t, 0.0f), 1.0f);
  if (t < 0.5f) {
    const float u = t * 2.0f;
    for (int k = 0; k < 3; ++k) c[k] = orc_mixf(slow[k], mid[k], u);
  } else {
    const float u = t * 2.0f - 1.0f;
    for (int k = 0; k < 3; ++k) c[k] = orc_mixf(mid[k], fast[k], u);
  }
}

static int orc_pixel_range(float wpos, float hf, uint32_t extent, int *lo, int *hi) {
  const float a = wpos - hf, b = wpos + hf;
  if (!(a < (float)extent) || !(b >= 0.0f)) return 0;
  *lo = a <= 0.0f ? 0 : (int)floorf(a);
  *hi = b >= (float)(extent - 1) ? (int)extent - 1 : (int)floorf(b);
  return *lo <= *hi;
}

void orc_render(size_t n, const orc_body *b, float camX, float camY, float scale,
                int mode, float pointScale, float minPoint, float brightness,
                float speedMax, uint32_t w, uint32_t h, float *rgba, float *stats) {
  for (size_t p = 0; p < (size_t)w * h; ++p) {
    rgba[4 * p + 0] = 0.0f;
    rgba[4 * p + 1] = 0.0f;
    rgba[4 * p + 2] = 0.02f;
    rgba[4 * p + 3] = 1.0f;
  }
  const float halfW = (float)w * 0.5f, halfH = (float)h * 0.5f;
  double mx = 0.0, my = 0.0, m = 0.0;
  float vmax = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    const float speed = sqrtf(b[i].vx * b[i].vx + b[i].vy * b[i].vy);
    m += b[i].mass;
    mx += (double)b[i].mass * b[i].px;
    my += (double)b[i].mass * b[i].py;
    vmax = fmaxf(vmax, speed);
    const float wx = (b[i].px - camX) * scale + halfW;
    const float wy = (b[i].py - camY) * scale + halfH;
    const float size = b[i].radius * 2.0f * scale * pointScale;
    const float ps = fmaxf(size, minPoint);
    const float alpha = fminf(fmaxf(size / minPoint, 0.08f), 1.0f);
    const float hf = ps * 0.5f;
    float c[3] = {0.35f, 0.75f, 1.0f};
    if (mode == 0) orc_ramp(speed / speedMax, c);
    int x0, x1, y0, y1;
    if (!orc_pixel_range(wx, hf, w, &x0, &x1) || !orc_pixel_range(wy, hf, h, &y0, &y1))
      continue;
    for (int py = y0; py <= y1; ++py) {
      for (int px = x0; px <= x1; ++px) {
        const float cx = (float)px + 0.5f, cy = (float)py + 0.5f;
        const float dx = (cx - wx) / hf, dy = (cy - wy) / hf;
        const float r2 = dx * dx + dy * dy;
        if (r2 > 1.0f) continue;
        const float a = (1.0f - r2) * alpha * brightness;
        float *d = rgba + 4 * ((size_t)py * w + px);
        const float s0 = c[0] * a, s1 = c[1] * a, s2 = c[2] * a;
        if (mode == 1) {
          d[0] = s0 + d[0];
          d[1] = s1 + d[1];
          d[2] = s2 + d[2];
          d[3] = a + d[3];
        } else {
          const float k1 = 1.0f - a;
          d[0] = s0 + d[0] * k1;
          d[1] = s1 + d[1] * k1;
          d[2] = s2 + d[2] * k1;
          d[3] = a + d[3] * k1;
        }
      }
    }
  }
  stats[0] = m > 0.0 ? (float)(mx / m) : 0.0f;
  stats[1] = m > 0.0 ? (float)(my / m) : 0.0f;
  stats[2] = vmax > 0.0f ? vmax : 1.0f;
}
