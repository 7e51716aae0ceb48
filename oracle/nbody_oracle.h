/*
 * nbody_oracle.h -- CPU restatement of the reference's per-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * Every function restates one piece of tyreecepaul/n-body-simulation and
 * cites the file:line it follows.  The library is built with
 * -O2 -ffp-contract=off -fno-fast-math so that every float operation is a
 * single IEEE-754 round-to-nearest operation, as written.
 *
 * Parity pinning: oracle/pin_oracle.py checks these functions bit-for-bit
 * against the reference itself (oracle/_ref, compiled from the reference's
 * own sources by oracle/Makefile) and tests/golden/ holds fixtures written
 * by the reference (tests/golden/make_golden.py).
 */
#ifndef NBODY_ORACLE_H
#define NBODY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 36-byte layout as the reference's Body (src/Body.h:5-13). */
typedef struct orc_body {
  float px, py, vx, vy, ax, ay, mass, radius;
  uint32_t id;
} orc_body;

/* Node arrays as in src/cuda/TreeKernels.cuh:88-95 (NodeArrays). */
typedef struct orc_tree {
  float *comX, *comY, *mass, *centerX, *centerY, *size;
  int32_t *children, *next, *start, *end;
  int32_t capacity;
  int32_t nodeCount;
  int32_t levelCount;
} orc_tree;

/* Body::update for every body (src/Body.h:20-23, src/Simulation.cpp:44-50). */
void orc_integrate(size_t n, orc_body *b, float dt);

/* Root square {cx, cy, size} from the bounding box, as
 * Quad::newContaining (src/QuadTree.cpp:30-51) and rootSquare
 * (src/cuda/CudaQuadTree.cu:25-30).  NaN coordinates never win a min/max
 * (std::min/std::max semantics). */
void orc_root_square(size_t n, const float *x, const float *y, float out[3]);

/* 64-bit Morton codes over the root square with the reference's double
 * quantisation (src/cuda/TreeKernels.cuh:37-66, CudaQuadTree.cu:32-47). */
void orc_morton(size_t n, const float *x, const float *y, const float root[3],
                uint64_t *codes);

/* Stable sort of indices by code (cub::DeviceRadixSort::SortPairs is stable;
 * CudaQuadTree.cu:405-407). */
void orc_stable_perm(size_t n, const uint64_t *codes, uint32_t *perm);

/* Breadth-first tree over Morton-sorted codes, exactly as buildHostLoop
 * (CudaQuadTree.cu:452-498) with splitNode/sumNode/finishNode
 * (TreeKernels.cuh:117-177).  Returns 0, or -1 on node-capacity overflow. */
int orc_build_tree(size_t n, const uint64_t *sortedCodes, const float *x,
                   const float *y, const float *m, const float root[3],
                   int leafCapacity, orc_tree *t);

/* accelerationAt (TreeKernels.cuh:197-245) for every body. */
void orc_tree_forces(size_t n, const float *x, const float *y, const float *m,
                     const orc_tree *t, float theta, float epsilon, float *ax,
                     float *ay);

/* Interaction counts of accelerationAt for selected targets: far (accepted
 * node with mass > 0), near (leaf body terms) and node visits. */
void orc_interaction_counts(size_t nt, const uint32_t *targets, const float *x,
                            const float *y, const orc_tree *t, float theta,
                            double out[3]);

/* QuadTree.cpp's own in-place partition tree + acceleration for every body
 * (QuadTree.cpp:154-389, Partition.h:7-18).  Reorders `b` like
 * QuadTree::build does; writes b[i].ax/ay. */
int orc_quadtree_forces(size_t n, orc_body *b, float theta, float epsilon,
                        int leafCapacity);

/* Collision candidate pairs: every pair of boxes that overlaps under
 * Collision.cpp's before()/overlaps() (Collision.cpp:88-98), returned as
 * (later, earlier) index pairs in pairLess order (Collision.cpp:333-340).
 * Returns the number of pairs, or -(needed) if cap is too small. */
int64_t orc_collision_pairs(size_t n, const orc_body *b, int32_t *later,
                            int32_t *earlier, int64_t cap);

/* collide(): pairs in pairLess order, each resolved in sequence with
 * Collision.cpp's resolve() (Collision.cpp:16-84, 346-348).
 * Returns the number of candidate pairs, or -1 on allocation failure. */
int64_t orc_collide(size_t n, orc_body *b);

/* One step as CudaSimulation::step (CudaSimulation.cu:51-58) but with
 * Collision.cpp's sequential resolution: iterate -> collide -> Morton
 * sort (bodies permuted into Morton order) -> tree -> forces.
 * Returns 0, or -1 on failure. */
int orc_step(size_t n, orc_body *b, float dt, float theta, float epsilon,
             int leafCapacity, int collisions);

/* Direct all-pairs accelerations, NaiveSimulation::attract
 * (src/naive/NaiveSimulation.cpp:17-57): for each i, over j != i in index
 * order, d = pos_j - pos_i, s = |d|^2 + eps^2,
 * acc += d * (m_j * (1/sqrt(s)) * (1/s)), IEEE single precision. */
void orc_naive_forces(size_t n, const float *x, const float *y, const float *m,
                      float epsilon, float *ax, float *ay);

/* One NaiveSimulation::step (NaiveSimulation.cpp:10-15): iterate -> collide
 * -> naive attract; bodies keep their order.  Returns 0, or -1. */
int orc_naive_step(size_t n, orc_body *b, float dt, float epsilon, int collisions);

/* The viewer's attractor pull (attractorKernel,
 * src/cuda/CudaSimulation.cu:14-31) added to ax/ay in IEEE single
 * precision: d = a - p, f = (m * (1/sqrt(|d|^2 + 1e-12))) / (|d|^2 + s^2),
 * acc += d * f. */
void orc_attractor(size_t n, const float *x, const float *y, float axp, float ayp,
                   float mass, float softening, float *ax, float *ay);

/* The viewer's point-sprite drawing restated (src/viewer/Renderer.cpp:8-52
 * shaders, 113-147 blending; the product's headless renderer defines the
 * same math): bodies in array order into rgba[h][w][4], row 0 at the
 * bottom, cleared to (0, 0, 0.02, 1); mode 0 speed ramp composited over,
 * mode 1 glow additive.  stats = {comX, comY, maxSpeed} as BodyStats
 * (Interop.cu:80-104), sums in FP64 in index order. */
void orc_render(size_t n, const orc_body *b, float camX, float camY, float scale,
                int mode, float pointScale, float minPoint, float brightness,
                float speedMax, uint32_t w, uint32_t h, float *rgba, float *stats);

/* FP64 direct sum with the tree's force law for the given targets
 * (exactTreeLawForces, src/cuda/CheckCuda.cu:453-475; eps generalised). */
void orc_direct_fp64(size_t n, const float *x, const float *y, const float *m,
                     double epsilon, size_t nt, const uint32_t *targets,
                     double *ax, double *ay);

/* Compensated (Neumaier) FP64 sums: out = {kinetic energy, px, py, Lz,
 * total mass}. */
void orc_energy_momentum(size_t n, const orc_body *b, double out[5]);

/* Pair potential energy of the tree force law, O(n^2) in FP64:
 * phi(r) = -(m_i m_j / eps) * (pi/2 - atan(r / eps)). */
double orc_potential_fp64(size_t n, const orc_body *b, double epsilon);

#ifdef __cplusplus
}
#endif
#endif
