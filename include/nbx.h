/*
 * nbx.h -- C ABI of the B200 Barnes-Hut + collision step.
 *
 * A drop-in for the per-step path of tyreecepaul/n-body-simulation:
 * Simulation::step = iterate -> collide -> attract (src/Simulation.cpp:11-16,
 * src/cuda/CudaSimulation.cu:51-58).  Plain C types only; every call returns
 * an nbx_status and never exits the process (the reference's CUDA_CHECK
 * aborts, src/cuda/DeviceBodies.cuh:18-27).  One handle = one CUDA stream
 * and its captured step graphs; handles are independent (no global state),
 * a handle must not be used from two threads at once.
 *
 * A handle holds one or more independent simulations ("instances") of fixed
 * sizes, advanced together: one instance is the reference's Simulation /
 * CudaSimulation; many is the batched ensemble.
 */
#ifndef NBX_H
#define NBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes. */
typedef enum nbx_status {
  NBX_OK = 0,
  NBX_ERR_ARG = 1,         /* bad argument or size mismatch */
  NBX_ERR_CUDA = 2,        /* a CUDA call failed (see nbx_last_error) */
  NBX_ERR_CAPACITY = 3,    /* tree-node or collision-pair capacity exceeded */
  NBX_ERR_NONFINITE = 4,   /* a body position became NaN or infinite */
  NBX_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  NBX_ERR_STATE = 6,       /* call not valid in the handle's state */
  NBX_ERR_NOMEM = 7        /* device or host allocation failed */
} nbx_status;

/* Same 36-byte layout as the reference's Body (src/Body.h:5-13):
 * pos, vel, acc (Vec2 = 2 floats each), mass, radius, id. */
typedef struct nbx_body {
  float pos_x, pos_y;
  float vel_x, vel_y;
  float acc_x, acc_y;
  float mass;
  float radius;
  uint32_t id;
} nbx_body;

/* Step parameters.  Defaults (nbx_params_default) are the reference's:
 * dt 0.05 (Simulation.cpp:8), theta 1, epsilon 1, leaf capacity 16
 * (Simulation.cpp:9, TreeKernels.cuh:32-34), collisions on
 * (CudaSimulation.cuh:39-42). */
typedef struct nbx_params {
  float dt;
  float theta;
  float epsilon;
  int32_t leaf_capacity;  /* 1..64 */
  int32_t collisions;     /* 0/1 */
  int32_t exact_math;     /* 1: force arithmetic exactly as the reference
                             writes it (no FMA contraction, IEEE reciprocal),
                             bit-identical to the CPU traversal on the same
                             tree; 0: contracted, hardware reciprocal */
  int32_t use_mlp;        /* far-field correction of accepted cells with
                             size/distance >= mlp_band: 0 none (the
                             reference), 1 learned MLP (nbx_mlp_*), 2 the
                             analytic quadrupole term (control) */
  float node_factor;      /* node capacity per body (default 8, the
                             reference bound 8n+8, CudaQuadTree.cu:270-273) */
  float pair_factor;      /* collision partner slots per body (default 32) */
  int32_t force_blocks;   /* 0 = auto; else blocks of the force launch */
  int32_t device;         /* CUDA device ordinal; -1 = the current device */
  float mlp_band;         /* learned correction on accepted cells with
                             size/distance >= mlp_band (default 0.5) */
  int32_t force_law;      /* 0: Barnes-Hut tree (Simulation, default);
                             1: direct all-pairs sum with the Plummer law of
                             NaiveSimulation::attract
                             (src/naive/NaiveSimulation.cpp:17-57,
                             src/cuda/CudaNaive.cu:17-57); no tree is built,
                             use_mlp must be 0 */
  int32_t force_block;    /* threads per block of the default force walk:
                             128, 256 or 512 (0 = 256) */
  int32_t leaf_pairs;     /* default force walk: 1 takes a leaf's bodies two
                             at a time with paired FP32 instructions, 0 one
                             at a time (default 1); the same terms either
                             way, summed in another order */
} nbx_params;

typedef struct nbx_handle nbx_handle;

/* Step phases for nbx_phase (the reference's Simulation::iterate/collide/
 * attract and CudaQuadTree::build/computeForces, CudaSimulation.cuh:34-37,
 * CudaQuadTree.cuh:26-32). */
typedef enum nbx_phase_id {
  NBX_PHASE_ITERATE = 0,
  NBX_PHASE_COLLIDE = 1,
  NBX_PHASE_BUILD = 2,   /* bounds, Morton codes, sort, permute, tree */
  NBX_PHASE_FORCES = 3,  /* traversal of the last built tree */
  NBX_PHASE_ATTRACT = 4, /* BUILD then FORCES */
  NBX_PHASE_STEP = 5     /* ITERATE, COLLIDE (if on), ATTRACT */
} nbx_phase_id;

/* Fills p with the reference defaults.  (Simulation.cpp:7-9) */
int nbx_params_default(nbx_params *p);

/* Creates a handle on the current CUDA device for `num_instances`
 * instances of the given sizes (bodies are laid out instance after
 * instance).  Replaces `CudaSimulation(n)` / `CudaQuadTree(n)` /
 * `CudaCollider(b)` construction (CudaSimulation.cu:34-38,
 * CudaQuadTree.cu:269-334). */
int nbx_create(const nbx_params *p, uint32_t num_instances,
               const uint32_t *instance_sizes, nbx_handle **out);

/* Releases every device allocation of the handle. */
int nbx_destroy(nbx_handle *h);

/* Parameters; takes effect at the next step (graphs are re-captured).
 * Replaces the public fields dt/theta/epsilon/collisions of CudaSimulation
 * (CudaSimulation.cuh:39-42) and QuadTree(theta, epsilon, leafCapacity)
 * (QuadTree.h:76-79). */
int nbx_set_params(nbx_handle *h, const nbx_params *p);
int nbx_get_params(const nbx_handle *h, nbx_params *p);

/* Bodies in and out, 36-byte Body records, all instances back to back.
 * Replaces DeviceBodies::upload/download (DeviceBodies.cu:25-72).  Upload
 * also fixes each instance's collision cell from its radii (CudaCollision.cu
 * :201-215).  id_order = 1 writes body with id k of instance j at
 * instance_start(j) + k (Main.cpp:55-62 sortById); it requires the ids of
 * each instance to be a permutation of 0..size-1. */
int nbx_upload_bodies(nbx_handle *h, const nbx_body *bodies, size_t n);
int nbx_download_bodies(nbx_handle *h, nbx_body *bodies, size_t n,
                        int id_order);

/* Advances every instance by `steps` Simulation::step()s
 * (Simulation.cpp:11-16).  Asynchronous: launches the captured step graph
 * per step and returns; errors raised on the device surface at nbx_sync. */
int nbx_step(nbx_handle *h, uint32_t steps);

/* One Simulation::step() on host-owned bodies, the call the drop-in
 * Simulation::step() makes (Simulation.cpp:11-16 over the caller's
 * vector): uploads `in` (as nbx_upload_bodies), steps once and writes the
 * bodies in their order after the step (as nbx_download_bodies with
 * id_order 0) to `out`; synchronous.  in may equal out.  When out is
 * pinned host memory the force pass runs in ranges and each range's
 * records are copied to out while the later ranges still compute, so most
 * of the device-to-host copy is hidden; otherwise it is upload, step,
 * download. */
int nbx_step_io(nbx_handle *h, const nbx_body *in, nbx_body *out, size_t n);

/* The viewer's attractor (CudaSimulation.cuh:9-15, attractorKernel
 * CudaSimulation.cu:14-31): while active, every step adds to each body's
 * acceleration the pull of a point mass at (x, y),
 * d * mass / (sqrt(|d|^2 + 1e-12) * (|d|^2 + softening^2)), d = (x, y) - pos,
 * after the gravitational sum.  Defaults: inactive, mass 1e6, softening 50.
 * Takes effect from the next step enqueued; no graph is re-captured. */
int nbx_set_attractor(nbx_handle *h, int active, float x, float y, float mass,
                      float softening);

/* CudaSimulation::reset (CudaSimulation.cu:40-49): replaces every body of a
 * single-instance handle, any count, reallocating the device state for it.
 * Parameters, the attractor and loaded network parameters are kept. */
int nbx_reset(nbx_handle *h, const nbx_body *bodies, size_t n);

/* Headless splat renderer: the viewer's point-sprite drawing
 * (viewer/Renderer.cpp:8-52 shaders, 113-147 blending) rasterised by CUDA
 * into a float RGBA image, no graphics API.  Camera: screen = (world -
 * centre) * scale pixels from the image centre, y up (Renderer.h:5-10). */
typedef struct nbx_camera {
  float center_x, center_y;
  float scale; /* pixels per world unit */
} nbx_camera;
typedef struct nbx_draw {   /* DrawSettings (Renderer.h:14-20) */
  int32_t mode;             /* 0: speed colour ramp, composited over in draw
                               order; 1: glow, additive (default) */
  float point_scale;        /* multiplies each body's true size (1) */
  float min_point_px;       /* smallest drawn point; smaller ones fade (1.5) */
  float brightness;         /* (0.6) */
  float speed_max;          /* speed at the top of the colour ramp (60) */
} nbx_draw;
int nbx_draw_default(nbx_draw *d);
/* Renders the handle's bodies in their current array order (the order the
 * viewer draws) into rgba[height][width][4] (host memory, premultiplied,
 * row 0 at the bottom, cleared to (0, 0, 0.02, 1)); rgba may be NULL.
 * stats (may be NULL) receives the viewer's BodyStats {centre-of-mass x,
 * y, max speed} (Interop.cu:14-45, 80-104).  width, height <= 16384. */
int nbx_render(nbx_handle *h, const nbx_camera *cam, const nbx_draw *draw,
               uint32_t width, uint32_t height, float *rgba, float *stats);
/* BodyStats alone, for a follow-the-centre camera. */
int nbx_body_stats(nbx_handle *h, float *stats);

/* nbx_step with the duration of each step's force pass recorded by CUDA
 * events on the handle's stream, around the force launch inside the step's
 * graph (the same kernels as nbx_step, plus two event records per step).
 * Asynchronous like nbx_step; nbx_force_times synchronises and returns the
 * first `count` per-step durations (ms) of the last nbx_step_timed call.
 * No counterpart in the reference, which times whole sim.step() calls
 * only (src/Main.cpp:172-180). */
int nbx_step_timed(nbx_handle *h, uint32_t steps);
int nbx_force_times(nbx_handle *h, float *ms, uint32_t count);

/* Waits for the handle's stream and reports (and clears) device-side
 * error bits: NBX_ERR_CAPACITY, NBX_ERR_NONFINITE, NBX_ERR_TIMEOUT. */
int nbx_sync(nbx_handle *h);

/* Runs one phase eagerly (no graph); for parity checks. */
int nbx_phase(nbx_handle *h, int phase);

/* --- introspection of the last build / collide (parity checks) --- */

/* Morton codes of the last build in pre-sort body order, and the sort
 * permutation (sorted position -> pre-sort index), instance-local values.
 * (CudaQuadTree.cu:400-407) */
int nbx_get_morton(nbx_handle *h, uint32_t instance, uint64_t *codes,
                   uint32_t *perm, size_t n);

/* Node count and level count of an instance's last tree
 * (CudaQuadTree::nodeCount/levelCount, CudaQuadTree.cuh:34-36). */
int nbx_tree_size(nbx_handle *h, uint32_t instance, uint32_t *node_count,
                  uint32_t *level_count);

/* Node arrays of the last tree in the reference's breadth-first layout
 * (TreeKernels.cuh:88-95, CudaQuadTree::download CudaQuadTree.cu:515-533);
 * each array holds node_count entries; any pointer may be NULL. */
int nbx_get_tree(nbx_handle *h, uint32_t instance, float *com_x, float *com_y,
                 float *mass, float *center_x, float *center_y, float *size,
                 int32_t *children, int32_t *next, int32_t *start,
                 int32_t *end, size_t capacity);

/* Candidate pairs of the last collide in resolution (pairLess) order,
 * (later, earlier) body indices in the pre-collide order
 * (Collision.cpp:333-348).  *count receives the pair total; nothing is
 * written past `capacity`. */
int nbx_get_pairs(nbx_handle *h, int32_t *later, int32_t *earlier,
                  int64_t capacity, int64_t *count);

/* Contact statistics of the last collide: *pairs the candidate pairs it
 * resolved, *depth the longest chain of pairs that each wait for an
 * earlier pair sharing a body (the length of the sequential dependence in
 * Collision.cpp:341-348, which bounds the ordered resolution's time).  No
 * counterpart in the reference. */
int nbx_collision_stats(nbx_handle *h, int64_t *pairs, uint32_t *depth);

/* Accelerations at arbitrary points (px[i], py[i]) from instance 0's last
 * tree, with the handle's theta/epsilon: QuadTree::acceleration(pos, bodies)
 * for any position (QuadTree.h:83-85, QuadTree.cpp:264-389). */
int nbx_accel_at(nbx_handle *h, const float *px, const float *py, uint32_t n,
                 float *ax, float *ay);

/* --- NBS2 trajectory files (Main.cpp:13-49, load_sim.py:1-28) ---
 * 28-byte header "NBS2", n_bodies, total_steps, output_every, num_frames =
 * 1 + total_steps / output_every, completed_frames, dt; then float32
 * mass[n] and radius[n] in id order; then frames of n records
 * {x, y, vx, vy} in id order.  completed_frames is rewritten in place after
 * every frame, so a killed run stays readable. */
typedef struct nbx_nbs2 nbx_nbs2;
int nbx_nbs2_open(const char *path, uint32_t n, uint32_t total_steps,
                  uint32_t output_every, float dt, const float *mass_by_id,
                  const float *radius_by_id, nbx_nbs2 **out);
/* One frame from body records in id order (nbx_download_bodies with
 * id_order = 1). */
int nbx_nbs2_write_frame(nbx_nbs2 *f, const nbx_body *bodies_by_id);
/* One frame already in record layout: {x, y, vx, vy} per body, id order. */
int nbx_nbs2_write_packed(nbx_nbs2 *f, const float *xyvv_by_id, uint32_t n);
int nbx_nbs2_close(nbx_nbs2 *f);

/* Device-path frame output for a single-instance handle (MainCuda.cu:90-105
 * downloads the bodies and scatters them by id on the host).  Records the
 * current state as the next frame of f: an id-order scatter of
 * {x, y, vx, vy} on the handle's stream, a copy into pinned host memory on a
 * second stream, and a writer thread that appends it to f -- so the copy and
 * the file write overlap the steps enqueued after the call.  Frames are
 * written in call order; two frames can be in flight, a third call waits for
 * the oldest to be written.  Do not write to f by other calls until
 * nbx_nbs2_flush has returned.  No counterpart in the reference. */
int nbx_nbs2_record(nbx_handle *h, nbx_nbs2 *f);
/* Waits until every recorded frame is written; returns the first error. */
int nbx_nbs2_flush(nbx_handle *h);

/* Failure detection check: enqueues one bounded device wait on a flag that
 * nothing sets -- the same loop, limit and status bit as the ordered
 * resolution's and the radix sort's waits -- so that the next nbx_sync
 * returns NBX_ERR_TIMEOUT (about a second later) and the handle stays usable
 * afterwards.  No counterpart in the reference, whose waits are
 * unbounded. */
int nbx_debug_expire_wait(nbx_handle *h);

/* --- FP64 checks --- */

/* FP64 direct-sum accelerations for bodies at the given current indices,
 * over the other bodies of each target's own instance, with the handle's
 * force law: the tree's m d / (|d| (d^2 + eps^2)) (exactTreeLawForces,
 * CheckCuda.cu:453-475), or with force_law = 1 the Plummer law
 * m d / (d^2 + eps^2)^1.5; eps = params.epsilon. */
int nbx_direct_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                    double *ax, double *ay);

/* nbx_direct_fp64 for callers that cannot allocate device memory (their
 * memory belongs to another allocator or is budgeted at start-up, or they
 * must not pay cudaMalloc's device-wide synchronisation inside a loop).  No
 * counterpart in the reference.  Every pointer is DEVICE memory owned by
 * the caller: body positions x, y and masses (n floats each, the bodies'
 * current order), targets (m indices, each in 0..n-1; a target outside
 * that range is not read through and gets NaN outputs), outputs ax, ay
 * (m doubles); runs on `stream` (cudaStream_t, NULL = default stream) on
 * the current device.  It sums the tree law m d / (|d| (d^2 + eps^2)) over
 * all n bodies given, as nbx_direct_fp64 does for a single-instance handle
 * with force_law 0 (no Plummer law, no per-instance source ranges).
 * Allocates nothing: its partial sums live in a fixed 4 MiB device array of
 * the library, held by every GPU that loads it until exit.  At most 4096
 * targets per call (NBX_ERR_CAPACITY beyond).  The first call on a device
 * looks up that array's address and keeps it; make it before any stream
 * capture, and do not call it again on a device after cudaDeviceReset.
 * Calls share the array: calls whose kernels overlap on the GPU race, so
 * order them on one stream.  Launch failures are those of its own launches;
 * an error left pending by earlier CUDA calls is not cleared. */
int nbx_direct_fp64_noalloc(const float *x, const float *y, const float *mass,
                            uint32_t n, const uint32_t *targets, uint32_t m,
                            double epsilon, double *ax, double *ay,
                            void *stream);

/* Relative force error of the last force pass against nbx_direct_fp64 for
 * the given targets: stats = {median, p99, max, mean}; per-target errors
 * are written to err if not NULL.  (CheckCuda.cu:580-625) */
int nbx_force_error_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                         double *stats, double *err);

/* Error of the reference's force law itself: for the given targets, the
 * relative difference between the FP64 direct sum of the tree law computed
 * with the reference's fastInvSqrt (QuadTree.cpp:11-26, applied to the
 * float distance squared) and the FP64 direct sum of the exact law;
 * stats = {median, p99, max, mean}.  No tree and no float summation enter,
 * so this is the floor under the force error of every form that keeps the
 * reference's law.  Tree law (force_law 0) only.  No counterpart in the
 * reference. */
int nbx_law_error_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                       double *stats);

/* Compensated FP64 sums over all bodies: {kinetic energy, px, py, Lz,
 * total mass}.  No counterpart in the reference. */
int nbx_energy_momentum_fp64(nbx_handle *h, double *out5);

/* FP64 potential energy of the handle's force law, the partner of
 * nbx_energy_momentum_fp64's kinetic energy for total-energy drift.  The
 * pair potential is the one whose gradient is the law: for the tree law
 * m d / (|d| (d^2 + eps^2)) (exactTreeLawForces, CheckCuda.cu:453-475) it
 * is -m_i m_j atan(eps / r) / eps (-m_i m_j / r for eps = 0); for
 * force_law 1, -m_i m_j / sqrt(r^2 + eps^2).  Pairs are taken within each
 * instance.  targets == NULL: *u = the exact sum over all pairs (every body
 * a target of an FP64 direct sum, O(n^2): for test sizes or occasional
 * checks; compensated over the targets).  Otherwise phi[k] receives the
 * potential per unit mass at body targets[k] (current index) from every
 * other body of its instance, and *u the sampled estimate
 * (n / m) * 1/2 * sum_k mass_k * phi[k].  No counterpart in the reference. */
int nbx_potential_fp64(nbx_handle *h, const uint32_t *targets, uint32_t m,
                       double *phi, double *u);

/* --- measurement helpers (no counterpart in the reference) --- */

/* The CUDA stream (cudaStream_t) all of the handle's work runs on, so that
 * callers can time it with events recorded on the same stream. */
int nbx_get_stream(nbx_handle *h, void **stream);

/* Runs one step eagerly with CUDA events between its stages and returns
 * the stage durations: labels holds max_marks strings of 32 chars, ms the
 * milliseconds, *count the number of stages. */
int nbx_profile_step(nbx_handle *h, uint32_t max_marks, char *labels,
                     float *ms, uint32_t *count);

/* Kernel launches in one captured step. */
int nbx_step_kernel_count(nbx_handle *h, uint32_t *kernels);

/* Interactions of the traversal over the last tree for every body:
 * out5 = {accepted nodes with mass > 0, leaf body terms, visited nodes,
 * warp iterations, leaf chunks staged (up to 32 bodies each)}. */
int nbx_interaction_count(nbx_handle *h, double *out5);

/* FP32 FMA throughput of the current device (TFLOP/s, 2 flops per FMA),
 * measured with a probe kernel. */
int nbx_fp32_peak_tflops(double *tflops);

/* Device status bits (cleared on read) and the last error message. */
int nbx_status_bits(nbx_handle *h, uint32_t *bits);
const char *nbx_last_error(const nbx_handle *h);

/* --- learned far-field correction (no counterpart in the reference) ---
 * A 9 -> 32 -> 32 -> 2 SiLU MLP with BF16 weights and FP32 accumulation
 * corrects the monopole of accepted cells with size/distance >= mlp_band
 * when params.use_mlp = 1.  Parameters are 1442 FP32 values:
 * W1[32][9], b1[32], W2[32][32], b2[32], W3[2][32], b3[2].  A training row
 * is 12 floats: 9 features, 2 targets, weight. */
#define NBX_MLP_PARAMS 1442
#define NBX_MLP_ROW 12

int nbx_mlp_set_params(nbx_handle *h, const float *params, uint32_t n);
int nbx_mlp_get_params(nbx_handle *h, float *params, uint32_t n);

/* Xavier-uniform weights, zero biases, from mt19937(seed). */
int nbx_mlp_init(nbx_handle *h, uint32_t seed);

/* Walks the last tree from the bodies at the given current indices with
 * MAC theta; every accepted cell with size/distance >= band yields a row
 * whose targets come from an FP64 direct sum over the cell's bodies.
 * Writes at most max_rows rows; *n_rows receives the number written.  The
 * rows need the cells' second moments, which a tree built by nbx_phase
 * (BUILD or ATTRACT) always has and a tree built by nbx_step only with
 * use_mlp != 0 (otherwise NBX_ERR_STATE). */
int nbx_mlp_harvest(nbx_handle *h, const uint32_t *targets, uint32_t n_targets,
                    float theta, float band, float *rows, uint32_t max_rows,
                    uint32_t *n_rows);

/* Adam on the mean weighted squared error of the rows, minibatches of
 * `batch` rows in an order shuffled per epoch by mt19937(seed);
 * epoch_loss (epochs entries, may be NULL) receives the mean loss. */
int nbx_mlp_train(nbx_handle *h, const float *rows, uint32_t n_rows,
                  uint32_t epochs, uint32_t batch, float lr, uint32_t seed,
                  float *epoch_loss);

/* Gradient (1442 floats) and loss of the mean weighted squared error over
 * all rows, with the training kernels (for gradient checks). */
int nbx_mlp_gradient(nbx_handle *h, const float *rows, uint32_t n_rows,
                     float *grad, float *loss);

/* Network outputs (2 per row) for n feature rows of 9 floats, with the
 * training kernels (tensor_cores = 0) or the tensor-core inference path
 * of the traversal (tensor_cores = 1). */
int nbx_mlp_eval(nbx_handle *h, const float *features, uint32_t n, float *out,
                 int tensor_cores);

/* --- autotuner (no counterpart in the reference) ---
 * Times `steps` steps from the current state for each candidate -- for the
 * default plain walk the block shape (force_block 128, 256, 512 threads)
 * and the leaf width (leaf_pairs 1 or 0); force launch grids {one warp per
 * 32 bodies, 1/2, 1 or 2 SMs' worth of resident blocks per SM}; and, if
 * allow_leaf, leaf capacities {8, 12, 16, 24, 32} (a leaf capacity other
 * than 16 changes the tree, so results then differ from the reference's) --
 * keeps the fastest in the handle's parameters, and restores the state.
 * *best receives the chosen parameters, *best_ms their time per step. */
int nbx_autotune(nbx_handle *h, int allow_leaf, uint32_t steps,
                 nbx_params *best, float *best_ms);

/* --- host-side scenario generators (product host code) --- */

/* uniformDisc(n, seed): src/Utils.cpp:6-54. */
int nbx_uniform_disc(uint32_t n, uint32_t seed, nbx_body *out);

/* Two discs of n/2 and n - n/2 bodies (seeds seed, seed+1) centred at
 * (-sep/2, 0) and (+sep/2, 0) with sep = 6R (R = 5*sqrt(n/2), the disc
 * radius), bulk velocities (0, -f*v) and (0, +f*v) with
 * v = sqrt(M_total / (6R)), the second disc's spin reversed, ids renumbered
 * 0..n-1 (after viewer/Scenarios.cpp:36-48). */
int nbx_two_discs(uint32_t n, uint32_t seed, float approach_fraction,
                  nbx_body *out);

/* n unit-mass, radius-1 bodies at rest uniform in [-h, h]^2 with
 * h = 3*sqrt(n), mt19937(seed): the viewer's ColdSquare
 * (viewer/Scenarios.cpp:50-57), = nbx_make_scenario(NBX_SCENARIO_COLD_SQUARE). */
int nbx_cold_square(uint32_t n, uint32_t seed, nbx_body *out);

/* The viewer's scenarios and edits (viewer/Scenarios.h:1-23), for
 * injecting states into a handle without a GUI: edit a host copy, then
 * nbx_reset() the handle with it (viewer/main.cpp:122-129).  Results are
 * bit-identical to the viewer's build (its -O2 for these, -Ofast for
 * uniformDisc). */
enum {
  NBX_SCENARIO_DISC = 0,         /* uniformDisc(n, seed) */
  NBX_SCENARIO_TWO_GALAXIES = 1, /* two discs on a glancing course */
  NBX_SCENARIO_COLD_SQUARE = 2   /* unit masses at rest, half-width 3 sqrt(n) */
};
/* makeScenario (Scenarios.cpp:28-62): n bodies, ids 0..n-1.  n >= 1 for a
 * disc and n >= 2 for two galaxies (smaller sizes make the reference return
 * more bodies than asked: uniformDisc(0) still holds its central body). */
int nbx_make_scenario(int kind, uint32_t n, uint32_t seed, nbx_body *out);
/* renumber (Scenarios.cpp:22-26): ids 0..n-1 in array order. */
void nbx_renumber(nbx_body *bodies, size_t n);
/* addHeavyBody (Scenarios.cpp:64-70): writes body n (the array must hold
 * n + 1) at rest at (x, y); returns the new count. */
size_t nbx_add_heavy_body(nbx_body *bodies, size_t n, float x, float y, float mass);
/* addCluster (Scenarios.cpp:72-86): writes bodies n .. n+count-1 (unit
 * mass and radius, velocity (vx, vy)) in a small disc around (x, y),
 * mt19937(seed); returns the new count. */
size_t nbx_add_cluster(nbx_body *bodies, size_t n, float x, float y, float vx,
                       float vy, size_t count, uint32_t seed);

/* Instance sizes of the batched ensemble: instance i has
 * round(exp(U(ln lo, ln hi))) bodies, U drawn from mt19937(i). */
int nbx_ensemble_sizes(uint32_t count, uint32_t lo, uint32_t hi,
                       uint32_t *sizes);

/* Library build/version string. */
const char *nbx_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NBX_H */
