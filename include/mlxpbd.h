/*
 * mlxpbd.h -- C ABI of the B200 multi-layer XPBD step.
 *
 * This is the drop-in boundary for the reference's static
 * `xpbdLayer3D.layerSolve` (3d/integrator/xpbdLayer3D.m:44-93) and the helpers
 * `xpbdLayer3D.integrate` calls around it (xpbdLayer3D.m:601-745).  Every entry
 * point takes plain pointers and sizes, returns an int status (MLX_OK == 0) and
 * never throws; the message of the last failure on the calling thread is
 * available from mlx_last_error().
 *
 * Array conventions follow the MATLAB caller exactly, so a mex gateway can pass
 * mxArray data pointers straight through:
 *   - positions, velocities, forces, masses: 3N doubles, AoS [x1 y1 z1 x2 ...]
 *     (Mesh3D.p, Mesh3D.m:181);
 *   - index arrays are 1-based int32 and matrices are column-major
 *     (Mesh3D.t is T x 4, Mesh3D.m:193);
 *   - page arrays (DmInv 3x3xT, alpha 6x6xT) are column-major pages;
 *   - logical masks are one byte per entry (MATLAB `logical`).
 * The library never keeps a caller pointer beyond the call that received it.
 */
#ifndef MLXPBD_H
#define MLXPBD_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLX_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
  MLX_OK = 0,
  MLX_ERR_ARGUMENT = 1,     /* bad pointer / size / value                    */
  MLX_ERR_UNSUPPORTED = 2,  /* valid input this build does not handle        */
  MLX_ERR_CUDA = 3,         /* a CUDA runtime call failed                     */
  MLX_ERR_NO_DEVICE = 4,    /* no usable sm_100 device                        */
  MLX_ERR_NUMERIC = 5,      /* NaN/Inf detected in the state                  */
  MLX_ERR_LIMIT = 6,        /* an iteration or wait limit was reached         */
  MLX_ERR_ALLOC = 7         /* device or host allocation failed              */
};

/* ---- element energies (xpbdLayer3D.energyType, xpbdLayer3D.m:22) -------- */
enum {
  MLX_ENERGY_NEOHOOKEAN = 1,   /* stable Neo-Hookean D/H pair per tet; the 3D
                                  form of 2d/mex/mexNeoHookeanDConstraint.cpp and
                                  mexNeoHookeanHConstraint.cpp                   */
  MLX_ENERGY_STVK_VOIGT = 2    /* matStvkVoigtConstraint3D.m:1-45              */
};

/* ---- arithmetic of the bulk projection ---------------------------------- */
enum {
  MLX_FP32 = 0,   /* positions, lambdas and tet rest data in FP32; rigid-body
                     state, its reductions and the residual norm in FP64      */
  MLX_FP64 = 1    /* everything in FP64 (the reference's own precision)      */
};

/* Mesh precompute consumed by layerSolve: the Mesh3D fields of
 * xpbdLayer3D.m:713-729 (mass, t, pinnedDOFs, DmInv, alpha, beta, colours,
 * volume).  Compliance is given in ONE of two forms:
 *   (a) alpha/beta pages exactly as Mesh3D.updateMaterials builds them
 *       (Mesh3D.m:445-460).  They must be block diagonal (3x3 (+) 3x3 with a
 *       diagonal lower block) -- which updateMaterials always produces;
 *   (b) per-tet Lame parameters mu/lambda and Rayleigh alpha1, from which the
 *       same blocks are formed on the device (TriangleMaterial.m:18-64).
 * Neo-Hookean meshes need mu/lambda (form b). */
typedef struct mlx_mesh_desc {
  int32_t num_vertices;          /* N                                         */
  int32_t num_tets;              /* T                                         */
  const int32_t* t;              /* T x 4, column-major, 1-based              */
  const double* mass;            /* 3N lumped masses (computeMass.m:24-39)    */
  const double* DmInv;           /* 3 x 3 x T (computeB3D.m:24)               */
  const double* volume;          /* T (Mesh3D.elV)                            */
  const int32_t* element_color;  /* T, 1-based (naiveGraphColoring.m)         */
  int32_t num_colors;            /* max(element_color)                        */
  const int32_t* pinned_dofs;    /* 1-based DOF ids, sorted (pin.m:8)         */
  int32_t num_pinned_dofs;
  int32_t energy_type;           /* MLX_ENERGY_*                              */
  const double* alpha;           /* form (a): 6 x 6 x T, or NULL              */
  const double* beta;            /* form (a): 6 x 6 x T, or NULL              */
  const double* mu;              /* form (b): T, or NULL                      */
  const double* lambda;          /* form (b): T, or NULL                      */
  const double* alpha1;          /* form (b): T, or NULL (= 0)                */
  int32_t precision;             /* MLX_FP32 / MLX_FP64                       */
  int32_t device;                /* CUDA ordinal                              */
} mlx_mesh_desc;

/* The layer description of one call (xpbdLayer3D.m:44-49,54,59-60,84),
 * produced by buildLayers + findBoundaryVertices (xpbdLayer3D.m:646-652).
 * Per-layer arrays have `num_columns` columns (numel(sortedLayers)); user
 * layer l (0-based) reads column layers_map[l]-1. */
typedef struct mlx_layer_desc {
  int32_t num_layers;                  /* numel(layers)                       */
  int32_t num_columns;                 /* numel(sortedLayers)                 */
  const int32_t* layers_map;           /* num_layers, 1-based                 */
  const int32_t* iterations;           /* num_layers                          */
  const uint8_t* is_elastic_element;   /* T x num_columns                     */
  const uint8_t* is_rigid_element;     /* T x num_columns                     */
  const int32_t* rigid_body_sets;      /* T x num_columns, 0 = elastic        */
  const int32_t* vertex_rigid_body;    /* N x num_columns, 0 = elastic        */
  const uint8_t* is_boundary_vertex;   /* N x num_columns                     */
  const uint8_t* is_rigid_vertex;      /* N x num_columns                     */
  const int32_t* num_rigids;           /* num_columns                         */
} mlx_layer_desc;

/* Scalar settings of layerSolve (xpbdLayer3D.m:53-67,85-86,91-92). */
typedef struct mlx_solve_params {
  double h;
  double boundary_compliance;
  double contact_resistance;
  double run_until;                    /* runUntilResSmallerThan, <0 = off    */
  double give_up_threshold;
  double gravity_compliance;           /* accepted; gravity constraint is
                                          disabled in the reference (:325-327)*/
  double gravity;
  double stop_at_improvement_percent;
  int32_t compute_residuals;
  int32_t hanging_stop;                /* <0 = off                            */
  int32_t give_up_enabled;
  int32_t last_layer_give_up_enabled;
  int32_t use_gravity_constraints;
  int32_t use_rigid_contacts;
  int32_t contact_coloring;            /* 0: the reference's order -- elastic
                                          contacts after the colour sweep
                                          (xpbdLayer3D.m:315-341); 1: each
                                          vertex's elastic contacts in the
                                          first colour phase whose tets do not
                                          touch the vertex (after the sweep
                                          when every colour does).  No
                                          counterpart in the reference; device-
                                          detected contacts only
                                          (mlx_sim_set_obstacles). */
} mlx_solve_params;

/* Step-start contacts (xpbdLayer3D.m:675-681; contactInfo3D.m:32-55). */
typedef struct mlx_contacts {
  int32_t num_contacts;                /* K                                   */
  const double* normals;               /* K x 3, column-major                 */
  const double* point_colliders;       /* K x 3, column-major                 */
  const int32_t* vertex_ids;           /* K, 1-based                          */
  const double* compliance;            /* K (xpbdContactCompliance)           */
} mlx_contacts;

/* Per-step vectors of layerSolve. */
typedef struct mlx_solve_inputs {
  const double* xi;                    /* 3N                                  */
  const double* lambdai;               /* T x 6 column-major; NULL = zeros    */
                                       /* (what integrate passes)             */
  const double* oldp;                  /* 3N                                  */
  const double* old_oldp;              /* 3N (accepted; unused by the path)   */
  const double* f;                     /* 3N (accepted; unused by the path)   */
  const double* residualv;             /* 3N                                  */
  const double* pinnedx;               /* num_pinned_dofs                     */
  const double* residual_in;           /* residualArray on entry              */
  int32_t residual_in_len;
  double sum_non_monitored_time;
} mlx_solve_inputs;

typedef struct mlx_solve_outputs {
  double* xi;                          /* 3N                                  */
  double* lambdai;                     /* T x 6, optional (NULL = skip)       */
  double* residual;                    /* residualArray on exit (capacity)    */
  int32_t residual_capacity;
  int32_t residual_len;                /* written                             */
  double run_until;                    /* written                             */
  double sum_non_monitored_time;       /* written (host stop rules add their
                                          residual time; a replayed call,
                                          whose rules run on the device,
                                          passes the input through)           */
  int32_t total_iterations;            /* written: projectGS iterations run   */
} mlx_solve_outputs;

typedef struct mlx_solver mlx_solver;  /* device-resident mesh + work buffers */

/* ---- library ------------------------------------------------------------ */
const char* mlx_last_error(void);
int mlx_abi_version(void);
/* Number of visible sm_100 devices (0 when none). */
int mlx_device_count(void);

/* ---- solver (replaces the device residency of layerSolve's runOnGPU path,
 *      xpbdLayer3D.m:96-103 / 227-231) ------------------------------------ */
int mlx_create(const mlx_mesh_desc* mesh, mlx_solver** out);
int mlx_destroy(mlx_solver* solver);

/* xpbdLayer3D.layerSolve (xpbdLayer3D.m:44-232) with host buffers: uploads
 * the per-step vectors, runs every layer on the device, downloads xi.  The
 * outputs mirror [xi, sumNonMonitoredTime, residualArray, runUntil].  A call
 * with the same layers and params as the previous one and no host contacts
 * replays the loop recorded once as a CUDA graph; with compute_residuals the
 * stop rules then run on the device (the same results bit for bit; the
 * residual array may hold up to 16,384 entries on entry, else the call keeps
 * the host rules). */
int mlx_layer_solve(mlx_solver* solver,
                    const mlx_layer_desc* layers,
                    const mlx_solve_params* params,
                    const mlx_contacts* contacts,
                    const mlx_solve_inputs* in,
                    mlx_solve_outputs* out);

/* ---- device-resident stepping ------------------------------------------
 * xpbdLayer3D.integrate (xpbdLayer3D.m:621-745) with the state kept on the
 * device between steps: one solver holds one resident simulation.  The layer
 * description is fixed for all steps (fixed rigid clusters, or layers built
 * once), contacts are not detected, iterations are fixed
 * (compute_residuals = 0).  Frame 1 semantics: the pinned values are the
 * initial positions of the pinned DOFs (xpbdLayer3D.m:629-632). */
int mlx_sim_init(mlx_solver* solver, const mlx_layer_desc* layers,
                 const mlx_solve_params* params, const double* p0, const double* v0,
                 double air_drag);
/* Adds dv to the velocity DOFs `dofs` (1-based), as
 * VelocityImpulseAnimationScripter.scriptMesh does before a step
 * (3d/animations/VelocityImpulseAnimationScripter.m:16-30). */
int mlx_sim_add_velocity(mlx_solver* solver, const int32_t* dofs, const double* dv, int32_t n);
/* Runs `nsteps` steps; use_graph replays one captured CUDA graph per step.
 * With compute_residuals in the parameters the layers iterate until the
 * stop rules of simpleMonitorError end them (see mlx_sim_monitor).
 * device_ms (optional) receives the CUDA-event time of the steps. */
int mlx_sim_step(mlx_solver* solver, int32_t nsteps, int32_t use_graph, double* device_ms);
/* Copies positions and velocities (3N each, either may be NULL) to the host. */
int mlx_sim_get_state(mlx_solver* solver, double* p, double* v);
/* Colour-sweep timing of the resident stepper: with `on`, every iteration's
 * run of colour-projection kernels is bracketed by a pair of CUDA events on
 * the solver's stream (recorded inside the captured step).  sweep_stats
 * returns the summed device time, the algorithmic bytes of the projected tets
 * and the number of colour kernels since the last reset. */
int mlx_sim_sweep_timing(mlx_solver* solver, int32_t on);
int mlx_sim_sweep_stats(mlx_solver* solver, double* ms, double* bytes, long long* launches, int32_t reset);
/* Kernel launches per step of the resident stepper (after a step ran), and
 * kernel launches of the last mlx_layer_solve call. */
long long mlx_sim_launches_per_step(const mlx_solver* solver);
long long mlx_last_call_launches(const mlx_solver* solver);
/* No counterpart in the reference.  Per-colour tile autotuner of the
 * resident stepper: for every layer and colour, times `reps` launches of the
 * colour kernel at block sizes 32..256 on the current state, keeps the
 * fastest (positions and multipliers are restored) and recaptures the step.
 * before_ms / after_ms (optional) receive one step's device time with the
 * default and the tuned tiles. */
int mlx_sim_autotune(mlx_solver* solver, int32_t reps, double* before_ms, double* after_ms);
/* No counterpart in the reference.  Writes a one-line description of how
 * fixed-iteration layers are launched on this solver's device (thread-block
 * cluster size and threads, or per-colour launches) into buf (NUL-terminated,
 * at most n bytes).  Returns the length of the full description. */
int mlx_launch_path(const mlx_solver* solver, char* buf, int32_t n);

/* ---- analytic obstacles (contact finders) ------------------------------
 * One obstacle per contact finder of simulate3D (3d/simulate3D.m:156-171),
 * in finder order:
 *   MLX_OBSTACLE_PLANE  PlaneContactFinder3D(normal, position)
 *                       (3d/contact/PlaneContactFinder3D.m:16-32): `normal`
 *                       as given (the test uses it normalised, the offset
 *                       D = dot(normal, position) as given), `center` = position;
 *   MLX_OBSTACLE_SPHERE SphereContactFinder(radius, position)
 *                       (3d/contact/SphereContactFinder.m:13-21): `radius`,
 *                       `center`; its contacts keep contactInfo3D's default
 *                       compliance 1e-4 (the `compliance` field is ignored);
 *   MLX_OBSTACLE_BOX    PlatformContactDetector(degrees, scale, position)
 *                       (3d/contact/PlatformContactDetector.m:22-63):
 *                       `rotation` = RotationMatrixDegrees(degrees), row-major,
 *                       `scale` = [width depth height], `center` = position.
 * `compliance` is the finder's xpbdContactCompliance (1e-4 by default). */
#define MLX_OBSTACLE_PLANE 1
#define MLX_OBSTACLE_SPHERE 2
#define MLX_OBSTACLE_BOX 3
#define MLX_MAX_OBSTACLES 32
typedef struct mlx_obstacle {
  int32_t type;
  double normal[3];
  double center[3];
  double radius;
  double rotation[9];
  double scale[3];
  double compliance;
} mlx_obstacle;

/* Contact detection on the device for positions p (3N, host): the
 * concatenated contact lists of the finders, each finder's contacts in
 * ascending vertex order, as simulate3D builds them.  Writes, when
 * *num_contacts <= max_contacts, 1-based vertex ids (K), normals and collider
 * points (K x 3, column-major) and compliances (K); *num_contacts is always
 * set.  Returns MLX_ERR_LIMIT when the contacts do not fit. */
int mlx_find_contacts(mlx_solver* solver, const mlx_obstacle* obstacles, int32_t num_obstacles, const double* p,
                      int32_t max_contacts, int32_t* vertex_ids, double* normals, double* point_colliders,
                      double* compliance, int32_t* num_contacts);

/* Resident stepper with obstacles: every step detects the contacts of the
 * step-start positions on the device, projects them in every layer
 * (contactConstraints, xpbdLayer3D.m:422-485) and applies
 * contactVelocityUpdate with restitution e (xpbdLayer3D.m:740 uses 1e-2)
 * after the step, without a host round trip.  num_obstacles = 0 removes them.
 * Call after mlx_sim_init. */
int mlx_sim_set_obstacles(mlx_solver* solver, const mlx_obstacle* obstacles, int32_t num_obstacles,
                          double restitution);
/* Residual monitor of the last resident step run with compute_residuals:
 * its residualArray (the leading initial residual 0 included; at most
 * `capacity` entries copied, *len = full length), the projectGS iterations of
 * all layers, runUntilResSmallerThan after the step (it carries over to the
 * next step as in xpbdLayer3D.integrate) and a status (0 ok, 1 a layer hit
 * the iteration cap of 1e6, 2 the residual array overflowed).  In a graph
 * step (use_graph) the stop rules of simpleMonitorError run on the device
 * (conditional graph nodes); without a graph they run on the host. */
int mlx_sim_monitor(mlx_solver* solver, double* residuals, int32_t capacity, int32_t* len,
                    int32_t* total_iterations, double* run_until, int32_t* status);
/* Number of contacts of the last resident step (reads one int from the device). */
int mlx_sim_contact_count(mlx_solver* solver, int32_t* num_contact_vertices);

/* ---- preconditioned conjugate gradients ---------------------------------
 * solvePCG(iterations, Afun, b, zeros, preconditioner)
 * (2d/tools/solver/solvePCG.m:1-56) on the device for the linearly implicit
 * system of the mesh, A = M + h^2 K0: lumped masses and the linear-elasticity
 * stiffness at the rest shape from each tet's DmInv, volume, mu and lambda
 * (the system quickSolve3D.m:170 hands to solvePCG, without damping, at the
 * rest tangent), restricted to the unpinned DOFs; preconditioner: the 3x3
 * block-Jacobi inverse of A.  b and x are 3N (pinned components of x are 0);
 * resvec (optional, `iterations` values) receives ||A x - b|| after every
 * iteration, as solvePCG's second output.  Needs mu and lambda in the mesh
 * description. */
int mlx_pcg_solve(mlx_solver* solver, double h, const double* b, int32_t iterations, double* x, double* resvec);

/* The PCG in the layer solve.  No counterpart in the reference's layerSolve
 * (its PCG, solvePCG.m, serves the non-XPBD quick solve).  With
 * pcg_iterations > 0 the last layer of a Neo-Hookean mesh (no rigid bodies)
 * takes Newton-PCG corrections: the XPBD projection linearised at the current
 * positions, (M + J^T W J) dx = -J^T (W C + lambda) with W = alpha~^-1 on
 * the free DOFs, solved by `pcg_iterations` iterations of solvePCG's method
 * with the 3x3 block-Jacobi preconditioner; then x += dx and
 * lambda = -W (C + J dx).  One correction comes before the layer's
 * Gauss-Seidel and one after every `every` of its iterations (0: only the
 * first).  The stop rules are unchanged.  Applies to mlx_layer_solve and
 * the resident stepper (also inside its captured step, as a conditional
 * node); pcg_iterations = 0 (the default) restores the reference's
 * projectGS.  MLX_ERR_UNSUPPORTED for StVK meshes. */
int mlx_layer_pcg(mlx_solver* solver, int32_t pcg_iterations, int32_t every);

/* Diagnostic of the bounded device waits (no counterpart in the reference):
 * one thread runs the wait the library's kernels use -- kind 0: the grid
 * barrier of the persistent layer kernel, kind 1: the mbarrier wait of the
 * tensor-core GEMM -- on a condition nothing satisfies, so it gives up after
 * limit_ns (clamped to [1 ms, 2 s]) and *timed_out is set to 1.  Shows that a
 * wait that runs out ends with a status and leaves the context usable. */
int mlx_wait_probe(int32_t device, int32_t kind, int64_t limit_ns, int32_t* timed_out);

/* xpbdLayer3D.buildLayers (3d/integrator/xpbdLayer3D.m:601-619) followed by
 * xpbdLayer2D.findBoundaryVertices (2d/integrator/xpbdLayer2D.m:551-569) on
 * the device, replacing mexEdiffNorm3D + sort + mexUnionFindByVertice and
 * the mask computation of the host.  ordering 0: strain-rate order of p and
 * oldp (3N each, host) with the mesh's DmInv (9 values per element, as in
 * mlx_mesh_desc; copied to the device once per pointer) and step h;
 * ordering 1: `order` (T, 1-based element ids, e.g. a random permutation).
 * sorted_layers: ascending layer percentages (num_layers); forced_elastic:
 * T flags (pinned tets).  Outputs (host, column-major, one column per sorted
 * layer): rigidBodySetsPerLayer (T x L, 0 = elastic, bodies numbered by
 * their smallest element), numRigids (L), isElasticElement (T x L),
 * isBoundaryVertex, isRigidVertex (N x L), vertexRigidBody (N x L); the four
 * mask outputs may be NULL.  Results are the bits of the host builder. */
int mlx_build_layers(mlx_solver* solver, const double* p, const double* oldp, double h, int32_t ordering,
                     const int32_t* order, const double* DmInv, const double* sorted_layers, int32_t num_layers,
                     const uint8_t* forced_elastic, int32_t* rigid_body_sets, int32_t* num_rigids,
                     uint8_t* is_elastic_element, uint8_t* is_boundary_vertex, uint8_t* is_rigid_vertex,
                     int32_t* vertex_rigid_body);

/* ---- learned warm start: the perceptron ----------------------------------
 * No counterpart in the reference.  n_in -> n_hidden (GELU) x
 * n_hidden_layers -> n_out, BF16 weights and activations with FP32
 * accumulation on the tensor cores (tcgen05), FP32 master parameters and
 * Adam.  Parameters are flat FP32: per layer W (n_out x n_in, row-major) then
 * b.  n_hidden is 64 or 128; batches hold at most max_batch rows.  Inputs,
 * outputs and targets are row-major FP32 host arrays.  The loss is the mean
 * squared error over the n_out outputs of the batch. */
typedef struct mlx_mlp mlx_mlp;
int mlx_mlp_create(int32_t n_in, int32_t n_hidden, int32_t n_hidden_layers, int32_t n_out, int32_t max_batch,
                   uint64_t seed, int32_t device, mlx_mlp** out);
int mlx_mlp_destroy(mlx_mlp* mlp);
long long mlx_mlp_num_params(const mlx_mlp* mlp);
int mlx_mlp_set_params(mlx_mlp* mlp, const float* params, long long n);
int mlx_mlp_get_params(mlx_mlp* mlp, float* params, long long n);
int mlx_mlp_forward(mlx_mlp* mlp, const float* x, int32_t batch, float* y);
/* Loss and (optional) flat gradient of one batch, without an update. */
int mlx_mlp_loss_grad(mlx_mlp* mlp, const float* x, const float* target, int32_t batch, float* loss, float* grad);
/* Adam over `epochs` shuffled passes of n_samples rows in batches of `batch`
 * (learning rate lr); losses (optional) receives each epoch's mean loss. */
int mlx_mlp_train(mlx_mlp* mlp, const float* x, const float* target, int32_t n_samples, int32_t batch, int32_t epochs,
                  float lr, uint64_t seed, float* losses);

/* Learned warm start of the resident stepper's first layer (its rigid
 * clusters).  No counterpart in the reference.  For every cluster, right
 * after makeRigidsFromConnectivity, 44 features are formed on the device: its
 * COM velocity, angular velocity, COM displacement from the positions given
 * to mlx_sim_init and the rotation vector of its deformation from them (FP64
 * polar decomposition), and for the 4 clusters nearest at rest their
 * relative velocities, COM distance change and mass ratio.  8 outputs per
 * cluster: a COM-velocity and angular-velocity correction applied before the
 * symplectic rigid step (6), the cluster's starting boundary multiplier (0 in
 * the reference) (1), and the predicted residual of its rigid fit, log10 of
 * the RMS distance (m) of its vertices' final positions from the best-fit
 * rigid motion of the step (1).  A cluster whose predicted residual exceeds
 * `fallback_residual` (m; <= 0: never) gets no correction -- the plain
 * solve's start -- and is counted (mlx_sim_warm_start_fetch).
 *   mode 1: `net` (44 -> 8) maps normalised features
 *           ((f - feature_mean) / feature_std) to normalised outputs
 *           (denormalised with output_mean / output_std);
 *   mode 2: `corrections` (num_clusters x 8, output units) are applied;
 *   mode 0: nothing is applied.
 * With `record` every step keeps its raw features and the targets -- the
 * corrections that would have put each cluster on the best-fit rigid motion
 * to its final positions, its mean final boundary multiplier and the log10
 * RMS residual of that fit -- for mlx_sim_warm_start_fetch, which also
 * returns how many clusters fell back in the last step.  The stop rules are
 * unchanged: a warm start changes the iterations needed to reach the
 * residual, not the residual. */
int mlx_sim_warm_start(mlx_solver* solver, int32_t record, int32_t mode, mlx_mlp* net, double fallback_residual,
                       const float* feature_mean, const float* feature_std, const float* output_mean,
                       const float* output_std, const float* corrections, int32_t* num_clusters);
int mlx_sim_warm_start_fetch(mlx_solver* solver, float* features, float* targets, int32_t capacity,
                             int32_t* num_clusters, int32_t* num_fallbacks);

/* Multiplier warm start of the resident stepper.  No counterpart in the
 * reference, which zeroes every tet's multipliers at the start of a step
 * (xpbdLayer3D.m:666) and rebuilds them in every step's projectGS.  With `on`,
 * the last layer (the fine layer) starts from the converged multipliers of
 * the previous steps,
 *   lambda0 = a lambda_{n-1} + b (lambda_{n-1} - lambda_{n-2}),
 * and its positions move by the displacement the change of multipliers
 * implies, M^-1 grad C(x)^T (lambda0 - lambda), so that the layer's
 * Gauss-Seidel continues from a state with the same fixed point to first
 * order (a = `scale`, b = `extrapolation`).  The first step after this call
 * starts from the plain state and the second uses b = 0.  on = 0 (the
 * default) restores the reference's start.  The stop rules are unchanged.
 * Measured: <= 5 % fewer iterations to residual 1e-4 on the Neo-Hookean
 * blocks and none on the contact-heavy drop, with positions 3e-4 to 6e-4 of
 * the bounding-box diagonal away from the plain solve's after one step (the
 * fixed point of Gauss-Seidel on these nonlinear constraints depends on the
 * path), so it stays an option. */
int mlx_sim_multiplier_warm_start(mlx_solver* solver, int32_t on, double scale, double extrapolation);

/* ---- allocation-free residual ------------------------------------------
 * No counterpart in the reference.  The elastic constraint residual of
 * simpleEvaluateAllConstraintResiduals (StVK Voigt tets, no contacts) on
 * device arrays the caller owns, for callers that cannot allocate device
 * memory (a MATLAB mexcuda function working on gpuArray memory, a fixed-rate
 * loop where cudaMalloc would stall).  Inputs are device pointers in the
 * MATLAB layout of mlx_mesh_desc / mlx_solve_inputs; d_residual receives one
 * double.  The call only enqueues work on `stream` (a cudaStream_t, NULL =
 * default stream) and allocates nothing: its scratch is a fixed device array
 * of MLX_NOALLOC_MAX_TETS/256 doubles inside the library, shared by all calls
 * (calls that overlap on the GPU race; serialise them).  The first call in a
 * CUDA context (on a device, and again after cudaDeviceReset) looks that
 * array up and should come before any stream capture.  Types: d_t is int32
 * (T x 4, 1-based: int32(mesh.t) in MATLAB, whose mesh.t is double); d_x,
 * d_DmInv, d_alpha, d_lambda and d_volume are double.  A tet whose vertex
 * index lies outside [1, num_vertices] is not read and makes the residual
 * NaN.  An error already pending on entry is reported (MLX_ERR_CUDA) and
 * nothing is launched.  More than MLX_NOALLOC_MAX_TETS tets is rejected with
 * MLX_ERR_ARGUMENT. */
#define MLX_NOALLOC_MAX_TETS 524288
int mlx_stvk_residual_noalloc(int32_t num_vertices, int32_t num_tets, const double* d_x,
                              const int32_t* d_t, const double* d_DmInv, const double* d_alpha,
                              const double* d_lambda, const double* d_volume, double h,
                              double* d_residual, void* stream);

/* ---- host-side helpers of the step (run on the CPU in the reference too) */

/* naiveGraphColoring (2d/tools/functionalities/naiveGraphColoring.m:1-19):
 * greedy first-fit colour per tet in index order.  Returns num_colors. */
int mlx_greedy_coloring(const int32_t* t, int32_t num_tets, int32_t num_vertices,
                        int32_t* element_color, int32_t* num_colors);

/* mexEdiffNorm3D applied to F = B*p and B*oldp (xpbdLayer3D.m:606-608,
 * 3d/mex/mexEdiffNorm3D.cpp:25-61): per-tet strain-rate norm. */
int mlx_strain_rate_norms(const int32_t* t, int32_t num_tets, const double* DmInv,
                          const double* p, const double* oldp, double h,
                          double* norms);

/* buildLayers' ordering + mexUnionFindByVertice (xpbdLayer3D.m:601-619,
 * 2d/mex/mexUnionFindByVertice.cpp:117-178).  `order` is the 1-based element
 * order (strain-rate ascending), `sorted_layers` the ascending unique
 * percentages.  Writes T x num_sorted rigid IDs and num_sorted counts. */
int mlx_union_find_layers(const int32_t* order, int32_t num_tets,
                          const double* sorted_layers, int32_t num_sorted,
                          const uint8_t* forced_elastic, const int32_t* t,
                          int32_t num_vertices, int32_t* rigid_body_sets,
                          int32_t* num_rigids);

/* xpbdLayer2D.findBoundaryVertices (2d/integrator/xpbdLayer2D.m:551-569). */
int mlx_find_boundary_vertices(const int32_t* t, int32_t num_tets,
                               int32_t num_vertices,
                               const int32_t* rigid_body_sets, int32_t num_columns,
                               uint8_t* is_boundary_vertex,
                               uint8_t* is_elastic_element,
                               uint8_t* is_rigid_vertex,
                               int32_t* vertex_rigid_body);

/* The per-step vector arithmetic of xpbdLayer3D.integrate around layerSolve,
 * each phase one fused pass over the DOFs (split over host threads for large
 * meshes), with the reference's operation order so results are the same
 * doubles as the element-wise MATLAB expressions.
 *
 * mlx_any_nan: any(isnan(x)) of the step-start check (xpbdLayer3D.m:629).
 * Returns 1 or 0 (0 for n <= 0), or minus MLX_ERR_ARGUMENT for a NULL x.
 *
 * mlx_integrate_begin (xpbdLayer3D.m:638-643, 662-664): forces
 * f = [0, 0, mass_z * gravity] + custom force (`custom_force_vec` of
 * num_dofs values, or the scalar `custom_force` when it is NULL) and the
 * residual velocity (1 - air_drag) * (v + h f / mass) with the h f / mass
 * term left out at the 1-based `pinned_dofs`.  f and residualv may not alias
 * the inputs.
 *
 * mlx_integrate_end (xpbdLayer3D.m:737): v = (xi - oldp) / h.  v may alias
 * neither input. */
int32_t mlx_any_nan(int64_t n, const double* x);
int mlx_integrate_begin(int32_t num_dofs, double h, double gravity, double air_drag,
                        double custom_force, const double* custom_force_vec,
                        const double* mass, const double* v,
                        const int32_t* pinned_dofs, int32_t num_pinned,
                        double* f, double* residualv);
int mlx_integrate_end(int32_t num_dofs, double h, const double* xi, const double* oldp,
                      double* v);

/* xpbdLayer2D.contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603),
 * called after the step with the step-start contacts (xpbdLayer3D.m:740):
 * normals K x dim column-major, 1-based vertex ids (the first column of
 * contactVertexID), v of num_dofs = dim x vertices values; the updated
 * velocities go to v_out, which may be v itself.  A vertex with several
 * contacts keeps its last contact's value. */
int mlx_contact_velocity_update(int32_t num_contacts, const double* normals,
                                const int32_t* vertex_ids, int32_t dim, int64_t num_dofs,
                                const double* v, double h, double gravity,
                                double restitution, double* v_out);

#ifdef __cplusplus
}
#endif
#endif /* MLXPBD_H */
