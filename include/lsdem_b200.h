/*
 * lsdem_b200 — C ABI of the B200-native level-set DEM step.
 *
 * Plain pointers and sizes only. Vectors are 3 doubles (x, y, z), quaternions
 * 4 doubles (q0 scalar first, local -> world), symmetric tensors 6 doubles
 * (xx, yy, zz, xy, xz, yz), integer triples 3 ints. Every call returns an
 * LSDEM_* status; lsdem_last_error() gives the message of the last failure.
 *
 * Each entry point replaces a part of the reference solver's host API or of
 * its internal extern "C" launcher layer; the reference interface is cited
 * (paths relative to the reference project root).
 */
#ifndef LSDEM_B200_H
#define LSDEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define LSDEM_OK 0
#define LSDEM_ERR_ARG 1      /* invalid argument (reference: cerr + return) */
#define LSDEM_ERR_CUDA 2     /* CUDA runtime error (reference: CUDA_CHECK throws) */
#define LSDEM_ERR_NOMEM 3    /* device allocation failed */
#define LSDEM_ERR_STATE 4    /* call out of order (e.g. step before initialize) */
#define LSDEM_ERR_NODEVICE 5 /* no usable CUDA device (reference: exit(1)) */

/* Compatibility switches (lsdem_set_flags). Both quirks of the reference are
 * kept by default; setting a bit replaces the quirk by the exact form. */
#define LSDEM_FIX_GRADIENT 1 /* x weight of the SDF gradient (LSParticleContactDetectionKernel.cuh:34-52) */
#define LSDEM_FIX_SQRTF 2    /* FP64 sqrt in the damping terms (contactKernel.cuh:51,53,58) */

/* Contact list kinds for lsdem_get_contacts / lsdem_count_contacts. */
#define LSDEM_CONTACT_PARTICLE 0 /* particle-particle (LSSolver.h:706-763) */
#define LSDEM_CONTACT_WALL 1     /* particle-wall (LSSolver.h:765-822) */
#define LSDEM_CONTACT_GHOST 2    /* particle-periodic image (PeriodicBoundary.h:75-141) */

typedef struct lsdem_solver lsdem_solver;

/* External force hook, called exactly once per step after the contact and
 * bond forces and before the second half kick, with the simulation time of the
 * step. Replaces the virtual LSSolver::addExternalForceTorque (LSSolver.h:508).
 * Kernels it launches on the solver's stream (or the legacy default stream
 * when the solver uses it) see the step's forces. With a hook, lsdem_step reads
 * each step's capacity status before the hook runs (one host synchronisation per
 * step, as the reference's per-step reads); a step whose lists overflowed is re-run
 * with grown capacities before its hook is called, so no step's hook runs twice. */
typedef void (*lsdem_hook)(void* user, double time);

/* Solver lifetime. Replaces LSSolver(dir, stream, maxGPUThread, device) (LSSolver.h:14).
 * `stream` is a cudaStream_t (NULL: legacy default stream, as the reference).
 * No device work happens before lsdem_initialize. */
int lsdem_create(int device, void* stream, lsdem_solver** out);
void lsdem_destroy(lsdem_solver* s);
const char* lsdem_last_error(const lsdem_solver* s);
int lsdem_set_flags(lsdem_solver* s, int flags);

/* Mass, centroid, inertia and inverse inertia of a level-set body by smoothed
 * Heaviside integration of its SDF grid (LSSolver.h:66-135). out[16] = mass,
 * centroid(3), inertia(6), inverse inertia(6). Host only; needs no device. */
int lsdem_mass_properties(const double* sdf, const int* size3, const double* origin3, double spacing,
                          double density, double* out16);
/* The same integrals computed on `device` as parallel sums over the grid nodes (the
 * summation order differs from the host loop's: agreement to rounding, relative 1e-12
 * in the tests); reproducible run to run. For large grids and many templates. */
int lsdem_mass_properties_gpu(const double* sdf, const int* size3, const double* origin3, double spacing,
                              double density, double* out16, int device);

/* Grid box of a level-set grid built around a triangle mesh with the given
 * spacing and padding layers: the vertices' bounding box grown by max(1, pad)
 * spacings, snapped outward to multiples of the spacing
 * (LevelSetObject::Base::buildGrid, FunDEM/kernel/helper/LevelSetObjectGenerator.h:122-170).
 * Host only. */
int lsdem_mesh_grid_box(const double* verts, int n_verts, double spacing, int pad, double* origin3, int* size3);

/* Level-set grid of a closed triangle mesh, computed on `device`: at every grid
 * node the distance to the nearest triangle, negative inside by the solid-angle
 * sum, divided by the gradient norm as buildGrid does (-+h/2 where that is
 * <= 1e-12) — LevelSetObject::Base::buildGrid over
 * TriangleMeshParticle::evaluateImplicitFunctionValueAndGradient
 * (LevelSetObjectGenerator.h:122-224, 454-500, 758-802, 888-914).
 * positive_inside = TriangleMeshParticle::setLevelSetPositiveInside. verts: n_verts
 * x 3, tris: n_tris x 3 vertex indices, sdf_out: size3[0] x size3[1] x size3[2]
 * values in the order ix + nx (iy + ny iz), host memory; blocking. LSDEM_ERR_ARG
 * for a mesh the reference's isValid rejects (no vertices or triangles, an index
 * out of range or repeated within a triangle). */
int lsdem_mesh_grid(const double* verts, int n_verts, const int* tris, int n_tris, const double* origin3,
                    const int* size3, double spacing, int positive_inside, double* sdf_out, int device);

/* Registers a shape template (surface nodes in the body frame + SDF grid with
 * index ix + nx*(iy + ny*iz), phi < 0 inside). Identical templates are shared.
 * Replaces the per-particle copies appended by LSParticle::add (LSParticle.h:115-212). */
int lsdem_add_shape(lsdem_solver* s, const double* nodes, int n_nodes, const double* sdf, const int* size3,
                    const double* origin3, double spacing, int* shape_id);

/* Appends n particles of registered shapes with explicit inverse mass and
 * body-frame inverse inertia (LSSolver.h:190-223 + LSParticle::add). `scale`
 * (nullable) uniformly scales the template (nodes, grid, SDF values).
 * Quaternions are normalised, kn/ks/mu clamped at 0, restitution outside
 * (0, 1] set to 1 (LSParticle.h:193-202). `first_index` (nullable) receives
 * the index of the first new particle. */
int lsdem_add_particles(lsdem_solver* s, int n, const int* shape, const double* scale, const double* pos,
                        const double* vel, const double* angvel, const double* quat, const double* inv_mass,
                        const double* inv_inertia6, const double* kn, const double* ks, const double* mu,
                        const double* e, int* first_index);

/* One particle with mass and inertia from the SDF and density, frame moved to
 * the centroid: LSSolver::addLSParticle (LSSolver.h:51-163). */
int lsdem_add_ls_particle(lsdem_solver* s, const double* nodes, int n_nodes, const double* sdf, const int* size3,
                          const double* origin3, double spacing, const double* pos, const double* vel,
                          const double* angvel, const double* quat, double kn, double ks, double mu, double e,
                          double density, int* index);

/* A fixed level-set wall (LSSolver::addWall, LSSolver.h:245-272). */
int lsdem_add_wall(lsdem_solver* s, const double* verts, int n_verts, const double* sdf, const int* size3,
                   const double* origin3, double spacing, const double* pos, const double* quat, double mu, double e,
                   int* index);
/* LSSolver::moveLSParticle / moveWall / setFixedVelocityToWall / setFixedAngularVelocityToWall (LSSolver.h:280-320). */
int lsdem_move_particle(lsdem_solver* s, int index, const double* offset3);
int lsdem_move_wall(lsdem_solver* s, int index, const double* offset3);
int lsdem_set_wall_velocity(lsdem_solver* s, int index, const double* v3);
int lsdem_set_wall_angular_velocity(lsdem_solver* s, int index, const double* w3);

/* V-bond between two particles (LSSolver::addBondedInteraction, LSSolver.h:344-379;
 * VBondedInteraction::add, VBondedInteraction.h:74-195). */
int lsdem_add_bond(lsdem_solver* s, int master, int slave, const double* point3, const double* normal3,
                   double radius, double initial_length, double youngs, double poisson, double tensile,
                   double cohesion, double mu);
/* Bonds from the current particle-particle contacts (LSSolver::createBondsFromContacts, LSSolver.h:385-418). */
int lsdem_create_bonds_from_contacts(lsdem_solver* s, double radius, double initial_length, double youngs,
                                     double poisson, double tensile, double cohesion, double mu);

/* Arithmetic form of the narrowphase and contact forces (no counterpart in the
 * reference, which is FP64 throughout): LSDEM_PREC_FP64 (default, the reference's
 * arithmetic), LSDEM_PREC_FP32_FP16 / LSDEM_PREC_FP32_BF16 (FP32 geometry and contact
 * law on SDF templates stored as phi / spacing in FP16 / BF16; positions, quaternions,
 * integration and the tangential-spring history stay FP64). Takes effect at initialize. */
#define LSDEM_PREC_FP64 0
#define LSDEM_PREC_FP32_FP16 1
#define LSDEM_PREC_FP32_BF16 2
int lsdem_set_precision(lsdem_solver* s, int mode);

/* Periodic axes bit mask (bit 0 x, 1 y, 2 z). x and y follow
 * addPeriodicBoundaryXD/YD (LSSolver.h:426-447); z applies the same rule. 0 removes
 * periodicity (removePeriodicBoundary, LSSolver.h:459-464). LSDEM_PERIODIC_SECTOR
 * (alone) is the quarter-sector periodicity of addPeriodicBoundarySector
 * (LSSolver.h:448-452, PeriodicBoundary.h:313-420): about the z axis through the
 * domain minimum, particles leaving across x = min.x or y = min.y are turned by
 * -/+90 degrees, images turned by 90, 180 and 270 degrees (contact image codes 8, 16,
 * 32). Combined with x/y/z bits: LSDEM_ERR_ARG. */
#define LSDEM_PERIODIC_SECTOR 8
int lsdem_set_periodic(lsdem_solver* s, int axes);

/* Uploads the model and builds the grids for the domain [min, max)
 * (LSSolver::upload + checkSolverInput, LSSolver.h:566-623). Called again after
 * steps (a new solve() phase), it starts from the current state with the host-side
 * edits made since (moves, wall velocities, new bodies or bonds), keeps the last
 * step's forces for the first half kick and, while the bodies, their surface nodes and
 * the periodic image sets are unchanged, the contact history (the reference keeps its
 * contact arrays, SolidInteraction.h:24-27); the simulation time restarts at 0, as each
 * of the reference's phases (LSSolver.h:994-996). */
int lsdem_initialize(lsdem_solver* s, const double* min3, const double* max3, const double* gravity3);

/* Advances nsteps time steps of size dt (loop body of LSSolver::compute*, LSSolver.h:1000-1128):
 * half kick, drift, hash, narrowphase + contact forces, periodic images, bonds,
 * hook, half kick. No host synchronisation inside a batch of steps. */
int lsdem_step(lsdem_solver* s, double dt, long long nsteps, lsdem_hook hook, void* user);

/* When on, the last step of every lsdem_step call also records contact point,
 * normal, overlap and elastic energies (needed for output and bond creation). */
int lsdem_set_record_contacts(lsdem_solver* s, int on);
/* Capacities: per-particle candidate slots (particles, walls, ghosts), contact
 * list, steps per batch. Values <= 0 keep the current setting. */
int lsdem_set_capacity(lsdem_solver* s, int pp_slots, int wall_slots, int ghost_slots, long long contacts,
                       int batch_steps);

/* Sizes: 0 particles, 1 walls, 2 bonds, 3 surface nodes, 4 shapes, 5 grid cells,
 * 6 steps taken, 7 overflow re-runs so far, 8 kernels launched by steps so far,
 * 9 steps that sorted the cells and rebuilt the neighbour lists (counted while
 * lsdem_set_neighbour_lists is on). */
long long lsdem_num(const lsdem_solver* s, int what);
double lsdem_time(const lsdem_solver* s);

/* Particle state in particle order (nullable outputs are skipped). Synchronous. */
int lsdem_get_state(lsdem_solver* s, double* pos, double* vel, double* angvel, double* quat, double* force,
                    double* torque);
int lsdem_get_wall_state(lsdem_solver* s, double* pos, double* vel, double* angvel, double* quat);
/* Overwrites particle state on the device (history is kept). */
int lsdem_set_state(lsdem_solver* s, const double* pos, const double* vel, const double* angvel, const double* quat);
/* Per-particle constants: inverse mass, body-frame inverse inertia (6), radius,
 * kn, ks, mu, e, shape id, scale, grid origin (3), inverse grid spacing, first node id. */
int lsdem_get_particle_params(const lsdem_solver* s, double* inv_mass, double* inv_inertia6, double* radius,
                              double* kn, double* ks, double* mu, double* e, int* shape, double* scale,
                              double* origin3, double* invh, long long* node_base);
int lsdem_get_wall_params(const lsdem_solver* s, double* radius, double* mu, double* e, int* shape, double* origin3,
                          double* invh);
/* Shape template in the caller's node order. */
int lsdem_get_shape(const lsdem_solver* s, int shape, double* nodes, double* sdf, int* size3, double* origin3,
                    double* spacing, int* n_nodes);

/* Broadphase of the last step: particle cell keys (-1 outside), stable sorted
 * particle index and key, per-cell [start, end) or -1 (launchUpdateSpatialGridHashStartEnd,
 * mySpatialGrid.h:33-49 / buildHashStartEnd.h). Grid: min, max, inverse cell size, cell counts.
 * With neighbour lists on (lsdem_set_neighbour_lists), lsdem_get_hash sorts the last step's
 * keys when called, and the next step rebuilds the lists. */
int lsdem_get_grid(const lsdem_solver* s, double* min3, double* max3, double* inv3, int* size3);
int lsdem_get_wall_grid(const lsdem_solver* s, double* min3, double* max3, double* inv3, int* size3);
int lsdem_get_hash(lsdem_solver* s, int* key, int* sorted_idx, int* sorted_key, int* cell_start, int* cell_end);

/* Contacts of the last step of one kind: global surface-node id, partner index
 * (particle, wall, or the particle whose image was hit), image set (ghosts),
 * tangential spring; geometry when recorded (nullable outputs skipped).
 * Order: by owner particle, candidate slot, node. */
int lsdem_count_contacts(lsdem_solver* s, int kind, long long* n);
int lsdem_get_contacts(lsdem_solver* s, int kind, long long cap, long long* node, int* partner, int* image,
                       double* spring, double* point, double* normal, double* overlap, double* en_n, double* en_s);

/* Bond state: master/slave ids, bonded flag, Un, Us, Ub, Ut, max normal and
 * shear stress, bond point (addBondedForceTorqueKernel outputs). */
int lsdem_get_bonds(lsdem_solver* s, int* ids2, int* bonded, double* state9);
/* The constants of every bond as added (no counterpart in the reference, whose
 * VBondedInteraction keeps them in its host mirrors, VBondedInteraction.h:74-195):
 * B[4] stiffness coefficients, geo[5] radius, initial length, tensile strength,
 * cohesion, friction coefficient, frames[24] master n1, n2, n3, local point, slave
 * n1, n2, n3, local point. Any pointer may be NULL. */
int lsdem_get_bond_params(lsdem_solver* s, double* B4, double* geo5, double* frames24);

/* Device pointers (double3 arrays in particle order, AoS) for external-force
 * kernels: what LSParticle::force()/torque()/velocity()/angularVelocity()
 * return to the reference's apps (LSParticle.h:665-669). Valid after initialize. */
int lsdem_device_pointers(lsdem_solver* s, void** force, void** torque, void** vel, void** angvel, void** pos,
                          void** quat);
/* The solver's CUDA stream (cudaStream_t). */
void* lsdem_stream(const lsdem_solver* s);

/* Device timing of the step phases with CUDA events on the solver stream
 * (no counterpart in the reference, which has no timers). Phases: 0 kick+drift+keys,
 * 1 cell sort, 2 candidates, 3 particle/wall narrowphase + forces (precision forms:
 * the FP32 screen), 4 periodic wrap + ghost images + ghost candidates, 5 ghost
 * narrowphase + forces (precision forms: the screen), 6 bonds, 7 second half kick,
 * 8 precision forms: FP64 contact pass of both narrowphases (learned form: with the
 * compaction of the network's survivors), 9 whole steps (step timing, below), 10
 * learned form: the network passes on the tensor cores. ms and calls hold
 * LSDEM_NUM_PHASES entries. Enabling resets the totals of every phase but 9. */
#define LSDEM_NUM_PHASES 11
int lsdem_set_profiling(lsdem_solver* s, int on);
int lsdem_get_profile(const lsdem_solver* s, double* ms, long long* calls);
/* Benchmark support (no counterpart in the reference): when on, every step is
 * bracketed by CUDA events on the solver stream (profile phase 9; the state backup
 * of each batch of steps is timed with the batch's first step), and when
 * l2_flush_bytes > 0 a scratch buffer of that size is written before each step,
 * outside the events, so that no step starts with data left in L2 by the one
 * before. Resets the phase-9 totals. */
int lsdem_set_step_timing(lsdem_solver* s, int on, long long l2_flush_bytes);
/* Work counts of the last step: candidate pairs (particle, wall, ghost) and contacts. */
int lsdem_step_stats(lsdem_solver* s, long long* out4);
/* Precision forms: counters of the FP32 screen summed over all steps run while
 * enabled (no counterpart in the reference): pairs screened, clusters tested,
 * clusters kept by the culls, 16-bit grid lookups of nodes, node tests, nodes
 * queued for the FP64 test, network evaluations of nodes (learned SDF), 8-node
 * sub-clusters kept.
 * Enabling resets them; off by default. */
int lsdem_set_screen_stats(lsdem_solver* s, int on);
int lsdem_get_screen_stats(lsdem_solver* s, long long* out8);
/* Precision forms without the network: of the screen's queued nodes, those of particle,
 * wall and image pairs (out3), summed like lsdem_get_screen_stats (no counterpart in the
 * reference). */
int lsdem_get_screen_queue(lsdem_solver* s, long long* out3);

/* Learned per-shape SDF (no counterpart in the reference). After lsdem_initialize,
 * trains one 3-64-64-1 SiLU network per shape template on the GPU (own forward,
 * backward and Adam kernels; FP32 master weights) on `samples` points of the
 * template's grid box (half uniform, half near the surface) with FP64 grid targets,
 * `iterations` Adam steps of `batch` points (a multiple of 128) at learning rate lr
 * (cosine schedule), then measures each network's largest error against the grid
 * over all grid nodes and `samples` further points, with the BF16 tensor-core
 * inference code of the narrowphase. loss_out[shape]: mean squared error of
 * phi / R of the last batch (R: half the largest grid extent); err_out[shape]: the
 * measured bound (template units). Either may be NULL. */
int lsdem_train_learned_sdf(lsdem_solver* s, int iterations, int batch, int samples, double lr,
                            unsigned long long seed, double* loss_out, double* err_out);
/* Training options of the learned SDF (no counterpart in the reference), before
 * lsdem_train_learned_sdf: the target phi / R is clipped to [clip_lo, clip_hi]
 * (defaults -0.25, 0.5; the one-sided error is measured against the clipped value,
 * so clip_lo <= -0.05 and clip_hi >= 0.1 keep the trust band inside the range), and
 * near_fraction (default 0.5) of the samples are drawn near the surface, the rest
 * uniform in the grid box. LSDEM_ERR_ARG outside those ranges. */
int lsdem_set_learned_training(lsdem_solver* s, double clip_lo, double clip_hi, double near_fraction);
/* Precision forms: when on, the screen rejects a node by the network where
 * phi_net exceeds the trust band delta (2 % of the shape size) plus 1.25 x the
 * measured one-sided error max(phi_net - phi_grid) over the validation points with
 * phi_grid <= delta; every other node goes on to the grid screen and the FP64 test.
 * Nodes of 8-node sub-clusters whose grid estimate of phi lies below that threshold
 * skip the network and take the grid test directly. */
int lsdem_set_learned_sdf(lsdem_solver* s, int on);
/* FP32 weights of a shape's network (LSDEM_MLP_PARAMS floats: W1[64][3], b1[64],
 * W2[64][64], b2[64], w3[64], b3, padding) and norm[8] = centre xyz, R, measured
 * error max |phi_net - phi_grid|, network threshold in template spacings, one-sided
 * error inside the trust band, trust band (template units). */
#define LSDEM_MLP_PARAMS 4484
int lsdem_get_learned_sdf(lsdem_solver* s, int shape, float* params, float* norm);
/* The network of `shape` at n template-frame points (double xyz), through the
 * narrowphase's inference code: phi in template units. */
int lsdem_mlp_eval(lsdem_solver* s, int shape, int n, const double* pts, float* phi);
/* Gradient check support: loss (mean squared error) and its gradient with respect
 * to the LSDEM_MLP_PARAMS weights over n points (n a multiple of 128; pts: x, y, z,
 * target per point), computed by the training kernel on `device`; y (optional):
 * the FP32 forward output per point. */
int lsdem_mlp_gradient(int device, int n, const float* params, const float* pts, float* loss, float* grad, float* y);

/* Scene set-up helper: random sequential addition of spheres (in the given
 * order) in [lo, hi), periodic or not (the reference's sphere-packing helper,
 * FunDEM/kernel/helper/SpherePackingGenerator.h:75-217, does the same job on the host).
 * keep (nullable): spheres with keep[i] != 0 stay at pos_out[i] and are placed around. */
int lsdem_pack_rsa(int n, const double* radius, const double* lo, const double* hi, int periodic,
                   unsigned long long seed, int max_tries, const int* keep, double* pos_out);

/* Triangles of a body's nodes (kind 0: particle, its surface nodes in the order
 * given at insertion; kind 1: wall, its vertices), kept for the mesh files of
 * lsdem_write_vtu: the boundaryNodeConnectivity / objTriangleVertexID argument of
 * LSParticle::add (FunDEM/kernel/LSParticle.h:165-172) through addLSParticle and
 * addWall (LSSolver.h:51-65, 245-254). tris: n_tris x 3 node indices of that body;
 * n_tris = 0 clears them. Host only. */
int lsdem_set_triangles(lsdem_solver* s, int kind, int index, const int* tris, int n_tris);

/* One output frame: the VTU files of LSSolver::output (LSSolver.h:637-665) under
 * the phase directory `dir`, with the reference's file names, layout, array
 * names and types (inline base64 binary, UInt64 headers):
 *   dir/LSParticle/LSObjectMesh_NNNN.vtu   surface nodes (world position,
 *       particleID, velocity) and their triangles (LSParticle.h:311-506);
 *   dir/LSParticle/Particle_NNNN.vtu       particle centres, velocity, angular
 *       velocity, orientation, radius (LSParticle.h:508-654);
 *   dir/LSParticleInteraction/LSInteraction_NNNN.vtu   particle contacts
 *       (SolidInteraction.h:154-317);
 *   dir/LSParticleInteraction/VBondedInteraction_NNNN.vtu   bonds, when there are
 *       any (VBondedInteraction.h:262-448);
 *   dir/Wall/LSObjectMesh_NNNN.vtu         wall vertices and triangles;
 *   dir/LSParticle-WallInteraction/LSInteraction_NNNN.vtu  wall contacts.
 * Arrays are computed and base64-encoded on the device in chunks of 32 MB, the
 * encoded chunks copied through two pinned buffers while the previous chunk is
 * written. Contacts need recorded geometry (lsdem_set_record_contacts). Returns
 * when the files are written; the solver's stream is ordered before the writer. */
int lsdem_write_vtu(lsdem_solver* s, const char* dir, unsigned long long frame, unsigned long long step,
                    double time);

/* Steps without profiling or contact recording are replayed from a CUDA graph of
 * the step's launches up to the external-force hook (captured once per history
 * parity and re-captured when the step's arguments change; on the legacy default
 * stream the replay runs on a private blocking stream, ordered with it both ways);
 * the hook and the second half kick follow the replay. on = 0 launches every kernel
 * of every step instead. Default on. No counterpart in the reference (which
 * launches each kernel and synchronises with the host every step). */
int lsdem_set_graphs(lsdem_solver* s, int on);

/* Neighbour lists (exact; default on): the candidate search tests, per particle, the
 * bodies it found within its reach plus a margin (a tenth of the largest bounding
 * radius) at the last rebuild, keeping those whose cell is in its cell window and
 * which pass the same bounding-sphere test, in the walk's order. The cell sort and the
 * rebuild run only in steps where a particle moved 0.04 of the largest bounding
 * radius since the last rebuild (a periodic wrap included). The candidate pairs,
 * their order and so every result are the same as with on = 0, which sorts and walks
 * the 27 cells every step as the reference does (LSSolver.h:1000-1011,
 * mySpatialGrid.cu, LSParticleContactDetectionKernel.cu). */
int lsdem_set_neighbour_lists(lsdem_solver* s, int on);

/* Snapshot of the dynamic state (no counterpart in the reference, which writes its
 * state only as VTU frames): particle position, velocity, angular velocity,
 * orientation, force and torque, wall pose and velocities, bond flags and state, the
 * contact history of the last step (candidate slots, contact nodes and FP64 springs),
 * time and step count, in one binary file. lsdem_snapshot_load restores it into a
 * solver initialized with the same bodies, surface nodes, bonds and image sets
 * (LSDEM_ERR_ARG otherwise), growing capacities to the file's; the steps that follow
 * are those the saved solver would have taken. Both need lsdem_initialize first. */
int lsdem_snapshot_save(lsdem_solver* s, const char* path);
int lsdem_snapshot_load(lsdem_solver* s, const char* path);

/* Broadphase cell sort that allocates no device memory: cell keys of n body
 * centres (pos_dev: device array of n x 3 doubles), their stable sorted order
 * and per-cell [start, end) (-1 when empty) for the grid (min, max, inverse
 * cell size, cell counts), written to caller-provided device arrays
 * (sorted_key_dev may be NULL) on `stream` (a cudaStream_t, NULL = legacy default).
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory when they call in (latency-critical loops in which an allocation
 * may block or synchronise, hosts whose device memory belongs to their own pool
 * or fixed budget). Its scratch is one fixed device array of the library, which
 * limits a call to 262,144 bodies and 262,144 cells (LSDEM_ERR_ARG beyond, with
 * a message on stderr). The first call on a device looks up that array's device
 * address, so it should come before any stream capture; that address is kept
 * for the life of the process, so the entry point must not be used on a device
 * again after cudaDeviceReset. All calls share the array; calls that overlap on
 * the GPU race. */
int lsdem_cell_sort_static(const void* pos_dev, int n, const double* min3, const double* max3, const double* inv3,
                           const int* size3, int* key_dev, int* sorted_idx_dev, int* sorted_key_dev,
                           int* cell_start_dev, int* cell_end_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif
