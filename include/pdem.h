/* peclet-dem B200 substep: C ABI.
 *
 * Drop-in boundary for the reference's `peclet.dem.Simulation` (nanobind module `_dem`,
 * src/dem_bindings.cpp:51-464, facade src/sim.hpp:909-1670). Every entry point takes a handle, plain
 * host pointers and sizes, returns an int status (PDEM_OK or an error code, message from
 * pdem_last_error()) and never throws across the ABI. Host arrays are double precision; the handle's
 * precision (64: FP64 step, 32: the reference's float arithmetic) decides what the device computes.
 * Getters return the number of values available (which may exceed `cap`; only `cap` are written).
 *
 * Each declaration cites the reference interface it replaces (file:line).
 */
#ifndef PDEM_H
#define PDEM_H

#ifdef __cplusplus
extern "C" {
#endif

#define PDEM_MIXED 3264 /* pdem_create precision: FP32 step with FP64 master positions/orientations */
#define PDEM_OK 0
#define PDEM_ERR_RUNTIME 1     /* std::runtime_error in the reference  -> RuntimeError */
#define PDEM_ERR_INVALID 2     /* std::invalid_argument in the reference -> ValueError  */
#define PDEM_ERR_UNSUPPORTED 3 /* a mode this build does not provide                     */
#define PDEM_ERR_CUDA 4        /* CUDA runtime failure (no device, out of memory, ...)   */

typedef void* pdem_handle;

/* last error message of this thread */
const char* pdem_last_error(void);
/* "CUDA sm_100a" and the device name; for diagnostics */
const char* pdem_execution_space(void);

/* select the CUDA device later pdem_create calls of this thread use (one process per GPU); the
 * reference runs on Kokkos' default device, src/dem_bindings.cpp:54-55 */
int pdem_set_device(int device);

/* Simulation(capacity)                         src/dem_bindings.cpp:72, src/sim.hpp:911-916
 * precision: 64 = FP64 step (the drop-in), 32 = the reference's float arithmetic,
 * PDEM_MIXED = float step whose positions and orientations are kept and returned in FP64 */
int pdem_create(int capacity, int precision, pdem_handle* out);
void pdem_destroy(pdem_handle h);

/* initialize_shape / initialize / set_sphere_shape   src/dem_bindings.cpp:73-80, src/sim.hpp:949-1021 */
int pdem_initialize_shape(pdem_handle h, int shape_type, double radius, double height, double thickness);
/* set_sdf_shape                                 src/dem_bindings.cpp:86-103, src/sim.hpp:1034-1084 */
int pdem_set_sdf_shape(pdem_handle h, const double* grid, int nx, int ny, int nz, const double* origin,
                       const double* spacing, const double* shell, int nshell, const double* inv_inertia,
                       double bounding_radius);
/* extension: replace the active shape's surface point shell (keeps its analytic SDF)          */
int pdem_set_shell_points(pdem_handle h, const double* pts, int n);
/* set_domain(lx,ly,lz,px,py,pz)                 src/dem_bindings.cpp:104-106, src/sim.hpp:1086-1089 */
int pdem_set_domain(pdem_handle h, double lx, double ly, double lz, int px, int py, int pz);
/* set_domain(min, max)                          src/dem_bindings.cpp:109-118, src/sim.hpp:1091-1099 */
int pdem_set_domain_minmax(pdem_handle h, const double* mn, const double* mx);
/* enable_periodicity                            src/dem_bindings.cpp:119, src/sim.hpp:1100-1104 */
int pdem_enable_periodicity(pdem_handle h, int x, int y, int z);
/* set_gravity                                   src/dem_bindings.cpp:125, src/sim.hpp:1111 */
int pdem_set_gravity(pdem_handle h, double gx, double gy, double gz);
/* set_thermostat                                src/dem_bindings.cpp:127, src/sim.hpp:1112-1116 */
int pdem_set_thermostat(pdem_handle h, double temperature, double tau, double kB);
/* set_solver_iterations                         src/dem_bindings.cpp:130, src/sim.hpp:1117-1120 */
int pdem_set_solver_iterations(pdem_handle h, int pos, int vel);
/* set_velocity_use_gs                           src/dem_bindings.cpp:154, src/sim.hpp:1123 */
int pdem_set_velocity_use_gs(pdem_handle h, int use_gs);
/* set_stabilization / set_stabilization_mode    src/dem_bindings.cpp:142-153, src/sim.hpp:1128-1150 */
int pdem_set_stabilization_mode(pdem_handle h, const char* mode);
/* set_hertz_material                            src/dem_bindings.cpp:132, src/sim.hpp:1153-1164 */
int pdem_set_hertz_material(pdem_handle h, int mat, double youngs, double poisson);
/* set_global_scale                              src/dem_bindings.cpp:157, src/sim.hpp:1171-1174 */
int pdem_set_global_scale(pdem_handle h, double s);
/* set_dt                                        src/dem_bindings.cpp:159, src/sim.hpp:1175 */
int pdem_set_dt(pdem_handle h, double dt);
/* set_material_params                           src/dem_bindings.cpp:160, src/sim.hpp:1179-1183 */
int pdem_set_material_params(pdem_handle h, double restitution_normal, double restitution_tangent,
                             double friction);
/* set_material_ids                              src/dem_bindings.cpp:163, src/sim.hpp:1187-1193 */
int pdem_set_material_ids(pdem_handle h, const int* ids, int n);
/* set_pair_material                             src/dem_bindings.cpp:166, src/sim.hpp:1196-1216 */
int pdem_set_pair_material(pdem_handle h, int a, int b, double restitution, double friction);
/* set_wall_material_id                          src/dem_bindings.cpp:170, src/sim.hpp:1218-1225 */
int pdem_set_wall_material_id(pdem_handle h, int wid, int mat);
/* add_plane (both overloads)                    src/dem_bindings.cpp:173-183, src/sim.hpp:1226-1232 */
int pdem_add_plane(pdem_handle h, double px, double py, double pz, double nx, double ny, double nz);
/* add_sdf_wall                                  src/dem_bindings.cpp:190-205, src/sim.hpp:1242-1274 */
int pdem_add_sdf_wall(pdem_handle h, const double* grid, int nx, int ny, int nz, const double* origin,
                      const double* spacing, double restitution, double friction, int* out_index);
/* set_wall_velocity                             src/dem_bindings.cpp:208-223, src/sim.hpp:1280-1287 */
int pdem_set_wall_velocity(pdem_handle h, int index, const double* lin_vel, const double* ang_vel,
                           const double* center);
/* set_positions (N,3)                           src/dem_bindings.cpp:225-251, src/sim.hpp:1290-1330 */
int pdem_set_positions(pdem_handle h, const double* xyz, int n);
/* set_velocities / set_external_forces / clear_external_forces / set_quaternions /
 * set_angular_velocities / set_inv_inertia / set_inv_mass     src/dem_bindings.cpp:252-288,
 *                                                             src/sim.hpp:1347-1405 */
int pdem_set_velocities(pdem_handle h, const double* v, int n);
int pdem_set_external_forces(pdem_handle h, const double* f, int n);
int pdem_clear_external_forces(pdem_handle h);
int pdem_set_quaternions(pdem_handle h, const double* q, int n);
int pdem_set_angular_velocities(pdem_handle h, const double* w, int n);
int pdem_set_inv_inertia(pdem_handle h, const double* ii, int n);
int pdem_set_inv_mass(pdem_handle h, const double* im, int n);
/* set_scales / set_scales_uniform / set_growth_params / get_growth_factor / get_growth_rate
 *                                               src/dem_bindings.cpp:291-305, src/sim.hpp:1331-1426 */
int pdem_set_scales(pdem_handle h, const double* s, int n);
int pdem_set_scales_uniform(pdem_handle h, double s);
int pdem_set_growth_params(pdem_handle h, double rate, double new_factor);
double pdem_get_growth_factor(pdem_handle h);
double pdem_get_growth_rate(pdem_handle h);
/* get_positions / velocities / quaternions / angular_velocities / inv_inertia / scales / masses
 *                                               src/dem_bindings.cpp:289-346, src/sim.hpp:1406-1452 */
long pdem_get_positions(pdem_handle h, double* out, long cap);
long pdem_get_velocities(pdem_handle h, double* out, long cap);
long pdem_get_quaternions(pdem_handle h, double* out, long cap);
long pdem_get_angular_velocities(pdem_handle h, double* out, long cap);
long pdem_get_inv_inertia(pdem_handle h, double* out, long cap);
long pdem_get_scales(pdem_handle h, double* out, long cap);
long pdem_get_masses(pdem_handle h, double* out, long cap);
/* step(dt): ONE XPBD substep                    src/dem_bindings.cpp:342, src/sim.hpp:1456-1459,97-488 */
int pdem_step(pdem_handle h, double dt);
/* n substeps in one call (the caller's substep loop moved across the boundary; each substep is
 * exactly pdem_step, and the step's own host reads stay, so this is not a captured graph) */
int pdem_step_n(pdem_handle h, double dt, int n);
/* the last substep's counters: candidate pairs P, contacts C, manifolds M, colours of the two
 * colourings K, velocity / stabilization / position sweeps I_v / I_s / I_p, the error bits of
 * bounded device loops (0 = none), the maximum overlap, and the Jones-Plassmann rounds of the two
 * colourings */
typedef struct {
  long pairs, contacts, manifolds;
  int colors_velocity, colors_position;
  int velocity_sweeps, stabilization_sweeps, position_sweeps;
  int status;
  double max_overlap;
  int color_rounds_velocity, color_rounds_position;
} pdem_counters_t;
int pdem_counters(pdem_handle h, pdem_counters_t* out);
/* step_hertz(dt, substeps, skin_frac)           src/dem_bindings.cpp:139, src/sim.hpp:1167-1170,628-750 */
int pdem_step_hertz(pdem_handle h, double dt, int substeps, double skin_frac);
/* compute_overlaps                              src/dem_bindings.cpp:368, src/sim.hpp:1462,494-541 */
int pdem_compute_overlaps(pdem_handle h, double* out);
/* num_particles / num_contacts / num_manifolds / max_overlap (+ get_* aliases)
 *                                               src/dem_bindings.cpp:357-366, src/sim.hpp:1544-1556 */
int pdem_num_particles(pdem_handle h);
int pdem_num_contacts(pdem_handle h);
int pdem_num_manifolds(pdem_handle h);
double pdem_max_overlap(pdem_handle h);
/* export_lammps / write_vtp                     src/dem_bindings.cpp:355,369-371, src/sim.hpp:1466-1475,1560-1601 */
int pdem_export_lammps(pdem_handle h, const char* filename, int step);
int pdem_write_vtp(pdem_handle h, const char* filename);

/* ---- diagnostics: intermediate products of the last substep, canonical order ----
 * (the reference keeps them in its Particles SoA, src/particles.hpp:49-151, without a getter)
 * counts: pairs, contacts, manifolds, bodies incl. ghosts, ledger size, capacity, contact capacity,
 *         pair capacity
 * contacts: 17 doubles each (bodyA bodyB n[3] rA[3] rB[3] dist lambdaN wallVel[3] restitution);
 *           contact_mu: the per-contact friction
 * manifolds: 23 doubles each (bodyA bodyB Nsum[3] TauA[3] TauB[3] rA[3] rB[3] points wallVel[3] e mu)
 * lambda: 4 doubles per manifold (normal accumulator, tangential accumulator[3])
 * ledger: committed sorted keys + 5 doubles (lambda, lambdaT[3], position impulse) */
int pdem_debug_counts(pdem_handle h, long* out8);
long pdem_debug_pairs(pdem_handle h, int* out, long cap);
long pdem_debug_contacts(pdem_handle h, double* out, long cap);
long pdem_debug_contact_mu(pdem_handle h, double* out, long cap);
long pdem_debug_manifolds(pdem_handle h, double* out, long cap);
long pdem_debug_manifold_colors(pdem_handle h, int* out, long cap);
long pdem_debug_contact_colors(pdem_handle h, int* out, long cap);
long pdem_debug_lambda(pdem_handle h, double* out, long cap);
long pdem_debug_pair_keys(pdem_handle h, unsigned long long* out, long cap);
long pdem_debug_ledger(pdem_handle h, unsigned long long* keys, double* vals, long cap);
long pdem_debug_grounded(pdem_handle h, int* out, long cap);
long pdem_debug_pos_lambda(pdem_handle h, double* out, long cap);
long pdem_debug_hertz(pdem_handle h, unsigned long long* keys, double* xi, long cap);
/* test hook: set the contact buffer capacity (overflow / clamp behaviour) */
int pdem_debug_set_max_contacts(pdem_handle h, int max_contacts);
/* test hook: polls before a grid-wide barrier wait of the persistent loops gives up (<= 0: the
 * default, seconds of waiting). A wait that gives up sets an error bit; the kernel returns, the
 * step reports PDEM_ERR_CUDA at its next read-back and clears the bit; the substep's state is then
 * partial and the caller sets the bodies' state again. Lets a test make the wait run out. */
int pdem_debug_set_barrier_spins(pdem_handle h, long spins);
/* the broadphase's own stable radix sort (the Morton sort of the LBVH build) on HOST arrays of n
 * (key, value) pairs, by the low end_bit bits of the keys (a test entry point: it allocates
 * device memory for the call and synchronises) */
int pdem_debug_radix_sort(const unsigned long long* keys, const int* vals, int n, int end_bit,
                          unsigned long long* out_keys, int* out_vals);

/* ---- batched form (no reference counterpart: the reference steps one scene per Simulation) ----
 * Several independent scenes share one simulation: scene s owns the bodies
 * [first_body[s], first_body[s+1]) of the arrays given to set_positions (call set_scenes after it;
 * first_body[0] = 0, first_body[nscenes] = particle count, at most 1023 scenes). Every scene is
 * stepped exactly as a simulation of that scene alone would step it: candidate pairs only inside
 * a scene, its own contact margin (0.1 x its largest radius), restitution and friction, walls and
 * adaptive iteration stops, and the colour priorities of its own indices. Scenes may overlap in
 * space. Shared: shape, global scale, gravity, iterations, dt, stabilization mode, planes (walls
 * with scene -1). Not supported: periodic domains, growth, thermostat, zero-gravity friction,
 * the Hertz engine. */
int pdem_set_scenes(pdem_handle h, int nscenes, const int* first_body);
int pdem_set_scene_material(pdem_handle h, int scene, double e_n, double mu);
/* the wall (index from add_sdf_wall) is met only by the bodies of `scene` (-1: by every scene) */
int pdem_set_wall_scene(pdem_handle h, int wall, int scene);
/* per scene, 5 values: max overlap, max approach, velocity / stabilization / position sweeps of
 * the last substep; returns the number of scenes (0 when not batched, -1 on error) */
long pdem_scene_counters(pdem_handle h, double* out, long cap);

/* ---- instrumentation (no reference counterpart; the reference's Kokkos labels serve Kokkos Tools) ----
 * profile_enable(1) resets and starts per-stage device timing (CUDA events between stage
 * boundaries of every step) and the count of this library's kernel launches; profile_read returns
 * the number of stages and fills per-stage milliseconds and call counts, in this order:
 * predict, ghosts, broadphase, narrowphase, manifolds, colour_velocity, warm_start, velocity,
 * stabilization, ledger, friction, integrate, colour_position, position, commit, hertz_pairs,
 * hertz_rebuild, hertz_integrate */
int pdem_profile_enable(pdem_handle h, int on);
int pdem_profile_read(pdem_handle h, double* ms, long* calls, int cap, long* launches);
/* host wall-clock milliseconds spent issuing each stage since profile_enable (same order): a stage
 * whose host time matches its device time is paced by the host (launches, read-backs) */
int pdem_profile_read_host(pdem_handle h, double* ms, int cap);
/* device-timeline interval: timer_start records an event on the simulation's stream, timer_stop
 * records another, waits for it and returns the milliseconds between them (everything the stream
 * ran, and any idle time, in between) */
int pdem_timer_start(pdem_handle h);
int pdem_timer_stop(pdem_handle h, double* ms);
/* substeps since profile_enable that kept the previous substep's manifold grouping, contact
 * colours and manifold colours (their lists were unchanged) */
int pdem_debug_reuse(pdem_handle h, long* out3);
/* substeps since profile_enable whose contact grouping took the rank scatter (the list in key
 * order up to its boundary contacts), and those of them whose list the scatter rejected (sorted) */
int pdem_debug_ranked(pdem_handle h, long* out2);
/* device allocations made by this library's growable buffers since it was loaded */
long pdem_debug_allocs(void);
/* sweeps executed since profile_enable: velocity, stabilization, position; and substeps */
int pdem_debug_sweeps(pdem_handle h, long* out4);

/* ---- candidate pairs without allocation (no counterpart in the reference) ----
 * The broadphase of the step (same predicate and canonical (i, j) order as the pair list that
 * pdem_compute_overlaps builds) over caller-owned DEVICE arrays: d_xyz (n x 3 doubles), d_radius (n
 * doubles); pairs go to d_pairs (pair_cap x 2 ints), their number to *out_count (when it exceeds
 * pair_cap nothing is written). All scratch is a fixed static device buffer: this call allocates
 * no device or pinned memory, so callers that own the whole device memory budget can use it.
 * n is at most 16384 (PDEM_ERR_INVALID above). The first call on a device does a one-time set-up
 * and should come before any stream capture; calls that overlap in time share the scratch and
 * race. Work is ordered on `stream` (a cudaStream_t, NULL = default stream); the call returns
 * after synchronising it. */
int pdem_find_pairs_static(const double* d_xyz, const double* d_radius, int n, double margin, double box_cap,
                           int* d_pairs, long pair_cap, long* out_count, void* stream);

/* get_domain_min / get_domain_max              src/dem_bindings.cpp:124-127, src/sim.hpp:1105-1110 */
int pdem_get_domain(pdem_handle h, double* mn, double* mx);
/* get_positions_view / get_velocities_view / get_external_forces_view / get_inv_mass_view
 *                                               src/dem_bindings.cpp:302-334
 * zero-copy device arrays: field 0 positions, 1 velocities, 2 external forces (writable: the step
 * reads it), 3 inverse mass. Returns the device pointer, the number of rows, the row stride in
 * elements (4: x, y, z and a pad; 1 for the inverse mass) and the element size (8 at FP64, 4 at
 * FP32 and in the mixed form, whose positions here are the float state). The stream is
 * synchronised first. Valid until a call that can grow the particle buffers. */
int pdem_device_view(pdem_handle h, int field, void** ptr, long* rows, int* row_stride, int* elem_bytes);
/* batched form: the block size the launch shape autotuner chose for the per-scene sweep loops
 * (0 while it is still trying the candidates 64, 128, 256, 512 over the first batched substeps;
 * the environment variable PDEM_SCENE_BLOCK fixes it instead) and the mean sweep-loop time of each
 * candidate in ms (cap values) */
int pdem_scene_block(pdem_handle h, int* block, double* ms, int cap);
/* batched form: the block size the autotuner chose for the colouring launch (0 while it is still
 * timing the candidates 256, 512, 1024 over the first batched colourings; PDEM_COLOR_BLOCK fixes it
 * instead) and each candidate's mean launch time in ms (cap values) */
int pdem_color_block(pdem_handle h, int* block, double* ms, int cap);
/* get_sdf_grid(resolution)                      src/dem_bindings.cpp:344-355, src/sim.hpp:1538-1542
 * packed-bed SDF over the domain (src/output_sdf.hpp:25-196), flat x-fastest; returns rx*ry*rz
 * (only cap written), or -1 with pdem_last_error() set */
long pdem_get_sdf_grid(pdem_handle h, int rx, int ry, int rz, double* out, long cap);
/* export_sdf(filename, resolution)              src/dem_bindings.cpp:369-376, src/sim.hpp:1478-1483 */
int pdem_export_sdf(pdem_handle h, const char* filename, int rx, int ry, int rz);

/* ---- forward, adjoint and tangent-linear runs of the Hertz-Mindlin substep for spheres (no
 * counterpart in the reference; the force law is the Hertz engine's, src/solver_hertz.hpp:88-144,
 * its kick-drift src/solver_hertz.hpp:374-425; planes are walls at rest with the same law) ----
 * All arrays are DEVICE arrays of the call's precision (32: float, 64: double) unless stated;
 * contacts are int pairs (i, j): j >= 0 the sphere j > i, j < 0 the plane -j - 1. A state block is
 * x, v, w (3 n each) then the history of every contact (3 each): pdem_hz_state_size values. The
 * contact list stays fixed over the substeps of one call. Work goes to `stream`; forward,
 * backward and jvp do not synchronise it. */
typedef struct {
  int n, ncontact, nplane;
  const int* contacts;  /* ncontact x (i, j) */
  const void* planes;   /* nplane x (point, unit normal into the domain) */
  const void* radius;       /* n */
  const void* inv_mass;     /* n: 1 / mass (0: fixed) */
  const void* inv_inertia;  /* n: 1 / scalar moment of inertia */
  double youngs, restitution, friction, poisson, dt, gravity[3];
} pdem_hz_model;
long pdem_hz_state_size(int n, int ncontact);
/* work buffer of forward, backward and jvp, in values of the precision */
long pdem_hz_work_size(int n, int ncontact);
/* candidate contacts per sphere i, in i order: the spheres i < j of i's scene (scenes are the
 * ranges [first[s], first[s + 1]), nscene + 1 ints from 0 to n, given on the HOST (first) and the
 * device (d_first) alike) with
 * |x_i - x_j| < r_i + r_j + skin, then the planes k with (x_i - p0_k).n_k < r_i + skin.
 * d_cnt n ints and d_off n + 1 ints of scratch; when the count exceeds cap nothing is written.
 * Synchronises the stream. */
int pdem_hz_contacts(int precision, const void* d_x, const void* d_radius, const int* first, const int* d_first,
                     int nscene, const void* d_planes, int nplane, double skin, int* d_cnt, int* d_off, int* d_contacts,
                     long cap, long* count, void* stream);
/* `steps` substeps from the state in block 0 of d_traj: store = 1 writes substep k to block k
 * (steps + 1 blocks), store = 0 ping-pongs blocks 0 and 1 and leaves the final state in block 1 */
int pdem_hz_forward(int precision, const pdem_hz_model* model, int steps, int store, void* d_traj, void* d_work,
                    void* stream);
/* reverse of a stored forward (steps + 1 blocks in d_traj): d_adj holds the adjoint of the final
 * state on entry and that of block 0 on return; gradients with respect to (E, e, mu) accumulate
 * into d_grad (3 doubles, device, not cleared). mode 0: hand reversal of each contact law;
 * mode 1: dual-number local Jacobians (the cross-check, slower) */
int pdem_hz_backward(int precision, const pdem_hz_model* model, int steps, const void* d_traj, void* d_adj,
                     double* d_grad, void* d_work, int mode, void* stream);
/* tangent-linear run: the state (2 blocks) and its tangent (2 blocks) advance `steps` substeps
 * from block 0 together, with the parameter tangent theta_dot (3 doubles, HOST: dE, de, dmu);
 * both end in block 1 */
int pdem_hz_jvp(int precision, const pdem_hz_model* model, int steps, void* d_state, void* d_tangent,
                const double* theta_dot, void* d_work, void* stream);

/* ---- adjoint of the XPBD substep (added form; no reference counterpart) ----
 * The plain FP64 step (pdem_step, src/sim.hpp:97-488) differentiated over a recorded rollout:
 * one scene of spheres without point shells, planes as walls, gravity on with the coloured
 * Gauss-Seidel (PGS) velocity solve, stabilization "off", "onesided" or "escalate", no periodicity, growth,
 * thermostat or pair materials; every entry coloured (no Jacobi leftovers). Other set-ups are
 * refused with PDEM_ERR_INVALID at pdem_xa_begin / pdem_xa_step. Rows are DEVICE doubles:
 * positions, velocities and angular velocities n x 3, quaternions n x 4 (x, y, z, w).
 * pdem_xa_begin sets the start state of a rollout (n = every particle), clears the warm-start
 * ledger, the support levels and the topology caches (a rollout is a function of its start
 * state and the material only) and starts a new record; pdem_xa_step runs `substeps` substeps
 * of pdem_step (dt <= 0: the current substep length), recording each one's start state, ledger
 * and frozen active set (contacts, manifolds, colourings, side flags, sweep counts);
 * pdem_xa_state returns the current state rows. pdem_xa_backward takes the adjoint of the
 * rollout's end state and returns the gradients with respect to its start state (rows as
 * above) and to (eN, eT, mu) of pdem_set_material_params (dtheta: 3 doubles, HOST); it replays
 * each substep from its record and reverses it, the sweeps in reverse colour and sweep order
 * over the frozen colouring. The backward uses the rollout's own substep length, material and
 * gravity; the masses, inertia, scales, external forces and planes must stay as they were during
 * the rollout until its backward. Synchronise the caller's stream before these calls; each returns
 * with the library's stream synchronised. pdem_xa_info: out[0] substeps recorded, out[1] bytes
 * of the record, out[2] bytes of the reverse workspace, out[3] the largest sweep count;
 * err[0] the largest deviation of a replayed substep's end positions from the recorded next
 * state over the last backward, in units of the global scale, err[1] the same for velocities
 * (m/s). */
int pdem_xa_begin(pdem_handle h, const double* x, const double* q, const double* v, const double* w, int n);
int pdem_xa_step(pdem_handle h, double dt, int substeps);
int pdem_xa_state(pdem_handle h, double* x, double* q, double* v, double* w);
int pdem_xa_backward(pdem_handle h, const double* gx, const double* gq, const double* gv, const double* gw,
                     double* dx, double* dq, double* dv, double* dw, double* dtheta);
int pdem_xa_info(pdem_handle h, long* out, double* err);
/* the record's discrete decisions, 7 longs per substep (contacts, manifolds, colours of the
 * velocity and position colourings, main, stabilization and position sweeps), at most cap values;
 * returns the number of substeps recorded (or -1 on error). Equal signatures of two rollouts mean
 * the same contact sets, colourings and adaptive stops (a certified finite difference). */
long pdem_xa_signature(pdem_handle h, long* out, long cap);
/* the branch signature of the record: every substep replayed (no reverse) and every sweep
 * update's branch decisions (normal impulse clamp, restitution cut-off, friction cone, active
 * position contact) hashed into *hash. With equal signatures (pdem_xa_signature) and equal branch
 * hashes, two rollouts ran the same smooth piece of the step: their central difference is a
 * certified check of the gradient. */
int pdem_xa_branches(pdem_handle h, unsigned long long* hash);

#ifdef __cplusplus
}
#endif
#endif /* PDEM_H */
