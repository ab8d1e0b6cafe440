/*
 * wake_gpu.h - C ABI of the B200 lattice-update library (libwake_b200.so).
 *
 * Two layers:
 *
 * 1. Drop-in kernel entry points. Same symbol names, parameter lists and
 *    meaning as the ISPC exports that the reference host declares in
 *    `namespace ispc { extern "C" { ... } }` (src/grid/lattice_grid_2d.cpp:8-42,
 *    src/grid/lattice_grid_3d.cpp:7-42, src/scenarios/karman_vortex.cpp:10-21,
 *    src/scenarios/sphere_3d_wake.cpp:10-21, src/thermal/thermal_solver.cpp:6-44).
 *    A build that links this library instead of the reference's
 *    wake_ispc_kernels static library runs the reference host unchanged.
 *    Pointers may be device memory (used in place) or ordinary host memory
 *    (staged through the device). Each call is synchronous, like the
 *    reference's, and returns void; failures are reported by
 *    wake_gpu_last_error() (the reference has no error channel).
 *    The ISPC `uniform float &` outputs of the momentum-exchange kernels are
 *    plain pointers here (identical calling convention).
 *
 * 2. The fused engine (wake_grid_*): one resident lattice per handle,
 *    advanced by one fused pull-stream + boundaries + moments +
 *    momentum-exchange + collide kernel per step. This is the fast path a
 *    GPU LatticeGrid2D/3D::step uses. Functions return 0 on success and a
 *    negative WAKE_ERR_* code on failure (message in wake_gpu_last_error()).
 */
#ifndef WAKE_GPU_H
#define WAKE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ errors */
#define WAKE_OK 0
#define WAKE_ERR_INVALID (-1)   /* bad argument, size or state */
#define WAKE_ERR_CUDA (-2)      /* CUDA runtime failure */
#define WAKE_ERR_NOMEM (-3)     /* device allocation failed */
#define WAKE_ERR_NUMERIC (-4)   /* non-finite or non-positive density seen on the device */

/* Last error of the calling thread ("" if none); cleared by wake_gpu_clear_error. */
const char* wake_gpu_last_error(void);
int wake_gpu_last_error_code(void);
void wake_gpu_clear_error(void);
/* Library version string. */
const char* wake_gpu_version(void);
/* Device blocks of destroyed grids and batches are kept for reuse instead of
 * being freed (cudaFree synchronises the whole device). trim frees every cached
 * block of the current device and returns the bytes freed; cache_bytes reports
 * what the cache holds. An allocation that fails trims the cache and retries. */
long long wake_gpu_cache_trim(void);
long long wake_gpu_cache_bytes(void);

/* ------------------------------------------------- drop-in kernel entry points */
/* D2Q9: src/ispc/d2q9_collision_bgk.ispc:5-16 */
void d2q9_collide_bgk(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau, float gx, float gy, int count);
/* src/ispc/d2q9_collision_trt.ispc:7-19 */
void d2q9_collide_trt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau_s, float tau_a, float gx, float gy, int count);
/* src/ispc/d2q9_collision_mrt.ispc:6-18 */
void d2q9_collide_mrt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                      float uy[], float tau_shear, float tau_bulk, float gx, float gy, int count);
/* src/ispc/d2q9_streaming.ispc:4-9 */
void d2q9_stream_periodic(const float f_src[], float f_dst[], int nx, int ny);
/* src/ispc/d2q9_streaming.ispc:33-41 */
void d2q9_stream_with_boundaries(const float f_src[], float f_dst[], const uint8_t cell_type[], int nx, int ny,
                                 float uw_x, float uw_y);
/* src/ispc/d2q9_boundaries.ispc:5-11 */
void d2q9_apply_bounce_back(float f[], const uint8_t cell_type[], float uw_x, float uw_y, int count);
/* src/ispc/d2q9_boundaries.ispc:43-52 */
void d2q9_apply_zou_he_inflow_west(float f[], float rho[], float ux[], float uy[], float u_in_x, float u_in_y,
                                   int nx, int ny);
/* src/ispc/d2q9_boundaries.ispc:85-93 */
void d2q9_apply_zou_he_outflow_east(float f[], float rho[], float ux[], float uy[], float rho_out, int nx, int ny);
/* src/ispc/d2q9_boundaries.ispc:125-131 */
void d2q9_apply_convective_outflow_east(float f[], const float f_prev[], float u_conv, int nx, int ny);
/* src/ispc/d2q9_les.ispc:6-15 */
void d2q9_compute_smagorinsky_tau(const float f[], const float rho[], const float ux[], const float uy[],
                                  float tau_eff[], float tau_0, float smagorinsky_constant, int count);
/* src/ispc/d2q9_moments.ispc:4-10, 35-43, 68-73 */
void d2q9_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], int count);
void d2q9_compute_macroscopic_moments_forced(const float f[], float rho[], float ux[], float uy[], float gx,
                                             float gy, int count);
void d2q9_compute_velocity_magnitude(const float ux[], const float uy[], float speed[], int count);
/* src/ispc/forces_momentum_exchange.ispc:6-18 (uniform float & -> float *) */
void d2q9_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[], int nx,
                                           int ny, float center_x, float center_y, float max_radius,
                                           float* fx_out, float* fy_out, float* torque_z_out);

/* D3Q19: src/ispc/d3q19_collision_bgk.ispc:4-17, d3q19_collision_trt.ispc:5-19, d3q19_collision_mrt.ispc:26-40 */
void d3q19_collide_bgk(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau, float gx, float gy, float gz, int count);
void d3q19_collide_trt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau_s, float tau_a, float gx, float gy, float gz, int count);
void d3q19_collide_mrt(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                       float uy[], float uz[], float tau_shear, float tau_bulk, float gx, float gy, float gz,
                       int count);
/* src/ispc/d3q19_streaming.ispc:4-10, 39-49 */
void d3q19_stream_periodic(const float f_src[], float f_dst[], int nx, int ny, int nz);
void d3q19_stream_with_boundaries(const float f_src[], float f_dst[], const uint8_t cell_type[], int nx, int ny,
                                  int nz, float uw_x, float uw_y, float uw_z);
/* src/ispc/d3q19_curved.ispc:7-20 */
void d3q19_apply_curved_bfl(float f_dst[], const float f_src[], const int fluid_indices[], const int q_dirs[],
                            const float delta_fractions[], const float uw_x[], const float uw_y[],
                            const float uw_z[], int nx, int ny, int nz, int num_boundary_links);
/* src/ispc/d3q19_les.ispc:7-17 */
void d3q19_compute_smagorinsky_tau(const float f[], const float rho[], const float ux[], const float uy[],
                                   const float uz[], float tau_eff[], float tau_0, float smagorinsky_constant,
                                   int count);
/* src/ispc/d3q19_moments.ispc:4-11, 35-45, 69-75 */
void d3q19_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], float uz[], int count);
void d3q19_compute_macroscopic_moments_forced(const float f[], float rho[], float ux[], float uy[], float uz[],
                                              float gx, float gy, float gz, int count);
void d3q19_compute_velocity_magnitude(const float ux[], const float uy[], const float uz[], float speed[],
                                      int count);
/* src/ispc/forces_momentum_exchange.ispc:71-84 */
void d3q19_compute_momentum_exchange_forces(const float f_post_collision[], const uint8_t cell_type[], int nx,
                                            int ny, int nz, float center_x, float center_y, float center_z,
                                            float max_radius, float* fx_out, float* fy_out, float* fz_out);

/* Allocation-free variant of d3q19_compute_momentum_exchange_forces. It has no
 * counterpart in the reference. It is meant for callers that cannot allocate
 * device memory while they run: a serving loop that has committed all of HBM to
 * resident lattices, or a latency-critical loop in which cudaMalloc / cudaFree
 * would synchronise the device. Instead of allocating scratch, it keeps its
 * per-block partial sums in a fixed 384 KiB device array of the library (held by
 * every GPU that loads the library until the process exits), which limits the
 * lattice to nx*ny*nz <= 4,194,304 nodes; larger sizes are rejected with
 * WAKE_ERR_INVALID. Every pointer must be memory of the current GPU or managed
 * memory (host buffers would need allocated staging). The buffers use the
 * reference's unpadded layout, f [19][nx*ny*nz] and cell_type [nx*ny*nz], with
 * the populations the reference passes (its f_src after a step); a resident
 * lattice's state buffers are padded per plane and hold post-collision values,
 * so pass what wake_grid_get_populations writes instead. The kernels run on the
 * legacy default stream and the call returns after cudaStreamSynchronize(0):
 * inputs written on other streams (a resident grid's or batch's streams do not
 * synchronise with the legacy stream) must be complete before the call. Returns
 * 0 or a WAKE_ERR_* code. The first call on each device looks up the array's
 * device address (once per device); make that first call before any stream
 * capture. All calls share the array: calls that overlap on the GPU race. The
 * partial sums are added in another order than the allocating entry point's
 * above 303,104 nodes, so the two agree to FP64 rounding there, not bit for bit. */
int d3q19_compute_momentum_exchange_forces_noalloc(const float f_post_collision[], const uint8_t cell_type[], int nx,
                                                   int ny, int nz, float center_x, float center_y, float center_z,
                                                   float max_radius, float* fx_out, float* fy_out, float* fz_out);

/* D3Q27: src/ispc/d3q27_collision_mrt.ispc:5-18 (TRT), d3q27_moments.ispc:4-11, d3q27_streaming.ispc:4-10 */
void d3q27_collide(const float f_in[], float f_out[], const uint8_t cell_type[], float rho[], float ux[],
                   float uy[], float uz[], float tau_s, float tau_a, float gx, float gy, float gz, int count);
void d3q27_compute_macroscopic_moments(const float f[], float rho[], float ux[], float uy[], float uz[], int count);
void d3q27_stream_periodic(const float f_src[], float f_dst[], int nx, int ny, int nz);

/* Thermal D2Q9: src/ispc/thermal_kernels.ispc:4-13, 48-55, 63-69 */
void thermal_collide_d2q9(const float g_in[], float g_out[], const uint8_t cell_type[], const float ux[],
                          const float uy[], float temperature[], float tau_T, int count);
void thermal_compute_buoyancy_force_2d(const float temperature[], float gy_body[], float t_ref, float beta,
                                       float g_gravity, int count);
void thermal_apply_isothermal_wall(float g[], int nx, int ny, int y_wall, float t_wall);

/* Immersed boundary, 2D: src/ispc/ibm_kernels.ispc:12-22 (velocity at the markers, Roma-Peskin
 * 4-point delta, periodic in x) and 56-67 (marker forces times arc length spread onto the
 * lattice body force; overlapping markers add atomically, so sums may differ from the
 * reference's marker-order loop in the last bits). Called by ImmersedBoundary
 * (src/ibm/immersed_boundary.cpp:87, 111). */
void ibm_interpolate_velocity_2d(const float ux[], const float uy[], const float marker_x[], const float marker_y[],
                                 float marker_ux[], float marker_uy[], int nx, int ny, int num_markers);
void ibm_spread_force_2d(const float marker_x[], const float marker_y[], const float marker_fx[],
                         const float marker_fy[], const float marker_ds[], float euler_gx[], float euler_gy[], int nx,
                         int ny, int num_markers);

/* Field analytics: src/ispc/analytics_kernels.ispc:4-10 (2D vorticity), 33-44
 * (3D vorticity vector + Q-criterion). Central differences with periodic wrap;
 * products and sums rounded in the reference's order without contraction.
 * Called by FieldAnalytics (src/analytics/field_analytics.cpp:5-14). */
void compute_vorticity_2d(const float ux[], const float uy[], float vorticity[], int nx, int ny);
void compute_vorticity_and_q_criterion_3d(const float ux[], const float uy[], const float uz[], float omega_x[],
                                          float omega_y[], float omega_z[], float q_criterion[], int nx, int ny,
                                          int nz);

/* ---------------------------------------------------------- fused engine */
typedef struct wake_grid wake_grid;

/* Storage of the resident populations. */
#define WAKE_STORE_F32 0
#define WAKE_STORE_F16 1   /* FP16 of f_q / w_q - 1 */
#define WAKE_STORE_BF16 2  /* BF16 of f_q / w_q - 1 */
#define WAKE_STORE_F16C 3  /* FP16C (1 sign, 4 exponent, 11 mantissa bits; |h| < 2) of h = f_q / w_q - 1 */

/* Collision models (values of the reference's CollisionType, include/wake/core/types.hpp:80-85). */
#define WAKE_BGK 0
#define WAKE_TRT 1
#define WAKE_MRT 2

/* Cell types (include/wake/core/types.hpp:69-77). */
#define WAKE_CELL_FLUID 0
#define WAKE_CELL_SOLID 1
#define WAKE_CELL_INFLOW 2
#define WAKE_CELL_OUTFLOW 3
#define WAKE_CELL_MOVING_WALL 6

/* q = 9 (nz must be 1), 19 or 27. Like LatticeGrid2D/3D's constructors
 * (lattice_grid_2d.cpp:46-62, lattice_grid_3d.cpp:46-64) the lattice starts at
 * rest with rho = 1 and every cell Fluid. Returns NULL on failure. */
wake_grid* wake_grid_create(int q, int nx, int ny, int nz, float tau, int storage);
void wake_grid_destroy(wake_grid* g);

/* Work on this CUDA stream (cudaStream_t passed as void*); NULL = library stream. */
int wake_grid_set_stream(wake_grid* g, void* stream);

/* Collision model. les = 1 applies the Smagorinsky tau per node (the reference
 * computes it but never feeds it to the collision, lattice_grid_2d.cpp:205).
 * lambda_trt: TRT magic parameter (reference 0.25). tau_bulk: MRT bulk rate
 * (reference 1.63 in 2D, 1.19 in 3D). mrt_exact: D3Q19 only, 0 = the
 * reference's 7-digit inverse table, 1 = exact inverse. s3, s4: D3Q27 MRT
 * third- and higher-order rates. */
int wake_grid_set_model(wake_grid* g, int collision, int les, float cs_smag, float lambda_trt, float tau_bulk,
                        int mrt_exact, float s3, float s4);
int wake_grid_set_relaxation_time(wake_grid* g, float tau);

/* Geometry (lattice_grid_2d.cpp:122-184, lattice_grid_3d.cpp:133-215). */
int wake_grid_set_cell_type(wake_grid* g, int x, int y, int z, int type);
int wake_grid_set_cell_types(wake_grid* g, const uint8_t* types /* host [nx*ny*nz] */);
int wake_grid_get_cell_types(wake_grid* g, uint8_t* types /* host [nx*ny*nz] */);
int wake_grid_set_solid_box(wake_grid* g, int x0, int y0, int z0, int x1, int y1, int z1);
int wake_grid_set_solid_circle(wake_grid* g, float cx, float cy, float radius);
int wake_grid_set_solid_sphere(wake_grid* g, float cx, float cy, float cz, float radius);
/* Velocity inlet (Zou-He) on x = 0 and pressure outlet on x = nx-1. 2D follows
 * the reference exactly (rows 1..ny-2, d2q9_boundaries.ispc:56,98); 3D applies
 * the D3Q19 on-site scheme on Inflow / Outflow cells of those faces. */
int wake_grid_set_inflow_west(wake_grid* g, float ux, float uy, float uz);
int wake_grid_set_outflow_east(wake_grid* g, float rho_out);
/* Moving lid: 2D north row (set_moving_wall_north), 3D top y = ny-1 plane. */
int wake_grid_set_moving_wall(wake_grid* g, float uw_x, float uw_y, float uw_z);
/* 3D: wrap y / z instead of half-way bounce-back walls. */
int wake_grid_set_periodic(wake_grid* g, int periodic_y, int periodic_z);
/* BFL curved links (arrays in host memory; uw may be NULL for resting walls). */
int wake_grid_set_curved_links(wake_grid* g, int n, const int* fluid_indices, const int* q_dirs,
                               const float* delta, const float* uw_x, const float* uw_y, const float* uw_z);
/* Link builder of LatticeGrid3D::build_curved_sphere_links (lattice_grid_3d.cpp:217-290). */
int wake_grid_build_curved_sphere_links(wake_grid* g, float cx, float cy, float cz, float radius);
int wake_grid_num_curved_links(wake_grid* g);
int wake_grid_get_curved_links(wake_grid* g, int* fluid_indices, int* q_dirs, float* delta);

/* Initial state: equilibrium of uniform / per-node fields (initialize,
 * initialize_custom: lattice_grid_2d.cpp:64-120), or raw populations f_src
 * [q][node] in host memory. The equilibrium is evaluated on the device in the
 * reference's float order; the fields may be host or device arrays. */
int wake_grid_initialize(wake_grid* g, float rho, float ux, float uy, float uz);
int wake_grid_initialize_fields(wake_grid* g, const float* rho, const float* ux, const float* uy, const float* uz);
/* Equilibrium of rho and u + amplitude * (2 r - 1) per component, r the 24-bit
 * uniform (top 24 bits * 2^-24) of SplitMix64 output offset + 1 + a * N + i
 * of `seed` for component a of node i, generated on the device. Same bits as
 * building the noisy fields on the host and calling initialize_fields. No
 * reference counterpart (the scenarios draw their noise on the host). */
int wake_grid_initialize_noise(wake_grid* g, float rho, float ux, float uy, float uz, float amplitude,
                               unsigned long long seed, long long offset);
int wake_grid_set_populations(wake_grid* g, const float* f /* host [q][nx*ny*nz] */);
/* Same, from device memory (no host staging). */
int wake_grid_set_populations_device(wake_grid* g, const float* f_dev /* device [q][nx*ny*nz] */);

/* Momentum-exchange monitor (forces_momentum_exchange.ispc:6-138): one force
 * record per step, (Fx, Fy, Tz) in 2D and (Fx, Fy, Fz) in 3D, summed in FP64
 * in a fixed order. history_capacity records are kept (ring). */
int wake_grid_enable_forces(wake_grid* g, float cx, float cy, float cz, float r_max, int history_capacity);
int wake_grid_disable_forces(wake_grid* g);
/* Copies up to max records, oldest first, of the last min(steps, capacity)
 * steps into a host or device buffer (only those records cross the bus);
 * returns the number copied or a negative error. */
int wake_grid_get_force_history(wake_grid* g, double* out /* [max][3] */, int max);
/* Number of steps recorded since forces were enabled. */
long long wake_grid_force_count(wake_grid* g);

/* Advance n steps with body force (gx, gy, gz). */
int wake_grid_step(wake_grid* g, int n, float gx, float gy, float gz);
/* Capture n steps in a CUDA graph (replayed by wake_grid_step whenever n is a
 * multiple of the captured count and nothing was reconfigured). 0 disables. */
int wake_grid_use_graph(wake_grid* g, int steps_per_graph);
/* Do now the one-time work that the next wake_grid_step with this body force
 * would do first: re-collide after a parameter or geometry change and, when a
 * graph size is set, capture and instantiate the graph from the current buffer
 * parity. Advances nothing; returns after that work has finished, so that a
 * timed run of wake_grid_step measures the steps alone. No reference
 * counterpart. */
int wake_grid_prepare_steps(wake_grid* g, float gx, float gy, float gz);
long long wake_grid_step_count(wake_grid* g);
/* Block until the grid's stream is idle; reports device-side numeric errors. */
int wake_grid_synchronize(wake_grid* g);

/* Reference-visible state after the last step: f_src [q][node], and
 * rho/ux/uy/uz/speed (moments_forced + velocity magnitude). Host or device
 * pointers; uz may be NULL in 2D. */
int wake_grid_get_populations(wake_grid* g, float* f);
int wake_grid_get_macroscopic(wake_grid* g, float* rho, float* ux, float* uy, float* uz, float* speed);
/* Diagnostics over Fluid cells (lattice_grid_2d.cpp:267-295), summed in FP64. */
int wake_grid_diagnostics(wake_grid* g, double* total_mass, double* kinetic_energy, double* max_speed);
/* Mass over every non-solid cell, FP64 (global conservation check). */
int wake_grid_total_mass(wake_grid* g, double* mass);

/* Introspection for benchmarks and tests. */
int wake_grid_info(wake_grid* g, int* q, int* nx, int* ny, int* nz, int* storage, long long* pitch);
/* Device pointer of the state buffer holding g^k (which = 0) or the other one (which = 1). */
void* wake_grid_state_buffer(wake_grid* g, int which);
/* Launch shape of the fused kernel: threads per block (32..512, multiple of 32). */
int wake_grid_set_block(wake_grid* g, int threads_per_block);
int wake_grid_get_block(wake_grid* g);
/* Step kernels: 0 automatic (default), 1 direct (a launch over the pure-gather
 * spans reading global memory, beside a launch over the remaining rows), 2 one
 * persistent launch per step that stages the pure-gather rows in shared memory
 * by bulk copies, tiles of up to 1024 nodes, and runs the remaining rows beside
 * them (used when a row is a whole number of 16-byte chunks and at most 1024
 * nodes), 3 (TRT) one block per row whose every node is a pure gather, 4 (TRT)
 * those rows moved through shared memory by bulk copies in both directions, a
 * few rows in flight per block (rows of at most 512 nodes and a whole number of
 * 16-byte chunks). A variant whose conditions do not hold runs the direct
 * kernels. Automatic: 4 for 16-bit storage where it applies, else 1.
 * get_kernel prepares the grid and returns the variant in use (1 to 4). For
 * TRT every variant computes two nodes per thread in packed FP32 with the same
 * roundings, so all give the same bits. No reference counterpart. */
int wake_grid_set_kernel(wake_grid* g, int variant);
int wake_grid_get_kernel(wake_grid* g);
/* Kernel launches one fused step issues with the current geometry (pure-gather
 * rows, general rows, momentum-exchange reduction). No reference counterpart. */
int wake_grid_launches_per_step(wake_grid* g);
/* CUDA-event timing of each pure-gather (bulk) launch. While on, steps run as
 * plain launches (no graph). bulk_launch_times synchronizes, returns the summed
 * duration of the launches recorded since the last read, their count and the
 * nodes one launch updates, and restarts the count. No reference counterpart. */
int wake_grid_time_bulk_launches(wake_grid* g, int on);
int wake_grid_bulk_launch_times(wake_grid* g, double* total_ms, long long* launches, long long* nodes_per_launch);

/* Coupled temperature (D2Q9 lattices only; no reference counterpart: the
 * reference's ThermalSolver2D, src/thermal/thermal_solver.cpp:83-123, carries a
 * D2Q9 temperature and drives the flow with one domain-averaged force,
 * src/scenarios/thermal_convection.cpp:70). A D2Q5 temperature lattice advances
 * in the same fused step as the flow: per node T = sum g, the flow collides
 * with the body force (gx, gy + beta_g (T - t_ref)) (local Boussinesq), the
 * temperature relaxes with tau_t to w_q T (1 + 3 c_q.u). The y walls hold
 * t_south (y = -1/2) and t_north (y = ny - 1/2) by anti-bounce-back; solid
 * nodes are adiabatic. enable before the first step (the temperature starts at
 * t_ref); initialize_temperature sets a per-node start (host or device array of
 * N floats) and restarts the coupled run at step 0 from the flow's initial
 * state. The collision model, tau and body force are fixed once the grid has
 * stepped. get_temperature returns the temperature of the last step (N floats).
 * Thermal grids run every node on the general per-node path. */
int wake_grid_enable_thermal(wake_grid* g, float tau_t, float t_ref, float beta_g, float t_south, float t_north);
int wake_grid_initialize_temperature(wake_grid* g, const float* T);
int wake_grid_get_temperature(wake_grid* g, float* T);

/* Rotated solid ellipse, semi-axes a (along the rotated x axis) and b, angle in
 * radians; extruded along z in 3D. Cell-centre test in float like
 * GeometryPrimitives::voxelize_ellipsoid (src/geometry/primitives.cpp:73-99),
 * which has no rotation and no 2D form. */
int wake_grid_set_solid_ellipse(wake_grid* g, float cx, float cy, float a, float b, float angle);

/* Device memory: what the grid holds now, and an upper estimate for a new grid
 * of that shape (state buffers, FP32 initialisation scratch, flags, tables;
 * with_fields bit 0 adds the macroscopic-field scratch, bit 1 a coupled temperature). release_scratch first
 * completes any pending setup (flags, initial collide), then frees the FP32
 * population and field scratch (re-allocated on demand by the readers). A
 * parameter change after it and before the first step re-collides f^0 as held
 * in the state buffer, i.e. at storage precision.
 * No reference counterpart (the reference allocates host AlignedBuffers,
 * include/wake/core/memory.hpp:52-159). */
long long wake_grid_device_bytes(wake_grid* g);
long long wake_grid_estimate_bytes(int q, int nx, int ny, int nz, int storage, int with_fields);
int wake_grid_release_scratch(wake_grid* g);

/* ------------------------------------------------------------------ batches
 * A batch advances many resident grids together: one bulk launch over the
 * pure-gather rows of every member, one launch over the remaining rows and one
 * momentum-exchange reduction per step, whatever the members' sizes. Members
 * share the lattice and storage (checked by add) and the collision model and LES
 * switch (checked by step); sizes, tau, boundaries, geometry and force monitors
 * are per member. A member stays an ordinary grid: its readers (populations,
 * fields, force history, diagnostics) work between batch steps, and its results
 * are identical to stepping it alone. Its work runs on the batch stream while it
 * is a member. Remove a grid before destroying it. No reference counterpart:
 * the reference steps one LatticeGrid per call (src/grid/lattice_grid_2d.cpp:195-265). */
typedef struct wake_batch wake_batch;
wake_batch* wake_batch_create(int q, int storage);
void wake_batch_destroy(wake_batch* b);          /* members stay valid, back on their own streams */
int wake_batch_add(wake_batch* b, wake_grid* g);  /* returns the member index */
int wake_batch_remove(wake_batch* b, wake_grid* g);
int wake_batch_size(wake_batch* b);
int wake_batch_set_stream(wake_batch* b, void* stream);
int wake_batch_use_graph(wake_batch* b, int steps_per_graph);
int wake_batch_set_block(wake_batch* b, int threads_bulk, int threads_general);
int wake_batch_get_block(wake_batch* b);
/* As wake_grid_set_kernel, for the batch (persistent tiles only when every member allows them). */
int wake_batch_set_kernel(wake_batch* b, int variant);
int wake_batch_step(wake_batch* b, int n);
int wake_batch_synchronize(wake_batch* b);        /* first member error, if any */
int wake_batch_info(wake_batch* b, long long* nodes, int* bulk_rows, int* general_rows, int* launches_per_step);
/* Times `steps` real steps per bulk block size (those of 32, 64, 128, 256 within
 * the build's bound, 64 by default) and keeps the fastest; members advance
 * `steps` per size tried. Results do not depend on the choice. */
int wake_batch_autotune(wake_batch* b, int steps, int* best_threads);
/* Host seconds spent so far inside wake_batch_step, by phase: preparing members and
 * tables, capturing and instantiating CUDA graphs, issuing launches (including any wait
 * for launch-queue space). For finding where a serving loop's time goes. */
int wake_batch_host_seconds(wake_batch* b, double* prepare_s, double* capture_s, double* launch_s);

/* ------------------------------------------------------------------ field analytics and VTK
 * FieldAnalytics (src/analytics/field_analytics.cpp:18-63) on the device, from
 * the moments of the grid's current state (the same ux/uy/uz the reference
 * passes from grid.ux_data()): 2D vorticity, 3D vorticity vector + Q-criterion,
 * and the largest |vorticity| in 2D. Outputs are host or device memory, one
 * float per node. wake_field_abs_max = compute_max_vorticity_2d on any float
 * array (host or device; NaN values are skipped, as std::max from 0 does). */
int wake_grid_compute_vorticity(wake_grid* g, float* vorticity);
int wake_grid_compute_3d_features(wake_grid* g, float* omega_x, float* omega_y, float* omega_z, float* q_criterion);
int wake_grid_max_vorticity(wake_grid* g, float* max_vorticity);
int wake_field_abs_max(const float* values, long long count, float* max_abs);

/* VTK XML ImageData (.vti, ASCII) and ParaView .pvd collections in the bytes
 * wake::VtkExporter writes (src/export/vtk_exporter.cpp:8-223) for the same
 * fields: Velocity, Speed, Density, then Vorticity (2D) or Q_Criterion and
 * Vorticity (3D) when given, then CellType. Arrays are host memory, x fastest;
 * vorticity_x/y/z are the three components as separate arrays (written
 * interleaved, as the reference's Vec3 array). Formatting runs on `threads`
 * host threads (<= 0: all cores) and gives the same bytes for any count.
 * wake_grid_export_vti writes a grid's current state (moments, cell types and,
 * when `analytics` is nonzero, the device-computed vorticity / Q-criterion).
 * Return 0, or WAKE_ERR_INVALID when the file cannot be written. */
int wake_vtk_write_vti_2d(const char* path, int nx, int ny, const float* ux, const float* uy, const float* speed,
                          const float* rho, const float* vorticity, const uint8_t* cell_type, int threads);
int wake_vtk_write_vti_3d(const char* path, int nx, int ny, int nz, const float* ux, const float* uy,
                          const float* uz, const float* speed, const float* rho, const float* q_criterion,
                          const float* vorticity_x, const float* vorticity_y, const float* vorticity_z,
                          const uint8_t* cell_type, int threads);
int wake_vtk_write_pvd(const char* manifest_path, const char* file_prefix, int start_step, int end_step,
                       int step_interval, float dt);
int wake_grid_export_vti(wake_grid* g, const char* path, int analytics, int threads);

/* ------------------------------------------------------------------ telemetry files
 * The reference's telemetry formats (wake::TelemetryExporter,
 * src/export/csv_telemetry.cpp:21-125): aerodynamic CSV
 * "step,time,fx,fy,fz,cd,cl,cm", performance CSV
 * "step,step_time_ms,mlups,max_speed,total_mass,kinetic_energy" and the summary
 * JSON, identical bytes for identical records. Coefficients follow
 * compute_aerodynamic_coefficients (include/wake/forces/momentum_exchange.hpp:20-37)
 * in float. record_history turns a grid's FP64 force history (n rows of
 * Fx, Fy, Tz in 2D / Fx, Fy, Fz in 3D, row i = step first_step + i) into records
 * of the steps divisible by `every` (the scenarios record every 10th step,
 * src/scenarios/karman_vortex.cpp:126). Host code only; no device work. */
typedef struct wake_telemetry wake_telemetry;
wake_telemetry* wake_telemetry_create(void);
void wake_telemetry_destroy(wake_telemetry* t);
void wake_telemetry_clear(wake_telemetry* t);
int wake_telemetry_record_aero(wake_telemetry* t, unsigned long long step, float time, float fx, float fy, float fz,
                               float torque_z, float rho_inf, float u_inf, float area, float chord);
int wake_telemetry_record_history(wake_telemetry* t, const double* hist, int n, long long first_step, int every,
                                  int is3d, float rho_inf, float u_inf, float area, float chord);
int wake_telemetry_record_performance(wake_telemetry* t, unsigned long long step, double step_time_ms, double mlups,
                                      float max_speed, float total_mass, float kinetic_energy);
int wake_telemetry_count(wake_telemetry* t, int which); /* 0: aerodynamic records, 1: performance records */
int wake_telemetry_get_coefficients(wake_telemetry* t, int i, float* cd_cl_cm);
int wake_telemetry_write_aero_csv(wake_telemetry* t, const char* path);
int wake_telemetry_write_performance_csv(wake_telemetry* t, const char* path);
int wake_telemetry_write_summary_json(wake_telemetry* t, const char* path, const char* simulation_name,
                                      float strouhal_number, float shedding_frequency);

/* FP64 Strouhal frequency of a lift history (strouhal_analyzer.cpp:39-84:
 * mean removed, Hann window over the first min(n, 4096) samples, radix-2 FFT,
 * peak bin >= 1). Returns the frequency; St = f D / U. */
double wake_strouhal_frequency(const double* signal, int n, double dt);

#ifdef __cplusplus
}
#endif

#endif /* WAKE_GPU_H */
