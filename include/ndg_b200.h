/* ndg_b200: C ABI of the B200 (sm_100a) DG spectral-element wave solver.
 *
 * Drop-in for the GPU path of NDG_cuda's 2D wave-equation time step. Every
 * entry point takes plain pointers and sizes; device memory, streams and
 * kernels stay inside the library. Each declaration names the reference
 * interface it replaces (paths inside the NDG_cuda repository).
 *
 * Conventions
 *  - Every call returns an ndg_status; on failure ndg_last_error() returns a
 *    message for the calling thread. Nothing calls exit().
 *  - One context per host thread; calls on one context are not thread-safe.
 *    All device work is ordered on the context's stream; calls that return
 *    host data synchronise that stream.
 *  - Element fields are laid out as the reference's Element2D_t arrays:
 *    element after element, (N+1)^2 values each, node index i*(N+1)+j with i
 *    along xi and j along eta (include/entities/Element2D_t.h:36-38).
 *  - Several independent instances (same mesh, different fields) can share
 *    one context; instance fields follow each other in the field arrays.
 */
#ifndef NDG_B200_H
#define NDG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ndg_status {
    NDG_OK = 0,
    NDG_ERR_INVALID_ARG = 1,
    NDG_ERR_MESH = 2,
    NDG_ERR_CUDA = 3,
    NDG_ERR_NONFINITE = 4,
    NDG_ERR_OOM = 5,
    NDG_ERR_TIMEOUT = 6,
    NDG_ERR_UNSUPPORTED = 7
} ndg_status;

/* Opaque solver context. */
typedef struct ndg_ctx ndg_ctx;

/* Arithmetic of the stage kernels.
 * NDG_FP64: FP64 with fused multiply-adds and reciprocal multiplies.
 * NDG_FP64_STRICT: FP64 rounded operation by operation in the reference's
 *   order (no contraction, true divisions): bit-identical to the reference's
 *   CPU path on the same inputs.
 * NDG_FP32: traces, fluxes, metrics and the volume term in FP32 (traces
 *   stored in FP32); the solution, the RK register and the RK update stay
 *   FP64. Every mesh: uniform meshes use the fused FP32 stage kernel;
 *   mixed-order and nonconforming meshes after adaptation run the mixed-order
 *   kernels in FP32 (mortar interpolation and projection included). */
typedef enum ndg_precision { NDG_FP64 = 0, NDG_FP64_STRICT = 1, NDG_FP32 = 2 } ndg_precision;

/* Tables of NDG_t (include/entities/NDG_t.cuh:11-29). */
typedef enum ndg_table {
    NDG_TABLE_NODES = 0,
    NDG_TABLE_WEIGHTS = 1,
    NDG_TABLE_BARYCENTRIC_WEIGHTS = 2,
    NDG_TABLE_LAGRANGE_LEFT = 3,
    NDG_TABLE_LAGRANGE_RIGHT = 4,
    NDG_TABLE_LAGRANGE_DERIVATIVE_LEFT = 5,
    NDG_TABLE_LAGRANGE_DERIVATIVE_RIGHT = 6,
    NDG_TABLE_DERIVATIVE_MATRICES = 7,
    NDG_TABLE_G_HAT_DERIVATIVE_MATRICES = 8,
    NDG_TABLE_DERIVATIVE_MATRICES_HAT = 9,
    NDG_TABLE_INTERPOLATION_MATRICES = 10,
    NDG_TABLE_POLYNOMIALS = 11
} ndg_table;

typedef enum ndg_field {
    NDG_FIELD_P = 0, NDG_FIELD_U = 1, NDG_FIELD_V = 2,          /* Element2D_t::p_, u_, v_ */
    NDG_FIELD_G_P = 3, NDG_FIELD_G_U = 4, NDG_FIELD_G_V = 5,    /* Element2D_t::G_p_ ... (last stage's time derivative) */
    NDG_FIELD_K_P = 6, NDG_FIELD_K_U = 7, NDG_FIELD_K_V = 8     /* Element2D_t::p_intermediate_ ... (RK register) */
} ndg_field;

/* Boundary condition codes of the zone description (CGNS BCType_t subset read by
 * Mesh2D_t::read_cgns, src/meshes/Mesh2D_t.cpp:725-816). */
typedef enum ndg_bc { NDG_BC_WALL = 0, NDG_BC_SYMMETRY = 1, NDG_BC_INFLOW = 2, NDG_BC_OUTFLOW = 3, NDG_BC_NULL = 4 } ndg_bc;

/* Boundary lists of ndg_mesh_get_boundary (Mesh2D_t::wall_boundaries_ ...,
 * interfaces_origin_ ..., include/meshes/Mesh2D_t.h:29-38). */
typedef enum ndg_boundary_list {
    NDG_LIST_WALL = 0, NDG_LIST_SYMMETRY = 1, NDG_LIST_INFLOW = 2, NDG_LIST_OUTFLOW = 3,
    NDG_LIST_INTERFACE_ORIGIN = 4, NDG_LIST_INTERFACE_ORIGIN_SIDE = 5, NDG_LIST_INTERFACE_DESTINATION = 6
} ndg_boundary_list;

/* One unstructured 2D zone in CGNS terms: what Mesh2D_t::read_cgns reads from
 * a file (src/meshes/Mesh2D_t.cpp:422-645), as arrays.
 *  - section_type: 0 = QUAD_4 (domain), 1 = BAR_2 (ghost/boundary elements);
 *    section_start/end: 1-based element numbers; section_connectivity:
 *    1-based node numbers, 4 per quad and 2 per bar, sections concatenated.
 *  - boco_type: ndg_bc; boco_points: 1-based element numbers, concatenated.
 *  - conn_*: Abutting1to1 self connectivity (periodic), 1-based element
 *    numbers of the receiving ghost and of its donor ghost. */
typedef struct ndg_zone {
    int64_t n_nodes;
    const double* x;
    const double* y;
    int32_t n_sections;
    const int32_t* section_type;
    const int64_t* section_start;
    const int64_t* section_end;
    const int64_t* section_connectivity;
    int32_t n_bocos;
    const int32_t* boco_type;
    const int64_t* boco_count;
    const int64_t* boco_points;
    int32_t n_conns;
    const int64_t* conn_count;
    const int64_t* conn_points;
    const int64_t* conn_donors;
} ndg_zone;

/* Constructor arguments of Mesh2D_t (include/meshes/Mesh2D_t.cuh:25) and
 * the CFL of Solver2D_t (include/solvers/Solver2D_t.cuh:16). */
typedef struct ndg_mesh_params {
    int32_t initial_N;
    int32_t maximum_N;
    int64_t n_interpolation_points;
    int32_t max_split_level;
    int64_t adaptivity_interval;
    double tolerance_min;
    double tolerance_max;
    double cfl;
} ndg_mesh_params;

/* Message of the last failed call on this thread ("" if none). */
const char* ndg_last_error(void);
const char* ndg_version(void);

/* Context: owns device memory and the stream of one solver.
 * device < 0 makes a host-only context (tables and mesh topology, no GPU).
 * stream is a cudaStream_t (NULL = a stream created by the context).
 * Replaces the stream/ownership plumbing of Mesh2D_t (include/meshes/Mesh2D_t.cuh:163). */
ndg_status ndg_ctx_create(int32_t device, void* stream, ndg_ctx** out);
ndg_status ndg_ctx_destroy(ndg_ctx* ctx);
ndg_status ndg_ctx_set_precision(ndg_ctx* ctx, int32_t precision);
ndg_status ndg_ctx_synchronize(ndg_ctx* ctx);
/* Keep a copy of each stage's time derivative G (Element2D_t::G_p_ ...) so
 * that ndg_get_field can return it; off by default (it costs HBM traffic). */
ndg_status ndg_ctx_keep_derivative(ndg_ctx* ctx, int32_t enable);
/* How a stage runs on a mixed-order mesh (after adaptation), replacing the
 * reference's per-stage launch chain (include/solvers/Solver2D_t.tcu:44-70):
 * mode 0 (default) one launch per order group, as concurrent branches of
 * the step graph, each with its order's own tile, registers and shared
 * memory; mode 1 one launch per stage whose CTAs take the tiles of every
 * order group from one queue, largest order first, each running its tile's
 * order; mode 2 as mode 0, but every order group that is not all
 * conforming elements runs in two launches: its element side fluxes (face
 * fluxes and mortar projections), then the uniform-style element tile over
 * them. Mode 0 runs a group that way where it has at least 2,048
 * elements (times the instances) and its order no conforming part, else
 * fused. Each computes the same operations
 * either way (bit-identical in NDG_FP64_STRICT; the compiler may contract
 * differently otherwise). Meshes of one order are not affected. */
ndg_status ndg_set_mixed_launch(ndg_ctx* ctx, int32_t mode);

/* NDG_t<LegendrePolynomial_t>(N_max, n_interpolation_points, stream)
 * (include/entities/NDG_t.cuh:11, include/entities/NDG_t.tcu:13-72). */
ndg_status ndg_tables_build(ndg_ctx* ctx, int32_t N_max, int64_t n_interpolation_points);
/* One table of order N into out[capacity]; *count = number of values. */
ndg_status ndg_tables_get(const ndg_ctx* ctx, int32_t table, int32_t N, double* out, int64_t capacity, int64_t* count);
/* The same without a context (host FP64, no GPU). */
ndg_status ndg_tables_compute(int32_t N_max, int64_t n_interpolation_points, int32_t table, int32_t N, double* out, int64_t capacity, int64_t* count);

/* Mesh2D_t(filename, initial_N, maximum_N, ...) for a zone given as arrays
 * (include/meshes/Mesh2D_t.cuh:25, src/meshes/Mesh2D_t.cu:32-82). Builds the
 * reference's element, face, boundary and interface numbering, then the
 * device layout. n_instances independent solutions share the mesh. */
ndg_status ndg_mesh_load_zone(ndg_ctx* ctx, const ndg_zone* zone, const ndg_mesh_params* params, int32_t n_instances);
/* Same, from a mesh file: .su2 (Mesh2D_t::read_su2, src/meshes/Mesh2D_t.cpp:78-421). */
ndg_status ndg_mesh_load_file(ndg_ctx* ctx, const char* path, const ndg_mesh_params* params, int32_t n_instances);
ndg_status ndg_mesh_counts(const ndg_ctx* ctx, int64_t* n_elements, int64_t* n_elements_total, int64_t* n_faces, int64_t* n_nodes);
/* Topology views with the reference's numbering (Face2D_t fields,
 * include/entities/Face2D_t.h:37-58; Element2D_t nodes_/faces_/N_). */
ndg_status ndg_mesh_get_faces(const ndg_ctx* ctx, int64_t* nodes, int64_t* elements, int64_t* sides, int32_t* N,
                              double* normal, double* tangent, double* offset, double* scale);
ndg_status ndg_mesh_get_elements(const ndg_ctx* ctx, int64_t* nodes, int32_t* N, double* delta_xy_min, int64_t* first_face);
ndg_status ndg_mesh_get_boundary(const ndg_ctx* ctx, int32_t list, int64_t* out, int64_t capacity, int64_t* count);
/* Per element (domain and ghosts): Element2D_t::split_level_, status_
 * (Hilbert H, A, R, B = 0..3) and rotation_ (include/entities/Element2D_t.h),
 * and the number of faces on each of its 4 sides (faces_[s].size()). Any
 * pointer may be NULL. */
ndg_status ndg_mesh_get_element_state(const ndg_ctx* ctx, int32_t* split_level, int32_t* status, int32_t* rotation, int32_t* n_faces_side);
/* The faces of every element side, element by element and side by side
 * (Element2D_t::faces_), into out[capacity]; *count = total number. */
ndg_status ndg_mesh_get_element_faces(const ndg_ctx* ctx, int64_t* out, int64_t capacity, int64_t* count);
ndg_status ndg_mesh_get_nodes(const ndg_ctx* ctx, double* xy);
/* Degrees of freedom per field and instance: sum over elements of (N+1)^2. */
ndg_status ndg_mesh_field_size(const ndg_ctx* ctx, int64_t* n_values);

/* Mesh2D_t::initial_conditions (src/meshes/Mesh2D_t.cu:5030): the reference
 * plane wave g(x, 0) in every instance; G and the RK register are zeroed. */
ndg_status ndg_initial_conditions(ndg_ctx* ctx);
/* Copies one field of one instance from/to host memory (field_size values).
 * instance < 0 addresses all instances back to back. */
ndg_status ndg_set_field(ndg_ctx* ctx, int32_t instance, int32_t field, const double* values);
ndg_status ndg_get_field(ndg_ctx* ctx, int32_t instance, int32_t field, double* values);

/* Solver2D_t::get_delta_t (src/solvers/Solver2D_t.cu:17-31): min over
 * elements of CFL * delta_xy_min / (N^2 c), reduced on the device. */
ndg_status ndg_get_delta_t(ndg_ctx* ctx, double* delta_t);
/* The CFL of Solver2D_t(CFL, ...) (include/solvers/Solver2D_t.cuh:16):
 * recomputes the mesh's step for a new CFL (the load used
 * ndg_mesh_params.cfl); later ndg_run/ndg_solve steps use it. */
ndg_status ndg_set_cfl(ndg_ctx* ctx, double cfl);
/* One low-storage RK3 stage m in {0,1,2} at step start `time` with step dt:
 * interpolate_to_boundaries, boundary_conditions, project_to_faces,
 * calculate_wave_fluxes, project_to_elements, compute_dg_wave_derivative,
 * rk3_(first_)step (include/solvers/Solver2D_t.tcu:46-70), fused. */
ndg_status ndg_stage(ndg_ctx* ctx, int32_t m, double time, double dt);
/* n_steps RK3 steps, each with dt = get_delta_t; *time advances by dt per step. */
ndg_status ndg_run(ndg_ctx* ctx, int64_t n_steps, double* time);
/* The reference's time loop to t_end (include/solvers/Solver2D_t.tcu:7-135
 * without output): the last step is shortened to land on t_end, and with
 * adaptivity_interval > 0 the error is estimated and the mesh adapted after
 * every adaptivity_interval-th step. *time is the start time in and the end
 * time out. */
ndg_status ndg_solve(ndg_ctx* ctx, double t_end, double* time, int64_t* n_steps);

/* Mesh2D_t::estimate_error (src/meshes/Mesh2D_t.cu:5158, Element2D_t::estimate_p_error,
 * src/entities/Element2D_t.cpp:274-343): Legendre-coefficient decay of the
 * pressure in every element of every instance, on the device. */
ndg_status ndg_estimate_error(ndg_ctx* ctx);
/* Per element of one instance: p_error_, p_sigma_, refine_ (error >
 * tolerance_min), coarsen_ (error < tolerance_max). Any pointer may be NULL. */
ndg_status ndg_get_error(ndg_ctx* ctx, int32_t instance, double* p_error, double* p_sigma, int32_t* refine, int32_t* coarsen);

/* Mesh2D_t::adapt(N_max, nodes, barycentric_weights) (src/meshes/Mesh2D_t.cpp:1644-2268)
 * from the last ndg_estimate_error: elements with refine_ and p_sigma_ >= 1
 * below maximum_N gain 2 orders (p_adapt, :5026) with their solution
 * interpolated (Element2D_t::interpolate_from, src/entities/Element2D_t.cpp:464-579);
 * boundary and interface ghosts and faces take their neighbours' orders
 * (adjust_boundaries, adjust_interfaces, adjust_faces, :7482-7538). Later
 * steps run the mixed-order (mortar) stage path. Needs one instance.
 * Elements with refine_, p_sigma_ < 1 and split_level_ < max_split_level
 * split in four (see ndg_adapt_flags). The estimate is consumed. */
ndg_status ndg_adapt(ndg_ctx* ctx);
/* The same adaptation from caller-given refine_ flags and p_sigma_ decay
 * rates, one per domain element (the element state Mesh2D_t::adapt reads).
 * Element splitting (h-refinement) follows the reference's rules and
 * numbering: hp_adapt, split_faces, split_boundaries and split_interfaces
 * (src/meshes/Mesh2D_t.cpp:5186-6757); children take their solution by
 * interpolation from the parent (Element2D_t.cpp:345-463). On a host-only
 * context (device < 0) only the topology is adapted. */
ndg_status ndg_adapt_flags(ndg_ctx* ctx, const int32_t* refine, const double* p_sigma);

/* Benchmark aid: launches stage m n_launches times back to back (the state
 * advances), timing each launch with CUDA events on the context's stream;
 * *avg_ms = mean kernel duration. */
ndg_status ndg_time_stage(ndg_ctx* ctx, int32_t m, int32_t n_launches, double* avg_ms);

/* Autotuner (no reference counterpart). The uniform-order stage kernel is
 * compiled for several tiles (elements per CTA: 2, 4, 8, 16 where a tile
 * fits 512 threads and 113 KB of shared memory) besides its default.
 * ndg_autotune times n_launches launches of each tile, and of the default,
 * on the loaded mesh and instances in the context's current form (FP64 or
 * FP32), keeps the fastest for later stepping and returns it (0 = the
 * default) with its mean launch time. The fields are restored afterwards.
 * Tiles do not change results: every element computes the same operations
 * whatever tile holds it. Mixed-order meshes and the strict form keep their
 * tiles (the call returns 0). Tiles reset when the mesh changes. */
ndg_status ndg_autotune(ndg_ctx* ctx, int32_t n_launches, int32_t* elements_per_block, double* best_ms);
/* Sets the tile of the current form by hand (0 = the default). */
ndg_status ndg_set_tile(ndg_ctx* ctx, int32_t elements_per_block);
/* The candidate tiles of the loaded order and current form, and the default. */
ndg_status ndg_tile_candidates(const ndg_ctx* ctx, int32_t* out, int32_t capacity, int32_t* count, int32_t* default_tile);

/* No counterpart in the reference. Host wall time of the last adaptation
 * (ndg_adapt or ndg_adapt_flags) by phase, in ms: ms[0] the decisions and
 * renumbering counts on the device (with the upload of the topology they
 * read and the download of their results), ms[1] the rebuild of the
 * topology on the host, ms[2] the field transfer to the new elements,
 * ms[3] the device plan of the new mesh. */
ndg_status ndg_adapt_timings(const ndg_ctx* ctx, double* ms);

/* Kernel launches issued by this context so far (for launch accounting). */
ndg_status ndg_launch_count(const ndg_ctx* ctx, int64_t* launches);

/* No counterpart in the reference. The CFL time step of ndg_get_delta_t,
 * min over elements of cfl * delta_xy_min / N^2 (bit-identical), computed
 * from caller-owned device arrays of n_elements values on the current device
 * and returned in *delta_t (host memory) after the stream has been
 * synchronised. It allocates no device memory (no cudaMalloc/cudaFree, no
 * allocating library routine) and needs no context: for callers that manage
 * all device memory through their own pool, or whose time loop cannot afford
 * the device-wide synchronisation of cudaMalloc/cudaFree. The partial minima go to one fixed 33 KB scratch array
 * per device, so n_elements is at most 4,194,304 (NDG_ERR_INVALID_ARG
 * beyond), and calls that overlap in time on one device race on that array:
 * serialise them. Each call looks up the array's address on the current
 * device (nothing is cached between calls); the first call on a device also
 * loads the library's kernels there. Every call copies the result to the
 * host and synchronises its stream before it returns, so it can never be
 * captured into a graph: do not make it on a capturing stream, nor while
 * another thread runs a global-mode capture on the device. stream is a
 * cudaStream_t of the current device (NULL: the default
 * stream); a stream of another device is refused with NDG_ERR_INVALID_ARG. */
ndg_status ndg_delta_t_from_device(const double* delta_xy_min, const int32_t* elem_N, int64_t n_elements,
                                   double cfl, void* stream, double* delta_t);

/* ------------------------------------------------------------------------
 * Solution output. */

/* Mesh2D_t::get_solution and get_complete_solution (src/meshes/Mesh2D_t.cpp:4237-4296;
 * Element2D_t::interpolate_solution and interpolate_complete_solution,
 * src/entities/Element2D_t.cpp:580-646) for one instance, on the device:
 * every domain element's fields on an n x n grid of equispaced reference
 * points xi_i = i / (n - 1) * 2 - 1, n = the mesh's n_interpolation_points
 * (>= 2). Each array holds n_elements n^2 values, point (i, j) of element e
 * at e n^2 + i n + j; any pointer may be NULL. x, y: physical coordinates
 * (quad_map); p, u, v: the fields interpolated with the order's
 * interpolation matrix; dp_dt, du_dt, dv_dt: the last stage's time
 * derivative (needs ndg_ctx_keep_derivative before stepping);
 * *_analytical_error: sum_mn |g(x_mn, time) - q_mn| I_im I_jn over the Gauss
 * nodes, g the reference plane wave. Rounded in the reference's order: x, y,
 * the fields and the derivatives equal its CPU output bit for bit, the
 * analytic error to the rounding of the exponential. */
typedef struct ndg_solution_output {
    double *x, *y, *p, *u, *v;
    double *dp_dt, *du_dt, *dv_dt;
    double *p_analytical_error, *u_analytical_error, *v_analytical_error;
} ndg_solution_output;
ndg_status ndg_get_solution(ndg_ctx* ctx, int32_t instance, double time, const ndg_solution_output* out);

/* L2 error of one instance against the reference plane wave g(x, time)
 * (include/functions/analytical_solution.tpp:4-10), per field:
 * l2[f] = sqrt(sum_e sum_ij w_i w_j J_ij (q_ij - g_ij)^2), w the Gauss
 * weights and J the Jacobian of the element map (Element2D_t.cpp:743-777).
 * The reference writes only the pointwise |g - q| (get_complete_solution);
 * this is the norm of it over the domain, the same formula as the oracle's. */
ndg_status ndg_l2_error(ndg_ctx* ctx, int32_t instance, double time, double* l2);

/* Output files in the role of DataWriter_t (src/helpers/DataWriter_t.cpp,
 * include/helpers/DataWriter_t.h; VTK is not needed): per output time a
 * parallel unstructured grid <stem>_t<time, 9 decimals, '.' -> '_'>s<ext>
 * (PUnstructuredGrid summary) with its piece <that name without ext>_0.vtu
 * (base64 binary arrays), and for the complete output the element grid
 * <stem>_element_t...s<ext>; time series <output_filename>.series and
 * <stem>_element<ext>.series (JSON), created empty by ndg_writer_create
 * (DataWriter_t::DataWriter_t) and extended at every write. Array names,
 * components and cell layout are the reference's (see writer.cpp). */
typedef struct ndg_writer ndg_writer;
ndg_status ndg_writer_create(const char* output_filename, ndg_writer** writer);
ndg_status ndg_writer_destroy(ndg_writer* writer);
/* DataWriter_t::write_data (complete = 0: x, y, p, u, v) and
 * write_complete_data (complete = 1: also the derivatives, analytic errors
 * and the per-element arrays; NULL ones are written as zeros) from host
 * arrays: point arrays of n_elements n_interp^2 values as ndg_get_solution
 * returns them, element arrays of n_elements values. No GPU needed. */
typedef struct ndg_output_arrays {
    int32_t complete;
    const double *x, *y, *p, *u, *v;
    const double *dp_dt, *du_dt, *dv_dt;
    const double *p_analytical_error, *u_analytical_error, *v_analytical_error;
    const int32_t* N;
    const int32_t *status, *rotation;
    int32_t rank;
    const double *p_error, *u_error, *v_error, *p_sigma, *u_sigma, *v_sigma;
    const int32_t *refine, *coarsen, *split_level;
} ndg_output_arrays;
ndg_status ndg_writer_write_arrays(ndg_writer* writer, double time, int64_t n_elements, int64_t n_interp, const ndg_output_arrays* arrays);
/* Mesh2D_t::write_data / write_complete_data (src/meshes/Mesh2D_t.cpp:1601-1642)
 * for one instance of a context: ndg_get_solution at `time`, and for the
 * complete output the element orders, Hilbert status and rotation, split
 * levels and the last error estimate (zeros when none is held, as the
 * reference's elements hold before their first estimate; the reference
 * estimates only the pressure, so the velocity errors and decay rates are
 * zeros). The time derivative is written as zeros unless the context keeps
 * it (ndg_ctx_keep_derivative). */
ndg_status ndg_writer_write(ndg_writer* writer, ndg_ctx* ctx, int32_t instance, double time, int32_t complete);

/* Solver2D_t::pre_condition and pre_condition_iterative
 * (include/solvers/Solver2D_t.tpp:136-334): RK3 steps of dt = get_delta_t
 * (never shortened) from time 0; after every pre_condition_interval-th step
 * the error is estimated and the mesh adapted, n_adaptivity_steps times.
 * iterative = 0 (sequential): the initial conditions are set once at the
 * end, on the adapted mesh; iterative = 1: after every adaptation the
 * initial conditions are set again and the time restarts from 0.
 * pre_condition_interval = 0 is rejected (the reference exits with 77).
 * Needs one instance. *n_steps (may be NULL) = the steps taken. */
ndg_status ndg_pre_condition(ndg_ctx* ctx, int64_t n_adaptivity_steps, int64_t pre_condition_interval, int32_t iterative, int64_t* n_steps);

/* ------------------------------------------------------------------------
 * Discrete adjoint. No counterpart in the reference, whose wave speed is the
 * constant c = 1 (include/helpers/constants.h:15); with c = 1 the operator
 * below is the reference's.
 *
 * Operator: a wave speed c_e > 0 per domain element in
 *   p_t + c (u_x + v_y) = 0,  u_t + c p_x = 0,  v_t + c p_y = 0:
 * the reference's fluxes x_flux = (c u, p, 0), y_flux = (c v, 0, p)
 * (src/solvers/Solver2D_t.cpp:31-37) become c_e (u, p, 0), c_e (v, 0, p)
 * inside element e, and its upwind face flux (Solver2D_t.cpp:48-63, with
 * w = p +- u.n) is multiplied by the face speed (c_left + c_right) / 2.
 * Time stepping: the reference's low-storage RK3 with a fixed step dt.
 * Meshes of one order with conforming faces (no adaptation since the load)
 * and wall, symmetry, outflow or periodic boundaries (inflow sides make the
 * step affine rather than linear and are rejected).
 *
 * Misfit: receivers at points (x_r, y_r) sample the pressure interpolated
 * in their element after every step n = 1..n_steps; with targets d[n][r],
 *   J = dt / 2 sum_n sum_r (p_r(t_n) - d[n][r])^2.
 * ndg_adjoint_backward returns dJ/d(p0, u0, v0) (the initial fields) and
 * dJ/dc (per element), the exact gradient of the discrete forward map (the
 * transpose of every stage, in reverse), with dt held fixed.
 * Memory: the forward keeps the state every checkpoint_interval steps and
 * the 3 checkpoint_interval stage inputs of its last interval; the backward
 * recomputes each earlier interval's stage inputs from its checkpoint, the
 * recomputation of interval j - 1 overlapping the adjoint stages over
 * interval j (two interval buffers when the memory allows, one otherwise). */
typedef struct ndg_adjoint ndg_adjoint;

/* An adjoint problem on the context's mesh, with n_receivers (at most 64)
 * receivers at receiver_xy[2 r], [2 r + 1]; the wave speed starts at 1. */
ndg_status ndg_adjoint_create(ndg_ctx* ctx, int32_t n_receivers, const double* receiver_xy, ndg_adjoint** out);
ndg_status ndg_adjoint_destroy(ndg_adjoint* adj);
/* Arithmetic of the adjoint problem's kernels: NDG_FP64 (default) or
 * NDG_FP32 (traces, fluxes, metrics, the volume term and their transposes
 * in FP32; states, RK updates, misfit and gradient accumulation in FP64). */
ndg_status ndg_adjoint_set_precision(ndg_adjoint* adj, int32_t precision);
/* Wave speed per domain element (n_elements values, all > 0). */
ndg_status ndg_adjoint_set_speed(ndg_adjoint* adj, const double* c);
/* The CFL step of the variable-speed operator: min over elements of
 * cfl * delta_xy_min / (N^2 c_e). */
ndg_status ndg_adjoint_delta_t(ndg_adjoint* adj, double cfl, double* delta_t);
/* Receivers: their element and reference coordinates (xi, eta); any pointer
 * may be NULL. */
ndg_status ndg_adjoint_receivers(const ndg_adjoint* adj, int64_t* element, double* xi_eta);
/* Forward solve from (p0, u0, v0) (field_size values each; u0 or v0 NULL =
 * zero) for n_steps steps of dt, keeping checkpoints every
 * checkpoint_interval steps (0: one interval). targets: (n_steps + 1) x
 * n_receivers values, row n for step n (row 0 unused); NULL = zero.
 * samples (optional, same shape) receives the receivers' pressure (row 0:
 * the initial state's). *misfit = J. */
ndg_status ndg_adjoint_forward(ndg_adjoint* adj, const double* p0, const double* u0, const double* v0, const double* targets,
                               double dt, int64_t n_steps, int64_t checkpoint_interval, double* samples, double* misfit);
/* Gradient of the last forward's misfit: grad_p0, grad_u0, grad_v0
 * (field_size values each) and grad_c (n_elements values); any may be
 * NULL. */
ndg_status ndg_adjoint_backward(ndg_adjoint* adj, double* grad_p0, double* grad_u0, double* grad_v0, double* grad_c);
/* The operator and its transpose on given states (3 field_size values each,
 * p then u then v): Lx = L(c) x, LTy = L(c)^T y, and dc[e] = d(y . L(c) x)/dc_e.
 * Any output may be NULL. For the transpose (dot-product) test. */
ndg_status ndg_adjoint_operator(ndg_adjoint* adj, const double* x, const double* y, double* Lx, double* LTy, double* dc);
/* Device time (CUDA events on the context's stream) of the last forward's
 * stepping and of the last backward's recompute + adjoint stepping, in ms,
 * and the kernel launches of each. Any pointer may be NULL. */
ndg_status ndg_adjoint_timings(const ndg_adjoint* adj, double* forward_ms, double* backward_ms, int64_t* forward_launches, int64_t* backward_launches);
/* Benchmark aid: mean duration (CUDA events) of n_launches back-to-back
 * launches of one kernel on the current state, after a forward and a
 * backward: which = 0 the forward stage, 1 the forward stage keeping its
 * input (the recomputation's), 2 the adjoint stage. The state advances; run
 * a new forward before the next backward. */
ndg_status ndg_adjoint_time_stage(ndg_adjoint* adj, int32_t which, int32_t n_launches, double* avg_ms);

#ifdef __cplusplus
}
#endif

#endif
