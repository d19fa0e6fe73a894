/* CPU restatement of the reference's DG spectral-element wave step
 * (NDG_cuda, SEM::Host::*), in plain C, FP64, single thread.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the tests, the smoke
 * check and the benchmark's CPU-baseline leg compare the CUDA path against.
 * The product library never links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks this restatement bit-for-bit
 * against the reference's own CPU path compiled from its sources
 * (oracle/_ref/libndgref.so) and against the reference's golden vectors
 * (tests/polynomials_test.cu:187,209 Legendre N=16 nodes/weights). */
#ifndef NDG_ORACLE_H
#define NDG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ndgo_ctx ndgo_ctx;

/* Tables: fills `out` with table `table` of order N for an NDG built with
 * N_max and n_interp output points; returns the number of values.
 * table: 0 nodes, 1 weights, 2 barycentric, 3 lagrange left, 4 lagrange right,
 * 5 lagrange derivative left, 6 lagrange derivative right, 7 derivative,
 * 8 cg derivative, 9 derivative hat, 10 interpolation, 11 polynomials. */
int ndgo_table(int N_max, int64_t n_interp, int table, int N, double* out);

/* Zone input, the in-memory form of one unstructured CGNS zone:
 * sec_type 0 = QUAD_4, 1 = BAR_2; sec_start/sec_end 1-based element numbers;
 * sec_conn concatenated 1-based node indices (4 or 2 per element);
 * boco_type 0 wall, 1 symmetry, 2 inflow, 3 outflow, 4 null; boco points are
 * 1-based element numbers; conn points/donors 1-based element numbers. */
ndgo_ctx* ndgo_create(int initial_N, int N_max, double cfl,
                      int64_t n_nodes, const double* x, const double* y,
                      int n_sections, const int* sec_type, const int64_t* sec_start, const int64_t* sec_end, const int64_t* sec_conn,
                      int n_bocos, const int* boco_type, const int64_t* boco_count, const int64_t* boco_points,
                      int n_conns, const int64_t* conn_count, const int64_t* conn_points, const int64_t* conn_donors);
void ndgo_destroy(ndgo_ctx* ctx);

void ndgo_counts(const ndgo_ctx* ctx, int64_t* n_elements, int64_t* n_elements_total, int64_t* n_faces, int64_t* n_nodes);
void ndgo_initial_conditions(ndgo_ctx* ctx);
double ndgo_get_delta_t(const ndgo_ctx* ctx);
void ndgo_stage(ndgo_ctx* ctx, int m, double time, double dt);
double ndgo_run(ndgo_ctx* ctx, int64_t n_steps, double time);

/* which: 0 p, 1 u, 2 v, 3 G_p, 4 G_u, 5 G_v, 6 k_p, 7 k_u, 8 k_v.
 * Element-by-element concatenation, (N+1)^2 values each, index i*(N+1)+j. */
int64_t ndgo_get_field(const ndgo_ctx* ctx, int which, double* out);
int64_t ndgo_set_field(ndgo_ctx* ctx, int which, const double* in);
void ndgo_element_N(const ndgo_ctx* ctx, int* N);

void ndgo_get_faces(const ndgo_ctx* ctx, int64_t* nodes, int64_t* elements, int64_t* sides, int* N, double* normal, double* tangent, double* offset, double* scale);
void ndgo_get_elements(const ndgo_ctx* ctx, int64_t* nodes, int* N, double* delta_xy_min, int64_t* first_face);
void ndgo_get_nodes(const ndgo_ctx* ctx, double* xy);
int64_t ndgo_get_boundary(const ndgo_ctx* ctx, int kind, int64_t* out);

void ndgo_estimate_error(ndgo_ctx* ctx, double tolerance_min, double tolerance_max);
void ndgo_get_error(const ndgo_ctx* ctx, double* p_error, double* p_sigma, int* refine, int* coarsen);
/* Mesh2D_t::get_complete_solution: out[11] = x, y, p, u, v, dp/dt, du/dt,
 * dv/dt, p/u/v analytic error on n_interp^2 points per element. */
int ndgo_complete_solution(const ndgo_ctx* ctx, int64_t n_interp, double time, double** out);
/* L2 error against the plane wave at `time`: out[3] for p, u, v. */
void ndgo_l2_error(const ndgo_ctx* ctx, double time, double* out);

/* Variable-speed operator (a wave speed per domain element: fluxes
 * c_e (u, p, 0), c_e (v, 0, p) and the upwind face flux times the mean of
 * the two sides' speeds; NULL restores the reference's constant c = 1) and
 * its discrete adjoint, for meshes of one order with conforming faces.
 * States: p, u, v blocks of field-size values each. */
void ndgo_set_speed(ndgo_ctx* ctx, const double* speed);
/* Lx = L(c) x (one stage's time derivative; boundary time 0). */
int ndgo_operator(ndgo_ctx* ctx, const double* x, double* Lx);
/* LTy = L(c)^T y and dc = d(y . L(c) x)/dc. Returns -1 on a non-conforming face. */
int ndgo_operator_transpose(ndgo_ctx* ctx, const double* x, const double* y, double* LTy, double* dc);
/* Forward solve of n_steps RK3 steps of dt from (p0, u0, v0) (u0, v0 may be
 * NULL) with receivers (element, (N+1)^2 interpolation weights each) sampled
 * after every step into samples ((n_steps+1) x n_rec, row 0 the initial
 * state), the misfit J = dt/2 sum (sample - target)^2 over steps 1..n_steps
 * (targets of the same shape, NULL = 0), and its gradient by the discrete
 * adjoint (every stage input kept in memory). Returns J. */
double ndgo_adjoint_solve(ndgo_ctx* ctx, const double* p0, const double* u0, const double* v0, double dt, int64_t n_steps,
                          int n_rec, const int64_t* rec_elem, const double* rec_w, const double* targets,
                          double* samples, double* grad_p, double* grad_u, double* grad_v, double* grad_c);

#ifdef __cplusplus
}
#endif

#endif
