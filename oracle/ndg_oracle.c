/* CPU restatement of the reference's DG spectral-element step for the 2D
 * first-order wave equation (NDG_cuda, SEM::Host::*), plain C, FP64.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the tests, the smoke check and
 * the benchmark's CPU-baseline leg. The product never links or calls it.
 *
 * Every loop keeps the reference's order of operations, and the file is
 * built without FMA contraction (oracle/Makefile), so on x86-64 it rounds
 * exactly as the reference's own CPU build does. Citations are paths inside
 * the reference repository. */
#include "ndg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NDGO_PI 3.14159265358979323846

/* ------------------------------------------------------------------ */
/* Polynomial tables                                                    */
/* ------------------------------------------------------------------ */

/* src/polynomials/LegendrePolynomial_t.cpp:8-32 (Algorithm 22). */
static void legendre_polynomial_and_derivative(int N, double x, double* L_N, double* L_N_prime) {
    if (N == 0) {
        *L_N = 1.0;
        *L_N_prime = 0.0;
    } else if (N == 1) {
        *L_N = x;
        *L_N_prime = 1.0;
    } else {
        double L_N_2 = 1.0, L_N_1 = x, L_N_2_prime = 0.0, L_N_1_prime = 1.0;
        for (int k = 2; k <= N; ++k) {
            *L_N = (2 * k - 1) * x * L_N_1 / k - (k - 1) * L_N_2 / k;
            *L_N_prime = L_N_2_prime + (2 * k - 1) * L_N_1;
            L_N_2 = L_N_1;
            L_N_1 = *L_N;
            L_N_2_prime = L_N_1_prime;
            L_N_1_prime = *L_N_prime;
        }
    }
}

/* src/polynomials/LegendrePolynomial_t.cpp:34-58. */
static double legendre_polynomial(int N, double x) {
    if (N == 0) return 1.0;
    if (N == 1) return x;
    double L_N_2 = 1.0, L_N_1 = x, L_N = 0.0;
    for (int k = 2; k <= N; ++k) {
        L_N = (2 * k - 1) * x * L_N_1 / k - (k - 1) * L_N_2 / k;
        L_N_2 = L_N_1;
        L_N_1 = L_N;
    }
    return L_N;
}

/* src/polynomials/LegendrePolynomial_t.cpp:60-101 (Algorithm 23):
 * Newton from the Chebyshev guess, at most 1000 iterations. */
static void legendre_nodes_and_weights(int N, double* nodes, double* weights) {
    for (int i = 0; i < (N + 1) / 2; ++i) {
        if (N == 1) {
            nodes[0] = -sqrt(1.0 / 3.0);
            weights[0] = 1.0;
            nodes[1] = -nodes[0];
            weights[1] = weights[0];
        } else {
            nodes[i] = -cos(NDGO_PI * (2 * i + 1) / (2 * N + 2));
            for (int k = 0; k < 1000; ++k) {
                double L, Lp;
                legendre_polynomial_and_derivative(N + 1, nodes[i], &L, &Lp);
                const double delta = -L / Lp;
                nodes[i] += delta;
                if (fabs(delta) <= DBL_MIN * 2 * fabs(nodes[i])) break;
            }
            double dummy, Lp_final;
            legendre_polynomial_and_derivative(N + 1, nodes[i], &dummy, &Lp_final);
            nodes[N - i] = -nodes[i];
            weights[i] = 2.0 / ((1 - pow(nodes[i], 2)) * pow(Lp_final, 2));
            weights[N - i] = weights[i];
        }
    }
    if (N == 0) {
        nodes[0] = 0.0;
        weights[0] = 2.0;
    }
    if (N % 2 == 0) {
        double dummy, Lp_final;
        legendre_polynomial_and_derivative(N + 1, 0.0, &dummy, &Lp_final);
        nodes[N / 2] = 0.0;
        weights[N / 2] = 2 / pow(Lp_final, 2);
    }
}

/* include/entities/NDG_t.tpp:200-208 (cppreference 2-ulp test). */
static int almost_equal(double x, double y) {
    return fabs(x - y) <= DBL_EPSILON * fabs(x + y) * 2 || fabs(x - y) < DBL_MIN;
}

typedef struct {
    int N_max;
    int64_t n_interp;
    double* t[12][33]; /* [table][N]; N_max <= 32 */
} ndgo_tables;

enum { T_NODES, T_WEIGHTS, T_BARY, T_LL, T_LR, T_DLL, T_DLR, T_D, T_DCG, T_DHAT, T_INTERP, T_POLY };

/* include/entities/NDG_t.tpp:10-59: the per-order table sequence. */
static int tables_build(ndgo_tables* T, int N_max, int64_t n_interp) {
    if (N_max < 0 || N_max > 32) return -1;
    memset(T, 0, sizeof(*T));
    T->N_max = N_max;
    T->n_interp = n_interp;
    for (int N = 0; N <= N_max; ++N) {
        const int n = N + 1;
        for (int k = 0; k < 12; ++k) {
            size_t sz = (k >= T_D && k <= T_DHAT) || k == T_POLY ? (size_t)(n * n) : (k == T_INTERP ? (size_t)(n * n_interp) : (size_t)n);
            T->t[k][N] = (double*)calloc(sz > 0 ? sz : 1, sizeof(double));
        }
        double* x = T->t[T_NODES][N];
        double* w = T->t[T_WEIGHTS][N];
        double* bw = T->t[T_BARY][N];
        double* D = T->t[T_D][N];
        legendre_nodes_and_weights(N, x, w);
        /* NDG_t.tpp:176-188 (Algorithm 30) */
        for (int j = 0; j <= N; ++j) {
            double xjxi = 1.0;
            for (int i = 0; i < j; ++i) xjxi *= x[j] - x[i];
            for (int i = j + 1; i <= N; ++i) xjxi *= x[j] - x[i];
            bw[j] = 1.0 / xjxi;
        }
        /* NDG_t.tpp:328-334 */
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N; ++j)
                T->t[T_POLY][N][i * n + j] = legendre_polynomial(i, x[j]) * w[j] * (2 * i + 1) * 0.5;
        /* NDG_t.tpp:252-261 (Algorithm 37, off-diagonal) */
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N; ++j)
                if (i != j) D[i * n + j] = bw[j] / (bw[i] * (x[i] - x[j]));
        /* NDG_t.tpp:301-325 */
        for (int64_t j = 0; j < n_interp; ++j) {
            int row_has_match = 0;
            const double xc = 2.0 * j / (n_interp - 1) - 1.0;
            double* row = T->t[T_INTERP][N] + j * n;
            for (int k = 0; k <= N; ++k) {
                row[k] = 0.0;
                if (almost_equal(xc, x[k])) {
                    row[k] = 1.0;
                    row_has_match = 1;
                }
            }
            if (!row_has_match) {
                double total = 0.0;
                for (int k = 0; k <= N; ++k) {
                    row[k] = bw[k] / (xc - x[k]);
                    total += row[k];
                }
                for (int k = 0; k <= N; ++k) row[k] /= total;
            }
        }
        /* NDG_t.tpp:210-228 (Algorithm 34) and :230-250 (Algorithm 36) */
        for (int side = 0; side < 2; ++side) {
            const double xs = side == 0 ? -1.0 : 1.0;
            double* l = T->t[side == 0 ? T_LL : T_LR][N];
            double* dl = T->t[side == 0 ? T_DLL : T_DLR][N];
            for (int i = 0; i <= N; ++i) l[i] = bw[i] / (xs - x[i]);
            for (int i = 0; i <= N; ++i) dl[i] = bw[i] / ((xs - x[i]) * (xs - x[i]));
        }
        for (int side = 0; side < 2; ++side) {
            double* l = T->t[side == 0 ? T_LL : T_LR][N];
            double sum = 0.0;
            for (int i = 0; i <= N; ++i) sum += l[i];
            for (int i = 0; i <= N; ++i) l[i] /= sum;
        }
        for (int side = 0; side < 2; ++side) {
            const double xs = side == 0 ? -1.0 : 1.0;
            double* dl = T->t[side == 0 ? T_DLL : T_DLR][N];
            double sum = 0.0;
            for (int i = 0; i <= N; ++i) sum += bw[i] / (xs - x[i]);
            for (int i = 0; i <= N; ++i) dl[i] /= sum;
        }
        /* NDG_t.tpp:263-274 (diagonal, negative row sum) */
        for (int i = 0; i <= N; ++i) {
            D[i * (N + 2)] = 0.0;
            for (int j = 0; j < i; ++j) D[i * (N + 2)] -= D[i * n + j];
            for (int j = i + 1; j <= N; ++j) D[i * (N + 2)] -= D[i * n + j];
        }
        /* NDG_t.tpp:287-298 (Algorithm 57) */
        for (int j = 0; j <= N; ++j)
            for (int m = 0; m <= N; ++m) {
                double s = 0.0;
                for (int k = 0; k <= N; ++k) s += D[k * n + m] * D[k * n + j] * w[k];
                T->t[T_DCG][N][j * n + m] = s / w[j];
            }
        /* NDG_t.tpp:277-284 */
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N; ++j)
                T->t[T_DHAT][N][i * n + j] = -D[j * n + i] * w[j] / w[i];
    }
    return 0;
}

static void tables_free(ndgo_tables* T) {
    for (int k = 0; k < 12; ++k)
        for (int N = 0; N <= T->N_max; ++N) free(T->t[k][N]);
}

int ndgo_table(int N_max, int64_t n_interp, int table, int N, double* out) {
    ndgo_tables T;
    if (table < 0 || table > 11 || N < 0 || N > N_max) return -1;
    if (tables_build(&T, N_max, n_interp) != 0) return -1;
    const int n = N + 1;
    const int count = (table >= T_D && table <= T_DHAT) || table == T_POLY ? n * n : (table == T_INTERP ? (int)(n * n_interp) : n);
    memcpy(out, T.t[table][N], (size_t)count * sizeof(double));
    tables_free(&T);
    return count;
}

/* ------------------------------------------------------------------ */
/* Mesh                                                                 */
/* ------------------------------------------------------------------ */

struct ndgo_ctx {
    ndgo_tables T;
    double cfl;
    /* nodes */
    int64_t n_nodes;
    double* nx;
    double* ny;
    /* elements: domain first, then ghost (boundary) elements */
    int64_t n_elem;       /* domain */
    int64_t n_elem_total; /* domain + ghosts */
    int* eN;
    int64_t* enodes;     /* 4 per element */
    int64_t* eface;      /* first face per side (4 per element), -1 if none */
    int* eface_cnt;      /* faces per side (always 1 or 0 here: conforming input) */
    int64_t* off2;       /* offset of the element's (N+1)^2 block */
    int64_t* off1;       /* offset of the element's 4*(N+1) side block */
    double *xi_x, *eta_x, *xi_y, *eta_y, *jac; /* named as the reference: dxi_dx_ etc. */
    double* sf;                                  /* scaling_factor_, 4 sides */
    double* dxy_min;
    double* center;
    double *p, *u, *v, *Gp, *Gu, *Gv, *kp, *ku, *kv;
    double *pe, *ue, *ve;    /* p/u/v_extrapolated_, 4 sides */
    double *pfe, *ufe, *vfe; /* p/u/v_flux_extrapolated_, 4 sides */
    double* p_error;
    double* p_sigma;
    int* refine;
    int* coarsen;
    /* faces */
    int64_t n_faces;
    int* fN;
    int64_t* fnodes;
    int64_t* felem;
    int64_t* fside;
    double *normal, *tangent, *length, *offset, *scale;
    int64_t* foff; /* offset of the face's N+1 block */
    double *fp0, *fp1, *fu0, *fu1, *fv0, *fv1, *fluxp, *fluxu, *fluxv;
    /* boundaries */
    int64_t nb[4];
    int64_t* blist[4]; /* wall, symmetry, inflow, outflow */
    int64_t n_if;
    int64_t *if_origin, *if_origin_side, *if_dest;
    /* variable-speed operator (NULL: the reference's constant c = 1):
     * speed per domain element, and per element (ghosts included) the
     * domain element whose speed it carries */
    double* speed;
    int64_t* speed_owner;
};

static void* xcalloc(size_t n, size_t sz) { return calloc(n > 0 ? n : 1, sz); }

/* include/functions/quad_metrics.tpp:2-7 (Algorithm 100). m[0] = (x_xi, x_eta), m[1] = (y_xi, y_eta). */
static void quad_metrics(double xi, double eta, const double* px, const double* py, double m[2][2]) {
    m[0][0] = ((1 - eta) * (px[1] - px[0]) + (1 + eta) * (px[2] - px[3])) / 4;
    m[0][1] = ((1 - xi) * (px[3] - px[0]) + (1 + xi) * (px[2] - px[1])) / 4;
    m[1][0] = ((1 - eta) * (py[1] - py[0]) + (1 + eta) * (py[2] - py[3])) / 4;
    m[1][1] = ((1 - xi) * (py[3] - py[0]) + (1 + xi) * (py[2] - py[1])) / 4;
}

/* include/functions/quad_map.tpp:2-7 (Algorithm 95), per component with the
 * reference's Vec2 evaluation order. */
static void quad_map(double xi, double eta, const double* px, const double* py, double* gx, double* gy) {
    *gx = (px[0] * (1 - xi) * (1 - eta) + px[1] * (xi + 1) * (1 - eta) + px[2] * (xi + 1) * (eta + 1) + px[3] * (1 - xi) * (eta + 1)) / 4;
    *gy = (py[0] * (1 - xi) * (1 - eta) + py[1] * (xi + 1) * (1 - eta) + py[2] * (xi + 1) * (eta + 1) + py[3] * (1 - xi) * (eta + 1)) / 4;
}

static double magnitude(double x, double y) { return sqrt(x * x + y * y); }

/* include/helpers/constants.h:15-18 and include/functions/analytical_solution.tpp:4-10. */
static const double C_c = 1;
static const double C_xy0x = -0.2, C_xy0y = -0.2;
static const double C_kx = 0.707106781186548, C_ky = 0.707106781186548;
static const double C_d = 0.120112240878645;

static void analytic_g(double x, double y, double t, double* p, double* u, double* v) {
    const double a = C_kx * (x - C_xy0x) + C_ky * (y - C_xy0y) - C_c * t;
    *p = exp(-a * a / (C_d * C_d));
    *u = *p * C_kx / C_c;
    *v = *p * C_ky / C_c;
}

static int64_t section_of(int n_sections, const int64_t* start, const int64_t* end, int64_t elem) {
    for (int k = 0; k < n_sections; ++k)
        if (elem >= start[k] && elem <= end[k]) return k;
    return -1;
}

ndgo_ctx* ndgo_create(int initial_N, int N_max, double cfl,
                      int64_t n_nodes, const double* x, const double* y,
                      int n_sections, const int* sec_type, const int64_t* sec_start, const int64_t* sec_end, const int64_t* sec_conn,
                      int n_bocos, const int* boco_type, const int64_t* boco_count, const int64_t* boco_points,
                      int n_conns, const int64_t* conn_count, const int64_t* conn_points, const int64_t* conn_donors) {
    if (initial_N < 0 || initial_N > N_max) return NULL;
    ndgo_ctx* c = (ndgo_ctx*)calloc(1, sizeof(ndgo_ctx));
    if (!c || tables_build(&c->T, N_max, 2) != 0) {
        free(c);
        return NULL;
    }
    c->cfl = cfl;
    c->n_nodes = n_nodes;
    c->nx = (double*)xcalloc((size_t)n_nodes, sizeof(double));
    c->ny = (double*)xcalloc((size_t)n_nodes, sizeof(double));
    memcpy(c->nx, x, (size_t)n_nodes * sizeof(double));
    memcpy(c->ny, y, (size_t)n_nodes * sizeof(double));

    /* Mesh2D_t.cpp:658-713: domain QUAD_4 sections first, then BAR_2 ghosts. */
    int64_t n_dom = 0, n_ghost = 0;
    for (int k = 0; k < n_sections; ++k) {
        if (sec_type[k] == 0) n_dom += sec_end[k] - sec_start[k] + 1;
        else n_ghost += sec_end[k] - sec_start[k] + 1;
    }
    const int64_t ne = n_dom + n_ghost;
    c->n_elem = n_dom;
    c->n_elem_total = ne;
    c->eN = (int*)xcalloc((size_t)ne, sizeof(int));
    c->enodes = (int64_t*)xcalloc((size_t)(4 * ne), sizeof(int64_t));
    int64_t* sec_first = (int64_t*)xcalloc((size_t)n_sections, sizeof(int64_t));
    {
        int64_t dom_i = 0, ghost_i = n_dom, conn_off = 0;
        for (int k = 0; k < n_sections; ++k) {
            const int64_t cnt = sec_end[k] - sec_start[k] + 1;
            if (sec_type[k] == 0) {
                sec_first[k] = dom_i;
                for (int64_t j = 0; j < cnt; ++j) {
                    const int64_t e = dom_i + j;
                    c->eN[e] = initial_N;
                    for (int q = 0; q < 4; ++q) c->enodes[4 * e + q] = sec_conn[conn_off + 4 * j + q] - 1;
                }
                dom_i += cnt;
                conn_off += 4 * cnt;
            } else {
                sec_first[k] = ghost_i;
                for (int64_t j = 0; j < cnt; ++j) {
                    const int64_t e = ghost_i + j;
                    c->eN[e] = initial_N;
                    c->enodes[4 * e + 0] = sec_conn[conn_off + 2 * j] - 1;
                    c->enodes[4 * e + 1] = sec_conn[conn_off + 2 * j + 1] - 1;
                    c->enodes[4 * e + 2] = sec_conn[conn_off + 2 * j + 1] - 1;
                    c->enodes[4 * e + 3] = sec_conn[conn_off + 2 * j] - 1;
                }
                ghost_i += cnt;
                conn_off += 2 * cnt;
            }
        }
    }

    /* Mesh2D_t.cpp:1110-1190 (build_faces): faces in first-seen order over the
     * domain elements; a face seen again in reverse gets its right element;
     * ghosts attach as right elements, swapping their nodes when needed. */
    int64_t* e2f = (int64_t*)xcalloc((size_t)(4 * ne), sizeof(int64_t));
    int64_t cap = 4 * ne;
    c->fnodes = (int64_t*)xcalloc((size_t)(2 * cap), sizeof(int64_t));
    c->felem = (int64_t*)xcalloc((size_t)(2 * cap), sizeof(int64_t));
    c->fside = (int64_t*)xcalloc((size_t)(2 * cap), sizeof(int64_t));
    /* node -> faces adjacency, as growable lists */
    int64_t* n2f_cnt = (int64_t*)xcalloc((size_t)n_nodes, sizeof(int64_t));
    int64_t* n2f_cap = (int64_t*)xcalloc((size_t)n_nodes, sizeof(int64_t));
    int64_t** n2f = (int64_t**)xcalloc((size_t)n_nodes, sizeof(int64_t*));
#define N2F_PUSH(node, face)                                                              \
    do {                                                                                  \
        int64_t nd_ = (node);                                                             \
        if (n2f_cnt[nd_] == n2f_cap[nd_]) {                                               \
            n2f_cap[nd_] = n2f_cap[nd_] ? 2 * n2f_cap[nd_] : 4;                           \
            n2f[nd_] = (int64_t*)realloc(n2f[nd_], (size_t)n2f_cap[nd_] * sizeof(int64_t)); \
        }                                                                                 \
        n2f[nd_][n2f_cnt[nd_]++] = (face);                                                \
    } while (0)
    int64_t nf = 0;
    for (int64_t i = 0; i < n_dom; ++i) {
        for (int j = 0; j < 4; ++j) {
            const int64_t a = c->enodes[4 * i + j];
            const int64_t b = c->enodes[4 * i + (j + 1 < 4 ? j + 1 : 0)];
            int found = 0;
            for (int64_t q = 0; q < n2f_cnt[a]; ++q) {
                const int64_t f = n2f[a][q];
                if (c->fnodes[2 * f] == b && c->fnodes[2 * f + 1] == a) {
                    found = 1;
                    c->felem[2 * f + 1] = i;
                    c->fside[2 * f + 1] = j;
                    e2f[4 * i + j] = f;
                    break;
                }
            }
            if (!found) {
                e2f[4 * i + j] = nf;
                N2F_PUSH(a, nf);
                if (b != a) N2F_PUSH(b, nf);
                c->fnodes[2 * nf] = a;
                c->fnodes[2 * nf + 1] = b;
                c->felem[2 * nf] = i;
                c->felem[2 * nf + 1] = -1;
                c->fside[2 * nf] = j;
                c->fside[2 * nf + 1] = -1;
                ++nf;
            }
        }
    }
    for (int64_t i = n_dom; i < ne; ++i) {
        const int64_t a = c->enodes[4 * i], b = c->enodes[4 * i + 1];
        for (int64_t q = 0; q < n2f_cnt[a]; ++q) {
            const int64_t f = n2f[a][q];
            if (c->fnodes[2 * f] == b && c->fnodes[2 * f + 1] == a) {
                c->felem[2 * f + 1] = i;
                c->fside[2 * f + 1] = 0;
                e2f[4 * i] = f;
                for (int s = 1; s < 4; ++s) e2f[4 * i + s] = -1;
                break;
            }
            if (c->fnodes[2 * f] == a && c->fnodes[2 * f + 1] == b) {
                c->felem[2 * f + 1] = i;
                c->fside[2 * f + 1] = 0;
                e2f[4 * i] = f;
                for (int s = 1; s < 4; ++s) e2f[4 * i + s] = -1;
                c->enodes[4 * i] = b;
                c->enodes[4 * i + 1] = a;
                break;
            }
        }
    }
    for (int64_t nd = 0; nd < n_nodes; ++nd) free(n2f[nd]);
    free(n2f);
    free(n2f_cnt);
    free(n2f_cap);
    c->n_faces = nf;

    /* Mesh2D_t.cpp:725-816: boundary lists, section-relative element numbers. */
    {
        int64_t off = 0;
        for (int k = 0; k < 4; ++k) c->nb[k] = 0;
        for (int bc = 0; bc < n_bocos; ++bc)
            if (boco_type[bc] >= 0 && boco_type[bc] < 4) c->nb[boco_type[bc]] += boco_count[bc];
        for (int k = 0; k < 4; ++k) {
            c->blist[k] = (int64_t*)xcalloc((size_t)c->nb[k], sizeof(int64_t));
            c->nb[k] = 0;
        }
        for (int bc = 0; bc < n_bocos; ++bc) {
            const int t = boco_type[bc];
            for (int64_t j = 0; j < boco_count[bc]; ++j) {
                const int64_t el = boco_points[off + j];
                if (t >= 0 && t < 4) {
                    const int64_t s = section_of(n_sections, sec_start, sec_end, el);
                    c->blist[t][c->nb[t]++] = sec_first[s] + el - sec_start[s];
                }
            }
            off += boco_count[bc];
        }
    }
    /* Mesh2D_t.cpp:818-875: self interfaces (periodic), origin = the domain
     * element next to the donor ghost, destination = the receiving ghost. */
    {
        int64_t total = 0;
        for (int k = 0; k < n_conns; ++k) total += conn_count[k];
        c->n_if = total;
        c->if_origin = (int64_t*)xcalloc((size_t)total, sizeof(int64_t));
        c->if_origin_side = (int64_t*)xcalloc((size_t)total, sizeof(int64_t));
        c->if_dest = (int64_t*)xcalloc((size_t)total, sizeof(int64_t));
        int64_t off = 0;
        for (int k = 0; k < n_conns; ++k) {
            for (int64_t j = 0; j < conn_count[k]; ++j) {
                const int64_t el = conn_points[off + j], donor = conn_donors[off + j];
                const int64_t so = section_of(n_sections, sec_start, sec_end, el);
                const int64_t sd = section_of(n_sections, sec_start, sec_end, donor);
                const int64_t donor_ghost = sec_first[sd] + donor - sec_start[sd];
                const int64_t f = e2f[4 * donor_ghost];
                const int64_t fs = c->felem[2 * f] == donor_ghost;
                c->if_origin[off + j] = c->felem[2 * f + fs];
                c->if_origin_side[off + j] = c->fside[2 * f + fs];
                c->if_dest[off + j] = sec_first[so] + el - sec_start[so];
            }
            off += conn_count[k];
        }
    }
    free(sec_first);

    /* Storage (Element2D_t.cpp:648-735, Face2D_t.cpp:36-43) and the face list
     * per side (Mesh2D_t.cpp:4186-4206). */
    c->eface = (int64_t*)xcalloc((size_t)(4 * ne), sizeof(int64_t));
    c->eface_cnt = (int*)xcalloc((size_t)(4 * ne), sizeof(int));
    for (int64_t e = 0; e < ne; ++e)
        for (int s = 0; s < 4; ++s) {
            if (e < n_dom || s == 0) {
                c->eface[4 * e + s] = e2f[4 * e + s];
                c->eface_cnt[4 * e + s] = 1;
            } else {
                c->eface[4 * e + s] = -1;
                c->eface_cnt[4 * e + s] = 0;
            }
        }
    free(e2f);
    c->off2 = (int64_t*)xcalloc((size_t)ne, sizeof(int64_t));
    c->off1 = (int64_t*)xcalloc((size_t)ne, sizeof(int64_t));
    int64_t s2 = 0, s1 = 0;
    for (int64_t e = 0; e < ne; ++e) {
        const int64_t n = c->eN[e] + 1;
        c->off2[e] = s2;
        c->off1[e] = s1;
        s2 += n * n;
        s1 += 4 * n;
    }
    double** arr2[] = {&c->xi_x, &c->eta_x, &c->xi_y, &c->eta_y, &c->jac, &c->p, &c->u, &c->v, &c->Gp, &c->Gu, &c->Gv, &c->kp, &c->ku, &c->kv};
    for (size_t k = 0; k < sizeof(arr2) / sizeof(arr2[0]); ++k) *arr2[k] = (double*)xcalloc((size_t)s2, sizeof(double));
    double** arr1[] = {&c->sf, &c->pe, &c->ue, &c->ve, &c->pfe, &c->ufe, &c->vfe};
    for (size_t k = 0; k < sizeof(arr1) / sizeof(arr1[0]); ++k) *arr1[k] = (double*)xcalloc((size_t)s1, sizeof(double));
    c->dxy_min = (double*)xcalloc((size_t)ne, sizeof(double));
    c->center = (double*)xcalloc((size_t)(2 * ne), sizeof(double));
    c->p_error = (double*)xcalloc((size_t)ne, sizeof(double));
    c->p_sigma = (double*)xcalloc((size_t)ne, sizeof(double));
    c->refine = (int*)xcalloc((size_t)ne, sizeof(int));
    c->coarsen = (int*)xcalloc((size_t)ne, sizeof(int));

    c->fN = (int*)xcalloc((size_t)nf, sizeof(int));
    c->foff = (int64_t*)xcalloc((size_t)nf, sizeof(int64_t));
    int64_t sfc = 0;
    for (int64_t f = 0; f < nf; ++f) {
        c->fN[f] = initial_N;
        c->foff[f] = sfc;
        sfc += initial_N + 1;
    }
    double** arrf[] = {&c->fp0, &c->fp1, &c->fu0, &c->fu1, &c->fv0, &c->fv1, &c->fluxp, &c->fluxu, &c->fluxv};
    for (size_t k = 0; k < sizeof(arrf) / sizeof(arrf[0]); ++k) *arrf[k] = (double*)xcalloc((size_t)sfc, sizeof(double));
    c->normal = (double*)xcalloc((size_t)(2 * nf), sizeof(double));
    c->tangent = (double*)xcalloc((size_t)(2 * nf), sizeof(double));
    c->length = (double*)xcalloc((size_t)nf, sizeof(double));
    c->offset = (double*)xcalloc((size_t)(2 * nf), sizeof(double));
    c->scale = (double*)xcalloc((size_t)(2 * nf), sizeof(double));

    /* Element2D_t.cpp:743-777 (compute_geometry), domain elements. */
    for (int64_t e = 0; e < n_dom; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* xn = c->T.t[T_NODES][N];
        double px[4], py[4];
        for (int q = 0; q < 4; ++q) {
            px[q] = c->nx[c->enodes[4 * e + q]];
            py[q] = c->ny[c->enodes[4 * e + q]];
        }
        double* sf = c->sf + c->off1[e];
        for (int i = 0; i <= N; ++i) {
            for (int j = 0; j <= N; ++j) {
                double m[2][2];
                quad_metrics(xn[i], xn[j], px, py, m);
                const int64_t k = c->off2[e] + i * n + j;
                c->xi_x[k] = m[0][0];
                c->eta_x[k] = m[0][1];
                c->xi_y[k] = m[1][0];
                c->eta_y[k] = m[1][1];
                c->jac[k] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
            }
            double mb[2][2], mr[2][2], mt[2][2], ml[2][2];
            quad_metrics(xn[i], -1.0, px, py, mb);
            quad_metrics(1.0, xn[i], px, py, mr);
            quad_metrics(xn[i], 1.0, px, py, mt);
            quad_metrics(-1.0, xn[i], px, py, ml);
            sf[0 * n + i] = sqrt(mb[0][0] * mb[0][0] + mb[1][0] * mb[1][0]);
            sf[1 * n + i] = sqrt(mr[0][1] * mr[0][1] + mr[1][1] * mr[1][1]);
            sf[2 * n + i] = sqrt(mt[0][0] * mt[0][0] + mt[1][0] * mt[1][0]);
            sf[3 * n + i] = sqrt(ml[0][1] * ml[0][1] + ml[1][1] * ml[1][1]);
        }
        const double d01 = magnitude(px[1] - px[0], py[1] - py[0]);
        const double d23 = magnitude(px[2] - px[3], py[2] - py[3]);
        const double d12 = magnitude(px[1] - px[2], py[1] - py[2]);
        const double d03 = magnitude(px[0] - px[3], py[0] - py[3]);
        const double d13 = magnitude(px[1] - px[3], py[1] - py[3]);
        const double d20 = magnitude(px[2] - px[0], py[2] - py[0]);
        c->dxy_min[e] = fmin(fmin(fmin(d01, d23), fmin(d12, d03)), fmin(d13, d20));
        c->center[2 * e] = (px[0] + px[1] + px[2] + px[3]) / 4;
        c->center[2 * e + 1] = (py[0] + py[1] + py[2] + py[3]) / 4;
    }
    /* Element2D_t.cpp:779-790 (compute_boundary_geometry), ghosts. */
    for (int64_t e = n_dom; e < ne; ++e) {
        const int N = c->eN[e];
        const double* xn = c->T.t[T_NODES][N];
        double px[4], py[4];
        for (int q = 0; q < 4; ++q) {
            px[q] = c->nx[c->enodes[4 * e + q]];
            py[q] = c->ny[c->enodes[4 * e + q]];
        }
        for (int i = 0; i <= N; ++i) {
            double mb[2][2];
            quad_metrics(xn[i], -1.0, px, py, mb);
            c->sf[c->off1[e] + i] = sqrt(mb[0][0] * mb[0][0] + mb[1][0] * mb[1][0]);
        }
        c->dxy_min[e] = magnitude(px[1] - px[0], py[1] - py[0]);
        c->center[2 * e] = (px[0] + px[1]) / 2;
        c->center[2 * e + 1] = (py[0] + py[1]) / 2;
    }
    /* Mesh2D_t.cpp:4208-4235 and Face2D_t.cpp:56-81 (face geometry). */
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t eL = c->felem[2 * f], eR = c->felem[2 * f + 1];
        const int64_t sL = c->fside[2 * f], sR = c->fside[2 * f + 1];
        const int64_t nL = c->enodes[4 * eL + sL], nL1 = c->enodes[4 * eL + (sL + 1 < 4 ? sL + 1 : 0)];
        const int64_t nR = c->enodes[4 * eR + sR], nR1 = c->enodes[4 * eR + (sR + 1 < 4 ? sR + 1 : 0)];
        const double f0x = c->nx[c->fnodes[2 * f]], f0y = c->ny[c->fnodes[2 * f]];
        const double f1x = c->nx[c->fnodes[2 * f + 1]], f1y = c->ny[c->fnodes[2 * f + 1]];
        double tx = f1x - f0x, ty = f1y - f0y;
        const double len = magnitude(tx, ty);
        tx /= len;
        ty /= len;
        double nxv = ty, nyv = -tx;
        const double eLdx = c->nx[nL1] - c->nx[nL], eLdy = c->ny[nL1] - c->ny[nL];
        const double sign = copysign(1.0, tx * eLdx + ty * eLdy);
        nxv *= sign;
        nyv *= sign;
        tx *= sign;
        ty *= sign;
        const double eRdx = c->nx[nR1] - c->nx[nR], eRdy = c->ny[nR1] - c->ny[nR];
        const double fdx = f1x - f0x, fdy = f1y - f0y;
        c->length[f] = len;
        c->normal[2 * f] = nxv;
        c->normal[2 * f + 1] = nyv;
        c->tangent[2 * f] = tx;
        c->tangent[2 * f + 1] = ty;
        c->offset[2 * f] = magnitude(f0x - c->nx[nL], f0y - c->ny[nL]) / magnitude(eLdx, eLdy);
        c->offset[2 * f + 1] = magnitude(f1x - c->nx[nR], f1y - c->ny[nR]) / magnitude(eRdx, eRdy);
        c->scale[2 * f] = magnitude(fdx, fdy) / magnitude(eLdx, eLdy);
        c->scale[2 * f + 1] = magnitude(fdx, fdy) / magnitude(eRdx, eRdy);
    }
    return c;
}

void ndgo_destroy(ndgo_ctx* c) {
    if (!c) return;
    tables_free(&c->T);
    void* ptrs[] = {c->nx, c->ny, c->eN, c->enodes, c->eface, c->eface_cnt, c->off2, c->off1, c->xi_x, c->eta_x, c->xi_y, c->eta_y, c->jac, c->sf, c->dxy_min, c->center,
                    c->p, c->u, c->v, c->Gp, c->Gu, c->Gv, c->kp, c->ku, c->kv, c->pe, c->ue, c->ve, c->pfe, c->ufe, c->vfe, c->p_error, c->p_sigma, c->refine, c->coarsen,
                    c->fN, c->fnodes, c->felem, c->fside, c->normal, c->tangent, c->length, c->offset, c->scale, c->foff,
                    c->fp0, c->fp1, c->fu0, c->fu1, c->fv0, c->fv1, c->fluxp, c->fluxu, c->fluxv,
                    c->blist[0], c->blist[1], c->blist[2], c->blist[3], c->if_origin, c->if_origin_side, c->if_dest,
                    c->speed, c->speed_owner};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
    free(c);
}

void ndgo_counts(const ndgo_ctx* c, int64_t* n_elements, int64_t* n_elements_total, int64_t* n_faces, int64_t* n_nodes) {
    *n_elements = c->n_elem;
    *n_elements_total = c->n_elem_total;
    *n_faces = c->n_faces;
    *n_nodes = c->n_nodes;
}

/* Mesh2D_t.cpp:1192-1216 (initial_conditions). */
void ndgo_initial_conditions(ndgo_ctx* c) {
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* xn = c->T.t[T_NODES][N];
        double px[4], py[4];
        for (int q = 0; q < 4; ++q) {
            px[q] = c->nx[c->enodes[4 * e + q]];
            py[q] = c->ny[c->enodes[4 * e + q]];
        }
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N; ++j) {
                double gx, gy, p, u, v;
                quad_map(xn[i], xn[j], px, py, &gx, &gy);
                analytic_g(gx, gy, 0.0, &p, &u, &v);
                const int64_t k = c->off2[e] + i * n + j;
                c->p[k] = p;
                c->u[k] = u;
                c->v[k] = v;
                c->Gp[k] = 0;
                c->Gu[k] = 0;
                c->Gv[k] = 0;
            }
    }
}

/* src/solvers/Solver2D_t.cpp:19-29 (get_delta_t), one rank. */
double ndgo_get_delta_t(const ndgo_ctx* c) {
    double dt = INFINITY;
    for (int64_t e = 0; e < c->n_elem; ++e) dt = fmin(c->cfl * c->dxy_min[e] / (c->eN[e] * c->eN[e] * C_c), dt);
    return dt;
}

/* Element2D_t.cpp:86-125 (interpolate_to_boundaries). */
static void interpolate_to_boundaries(ndgo_ctx* c) {
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* lm = c->T.t[T_LL][N];
        const double* lp = c->T.t[T_LR][N];
        const double* q[3] = {c->p + c->off2[e], c->u + c->off2[e], c->v + c->off2[e]};
        double* ex[3] = {c->pe + c->off1[e], c->ue + c->off1[e], c->ve + c->off1[e]};
        for (int i = 0; i <= N; ++i) {
            for (int f = 0; f < 3; ++f) {
                ex[f][0 * n + i] = 0.0;
                ex[f][2 * n + N - i] = 0.0;
                ex[f][1 * n + i] = 0.0;
                ex[f][3 * n + N - i] = 0.0;
            }
            for (int j = 0; j <= N; ++j)
                for (int f = 0; f < 3; ++f) {
                    ex[f][0 * n + i] += lm[j] * q[f][i * n + j];
                    ex[f][2 * n + N - i] += lp[j] * q[f][i * n + j];
                    ex[f][1 * n + i] += lp[j] * q[f][j * n + i];
                    ex[f][3 * n + N - i] += lm[j] * q[f][j * n + i];
                }
        }
    }
}

/* The ghost-trace projection shared by the wall, symmetry and outflow
 * boundaries (Mesh2D_t.cpp:4366-4424, the multi-face branch, which is the one
 * that runs because a ghost's side-0 face list is never empty), followed by
 * the velocity mirror of the wall/symmetry boundaries (:4426-4434). */
static void ghost_projection(ndgo_ctx* c, int64_t ge, int mirror) {
    const int N = c->eN[ge];
    const double* xe = c->T.t[T_NODES][N];
    const double* we = c->T.t[T_WEIGHTS][N];
    const double* bwe = c->T.t[T_BARY][N];
    double* gp = c->pe + c->off1[ge];
    double* gu = c->ue + c->off1[ge];
    double* gv = c->ve + c->off1[ge];
    const double* sf = c->sf + c->off1[ge];
    for (int i = 0; i <= N; ++i) gp[i] = gu[i] = gv[i] = 0.0;
    for (int fi = 0; fi < c->eface_cnt[4 * ge]; ++fi) {
        const int64_t f = c->eface[4 * ge + fi];
        const int fs = c->felem[2 * f] == ge;
        const int64_t nb = c->felem[2 * f + fs];
        const int64_t nbs = c->fside[2 * f + fs];
        const int Nn = c->eN[nb], nn = Nn + 1;
        const double* xnb = c->T.t[T_NODES][Nn];
        const double* wnb = c->T.t[T_WEIGHTS][Nn];
        const double* np_ = c->pe + c->off1[nb] + nbs * nn;
        const double* nu_ = c->ue + c->off1[nb] + nbs * nn;
        const double* nv_ = c->ve + c->off1[nb] + nbs * nn;
        for (int j = 0; j <= Nn; ++j) {
            const double coord = (xnb[Nn - j] + 1) * c->scale[2 * f + fs] + 2 * c->offset[2 * f + fs] - 1;
            int found = 0;
            for (int i = 0; i <= N; ++i) {
                if (almost_equal(coord, xe[i])) {
                    gp[i] += wnb[j] / we[i] * np_[j] * sf[i];
                    gu[i] += wnb[j] / we[i] * nu_[j] * sf[i];
                    gv[i] += wnb[j] / we[i] * nv_[j] * sf[i];
                    found = 1;
                    break;
                }
            }
            if (!found) {
                double s = 0.0;
                for (int i = 0; i <= N; ++i) s += bwe[i] / (coord - xe[i]);
                for (int i = 0; i <= N; ++i) {
                    const double T = bwe[i] / ((coord - xe[i]) * s);
                    gp[i] += T * wnb[j] / we[i] * np_[j] * sf[i];
                    gu[i] += T * wnb[j] / we[i] * nu_[j] * sf[i];
                    gv[i] += T * wnb[j] / we[i] * nv_[j] * sf[i];
                }
            }
        }
    }
    if (mirror) {
        const int64_t f = c->eface[4 * ge];
        const double nxv = c->normal[2 * f], nyv = c->normal[2 * f + 1];
        const double tx = c->tangent[2 * f], ty = c->tangent[2 * f + 1];
        for (int k = 0; k <= N; ++k) {
            const double Vx = gu[k], Vy = gv[k];
            const double l0 = -(Vx * nxv + Vy * nyv);
            const double l1 = Vx * tx + Vy * ty;
            gu[k] = nxv * l0 + tx * l1;
            gv[k] = nyv * l0 + ty * l1;
        }
    }
}

/* Mesh2D_t.cpp:3731-3782 (boundary_conditions) with the inflow boundary of
 * :4575-4599 and the periodic copy of :4712-4730. */
static void boundary_conditions(ndgo_ctx* c, double t) {
    for (int64_t b = 0; b < c->nb[0]; ++b) ghost_projection(c, c->blist[0][b], 1);
    for (int64_t b = 0; b < c->nb[1]; ++b) ghost_projection(c, c->blist[1][b], 1);
    for (int64_t b = 0; b < c->nb[2]; ++b) {
        const int64_t ge = c->blist[2][b];
        const int N = c->eN[ge];
        const double* xn = c->T.t[T_NODES][N];
        const double p0x = c->nx[c->enodes[4 * ge]], p0y = c->ny[c->enodes[4 * ge]];
        const double p1x = c->nx[c->enodes[4 * ge + 1]], p1y = c->ny[c->enodes[4 * ge + 1]];
        for (int k = 0; k <= N; ++k) {
            const double interp = (xn[k] + 1) / 2;
            const double gx = p1x * interp + p0x * (1 - interp);
            const double gy = p1y * interp + p0y * (1 - interp);
            analytic_g(gx, gy, t, c->pe + c->off1[ge] + k, c->ue + c->off1[ge] + k, c->ve + c->off1[ge] + k);
        }
    }
    for (int64_t b = 0; b < c->nb[3]; ++b) ghost_projection(c, c->blist[3][b], 0);
    for (int64_t q = 0; q < c->n_if; ++q) {
        const int64_t src = c->if_origin[q], dst = c->if_dest[q], side = c->if_origin_side[q];
        const int N = c->eN[src], n = N + 1;
        for (int k = 0; k <= N; ++k) {
            c->pe[c->off1[dst] + k] = c->pe[c->off1[src] + side * n + k];
            c->ue[c->off1[dst] + k] = c->ue[c->off1[src] + side * n + k];
            c->ve[c->off1[dst] + k] = c->ve[c->off1[src] + side * n + k];
        }
    }
}

/* Mesh2D_t.cpp:3803-3893 (project_to_faces). */
static void project_to_faces(ndgo_ctx* c) {
    for (int64_t f = 0; f < c->n_faces; ++f) {
        const int Nf = c->fN[f];
        const double* xf = c->T.t[T_NODES][Nf];
        for (int side = 0; side < 2; ++side) {
            const int64_t e = c->felem[2 * f + side];
            const int64_t es = c->fside[2 * f + side];
            const int Ne = c->eN[e], ne_ = Ne + 1;
            const double* xe = c->T.t[T_NODES][Ne];
            const double* bwe = c->T.t[T_BARY][Ne];
            const double* ep = c->pe + c->off1[e] + es * ne_;
            const double* eu = c->ue + c->off1[e] + es * ne_;
            const double* ev = c->ve + c->off1[e] + es * ne_;
            double* fp = (side == 0 ? c->fp0 : c->fp1) + c->foff[f];
            double* fu = (side == 0 ? c->fu0 : c->fu1) + c->foff[f];
            double* fv = (side == 0 ? c->fv0 : c->fv1) + c->foff[f];
            const int64_t en0 = c->enodes[4 * e + es];
            const int64_t en1 = c->enodes[4 * e + ((es + 1) * !(es + 1 == 4))];
            const int conforming = side == 0 ? (Nf == Ne && c->fnodes[2 * f] == en0 && c->fnodes[2 * f + 1] == en1)
                                             : (Nf == Ne && c->fnodes[2 * f + 1] == en0 && c->fnodes[2 * f] == en1);
            if (conforming) {
                for (int i = 0; i <= Nf; ++i) {
                    const int d = side == 0 ? i : Nf - i;
                    fp[d] = ep[i];
                    fu[d] = eu[i];
                    fv[d] = ev[i];
                }
            } else {
                for (int i = 0; i <= Nf; ++i) {
                    const double coord = (xf[side == 0 ? i : Nf - i] + 1) * c->scale[2 * f + side] + 2 * c->offset[2 * f + side] - 1;
                    double pn = 0.0, un = 0.0, vn = 0.0, den = 0.0;
                    for (int j = 0; j <= Ne; ++j) {
                        if (almost_equal(coord, xe[j])) {
                            pn = ep[j];
                            un = eu[j];
                            vn = ev[j];
                            den = 1.0;
                            break;
                        }
                        const double t = bwe[j] / (coord - xe[j]);
                        pn += t * ep[j];
                        un += t * eu[j];
                        vn += t * ev[j];
                        den += t;
                    }
                    fp[i] = pn / den;
                    fu[i] = un / den;
                    fv[i] = vn / den;
                }
            }
        }
    }
}

/* Face speed of the variable-speed operator: the mean of its two sides'
 * speeds (a ghost carries the speed of the element it stands for). */
static double face_speed(const ndgo_ctx* c, int64_t f) {
    return 0.5 * (c->speed[c->speed_owner[c->felem[2 * f]]] + c->speed[c->speed_owner[c->felem[2 * f + 1]]]);
}

/* src/solvers/Solver2D_t.cpp:48-63 (calculate_wave_fluxes, upwind). */
static void calculate_wave_fluxes(ndgo_ctx* c) {
    if (c->speed) {
        /* variable speed: the unit-speed upwind flux times the face speed */
        for (int64_t f = 0; f < c->n_faces; ++f) {
            const double nxv = c->normal[2 * f], nyv = c->normal[2 * f + 1], cf = face_speed(c, f);
            for (int i = 0; i <= c->fN[f]; ++i) {
                const int64_t k = c->foff[f] + i;
                const double wL = c->fp0[k] + (c->fu0[k] * nxv + c->fv0[k] * nyv);
                const double wR = c->fp1[k] - (c->fu1[k] * nxv + c->fv1[k] * nyv);
                c->fluxp[k] = cf * (wL - wR) / 2;
                c->fluxu[k] = cf * nxv * (wL + wR) / 2;
                c->fluxv[k] = cf * nyv * (wL + wR) / 2;
            }
        }
        return;
    }
    for (int64_t f = 0; f < c->n_faces; ++f) {
        const double nxv = c->normal[2 * f], nyv = c->normal[2 * f + 1];
        for (int i = 0; i <= c->fN[f]; ++i) {
            const int64_t k = c->foff[f] + i;
            const double wL = c->fp0[k] + C_c * (c->fu0[k] * nxv + c->fv0[k] * nyv);
            const double wR = c->fp1[k] - C_c * (c->fu1[k] * nxv + c->fv1[k] * nyv);
            c->fluxp[k] = C_c * (wL - wR) / 2;
            c->fluxu[k] = nxv * (wL + wR) / 2;
            c->fluxv[k] = nyv * (wL + wR) / 2;
        }
    }
}

/* Mesh2D_t.cpp:3895-4006 (project_to_elements). */
static void project_to_elements(ndgo_ctx* c) {
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* xe = c->T.t[T_NODES][N];
        const double* we = c->T.t[T_WEIGHTS][N];
        const double* bwe = c->T.t[T_BARY][N];
        for (int s = 0; s < 4; ++s) {
            const double* sf = c->sf + c->off1[e] + s * n;
            double* op = c->pfe + c->off1[e] + s * n;
            double* ou = c->ufe + c->off1[e] + s * n;
            double* ov = c->vfe + c->off1[e] + s * n;
            const int64_t en0 = c->enodes[4 * e + s];
            const int64_t en1 = c->enodes[4 * e + ((s + 1) * !(s + 1 == 4))];
            const int cnt = c->eface_cnt[4 * e + s];
            const int64_t f0 = c->eface[4 * e + s];
            if (cnt == 1 && c->fN[f0] == N && c->fnodes[2 * f0] == en0 && c->fnodes[2 * f0 + 1] == en1) {
                for (int j = 0; j <= N; ++j) {
                    const int64_t k = c->foff[f0] + j;
                    op[j] = c->fluxp[k] * sf[j];
                    ou[j] = c->fluxu[k] * sf[j];
                    ov[j] = c->fluxv[k] * sf[j];
                }
            } else if (cnt == 1 && c->fN[f0] == N && c->fnodes[2 * f0 + 1] == en0 && c->fnodes[2 * f0] == en1) {
                for (int j = 0; j <= N; ++j) {
                    const int64_t k = c->foff[f0] + j;
                    op[N - j] = -c->fluxp[k] * sf[j];
                    ou[N - j] = -c->fluxu[k] * sf[j];
                    ov[N - j] = -c->fluxv[k] * sf[j];
                }
            } else {
                for (int i = 0; i <= N; ++i) op[i] = ou[i] = ov[i] = 0.0;
                /* Zones built here have at most one face per element side; the
                 * reference's loop over several faces per side arises only
                 * after h-adaptation. */
                for (int fi = 0; fi < cnt; ++fi) {
                    const int64_t f = f0;
                    const int Nf = c->fN[f];
                    const double* xf = c->T.t[T_NODES][Nf];
                    const double* wf = c->T.t[T_WEIGHTS][Nf];
                    const int fwd = e == c->felem[2 * f];
                    const int fs = fwd ? 0 : 1;
                    const double sgn = fwd ? 1.0 : -1.0;
                    for (int j = 0; j <= Nf; ++j) {
                        const int64_t k = c->foff[f] + j;
                        const double coord = (xf[fwd ? j : Nf - j] + 1) * c->scale[2 * f + fs] + 2 * c->offset[2 * f + fs] - 1;
                        int found = 0;
                        for (int i = 0; i <= N; ++i) {
                            if (almost_equal(coord, xe[i])) {
                                op[i] += sgn * wf[j] / we[i] * c->fluxp[k] * sf[i] * c->scale[2 * f + fs];
                                ou[i] += sgn * wf[j] / we[i] * c->fluxu[k] * sf[i] * c->scale[2 * f + fs];
                                ov[i] += sgn * wf[j] / we[i] * c->fluxv[k] * sf[i] * c->scale[2 * f + fs];
                                found = 1;
                                break;
                            }
                        }
                        if (!found) {
                            double s_ = 0.0;
                            for (int i = 0; i <= N; ++i) s_ += bwe[i] / (coord - xe[i]);
                            for (int i = 0; i <= N; ++i) {
                                const double T = bwe[i] / ((coord - xe[i]) * s_);
                                op[i] += sgn * T * wf[j] / we[i] * c->fluxp[k] * sf[i] * c->scale[2 * f + fs];
                                ou[i] += sgn * T * wf[j] / we[i] * c->fluxu[k] * sf[i] * c->scale[2 * f + fs];
                                ov[i] += sgn * T * wf[j] / we[i] * c->fluxv[k] * sf[i] * c->scale[2 * f + fs];
                            }
                        }
                    }
                }
            }
        }
    }
}

/* src/solvers/Solver2D_t.cpp:66-136 (compute_dg_wave_derivative, Algorithm 114)
 * with the fluxes x_flux = (c u, p, 0), y_flux = (c v, 0, p) of :31-37; with
 * a speed per element, c_e (u, p, 0) and c_e (v, 0, p). */
static void compute_dg_wave_derivative(ndgo_ctx* c) {
    double fl[3][33], fd[3][33];
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* Dh = c->T.t[T_DHAT][N];
        const double* lm = c->T.t[T_LL][N];
        const double* lp = c->T.t[T_LR][N];
        const double* w = c->T.t[T_WEIGHTS][N];
        const int64_t o2 = c->off2[e], o1 = c->off1[e];
        const double* P = c->p + o2;
        const double* U = c->u + o2;
        const double* V = c->v + o2;
        double* G[3] = {c->Gp + o2, c->Gu + o2, c->Gv + o2};
        const double* FE[3] = {c->pfe + o1, c->ufe + o1, c->vfe + o1};
        const double ce = c->speed ? c->speed[e] : 0.0;
        for (int j = 0; j <= N; ++j) {
            for (int i = 0; i <= N; ++i) {
                const int k = i * n + j;
                double fx[3] = {C_c * U[k], P[k], 0};
                double fy[3] = {C_c * V[k], 0, P[k]};
                if (c->speed) {
                    fx[0] = ce * U[k], fx[1] = ce * P[k];
                    fy[0] = ce * V[k], fy[2] = ce * P[k];
                }
                for (int f = 0; f < 3; ++f) fl[f][i] = c->eta_y[o2 + k] * fx[f] - c->eta_x[o2 + k] * fy[f];
            }
            for (int f = 0; f < 3; ++f)
                for (int i = 0; i <= N; ++i) {
                    fd[f][i] = 0.0;
                    for (int m = 0; m <= N; ++m) fd[f][i] += Dh[i * n + m] * fl[f][m];
                }
            for (int i = 0; i <= N; ++i)
                for (int f = 0; f < 3; ++f) fd[f][i] += (FE[f][1 * n + j] * lp[i] + FE[f][3 * n + N - j] * lm[i]) / w[i];
            for (int i = 0; i <= N; ++i)
                for (int f = 0; f < 3; ++f) G[f][i * n + j] = -fd[f][i];
        }
        for (int i = 0; i <= N; ++i) {
            for (int j = 0; j <= N; ++j) {
                const int k = i * n + j;
                double fx[3] = {C_c * U[k], P[k], 0};
                double fy[3] = {C_c * V[k], 0, P[k]};
                if (c->speed) {
                    fx[0] = ce * U[k], fx[1] = ce * P[k];
                    fy[0] = ce * V[k], fy[2] = ce * P[k];
                }
                for (int f = 0; f < 3; ++f) fl[f][j] = -c->xi_y[o2 + k] * fx[f] + c->xi_x[o2 + k] * fy[f];
            }
            for (int f = 0; f < 3; ++f)
                for (int j = 0; j <= N; ++j) {
                    fd[f][j] = 0.0;
                    for (int m = 0; m <= N; ++m) fd[f][j] += Dh[j * n + m] * fl[f][m];
                }
            for (int j = 0; j <= N; ++j)
                for (int f = 0; f < 3; ++f) fd[f][j] += (FE[f][2 * n + N - i] * lp[j] + FE[f][0 * n + i] * lm[j]) / w[j];
            for (int j = 0; j <= N; ++j)
                for (int f = 0; f < 3; ++f) G[f][i * n + j] = (G[f][i * n + j] - fd[f][j]) / c->jac[o2 + i * n + j];
        }
    }
}

/* src/solvers/Solver2D_t.cpp:138-172 (rk3_first_step, rk3_step) with the
 * Williamson coefficients of include/solvers/Solver2D_t.tpp:16-18. */
static const double RK_A[3] = {0, -5.0 / 9.0, -153.0 / 128.0};
static const double RK_B[3] = {0, 1.0 / 3.0, 0.75};
static const double RK_G[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

static void rk3(ndgo_ctx* c, int m, double dt) {
    double* q[3] = {c->p, c->u, c->v};
    double* G[3] = {c->Gp, c->Gu, c->Gv};
    double* K[3] = {c->kp, c->ku, c->kv};
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int n = c->eN[e] + 1;
        for (int64_t k = c->off2[e]; k < c->off2[e] + n * n; ++k)
            for (int f = 0; f < 3; ++f) {
                K[f][k] = (m == 0) ? G[f][k] : RK_A[m] * K[f][k] + G[f][k];
                q[f][k] += RK_G[m] * dt * K[f][k];
            }
    }
}

void ndgo_stage(ndgo_ctx* c, int m, double time, double dt) {
    const double t = time + RK_B[m] * dt;
    interpolate_to_boundaries(c);
    boundary_conditions(c, t);
    project_to_faces(c);
    calculate_wave_fluxes(c);
    project_to_elements(c);
    compute_dg_wave_derivative(c);
    rk3(c, m, dt);
}

double ndgo_run(ndgo_ctx* c, int64_t n_steps, double time) {
    for (int64_t s = 0; s < n_steps; ++s) {
        const double dt = ndgo_get_delta_t(c);
        ndgo_stage(c, 0, time, dt);
        ndgo_stage(c, 1, time, dt);
        ndgo_stage(c, 2, time, dt);
        time += dt;
    }
    return time;
}

static double* field_ptr(const ndgo_ctx* c, int which) {
    double* a[] = {c->p, c->u, c->v, c->Gp, c->Gu, c->Gv, c->kp, c->ku, c->kv};
    return (which >= 0 && which < 9) ? a[which] : NULL;
}

int64_t ndgo_get_field(const ndgo_ctx* c, int which, double* out) {
    const double* src = field_ptr(c, which);
    if (!src) return -1;
    const int64_t total = c->n_elem > 0 ? c->off2[c->n_elem - 1] + (c->eN[c->n_elem - 1] + 1) * (c->eN[c->n_elem - 1] + 1) : 0;
    memcpy(out, src, (size_t)total * sizeof(double));
    return total;
}

int64_t ndgo_set_field(ndgo_ctx* c, int which, const double* in) {
    double* dst = field_ptr(c, which);
    if (!dst) return -1;
    const int64_t total = c->n_elem > 0 ? c->off2[c->n_elem - 1] + (c->eN[c->n_elem - 1] + 1) * (c->eN[c->n_elem - 1] + 1) : 0;
    memcpy(dst, in, (size_t)total * sizeof(double));
    return total;
}

void ndgo_element_N(const ndgo_ctx* c, int* N) {
    for (int64_t e = 0; e < c->n_elem; ++e) N[e] = c->eN[e];
}

void ndgo_get_faces(const ndgo_ctx* c, int64_t* nodes, int64_t* elements, int64_t* sides, int* N, double* normal, double* tangent, double* offset, double* scale) {
    for (int64_t f = 0; f < c->n_faces; ++f) {
        for (int k = 0; k < 2; ++k) {
            nodes[2 * f + k] = c->fnodes[2 * f + k];
            elements[2 * f + k] = c->felem[2 * f + k];
            sides[2 * f + k] = c->fside[2 * f + k];
            normal[2 * f + k] = c->normal[2 * f + k];
            tangent[2 * f + k] = c->tangent[2 * f + k];
            offset[2 * f + k] = c->offset[2 * f + k];
            scale[2 * f + k] = c->scale[2 * f + k];
        }
        N[f] = c->fN[f];
    }
}

void ndgo_get_elements(const ndgo_ctx* c, int64_t* nodes, int* N, double* delta_xy_min, int64_t* first_face) {
    for (int64_t e = 0; e < c->n_elem_total; ++e) {
        for (int k = 0; k < 4; ++k) {
            nodes[4 * e + k] = c->enodes[4 * e + k];
            first_face[4 * e + k] = c->eface[4 * e + k];
        }
        N[e] = c->eN[e];
        delta_xy_min[e] = c->dxy_min[e];
    }
}

void ndgo_get_nodes(const ndgo_ctx* c, double* xy) {
    for (int64_t i = 0; i < c->n_nodes; ++i) {
        xy[2 * i] = c->nx[i];
        xy[2 * i + 1] = c->ny[i];
    }
}

int64_t ndgo_get_boundary(const ndgo_ctx* c, int kind, int64_t* out) {
    const int64_t* src;
    int64_t cnt;
    if (kind >= 0 && kind < 4) {
        src = c->blist[kind];
        cnt = c->nb[kind];
    } else if (kind == 4) {
        src = c->if_origin;
        cnt = c->n_if;
    } else if (kind == 5) {
        src = c->if_origin_side;
        cnt = c->n_if;
    } else if (kind == 6) {
        src = c->if_dest;
        cnt = c->n_if;
    } else {
        return -1;
    }
    if (out) memcpy(out, src, (size_t)cnt * sizeof(int64_t));
    return cnt;
}

/* Element2D_t.cpp:274-317 (estimate_p_error) and :319-343 (exponential_decay),
 * with n_points_least_squares_max = 4 (include/helpers/constants.h:19). */
void ndgo_estimate_error(ndgo_ctx* c, double tolerance_min, double tolerance_max) {
    double spectrum[33];
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* poly = c->T.t[T_POLY][N];
        const double* P = c->p + c->off2[e];
        const int npl = (N + 1 < 4) ? N + 1 : 4;
        for (int ni = 0; ni < npl; ++ni) {
            spectrum[ni] = 0.0;
            const double pd = N + ni + 1 - npl;
            const int p = (int)pd;
            for (int i = 0; i < pd; ++i) {
                double lx = 0.0, ly = 0.0;
                for (int k = 0; k <= N; ++k)
                    for (int l = 0; l <= N; ++l) {
                        lx += P[k * n + l] * poly[i * n + k] * poly[p * n + l];
                        ly += P[k * n + l] * poly[p * n + k] * poly[i * n + l];
                    }
                spectrum[ni] += fabs(lx) + fabs(ly);
            }
            double lx = 0.0;
            for (int k = 0; k <= N; ++k)
                for (int l = 0; l <= N; ++l) lx += P[k * n + l] * poly[p * n + k] * poly[p * n + l];
            spectrum[ni] += fabs(lx);
        }
        double x_avg = 0.0, y_avg = 0.0;
        for (int i = 0; i < npl; ++i) {
            x_avg += N + i + 1 - npl;
            y_avg += log(spectrum[i]);
        }
        x_avg /= npl;
        y_avg /= npl;
        double num = 0.0, den = 0.0;
        for (int i = 0; i < npl; ++i) {
            const int p = N + i + 1 - npl;
            num += (p - x_avg) * (log(spectrum[i]) - y_avg);
            den += (p - x_avg) * (p - x_avg);
        }
        const double sigma_signed = num / den;
        const double C = exp(y_avg - sigma_signed * x_avg);
        const double sigma = fabs(sigma_signed);
        c->p_sigma[e] = sigma;
        c->p_error[e] = sqrt(spectrum[npl - 1] * spectrum[npl - 1] + C * C * 0.5 / sigma * exp(-2 * sigma * (N + 1)));
        c->refine[e] = c->p_error[e] > tolerance_min;
        c->coarsen[e] = c->p_error[e] < tolerance_max;
    }
}

void ndgo_get_error(const ndgo_ctx* c, double* p_error, double* p_sigma, int* refine, int* coarsen) {
    for (int64_t e = 0; e < c->n_elem; ++e) {
        p_error[e] = c->p_error[e];
        p_sigma[e] = c->p_sigma[e];
        refine[e] = c->refine[e];
        coarsen[e] = c->coarsen[e];
    }
}

/* ------------------------------------------------------------------------
 * Variable-speed operator and its discrete adjoint (the CPU reference
 * gradient of the library's adjoint). Plain loops: every forward pass of
 * ndgo_stage is transposed on its own, in reverse order, on meshes of one
 * order with conforming faces; the c-derivative of the face flux is taken
 * per face (both sides' owners receive half of it). */

static int64_t total1(const ndgo_ctx* c) { return c->off1[c->n_elem_total - 1] + 4 * (c->eN[c->n_elem_total - 1] + 1); }
static int64_t total_faces(const ndgo_ctx* c) { return c->n_faces ? c->foff[c->n_faces - 1] + c->fN[c->n_faces - 1] + 1 : 0; }
static int64_t domain_size(const ndgo_ctx* c) { return c->off2[c->n_elem - 1] + (c->eN[c->n_elem - 1] + 1) * (c->eN[c->n_elem - 1] + 1); }

void ndgo_set_speed(ndgo_ctx* c, const double* speed) {
    free(c->speed);
    free(c->speed_owner);
    c->speed = NULL;
    c->speed_owner = NULL;
    if (!speed) return;
    c->speed = (double*)xcalloc((size_t)c->n_elem, sizeof(double));
    memcpy(c->speed, speed, (size_t)c->n_elem * sizeof(double));
    c->speed_owner = (int64_t*)xcalloc((size_t)c->n_elem_total, sizeof(int64_t));
    for (int64_t e = 0; e < c->n_elem_total; ++e) c->speed_owner[e] = e;
    /* a boundary ghost carries the speed of the element across its face */
    for (int64_t g = c->n_elem; g < c->n_elem_total; ++g) {
        const int64_t f = c->eface[4 * g];
        if (f >= 0) c->speed_owner[g] = c->felem[2 * f] == g ? c->felem[2 * f + 1] : c->felem[2 * f];
    }
    /* a periodic ghost carries the speed of the element whose trace it copies */
    for (int64_t q = 0; q < c->n_if; ++q) c->speed_owner[c->if_dest[q]] = c->if_origin[q];
}

typedef struct {
    double *pe, *ue, *ve;    /* adjoints of the side traces */
    double *pfe, *ufe, *vfe; /* adjoints of the element side fluxes */
    double *f0[3], *f1[3];   /* adjoints of the face traces (left, right) */
    double* fl[3];           /* adjoints of the face fluxes */
} adj_work;

static void adj_work_alloc(const ndgo_ctx* c, adj_work* w) {
    const size_t s1 = (size_t)total1(c), sf = (size_t)total_faces(c);
    w->pe = (double*)xcalloc(s1, sizeof(double));
    w->ue = (double*)xcalloc(s1, sizeof(double));
    w->ve = (double*)xcalloc(s1, sizeof(double));
    w->pfe = (double*)xcalloc(s1, sizeof(double));
    w->ufe = (double*)xcalloc(s1, sizeof(double));
    w->vfe = (double*)xcalloc(s1, sizeof(double));
    for (int f = 0; f < 3; ++f) {
        w->f0[f] = (double*)xcalloc(sf, sizeof(double));
        w->f1[f] = (double*)xcalloc(sf, sizeof(double));
        w->fl[f] = (double*)xcalloc(sf, sizeof(double));
    }
}

static void adj_work_free(adj_work* w) {
    free(w->pe), free(w->ue), free(w->ve), free(w->pfe), free(w->ufe), free(w->vfe);
    for (int f = 0; f < 3; ++f) free(w->f0[f]), free(w->f1[f]), free(w->fl[f]);
}

static void adj_work_zero(const ndgo_ctx* c, adj_work* w) {
    const size_t s1 = (size_t)total1(c), sf = (size_t)total_faces(c);
    double* a1[] = {w->pe, w->ue, w->ve, w->pfe, w->ufe, w->vfe};
    for (int k = 0; k < 6; ++k) memset(a1[k], 0, s1 * sizeof(double));
    for (int f = 0; f < 3; ++f) {
        memset(w->f0[f], 0, sf * sizeof(double));
        memset(w->f1[f], 0, sf * sizeof(double));
        memset(w->fl[f], 0, sf * sizeof(double));
    }
}

/* The forward passes of one stage up to the element time derivative G, on
 * the state in c->p, c->u, c->v (no RK update). */
static void operator_passes(ndgo_ctx* c) {
    interpolate_to_boundaries(c);
    boundary_conditions(c, 0.0);
    project_to_faces(c);
    calculate_wave_fluxes(c);
    project_to_elements(c);
    compute_dg_wave_derivative(c);
}

/* Transpose of ghost_projection (the velocity mirror, then the projection of
 * the neighbour's side trace), adding to the neighbour's trace adjoints and
 * consuming the ghost's. */
static void ghost_projection_transpose(ndgo_ctx* c, adj_work* w, int64_t ge, int mirror) {
    const int N = c->eN[ge];
    const double* xe = c->T.t[T_NODES][N];
    const double* we = c->T.t[T_WEIGHTS][N];
    const double* bwe = c->T.t[T_BARY][N];
    double* gp = w->pe + c->off1[ge];
    double* gu = w->ue + c->off1[ge];
    double* gv = w->ve + c->off1[ge];
    const double* sf = c->sf + c->off1[ge];
    if (mirror) {
        const int64_t f = c->eface[4 * ge];
        const double nxv = c->normal[2 * f], nyv = c->normal[2 * f + 1];
        const double tx = c->tangent[2 * f], ty = c->tangent[2 * f + 1];
        for (int k = 0; k <= N; ++k) {
            /* the mirror -n n^T + t t^T is symmetric: its own transpose */
            const double Vx = gu[k], Vy = gv[k];
            const double l0 = -(Vx * nxv + Vy * nyv);
            const double l1 = Vx * tx + Vy * ty;
            gu[k] = nxv * l0 + tx * l1;
            gv[k] = nyv * l0 + ty * l1;
        }
    }
    for (int fi = 0; fi < c->eface_cnt[4 * ge]; ++fi) {
        const int64_t f = c->eface[4 * ge + fi];
        const int fs = c->felem[2 * f] == ge;
        const int64_t nb = c->felem[2 * f + fs];
        const int64_t nbs = c->fside[2 * f + fs];
        const int Nn = c->eN[nb], nn = Nn + 1;
        const double* xnb = c->T.t[T_NODES][Nn];
        const double* wnb = c->T.t[T_WEIGHTS][Nn];
        double* np_ = w->pe + c->off1[nb] + nbs * nn;
        double* nu_ = w->ue + c->off1[nb] + nbs * nn;
        double* nv_ = w->ve + c->off1[nb] + nbs * nn;
        for (int j = 0; j <= Nn; ++j) {
            const double coord = (xnb[Nn - j] + 1) * c->scale[2 * f + fs] + 2 * c->offset[2 * f + fs] - 1;
            int found = 0;
            for (int i = 0; i <= N; ++i) {
                if (almost_equal(coord, xe[i])) {
                    np_[j] += wnb[j] / we[i] * sf[i] * gp[i];
                    nu_[j] += wnb[j] / we[i] * sf[i] * gu[i];
                    nv_[j] += wnb[j] / we[i] * sf[i] * gv[i];
                    found = 1;
                    break;
                }
            }
            if (!found) {
                double s = 0.0;
                for (int i = 0; i <= N; ++i) s += bwe[i] / (coord - xe[i]);
                for (int i = 0; i <= N; ++i) {
                    const double T = bwe[i] / ((coord - xe[i]) * s);
                    np_[j] += T * wnb[j] / we[i] * sf[i] * gp[i];
                    nu_[j] += T * wnb[j] / we[i] * sf[i] * gu[i];
                    nv_[j] += T * wnb[j] / we[i] * sf[i] * gv[i];
                }
            }
        }
    }
    for (int k = 0; k <= N; ++k) gp[k] = gu[k] = gv[k] = 0.0;
}

/* lq += L(c)^T mu; dc (optional) += d(mu . L(c) q)/dc where q is the state
 * whose forward passes were run last (its face traces and fluxes are in c).
 * mu, lq: field blocks p, u, v of domain_size values each. Returns -1 on a
 * non-conforming face. */
static int operator_transpose(ndgo_ctx* c, adj_work* w, const double* mu, double* lq, double* dc) {
    const int64_t fsz = domain_size(c);
    adj_work_zero(c, w);
    /* compute_dg_wave_derivative^T */
    double lfl[3][33];
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* Dh = c->T.t[T_DHAT][N];
        const double* lm = c->T.t[T_LL][N];
        const double* lp = c->T.t[T_LR][N];
        const double* wt = c->T.t[T_WEIGHTS][N];
        const int64_t o2 = c->off2[e], o1 = c->off1[e];
        const double ce = c->speed ? c->speed[e] : 1.0;
        const double* P = c->p + o2;
        const double* U = c->u + o2;
        const double* V = c->v + o2;
        const double* M[3] = {mu + o2, mu + fsz + o2, mu + 2 * fsz + o2};
        double* LQ[3] = {lq + o2, lq + fsz + o2, lq + 2 * fsz + o2};
        double* LFE[3] = {w->pfe + o1, w->ufe + o1, w->vfe + o1};
        double dce = 0.0;
        for (int pass = 0; pass < 2; ++pass) {
            for (int a = 0; a <= N; ++a) {
                /* pass 0: xi lines (column j = a); pass 1: eta lines (row i = a) */
                double nu[3][33];
                for (int b = 0; b <= N; ++b) {
                    const int k = pass == 0 ? b * n + a : a * n + b;
                    for (int f = 0; f < 3; ++f) nu[f][b] = -M[f][k] / c->jac[o2 + k];
                }
                for (int f = 0; f < 3; ++f)
                    for (int m = 0; m <= N; ++m) {
                        lfl[f][m] = 0.0;
                        for (int b = 0; b <= N; ++b) lfl[f][m] += Dh[b * n + m] * nu[f][b];
                    }
                for (int f = 0; f < 3; ++f)
                    for (int b = 0; b <= N; ++b) {
                        if (pass == 0) {
                            LFE[f][1 * n + a] += nu[f][b] * lp[b] / wt[b];
                            LFE[f][3 * n + N - a] += nu[f][b] * lm[b] / wt[b];
                        } else {
                            LFE[f][2 * n + N - a] += nu[f][b] * lp[b] / wt[b];
                            LFE[f][0 * n + a] += nu[f][b] * lm[b] / wt[b];
                        }
                    }
                for (int m = 0; m <= N; ++m) {
                    const int k = pass == 0 ? m * n + a : a * n + m;
                    double lfx[3], lfy[3];
                    for (int f = 0; f < 3; ++f) {
                        if (pass == 0) {
                            lfx[f] = c->eta_y[o2 + k] * lfl[f][m];
                            lfy[f] = -c->eta_x[o2 + k] * lfl[f][m];
                        } else {
                            lfx[f] = -c->xi_y[o2 + k] * lfl[f][m];
                            lfy[f] = c->xi_x[o2 + k] * lfl[f][m];
                        }
                    }
                    /* fx = ce (u, p, 0), fy = ce (v, 0, p) */
                    LQ[1][k] += ce * lfx[0];
                    LQ[0][k] += ce * lfx[1];
                    LQ[2][k] += ce * lfy[0];
                    LQ[0][k] += ce * lfy[2];
                    dce += U[k] * lfx[0] + P[k] * lfx[1] + V[k] * lfy[0] + P[k] * lfy[2];
                }
            }
        }
        if (dc) dc[e] += dce;
    }
    /* project_to_elements^T (conforming faces) */
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        for (int s = 0; s < 4; ++s) {
            const double* sf = c->sf + c->off1[e] + s * n;
            const double* op = w->pfe + c->off1[e] + s * n;
            const double* ou = w->ufe + c->off1[e] + s * n;
            const double* ov = w->vfe + c->off1[e] + s * n;
            const int64_t en0 = c->enodes[4 * e + s];
            const int64_t en1 = c->enodes[4 * e + ((s + 1) * !(s + 1 == 4))];
            const int64_t f0 = c->eface[4 * e + s];
            if (c->eface_cnt[4 * e + s] != 1 || c->fN[f0] != N) return -1;
            if (c->fnodes[2 * f0] == en0 && c->fnodes[2 * f0 + 1] == en1) {
                for (int j = 0; j <= N; ++j) {
                    const int64_t k = c->foff[f0] + j;
                    w->fl[0][k] += op[j] * sf[j];
                    w->fl[1][k] += ou[j] * sf[j];
                    w->fl[2][k] += ov[j] * sf[j];
                }
            } else if (c->fnodes[2 * f0 + 1] == en0 && c->fnodes[2 * f0] == en1) {
                for (int j = 0; j <= N; ++j) {
                    const int64_t k = c->foff[f0] + j;
                    w->fl[0][k] -= op[N - j] * sf[j];
                    w->fl[1][k] -= ou[N - j] * sf[j];
                    w->fl[2][k] -= ov[N - j] * sf[j];
                }
            } else {
                return -1;
            }
        }
    }
    /* calculate_wave_fluxes^T, with the face-speed derivative */
    for (int64_t f = 0; f < c->n_faces; ++f) {
        const double nxv = c->normal[2 * f], nyv = c->normal[2 * f + 1];
        const double cf = c->speed ? face_speed(c, f) : 1.0;
        double dcf = 0.0;
        for (int i = 0; i <= c->fN[f]; ++i) {
            const int64_t k = c->foff[f] + i;
            const double gp = w->fl[0][k], gu = w->fl[1][k], gv = w->fl[2][k];
            dcf += gp * c->fluxp[k] + gu * c->fluxu[k] + gv * c->fluxv[k];
            const double lwL = cf * (gp / 2 + (nxv * gu + nyv * gv) / 2);
            const double lwR = cf * (-gp / 2 + (nxv * gu + nyv * gv) / 2);
            w->f0[0][k] += lwL;
            w->f0[1][k] += lwL * nxv;
            w->f0[2][k] += lwL * nyv;
            w->f1[0][k] += lwR;
            w->f1[1][k] -= lwR * nxv;
            w->f1[2][k] -= lwR * nyv;
        }
        if (dc && c->speed) {
            dc[c->speed_owner[c->felem[2 * f]]] += 0.5 * dcf / cf;
            dc[c->speed_owner[c->felem[2 * f + 1]]] += 0.5 * dcf / cf;
        }
    }
    /* project_to_faces^T (conforming) */
    for (int64_t f = 0; f < c->n_faces; ++f) {
        const int Nf = c->fN[f];
        for (int side = 0; side < 2; ++side) {
            const int64_t e = c->felem[2 * f + side];
            const int64_t es = c->fside[2 * f + side];
            const int ne_ = c->eN[e] + 1;
            double* ep = w->pe + c->off1[e] + es * ne_;
            double* eu = w->ue + c->off1[e] + es * ne_;
            double* ev = w->ve + c->off1[e] + es * ne_;
            double* const* src = side == 0 ? w->f0 : w->f1;
            for (int i = 0; i <= Nf; ++i) {
                const int d = side == 0 ? i : Nf - i;
                const int64_t k = c->foff[f] + d;
                ep[i] += src[0][k];
                eu[i] += src[1][k];
                ev[i] += src[2][k];
            }
        }
    }
    /* boundary_conditions^T, in reverse order */
    for (int64_t q = c->n_if - 1; q >= 0; --q) {
        const int64_t src = c->if_origin[q], dst = c->if_dest[q], side = c->if_origin_side[q];
        const int N = c->eN[src], n = N + 1;
        for (int k = 0; k <= N; ++k) {
            w->pe[c->off1[src] + side * n + k] += w->pe[c->off1[dst] + k];
            w->ue[c->off1[src] + side * n + k] += w->ue[c->off1[dst] + k];
            w->ve[c->off1[src] + side * n + k] += w->ve[c->off1[dst] + k];
            w->pe[c->off1[dst] + k] = w->ue[c->off1[dst] + k] = w->ve[c->off1[dst] + k] = 0.0;
        }
    }
    for (int64_t b = c->nb[3] - 1; b >= 0; --b) ghost_projection_transpose(c, w, c->blist[3][b], 0);
    for (int64_t b = c->nb[1] - 1; b >= 0; --b) ghost_projection_transpose(c, w, c->blist[1][b], 1);
    for (int64_t b = c->nb[0] - 1; b >= 0; --b) ghost_projection_transpose(c, w, c->blist[0][b], 1);
    /* interpolate_to_boundaries^T */
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* lm = c->T.t[T_LL][N];
        const double* lp = c->T.t[T_LR][N];
        const int64_t o2 = c->off2[e], o1 = c->off1[e];
        double* LQ[3] = {lq + o2, lq + fsz + o2, lq + 2 * fsz + o2};
        const double* ex[3] = {w->pe + o1, w->ue + o1, w->ve + o1};
        for (int i = 0; i <= N; ++i)
            for (int j = 0; j <= N; ++j)
                for (int f = 0; f < 3; ++f) {
                    LQ[f][i * n + j] += lm[j] * ex[f][0 * n + i] + lp[j] * ex[f][2 * n + N - i];
                    LQ[f][j * n + i] += lp[j] * ex[f][1 * n + i] + lm[j] * ex[f][3 * n + N - i];
                }
    }
    return 0;
}

static void set_state(ndgo_ctx* c, const double* p, const double* u, const double* v) {
    const size_t bytes = (size_t)domain_size(c) * sizeof(double);
    memcpy(c->p, p, bytes);
    if (u) memcpy(c->u, u, bytes); else memset(c->u, 0, bytes);
    if (v) memcpy(c->v, v, bytes); else memset(c->v, 0, bytes);
}

int ndgo_operator(ndgo_ctx* c, const double* x, double* Lx) {
    const int64_t fsz = domain_size(c);
    set_state(c, x, x + fsz, x + 2 * fsz);
    operator_passes(c);
    memcpy(Lx, c->Gp, (size_t)fsz * sizeof(double));
    memcpy(Lx + fsz, c->Gu, (size_t)fsz * sizeof(double));
    memcpy(Lx + 2 * fsz, c->Gv, (size_t)fsz * sizeof(double));
    return 0;
}

int ndgo_operator_transpose(ndgo_ctx* c, const double* x, const double* y, double* LTy, double* dc) {
    const int64_t fsz = domain_size(c);
    set_state(c, x, x + fsz, x + 2 * fsz);
    operator_passes(c);
    memset(LTy, 0, 3 * (size_t)fsz * sizeof(double));
    if (dc) memset(dc, 0, (size_t)c->n_elem * sizeof(double));
    adj_work w;
    adj_work_alloc(c, &w);
    const int rc = operator_transpose(c, &w, y, LTy, dc);
    adj_work_free(&w);
    return rc;
}

static double sample(const ndgo_ctx* c, int64_t elem, const double* wr) {
    const int n = c->eN[elem] + 1;
    const double* p = c->p + c->off2[elem];
    double s = 0.0;
    for (int i = 0; i < n * n; ++i) s += wr[i] * p[i];
    return s;
}

double ndgo_adjoint_solve(ndgo_ctx* c, const double* p0, const double* u0, const double* v0, double dt, int64_t n_steps,
                          int n_rec, const int64_t* rec_elem, const double* rec_w, const double* targets,
                          double* samples, double* grad_p, double* grad_u, double* grad_v, double* grad_c) {
    const int64_t fsz = domain_size(c);
    const int NN = (c->eN[0] + 1) * (c->eN[0] + 1);
    const size_t state = 3 * (size_t)fsz;
    double* Q = (double*)xcalloc((size_t)n_steps * 3 * state, sizeof(double));
    double* smp = (double*)xcalloc((size_t)(n_steps + 1) * (size_t)(n_rec > 0 ? n_rec : 1), sizeof(double));
    set_state(c, p0, u0, v0);
    for (int r = 0; r < n_rec; ++r) smp[r] = sample(c, rec_elem[r], rec_w + (size_t)r * NN);
    double J = 0.0;
    for (int64_t s = 1; s <= n_steps; ++s) {
        for (int m = 0; m < 3; ++m) {
            double* q = Q + ((size_t)(s - 1) * 3 + (size_t)m) * state;
            memcpy(q, c->p, (size_t)fsz * sizeof(double));
            memcpy(q + fsz, c->u, (size_t)fsz * sizeof(double));
            memcpy(q + 2 * fsz, c->v, (size_t)fsz * sizeof(double));
            ndgo_stage(c, m, 0.0, dt);
        }
        for (int r = 0; r < n_rec; ++r) {
            smp[s * n_rec + r] = sample(c, rec_elem[r], rec_w + (size_t)r * NN);
            const double d = smp[s * n_rec + r] - (targets ? targets[s * n_rec + r] : 0.0);
            J += d * d;
        }
    }
    J *= 0.5 * dt;
    if (samples) memcpy(samples, smp, (size_t)(n_steps + 1) * (size_t)n_rec * sizeof(double));

    /* reverse sweep */
    double* lq = (double*)xcalloc(state, sizeof(double));
    double* lk = (double*)xcalloc(state, sizeof(double));
    double* mu = (double*)xcalloc(state, sizeof(double));
    double* dc = (double*)xcalloc((size_t)c->n_elem, sizeof(double));
    adj_work w;
    adj_work_alloc(c, &w);
    int rc = 0;
    for (int64_t s = n_steps; s >= 1 && rc == 0; --s) {
        /* the misfit's derivative at the end of step s */
        for (int r = 0; r < n_rec; ++r) {
            const double res = dt * (smp[s * n_rec + r] - (targets ? targets[s * n_rec + r] : 0.0));
            const double* wr = rec_w + (size_t)r * NN;
            for (int i = 0; i < NN; ++i) lq[c->off2[rec_elem[r]] + i] += res * wr[i];
        }
        for (int m = 2; m >= 0 && rc == 0; --m) {
            const double* q = Q + ((size_t)(s - 1) * 3 + (size_t)m) * state;
            for (size_t i = 0; i < state; ++i) mu[i] = lk[i] + RK_G[m] * dt * lq[i];
            set_state(c, q, q + fsz, q + 2 * fsz);
            operator_passes(c);
            rc = operator_transpose(c, &w, mu, lq, dc);
            for (size_t i = 0; i < state; ++i) lk[i] = RK_A[m] * mu[i];
        }
    }
    if (grad_p) memcpy(grad_p, lq, (size_t)fsz * sizeof(double));
    if (grad_u) memcpy(grad_u, lq + fsz, (size_t)fsz * sizeof(double));
    if (grad_v) memcpy(grad_v, lq + 2 * fsz, (size_t)fsz * sizeof(double));
    if (grad_c) memcpy(grad_c, dc, (size_t)c->n_elem * sizeof(double));
    adj_work_free(&w);
    free(lq), free(lk), free(mu), free(dc), free(Q), free(smp);
    return rc == 0 ? J : NAN;
}

/* Mesh2D_t::get_complete_solution (src/meshes/Mesh2D_t.cpp:4251-4296) with
 * Element2D_t::interpolate_complete_solution (src/entities/Element2D_t.cpp:606-646):
 * per domain element, on the n_interp x n_interp grid of reference points
 * i / (n_interp - 1) * 2 - 1, the coordinates (quad_map), the fields and
 * their time derivatives interpolated with the order's interpolation
 * matrix, and the interpolated |g(x_mn, time) - q_mn| over the Gauss nodes,
 * each sum in the reference's order. out[11] = x, y, p, u, v, dp/dt, du/dt,
 * dv/dt, p/u/v analytic error, n_elements n_interp^2 values each (any may
 * be NULL). Returns 0, or -1 when the tables cannot be built. */
int ndgo_complete_solution(const ndgo_ctx* c, int64_t n_interp, double time, double** out) {
    ndgo_tables T;
    if (n_interp < 2 || tables_build(&T, c->T.N_max, n_interp) != 0) return -1;
    const int64_t PP = n_interp * n_interp;
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const int64_t o2 = c->off2[e];
        double px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            px[k] = c->nx[c->enodes[4 * e + k]];
            py[k] = c->ny[c->enodes[4 * e + k]];
        }
        const double* I = T.t[T_INTERP][N];
        const double* xn = T.t[T_NODES][N];
        const double* q[6] = {c->p + o2, c->u + o2, c->v + o2, c->Gp + o2, c->Gu + o2, c->Gv + o2};
        for (int64_t i = 0; i < n_interp; ++i) {
            for (int64_t j = 0; j < n_interp; ++j) {
                const int64_t o = e * PP + i * n_interp + j;
                const double xi = (double)i / (double)(n_interp - 1) * 2 - 1;
                const double eta = (double)j / (double)(n_interp - 1) * 2 - 1;
                double gx, gy;
                quad_map(xi, eta, px, py, &gx, &gy);
                double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int m = 0; m < n; ++m) {
                    for (int nn = 0; nn < n; ++nn) {
                        const double im = I[i * n + m], jn = I[j * n + nn];
                        for (int f = 0; f < 6; ++f) acc[f] += q[f][m * n + nn] * im * jn;
                        double nxg, nyg, g[3];
                        quad_map(xn[m], xn[nn], px, py, &nxg, &nyg);
                        analytic_g(nxg, nyg, time, &g[0], &g[1], &g[2]);
                        for (int f = 0; f < 3; ++f) acc[6 + f] += fabs(g[f] - q[f][m * n + nn]) * im * jn;
                    }
                }
                if (out[0]) out[0][o] = gx;
                if (out[1]) out[1][o] = gy;
                for (int f = 0; f < 9; ++f)
                    if (out[2 + f]) out[2 + f][o] = acc[f];
            }
        }
    }
    tables_free(&T);
    return 0;
}

/* The L2 error against the reference plane wave g(x, time) per field:
 * sqrt(sum_e sum_ij w_i w_j J_ij (q_ij - g_ij)^2), with the weights of the
 * element's order and J as compute_geometry forms it (Element2D_t.cpp:743-777);
 * elements, then nodes, in order. */
void ndgo_l2_error(const ndgo_ctx* c, double time, double* out) {
    double s[3] = {0, 0, 0};
    const double* q[3] = {c->p, c->u, c->v};
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int N = c->eN[e], n = N + 1;
        const double* xn = c->T.t[T_NODES][N];
        const double* w = c->T.t[T_WEIGHTS][N];
        double px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            px[k] = c->nx[c->enodes[4 * e + k]];
            py[k] = c->ny[c->enodes[4 * e + k]];
        }
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) {
                const int64_t k = c->off2[e] + i * n + j;
                double gx, gy, g[3];
                quad_map(xn[i], xn[j], px, py, &gx, &gy);
                analytic_g(gx, gy, time, &g[0], &g[1], &g[2]);
                const double ww = w[i] * w[j] * c->jac[k];
                for (int f = 0; f < 3; ++f) {
                    const double d = q[f][k] - g[f];
                    s[f] += ww * d * d;
                }
            }
        }
    }
    for (int f = 0; f < 3; ++f) out[f] = sqrt(s[f]);
}
