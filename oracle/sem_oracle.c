/*
 * sem_oracle.c -- CPU FP64 oracle of the CG-SEM elastic time loop.
 *
 * TEST INFRASTRUCTURE ONLY (see sem_oracle.h).  Restates the reference's CPU
 * time-loop semantics with the same floating-point evaluation order; compile
 * with -ffp-contract=off so no multiply-add is fused.
 */
#include "sem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

void orc_set_threads(int32_t n) { g_threads = n < 1 ? 1 : n; }

/* ------------------------------------------------------------------------
 * GLL tables (forward/share/include/gf/gll.hpp:21-131)
 * ---------------------------------------------------------------------- */

/* Legendre P_n(x) by Bonnet's recurrence (gll.hpp:21-33). */
static double leg_p(int n, double x) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    double p_prev = 1.0, p_cur = x, p_next = 0.0;
    for (int m = 1; m < n; ++m) {
        p_next = ((2.0 * m + 1.0) * x * p_cur - m * p_prev) / (m + 1.0);
        p_prev = p_cur;
        p_cur = p_next;
    }
    return p_next;
}

/* P_n'(x) (gll.hpp:36-47). */
static double leg_dp(int n, double x) {
    if (n == 0) return 0.0;
    if (fabs(x - 1.0) < 1e-14) return 0.5 * n * (n + 1.0);
    if (fabs(x + 1.0) < 1e-14) return (n % 2 == 0 ? -1.0 : 1.0) * 0.5 * n * (n + 1.0);
    double pn = leg_p(n, x);
    double pnm1 = leg_p(n - 1, x);
    return n * (x * pn - pnm1) / (x * x - 1.0);
}

int orc_gll(int32_t N, double* nodes, double* weights, double* D) {
    if (N < 1) return -1;
    const int ng = N + 1;
    /* nodes: endpoints fixed, interior roots of P_N' by Newton (gll.hpp:55-88) */
    nodes[0] = -1.0;
    nodes[N] = 1.0;
    for (int i = 1; i < N; ++i) {
        double x = -cos(M_PI * i / N);
        for (int it = 0; it < 100; ++it) {
            double f = leg_dp(N, x);
            double df = (2.0 * x * f - N * (N + 1.0) * leg_p(N, x)) / (1.0 - x * x);
            if (fabs(df) < 1.0e-14) return -1;
            double step = -f / df;
            x += step;
            if (fabs(step) < 1.0e-15 * (1.0 + fabs(x))) break;
        }
        nodes[i] = x;
    }
    /* weights 2/(N(N+1)P_N^2) (gll.hpp:93-104) */
    for (int i = 0; i < ng; ++i) {
        double pn = leg_p(N, nodes[i]);
        weights[i] = 2.0 / (N * (N + 1.0) * pn * pn);
    }
    /* derivative matrix (gll.hpp:109-131) */
    double pn_at[64];
    for (int i = 0; i < ng; ++i) pn_at[i] = leg_p(N, nodes[i]);
    for (int i = 0; i < ng; ++i) {
        for (int j = 0; j < ng; ++j) {
            double v;
            if (i == j) {
                if (i == 0) v = -0.25 * N * (N + 1.0);
                else if (i == N) v = 0.25 * N * (N + 1.0);
                else v = 0.0;
            } else {
                v = pn_at[i] / (pn_at[j] * (nodes[i] - nodes[j]));
            }
            D[i * ng + j] = v;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Element internal force (forward/elastic/src/element_cpu.cpp:19-162)
 * ---------------------------------------------------------------------- */

/* Displacement gradient in physical space at node (i,j,k) of one element,
 * reading the stored inverse Jacobian the way the reference kernel does:
 * grad[c][m] = du_c/dxi*dd[3m] + du_c/deta*dd[3m+1] + du_c/dzeta*dd[3m+2]. */
static void node_gradient(int i, int j, int k, int ng, const double* D, const double* u_e,
                          const double* dd, double grad[3][3]) {
    double gxi[3] = {0.0, 0.0, 0.0};
    double geta[3] = {0.0, 0.0, 0.0};
    double gzeta[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < ng; ++s) {
        const double a = D[i * ng + s];
        const double b = D[j * ng + s];
        const double c = D[k * ng + s];
        const double* ua = u_e + 3 * ((s * ng + j) * ng + k);
        const double* ub = u_e + 3 * ((i * ng + s) * ng + k);
        const double* uc = u_e + 3 * ((i * ng + j) * ng + s);
        for (int d = 0; d < 3; ++d) {
            gxi[d] += a * ua[d];
            geta[d] += b * ub[d];
            gzeta[d] += c * uc[d];
        }
    }
    for (int c = 0; c < 3; ++c) {
        grad[c][0] = gxi[c] * dd[0] + geta[c] * dd[1] + gzeta[c] * dd[2];
        grad[c][1] = gxi[c] * dd[3] + geta[c] * dd[4] + gzeta[c] * dd[5];
        grad[c][2] = gxi[c] * dd[6] + geta[c] * dd[7] + gzeta[c] * dd[8];
    }
}

/* Subtract sig . (Dts * dd[col], dd[col+3], dd[col+6]) * factor at node rn. */
static inline void add_divergence(double* r_node, const double sig[3][3], double Dts,
                                  const double* dd, int col, double factor) {
    const double g0 = Dts * dd[col];
    const double g1 = Dts * dd[col + 3];
    const double g2 = Dts * dd[col + 6];
    r_node[0] -= (sig[0][0] * g0 + sig[0][1] * g1 + sig[0][2] * g2) * factor;
    r_node[1] -= (sig[1][0] * g0 + sig[1][1] * g1 + sig[1][2] * g2) * factor;
    r_node[2] -= (sig[2][0] * g0 + sig[2][1] * g1 + sig[2][2] * g2) * factor;
}

static void one_element(int ng, const double* dd_e, const double* jac_e, const double* lam_e,
                        const double* mu_e, const double* D, const double* w, const double* u_e,
                        double* r_e) {
    for (int i = 0; i < ng; ++i)
        for (int j = 0; j < ng; ++j)
            for (int k = 0; k < ng; ++k) {
                const int n = (i * ng + j) * ng + k;
                const double lam = lam_e[n];
                const double mu = mu_e[n];
                if (mu <= 0.0) continue; /* element_cpu.cpp:42-43 */
                const double* dd = dd_e + 9 * n;
                double grad[3][3];
                node_gradient(i, j, k, ng, D, u_e, dd, grad);
                double eps[3][3];
                for (int l = 0; l < 3; ++l)
                    for (int m = 0; m < 3; ++m) eps[l][m] = 0.5 * (grad[l][m] + grad[m][l]);
                const double tr = eps[0][0] + eps[1][1] + eps[2][2];
                double sig[3][3];
                for (int l = 0; l < 3; ++l) {
                    for (int m = 0; m < 3; ++m) sig[l][m] = 2.0 * mu * eps[l][m];
                    sig[l][l] += lam * tr;
                }
                const double factor = jac_e[n] * w[i] * w[j] * w[k];
                for (int s = 0; s < ng; ++s)
                    add_divergence(r_e + 3 * ((s * ng + j) * ng + k), sig, D[i * ng + s], dd, 0,
                                   factor);
                for (int s = 0; s < ng; ++s)
                    add_divergence(r_e + 3 * ((i * ng + s) * ng + k), sig, D[j * ng + s], dd, 1,
                                   factor);
                for (int s = 0; s < ng; ++s)
                    add_divergence(r_e + 3 * ((i * ng + j) * ng + s), sig, D[k * ng + s], dd, 2,
                                   factor);
            }
}

void orc_element_residual(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                          const double* lambda_, const double* mu, const double* D,
                          const double* weights, int32_t ngll, const double* u, double* r) {
    const long nn = (long)ngll * ngll * ngll;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long e = 0; e < n_elem; ++e)
        one_element(ngll, dxi_dx + e * nn * 9, jacobian + e * nn, lambda_ + e * nn, mu + e * nn,
                    D, weights, u + e * nn * 3, r + e * nn * 3);
}

void orc_element_strain(const double* dxi_dx_e, const double* D, int32_t ngll,
                        const double* u_e, double* strain_e) {
    const int ng = ngll;
    for (int i = 0; i < ng; ++i)
        for (int j = 0; j < ng; ++j)
            for (int k = 0; k < ng; ++k) {
                const int n = (i * ng + j) * ng + k;
                double grad[3][3];
                node_gradient(i, j, k, ng, D, u_e, dxi_dx_e + 9 * n, grad);
                double* s = strain_e + 6 * n;
                s[0] = grad[0][0];
                s[1] = grad[1][1];
                s[2] = grad[2][2];
                s[3] = 0.5 * (grad[0][1] + grad[1][0]);
                s[4] = 0.5 * (grad[0][2] + grad[2][0]);
                s[5] = 0.5 * (grad[1][2] + grad[2][1]);
            }
}

/* ------------------------------------------------------------------------
 * Time loop state
 * ---------------------------------------------------------------------- */

struct orc_handle {
    orc_problem p;
    int ng, nn;
    double gll_x[16], gll_w[16], D[256];
    double *u, *v, *a, *ut, *r;          /* global [n_node*3]            */
    double *u_el, *r_el;                 /* element-local [n_cell*nn*3]  */
    double *m_node, *d_node;             /* global [n_node]              */
    int has_cpml;
    double *pml_new, *pml_old, *pml_mem; /* [n_cell*nn*3], [..*3], [..*9] */
    int* src_local;                      /* [n_src] local cell or -1      */
    int step;
};

orc_handle* orc_create(const orc_problem* p) {
    if (!p || p->n_cell < 0 || p->ngll < 2 || p->ngll > 16 || p->n_node < 0) return NULL;
    orc_handle* h = (orc_handle*)calloc(1, sizeof(orc_handle));
    if (!h) return NULL;
    h->p = *p;
    h->ng = p->ngll;
    h->nn = p->ngll * p->ngll * p->ngll;
    if (orc_gll(p->ngll - 1, h->gll_x, h->gll_w, h->D) != 0) {
        free(h);
        return NULL;
    }
    const long G3 = (long)p->n_node * 3;
    const long L3 = (long)p->n_cell * h->nn * 3;
    h->u = calloc(G3 + 1, sizeof(double));
    h->v = calloc(G3 + 1, sizeof(double));
    h->a = calloc(G3 + 1, sizeof(double));
    h->ut = calloc(G3 + 1, sizeof(double));
    h->r = calloc(G3 + 1, sizeof(double));
    h->u_el = calloc(L3 + 1, sizeof(double));
    h->r_el = calloc(L3 + 1, sizeof(double));
    h->m_node = calloc((size_t)p->n_node + 1, sizeof(double));
    h->d_node = calloc((size_t)p->n_node + 1, sizeof(double));
    /* global lumped mass (accumulate) and damping (assign), solver.cpp:195-202 */
    for (long e = 0; e < p->n_cell; ++e)
        for (int n = 0; n < h->nn; ++n) {
            const long q = e * h->nn + n;
            const int g = p->ibool[q];
            h->m_node[g] += p->mass[q];
            h->d_node[g] = p->damping ? p->damping[q] : 0.0;
        }
    /* C-PML memory state, sized for all cells (pml.cpp:41-53) */
    h->has_cpml = (p->pml_coef_abar != NULL && p->pml_region != NULL);
    if (h->has_cpml) {
        h->pml_new = calloc(L3 + 1, sizeof(double));
        h->pml_old = calloc(L3 + 1, sizeof(double));
        h->pml_mem = calloc(L3 * 3 + 1, sizeof(double));
    }
    /* source element lookup by id (solver.cpp:250-258) */
    h->src_local = (int*)malloc(sizeof(int) * (p->n_src > 0 ? p->n_src : 1));
    for (int si = 0; si < p->n_src; ++si) {
        h->src_local[si] = -1;
        for (long e = 0; e < p->n_cell; ++e) {
            const long id = p->cell_ids ? p->cell_ids[e] : e;
            if (id == p->src_cell_ids[si]) {
                h->src_local[si] = (int)e;
                break;
            }
        }
    }
    return h;
}

void orc_destroy(orc_handle* h) {
    if (!h) return;
    free(h->u); free(h->v); free(h->a); free(h->ut); free(h->r);
    free(h->u_el); free(h->r_el); free(h->m_node); free(h->d_node);
    free(h->pml_new); free(h->pml_old); free(h->pml_mem); free(h->src_local);
    free(h);
}

int32_t orc_current_step(const orc_handle* h) { return h->step; }

void orc_get_state(const orc_handle* h, double* u, double* v, double* a) {
    const size_t b = sizeof(double) * (size_t)h->p.n_node * 3;
    if (u) memcpy(u, h->u, b);
    if (v) memcpy(v, h->v, b);
    if (a) memcpy(a, h->a, b);
}

void orc_set_state(orc_handle* h, int32_t step, const double* u, const double* v,
                   const double* a) {
    const size_t b = sizeof(double) * (size_t)h->p.n_node * 3;
    if (u) memcpy(h->u, u, b);
    if (v) memcpy(h->v, v, b);
    if (a) memcpy(h->a, a, b);
    h->step = step;
}

void orc_get_node_mass(const orc_handle* h, double* mass) {
    memcpy(mass, h->m_node, sizeof(double) * (size_t)h->p.n_node);
}

/* gather_from_rank (assembly.cpp:28-41) */
static void gather(const orc_handle* h, const double* glob, double* el) {
    const long total = (long)h->p.n_cell * h->nn;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long q = 0; q < total; ++q) {
        const long g = h->p.ibool[q];
        el[q * 3 + 0] = glob[g * 3 + 0];
        el[q * 3 + 1] = glob[g * 3 + 1];
        el[q * 3 + 2] = glob[g * 3 + 2];
    }
}

/* scatter_to_rank (assembly.cpp:10-26): zero, then element-major sum */
static void scatter(const orc_handle* h, const double* el, double* glob) {
    memset(glob, 0, sizeof(double) * (size_t)h->p.n_node * 3);
    const long total = (long)h->p.n_cell * h->nn;
    for (long q = 0; q < total; ++q) {
        const long g = h->p.ibool[q];
        glob[g * 3 + 0] += el[q * 3 + 0];
        glob[g * 3 + 1] += el[q * 3 + 1];
        glob[g * 3 + 2] += el[q * 3 + 2];
    }
}

static const double kTheta = 1.0 / 8.0; /* pml.cpp:35 */

static inline int pml_region_of(const orc_handle* h, long e) { return h->p.pml_region[e]; }

/* cpml_update_displ_fields (pml.cpp:55-110) */
static void cpml_fields(orc_handle* h) {
    const double dt = h->p.dt;
    const double c1 = (1.0 - 2.0 * kTheta) * 0.5 * dt;
    const double c2 = (1.0 - kTheta) * 0.5 * dt * dt;
    double* t = h->pml_old;
    h->pml_old = h->pml_new;
    h->pml_new = t;
    const int nn = h->nn;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long e = 0; e < h->p.n_cell; ++e) {
        if (pml_region_of(h, e) == 0) continue;
        for (int n = 0; n < nn; ++n) {
            const long q = e * nn + n;
            const long g = h->p.ibool[q];
            for (int d = 0; d < 3; ++d)
                h->pml_new[q * 3 + d] = h->u[g * 3 + d] + c1 * h->v[g * 3 + d];
        }
    }
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long e = 0; e < h->p.n_cell; ++e) {
        if (pml_region_of(h, e) == 0) continue;
        for (int n = 0; n < nn; ++n) {
            const long q = e * nn + n;
            const long g = h->p.ibool[q];
            for (int d = 0; d < 3; ++d) h->pml_old[q * 3 + d] += c2 * h->a[g * 3 + d];
        }
    }
}

/* cpml_accel_contribution (pml.cpp:151-216) */
static void cpml_accel(orc_handle* h) {
    const int ng = h->ng, nn = h->nn;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long e = 0; e < h->p.n_cell; ++e) {
        if (pml_region_of(h, e) == 0) continue;
        for (int n = 0; n < nn; ++n) {
            const int nk = n % ng, nj = (n / ng) % ng, ni = n / (ng * ng);
            const double wgll = h->gll_w[ni] * h->gll_w[nj] * h->gll_w[nk];
            const long q = e * nn + n;
            const long g = h->p.ibool[q];
            const double rho = h->p.density[q];
            const double jac = h->p.jacobian[q];
            const double rho_inv = (rho > 0.0) ? 1.0 / rho : 0.0;
            const double* A = h->p.pml_coef_abar + q * 5;
            const double scale = wgll * rho_inv * jac;
            for (int c = 0; c < 3; ++c) {
                const double uu = h->u[g * 3 + c];
                const double vv = h->v[g * 3 + c];
                const double* m = h->pml_mem + q * 9 + c * 3;
                const double acc =
                    scale * (A[0] * vv + A[1] * uu + A[2] * m[0] + A[3] * m[1] + A[4] * m[2]);
                h->r_el[q * 3 + c] += acc;
            }
        }
    }
}

/* cpml_update_displ_memory (pml.cpp:112-149) */
static void cpml_memory(orc_handle* h) {
    const int nn = h->nn;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long e = 0; e < h->p.n_cell; ++e) {
        if (pml_region_of(h, e) == 0) continue;
        for (int n = 0; n < nn; ++n) {
            const long q = e * nn + n;
            const double* coef = h->p.pml_coef_alpha + q * 9;
            for (int c = 0; c < 3; ++c) {
                const double nv = h->pml_new[q * 3 + c];
                const double ov = h->pml_old[q * 3 + c];
                for (int d = 0; d < 3; ++d) {
                    double* m = h->pml_mem + q * 9 + c * 3 + d;
                    *m = coef[d * 3 + 0] * *m + coef[d * 3 + 1] * nv + coef[d * 3 + 2] * ov;
                }
            }
        }
    }
}

int32_t orc_advance(orc_handle* h, int32_t n_steps, int32_t max_snap, int32_t* rec_step,
                    double* rec_strain, double* rec_u, double* rec_v, double* rec_a) {
    const orc_problem* p = &h->p;
    const int ng = h->ng, nn = h->nn;
    const double dt = p->dt;
    const double beta = 0.0, gamma = 0.5; /* solver.cpp:338-339 */
    const long G3 = (long)p->n_node * 3;
    int32_t n_snap = 0;
    for (int32_t it = 0; it < n_steps; ++it) {
        const int step = h->step;
        /* 1. Newmark predictor (solver.cpp:40-49) */
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
        for (long i = 0; i < G3; ++i)
            h->ut[i] = h->u[i] + dt * h->v[i] + (0.5 * dt * dt * (1.0 - 2.0 * beta)) * h->a[i];
        /* 3. gather predicted displacement (solver.cpp:539-542) */
        gather(h, h->ut, h->u_el);
        /* 3a. C-PML fields before the kernel (solver.cpp:545-548) */
        if (h->has_cpml) cpml_fields(h);
        /* 3b. zero + element kernel (solver.cpp:551-555) */
        memset(h->r_el, 0, sizeof(double) * (size_t)p->n_cell * nn * 3);
        orc_element_residual(p->n_cell, p->dxi_dx, p->jacobian, p->lambda_, p->mu, h->D,
                             h->gll_w, ng, h->u_el, h->r_el);
        /* 4. C-PML accel, else legacy velocity damping (solver.cpp:558-574) */
        if (h->has_cpml) {
            cpml_accel(h);
        } else {
            for (long g = 0; g < p->n_node; ++g) {
                const double d = h->d_node[g];
                if (d > 0.0) {
                    h->v[g * 3 + 0] -= d * h->v[g * 3 + 0];
                    h->v[g * 3 + 1] -= d * h->v[g * 3 + 1];
                    h->v[g * 3 + 2] -= d * h->v[g * 3 + 2];
                }
            }
        }
        /* 5. source injection (solver.cpp:577-605) */
        {
            const double sv = (step < p->n_stf) ? p->stf[step] : 0.0;
            if (sv != 0.0) {
                for (int si = 0; si < p->n_src; ++si) {
                    const int el = h->src_local[si];
                    if (el < 0) continue;
                    for (int k = 0; k < ng; ++k)
                        for (int j = 0; j < ng; ++j)
                            for (int i = 0; i < ng; ++i) {
                                const int node = (i * ng + j) * ng + k;
                                const double wv = p->src_weights[(long)si * nn + node];
                                if (wv == 0.0) continue;
                                h->r_el[((long)el * nn + node) * 3 + p->direction] += sv * wv;
                            }
                }
            }
        }
        /* 6. scatter (solver.cpp:608-609) */
        scatter(h, h->r_el, h->r);
        /* 7. Newmark corrector (solver.cpp:52-69) */
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
        for (long i = 0; i < G3; ++i) {
            const double m = h->m_node[i / 3];
            if (m <= 0.0) {
                h->a[i] = 0.0;
                continue;
            }
            const double a_old = h->a[i];
            const double a_new = h->r[i] / m;
            h->u[i] += dt * h->v[i] + dt * dt * ((0.5 - beta) * a_old + beta * a_new);
            h->v[i] += dt * ((1.0 - gamma) * a_old + gamma * a_new);
            h->a[i] = a_new;
        }
        /* 8. C-PML memory after the corrector (solver.cpp:619-621) */
        if (h->has_cpml) cpml_memory(h);
        /* snapshot (solver.cpp:631-675): strain from the gathered corrected u */
        if (p->snapshot_stride > 0 && step % p->snapshot_stride == 0 && p->n_rec > 0) {
            if (n_snap >= max_snap) return -1;
            if (rec_step) rec_step[n_snap] = step;
            const long base = (long)n_snap * p->n_rec * nn;
            double u_e[3 * 4096];
            for (int ci = 0; ci < p->n_rec; ++ci) {
                const long e = p->rec_cell_local[ci];
                for (int n = 0; n < nn; ++n) {
                    const long g = p->ibool[e * nn + n];
                    for (int d = 0; d < 3; ++d) u_e[n * 3 + d] = h->u[g * 3 + d];
                }
                if (rec_strain)
                    orc_element_strain(p->dxi_dx + e * nn * 9, h->D, ng, u_e,
                                       rec_strain + (base + (long)ci * nn) * 6);
                for (int n = 0; n < nn; ++n) {
                    const long g = p->ibool[e * nn + n];
                    const long o = (base + (long)ci * nn + n) * 3;
                    for (int d = 0; d < 3; ++d) {
                        if (rec_u) rec_u[o + d] = h->u[g * 3 + d];
                        if (rec_v) rec_v[o + d] = h->v[g * 3 + d];
                        if (rec_a) rec_a[o + d] = h->a[g * 3 + d];
                    }
                }
            }
            ++n_snap;
        }
        h->step++;
    }
    return n_snap;
}
