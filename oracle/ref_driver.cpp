// ref_driver.cpp -- drives the reference's own compiled CPU functions.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the
// reference sources forward/elastic/src/element_cpu.cpp,
// forward/share/src/assembly.cpp and forward/share/src/pml.cpp (unmodified,
// compiled where they lie) into oracle/_ref/libgf_ref.so.  The functions the
// reference keeps inside run_forward (Newmark predict/correct in an
// anonymous namespace, solver.cpp:40-69; mass/damping assembly 193-202;
// source loop 577-605; snapshot strain lambda 282-335) cannot be linked
// because solver.cpp needs HDF5, so this file restates the CPU loop of
// solver.cpp:510-688 around the linked reference functions.
//
// It exports the same C interface as sem_oracle.h with the prefix ref_
// instead of orc_, so tests can run both on identical inputs.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../sem_oracle.h"
#include "gf/assembly.hpp"
#include "gf/element.hpp"
#include "gf/gll.hpp"
#include "gf/pml.hpp"
#include "gf/types.hpp"

namespace {

int g_ref_threads = 1;

struct RefRun {
    orc_problem p{};
    gf::RankData part;
    std::vector<double> gll_w, D;
    std::vector<double> u, v, a, ut, r, m_node, d_node;
    std::vector<double> u_el, r_el;
    std::vector<int> src_local;
    int ng = 0, nn = 0, step = 0;
};

// compute_element_residual<BackendCPU> on disjoint element ranges from
// several threads; each call only writes its own elements' residual.
void element_residual_threaded(RefRun& s) {
    const int n_cell = s.part.n_local_cell;
    const int nt = std::max(1, std::min(g_ref_threads, n_cell > 0 ? n_cell : 1));
    auto run = [&](int e0, int e1) {
        if (e1 <= e0) return;
        const size_t nn = s.nn;
        gf::compute_element_residual<gf::BackendCPU>(
            e1 - e0, s.part.dxi_dx.data() + e0 * nn * 9, s.part.jacobian.data() + e0 * nn,
            s.part.lambda_.data() + e0 * nn, s.part.mu_.data() + e0 * nn, s.D.data(),
            s.gll_w.data(), s.ng, s.u_el.data() + e0 * nn * 3, s.r_el.data() + e0 * nn * 3);
    };
    if (nt == 1) {
        run(0, n_cell);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) {
        const int e0 = (int)((long)n_cell * t / nt), e1 = (int)((long)n_cell * (t + 1) / nt);
        pool.emplace_back(run, e0, e1);
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

void ref_set_threads(int32_t n) { g_ref_threads = n < 1 ? 1 : n; }

int ref_gll(int32_t N, double* nodes, double* weights, double* D) {
    try {
        auto x = gf::gll_nodes(N);
        auto w = gf::gll_weights(N, x);
        auto d = gf::gll_derivative_matrix(N, x);
        std::memcpy(nodes, x.data(), x.size() * sizeof(double));
        std::memcpy(weights, w.data(), w.size() * sizeof(double));
        std::memcpy(D, d.data(), d.size() * sizeof(double));
        return 0;
    } catch (...) {
        return -1;
    }
}

void ref_element_residual(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                          const double* lambda_, const double* mu, const double* D,
                          const double* weights, int32_t ngll, const double* u, double* r) {
    gf::compute_element_residual<gf::BackendCPU>(n_elem, dxi_dx, jacobian, lambda_, mu, D,
                                                 weights, ngll, u, r);
}

void* ref_create(const orc_problem* p) {
    if (!p || p->ngll < 2) return nullptr;
    auto* s = new RefRun();
    s->p = *p;
    s->ng = p->ngll;
    s->nn = p->ngll * p->ngll * p->ngll;
    const size_t L = (size_t)p->n_cell * s->nn;
    gf::RankData& part = s->part;
    part.n_local_cell = p->n_cell;
    part.ngll = p->ngll;
    part.n_rank_node = p->n_node;
    part.dxi_dx.assign(p->dxi_dx, p->dxi_dx + L * 9);
    part.jacobian.assign(p->jacobian, p->jacobian + L);
    part.lambda_.assign(p->lambda_, p->lambda_ + L);
    part.mu_.assign(p->mu, p->mu + L);
    part.mass.assign(p->mass, p->mass + L);
    if (p->density) part.density.assign(p->density, p->density + L);
    if (p->damping) part.pml_damping.assign(p->damping, p->damping + L);
    else part.pml_damping.assign(L, 0.0);
    part.local_cell2rank_node.assign(p->ibool, p->ibool + L);
    if (p->cell_ids) part.local_cell_ids.assign(p->cell_ids, p->cell_ids + p->n_cell);
    else
        for (int e = 0; e < p->n_cell; ++e) part.local_cell_ids.push_back(e);
    if (p->pml_region && p->pml_coef_abar) {
        part.pml_region.assign(p->pml_region, p->pml_region + p->n_cell);
        part.pml_coef_alpha.assign(p->pml_coef_alpha, p->pml_coef_alpha + L * 9);
        part.pml_coef_abar.assign(p->pml_coef_abar, p->pml_coef_abar + L * 5);
        part.has_cpml = true;
        gf::cpml_initialize(part, s->nn);
    }
    auto x = gf::gll_nodes(p->ngll - 1);
    s->gll_w = gf::gll_weights(p->ngll - 1, x);
    s->D = gf::gll_derivative_matrix(p->ngll - 1, x);
    const size_t G3 = (size_t)p->n_node * 3;
    s->u.assign(G3, 0.0);
    s->v.assign(G3, 0.0);
    s->a.assign(G3, 0.0);
    s->ut.assign(G3, 0.0);
    s->r.assign(G3, 0.0);
    s->u_el.assign(L * 3, 0.0);
    s->r_el.assign(L * 3, 0.0);
    // solver.cpp:193-202
    s->m_node.assign(p->n_node, 0.0);
    s->d_node.assign(p->n_node, 0.0);
    for (int e = 0; e < p->n_cell; ++e)
        for (int n = 0; n < s->nn; ++n) {
            const int g = part.local_cell2rank_node[(size_t)e * s->nn + n];
            s->m_node[g] += part.mass[(size_t)e * s->nn + n];
            s->d_node[g] = part.pml_damping[(size_t)e * s->nn + n];
        }
    // solver.cpp:250-258
    s->src_local.assign(p->n_src, -1);
    for (int si = 0; si < p->n_src; ++si)
        for (int e = 0; e < p->n_cell; ++e)
            if (part.local_cell_ids[e] == p->src_cell_ids[si]) {
                s->src_local[si] = e;
                break;
            }
    return s;
}

void ref_destroy(void* h) { delete static_cast<RefRun*>(h); }

int32_t ref_current_step(const void* h) { return static_cast<const RefRun*>(h)->step; }

void ref_get_state(const void* h, double* u, double* v, double* a) {
    auto* s = static_cast<const RefRun*>(h);
    if (u) std::memcpy(u, s->u.data(), s->u.size() * sizeof(double));
    if (v) std::memcpy(v, s->v.data(), s->v.size() * sizeof(double));
    if (a) std::memcpy(a, s->a.data(), s->a.size() * sizeof(double));
}

int32_t ref_advance(void* h, int32_t n_steps, int32_t max_snap, int32_t* rec_step,
                    double* rec_strain, double* rec_u, double* rec_v, double* rec_a) {
    auto& s = *static_cast<RefRun*>(h);
    const orc_problem& p = s.p;
    const int ng = s.ng, nn = s.nn;
    const double beta = 0.0, gamma = 0.5, dt = p.dt;
    int32_t n_snap = 0;
    for (int32_t it = 0; it < n_steps; ++it) {
        const int step = s.step;
        for (size_t i = 0; i < s.u.size(); ++i)
            s.ut[i] = s.u[i] + dt * s.v[i] + (0.5 * dt * dt * (1.0 - 2.0 * beta)) * s.a[i];
        gf::gather_from_rank(s.ut, s.part.local_cell2rank_node, p.n_cell, nn, s.u_el);
        if (s.part.has_cpml) gf::cpml_update_displ_fields(s.part, s.u, s.v, s.a, dt, nn);
        std::fill(s.r_el.begin(), s.r_el.end(), 0.0);
        element_residual_threaded(s);
        if (s.part.has_cpml) {
            gf::cpml_accel_contribution(s.part, s.u, s.v, s.part.local_cell2rank_node, s.gll_w,
                                        s.r_el, p.n_cell, nn);
        } else {
            for (int g = 0; g < p.n_node; ++g) {
                const double d = s.d_node[g];
                if (d > 0.0)
                    for (int c = 0; c < 3; ++c) s.v[g * 3 + c] -= d * s.v[g * 3 + c];
            }
        }
        const double sv = (step < p.n_stf) ? p.stf[step] : 0.0;
        if (sv != 0.0)
            for (int si = 0; si < p.n_src; ++si) {
                const int el = s.src_local[si];
                if (el < 0) continue;
                for (int k = 0; k < ng; ++k)
                    for (int j = 0; j < ng; ++j)
                        for (int i = 0; i < ng; ++i) {
                            const int node = (i * ng + j) * ng + k;
                            const double wv = p.src_weights[(size_t)si * nn + node];
                            if (wv == 0.0) continue;
                            s.r_el[((size_t)el * nn + node) * 3 + p.direction] += sv * wv;
                        }
            }
        gf::scatter_to_rank(s.r_el, s.part.local_cell2rank_node, p.n_cell, nn, s.r);
        for (size_t i = 0; i < s.r.size(); ++i) {
            const double m = s.m_node[i / 3];
            if (m <= 0.0) {
                s.a[i] = 0.0;
                continue;
            }
            const double a_old = s.a[i];
            const double a_new = s.r[i] / m;
            s.u[i] += dt * s.v[i] + dt * dt * ((0.5 - beta) * a_old + beta * a_new);
            s.v[i] += dt * ((1.0 - gamma) * a_old + gamma * a_new);
            s.a[i] = a_new;
        }
        if (s.part.has_cpml) gf::cpml_update_displ_memory(s.part, nn);
        if (p.snapshot_stride > 0 && step % p.snapshot_stride == 0 && p.n_rec > 0) {
            if (n_snap >= max_snap) return -1;
            if (rec_step) rec_step[n_snap] = step;
            const size_t base = (size_t)n_snap * p.n_rec * nn;
            for (int ci = 0; ci < p.n_rec; ++ci) {
                const int e = p.rec_cell_local[ci];
                std::vector<double> ue(nn * 3);
                for (int n = 0; n < nn; ++n) {
                    const int g = s.part.local_cell2rank_node[(size_t)e * nn + n];
                    for (int d = 0; d < 3; ++d) ue[n * 3 + d] = s.u[g * 3 + d];
                }
                for (int i = 0; i < ng; ++i)
                    for (int j = 0; j < ng; ++j)
                        for (int k = 0; k < ng; ++k) {
                            const int n = (i * ng + j) * ng + k;
                            const double* dx = &s.part.dxi_dx[((size_t)e * nn + n) * 9];
                            double gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0}, gz[3] = {0, 0, 0};
                            for (int q = 0; q < ng; ++q) {
                                const double Di = s.D[i * ng + q], Dj = s.D[j * ng + q],
                                             Dk = s.D[k * ng + q];
                                const int a0 = (q * ng + j) * ng + k, a1 = (i * ng + q) * ng + k,
                                          a2 = (i * ng + j) * ng + q;
                                for (int d = 0; d < 3; ++d) {
                                    gx[d] += Di * ue[3 * a0 + d];
                                    gy[d] += Dj * ue[3 * a1 + d];
                                    gz[d] += Dk * ue[3 * a2 + d];
                                }
                            }
                            double du[3][3];
                            for (int c = 0; c < 3; ++c) {
                                du[c][0] = gx[c] * dx[0] + gy[c] * dx[1] + gz[c] * dx[2];
                                du[c][1] = gx[c] * dx[3] + gy[c] * dx[4] + gz[c] * dx[5];
                                du[c][2] = gx[c] * dx[6] + gy[c] * dx[7] + gz[c] * dx[8];
                            }
                            if (rec_strain) {
                                double* o = rec_strain + (base + (size_t)ci * nn + n) * 6;
                                o[0] = du[0][0];
                                o[1] = du[1][1];
                                o[2] = du[2][2];
                                o[3] = 0.5 * (du[0][1] + du[1][0]);
                                o[4] = 0.5 * (du[0][2] + du[2][0]);
                                o[5] = 0.5 * (du[1][2] + du[2][1]);
                            }
                            const int g = s.part.local_cell2rank_node[(size_t)e * nn + n];
                            const size_t o3 = (base + (size_t)ci * nn + n) * 3;
                            for (int d = 0; d < 3; ++d) {
                                if (rec_u) rec_u[o3 + d] = s.u[g * 3 + d];
                                if (rec_v) rec_v[o3 + d] = s.v[g * 3 + d];
                                if (rec_a) rec_a[o3 + d] = s.a[g * 3 + d];
                            }
                        }
            }
            ++n_snap;
        }
        s.step++;
    }
    return n_snap;
}

}  // extern "C"
