/*
 * sem_oracle.h -- CPU FP64 oracle of the CG-SEM elastic time loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The product library never links or calls it.
 *
 * It restates the CPU branch of the reference forward solver
 * (forward/share/src/solver.cpp:510-688) together with the functions that
 * branch calls:
 *   - GLL tables                 forward/share/include/gf/gll.hpp:48-131
 *   - element internal force     forward/elastic/src/element_cpu.cpp:19-162
 *   - gather / scatter           forward/share/src/assembly.cpp:10-41
 *   - C-PML fields/accel/memory  forward/share/src/pml.cpp:55-216
 *   - Newmark predict / correct  forward/share/src/solver.cpp:40-69
 *   - global mass / damping      forward/share/src/solver.cpp:193-202
 *   - source injection           forward/share/src/solver.cpp:577-605
 *   - snapshot strain + copy-out forward/share/src/solver.cpp:282-335, 640-675
 * Every floating-point expression is evaluated in the same order as in the
 * reference so that, compiled without FP contraction, the results are
 * bit-identical to the reference's own compiled functions (oracle/_ref).
 */
#ifndef GF_SEM_ORACLE_H
#define GF_SEM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Merged partition set plus run configuration (RankData + ConfigData,
 * forward/share/include/gf/types.hpp:27-140).  All arrays are borrowed for
 * the lifetime of the handle. */
typedef struct orc_problem {
    int32_t n_cell;            /* n_local_cell                                   */
    int32_t ngll;              /* N+1                                            */
    int32_t n_node;            /* n_rank_node (max ibool + 1)                    */
    const int32_t* ibool;      /* [n_cell*ngll^3] local_cell2rank_node           */
    const int64_t* cell_ids;   /* [n_cell] local_cell_ids, NULL -> 0..n_cell-1   */
    const double* dxi_dx;      /* [n_cell*ngll^3*9]                              */
    const double* jacobian;    /* [n_cell*ngll^3]                                */
    const double* lambda_;     /* [n_cell*ngll^3]                                */
    const double* mu;          /* [n_cell*ngll^3]                                */
    const double* density;     /* [n_cell*ngll^3]  (C-PML only)                  */
    const double* mass;        /* [n_cell*ngll^3]  element-local lumped mass     */
    const double* damping;     /* [n_cell*ngll^3]  legacy ramp, NULL -> zeros    */
    const int32_t* pml_region; /* [n_cell]         NULL -> no C-PML              */
    const double* pml_coef_alpha; /* [n_cell*ngll^3*9]                           */
    const double* pml_coef_abar;  /* [n_cell*ngll^3*5]; NULL -> no C-PML         */
    double dt;
    int32_t snapshot_stride;   /* <= 0 disables snapshots                        */
    int32_t direction;         /* 0=x 1=y 2=z                                    */
    int32_t n_src;
    const int64_t* src_cell_ids;  /* [n_src] cell ids matched against cell_ids  */
    const double* src_weights;    /* [n_src*ngll^3]                              */
    int32_t n_stf;
    const double* stf;            /* [n_stf] stf_values                          */
    int32_t n_rec;
    const int32_t* rec_cell_local; /* [n_rec] merged local cell indices          */
} orc_problem;

typedef struct orc_handle orc_handle;

/* GLL nodes, weights and derivative matrix D[i*ngll+j] = l_j'(xi_i).
 * Returns 0 on success, -1 if N < 1 or the Newton iteration breaks down. */
int orc_gll(int32_t N, double* nodes, double* weights, double* D);

/* r += K_e u for n_elem elements (element_cpu.cpp:19-162). */
void orc_element_residual(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                          const double* lambda_, const double* mu, const double* D,
                          const double* weights, int32_t ngll, const double* u, double* r);

/* Strain (Voigt xx,yy,zz,xy,xz,yz) at every node of one element from its
 * element-local displacement (solver.cpp:282-335). */
void orc_element_strain(const double* dxi_dx_e, const double* D, int32_t ngll,
                        const double* u_e, double* strain_e);

/* Threads used by orc_advance for element-parallel loops (results do not
 * depend on the count). */
void orc_set_threads(int32_t n);

orc_handle* orc_create(const orc_problem* p);
void orc_destroy(orc_handle* h);

/* Advance n_steps solver steps.  At each step with step % stride == 0 a
 * snapshot of the recording cells is appended to the caller buffers:
 *   rec_strain [max_snap, n_rec, ngll^3, 6]
 *   rec_u/v/a  [max_snap, n_rec, ngll^3, 3]
 *   rec_step   [max_snap]
 * Any buffer may be NULL.  Returns the number of snapshots written, or -1
 * when more than max_snap snapshots fall in the range. */
int32_t orc_advance(orc_handle* h, int32_t n_steps, int32_t max_snap, int32_t* rec_step,
                    double* rec_strain, double* rec_u, double* rec_v, double* rec_a);

int32_t orc_current_step(const orc_handle* h);

/* Copy global state [n_node*3] (u, v, a). */
void orc_get_state(const orc_handle* h, double* u, double* v, double* a);
void orc_set_state(orc_handle* h, int32_t step, const double* u, const double* v,
                   const double* a);

/* Assembled global lumped mass [n_node]. */
void orc_get_node_mass(const orc_handle* h, double* mass);

#ifdef __cplusplus
}
#endif
#endif
