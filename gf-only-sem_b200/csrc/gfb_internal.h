// gfb_internal.h -- helpers shared between the translation units of libgfb.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/gfb.h"

namespace gfb {

// Record `msg` as this thread's gfb_last_error() and return `st`.
gfb_status set_error(gfb_status st, const char* msg);

// GLL weights and derivative matrix for ngll points per axis.
bool gll_tables_for(int ngll, std::vector<double>& w, std::vector<double>& D);

// What other translation units see of a solver: its stream, sizes and the
// device arrays of the time loop (layouts of gfb_kernels.cuh).
struct SolverView {
    int device = 0;
    cudaStream_t stream = nullptr;
    int precision = GFB_FP64;
    int n_field = 1;
    int n_model = 1;
    long long n_node = 0;
    double dt = 0.0;
    double* u = nullptr;           // [node][3*n_field]
    double* v = nullptr;
    void* a = nullptr;             // Real [node][3*n_field]
    void* ut = nullptr;            // Real [node][n_field][4]
    void* force = nullptr;         // Real [node][n_field][4]
    const double* mass = nullptr;  // [node]
    const int* mstep = nullptr;    // [model] next step index (device)
    const std::vector<int>* node_inv = nullptr;   // node -> device node (empty: identity)
    const std::vector<int>* node_perm = nullptr;  // device node -> node (empty: identity)
};

SolverView solver_view(gfb_solver* s);

// Recompute the predicted displacement from u, v, a on the solver's stream
// (after u, v, a were written from outside the time loop).
gfb_status solver_predict(gfb_solver* s);

// Keep (u, v, a) at every node from now on (the FP32 path otherwise holds
// the half-step velocity and no acceleration at its plain nodes); for code
// that reads or writes v and a of any node between steps.
gfb_status solver_full_state(gfb_solver* s);

// Learned absorbing layer attached to a solver (gfb_layer.cu): launched
// between the element phase and the node phase of every step; freed with the
// solver.
struct Layer;
gfb_status layer_step(gfb_solver* s, Layer* layer);
void layer_free(Layer* layer);
Layer* solver_layer(gfb_solver* s);
gfb_status solver_set_layer(gfb_solver* s, Layer* layer);

}  // namespace gfb
