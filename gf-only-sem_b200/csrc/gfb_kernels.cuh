// gfb_kernels.cuh -- sm_100a kernels of the CG-SEM elastic time loop.
//
// One time step is NC colour launches of elem_step_kernel followed by one
// launch of node_update_kernel:
//
//   elem_step_kernel (colour c)  -- for every cell of colour c: gather the
//       predicted displacement through ibool into shared memory, GLL
//       derivative contractions, stress, weighted transposed-derivative
//       divergence (forward/elastic/src/element_cpu.cpp:19-162), C-PML
//       acceleration term and memory update on C-PML cells
//       (forward/share/src/pml.cpp:55-216), point-force injection
//       (forward/share/src/solver.cpp:577-605), then a plain read-modify-
//       write of the global force.  Cells of one colour share no node, and
//       colours run in a fixed order, so assembly needs no atomics and is
//       bit-reproducible run to run.  The first colour touching a node
//       stores instead of adding, which replaces the memset of the global
//       residual (cuda_step.cu:289-290).
//   node_update_kernel -- Newmark corrector with the diagonal mass and the
//       legacy velocity damping (solver.cpp:52-69, 564-574), followed by the
//       predictor of the next step (solver.cpp:40-49), so no separate
//       predictor launch is needed.
//
// Layouts on the device (cells in colour order):
//   ibool  [cell][NN]            node id | FIRST_TOUCH bit
//   geom   [cell][12][NN] Real   dxi_dx(9), jac*w_i*w_j*w_k, lambda, mu
//   state  u, v (double), a (Real): [node][3*n_field];
//          predicted displacement ut and force (Real): [node][n_field][4]
//   C-PML  coef [slot][15][NN] Real (alpha 9, abar 5, w*J/rho),
//          mem [slot][n_field*9][NN], prev [slot][n_field*3][NN]
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gfb {

constexpr uint32_t kFirstTouch = 0x80000000u;  // lowest colour touching the node: store
constexpr uint32_t kLastTouch = 0x40000000u;   // highest colour touching the node: finalise
constexpr uint32_t kNodeMask = 0x3fffffffu;

// Predicted displacement and force of the time loop are stored
// [node][field][4] (x, y, z, pad) so a field of a node is one 16-byte
// vector; u, v, a are [node][3*field].  Index of component f of node g.
__device__ __forceinline__ long long padded_index(long long g, int f, int F) {
    return g * (F / 3) * 4 + (f / 3) * 4 + (f % 3);
}

// Node-table rows used by the pipelined kernels: the NN node words of a
// cell, then the index of the model the cell belongs to, padded to whole
// 16-byte copies.
__host__ __device__ constexpr int ib_row_words(int nn) { return (nn + 1 + 3) / 4 * 4; }

// Time-step constants of one model (several independent models can share
// one solver): dt, dt^2/2 (beta = 0) and the C-PML field coefficients
// c1 = (1-2 theta) dt/2, c2 = (1-theta) dt^2/2 of pml.cpp:35, 63-64.
struct ModelConst {
    double dt, half_dt2, c1, c2;
};
constexpr int kMaxModels = 255;
// Wavefields one solver advances together: force directions times source
// positions (a source set per position, each with its cells, weights and
// source time function).
constexpr int kMaxFields = 12;

// Direction and source set of wavefield f (kernel parameters are indexed
// with compile-time indices only).
template <int NFLD>
__device__ __forceinline__ void field_source(const int (&dir)[kMaxFields], const int (&fset)[kMaxFields], int f,
                                             int& d, int& k) {
    d = dir[0];
    k = fset[0];
#pragma unroll
    for (int q = 1; q < NFLD; ++q)
        if (f == q) {
            d = dir[q];
            k = fset[q];
        }
}

template <int NG>
struct Shape {
    static constexpr int NN = NG * NG * NG;
    static constexpr int NNP = (NN + 31) / 32 * 32;
    static constexpr int EPB = NNP <= 32 ? 8 : (NNP <= 64 ? 4 : (NNP <= 128 ? 2 : 1));
    static constexpr int THREADS = NNP * EPB;
};

template <typename Real>
struct NodeArgs {
    long long n_node;
    double* u;              // [node][3*n_field]
    double* v;
    Real* a;
    Real* ut;               // [node][field][4]
    const Real* force;      // [node][field][4]
    const double* mass;     // [n_node] assembled lumped mass
    const Real* inv_mass;   // [n_node] 1/m (FP32 path) or nullptr
    const double* damping;  // [n_node] or nullptr
    double dt, half_dt2, beta, gamma;
    // several models: model of each node, its constants, whether it still steps
    const uint8_t* node_model;
    const ModelConst* mc;
    const int* mlive;
    const long long* live_node_end;  // [2] end of the stepping C-PML / plain nodes (several models), or null
    // [model] 1 when the model's next step evaluates the element force in
    // full (the node pass then stores the predicted displacement), 0 when
    // it adds the force of the step's increment (the node pass stores the
    // increment of the predicted displacement); nullptr: always in full
    const int* mnext;
    // plain nodes keep the half-step velocity w = v + dt/2 a (in float, in
    // w32 [node][3*n_field]) and no acceleration (see update_node_field)
    bool half_v;
    float* w32;
};

// C-PML at global nodes (FP32 path).
//
// The reference keeps C-PML memory per cell and GLL node (pml.cpp:112-149)
// and adds each cell's term w J/rho (A1 v + A2 u + A3 m_x + A4 m_y + A5 m_z)
// to the cell residual before assembly (pml.cpp:151-216).  At a node shared
// by several C-PML cells the memory of an axis that is active in those
// cells follows the same recursion m = a0 m + a1 new + a2 old with the same
// new/old (they are node values) and the same axis coefficients (functions
// of the node position), and A_{3+q} = 0 exactly in cells where axis q is
// inactive.  So the memory is kept once per node and axis, and the assembled
// term is B1 v + B2 u + B3 m_x + B4 m_y + B5 m_z with B_k = sum over the
// node's C-PML cells of w J/rho A_k.  The host checks the axis coefficients
// agree across cells before choosing this form.
// The C-PML nodes are the device nodes [0, n_slot): a node's slot is its
// index.
template <typename Real>
struct NodePml {
    const Real* coef;    // [slot][14]: B1..B5, alpha x(3), y(3), z(3)
    Real* mem;           // [axis][slot][F]; only live axes are read or written
    Real* prev;          // [slot][F]  last step's u + c1 v
    long long n_slot;
    double c1, c2;
};

template <typename Real>
struct ElemArgs {
    int e_begin, e_end;
    const uint32_t* ibool;
    const Real* geom;
    const Real* ut;
    Real* force;
    const Real* dmat;  // [NG*NG]
    // C-PML
    const int* pml_slot;   // [cell] -1 if not a C-PML cell
    const Real* pml_coef;  // [slot][15][NN]
    Real* pml_mem;         // [slot][F*3][NN]
    Real* pml_prev;        // [slot][F][NN]
    const double* u;     // [node][3*n_field]
    const double* v;
    const Real* a;
    long long n_node;
    double c1, c2;
    // source
    const int* src_head;  // [cell] first source slot or -1
    const int* src_next;  // [slot]
    const Real* src_w;    // [slot][NN]
    const Real* mstf;     // [model][set] source time function value of this step (nullptr: none)
    const int* src_set;   // [slot] source set of the slot (nullptr: every slot is set 0)
    int n_set;            // source sets (one per source position)
    const int* mlive;     // [model] 1 while the model still steps
    const int* mdirect;   // [model] 1: this step evaluates the force in full (first touch stores), 0: adds the
                          // increment's force to the stored one; nullptr: in full
    const ModelConst* mc; // [model]
    int dir[kMaxFields];  // force direction of each wavefield
    int fset[kMaxFields]; // source set of each wavefield
    // finalisation of the nodes whose last touching colour this is (the
    // node update fused into the element kernel); fuse == 0 keeps the
    // force in memory for a separate node pass
    int fuse;
    NodeArgs<Real> nu;
    NodePml<Real> np;
};

template <typename Real, int NG, int NFLD>
__device__ __forceinline__ void elem_body(const ElemArgs<Real>& A, Real* smem) {
    using S = Shape<NG>;
    constexpr int NN = S::NN, NNP = S::NNP, EPB = S::EPB, F = 3 * NFLD;
    Real* sD = smem;                       // NG*NG, padded to 64
    Real* su = smem + 64;                  // [EPB][F][NNP]
    Real* sG = su + EPB * F * NNP;         // [EPB][3*F][NNP]
    const int tid = threadIdx.x;
    const int el = tid / NNP, p = tid - el * NNP;
    const int e = A.e_begin + blockIdx.x * EPB + el;
    const bool active = (p < NN) && (e < A.e_end);
    if (tid < NG * NG) sD[tid] = A.dmat[tid];
    Real* mu_s = su + el * F * NNP;
    Real* mG = sG + el * 3 * F * NNP;

    uint32_t gword = 0;
    Real dd[9], jw = Real(0), lam = Real(0), mu = Real(0);
    if (active) {
        gword = __ldg(A.ibool + (size_t)e * NN + p);
        const uint32_t g = gword & kNodeMask;
        const Real* src = A.ut + (size_t)g * F;
#pragma unroll
        for (int f = 0; f < F; ++f) mu_s[f * NNP + p] = src[f];
        const Real* gp = A.geom + (size_t)e * 12 * NN + p;
#pragma unroll
        for (int f = 0; f < 9; ++f) dd[f] = __ldg(gp + f * NN);
        jw = __ldg(gp + 9 * NN);
        lam = __ldg(gp + 10 * NN);
        mu = __ldg(gp + 11 * NN);
    }
    __syncthreads();
    const int i = p / (NG * NG), j = (p / NG) % NG, k = p % NG;
    if (active) {
#pragma unroll
        for (int d = 0; d < NFLD; ++d) {
            if (mu <= Real(0)) {  // element_cpu.cpp:42-43: the point adds nothing
#pragma unroll
                for (int q = 0; q < 9; ++q) mG[((q / 3) * F + d * 3 + (q % 3)) * NNP + p] = Real(0);
                continue;
            }
            Real gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0}, gz[3] = {0, 0, 0};
#pragma unroll
            for (int s = 0; s < NG; ++s) {
                const Real Di = sD[i * NG + s], Dj = sD[j * NG + s], Dk = sD[k * NG + s];
                const int pa = (s * NG + j) * NG + k, pb = (i * NG + s) * NG + k,
                          pc = (i * NG + j) * NG + s;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const Real* uc = mu_s + (d * 3 + c) * NNP;
                    gx[c] += Di * uc[pa];
                    gy[c] += Dj * uc[pb];
                    gz[c] += Dk * uc[pc];
                }
            }
            // physical gradient with the reference's reading of dxi_dx
            Real gr[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                gr[c][0] = gx[c] * dd[0] + gy[c] * dd[1] + gz[c] * dd[2];
                gr[c][1] = gx[c] * dd[3] + gy[c] * dd[4] + gz[c] * dd[5];
                gr[c][2] = gx[c] * dd[6] + gy[c] * dd[7] + gz[c] * dd[8];
            }
            const Real exx = gr[0][0], eyy = gr[1][1], ezz = gr[2][2];
            const Real exy = Real(0.5) * (gr[0][1] + gr[1][0]);
            const Real exz = Real(0.5) * (gr[0][2] + gr[2][0]);
            const Real eyz = Real(0.5) * (gr[1][2] + gr[2][1]);
            const Real tr = exx + eyy + ezz;
            const Real m2 = Real(2) * mu;
            Real sg[3][3];
            sg[0][0] = m2 * exx + lam * tr;
            sg[1][1] = m2 * eyy + lam * tr;
            sg[2][2] = m2 * ezz + lam * tr;
            sg[0][1] = sg[1][0] = m2 * exy;
            sg[0][2] = sg[2][0] = m2 * exz;
            sg[1][2] = sg[2][1] = m2 * eyz;
            // flux along reference axis a: jw * sigma . (dd[a], dd[3+a], dd[6+a])
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    mG[(a * F + d * 3 + c) * NNP + p] =
                        jw * (sg[c][0] * dd[a] + sg[c][1] * dd[3 + a] + sg[c][2] * dd[6 + a]);
            }
        }
    }
    __syncthreads();
    if (!active) return;

    Real r[F];
#pragma unroll
    for (int f = 0; f < F; ++f) {
        Real acc = Real(0);
#pragma unroll
        for (int s = 0; s < NG; ++s) {
            acc += sD[s * NG + i] * mG[(0 * F + f) * NNP + (s * NG + j) * NG + k];
            acc += sD[s * NG + j] * mG[(1 * F + f) * NNP + (i * NG + s) * NG + k];
            acc += sD[s * NG + k] * mG[(2 * F + f) * NNP + (i * NG + j) * NG + s];
        }
        r[f] = -acc;
    }
    const uint32_t g = gword & kNodeMask;

    // C-PML acceleration term with last step's memory, then the memory
    // update that the reference performs after the corrector (it only uses
    // values fixed at the start of the step).
    const int slot = A.pml_slot ? __ldg(A.pml_slot + e) : -1;
    if (slot >= 0) {
        const Real* cf = A.pml_coef + (size_t)slot * 15 * NN + p;
        Real al[9], ab[5];
#pragma unroll
        for (int q = 0; q < 9; ++q) al[q] = __ldg(cf + q * NN);
#pragma unroll
        for (int q = 0; q < 5; ++q) ab[q] = __ldg(cf + (9 + q) * NN);
        const Real scale = __ldg(cf + 14 * NN);
        Real* mem = A.pml_mem + (size_t)slot * (F * 3) * NN + p;
        Real* prev = A.pml_prev + (size_t)slot * F * NN + p;
#pragma unroll
        for (int f = 0; f < F; ++f) {
            const double un = A.u[(size_t)g * F + f];
            const double vn = A.v[(size_t)g * F + f];
            const Real an = A.a[(size_t)g * F + f];
            const Real nv = Real(un + A.c1 * vn);
            const Real ov = prev[f * NN] + Real(A.c2) * an;
            Real m0 = mem[(f * 3 + 0) * NN], m1 = mem[(f * 3 + 1) * NN], m2 = mem[(f * 3 + 2) * NN];
            r[f] += scale * (ab[0] * Real(vn) + ab[1] * Real(un) + ab[2] * m0 + ab[3] * m1 + ab[4] * m2);
            m0 = al[0] * m0 + al[1] * nv + al[2] * ov;
            m1 = al[3] * m1 + al[4] * nv + al[5] * ov;
            m2 = al[6] * m2 + al[7] * nv + al[8] * ov;
            mem[(f * 3 + 0) * NN] = m0;
            mem[(f * 3 + 1) * NN] = m1;
            mem[(f * 3 + 2) * NN] = m2;
            prev[f * NN] = nv;
        }
    }
    // point-force source (one model): wavefield d takes the slots of its
    // source set, scaled by that set's source time function
    if (A.mstf) {
        int s = A.src_head ? __ldg(A.src_head + e) : -1;
        while (s >= 0) {
            const Real w = __ldg(A.src_w + (size_t)s * NN + p);
            const int ks = A.src_set ? __ldg(A.src_set + s) : 0;
            if (w != Real(0)) {
#pragma unroll
                for (int d = 0; d < NFLD; ++d) {
                    const Real stf = A.mstf[A.fset[d]];
                    if (stf == Real(0) || A.fset[d] != ks) continue;
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        if (c == A.dir[d]) r[d * 3 + c] += stf * w;
                }
            }
            s = __ldg(A.src_next + s);
        }
    }
    // colour-ordered assembly: exclusive access to node g in this launch
    Real* out = A.force + (size_t)g * F;
    if (gword & kFirstTouch) {
#pragma unroll
        for (int f = 0; f < F; ++f) out[f] = r[f];
    } else {
#pragma unroll
        for (int f = 0; f < F; ++f) out[f] += r[f];
    }
}

template <typename Real, int NG, int NFLD>
__global__ void __launch_bounds__(Shape<NG>::THREADS) elem_step_kernel(ElemArgs<Real> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    elem_body<Real, NG, NFLD>(A, reinterpret_cast<Real*>(smem_raw));
}

template <typename Real, int NG, int NFLD>
constexpr size_t elem_smem_bytes() {
    using S = Shape<NG>;
    return sizeof(Real) * (64 + (size_t)S::EPB * 3 * NFLD * S::NNP * 4);
}

// 16-byte vector helpers (a float4, or two double2 for FP64 vectors).
__device__ __forceinline__ void load4(const float* p, float (&v)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void load4_nc(const float* p, float (&v)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4_nc(const double* p, double (&v)[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void store4(float* p, float a, float b, float c, float d) {
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ void store4(double* p, double a, double b, double c, double d) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
    reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
}

// FP64 operations rounded one by one (no contraction into FMA), so that the
// node update rounds the same way in every instantiation of the kernels
// that inline it (a solver of one model and of several must agree bit for
// bit) and in the reference's evaluation order.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

// Finalise wavefield d of node g from its complete assembled force fv:
// node C-PML term (when PML), Newmark corrector with the diagonal mass
// (solver.cpp:52-69, legacy damping of 564-574 applied to v first) and the
// next step's predictor (40-49), written as one 16-byte vector.  Every load
// is issued before the first store, so a thread's memory round trips
// overlap.  On the FP32 path 1/m == 0 marks a node with m <= 0 (the host
// stores 0 there), so the f64 mass is not read.
template <typename Real, int NFLD, bool PML>
__device__ __forceinline__ void update_node_field(const NodeArgs<Real>& A, const NodePml<Real>& P, long long g,
                                                  int d, const Real (&fv)[3], int sl, const ModelConst& K,
                                                  bool full = true) {
    constexpr int F = 3 * NFLD;
    const long long i0 = g * F + d * 3;
    double* __restrict__ pu = A.u + i0;
    double* __restrict__ pv = A.v + i0;
    Real* __restrict__ pa = A.a + i0;
    if (!PML && A.half_v) {
        // Newmark with beta = 0, gamma = 1/2 (solver.cpp:40-69) written on
        // the half-step velocity w = v + dt/2 a: u_{n+1} = u_n + dt w_n,
        // a_{n+1} = f/m, w_{n+1} = w_n + dt a_{n+1}, and the next predicted
        // displacement u_{n+1} + dt w_{n+1} (its increment dt w_{n+1}).  The
        // same values as the (u, v, a) form in exact arithmetic, without the
        // acceleration's read and write; v and a are recovered from w and
        // the assembled force when they are needed (records, state).  w is
        // held in float (its rounding adds a random walk of ~1e-7 relative
        // per step, far below the float rounding of the predicted
        // displacement that bounds this path), u in double.
        float* __restrict__ pw = A.w32 + i0;
        double uu[3], ww[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            uu[c] = pu[c];
            ww[c] = (double)pw[c];
        }
        const Real im = __ldg(A.inv_mass + g);
        Real out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (im != Real(0)) {  // m <= 0: the node stays as it is (a = 0, solver.cpp:58-61)
                const double a_new = (double)(Real)(fv[c] * im);
                uu[c] = dadd(uu[c], dmul(K.dt, ww[c]));
                ww[c] = (double)(float)dadd(ww[c], dmul(K.dt, a_new));
                pu[c] = uu[c];
                pw[c] = (float)ww[c];
            }
            out[c] = full ? (Real)dadd(uu[c], dmul(K.dt, ww[c])) : (Real)dmul(K.dt, ww[c]);
        }
        store4(A.ut + ((size_t)g * NFLD + d) * 4, out[0], out[1], out[2], Real(0));
        return;
    }
    double vv[3], uu[3];
    Real ao[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vv[c] = pv[c];
        uu[c] = pu[c];
        ao[c] = pa[c];
    }
    const Real im = A.inv_mass ? __ldg(A.inv_mass + g) : Real(0);
    const bool massless = A.inv_mass ? (im == Real(0)) : (__ldg(A.mass + g) <= 0.0);
    const double m = A.inv_mass ? 1.0 : __ldg(A.mass + g);
    const double dmp = A.damping ? __ldg(A.damping + g) : 0.0;
    Real cf[14], mm[3][3], pr[3];
    if (PML) {
        if (sl >= 0) {
#pragma unroll
            for (int q = 0; q < 14; ++q) cf[q] = __ldg(P.coef + (size_t)sl * 14 + q);
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    mm[q][c] = cf[2 + q] != Real(0) ? P.mem[((size_t)q * P.n_slot + sl) * F + d * 3 + c] : Real(0);
#pragma unroll
            for (int c = 0; c < 3; ++c) pr[c] = P.prev[(size_t)sl * F + d * 3 + c];
        }
    }
    Real out[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (dmp > 0.0) vv[c] = __dsub_rn(vv[c], dmul(dmp, vv[c]));
        Real force = fv[c];
        if (PML && sl >= 0) {
            const Real nv = (Real)dadd(uu[c], dmul(K.c1, vv[c]));
            const Real ov = pr[c] + (Real)K.c2 * ao[c];
            force += cf[0] * (Real)vv[c] + cf[1] * (Real)uu[c] + cf[2] * mm[0][c] + cf[3] * mm[1][c] + cf[4] * mm[2][c];
#pragma unroll
            for (int q = 0; q < 3; ++q)
                if (cf[2 + q] != Real(0))
                    P.mem[((size_t)q * P.n_slot + sl) * F + d * 3 + c] =
                        cf[5 + 3 * q] * mm[q][c] + cf[6 + 3 * q] * nv + cf[7 + 3 * q] * ov;
            P.prev[(size_t)sl * F + d * 3 + c] = nv;
        }
        double a_new;
        if (massless) {
            a_new = 0.0;
        } else {
            a_new = A.inv_mass ? (double)(force * im) : __ddiv_rn((double)force, m);
            a_new = (double)(Real)a_new;
            const double a_old = (double)ao[c];
            // solver.cpp:62-66
            const double ta = dadd(dmul(0.5 - A.beta, a_old), dmul(A.beta, a_new));
            uu[c] = dadd(uu[c], dadd(dmul(K.dt, vv[c]), dmul(dmul(K.dt, K.dt), ta)));
            vv[c] = dadd(vv[c], dmul(K.dt, dadd(dmul(1.0 - A.gamma, a_old), dmul(A.gamma, a_new))));
        }
        pu[c] = uu[c];
        pv[c] = vv[c];
        pa[c] = (Real)a_new;
        // the next step's predicted displacement (solver.cpp:40-49), or its
        // increment over this step's (u_{n+1} is this step's prediction)
        const double inc = dadd(dmul(K.dt, vv[c]), dmul(K.half_dt2, a_new));
        out[c] = full ? (Real)dadd(uu[c], inc) : (Real)inc;
    }
    store4(A.ut + ((size_t)g * NFLD + d) * 4, out[0], out[1], out[2], Real(0));
}

// Separate node pass (used when the element kernel does not finalise nodes):
// one thread per (node, wavefield), the wavefields of a node in adjacent
// threads, so a warp streams contiguous u, v, a and force/prediction
// vectors and reads each node's mass once.  With node-form C-PML the pass
// is two launches over contiguous node ranges: node_update_kernel over the
// plain nodes [g0, n_node) without the C-PML registers, node_pml_kernel
// over the C-PML nodes [0, g0).
// Constants of the model node g belongs to; false when that model has
// taken all its steps (its state stays as it is).
template <typename Real, bool MULTI>
__device__ __forceinline__ bool node_constants(const NodeArgs<Real>& A, const NodePml<Real>& P, long long g,
                                               ModelConst& K, bool& full) {
    if (!MULTI) {
        K = ModelConst{A.dt, A.half_dt2, P.c1, P.c2};
        full = A.mnext ? A.mnext[0] != 0 : true;
        return true;
    }
    const int m = __ldg(A.node_model + g);
    if (!__ldg(A.mlive + m)) return false;
    K = A.mc[m];
    full = A.mnext ? A.mnext[m] != 0 : true;
    return true;
}

template <typename Real, int NFLD, bool MULTI>
__global__ void __launch_bounds__(256, 3) node_update_kernel(NodeArgs<Real> A, NodePml<Real> P, long long g0) {
    const long long g1 = (MULTI && A.live_node_end) ? min(A.n_node, A.live_node_end[1]) : A.n_node;
    const long long total = max(0LL, g1 - g0) * NFLD;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const long long gl = t / NFLD;
        const int d = (int)(t - gl * NFLD);
        const long long g = g0 + gl;
        ModelConst K;
        bool full;
        if (!node_constants<Real, MULTI>(A, P, g, K, full)) continue;
        Real fv4[4];
        load4_nc(A.force + ((size_t)g * NFLD + d) * 4, fv4);
        const Real fv[3] = {fv4[0], fv4[1], fv4[2]};
        update_node_field<Real, NFLD, false>(A, P, g, d, fv, -1, K, full);
    }
}

template <typename Real, int NFLD, bool MULTI>
__global__ void __launch_bounds__(256, 2) node_pml_kernel(NodeArgs<Real> A, NodePml<Real> P) {
    const long long n1 = (MULTI && A.live_node_end) ? min(P.n_slot, A.live_node_end[0]) : P.n_slot;
    const long long total = n1 * NFLD;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const long long g = t / NFLD;
        const int d = (int)(t - g * NFLD);
        ModelConst K;
        bool full;
        if (!node_constants<Real, MULTI>(A, P, g, K, full)) continue;
        Real fv4[4];
        load4_nc(A.force + ((size_t)g * NFLD + d) * 4, fv4);
        const Real fv[3] = {fv4[0], fv4[1], fv4[2]};
        update_node_field<Real, NFLD, true>(A, P, g, d, fv, (int)g, K, full);
    }
}

// Start of a step for every model: whether it still steps, and its source
// time function value (solver.cpp:577-605 uses stf_values[step]; steps past
// the end of the series inject nothing).  mstep[m] is the step about to be
// computed and moves on by one while the model steps, so a captured step
// replays correctly.
// Series q = m * n_set + k is source set k of model m.
//
// Element force in full or by increments: a step whose element phase
// evaluates the force of the full predicted displacement (mdirect = 1: the
// first colour touching a node stores) is followed by up to period-1 steps
// that add the force of the predicted displacement's increment to the
// stored force (mdirect = 0); the source then adds the increment of the
// source time function.  A one-shot force_direct[m] (set by the host after
// the predicted displacement was rewritten from u, v, a) makes the step a
// full one.  mnext[m] tells the node pass what the next step needs.
template <typename Real>
__global__ void step_begin_kernel(int n_model, int n_set, int* mstep, const int* nsteps, const int* n_stf,
                                  const long long* stf_off, const Real* stf_all, Real* mstf, int* mlive, int period,
                                  int* force_direct, int* mdirect, int* mnext) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_model) return;
    const int t = mstep[m];
    const bool live = t < nsteps[m];
    mlive[m] = live ? 1 : 0;
    bool full = true;
    if (mdirect) {
        full = period <= 1 || force_direct[m] != 0 || t % period == 0;
        force_direct[m] = 0;
        mdirect[m] = full ? 1 : 0;
        mnext[m] = (period <= 1 || (t + 1) % period == 0) ? 1 : 0;
    }
    for (int k = 0; k < n_set; ++k) {
        const int q = m * n_set + k;
        const Real now = (live && t < n_stf[q]) ? stf_all[stf_off[q] + t] : Real(0);
        const Real before = (!full && t >= 1 && t - 1 < n_stf[q]) ? stf_all[stf_off[q] + t - 1] : Real(0);
        mstf[q] = full ? now : (live ? now - before : Real(0));
    }
    mstep[m] = t + (live ? 1 : 0);
}

// Several models in one solver: after step_begin_kernel, the end of the
// cells still stepping in each colour and of the nodes still stepping in the
// C-PML and plain node ranges.  Cells of a colour and nodes of a range are
// grouped by model, so everything past the largest end of a live model
// belongs to finished models and the launches of this step stop there
// (cells and nodes before it of finished models are still skipped one by
// one).  cell_end [model][colour], node_end [model][2] (C-PML, plain); one
// block, a thread per colour or range.
static __global__ void live_bounds_kernel(int n_model, int n_colour, const int* mlive, const int* cell_end,
                                   const int* colour_first, const long long* node_end, long long plain_first,
                                   int* live_cell_end, long long* live_node_end) {
    for (int c = threadIdx.x; c < n_colour + 2; c += blockDim.x) {
        if (c < n_colour) {
            int e = colour_first[c];
            for (int m = 0; m < n_model; ++m)
                if (mlive[m]) e = max(e, cell_end[m * n_colour + c]);
            live_cell_end[c] = e;
        } else {
            const int r = c - n_colour;
            long long g = r == 0 ? 0 : plain_first;
            for (int m = 0; m < n_model; ++m)
                if (mlive[m]) g = max(g, node_end[m * 2 + r]);
            live_node_end[r] = g;
        }
    }
}

// ---------------------------------------------------------------------------
// elem_pipe_kernel: persistent, software-pipelined element/assembly kernel.
//
// Blocks loop over groups of EPB cells of one colour.  While group i is
// computed, the gathered displacement of group i+1 and the geometry + node
// table of group i+2 are in flight as cp.async copies into rotating shared
// stages (3 stages for geometry/ibool, 2 for the gathered vectors), so each
// SM keeps tens of KB of loads outstanding independent of how many blocks
// fit.  Thread per GLL point; the n_field wavefields are looped per thread.
// Node table rows on the device hold the cell's model index after its node
// words and are padded so every copy is a 16-byte cp.async.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Bulk copies (TMA, no tensor map, no multicast) completing on an mbarrier
// of this block: one thread announces the bytes of a stage and issues its
// copies; every thread waits for the phase with a bounded poll.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// The phase of parity `parity` completed; false after kMbarPolls polls
// (each try_wait may suspend the thread for a while), which only a lost
// copy would cause.
constexpr long kMbarPolls = 1L << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (long k = 0; k < kMbarPolls; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// bytes: a multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_copy_g2s(void* smem, const void* gmem, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(smem)), "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

template <typename Real, int NG, int NFLD>
struct PipeShape {
    static constexpr int NN = NG * NG * NG;
    static constexpr int NNP = (NN + 31) / 32 * 32;
    static constexpr int EPB = NNP <= 32 ? 8 : (NNP <= 64 ? 4 : (NNP <= 128 ? 2 : 1));
    static constexpr int THREADS = NNP * EPB;
    static constexpr int GEO_B = 12 * NN * (int)sizeof(Real);         // geometry bytes per cell
    static constexpr int IB_B = ib_row_words(NN) * 4;                  // node-table bytes per cell
    static constexpr int BUF_B = NN * NFLD * 4 * (int)sizeof(Real);    // field vectors per cell
    // a geometry stage also receives the cell's old force vectors once the
    // geometry has been read into registers
    static constexpr int GEO_SLOT = GEO_B > BUF_B ? GEO_B : BUF_B;
    static constexpr int GSTAGE = EPB * GEO_SLOT;
    static constexpr int ISTAGE = EPB * IB_B;
    static constexpr int BSTAGE = EPB * BUF_B;
    static constexpr int D_B = 64 * (int)sizeof(Real);
    static constexpr int SMEM = D_B + 2 * GSTAGE + 3 * ISTAGE + 2 * BSTAGE;
    static constexpr int MIN_BLOCKS = (64 * 1024) / (THREADS * 64) > 0 ? (64 * 1024) / (THREADS * 64) : 1;
    static_assert(GEO_B % 16 == 0 && IB_B % 16 == 0 && BUF_B % 16 == 0, "16-byte copies");
};

template <typename Real, int NG, int NFLD>
__global__ void __launch_bounds__(PipeShape<Real, NG, NFLD>::THREADS, (sizeof(Real) == 4 ? PipeShape<Real, NG, NFLD>::MIN_BLOCKS : 1))
    elem_pipe_kernel(ElemArgs<Real> A, const uint32_t* __restrict__ ibool_padded, int n_groups) {
    using S = PipeShape<Real, NG, NFLD>;
    constexpr int NN = S::NN, NNP = S::NNP, EPB = S::EPB, THREADS = S::THREADS;
    constexpr int VW = 16 / (int)sizeof(Real);               // Reals per 16-byte copy
    constexpr int CPV = 4 * (int)sizeof(Real) / 16;          // 16-byte copies per field vector
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* sD = reinterpret_cast<Real*>(smem_raw);
    unsigned char* gbase = smem_raw + S::D_B;
    unsigned char* ibase = gbase + 2 * S::GSTAGE;
    unsigned char* bbase = ibase + 3 * S::ISTAGE;
    const int tid = threadIdx.x;
    const int el = tid / NNP, p = tid - el * NNP;
    if (tid < NG * NG) sD[tid] = A.dmat[tid];

    auto geo_of = [&](int st, int c) -> Real* {
        return reinterpret_cast<Real*>(gbase + st * S::GSTAGE + c * S::GEO_SLOT);
    };
    auto ib_of = [&](int st, int c) -> uint32_t* {
        return reinterpret_cast<uint32_t*>(ibase + st * S::ISTAGE + c * S::IB_B);
    };
    auto buf_of = [&](int st, int c) -> Real* {
        return reinterpret_cast<Real*>(bbase + st * S::BSTAGE + c * S::BUF_B);
    };
    auto issue_ib = [&](int grp, int st) {
        constexpr int CI = S::IB_B / 16;
        for (int q = tid; q < EPB * CI; q += THREADS) {
            const int c = q / CI, r = q - c * CI;
            const int e = A.e_begin + grp * EPB + c;
            if (e < A.e_end)
                cp_async16(reinterpret_cast<unsigned char*>(ib_of(st, c)) + r * 16,
                           reinterpret_cast<const unsigned char*>(ibool_padded) + (size_t)e * S::IB_B + r * 16);
        }
    };
    auto issue_geo = [&](int grp, int st) {
        constexpr int CG = S::GEO_B / 16;
        for (int q = tid; q < EPB * CG; q += THREADS) {
            const int c = q / CG, r = q - c * CG;
            const int e = A.e_begin + grp * EPB + c;
            if (e < A.e_end)
                cp_async16(reinterpret_cast<unsigned char*>(geo_of(st, c)) + r * 16,
                           reinterpret_cast<const unsigned char*>(A.geom) + (size_t)e * S::GEO_B + r * 16);
        }
    };
    // this point's predicted-displacement vectors (node table in stage ist)
    auto issue_gather = [&](int grp, int ist, int bs) {
        const int e = A.e_begin + grp * EPB + el;
        if (e >= A.e_end || p >= NN) return;
        const uint32_t g = ib_of(ist, el)[p] & kNodeMask;
#pragma unroll
        for (int d = 0; d < NFLD; ++d)
#pragma unroll
            for (int h = 0; h < CPV; ++h)
                cp_async16(buf_of(bs, el) + (p * NFLD + d) * 4 + h * VW, A.ut + ((size_t)g * NFLD + d) * 4 + h * VW);
    };

    // prologue: node table of the first group, then its vectors and
    // geometry and the node table of the second group
    const int grp0 = blockIdx.x;
    if (grp0 < n_groups) issue_ib(grp0, 0);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    if (grp0 < n_groups) {
        issue_gather(grp0, 0, 0);
        issue_geo(grp0, 0);
    }
    if (grp0 + (int)gridDim.x < n_groups) issue_ib(grp0 + gridDim.x, 1);
    cp_async_commit();

    const int i = p / (NG * NG), j = (p / NG) % NG, k = p % NG;
    int it = 0;
    for (int grp = grp0; grp < n_groups; grp += gridDim.x, ++it) {
        const int cur = it & 1, ist = it % 3;
        cp_async_wait_all();
        __syncthreads();  // vectors + geometry of this group, node table of the next
        const int e = A.e_begin + grp * EPB + el;
        const int mdl = (e < A.e_end) ? (int)ib_of(ist, el)[NN] : 0;
        const bool active = (e < A.e_end) && (p < NN) && (!A.mlive || __ldg(A.mlive + mdl));
        const uint32_t first_bit = (!A.mdirect || __ldg(A.mdirect + mdl)) ? kFirstTouch : 0u;
        Real* geo = geo_of(cur, el);
        Real* buf = buf_of(cur, el);
        uint32_t gword = 0;
        Real dd[9], jw = Real(0), lam = Real(0), mu = Real(0);
        if (active) {
            gword = ib_of(ist, el)[p];
#pragma unroll
            for (int q = 0; q < 9; ++q) dd[q] = geo[q * NN + p];
            jw = geo[9 * NN + p];
            lam = geo[10 * NN + p];
            mu = geo[11 * NN + p];
        }
        __syncthreads();  // geometry stage now takes this group's old force vectors
        if (active && !(gword & first_bit)) {
            const uint32_t g = gword & kNodeMask;
#pragma unroll
            for (int d = 0; d < NFLD; ++d)
#pragma unroll
                for (int h = 0; h < CPV; ++h)
                    cp_async16(geo + (p * NFLD + d) * 4 + h * VW, A.force + ((size_t)g * NFLD + d) * 4 + h * VW);
        }
        cp_async_commit();  // group: old force of this group
        const int nxt = grp + gridDim.x;
        if (nxt < n_groups) {
            issue_gather(nxt, (it + 1) % 3, cur ^ 1);
            issue_geo(nxt, cur ^ 1);
        }
        if (nxt + (int)gridDim.x < n_groups) issue_ib(nxt + gridDim.x, (it + 2) % 3);
        cp_async_commit();  // group: next group's vectors and geometry, node table after that

        Real st[NFLD][6];
#pragma unroll
        for (int d = 0; d < NFLD; ++d)
#pragma unroll
            for (int q = 0; q < 6; ++q) st[d][q] = Real(0);
        if (active && mu > Real(0)) {  // element_cpu.cpp:42-43: mu <= 0 adds nothing
#pragma unroll
            for (int d = 0; d < NFLD; ++d) {
                Real gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0}, gz[3] = {0, 0, 0};
#pragma unroll
                for (int s = 0; s < NG; ++s) {
                    Real va[4], vb[4], vc[4];
                    load4(buf + ((((s * NG + j) * NG + k) * NFLD) + d) * 4, va);
                    load4(buf + ((((i * NG + s) * NG + k) * NFLD) + d) * 4, vb);
                    load4(buf + ((((i * NG + j) * NG + s) * NFLD) + d) * 4, vc);
                    const Real Di = sD[i * NG + s], Dj = sD[j * NG + s], Dk = sD[k * NG + s];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        gx[c] += Di * va[c];
                        gy[c] += Dj * vb[c];
                        gz[c] += Dk * vc[c];
                    }
                }
                Real gr[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    gr[c][0] = gx[c] * dd[0] + gy[c] * dd[1] + gz[c] * dd[2];
                    gr[c][1] = gx[c] * dd[3] + gy[c] * dd[4] + gz[c] * dd[5];
                    gr[c][2] = gx[c] * dd[6] + gy[c] * dd[7] + gz[c] * dd[8];
                }
                const Real tr = gr[0][0] + gr[1][1] + gr[2][2];
                const Real m2 = Real(2) * mu;
                st[d][0] = m2 * gr[0][0] + lam * tr;
                st[d][1] = m2 * gr[1][1] + lam * tr;
                st[d][2] = m2 * gr[2][2] + lam * tr;
                st[d][3] = m2 * (Real(0.5) * (gr[0][1] + gr[1][0]));
                st[d][4] = m2 * (Real(0.5) * (gr[0][2] + gr[2][0]));
                st[d][5] = m2 * (Real(0.5) * (gr[1][2] + gr[2][1]));
            }
        }
        __syncthreads();  // the vector buffer is reused for the fluxes
        Real r[NFLD][3];
#pragma unroll
        for (int d = 0; d < NFLD; ++d) r[d][0] = r[d][1] = r[d][2] = Real(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (active) {
                const Real ea = dd[a], eb = dd[3 + a], ec = dd[6 + a];
#pragma unroll
                for (int d = 0; d < NFLD; ++d)
                    store4(buf + (p * NFLD + d) * 4, jw * (st[d][0] * ea + st[d][3] * eb + st[d][4] * ec),
                           jw * (st[d][3] * ea + st[d][1] * eb + st[d][5] * ec),
                           jw * (st[d][4] * ea + st[d][5] * eb + st[d][2] * ec), Real(0));
            }
            __syncthreads();
            if (active) {
                const int ia = (a == 0) ? i : ((a == 1) ? j : k);
#pragma unroll
                for (int s = 0; s < NG; ++s) {
                    const int q = (a == 0) ? ((s * NG + j) * NG + k)
                                           : ((a == 1) ? ((i * NG + s) * NG + k) : ((i * NG + j) * NG + s));
                    const Real w = sD[s * NG + ia];
#pragma unroll
                    for (int d = 0; d < NFLD; ++d) {
                        Real v[4];
                        load4(buf + (q * NFLD + d) * 4, v);
                        r[d][0] -= w * v[0];
                        r[d][1] -= w * v[1];
                        r[d][2] -= w * v[2];
                    }
                }
            }
            if (a < 2) __syncthreads();
        }
        if (active) {
            const uint32_t g = gword & kNodeMask;
            // C-PML per cell (pml.cpp:55-216)
            const int slot = A.pml_slot ? __ldg(A.pml_slot + e) : -1;
            if (slot >= 0) {
                const double c1 = A.mc ? A.mc[mdl].c1 : A.c1, c2 = A.mc ? A.mc[mdl].c2 : A.c2;
                const Real* cf = A.pml_coef + (size_t)slot * 15 * NN + p;
                Real al[9], ab[5];
#pragma unroll
                for (int q = 0; q < 9; ++q) al[q] = __ldg(cf + q * NN);
#pragma unroll
                for (int q = 0; q < 5; ++q) ab[q] = __ldg(cf + (9 + q) * NN);
                const Real scale = __ldg(cf + 14 * NN);
                Real* mem = A.pml_mem + (size_t)slot * (3 * NFLD * 3) * NN + p;
                Real* prev = A.pml_prev + (size_t)slot * (3 * NFLD) * NN + p;
#pragma unroll
                for (int d = 0; d < NFLD; ++d) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int f = d * 3 + c;
                        const double un = A.u[(size_t)g * 3 * NFLD + f];
                        const double vn = A.v[(size_t)g * 3 * NFLD + f];
                        const Real an = A.a[(size_t)g * 3 * NFLD + f];
                        const Real nv = Real(un + c1 * vn);
                        const Real ov = prev[f * NN] + Real(c2) * an;
                        Real m0 = mem[(f * 3 + 0) * NN], m1 = mem[(f * 3 + 1) * NN], m2 = mem[(f * 3 + 2) * NN];
                        r[d][c] += scale * (ab[0] * Real(vn) + ab[1] * Real(un) + ab[2] * m0 + ab[3] * m1 + ab[4] * m2);
                        mem[(f * 3 + 0) * NN] = al[0] * m0 + al[1] * nv + al[2] * ov;
                        mem[(f * 3 + 1) * NN] = al[3] * m1 + al[4] * nv + al[5] * ov;
                        mem[(f * 3 + 2) * NN] = al[6] * m2 + al[7] * nv + al[8] * ov;
                        prev[f * NN] = nv;
                    }
                }
            }
            // point force (solver.cpp:577-605): wavefield d takes the slots
            // of its source set, scaled by that set's source time function
            if (A.mstf) {
                int s = A.src_head ? __ldg(A.src_head + e) : -1;
                while (s >= 0) {
                    const Real w = __ldg(A.src_w + (size_t)s * NN + p);
                    const int ks = A.src_set ? __ldg(A.src_set + s) : 0;
                    if (w != Real(0)) {
#pragma unroll
                        for (int d = 0; d < NFLD; ++d) {
                            const Real stf = __ldg(A.mstf + mdl * A.n_set + A.fset[d]);
                            if (stf == Real(0) || A.fset[d] != ks) continue;
#pragma unroll
                            for (int c = 0; c < 3; ++c)
                                if (c == A.dir[d]) r[d][c] += stf * w;
                        }
                    }
                    s = __ldg(A.src_next + s);
                }
            }
        }
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this group's old force
        __syncthreads();
        if (active) {
            const uint32_t g = gword & kNodeMask;
            const bool first = gword & first_bit;
            // the highest colour touching a node completes its force here and
            // finalises it: no cell reads the node later in this step
            const bool fin = A.fuse && (gword & kLastTouch);
#pragma unroll
            for (int d = 0; d < NFLD; ++d) {
                Real fo[4] = {Real(0), Real(0), Real(0), Real(0)};
                if (!first) load4(geo + (p * NFLD + d) * 4, fo);
                if (fin) {
                    const Real fv[3] = {fo[0] + r[d][0], fo[1] + r[d][1], fo[2] + r[d][2]};
                    const ModelConst K = A.mc ? A.mc[mdl] : ModelConst{A.nu.dt, A.nu.half_dt2, A.np.c1, A.np.c2};
                    if (A.np.coef)
                        update_node_field<Real, NFLD, true>(A.nu, A.np, g, d, fv, g < A.np.n_slot ? (int)g : -1, K);
                    else
                        update_node_field<Real, NFLD, false>(A.nu, A.np, g, d, fv, -1, K);
                } else {
                    store4(A.force + ((size_t)g * NFLD + d) * 4, fo[0] + r[d][0], fo[1] + r[d][1], fo[2] + r[d][2],
                           Real(0));
                }
            }
        }
    }
    cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// elem_col_kernel: element/assembly kernel with one thread per
// (cell, wavefield, xi-line).
//
// The thread-per-point kernel above reads 15 neighbour vectors per point for
// the gradient and 15 flux vectors for the divergence, all from shared
// memory, and shared-memory bandwidth is what bounds it.  Here a thread owns
// the NG points (i = 0..NG-1, j, k) of one xi-line of one wavefield: the xi
// contractions of the gradient and of the divergence run on values held in
// registers, and only the eta and zeta neighbours go through shared memory,
// as one float per component (structure-of-arrays, no padding lane).  The
// per-(cell, wavefield) arrays are SP floats apart with SP = NG*NG (mod 32),
// so that the eta/zeta reads of a warp that spans two or three of them fall
// in distinct banks.  The D entries indexed by the loop counter come from
// the kernel parameters (constant bank); those indexed by the thread's own j
// and k are kept in registers.
//
// XCH (line owners): instead of every thread reading the five eta and five
// zeta neighbours of each of its points (30 shared loads per point for the
// gradient, 30 for the divergence), the thread with column (j, k) also owns
// the eta line (i = j, k) and the zeta line (i = k, j) of its (cell,
// wavefield): it reads the line, contracts it with D in registers and
// writes the derivative back in place, so a point costs one shared load per
// direction and component afterwards.  Phases per group: own points'
// displacement into both arrays | line contractions | gradient, stress and
// fluxes (the eta and zeta fluxes replace the derivatives in place) | line
// contractions of the fluxes | divergence and assembly; four barriers instead
// of two, and 40 % fewer shared-memory wavefronts.  The arrays' point layout
// (PIE, PIZ) and slot stride SP put a warp's own-point accesses and its
// line accesses in distinct banks.  The eta and zeta sums of the divergence
// are added in another order than in the default layout, so the two agree
// to rounding, not bit for bit.
//
// Pipelining: the geometry of the next group and the node table of the one
// after are bulk copies (TMA engine, one per cell, issued by one thread and
// completing on a per-stage mbarrier) into rotating shared stages; the
// writes bypass the LSU pipe that the shared-memory exchange keeps busy,
// which 16-byte cp.async by every thread did not; the next group's
// predicted-displacement vectors are register loads issued one group ahead,
// this group's old force vectors are prefetched into L2 at the start of the
// group and loaded into registers once its gradient phase is done.
// ---------------------------------------------------------------------------

// Cells per group of the line kernel: about 150 threads by default; the
// autotuner also tries the neighbouring counts at ngll 5.
__host__ __device__ constexpr int col_default_epb(int ng, int nfld) {
    return (150 / (nfld * ng * ng)) > 0 ? 150 / (nfld * ng * ng) : 1;
}

// XCH: the eta and zeta contractions done by line owners (see
// elem_col_kernel) in two [3][GR][SP] arrays laid out point (i, j, k) ->
// PI*i + NG*j + k with PI = PIE (eta array) or PIZ (zeta array).
template <int NG, int NFLD, int EPB_ = col_default_epb(NG, NFLD), bool XCH = false>
struct ColShape {
    static constexpr int NN = NG * NG * NG;
    static constexpr int NG2 = NG * NG;
    static constexpr int EPB = EPB_;                      // cells per group
    static constexpr int GR = EPB * NFLD;                 // (cell, wavefield) lines per group
    static constexpr int ACTIVE = GR * NG2;               // threads with work
    static constexpr int THREADS = (ACTIVE + 31) / 32 * 32;
    // at NG = 5 (PIE, PIZ, SP) = (37, 33, 185): the own-point accesses and
    // the eta- (zeta-) line accesses of a warp fall in distinct banks
    static constexpr int PIE = NG2 + 12, PIZ = NG2 + 8;
    static constexpr int SP = XCH ? NG * PIE : NN + ((NG2 - NN) % 32 + 32) % 32;  // >= NN, == NG2 (mod 32)
    static constexpr int GEO_B = 12 * NN * 4;
    static constexpr int GEO_W = GEO_B / 4;
    static constexpr int GEO_SLOT = GEO_B + 4 * (((24 - GEO_W) % 32 + 32) % 32 / 4 * 4);
    static constexpr int IB_B = ib_row_words(NN) * 4;
    static constexpr int ARR = 3 * GR * SP;               // floats of one [3][GR][SP] array
    static constexpr int N_ARR = XCH ? 2 : 3;
    // dynamic shared memory without the per-model values (col_model_smem)
    static constexpr int SMEM = 2 * EPB * GEO_SLOT + 3 * EPB * IB_B + (N_ARR * ARR + 64) * 4;
    static constexpr int MIN_BLOCKS = THREADS <= 160 ? 3 : 2;
    static_assert(GEO_B % 16 == 0 && GEO_SLOT % 16 == 0 && IB_B % 16 == 0, "16-byte copies");
};

struct ColArgs {
    int e_begin, e_end, n_groups;
    const int* live_end;           // [colour] end of the stepping cells (several models), or null
    int colour;
    const uint32_t* ibool_padded;  // [cell][ib_row_words(NN)]: node words, model index
    const float* geom;             // [cell][12][NN]
    const float* ut;               // [node][NFLD][4]
    float* force;                  // [node][NFLD][4]
    const float* dmat;             // [NG*NG]
    const int* src_head;
    const int* src_next;
    const float* src_w;
    const float* mstf;             // [model][set] source time function value of this step
    const int* src_set;            // [slot] source set (nullptr: all set 0)
    int n_set;                     // n_model * n_set <= kMaxModels
    const int* mlive;              // [model] 1 while the model still steps
    const int* mdirect;            // [model] 1: force in full this step, 0: by increment (nullptr: in full)
    int n_model;                   // <= kMaxModels
    int dir[kMaxFields];
    int fset[kMaxFields];
    unsigned* err;                 // set to 1 when a bulk copy's wait gave up (the launch did not finish)
    float D[36];                   // D[i*NG+s], read with compile-time indices only
};

// Shared bytes of the per-model values of elem_col_kernel: source time
// function values [n_model][n_set], live and full-force flags [n_model].
__host__ __device__ constexpr int col_model_smem(int n_model, int n_set) { return (n_model * n_set + 2 * n_model) * 4; }

template <int NG, int NFLD, int EPB_, bool XCH = false>
__global__ void __launch_bounds__(ColShape<NG, NFLD, EPB_, XCH>::THREADS, ColShape<NG, NFLD, EPB_, XCH>::MIN_BLOCKS)
    elem_col_kernel(ColArgs A) {
    using S = ColShape<NG, NFLD, EPB_, XCH>;
    constexpr int NN = S::NN, NG2 = S::NG2, EPB = S::EPB, GR = S::GR, SP = S::SP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* gbase = smem_raw;
    unsigned char* ibase = gbase + 2 * EPB * S::GEO_SLOT;
    float* us = reinterpret_cast<float*>(ibase + 3 * EPB * S::IB_B);  // [3][GR][SP] displacement
    float* fe = us + S::ARR;                                          // [3][GR][SP] eta flux
    float* fz = fe + S::ARR;                                          // [3][GR][SP] zeta flux
    float* sD = us + S::N_ARR * S::ARR;
    // XCH: [3][GR][SP] eta and zeta arrays (u, then its derivative, the
    // flux, then the flux's contraction, each in place)
    float* xe = us;
    float* xz = us + S::ARR;

    // cells of this colour that still step (several models: the cells past
    // the last one of a live model belong to finished models)
    const int e_end = A.live_end ? min(A.e_end, A.live_end[A.colour]) : A.e_end;
    const int n_groups = e_end > A.e_begin ? (e_end - A.e_begin + EPB - 1) / EPB : 0;
    const int tid = threadIdx.x;
    const bool lane_ok = tid < S::ACTIVE;
    const int line = lane_ok ? tid / NG2 : 0;  // (cell, wavefield) line of this thread
    const int col = lane_ok ? tid - line * NG2 : 0;
    const int cl = line / NFLD, fld = line - cl * NFLD;
    const int j = col / NG, k = col - j * NG;
    int dir, fs;
    field_source<NFLD>(A.dir, A.fset, fld, dir, fs);
    // per-model step flags and source values of this step, read once per block
    // (in the dynamic shared memory after sD: col_model_smem bytes)
    float* s_stf = sD + 64;
    int* s_live = reinterpret_cast<int*>(s_stf + A.n_model * A.n_set);
    int* s_direct = s_live + A.n_model;
    for (int m = tid; m < A.n_model * A.n_set; m += S::THREADS) s_stf[m] = A.mstf[m];
    for (int m = tid; m < A.n_model; m += S::THREADS) {
        s_live[m] = A.mlive[m];
        s_direct[m] = A.mdirect ? A.mdirect[m] : 1;
    }
    if (tid < NG2) sD[tid] = A.dmat[tid];
    __syncthreads();
    float Dj[NG], Dk[NG], Tj[NG], Tk[NG];
#pragma unroll
    for (int s = 0; s < NG; ++s) {
        Dj[s] = sD[j * NG + s];
        Dk[s] = sD[k * NG + s];
        Tj[s] = sD[s * NG + j];
        Tk[s] = sD[s * NG + k];
    }

    auto geo_of = [&](int st, int c) -> const float* {
        return reinterpret_cast<const float*>(gbase + (st * EPB + c) * S::GEO_SLOT);
    };
    auto ib_of = [&](int st, int c) -> const uint32_t* {
        return reinterpret_cast<const uint32_t*>(ibase + (st * EPB + c) * S::IB_B);
    };
    // node words of this thread's line of group grp (node table in stage st)
    auto line_nodes = [&](int grp, int st, uint32_t (&w)[NG]) -> bool {
        const bool ok = lane_ok && grp < n_groups && A.e_begin + grp * EPB + cl < e_end;
#pragma unroll
        for (int i = 0; i < NG; ++i) w[i] = ok ? ib_of(st, cl)[i * NG2 + col] : 0u;
        return ok;
    };
    auto load_vectors = [&](const uint32_t (&w)[NG], bool ok, float4 (&v)[NG]) {
#pragma unroll
        for (int i = 0; i < NG; ++i)
            v[i] = ok ? __ldg(reinterpret_cast<const float4*>(A.ut) + (size_t)(w[i] & kNodeMask) * NFLD + fld)
                      : make_float4(0.f, 0.f, 0.f, 0.f);
    };

    // bulk-copy stages: barriers 0, 1 for the geometry, 2..4 for the node table
    __shared__ __align__(8) uint64_t s_bar[5];
    auto tma_geo = [&](int grp, int st) {
        if (tid != 0) return;
        const int e0 = A.e_begin + grp * EPB, nc = min(EPB, e_end - e0);
        fence_proxy_async_smem();
        mbar_expect_tx(&s_bar[st], (unsigned)(nc * S::GEO_B));
        for (int c = 0; c < nc; ++c)
            bulk_copy_g2s(gbase + (st * EPB + c) * S::GEO_SLOT,
                          reinterpret_cast<const unsigned char*>(A.geom) + (size_t)(e0 + c) * S::GEO_B, S::GEO_B,
                          &s_bar[st]);
    };
    auto tma_ib = [&](int grp, int st) {
        if (tid != 0) return;
        const int e0 = A.e_begin + grp * EPB, nc = min(EPB, e_end - e0);
        fence_proxy_async_smem();
        mbar_expect_tx(&s_bar[2 + st], (unsigned)(nc * S::IB_B));
        for (int c = 0; c < nc; ++c)
            bulk_copy_g2s(ibase + (st * EPB + c) * S::IB_B,
                          reinterpret_cast<const unsigned char*>(A.ibool_padded) + (size_t)(e0 + c) * S::IB_B,
                          S::IB_B, &s_bar[2 + st]);
    };
    // a wait that gave up: flag it, give the copies in flight a second
    // bounded wait, and leave (every thread together)
    auto give_up = [&](int b0, unsigned p0, int b1, unsigned p1) {
        if (tid == 0) {
            atomicOr(A.err, 1u);
            if (b0 >= 0) mbar_wait(&s_bar[b0], p0);
            if (b1 >= 0) mbar_wait(&s_bar[b1], p1);
        }
    };

    const int G = gridDim.x;
    const int grp0 = blockIdx.x;
    if (tid == 0) {
        for (int b = 0; b < 5; ++b) mbar_init(&s_bar[b], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (grp0 < n_groups) tma_ib(grp0, 0);
    if (__syncthreads_or(grp0 < n_groups && !mbar_wait(&s_bar[2], 0))) {
        give_up(2, 0, -1, 0);
        return;
    }
    uint32_t nw[NG];
    float4 pre[NG];
    bool pre_ok = line_nodes(grp0, 0, nw);
    load_vectors(nw, pre_ok, pre);
    if (grp0 < n_groups) tma_geo(grp0, 0);
    if (grp0 + G < n_groups) tma_ib(grp0 + G, 1);

    const int ubase = line * SP + col;        // + c*GR*SP + i*NG2
    const int ebase = line * SP + col - j * NG;  // + s*NG  (eta line: i*NG2 + s*NG + k)
    const int zbase = line * SP + j * NG;        // + s     (zeta line: i*NG2 + j*NG + s)
    // XCH: own points (i, j, k) at xown + i*PI; the eta line this thread owns
    // is (i = j, k = k) of its (cell, wavefield): points xline_e + s*NG; the
    // zeta line is (i = k, j = j): points xline_z + s
    const int xown_e = line * SP + j * NG + k, xown_z = xown_e;
    const int xline_e = line * SP + j * S::PIE + k;
    const int xline_z = line * SP + k * S::PIZ + j * NG;

    int it = 0;
    for (int grp = grp0; grp < n_groups; grp += G, ++it) {
        const int e = A.e_begin + grp * EPB + cl;
        const int mdl = pre_ok ? (int)ib_of(it % 3, cl)[NN] : 0;
        const bool act = pre_ok && s_live[mdl];
        // first touch stores only on a full-force step; by increments
        // every touch adds to the stored force
        const uint32_t first_bit = s_direct[mdl] ? kFirstTouch : 0u;
        uint32_t cw[NG];
        float u0[NG], u1[NG], u2[NG];
#pragma unroll
        for (int i = 0; i < NG; ++i) {
            cw[i] = nw[i];
            u0[i] = pre[i].x;
            u1[i] = pre[i].y;
            u2[i] = pre[i].z;
            if (act) {
                if constexpr (XCH) {
                    xe[0 * GR * SP + xown_e + i * S::PIE] = u0[i];
                    xe[1 * GR * SP + xown_e + i * S::PIE] = u1[i];
                    xe[2 * GR * SP + xown_e + i * S::PIE] = u2[i];
                    xz[0 * GR * SP + xown_z + i * S::PIZ] = u0[i];
                    xz[1 * GR * SP + xown_z + i * S::PIZ] = u1[i];
                    xz[2 * GR * SP + xown_z + i * S::PIZ] = u2[i];
                } else {
                    us[0 * GR * SP + ubase + i * NG2] = u0[i];
                    us[1 * GR * SP + ubase + i * NG2] = u1[i];
                    us[2 * GR * SP + ubase + i * NG2] = u2[i];
                }
            }
        }
        const int nx = grp + G;
        {
            // stage it&1 holds this group's geometry (use it/2 of that stage),
            // stage (it+1)%3 the next group's node table (use (it+1)/3)
            const unsigned pg = (unsigned)(it >> 1) & 1u, pi = (unsigned)((it + 1) / 3) & 1u;
            const int bi = nx < n_groups ? 2 + (it + 1) % 3 : -1;
            bool bad = !mbar_wait(&s_bar[it & 1], pg);
            if (bi >= 0) bad = !mbar_wait(&s_bar[bi], pi) || bad;
            if (__syncthreads_or(bad)) {  // displacement of this group, its geometry, the next node table
                give_up(it & 1, pg, bi, pi);
                return;
            }
        }
        if (nx < n_groups) tma_geo(nx, (it + 1) & 1);
        if (nx + G < n_groups) tma_ib(nx + G, (it + 2) % 3);
        // old force vectors of the nodes this colour does not touch first:
        // start their DRAM reads into L2 now, so the loads issued after the
        // flux phase find them there (no registers held meanwhile)
        if (act) {
#pragma unroll
            for (int i = 0; i < NG; ++i)
                if (!(cw[i] & first_bit)) {
                    const float4* pf = reinterpret_cast<const float4*>(A.force) + (size_t)(cw[i] & kNodeMask) * NFLD + fld;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(pf));
                }
        }
        const float stf = act ? s_stf[mdl * A.n_set + fs] : 0.f;
        const int src = (act && stf != 0.f && A.src_head) ? __ldg(A.src_head + e) : -1;
        pre_ok = line_nodes(nx, (it + 1) % 3, nw);
        load_vectors(nw, pre_ok, pre);

        // old force of the nodes this colour does not touch first
        float4 of[NG];
        auto load_old_force = [&]() {
#pragma unroll
            for (int i = 0; i < NG; ++i)
                of[i] = (act && !(cw[i] & first_bit))
                            ? *(reinterpret_cast<const float4*>(A.force) + (size_t)(cw[i] & kNodeMask) * NFLD + fld)
                            : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        if constexpr (XCH) {
            // line owners: d/d-eta along this thread's eta line and d/d-zeta
            // along its zeta line, in place (the lines of a (cell, wavefield)
            // are disjoint; the two arrays hold the same displacement)
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float* le = xe + c * GR * SP + xline_e;
                    float* lz = xz + c * GR * SP + xline_z;
                    float ve[NG], vz[NG];
#pragma unroll
                    for (int t = 0; t < NG; ++t) {
                        ve[t] = le[t * NG];
                        vz[t] = lz[t];
                    }
#pragma unroll
                    for (int s2 = 0; s2 < NG; ++s2) {
                        float de = 0.f, dz = 0.f;
#pragma unroll
                        for (int t = 0; t < NG; ++t) {
                            de += A.D[s2 * NG + t] * ve[t];
                            dz += A.D[s2 * NG + t] * vz[t];
                        }
                        le[s2 * NG] = de;
                        lz[s2] = dz;
                    }
                }
            }
            __syncthreads();  // the eta and zeta derivatives of the whole group
        }
        // gradient, stress and the three fluxes at each point of the line
        float fx0[NG], fx1[NG], fx2[NG];
        const float* geo = geo_of(it & 1, cl);
#pragma unroll
        for (int i = 0; i < NG; ++i) {
            fx0[i] = fx1[i] = fx2[i] = 0.f;
            if (!act) continue;
            const int p = i * NG2 + col;
            float dd[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) dd[q] = geo[q * NN + p];
            const float jw = geo[9 * NN + p], lam = geo[10 * NN + p], mu = geo[11 * NN + p];
            float gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int s = 0; s < NG; ++s) {
                const float Di = A.D[i * NG + s];
                gx[0] += Di * u0[s];
                gx[1] += Di * u1[s];
                gx[2] += Di * u2[s];
            }
            if constexpr (XCH) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    gy[c] = xe[c * GR * SP + xown_e + i * S::PIE];
                    gz[c] = xz[c * GR * SP + xown_z + i * S::PIZ];
                }
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float* uc = us + c * GR * SP + i * NG2;
#pragma unroll
                    for (int s = 0; s < NG; ++s) {
                        gy[c] += Dj[s] * uc[ebase + s * NG];
                        gz[c] += Dk[s] * uc[zbase + s];
                    }
                }
            }
            float st0 = 0.f, st1 = 0.f, st2 = 0.f, st3 = 0.f, st4 = 0.f, st5 = 0.f;
            if (mu > 0.f) {  // element_cpu.cpp:42-43: mu <= 0 adds nothing
                float gr[3][3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    gr[c][0] = gx[c] * dd[0] + gy[c] * dd[1] + gz[c] * dd[2];
                    gr[c][1] = gx[c] * dd[3] + gy[c] * dd[4] + gz[c] * dd[5];
                    gr[c][2] = gx[c] * dd[6] + gy[c] * dd[7] + gz[c] * dd[8];
                }
                const float tr = gr[0][0] + gr[1][1] + gr[2][2];
                const float m2 = 2.f * mu;
                st0 = m2 * gr[0][0] + lam * tr;
                st1 = m2 * gr[1][1] + lam * tr;
                st2 = m2 * gr[2][2] + lam * tr;
                st3 = m2 * (0.5f * (gr[0][1] + gr[1][0]));
                st4 = m2 * (0.5f * (gr[0][2] + gr[2][0]));
                st5 = m2 * (0.5f * (gr[1][2] + gr[2][1]));
            }
            // flux along axis a: jw * sigma . (dd[a], dd[3+a], dd[6+a])
            fx0[i] = jw * (st0 * dd[0] + st3 * dd[3] + st4 * dd[6]);
            fx1[i] = jw * (st3 * dd[0] + st1 * dd[3] + st5 * dd[6]);
            fx2[i] = jw * (st4 * dd[0] + st5 * dd[3] + st2 * dd[6]);
            const float e0 = jw * (st0 * dd[1] + st3 * dd[4] + st4 * dd[7]);
            const float e1 = jw * (st3 * dd[1] + st1 * dd[4] + st5 * dd[7]);
            const float e2 = jw * (st4 * dd[1] + st5 * dd[4] + st2 * dd[7]);
            const float z0 = jw * (st0 * dd[2] + st3 * dd[5] + st4 * dd[8]);
            const float z1 = jw * (st3 * dd[2] + st1 * dd[5] + st5 * dd[8]);
            const float z2 = jw * (st4 * dd[2] + st5 * dd[5] + st2 * dd[8]);
            if constexpr (XCH) {  // own points: the derivatives read above are replaced
                xe[0 * GR * SP + xown_e + i * S::PIE] = e0;
                xe[1 * GR * SP + xown_e + i * S::PIE] = e1;
                xe[2 * GR * SP + xown_e + i * S::PIE] = e2;
                xz[0 * GR * SP + xown_z + i * S::PIZ] = z0;
                xz[1 * GR * SP + xown_z + i * S::PIZ] = z1;
                xz[2 * GR * SP + xown_z + i * S::PIZ] = z2;
            } else {
                fe[0 * GR * SP + ubase + i * NG2] = e0;
                fe[1 * GR * SP + ubase + i * NG2] = e1;
                fe[2 * GR * SP + ubase + i * NG2] = e2;
                fz[0 * GR * SP + ubase + i * NG2] = z0;
                fz[1 * GR * SP + ubase + i * NG2] = z1;
                fz[2 * GR * SP + ubase + i * NG2] = z2;
            }
        }
        load_old_force();
        __syncthreads();  // fluxes of the whole group
        if constexpr (XCH) {
            // line owners: the eta (zeta) contraction of the divergence along
            // this thread's eta (zeta) line, in place
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float* le = xe + c * GR * SP + xline_e;
                    float* lz = xz + c * GR * SP + xline_z;
                    float ve[NG], vz[NG];
#pragma unroll
                    for (int t = 0; t < NG; ++t) {
                        ve[t] = le[t * NG];
                        vz[t] = lz[t];
                    }
#pragma unroll
                    for (int s2 = 0; s2 < NG; ++s2) {
                        float de = 0.f, dz = 0.f;
#pragma unroll
                        for (int t = 0; t < NG; ++t) {
                            de += A.D[t * NG + s2] * ve[t];
                            dz += A.D[t * NG + s2] * vz[t];
                        }
                        le[s2 * NG] = de;
                        lz[s2] = dz;
                    }
                }
            }
            __syncthreads();  // contractions of the whole group
        }
        if (act) {
#pragma unroll
            for (int i = 0; i < NG; ++i) {
                const int p = i * NG2 + col;
                float r[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int s = 0; s < NG; ++s) {
                    const float Ti = A.D[s * NG + i];
                    r[0] += Ti * fx0[s];
                    r[1] += Ti * fx1[s];
                    r[2] += Ti * fx2[s];
                }
                if constexpr (XCH) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        r[c] += xe[c * GR * SP + xown_e + i * S::PIE];
                        r[c] += xz[c * GR * SP + xown_z + i * S::PIZ];
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float* ec = fe + c * GR * SP + i * NG2;
                        const float* zc = fz + c * GR * SP + i * NG2;
#pragma unroll
                        for (int s = 0; s < NG; ++s) {
                            r[c] += Tj[s] * ec[ebase + s * NG];
                            r[c] += Tk[s] * zc[zbase + s];
                        }
                    }
                }
                r[0] = -r[0];
                r[1] = -r[1];
                r[2] = -r[2];
                // point force (solver.cpp:577-605)
                for (int sl = src; sl >= 0; sl = __ldg(A.src_next + sl)) {
                    if (A.src_set && __ldg(A.src_set + sl) != fs) continue;
                    const float w = __ldg(A.src_w + (size_t)sl * NN + p);
                    if (w != 0.f) {
                        const float sw = stf * w;
                        if (dir == 0) r[0] += sw;
                        else if (dir == 1) r[1] += sw;
                        else r[2] += sw;
                    }
                }
                float4* dst = reinterpret_cast<float4*>(A.force) + (size_t)(cw[i] & kNodeMask) * NFLD + fld;
                *dst = make_float4(of[i].x + r[0], of[i].y + r[1], of[i].z + r[2], 0.f);
            }
        }
    }
}

// Predictor only (start of a run or after a state overwrite).
// Nodes g >= hv_begin hold the half-step velocity (v + dt/2 a) in w32.
template <typename Real>
__global__ void predict_kernel(long long n_node, int F, const double* u, const double* v, const Real* a,
                               Real* ut, double dt, double half_dt2, const uint8_t* node_model,
                               const ModelConst* mc, long long hv_begin, const float* w32) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long total = n_node * F;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const long long g = idx / F;
        const int f = (int)(idx - g * F);
        double h = dt, h2 = half_dt2;
        if (node_model) {
            const ModelConst& K = mc[node_model[g]];
            h = K.dt;
            h2 = K.half_dt2;
        }
        ut[padded_index(g, f, F)] =
            g >= hv_begin ? (Real)(u[idx] + h * (double)w32[idx]) : (Real)(u[idx] + h * v[idx] + h2 * (double)a[idx]);
        if (f % 3 == 2) ut[padded_index(g, f, F) + 1] = Real(0);
    }
}

template <typename Real, typename Out>
struct RecArgs {
    int n_rec;
    const int* rec_cell;    // [n_rec] device cell index
    const uint32_t* ibool;
    const Real* geom;
    const Real* dmat;
    const double* u;        // [node][3*n_field]
    const double* v;
    const Real* a;
    long long n_node;
    Out* out;               // [NFLD][n_rec][NN][15]
    // nodes g >= hv_begin hold the half-step velocity w (w32): a = f/m from
    // the step's assembled force, v = w - dt/2 a
    long long hv_begin;
    const float* w32;
    const Real* force;      // [node][NFLD][4]
    const Real* inv_mass;   // [node]
    const uint8_t* node_model;
    const ModelConst* mc;
    double dt;
};

// Snapshot of the recording cells: strain from the gathered corrected
// displacement (solver.cpp:282-335) plus u, v, a at every cell node
// (solver.cpp:485-504).  One block per recording cell.
template <typename Real, int NG, int NFLD, typename Out>
__global__ void record_kernel(RecArgs<Real, Out> A) {
    using S = Shape<NG>;
    constexpr int NN = S::NN, F = 3 * NFLD;
    __shared__ double su[F][NN];
    __shared__ double sD[NG * NG];
    const int ci = blockIdx.x;
    const int p = threadIdx.x;
    if (p < NG * NG) sD[p] = (double)A.dmat[p];
    const int e = A.rec_cell[ci];
    uint32_t g = 0;
    if (p < NN) {
        g = A.ibool[(size_t)e * NN + p] & kNodeMask;
        for (int f = 0; f < F; ++f) su[f][p] = A.u[(size_t)g * F + f];
    }
    __syncthreads();
    if (p >= NN) return;
    const int i = p / (NG * NG), j = (p / NG) % NG, k = p % NG;
    double dd[9];
    const Real* gp = A.geom + (size_t)e * 12 * NN + p;
    for (int q = 0; q < 9; ++q) dd[q] = (double)gp[q * NN];
    for (int d = 0; d < NFLD; ++d) {
        double gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0}, gz[3] = {0, 0, 0};
        for (int s = 0; s < NG; ++s) {
            const double Di = sD[i * NG + s], Dj = sD[j * NG + s], Dk = sD[k * NG + s];
            for (int c = 0; c < 3; ++c) {
                gx[c] += Di * su[d * 3 + c][(s * NG + j) * NG + k];
                gy[c] += Dj * su[d * 3 + c][(i * NG + s) * NG + k];
                gz[c] += Dk * su[d * 3 + c][(i * NG + j) * NG + s];
            }
        }
        double gr[3][3];
        for (int c = 0; c < 3; ++c) {
            gr[c][0] = gx[c] * dd[0] + gy[c] * dd[1] + gz[c] * dd[2];
            gr[c][1] = gx[c] * dd[3] + gy[c] * dd[4] + gz[c] * dd[5];
            gr[c][2] = gx[c] * dd[6] + gy[c] * dd[7] + gz[c] * dd[8];
        }
        Out* o = A.out + (((size_t)d * A.n_rec + ci) * NN + p) * 15;
        o[0] = (Out)gr[0][0];
        o[1] = (Out)gr[1][1];
        o[2] = (Out)gr[2][2];
        o[3] = (Out)(0.5 * (gr[0][1] + gr[1][0]));
        o[4] = (Out)(0.5 * (gr[0][2] + gr[2][0]));
        o[5] = (Out)(0.5 * (gr[1][2] + gr[2][1]));
        if ((long long)g >= A.hv_begin) {
            const double h = A.node_model ? A.mc[A.node_model[g]].dt : A.dt;
            const Real im = A.inv_mass[g];
            for (int c = 0; c < 3; ++c) {
                const double an = (double)(Real)(A.force[((size_t)g * NFLD + d) * 4 + c] * im);
                o[6 + c] = (Out)A.u[(size_t)g * F + d * 3 + c];
                o[9 + c] = (Out)((double)A.w32[(size_t)g * F + d * 3 + c] - 0.5 * h * an);
                o[12 + c] = (Out)an;
            }
        } else {
            for (int c = 0; c < 3; ++c) {
                o[6 + c] = (Out)A.u[(size_t)g * F + d * 3 + c];
                o[9 + c] = (Out)A.v[(size_t)g * F + d * 3 + c];
                o[12 + c] = (Out)A.a[(size_t)g * F + d * 3 + c];
            }
        }
    }
}


// Half-step velocity state (w32) <-> (v, a) at the nodes g >= hv_begin.
// to_full: v_out = w - dt/2 a, a_out = a with a = f/m from the assembled
// force (a_from_force) or the stored a (state set since the last step);
// otherwise (from_full): w = v + dt/2 a.  One thread per (node, value).
template <typename Real>
__global__ void half_v_kernel(long long n_node, int F, long long hv_begin, bool to_full, bool a_from_force,
                              const double* v, float* w32, const Real* a, const Real* force, const Real* inv_mass,
                              const uint8_t* node_model, const ModelConst* mc, double dt, double* v_out,
                              Real* a_out) {
    const long long total = (n_node - hv_begin) * F;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = hv_begin + t / F;
        const int f = (int)(t % F);
        const size_t i = (size_t)g * F + f;
        const double h = node_model ? mc[node_model[g]].dt : dt;
        if (to_full) {
            const double an = a_from_force ? (double)(Real)(force[padded_index(g, f, F)] * inv_mass[g]) : (double)a[i];
            v_out[i] = (double)w32[i] - 0.5 * h * an;
            a_out[i] = (Real)an;
        } else {
            w32[i] = (float)(v[i] + 0.5 * h * (double)a[i]);
        }
    }
}

// Recording nodes merged across the recording cells that share them (the
// strain Green's-function extraction of postprocess/cpp/main.cpp:300-425):
// strain mass-weighted, sum(m_p e_p) / sum(m_p) over the node's (cell, point)
// occurrences; u, v, a averaged.  One thread per (wavefield, node, value),
// reading the snapshot's cell-point records (out[field][rec][NN][15]) and
// writing merged[field][node][15] behind them in the same slot.
template <typename Out>
__global__ void merge_nodes_kernel(int n_field, int n_unique, long long per_field, const int* ptr, const int* occ,
                                   const double* w, Out* slot) {
    const long long total = (long long)n_field * n_unique * 15;
    Out* merged = slot + (size_t)n_field * per_field;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t % 15);
        const long long fn = t / 15;
        const int node = (int)(fn % n_unique), f = (int)(fn / n_unique);
        const Out* src = slot + (size_t)f * per_field;
        double acc = 0.0, ws = 0.0;
        for (int k = ptr[node]; k < ptr[node + 1]; ++k) {
            const double wk = c < 6 ? w[k] : 1.0;
            acc += wk * (double)src[(size_t)occ[k] * 15 + c];
            ws += wk;
        }
        merged[((size_t)f * n_unique + node) * 15 + c] = (Out)(ws > 0.0 ? acc / ws : 0.0);
    }
}

}  // namespace gfb
