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
//   state  [node][F]             F = 3 * n_field; u, v in double, a/ut/force in Real
//   C-PML  coef [slot][15][NN] Real (alpha 9, abar 5, w*J/rho),
//          mem [slot][n_field*9][NN], prev [slot][n_field*3][NN]
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gfb {

constexpr uint32_t kFirstTouch = 0x80000000u;
constexpr uint32_t kNodeMask = 0x3fffffffu;

template <int NG>
struct Shape {
    static constexpr int NN = NG * NG * NG;
    static constexpr int NNP = (NN + 31) / 32 * 32;
    static constexpr int EPB = NNP <= 32 ? 8 : (NNP <= 64 ? 4 : (NNP <= 128 ? 2 : 1));
    static constexpr int THREADS = NNP * EPB;
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
    const double* u;
    const double* v;
    const Real* a;
    double c1, c2;
    // source
    const int* src_head;  // [cell] first source slot or -1
    const int* src_next;  // [slot]
    const Real* src_w;    // [slot][NN]
    Real stf;
    int dir0, dir1, dir2;
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
    // point-force source
    if (A.stf != Real(0)) {
        int s = A.src_head ? __ldg(A.src_head + e) : -1;
        while (s >= 0) {
            const Real w = __ldg(A.src_w + (size_t)s * NN + p);
            if (w != Real(0)) {
                const Real sw = A.stf * w;
                const int dirs[3] = {A.dir0, A.dir1, A.dir2};
#pragma unroll
                for (int d = 0; d < NFLD; ++d)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        if (c == dirs[d]) r[d * 3 + c] += sw;
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

template <typename Real>
struct NodeArgs {
    long long n;      // n_node * F
    int F;
    double* u;
    double* v;
    Real* a;
    Real* ut;
    const Real* force;
    const double* mass;     // [n_node] assembled lumped mass
    const Real* inv_mass;   // [n_node] 1/m (FP32 path) or nullptr
    const double* damping;  // [n_node] or nullptr
    double dt, half_dt2, beta, gamma;
};

// Newmark corrector (solver.cpp:52-69, with the legacy damping of 564-574
// applied to v first) followed by the next step's predictor (40-49).
template <typename Real>
__global__ void node_update_kernel(NodeArgs<Real> A) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < A.n; idx += stride) {
        const long long g = idx / A.F;
        double vv = A.v[idx];
        if (A.damping) {
            const double d = A.damping[g];
            if (d > 0.0) vv -= d * vv;
        }
        double uu = A.u[idx];
        const double m = A.mass[g];
        double a_new;
        if (m <= 0.0) {
            a_new = 0.0;
        } else {
            const double a_old = (double)A.a[idx];
            if (A.inv_mass) a_new = (double)(A.force[idx] * A.inv_mass[g]);
            else a_new = (double)A.force[idx] / m;
            a_new = (double)(Real)a_new;
            uu += A.dt * vv + A.dt * A.dt * ((0.5 - A.beta) * a_old + A.beta * a_new);
            vv += A.dt * ((1.0 - A.gamma) * a_old + A.gamma * a_new);
        }
        A.u[idx] = uu;
        A.v[idx] = vv;
        A.a[idx] = (Real)a_new;
        A.ut[idx] = (Real)(uu + A.dt * vv + A.half_dt2 * a_new);
    }
}

// Predictor only (start of a run or after a state overwrite).
template <typename Real>
__global__ void predict_kernel(long long n, const double* u, const double* v, const Real* a,
                               Real* ut, double dt, double half_dt2) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride)
        ut[idx] = (Real)(u[idx] + dt * v[idx] + half_dt2 * (double)a[idx]);
}

template <typename Real>
struct RecArgs {
    int n_rec;
    const int* rec_cell;    // [n_rec] device cell index
    const uint32_t* ibool;
    const Real* geom;
    const Real* dmat;
    const double* u;
    const double* v;
    const Real* a;
    double* out;            // [NFLD][n_rec][NN][15]
};

// Snapshot of the recording cells: strain from the gathered corrected
// displacement (solver.cpp:282-335) plus u, v, a at every cell node
// (solver.cpp:485-504).  One block per recording cell.
template <typename Real, int NG, int NFLD>
__global__ void record_kernel(RecArgs<Real> A) {
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
        double* o = A.out + (((size_t)d * A.n_rec + ci) * NN + p) * 15;
        o[0] = gr[0][0];
        o[1] = gr[1][1];
        o[2] = gr[2][2];
        o[3] = 0.5 * (gr[0][1] + gr[1][0]);
        o[4] = 0.5 * (gr[0][2] + gr[2][0]);
        o[5] = 0.5 * (gr[1][2] + gr[2][1]);
        for (int c = 0; c < 3; ++c) {
            o[6 + c] = A.u[(size_t)g * F + d * 3 + c];
            o[9 + c] = A.v[(size_t)g * F + d * 3 + c];
            o[12 + c] = (double)A.a[(size_t)g * F + d * 3 + c];
        }
    }
}

}  // namespace gfb
