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

// Predicted displacement and force of the time loop are stored
// [node][field][4] (x, y, z, pad) so a field of a node is one 16-byte
// vector; u, v, a are [node][3*field].  Index of component f of node g.
__device__ __forceinline__ long long padded_index(long long g, int f, int F) {
    return g * (F / 3) * 4 + (f / 3) * 4 + (f % 3);
}

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

// ---------------------------------------------------------------------------
// elem_field_kernel: the time loop's element/assembly kernel.
//
// One thread per (GLL point, wavefield): the three wavefields of a point run
// in three different warps, so a thread holds one field's gradient and
// stress and there are three times more warps to cover the gather latency
// than with one thread per point.  Per cell:
//   1. the cell's geometry block [12][NN] (contiguous, 16-byte multiple) is
//      staged into shared memory with 16-byte loads by all the cell's
//      threads; each thread gathers its node's field as one 16-byte vector
//      ([node][field][4] layout) into shared memory;
//   2. gradient from 3 x NG neighbour vectors, Hooke stress in registers;
//   3. for each reference axis: the flux jw * sigma . (dd[a], dd[3+a],
//      dd[6+a]) goes to the same shared buffer, and the divergence
//      contribution is summed from NG neighbour vectors of that axis;
//   4. C-PML per-cell term (FP64 path / per-cell form), point force, and
//      the colour-ordered read-modify-write of the node's force vector.
// Shared memory per cell: 12*NN + 4*NN*n_field words.
// ---------------------------------------------------------------------------

template <int NG, int NFLD>
struct FieldShape {
    static constexpr int NN = NG * NG * NG;
    static constexpr int NNP = (NN + 31) / 32 * 32;
    static constexpr int TPE = NNP * NFLD;                  // threads per cell
    static constexpr int EPB = TPE >= 256 ? 1 : 256 / TPE;  // cells per block
    static constexpr int THREADS = TPE * EPB;
    static constexpr int GEO = 12 * NN;                     // geometry words per cell
    static constexpr int BUF = 4 * NN * NFLD;               // vector words per cell
};

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

template <typename Real, int NG, int NFLD>
constexpr size_t field_smem_bytes() {
    using S = FieldShape<NG, NFLD>;
    return sizeof(Real) * (64 + (size_t)S::EPB * (S::GEO + S::BUF));
}

template <typename Real, int NG, int NFLD>
__global__ void __launch_bounds__(FieldShape<NG, NFLD>::THREADS) elem_field_kernel(ElemArgs<Real> A) {
    using S = FieldShape<NG, NFLD>;
    constexpr int NN = S::NN, NNP = S::NNP, TPE = S::TPE, EPB = S::EPB, F = 3 * NFLD;
    static_assert((S::GEO * sizeof(Real)) % 16 == 0, "geometry block must be a 16-byte multiple");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* sD = reinterpret_cast<Real*>(smem_raw);
    const int tid = threadIdx.x;
    const int el = tid / TPE;
    const int rem = tid - el * TPE;
    const int d = rem / NNP;
    const int p = rem - d * NNP;
    const int e = A.e_begin + blockIdx.x * EPB + el;
    const bool cell_ok = e < A.e_end;
    const bool active = cell_ok && p < NN;
    Real* geo = sD + 64 + el * (S::GEO + S::BUF);
    Real* buf = geo + S::GEO;
    if (tid < NG * NG) sD[tid] = A.dmat[tid];
    if (cell_ok) {
        constexpr int CH = (int)(S::GEO * sizeof(Real) / 16);
        const uint4* src = reinterpret_cast<const uint4*>(A.geom + (size_t)e * S::GEO);
        uint4* dst = reinterpret_cast<uint4*>(geo);
        for (int q = rem; q < CH; q += TPE) dst[q] = __ldg(src + q);
    }
    uint32_t gword = 0;
    if (active) {
        gword = __ldg(A.ibool + (size_t)e * NN + p);
        Real v[4];
        load4_nc(A.ut + ((size_t)(gword & kNodeMask) * NFLD + d) * 4, v);
        store4(buf + (p * NFLD + d) * 4, v[0], v[1], v[2], v[3]);
    }
    __syncthreads();
    const int i = p / (NG * NG), j = (p / NG) % NG, k = p % NG;
    Real dd[9], jw = Real(0);
    Real s00 = 0, s11 = 0, s22 = 0, s01 = 0, s02 = 0, s12 = 0;
    if (active) {
#pragma unroll
        for (int q = 0; q < 9; ++q) dd[q] = geo[q * NN + p];
        jw = geo[9 * NN + p];
        const Real lam = geo[10 * NN + p], mu = geo[11 * NN + p];
        if (mu > Real(0)) {  // element_cpu.cpp:42-43: mu <= 0 adds nothing
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
            s00 = m2 * gr[0][0] + lam * tr;
            s11 = m2 * gr[1][1] + lam * tr;
            s22 = m2 * gr[2][2] + lam * tr;
            s01 = m2 * (Real(0.5) * (gr[0][1] + gr[1][0]));
            s02 = m2 * (Real(0.5) * (gr[0][2] + gr[2][0]));
            s12 = m2 * (Real(0.5) * (gr[1][2] + gr[2][1]));
        }
    }
    __syncthreads();  // buf is reused for the fluxes
    Real r0 = Real(0), r1 = Real(0), r2 = Real(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (active) {
            const Real ea = dd[a], eb = dd[3 + a], ec = dd[6 + a];
            store4(buf + (p * NFLD + d) * 4, jw * (s00 * ea + s01 * eb + s02 * ec),
                   jw * (s01 * ea + s11 * eb + s12 * ec), jw * (s02 * ea + s12 * eb + s22 * ec), Real(0));
        }
        __syncthreads();
        if (active) {
            const int ia = (a == 0) ? i : ((a == 1) ? j : k);
#pragma unroll
            for (int s = 0; s < NG; ++s) {
                const int q = (a == 0) ? ((s * NG + j) * NG + k) : ((a == 1) ? ((i * NG + s) * NG + k) : ((i * NG + j) * NG + s));
                Real v[4];
                load4(buf + (q * NFLD + d) * 4, v);
                const Real w = sD[s * NG + ia];
                r0 -= w * v[0];
                r1 -= w * v[1];
                r2 -= w * v[2];
            }
        }
        if (a < 2) __syncthreads();
    }
    if (!active) return;
    const uint32_t g = gword & kNodeMask;
    // C-PML per cell (pml.cpp:55-216), as in elem_step_kernel
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
        Real rr[3] = {r0, r1, r2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int f = d * 3 + c;
            const double un = A.u[(size_t)g * F + f];
            const double vn = A.v[(size_t)g * F + f];
            const Real an = A.a[(size_t)g * F + f];
            const Real nv = Real(un + A.c1 * vn);
            const Real ov = prev[f * NN] + Real(A.c2) * an;
            Real m0 = mem[(f * 3 + 0) * NN], m1 = mem[(f * 3 + 1) * NN], m2 = mem[(f * 3 + 2) * NN];
            rr[c] += scale * (ab[0] * Real(vn) + ab[1] * Real(un) + ab[2] * m0 + ab[3] * m1 + ab[4] * m2);
            m0 = al[0] * m0 + al[1] * nv + al[2] * ov;
            m1 = al[3] * m1 + al[4] * nv + al[5] * ov;
            m2 = al[6] * m2 + al[7] * nv + al[8] * ov;
            mem[(f * 3 + 0) * NN] = m0;
            mem[(f * 3 + 1) * NN] = m1;
            mem[(f * 3 + 2) * NN] = m2;
            prev[f * NN] = nv;
        }
        r0 = rr[0];
        r1 = rr[1];
        r2 = rr[2];
    }
    // point force (solver.cpp:577-605)
    if (A.stf != Real(0)) {
        const int dir = (d == 0) ? A.dir0 : ((d == 1) ? A.dir1 : A.dir2);
        int s = A.src_head ? __ldg(A.src_head + e) : -1;
        while (s >= 0) {
            const Real w = __ldg(A.src_w + (size_t)s * NN + p);
            if (w != Real(0)) {
                const Real sw = A.stf * w;
                if (dir == 0) r0 += sw;
                else if (dir == 1) r1 += sw;
                else r2 += sw;
            }
            s = __ldg(A.src_next + s);
        }
    }
    Real* out = A.force + ((size_t)g * NFLD + d) * 4;
    if (gword & kFirstTouch) {
        store4(out, r0, r1, r2, Real(0));
    } else {
        Real v[4];
        load4(out, v);
        store4(out, v[0] + r0, v[1] + r1, v[2] + r2, Real(0));
    }
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
        const int f = (int)(idx - g * A.F);
        const long long pi = padded_index(g, f, A.F);
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
            if (A.inv_mass) a_new = (double)(A.force[pi] * A.inv_mass[g]);
            else a_new = (double)A.force[pi] / m;
            a_new = (double)(Real)a_new;
            uu += A.dt * vv + A.dt * A.dt * ((0.5 - A.beta) * a_old + A.beta * a_new);
            vv += A.dt * ((1.0 - A.gamma) * a_old + A.gamma * a_new);
        }
        A.u[idx] = uu;
        A.v[idx] = vv;
        A.a[idx] = (Real)a_new;
        A.ut[pi] = (Real)(uu + A.dt * vv + A.half_dt2 * a_new);
    }
}

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
template <typename Real>
struct NodePml {
    const int* slot;     // [n_node] -1 or C-PML node slot
    const Real* coef;    // [slot][14]: B1..B5, alpha x(3), y(3), z(3)
    Real* mem;           // [slot][F][3]
    Real* prev;          // [slot][F]  last step's u + c1 v
    double c1, c2;
};

template <typename Real>
__global__ void node_update_pml_kernel(NodeArgs<Real> A, NodePml<Real> P) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < A.n; idx += stride) {
        const long long g = idx / A.F;
        const int f = (int)(idx - g * A.F);
        const long long pi = padded_index(g, f, A.F);
        double vv = A.v[idx];
        double uu = A.u[idx];
        const double a_old = (double)A.a[idx];
        Real force = A.force[pi];
        const int sl = __ldg(P.slot + g);
        if (sl >= 0) {
            const Real* cf = P.coef + (size_t)sl * 14;
            Real* m = P.mem + ((size_t)sl * A.F + f) * 3;
            Real* pv = P.prev + (size_t)sl * A.F + f;
            const Real nv = (Real)(uu + P.c1 * vv);
            const Real ov = *pv + (Real)P.c2 * (Real)a_old;
            const Real m0 = m[0], m1 = m[1], m2 = m[2];
            force += __ldg(cf + 0) * (Real)vv + __ldg(cf + 1) * (Real)uu + __ldg(cf + 2) * m0 +
                     __ldg(cf + 3) * m1 + __ldg(cf + 4) * m2;
            if (__ldg(cf + 2) != Real(0)) m[0] = __ldg(cf + 5) * m0 + __ldg(cf + 6) * nv + __ldg(cf + 7) * ov;
            if (__ldg(cf + 3) != Real(0)) m[1] = __ldg(cf + 8) * m1 + __ldg(cf + 9) * nv + __ldg(cf + 10) * ov;
            if (__ldg(cf + 4) != Real(0)) m[2] = __ldg(cf + 11) * m2 + __ldg(cf + 12) * nv + __ldg(cf + 13) * ov;
            *pv = nv;
        }
        const double mass = A.mass[g];
        double a_new;
        if (mass <= 0.0) {
            a_new = 0.0;
        } else {
            a_new = (double)(Real)(force * A.inv_mass[g]);
            uu += A.dt * vv + A.dt * A.dt * ((0.5 - A.beta) * a_old + A.beta * a_new);
            vv += A.dt * ((1.0 - A.gamma) * a_old + A.gamma * a_new);
        }
        A.u[idx] = uu;
        A.v[idx] = vv;
        A.a[idx] = (Real)a_new;
        A.ut[pi] = (Real)(uu + A.dt * vv + A.half_dt2 * a_new);
    }
}

// Predictor only (start of a run or after a state overwrite).
template <typename Real>
__global__ void predict_kernel(long long n, int F, const double* u, const double* v, const Real* a,
                               Real* ut, double dt, double half_dt2) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const long long g = idx / F;
        ut[padded_index(g, (int)(idx - g * F), F)] = (Real)(u[idx] + dt * v[idx] + half_dt2 * (double)a[idx]);
    }
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
