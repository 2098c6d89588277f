// gfb_prep.cu -- the solver's mesh inputs computed on the device.
//
// The reference produces these arrays on the host, in Python:
//   * GLL geometry of trilinear hexes: coordinates, det J, inv(J) raveled and
//     the geometric mass det J w_i w_j w_k (preprocess/gll_geometry.py:132-186);
//   * the global node numbering ibool by a lexicographic sort of quantised
//     coordinates (preprocess/partition.py:192-254);
//   * the C-PML region of each cell, the per-point profiles K, d, alpha, the
//     convolution coefficients and A1..A5 (preprocess/pml_cpml.py:42-147,
//     174-253, 261-345, 353-515).
// Here each is a kernel (one thread per GLL point; the sort is CUB's radix
// sort in three stable passes), with host arrays in and out through the C
// ABI.  Element-wise formulas keep the reference's operation order with every
// product and sum rounded separately (no fused multiply-add), so they round
// as numpy does; sums of products that numpy hands to BLAS (the trilinear
// map) and exp/log/pow may differ from numpy in the last bits.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/gfb.h"
#include "gfb_internal.h"

namespace {

gfb_status prep_fail(gfb_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return gfb::set_error(st, buf);
}

#define PCU(call)                                                                               \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return prep_fail(_e == cudaErrorMemoryAllocation ? GFB_ERR_NOMEM : GFB_ERR_CUDA,    \
                             "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// Device buffers of one call, freed on every return path.
struct Scratch {
    std::vector<void*> ptrs;
    template <typename T>
    cudaError_t alloc(T** p, size_t n) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = static_cast<T*>(q);
        return e;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
};

gfb_status open_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return prep_fail(GFB_ERR_NO_DEVICE, "no CUDA-capable GPU found");
    if (device < 0 || device >= n) return prep_fail(GFB_ERR_INVALID, "device %d not present", device);
    PCU(cudaSetDevice(device));
    return GFB_OK;
}

unsigned blocks_for(long long n, int threads) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 1LL << 30));
}

// GMSH hex corner order in reference coordinates (gll_geometry.py:14-26).
__constant__ double c_corner[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// ---------------------------------------------------------------------------
// GLL geometry: one thread per (cell, point)
// ---------------------------------------------------------------------------

__global__ void geometry_kernel(long long n_cell, int ng, const double* __restrict__ gx, const double* __restrict__ gw,
                                const double* __restrict__ corners, double* __restrict__ coords,
                                double* __restrict__ jac, double* __restrict__ dxi, double* __restrict__ mass) {
    const int nn = ng * ng * ng;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cell * nn) return;
    const long long e = t / nn;
    const int p = (int)(t - e * nn);
    // point order (xi slowest, zeta fastest) as meshgrid(pts, pts, pts, 'ij')
    const int i = p / (ng * ng), j = (p / ng) % ng, k = p % ng;
    const double xi = gx[i], eta = gx[j], zeta = gx[k];
    const double* X = corners + e * 24;
    double J[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int a = 0; a < 8; ++a) {
        const double ca = c_corner[a][0], cb = c_corner[a][1], cc = c_corner[a][2];
        const double fa = __dadd_rn(1.0, __dmul_rn(xi, ca));
        const double fb = __dadd_rn(1.0, __dmul_rn(eta, cb));
        const double fc = __dadd_rn(1.0, __dmul_rn(zeta, cc));
        const double dS[3] = {__dmul_rn(__dmul_rn(__dmul_rn(0.125, ca), fb), fc),
                              __dmul_rn(__dmul_rn(__dmul_rn(0.125, fa), cb), fc),
                              __dmul_rn(__dmul_rn(__dmul_rn(0.125, fa), fb), cc)};
        for (int c = 0; c < 3; ++c) {
            const double xa = X[a * 3 + c];
            // J[m][c] = sum_a dS[a][m] x_a[c]  (J = dS.T @ corners, gll_geometry.py:173)
            for (int m = 0; m < 3; ++m) J[m][c] = __dadd_rn(J[m][c], __dmul_rn(dS[m], xa));
        }
    }
    // Coordinates: the same trilinear map evaluated one axis at a time
    // (along xi between corner pairs, then eta, then zeta).  On a cell face
    // the weights of the far corners are exactly 0 and 1, so a point shared
    // by two cells goes through the same rounded operations on the same
    // corner values in both: bit-identical coordinates, and the quantised
    // sort cannot split a shared node.  (The one-sum form S @ corners adds
    // the four face corners in a different order in each cell, and a point
    // whose copies differ in the last bit can round to two grid values.)
    const double lw[3] = {__dmul_rn(0.5, __dsub_rn(1.0, xi)), __dmul_rn(0.5, __dsub_rn(1.0, eta)),
                          __dmul_rn(0.5, __dsub_rn(1.0, zeta))};
    const double hw[3] = {__dmul_rn(0.5, __dadd_rn(1.0, xi)), __dmul_rn(0.5, __dadd_rn(1.0, eta)),
                          __dmul_rn(0.5, __dadd_rn(1.0, zeta))};
    // corner of (xi side, eta side, zeta side) in GMSH order
    const int cidx[2][2][2] = {{{0, 4}, {3, 7}}, {{1, 5}, {2, 6}}};
    for (int c = 0; c < 3; ++c) {
        double s[2];
        for (int kb = 0; kb < 2; ++kb) {
            double r[2];
            for (int jb = 0; jb < 2; ++jb)
                r[jb] = __dadd_rn(__dmul_rn(lw[0], X[cidx[0][jb][kb] * 3 + c]),
                                  __dmul_rn(hw[0], X[cidx[1][jb][kb] * 3 + c]));
            s[kb] = __dadd_rn(__dmul_rn(lw[1], r[0]), __dmul_rn(hw[1], r[1]));
        }
        coords[t * 3 + c] = __dadd_rn(__dmul_rn(lw[2], s[0]), __dmul_rn(hw[2], s[1]));
    }
    const double a = J[0][0], b = J[0][1], c = J[0][2];
    const double d = J[1][0], ee = J[1][1], f = J[1][2];
    const double g = J[2][0], h = J[2][1], ii = J[2][2];
    // cofactors, det and inverse (inv(J) raveled row-major)
    const double A = __dsub_rn(__dmul_rn(ee, ii), __dmul_rn(f, h));
    const double B = __dsub_rn(__dmul_rn(f, g), __dmul_rn(d, ii));
    const double C = __dsub_rn(__dmul_rn(d, h), __dmul_rn(ee, g));
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(a, A), __dmul_rn(b, B)), __dmul_rn(c, C));
    jac[t] = det;
    const double rdet = det > 0.0 ? __ddiv_rn(1.0, det) : 0.0;
    double* o = dxi + t * 9;
    o[0] = __dmul_rn(A, rdet);
    o[1] = __dmul_rn(__dsub_rn(__dmul_rn(c, h), __dmul_rn(b, ii)), rdet);
    o[2] = __dmul_rn(__dsub_rn(__dmul_rn(b, f), __dmul_rn(c, ee)), rdet);
    o[3] = __dmul_rn(B, rdet);
    o[4] = __dmul_rn(__dsub_rn(__dmul_rn(a, ii), __dmul_rn(c, g)), rdet);
    o[5] = __dmul_rn(__dsub_rn(__dmul_rn(c, d), __dmul_rn(a, f)), rdet);
    o[6] = __dmul_rn(C, rdet);
    o[7] = __dmul_rn(__dsub_rn(__dmul_rn(b, g), __dmul_rn(a, h)), rdet);
    o[8] = __dmul_rn(__dsub_rn(__dmul_rn(a, ee), __dmul_rn(b, d)), rdet);
    // mass = det J * (w_i w_j) w_k
    mass[t] = __dmul_rn(det, __dmul_rn(__dmul_rn(gw[i], gw[j]), gw[k]));
}

// ---------------------------------------------------------------------------
// node numbering: quantise, three stable radix passes, flag, scan, scatter
// ---------------------------------------------------------------------------

// per-block min/max of each axis -> part[block][6]
__global__ void extent_kernel(long long n, const double* __restrict__ xyz, double* __restrict__ part) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const double v = xyz[q * 3 + c];
            lo[c] = fmin(lo[c], v);
            hi[c] = fmax(hi[c], v);
        }
    __shared__ double s[6][256];
    for (int c = 0; c < 3; ++c) {
        s[c][threadIdx.x] = lo[c];
        s[3 + c][threadIdx.x] = hi[c];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 3; ++c) {
                s[c][threadIdx.x] = fmin(s[c][threadIdx.x], s[c][threadIdx.x + w]);
                s[3 + c][threadIdx.x] = fmax(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[blockIdx.x * 6 + threadIdx.x] = s[threadIdx.x][0];
}

// q[c][i] = rint(x_i[c] * scale) as int64 (partition.py: np.rint(flat * scale))
__global__ void quantise_kernel(long long n, const double* __restrict__ xyz, double scale, long long* __restrict__ q) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; ++c) q[c * n + i] = (long long)rint(__dmul_rn(xyz[i * 3 + c], scale));
}

__global__ void iota_kernel(long long n, int* __restrict__ v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int)i;
}

__global__ void gather_key_kernel(long long n, const long long* __restrict__ q, const int* __restrict__ perm,
                                  long long* __restrict__ key) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = q[perm[i]];
}

// 1 where the sorted point differs from its predecessor in any coordinate
__global__ void new_flag_kernel(long long n, const long long* __restrict__ q, const int* __restrict__ perm,
                                int* __restrict__ flag) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0) {
        flag[i] = 1;
        return;
    }
    const int a = perm[i], b = perm[i - 1];
    flag[i] = (q[a] != q[b] || q[n + a] != q[n + b] || q[2 * n + a] != q[2 * n + b]) ? 1 : 0;
}

__global__ void scatter_ids_kernel(long long n, const int* __restrict__ perm, const int* __restrict__ incl,
                                   int* __restrict__ ibool) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ibool[perm[i]] = incl[i] - 1;
}

// ---------------------------------------------------------------------------
// C-PML
// ---------------------------------------------------------------------------

enum { X_ONLY = 1, Y_ONLY = 2, Z_ONLY = 3, XY_ONLY = 4, XZ_ONLY = 5, YZ_ONLY = 6, XYZ = 7 };

struct CpmlParams {
    double bound[6];  // xmin xmax ymin ymax zmin zmax
    double width[6];  // same faces; 0 = no layer
    double f0, dt, log_r, tol;
};

// region from the cell's GLL centroid (pml_cpml.py:174-253)
__global__ void region_kernel(long long n_cell, int nn, const double* __restrict__ xyz,
                              const uint8_t* __restrict__ is_pml, CpmlParams P, int* __restrict__ region) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_cell) return;
    if (!is_pml[e]) {
        region[e] = 0;
        return;
    }
    bool act[3];
    for (int ax = 0; ax < 3; ++ax) {
        double s = 0.0;
        for (int p = 0; p < nn; ++p) s += xyz[(e * nn + p) * 3 + ax];
        const double ctr = s / nn;
        bool a = false;
        const double wlo = P.width[2 * ax], whi = P.width[2 * ax + 1];
        if (wlo > 0.0) a = a || ctr < __dadd_rn(__dadd_rn(P.bound[2 * ax], wlo), __dmul_rn(P.tol, wlo));
        if (whi > 0.0) a = a || ctr > __dsub_rn(__dsub_rn(P.bound[2 * ax + 1], whi), __dmul_rn(P.tol, whi));
        act[ax] = a;
    }
    int r = XYZ;
    if (act[0] && act[1] && !act[2]) r = XY_ONLY;
    else if (act[0] && !act[1] && act[2]) r = XZ_ONLY;
    else if (!act[0] && act[1] && act[2]) r = YZ_ONLY;
    else if (act[0] && !act[1] && !act[2]) r = X_ONLY;
    else if (!act[0] && act[1] && !act[2]) r = Y_ONLY;
    else if (!act[0] && !act[1] && act[2]) r = Z_ONLY;
    region[e] = r;
}

__device__ bool axis_active(int r, int ax) {
    switch (ax) {
        case 0: return r == X_ONLY || r == XY_ONLY || r == XZ_ONLY || r == XYZ;
        case 1: return r == Y_ONLY || r == XY_ONLY || r == YZ_ONLY || r == XYZ;
        default: return r == Z_ONLY || r == XZ_ONLY || r == YZ_ONLY || r == XYZ;
    }
}

// |x| < MIN_DISTANCE -> MIN_DISTANCE (pml_cpml.py _safe)
__device__ double safe(double x) { return fabs(x) < 1e-6 ? 1e-6 : x; }

// coef0, coef1, coef2 of the recursive convolution for b (pml_cpml.py:261-305)
__device__ void conv_coef(double b, double dt, double* o) {
    const double temp = exp(__dmul_rn(__dmul_rn(-0.5, b), dt));
    o[0] = __dmul_rn(temp, temp);
    if (fabs(b) >= 1e-6) {
        o[1] = __ddiv_rn(__dsub_rn(1.0, temp), b);
        o[2] = __dmul_rn(o[1], temp);
    } else {
        const double dt2 = __dmul_rn(dt, dt), dt3 = __dmul_rn(dt2, dt), dt4 = __dmul_rn(dt3, dt);
        const double b2 = __dmul_rn(b, b), b3 = __dmul_rn(b2, b);
        const double h = __dmul_rn(dt, 0.5);
        o[1] = __dadd_rn(h, __dsub_rn(__dadd_rn(__dmul_rn(__dmul_rn(-0.125, dt2), b),
                                                __dmul_rn(__dmul_rn(1.0 / 48.0, dt3), b2)),
                                      __dmul_rn(__dmul_rn(1.0 / 384.0, dt4), b3)));
        o[2] = __dadd_rn(h, __dsub_rn(__dadd_rn(__dmul_rn(__dmul_rn(-0.375, dt2), b),
                                                __dmul_rn(__dmul_rn(7.0 / 48.0, dt3), b2)),
                                      __dmul_rn(__dmul_rn(5.0 / 128.0, dt4), b3)));
    }
}

#define MUL __dmul_rn
#define ADD __dadd_rn
#define SUB __dsub_rn
#define DIV __ddiv_rn

// one thread per (cell, point): profiles, coef_alpha [9], abar [5]
__global__ void cpml_kernel(long long n_cell, int nn, const double* __restrict__ xyz, const int* __restrict__ region,
                            const double* __restrict__ vp, CpmlParams P, double* __restrict__ calpha,
                            double* __restrict__ abar) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cell * nn) return;
    const long long e = t / nn;
    const int r = region[e];
    double K[3] = {1.0, 1.0, 1.0}, d[3] = {0.0, 0.0, 0.0}, al[3] = {0.0, 0.0, 0.0};
    if (r != 0) {
        const double amax[3] = {MUL(MUL(M_PI, P.f0), 0.9), MUL(MUL(M_PI, P.f0), 1.0), MUL(MUL(M_PI, P.f0), 1.1)};
        // faces in order; a later face of the same axis overwrites (pml_cpml.py:42-147)
        for (int f = 0; f < 6; ++f) {
            const int ax = f / 2;
            const double width = P.width[f];
            if (!(width > 0.0) || !axis_active(r, ax)) continue;
            const double dist = fmin(fmax(DIV(fabs(SUB(xyz[t * 3 + ax], P.bound[f])), width), 0.0), 1.0);
            double Kv = ADD(1.0, MUL(SUB(1.0, 1.0), dist));  // K_MIN + (K_MAX - 1) dist, K_MIN = K_MAX = 1
            // -((n + 1) vp ln R / (2 width)) dist^(1.2 n), n = 2
            double dv = MUL(-DIV(MUL(MUL(3.0, vp[t]), P.log_r), MUL(2.0, width)), pow(dist, 1.2 * 2.0));
            double av = MUL(amax[ax], SUB(1.0, dist));
            if (Kv < 1.0 || dv < 0.0) {
                Kv = 1.0;
                dv = 0.0;
            }
            av = fmax(av, 0.0);
            K[ax] = Kv;
            d[ax] = dv;
            al[ax] = av;
        }
    }
    double* ca = calpha + t * 9;
    for (int ax = 0; ax < 3; ++ax) conv_coef(r != 0 ? al[ax] : 0.0, P.dt, ca + ax * 3);
    double* o = abar + t * 5;
    if (r == 0) {
        for (int c = 0; c < 5; ++c) o[c] = 0.0;
        return;
    }
    const double kx = K[0], ky = K[1], kz = K[2];
    const double ax = al[0], ay = al[1], az = al[2];
    const double bx = ADD(ax, DIV(d[0], fmax(kx, 1.0)));
    const double by = ADD(ay, DIV(d[1], fmax(ky, 1.0)));
    const double bz = ADD(az, DIV(d[2], fmax(kz, 1.0)));
    double A0, A1, A2, A3 = 0.0, A4 = 0.0, A5 = 0.0;
    // A1..A5 per region (pml_cpml.py:353-515); products evaluated left to right
    switch (r) {
        case XYZ:
            A0 = MUL(MUL(kx, ky), kz);
            A1 = MUL(A0, SUB(SUB(SUB(ADD(ADD(bx, by), bz), ax), ay), az));
            A2 = ADD(ADD(MUL(MUL(A0, SUB(bx, ax)), SUB(SUB(by, ay), ax)), MUL(MUL(A0, SUB(by, ay)), SUB(SUB(bz, az), ay))),
                     MUL(MUL(A0, SUB(bz, az)), SUB(SUB(bx, ax), az)));
            A3 = DIV(MUL(MUL(MUL(MUL(A0, MUL(ax, ax)), SUB(bx, ax)), SUB(by, ax)), SUB(bz, ax)),
                     MUL(safe(SUB(ay, ax)), safe(SUB(az, ax))));
            A4 = DIV(MUL(MUL(MUL(MUL(A0, MUL(ay, ay)), SUB(bx, ay)), SUB(by, ay)), SUB(bz, ay)),
                     MUL(safe(SUB(ax, ay)), safe(SUB(az, ay))));
            A5 = DIV(MUL(MUL(MUL(MUL(A0, MUL(az, az)), SUB(bx, az)), SUB(by, az)), SUB(bz, az)),
                     MUL(safe(SUB(ay, az)), safe(SUB(az, ax))));
            break;
        case XY_ONLY:
            A0 = MUL(kx, ky);
            A1 = MUL(A0, SUB(SUB(ADD(bx, by), ax), ay));
            A2 = SUB(MUL(MUL(A0, SUB(bx, ax)), SUB(SUB(by, ay), ax)), MUL(MUL(A0, SUB(by, ay)), ay));
            A3 = DIV(MUL(MUL(MUL(A0, MUL(ax, ax)), SUB(bx, ax)), SUB(by, ax)), safe(SUB(ay, ax)));
            A4 = DIV(MUL(MUL(MUL(A0, MUL(ay, ay)), SUB(bx, ay)), SUB(by, ay)), safe(SUB(ax, ay)));
            break;
        case XZ_ONLY:
            A0 = MUL(kx, kz);
            A1 = MUL(A0, SUB(SUB(ADD(bx, bz), ax), az));
            A2 = ADD(MUL(MUL(A0, SUB(bx, ax)), -ax), MUL(MUL(A0, SUB(bz, az)), SUB(SUB(bx, ax), az)));
            A3 = DIV(MUL(MUL(MUL(A0, MUL(ax, ax)), SUB(bx, ax)), SUB(bz, ax)), safe(SUB(az, ax)));
            A5 = DIV(MUL(MUL(MUL(A0, MUL(az, az)), SUB(bx, az)), SUB(bz, az)), safe(SUB(ax, az)));
            break;
        case YZ_ONLY:
            A0 = MUL(ky, kz);
            A1 = MUL(A0, SUB(SUB(ADD(by, bz), ay), az));
            A2 = SUB(MUL(MUL(A0, SUB(by, ay)), SUB(SUB(bz, az), ay)), MUL(MUL(A0, SUB(bz, az)), az));
            A4 = DIV(MUL(MUL(MUL(A0, MUL(ay, ay)), SUB(by, ay)), SUB(bz, ay)), safe(SUB(az, ay)));
            A5 = DIV(MUL(MUL(MUL(A0, MUL(az, az)), SUB(by, az)), SUB(bz, az)), safe(SUB(ay, az)));
            break;
        case X_ONLY: {
            const double diff = SUB(bx, ax);
            A1 = MUL(kx, diff);
            A2 = MUL(MUL(-kx, ax), diff);
            A3 = MUL(MUL(kx, MUL(ax, ax)), diff);
            break;
        }
        case Y_ONLY: {
            const double diff = SUB(by, ay);
            A1 = MUL(ky, diff);
            A2 = MUL(MUL(-ky, ay), diff);
            A4 = MUL(MUL(ky, MUL(ay, ay)), diff);
            break;
        }
        default: {  // Z_ONLY
            const double diff = SUB(bz, az);
            A1 = MUL(kz, diff);
            A2 = MUL(MUL(-kz, az), diff);
            A5 = MUL(MUL(kz, MUL(az, az)), diff);
            break;
        }
    }
    o[0] = A1;
    o[1] = A2;
    o[2] = A3;
    o[3] = A4;
    o[4] = A5;
}

#undef MUL
#undef ADD
#undef SUB
#undef DIV

// cells per chunk of the per-cell kernels: device memory stays bounded
// whatever the mesh size
constexpr long long kChunkCells = 1 << 18;

}  // namespace

extern "C" {

gfb_status gfb_prep_geometry(int32_t device, int64_t n_cell, int32_t ngll, const double* gll_x, const double* gll_w,
                             const double* corners, double* coords, double* jacobian, double* dxi_dx,
                             double* mass_geo) {
    if (n_cell < 0 || ngll < 2 || ngll > 10 || !gll_x || !gll_w || (n_cell > 0 && !corners))
        return prep_fail(GFB_ERR_INVALID, "invalid geometry arguments");
    if (!coords || !jacobian || !dxi_dx || !mass_geo) return prep_fail(GFB_ERR_INVALID, "NULL output array");
    gfb_status st;
    if ((st = open_device(device))) return st;
    if (n_cell == 0) return GFB_OK;
    const int nn = ngll * ngll * ngll;
    const long long chunk = std::min<long long>(kChunkCells, n_cell);
    Scratch S;
    double *gx, *gw, *dc, *dx, *dj, *dd, *dm;
    PCU(S.alloc(&gx, ngll));
    PCU(S.alloc(&gw, ngll));
    PCU(S.alloc(&dc, (size_t)chunk * 24));
    PCU(S.alloc(&dx, (size_t)chunk * nn * 3));
    PCU(S.alloc(&dj, (size_t)chunk * nn));
    PCU(S.alloc(&dd, (size_t)chunk * nn * 9));
    PCU(S.alloc(&dm, (size_t)chunk * nn));
    PCU(cudaMemcpy(gx, gll_x, ngll * sizeof(double), cudaMemcpyHostToDevice));
    PCU(cudaMemcpy(gw, gll_w, ngll * sizeof(double), cudaMemcpyHostToDevice));
    for (long long e0 = 0; e0 < n_cell; e0 += chunk) {
        const long long ne = std::min(chunk, n_cell - e0);
        const long long np = ne * nn;
        PCU(cudaMemcpy(dc, corners + e0 * 24, (size_t)ne * 24 * sizeof(double), cudaMemcpyHostToDevice));
        geometry_kernel<<<blocks_for(np, 256), 256>>>(ne, ngll, gx, gw, dc, dx, dj, dd, dm);
        PCU(cudaGetLastError());
        PCU(cudaMemcpy(coords + e0 * nn * 3, dx, (size_t)np * 3 * sizeof(double), cudaMemcpyDeviceToHost));
        PCU(cudaMemcpy(jacobian + e0 * nn, dj, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost));
        PCU(cudaMemcpy(dxi_dx + e0 * nn * 9, dd, (size_t)np * 9 * sizeof(double), cudaMemcpyDeviceToHost));
        PCU(cudaMemcpy(mass_geo + e0 * nn, dm, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return GFB_OK;
}

gfb_status gfb_prep_numbering(int32_t device, int64_t n_point, const double* coords, int32_t* ibool,
                              int32_t* n_node) {
    if (n_point < 0 || (n_point > 0 && (!coords || !ibool)) || !n_node)
        return prep_fail(GFB_ERR_INVALID, "invalid numbering arguments");
    if (n_point >= (1LL << 31)) return prep_fail(GFB_ERR_UNSUPPORTED, "more than 2^31-1 points");
    gfb_status st;
    if ((st = open_device(device))) return st;
    *n_node = 0;
    if (n_point == 0) return GFB_OK;
    const long long n = n_point;
    Scratch S;
    double *xyz, *part;
    long long *q, *key, *key2;
    int *perm, *perm2, *flag, *incl, *ib;
    const int nb = 4 * 148;
    PCU(S.alloc(&xyz, (size_t)n * 3));
    PCU(S.alloc(&part, (size_t)nb * 6));
    PCU(S.alloc(&q, (size_t)n * 3));
    PCU(S.alloc(&key, (size_t)n));
    PCU(S.alloc(&key2, (size_t)n));
    PCU(S.alloc(&perm, (size_t)n));
    PCU(S.alloc(&perm2, (size_t)n));
    PCU(S.alloc(&flag, (size_t)n));
    PCU(S.alloc(&incl, (size_t)n));
    PCU(S.alloc(&ib, (size_t)n));
    PCU(cudaMemcpy(xyz, coords, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice));
    // extent = max over axes of (max - min), at least machine epsilon
    extent_kernel<<<nb, 256>>>(n, xyz, part);
    PCU(cudaGetLastError());
    std::vector<double> hp((size_t)nb * 6);
    PCU(cudaMemcpy(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = 0; b < nb; ++b)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], hp[b * 6 + c]);
            hi[c] = std::max(hi[c], hp[b * 6 + 3 + c]);
        }
    double extent = 2.220446049250313e-16;
    for (int c = 0; c < 3; ++c) extent = std::max(extent, hi[c] - lo[c]);
    const double tol = 1e-12 * extent;
    const double scale = 1.0 / tol;
    const unsigned g = blocks_for(n, 256);
    quantise_kernel<<<g, 256>>>(n, xyz, scale, q);
    PCU(cudaGetLastError());
    iota_kernel<<<g, 256>>>(n, perm);
    PCU(cudaGetLastError());
    // lexicographic order (x, then y, then z): stable passes by z, y, x
    size_t temp_bytes = 0;
    PCU(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, key, key2, perm, perm2, (int)n));
    void* temp = nullptr;
    PCU(S.alloc(reinterpret_cast<unsigned char**>(&temp), temp_bytes));
    for (int c = 2; c >= 0; --c) {
        gather_key_kernel<<<g, 256>>>(n, q + (size_t)c * n, perm, key);
        PCU(cudaGetLastError());
        PCU(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, key, key2, perm, perm2, (int)n));
        std::swap(perm, perm2);
    }
    new_flag_kernel<<<g, 256>>>(n, q, perm, flag);
    PCU(cudaGetLastError());
    size_t scan_bytes = 0;
    PCU(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, flag, incl, (int)n));
    void* scan_temp = nullptr;
    PCU(S.alloc(reinterpret_cast<unsigned char**>(&scan_temp), scan_bytes));
    PCU(cub::DeviceScan::InclusiveSum(scan_temp, scan_bytes, flag, incl, (int)n));
    scatter_ids_kernel<<<g, 256>>>(n, perm, incl, ib);
    PCU(cudaGetLastError());
    int last = 0;
    PCU(cudaMemcpy(&last, incl + (n - 1), sizeof(int), cudaMemcpyDeviceToHost));
    PCU(cudaMemcpy(ibool, ib, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    *n_node = last;
    return GFB_OK;
}

gfb_status gfb_prep_cpml(int32_t device, int64_t n_cell, int32_t ngll, const double* coords, const uint8_t* is_pml,
                         const double* vp, const double* bounds, const double* widths, double f0, double dt,
                         double log_r, int32_t* region, double* coef_alpha, double* abar) {
    if (n_cell < 0 || ngll < 2 || ngll > 10 || !bounds || !widths || !region || !coef_alpha || !abar ||
        (n_cell > 0 && (!coords || !is_pml || !vp)))
        return prep_fail(GFB_ERR_INVALID, "invalid C-PML arguments");
    gfb_status st;
    if ((st = open_device(device))) return st;
    if (n_cell == 0) return GFB_OK;
    const int nn = ngll * ngll * ngll;
    CpmlParams P;
    for (int f = 0; f < 6; ++f) {
        P.bound[f] = bounds[f];
        P.width[f] = widths[f];
    }
    P.f0 = f0;
    P.dt = dt;
    P.log_r = log_r;
    P.tol = 1e-6;
    const long long chunk = std::min<long long>(kChunkCells, n_cell);
    Scratch S;
    double *xyz, *dv, *dca, *dab;
    uint8_t* dpml;
    int* dreg;
    PCU(S.alloc(&xyz, (size_t)chunk * nn * 3));
    PCU(S.alloc(&dv, (size_t)chunk * nn));
    PCU(S.alloc(&dca, (size_t)chunk * nn * 9));
    PCU(S.alloc(&dab, (size_t)chunk * nn * 5));
    PCU(S.alloc(&dpml, (size_t)chunk));
    PCU(S.alloc(&dreg, (size_t)chunk));
    for (long long e0 = 0; e0 < n_cell; e0 += chunk) {
        const long long ne = std::min(chunk, n_cell - e0);
        const long long np = ne * nn;
        PCU(cudaMemcpy(xyz, coords + e0 * nn * 3, (size_t)np * 3 * sizeof(double), cudaMemcpyHostToDevice));
        PCU(cudaMemcpy(dv, vp + e0 * nn, (size_t)np * sizeof(double), cudaMemcpyHostToDevice));
        PCU(cudaMemcpy(dpml, is_pml + e0, (size_t)ne, cudaMemcpyHostToDevice));
        region_kernel<<<blocks_for(ne, 128), 128>>>(ne, nn, xyz, dpml, P, dreg);
        PCU(cudaGetLastError());
        cpml_kernel<<<blocks_for(np, 256), 256>>>(ne, nn, xyz, dreg, dv, P, dca, dab);
        PCU(cudaGetLastError());
        PCU(cudaMemcpy(region + e0, dreg, (size_t)ne * sizeof(int32_t), cudaMemcpyDeviceToHost));
        PCU(cudaMemcpy(coef_alpha + e0 * nn * 9, dca, (size_t)np * 9 * sizeof(double), cudaMemcpyDeviceToHost));
        PCU(cudaMemcpy(abar + e0 * nn * 5, dab, (size_t)np * 5 * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return GFB_OK;
}

}  // extern "C"
