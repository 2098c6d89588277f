// gfb_layer.cu -- learned absorbing layer: a small per-boundary-node network
// that adds a force correction on the nodes of a thin (one-element) C-PML
// layer so that the truncated domain behaves like the same domain with a
// thick C-PML, its training data (replay of a thick-C-PML run) and its
// training.  No counterpart in the reference, which only has C-PML
// (forward/share/src/pml.cpp) and the legacy damping layer.
//
// Network, per node and wavefield (one network per depth class "net"):
//   x  = 9 channels (u, v, a in the node's face frame, each channel divided
//        by its scale) x 4 time taps (the states of steps n-1 .. n-4),
//        normalised to unit length: xh = x / |x|
//   h1 = relu(+-W1 xh), h2 = relu(W2 h1), y = W3 h2     (no biases)
//   sigma_j = softplus((y_j(+xh) + y_j(-xh)) / 2)
//   correction_j = -(s_c / s_v) sigma_j v_j   (face frame; v_j the velocity
//                  at the end of the step, the damping taken implicitly)
// The network predicts damping coefficients of a dashpot on each face axis
// (a learned, history-dependent generalisation of a viscous absorbing
// boundary): the correction only takes energy out and adds no stiffness, so
// the explicit step stays stable; sigma depends on the shape of the recent
// history, not its size, so the correction is linear in the wavefield's
// amplitude like the exact absorbing operator.  sigma is capped at m / dt.
// Weights are BF16; inference runs on the tensor cores (mma.sync m16n8k16,
// FP32 accumulate); training keeps FP32 master weights, rounds them to BF16
// for its forward/backward pass and runs on the CUDA cores.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/gfb.h"
#include "gfb_internal.h"
#include "gfb_kernels.cuh"

namespace gfb {

constexpr int kIn = GFB_LAYER_NIN;    // 36
constexpr int kHid = GFB_LAYER_NHID;  // 64
constexpr int kOut = GFB_LAYER_NOUT;  // 3
constexpr int kTaps = 4;
// BF16 inference layout of one network, rows padded for conflict-free
// 32-bit fragment loads from shared memory:
//   W1 [64][56] (k = 0..35 used), W2 [64][72], W3 [8][72] (rows 0..2 used)
constexpr int kW1S = 56, kW2S = 72, kW3S = 72;
constexpr int kW1 = 0, kW2 = kW1 + kHid * kW1S, kW3 = kW2 + kHid * kW2S, kWNet = kW3 + 8 * kW3S;
static_assert(kWNet == GFB_LAYER_WEIGHTS, "weight layout");
// FP32 master layout of one network: W1 [64][36], W2 [64][64], W3 [3][64]
constexpr int kM1 = 0, kM2 = kHid * kIn, kM3 = kM2 + kHid * kHid, kMNet = kM3 + kOut * kHid;
static_assert(kMNet == GFB_LAYER_PARAMS, "parameter layout");

#define LCU(call)                                                                              \
    do {                                                                                       \
        cudaError_t _e = (call);                                                               \
        if (_e != cudaSuccess) {                                                               \
            std::string _m = std::string(#call) + ": " + cudaGetErrorString(_e);               \
            return set_error(_e == cudaErrorMemoryAllocation ? GFB_ERR_NOMEM : GFB_ERR_CUDA,   \
                             _m.c_str());                                                      \
        }                                                                                      \
    } while (0)

// ---------------------------------------------------------------------------
// boundary nodes and their features
// ---------------------------------------------------------------------------

// One boundary node: device node, network, local frame.  frame[j] in
// {+-1, +-2, +-3}: local axis j is global axis |frame[j]|-1, with its sign.
struct BNode {
    int node;
    int net;
    int frame;  // 3 signed 4-bit fields
    int pad;
};

__host__ __device__ inline int frame_axis(int frame, int j) {
    const int f = ((frame >> (4 * j)) & 0xf) - 8;
    return (f < 0 ? -f : f) - 1;
}
__host__ __device__ inline float frame_sign(int frame, int j) { return (((frame >> (4 * j)) & 0xf) - 8) < 0 ? -1.f : 1.f; }
// v[ax] for a runtime axis, by selects (an indexed load would put the
// array in local memory)
__device__ inline float pick3(const float* v, int ax) { return ax == 0 ? v[0] : (ax == 1 ? v[1] : v[2]); }

// History of the boundary nodes: ring[slot][b][field][9] global-frame
// (u, v, a) of one step; state m lives in slot m % 3.
struct History {
    float* ring = nullptr;
};

// Features of sample (b, field) at step n (arrays hold the state of n-1;
// the ring holds n-2 .. n-4) into x[36] (face frame, scaled by sc[0..2]),
// and the state of n-1 in global frame into cur[9].
__device__ inline void node_features(const BNode& bn, int f, int NF, long long n, const double* u, const double* v,
                                     const float* a, const float* ring, long long n_bnd, int b, const float* sc,
                                     float* x, float* cur) {
    const long long g = bn.node;
    const int F = 3 * NF;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        cur[c] = (float)u[g * F + f * 3 + c];
        cur[3 + c] = (float)v[g * F + f * 3 + c];
        cur[6 + c] = a[g * F + f * 3 + c];
    }
#pragma unroll
    for (int tap = 0; tap < kTaps; ++tap) {
        float val[9];
        if (tap == 0) {
#pragma unroll
            for (int q = 0; q < 9; ++q) val[q] = cur[q];
        } else {
            const long long m = n - 1 - tap;
            if (m < 0) {
#pragma unroll
                for (int q = 0; q < 9; ++q) val[q] = 0.f;
            } else {
                const float* r = ring + ((size_t)(m % 3) * n_bnd + b) * NF * 9 + f * 9;
#pragma unroll
                for (int q = 0; q < 9; ++q) val[q] = r[q];
            }
        }
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                x[tap * 9 + ch * 3 + j] = frame_sign(bn.frame, j) * pick3(val + ch * 3, frame_axis(bn.frame, j)) / sc[ch];
    }
}

// ---------------------------------------------------------------------------
// inference (time loop): persistent warps over tiles of 16 samples of one
// network; all networks' BF16 weights in shared memory
// ---------------------------------------------------------------------------

struct LayerArgs {
    const BNode* bnd;
    long long n_bnd;
    const int* tile_net;      // [n_tile]
    const int* tile_sample;   // [n_tile][16]: b * NF + field, or -1
    int n_tile;
    int n_net;
    const __nv_bfloat16* w;   // [n_net][kWNet]
    float sc[4];              // channel scales u, v, a; output scale
    const float* gain;        // [n_net][3] damping gain per network and face axis
    const double* u;
    const double* v;
    const float* a;
    float* force;             // [node][NF][4]
    const double* mass;
    float* ring;
    const int* mstep;         // next step index (device counter); this step is mstep - 1
    double dt;
    double* acc;              // [2 parity][2]: work of the correction, boundary kinetic energy
    double* monitor;          // [0] residual (running mean), [1] steps seen, [2] steps above threshold in a row
    int* active;              // 1 while the correction is applied
    double threshold;
};

__device__ inline uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 t = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&t);
}

__device__ inline void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Warps per block of layer_kernel: every block stages all networks' weights
// in shared memory once (up to ~180 KB: one block per SM), so the warps of
// one block are all the warps an SM gets; 12 x 32 threads at ~160 registers
// fill the register file (the feature gathers need the warps).
constexpr int kLayerWarps = 12;

template <int NF>
__global__ void __launch_bounds__(kLayerWarps * 32) layer_kernel(LayerArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(smem_raw);                  // [n_net][kWNet]
    __nv_bfloat16* sx = sw + (size_t)A.n_net * kWNet;                                 // [warps][16][56]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const uint4* src = reinterpret_cast<const uint4*>(A.w);
        uint4* dst = reinterpret_cast<uint4*>(sw);
        const int n16 = A.n_net * kWNet * 2 / 16;
        for (int q = tid; q < n16; q += blockDim.x) dst[q] = src[q];
    }
    const long long n = (long long)__ldg(A.mstep) - 1;  // the step being computed
    const int par = (int)(n & 1);
    // monitor: the previous step's work and energy (parity of n-1), read and
    // cleared by one thread; blocks of this step accumulate into parity n
    if (blockIdx.x == 0 && tid == 0 && n > 0) {
        double* pa = A.acc + (1 - par) * 2;
        const double work = pa[0], ekin = pa[1];
        pa[0] = 0.0;
        pa[1] = 0.0;
        if (*A.active) {
            // residual of the step: energy put in by the correction relative
            // to the kinetic energy of the layer nodes; off for good after 3
            // steps in a row above the threshold, or at once on a non-finite
            // value or a residual 100 times the threshold
            const double r = (ekin > 0.0) ? work / ekin : 0.0;
            const double k = A.monitor[1] + 1.0;
            A.monitor[0] += (r - A.monitor[0]) / fmin(k, 50.0);  // running mean over <= 50 steps (reported)
            A.monitor[1] = k;
            A.monitor[2] = (r > A.threshold) ? A.monitor[2] + 1.0 : 0.0;
            if (!isfinite(work) || !isfinite(ekin) || A.monitor[2] >= 3.0 || r > 100.0 * A.threshold) *A.active = 0;
        }
    }
    __syncthreads();
    const bool on = *((volatile int*)A.active) != 0;
    __nv_bfloat16* xs = sx + warp * 16 * kW1S;
    double work = 0.0, ekin = 0.0;
    for (int t = blockIdx.x * kLayerWarps + warp; t < A.n_tile; t += gridDim.x * kLayerWarps) {
        const int net = A.tile_net[t];
        const __nv_bfloat16* W = sw + (size_t)net * kWNet;
        // features: lane -> (row lane/2, half lane%2) ... two lanes per sample
        const int row = lane >> 1, half = lane & 1;
        const int smp = A.tile_sample[t * 16 + row];
        float x[kIn], cur[9];
        BNode bn{};
        int b = -1, f = 0;
        if (smp >= 0) {
            b = smp / NF;
            f = smp - b * NF;
            bn = A.bnd[b];
            node_features(bn, f, NF, n, A.u, A.v, A.a, A.ring, A.n_bnd, b, A.sc, x, cur);
            float nrm = 0.f;
#pragma unroll
            for (int q = 0; q < kIn; ++q) nrm += x[q] * x[q];
            const float inv = nrm > 0.f ? rsqrtf(nrm) : 0.f;
#pragma unroll
            for (int q = 0; q < kIn; ++q) x[q] *= inv;
        } else {
#pragma unroll
            for (int q = 0; q < kIn; ++q) x[q] = 0.f;
#pragma unroll
            for (int q = 0; q < 9; ++q) cur[q] = 0.f;
        }
        // half 0 writes k = 0..27, half 1 writes k = 28..55 (zero padding);
        // both x indices are compile-time, so x stays in registers
#pragma unroll
        for (int q = 0; q < 28; ++q) {
            const float hi = q + 28 < kIn ? x[q + 28 < kIn ? q + 28 : 0] : 0.f;
            xs[row * kW1S + half * 28 + q] = __float2bfloat16_rn(half ? hi : x[q]);
        }
        __syncwarp();
        const int r0 = lane >> 2, c0 = 2 * (lane & 3);
        // layer 1: z1 [16 x 64] = X [16 x 48] . W1^T
        float z[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) z[j][0] = z[j][1] = z[j][2] = z[j][3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 3; ++ks) {
            const uint32_t a0 = *reinterpret_cast<const uint32_t*>(xs + r0 * kW1S + ks * 16 + c0);
            const uint32_t a1 = *reinterpret_cast<const uint32_t*>(xs + (r0 + 8) * kW1S + ks * 16 + c0);
            const uint32_t a2 = *reinterpret_cast<const uint32_t*>(xs + r0 * kW1S + ks * 16 + c0 + 8);
            const uint32_t a3 = *reinterpret_cast<const uint32_t*>(xs + (r0 + 8) * kW1S + ks * 16 + c0 + 8);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const __nv_bfloat16* wr = W + kW1 + (8 * j + r0) * kW1S + ks * 16 + c0;
                mma_bf16(z[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wr),
                         *reinterpret_cast<const uint32_t*>(wr + 8));
            }
        }
        __syncwarp();
        // layers 2 and 3 for +x and -x
        float y[2][4];
#pragma unroll
        for (int br = 0; br < 2; ++br) {
            const float sg = br == 0 ? 1.f : -1.f;
            float h[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) h[j][0] = h[j][1] = h[j][2] = h[j][3] = 0.f;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint32_t a0 = pack_bf16(fmaxf(sg * z[2 * ks][0], 0.f), fmaxf(sg * z[2 * ks][1], 0.f));
                const uint32_t a1 = pack_bf16(fmaxf(sg * z[2 * ks][2], 0.f), fmaxf(sg * z[2 * ks][3], 0.f));
                const uint32_t a2 = pack_bf16(fmaxf(sg * z[2 * ks + 1][0], 0.f), fmaxf(sg * z[2 * ks + 1][1], 0.f));
                const uint32_t a3 = pack_bf16(fmaxf(sg * z[2 * ks + 1][2], 0.f), fmaxf(sg * z[2 * ks + 1][3], 0.f));
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const __nv_bfloat16* wr = W + kW2 + (8 * j + r0) * kW2S + ks * 16 + c0;
                    mma_bf16(h[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wr),
                             *reinterpret_cast<const uint32_t*>(wr + 8));
                }
            }
            y[br][0] = y[br][1] = y[br][2] = y[br][3] = 0.f;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint32_t a0 = pack_bf16(fmaxf(h[2 * ks][0], 0.f), fmaxf(h[2 * ks][1], 0.f));
                const uint32_t a1 = pack_bf16(fmaxf(h[2 * ks][2], 0.f), fmaxf(h[2 * ks][3], 0.f));
                const uint32_t a2 = pack_bf16(fmaxf(h[2 * ks + 1][0], 0.f), fmaxf(h[2 * ks + 1][1], 0.f));
                const uint32_t a3 = pack_bf16(fmaxf(h[2 * ks + 1][2], 0.f), fmaxf(h[2 * ks + 1][3], 0.f));
                const __nv_bfloat16* wr = W + kW3 + r0 * kW3S + ks * 16 + c0;
                mma_bf16(y[br], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(wr),
                         *reinterpret_cast<const uint32_t*>(wr + 8));
            }
        }
        // outputs: lane holds columns c0, c0+1 of rows r0 (y[.][0..1]) and
        // r0+8 (y[.][2..3]); columns 0..2 are the face-frame damping logits
        float sig[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float fz = 0.5f * (y[0][q] + y[1][q]);
            sig[q] = fz > 20.f ? fz : log1pf(__expf(fz));  // softplus
        }
        // gather the three columns of each row in lanes with lane%4 == 0
        const float s2a = __shfl_down_sync(0xffffffffu, sig[0], 1);  // column 2 of row r0
        const float s2b = __shfl_down_sync(0xffffffffu, sig[2], 1);  // column 2 of row r0+8
        const float gain = A.sc[3] / A.sc[1];
#pragma unroll
        for (int rr = 0; rr < 2; ++rr) {
            const int orow = r0 + 8 * rr;
            // the state of row orow lives in lane 2*orow (half 0)
            float cv[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) cv[q] = __shfl_sync(0xffffffffu, cur[q], 2 * orow);
            const int osmp = __shfl_sync(0xffffffffu, smp, 2 * orow);
            const int oframe = __shfl_sync(0xffffffffu, bn.frame, 2 * orow);
            const int onode = __shfl_sync(0xffffffffu, bn.node, 2 * orow);
            if ((lane & 3) == 0 && osmp >= 0) {
                const float sl[3] = {rr == 0 ? sig[0] : sig[2], rr == 0 ? sig[1] : sig[3], rr == 0 ? s2a : s2b};
                const double m = A.mass[onode];
                const float cap = (float)(m / A.dt);
                const int of = osmp % NF;
                float4* dst = reinterpret_cast<float4*>(A.force) + (size_t)onode * NF + of;
                float4 fo = *dst;
                const float fe[3] = {fo.x, fo.y, fo.z};
                const float hdm = (float)(0.5 * A.dt / m);
                float gc[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int ax = frame_axis(oframe, j);
                    // non-finite stays non-finite (the monitor's signal)
                    float dj = gain * __ldg(A.gain + net * 3 + j) * sl[j];
                    if (isfinite(dj)) dj = fminf(dj, cap);
                    // trapezoidal dashpot: velocity at the end of the step
                    // estimated from this step's force, the damping taken
                    // implicitly, so any sigma >= 0 stays stable
                    const float vbar = pick3(cv + 3, ax) + (float)(0.5 * A.dt) * pick3(cv + 6, ax) + hdm * pick3(fe, ax);
                    const float gj = -dj * vbar / (1.f + dj * hdm);
                    gc[0] = ax == 0 ? gj : gc[0];
                    gc[1] = ax == 1 ? gj : gc[1];
                    gc[2] = ax == 2 ? gj : gc[2];
                }
                const bool fin = isfinite(gc[0]) && isfinite(gc[1]) && isfinite(gc[2]);
                if (on && fin) {
                    fo.x += gc[0];
                    fo.y += gc[1];
                    fo.z += gc[2];
                    *dst = fo;
                }
                // work of the correction over the step and kinetic energy
                work += fin ? A.dt * ((double)gc[0] * cv[3] + (double)gc[1] * cv[4] + (double)gc[2] * cv[5])
                            : nan("");
                ekin += 0.5 * m * ((double)cv[3] * cv[3] + (double)cv[4] * cv[4] + (double)cv[5] * cv[5]);
            }
        }
        // push the state of step n-1 into the ring (half 0 lanes own a sample)
        if (smp >= 0 && half == 0) {
            float* r = A.ring + ((size_t)((n - 1) % 3 + 3) % 3 * A.n_bnd + b) * NF * 9 + f * 9;
            if (n >= 1)
#pragma unroll
                for (int q = 0; q < 9; ++q) r[q] = cur[q];
        }
        __syncwarp();
    }
    // block sums of the monitor terms
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        work += __shfl_down_sync(0xffffffffu, work, o);
        ekin += __shfl_down_sync(0xffffffffu, ekin, o);
    }
    if (lane == 0) {
        atomicAdd(A.acc + par * 2 + 0, work);
        atomicAdd(A.acc + par * 2 + 1, ekin);
    }
}

// ---------------------------------------------------------------------------
// the layer object attached to a solver
// ---------------------------------------------------------------------------

struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    gfb_status alloc(T** out, size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess)
            return set_error(GFB_ERR_NOMEM, "learned layer: cudaMalloc failed");
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return GFB_OK;
    }
};

// Boundary nodes (device numbering), tiles of 16 samples of one network.
struct Boundary {
    long long n_bnd = 0;
    int n_net = 0, n_tile = 0, nf = 1;
    BNode* bnd = nullptr;
    int* tile_net = nullptr;
    int* tile_sample = nullptr;
    float* ring = nullptr;
    std::vector<BNode> host;
};

gfb_status build_boundary(const SolverView& v, const gfb_layer* L, DevMem& mem, Boundary& B) {
    if (!L || L->n_node <= 0 || !L->node || !L->frame || !L->net || L->n_net < 1 || L->n_net > 64)
        return set_error(GFB_ERR_INVALID, "learned layer: bad layer description");
    B.n_bnd = L->n_node;
    B.n_net = L->n_net;
    B.nf = v.n_field;
    B.host.resize(L->n_node);
    std::vector<std::vector<int>> per_net(L->n_net);
    for (int i = 0; i < L->n_node; ++i) {
        const int g = L->node[i];
        if (g < 0 || g >= v.n_node) return set_error(GFB_ERR_INVALID, "learned layer: node id out of range");
        if (L->net[i] >= L->n_net) return set_error(GFB_ERR_INVALID, "learned layer: network index out of range");
        int fr = 0, seen = 0;
        for (int j = 0; j < 3; ++j) {
            const int f = L->frame[i * 3 + j];
            if (f == 0 || f < -3 || f > 3) return set_error(GFB_ERR_INVALID, "learned layer: bad frame");
            seen |= 1 << ((f < 0 ? -f : f) - 1);
            fr |= (f + 8) << (4 * j);
        }
        if (seen != 7) return set_error(GFB_ERR_INVALID, "learned layer: frame is not a permutation of the axes");
        const int d = v.node_inv->empty() ? g : (*v.node_inv)[g];
        B.host[i] = BNode{d, (int)L->net[i], fr, 0};
        for (int f = 0; f < v.n_field; ++f) per_net[L->net[i]].push_back(i * v.n_field + f);
    }
    std::vector<int> tn, ts;
    for (int k = 0; k < L->n_net; ++k) {
        const auto& sm = per_net[k];
        for (size_t q = 0; q < sm.size(); q += 16) {
            tn.push_back(k);
            for (size_t r = 0; r < 16; ++r) ts.push_back(q + r < sm.size() ? sm[q + r] : -1);
        }
    }
    B.n_tile = (int)tn.size();
    gfb_status st;
    if ((st = mem.alloc(&B.bnd, B.host.size()))) return st;
    if ((st = mem.alloc(&B.tile_net, tn.size()))) return st;
    if ((st = mem.alloc(&B.tile_sample, ts.size()))) return st;
    if ((st = mem.alloc(&B.ring, (size_t)3 * B.n_bnd * v.n_field * 9))) return st;
    LCU(cudaMemcpy(B.bnd, B.host.data(), B.host.size() * sizeof(BNode), cudaMemcpyHostToDevice));
    LCU(cudaMemcpy(B.tile_net, tn.data(), tn.size() * 4, cudaMemcpyHostToDevice));
    LCU(cudaMemcpy(B.tile_sample, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice));
    LCU(cudaMemset(B.ring, 0, (size_t)3 * B.n_bnd * v.n_field * 9 * sizeof(float)));
    return GFB_OK;
}

struct Layer {
    DevMem mem;
    Boundary B;
    __nv_bfloat16* w = nullptr;
    float sc[4] = {1.f, 1.f, 1.f, 1.f};
    float* gain = nullptr;      // [n_net][3]
    int n_net = 0;
    double* acc = nullptr;      // [4]
    double* monitor = nullptr;  // [3]
    int* active = nullptr;
    double threshold = 0.0;
    int blocks = 0;
    size_t smem = 0;
};

template <int NF>
gfb_status launch_layer(const SolverView& v, Layer* L) {
    LayerArgs A;
    A.bnd = L->B.bnd;
    A.n_bnd = L->B.n_bnd;
    A.tile_net = L->B.tile_net;
    A.tile_sample = L->B.tile_sample;
    A.n_tile = L->B.n_tile;
    A.n_net = L->B.n_net;
    A.w = L->w;
    for (int q = 0; q < 4; ++q) A.sc[q] = L->sc[q];
    A.gain = L->gain;
    A.u = v.u;
    A.v = v.v;
    A.a = static_cast<const float*>(v.a);
    A.force = static_cast<float*>(v.force);
    A.mass = v.mass;
    A.ring = L->B.ring;
    A.mstep = v.mstep;
    A.dt = v.dt;
    A.acc = L->acc;
    A.monitor = L->monitor;
    A.active = L->active;
    A.threshold = L->threshold;
    layer_kernel<NF><<<L->blocks, kLayerWarps * 32, L->smem, v.stream>>>(A);
    LCU(cudaGetLastError());
    return GFB_OK;
}

gfb_status layer_step(gfb_solver* s, Layer* L) {
    const SolverView v = solver_view(s);
    if (v.n_field == 1) return launch_layer<1>(v, L);
    if (v.n_field == 2) return launch_layer<2>(v, L);
    return launch_layer<3>(v, L);
}

void layer_free(Layer* L) { delete L; }

// Padded BF16 inference layout from FP32 master weights of one network.
void pack_weights(const float* m, __nv_bfloat16* w) {
    for (int q = 0; q < kWNet; ++q) w[q] = __float2bfloat16_rn(0.f);
    for (int n = 0; n < kHid; ++n)
        for (int k = 0; k < kIn; ++k) w[kW1 + n * kW1S + k] = __float2bfloat16_rn(m[kM1 + n * kIn + k]);
    for (int n = 0; n < kHid; ++n)
        for (int k = 0; k < kHid; ++k) w[kW2 + n * kW2S + k] = __float2bfloat16_rn(m[kM2 + n * kHid + k]);
    for (int n = 0; n < kOut; ++n)
        for (int k = 0; k < kHid; ++k) w[kW3 + n * kW3S + k] = __float2bfloat16_rn(m[kM3 + n * kHid + k]);
}

// ---------------------------------------------------------------------------
// training data: replay of a thick-C-PML run on the thin domain
// ---------------------------------------------------------------------------

// thin (u, v, a) <- thick (u, v, a) through the node map (device numbering)
__global__ void replay_gather_kernel(long long n_node, int F, const int* map, const double* tu, const double* tv,
                                     const float* ta, double* u, double* v, float* a) {
    const long long total = n_node * F;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long g = i / F;
        const int c = (int)(i - g * F);
        const long long h = (long long)map[g] * F + c;
        u[i] = tu[h];
        v[i] = tv[h];
        a[i] = ta[h];
    }
}

// features of step n for every (b, field) into stage[b][field][36]; push the
// state of n-1 into the ring
template <int NF>
__global__ void replay_features_kernel(const BNode* bnd, long long n_bnd, long long n, const double* u,
                                       const double* v, const float* a, float* ring, float* stage) {
    const float one[3] = {1.f, 1.f, 1.f};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_bnd * NF;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / NF), f = (int)(i - (long long)b * NF);
        float x[kIn], cur[9];
        const BNode bn = bnd[b];
        node_features(bn, f, NF, n, u, v, a, ring, n_bnd, b, one, x, cur);
        float* st = stage + i * kIn;
#pragma unroll
        for (int q = 0; q < kIn; ++q) st[q] = x[q];
        if (n >= 1) {
            float* r = ring + ((size_t)((n - 1) % 3) * n_bnd + b) * NF * 9 + f * 9;
#pragma unroll
            for (int q = 0; q < 9; ++q) r[q] = cur[q];
        }
    }
}

// target m (a_thick - a_thin) in face frame; append (x, t) of every
// node_stride-th node to its network's data set
template <int NF>
__global__ void replay_targets_kernel(const BNode* bnd, long long n_bnd, int node_stride, int phase, const int* map,
                                      const float* a_thin, const float* a_thick, const double* mass,
                                      const float* stage, float* X, float* T, unsigned long long* count,
                                      long long capacity) {
    const int F = 3 * NF;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_bnd * NF;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / NF), f = (int)(i - (long long)b * NF);
        if ((b + phase) % node_stride != 0) continue;
        const BNode bn = bnd[b];
        const long long g = bn.node, h = map[g];
        float t[3];
        for (int j = 0; j < 3; ++j) {
            const int ax = frame_axis(bn.frame, j);
            t[j] = frame_sign(bn.frame, j) *
                   (float)(mass[g] * ((double)a_thick[h * F + f * 3 + ax] - (double)a_thin[g * F + f * 3 + ax]));
        }
        const unsigned long long k = atomicAdd(count + bn.net, 1ull);
        if ((long long)k >= capacity) continue;
        float* xo = X + ((size_t)bn.net * capacity + k) * kIn;
        float* to = T + ((size_t)bn.net * capacity + k) * kOut;
        for (int q = 0; q < kIn; ++q) xo[q] = stage[i * kIn + q];
        for (int q = 0; q < kOut; ++q) to[q] = t[q];
    }
}

// ---------------------------------------------------------------------------
// training: forward/backward of one sample per thread on the CUDA cores
// ---------------------------------------------------------------------------

constexpr int kTB = 64;  // samples per block

struct TrainArgs {
    const float* X;      // [n][36] raw face-frame features of this network
    const float* T;      // [n][3]
    const int* idx;      // [n_batch] sample indices of the minibatch
    int n_batch;
    const float* wm;     // [kMNet] master weights (rounded to BF16 when loaded)
    float sc[4];
    float* grad;         // [kMNet]
    double* loss;        // sum of squared errors
};

__device__ inline float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__global__ void __launch_bounds__(kTB) train_kernel(TrainArgs A) {
    extern __shared__ __align__(16) float ts[];
    float* w1 = ts;                    // [64][36]
    float* w2 = w1 + kHid * kIn;       // [64][64]
    float* w3 = w2 + kHid * kHid;      // [3][64]
    float* xs = w3 + kOut * kHid;      // [kTB][36]
    float* z1 = xs + kTB * kIn;        // [kTB][64]
    float* hp = z1 + kTB * kHid;       // [kTB][64] relu(W2 relu(z1))
    float* hm = hp + kTB * kHid;       // [kTB][64] relu(W2 relu(-z1))
    float* dp = hm + kTB * kHid;       // [kTB][64] dz2 (+)
    float* dm = dp + kTB * kHid;       // [kTB][64] dz2 (-)
    float* d1 = dm + kTB * kHid;       // [kTB][64] dz1
    float* ep = d1 + kTB * kHid;       // [kTB][3] d loss / d y, the same for both branches
    const int tid = threadIdx.x;
    for (int q = tid; q < kMNet; q += kTB) ts[q] = bf16r(A.wm[q]);
    const int s = blockIdx.x * kTB + tid;
    const bool ok = s < A.n_batch;
    float x[kIn], t[kOut];
    if (ok) {
        const int i = A.idx[s];
        float nrm = 0.f;
        for (int q = 0; q < kIn; ++q) {
            x[q] = A.X[(size_t)i * kIn + q] / A.sc[(q % 9) / 3];
            nrm += x[q] * x[q];
        }
        nrm = sqrtf(nrm);
        const float inv = nrm > 0.f ? 1.f / nrm : 0.f;
        for (int q = 0; q < kIn; ++q) x[q] *= inv;
        for (int q = 0; q < kOut; ++q) t[q] = A.T[(size_t)i * kOut + q] / A.sc[3] * inv;
    } else {
        for (int q = 0; q < kIn; ++q) x[q] = 0.f;
        for (int q = 0; q < kOut; ++q) t[q] = 0.f;
    }
    __syncthreads();
    for (int q = 0; q < kIn; ++q) xs[tid * kIn + q] = x[q];
    // forward
    for (int nn = 0; nn < kHid; ++nn) {
        float acc = 0.f;
        for (int k = 0; k < kIn; ++k) acc += w1[nn * kIn + k] * x[k];
        z1[tid * kHid + nn] = acc;
    }
    float y[2][kOut];
    for (int br = 0; br < 2; ++br) {
        const float sg = br == 0 ? 1.f : -1.f;
        float* h = br == 0 ? hp : hm;
        for (int nn = 0; nn < kHid; ++nn) {
            float acc = 0.f;
            for (int k = 0; k < kHid; ++k) acc += w2[nn * kHid + k] * fmaxf(sg * z1[tid * kHid + k], 0.f);
            h[tid * kHid + nn] = fmaxf(acc, 0.f);
        }
        for (int o = 0; o < kOut; ++o) {
            float acc = 0.f;
            for (int k = 0; k < kHid; ++k) acc += w3[o * kHid + k] * h[tid * kHid + k];
            y[br][o] = acc;
        }
    }
    // c_j = -softplus(f_j) vh_j with f = (y(+x) + y(-x)) / 2 and vh the
    // newest velocity channels of the normalised features
    double l = 0.0;
    float dyv[kOut];
    for (int o = 0; o < kOut; ++o) {
        const float fz = 0.5f * (y[0][o] + y[1][o]);
        const float sp = fz > 20.f ? fz : log1pf(expf(fz));
        const float sgm = 1.f / (1.f + expf(-fz));
        const float vh = x[3 + o];
        const float e = ok ? -sp * vh - t[o] : 0.f;
        l += 0.5 * (double)e * e;
        dyv[o] = 0.5f * e * (-vh) * sgm;  // d loss / d y(+x) = d loss / d y(-x)
        ep[tid * kOut + o] = dyv[o];
    }
    // backward to dz2 (+/-) and dz1
    for (int br = 0; br < 2; ++br) {
        const float* h = br == 0 ? hp : hm;
        float* dz = br == 0 ? dp : dm;
        for (int k = 0; k < kHid; ++k) {
            float g = 0.f;
            for (int o = 0; o < kOut; ++o) g += w3[o * kHid + k] * dyv[o];
            dz[tid * kHid + k] = h[tid * kHid + k] > 0.f ? g : 0.f;
        }
    }
    for (int k = 0; k < kHid; ++k) {
        float gp = 0.f, gm = 0.f;
        for (int nn = 0; nn < kHid; ++nn) {
            gp += w2[nn * kHid + k] * dp[tid * kHid + nn];
            gm += w2[nn * kHid + k] * dm[tid * kHid + nn];
        }
        const float zz = z1[tid * kHid + k];
        d1[tid * kHid + k] = (zz > 0.f ? gp : 0.f) - (zz < 0.f ? gm : 0.f);
    }
    __syncthreads();
    // weight gradients summed over the block's samples
    for (int q = tid; q < kMNet; q += kTB) {
        float g = 0.f;
        if (q < kM2) {
            const int nn = q / kIn, k = q - nn * kIn;
            for (int r = 0; r < kTB; ++r) g += d1[r * kHid + nn] * xs[r * kIn + k];
        } else if (q < kM3) {
            const int qq = q - kM2, nn = qq / kHid, k = qq - nn * kHid;
            for (int r = 0; r < kTB; ++r) {
                const float zz = z1[r * kHid + k];
                g += dp[r * kHid + nn] * fmaxf(zz, 0.f) + dm[r * kHid + nn] * fmaxf(-zz, 0.f);
            }
        } else {
            const int qq = q - kM3, o = qq / kHid, k = qq - o * kHid;
            for (int r = 0; r < kTB; ++r) g += ep[r * kOut + o] * (hp[r * kHid + k] + hm[r * kHid + k]);
        }
        atomicAdd(A.grad + q, g);
    }
    // loss
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((tid & 31) == 0) atomicAdd(A.loss, l);
}

constexpr size_t kTrainSmem = sizeof(float) * (kMNet + kTB * kIn + 6 * kTB * kHid + kTB * kOut);

__global__ void adam_kernel(int n, float* w, float* m, float* v, const float* g, float scale, float lr, float b1,
                            float b2, float eps, int t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * scale;
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    const float mh = m[i] / (1.f - powf(b1, (float)t)), vh = v[i] / (1.f - powf(b2, (float)t));
    w[i] -= lr * mh / (sqrtf(vh) + eps);
}

// per-channel sums of squares of features (u, v, a) and targets
__global__ void moments_kernel(const float* X, const float* T, long long n, double* out) {
    double s[4] = {0, 0, 0, 0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < kIn; ++q) {
            const double x = X[i * kIn + q];
            s[(q % 9) / 3] += x * x;
        }
        for (int q = 0; q < kOut; ++q) {
            const double t = T[i * kOut + q];
            s[3] += t * t;
        }
    }
    for (int c = 0; c < 4; ++c) {
        double r = s[c];
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(out + c, r);
    }
}

}  // namespace gfb

// ===========================================================================
// C ABI
// ===========================================================================

struct gfb_trainer {
    int device = 0;
    int n_net = 0;
    long long capacity = 0;
    gfb::DevMem mem;
    float* X = nullptr;                 // [n_net][capacity][36]
    float* T = nullptr;                 // [n_net][capacity][3]
    unsigned long long* count = nullptr;
    float* wm = nullptr;                // [n_net][kMNet] master weights
    float* am = nullptr;                // Adam moments
    float* av = nullptr;
    float* grad = nullptr;              // [kMNet]
    int* idx = nullptr;                 // [max batch]
    double* dsum = nullptr;             // scratch sums
    float sc[4] = {1.f, 1.f, 1.f, 1.f};
    bool have_scales = false;
    int adam_t = 0;
    int max_batch = 1 << 16;
    cudaStream_t stream = nullptr;
    ~gfb_trainer() {
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

gfb_status gfb_layer_attach(gfb_solver* s, const gfb_layer* layer, const uint16_t* weights, const float* scales,
                            double threshold) {
    using namespace gfb;
    if (!s || !layer || !weights || !scales) return set_error(GFB_ERR_INVALID, "NULL argument");
    const SolverView v = solver_view(s);
    if (v.precision != GFB_FP32) return set_error(GFB_ERR_UNSUPPORTED, "the learned layer runs on the FP32 path");
    if (v.n_field > 3) return set_error(GFB_ERR_UNSUPPORTED, "the learned layer takes at most 3 wavefields");
    if (v.n_model != 1) return set_error(GFB_ERR_UNSUPPORTED, "the learned layer needs a single-model solver");
    LCU(cudaSetDevice(v.device));
    auto L = std::make_unique<Layer>();
    gfb_status st;
    if ((st = build_boundary(v, layer, L->mem, L->B))) return st;
    if ((st = L->mem.alloc(&L->w, (size_t)layer->n_net * kWNet))) return st;
    LCU(cudaMemcpy(L->w, weights, (size_t)layer->n_net * kWNet * 2, cudaMemcpyHostToDevice));
    for (int q = 0; q < 4; ++q) {
        if (!(scales[q] > 0.f)) return set_error(GFB_ERR_INVALID, "learned layer: scales must be positive");
        L->sc[q] = scales[q];
    }
    L->n_net = layer->n_net;
    if ((st = L->mem.alloc(&L->gain, (size_t)layer->n_net * 3))) return st;
    {
        const std::vector<float> ones((size_t)layer->n_net * 3, 1.f);
        LCU(cudaMemcpy(L->gain, ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if ((st = L->mem.alloc(&L->acc, 4))) return st;
    if ((st = L->mem.alloc(&L->monitor, 3))) return st;
    if ((st = L->mem.alloc(&L->active, 1))) return st;
    LCU(cudaMemset(L->acc, 0, 4 * sizeof(double)));
    LCU(cudaMemset(L->monitor, 0, 3 * sizeof(double)));
    const int one = 1;
    LCU(cudaMemcpy(L->active, &one, sizeof(int), cudaMemcpyHostToDevice));
    L->threshold = threshold;
    L->smem = (size_t)layer->n_net * kWNet * 2 + kLayerWarps * 16 * kW1S * 2;
    if (L->smem > 227 * 1024) return set_error(GFB_ERR_UNSUPPORTED, "learned layer: too many networks");
    int n_sm = 0, per_sm = 0;
    LCU(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, v.device));
    auto set = [&](auto kern) -> gfb_status {
        LCU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem));
        LCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLayerWarps * 32, L->smem));
        return GFB_OK;
    };
    if (v.n_field == 1) st = set(layer_kernel<1>);
    else if (v.n_field == 2) st = set(layer_kernel<2>);
    else st = set(layer_kernel<3>);
    if (st) return st;
    if (per_sm < 1) return set_error(GFB_ERR_UNSUPPORTED, "learned layer: kernel does not fit on an SM");
    L->blocks = std::max(1, std::min(per_sm * n_sm, (L->B.n_tile + kLayerWarps - 1) / kLayerWarps));
    return solver_set_layer(s, L.release());
}

gfb_status gfb_layer_set_gains(gfb_solver* s, int32_t n_net, const float* gains) {
    using namespace gfb;
    if (!s || !gains) return set_error(GFB_ERR_INVALID, "NULL argument");
    Layer* L = solver_layer(s);
    if (!L) return set_error(GFB_ERR_STATE, "no learned layer attached");
    if (n_net != L->n_net) return set_error(GFB_ERR_INVALID, "learned layer: gains for another network count");
    for (int q = 0; q < 3 * n_net; ++q)
        if (!(gains[q] >= 0.f) || !std::isfinite(gains[q]))
            return set_error(GFB_ERR_INVALID, "learned layer: gains must be finite and >= 0");
    const SolverView v = solver_view(s);
    LCU(cudaSetDevice(v.device));
    LCU(cudaStreamSynchronize(v.stream));
    LCU(cudaMemcpy(L->gain, gains, (size_t)n_net * 3 * sizeof(float), cudaMemcpyHostToDevice));
    return GFB_OK;
}

gfb_status gfb_layer_status(gfb_solver* s, int32_t* active, double* residual) {
    using namespace gfb;
    if (!s) return set_error(GFB_ERR_INVALID, "solver is NULL");
    Layer* L = solver_layer(s);
    if (!L) return set_error(GFB_ERR_STATE, "no learned layer attached");
    const SolverView v = solver_view(s);
    LCU(cudaSetDevice(v.device));
    LCU(cudaStreamSynchronize(v.stream));
    int a = 0;
    double mon[2] = {0, 0};
    LCU(cudaMemcpy(&a, L->active, sizeof(int), cudaMemcpyDeviceToHost));
    LCU(cudaMemcpy(mon, L->monitor, sizeof(mon), cudaMemcpyDeviceToHost));
    if (active) *active = a;
    if (residual) *residual = mon[0];
    return GFB_OK;
}

gfb_status gfb_trainer_create(int32_t n_net, int64_t capacity, int32_t device, uint64_t seed, gfb_trainer** out) {
    using namespace gfb;
    if (!out) return set_error(GFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (n_net < 1 || n_net > 64 || capacity < 1) return set_error(GFB_ERR_INVALID, "trainer: bad sizes");
    LCU(cudaSetDevice(device));
    auto t = std::make_unique<gfb_trainer>();
    t->device = device;
    t->n_net = n_net;
    t->capacity = capacity;
    LCU(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    gfb_status st;
    if ((st = t->mem.alloc(&t->X, (size_t)n_net * capacity * kIn))) return st;
    if ((st = t->mem.alloc(&t->T, (size_t)n_net * capacity * kOut))) return st;
    if ((st = t->mem.alloc(&t->count, n_net))) return st;
    if ((st = t->mem.alloc(&t->wm, (size_t)n_net * kMNet))) return st;
    if ((st = t->mem.alloc(&t->am, (size_t)n_net * kMNet))) return st;
    if ((st = t->mem.alloc(&t->av, (size_t)n_net * kMNet))) return st;
    if ((st = t->mem.alloc(&t->grad, kMNet))) return st;
    if ((st = t->mem.alloc(&t->idx, t->max_batch))) return st;
    if ((st = t->mem.alloc(&t->dsum, 8))) return st;
    LCU(cudaMemset(t->count, 0, n_net * sizeof(unsigned long long)));
    LCU(cudaMemset(t->am, 0, (size_t)n_net * kMNet * sizeof(float)));
    LCU(cudaMemset(t->av, 0, (size_t)n_net * kMNet * sizeof(float)));
    // He initialisation, seeded
    std::mt19937_64 rng(seed);
    std::vector<float> w((size_t)n_net * kMNet);
    for (int k = 0; k < n_net; ++k) {
        float* m = w.data() + (size_t)k * kMNet;
        std::normal_distribution<float> n1(0.f, std::sqrt(2.f / kIn)), n2(0.f, std::sqrt(2.f / kHid)),
            n3(0.f, std::sqrt(1.f / kHid));
        for (int q = 0; q < kM2; ++q) m[q] = n1(rng);
        for (int q = kM2; q < kM3; ++q) m[q] = n2(rng);
        for (int q = kM3; q < kMNet; ++q) m[q] = n3(rng);
    }
    LCU(cudaMemcpy(t->wm, w.data(), w.size() * 4, cudaMemcpyHostToDevice));
    LCU(cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    *out = t.release();
    return GFB_OK;
}

gfb_status gfb_trainer_destroy(gfb_trainer* t) {
    if (t) {
        cudaSetDevice(t->device);
        cudaStreamSynchronize(t->stream);
        delete t;
    }
    return GFB_OK;
}

gfb_status gfb_trainer_collect(gfb_trainer* t, gfb_solver* thin, gfb_solver* thick, const int32_t* thin_to_thick,
                               const gfb_layer* layer, int32_t n_steps, int32_t sample_stride, int32_t node_stride) {
    using namespace gfb;
    if (!t || !thin || !thick || !thin_to_thick || !layer) return set_error(GFB_ERR_INVALID, "NULL argument");
    if (n_steps < 0 || sample_stride < 1 || node_stride < 1) return set_error(GFB_ERR_INVALID, "trainer: bad strides");
    const SolverView a = solver_view(thin), b = solver_view(thick);
    if (a.precision != GFB_FP32 || b.precision != GFB_FP32 || a.n_field != b.n_field || a.n_field > 3 || a.device != b.device ||
        a.device != t->device || a.n_model != 1 || b.n_model != 1)
        return set_error(GFB_ERR_INVALID, "trainer: thin and thick solvers must be single-model FP32 solvers with "
                                          "the same wavefields on the trainer's device");
    if (layer->n_net != t->n_net) return set_error(GFB_ERR_INVALID, "trainer: network count differs from the layer's");
    if (solver_layer(thin)) return set_error(GFB_ERR_STATE, "trainer: the thin solver must have no layer attached");
    LCU(cudaSetDevice(t->device));
    // the replay reads and writes u, v, a at every node
    gfb_status st0;
    if ((st0 = solver_full_state(thin)) || (st0 = solver_full_state(thick))) return st0;
    DevMem mem;
    Boundary B;
    gfb_status st;
    if ((st = build_boundary(a, layer, mem, B))) return st;
    // node map in device numbering
    std::vector<int> dmap(a.n_node);
    for (long long d = 0; d < a.n_node; ++d) {
        const long long g = a.node_perm->empty() ? d : (*a.node_perm)[d];
        const int h = thin_to_thick[g];
        if (h < 0 || h >= b.n_node) return set_error(GFB_ERR_INVALID, "trainer: node map out of range");
        dmap[d] = b.node_inv->empty() ? h : (*b.node_inv)[h];
    }
    int* map = nullptr;
    float* stage = nullptr;
    if ((st = mem.alloc(&map, dmap.size()))) return st;
    if ((st = mem.alloc(&stage, (size_t)B.n_bnd * a.n_field * kIn))) return st;
    LCU(cudaMemcpy(map, dmap.data(), dmap.size() * 4, cudaMemcpyHostToDevice));
    int s0 = 0, s1 = 0;
    if ((st = gfb_current_step(thin, &s0)) || (st = gfb_current_step(thick, &s1))) return st;
    if (s0 != s1) return set_error(GFB_ERR_STATE, "trainer: thin and thick solvers are at different steps");
    const int F = 3 * a.n_field;
    const int grid = 148 * 8;
    for (int it = 0; it < n_steps; ++it) {
        const long long n = s0 + it;
        // thin state of step n-1 = thick state of step n-1 on the shared nodes
        LCU(cudaStreamSynchronize(b.stream));
        replay_gather_kernel<<<grid, 256, 0, a.stream>>>(a.n_node, F, map, b.u, b.v, static_cast<const float*>(b.a),
                                                         a.u, a.v, static_cast<float*>(a.a));
        LCU(cudaGetLastError());
        if ((st = solver_predict(thin))) return st;
        if (a.n_field == 1) replay_features_kernel<1><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, n, a.u, a.v, static_cast<const float*>(a.a), B.ring, stage);
        else if (a.n_field == 2) replay_features_kernel<2><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, n, a.u, a.v, static_cast<const float*>(a.a), B.ring, stage);
        else replay_features_kernel<3><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, n, a.u, a.v, static_cast<const float*>(a.a), B.ring, stage);
        LCU(cudaGetLastError());
        LCU(cudaStreamSynchronize(a.stream));
        if ((st = gfb_advance(thick, 1)) || (st = gfb_advance(thin, 1))) return st;
        LCU(cudaStreamSynchronize(b.stream));
        if (n >= kTaps && (n % sample_stride) == 0) {
            const int phase = (int)((n / sample_stride) % node_stride);
            const float* at = static_cast<const float*>(a.a);
            const float* ak = static_cast<const float*>(b.a);
            if (a.n_field == 1) replay_targets_kernel<1><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, node_stride, phase, map, at, ak, a.mass, stage, t->X, t->T, t->count, t->capacity);
            else if (a.n_field == 2) replay_targets_kernel<2><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, node_stride, phase, map, at, ak, a.mass, stage, t->X, t->T, t->count, t->capacity);
            else replay_targets_kernel<3><<<grid, 256, 0, a.stream>>>(B.bnd, B.n_bnd, node_stride, phase, map, at, ak, a.mass, stage, t->X, t->T, t->count, t->capacity);
            LCU(cudaGetLastError());
        }
    }
    LCU(cudaStreamSynchronize(a.stream));
    return GFB_OK;
}

gfb_status gfb_trainer_samples(gfb_trainer* t, int64_t* counts) {
    using namespace gfb;
    if (!t || !counts) return set_error(GFB_ERR_INVALID, "NULL argument");
    LCU(cudaSetDevice(t->device));
    std::vector<unsigned long long> c(t->n_net);
    LCU(cudaMemcpy(c.data(), t->count, c.size() * 8, cudaMemcpyDeviceToHost));
    for (int k = 0; k < t->n_net; ++k) counts[k] = (int64_t)std::min<unsigned long long>(c[k], t->capacity);
    return GFB_OK;
}

gfb_status gfb_trainer_set_scales(gfb_trainer* t, const float* scales) {
    using namespace gfb;
    if (!t || !scales) return set_error(GFB_ERR_INVALID, "NULL argument");
    for (int q = 0; q < 4; ++q) {
        if (!(scales[q] > 0.f)) return set_error(GFB_ERR_INVALID, "trainer: scales must be positive");
        t->sc[q] = scales[q];
    }
    t->have_scales = true;
    return GFB_OK;
}

// Channel scales from the collected samples: RMS of u, v, a features and of
// the targets, over all networks.
static gfb_status trainer_scales(gfb_trainer* t) {
    using namespace gfb;
    std::vector<int64_t> cnt(t->n_net);
    gfb_status st;
    if ((st = gfb_trainer_samples(t, cnt.data()))) return st;
    LCU(cudaMemsetAsync(t->dsum, 0, 4 * sizeof(double), t->stream));
    long long total = 0;
    for (int k = 0; k < t->n_net; ++k) {
        if (cnt[k] == 0) continue;
        moments_kernel<<<148 * 4, 256, 0, t->stream>>>(t->X + (size_t)k * t->capacity * kIn,
                                                       t->T + (size_t)k * t->capacity * kOut, cnt[k], t->dsum);
        LCU(cudaGetLastError());
        total += cnt[k];
    }
    if (total == 0) return set_error(GFB_ERR_STATE, "trainer: no samples collected");
    double s[4];
    LCU(cudaMemcpyAsync(s, t->dsum, sizeof(s), cudaMemcpyDeviceToHost, t->stream));
    LCU(cudaStreamSynchronize(t->stream));
    for (int c = 0; c < 3; ++c) t->sc[c] = (float)std::sqrt(s[c] / (total * 12.0));
    t->sc[3] = (float)std::sqrt(s[3] / (total * 3.0));
    for (int c = 0; c < 4; ++c)
        if (!(t->sc[c] > 0.f) || !std::isfinite(t->sc[c])) t->sc[c] = 1.f;
    t->have_scales = true;
    return GFB_OK;
}

static gfb_status trainer_grad(gfb_trainer* t, int net, const float* X, const float* T, int n_batch, double* loss) {
    using namespace gfb;
    LCU(cudaMemsetAsync(t->grad, 0, kMNet * sizeof(float), t->stream));
    LCU(cudaMemsetAsync(t->dsum, 0, sizeof(double), t->stream));
    TrainArgs A;
    A.X = X;
    A.T = T;
    A.idx = t->idx;
    A.n_batch = n_batch;
    A.wm = t->wm + (size_t)net * kMNet;
    for (int q = 0; q < 4; ++q) A.sc[q] = t->sc[q];
    A.grad = t->grad;
    A.loss = t->dsum;
    train_kernel<<<(n_batch + kTB - 1) / kTB, kTB, kTrainSmem, t->stream>>>(A);
    LCU(cudaGetLastError());
    if (loss) {
        LCU(cudaMemcpyAsync(loss, t->dsum, sizeof(double), cudaMemcpyDeviceToHost, t->stream));
        LCU(cudaStreamSynchronize(t->stream));
    }
    return GFB_OK;
}

gfb_status gfb_trainer_fit(gfb_trainer* t, int32_t epochs, int32_t batch, float lr, uint64_t seed, double* loss) {
    using namespace gfb;
    if (!t) return set_error(GFB_ERR_INVALID, "trainer is NULL");
    if (epochs < 0 || batch < 1 || batch > t->max_batch || !(lr > 0.f))
        return set_error(GFB_ERR_INVALID, "trainer: bad epochs, batch or learning rate");
    LCU(cudaSetDevice(t->device));
    gfb_status st;
    if (!t->have_scales && (st = trainer_scales(t))) return st;
    std::vector<int64_t> cnt(t->n_net);
    if ((st = gfb_trainer_samples(t, cnt.data()))) return st;
    std::mt19937_64 rng(seed);
    std::vector<int> perm;
    for (int ep = 0; ep < epochs; ++ep) {
        double ep_loss = 0.0;
        long long ep_n = 0;
        for (int k = 0; k < t->n_net; ++k) {
            if (cnt[k] == 0) continue;
            perm.resize(cnt[k]);
            for (long long i = 0; i < cnt[k]; ++i) perm[i] = (int)i;
            std::shuffle(perm.begin(), perm.end(), rng);
            for (long long b0 = 0; b0 < cnt[k]; b0 += batch) {
                const int nb = (int)std::min<long long>(batch, cnt[k] - b0);
                LCU(cudaMemcpyAsync(t->idx, perm.data() + b0, nb * 4, cudaMemcpyHostToDevice, t->stream));
                double l = 0.0;
                if ((st = trainer_grad(t, k, t->X + (size_t)k * t->capacity * kIn,
                                       t->T + (size_t)k * t->capacity * kOut, nb, &l)))
                    return st;
                ep_loss += l;
                ep_n += nb;
                ++t->adam_t;
                adam_kernel<<<(kMNet + 255) / 256, 256, 0, t->stream>>>(
                    kMNet, t->wm + (size_t)k * kMNet, t->am + (size_t)k * kMNet, t->av + (size_t)k * kMNet, t->grad,
                    1.f / nb, lr, 0.9f, 0.999f, 1e-8f, t->adam_t);
                LCU(cudaGetLastError());
            }
        }
        if (loss) loss[ep] = ep_n ? ep_loss / ep_n : 0.0;
    }
    LCU(cudaStreamSynchronize(t->stream));
    return GFB_OK;
}

gfb_status gfb_trainer_evaluate(gfb_trainer* t, double* loss) {
    using namespace gfb;
    if (!t || !loss) return set_error(GFB_ERR_INVALID, "NULL argument");
    LCU(cudaSetDevice(t->device));
    gfb_status st;
    if (!t->have_scales && (st = trainer_scales(t))) return st;
    std::vector<int64_t> cnt(t->n_net);
    if ((st = gfb_trainer_samples(t, cnt.data()))) return st;
    double sum = 0.0;
    long long n = 0;
    std::vector<int> id(t->max_batch);
    for (int k = 0; k < t->n_net; ++k)
        for (long long b0 = 0; b0 < cnt[k]; b0 += t->max_batch) {
            const int nb = (int)std::min<long long>(t->max_batch, cnt[k] - b0);
            for (int i = 0; i < nb; ++i) id[i] = (int)(b0 + i);
            LCU(cudaMemcpyAsync(t->idx, id.data(), nb * 4, cudaMemcpyHostToDevice, t->stream));
            double l = 0.0;
            if ((st = trainer_grad(t, k, t->X + (size_t)k * t->capacity * kIn, t->T + (size_t)k * t->capacity * kOut,
                                   nb, &l)))
                return st;
            sum += l;
            n += nb;
        }
    *loss = n ? sum / n : 0.0;
    return GFB_OK;
}

gfb_status gfb_trainer_gradient(gfb_trainer* t, int32_t net, int32_t n, const float* x, const float* y, float* grad,
                                double* loss) {
    using namespace gfb;
    if (!t || !x || !y || !grad) return set_error(GFB_ERR_INVALID, "NULL argument");
    if (net < 0 || net >= t->n_net || n < 1 || n > t->max_batch) return set_error(GFB_ERR_INVALID, "trainer: bad net or n");
    LCU(cudaSetDevice(t->device));
    DevMem mem;
    float *dx = nullptr, *dy = nullptr;
    gfb_status st;
    if ((st = mem.alloc(&dx, (size_t)n * kIn)) || (st = mem.alloc(&dy, (size_t)n * kOut))) return st;
    LCU(cudaMemcpy(dx, x, (size_t)n * kIn * 4, cudaMemcpyHostToDevice));
    LCU(cudaMemcpy(dy, y, (size_t)n * kOut * 4, cudaMemcpyHostToDevice));
    std::vector<int> id(n);
    for (int i = 0; i < n; ++i) id[i] = i;
    LCU(cudaMemcpy(t->idx, id.data(), n * 4, cudaMemcpyHostToDevice));
    double l = 0.0;
    if ((st = trainer_grad(t, net, dx, dy, n, &l))) return st;
    LCU(cudaMemcpy(grad, t->grad, kMNet * 4, cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return GFB_OK;
}

gfb_status gfb_trainer_get_params(gfb_trainer* t, float* params, float* scales) {
    using namespace gfb;
    if (!t) return set_error(GFB_ERR_INVALID, "trainer is NULL");
    LCU(cudaSetDevice(t->device));
    LCU(cudaStreamSynchronize(t->stream));
    if (params) LCU(cudaMemcpy(params, t->wm, (size_t)t->n_net * kMNet * 4, cudaMemcpyDeviceToHost));
    if (scales)
        for (int q = 0; q < 4; ++q) scales[q] = t->sc[q];
    return GFB_OK;
}

gfb_status gfb_trainer_set_params(gfb_trainer* t, const float* params) {
    using namespace gfb;
    if (!t || !params) return set_error(GFB_ERR_INVALID, "NULL argument");
    LCU(cudaSetDevice(t->device));
    LCU(cudaStreamSynchronize(t->stream));
    LCU(cudaMemcpy(t->wm, params, (size_t)t->n_net * kMNet * 4, cudaMemcpyHostToDevice));
    return GFB_OK;
}

gfb_status gfb_layer_pack(int32_t n_net, const float* params, uint16_t* weights) {
    using namespace gfb;
    if (n_net < 1 || !params || !weights) return set_error(GFB_ERR_INVALID, "bad arguments");
    for (int k = 0; k < n_net; ++k)
        pack_weights(params + (size_t)k * kMNet, reinterpret_cast<__nv_bfloat16*>(weights) + (size_t)k * kWNet);
    return GFB_OK;
}

}  // extern "C"
