// gfb_solver.cu -- host side of the B200 CG-SEM elastic time loop (C ABI in
// include/gfb.h).  Builds the device layout from the reference's merged
// partition arrays, launches the kernels of gfb_kernels.cuh and manages the
// snapshot ring.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/gfb.h"
#include "gfb_internal.h"
#include "gfb_kernels.cuh"

namespace {

thread_local std::string g_err;

// Steps between full evaluations of the element force on the FP32 path:
// the steps between add the force of the predicted displacement's
// increment.  Each full evaluation rounds the whole predicted displacement
// to float, a perturbation the stiffness amplifies into the highest
// (undamped) modes; by increments the rounded quantity is a step's change,
// ~dt*omega smaller, and the periodic full evaluation keeps the float sum
// of increments from drifting.  The acceleration error after the deformed
// 128x128x64 run (6000 steps) was 1.0e-4 / 5.9e-5 / 5.2e-5 for periods of
// 100 / 400 / 800 steps: the rounding of the increments grows like the
// square root of the period, that of the full evaluations like their count.
constexpr int kRefreshSteps = 800;

gfb_status fail(gfb_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

#define CU(call)                                                                           \
    do {                                                                                   \
        cudaError_t _e = (call);                                                           \
        if (_e != cudaSuccess)                                                             \
            return fail(_e == cudaErrorMemoryAllocation ? GFB_ERR_NOMEM : GFB_ERR_CUDA,   \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// GLL nodes, weights and derivative matrix D[i*ng+j] = l_j'(x_i): the
// tables of forward/share/include/gf/gll.hpp:48-131 (Newton on P_N').
double legendre(int n, double x) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    double a = 1.0, b = x, c = 0.0;
    for (int m = 1; m < n; ++m) {
        c = ((2.0 * m + 1.0) * x * b - m * a) / (m + 1.0);
        a = b;
        b = c;
    }
    return c;
}

double legendre_d(int n, double x) {
    if (n == 0) return 0.0;
    if (std::abs(x - 1.0) < 1e-14) return 0.5 * n * (n + 1.0);
    if (std::abs(x + 1.0) < 1e-14) return (n % 2 == 0 ? -1.0 : 1.0) * 0.5 * n * (n + 1.0);
    return n * (x * legendre(n, x) - legendre(n - 1, x)) / (x * x - 1.0);
}

bool gll_tables(int N, std::vector<double>& x, std::vector<double>& w, std::vector<double>& D) {
    const int ng = N + 1;
    x.assign(ng, 0.0);
    w.assign(ng, 0.0);
    D.assign(ng * ng, 0.0);
    x[0] = -1.0;
    x[N] = 1.0;
    for (int i = 1; i < N; ++i) {
        double t = -std::cos(M_PI * i / N);
        for (int it = 0; it < 100; ++it) {
            const double f = legendre_d(N, t);
            const double df = (2.0 * t * f - N * (N + 1.0) * legendre(N, t)) / (1.0 - t * t);
            if (std::abs(df) < 1.0e-14) return false;
            const double st = -f / df;
            t += st;
            if (std::abs(st) < 1.0e-15 * (1.0 + std::abs(t))) break;
        }
        x[i] = t;
    }
    std::vector<double> pn(ng);
    for (int i = 0; i < ng; ++i) {
        pn[i] = legendre(N, x[i]);
        w[i] = 2.0 / (N * (N + 1.0) * pn[i] * pn[i]);
    }
    for (int i = 0; i < ng; ++i)
        for (int j = 0; j < ng; ++j)
            D[i * ng + j] = (i == j) ? (i == 0 ? -0.25 * N * (N + 1.0) : (i == N ? 0.25 * N * (N + 1.0) : 0.0))
                                     : pn[i] / (pn[j] * (x[i] - x[j]));
    return true;
}

// fn(i0, i1) over [0, n) split across the host's threads, each thread
// taking at least `grain` items
template <typename F>
void parallel_for(long long n, F&& fn, long long grain = 65536) {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    nt = (unsigned)std::max(1LL, std::min((long long)nt, n / std::max(1LL, grain)));
    if (nt == 1) {
        fn(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(fn, n * t / nt, n * (t + 1) / nt);
    for (auto& x : th) x.join();
}

// Append to out, in increasing q, value(q) for every q in [0, n) with
// keep(q); the host threads count and fill chunks of q in parallel.
template <typename Keep, typename Value>
void parallel_compact(long long n, Keep&& keep, Value&& value, std::vector<int>& out) {
    const long long n_chunk = std::max(1LL, std::min<long long>(256, n / 65536));
    std::vector<long long> cnt(n_chunk + 1, 0);
    auto bounds = [&](long long c) { return n * c / n_chunk; };
    parallel_for(n_chunk, [&](long long c0, long long c1) {
        for (long long c = c0; c < c1; ++c) {
            long long k = 0;
            for (long long q = bounds(c); q < bounds(c + 1); ++q) k += keep(q) ? 1 : 0;
            cnt[c + 1] = k;
        }
    }, 1);
    for (long long c = 0; c < n_chunk; ++c) cnt[c + 1] += cnt[c];
    const size_t base = out.size();
    out.resize(base + (size_t)cnt[n_chunk]);
    parallel_for(n_chunk, [&](long long c0, long long c1) {
        for (long long c = c0; c < c1; ++c) {
            size_t o = base + (size_t)cnt[c];
            for (long long q = bounds(c); q < bounds(c + 1); ++q)
                if (keep(q)) out[o++] = value(q);
        }
    }, 1);
}

// The points of the mesh grouped by the thread that owns their node.
// Owner t holds the nodes [bound[t], bound[t+1]) and the points q that list
// one of them, in increasing q: q[off[t] .. off[t+1]).  Built once by a
// parallel partition of the points; a pass that must visit each node's
// points in mesh order (sums in the reference's order) then reads only its
// own points instead of scanning every point per thread.
struct NodeBuckets {
    int n_owner = 1;
    long long n_node = 0;
    std::vector<long long> bound;  // [n_owner + 1]
    std::vector<size_t> off;       // [n_owner + 1]
    std::vector<long long> q;      // [points]
    int owner(long long g) const {
        int t = (int)(g * n_owner / std::max(1LL, n_node));
        while (t + 1 < n_owner && bound[t + 1] <= g) ++t;
        while (t > 0 && bound[t] > g) --t;
        return t;
    }
    // fn(t, g0, g1, points, count) on one thread per owner
    template <typename F>
    void for_each_owner(F&& fn) const {
        std::vector<std::thread> th;
        for (int t = 0; t < n_owner; ++t)
            th.emplace_back([&, t] { fn(t, bound[t], bound[t + 1], q.data() + off[t], off[t + 1] - off[t]); });
        for (auto& x : th) x.join();
    }
};

NodeBuckets bucket_points(const int* ibool, long long P, long long n_node) {
    NodeBuckets b;
    const long long hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    b.n_owner = (int)std::max(1LL, std::min(hw, n_node / (1LL << 18)));
    b.n_node = n_node;
    const int T = b.n_owner;
    b.bound.resize(T + 1);
    for (int t = 0; t <= T; ++t) b.bound[t] = n_node * t / T;
    const long long n_chunk = std::max(1LL, std::min<long long>(4 * hw, P / 65536));
    auto cb = [&](long long c) { return P * c / n_chunk; };
    std::vector<size_t> pos((size_t)n_chunk * T, 0);
    parallel_for(n_chunk, [&](long long c0, long long c1) {
        for (long long c = c0; c < c1; ++c)
            for (long long q = cb(c); q < cb(c + 1); ++q) pos[(size_t)c * T + b.owner(ibool[q])]++;
    }, 1);
    b.off.assign(T + 1, 0);
    size_t run = 0;
    for (int t = 0; t < T; ++t) {
        b.off[t] = run;
        for (long long c = 0; c < n_chunk; ++c) {
            const size_t k = pos[(size_t)c * T + t];
            pos[(size_t)c * T + t] = run;
            run += k;
        }
    }
    b.off[T] = run;
    b.q.resize(run);
    parallel_for(n_chunk, [&](long long c0, long long c1) {
        for (long long c = c0; c < c1; ++c) {
            size_t* pc = pos.data() + (size_t)c * T;
            for (long long q = cb(c); q < cb(c + 1); ++q) b.q[pc[b.owner(ibool[q])]++] = q;
        }
    }, 1);
    return b;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

struct Snapshot {
    int step;
    int slot;                  // ring slot (device + pinned host), -1 once spilled
    std::unique_ptr<unsigned char[]> host;  // spilled raw copy [NFLD][n_rec][NN][15] (float or double)
    int fields_read = 0;
    int readers = 0;           // gfb_read_record calls copying out of the slot
    bool done = false;         // read (or released); removed once no reader holds it
    std::vector<char> read_mask;
};

}  // namespace

struct gfb_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;
    int prec = GFB_FP64;
    int ng = 0, nn = 0, nfld = 1, F = 3;
    int n_cell = 0, n_node = 0;
    double dt = 0.0;
    int stride = 0;
    int dirs[gfb::kMaxFields] = {0, 1, 2};
    int fset[gfb::kMaxFields] = {};    // source set of each wavefield
    int n_set = 1;                     // source sets (positions), one model only when > 1
    std::vector<gfb_source> sets;      // the sets during gfb_create (host arrays borrowed)
    bool stf_from_sets = false;        // source time functions per set (else per model)
    int* src_set = nullptr;            // [slot] set of each source slot (n_set > 1)
    int flags = 0;
    bool fuse = false;  // node update in the element kernel's last colour
    int step = 0;
    std::vector<int> colour_begin;  // [n_colour+1] device cell ranges
    bool has_cpml = false, has_damping = false, has_src = false;
    int n_pml = 0, n_src = 0, n_rec = 0, slots = 0;
    double c1 = 0.0, c2 = 0.0;
    // device memory
    std::vector<std::unique_ptr<DevBuf>> bufs;
    uint32_t* ibool = nullptr;
    uint32_t* ibool_padded = nullptr;  // [cell][NNP] for the pipelined kernel
    int pipe_blocks = 0;               // persistent grid of the element kernel
    int col_blocks = 0;                // persistent grid of the line kernel (FP32)
    int col_variant = 0;               // line kernel: 0 default (line owners where built), 1 fewer cells, 2 more, 3 default cells, exchange by every thread
    int n_col_variants = 1;
    int col_epb = 0;                   // cells per group of the variant in use
    bool point_kernel = false;         // thread-per-point element kernel on the FP32 path
    void* geom = nullptr;
    void* dmat = nullptr;
    float dmat_host[36] = {};          // D of the line kernel's parameters
    double *u = nullptr, *v = nullptr;
    void *a = nullptr, *ut = nullptr, *force = nullptr;
    double* mass = nullptr;
    void* inv_mass = nullptr;
    double* damping = nullptr;
    int* pml_slot = nullptr;
    void *pml_coef = nullptr, *pml_mem = nullptr, *pml_prev = nullptr;
    int *src_head = nullptr, *src_next = nullptr;
    void* src_w = nullptr;
    int* rec_cell = nullptr;
    // recording nodes merged across cells: unique node ids (ascending), CSR
    // of their (recording cell, point) occurrences and mass weights
    int n_unique = 0;
    std::vector<int64_t> rec_node_ids;
    int *gf_ptr = nullptr, *gf_occ = nullptr;
    double* gf_w = nullptr;
    // models sharing the solver (one for gfb_create): constants, step
    // counters and source time functions on the device, so that a step
    // captured in a CUDA graph replays correctly
    int n_model = 1;
    std::vector<int> model_nsteps;
    gfb::ModelConst* d_mc = nullptr;
    uint8_t* d_node_model = nullptr;   // [node] (several models only)
    // several models: per model the end of its cells in each colour and of
    // its nodes in the C-PML and plain ranges; the bounds of this step
    int* d_cell_end = nullptr;          // [model][colour]
    int* d_colour_first = nullptr;      // [colour]
    long long* d_node_end = nullptr;    // [model][2]
    int* d_live_cell_end = nullptr;     // [colour]
    long long* d_live_node_end = nullptr;  // [2]
    int *d_mlive = nullptr, *d_mstep = nullptr, *d_nsteps = nullptr, *d_nstf = nullptr;
    // element force in full every `refresh` steps and by increments between
    // (FP32 path; 1 = in full every step): per model this step's kind, the
    // next step's kind and a one-shot request for a full step
    int refresh = 1;
    bool by_increments_ok = false;     // the force may be updated by increments (FP32, node-form or no C-PML, ...)
    int *d_mdirect = nullptr, *d_mnext = nullptr, *d_force_direct = nullptr;
    int* d_kernel_err = nullptr;       // set by a kernel whose bounded wait gave up
    // plain nodes (device nodes >= hv_begin) keep the half-step velocity
    // v + dt/2 a in v and no acceleration (FP32 path); a_in_force: the
    // assembled force holds the last step's (a = f/m), else a is the stored
    // one (state set since the last step)
    bool half_v = false;
    long long hv_begin = 0;
    float* w32 = nullptr;              // [node][F] half-step velocity of the nodes >= hv_begin
    bool a_in_force = false;
    long long* d_stf_off = nullptr;
    void *d_mstf = nullptr, *d_stf_all = nullptr;
    bool use_graph = true;
    cudaGraphExec_t gexec = nullptr;   // one step: step start, colours, node pass
    gfb::Layer* layer = nullptr;       // learned absorbing layer (or none)
    long long graph_launches = 0;
    void* ring = nullptr;              // device snapshot ring [slots]
    std::vector<void*> pinned;         // pinned host copy of each slot
    bool rec_f32 = false;              // snapshot values stored as float
    std::vector<cudaEvent_t> rec_evt;  // record kernel of the slot done
    std::vector<cudaEvent_t> copy_evt; // device->host copy of the slot done
    std::vector<char> copy_issued;
    int next_slot = 0;
    // pending snapshots and slot ownership are shared between gfb_advance
    // and gfb_read_record, which may run on different host threads
    std::mutex rec_mu;
    std::condition_variable rec_cv;
    std::deque<Snapshot> pending;
    // C-PML kept at global nodes (FP32 path)
    bool node_pml = false;
    int n_pml_node = 0;
    std::vector<int> node_perm, node_inv;  // device node -> node and back (empty: identity)
    void *npml_coef = nullptr, *npml_mem = nullptr, *npml_prev = nullptr;
    long long device_bytes = 0, upload_bytes = 0, launches = 0;

    template <typename T>
    gfb_status alloc(T** out, size_t count) {
        auto b = std::make_unique<DevBuf>();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&b->p, count * sizeof(T));
        if (e != cudaSuccess)
            return fail(GFB_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                        cudaGetErrorString(e));
        *out = static_cast<T*>(b->p);
        device_bytes += (long long)(count * sizeof(T));
        bufs.push_back(std::move(b));
        return GFB_OK;
    }
    ~gfb_solver() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (layer) gfb::layer_free(layer);
        for (auto e : rec_evt) cudaEventDestroy(e);
        for (auto e : copy_evt) cudaEventDestroy(e);
        for (auto p : pinned) cudaFreeHost(p);
        bufs.clear();
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

namespace {

// Host<->device copies ordered on the solver's stream and complete on return
// (a plain cudaMemcpy from pageable memory may return before the data has
// reached the device, and the solver's non-blocking stream does not order
// against the legacy default stream).
gfb_status h2d(gfb_solver* s, void* dst, const void* src, size_t bytes) {
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->upload_bytes += (long long)bytes;
    return GFB_OK;
}

gfb_status d2h(gfb_solver* s, void* dst, const void* src, size_t bytes) {
    CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return GFB_OK;
}

template <typename Real>
gfb_status upload(gfb_solver* s, void** dst, const std::vector<Real>& h) {
    Real* d = nullptr;
    gfb_status st = s->alloc(&d, h.size());
    if (st) return st;
    CU(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(Real), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->upload_bytes += (long long)(h.size() * sizeof(Real));
    *dst = d;
    return GFB_OK;
}

// Pinned staging buffers of staged_upload: two 64 MB page-locked buffers
// (portable, so any device's copies may read them), allocated by the first
// gfb_create that uploads and kept for the rest of the process: pinning and
// unpinning them on every create cost more than the copies they serve.  The
// mutex serialises the creates that use them.
struct Staging {
    std::mutex mu;
    void* buf[2] = {nullptr, nullptr};
    size_t bytes = 0;
};
Staging& staging() {
    static Staging* st = new Staging();  // never destroyed: freed with the process
    return *st;
}

// Fill the device array dst of n_item items of item_bytes each.  The host
// threads pack the items chunk by chunk (pack(i0, i1, out) writes items
// [i0, i1) to out) into the two pinned staging buffers in turn, and the copy
// of one chunk to the device runs while the next is packed: no host copy of
// the whole array and no copy from pageable memory.  The caller holds
// staging().mu.
template <typename Pack>
gfb_status staged_upload(gfb_solver* s, void* dst, size_t item_bytes, long long n_item, Pack&& pack) {
    if (n_item <= 0) return GFB_OK;
    Staging& S = staging();
    const size_t stage = size_t(64) << 20;
    if (S.bytes == 0) {
        for (int k = 0; k < 2; ++k) CU(cudaHostAlloc(&S.buf[k], stage, cudaHostAllocPortable));
        S.bytes = stage;
    }
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events() {
            for (auto x : e)
                if (x) {
                    cudaEventSynchronize(x);
                    cudaEventDestroy(x);
                }
        }
    } done;
    for (int k = 0; k < 2; ++k) CU(cudaEventCreateWithFlags(&done.e[k], cudaEventDisableTiming));
    const long long per = std::max<long long>(1, (long long)(S.bytes / item_bytes));
    if ((size_t)per * item_bytes > S.bytes) return fail(GFB_ERR_UNSUPPORTED, "item of %zu bytes", item_bytes);
    long long c = 0;
    for (long long i0 = 0; i0 < n_item; i0 += per, ++c) {
        const int k = (int)(c & 1);
        const long long i1 = std::min(n_item, i0 + per);
        CU(cudaEventSynchronize(done.e[k]));  // the copy of chunk c-2 has read the buffer
        pack(i0, i1, static_cast<unsigned char*>(S.buf[k]));
        CU(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + (size_t)i0 * item_bytes, S.buf[k],
                           (size_t)(i1 - i0) * item_bytes, cudaMemcpyHostToDevice, s->stream));
        CU(cudaEventRecord(done.e[k], s->stream));
    }
    CU(cudaStreamSynchronize(s->stream));
    s->upload_bytes += (long long)((size_t)n_item * item_bytes);
    return GFB_OK;
}

// The pinned host slots of the snapshot ring, allocated by a helper thread
// while gfb_create does the rest of its work (page-locking hundreds of MB
// takes a large part of a second).  finish() hands them over; slots not
// handed over are freed.
struct PinnedRing {
    std::vector<void*> slot;
    cudaError_t err = cudaSuccess;
    std::thread worker;
    bool taken = false;
    void start(int device, int n, size_t bytes) {
        slot.assign(n, nullptr);
        worker = std::thread([this, device, n, bytes] {
            err = cudaSetDevice(device);
            for (int k = 0; k < n && err == cudaSuccess; ++k) {
                err = cudaHostAlloc(&slot[k], bytes, cudaHostAllocDefault);
                if (err != cudaSuccess) slot[k] = nullptr;
            }
        });
    }
    cudaError_t finish() {
        if (worker.joinable()) worker.join();
        return err;
    }
    ~PinnedRing() {
        if (worker.joinable()) worker.join();
        if (!taken)
            for (void* q : slot)
                if (q) cudaFreeHost(q);
    }
};

// Seconds spent in each stage of gfb_create, printed to stderr when the
// environment variable GFB_TRACE is set.
struct StageClock {
    bool on = std::getenv("GFB_TRACE") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char* what) {
        if (!on) return;
        const auto n = std::chrono::steady_clock::now();
        std::fprintf(stderr, "gfb_create %-28s %8.3f s\n", what, std::chrono::duration<double>(n - t).count());
        t = n;
    }
};

// ---------------------------------------------------------------------------
// kernel dispatch
// ---------------------------------------------------------------------------

template <typename Real>
void node_args(const gfb_solver* s, gfb::NodeArgs<Real>& A, gfb::NodePml<Real>& P) {
    A.n_node = s->n_node;
    A.u = s->u;
    A.v = s->v;
    A.a = static_cast<Real*>(s->a);
    A.ut = static_cast<Real*>(s->ut);
    A.force = static_cast<const Real*>(s->force);
    A.mass = s->mass;
    A.inv_mass = static_cast<const Real*>(s->inv_mass);
    A.damping = s->has_damping ? s->damping : nullptr;
    A.dt = s->dt;
    A.beta = 0.0;
    A.gamma = 0.5;
    A.half_dt2 = 0.5 * s->dt * s->dt * (1.0 - 2.0 * A.beta);
    A.node_model = s->d_node_model;
    A.mc = s->d_mc;
    A.mlive = s->d_mlive;
    A.live_node_end = s->d_live_node_end;  // null with one model
    A.mnext = s->refresh > 1 ? s->d_mnext : nullptr;
    A.half_v = s->half_v;
    A.w32 = s->w32;
    P = gfb::NodePml<Real>{};
    if (s->node_pml) {
        P.coef = static_cast<const Real*>(s->npml_coef);
        P.mem = static_cast<Real*>(s->npml_mem);
        P.prev = static_cast<Real*>(s->npml_prev);
        P.n_slot = s->n_pml_node;
    }
    P.c1 = s->c1;
    P.c2 = s->c2;
}

template <typename Real, int NG, int NFLD>
gfb_status launch_elem_t(gfb_solver* s, int c) {
    using S = gfb::PipeShape<Real, NG, NFLD>;
    gfb::ElemArgs<Real> A;
    A.e_begin = s->colour_begin[c];
    A.e_end = s->colour_begin[c + 1];
    if (A.e_end <= A.e_begin) return GFB_OK;
    A.ibool = s->ibool;
    A.geom = static_cast<const Real*>(s->geom);
    A.ut = static_cast<const Real*>(s->ut);
    A.force = static_cast<Real*>(s->force);
    A.dmat = static_cast<const Real*>(s->dmat);
    A.pml_slot = (s->has_cpml && !s->node_pml) ? s->pml_slot : nullptr;
    A.pml_coef = static_cast<const Real*>(s->pml_coef);
    A.pml_mem = static_cast<Real*>(s->pml_mem);
    A.pml_prev = static_cast<Real*>(s->pml_prev);
    A.u = s->u;
    A.v = s->v;
    A.a = static_cast<const Real*>(s->a);
    A.n_node = s->n_node;
    A.c1 = s->c1;
    A.c2 = s->c2;
    A.src_head = s->has_src ? s->src_head : nullptr;
    A.src_next = s->src_next;
    A.src_w = static_cast<const Real*>(s->src_w);
    A.mstf = static_cast<const Real*>(s->d_mstf);
    A.src_set = s->src_set;
    A.n_set = s->n_set;
    A.mlive = s->d_mlive;
    A.mdirect = s->refresh > 1 ? s->d_mdirect : nullptr;
    A.mc = s->d_mc;
    for (int d = 0; d < gfb::kMaxFields; ++d) {
        A.dir[d] = s->dirs[d];
        A.fset[d] = s->fset[d];
    }
    A.fuse = s->fuse ? 1 : 0;
    node_args(s, A.nu, A.np);
    const int n = A.e_end - A.e_begin;
    const int groups = (n + S::EPB - 1) / S::EPB;
    const int blocks = std::max(1, std::min(groups, s->pipe_blocks));
    gfb::elem_pipe_kernel<Real, NG, NFLD><<<blocks, S::THREADS, S::SMEM, s->stream>>>(A, s->ibool_padded, groups);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

// The FP32 path runs the line kernel unless per-cell C-PML, the fused node
// update or GFB_FLAG_POINT_KERNEL asks for the thread-per-point kernel.
bool col_kernel_eligible(const gfb_solver* s) {
    return s->prec == GFB_FP32 && !(s->has_cpml && !s->node_pml) && !s->fuse;
}
bool use_col_kernel(const gfb_solver* s) { return col_kernel_eligible(s) && !s->point_kernel; }

template <int NG, int NFLD, int EPB, bool XCH = false>
gfb_status launch_col_e(gfb_solver* s, int c) {
    using S = gfb::ColShape<NG, NFLD, EPB, XCH>;
    gfb::ColArgs A;
    A.e_begin = s->colour_begin[c];
    A.e_end = s->colour_begin[c + 1];
    if (A.e_end <= A.e_begin) return GFB_OK;
    const int n = A.e_end - A.e_begin;
    A.n_groups = (n + S::EPB - 1) / S::EPB;
    A.live_end = s->d_live_cell_end;  // null with one model
    A.colour = c;
    A.ibool_padded = s->ibool_padded;
    A.geom = static_cast<const float*>(s->geom);
    A.ut = static_cast<const float*>(s->ut);
    A.force = static_cast<float*>(s->force);
    A.dmat = static_cast<const float*>(s->dmat);
    A.src_head = s->has_src ? s->src_head : nullptr;
    A.src_next = s->src_next;
    A.src_w = static_cast<const float*>(s->src_w);
    A.mstf = static_cast<const float*>(s->d_mstf);
    A.src_set = s->src_set;
    A.n_set = s->n_set;
    A.mlive = s->d_mlive;
    A.mdirect = s->refresh > 1 ? s->d_mdirect : nullptr;
    A.n_model = s->n_model;
    for (int d = 0; d < gfb::kMaxFields; ++d) {
        A.dir[d] = s->dirs[d];
        A.fset[d] = s->fset[d];
    }
    for (int q = 0; q < 36; ++q) A.D[q] = q < NG * NG ? s->dmat_host[q] : 0.f;
    const int blocks = std::max(1, std::min(A.n_groups, s->col_blocks));
    A.err = reinterpret_cast<unsigned*>(s->d_kernel_err);
    const int smem = S::SMEM + gfb::col_model_smem(s->n_model, s->n_set);
    gfb::elem_col_kernel<NG, NFLD, EPB, XCH><<<blocks, S::THREADS, smem, s->stream>>>(A);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

// Candidates of the line kernel.  At ngll 5 with up to three wavefields:
// 0 the default cells per group with the eta/zeta contractions done by line
// owners (ColShape's XCH; the fastest measured), and with the exchange done
// by every thread 1 one fewer cell per group ("LO"), 2 one more ("HI"),
// 3 the default count.  Elsewhere: 0 the default count, exchange by every
// thread.
constexpr int col_epb_lo(int nfld) { return nfld == 3 ? 1 : (nfld == 2 ? 2 : 4); }
constexpr int col_epb_hi(int nfld) { return nfld == 3 ? 3 : (nfld == 2 ? 4 : 8); }
template <int NG, int NFLD>
struct ColEpb {
    static constexpr int D = gfb::col_default_epb(NG, NFLD);
    // the other variants exist for ngll 5 with up to three wavefields (more
    // would exceed a block's threads)
    static constexpr int N = (NG == 5 && NFLD <= 3) ? 4 : 1;
};

template <int NG, int NFLD>
gfb_status launch_col_t(gfb_solver* s, int c) {
    using E = ColEpb<NG, NFLD>;
    if constexpr (E::N > 1) {
        if (s->col_variant == 0) return launch_col_e<NG, NFLD, E::D, true>(s, c);
        if (s->col_variant == 1) return launch_col_e<NG, NFLD, col_epb_lo(NFLD)>(s, c);
        if (s->col_variant == 2) return launch_col_e<NG, NFLD, col_epb_hi(NFLD)>(s, c);
    }
    return launch_col_e<NG, NFLD, E::D>(s, c);
}

// Persistent grid of the line kernel variant EPB: occupancy x SMs.
template <int NG, int NFLD, int EPB, bool XCH = false>
gfb_status col_grid(gfb_solver* s, int* blocks) {
    using C = gfb::ColShape<NG, NFLD, EPB, XCH>;
    auto* fn = gfb::elem_col_kernel<NG, NFLD, EPB, XCH>;
    const int smem = C::SMEM + gfb::col_model_smem(s->n_model, s->n_set);
    CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0, n_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, C::THREADS, smem));
    CU(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, s->device));
    if (per_sm < 1) return fail(GFB_ERR_UNSUPPORTED, "line element kernel does not fit on an SM");
    *blocks = per_sm * n_sm;
    return GFB_OK;
}

template <int NG, int NFLD>
gfb_status col_grid_t(gfb_solver* s) {
    using E = ColEpb<NG, NFLD>;
    gfb_status st;
    s->n_col_variants = E::N;
    if constexpr (E::N > 1) {
        if (s->col_variant == 1) {
            s->col_epb = col_epb_lo(NFLD);
            return col_grid<NG, NFLD, col_epb_lo(NFLD)>(s, &s->col_blocks);
        }
        if (s->col_variant == 2) {
            s->col_epb = col_epb_hi(NFLD);
            return col_grid<NG, NFLD, col_epb_hi(NFLD)>(s, &s->col_blocks);
        }
        if (s->col_variant == 0) {
            s->col_epb = E::D;
            return col_grid<NG, NFLD, E::D, true>(s, &s->col_blocks);
        }
    }
    if ((st = col_grid<NG, NFLD, E::D>(s, &s->col_blocks))) return st;
    s->col_epb = E::D;
    return GFB_OK;
}

template <typename Real, int NG, int NFLD>
struct ColGridOp {
    static gfb_status run(gfb_solver* s) { return col_grid_t<NG, NFLD>(s); }
};

template <typename Real, int NG, int NFLD>
gfb_status set_smem_t(gfb_solver* s) {
    using S = gfb::PipeShape<Real, NG, NFLD>;
    CU(cudaFuncSetAttribute(gfb::elem_pipe_kernel<Real, NG, NFLD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            S::SMEM));
    int per_sm = 0, n_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gfb::elem_pipe_kernel<Real, NG, NFLD>, S::THREADS,
                                                     S::SMEM));
    CU(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, s->device));
    if (per_sm < 1) return fail(GFB_ERR_UNSUPPORTED, "element kernel does not fit on an SM");
    s->pipe_blocks = per_sm * n_sm;
    if constexpr (std::is_same<Real, float>::value) return col_grid_t<NG, NFLD>(s);
    return GFB_OK;
}

template <typename Real, int NG, int NFLD, typename Out>
gfb_status launch_record_o(gfb_solver* s, Out* out) {
    using S = gfb::Shape<NG>;
    gfb::RecArgs<Real, Out> A;
    A.n_rec = s->n_rec;
    A.rec_cell = s->rec_cell;
    A.ibool = s->ibool;
    A.geom = static_cast<const Real*>(s->geom);
    A.dmat = static_cast<const Real*>(s->dmat);
    A.u = s->u;
    A.v = s->v;
    A.a = static_cast<const Real*>(s->a);
    A.n_node = s->n_node;
    A.out = out;
    A.hv_begin = s->half_v ? s->hv_begin : s->n_node;
    A.w32 = s->w32;
    A.force = static_cast<const Real*>(s->force);
    A.inv_mass = static_cast<const Real*>(s->inv_mass);
    A.node_model = s->d_node_model;
    A.mc = s->d_mc;
    A.dt = s->dt;
    gfb::record_kernel<Real, NG, NFLD, Out><<<s->n_rec, S::NNP, 0, s->stream>>>(A);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

template <typename Real, int NG, int NFLD>
gfb_status launch_record_t(gfb_solver* s, void* out) {
    if (s->rec_f32) return launch_record_o<Real, NG, NFLD, float>(s, static_cast<float*>(out));
    return launch_record_o<Real, NG, NFLD, double>(s, static_cast<double*>(out));
}

// Instantiate (Real, NG, NFLD) combinations behind one switch.
template <typename Real, template <typename, int, int> class Op, typename... Args>
gfb_status dispatch(int ng, int nfld, Args... args) {
#define GFB_CASE(NGV, NFV) \
    if (ng == NGV && nfld == NFV) return Op<Real, NGV, NFV>::run(args...);
    GFB_CASE(3, 1) GFB_CASE(3, 2) GFB_CASE(3, 3)
    GFB_CASE(4, 1) GFB_CASE(4, 2) GFB_CASE(4, 3)
    GFB_CASE(5, 1) GFB_CASE(5, 2) GFB_CASE(5, 3)
    GFB_CASE(6, 1) GFB_CASE(6, 2) GFB_CASE(6, 3)
    // several source positions: three directions each, at ngll 5
    GFB_CASE(5, 6) GFB_CASE(5, 9) GFB_CASE(5, 12)
#undef GFB_CASE
    return fail(GFB_ERR_UNSUPPORTED, "ngll=%d with %d wavefields is not supported", ng, nfld);
}

template <typename Real, int NG, int NFLD>
struct ElemOp {
    static gfb_status run(gfb_solver* s, int c) {
        if constexpr (std::is_same<Real, float>::value)
            if (use_col_kernel(s)) return launch_col_t<NG, NFLD>(s, c);
        return launch_elem_t<Real, NG, NFLD>(s, c);
    }
};
template <typename Real, int NG, int NFLD>
struct SmemOp {
    static gfb_status run(gfb_solver* s) { return set_smem_t<Real, NG, NFLD>(s); }
};
template <typename Real, int NG, int NFLD>
struct RecOp {
    static gfb_status run(gfb_solver* s, void* out) { return launch_record_t<Real, NG, NFLD>(s, out); }
};

gfb_status launch_elem(gfb_solver* s, int c) {
    if (s->prec == GFB_FP64) return dispatch<double, ElemOp>(s->ng, s->nfld, s, c);
    return dispatch<float, ElemOp>(s->ng, s->nfld, s, c);
}

// Autotuner of the FP32 element phase: times full colour sweeps of every
// element-kernel candidate on this mesh (the line kernel with each cells-per-
// group count it is built with, and the thread-per-point kernel) and keeps
// the fastest.  A full sweep only rewrites the assembled force from the
// current predicted displacement (the first colour touching a node stores),
// so tuning leaves the solver's state as it was.
gfb_status autotune(gfb_solver* s) {
    if (!col_kernel_eligible(s)) return GFB_OK;
    const int n_colour = (int)s->colour_begin.size() - 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    struct Cand {
        bool point;
        int variant;
        float ms;
    };
    std::vector<Cand> cands;
    for (int v = 0; v < s->n_col_variants; ++v) cands.push_back({false, v, 0.0f});
    cands.push_back({true, 0, 0.0f});
    gfb_status st = GFB_OK;
    const long long l0 = s->launches;
    for (auto& c : cands) {
        s->point_kernel = c.point;
        s->col_variant = c.variant;
        if (!c.point && (st = dispatch<float, ColGridOp>(s->ng, s->nfld, s))) break;
        auto sweep = [&]() -> gfb_status {
            gfb_status r;
            for (int k = 0; k < n_colour; ++k)
                if ((r = launch_elem(s, k))) return r;
            return GFB_OK;
        };
        if ((st = sweep())) break;  // warm-up
        if (cudaEventRecord(e0, s->stream) != cudaSuccess) { st = fail(GFB_ERR_CUDA, "autotune event"); break; }
        for (int rep = 0; rep < 3 && !st; ++rep) st = sweep();
        if (st) break;
        if (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&c.ms, e0, e1) != cudaSuccess) {
            st = fail(GFB_ERR_CUDA, "autotune timing failed");
            break;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->launches = l0;
    if (st) return st;
    const Cand* best = &cands[0];
    for (const auto& c : cands)
        if (c.ms < best->ms) best = &c;
    s->point_kernel = best->point;
    s->col_variant = best->point ? 0 : best->variant;
    return dispatch<float, ColGridOp>(s->ng, s->nfld, s);
}

gfb_status launch_record(gfb_solver* s, void* out) {
    if (s->prec == GFB_FP64) return dispatch<double, RecOp>(s->ng, s->nfld, s, out);
    return dispatch<float, RecOp>(s->ng, s->nfld, s, out);
}

int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

template <typename Real, int NFLD, bool MULTI>
gfb_status launch_node_m(gfb_solver* s) {
    gfb::NodeArgs<Real> A;
    gfb::NodePml<Real> P;
    node_args(s, A, P);
    // node-form C-PML nodes are device nodes [0, n_pml_node)
    const long long g0 = s->node_pml ? s->n_pml_node : 0;
    if (g0 < s->n_node) {
        const int grid = grid_for((long long)(s->n_node - g0) * NFLD, 256);
        gfb::node_update_kernel<Real, NFLD, MULTI><<<grid, 256, 0, s->stream>>>(A, P, g0);
        CU(cudaGetLastError());
        s->launches++;
    }
    if (g0 > 0) {
        const int gp = grid_for(g0 * NFLD, 256);
        gfb::node_pml_kernel<Real, NFLD, MULTI><<<gp, 256, 0, s->stream>>>(A, P);
        CU(cudaGetLastError());
        s->launches++;
    }
    return GFB_OK;
}

template <typename Real, int NFLD>
gfb_status launch_node_f(gfb_solver* s) {
    return s->n_model > 1 ? launch_node_m<Real, NFLD, true>(s) : launch_node_m<Real, NFLD, false>(s);
}

template <typename Real>
gfb_status launch_node_t(gfb_solver* s) {
    switch (s->nfld) {
        case 1: return launch_node_f<Real, 1>(s);
        case 2: return launch_node_f<Real, 2>(s);
        case 3: return launch_node_f<Real, 3>(s);
        case 6: return launch_node_f<Real, 6>(s);
        case 9: return launch_node_f<Real, 9>(s);
        case 12: return launch_node_f<Real, 12>(s);
        default: return fail(GFB_ERR_UNSUPPORTED, "%d wavefields in the node pass", s->nfld);
    }
}

gfb_status launch_node(gfb_solver* s) {
    return s->prec == GFB_FP64 ? launch_node_t<double>(s) : launch_node_t<float>(s);
}

template <typename Real>
gfb_status launch_predict_t(gfb_solver* s) {
    const long long n = (long long)s->n_node * s->F;
    const double h = 0.5 * s->dt * s->dt * (1.0 - 2.0 * 0.0);
    gfb::predict_kernel<Real><<<grid_for(n, 256), 256, 0, s->stream>>>(
        (long long)s->n_node, s->F, s->u, s->v, static_cast<const Real*>(s->a), static_cast<Real*>(s->ut), s->dt, h,
        s->d_node_model, s->d_mc, s->half_v ? s->hv_begin : (long long)s->n_node, s->w32);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

// Half-step velocity state of the plain nodes to (v, a): into v_out / a_out,
// or in place (v_out == v, a_out == a) when leaving the form for good.
gfb_status half_v_to_full(gfb_solver* s, double* v_out, float* a_out) {
    const long long total = (long long)(s->n_node - s->hv_begin) * s->F;
    if (total <= 0) return GFB_OK;
    gfb::half_v_kernel<float><<<grid_for(total, 256), 256, 0, s->stream>>>(
        (long long)s->n_node, s->F, s->hv_begin, true, s->a_in_force, s->v, s->w32, static_cast<const float*>(s->a),
        static_cast<const float*>(s->force), static_cast<const float*>(s->inv_mass), s->d_node_model, s->d_mc, s->dt,
        v_out, a_out);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

// (v, a) of the plain nodes to the half-step velocity, in place.
gfb_status half_v_from_full(gfb_solver* s) {
    const long long total = (long long)(s->n_node - s->hv_begin) * s->F;
    if (total <= 0) return GFB_OK;
    gfb::half_v_kernel<float><<<grid_for(total, 256), 256, 0, s->stream>>>(
        (long long)s->n_node, s->F, s->hv_begin, false, false, s->v, s->w32, static_cast<const float*>(s->a), nullptr,
        nullptr, s->d_node_model, s->d_mc, s->dt, nullptr, nullptr);
    CU(cudaGetLastError());
    s->launches++;
    return GFB_OK;
}

// Leave the half-step velocity form (the learned layer and its trainer read
// and write v and a at any node): v and a in place, from here on.
gfb_status leave_half_v(gfb_solver* s) {
    if (!s->half_v) return GFB_OK;
    gfb_status st = half_v_to_full(s, s->v, static_cast<float*>(s->a));
    if (st) return st;
    CU(cudaStreamSynchronize(s->stream));
    s->half_v = false;
    s->hv_begin = s->n_node;
    if (s->gexec) {
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return GFB_OK;
}

// The predicted displacement rewritten in full from u, v, a (the start of a
// run, or after a state overwrite): the next step evaluates the element
// force in full.
gfb_status launch_predict(gfb_solver* s) {
    gfb_status st = s->prec == GFB_FP64 ? launch_predict_t<double>(s) : launch_predict_t<float>(s);
    if (st) return st;
    if (s->refresh > 1) CU(cudaMemsetAsync(s->d_force_direct, 1, (size_t)s->n_model * sizeof(int), s->stream));
    return GFB_OK;
}

// A snapshot: the recording cells' records [field][rec][NN][15], then the
// same values merged per recording node [field][node][15].
size_t snapshot_cell_values(const gfb_solver* s) { return (size_t)s->nfld * s->n_rec * s->nn * 15; }
size_t snapshot_values(const gfb_solver* s) {
    return snapshot_cell_values(s) + (size_t)s->nfld * s->n_unique * 15;
}
size_t snapshot_bytes(const gfb_solver* s) { return snapshot_values(s) * (s->rec_f32 ? 4 : 8); }

// Convert n snapshot values starting at value `off` of a raw snapshot
// (float or double, as recorded) to double.
// Scatter n_out recorded points of 15 values (strain 6, u 3, v 3, a 3) into
// the caller's arrays: output point q takes the 15 values at
// raw + src_index(q) * 15 (float or double as recorded).  Threads split the
// points; a NULL array is skipped.
template <typename Index, typename Out>
void unpack_points(const gfb_solver* s, const void* raw, long long n_out, Index src_index, Out* strain, Out* u,
                   Out* v, Out* a) {
    auto run = [&](auto* src) {
        parallel_for(n_out, [&](long long q0, long long q1) {
            for (long long q = q0; q < q1; ++q) {
                const auto* o = src + (size_t)src_index(q) * 15;
                if (strain)
                    for (int c = 0; c < 6; ++c) strain[q * 6 + c] = (Out)o[c];
                for (int c = 0; c < 3; ++c) {
                    if (u) u[q * 3 + c] = (Out)o[6 + c];
                    if (v) v[q * 3 + c] = (Out)o[9 + c];
                    if (a) a[q * 3 + c] = (Out)o[12 + c];
                }
            }
        }, 16384);
    };
    if (s->rec_f32) run(static_cast<const float*>(raw));
    else run(static_cast<const double*>(raw));
}

// Copy a snapshot out of its pinned slot into pageable memory, as recorded,
// so the slot can take a new snapshot (only when the caller has not read it
// yet).
gfb_status spill(gfb_solver* s, Snapshot& snap) {
    CU(cudaEventSynchronize(s->copy_evt[snap.slot]));
    const size_t n = snapshot_bytes(s);
    snap.host.reset(new unsigned char[n]);  // no zero fill: every byte is copied below
    unsigned char* dst = snap.host.get();
    const unsigned char* src = static_cast<const unsigned char*>(s->pinned[snap.slot]);
    const size_t chunk = 1 << 16;
    parallel_for((long long)((n + chunk - 1) / chunk), [&](long long c0, long long c1) {
        const size_t b0 = (size_t)c0 * chunk, b1 = std::min(n, (size_t)c1 * chunk);
        std::memcpy(dst + b0, src + b0, b1 - b0);
    }, 32);
    snap.slot = -1;
    return GFB_OK;
}

// ---------------------------------------------------------------------------
// solver construction
// ---------------------------------------------------------------------------

// C-PML at global nodes: B_k = sum over C-PML cells at the node of
// w J/rho A_k (k = 1..5, accumulated in FP64 in cell order), and for each
// axis the convolution coefficients of the cells where that axis acts.
// live_pts[t]: the live C-PML points (some A_k != 0) of owner t's nodes in
// increasing point order, so each owner thread accumulates its nodes in mesh
// order; the slot of node g is its device index (the C-PML nodes are the
// first n_slot device nodes); coef is [slot][14].  Returns false (per-cell
// form) if two cells disagree on an axis's coefficients at a shared node
// (beyond 1e-6 relative).
bool accumulate_node_pml(const gfb_solver* s, const gfb_mesh* m, const std::vector<double>& w,
                         const std::vector<std::vector<long long>>& live_pts, int n_slot, std::vector<double>& coef) {
    const int ng = s->ng, nn = s->nn;
    coef.assign((size_t)n_slot * 14, 0.0);
    std::vector<unsigned char> have(n_slot, 0);
    std::atomic<bool> agree(true);
    std::vector<std::thread> th;
    for (size_t t = 0; t < live_pts.size(); ++t)
        th.emplace_back([&, t] {
            for (const long long q : live_pts[t]) {
                const int p = (int)(q % nn);
                const double* A = m->pml_coef_abar + q * 5;
                const int g = m->ibool[q];
                const int sl = s->node_inv.empty() ? g : s->node_inv[g];
                double* c = &coef[(size_t)sl * 14];
                const int nk = p % ng, nj = (p / ng) % ng, ni = p / (ng * ng);
                const double wgll = w[ni] * w[nj] * w[nk];
                const double rho = m->density[q];
                const double scale = wgll * ((rho > 0.0) ? 1.0 / rho : 0.0) * m->jacobian[q];
                for (int kk = 0; kk < 5; ++kk) c[kk] += scale * A[kk];
                const double* al = m->pml_coef_alpha + q * 9;
                for (int ax = 0; ax < 3; ++ax) {
                    if (A[2 + ax] == 0.0) continue;
                    if (!(have[sl] & (1u << ax))) {
                        for (int k = 0; k < 3; ++k) c[5 + ax * 3 + k] = al[ax * 3 + k];
                        have[sl] |= (unsigned char)(1u << ax);
                    } else {
                        for (int k = 0; k < 3; ++k) {
                            const double a0 = c[5 + ax * 3 + k], a1 = al[ax * 3 + k];
                            // the cells' coefficients at a node come from the same position
                            // through different cell maps: equal up to rounding (seen up to
                            // ~1e-9 relative on deformed meshes); different profiles differ
                            // at O(1)
                            if (std::abs(a0 - a1) > 1e-6 * std::max(std::abs(a0), std::abs(a1))) {
                                agree.store(false);
                                return;
                            }
                        }
                    }
                }
            }
        });
    for (auto& x : th) x.join();
    return agree.load();
}

// Upload the node-form C-PML: the C-PML nodes are device nodes [0, n)
// (slot = device node), coefficients [slot][14], memory [axis][slot][F]
// and the previous field [slot][F], both zero.
template <typename Real>
gfb_status upload_node_pml(gfb_solver* s, const std::vector<double>& coef) {
    gfb_status st;
    const int n = (int)(coef.size() / 14);
    Real* dc = nullptr;
    if ((st = s->alloc(&dc, (size_t)std::max(n, 1) * 14))) return st;
    st = staged_upload(s, dc, 14 * sizeof(Real), n, [&](long long i0, long long i1, unsigned char* out) {
        Real* o = reinterpret_cast<Real*>(out);
        parallel_for((i1 - i0) * 14, [&](long long a0, long long a1) {
            for (long long i = a0; i < a1; ++i) o[i] = (Real)coef[(size_t)i0 * 14 + i];
        });
    });
    if (st) return st;
    s->npml_coef = dc;
    Real *mem = nullptr, *prev = nullptr;
    if ((st = s->alloc(&mem, (size_t)std::max(n, 1) * s->F * 3))) return st;
    if ((st = s->alloc(&prev, (size_t)std::max(n, 1) * s->F))) return st;
    CU(cudaMemset(mem, 0, (size_t)std::max(n, 1) * s->F * 3 * sizeof(Real)));
    CU(cudaMemset(prev, 0, (size_t)std::max(n, 1) * s->F * sizeof(Real)));
    s->npml_mem = mem;
    s->npml_prev = prev;
    s->n_pml_node = n;
    s->node_pml = true;
    return GFB_OK;
}

template <typename Real>
gfb_status build_device(gfb_solver* s, const gfb_mesh* m, const gfb_source* src, int n_model,
                        const gfb_model* models, const std::vector<int>& perm, const std::vector<int>& inv_perm,
                        const std::vector<uint32_t>& ibool_dev, const std::vector<double>& node_mass,
                        const std::vector<double>& node_damp, const std::vector<long long>& first_q,
                        std::vector<uint8_t>& first_flag, const std::vector<uint8_t>& node_live,
                        const std::vector<std::vector<long long>>& live_pts, const std::vector<double>& w,
                        const std::vector<double>& D, StageClock& clk) {
    const int ng = s->ng, nn = s->nn;
    const long long n_cell = s->n_cell;
    gfb_status st;
    std::lock_guard<std::mutex> staging_lock(staging().mu);
    PinnedRing host_ring;
    // recording nodes: unique node ids in ascending order (the recording
    // map's gll_node_ids), each node's (cell, point) occurrences, and the
    // mass of each occurrence as the merge weight
    if (s->n_rec > 0) {
        std::vector<std::pair<int, int>> occ;  // (node, record index)
        occ.reserve((size_t)s->n_rec * nn);
        for (int ci = 0; ci < s->n_rec; ++ci)
            for (int p = 0; p < nn; ++p)
                occ.push_back({m->ibool[(size_t)m->rec_cell_local[ci] * nn + p], ci * nn + p});
        std::sort(occ.begin(), occ.end());
        std::vector<int> ptr{0}, idx;
        std::vector<double> wts;
        s->rec_node_ids.clear();
        for (size_t k = 0; k < occ.size(); ++k) {
            if (k == 0 || occ[k].first != occ[k - 1].first) {
                if (k) ptr.push_back((int)k);
                s->rec_node_ids.push_back(occ[k].first);
            }
            idx.push_back(occ[k].second);
            const int ci = occ[k].second / nn, p = occ[k].second - ci * nn;
            wts.push_back(m->mass[(size_t)m->rec_cell_local[ci] * nn + p]);
        }
        ptr.push_back((int)occ.size());
        s->n_unique = (int)s->rec_node_ids.size();
        if ((st = s->alloc(&s->gf_ptr, ptr.size())) || (st = h2d(s, s->gf_ptr, ptr.data(), ptr.size() * 4))) return st;
        if ((st = s->alloc(&s->gf_occ, idx.size())) || (st = h2d(s, s->gf_occ, idx.data(), idx.size() * 4))) return st;
        if ((st = s->alloc(&s->gf_w, wts.size())) || (st = h2d(s, s->gf_w, wts.data(), wts.size() * 8))) return st;
    }
    // the snapshot size is known now: pin the host ring meanwhile
    if (s->n_rec > 0) host_ring.start(s->device, s->slots, snapshot_bytes(s));
    clk.mark("recording nodes");
    // C-PML at global nodes (FP32 path) when the cells agree at shared nodes.
    // Device node order: the node-form C-PML nodes first (so they are device
    // nodes [0, n_pml_node)), then the others; within each, nodes in the
    // order cells (in mesh order) first touch them, so the nodes of a cell
    // and of its neighbours sit close in memory whatever the input
    // numbering (the reference's coordinate sort scatters them on deformed
    // meshes)
    // first_flag[q]: 1 if q is its node's first touch, 2 if that node is a
    // live C-PML node numbered first
    auto number_nodes = [&](bool pml_first) {
        s->node_perm.clear();
        s->node_inv.clear();
        s->node_perm.reserve(s->n_node);
        const long long P = n_cell * nn;
        parallel_for(s->n_node, [&](long long g0, long long g1) {
            for (long long g = g0; g < g1; ++g)
                if (first_q[g] >= 0) first_flag[first_q[g]] = (pml_first && node_live[g]) ? 2 : 1;
        });
        auto node_of = [&](long long q) { return m->ibool[q]; };
        for (int pass = pml_first ? 0 : 1; pass < 2; ++pass) {
            const uint8_t want = pass == 0 ? 2 : 1;
            parallel_compact(P, [&](long long q) { return first_flag[q] == want; }, node_of, s->node_perm);
        }
        parallel_compact(s->n_node, [&](long long g) { return first_q[g] < 0; },  // nodes no cell uses
                         [](long long g) { return (int)g; }, s->node_perm);
        std::atomic<bool> ident(true);
        parallel_for(s->n_node, [&](long long d0, long long d1) {
            for (long long d = d0; d < d1; ++d)
                if (s->node_perm[d] != (int)d) {
                    ident.store(false);
                    return;
                }
        });
        if (ident.load()) {
            s->node_perm.clear();
        } else {
            s->node_inv.assign(s->n_node, 0);
            parallel_for(s->n_node, [&](long long d0, long long d1) {
                for (long long d = d0; d < d1; ++d) s->node_inv[s->node_perm[d]] = (int)d;
            });
        }
    };
    // node-form C-PML (FP32 path): its nodes are numbered first and its
    // coefficients accumulated straight into their device slots; if two
    // cells disagree at a node, the per-cell form is used and the nodes are
    // numbered again without the C-PML group
    bool node_form = !node_live.empty();
    number_nodes(node_form);
    clk.mark("node numbering");
    std::vector<double> pcoef;
    if (node_form) {
        long long n_live = 0;
        for (size_t g = 0; g < node_live.size(); ++g) n_live += node_live[g];
        if (!accumulate_node_pml(s, m, w, live_pts, (int)n_live, pcoef)) {
            node_form = false;
            pcoef.clear();
            number_nodes(false);
        }
    }
    clk.mark("C-PML node plan");
    auto dev_node = [&](long long g) -> long long { return s->node_inv.empty() ? g : s->node_inv[g]; };
    // ibool in device node numbers, and the rows of the pipelined kernels:
    // node words, then the cell's model, zero padding
    {
        auto dev_word = [&](uint32_t x) {
            return s->node_inv.empty() ? x
                                       : (x & ~gfb::kNodeMask) | (uint32_t)s->node_inv[x & gfb::kNodeMask];
        };
        uint32_t* d = nullptr;
        if ((st = s->alloc(&d, (size_t)n_cell * nn))) return st;
        st = staged_upload(s, d, (size_t)nn * 4, n_cell, [&](long long e0, long long e1, unsigned char* out) {
            uint32_t* o = reinterpret_cast<uint32_t*>(out);
            parallel_for(e1 - e0, [&](long long a0, long long a1) {
                for (long long i = a0 * nn; i < a1 * nn; ++i) o[i] = dev_word(ibool_dev[e0 * nn + i]);
            }, 1024);
        });
        if (st) return st;
        s->ibool = d;
        const int nnp = gfb::ib_row_words(nn);
        uint32_t* dp = nullptr;
        if ((st = s->alloc(&dp, (size_t)n_cell * nnp))) return st;
        st = staged_upload(s, dp, (size_t)nnp * 4, n_cell, [&](long long e0, long long e1, unsigned char* out) {
            uint32_t* o = reinterpret_cast<uint32_t*>(out);
            parallel_for(e1 - e0, [&](long long a0, long long a1) {
                for (long long i = a0; i < a1; ++i) {
                    const long long e = e0 + i;
                    uint32_t* row = o + i * nnp;
                    for (int p = 0; p < nn; ++p) row[p] = dev_word(ibool_dev[e * nn + p]);
                    int mi = 0;
                    while (perm[e] >= models[mi].cell_end) ++mi;
                    row[nn] = (uint32_t)mi;
                    for (int p = nn + 1; p < nnp; ++p) row[p] = 0u;
                }
            }, 1024);
        });
        if (st) return st;
        s->ibool_padded = dp;
    }
    clk.mark("ibool upload");
    // geometry [cell][12][NN] in colour order
    {
        Real* dg = nullptr;
        if ((st = s->alloc(&dg, (size_t)n_cell * 12 * nn))) return st;
        st = staged_upload(s, dg, (size_t)12 * nn * sizeof(Real), n_cell,
                           [&](long long e0, long long e1, unsigned char* out) {
            parallel_for(e1 - e0, [&](long long a0, long long a1) {
                for (long long i = a0; i < a1; ++i) {
                    const long long e = perm[e0 + i];
                    Real* o = reinterpret_cast<Real*>(out) + i * 12 * nn;
                    for (int p = 0; p < nn; ++p) {
                        const long long q = e * nn + p;
                        for (int f = 0; f < 9; ++f) o[f * nn + p] = (Real)m->dxi_dx[q * 9 + f];
                        const int i0 = p / (ng * ng), j = (p / ng) % ng, k = p % ng;
                        // factor = detJ * w_i * w_j * w_k (element_cpu.cpp:108)
                        o[9 * nn + p] = (Real)(m->jacobian[q] * w[i0] * w[j] * w[k]);
                        o[10 * nn + p] = (Real)m->lambda_[q];
                        o[11 * nn + p] = (Real)m->mu[q];
                    }
                }
            }, 256);
        });
        if (st) return st;
        s->geom = dg;
    }
    clk.mark("geometry upload");
    {
        std::vector<Real> d(D.size());
        for (size_t i = 0; i < D.size(); ++i) d[i] = (Real)D[i];
        for (size_t i = 0; i < D.size() && i < 36; ++i) s->dmat_host[i] = (float)D[i];
        if ((st = upload(s, &s->dmat, d))) return st;
    }
    const long long nF = (long long)s->n_node * s->F;
    const long long nP = (long long)s->n_node * s->nfld * 4;  // [node][field][4]
    if ((st = s->alloc(&s->u, nF))) return st;
    if ((st = s->alloc(&s->v, nF))) return st;
    Real* a = nullptr;
    Real* ut = nullptr;
    Real* force = nullptr;
    if ((st = s->alloc(&a, nF))) return st;
    if ((st = s->alloc(&ut, nP))) return st;
    if ((st = s->alloc(&force, nP))) return st;
    s->a = a;
    s->ut = ut;
    s->force = force;
    CU(cudaMemset(s->u, 0, nF * sizeof(double)));
    CU(cudaMemset(s->v, 0, nF * sizeof(double)));
    CU(cudaMemset(a, 0, nF * sizeof(Real)));
    CU(cudaMemset(ut, 0, nP * sizeof(Real)));
    CU(cudaMemset(force, 0, nP * sizeof(Real)));
    clk.mark("state arrays");
    // lumped mass, 1/m (FP32 path; 0 marks m <= 0) and damping in device
    // order, gathered by the host threads straight into the pinned chunks
    auto gathered = [&](void* dst, size_t es, auto value) -> gfb_status {
        return staged_upload(s, dst, es, s->n_node, [&](long long i0, long long i1, unsigned char* out) {
            parallel_for(i1 - i0, [&](long long a0, long long a1) {
                for (long long i = a0; i < a1; ++i) {
                    const long long d = i0 + i;
                    value(s->node_perm.empty() ? d : (long long)s->node_perm[d], out + (size_t)i * es);
                }
            }, 65536);
        });
    };
    {
        double* d = nullptr;
        if ((st = s->alloc(&d, (size_t)s->n_node))) return st;
        if ((st = gathered(d, 8, [&](long long g, unsigned char* o) { std::memcpy(o, &node_mass[g], 8); }))) return st;
        s->mass = d;
    }
    if (s->prec == GFB_FP32) {
        Real* d = nullptr;
        if ((st = s->alloc(&d, (size_t)s->n_node))) return st;
        st = gathered(d, sizeof(Real), [&](long long g, unsigned char* o) {
            const Real im = node_mass[g] > 0.0 ? (Real)(1.0 / node_mass[g]) : Real(0);
            std::memcpy(o, &im, sizeof(Real));
        });
        if (st) return st;
        s->inv_mass = d;
    }
    if (s->has_damping) {
        double* d = nullptr;
        if ((st = s->alloc(&d, (size_t)s->n_node))) return st;
        if ((st = gathered(d, 8, [&](long long g, unsigned char* o) { std::memcpy(o, &node_damp[g], 8); }))) return st;
        s->damping = d;
    }
    clk.mark("mass and damping");
    if (node_form && (st = upload_node_pml<Real>(s, pcoef))) return st;
    // C-PML per cell
    if (s->has_cpml && !s->node_pml) {
        std::vector<int> slot(n_cell, -1);
        std::vector<long long> slot_cell;
        for (long long ed = 0; ed < n_cell; ++ed)
            if (m->pml_region[perm[ed]] != 0) {
                slot[ed] = (int)slot_cell.size();
                slot_cell.push_back(perm[ed]);
            }
        s->n_pml = (int)slot_cell.size();
        {
            int* d = nullptr;
            if ((st = s->alloc(&d, slot.size()))) return st;
            if ((st = h2d(s, d, slot.data(), slot.size() * 4))) return st;
            s->pml_slot = d;
        }
        Real* dcoef = nullptr;
        if ((st = s->alloc(&dcoef, (size_t)s->n_pml * 15 * nn))) return st;
        st = staged_upload(s, dcoef, (size_t)15 * nn * sizeof(Real), s->n_pml,
                           [&](long long s0, long long s1, unsigned char* out) {
          parallel_for(s1 - s0, [&](long long a0, long long a1) {
            for (long long i = a0; i < a1; ++i) {
                const long long e = slot_cell[s0 + i];
                Real* o = reinterpret_cast<Real*>(out) + i * 15 * nn;
                for (int p = 0; p < nn; ++p) {
                    const long long q = e * nn + p;
                    for (int f = 0; f < 9; ++f) o[f * nn + p] = (Real)m->pml_coef_alpha[q * 9 + f];
                    for (int f = 0; f < 5; ++f) o[(9 + f) * nn + p] = (Real)m->pml_coef_abar[q * 5 + f];
                    const int nk = p % ng, nj = (p / ng) % ng, ni = p / (ng * ng);
                    const double wgll = w[ni] * w[nj] * w[nk];  // pml.cpp:171-174
                    const double rho = m->density[q];
                    const double rho_inv = (rho > 0.0) ? 1.0 / rho : 0.0;
                    o[14 * nn + p] = (Real)(wgll * rho_inv * m->jacobian[q]);
                }
            }
          }, 256);
        });
        if (st) return st;
        s->pml_coef = dcoef;
        Real *mem = nullptr, *prev = nullptr;
        if ((st = s->alloc(&mem, (size_t)s->n_pml * s->F * 3 * nn))) return st;
        if ((st = s->alloc(&prev, (size_t)s->n_pml * s->F * nn))) return st;
        CU(cudaMemset(mem, 0, (size_t)s->n_pml * s->F * 3 * nn * sizeof(Real)));
        CU(cudaMemset(prev, 0, (size_t)s->n_pml * s->F * nn * sizeof(Real)));
        s->pml_mem = mem;
        s->pml_prev = prev;
    }
    clk.mark("C-PML arrays");
    // source: cells located by id (solver.cpp:250-258), chained per cell;
    // the slots of every source set (one per source position) in one list,
    // each slot tagged with its set
    {
        long long n_slot = 0;
        for (const auto& ss : s->sets) n_slot += std::max(0, ss.n_src_cell);
        if (n_slot > 0) {
            std::unordered_map<long long, long long> cell_of;
            cell_of.reserve((size_t)n_cell * 2);
            for (long long e = n_cell - 1; e >= 0; --e) cell_of[m->cell_ids ? m->cell_ids[e] : e] = e;
            std::vector<int> head(n_cell, -1), next(n_slot, -1), tail(n_cell, -1), set_of(n_slot, 0);
            std::vector<Real> wts((size_t)n_slot * nn, Real(0));
            int used = 0;
            long long si = 0;
            for (int k = 0; k < (int)s->sets.size(); ++k) {
                const gfb_source& ss = s->sets[k];
                for (int q = 0; q < ss.n_src_cell; ++q, ++si) {
                    set_of[si] = k;
                    auto it = cell_of.find(ss.cell_ids[q]);  // the first cell with the id
                    if (it == cell_of.end()) continue;       // not in this mesh (reference: -1, skipped)
                    const int ed = inv_perm[it->second];
                    for (int p = 0; p < nn; ++p) wts[(size_t)si * nn + p] = (Real)ss.weights[(size_t)q * nn + p];
                    if (head[ed] < 0) head[ed] = (int)si;
                    else next[tail[ed]] = (int)si;
                    tail[ed] = (int)si;
                    ++used;
                }
            }
            s->has_src = used > 0;
            s->n_src = (int)n_slot;
            int *dh = nullptr, *dn = nullptr;
            if ((st = s->alloc(&dh, head.size()))) return st;
            if ((st = s->alloc(&dn, next.size()))) return st;
            if ((st = h2d(s, dh, head.data(), head.size() * 4))) return st;
            if ((st = h2d(s, dn, next.data(), next.size() * 4))) return st;
            s->src_head = dh;
            s->src_next = dn;
            if ((st = upload(s, &s->src_w, wts))) return st;
            if (s->n_set > 1) {
                if ((st = s->alloc(&s->src_set, set_of.size()))) return st;
                if ((st = h2d(s, s->src_set, set_of.data(), set_of.size() * 4))) return st;
            }
        }
    }
    clk.mark("source");
    // models: constants, step counters, source time functions
    {
        // source time function series: one per model, or one per source
        // set of the single model (series q = model * n_set + set)
        const int n_series = n_model * s->n_set;
        std::vector<gfb::ModelConst> mc(n_model);
        std::vector<int> nsteps(n_model), nstf(n_series), zero(n_model, 0), one(n_model, 1);
        std::vector<long long> off(n_series);
        std::vector<Real> stf_all, mstf(n_series, Real(0));
        const double theta = 1.0 / 8.0;  // pml.cpp:35, 63-64
        for (int k = 0; k < n_model; ++k) {
            const double dt = models[k].dt;
            mc[k] = gfb::ModelConst{dt, 0.5 * dt * dt, (1.0 - 2.0 * theta) * 0.5 * dt, (1.0 - theta) * 0.5 * dt * dt};
            nsteps[k] = models[k].n_steps;
        }
        for (int q = 0; q < n_series; ++q) {
            const int n = s->stf_from_sets ? s->sets[q].n_stf : models[q].n_stf;
            const double* v = s->stf_from_sets ? s->sets[q].stf : models[q].stf;
            nstf[q] = std::max(0, n);
            off[q] = (long long)stf_all.size();
            for (int t = 0; t < nstf[q]; ++t) stf_all.push_back((Real)v[t]);
        }
        s->model_nsteps = nsteps;
        if (stf_all.empty()) stf_all.push_back(Real(0));
        auto put_int = [&](int** d, const std::vector<int>& h) -> gfb_status {
            gfb_status r;
            if ((r = s->alloc(d, h.size()))) return r;
            return h2d(s, *d, h.data(), h.size() * 4);
        };
        if ((st = s->alloc(&s->d_mc, mc.size()))) return st;
        if ((st = h2d(s, s->d_mc, mc.data(), mc.size() * sizeof(gfb::ModelConst)))) return st;
        if ((st = put_int(&s->d_nsteps, nsteps))) return st;
        if ((st = put_int(&s->d_nstf, nstf))) return st;
        if ((st = put_int(&s->d_mstep, zero))) return st;
        if ((st = put_int(&s->d_mlive, one))) return st;
        if ((st = put_int(&s->d_mdirect, one))) return st;
        if ((st = put_int(&s->d_mnext, one))) return st;
        if ((st = put_int(&s->d_force_direct, zero))) return st;
        if ((st = put_int(&s->d_kernel_err, std::vector<int>(1, 0)))) return st;
        if ((st = s->alloc(&s->d_stf_off, off.size()))) return st;
        if ((st = h2d(s, s->d_stf_off, off.data(), off.size() * 8))) return st;
        if ((st = upload(s, &s->d_stf_all, stf_all))) return st;
        if ((st = upload(s, &s->d_mstf, mstf))) return st;
        if (n_model > 1) {
            std::vector<uint8_t> nm(s->n_node, 0);
            for (int k = 0; k < n_model; ++k)
                for (int g = models[k].node_begin; g < models[k].node_end; ++g) nm[dev_node(g)] = (uint8_t)k;
            if ((st = s->alloc(&s->d_node_model, nm.size()))) return st;
            if ((st = h2d(s, s->d_node_model, nm.data(), nm.size()))) return st;
            // ends of each model's cells per colour and nodes per range
            const int nc = (int)s->colour_begin.size() - 1;
            const long long g0 = s->node_pml ? s->n_pml_node : 0;
            std::vector<int> cell_end((size_t)n_model * nc), first(nc), live_cell(nc);
            for (int k = 0; k < n_model; ++k)
                for (int c = 0; c < nc; ++c) cell_end[(size_t)k * nc + c] = s->colour_begin[c];
            for (int c = 0; c < nc; ++c) {
                first[c] = s->colour_begin[c];
                live_cell[c] = s->colour_begin[c + 1];
                for (int ed = s->colour_begin[c]; ed < s->colour_begin[c + 1]; ++ed) {
                    int mi = 0;
                    while (perm[ed] >= models[mi].cell_end) ++mi;
                    cell_end[(size_t)mi * nc + c] = ed + 1;
                }
            }
            std::vector<long long> node_end((size_t)n_model * 2), live_node{g0, (long long)s->n_node};
            for (int k = 0; k < n_model; ++k) {
                node_end[(size_t)k * 2] = 0;
                node_end[(size_t)k * 2 + 1] = g0;
            }
            for (long long d = 0; d < s->n_node; ++d) {
                long long& e = node_end[(size_t)nm[d] * 2 + (d < g0 ? 0 : 1)];
                e = std::max(e, d + 1);
            }
            auto put = [&](auto** dst, const auto& h) -> gfb_status {
                gfb_status r;
                if ((r = s->alloc(dst, h.size()))) return r;
                return h2d(s, *dst, h.data(), h.size() * sizeof(h[0]));
            };
            if ((st = put(&s->d_cell_end, cell_end)) || (st = put(&s->d_colour_first, first)) ||
                (st = put(&s->d_live_cell_end, live_cell)) || (st = put(&s->d_node_end, node_end)) ||
                (st = put(&s->d_live_node_end, live_node)))
                return st;
        }
    }
    if (s->node_pml) {
        s->n_pml = 0;
        for (long long e = 0; e < n_cell; ++e) s->n_pml += m->pml_region[e] != 0;
    }
    clk.mark("models");
    // recording cells and snapshot ring
    if (s->n_rec > 0) {
        std::vector<int> rc(s->n_rec);
        for (int ci = 0; ci < s->n_rec; ++ci) rc[ci] = inv_perm[m->rec_cell_local[ci]];
        int* d = nullptr;
        if ((st = s->alloc(&d, rc.size()))) return st;
        if ((st = h2d(s, d, rc.data(), rc.size() * 4))) return st;
        s->rec_cell = d;
        unsigned char* ring = nullptr;
        if ((st = s->alloc(&ring, snapshot_bytes(s) * s->slots))) return st;
        s->ring = ring;
        s->rec_evt.assign(s->slots, nullptr);
        s->copy_evt.assign(s->slots, nullptr);
        s->copy_issued.assign(s->slots, 0);
        for (int k = 0; k < s->slots; ++k) {
            CU(cudaEventCreateWithFlags(&s->rec_evt[k], cudaEventDisableTiming));
            CU(cudaEventCreateWithFlags(&s->copy_evt[k], cudaEventDisableTiming));
        }
        CU(host_ring.finish());
        s->pinned = host_ring.slot;  // the solver frees them from here on
        host_ring.taken = true;
    }
    clk.mark("snapshot ring");
    return GFB_OK;
}

gfb_status validate(const gfb_mesh* m, const gfb_config* c) {
    if (!m || !c) return fail(GFB_ERR_INVALID, "mesh and config are required");
    if (m->ngll < 3 || m->ngll > 6)
        return fail(GFB_ERR_UNSUPPORTED, "ngll=%d outside the supported 3..6", m->ngll);
    if (m->n_cell <= 0) return fail(GFB_ERR_INVALID, "n_cell must be positive (got %d)", m->n_cell);
    if (m->n_node <= 0 || (uint32_t)m->n_node > gfb::kNodeMask)
        return fail(GFB_ERR_INVALID, "n_node=%d out of range", m->n_node);
    if (!m->ibool || !m->dxi_dx || !m->jacobian || !m->lambda_ || !m->mu || !m->mass)
        return fail(GFB_ERR_INVALID, "ibool, dxi_dx, jacobian, lambda, mu and mass are required");
    if (m->pml_coef_abar && (!m->pml_region || !m->pml_coef_alpha || !m->density))
        return fail(GFB_ERR_INVALID, "C-PML needs pml_region, pml_coef_alpha and density");
    if (!(c->dt > 0.0)) return fail(GFB_ERR_INVALID, "dt must be positive");
    if (c->precision != GFB_FP64 && c->precision != GFB_FP32)
        return fail(GFB_ERR_INVALID, "unknown precision %d", c->precision);
    if (c->n_field < 1 || c->n_field > 3) return fail(GFB_ERR_INVALID, "n_field must be 1..3");
    for (int d = 0; d < c->n_field; ++d)
        if (c->field_dir[d] < 0 || c->field_dir[d] > 2)
            return fail(GFB_ERR_INVALID, "field_dir[%d]=%d must be 0, 1 or 2", d, c->field_dir[d]);
    if (m->n_rec_cell < 0 || (m->n_rec_cell > 0 && !m->rec_cell_local))
        return fail(GFB_ERR_INVALID, "bad recording map");
    for (int ci = 0; ci < m->n_rec_cell; ++ci)
        if (m->rec_cell_local[ci] < 0 || m->rec_cell_local[ci] >= m->n_cell)
            return fail(GFB_ERR_INVALID, "rec_cell_local[%d]=%d out of range", ci, m->rec_cell_local[ci]);
    return GFB_OK;
}


template <typename Real>
gfb_status launch_step_begin_t(gfb_solver* s) {
    const int threads = 128;
    const int blocks = (s->n_model + threads - 1) / threads;
    gfb::step_begin_kernel<Real><<<blocks, threads, 0, s->stream>>>(
        s->n_model, s->n_set, s->d_mstep, s->d_nsteps, s->d_nstf, s->d_stf_off, static_cast<const Real*>(s->d_stf_all),
        static_cast<Real*>(s->d_mstf), s->d_mlive, s->refresh, s->d_force_direct,
        s->refresh > 1 ? s->d_mdirect : nullptr, s->d_mnext);
    CU(cudaGetLastError());
    s->launches++;
    if (s->d_live_cell_end) {
        const int nc = (int)s->colour_begin.size() - 1;
        gfb::live_bounds_kernel<<<1, 128, 0, s->stream>>>(s->n_model, nc, s->d_mlive, s->d_cell_end,
                                                          s->d_colour_first, s->d_node_end,
                                                          s->node_pml ? (long long)s->n_pml_node : 0LL,
                                                          s->d_live_cell_end, s->d_live_node_end);
        CU(cudaGetLastError());
        s->launches++;
    }
    return GFB_OK;
}

// The device work of one step: step start, NC colour launches, node pass.
// With ev != nullptr, events 0..2 bracket the element and node phases.
gfb_status step_body(gfb_solver* s, cudaEvent_t* ev) {
    gfb_status st;
    const int n_colour = (int)s->colour_begin.size() - 1;
    if (ev) CU(cudaEventRecord(ev[0], s->stream));
    st = s->prec == GFB_FP64 ? launch_step_begin_t<double>(s) : launch_step_begin_t<float>(s);
    if (st) return st;
    for (int c = 0; c < n_colour; ++c)
        if ((st = launch_elem(s, c))) return st;
    if (s->layer && (st = gfb::layer_step(s, s->layer))) return st;
    if (ev) CU(cudaEventRecord(ev[1], s->stream));
    if (!s->fuse)
        if ((st = launch_node(s))) return st;
    if (ev) CU(cudaEventRecord(ev[2], s->stream));
    return GFB_OK;
}

// Capture step_body once as a CUDA graph; every argument it launches with
// (device pointers, colour ranges, grid sizes) is fixed for the solver's
// lifetime, and the step-dependent values live on the device.
gfb_status capture_step(gfb_solver* s) {
    const long long l0 = s->launches;
    CU(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    gfb_status st = step_body(s, nullptr);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return fail(GFB_ERR_CUDA, "step capture failed: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&s->gexec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(GFB_ERR_CUDA, "step graph instantiation failed: %s", cudaGetErrorString(ei));
    s->graph_launches = s->launches - l0;
    s->launches = l0;
    return GFB_OK;
}

// One solver step: the device work (a graph launch, or eager launches when
// phases are timed), then the snapshot when the step is a snapshot step.
gfb_status one_step(gfb_solver* s, cudaEvent_t* ev) {
    gfb_status st;
    const int step = s->step;
    if (!ev && s->use_graph) {
        if (!s->gexec && (st = capture_step(s))) return st;
        CU(cudaGraphLaunch(s->gexec, s->stream));
        s->launches += s->graph_launches;
    } else if ((st = step_body(s, ev))) {
        return st;
    }
    if (s->stride > 0 && s->n_rec > 0 && step % s->stride == 0) {
        // round-robin slot; an unread snapshot still in it moves to pageable
        // memory first.  The record kernel waits (on the GPU) for the last
        // device->host copy out of the slot; the copy of this snapshot runs
        // on the copy stream, overlapped with the following steps.
        // keep the host at most half the ring ahead of the snapshot copies, so
        // a reader thread gets the time to release a slot before it is
        // needed again (replayed steps are queued much faster than they run)
        const int slot = s->next_slot;
        if (s->slots > 1) {
            const int back = (slot - s->slots / 2 + s->slots) % s->slots;
            if (s->copy_issued[back]) CU(cudaEventSynchronize(s->copy_evt[back]));
        }
        std::unique_lock<std::mutex> lk(s->rec_mu);
        s->next_slot = (s->next_slot + 1) % s->slots;
        for (;;) {
            // the unread snapshot still in this slot, looked up again after
            // every wait (a reader may have released and removed it)
            while (!s->pending.empty() && s->pending.front().done && s->pending.front().readers == 0)
                s->pending.pop_front();
            Snapshot* old = nullptr;
            for (auto& p : s->pending)
                if (p.slot == slot) {
                    old = &p;
                    break;
                }
            if (!old) break;
            if (old->readers > 0) {
                s->rec_cv.wait(lk);  // a reader is copying it out
                continue;
            }
            if ((st = spill(s, *old))) return st;
        }
        if (s->copy_issued[slot]) CU(cudaStreamWaitEvent(s->stream, s->copy_evt[slot], 0));
        void* dslot = static_cast<unsigned char*>(s->ring) + (size_t)slot * snapshot_bytes(s);
        if ((st = launch_record(s, dslot))) return st;
        {
            const long long total = (long long)s->nfld * s->n_unique * 15;
            const int grid = grid_for(total, 256);
            const long long per_field = (long long)s->n_rec * s->nn * 15;
            if (s->rec_f32)
                gfb::merge_nodes_kernel<float><<<grid, 256, 0, s->stream>>>(s->nfld, s->n_unique, per_field, s->gf_ptr,
                                                                              s->gf_occ, s->gf_w, static_cast<float*>(dslot));
            else
                gfb::merge_nodes_kernel<double><<<grid, 256, 0, s->stream>>>(
                    s->nfld, s->n_unique, per_field, s->gf_ptr, s->gf_occ, s->gf_w, static_cast<double*>(dslot));
            CU(cudaGetLastError());
            s->launches++;
        }
        CU(cudaEventRecord(s->rec_evt[slot], s->stream));
        CU(cudaStreamWaitEvent(s->copy_stream, s->rec_evt[slot], 0));
        CU(cudaMemcpyAsync(s->pinned[slot], dslot, snapshot_bytes(s), cudaMemcpyDeviceToHost, s->copy_stream));
        CU(cudaEventRecord(s->copy_evt[slot], s->copy_stream));
        s->copy_issued[slot] = 1;
        Snapshot snap;
        snap.step = step;
        snap.slot = slot;
        snap.read_mask.assign(s->nfld, 0);
        s->pending.push_back(std::move(snap));
    }
    if (ev) CU(cudaEventRecord(ev[3], s->stream));
    s->step++;
    s->a_in_force = true;
    return GFB_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int32_t gfb_abi_version(void) { return GFB_ABI_VERSION; }

gfb_status gfb_device_count(int32_t* n) {
    if (!n) return fail(GFB_ERR_INVALID, "device count: NULL output");
    int k = 0;
    if (cudaGetDeviceCount(&k) != cudaSuccess) k = 0;
    *n = k;
    return GFB_OK;
}

gfb_status gfb_kernel_arch(int32_t device, int32_t* binary_version, int32_t* ptx_version) {
    if (!binary_version || !ptx_version) return fail(GFB_ERR_INVALID, "kernel arch: NULL output");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(GFB_ERR_NO_DEVICE, "no CUDA-capable GPU found");
    if (device < 0 || device >= ndev) return fail(GFB_ERR_INVALID, "device %d not present", device);
    CU(cudaSetDevice(device));
    cudaFuncAttributes fa{};
    CU(cudaFuncGetAttributes(&fa, gfb::predict_kernel<float>));
    *binary_version = fa.binaryVersion;
    *ptx_version = fa.ptxVersion;
    return GFB_OK;
}

const char* gfb_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace {

// Greedy colouring of the cells in mesh order with a colour mask of T per
// node; false when some cell would need a colour beyond T's width.
template <typename T>
bool greedy_colour(const gfb_mesh* m, int nn, std::vector<T>& used, std::vector<int>& colour, int& n_colour) {
    used.assign(m->n_node, T(0));
    n_colour = 0;
    for (long long e = 0; e < m->n_cell; ++e) {
        T u = 0;
        const int* ib = m->ibool + e * nn;
        for (int p = 0; p < nn; ++p) u |= used[ib[p]];
        const T avail = (T)~u;
        if (avail == 0) return false;
        const int col = __builtin_ctzll((unsigned long long)avail);
        colour[e] = col;
        n_colour = std::max(n_colour, col + 1);
        const T bit = (T)((T)1 << col);
        for (int p = 0; p < nn; ++p) used[ib[p]] |= bit;
    }
    return true;
}

// Wavefields of a solver with several source positions: count, force
// direction and source set of each, and the sets.
struct FieldSpec {
    int n_field = 0;
    int dir[gfb::kMaxFields] = {};
    int fset[gfb::kMaxFields] = {};
    int n_set = 0;
    const gfb_source* sets = nullptr;
};

// w_tab / D_tab: GLL weights [ngll] and derivative matrix [ngll*ngll] to use
// instead of the tables computed from ngll (NULL: computed).  fs: the
// wavefields and source sets (NULL: config's wavefields, all with src).
gfb_status create_impl(const gfb_mesh* m, const gfb_config* c, const gfb_source* src, int n_model,
                       const gfb_model* models, gfb_solver** out, const double* w_tab = nullptr,
                       const double* D_tab = nullptr, const FieldSpec* fs = nullptr) {
    gfb_status st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(GFB_ERR_NO_DEVICE, "no CUDA-capable GPU found");
    if (c->device < 0 || c->device >= ndev) return fail(GFB_ERR_INVALID, "device %d not present", c->device);
    CU(cudaSetDevice(c->device));

    auto s = std::make_unique<gfb_solver>();
    s->device = c->device;
    s->prec = c->precision;
    s->ng = m->ngll;
    s->nn = m->ngll * m->ngll * m->ngll;
    s->nfld = fs ? fs->n_field : c->n_field;
    s->F = 3 * s->nfld;
    s->n_cell = m->n_cell;
    s->n_node = m->n_node;
    s->dt = c->dt;
    s->stride = c->snapshot_stride;
    for (int d = 0; d < gfb::kMaxFields; ++d) {
        s->dirs[d] = fs ? fs->dir[d] : (d < c->n_field ? c->field_dir[d] : 0);
        s->fset[d] = fs ? fs->fset[d] : 0;
    }
    s->n_set = fs ? fs->n_set : 1;
    s->stf_from_sets = fs != nullptr;
    if (fs) s->sets.assign(fs->sets, fs->sets + fs->n_set);
    else if (src) s->sets.assign(1, *src);
    s->has_cpml = m->pml_coef_abar != nullptr;
    s->flags = c->flags;
    s->rec_f32 = (c->flags & GFB_FLAG_RECORD_F32) != 0;
    s->fuse = (c->flags & GFB_FLAG_FUSED_NODE) != 0;
    s->use_graph = !(c->flags & GFB_FLAG_NO_GRAPH);
    s->point_kernel = (c->flags & GFB_FLAG_POINT_KERNEL) != 0;
    s->n_model = n_model;
    s->n_rec = m->n_rec_cell;
    s->slots = std::max(1, c->record_slots);
    const double theta = 1.0 / 8.0;  // pml.cpp:35, 63-64
    s->c1 = (1.0 - 2.0 * theta) * 0.5 * c->dt;
    s->c2 = (1.0 - theta) * 0.5 * c->dt * c->dt;
    CU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));

    StageClock clk;
    const int nn = s->nn;
    const long long P = (long long)m->n_cell * nn;
    // ibool range and per-cell distinctness (a repeated node inside one cell
    // would make two threads of one block update the same force entry); the
    // first offending entry in mesh order is reported: an entry out of range,
    // or the second occurrence of a node in its cell
    {
        std::mutex bad_mu;
        long long bad_q = -1;
        bool bad_range = false;
        parallel_for(m->n_cell, [&](long long e0, long long e1) {
            std::vector<uint64_t> key(nn);
            for (long long e = e0; e < e1; ++e) {
                int rng_at = nn, dup_at = nn;
                for (int p = 0; p < nn; ++p) {
                    const int g = m->ibool[e * nn + p];
                    if (rng_at == nn && (g < 0 || g >= m->n_node)) rng_at = p;
                    key[p] = ((uint64_t)(uint32_t)g << 32) | (uint32_t)p;
                }
                std::sort(key.begin(), key.end());
                for (int k = 1; k < nn; ++k)
                    if ((key[k] >> 32) == (key[k - 1] >> 32)) dup_at = std::min(dup_at, (int)(key[k] & 0xffffffffu));
                const int at = std::min(rng_at, dup_at);
                if (at < nn) {
                    std::lock_guard<std::mutex> lk(bad_mu);
                    if (bad_q < 0 || e * nn + at < bad_q) {
                        bad_q = e * nn + at;
                        bad_range = at == rng_at;
                    }
                    return;  // later cells of this range come after it
                }
            }
        }, 4096);
        if (bad_q >= 0) {
            if (bad_range)
                return fail(GFB_ERR_INVALID, "ibool[%lld]=%d outside [0,%d)", bad_q, m->ibool[bad_q], m->n_node);
            return fail(GFB_ERR_INVALID, "cell %lld lists node %d twice", bad_q / nn, m->ibool[bad_q]);
        }
    }
    clk.mark("mesh check");
    // global lumped mass (accumulate) and damping (assign), solver.cpp:193-202.
    // Each thread owns a range of nodes and scans every entry in mesh order,
    // so every node sums (and assigns) in the reference's order
    // The same pass records each node's first touch (the first point in
    // mesh order that lists it), from which the device numbering follows.
    const NodeBuckets nb = bucket_points(m->ibool, P, m->n_node);
    clk.mark("point buckets");
    std::vector<double> node_mass(m->n_node, 0.0), node_damp(m->n_node, 0.0);
    std::vector<long long> first_q(m->n_node, -1);
    std::vector<uint8_t> first_flag((size_t)P, 0);  // 1: the point is its node's first touch
    // the FP32 path keeps C-PML per node when it can: the same pass marks
    // the live C-PML points (some A_k != 0 in a C-PML cell) and their nodes
    const bool want_node_pml = s->has_cpml && s->prec == GFB_FP32 && !(c->flags & GFB_FLAG_CELL_PML);
    std::vector<uint8_t> node_live(want_node_pml ? (size_t)m->n_node : 0, 0);
    std::vector<std::vector<long long>> live_pts(want_node_pml ? nb.n_owner : 0);
    nb.for_each_owner([&](int t, long long, long long, const long long* qs, size_t nq) {
        for (size_t k = 0; k < nq; ++k) {
            const long long q = qs[k];
            const int g = m->ibool[q];
            node_mass[g] += m->mass[q];
            node_damp[g] = m->damping ? m->damping[q] : 0.0;
            if (first_q[g] < 0) {
                first_q[g] = q;
                first_flag[q] = 1;
            }
            if (want_node_pml && m->pml_region[q / nn] != 0) {
                const double* A = m->pml_coef_abar + q * 5;
                if (A[0] != 0.0 || A[1] != 0.0 || A[2] != 0.0 || A[3] != 0.0 || A[4] != 0.0) {
                    node_live[g] = 1;
                    live_pts[t].push_back(q);
                }
            }
        }
    });
    clk.mark("lumped mass");
    s->has_damping = false;
    if (!s->has_cpml && m->damping)
        for (double d : node_damp)
            if (d > 0.0) {
                s->has_damping = true;
                break;
            }
    // greedy colouring in cell order: colour = lowest colour unused by any
    // cell already sharing a node (structured meshes get the 8 parity
    // colours).  Byte masks per node first (an eighth of the memory
    // traffic); a mesh that needs a ninth colour is coloured again with
    // 64-bit masks, which gives the same colours
    std::vector<uint8_t> used8;
    std::vector<uint64_t> used64;
    std::vector<int> colour(m->n_cell);
    int n_colour = 0;
    const bool narrow = greedy_colour(m, nn, used8, colour, n_colour);
    if (!narrow) {
        std::vector<uint8_t>().swap(used8);
        if (!greedy_colour(m, nn, used64, colour, n_colour))
            return fail(GFB_ERR_UNSUPPORTED, "mesh needs more than 64 colours");
    }
    auto used_mask = [&](uint32_t g) -> uint64_t { return narrow ? (uint64_t)used8[g] : used64[g]; };
    clk.mark("colouring");
    std::vector<int> perm(m->n_cell), inv_perm(m->n_cell);
    s->colour_begin.assign(n_colour + 1, 0);
    for (long long e = 0; e < m->n_cell; ++e) s->colour_begin[colour[e] + 1]++;
    for (int k = 0; k < n_colour; ++k) s->colour_begin[k + 1] += s->colour_begin[k];
    {
        std::vector<int> fill(s->colour_begin.begin(), s->colour_begin.end() - 1);
        for (long long e = 0; e < m->n_cell; ++e) {
            const int ed = fill[colour[e]]++;
            perm[ed] = (int)e;
            inv_perm[e] = ed;
        }
    }
    // device ibool with the first/last-touch bits: the lowest colour
    // touching a node stores its force, later colours add, the highest
    // colour finalises the node
    std::vector<uint32_t> ibool_dev((size_t)P);
    parallel_for(m->n_cell, [&](long long e0, long long e1) {
        for (long long ed = e0; ed < e1; ++ed) {
            const long long e = perm[ed];
            for (int p = 0; p < nn; ++p) {
                const uint32_t g = (uint32_t)m->ibool[e * nn + p];
                const uint64_t um = used_mask(g);
                const bool first = __builtin_ctzll(um) == colour[e];
                const bool last = 63 - __builtin_clzll(um) == colour[e];
                ibool_dev[ed * nn + p] = g | (first ? gfb::kFirstTouch : 0u) | (last ? gfb::kLastTouch : 0u);
            }
        }
    });
    clk.mark("colour order");
    std::vector<double> x, w, D;
    if (!gll_tables(m->ngll - 1, x, w, D)) return fail(GFB_ERR_INVALID, "GLL table construction failed");
    if (w_tab) w.assign(w_tab, w_tab + m->ngll);
    if (D_tab) D.assign(D_tab, D_tab + (size_t)m->ngll * m->ngll);
    if (s->prec == GFB_FP64) {
        if ((st = dispatch<double, SmemOp>(s->ng, s->nfld, s.get()))) return st;
        st = build_device<double>(s.get(), m, src, n_model, models, perm, inv_perm, ibool_dev, node_mass, node_damp,
                                  first_q, first_flag, node_live, live_pts, w, D, clk);
    } else {
        if ((st = dispatch<float, SmemOp>(s->ng, s->nfld, s.get()))) return st;
        st = build_device<float>(s.get(), m, src, n_model, models, perm, inv_perm, ibool_dev, node_mass, node_damp,
                                 first_q, first_flag, node_live, live_pts, w, D, clk);
    }
    if (st) return st;
    CU(cudaStreamSynchronize(s->stream));
    clk.mark("device set-up");
    // FP32 path: the element force of most steps from the predicted
    // displacement's increment (see step_begin_kernel), where the C-PML
    // term is added at the nodes (node form or none) and no node is
    // finalised inside the element kernel
    s->by_increments_ok = s->prec == GFB_FP32 && (!s->has_cpml || s->node_pml) && !s->fuse &&
                          !(c->flags & GFB_FLAG_DIRECT_FORCE);
    s->refresh = s->by_increments_ok ? kRefreshSteps : 1;
    // plain nodes in the half-step velocity form where nothing reads their
    // (v, a) inside the step: the FP32 path with node-form or no C-PML, no
    // legacy damping (it acts on v_n, solver.cpp:564-574), no node update in
    // the element kernel
    s->half_v = s->prec == GFB_FP32 && (!s->has_cpml || s->node_pml) && !s->fuse && !s->has_damping &&
                !(c->flags & GFB_FLAG_DIRECT_FORCE);
    s->hv_begin = s->half_v ? (s->node_pml ? s->n_pml_node : 0) : s->n_node;
    if (s->half_v) {  // the state starts at rest: w = 0
        if ((st = s->alloc(&s->w32, (size_t)s->n_node * s->F))) return st;
        CU(cudaMemsetAsync(s->w32, 0, (size_t)s->n_node * s->F * sizeof(float), s->stream));
    }
    if ((c->flags & GFB_FLAG_AUTOTUNE) && (st = autotune(s.get()))) return st;
    CU(cudaDeviceSynchronize());
    clk.mark("autotune");
    s->sets.clear();  // the caller's source arrays were borrowed for the call
    *out = s.release();
    return GFB_OK;
}

}  // namespace

extern "C" {

gfb_status gfb_create(const gfb_mesh* m, const gfb_config* c, const gfb_source* src, gfb_solver** out) {
    if (!out) return fail(GFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    gfb_status st = validate(m, c);
    if (st) return st;
    gfb_model one{};
    one.cell_begin = 0;
    one.cell_end = m->n_cell;
    one.node_begin = 0;
    one.node_end = m->n_node;
    one.dt = c->dt;
    one.n_steps = INT32_MAX;
    one.n_stf = src ? src->n_stf : 0;
    one.stf = src ? src->stf : nullptr;
    return create_impl(m, c, src, 1, &one, out);
}

gfb_status gfb_create_sources(const gfb_mesh* m, const gfb_config* c, int32_t n_source, const gfb_source* sources,
                              int32_t n_field, const int32_t* field_dir, const int32_t* field_source,
                              gfb_solver** out) {
    if (!out) return fail(GFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!m || !c) return fail(GFB_ERR_INVALID, "mesh and config are required");
    if (n_source < 1 || n_source > gfb::kMaxFields || !sources)
        return fail(GFB_ERR_INVALID, "n_source must be 1..%d", gfb::kMaxFields);
    if (!field_dir || !field_source) return fail(GFB_ERR_INVALID, "field_dir and field_source are required");
    const bool shape_ok = (n_field >= 1 && n_field <= 3) || (m->ngll == 5 && (n_field == 6 || n_field == 9 || n_field == 12));
    if (!shape_ok)
        return fail(GFB_ERR_UNSUPPORTED, "%d wavefields: 1..3 at any ngll, or 6, 9, 12 at ngll 5", n_field);
    if (c->precision == GFB_FP64 && n_field > 6)
        return fail(GFB_ERR_UNSUPPORTED, "the FP64 path advances at most 6 wavefields (%d asked)", n_field);
    FieldSpec fs;
    fs.n_field = n_field;
    fs.n_set = n_source;
    fs.sets = sources;
    for (int f = 0; f < n_field; ++f) {
        if (field_dir[f] < 0 || field_dir[f] > 2)
            return fail(GFB_ERR_INVALID, "field_dir[%d]=%d must be 0, 1 or 2", f, field_dir[f]);
        if (field_source[f] < 0 || field_source[f] >= n_source)
            return fail(GFB_ERR_INVALID, "field_source[%d]=%d must be 0..%d", f, field_source[f], n_source - 1);
        fs.dir[f] = field_dir[f];
        fs.fset[f] = field_source[f];
    }
    for (int k = 0; k < n_source; ++k) {
        const gfb_source& ss = sources[k];
        if (ss.n_src_cell < 0 || (ss.n_src_cell > 0 && (!ss.cell_ids || !ss.weights)) || ss.n_stf < 0 ||
            (ss.n_stf > 0 && !ss.stf))
            return fail(GFB_ERR_INVALID, "source %d: bad cells, weights or source time function", k);
    }
    gfb_config cc = *c;
    cc.n_field = 1;  // the wavefields are those of field_dir / field_source
    cc.field_dir[0] = 0;
    gfb_status st = validate(m, &cc);
    if (st) return st;
    gfb_model one{};
    one.cell_end = m->n_cell;
    one.node_end = m->n_node;
    one.dt = c->dt;
    one.n_steps = INT32_MAX;
    return create_impl(m, c, nullptr, 1, &one, out, nullptr, nullptr, &fs);
}

gfb_status gfb_create_batch(const gfb_mesh* m, const gfb_config* c, const gfb_source* src, int32_t n_model,
                            const gfb_model* models, gfb_solver** out) {
    if (!out) return fail(GFB_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!models || n_model < 1 || n_model > 255) return fail(GFB_ERR_INVALID, "n_model must be 1..255");
    if (!m || !c) return fail(GFB_ERR_INVALID, "mesh and config are required");
    gfb_config cc = *c;
    cc.dt = models[0].dt;
    gfb_status st = validate(m, &cc);
    if (st) return st;
    for (int k = 0; k < n_model; ++k) {
        const gfb_model& md = models[k];
        const int cb = k ? models[k - 1].cell_end : 0, nb = k ? models[k - 1].node_end : 0;
        if (md.cell_begin != cb || md.cell_end <= md.cell_begin || md.node_begin != nb || md.node_end <= md.node_begin)
            return fail(GFB_ERR_INVALID, "model %d: cells and nodes must follow the previous model's", k);
        if (!(md.dt > 0.0)) return fail(GFB_ERR_INVALID, "model %d: dt must be positive", k);
        if (md.n_steps < 0 || md.n_stf < 0 || (md.n_stf > 0 && !md.stf))
            return fail(GFB_ERR_INVALID, "model %d: bad step count or source time function", k);
    }
    if (models[n_model - 1].cell_end != m->n_cell || models[n_model - 1].node_end != m->n_node)
        return fail(GFB_ERR_INVALID, "models must cover all %d cells and %d nodes", m->n_cell, m->n_node);
    const int nn = m->ngll * m->ngll * m->ngll;
    for (int k = 0; k < n_model; ++k)
        for (long long q = (long long)models[k].cell_begin * nn; q < (long long)models[k].cell_end * nn; ++q)
            if (m->ibool[q] < models[k].node_begin || m->ibool[q] >= models[k].node_end)
                return fail(GFB_ERR_INVALID, "model %d: cell %lld uses node %d of another model", k, q / nn, m->ibool[q]);
    return create_impl(m, &cc, src, n_model, models, out);
}

gfb_status gfb_destroy(gfb_solver* s) {
    if (!s) return GFB_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
    return GFB_OK;
}

namespace {
// A kernel whose bounded wait on its own bulk copies gave up left the step
// unfinished: report it at the next synchronisation.
gfb_status check_kernel_err(gfb_solver* s) {
    if (!s->d_kernel_err) return GFB_OK;
    int e = 0;
    CU(cudaMemcpy(&e, s->d_kernel_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(GFB_ERR_CUDA, "element kernel: a bulk copy did not complete; the state is invalid");
    return GFB_OK;
}
}  // namespace

gfb_status gfb_advance(gfb_solver* s, int32_t n_steps) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (n_steps < 0) return fail(GFB_ERR_INVALID, "n_steps must be >= 0");
    CU(cudaSetDevice(s->device));
    for (int it = 0; it < n_steps; ++it) {
        gfb_status st = one_step(s, nullptr);
        if (st) return st;
    }
    return GFB_OK;
}

gfb_status gfb_advance_timed(gfb_solver* s, int32_t n_steps, double* ms) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (n_steps < 0) return fail(GFB_ERR_INVALID, "n_steps must be >= 0");
    CU(cudaSetDevice(s->device));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(GFB_ERR_CUDA, "cudaEventCreate failed");
    }
    gfb_status st = GFB_OK;
    if (cudaEventRecord(e0, s->stream) != cudaSuccess) st = fail(GFB_ERR_CUDA, "cudaEventRecord failed");
    for (int it = 0; it < n_steps && !st; ++it) st = one_step(s, nullptr);
    float t = 0.0f;
    if (!st && (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
        st = fail(GFB_ERR_CUDA, "step timing failed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!st && ms) *ms += t;
    return st ? st : check_kernel_err(s);
}

gfb_status gfb_advance_profiled(gfb_solver* s, int32_t n_steps, double* ms_element, double* ms_node,
                                double* ms_record) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (n_steps < 0) return fail(GFB_ERR_INVALID, "n_steps must be >= 0");
    CU(cudaSetDevice(s->device));
    std::vector<cudaEvent_t> ev((size_t)n_steps * 4, nullptr);
    gfb_status st = GFB_OK;
    for (auto& e : ev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            st = fail(GFB_ERR_CUDA, "cudaEventCreate failed");
            break;
        }
    }
    for (int it = 0; it < n_steps && !st; ++it) st = one_step(s, ev.data() + (size_t)it * 4);
    double acc[3] = {0, 0, 0};
    if (!st && n_steps > 0) {
        if (cudaEventSynchronize(ev.back()) != cudaSuccess) st = fail(GFB_ERR_CUDA, "event synchronize failed");
        for (int it = 0; it < n_steps && !st; ++it) {
            for (int k = 0; k < 3; ++k) {
                float t = 0.0f;
                if (cudaEventElapsedTime(&t, ev[(size_t)it * 4 + k], ev[(size_t)it * 4 + k + 1]) != cudaSuccess) {
                    st = fail(GFB_ERR_CUDA, "cudaEventElapsedTime failed");
                    break;
                }
                acc[k] += t;
            }
        }
    }
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
    if (st) return st;
    if (ms_element) *ms_element += acc[0];
    if (ms_node) *ms_node += acc[1];
    if (ms_record) *ms_record += acc[2];
    return GFB_OK;
}

gfb_status gfb_get_info(const gfb_solver* s, gfb_info* info) {
    if (!s || !info) return fail(GFB_ERR_INVALID, "NULL argument");
    info->n_colour = (int32_t)s->colour_begin.size() - 1;
    info->n_pml_cell = s->n_pml;
    info->n_rec_cell = s->n_rec;
    info->n_field = s->nfld;
    info->precision = s->prec;
    info->n_cell = s->n_cell;
    info->n_node = s->n_node;
    info->ngll = s->ng;
    info->device_bytes = s->device_bytes;
    info->upload_bytes = s->upload_bytes;
    info->kernel_launches = s->launches;
    info->n_pml_node = s->node_pml ? s->n_pml_node : 0;
    info->elem_blocks = use_col_kernel(s) ? s->col_blocks : s->pipe_blocks;
    info->elem_kernel = use_col_kernel(s) ? 1 : 0;
    info->cells_per_group = use_col_kernel(s) ? s->col_epb : 0;
    info->force_refresh = s->refresh;
    info->half_v = s->half_v ? 1 : 0;
    info->elem_variant = use_col_kernel(s) ? s->col_variant : -1;
    info->n_elem_variants = col_kernel_eligible(s) ? s->n_col_variants : 0;
    return GFB_OK;
}

gfb_status gfb_set_force_refresh(gfb_solver* s, int32_t steps) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (steps < 1) return fail(GFB_ERR_INVALID, "force refresh period must be >= 1");
    if (steps > 1 && !s->by_increments_ok)
        return fail(GFB_ERR_UNSUPPORTED, "this solver evaluates the element force in full every step");
    gfb_status st;
    CU(cudaStreamSynchronize(s->stream));
    // between full evaluations the node pass leaves the predicted
    // displacement's increment in place of it: rewrite it in full
    if (s->refresh > 1 && (st = launch_predict(s))) return st;
    s->refresh = steps;
    // the next step evaluates the force in full (from a period of 1 the
    // stored force is this step's, but the next step must not add to it)
    if (steps > 1) CU(cudaMemsetAsync(s->d_force_direct, 1, (size_t)s->n_model * sizeof(int), s->stream));
    if (s->gexec) {
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return GFB_OK;
}

gfb_status gfb_select_element_kernel(gfb_solver* s, int32_t variant) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (!col_kernel_eligible(s)) return fail(GFB_ERR_UNSUPPORTED, "this solver has one element kernel");
    if (variant < -1 || variant >= s->n_col_variants)
        return fail(GFB_ERR_INVALID, "element kernel variant out of range");
    gfb_status st;
    CU(cudaStreamSynchronize(s->stream));
    s->point_kernel = variant < 0;
    s->col_variant = variant < 0 ? 0 : variant;
    if ((st = dispatch<float, ColGridOp>(s->ng, s->nfld, s))) return st;
    // the next step evaluates the force in full with the new kernel, from
    // the predicted displacement rewritten in full (between full
    // evaluations the node pass leaves its increment there)
    if (s->refresh > 1 && (st = launch_predict(s))) return st;
    if (s->gexec) {
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return GFB_OK;
}

gfb_status gfb_synchronize(gfb_solver* s) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    return check_kernel_err(s);
}

gfb_status gfb_current_step(const gfb_solver* s, int32_t* step) {
    if (!s || !step) return fail(GFB_ERR_INVALID, "NULL argument");
    *step = s->step;
    return GFB_OK;
}

gfb_status gfb_get_state(gfb_solver* s, int32_t field, double* u, double* v, double* a) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (field < 0 || field >= s->nfld) return fail(GFB_ERR_INVALID, "field %d out of range", field);
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    const size_t nF = (size_t)s->n_node * s->F;
    std::vector<double> tmp(nF);
    gfb_status st;
    auto pick = [&](double* dst) {  // device layout [device node][3*n_field]
        for (long long g = 0; g < s->n_node; ++g) {
            const long long d = s->node_inv.empty() ? g : s->node_inv[g];
            for (int c = 0; c < 3; ++c) dst[g * 3 + c] = tmp[d * s->F + field * 3 + c];
        }
    };
    if (u) {
        if ((st = d2h(s, tmp.data(), s->u, nF * 8))) return st;
        pick(u);
    }
    // half-step velocity form: (v, a) of the plain nodes recovered into
    // temporary device arrays (the C-PML nodes copied as they are)
    double* dv = s->v;
    void* da = s->a;
    std::unique_ptr<DevBuf> tv, ta;
    if (s->half_v && (v || a)) {
        tv = std::make_unique<DevBuf>();
        ta = std::make_unique<DevBuf>();
        CU(cudaMalloc(&tv->p, nF * 8));
        CU(cudaMalloc(&ta->p, nF * 4));
        CU(cudaMemcpyAsync(tv->p, s->v, nF * 8, cudaMemcpyDeviceToDevice, s->stream));
        CU(cudaMemcpyAsync(ta->p, s->a, nF * 4, cudaMemcpyDeviceToDevice, s->stream));
        if ((st = half_v_to_full(s, static_cast<double*>(tv->p), static_cast<float*>(ta->p)))) return st;
        CU(cudaStreamSynchronize(s->stream));
        dv = static_cast<double*>(tv->p);
        da = ta->p;
    }
    if (v) {
        if ((st = d2h(s, tmp.data(), dv, nF * 8))) return st;
        pick(v);
    }
    if (a) {
        if (s->prec == GFB_FP64) {
            if ((st = d2h(s, tmp.data(), da, nF * 8))) return st;
        } else {
            std::vector<float> f(nF);
            if ((st = d2h(s, f.data(), da, nF * 4))) return st;
            for (size_t i = 0; i < nF; ++i) tmp[i] = f[i];
        }
        pick(a);
    }
    return GFB_OK;
}

gfb_status gfb_set_state(gfb_solver* s, int32_t field, int32_t step, const double* u, const double* v,
                         const double* a) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (field < 0 || field >= s->nfld) return fail(GFB_ERR_INVALID, "field %d out of range", field);
    if (step < 0) return fail(GFB_ERR_INVALID, "step must be >= 0");
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    const size_t nF = (size_t)s->n_node * s->F;
    std::vector<double> tmp(nF);
    gfb_status st0;
    auto put = [&](const double* src, void* dev, bool is_real_float) -> gfb_status {
        gfb_status st;
        if (is_real_float) {
            std::vector<float> f(nF);
            if ((st = d2h(s, f.data(), dev, nF * 4))) return st;
            for (long long g = 0; g < s->n_node; ++g) {
                const long long d = s->node_inv.empty() ? g : s->node_inv[g];
                for (int c = 0; c < 3; ++c) f[d * s->F + field * 3 + c] = src ? (float)src[g * 3 + c] : 0.0f;
            }
            if ((st = h2d(s, dev, f.data(), nF * 4))) return st;
        } else {
            if ((st = d2h(s, tmp.data(), dev, nF * 8))) return st;
            for (long long g = 0; g < s->n_node; ++g) {
                const long long d = s->node_inv.empty() ? g : s->node_inv[g];
                for (int c = 0; c < 3; ++c) tmp[d * s->F + field * 3 + c] = src ? src[g * 3 + c] : 0.0;
            }
            if ((st = h2d(s, dev, tmp.data(), nF * 8))) return st;
        }
        return GFB_OK;
    };
    gfb_status st;
    // half-step velocity form: the other fields' (v, a) first, so that the
    // wavefield written here and the others are all (v, a) when converted
    if (s->half_v) {
        if ((st0 = half_v_to_full(s, s->v, static_cast<float*>(s->a)))) return st0;  // in place
        CU(cudaStreamSynchronize(s->stream));
        s->a_in_force = false;  // a now holds every field's acceleration
    }
    if ((st = put(u, s->u, false))) return st;
    if ((st = put(v, s->v, false))) return st;
    if ((st = put(a, s->a, s->prec == GFB_FP32))) return st;
    if (s->half_v && (st = half_v_from_full(s))) return st;
    s->a_in_force = false;
    if (s->has_cpml && !s->node_pml) {
        const size_t es = s->prec == GFB_FP64 ? 8 : 4;
        CU(cudaMemset(s->pml_mem, 0, (size_t)s->n_pml * s->F * 3 * s->nn * es));
        CU(cudaMemset(s->pml_prev, 0, (size_t)s->n_pml * s->F * s->nn * es));
    }
    if (s->node_pml && s->n_pml_node > 0) {
        CU(cudaMemset(s->npml_mem, 0, (size_t)s->n_pml_node * s->F * 3 * sizeof(float)));
        CU(cudaMemset(s->npml_prev, 0, (size_t)s->n_pml_node * s->F * sizeof(float)));
    }
    if ((st = launch_predict(s))) return st;
    {
        std::vector<int> ms(s->n_model, step);
        if ((st = h2d(s, s->d_mstep, ms.data(), ms.size() * 4))) return st;
    }
    CU(cudaStreamSynchronize(s->stream));
    s->step = step;
    return GFB_OK;
}

namespace {

// Device arrays of a checkpoint, in order: pointer and byte count.
std::vector<std::pair<void*, size_t>> checkpoint_arrays(gfb_solver* s) {
    const size_t es = s->prec == GFB_FP64 ? 8 : 4;
    const size_t nF = (size_t)s->n_node * s->F;
    std::vector<std::pair<void*, size_t>> a;
    a.push_back({s->u, nF * 8});
    a.push_back({s->v, nF * 8});
    a.push_back({s->a, nF * es});
    a.push_back({s->ut, (size_t)s->n_node * s->nfld * 4 * es});
    if (s->has_cpml && !s->node_pml) {
        a.push_back({s->pml_mem, (size_t)s->n_pml * s->F * 3 * s->nn * es});
        a.push_back({s->pml_prev, (size_t)s->n_pml * s->F * s->nn * es});
    }
    if (s->node_pml && s->n_pml_node > 0) {
        a.push_back({s->npml_mem, (size_t)s->n_pml_node * s->F * 3 * es});
        a.push_back({s->npml_prev, (size_t)s->n_pml_node * s->F * es});
    }
    a.push_back({s->d_mstep, (size_t)s->n_model * 4});
    if (s->half_v) a.push_back({s->w32, (size_t)s->n_node * s->F * 4});
    if (s->refresh > 1) {
        // the stored force is state when it is updated by increments
        a.push_back({s->force, (size_t)s->n_node * s->nfld * 4 * es});
        a.push_back({s->d_force_direct, (size_t)s->n_model * 4});
    }
    return a;
}

struct CheckpointHeader {
    char magic[8];
    int64_t bytes;
    int32_t version, precision, n_field, n_model;
    int64_t n_node, n_cell, n_pml, n_pml_node;
    int32_t step, flags;
    int32_t half_v, a_in_force;
};

void checkpoint_header(const gfb_solver* s, int64_t bytes, CheckpointHeader& h) {
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "GFBCKPT", 8);
    h.bytes = bytes;
    h.version = 1;
    h.precision = s->prec;
    h.n_field = s->nfld;
    h.n_model = s->n_model;
    h.n_node = s->n_node;
    h.n_cell = s->n_cell;
    h.n_pml = s->node_pml ? 0 : s->n_pml;
    h.n_pml_node = s->node_pml ? s->n_pml_node : 0;
    h.step = s->step;
    h.flags = s->flags;
    h.half_v = s->half_v ? 1 : 0;
    h.a_in_force = s->a_in_force ? 1 : 0;
}

}  // namespace

gfb_status gfb_checkpoint_size(gfb_solver* s, int64_t* bytes) {
    if (!s || !bytes) return fail(GFB_ERR_INVALID, "NULL argument");
    int64_t b = sizeof(CheckpointHeader);
    for (auto& a : checkpoint_arrays(s)) b += (int64_t)a.second;
    *bytes = b;
    return GFB_OK;
}

gfb_status gfb_checkpoint_save(gfb_solver* s, void* buf, int64_t bytes) {
    int64_t need = 0;
    gfb_status st = gfb_checkpoint_size(s, &need);
    if (st) return st;
    if (!buf || bytes < need) return fail(GFB_ERR_INVALID, "checkpoint buffer needs %lld bytes", (long long)need);
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    CheckpointHeader h;
    checkpoint_header(s, need, h);
    unsigned char* p = static_cast<unsigned char*>(buf);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    for (auto& a : checkpoint_arrays(s)) {
        if ((st = d2h(s, p, a.first, a.second))) return st;
        p += a.second;
    }
    return GFB_OK;
}

gfb_status gfb_checkpoint_load(gfb_solver* s, const void* buf, int64_t bytes) {
    int64_t need = 0;
    gfb_status st = gfb_checkpoint_size(s, &need);
    if (st) return st;
    if (!buf || bytes < (int64_t)sizeof(CheckpointHeader)) return fail(GFB_ERR_INVALID, "checkpoint buffer too small");
    CheckpointHeader h, mine;
    std::memcpy(&h, buf, sizeof(h));
    checkpoint_header(s, need, mine);
    mine.step = h.step;
    mine.a_in_force = h.a_in_force;
    if (std::memcmp(&h, &mine, sizeof(h)) != 0 || bytes < need)
        return fail(GFB_ERR_INVALID, "checkpoint does not belong to a solver built like this one");
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof(h);
    for (auto& a : checkpoint_arrays(s)) {
        if ((st = h2d(s, a.first, p, a.second))) return st;
        p += a.second;
    }
    s->step = h.step;
    s->a_in_force = h.a_in_force != 0;
    return GFB_OK;
}

gfb_status gfb_records_pending(gfb_solver* s, int32_t* n) {
    if (!s || !n) return fail(GFB_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->rec_mu);
    int32_t k = 0;
    for (const auto& p : s->pending) k += p.done ? 0 : 1;
    *n = k;
    return GFB_OK;
}

}  // extern "C"

namespace {

// gfb_read_record into double or float buffers.
template <typename Out>
gfb_status read_record_t(gfb_solver* s, int32_t field, int32_t* step, Out* strain, Out* u, Out* v, Out* a,
                         int32_t release) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    if (field < 0 || field >= s->nfld) return fail(GFB_ERR_INVALID, "field %d out of range", field);
    CU(cudaSetDevice(s->device));
    Snapshot* snap;
    int slot;
    {
        std::lock_guard<std::mutex> lk(s->rec_mu);
        auto it = s->pending.begin();
        while (it != s->pending.end() && it->done) ++it;  // read, still held by another reader
        if (it == s->pending.end()) return fail(GFB_ERR_STATE, "no snapshot pending");
        snap = &*it;
        snap->readers++;  // keeps the slot from being spilled or reused while copying
        slot = snap->slot;
    }
    // copy out without holding the lock (the stepping thread may go on)
    gfb_status st = GFB_OK;
    if (slot >= 0 && cudaEventSynchronize(s->copy_evt[slot]) != cudaSuccess)
        st = fail(GFB_ERR_CUDA, "snapshot copy failed");
    if (step) *step = snap->step;
    if (!st && (strain || u || v || a)) {
        const void* raw = slot >= 0 ? s->pinned[slot] : (const void*)snap->host.get();
        const long long first = (long long)field * s->n_rec * s->nn;  // points of the earlier fields
        unpack_points(s, raw, (long long)s->n_rec * s->nn, [first](long long q) { return first + q; }, strain, u,
                      v, a);
    }
    {
        std::lock_guard<std::mutex> lk(s->rec_mu);
        snap->readers--;
        if (!st) {
            if (!snap->read_mask[field]) {
                snap->read_mask[field] = 1;
                snap->fields_read++;
            }
            if (release || snap->fields_read == s->nfld) snap->done = true;
        }
        while (!s->pending.empty() && s->pending.front().done && s->pending.front().readers == 0)
            s->pending.pop_front();
    }
    s->rec_cv.notify_all();
    return st;
}

}  // namespace

extern "C" {

gfb_status gfb_read_record(gfb_solver* s, int32_t field, int32_t* step, double* strain, double* u,
                           double* v, double* a, int32_t release) {
    return read_record_t(s, field, step, strain, u, v, a, release);
}

gfb_status gfb_read_record_f32(gfb_solver* s, int32_t field, int32_t* step, float* strain, float* u, float* v,
                               float* a, int32_t release) {
    return read_record_t(s, field, step, strain, u, v, a, release);
}

gfb_status gfb_rec_nodes(gfb_solver* s, int32_t* n_node, int64_t* node_ids) {
    if (!s || !n_node) return fail(GFB_ERR_INVALID, "NULL argument");
    *n_node = s->n_unique;
    if (node_ids) std::memcpy(node_ids, s->rec_node_ids.data(), s->rec_node_ids.size() * 8);
    return GFB_OK;
}

gfb_status gfb_read_green(gfb_solver* s, int32_t* step, double* strain, double* u, double* v, double* a,
                          int32_t release) {
    if (!s) return fail(GFB_ERR_INVALID, "solver is NULL");
    CU(cudaSetDevice(s->device));
    Snapshot* snap;
    int slot;
    {
        std::lock_guard<std::mutex> lk(s->rec_mu);
        auto it = s->pending.begin();
        while (it != s->pending.end() && it->done) ++it;
        if (it == s->pending.end()) return fail(GFB_ERR_STATE, "no snapshot pending");
        snap = &*it;
        snap->readers++;
        slot = snap->slot;
    }
    gfb_status st = GFB_OK;
    if (slot >= 0 && cudaEventSynchronize(s->copy_evt[slot]) != cudaSuccess)
        st = fail(GFB_ERR_CUDA, "snapshot copy failed");
    if (step) *step = snap->step;
    if (!st) {
        // merged part [field][node][15] after the cell part, read out as
        // [node][field][...]: the Green's tensor of a node is its fields' strains
        const void* raw = slot >= 0 ? s->pinned[slot] : (const void*)snap->host.get();
        const long long cells = (long long)(snapshot_cell_values(s) / 15);
        const int nfld = s->nfld;
        const long long nu = s->n_unique;
        unpack_points(s, raw, nu * nfld,
                      [=](long long q) { return cells + (q % nfld) * nu + q / nfld; }, strain, u, v, a);
    }
    {
        std::lock_guard<std::mutex> lk(s->rec_mu);
        snap->readers--;
        if (!st && release) snap->done = true;
        while (!s->pending.empty() && s->pending.front().done && s->pending.front().readers == 0)
            s->pending.pop_front();
    }
    s->rec_cv.notify_all();
    return st;
}

gfb_status gfb_element_residual(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                                const double* lambda_, const double* mu, const double* D,
                                const double* weights, int32_t ngll, const double* u, double* r,
                                int32_t precision, int32_t device) {
    if (n_elem <= 0 || !dxi_dx || !jacobian || !lambda_ || !mu || !u || !r)
        return fail(GFB_ERR_INVALID, "element residual: missing input");
    if (ngll < 3 || ngll > 6) return fail(GFB_ERR_UNSUPPORTED, "ngll=%d outside 3..6", ngll);
    const int nn = ngll * ngll * ngll;
    const long long P = (long long)n_elem * nn;
    if (P >= (long long)gfb::kNodeMask) return fail(GFB_ERR_INVALID, "too many element nodes");
    // independent elements: every element-local point is its own node, one
    // colour, every point first-touch, so force == element-local residual
    std::vector<int32_t> ib(P);
    std::vector<double> mass(P, 1.0);
    for (long long q = 0; q < P; ++q) ib[q] = (int32_t)q;
    gfb_mesh m{};
    m.n_cell = n_elem;
    m.ngll = ngll;
    m.n_node = (int32_t)P;
    m.ibool = ib.data();
    m.dxi_dx = dxi_dx;
    m.jacobian = jacobian;
    m.lambda_ = lambda_;
    m.mu = mu;
    m.mass = mass.data();
    gfb_config c{};
    c.dt = 1.0;
    c.precision = precision;
    c.n_field = 1;
    c.device = device;
    c.record_slots = 1;
    gfb_solver* s = nullptr;
    gfb_status st = validate(&m, &c);
    if (st) return st;
    gfb_model one{};
    one.cell_end = n_elem;
    one.node_end = m.n_node;
    one.dt = c.dt;
    one.n_steps = INT32_MAX;
    // the caller's GLL tables, as compute_element_residual uses the tables
    // it is given (element_cpu.cpp:19-162); NULL selects the GLL tables of ngll
    if ((st = create_impl(&m, &c, nullptr, 1, &one, &s, weights, D))) return st;
    std::unique_ptr<gfb_solver, gfb_status (*)(gfb_solver*)> guard(s, gfb_destroy);
    // [point][4] padded vectors on the device
    const size_t nP = (size_t)P * 4;
    if (precision == GFB_FP64) {
        std::vector<double> h(nP, 0.0);
        for (long long q = 0; q < P; ++q)
            for (int c = 0; c < 3; ++c) h[q * 4 + c] = u[q * 3 + c];
        if ((st = h2d(s, s->ut, h.data(), nP * 8))) return st;
    } else {
        std::vector<float> h(nP, 0.0f);
        for (long long q = 0; q < P; ++q)
            for (int c = 0; c < 3; ++c) h[q * 4 + c] = (float)u[q * 3 + c];
        if ((st = h2d(s, s->ut, h.data(), nP * 4))) return st;
    }
    if ((st = launch_elem(s, 0))) return st;
    CU(cudaStreamSynchronize(s->stream));
    if (precision == GFB_FP64) {
        std::vector<double> h(nP);
        if ((st = d2h(s, h.data(), s->force, nP * 8))) return st;
        for (long long q = 0; q < P; ++q)
            for (int c = 0; c < 3; ++c) r[q * 3 + c] = h[q * 4 + c];
    } else {
        std::vector<float> h(nP);
        if ((st = d2h(s, h.data(), s->force, nP * 4))) return st;
        for (long long q = 0; q < P; ++q)
            for (int c = 0; c < 3; ++c) r[q * 3 + c] = h[q * 4 + c];
    }
    return GFB_OK;
}

}  // extern "C"

// Internal hooks shared with other translation units of this library.
namespace gfb {

gfb_status set_error(gfb_status st, const char* msg) { return fail(st, "%s", msg); }

bool gll_tables_for(int ngll, std::vector<double>& w, std::vector<double>& D) {
    std::vector<double> x;
    return gll_tables(ngll - 1, x, w, D);
}

SolverView solver_view(gfb_solver* s) {
    SolverView v;
    v.device = s->device;
    v.stream = s->stream;
    v.precision = s->prec;
    v.n_field = s->nfld;
    v.n_model = s->n_model;
    v.n_node = s->n_node;
    v.dt = s->dt;
    v.u = s->u;
    v.v = s->v;
    v.a = s->a;
    v.ut = s->ut;
    v.force = s->force;
    v.mass = s->mass;
    v.mstep = s->d_mstep;
    v.node_inv = &s->node_inv;
    v.node_perm = &s->node_perm;
    return v;
}

gfb_status solver_predict(gfb_solver* s) { return launch_predict(s); }

gfb_status solver_full_state(gfb_solver* s) { return leave_half_v(s); }

Layer* solver_layer(gfb_solver* s) { return s->layer; }

gfb_status solver_set_layer(gfb_solver* s, Layer* layer) {
    if (s->layer) layer_free(s->layer);
    s->layer = layer;
    if (layer) {
        gfb_status st = leave_half_v(s);
        if (st) return st;
    }
    if (layer) s->by_increments_ok = false;
    if (layer && s->refresh > 1) {
        // the layer adds its correction to the assembled force each step,
        // which must not accumulate: the force is evaluated in full from now
        s->refresh = 1;
        gfb_status st = launch_predict(s);
        if (st) return st;
    }
    // the captured step graph does not contain the layer's launch
    if (s->gexec) {
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return GFB_OK;
}

}  // namespace gfb
