// gfb_noalloc.cu -- element internal force for callers that cannot allocate
// device memory.
//
// gfb_element_residual (gfb_solver.cu) allocates device buffers for every
// call: the inputs and output, the cell geometry repacked into the kernel's
// layout, the node table and the GLL derivative table.  Some callers cannot
// do that: code that embeds the kernel in a time loop whose device memory is
// owned by a caching pool (allocating behind the pool's back fragments it
// and can fail under memory pressure), code that must not trigger the
// implicit device synchronisation of cudaMalloc/cudaFree inside a
// latency-critical loop, and code running where the allocator is
// intercepted or forbidden.  Those callers already hold device buffers for
// their inputs and output; what they cannot provide is the kernel's
// scratch.  This file keeps that scratch in one fixed, file-scope device
// array instead.
//
// The array is kScratchBytes (8 MiB) per GPU; every GPU that loads this
// library holds it until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <vector>

#include "../../include/gfb.h"
#include "gfb_internal.h"
#include "gfb_kernels.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;

// The scratch.  Host code must not pass this symbol to a kernel: on the
// host it is only a stand-in, not a device address.  Its device address is
// obtained once per device with cudaGetSymbolAddress (scratch_on_device).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 256;
std::mutex g_scratch_mutex;

// Device address of g_scratch per device, with the id of the CUDA context it
// was looked up in.  A device reset (cudaDeviceReset, or the primary context
// released and created again) loads the library's device code into a new
// context, where the array can sit at another address; the id tells the
// contexts apart, so the address is looked up again in the new one.
struct ScratchAddr {
    bool valid = false;
    unsigned long long ctx_id = 0;
    void* addr = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];

// Driver entry points for the current context and its id, fetched through
// the runtime (the library does not link the driver library itself).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

bool current_context_id(int dev, unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return false;
    if (!ctx) {
        // no context bound to this host thread yet: bind the device's
        // primary context (the one the runtime launches into)
        if (cudaSetDevice(dev) != cudaSuccess || get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    }
    return get_id(ctx, id) == CUDA_SUCCESS;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// Scratch layout for n_elem cells of nn nodes: repacked geometry
// [cell][12][nn] (f64), node table [cell][nn] (u32), derivative table (f64).
struct Layout {
    size_t geom, ibool, dmat, total;
};

Layout layout_for(long long n_elem, int ngll) {
    const long long nn = (long long)ngll * ngll * ngll;
    Layout L;
    L.geom = 0;
    L.ibool = align256(L.geom + (size_t)n_elem * 12 * nn * sizeof(double));
    L.dmat = align256(L.ibool + (size_t)n_elem * nn * sizeof(uint32_t));
    L.total = align256(L.dmat + (size_t)ngll * ngll * sizeof(double));
    return L;
}

// Device address of g_scratch on the current device dev: looked up with
// cudaGetSymbolAddress on the first call in each CUDA context of the device
// (the first call on the device, and the first after a device reset), and
// taken from the cache otherwise.  If the driver cannot report the
// context's id, the address is looked up on every call.
gfb_status scratch_on_device(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return gfb::set_error(GFB_ERR_INVALID, "device ordinal out of range");
    unsigned long long ctx_id = 0;
    const bool have_id = current_context_id(dev, &ctx_id);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchAddr& c = g_scratch_addr[dev];
    if (!have_id || !c.valid || c.ctx_id != ctx_id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the scratch array failed: %s",
                     cudaGetErrorString(e));
            return gfb::set_error(GFB_ERR_CUDA, msg);
        }
        c.addr = p;
        c.ctx_id = ctx_id;
        c.valid = have_id;
    }
    *out = static_cast<unsigned char*>(c.addr);
    return GFB_OK;
}

struct GllTables {
    double w[8];
    double D[64];
};

// Reference-layout inputs -> the element kernel's layout in the scratch.
// Every scratch word the element kernel reads for these cells is written
// here, so no clearing is needed between calls.
template <int NG>
__global__ void repack_kernel(int n_elem, const double* dxi_dx, const double* jacobian, const double* lambda_,
                              const double* mu, GllTables t, double* geom, uint32_t* ibool, double* dmat) {
    constexpr int NN = NG * NG * NG;
    const long long total = (long long)n_elem * NN;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const long long e = q / NN;
        const int p = (int)(q - e * NN);
        const int i = p / (NG * NG), j = (p / NG) % NG, k = p % NG;
        double* o = geom + e * 12 * NN + p;
        for (int f = 0; f < 9; ++f) o[f * NN] = dxi_dx[q * 9 + f];
        o[9 * NN] = jacobian[q] * t.w[i] * t.w[j] * t.w[k];
        o[10 * NN] = lambda_[q];
        o[11 * NN] = mu[q];
        // every point is its own node and the only touch of it: the
        // kernel stores its residual straight into r
        ibool[q] = (uint32_t)q | gfb::kFirstTouch;
    }
    if (blockIdx.x == 0 && threadIdx.x < NG * NG) dmat[threadIdx.x] = t.D[threadIdx.x];
}

template <int NG>
gfb_status run(int n_elem, const double* dxi_dx, const double* jacobian, const double* lambda_, const double* mu,
               const double* u, double* r, unsigned char* scratch, const Layout& L, const GllTables& t,
               cudaStream_t stream) {
    using S = gfb::Shape<NG>;
    double* geom = reinterpret_cast<double*>(scratch + L.geom);
    uint32_t* ibool = reinterpret_cast<uint32_t*>(scratch + L.ibool);
    double* dmat = reinterpret_cast<double*>(scratch + L.dmat);
    const long long total = (long long)n_elem * S::NN;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    repack_kernel<NG><<<blocks, 256, 0, stream>>>(n_elem, dxi_dx, jacobian, lambda_, mu, t, geom, ibool, dmat);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof(msg), "element residual (no-alloc): repack kernel launch failed: %s",
                 cudaGetErrorString(e));
        return gfb::set_error(GFB_ERR_CUDA, msg);
    }
    gfb::ElemArgs<double> A{};
    A.e_begin = 0;
    A.e_end = n_elem;
    A.ibool = ibool;
    A.geom = geom;
    A.ut = u;
    A.force = r;
    A.dmat = dmat;
    A.pml_slot = nullptr;
    A.src_head = nullptr;
    A.mstf = nullptr;  // no source
    const int eblocks = (n_elem + S::EPB - 1) / S::EPB;
    gfb::elem_step_kernel<double, NG, 1>
        <<<eblocks, S::THREADS, gfb::elem_smem_bytes<double, NG, 1>(), stream>>>(A);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof(msg), "element residual (no-alloc): element kernel launch failed: %s",
                 cudaGetErrorString(e));
        return gfb::set_error(GFB_ERR_CUDA, msg);
    }
    return GFB_OK;
}

// Largest cell count whose scratch fits in kScratchBytes.
long long max_cells_for(int ngll) {
    if (ngll < 3 || ngll > 6) return 0;
    long long lo = 0, hi = (long long)kScratchBytes;
    while (lo < hi) {  // largest n with layout_for(n).total <= kScratchBytes
        const long long mid = (lo + hi + 1) / 2;
        if (layout_for(mid, ngll).total <= kScratchBytes) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace

extern "C" {

gfb_status gfb_element_residual_noalloc(int32_t n_elem, const double* dxi_dx, const double* jacobian,
                                        const double* lambda_, const double* mu, int32_t ngll, const double* u,
                                        double* r, void* stream) {
    if (!dxi_dx || !jacobian || !lambda_ || !mu || !u || !r)
        return gfb::set_error(GFB_ERR_INVALID, "element residual (no-alloc): missing device pointer");
    if (ngll < 3 || ngll > 6)
        return gfb::set_error(GFB_ERR_UNSUPPORTED, "element residual (no-alloc): ngll must be 3..6");
    if (n_elem <= 0) return gfb::set_error(GFB_ERR_INVALID, "element residual (no-alloc): n_elem must be > 0");
    const long long max_cells = max_cells_for(ngll);
    if (n_elem > max_cells) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "element residual (no-alloc): %d cells exceed the maximum of %lld cells at ngll=%d "
                 "(fixed %zu-byte scratch); split the call",
                 n_elem, max_cells, ngll, kScratchBytes);
        return gfb::set_error(GFB_ERR_INVALID, msg);
    }
    // an error left by an earlier, unrelated call would otherwise be read
    // back after this call's launches and reported as theirs: clear it (a
    // sticky error of a broken context comes back at the launches anyway)
    (void)cudaGetLastError();
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return gfb::set_error(GFB_ERR_NO_DEVICE, "no current CUDA device");
    unsigned char* scratch = nullptr;
    gfb_status st = scratch_on_device(dev, &scratch);
    if (st) return st;
    std::vector<double> w, D;
    if (!gfb::gll_tables_for(ngll, w, D)) return gfb::set_error(GFB_ERR_INVALID, "GLL tables failed");
    GllTables t{};
    for (int i = 0; i < ngll; ++i) t.w[i] = w[i];
    for (int i = 0; i < ngll * ngll; ++i) t.D[i] = D[i];
    const Layout L = layout_for(n_elem, ngll);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (ngll) {
        case 3: return run<3>(n_elem, dxi_dx, jacobian, lambda_, mu, u, r, scratch, L, t, s);
        case 4: return run<4>(n_elem, dxi_dx, jacobian, lambda_, mu, u, r, scratch, L, t, s);
        case 5: return run<5>(n_elem, dxi_dx, jacobian, lambda_, mu, u, r, scratch, L, t, s);
        default: return run<6>(n_elem, dxi_dx, jacobian, lambda_, mu, u, r, scratch, L, t, s);
    }
}

}  // extern "C"
