// hp_noalloc.cu -- time-step size of a conserved state, without allocating.
//
// Every other entry point works through a handle, and hp_create obtains all
// device memory with cudaMalloc.  Some callers cannot do that: a Fortran /
// OpenACC host whose device arrays belong to its compiler runtime and whose
// memory budget is fixed when its data region opens, or a framework that owns
// the whole GPU through its own pool allocator (cudaMalloc would fail once the
// pool has taken the memory, and it can synchronise the device in the middle
// of an asynchronous pipeline).  hp_dt_noalloc serves them: the caller passes
// its own device buffers for the inputs and the output, and the only scratch
// the computation needs -- one partial minimum per thread block -- lives in
// the file-scope array below, which every GPU that loads this library holds
// until the process exits.
//
// It is a variant of the start-of-step pass of the step kernels (primitive
// recovery of src/sr_primitive.F90:23-161 followed by the time-step
// reduction of src/main.F90:529-556), compiled like the FP64 parity variant
// (no FMA contraction), so its result equals the dt that hp_step reports for
// the same state, bit for bit.
#define HP_NS v_noalloc
#define HP_R double
#define HP_LSQ_TABLE 1
#include "hp_kernels.cuh"

#include <cuda.h>

#include <mutex>

#include "../../include/hydraphase.h"

namespace {

constexpr int kBlock = 256;
constexpr int kMaxBlocks = HP_NOALLOC_MAX_CELLS / kBlock;

// One partial minimum (bit pattern of a non-negative double) per block.
// Shared by every call on the device; each call writes the slots it reads,
// so nothing has to be cleared between calls.  Calls that overlap on the GPU
// (different streams, or threads issuing concurrently) race on it.
static __device__ __align__(256) unsigned long long g_dt_partial[kMaxBlocks];

std::mutex g_mu;
constexpr int kMaxDevices = 64;
// Device address of g_dt_partial per device, with the id of the CUDA context
// it was looked up in.  A context torn down and made again on the same device
// (cudaDeviceReset, or an OpenACC runtime that shuts the device down and
// opens a new data region) reloads this module at a new address, so the
// address is looked up again whenever the current context's id changes
// (context ids are never reused within a process).
struct Scratch { unsigned long long ctx_id; unsigned long long* ptr; };
Scratch g_dev[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the current context, through the driver entry points the runtime
// hands out (no link-time dependency on the driver library).
cudaError_t current_ctx_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            return cudaErrorNotSupported;
        get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorContextIsDestroyed;
    return get_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorContextIsDestroyed;
}

// Device address of g_dt_partial on the current device and context (the
// host-side name of the array is only a stand-in; a kernel must be given the
// device address).  Looked up once per device and context.
cudaError_t scratch_on_device(int dev, unsigned long long** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long id = 0;
    cudaError_t e = current_ctx_id(&id);
    if (e != cudaSuccess) return e;
    if (!g_dev[dev].ptr || g_dev[dev].ctx_id != id) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dt_partial);
        if (e != cudaSuccess) return e;
        g_dev[dev].ptr = static_cast<unsigned long long*>(p);
        g_dev[dev].ctx_id = id;
    }
    *out = g_dev[dev].ptr;
    return cudaSuccess;
}

using namespace hp;
using namespace hp::v_noalloc;

__global__ void __launch_bounds__(kBlock) k_dt_partial(const double* cn, long long ld, const double* dl, int n,
                                                       DevParams P, unsigned long long* part) {
    __shared__ unsigned long long red[kBlock / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = ~0ull;
    if (i < n) {
        double c[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = cn[(size_t)k * (size_t)ld + i];
        PrimV q;
        prim_full(c, q, P);
        double ag = sqrt((P.gamag * q.pg) / q.rog);
        double ap = sqrt((P.gamap * (q.pp + P.pinf)) / q.rop);
        double qg = sqrt(q.ug * q.ug + q.vg * q.vg + q.wg * q.wg);
        double qp = sqrt(q.up * q.up + q.vp * q.vp + q.wp * q.wp);
        double x = dl[i] / (mx2(ag, ap) + mx2(qg, qp));
        if (x == x) key = (unsigned long long)__double_as_longlong(x);
    }
    key = warp_min_u64(key);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = key;
    __syncthreads();
    if (wid == 0) {
        unsigned long long v = lane < kBlock / 32 ? red[lane] : ~0ull;
        v = warp_min_u64(v);
        if (lane == 0) part[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(1024) k_dt_final(const unsigned long long* part, int nblocks, double cfl,
                                                   double* dt_out) {
    __shared__ unsigned long long red[32];
    // the reference's running minimum starts at 1.0E8 (src/main.F90:521)
    unsigned long long v = (unsigned long long)__double_as_longlong(1.0e8);
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        unsigned long long w = part[b];
        v = w < v ? w : v;
    }
    v = warp_min_u64(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        unsigned long long w = lane < (int)(blockDim.x >> 5) ? red[lane] : ~0ull;
        w = warp_min_u64(w);
        if (lane == 0) dt_out[0] = __longlong_as_double((long long)w) * cfl;
    }
}

}  // namespace

// See include/hydraphase.h.
extern "C" int hp_dt_noalloc(const double* cn_dev, int64_t ld, const double* dl_dev, int32_t ncells,
                             const hp_params* params, double* dt_dev, void* stream) {
    if (!cn_dev || !dl_dev || !params || !dt_dev || ncells < 1 || ld < ncells) return HP_E_ARG;
    if (ncells > HP_NOALLOC_MAX_CELLS) return HP_E_ARG;   // beyond the scratch array
    // an error left pending by the caller's own CUDA work stays the caller's:
    // report it without launching and without clearing it
    if (cudaPeekAtLastError() != cudaSuccess) return HP_E_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HP_E_CUDA;
    unsigned long long* part = nullptr;
    if (scratch_on_device(dev, &part) != cudaSuccess) return HP_E_CUDA;
    const hp_params& p = *params;
    DevParams P{};
    P.gamag = p.gamag; P.gamap = p.gamap; P.pinf = p.pinf; P.cpp = p.cpp; P.cpg = p.cpg; P.prg = p.prg;
    P.rrg = 287.0; P.prp = 10.0;
    P.emin = p.epslnmin; P.emax = p.epslnmax;
    P.fsd = 4.0 * p.surfacetension / p.diap;
    P.cfl = p.cfl;
    P.r_emm = 1.0 / (P.emax - P.emin);
    const int nblocks = (ncells + kBlock - 1) / kBlock;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_dt_partial<<<nblocks, kBlock, 0, st>>>(cn_dev, ld, dl_dev, ncells, P, part);
    k_dt_final<<<1, 1024, 0, st>>>(part, nblocks, p.cfl, dt_dev);
    // nothing was pending on entry, so an error now is this call's launch
    return cudaGetLastError() == cudaSuccess ? HP_OK : HP_E_CUDA;
}
