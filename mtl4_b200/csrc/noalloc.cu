// Allocation-free variant of the fused SpMV + dot product (q = A p and p.q).
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory pool or a hard real-time loop where cudaMalloc may block
// or fail, a device-memory budget that is already fully reserved, or a
// process that must not touch the CUDA allocator after start-up.  This entry
// point takes only caller-owned device buffers and keeps its one scratch
// buffer -- the per-CTA partial sums of the dot product and a completion
// counter -- in a file-scope static device array, so it allocates nothing.
//
// Limits and rules:
//  * the array holds kNoAllocMaxCtas partial sums, so the matrix may have at
//    most kNoAllocMaxCtas * 256 = 1,048,576 rows; larger sizes are rejected;
//  * every GPU that loads the library holds the array (about 32 KiB) until
//    the process exits;
//  * every call uses the same array: calls that may overlap on the GPU (on
//    different streams, or from different host threads) race on it and must
//    be serialized by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is kept per device together
//    with the id of the CUDA context it belongs to; after cudaDeviceReset the
//    next call sees a new context and looks the address up again (so that
//    call, too, should come before any capture);
//  * with n_rows > 0, row_ptr, col, val, p and q must all be non-null (a
//    matrix without entries still passes a valid col and val pointer).
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/mtl4_b200/mtlg.h"

namespace mtlg {
void set_error(const char* fmt, ...);   // the library's last-error message (mtlg.cu)
}

namespace {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxCtas = 4096;
constexpr int kMaxDevices = 64;

// [0, kNoAllocMaxCtas): per-CTA partial dot products; the next slot holds the
// completion counter (reset to zero by the last CTA and by every call).
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxCtas + 2];

static std::mutex g_mu;
static double* g_scratch_ptr[kMaxDevices] = {nullptr};
static unsigned long long g_scratch_ctx[kMaxDevices] = {0};

// Driver entry points reached through the runtime (no link against libcuda):
// the current context and its process-unique id.
typedef CUresult (*PFN_ctx_current)(CUcontext*);
typedef CUresult (*PFN_ctx_id)(CUcontext, unsigned long long*);

unsigned long long current_ctx_id()
{
    static PFN_ctx_current get_current = nullptr;
    static PFN_ctx_id get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
        cudaGetLastError();
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;   // unknown: the cached address is kept
}

// One row per thread, entries summed in storage order as mtlg_spmv does for
// rows of up to 32 entries (products rounded before each addition, the row's
// last (L mod 4) entries fused); the CTA's share of p.q goes to
// scratch[blockIdx.x]; the last CTA to finish sums the partials in CTA order
// and writes *dot.
__global__ void __launch_bounds__(kNoAllocBlock)
k_spmv_dot_noalloc(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                   const double* __restrict__ val, const double* __restrict__ p, double* __restrict__ q,
                   double* __restrict__ dot, double* __restrict__ scratch)
{
    __shared__ double s_red[kNoAllocBlock / 32];
    __shared__ int s_last;
    const int i = blockIdx.x * kNoAllocBlock + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        double acc = 0.0;
        const int a = rp[i], e = rp[i + 1], tail = a + ((e - a) & ~3);
        for (int k = a; k < e; ++k)
            acc = k >= tail ? __fma_rn(val[k], p[ci[k]], acc) : __dadd_rn(acc, __dmul_rn(val[k], p[ci[k]]));
        q[i] = acc;
        part = p[i] * acc;
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = part;
    __syncthreads();
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxCtas);
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kNoAllocBlock / 32; ++w) s += s_red[w];
        scratch[blockIdx.x] = s;
        __threadfence();
        s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(scratch + b);
        *dot = s;
        *counter = 0u;
    }
}

int scratch_ptr(double** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MTLG_ERR_CUDA;
    // cudaFree(0) makes the device's primary context current, so that the
    // id read next names the context the kernel will run in (allocates nothing)
    cudaFree(nullptr);
    const unsigned long long ctx = current_ctx_id();
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev] || (ctx != 0 && ctx != g_scratch_ctx[dev])) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return MTLG_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_ptr[dev];
    return MTLG_OK;
}

}  // namespace

extern "C" int mtlg_spmv_dot_noalloc(int64_t n_rows, int64_t n_cols, const int32_t* row_ptr, const int32_t* col,
                                     const double* val, const double* p, double* q, double* dot, void* stream)
{
    if (n_rows < 0 || n_cols < 0 || !dot || (n_rows > 0 && (!row_ptr || !col || !val || !p || !q))) {
        mtlg::set_error("invalid argument: negative size or null pointer");
        return MTLG_ERR_INVALID_ARG;
    }
    if (n_rows != n_cols) {
        mtlg::set_error("p.q needs a square matrix (%lld x %lld)", (long long)n_rows, (long long)n_cols);
        return MTLG_ERR_NOT_SQUARE;
    }
    if (n_rows > int64_t(kNoAllocMaxCtas) * kNoAllocBlock) {
        mtlg::set_error("%lld rows exceed the allocation-free limit of %d rows (%d CTA partial sums)",
                        (long long)n_rows, kNoAllocMaxCtas * kNoAllocBlock, kNoAllocMaxCtas);
        return MTLG_ERR_TOO_LARGE;
    }
    double* scratch = nullptr;
    const int st = scratch_ptr(&scratch);
    if (st != MTLG_OK) {
        mtlg::set_error("cudaGetSymbolAddress of the scratch array failed");
        return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the counter must start at zero even after an interrupted earlier call
    if (cudaMemsetAsync(scratch + kNoAllocMaxCtas, 0, sizeof(unsigned), s) != cudaSuccess) return MTLG_ERR_CUDA;
    if (n_rows == 0) {
        if (cudaMemsetAsync(dot, 0, sizeof(double), s) != cudaSuccess) return MTLG_ERR_CUDA;
        return MTLG_OK;
    }
    const int grid = int((n_rows + kNoAllocBlock - 1) / kNoAllocBlock);
    k_spmv_dot_noalloc<<<grid, kNoAllocBlock, 0, s>>>(int(n_rows), row_ptr, col, val, p, q, dot, scratch);
    return cudaGetLastError() == cudaSuccess ? MTLG_OK : MTLG_ERR_CUDA;
}
