// Jacobi-PCG on a caller-provided CSR matrix that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands the
// whole device to its own memory pool (every byte reserved up front), or a
// solver plugin loaded into a process whose GPU memory is owned by another
// runtime, where an extra allocation would fail or break the owner's
// accounting.  For them phgGpuSolverPCGNoAlloc runs the same PCG kernels as
// phgGpuSolverPCG, but its working vectors live in one fixed array of device
// memory that belongs to this library (g_pcg_scratch below).  The array is
// part of the library image: every GPU that loads the library holds its
// kStaticScratchBytes until the process exits, and it bounds the problem
// size to PHG_GPU_NOALLOC_MAX_ROWS rows.
#include "../../include/phg_gpu.h"

#include "common.cuh"
#include "solve.h"

namespace phgb {
void set_last_error(const char *msg);     // capi.cu
void set_last_warning(const char *msg);   // capi.cu
}

#include <float.h>
#include <math.h>
#include <stdio.h>


namespace {

constexpr int64_t kMaxRows = PHG_GPU_NOALLOC_MAX_ROWS;
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Layout of the scratch array (byte offsets).
constexpr size_t kVec = align_up(sizeof(double) * kMaxRows);
constexpr size_t kOffDiag = 0;
constexpr size_t kOffR = kOffDiag + kVec;
constexpr size_t kOffP = kOffR + kVec;
constexpr size_t kOffAp = kOffP + kVec;
constexpr size_t kOffRp = kOffAp + kVec;
constexpr size_t kOffPartials = kOffRp + align_up(sizeof(int32_t) * (kMaxRows + 1));
// grid-sum workspace for the largest grid any grid sum may use (reduce.cuh)
constexpr size_t kOffSums = kOffPartials + align_up(sizeof(double) * phgb::red_partials_doubles(phgb::kRedMaxBlocks));
constexpr size_t kOffState = kOffSums + align_up(sizeof(double) * 2);
constexpr size_t kOffTicket = kOffState + align_up(sizeof(phgb::PcgState));
constexpr size_t kStaticScratchBytes = kOffTicket + align_up(sizeof(unsigned) * phgb::kRedTickets);

// The scratch memory.  In host code this name is only a stand-in for the
// symbol, not a device address; the device address comes from
// cudaGetSymbolAddress with the device current, on every call, below.
static __device__ __align__(256) unsigned char g_pcg_scratch[kStaticScratchBytes];

// records the message for phgGpuLastError() (kept in capi.cu)
int fail(int code, const char *msg) {
    phgb::set_last_error(msg);
    return code;
}

// Device address of the scratch array in the current device's context.  It
// is looked up on every call (a host-side table lookup once the library's
// device code is loaded), so a context that was reset and created again gets
// the array's new address.  The first lookup on a device loads the device
// code; that first call must not happen during a stream capture.
int scratch_address(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return fail(PHG_GPU_ERR_CUDA, "cudaGetSymbolAddress failed for the PCG scratch array");
    }
    *out = (unsigned char *)p;
    return PHG_GPU_OK;
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

__global__ void narrow_rows_kernel(int64_t n, const int64_t *in, int32_t *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i];
}

__global__ void diagonal_kernel(int64_t n, const int32_t *rp, const int32_t *ci, const double *va, double *d) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int32_t j = rp[i]; j < rp[i + 1]; j++)
            if (ci[j] == i) { v = va[j]; break; }
        d[i] = v;
    }
}

#define CKS(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            char b_[256];                                                          \
            snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));     \
            return fail(PHG_GPU_ERR_CUDA, b_);                                     \
        }                                                                          \
    } while (0)

constexpr int kChunk = 16;

int solve(int64_t n, const int64_t *ptr, const int32_t *cols, const double *vals, const double *rhs, double *x,
          double rtol, double btol, double atol, int maxit, cudaStream_t s, double *residual) {
    using namespace phgb;
    set_last_warning("");
    if (n <= 0 || ptr == nullptr || cols == nullptr || vals == nullptr || rhs == nullptr || x == nullptr || maxit < 0)
        return fail(PHG_GPU_ERR_ARG, "phgGpuSolverPCGNoAlloc: invalid arguments");
    if (n > kMaxRows) {
        char b[160];
        snprintf(b, sizeof(b), "phgGpuSolverPCGNoAlloc: %lld rows exceed the limit of %lld",
                 (long long)n, (long long)kMaxRows);
        return fail(PHG_GPU_ERR_LIMIT, b);
    }
    int dev = 0;
    CKS(cudaGetDevice(&dev));
    const void *ptrs[] = {ptr, cols, vals, rhs, x};
    for (const void *p : ptrs)
        if (!on_device(p, dev))
            return fail(PHG_GPU_ERR_ARG, "phgGpuSolverPCGNoAlloc: arguments must be device memory "
                                         "of the current device");
    unsigned char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != PHG_GPU_OK) return rc;
    double *D = (double *)(base + kOffDiag), *r = (double *)(base + kOffR);
    double *p = (double *)(base + kOffP), *Ap = (double *)(base + kOffAp);
    int32_t *rp = (int32_t *)(base + kOffRp);
    double *partials = (double *)(base + kOffPartials), *sums = (double *)(base + kOffSums);
    PcgState *st = (PcgState *)(base + kOffState);
    unsigned *ticket = (unsigned *)(base + kOffTicket);

    int64_t nnz = 0, first = 0;
    CKS(cudaMemcpyAsync(&nnz, ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CKS(cudaMemcpyAsync(&first, ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CKS(cudaStreamSynchronize(s));
    if (first != 0 || nnz < 0 || nnz >= INT32_MAX)
        return fail(PHG_GPU_ERR_ARG, "phgGpuSolverPCGNoAlloc: bad row pointers");

    // the array keeps the previous call's contents: reset what must start at 0
    CKS(cudaMemsetAsync(ticket, 0, sizeof(unsigned) * phgb::kRedTickets, s));
    narrow_rows_kernel<<<vec_blocks(n + 1), 256, 0, s>>>(n + 1, ptr, rp);
    diagonal_kernel<<<vec_blocks(n), 256, 0, s>>>(n, rp, cols, vals, D);
    CKS(cudaGetLastError());
    const int lpr = spmv_lanes_for((double)nnz / (double)n);

    double h[2];
    CKS(launch_init_sums(n, 0, x, rhs, D, partials, ticket, sums, s));
    CKS(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
    CKS(cudaStreamSynchronize(s));
    const double x1 = h[0], rb = sqrt(h[1]);
    auto is_zero = [](double a) { return fabs(a) < 10.0 * DBL_MIN; };
    if (is_zero(rb)) {
        CKS(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
        CKS(cudaStreamSynchronize(s));
        if (residual) *residual = 0.0;
        return 0;
    }
    CsrView A{n, rp, cols, vals};
    if (!is_zero(x1 / (double)n)) {
        CKS(launch_spmv(A, lpr, x, Ap, s));
        CKS(launch_residual(n, rhs, Ap, r, s));
    } else {
        CKS(cudaMemcpyAsync(r, rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    CKS(launch_init_sums(n, 1, x, r, D, partials, ticket, sums, s));
    CKS(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
    CKS(cudaStreamSynchronize(s));
    const double r0 = sqrt(h[0]), rz0 = h[1];
    if (!isfinite(rz0)) return fail(PHG_GPU_ERR_NAN, "phgGpuSolverPCGNoAlloc: zero or non-finite diagonal");
    double tol = r0 * rtol;
    if (tol < rb * btol) tol = rb * btol;
    if (tol < atol) tol = atol;

    PcgState hs{};
    hs.rz_cur = rz0;
    hs.residual = r0;
    hs.tol = tol;
    hs.maxit = maxit;
    hs.done = !(r0 > tol && 0 < maxit);
    CKS(cudaMemcpyAsync(st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    PcgBuffers B{A, x, r, p, Ap, D, partials, st, nullptr};
    while (!hs.done) {
        for (int i = 0; i < kChunk; i++) CKS(launch_pcg_iteration(B, lpr, s));
        CKS(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
        CKS(cudaStreamSynchronize(s));
    }
    if (residual) *residual = hs.residual;
    if (hs.status == PCG_NONFINITE) return fail(PHG_GPU_ERR_NAN, "PCG: non-finite residual");
    // a breakdown ends the iteration as in the reference (solver-phg.c:547-571):
    // x as it is, the iteration count returned, a warning recorded
    if (hs.status == PCG_BREAKDOWN)
        phgb::set_last_warning("phgGpuSolverPCGNoAlloc: PCG stopped, the matrix may not be SPD");
    return hs.nits;
}

}  // namespace

extern "C" int phgGpuSolverPCGNoAlloc(int64_t n, const int64_t *ptr, const int32_t *cols, const double *vals,
                                      const double *rhs, double *x, double rtol, double btol, double atol,
                                      int maxit, void *stream, double *residual) {
    return solve(n, ptr, cols, vals, rhs, x, rtol, btol, atol, maxit, (cudaStream_t)stream, residual);
}
