// The C ABI (include/phg_gpu.h): the system object, buffer management and
// host-side orchestration of the assembly and solver kernels.
#include "../../include/phg_gpu.h"

#include "assemble.h"
#include "common.cuh"
#include "fe_tables.h"
#include "solve.h"

#include <math.h>
#include <float.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

using namespace phgb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(PHG_GPU_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call,          \
                        cudaGetErrorString(e_));                                              \
    } while (0)

#define CHECK_RC(x)               \
    do {                          \
        int rc_ = (x);            \
        if (rc_ != PHG_GPU_OK)    \
            return rc_;           \
    } while (0)

// A device buffer that only grows.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    int ensure(size_t n) {
        if (n <= cap && p != nullptr) return PHG_GPU_OK;
        if (p != nullptr) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t bytes = (n > 0 ? n : 1) * sizeof(T);
        cudaError_t e = cudaMalloc((void **)&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PHG_GPU_ERR_CUDA, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
        }
        cap = n > 0 ? n : 1;
        return PHG_GPU_OK;
    }
    void release() {
        if (p != nullptr) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

bool is_device_ptr(const void *ptr) {
    if (ptr == nullptr) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

__global__ void widen_kernel(int64_t n, const int32_t *in, int64_t *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

__global__ void narrow_kernel(int64_t n, const int64_t *in, int32_t *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i];
}

// phgMatSetupDiagonal (matvec.c:500-549): first entry of row i in column i.
__global__ void diag_kernel(int64_t n, const int32_t *rp, const int32_t *ci, const double *va, double *d) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int32_t j = rp[i]; j < rp[i + 1]; j++)
            if (ci[j] == i) { v = va[j]; break; }
        d[i] = v;
    }
}

constexpr int kGraphChunk = 16;

}  // namespace

namespace phgb {
// Lets other translation units of the library report through phgGpuLastError().
void set_last_error(const char *msg) { g_last_error = msg; }
}  // namespace phgb

struct phgGpuSystem_ {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // mesh
    int64_t nvert = 0, nelem = 0;
    DevBuf<double> verts;
    DevBuf<int32_t> elems;
    bool have_mesh = false;

    // DOF layout
    int order = 0, N = 0;
    int64_t ndof = 0;
    DevBuf<int32_t> e2l, inc_ptr, inc, cnt, cursor;
    DevBuf<uint8_t> bdry;
    DevBuf<int64_t> scan_ws;
    bool have_dofs = false;

    // element tables
    int tab_order = 0;
    DevBuf<double> wk, gk, wr, br;

    // assembly buffers
    DevBuf<double> Ke, Re, kappa, f, g;
    DevBuf<int32_t> cnt_keep, cnt_bdry;

    // assembled system
    int64_t n = 0, nnz = 0, bnnz = 0;
    DevBuf<int32_t> rp, ci, brp, bci;
    DevBuf<double> va, bva, rhs, diag;
    bool assembled = false;
    bool have_bdry_cols = false;

    // solver
    DevBuf<double> x, r, p, Ap, partials, hist, sums;
    DevBuf<PcgState> st;
    DevBuf<unsigned> ticket;
    DevBuf<int64_t> tmp64;
    PcgState *h_st = nullptr;
    double *h_sums = nullptr;
    int *h_status = nullptr;
    DevBuf<int> status;
    cudaGraphExec_t graph = nullptr;
    struct GraphKey {
        const void *x, *r, *p, *Ap, *D, *va, *hist;
        int64_t n;
        int lpr;
        cudaStream_t s;
        bool operator==(const GraphKey &o) const { return memcmp(this, &o, sizeof(*this)) == 0; }
    } gkey{};
    int lpr = 8;
    int64_t launches = 0;   // kernels launched by this system (graph nodes included)
};

namespace {

int set_device(phgGpuSystem *s) {
    CK(cudaSetDevice(s->device));
    return PHG_GPU_OK;
}

int check_status(phgGpuSystem *s, const char *where) {
    CK(cudaMemcpyAsync(s->h_status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const int st = *s->h_status;
    if (st == PHGB_DEV_OK) return PHG_GPU_OK;
    *s->h_status = 0;
    CK(cudaMemsetAsync(s->status.p, 0, sizeof(int), s->stream));
    switch (st) {
    case PHGB_DEV_BAD_INDEX: return fail(PHG_GPU_ERR_ARG, "%s: vertex or DOF index out of range", where);
    case PHGB_DEV_ROW_OVERFLOW:
        return fail(PHG_GPU_ERR_LIMIT, "%s: a matrix row has more than %d entries", where,
                    row_walk_max_row(s->order));
    default: return fail(PHG_GPU_ERR_STATE, "%s: internal consistency check failed (%d)", where, st);
    }
}

// Copies n elements from src (host or device) to the device buffer dst.
template <typename T>
int copy_in(phgGpuSystem *s, T *dst, const T *src, size_t n) {
    if (n == 0) return PHG_GPU_OK;
    CK(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDefault, s->stream));
    return PHG_GPU_OK;
}

template <typename T>
int copy_out(phgGpuSystem *s, T *dst, const T *src, size_t n) {
    if (n == 0 || dst == nullptr) return PHG_GPU_OK;
    CK(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDefault, s->stream));
    return PHG_GPU_OK;
}

// Uses a device input in place, or stages a host input in `buf`.
template <typename T>
int stage(phgGpuSystem *s, const T *src, size_t n, DevBuf<T> &buf, const T **out) {
    if (src == nullptr) { *out = nullptr; return PHG_GPU_OK; }
    if (is_device_ptr(src)) { *out = src; return PHG_GPU_OK; }
    CHECK_RC(buf.ensure(n));
    CHECK_RC(copy_in(s, buf.p, src, n));
    *out = buf.p;
    return PHG_GPU_OK;
}

int upload_tables(phgGpuSystem *s, int p) {
    if (s->tab_order == p) return PHG_GPU_OK;
    const ElementTables t = make_tables(p);
    CHECK_RC(s->wk.ensure(t.wk.size()));
    CHECK_RC(s->gk.ensure(t.gk.size()));
    CHECK_RC(s->wr.ensure(t.wr.size()));
    CHECK_RC(s->br.ensure(t.br.size()));
    CK(cudaMemcpy(s->wk.p, t.wk.data(), t.wk.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->gk.p, t.gk.data(), t.gk.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->wr.p, t.wr.data(), t.wr.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->br.p, t.br.data(), t.br.size() * sizeof(double), cudaMemcpyHostToDevice));
    s->tab_order = p;
    return PHG_GPU_OK;
}

int solver_buffers(phgGpuSystem *s) {
    const size_t n = (size_t)s->n;
    CHECK_RC(s->x.ensure(n));
    CHECK_RC(s->r.ensure(n));
    CHECK_RC(s->p.ensure(n));
    CHECK_RC(s->Ap.ensure(n));
    CHECK_RC(s->partials.ensure(2 * (size_t)vec_blocks((int64_t)n * 32) + 64));
    CHECK_RC(s->sums.ensure(2));
    CHECK_RC(s->st.ensure(1));
    CHECK_RC(s->ticket.ensure(1));
    return PHG_GPU_OK;
}

}  // namespace

extern "C" {

const char *phgGpuLastError(void) { return g_last_error.c_str(); }

int phgGpuVersion(void) { return 100; }

int phgGpuCreate(int device, void *stream, phgGpuSystem **out) {
    if (out == nullptr) return fail(PHG_GPU_ERR_ARG, "phgGpuCreate: null output");
    *out = nullptr;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(PHG_GPU_ERR_ARG, "phgGpuCreate: no CUDA device %d", device);
    phgGpuSystem *s = new phgGpuSystem();
    s->device = device;
    int rc = set_device(s);
    if (rc == PHG_GPU_OK) {
        if (stream != nullptr) {
            s->stream = (cudaStream_t)stream;
        } else {
            cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) rc = fail(PHG_GPU_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
            s->own_stream = true;
        }
    }
    if (rc == PHG_GPU_OK) {
        cudaError_t e1 = cudaMallocHost((void **)&s->h_st, sizeof(PcgState));
        cudaError_t e2 = cudaMallocHost((void **)&s->h_sums, 2 * sizeof(double));
        cudaError_t e3 = cudaMallocHost((void **)&s->h_status, sizeof(int));
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
            rc = fail(PHG_GPU_ERR_CUDA, "cudaMallocHost failed");
    }
    if (rc == PHG_GPU_OK) rc = s->status.ensure(1);
    if (rc == PHG_GPU_OK) {
        *s->h_status = 0;
        cudaError_t e = cudaMemset(s->status.p, 0, sizeof(int));
        if (e != cudaSuccess) rc = fail(PHG_GPU_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    }
    if (rc != PHG_GPU_OK) {
        phgGpuDestroy(s);
        return rc;
    }
    *out = s;
    return PHG_GPU_OK;
}

int phgGpuDestroy(phgGpuSystem *s) {
    if (s == nullptr) return PHG_GPU_OK;
    cudaSetDevice(s->device);
    if (s->stream != nullptr) cudaStreamSynchronize(s->stream);
    if (s->graph != nullptr) cudaGraphExecDestroy(s->graph);
    DevBuf<double> *dbufs[] = {&s->verts, &s->wk, &s->gk, &s->wr, &s->br, &s->Ke, &s->Re, &s->kappa, &s->f,
                               &s->g, &s->va, &s->bva, &s->rhs, &s->diag, &s->x, &s->r, &s->p, &s->Ap,
                               &s->partials, &s->hist, &s->sums};
    for (auto *b : dbufs) b->release();
    DevBuf<int32_t> *ibufs[] = {&s->elems, &s->e2l, &s->inc_ptr, &s->inc, &s->cnt, &s->cursor, &s->cnt_keep,
                                &s->cnt_bdry, &s->rp, &s->ci, &s->brp, &s->bci};
    for (auto *b : ibufs) b->release();
    s->bdry.release();
    s->scan_ws.release();
    s->tmp64.release();
    s->st.release();
    s->ticket.release();
    s->status.release();
    if (s->h_st) cudaFreeHost(s->h_st);
    if (s->h_sums) cudaFreeHost(s->h_sums);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->own_stream && s->stream != nullptr) cudaStreamDestroy(s->stream);
    delete s;
    return PHG_GPU_OK;
}

int phgGpuSetStream(phgGpuSystem *s, void *stream) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    CHECK_RC(set_device(s));
    CK(cudaStreamSynchronize(s->stream));
    if (s->own_stream) {
        cudaStreamDestroy(s->stream);
        s->own_stream = false;
        s->stream = nullptr;
    }
    if (stream == nullptr) {
        CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    } else {
        s->stream = (cudaStream_t)stream;
    }
    return PHG_GPU_OK;
}

int phgGpuSetMesh(phgGpuSystem *s, int64_t nvert, const double *verts, int64_t nelem,
                  const int32_t *elem_verts) {
    if (s == nullptr || verts == nullptr || elem_verts == nullptr || nvert <= 0 || nelem <= 0)
        return fail(PHG_GPU_ERR_ARG, "phgGpuSetMesh: invalid arguments");
    if (nvert > INT32_MAX || nelem > INT32_MAX / 20)
        return fail(PHG_GPU_ERR_LIMIT, "phgGpuSetMesh: mesh too large for 32-bit indices");
    CHECK_RC(set_device(s));
    CHECK_RC(s->verts.ensure(3 * (size_t)nvert));
    CHECK_RC(s->elems.ensure(4 * (size_t)nelem));
    CHECK_RC(copy_in(s, s->verts.p, verts, 3 * (size_t)nvert));
    CHECK_RC(copy_in(s, s->elems.p, elem_verts, 4 * (size_t)nelem));
    s->nvert = nvert;
    s->nelem = nelem;
    s->have_mesh = true;
    s->have_dofs = false;
    s->assembled = false;
    return PHG_GPU_OK;
}

int phgGpuSetDofMap(phgGpuSystem *s, int order, int64_t ndof, const int32_t *e2l, const uint8_t *bdry) {
    if (s == nullptr || e2l == nullptr || bdry == nullptr || ndof <= 0)
        return fail(PHG_GPU_ERR_ARG, "phgGpuSetDofMap: invalid arguments");
    if (order < 1 || order > 3) return fail(PHG_GPU_ERR_ARG, "phgGpuSetDofMap: order %d not in 1..3", order);
    if (!s->have_mesh) return fail(PHG_GPU_ERR_STATE, "phgGpuSetDofMap: call phgGpuSetMesh first");
    if (ndof >= INT32_MAX) return fail(PHG_GPU_ERR_LIMIT, "phgGpuSetDofMap: too many DOFs");
    CHECK_RC(set_device(s));
    const int N = nbas(order);
    const size_t nk = (size_t)s->nelem * N;
    CHECK_RC(s->e2l.ensure(nk));
    CHECK_RC(s->bdry.ensure((size_t)ndof));
    CHECK_RC(s->cnt.ensure((size_t)ndof));
    CHECK_RC(s->cursor.ensure((size_t)ndof));
    CHECK_RC(s->inc_ptr.ensure((size_t)ndof + 1));
    CHECK_RC(s->inc.ensure(nk));
    CHECK_RC(s->scan_ws.ensure((size_t)scan_workspace_elems(ndof)));
    CHECK_RC(copy_in(s, s->e2l.p, e2l, nk));
    CHECK_RC(copy_in(s, s->bdry.p, bdry, (size_t)ndof));
    CHECK_RC(upload_tables(s, order));
    CK(launch_incidence(N, s->nelem, ndof, s->e2l.p, s->cnt.p, s->inc_ptr.p, s->cursor.p, s->inc.p,
                        s->scan_ws.p, s->status.p, s->stream));
    s->launches += 6;
    s->order = order;
    s->N = N;
    s->ndof = ndof;
    CHECK_RC(check_status(s, "phgGpuSetDofMap"));
    s->have_dofs = true;
    s->assembled = false;
    return PHG_GPU_OK;
}

int phgGpuBuildLinearSystem(phgGpuSystem *s, const double *kappa, const double *f, const double *g) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->have_dofs) return fail(PHG_GPU_ERR_STATE, "phgGpuBuildLinearSystem: call phgGpuSetDofMap first");
    CHECK_RC(set_device(s));
    const int N = s->N;
    const int64_t ndof = s->ndof;
    const double *dk, *df, *dg;
    CHECK_RC(stage(s, kappa, (size_t)s->nelem, s->kappa, &dk));
    CHECK_RC(stage(s, f, (size_t)ndof, s->f, &df));
    CHECK_RC(stage(s, g, (size_t)ndof, s->g, &dg));
    CHECK_RC(s->Ke.ensure((size_t)s->nelem * N * N));
    CHECK_RC(s->Re.ensure((size_t)s->nelem * N));

    ElemArgs ea{};
    ea.nelem = s->nelem; ea.nvert = s->nvert; ea.ndof = ndof;
    ea.verts = s->verts.p; ea.elems = s->elems.p; ea.e2l = s->e2l.p;
    ea.kappa = dk; ea.f = df;
    ea.wk = s->wk.p; ea.gk = s->gk.p; ea.wr = s->wr.p; ea.br = s->br.p;
    ea.Ke = s->Ke.p; ea.Re = s->Re.p; ea.status = s->status.p;
    CK(launch_element_kernel(s->order, ea, s->stream));
    s->launches += 1;

    CHECK_RC(s->cnt_keep.ensure((size_t)ndof));
    CHECK_RC(s->cnt_bdry.ensure((size_t)ndof));
    CHECK_RC(s->rp.ensure((size_t)ndof + 1));
    CHECK_RC(s->brp.ensure((size_t)ndof + 1));
    WalkArgs wa{};
    wa.ndof = ndof; wa.inc_ptr = s->inc_ptr.p; wa.inc = s->inc.p; wa.e2l = s->e2l.p; wa.bdry = s->bdry.p;
    wa.Ke = s->Ke.p; wa.Re = s->Re.p; wa.g = dg;
    wa.cnt_keep = s->cnt_keep.p; wa.cnt_bdry = s->cnt_bdry.p; wa.status = s->status.p;
    CK(launch_row_walk(s->order, false, wa, s->stream));
    s->launches += 7;   // pass 1 + two scans
    CK(launch_scan(ndof, s->cnt_keep.p, s->rp.p, s->scan_ws.p, s->stream));
    int32_t tot[2];
    CK(cudaMemcpyAsync(&tot[0], s->rp.p + ndof, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(launch_scan(ndof, s->cnt_bdry.p, s->brp.p, s->scan_ws.p, s->stream));
    CK(cudaMemcpyAsync(&tot[1], s->brp.p + ndof, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CHECK_RC(check_status(s, "phgGpuBuildLinearSystem (count)"));
    if (tot[0] < 0 || tot[1] < 0) return fail(PHG_GPU_ERR_LIMIT, "matrix has more than 2^31 entries");
    s->nnz = tot[0];
    s->bnnz = tot[1];
    CHECK_RC(s->ci.ensure((size_t)s->nnz));
    CHECK_RC(s->va.ensure((size_t)s->nnz));
    CHECK_RC(s->bci.ensure((size_t)s->bnnz));
    CHECK_RC(s->bva.ensure((size_t)s->bnnz));
    CHECK_RC(s->rhs.ensure((size_t)ndof));
    CHECK_RC(s->diag.ensure((size_t)ndof));
    wa.ptr = s->rp.p; wa.cols = s->ci.p; wa.vals = s->va.p;
    wa.bptr = s->brp.p; wa.bcols = s->bci.p; wa.bvals = s->bva.p;
    wa.rhs = s->rhs.p; wa.diag = s->diag.p;
    CK(launch_row_walk(s->order, true, wa, s->stream));
    s->launches += 1;
    CHECK_RC(check_status(s, "phgGpuBuildLinearSystem"));
    s->n = ndof;
    s->assembled = true;
    s->have_bdry_cols = true;
    s->lpr = spmv_lanes_for((double)s->nnz / (double)ndof);
    return PHG_GPU_OK;
}

int phgGpuSetMatrix(phgGpuSystem *s, int64_t n, const int64_t *ptr, const int32_t *cols, const double *vals,
                    const double *rhs) {
    if (s == nullptr || n <= 0 || ptr == nullptr || cols == nullptr || vals == nullptr || rhs == nullptr)
        return fail(PHG_GPU_ERR_ARG, "phgGpuSetMatrix: invalid arguments");
    if (n >= INT32_MAX) return fail(PHG_GPU_ERR_LIMIT, "phgGpuSetMatrix: too many rows");
    CHECK_RC(set_device(s));
    int64_t nnz = 0;
    CK(cudaMemcpy(&nnz, ptr + n, sizeof(int64_t), cudaMemcpyDefault));
    int64_t first = 0;
    CK(cudaMemcpy(&first, ptr, sizeof(int64_t), cudaMemcpyDefault));
    if (first != 0 || nnz < 0) return fail(PHG_GPU_ERR_ARG, "phgGpuSetMatrix: bad row pointers");
    if (nnz >= INT32_MAX) return fail(PHG_GPU_ERR_LIMIT, "phgGpuSetMatrix: more than 2^31 entries");
    CHECK_RC(s->tmp64.ensure((size_t)n + 1));
    CHECK_RC(s->rp.ensure((size_t)n + 1));
    CHECK_RC(s->ci.ensure((size_t)nnz));
    CHECK_RC(s->va.ensure((size_t)nnz));
    CHECK_RC(s->rhs.ensure((size_t)n));
    CHECK_RC(s->diag.ensure((size_t)n));
    CHECK_RC(copy_in(s, s->tmp64.p, ptr, (size_t)n + 1));
    narrow_kernel<<<vec_blocks(n + 1), 256, 0, s->stream>>>(n + 1, s->tmp64.p, s->rp.p);
    CHECK_RC(copy_in(s, s->ci.p, cols, (size_t)nnz));
    CHECK_RC(copy_in(s, s->va.p, vals, (size_t)nnz));
    CHECK_RC(copy_in(s, s->rhs.p, rhs, (size_t)n));
    diag_kernel<<<vec_blocks(n), 256, 0, s->stream>>>(n, s->rp.p, s->ci.p, s->va.p, s->diag.p);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    s->n = n;
    s->nnz = nnz;
    s->bnnz = 0;
    s->assembled = true;
    s->have_bdry_cols = false;
    s->lpr = spmv_lanes_for((double)nnz / (double)n);
    return PHG_GPU_OK;
}

int phgGpuGetSizes(phgGpuSystem *s, int64_t *n, int64_t *nnz, int64_t *nnz_bdry) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    if (n) *n = s->n;
    if (nnz) *nnz = s->nnz;
    if (nnz_bdry) *nnz_bdry = s->bnnz;
    return PHG_GPU_OK;
}

static int get_csr(phgGpuSystem *s, const DevBuf<int32_t> &rp, const DevBuf<int32_t> &ci, const DevBuf<double> &va,
                   int64_t nnz, int64_t *ptr, int32_t *cols, double *vals) {
    CHECK_RC(set_device(s));
    if (ptr != nullptr) {
        CHECK_RC(s->tmp64.ensure((size_t)s->n + 1));
        widen_kernel<<<vec_blocks(s->n + 1), 256, 0, s->stream>>>(s->n + 1, rp.p, s->tmp64.p);
        CK(cudaGetLastError());
        CHECK_RC(copy_out(s, ptr, s->tmp64.p, (size_t)s->n + 1));
    }
    CHECK_RC(copy_out(s, cols, ci.p, (size_t)nnz));
    CHECK_RC(copy_out(s, vals, va.p, (size_t)nnz));
    CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuGetMatrix(phgGpuSystem *s, int64_t *ptr, int32_t *cols, double *vals) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    return get_csr(s, s->rp, s->ci, s->va, s->nnz, ptr, cols, vals);
}

int phgGpuGetBdryColumns(phgGpuSystem *s, int64_t *ptr, int32_t *cols, double *vals) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->assembled || !s->have_bdry_cols)
        return fail(PHG_GPU_ERR_STATE, "no boundary columns (system not built by phgGpuBuildLinearSystem)");
    return get_csr(s, s->brp, s->bci, s->bva, s->bnnz, ptr, cols, vals);
}

int phgGpuGetRHS(phgGpuSystem *s, double *rhs) {
    if (s == nullptr || rhs == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(copy_out(s, rhs, s->rhs.p, (size_t)s->n));
    CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuGetDiagonal(phgGpuSystem *s, double *d) {
    if (s == nullptr || d == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(copy_out(s, d, s->diag.p, (size_t)s->n));
    CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuMatVec(phgGpuSystem *s, const double *x, double *y) {
    if (s == nullptr || x == nullptr || y == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    const bool xdev = is_device_ptr(x), ydev = is_device_ptr(y);
    const double *dx;
    CHECK_RC(stage(s, x, (size_t)s->n, s->p, &dx));
    double *dy = ydev ? y : s->Ap.p;
    CsrView A{s->n, s->rp.p, s->ci.p, s->va.p};
    CK(launch_spmv(A, s->lpr, dx, dy, s->stream));
    s->launches += 1;
    if (!ydev) CHECK_RC(copy_out(s, y, dy, (size_t)s->n));
    // device-to-device calls stay asynchronous on the system's stream
    if (!(xdev && ydev)) CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuGetLaunchCount(phgGpuSystem *s, int64_t *count) {
    if (s == nullptr || count == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    *count = s->launches;
    return PHG_GPU_OK;
}

int phgGpuSolverPCG(phgGpuSystem *s, double rtol, double btol, double atol, int maxit, double *x,
                    double *residual, double *hist) {
    if (s == nullptr || x == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    if (maxit < 0) return fail(PHG_GPU_ERR_ARG, "maxit < 0");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    const int64_t n = s->n;
    CHECK_RC(copy_in(s, s->x.p, x, (size_t)n));
    double *dhist = nullptr;
    if (hist != nullptr) {
        CHECK_RC(s->hist.ensure((size_t)maxit + 1));
        dhist = s->hist.p;
    }
    CK(cudaMemsetAsync(s->ticket.p, 0, sizeof(unsigned), s->stream));

    // ||b|| and |x|_1 (solver-phg.c:498-518)
    CK(launch_init_sums(n, 0, s->x.p, s->rhs.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double x1 = s->h_sums[0], rb = sqrt(s->h_sums[1]);
    auto is_zero = [](double a) { return fabs(a) < 10.0 * DBL_MIN; };   // utils.h:451
    if (is_zero(rb)) {
        CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
        CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
        CK(cudaStreamSynchronize(s->stream));
        if (residual) *residual = 0.0;
        if (hist) hist[0] = 0.0;
        return 0;
    }
    CsrView A{n, s->rp.p, s->ci.p, s->va.p};
    if (!is_zero(x1 / (double)n)) {
        CK(launch_spmv(A, s->lpr, s->x.p, s->Ap.p, s->stream));
        CK(launch_residual(n, s->rhs.p, s->Ap.p, s->r.p, s->stream));
        s->launches += 2;
    } else {
        CK(cudaMemcpyAsync(s->r.p, s->rhs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
    }
    CK(launch_init_sums(n, 1, s->x.p, s->r.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double r0 = sqrt(s->h_sums[0]), rz0 = s->h_sums[1];
    if (!isfinite(rz0)) return fail(PHG_GPU_ERR_NAN, "phgGpuSolverPCG: zero or non-finite diagonal");
    // get_tol (solver-phg.c:104-115)
    double tol = r0 * rtol;
    if (tol < rb * btol) tol = rb * btol;
    if (tol < atol) tol = atol;

    PcgState init{};
    init.rz_cur = rz0;
    init.residual = r0;
    init.tol = tol;
    init.maxit = maxit;
    init.done = !(r0 > tol && 0 < maxit);
    *s->h_st = init;
    CK(cudaMemcpyAsync(s->st.p, s->h_st, sizeof(PcgState), cudaMemcpyHostToDevice, s->stream));
    if (dhist) CK(cudaMemcpyAsync(dhist, &s->h_st->residual, sizeof(double), cudaMemcpyHostToDevice, s->stream));

    PcgBuffers B{A, s->x.p, s->r.p, s->p.p, s->Ap.p, s->diag.p, s->partials.p, s->st.p, dhist};
    phgGpuSystem_::GraphKey key{};
    key.x = B.x; key.r = B.r; key.p = B.p; key.Ap = B.Ap; key.D = B.D; key.va = A.va; key.hist = dhist;
    key.n = n; key.lpr = s->lpr; key.s = s->stream;
    if (s->graph == nullptr || !(s->gkey == key)) {
        if (s->graph != nullptr) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < kGraphChunk; i++) launch_pcg_iteration(B, s->lpr, s->stream);
        CK(cudaStreamEndCapture(s->stream, &gr));
        cudaError_t e = cudaGraphInstantiate(&s->graph, gr, 0);
        cudaGraphDestroy(gr);
        CK(e);
        s->gkey = key;
    }
    while (!s->h_st->done) {
        CK(cudaGraphLaunch(s->graph, s->stream));
        s->launches += 3 * kGraphChunk;
        CK(cudaMemcpyAsync(s->h_st, s->st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
    const int nits = s->h_st->nits;
    if (hist) CHECK_RC(copy_out(s, hist, dhist, (size_t)nits + 1));
    CK(cudaStreamSynchronize(s->stream));
    if (residual) *residual = s->h_st->residual;
    if (s->h_st->status == PCG_BREAKDOWN)
        return fail(PHG_GPU_ERR_BREAKDOWN, "PCG breakdown after %d iterations: the matrix may not be SPD", nits);
    if (s->h_st->status == PCG_NONFINITE)
        return fail(PHG_GPU_ERR_NAN, "PCG: non-finite residual after %d iterations", nits);
    return nits;
}

}  // extern "C"
