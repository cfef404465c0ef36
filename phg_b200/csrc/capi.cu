// The C ABI (include/phg_gpu.h): the system object, buffer management and
// host-side orchestration of the assembly and solver kernels.
#include "../../include/phg_gpu.h"

#include "assemble.h"
#include "common.cuh"
#include "fe_tables.h"
#include "solve.h"
#include "q16.h"
#include "adjoint.h"
#include "block.h"
#include "bicgstab.h"
#include "gmres.h"
#include "mixed.h"

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
thread_local std::string g_last_warning;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// A condition the reference reports with a warning and survives (a PCG
// breakdown: solver-phg.c:547-571 prints "the matrix may not be SPD" and
// returns the iteration count).
void warn(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_warning = buf;
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

// Flags a NaN or infinite value of v in *status.
__global__ void nonfinite_kernel(int64_t n, const double *v, int *status) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!isfinite(v[i])) atomicExch(status, PHGB_DEV_NONFINITE);
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

// SpMV autotuner candidates: CSR with 4/8/16/32 lanes per row, SELL-C-sigma
// with the inner loop unrolled 2/4/8 times, q16 (FP64 values; only for
// matrices whose rows fit two 65536-column windows).
constexpr int kTuneCandidates = 8;
constexpr int kTune32 = 8;   // FP32 candidates of the mixed solver
const int kTuneKind[kTuneCandidates] = {SPMV_CSR,  SPMV_CSR,  SPMV_CSR,  SPMV_CSR,
                                        SPMV_SELL, SPMV_SELL, SPMV_SELL, SPMV_Q16};
const int kTuneParam[kTuneCandidates] = {4, 8, 16, 32, 2, 4, 8, 1};

}  // namespace

namespace phgb {
// Lets other translation units of the library report through phgGpuLastError().
void set_last_error(const char *msg) { g_last_error = msg; }
void set_last_warning(const char *msg) { g_last_warning = msg; }
}  // namespace phgb

struct phgGpuSystem_ {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // solver graphs without conditional nodes, relaunched by the host per
    // chunk ($PHG_GPU_PLAIN_GRAPHS=1 at creation): profilers do not see the
    // kernels inside conditional nodes
    bool plain_graphs = false;

    // mesh
    int64_t nvert = 0, nelem = 0;
    DevBuf<double> verts;
    DevBuf<int32_t> elems;
    bool have_mesh = false;
    bool geometry_given = false;           // s->geo holds PHG's geometry (phgGpuSetGeometry)
    bool geometry_valid = false;           // s->geo holds this mesh's geometry, checked by a build

    // DOF layout
    int order = 0, N = 0;
    int64_t ndof = 0;
    DevBuf<int32_t> e2l, inc_ptr, inc, cnt, cursor;
    DevBuf<uint8_t> bdry;
    DevBuf<int64_t> scan_ws;
    bool have_dofs = false;

    // element tables
    int tab_order = 0;
    DevBuf<double> gk, br, brt;            // basis derivatives / values at the points (device)
    std::vector<double> wk, wr;            // quadrature weights (passed to the kernel by value)

    // assembly buffers
    DevBuf<double> Ke, Re, kappa, f, g, geo;
    DevBuf<int32_t> sc_cols;          // row-walk scratch (nelem * N * N entries)
    DevBuf<double> sc_vals;
    DevBuf<int32_t> cnt_keep, cnt_bdry;
    DevBuf<int32_t> over_list;        // rows the row walk's second pass assembles
    DevBuf<int> nover;
    // the assembly pattern of this mesh and DOF map (slots of the
    // contributions, places of the row entries), for builds that only change
    // kappa, f, g or the mass coefficient: 0 none yet, 1 one build done (the
    // next records the pattern), 2 recorded (builds use the value walk)
    int pattern_state = 0;
    DevBuf<uint16_t> slot, tmap;
    DevBuf<int32_t> dpos;                  // per row, its diagonal's index among the kept entries
    // rows assembled from recorded row segments (phgGpuAssembleRows)
    DevBuf<int32_t> rec_row, rec_cols, rec_inc_ptr, rec_inc, rec_cnt, rec_cursor, rec_cap, rec_cap_ptr;
    DevBuf<int64_t> rec_ptr;
    DevBuf<double> rec_vals;

    // assembled system
    int64_t n = 0, nnz = 0, bnnz = 0;
    DevBuf<int32_t> rp, ci, brp, bci;
    DevBuf<double> va, bva, rhs, diag;
    bool assembled = false;
    double mass = 0.0;   // mass coefficient of the built system
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
        const void *extra[8];   // further buffers a graph's kernels use (layout arrays)
        int64_t n;
        int lpr;
        cudaStream_t s;
        bool operator==(const GraphKey &o) const { return memcmp(this, &o, sizeof(*this)) == 0; }
    } gkey{};
    int lpr = 8;
    int64_t launches = 0;   // kernels launched by this system (graph nodes included)

    // SpMV layout chosen by the autotuner, and the SELL-C-sigma copy
    SpmvPlan plan;
    bool sell_valid = false;
    int64_t sell_total = 0;
    DevBuf<int32_t> sell_perm, sell_ssz, sell_sptr, sell_cols;
    DevBuf<uint16_t> sell_len;
    DevBuf<double> sell_vals;
    DevBuf<float> sell_vals32;
    bool tuned = false;
    int64_t tuned_n = -1, tuned_nnz = -1;
    int unroll32 = 0;                 // FP32 product unroll (0: not tuned yet)
    int kind32 = 0;                   // FP32 product layout: 0 SELL, 1 pair SELL
    double tune32_ms[kTune32] = {};
    bool sell2_valid = false;
    DevBuf<int32_t> sell2_ssz, sell2_sptr, sell2_cols, sell2_order, sell2_perm;
    DevBuf<uint16_t> sell2_width, sell2_len;
    DevBuf<float> sell2_vals;
    bool sell_sorted = false;         // sell_perm / sell_len / sell_ssz of the current matrix
    bool order_valid = false;         // sell2_order (slices widest first) of the current matrix
    int64_t tuned32_n = -1, tuned32_nnz = -1;
    // 16-bit-column layout (q16.h), built when every row fits two windows
    bool q16_valid = false;           // built for the current matrix
    bool q16_fits = false;            // ... and usable
    DevBuf<int32_t> q16_ssz, q16_sptr, q16_perm, q16_b0, q16_b1;
    DevBuf<uint16_t> q16_len, q16_split, q16_cols;
    DevBuf<float> q16_v32;
    DevBuf<double> q16_v64;
    DevBuf<int32_t> q16_src;          // CSR index of each stored q16 entry (value refills)
    DevBuf<int> q16_nofit;
    int *h_nofit = nullptr;
    int64_t sell2_total = 0, q16_total = 0;   // stored entries (padding included)
    int64_t pair_entries = 0, q16_entries = 0; // the same, known from the slice widths
    double tune_ms[kTuneCandidates] = {};

    // mixed-precision solver
    DevBuf<float> r32, p32, Ap32, y32, D32;
    // adjoint gradient
    DevBuf<double> adj_u, adj_uobs, adj_rhs, adj_lambda, adj_grad;

    // block PCG
    DevBuf<double> bX, bR, bP, bAP, bB, bscal, bpart;
    DevBuf<float> bY32, bR32, bP32, bAP32, bva32;
    DevBuf<int> bint;
    DevBuf<unsigned> btick;
    int btile = 0;                      // autotuned SpMM tile (columns)
    int64_t btile_n = -1, btile_nnz = -1;
    int btile_K = -1;
    double btile_ms[4] = {};
    cudaGraphExec_t graph_block = nullptr;
    GraphKey gkey_block{};
    DevBuf<float> u32, s32;             // mixed solver: u = D^-1 r, s = A p
    DevBuf<GearState> gst;
    GearState *h_gst_mixed = nullptr;
    cudaGraphExec_t graph_mixed = nullptr;
    GraphKey gkey_mixed{};
    // BiCGstab: its seven working vectors in one buffer, its state
    DevBuf<double> bicg_vecs;
    DevBuf<BicgState> bicg_st;
    BicgState *h_bst = nullptr;
    cudaGraphExec_t graph_bicg = nullptr;
    GraphKey gkey_bicg{};
    // GMRES: z and the restart + 2 basis vectors, the small dense arrays, state
    DevBuf<double> gm_vecs, gm_small;
    DevBuf<GmresState> gm_st;
    GmresState *h_gst = nullptr;
    cudaGraphExec_t graph_gmres = nullptr;
    GraphKey gkey_gmres{};
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
    case PHGB_DEV_NONFINITE:
        return fail(PHG_GPU_ERR_NAN, "%s: a coordinate, kappa, f or g value is NaN or infinite", where);
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
    if ((int)t.wk.size() > kElemMaxQK || (int)t.wr.size() > kElemMaxQR)
        return fail(PHG_GPU_ERR_LIMIT, "quadrature rule larger than the element kernel's");
    // the kernel reads gk component-major with the basis index fastest, and
    // br both point-major (the RHS sums) and basis-major (f_h at the points)
    const int N = t.N, QK = t.nq_k, QR = t.nq_r;
    std::vector<double> gkc(t.gk.size()), brt(t.br.size());
    for (int q = 0; q < QK; q++)
        for (int k = 0; k < N; k++)
            for (int c = 0; c < 4; c++) gkc[((size_t)c * QK + q) * N + k] = t.gk[((size_t)q * N + k) * 4 + c];
    for (int q = 0; q < QR; q++)
        for (int k = 0; k < N; k++) brt[(size_t)k * QR + q] = t.br[(size_t)q * N + k];
    CHECK_RC(s->gk.ensure(gkc.size()));
    CHECK_RC(s->br.ensure(t.br.size()));
    CHECK_RC(s->brt.ensure(brt.size()));
    CK(cudaMemcpy(s->gk.p, gkc.data(), gkc.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->br.p, t.br.data(), t.br.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->brt.p, brt.data(), brt.size() * sizeof(double), cudaMemcpyHostToDevice));
    s->wk = t.wk;
    s->wr = t.wr;
    s->tab_order = p;
    return PHG_GPU_OK;
}

int solver_buffers(phgGpuSystem *s) {
    const size_t n = (size_t)s->n;
    CHECK_RC(s->x.ensure(n));
    CHECK_RC(s->r.ensure(n));
    CHECK_RC(s->p.ensure(n));
    CHECK_RC(s->Ap.ensure(n));
    // grid sums of two or three values over at most kRedMaxBlocks blocks
    CHECK_RC(s->partials.ensure((size_t)red_partials3_doubles(kRedMaxBlocks) + 64));
    CHECK_RC(s->sums.ensure(4));
    CHECK_RC(s->st.ensure(1));
    CHECK_RC(s->ticket.ensure(kRedTickets));
    return PHG_GPU_OK;
}

// Forgets every layout derived from the matrix (called when it changes).
// New values in an unchanged pattern: the layouts built so far keep their
// structure and take the values again.
int refresh_layout_values(phgGpuSystem *s) {
    const int64_t n = s->n;
    if (s->sell_valid) {
        CK(launch_sell_fill(n, s->rp.p, s->ci.p, s->va.p, s->sell_perm.p, s->sell_len.p, s->sell_sptr.p,
                            s->sell_cols.p, s->sell_vals.p, s->sell_vals32.p, s->stream));
        s->launches += 1;
    }
    if (s->sell2_valid) {
        const int64_t nsl = sell_positions(n) / 32;
        const SellView S{n, nsl, s->sell_perm.p, s->sell_len.p, nullptr, nullptr, nullptr, nullptr};
        CK(launch_sell2_fill(S, s->rp.p, s->ci.p, s->va.p, s->sell2_order.p, s->sell2_sptr.p, s->sell2_perm.p,
                             s->sell2_len.p, s->sell2_cols.p, s->sell2_vals.p, s->stream));
        s->launches += 1;
    }
    if (s->q16_valid && s->q16_fits) {
        CK(launch_q16_refill(s->q16_total, s->q16_src.p, s->va.p, s->q16_v32.p, s->q16_v64.p, s->stream));
        s->launches += 1;
    }
    return PHG_GPU_OK;
}

void invalidate_layouts(phgGpuSystem *s) {
    s->sell_sorted = false;
    s->order_valid = false;
    s->sell_valid = false;
    s->sell2_valid = false;
    s->q16_valid = false;
    s->q16_fits = false;
}

// Rows sorted by length in 256-row windows (the slices of every SELL layout).
int ensure_sell_sort(phgGpuSystem *s) {
    if (s->sell_sorted) return PHG_GPU_OK;
    const int64_t n = s->n, npos = sell_positions(n), nsl = npos / 32;
    CHECK_RC(s->sell_perm.ensure((size_t)npos));
    CHECK_RC(s->sell_len.ensure((size_t)npos));
    CHECK_RC(s->sell_ssz.ensure((size_t)nsl));
    CK(launch_sell_sort(n, s->rp.p, s->sell_perm.p, s->sell_len.p, s->sell_ssz.p, s->stream));
    s->launches += 1;
    s->sell_sorted = true;
    return PHG_GPU_OK;
}

// Builds the SELL-C-sigma copy of the current CSR (values in FP64 and FP32).
int ensure_sell(phgGpuSystem *s) {
    if (s->sell_valid) return PHG_GPU_OK;
    CHECK_RC(ensure_sell_sort(s));
    const int64_t n = s->n, npos = sell_positions(n), nsl = npos / 32;
    CHECK_RC(s->sell_sptr.ensure((size_t)nsl + 1));
    CHECK_RC(s->scan_ws.ensure((size_t)scan_workspace_elems(nsl)));
    CK(launch_scan(nsl, s->sell_ssz.p, s->sell_sptr.p, s->scan_ws.p, s->stream));
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, s->sell_sptr.p + nsl, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (total < 0) return fail(PHG_GPU_ERR_LIMIT, "SELL layout larger than 2^31 entries");
    CHECK_RC(s->sell_cols.ensure((size_t)total));
    CHECK_RC(s->sell_vals.ensure((size_t)total));
    CHECK_RC(s->sell_vals32.ensure((size_t)total));
    CK(launch_sell_fill(n, s->rp.p, s->ci.p, s->va.p, s->sell_perm.p, s->sell_len.p, s->sell_sptr.p,
                        s->sell_cols.p, s->sell_vals.p, s->sell_vals32.p, s->stream));
    s->launches += 4;
    s->sell_total = total;
    s->sell_valid = true;
    return PHG_GPU_OK;
}

// The order in which the pair and q16 layouts store the slices: widest
// first (a stable counting sort of the slice widths, on the host).
int ensure_slice_order(phgGpuSystem *s) {
    if (s->order_valid) return PHG_GPU_OK;
    CHECK_RC(ensure_sell_sort(s));
    const int64_t nsl = sell_positions(s->n) / 32;
    const SellView S{s->n, nsl, s->sell_perm.p, s->sell_len.p, nullptr, nullptr, nullptr, nullptr};
    CHECK_RC(s->sell2_width.ensure((size_t)nsl));
    CHECK_RC(s->sell2_order.ensure((size_t)nsl));
    CK(launch_sell2_heads(S, s->sell2_width.p, s->stream));
    s->launches += 1;
    std::vector<uint16_t> w((size_t)nsl);
    std::vector<int32_t> order((size_t)nsl);
    CK(cudaMemcpyAsync(w.data(), s->sell2_width.p, sizeof(uint16_t) * nsl, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    std::vector<int64_t> start(65537, 0);
    for (int64_t i = 0; i < nsl; i++) start[65535 - w[i] + 1]++;
    for (int b = 1; b <= 65536; b++) start[b] += start[b - 1];
    for (int64_t i = 0; i < nsl; i++) order[start[65535 - w[i]]++] = (int32_t)i;
    // stored entries of the pair and q16 layouts, exactly, in 64 bits
    s->pair_entries = 0;
    s->q16_entries = 0;
    for (int64_t i = 0; i < nsl; i++) {
        s->pair_entries += 64 * (((int64_t)w[i] + 1) / 2);
        s->q16_entries += 128 * (((int64_t)w[i] + 3) / 4);
    }
    CK(cudaMemcpyAsync(s->sell2_order.p, order.data(), sizeof(int32_t) * nsl, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->order_valid = true;
    return PHG_GPU_OK;
}

// The FP32 pair layout (mixed solver), built from CSR in the SELL slices.
int ensure_sell2(phgGpuSystem *s) {
    if (s->sell2_valid) return PHG_GPU_OK;
    CHECK_RC(ensure_slice_order(s));
    const int64_t nsl = sell_positions(s->n) / 32;
    CHECK_RC(s->sell2_ssz.ensure((size_t)nsl));
    CHECK_RC(s->sell2_sptr.ensure((size_t)nsl + 1));
    CHECK_RC(s->scan_ws.ensure((size_t)scan_workspace_elems(nsl)));
    const SellView S{s->n, nsl, s->sell_perm.p, s->sell_len.p, nullptr, nullptr, nullptr, nullptr};
    CK(launch_sell2_sizes(S, s->sell2_order.p, s->sell2_ssz.p, s->stream));
    CK(launch_scan(nsl, s->sell2_ssz.p, s->sell2_sptr.p, s->scan_ws.p, s->stream));
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, s->sell2_sptr.p + nsl, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->pair_entries >= (int64_t)INT32_MAX || (int64_t)total != s->pair_entries)
        return fail(PHG_GPU_ERR_LIMIT, "pair SELL layout larger than 2^31 entries");
    CHECK_RC(s->sell2_cols.ensure((size_t)total));
    CHECK_RC(s->sell2_vals.ensure((size_t)total));
    CHECK_RC(s->sell2_perm.ensure((size_t)nsl * 32));
    CHECK_RC(s->sell2_len.ensure((size_t)nsl * 32));
    CK(launch_sell2_fill(S, s->rp.p, s->ci.p, s->va.p, s->sell2_order.p, s->sell2_sptr.p, s->sell2_perm.p,
                         s->sell2_len.p, s->sell2_cols.p, s->sell2_vals.p, s->stream));
    s->launches += 3;
    s->sell2_total = total;
    s->sell2_valid = true;
    return PHG_GPU_OK;
}

// The 16-bit-column layout with FP32 and FP64 values.  Sets q16_fits to
// whether every row fits two column windows; the layout is used only then.
int ensure_q16(phgGpuSystem *s) {
    if (s->q16_valid) return PHG_GPU_OK;
    CHECK_RC(ensure_slice_order(s));
    const int64_t nsl = sell_positions(s->n) / 32, npos = nsl * 32;
    {   // the layout is an optimisation: without room for it (32-bit offsets,
        // or 90% of the free device memory) it is simply not offered
        auto grow = [](int64_t need, size_t cap, int64_t bytes) { return need > (int64_t)cap ? (need - (int64_t)cap) * bytes : 0; };
        const int64_t e = s->q16_entries;
        const int64_t extra = grow(e, s->q16_cols.cap, 2) + grow(e, s->q16_v32.cap, 4) + grow(e, s->q16_v64.cap, 8) +
                              grow(npos, s->q16_perm.cap, 16);
        size_t free_b = 0, total_b = 0;
        if (extra > 0) CK(cudaMemGetInfo(&free_b, &total_b));   // only when the buffers must grow
        if (e >= (int64_t)INT32_MAX || (extra > 0 && extra > (int64_t)(0.9 * (double)free_b))) {
            s->q16_valid = true;
            s->q16_fits = false;
            return PHG_GPU_OK;
        }
    }
    CHECK_RC(s->q16_ssz.ensure((size_t)nsl));
    CHECK_RC(s->q16_sptr.ensure((size_t)nsl + 1));
    CHECK_RC(s->scan_ws.ensure((size_t)scan_workspace_elems(nsl)));
    CHECK_RC(s->q16_nofit.ensure(1));
    if (s->h_nofit == nullptr) CK(cudaMallocHost((void **)&s->h_nofit, sizeof(int)));
    CK(launch_q16_sizes(nsl, s->sell_len.p, s->sell2_order.p, s->q16_ssz.p, s->stream));
    CK(launch_scan(nsl, s->q16_ssz.p, s->q16_sptr.p, s->scan_ws.p, s->stream));
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, s->q16_sptr.p + nsl, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if ((int64_t)total != s->q16_entries) return fail(PHG_GPU_ERR_CUDA, "q16 layout: slice sizes disagree");
    CHECK_RC(s->q16_cols.ensure((size_t)total));
    CHECK_RC(s->q16_v32.ensure((size_t)total));
    CHECK_RC(s->q16_v64.ensure((size_t)total));
    CHECK_RC(s->q16_src.ensure((size_t)total));
    CHECK_RC(s->q16_perm.ensure((size_t)npos));
    CHECK_RC(s->q16_len.ensure((size_t)npos));
    CHECK_RC(s->q16_split.ensure((size_t)npos));
    CHECK_RC(s->q16_b0.ensure((size_t)npos));
    CHECK_RC(s->q16_b1.ensure((size_t)npos));
    CK(cudaMemsetAsync(s->q16_nofit.p, 0, sizeof(int), s->stream));
    const Q16Out O{s->q16_sptr.p, s->q16_perm.p, s->q16_len.p, s->q16_split.p, s->q16_b0.p, s->q16_b1.p,
                   s->q16_cols.p, s->q16_v32.p, s->q16_v64.p, s->q16_src.p};
    CK(launch_q16_fill(nsl, s->rp.p, s->ci.p, s->va.p, s->sell_perm.p, s->sell_len.p, s->sell2_order.p, O,
                       s->q16_nofit.p, s->stream));
    CK(cudaMemcpyAsync(s->h_nofit, s->q16_nofit.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->launches += 3;
    s->q16_total = total;
    s->q16_valid = true;
    s->q16_fits = *s->h_nofit == 0;
    return PHG_GPU_OK;
}

SellView sell_view(phgGpuSystem *s) {
    return SellView{s->n, sell_positions(s->n) / 32, s->sell_perm.p, s->sell_len.p, s->sell_sptr.p,
                    s->sell_cols.p, s->sell_vals.p, s->sell_vals32.p};
}

Sell2View sell2_view(phgGpuSystem *s) {
    return Sell2View{s->sell2_sptr.p, s->sell2_cols.p, s->sell2_vals.p, s->sell2_perm.p, s->sell2_len.p};
}

Q16View q16_view(phgGpuSystem *s) {
    return Q16View{sell_positions(s->n) / 32, s->q16_sptr.p, s->q16_perm.p, s->q16_len.p, s->q16_split.p,
                   s->q16_b0.p, s->q16_b1.p, s->q16_cols.p, s->q16_v32.p, s->q16_v64.p};
}

// FP32 product of the mixed solver on layout `kind` (0 SELL, 1 pair SELL,
// 2 q16) with unroll `u`.
int launch_fp32_product(phgGpuSystem *s, int kind, int u, const float *x, float *y) {
    if (kind == 2) CK(launch_q16_spmv32(q16_view(s), u, x, y, s->stream));
    else CK(launch_spmv32k(sell_view(s), sell2_view(s), kind, u, x, y, s->stream));
    s->launches += 1;
    return PHG_GPU_OK;
}

// The arrays the mixed solver's FP32 layout `kind` needs for the current
// matrix (the reliable updates read the FP64 values of the same layout:
// SELL for kinds 0 and 1).
int ensure_layout32(phgGpuSystem *s, int kind) {
    if (kind == 2) return ensure_q16(s);
    CHECK_RC(ensure_sell(s));
    if (kind == 1) CHECK_RC(ensure_sell2(s));
    return PHG_GPU_OK;
}

const int kTune32Kind[kTune32] = {0, 0, 0, 1, 1, 1, 2, 2};
const int kTune32Unroll[kTune32] = {4, 8, 16, 2, 4, 8, 1, 2};

// Layout and unroll of the FP32 product (mixed solver), timed once per
// matrix shape: SELL unrolled 4/8/16, pair SELL unrolled 2/4/8, q16 unrolled
// 1/2 (when every row fits its two windows).  Later matrices of the shape
// build only the chosen layout; a q16 choice falls back to a new tuning when
// a matrix does not fit it.
int tune_spmv32(phgGpuSystem *s) {
    if (s->unroll32 != 0 && s->tuned32_n == s->n && s->tuned32_nnz == s->nnz) {
        CHECK_RC(ensure_layout32(s, s->kind32));
        if (s->kind32 != 2 || s->q16_fits) return PHG_GPU_OK;
    }
    CHECK_RC(ensure_sell(s));
    CHECK_RC(ensure_sell2(s));
    CHECK_RC(ensure_q16(s));
    CHECK_RC(s->r32.ensure((size_t)s->n));
    CHECK_RC(s->Ap32.ensure((size_t)s->n));
    CK(cudaMemsetAsync(s->r32.p, 0, sizeof(float) * s->n, s->stream));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    int best = -1;
    const int reps = 5;
    for (int c = 0; c < kTune32; c++) {
        s->tune32_ms[c] = 0.0;
        if (kTune32Kind[c] == 2 && !s->q16_fits) continue;
        for (int i = 0; i < 2; i++) CHECK_RC(launch_fp32_product(s, kTune32Kind[c], kTune32Unroll[c], s->r32.p, s->Ap32.p));
        CK(cudaEventRecord(a, s->stream));
        for (int i = 0; i < reps; i++)
            CHECK_RC(launch_fp32_product(s, kTune32Kind[c], kTune32Unroll[c], s->r32.p, s->Ap32.p));
        CK(cudaEventRecord(b, s->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        s->tune32_ms[c] = ms / reps;
        if (best < 0 || s->tune32_ms[c] < s->tune32_ms[best]) best = c;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->kind32 = kTune32Kind[best];
    s->unroll32 = kTune32Unroll[best];
    s->tuned32_n = s->n;
    s->tuned32_nnz = s->nnz;
    return PHG_GPU_OK;
}

// The layout arrays an FP64 plan's kernels read, for a graph's key: a graph
// is captured again when a reallocation moved any of them.
void plan_key(phgGpuSystem *s, phgGpuSystem_::GraphKey &key) {
    if (s->plan.kind == SPMV_CSR) {
        key.va = s->va.p;
        const void *e[8] = {s->rp.p, s->ci.p, nullptr, nullptr, nullptr, nullptr, nullptr, s->partials.p};
        memcpy(key.extra, e, sizeof(e));
    } else if (s->plan.kind == SPMV_SELL) {
        key.va = s->sell_vals.p;
        const void *e[8] = {s->sell_cols.p, s->sell_perm.p, s->sell_len.p, s->sell_sptr.p,
                            nullptr, nullptr, nullptr, s->partials.p};
        memcpy(key.extra, e, sizeof(e));
    } else {
        key.va = s->q16_v64.p;
        const void *e[8] = {s->q16_cols.p, s->q16_perm.p, s->q16_len.p, s->q16_split.p,
                            s->q16_b0.p, s->q16_b1.p, s->q16_sptr.p, s->partials.p};
        memcpy(key.extra, e, sizeof(e));
    }
}

SpmvPlan make_plan(phgGpuSystem *s, int kind, int param) {
    SpmvPlan P;
    P.kind = kind;
    P.lpr = kind == SPMV_CSR ? param : 8;
    P.unroll = kind == SPMV_CSR ? 4 : param;
    P.csr = CsrView{s->n, s->rp.p, s->ci.p, s->va.p};
    P.sell = SellView{s->n, sell_positions(s->n) / 32, s->sell_perm.p, s->sell_len.p, s->sell_sptr.p,
                      s->sell_cols.p, s->sell_vals.p, s->sell_vals32.p};
    P.q16 = q16_view(s);
    return P;
}

// Chooses the fastest SpMV layout for the current matrix shape by timing
// every candidate on the system's stream (once per (n, nnz)).  With
// build_layout false a plan chosen before is kept without building its
// layout for the current matrix (a caller that will not use the plan).
int tune_spmv(phgGpuSystem *s, bool build_layout = true) {
    if (s->tuned && s->tuned_n == s->n && s->tuned_nnz == s->nnz) {
        if (build_layout && s->plan.kind == SPMV_SELL) CHECK_RC(ensure_sell(s));
        // a q16 plan is checked against every new matrix (a matrix of the
        // same shape may not fit it); it is then timed again without q16
        bool keep = true;
        if (s->plan.kind == SPMV_Q16) {
            CHECK_RC(ensure_q16(s));
            keep = s->q16_fits;
        }
        if (keep) {
            s->plan = make_plan(s, s->plan.kind, s->plan.kind == SPMV_CSR ? s->plan.lpr : s->plan.unroll);
            return PHG_GPU_OK;
        }
    }
    CHECK_RC(ensure_sell(s));
    CHECK_RC(ensure_q16(s));
    CHECK_RC(solver_buffers(s));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    int best = 0;
    const int reps = 5;
    for (int c = 0; c < kTuneCandidates; c++) {
        s->tune_ms[c] = 0.0;
        if (kTuneKind[c] == SPMV_Q16 && !s->q16_fits) continue;
        const SpmvPlan P = make_plan(s, kTuneKind[c], kTuneParam[c]);
        for (int i = 0; i < 2; i++) CK(launch_spmv_plan(P, s->rhs.p, s->Ap.p, s->stream));
        CK(cudaEventRecord(a, s->stream));
        for (int i = 0; i < reps; i++) CK(launch_spmv_plan(P, s->rhs.p, s->Ap.p, s->stream));
        CK(cudaEventRecord(b, s->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        s->tune_ms[c] = ms / reps;
        s->launches += 2 + reps;
        if (s->tune_ms[c] < s->tune_ms[best]) best = c;   // candidate 0 (CSR) is always timed
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->plan = make_plan(s, kTuneKind[best], kTuneParam[best]);
    s->unroll32 = 0;
    s->tuned = true;
    s->tuned_n = s->n;
    s->tuned_nnz = s->nnz;
    return PHG_GPU_OK;
}

}  // namespace

extern "C" {

const char *phgGpuLastError(void) { return g_last_error.c_str(); }

const char *phgGpuLastWarning(void) { return g_last_warning.c_str(); }

int phgGpuVersion(void) { return 100; }

int phgGpuCreate(int device, void *stream, phgGpuSystem **out) {
    if (out == nullptr) return fail(PHG_GPU_ERR_ARG, "phgGpuCreate: null output");
    *out = nullptr;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(PHG_GPU_ERR_ARG, "phgGpuCreate: no CUDA device %d", device);
    phgGpuSystem *s = new phgGpuSystem();
    s->device = device;
    {
        const char *pg = getenv("PHG_GPU_PLAIN_GRAPHS");
        s->plain_graphs = pg != nullptr && pg[0] != '\0' && pg[0] != '0';
    }
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
        cudaError_t e2 = cudaMallocHost((void **)&s->h_sums, 4 * sizeof(double));
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
    if (s->graph_mixed != nullptr) cudaGraphExecDestroy(s->graph_mixed);
    if (s->h_gst_mixed) cudaFreeHost(s->h_gst_mixed);
    if (s->graph_bicg != nullptr) cudaGraphExecDestroy(s->graph_bicg);
    if (s->h_bst) cudaFreeHost(s->h_bst);
    if (s->graph_gmres != nullptr) cudaGraphExecDestroy(s->graph_gmres);
    if (s->h_gst) cudaFreeHost(s->h_gst);
    s->gm_vecs.release();
    s->gm_small.release();
    s->gm_st.release();
    s->bicg_vecs.release();
    s->bicg_st.release();
    DevBuf<float> *fbufs[] = {&s->r32, &s->p32, &s->Ap32, &s->y32, &s->D32, &s->sell_vals32, &s->sell2_vals};
    s->sell2_ssz.release(); s->sell2_sptr.release(); s->sell2_cols.release();
    s->sell2_order.release(); s->sell2_perm.release(); s->sell2_width.release(); s->sell2_len.release();
    for (auto *b : fbufs) b->release();
    s->sell_perm.release(); s->sell_ssz.release(); s->sell_sptr.release(); s->sell_cols.release();
    s->sell_len.release(); s->sell_vals.release(); s->gst.release(); s->u32.release(); s->s32.release();
    DevBuf<int32_t> *qi[] = {&s->q16_ssz, &s->q16_sptr, &s->q16_perm, &s->q16_b0, &s->q16_b1};
    for (auto *b : qi) b->release();
    DevBuf<uint16_t> *qu[] = {&s->q16_len, &s->q16_split, &s->q16_cols};
    for (auto *b : qu) b->release();
    s->q16_v32.release(); s->q16_v64.release(); s->q16_nofit.release();
    if (s->h_nofit) cudaFreeHost(s->h_nofit);
    s->adj_u.release(); s->adj_uobs.release(); s->adj_rhs.release(); s->adj_lambda.release(); s->adj_grad.release();
    if (s->graph_block != nullptr) cudaGraphExecDestroy(s->graph_block);
    DevBuf<double> *bb[] = {&s->bX, &s->bR, &s->bP, &s->bAP, &s->bB, &s->bscal, &s->bpart};
    for (auto *b : bb) b->release();
    DevBuf<float> *bf[] = {&s->bY32, &s->bR32, &s->bP32, &s->bAP32, &s->bva32};
    for (auto *b : bf) b->release();
    s->bint.release();
    s->btick.release();
    DevBuf<double> *dbufs[] = {&s->verts, &s->gk, &s->br, &s->brt, &s->Ke, &s->Re, &s->kappa, &s->f,
                               &s->g, &s->geo, &s->va, &s->bva, &s->rhs, &s->diag, &s->x, &s->r, &s->p, &s->Ap,
                               &s->partials, &s->hist, &s->sums};
    for (auto *b : dbufs) b->release();
    DevBuf<int32_t> *ibufs[] = {&s->elems, &s->e2l, &s->inc_ptr, &s->inc, &s->cnt, &s->cursor, &s->cnt_keep,
                                &s->cnt_bdry, &s->rp, &s->ci, &s->brp, &s->bci};
    for (auto *b : ibufs) b->release();
    s->bdry.release();
    s->sc_cols.release();
    s->sc_vals.release();
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
    s->pattern_state = 0;
    s->have_mesh = true;
    s->geometry_given = false;
    s->geometry_valid = false;
    s->have_dofs = false;
    s->assembled = false;
    return PHG_GPU_OK;
}

int phgGpuSetGeometry(phgGpuSystem *s, int64_t nelem, const double *geo) {
    if (s == nullptr || geo == nullptr) return fail(PHG_GPU_ERR_ARG, "phgGpuSetGeometry: invalid arguments");
    if (!s->have_mesh) return fail(PHG_GPU_ERR_STATE, "phgGpuSetGeometry: call phgGpuSetMesh first");
    if (nelem != s->nelem) return fail(PHG_GPU_ERR_ARG, "phgGpuSetGeometry: %lld elements, the mesh has %lld",
                                       (long long)nelem, (long long)s->nelem);
    for (size_t i = 0; i < 17 * (size_t)nelem; i++)
        if (!isfinite(geo[i])) return fail(PHG_GPU_ERR_ARG, "phgGpuSetGeometry: element %lld not finite",
                                           (long long)(i / 17));
    CHECK_RC(set_device(s));
    CHECK_RC(s->geo.ensure((size_t)geometry_doubles(nelem)));
    // 17 doubles per element on the host into the kernels' padded stride
    CK(cudaMemcpy2DAsync(s->geo.p, (size_t)geometry_stride() * sizeof(double), geo, 17 * sizeof(double),
                         17 * sizeof(double), (size_t)nelem, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->geometry_given = true;
    s->pattern_state = 0;
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
    s->pattern_state = 0;
    CHECK_RC(check_status(s, "phgGpuSetDofMap"));
    s->have_dofs = true;
    s->assembled = false;
    return PHG_GPU_OK;
}

// Element matrices, right-hand sides and nonzero masks of every element
// (the element loop's phgQuad* calls) into s->Ke, s->Re.
static int element_pass(phgGpuSystem *s, const double *kappa, double mass, const double *f) {
    const int N = s->N;
    const int64_t ndof = s->ndof;
    const double *dk, *df;
    CHECK_RC(stage(s, kappa, (size_t)s->nelem, s->kappa, &dk));
    CHECK_RC(stage(s, f, (size_t)ndof, s->f, &df));
    CHECK_RC(s->Ke.ensure((size_t)s->nelem * N * N));
    CHECK_RC(s->Re.ensure((size_t)s->nelem * N));
    CHECK_RC(s->geo.ensure((size_t)geometry_doubles(s->nelem)));
    ElemArgs ea{};
    ea.nelem = s->nelem; ea.nvert = s->nvert; ea.ndof = ndof;
    ea.verts = s->verts.p; ea.elems = s->elems.p; ea.e2l = s->e2l.p;
    ea.kappa = dk; ea.f = df; ea.mass = mass;
    ea.gk = s->gk.p; ea.br = s->br.p; ea.brt = s->brt.p; ea.wk_host = s->wk.data(); ea.wr_host = s->wr.data();
    ea.Ke = s->Ke.p; ea.Re = s->Re.p; ea.geo = s->geo.p; ea.status = s->status.p;
    // the geometry is computed once per mesh (a build that succeeded has
    // checked its vertex indices and coordinates)
    ea.geometry_given = s->geometry_given || s->geometry_valid;
    CK(launch_element_kernel(s->order, ea, s->stream));
    s->launches += ea.geometry_given ? 1 : 2;
    return PHG_GPU_OK;
}

static int build_system(phgGpuSystem *s, const double *kappa, double mass, const double *f, const double *g) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->have_dofs) return fail(PHG_GPU_ERR_STATE, "phgGpuBuildLinearSystem: call phgGpuSetDofMap first");
    if (!isfinite(mass)) return fail(PHG_GPU_ERR_ARG, "phgGpuBuildLinearSystemMass: mass coefficient not finite");
    CHECK_RC(set_device(s));
    const int64_t ndof = s->ndof;
    const double *dg;
    CHECK_RC(stage(s, g, (size_t)ndof, s->g, &dg));
    CHECK_RC(element_pass(s, kappa, mass, f));

    CHECK_RC(s->cnt_keep.ensure((size_t)ndof));
    CHECK_RC(s->cnt_bdry.ensure((size_t)ndof));
    CHECK_RC(s->rp.ensure((size_t)ndof + 1));
    CHECK_RC(s->brp.ensure((size_t)ndof + 1));
    CHECK_RC(s->rhs.ensure((size_t)ndof));
    CHECK_RC(s->diag.ensure((size_t)ndof));
    const size_t nscratch = (size_t)s->nelem * s->N * s->N;   // every row fits in its incidences x N slots
    CHECK_RC(s->sc_cols.ensure(nscratch));
    CHECK_RC(s->sc_vals.ensure(nscratch));
    WalkArgs wa{};
    wa.ndof = ndof; wa.inc_ptr = s->inc_ptr.p; wa.inc = s->inc.p; wa.e2l = s->e2l.p; wa.bdry = s->bdry.p;
    wa.Ke = s->Ke.p; wa.Re = s->Re.p; wa.g = dg;
    wa.cnt_keep = s->cnt_keep.p; wa.cnt_bdry = s->cnt_bdry.p; wa.status = s->status.p;
    wa.sc_cols = s->sc_cols.p; wa.sc_vals = s->sc_vals.p;
    wa.rhs = s->rhs.p; wa.diag = s->diag.p;
    CHECK_RC(s->over_list.ensure((size_t)ndof));
    CHECK_RC(s->nover.ensure(1));
    wa.over_list = s->over_list.p; wa.nover = s->nover.p;
    if (s->pattern_state == 2 && s->assembled && s->have_bdry_cols) {
        // the recorded pattern: values only, written in place
        wa.slot = s->slot.p; wa.tmap = s->tmap.p; wa.dpos = s->dpos.p;
        wa.ptr = s->rp.p; wa.cols = s->ci.p; wa.vals = s->va.p;
        wa.bptr = s->brp.p; wa.bcols = s->bci.p; wa.bvals = s->bva.p;
        CK(launch_value_walk(s->order, wa, s->stream));
        s->launches += 2;
        CK(cudaMemcpyAsync(s->h_status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        if (*s->h_status == PHGB_DEV_PATTERN_CHANGED) {   // an exact zero appeared or went: walk again
            *s->h_status = 0;
            CK(cudaMemsetAsync(s->status.p, 0, sizeof(int), s->stream));
            s->pattern_state = 1;
        } else {
            CHECK_RC(check_status(s, "phgGpuBuildLinearSystem"));
            s->geometry_valid = true;
            CHECK_RC(refresh_layout_values(s));
            s->mass = mass;
            return PHG_GPU_OK;
        }
    }
    // the second build on this mesh and DOF map records the pattern
    const bool record = s->pattern_state == 1;
    if (record) {
        CHECK_RC(s->slot.ensure(nscratch));
        CHECK_RC(s->tmap.ensure(nscratch));
        CHECK_RC(s->dpos.ensure((size_t)ndof));
        CK(cudaMemsetAsync(s->dpos.p, 0xff, sizeof(int32_t) * (size_t)ndof, s->stream));   // -1: no diagonal
        wa.slot = s->slot.p;
        wa.tmap = s->tmap.p;
        wa.dpos = s->dpos.p;
    } else {
        wa.slot = nullptr;
        wa.tmap = nullptr;
        wa.dpos = nullptr;
    }
    CK(launch_row_walk(s->order, wa, s->stream));
    s->launches += 8;   // walk (two passes) + two scans
    CK(launch_scan(ndof, s->cnt_keep.p, s->rp.p, s->scan_ws.p, s->stream));
    int32_t tot[2];
    CK(cudaMemcpyAsync(&tot[0], s->rp.p + ndof, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(launch_scan(ndof, s->cnt_bdry.p, s->brp.p, s->scan_ws.p, s->stream));
    CK(cudaMemcpyAsync(&tot[1], s->brp.p + ndof, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CHECK_RC(check_status(s, "phgGpuBuildLinearSystem (rows)"));
    s->geometry_valid = true;
    if (tot[0] < 0 || tot[1] < 0) return fail(PHG_GPU_ERR_LIMIT, "matrix has more than 2^31 entries");
    s->nnz = tot[0];
    s->bnnz = tot[1];
    CHECK_RC(s->ci.ensure((size_t)s->nnz));
    CHECK_RC(s->va.ensure((size_t)s->nnz));
    CHECK_RC(s->bci.ensure((size_t)s->bnnz));
    CHECK_RC(s->bva.ensure((size_t)s->bnnz));
    wa.ptr = s->rp.p; wa.cols = s->ci.p; wa.vals = s->va.p;
    wa.bptr = s->brp.p; wa.bcols = s->bci.p; wa.bvals = s->bva.p;
    CK(launch_compact(s->N, wa, s->stream));   // sets no status: the check above covers the build
    s->launches += 1;

    s->n = ndof;
    s->assembled = true;
    s->have_bdry_cols = true;
    invalidate_layouts(s);
    s->lpr = spmv_lanes_for((double)s->nnz / (double)ndof);
    s->mass = mass;
    s->pattern_state = record ? 2 : 1;
    return PHG_GPU_OK;
}

int phgGpuBuildLinearSystem(phgGpuSystem *s, const double *kappa, const double *f, const double *g) {
    return build_system(s, kappa, 0.0, f, g);
}

int phgGpuElementMatrices(phgGpuSystem *s, const double *kappa, double mass_coef, const double *f, double *Ke,
                          double *Re) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->have_dofs) return fail(PHG_GPU_ERR_STATE, "phgGpuElementMatrices: call phgGpuSetDofMap first");
    if (!isfinite(mass_coef)) return fail(PHG_GPU_ERR_ARG, "phgGpuElementMatrices: mass coefficient not finite");
    CHECK_RC(set_device(s));
    CHECK_RC(element_pass(s, kappa, mass_coef, f));
    CHECK_RC(check_status(s, "phgGpuElementMatrices"));
    s->geometry_valid = true;
    const size_t N = (size_t)s->N;
    if (Ke != nullptr) CHECK_RC(copy_out(s, Ke, s->Ke.p, (size_t)s->nelem * N * N));
    if (Re != nullptr) CHECK_RC(copy_out(s, Re, s->Re.p, (size_t)s->nelem * N));
    CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuBuildLinearSystemMass(phgGpuSystem *s, const double *kappa, double mass_coef, const double *f,
                                const double *g) {
    return build_system(s, kappa, mass_coef, f, g);
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
    s->pattern_state = 0;
    s->assembled = true;
    s->have_bdry_cols = false;
    invalidate_layouts(s);
    s->lpr = spmv_lanes_for((double)nnz / (double)n);
    return PHG_GPU_OK;
}

int phgGpuSetRHS(phgGpuSystem *s, const double *rhs) {
    if (s == nullptr || rhs == nullptr) return fail(PHG_GPU_ERR_ARG, "phgGpuSetRHS: invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "phgGpuSetRHS: no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(copy_in(s, s->rhs.p, rhs, (size_t)s->n));
    nonfinite_kernel<<<vec_blocks(s->n), 256, 0, s->stream>>>(s->n, s->rhs.p, s->status.p);
    CK(cudaGetLastError());
    s->launches += 1;
    return check_status(s, "phgGpuSetRHS");
}

int phgGpuAssembleRows(phgGpuSystem *s, int64_t n, int64_t nrec, const int32_t *rec_row, const int64_t *rec_ptr,
                       const int32_t *rec_cols, const double *rec_vals) {
    if (s == nullptr || n <= 0 || nrec < 0 || (nrec > 0 && (rec_row == nullptr || rec_ptr == nullptr)))
        return fail(PHG_GPU_ERR_ARG, "phgGpuAssembleRows: invalid arguments");
    if (n >= INT32_MAX || nrec >= INT32_MAX) return fail(PHG_GPU_ERR_LIMIT, "phgGpuAssembleRows: too many rows");
    CHECK_RC(set_device(s));
    int64_t nent = 0;
    if (nrec > 0) {
        int64_t first = 0;
        CK(cudaMemcpy(&nent, rec_ptr + nrec, sizeof(int64_t), cudaMemcpyDefault));
        CK(cudaMemcpy(&first, rec_ptr, sizeof(int64_t), cudaMemcpyDefault));
        if (first != 0 || nent < 0) return fail(PHG_GPU_ERR_ARG, "phgGpuAssembleRows: bad segment offsets");
        if (nent >= INT32_MAX) return fail(PHG_GPU_ERR_LIMIT, "phgGpuAssembleRows: more than 2^31 entries");
        if (nent > 0 && (rec_cols == nullptr || rec_vals == nullptr))
            return fail(PHG_GPU_ERR_ARG, "phgGpuAssembleRows: invalid arguments");
    }
    const size_t un = (size_t)n;
    const int32_t *drow = nullptr, *dcols = nullptr;
    const int64_t *dptr = nullptr;
    const double *dvals = nullptr;
    CHECK_RC(stage(s, rec_row, (size_t)nrec, s->rec_row, &drow));
    CHECK_RC(stage(s, rec_ptr, (size_t)nrec + 1, s->rec_ptr, &dptr));
    CHECK_RC(stage(s, rec_cols, (size_t)nent, s->rec_cols, &dcols));
    CHECK_RC(stage(s, rec_vals, (size_t)nent, s->rec_vals, &dvals));
    CHECK_RC(s->rec_inc_ptr.ensure(un + 1));
    CHECK_RC(s->rec_inc.ensure((size_t)nrec));
    CHECK_RC(s->rec_cnt.ensure(un));
    CHECK_RC(s->rec_cursor.ensure(un));
    CHECK_RC(s->rec_cap.ensure(un));
    CHECK_RC(s->rec_cap_ptr.ensure(un + 1));
    CHECK_RC(s->scan_ws.ensure((size_t)scan_workspace_elems(n)));
    CHECK_RC(s->sc_cols.ensure((size_t)nent));
    CHECK_RC(s->sc_vals.ensure((size_t)nent));
    CHECK_RC(s->over_list.ensure(un));
    CHECK_RC(s->nover.ensure(1));
    CHECK_RC(s->rp.ensure(un + 1));
    CHECK_RC(s->rhs.ensure(un));
    CHECK_RC(s->diag.ensure(un));
    // each row's segments in call order (the incidence lists with one
    // "basis" per segment), and each row's capacity (its segments' total)
    CK(launch_incidence(1, nrec, n, drow, s->rec_cnt.p, s->rec_inc_ptr.p, s->rec_cursor.p, s->rec_inc.p,
                        s->scan_ws.p, s->status.p, s->stream));
    CK(cudaMemsetAsync(s->rec_cap.p, 0, sizeof(int32_t) * un, s->stream));
    if (nrec > 0) CK(launch_record_lengths(nrec, drow, dptr, s->rec_cap.p, s->stream));
    CK(launch_scan(n, s->rec_cap.p, s->rec_cap_ptr.p, s->scan_ws.p, s->stream));
    CHECK_RC(check_status(s, "phgGpuAssembleRows (segments)"));
    RecordArgs ra{};
    ra.n = n; ra.rinc_ptr = s->rec_inc_ptr.p; ra.rinc = s->rec_inc.p; ra.rec_ptr = dptr; ra.rec_cols = dcols;
    ra.rec_vals = dvals; ra.cap_ptr = s->rec_cap_ptr.p; ra.cnt = s->rec_cnt.p; ra.sc_cols = s->sc_cols.p;
    ra.sc_vals = s->sc_vals.p; ra.status = s->status.p; ra.over_list = s->over_list.p; ra.nover = s->nover.p;
    CK(launch_record_walk(ra, s->stream));
    CK(launch_scan(n, s->rec_cnt.p, s->rp.p, s->scan_ws.p, s->stream));
    int32_t tot = 0;
    CK(cudaMemcpyAsync(&tot, s->rp.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(s->h_status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->launches += 12;
    const int st = *s->h_status;
    if (st != PHGB_DEV_OK) {
        *s->h_status = 0;
        CK(cudaMemsetAsync(s->status.p, 0, sizeof(int), s->stream));
        s->assembled = false;
        if (st == PHGB_DEV_DUPLICATE)
            return fail(PHG_GPU_ERR_ARG, "phgGpuAssembleRows: a row's first segment names a column twice");
        if (st == PHGB_DEV_ROW_OVERFLOW)
            return fail(PHG_GPU_ERR_LIMIT, "phgGpuAssembleRows: a row has more than %d entries", kRecordMaxRow);
        return fail(PHG_GPU_ERR_STATE, "phgGpuAssembleRows: internal consistency check failed (%d)", st);
    }
    s->nnz = tot;
    s->bnnz = 0;
    CHECK_RC(s->ci.ensure((size_t)s->nnz));
    CHECK_RC(s->va.ensure((size_t)s->nnz));
    CK(launch_record_compact(ra, s->rp.p, s->ci.p, s->va.p, s->stream));
    CK(cudaMemsetAsync(s->rhs.p, 0, sizeof(double) * un, s->stream));
    diag_kernel<<<vec_blocks(n), 256, 0, s->stream>>>(n, s->rp.p, s->ci.p, s->va.p, s->diag.p);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    s->launches += 2;
    s->n = n;
    s->pattern_state = 0;
    s->assembled = true;
    s->have_bdry_cols = false;
    invalidate_layouts(s);
    s->lpr = spmv_lanes_for((double)s->nnz / (double)n);
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
    CHECK_RC(tune_spmv(s));
    CK(launch_spmv_plan(s->plan, dx, dy, s->stream));
    s->launches += 1;
    if (!ydev) CHECK_RC(copy_out(s, y, dy, (size_t)s->n));
    // device-to-device calls stay asynchronous on the system's stream
    if (!(xdev && ydev)) CK(cudaStreamSynchronize(s->stream));
    return PHG_GPU_OK;
}

int phgGpuSolverPCGMixed(phgGpuSystem *s, double rtol, double btol, double atol, int maxit, double *x,
                         double *residual, int *nupdates) {
    g_last_warning.clear();
    if (s == nullptr || x == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    if (maxit < 0) return fail(PHG_GPU_ERR_ARG, "maxit < 0");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    CHECK_RC(tune_spmv(s, false));
    const int64_t n = s->n;
    const size_t un = (size_t)n;
    CHECK_RC(s->r32.ensure(un));
    CHECK_RC(s->p32.ensure(un));
    CHECK_RC(s->Ap32.ensure(un));
    CHECK_RC(s->y32.ensure(un));
    CHECK_RC(s->D32.ensure(un));
    CHECK_RC(s->u32.ensure(un));
    CHECK_RC(s->s32.ensure(un));
    CHECK_RC(s->gst.ensure(1));
    if (s->h_gst_mixed == nullptr) CK(cudaMallocHost((void **)&s->h_gst_mixed, sizeof(GearState)));
    CHECK_RC(copy_in(s, s->x.p, x, un));
    CK(cudaMemsetAsync(s->ticket.p, 0, sizeof(unsigned) * kRedTickets, s->stream));
    CHECK_RC(tune_spmv32(s));   // builds the chosen FP32 layout for this matrix
    if (s->plan.kind == SPMV_Q16) CHECK_RC(ensure_q16(s));   // the FP64 plan's layout (checked by tune_spmv)
    const bool q16 = s->kind32 == 2;
    // FP64 products (residuals): the q16 layout's FP64 values, or the FP64
    // plan (whose SELL arrays the kinds 0 and 1 have built)
    const SpmvPlan P = make_plan(s, s->plan.kind, s->plan.kind == SPMV_CSR ? s->plan.lpr : s->plan.unroll);
    const Q16View Q = q16_view(s);
    auto product64 = [&](const double *xin, double *yout) -> cudaError_t {
        return q16 ? launch_q16_spmv64(Q, xin, yout, s->stream) : launch_spmv_plan(P, xin, yout, s->stream);
    };

    CK(launch_init_sums(n, 0, s->x.p, s->rhs.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->launches += 1;
    const double x1 = s->h_sums[0], rb = sqrt(s->h_sums[1]);
    auto is_zero = [](double a) { return fabs(a) < 10.0 * DBL_MIN; };
    if (is_zero(rb)) {
        CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
        CHECK_RC(copy_out(s, x, s->x.p, un));
        CK(cudaStreamSynchronize(s->stream));
        if (residual) *residual = 0.0;
        if (nupdates) *nupdates = 0;
        return 0;
    }
    bool x_nonzero = !is_zero(x1 / (double)n);
    double tol = -1.0;
    int nits_total = 0, nupd = 0;
    double res_true = 0.0;
    const GearBuffers B{n, s->x.p, s->r.p, s->rhs.p, s->r32.p, s->u32.p, s->Ap32.p, s->p32.p, s->s32.p, s->y32.p, s->D32.p,
                        s->partials.p, s->gst.p};
    const GearLayouts L{s->kind32, s->unroll32, sell_view(s), sell2_view(s), Q};
    // the solve's graph, captured again when a buffer or the layout changed
    phgGpuSystem_::GraphKey key{};
    key.x = s->x.p; key.r = s->r32.p; key.p = s->p32.p; key.Ap = s->Ap32.p; key.D = s->D32.p;
    key.n = n; key.lpr = s->unroll32 + 100 * s->kind32;
    key.s = s->stream;
    if (q16) {
        key.va = Q.vals32; key.hist = Q.vals64;
        const void *e[8] = {Q.cols, Q.perm, Q.len, Q.split, Q.base0, Q.base1, Q.sptr, s->partials.p};
        memcpy(key.extra, e, sizeof(e));
    } else {
        key.va = s->sell2_vals.p; key.hist = s->sell_cols.p;
        const void *e[8] = {s->sell2_cols.p, s->sell2_perm.p, s->u32.p, s->sell2_sptr.p,
                            s->sell_vals.p, s->sell_vals32.p, s->s32.p, s->partials.p};
        memcpy(key.extra, e, sizeof(e));
    }
    if (s->graph_mixed == nullptr || !(s->gkey_mixed == key)) {
        if (s->graph_mixed != nullptr) { cudaGraphExecDestroy(s->graph_mixed); s->graph_mixed = nullptr; }
        CK(build_gear_graph(B, L, kGraphChunk, s->plain_graphs, s->stream, &s->graph_mixed, nullptr));
        s->gkey_mixed = key;
    }
    // the explicit FP64 residual b - A x is checked at the end; a recurrence
    // that drifted above the tolerance restarts from it (at most twice)
    for (int restart = 0; restart < 3; restart++) {
        if (x_nonzero) {
            CK(product64(s->x.p, s->Ap.p));
            CK(launch_residual(n, s->rhs.p, s->Ap.p, s->r.p, s->stream));
            s->launches += 2;
        } else {
            CK(cudaMemcpyAsync(s->r.p, s->rhs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
        }
        CK(launch_gear_init(B, s->diag.p, s->ticket.p, s->sums.p, s->stream));
        s->launches += 1;
        CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        const double r0 = sqrt(s->h_sums[0]), ru0 = s->h_sums[1];
        if (!isfinite(ru0)) return fail(PHG_GPU_ERR_NAN, "phgGpuSolverPCGMixed: zero or non-finite diagonal");
        if (tol < 0.0) {   // get_tol (solver-phg.c:104-115) on the initial residual
            tol = r0 * rtol;
            if (tol < rb * btol) tol = rb * btol;
            if (tol < atol) tol = atol;
        }
        GearState g{};
        g.tol = tol;
        g.maxit = maxit - nits_total;
        g.maxr = r0;
        g.delta = 0.1;
        g.residual = r0;
        g.gamma_cur = ru0;
        g.rr_cur = s->h_sums[2];
        g.first = 1;
        g.y_reset = 1;
        g.done = !(r0 > tol && nits_total < maxit);
        g.max_passes = g.maxit / kGraphChunk + 3;
        *s->h_gst_mixed = g;
        CK(cudaMemcpyAsync(s->gst.p, s->h_gst_mixed, sizeof(GearState), cudaMemcpyHostToDevice, s->stream));
        int plain_passes = 0;
        bool plain_limit = false;
        if (!g.done && !s->plain_graphs) CK(cudaGraphLaunch(s->graph_mixed, s->stream));
        if (!g.done && s->plain_graphs) {
            for (;;) {
                if (plain_passes >= g.max_passes) { plain_limit = true; break; }
                CK(cudaGraphLaunch(s->graph_mixed, s->stream));
                plain_passes++;
                CK(cudaMemcpyAsync(s->h_gst_mixed, s->gst.p, sizeof(GearState), cudaMemcpyDeviceToHost, s->stream));
                CK(cudaStreamSynchronize(s->stream));
                if (s->h_gst_mixed->done) break;
            }
        }
        CK(cudaMemcpyAsync(s->h_gst_mixed, s->gst.p, sizeof(GearState), cudaMemcpyDeviceToHost, s->stream));
        CK(launch_gear_fold(B, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        GearState &hg = *s->h_gst_mixed;
        if (plain_limit) hg.status = GEAR_PASS_LIMIT;
        if (s->plain_graphs) s->launches += 4 * (int64_t)kGraphChunk * plain_passes + 1;
        else s->launches += 2 * (int64_t)hg.nits + 2 * (int64_t)hg.nupdates + hg.passes + 1;
        nits_total += hg.nits;
        nupd += hg.nupdates;
        if (hg.status == PCG_NONFINITE) return fail(PHG_GPU_ERR_NAN, "mixed PCG: non-finite residual");
        if (hg.status == GEAR_PASS_LIMIT)
            return fail(PHG_GPU_ERR_STATE, "mixed PCG: the iteration loop exceeded its pass bound");
        // explicit FP64 residual of the accumulated solution
        CK(product64(s->x.p, s->Ap.p));
        CK(launch_residual(n, s->rhs.p, s->Ap.p, s->r.p, s->stream));
        CK(launch_init_sums(n, 1, s->x.p, s->r.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
        s->launches += 3;
        CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        res_true = sqrt(s->h_sums[0]);
        if (hg.status == PCG_BREAKDOWN) {
            // as the FP64 PCG: warn, keep the iterate, report its FP64 residual
            warn("mixed PCG stopped after %d iterations: the matrix may not be SPD", nits_total);
            break;
        }
        if (!(res_true > tol) || nits_total >= maxit) break;
        x_nonzero = true;
    }
    CHECK_RC(copy_out(s, x, s->x.p, un));
    CK(cudaStreamSynchronize(s->stream));
    if (residual) *residual = res_true;
    if (nupdates) *nupdates = nupd;
    return nits_total;
}

int phgGpuTimeSpMV(phgGpuSystem *s, int fp32, int reps, double *ms_per_launch) {
    if (s == nullptr || ms_per_launch == nullptr || reps <= 0) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    CHECK_RC(tune_spmv(s));
    SpmvPlan P = make_plan(s, s->plan.kind, s->plan.kind == SPMV_CSR ? s->plan.lpr : s->plan.unroll);
    if (fp32) {
        CHECK_RC(tune_spmv32(s));
        CHECK_RC(s->r32.ensure((size_t)s->n));
        CHECK_RC(s->Ap32.ensure((size_t)s->n));
        CK(cudaMemsetAsync(s->r32.p, 0, sizeof(float) * s->n, s->stream));
    }
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int i = 0; i < reps + 3; i++) {
        if (i == 3) CK(cudaEventRecord(a, s->stream));
        if (fp32) {
            CHECK_RC(launch_fp32_product(s, s->kind32, s->unroll32, s->r32.p, s->Ap32.p));
        } else {
            CK(launch_spmv_plan(P, s->rhs.p, s->Ap.p, s->stream));
            s->launches += 1;
        }
    }
    CK(cudaEventRecord(b, s->stream));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_per_launch = ms / reps;
    return PHG_GPU_OK;
}

int phgGpuSetSpMVPlan(phgGpuSystem *s, int kind, int param) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    int c = 0;
    while (c < kTuneCandidates && !(kTuneKind[c] == kind && kTuneParam[c] == param)) c++;
    if (c == kTuneCandidates) return fail(PHG_GPU_ERR_ARG, "no SpMV layout (%d, %d)", kind, param);
    CHECK_RC(set_device(s));
    if (kind == SPMV_SELL) CHECK_RC(ensure_sell(s));
    if (kind == SPMV_Q16) {
        CHECK_RC(ensure_q16(s));
        if (!s->q16_fits)
            return fail(PHG_GPU_ERR_ARG, "the q16 layout does not fit this matrix: a row spans more than two "
                        "65536-column windows");
    }
    s->plan = make_plan(s, kind, param);
    s->tuned = true;
    s->tuned_n = s->n;
    s->tuned_nnz = s->nnz;
    return PHG_GPU_OK;
}

int phgGpuSetSpMVPlan32(phgGpuSystem *s, int layout, int unroll) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    bool ok = false;
    for (int c = 0; c < kTune32; c++) ok = ok || (kTune32Kind[c] == layout && kTune32Unroll[c] == unroll);
    if (!ok) return fail(PHG_GPU_ERR_ARG, "no FP32 SpMV layout (%d, %d)", layout, unroll);
    CHECK_RC(set_device(s));
    CHECK_RC(tune_spmv(s));   // FP64 layout for this matrix (returns at once if chosen)
    CHECK_RC(ensure_layout32(s, layout));
    if (layout == 2 && !s->q16_fits)
        return fail(PHG_GPU_ERR_ARG, "the q16 layout does not fit this matrix: a row spans more than two "
                    "65536-column windows");
    s->kind32 = layout;
    s->unroll32 = unroll;
    s->tuned32_n = s->n;
    s->tuned32_nnz = s->nnz;
    return PHG_GPU_OK;
}

int phgGpuGetSpMVPlan(phgGpuSystem *s, int *kind, int *param, double *times_ms) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (!s->tuned) return fail(PHG_GPU_ERR_STATE, "the SpMV layout is chosen at the first solve or product");
    if (kind) *kind = s->plan.kind;
    if (param) *param = s->plan.kind == SPMV_CSR ? s->plan.lpr : s->plan.unroll;
    if (times_ms) {
        for (int c = 0; c < kTuneCandidates; c++) times_ms[c] = s->tune_ms[c];
        for (int c = 0; c < kTune32; c++) times_ms[kTuneCandidates + c] = s->tune32_ms[c];
        times_ms[kTuneCandidates + kTune32] = s->unroll32;
        times_ms[kTuneCandidates + kTune32 + 1] = s->kind32;
    }
    return kTuneCandidates;
}

int phgGpuSpMVBytes(phgGpuSystem *s, int fp32, int64_t *bytes) {
    if (s == nullptr || bytes == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    CHECK_RC(set_device(s));
    CHECK_RC(tune_spmv(s));
    const int64_t n = s->n, npos = sell_positions(n), nsl = npos / 32;
    const int64_t vec = (fp32 ? 8 : 16) * n, sl = 4 * (nsl + 1);   // x read once + y written; slice offsets
    if (fp32) {
        CHECK_RC(tune_spmv32(s));
        if (s->kind32 == 2) *bytes = 6 * s->q16_total + 16 * npos + sl + vec;
        else if (s->kind32 == 1) *bytes = 8 * s->sell2_total + 6 * npos + sl + vec;
        else *bytes = 8 * s->sell_total + 6 * npos + sl + vec;
    } else if (s->plan.kind == SPMV_SELL) {
        *bytes = 12 * s->sell_total + 6 * npos + sl + vec;
    } else if (s->plan.kind == SPMV_Q16) {
        *bytes = 10 * s->q16_total + 16 * npos + sl + vec;
    } else {
        *bytes = 12 * s->nnz + 4 * (n + 1) + vec;
    }
    return PHG_GPU_OK;
}

int phgGpuGetLaunchCount(phgGpuSystem *s, int64_t *count) {
    if (s == nullptr || count == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    *count = s->launches;
    return PHG_GPU_OK;
}

}  // extern "C"

namespace {

// FP64 Jacobi-PCG on the assembled matrix with right-hand side `drhs`
// (device), iterating on s->x (initial guess in, solution out).  Returns the
// iteration count or a negative error code.
int pcg_core(phgGpuSystem *s, const double *drhs, double rtol, double btol, double atol, int maxit,
             double *dhist, double *residual) {
    const int64_t n = s->n;
    CK(cudaMemsetAsync(s->ticket.p, 0, sizeof(unsigned) * kRedTickets, s->stream));
    // ||b|| and |x|_1 (solver-phg.c:498-518)
    CK(launch_init_sums(n, 0, s->x.p, drhs, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double x1 = s->h_sums[0], rb = sqrt(s->h_sums[1]);
    auto is_zero = [](double a) { return fabs(a) < 10.0 * DBL_MIN; };   // utils.h:451
    if (is_zero(rb)) {
        CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
        if (residual) *residual = 0.0;
        if (dhist) CK(cudaMemsetAsync(dhist, 0, sizeof(double), s->stream));
        return 0;
    }
    CsrView A{n, s->rp.p, s->ci.p, s->va.p};
    CHECK_RC(tune_spmv(s));
    if (!is_zero(x1 / (double)n)) {
        CK(launch_spmv_plan(s->plan, s->x.p, s->Ap.p, s->stream));
        CK(launch_residual(n, drhs, s->Ap.p, s->r.p, s->stream));
        s->launches += 2;
    } else {
        CK(cudaMemcpyAsync(s->r.p, drhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
    }
    CK(launch_init_sums(n, 1, s->x.p, s->r.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double r0 = sqrt(s->h_sums[0]), rz0 = s->h_sums[1];
    if (!isfinite(rz0)) return fail(PHG_GPU_ERR_NAN, "PCG: zero or non-finite diagonal");
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
    init.max_passes = maxit / kGraphChunk + 3;
    *s->h_st = init;
    CK(cudaMemcpyAsync(s->st.p, s->h_st, sizeof(PcgState), cudaMemcpyHostToDevice, s->stream));
    if (dhist) CK(cudaMemcpyAsync(dhist, &s->h_st->residual, sizeof(double), cudaMemcpyHostToDevice, s->stream));

    PcgBuffers B{A, s->x.p, s->r.p, s->p.p, s->Ap.p, s->diag.p, s->partials.p, s->st.p, dhist};
    phgGpuSystem_::GraphKey key{};
    key.x = B.x; key.r = B.r; key.p = B.p; key.Ap = B.Ap; key.D = B.D; key.hist = dhist;
    key.n = n; key.lpr = s->plan.kind * 100 + s->plan.lpr * 10 + s->plan.unroll; key.s = s->stream;
    plan_key(s, key);
    if (s->graph == nullptr || !(s->gkey == key)) {
        if (s->graph != nullptr) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
        // one graph launch per solve: chunks of iterations in a WHILE loop
        struct Ctx { PcgBuffers B; SpmvPlan P; } ctx{B, s->plan};
        auto body = [](void *c, cudaStream_t st) {
            const Ctx *x = (const Ctx *)c;
            for (int i = 0; i < kGraphChunk; i++) launch_pcg_iteration_plan(x->B, x->P, st);
        };
        CK(build_pcg_loop_graph(s->stream, body, &ctx, s->st.p, s->plain_graphs, &s->graph));
        s->gkey = key;
    }
    if (!init.done && !s->plain_graphs) CK(cudaGraphLaunch(s->graph, s->stream));
    int plain_passes = 0;
    bool plain_limit = false;
    if (!init.done && s->plain_graphs) {
        for (;;) {
            if (plain_passes >= init.max_passes) { plain_limit = true; break; }
            CK(cudaGraphLaunch(s->graph, s->stream));
            plain_passes++;
            CK(cudaMemcpyAsync(s->h_st, s->st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s->stream));
            CK(cudaStreamSynchronize(s->stream));
            if (s->h_st->done) break;
        }
    }
    CK(cudaMemcpyAsync(s->h_st, s->st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (plain_limit) s->h_st->status = kStatusPassLimit;
    if (s->plain_graphs) s->launches += 3 * (int64_t)kGraphChunk * plain_passes;
    else s->launches += 3 * (int64_t)kGraphChunk * s->h_st->passes + s->h_st->passes;
    const int nits = s->h_st->nits;
    if (residual) *residual = s->h_st->residual;
    if (s->h_st->status == kStatusPassLimit)
        return fail(PHG_GPU_ERR_STATE, "PCG: the iteration loop exceeded its pass bound");
    if (s->h_st->status == PCG_BREAKDOWN)
        warn("PCG stopped after %d iterations: the matrix may not be SPD", nits);
    if (s->h_st->status == PCG_NONFINITE)
        return fail(PHG_GPU_ERR_NAN, "PCG: non-finite residual after %d iterations", nits);
    return nits;
}

// BiCGstab with the Jacobi preconditioner (solver_BiCGstab,
// solver-phg.c:606-781) from the initial guess in s->x.
int bicg_core(phgGpuSystem *s, double rtol, double btol, double atol, int maxit, double *dhist,
              double *residual) {
    const int64_t n = s->n;
    const double *drhs = s->rhs.p;
    CK(cudaMemsetAsync(s->ticket.p, 0, sizeof(unsigned) * kRedTickets, s->stream));
    CK(launch_init_sums(n, 0, s->x.p, drhs, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double x1 = s->h_sums[0], rb = sqrt(s->h_sums[1]);
    auto is_zero = [](double a) { return fabs(a) < 10.0 * DBL_MIN; };   // utils.h:451
    if (is_zero(rb)) {   // solver-phg.c:630-633
        CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
        if (residual) *residual = 0.0;
        if (dhist) CK(cudaMemsetAsync(dhist, 0, sizeof(double), s->stream));
        return 0;
    }
    CHECK_RC(tune_spmv(s));
    const int64_t stride = bicg_stride(n);
    CHECK_RC(s->bicg_vecs.ensure((size_t)stride * kBicgVectors));
    CHECK_RC(s->bicg_st.ensure(1));
    if (s->h_bst == nullptr) CK(cudaMallocHost((void **)&s->h_bst, sizeof(BicgState)));
    double *V = s->bicg_vecs.p;
    BicgBuffers B{n, s->x.p, s->r.p, V, V + stride, V + 2 * stride, V + 3 * stride, V + 4 * stride,
                  V + 5 * stride, V + 6 * stride, s->diag.p, s->partials.p, s->bicg_st.p, dhist};
    // r = b - A x, or b when x = 0 (solver-phg.c:645-653)
    if (!is_zero(x1 / (double)n)) {
        CK(launch_spmv_plan(s->plan, s->x.p, s->Ap.p, s->stream));
        CK(launch_residual(n, drhs, s->Ap.p, B.rg, s->stream));
        s->launches += 2;
    } else {
        CK(cudaMemcpyAsync(B.rg, drhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
    }
    CK(launch_init_sums(n, 1, s->x.p, B.rg, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(B.rh, B.rg, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double rr0 = s->h_sums[0], r0 = sqrt(rr0);
    double tol = r0 * rtol;   // get_tol (solver-phg.c:104-115)
    if (tol < rb * btol) tol = rb * btol;
    if (tol < atol) tol = atol;

    BicgState init{};
    init.rho1 = rr0;   // r.rh with rh = r
    init.residual = r0;
    init.tol = tol;
    init.maxit = maxit;
    init.done = !(r0 > tol && 0 < maxit);
    *s->h_bst = init;
    CK(cudaMemcpyAsync(B.st, s->h_bst, sizeof(BicgState), cudaMemcpyHostToDevice, s->stream));
    if (dhist) CK(cudaMemcpyAsync(dhist, &s->h_bst->residual, sizeof(double), cudaMemcpyHostToDevice, s->stream));

    phgGpuSystem_::GraphKey key{};
    key.x = B.x; key.r = B.rg; key.p = B.rh; key.D = B.D; key.hist = dhist;
    key.n = n; key.lpr = s->plan.kind * 100 + s->plan.lpr * 10 + s->plan.unroll; key.s = s->stream;
    plan_key(s, key);
    if (s->graph_bicg == nullptr || !(s->gkey_bicg == key)) {
        if (s->graph_bicg != nullptr) { cudaGraphExecDestroy(s->graph_bicg); s->graph_bicg = nullptr; }
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < kGraphChunk; i++) launch_bicg_iteration(B, s->plan, s->stream);
        CK(cudaStreamEndCapture(s->stream, &gr));
        cudaError_t e = cudaGraphInstantiate(&s->graph_bicg, gr, 0);
        cudaGraphDestroy(gr);
        CK(e);
        s->gkey_bicg = key;
    }
    while (!s->h_bst->done) {
        CK(cudaGraphLaunch(s->graph_bicg, s->stream));
        s->launches += 5 * kGraphChunk;
        CK(cudaMemcpyAsync(s->h_bst, B.st, sizeof(BicgState), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    const int nits = s->h_bst->nits;
    double res = s->h_bst->residual;
    if (s->h_bst->status == BICG_SMALL_S) {
        // x += alpha p^, then the residual of b - A x (solver-phg.c:717-729)
        CK(launch_bicg_small_s(B, s->stream));
        CK(launch_spmv_plan(s->plan, s->x.p, s->Ap.p, s->stream));
        CK(launch_residual(n, drhs, s->Ap.p, B.rg, s->stream));
        CK(launch_init_sums(n, 1, s->x.p, B.rg, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
        s->launches += 4;
        CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        res = sqrt(s->h_sums[0]);
        s->h_bst->residual = res;
        if (dhist)
            CK(cudaMemcpyAsync(dhist + nits, &s->h_bst->residual, sizeof(double), cudaMemcpyHostToDevice,
                               s->stream));
    }
    if (residual) *residual = res;
    if (s->h_bst->status == BICG_BREAKDOWN)
        return fail(PHG_GPU_ERR_BREAKDOWN, "BiCGstab breakdown after %d iterations (rh.v = 0 or t.t = 0)", nits);
    if (s->h_bst->status == BICG_NONFINITE)
        return fail(PHG_GPU_ERR_NAN, "BiCGstab: non-finite values after %d iterations", nits);
    return nits;
}

}  // namespace

extern "C" {

int phgGpuSolverPCG(phgGpuSystem *s, double rtol, double btol, double atol, int maxit, double *x,
                    double *residual, double *hist) {
    g_last_warning.clear();
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
    const int nits = pcg_core(s, s->rhs.p, rtol, btol, atol, maxit, dhist, residual);
    if (nits < 0) return nits;
    CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
    if (hist) CHECK_RC(copy_out(s, hist, dhist, (size_t)nits + 1));
    CK(cudaStreamSynchronize(s->stream));
    return nits;
}

// GMRES_r (augk < 0) or FLGMRES_r (augk >= 1 augmenting corrections).
static int gmres_impl(phgGpuSystem *s, int restart, int augk, double rtol, double btol, double atol, int maxit,
                      double *x, double *residual) {
    g_last_warning.clear();
    if (s == nullptr || x == nullptr) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    if (maxit < 0) return fail(PHG_GPU_ERR_ARG, "maxit < 0");
    const bool flex = augk >= 0;
    const int mk = restart;
    if (flex) restart = mk + augk;   // the most steps a cycle takes
    if (mk < 1 || restart > kGmresMaxRestart)
        return fail(PHG_GPU_ERR_LIMIT, "GMRES: restart (plus augk) must be in 1..%d", kGmresMaxRestart);
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    const int64_t n = s->n;
    CHECK_RC(copy_in(s, s->x.p, x, (size_t)n));
    // ||b|| (solver-phg.c:1071-1075)
    CK(cudaMemsetAsync(s->ticket.p, 0, sizeof(unsigned) * kRedTickets, s->stream));
    CK(launch_init_sums(n, 0, s->x.p, s->rhs.p, s->diag.p, s->partials.p, s->ticket.p, s->sums.p, s->stream));
    s->launches += 1;
    CK(cudaMemcpyAsync(s->h_sums, s->sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const double b_norm = sqrt(s->h_sums[1]);
    if (fabs(b_norm) < 10.0 * DBL_MIN) {
        CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
        CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
        CK(cudaStreamSynchronize(s->stream));
        if (residual) *residual = 0.0;
        return 0;
    }
    CHECK_RC(tune_spmv(s));
    const int64_t stride = bicg_stride(n);
    // z, V_0..V_(R+1); FLGMRES_r also F_0..F_R and Z_0..Z_(augk-1)
    const int nvec = (restart + 3) + (flex ? (restart + 1) + augk : 0);
    CHECK_RC(s->gm_vecs.ensure((size_t)stride * nvec));
    CHECK_RC(s->gm_small.ensure((size_t)gmres_small_doubles(restart)));
    CHECK_RC(s->gm_st.ensure(1));
    if (s->h_gst == nullptr) CK(cudaMallocHost((void **)&s->h_gst, sizeof(GmresState)));
    const int R2 = restart + 2;
    GmresState init{};
    init.rtol = rtol;
    init.btol_bnorm = b_norm * btol;
    init.atol = atol;
    init.maxit = maxit;
    init.restart = restart;
    init.first = 1;
    init.flexible = flex ? 1 : 0;
    init.mk = mk;
    init.augk = flex ? augk : 0;
    init.H = s->gm_small.p;
    init.c1 = init.H + (size_t)R2 * R2;
    init.c2 = init.c1 + R2;
    init.s = init.c2 + R2;
    init.y = init.s + R2;
    *s->h_gst = init;
    CK(cudaMemsetAsync(s->gm_small.p, 0, sizeof(double) * (size_t)gmres_small_doubles(restart), s->stream));
    CK(cudaMemcpyAsync(s->gm_st.p, s->h_gst, sizeof(GmresState), cudaMemcpyHostToDevice, s->stream));

    double *F = flex ? s->gm_vecs.p + (int64_t)(restart + 3) * stride : nullptr;
    double *Zv = flex ? F + (int64_t)(restart + 1) * stride : nullptr;
    if (flex) CK(cudaMemsetAsync(Zv, 0, sizeof(double) * (size_t)stride * augk, s->stream));
    GmresBuffers B{n, s->x.p, s->rhs.p, s->diag.p, s->gm_vecs.p, s->gm_vecs.p + stride, stride, s->partials.p,
                   s->gm_st.p, F, Zv};
    phgGpuSystem_::GraphKey key{};
    key.x = B.x; key.r = B.z; key.p = B.V; key.D = B.D; key.Ap = B.st;
    key.n = (n * 100 + restart) * 2 + (flex ? 1 : 0); key.lpr = s->plan.kind * 100 + s->plan.lpr * 10 + s->plan.unroll; key.s = s->stream;
    plan_key(s, key);
    if (s->graph_gmres == nullptr || !(s->gkey_gmres == key)) {
        if (s->graph_gmres != nullptr) { cudaGraphExecDestroy(s->graph_gmres); s->graph_gmres = nullptr; }
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        launch_gmres_cycle(B, s->plan, restart, s->stream);
        CK(cudaStreamEndCapture(s->stream, &gr));
        cudaError_t e = cudaGraphInstantiate(&s->graph_gmres, gr, 0);
        cudaGraphDestroy(gr);
        CK(e);
        s->gkey_gmres = key;
    }
    const int per_cycle = 3 + restart * 2 + restart * (restart + 1) / 2;   // at most
    do {
        CK(cudaGraphLaunch(s->graph_gmres, s->stream));
        s->launches += per_cycle;
        CK(cudaMemcpyAsync(s->h_gst, s->gm_st.p, sizeof(GmresState), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    } while (!s->h_gst->finished);
    const int nits = s->h_gst->nits;
    if (residual) *residual = s->h_gst->residual;
    if (s->h_gst->status == GMRES_NONFINITE)
        return fail(PHG_GPU_ERR_NAN, "GMRES: non-finite values after %d iterations", nits);
    CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
    CK(cudaStreamSynchronize(s->stream));
    return nits;
}

int phgGpuSolverGMRES(phgGpuSystem *s, int restart, double rtol, double btol, double atol, int maxit, double *x,
                      double *residual) {
    return gmres_impl(s, restart, -1, rtol, btol, atol, maxit, x, residual);
}

int phgGpuSolverFLGMRES(phgGpuSystem *s, int restart, int augk, double rtol, double btol, double atol, int maxit,
                        double *x, double *residual) {
    if (augk <= 0) augk = 2;   // solver-phg.c:2086-2087
    return gmres_impl(s, restart, augk, rtol, btol, atol, maxit, x, residual);
}

int phgGpuSolverBiCGstab(phgGpuSystem *s, double rtol, double btol, double atol, int maxit, double *x,
                         double *residual, double *hist) {
    g_last_warning.clear();
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
    const int nits = bicg_core(s, rtol, btol, atol, maxit, dhist, residual);
    if (nits < 0) return nits;
    CHECK_RC(copy_out(s, x, s->x.p, (size_t)n));
    if (hist) CHECK_RC(copy_out(s, hist, dhist, (size_t)nits + 1));
    CK(cudaStreamSynchronize(s->stream));
    return nits;
}

int phgGpuAdjointGradient(phgGpuSystem *s, const double *u, const double *u_obs, double rtol, int maxit,
                          double *grad, double *J, int *nits_out) {
    g_last_warning.clear();
    if (s == nullptr || u == nullptr || u_obs == nullptr || grad == nullptr)
        return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (!s->assembled || !s->have_bdry_cols)
        return fail(PHG_GPU_ERR_STATE, "phgGpuAdjointGradient: needs a system built by phgGpuBuildLinearSystem");
    if (s->mass != 0.0)
        return fail(PHG_GPU_ERR_STATE, "phgGpuAdjointGradient: the system has a mass term (only kappa-scaled "
                                       "stiffness is differentiated)");
    if (maxit < 0) return fail(PHG_GPU_ERR_ARG, "maxit < 0");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    const int64_t n = s->n;
    const double *du, *duo;
    CHECK_RC(stage(s, u, (size_t)n, s->adj_u, &du));
    CHECK_RC(stage(s, u_obs, (size_t)n, s->adj_uobs, &duo));
    CHECK_RC(s->adj_rhs.ensure((size_t)n));
    CHECK_RC(s->adj_lambda.ensure((size_t)n));
    CHECK_RC(s->adj_grad.ensure((size_t)s->nelem));
    // adjoint right-hand side dJ/du on the free DOFs, and J
    CK(launch_adjoint_rhs(n, du, duo, s->bdry.p, s->adj_rhs.p, s->partials.p, s->sums.p, s->stream));
    s->launches += 2;
    double Jv = 0.0;
    CK(cudaMemcpyAsync(&Jv, s->sums.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    // the assembled matrix is symmetric (interior block + diagonal
    // Dirichlet block), so the adjoint system uses it as is
    CK(cudaMemsetAsync(s->x.p, 0, sizeof(double) * n, s->stream));
    double res = 0.0;
    const int nits = pcg_core(s, s->adj_rhs.p, rtol, 0.0, 0.0, maxit, nullptr, &res);
    if (nits < 0) return nits;
    if (s->h_st->status == PCG_BREAKDOWN)
        return fail(PHG_GPU_ERR_BREAKDOWN, "phgGpuAdjointGradient: adjoint PCG breakdown (matrix not SPD)");
    CK(cudaMemcpyAsync(s->adj_lambda.p, s->x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s->stream));
    const bool gdev = is_device_ptr(grad);
    double *dg = gdev ? grad : s->adj_grad.p;
    CK(launch_adjoint_grad(s->order, s->nelem, s->e2l.p, s->Ke.p, s->adj_lambda.p, du, dg, s->stream));
    s->launches += 1;
    if (!gdev) CHECK_RC(copy_out(s, grad, dg, (size_t)s->nelem));
    CK(cudaStreamSynchronize(s->stream));
    if (J) *J = Jv;
    if (nits_out) *nits_out = nits;
    return PHG_GPU_OK;
}


int phgGpuSolverBlockPCG(phgGpuSystem *s, int nrhs, const double *B, double *X, double rtol, int maxit,
                         int mixed, int *nits_out, double *res_out) {
    g_last_warning.clear();
    if (s == nullptr || B == nullptr || X == nullptr || nrhs <= 0) return fail(PHG_GPU_ERR_ARG, "invalid arguments");
    if (nrhs > 64) return fail(PHG_GPU_ERR_LIMIT, "phgGpuSolverBlockPCG: at most 64 right-hand sides per call");
    if (!s->assembled) return fail(PHG_GPU_ERR_STATE, "no assembled system");
    if (maxit < 0) return fail(PHG_GPU_ERR_ARG, "maxit < 0");
    CHECK_RC(set_device(s));
    CHECK_RC(solver_buffers(s));
    const int64_t n = s->n;
    int K = 8;   // padded column count: a power of two, at least one 8-column tile
    while (K < nrhs) K <<= 1;
    const size_t nk = (size_t)n * K;
    CHECK_RC(s->bX.ensure(nk));
    CHECK_RC(s->bR.ensure(nk));
    CHECK_RC(s->bP.ensure(nk));
    CHECK_RC(s->bAP.ensure(nk));
    CHECK_RC(s->bB.ensure((size_t)n * nrhs));
    CHECK_RC(s->bscal.ensure(7 * 64));
    CHECK_RC(s->bint.ensure(3 * 64 + 8));
    CHECK_RC(s->bpart.ensure(block_partials_doubles()));
    if (s->btick.p == nullptr) {
        CHECK_RC(s->btick.ensure(block_ticket_count()));
        CK(cudaMemsetAsync(s->btick.p, 0, sizeof(unsigned) * block_ticket_count(), s->stream));
    }
    if (mixed) {
        CHECK_RC(s->bY32.ensure(nk));
        CHECK_RC(s->bR32.ensure(nk));
        CHECK_RC(s->bP32.ensure(nk));
        CHECK_RC(s->bAP32.ensure(nk));
        CHECK_RC(s->bva32.ensure((size_t)s->nnz));
        CHECK_RC(s->D32.ensure((size_t)n));
        CK(launch_to_float(s->nnz, s->va.p, s->bva32.p, s->stream));
        s->launches += 1;
    }
    BlockPtrs P{};
    P.n = n;
    P.K = K;
    P.rp = s->rp.p;
    P.ci = s->ci.p;
    double *sc = s->bscal.p;
    P.rz_cur = sc; P.rz_prev = sc + 64; P.alpha = sc + 128; P.res = sc + 192; P.tol = sc + 256;
    P.maxr = sc + 320; P.pAp = sc + 384;
    P.nits = s->bint.p; P.done = s->bint.p + 64; P.status = s->bint.p + 128; P.flags = s->bint.p + 192;
    P.delta = 0.1;
    P.partials = s->bpart.p;
    P.tickets = s->btick.p;
    BlockVecs V{};
    V.va = s->va.p; V.D = s->diag.p; V.X = s->bX.p; V.R = s->bR.p; V.P = s->bP.p; V.AP = s->bAP.p;
    V.va32 = s->bva32.p; V.D32 = s->D32.p; V.Y32 = s->bY32.p; V.R32 = s->bR32.p; V.P32 = s->bP32.p;
    V.AP32 = s->bAP32.p;

    // autotune the SpMM tile once per matrix shape and column count
    if (!(s->btile != 0 && s->btile_n == n && s->btile_nnz == s->nnz && s->btile_K == K)) {
        CK(cudaMemsetAsync(s->bP.p, 0, sizeof(double) * nk, s->stream));
        CK(cudaMemsetAsync(s->bint.p, 0, sizeof(int) * (3 * 64 + 8), s->stream));   // flags: not done
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        const int cand[4] = {8, 16, 32, 64};
        int best = -1;
        for (int c = 0; c < 4; c++) {
            s->btile_ms[c] = 0.0;
            if (cand[c] > K) continue;
            for (int i = 0; i < 2; i++) {
                if (mixed) CK(launch_block_spmm32(P, cand[c], s->bva32.p, s->bP32.p, s->bAP32.p, s->stream));
                else CK(launch_block_spmm64(P, cand[c], s->va.p, s->bP.p, s->bAP.p, s->stream));
            }
            CK(cudaEventRecord(a, s->stream));
            for (int i = 0; i < 3; i++) {
                if (mixed) CK(launch_block_spmm32(P, cand[c], s->bva32.p, s->bP32.p, s->bAP32.p, s->stream));
                else CK(launch_block_spmm64(P, cand[c], s->va.p, s->bP.p, s->bAP.p, s->stream));
            }
            CK(cudaEventRecord(b, s->stream));
            CK(cudaEventSynchronize(b));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, a, b));
            s->btile_ms[c] = ms / 3;
            s->launches += 5;
            if (best < 0 || s->btile_ms[c] < s->btile_ms[best]) best = c;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        s->btile = cand[best < 0 ? 0 : best];
        s->btile_n = n; s->btile_nnz = s->nnz; s->btile_K = K;
    }
    const int T = s->btile;

    // R = B (zero initial guess), X = 0
    const double *dB;
    CHECK_RC(stage(s, B, (size_t)n * nrhs, s->bB, &dB));
    CK(launch_block_pack(n, nrhs, K, dB, s->bR.p, s->stream));
    CK(cudaMemsetAsync(s->bX.p, 0, sizeof(double) * nk, s->stream));
    int hflags[8] = {0, 0, 0, 1, maxit, 0, 0, 0};
    CK(cudaMemcpyAsync(P.flags, hflags, sizeof(hflags), cudaMemcpyHostToDevice, s->stream));
    CK(launch_block_init(P, mixed != 0, s->bR.p, s->diag.p, s->bR32.p, s->D32.p, s->bY32.p, rtol, s->stream));
    s->launches += 2;

    phgGpuSystem_::GraphKey key{};
    key.x = s->bX.p; key.r = s->bR.p; key.p = mixed ? (const void *)s->bP32.p : (const void *)s->bP.p;
    key.Ap = s->bva32.p; key.D = s->diag.p; key.va = s->va.p; key.hist = s->bpart.p;
    key.n = n; key.lpr = T * 1000 + K * 2 + (mixed ? 1 : 0); key.s = s->stream;
    if (s->graph_block == nullptr || !(s->gkey_block == key)) {
        if (s->graph_block != nullptr) { cudaGraphExecDestroy(s->graph_block); s->graph_block = nullptr; }
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < kGraphChunk; i++) launch_block_iteration(P, T, mixed != 0, V, s->stream);
        CK(cudaStreamEndCapture(s->stream, &gr));
        cudaError_t e = cudaGraphInstantiate(&s->graph_block, gr, 0);
        cudaGraphDestroy(gr);
        CK(e);
        s->gkey_block = key;
    }
    int all_done = 0;
    CK(cudaMemcpyAsync(&all_done, P.flags, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    while (!all_done) {
        CK(cudaGraphLaunch(s->graph_block, s->stream));
        s->launches += (mixed ? 4 : 3) * kGraphChunk;
        CK(cudaMemcpyAsync(&all_done, P.flags, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    // iteration counts and status, then the explicit FP64 residual B - A X per column
    std::vector<int> hint(3 * 64);
    CK(cudaMemcpyAsync(hint.data(), P.nits, sizeof(int) * 3 * 64, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemsetAsync(P.flags, 0, sizeof(int), s->stream));   // the kernels skip work once all are done
    CK(launch_block_spmm64(P, T, s->va.p, s->bX.p, s->bAP.p, s->stream));
    CK(launch_block_pack(n, nrhs, K, dB, s->bR.p, s->stream));
    CK(launch_block_sub((int64_t)nk, s->bR.p, s->bAP.p, s->stream));   // AP = R - AP
    CK(launch_block_init(P, false, s->bAP.p, s->diag.p, nullptr, nullptr, nullptr, 0.0, s->stream));
    s->launches += 4;
    std::vector<double> hres(64);
    CK(cudaMemcpyAsync(hres.data(), P.res, sizeof(double) * 64, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const bool xdev = is_device_ptr(X);
    double *dX = xdev ? X : s->bB.p;
    CK(launch_block_unpack(n, nrhs, K, s->bX.p, dX, s->stream));
    if (!xdev) CHECK_RC(copy_out(s, X, dX, (size_t)n * nrhs));
    CK(cudaStreamSynchronize(s->stream));
    if (res_out)
        for (int k = 0; k < nrhs; k++) res_out[k] = hres[k];
    if (nits_out)
        for (int k = 0; k < nrhs; k++) nits_out[k] = hint[k];
    for (int k = 0; k < nrhs; k++) {
        if (hint[128 + k] == 1) return fail(PHG_GPU_ERR_BREAKDOWN, "block PCG: breakdown in column %d", k);
        if (hint[128 + k] == 2) return fail(PHG_GPU_ERR_NAN, "block PCG: non-finite residual in column %d", k);
    }
    return PHG_GPU_OK;
}

int phgGpuGetBlockTile(phgGpuSystem *s, int *tile, double *times_ms) {
    if (s == nullptr) return fail(PHG_GPU_ERR_ARG, "null system");
    if (s->btile == 0) return fail(PHG_GPU_ERR_STATE, "no block solve yet");
    if (tile) *tile = s->btile;
    if (times_ms)
        for (int c = 0; c < 4; c++) times_ms[c] = s->btile_ms[c];
    return PHG_GPU_OK;
}
}  // extern "C"
