// Launch interfaces of the assembly kernels (assemble.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phgb {

// Largest quadrature rules of the element kernel (P3: order 4 with 14
// points for the stiffness, order 6 with 24 for the mass and RHS).
constexpr int kElemMaxQK = 14;
constexpr int kElemMaxQR = 24;

struct ElemArgs {
    int64_t nelem, nvert, ndof;
    const double *verts;
    const int32_t *elems, *e2l;
    const double *kappa, *f;                 // may be null
    double mass;                             // mass coefficient c (0: stiffness only)
    // element tables (device): gk = d phi_k / d lambda_c at stiffness point q
    // as gk[(c * QK + q) * N + k]; br = phi_k at rhs point q as br[q * N + k],
    // brt the same transposed (brt[k * QR + q])
    const double *gk, *br, *brt;
    const double *wk_host, *wr_host;         // quadrature weights (host; passed by value)
    double *geo;                             // nelem * geometry_doubles: J (16), volume per element
    bool geometry_given;                     // geo holds the caller's geometry (else computed here)
    double *Ke, *Re;
    int *status;
};

struct WalkArgs {
    int64_t ndof;
    const int32_t *inc_ptr, *inc, *e2l;
    const uint8_t *bdry;
    const double *Ke, *Re, *g;
    int32_t *cnt_keep, *cnt_bdry;            // entries kept / saved per row
    int32_t *sc_cols;                        // scratch: nelem * N * N entries
    double *sc_vals;
    const int32_t *ptr, *bptr;               // compaction: CSR row pointers
    int32_t *cols, *bcols;
    double *vals, *bvals, *rhs, *diag;
    int *status;
    // rows longer than the walk's shared-memory table: listed by the walk and
    // assembled by a second pass with a larger table (over_list: ndof
    // entries; *nover zeroed before the walk)
    int32_t *over_list;
    int *nover;
    // the pattern: recorded by the walk when non-null (nelem * N * N
    // entries each, indexed like the scratch regions), read by the value walk
    uint16_t *slot, *tmap;
    // per row, the index of its diagonal among its kept entries (recorded
    // with the pattern; rows without one keep the caller's -1)
    int32_t *dpos;
};

cudaError_t launch_element_kernel(int p, const ElemArgs &a, cudaStream_t s);
cudaError_t launch_incidence(int N, int64_t nelem, int64_t ndof, const int32_t *e2l, int32_t *cnt,
                             int32_t *inc_ptr, int32_t *cursor, int32_t *inc, int64_t *scan_ws,
                             int *status, cudaStream_t s);
int64_t scan_workspace_elems(int64_t n);
// out[0..n] = exclusive prefix sums of in[0..n-1], out[n] = total (int32).
cudaError_t launch_scan(int64_t n, const int32_t *in, int32_t *out, int64_t *ws, cudaStream_t s);
// One pass over the rows into the scratch regions (counts, RHS, diagonal),
// then, after the counts are scanned into ptr/bptr, the copy into the CSR.
cudaError_t launch_row_walk(int p, const WalkArgs &a, cudaStream_t s);
cudaError_t launch_compact(int N, const WalkArgs &a, cudaStream_t s);
// A build on the recorded pattern: writes vals, bvals, rhs and diag in place
// (ptr, cols, bptr, bcols as the recording build left them); a changed
// pattern sets PHGB_DEV_PATTERN_CHANGED.
cudaError_t launch_value_walk(int p, const WalkArgs &a, cudaStream_t s);

// Longest row the walk assembles (its second pass); longer rows are
// PHG_GPU_ERR_LIMIT.
int row_walk_max_row(int p);

// Rows from recorded row segments (phgMatAddEntries_ calls), in call order.
struct RecordArgs {
    int64_t n;                                // rows
    const int32_t *rinc_ptr, *rinc;           // per row, its records in call order
    const int64_t *rec_ptr;                   // entries of record r: [rec_ptr[r], rec_ptr[r + 1])
    const int32_t *rec_cols;
    const double *rec_vals;
    const int32_t *cap_ptr;                   // scratch offset of each row (its entries' total)
    int32_t *cnt;                             // entries of each row
    int32_t *sc_cols;
    double *sc_vals;
    int *status;
    int32_t *over_list;                       // rows over 256 entries, for the second pass
    int *nover;
};
// Longest row the record walk assembles.
constexpr int kRecordMaxRow = 1024;
cudaError_t launch_record_lengths(int64_t nrec, const int32_t *rec_row, const int64_t *rec_ptr, int32_t *cap,
                                  cudaStream_t s);
cudaError_t launch_record_walk(const RecordArgs &a, cudaStream_t s);
cudaError_t launch_record_compact(const RecordArgs &a, const int32_t *ptr, int32_t *cols, double *vals,
                                  cudaStream_t s);
int64_t geometry_doubles(int64_t nelem);
int geometry_stride();                       // doubles per element in geo

}  // namespace phgb
