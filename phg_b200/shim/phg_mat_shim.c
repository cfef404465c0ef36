/*
 * Per-call drop-in for PHG's row insertion, assembled on the GPU.
 *
 * Loaded ahead of a shared PHG library (LD_PRELOAD, or linked before
 * libphg), this library defines
 *
 *   void phgMatAddEntries_(MAT *mat, INT nrows, const INT *rows, INT ncols,
 *                          const INT *cols, const FLOAT *values,
 *                          BOOLEAN rows_are_global, BOOLEAN cols_are_global,
 *                          BOOLEAN replace)
 *   void phgMatAddEntry_(MAT *mat, INT row, INT col, FLOAT value,
 *                        BOOLEAN row_is_global, BOOLEAN col_is_global,
 *                        BOOLEAN replace)
 *   void phgMatAssemble(MAT *mat)
 *   void phgMatDestroy(MAT **mat)
 *
 * with the reference's signatures (include/phg/matvec.h).  For a serial,
 * unpermuted matrix (one process, no L2Vmap, local indices, adding rather
 * than replacing) the calls only record their row segments (a short append
 * under a lock, so OpenMP element loops may call in).  phgMatAssemble then
 * builds the rows from the recorded segments on the GPU with
 * phgGpuAssembleRows -- the first-touch column order and the sums of
 * add_columns_to_row (src/matvec.c:3045-3332), exact zeros dropped as
 * phgMatAddEntries_ drops them (:5459-5461) -- stores them in the matrix's
 * MAT_ROW arrays as PHG would have, and calls PHG's own phgMatAssemble
 * (boundary elimination and the rest).  Any call outside those cases first
 * replays the matrix's recorded segments through PHG's phgMatAddEntries_ in
 * their order, then goes to PHG, and the matrix stays with PHG from then on,
 * so the order of every contribution is kept.  A GPU failure at assembly
 * time (for instance a row's first segment naming a column twice, which PHG
 * keeps twice) also falls back to the replay.  Set PHG_MAT_SHIM_STATS to
 * print what was recorded at exit.
 */
#define _GNU_SOURCE
#include "phg.h"
#include "phg_gpu.h"

#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef void (*adds_fn)(MAT *, INT, const INT *, INT, const INT *, const FLOAT *, BOOLEAN, BOOLEAN, BOOLEAN);
typedef void (*add1_fn)(MAT *, INT, INT, FLOAT, BOOLEAN, BOOLEAN, BOOLEAN);
typedef void (*asm_fn)(MAT *);
typedef void (*dst_fn)(MAT **);

#define MAT_ROW_TRUNK 8   /* the reference's allocation trunk for rows (matvec.c:2823) */

typedef struct Rec {
    MAT *mat;
    int host;                 /* the matrix's calls go to PHG */
    int32_t *row;
    int64_t *ptr;             /* nrec + 1 */
    int32_t *cols;
    double *vals;
    int64_t nrec, nent, caprec, capent;
    struct Rec *next;
} Rec;

/* set while this thread is inside a PHG function called from here: PHG's
 * own internal calls to the interposed functions go straight to PHG */
static __thread int in_phg = 0;

static struct {
    pthread_mutex_t lock;
    Rec *recs;
    phgGpuSystem *sys;
    long recorded, assembled, replayed, forwarded;
    int stats_registered;
} S = {PTHREAD_MUTEX_INITIALIZER};

#define ORIG(type, name)                                        \
    static type orig_##name(void) {                             \
        static type f = NULL;                                   \
        if (f == NULL) f = (type)dlsym(RTLD_NEXT, #name);       \
        return f;                                               \
    }
ORIG(adds_fn, phgMatAddEntries_)
ORIG(add1_fn, phgMatAddEntry_)
ORIG(asm_fn, phgMatAssemble)
ORIG(dst_fn, phgMatDestroy)

static void print_stats(void) {
    fprintf(stderr, "phg_mat_shim: segments %ld recorded, %ld matrices assembled on the GPU, %ld replayed, "
            "%ld calls forwarded\n", S.recorded, S.assembled, S.replayed, S.forwarded);
}

static Rec *find(MAT *m, int create) {
    Rec *r;
    for (r = S.recs; r != NULL; r = r->next)
        if (r->mat == m) return r;
    if (!create) return NULL;
    r = (Rec *)calloc(1, sizeof(*r));
    r->mat = m;
    r->next = S.recs;
    S.recs = r;
    if (!S.stats_registered && getenv("PHG_MAT_SHIM_STATS") != NULL) {
        atexit(print_stats);
        S.stats_registered = 1;
    }
    return r;
}

static void drop(MAT *m) {
    Rec **pp = &S.recs;
    while (*pp != NULL) {
        if ((*pp)->mat == m) {
            Rec *r = *pp;
            *pp = r->next;
            free(r->row); free(r->ptr); free(r->cols); free(r->vals); free(r);
            return;
        }
        pp = &(*pp)->next;
    }
}

/* The cases recorded: what the reference handles in its serial branch with
 * local indices equal to vector indices (matvec.c:5147-5230). */
static int eligible(MAT *mat, BOOLEAN rows_global, BOOLEAN cols_global, BOOLEAN replace) {
#if USE_MPI
    (void)mat; (void)rows_global; (void)cols_global; (void)replace;
    return 0;
#else
    return !replace && !cols_global && !rows_global && mat->mode != PHG_REPLACE &&
           mat->type != PHG_MATRIX_FREE && mat->blocks == NULL && !mat->assembled && mat->rmap->nprocs == 1 &&
           mat->cmap->nprocs == 1 && mat->rmap->L2Vmap == NULL && mat->cmap->L2Vmap == NULL &&
           mat->rmap->localsize == mat->rmap->nlocal && mat->cmap->localsize == mat->cmap->nlocal;
#endif
}

static void grow(Rec *r, int64_t nrec, int64_t nent) {
    if (r->nrec + nrec > r->caprec) {
        int64_t c = r->caprec ? 2 * r->caprec : 4096;
        while (c < r->nrec + nrec) c *= 2;
        r->row = (int32_t *)realloc(r->row, sizeof(int32_t) * c);
        r->ptr = (int64_t *)realloc(r->ptr, sizeof(int64_t) * (c + 1));
        r->caprec = c;
        if (r->nrec == 0) r->ptr[0] = 0;
    }
    if (r->nent + nent > r->capent) {
        int64_t c = r->capent ? 2 * r->capent : 65536;
        while (c < r->nent + nent) c *= 2;
        r->cols = (int32_t *)realloc(r->cols, sizeof(int32_t) * c);
        r->vals = (double *)realloc(r->vals, sizeof(double) * c);
        r->capent = c;
    }
    if (r->row == NULL || r->ptr == NULL || r->cols == NULL || r->vals == NULL) {
        fprintf(stderr, "phg_mat_shim: out of host memory\n");
        abort();
    }
}

/* Hands the recorded segments to PHG in their order and leaves the matrix
 * with PHG (called with the lock held). */
static void replay(Rec *r) {
    int64_t k;
    r->host = 1;
    in_phg++;
    for (k = 0; k < r->nrec; k++) {
        const int64_t b = r->ptr[k];
        const INT row = r->row[k];
        orig_phgMatAddEntries_()(r->mat, 1, &row, (INT)(r->ptr[k + 1] - b), r->cols + b, r->vals + b, FALSE,
                                 FALSE, FALSE);
    }
    in_phg--;
    if (r->nrec > 0) S.replayed++;
    r->nrec = r->nent = 0;
    if (r->ptr != NULL) r->ptr[0] = 0;
}

/* Called with the lock held: whether the call was recorded; if not, the
 * matrix's segments so far have been replayed and the caller forwards. */
static int record(MAT *mat, INT nrows, const INT *rows, INT ncols, const INT *cols, const FLOAT *values,
                  BOOLEAN rows_global, BOOLEAN cols_global, BOOLEAN replace) {
    Rec *r = find(mat, 1);
    INT i;
    if (r->host || !eligible(mat, rows_global, cols_global, replace)) {
        if (!r->host) replay(r);
        return 0;
    }
    if (mat->mode == PHG_UNDEFINED) mat->mode = PHG_ADD;
    grow(r, nrows, (int64_t)nrows * ncols);
    for (i = 0; i < nrows; i++) {
        if (rows[i] < 0) continue;
        r->row[r->nrec] = rows[i];
        memcpy(r->cols + r->nent, cols, sizeof(INT) * (size_t)ncols);
        memcpy(r->vals + r->nent, values + (size_t)i * ncols, sizeof(FLOAT) * (size_t)ncols);
        r->nent += ncols;
        r->ptr[++r->nrec] = r->nent;
        S.recorded++;
    }
    return 1;
}

void phgMatAddEntries_(MAT *mat, INT nrows, const INT *rows, INT ncols, const INT *cols, const FLOAT *values,
                       BOOLEAN rows_are_global, BOOLEAN cols_are_global, BOOLEAN replace) {
    int done = 0;
    if (ncols <= 0 || nrows <= 0) return;
    if (!in_phg) {
        pthread_mutex_lock(&S.lock);
        done = record(mat, nrows, rows, ncols, cols, values, rows_are_global, cols_are_global, replace);
        pthread_mutex_unlock(&S.lock);
    }
    if (!done) {
        __atomic_add_fetch(&S.forwarded, 1, __ATOMIC_RELAXED);
        in_phg++;
        orig_phgMatAddEntries_()(mat, nrows, rows, ncols, cols, values, rows_are_global, cols_are_global, replace);
        in_phg--;
    }
}

void phgMatAddEntry_(MAT *mat, INT row, INT col, FLOAT value, BOOLEAN row_is_global, BOOLEAN col_is_global,
                     BOOLEAN replace) {
    int done = 0;
    /* the reference returns before anything else on these (matvec.c:5297) */
    if (row < 0 || col < 0 || value == 0.0) return;
    if (!in_phg) {
        pthread_mutex_lock(&S.lock);
        done = record(mat, 1, &row, 1, &col, &value, row_is_global, col_is_global, replace);
        pthread_mutex_unlock(&S.lock);
    }
    if (!done) {
        __atomic_add_fetch(&S.forwarded, 1, __ATOMIC_RELAXED);
        in_phg++;
        orig_phgMatAddEntry_()(mat, row, col, value, row_is_global, col_is_global, replace);
        in_phg--;
    }
}

/* The rows from the GPU into the matrix's MAT_ROW arrays; 0 on success. */
static int assemble_on_gpu(Rec *r) {
    MAT *mat = r->mat;
    const INT n = mat->rmap->nlocal;
    int64_t nn, nnz, nb, k;
    int64_t *ptr;
    int32_t *cols;
    double *vals;
    INT i;
    for (i = 0; i < n; i++)
        if (mat->rows[i].ncols != 0) return -1;   /* PHG holds entries of its own */
    if (S.sys == NULL) {
        const char *dev = getenv("PHG_GPU_DEVICE");
        if (phgGpuCreate(dev == NULL ? 0 : atoi(dev), NULL, &S.sys) != PHG_GPU_OK) return -1;
    }
    for (k = 0; k < r->nrec; k++)
        if (r->row[k] >= n) return -1;
    if (phgGpuAssembleRows(S.sys, n, r->nrec, r->row, r->ptr, r->cols, r->vals) != PHG_GPU_OK ||
        phgGpuGetSizes(S.sys, &nn, &nnz, &nb) != PHG_GPU_OK || nn != n) {
        fprintf(stderr, "phg_mat_shim: %s (the segments go to PHG)\n", phgGpuLastError());
        return -1;
    }
    ptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    vals = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    if (ptr == NULL || cols == NULL || vals == NULL || phgGpuGetMatrix(S.sys, ptr, cols, vals) != PHG_GPU_OK) {
        free(ptr); free(cols); free(vals);
        return -1;
    }
    /* check_mat_localsize (matvec.c:5107-5145), serial branch: what the
     * reference's first row conversion sets */
    if (mat->localsize < 0) {
        mat->bdry_localsize = mat->rmap->localsize - mat->rmap->nlocal;
        mat->localsize = mat->rmap->localsize;
    }
    for (i = 0; i < n; i++) {
        MAT_ROW *row = mat->rows + i;
        const INT m = (INT)(ptr[i + 1] - ptr[i]);
        if (m == 0) continue;
        row->alloc = ((m + MAT_ROW_TRUNK - 1) / MAT_ROW_TRUNK) * MAT_ROW_TRUNK;
        row->cols = (INT *)phgAlloc(row->alloc * sizeof(*row->cols));
        row->data = (FLOAT *)phgAlloc(row->alloc * sizeof(*row->data));
        row->ncols = m;
        memcpy(row->cols, cols + ptr[i], sizeof(INT) * (size_t)m);
        memcpy(row->data, vals + ptr[i], sizeof(FLOAT) * (size_t)m);
    }
    free(ptr); free(cols); free(vals);
    return 0;
}

void phgMatAssemble(MAT *mat) {
    Rec *r;
    if (in_phg) {
        orig_phgMatAssemble()(mat);
        return;
    }
    pthread_mutex_lock(&S.lock);
    r = find(mat, 0);
    if (r != NULL && !r->host && r->nrec > 0 && !mat->assembled) {
        if (assemble_on_gpu(r) == 0) {
            S.assembled++;
            r->nrec = r->nent = 0;
            r->ptr[0] = 0;
        } else {
            replay(r);
        }
    }
    if (r != NULL) drop(mat);
    pthread_mutex_unlock(&S.lock);
    in_phg++;
    orig_phgMatAssemble()(mat);
    in_phg--;
}

/* The records of a matrix PHG frees (its last reference, matvec.c:2292-2311)
 * go with it. */
void phgMatDestroy(MAT **mat) {
    if (!in_phg && mat != NULL && *mat != NULL && (*mat)->refcount <= 0) {
        pthread_mutex_lock(&S.lock);
        drop(*mat);
        pthread_mutex_unlock(&S.lock);
    }
    in_phg++;
    orig_phgMatDestroy()(mat);
    in_phg--;
}
