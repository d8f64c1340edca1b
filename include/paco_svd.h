/*
 * paco_svd.h -- C ABI of the B200 (sm_100a) SVD library libpacosvd.so.
 *
 * Drop-in for the operator surface of DEAVEN-MITCH/paco-svd: the two device
 * kernels launched by main.cpp (upper_bidiagonalization, svd_DC), the host
 * tiling helpers (getTilingSize, GenerateTiling) and the buffer contract of
 * main.cpp:33-123.  Plain pointers and sizes only; `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * All matrices are FP32, row-major, M >= N.  Every entry point returns a
 * PACO_* status; device-side failures (non-convergence, bounded-wait
 * timeouts, a tiling blob for another N) are recorded in the workspace and
 * reported by paco_sync_status().
 */
#ifndef PACO_SVD_H
#define PACO_SVD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum paco_status {
    PACO_OK = 0,
    PACO_ERR_INVALID_ARG = 1,     /* M < N, N <= 0, NULL pointer, short buffer  */
    PACO_ERR_UNSUPPORTED = 2,     /* shape outside the kernels' limits         */
    PACO_ERR_CUDA = 3,            /* a CUDA runtime call failed                 */
    PACO_ERR_DEVICE = 4,          /* a kernel recorded an error                 */
    PACO_ERR_NONCONVERGENCE = 5,  /* a secular root hit its iteration limit     */
    PACO_ERR_TIMEOUT = 6,         /* a bounded device-side wait gave up         */
    PACO_ERR_BAD_TILING = 7,      /* tiling blob does not describe this N       */
    PACO_ERR_NONFINITE = 8        /* NaN/Inf in the input matrix                */
};

/* Largest N accepted by the stage-1 kernels (row tiles live in shared memory). */
#define PACO_MAX_N 8192

/* Size in bytes of the tiling blob for an N-column bidiagonal.
 * Replaces svd_tiling.cpp:67 getTilingSize(int N, int svdBlockNum). */
int getTilingSize(int N, int svdBlockNum);

/* Writes the leaf partition of svd_tiling.cpp:83-130 (3-column leaves,
 * remainder cases for N%3) into TilingHost (getTilingSize bytes).
 * Replaces svd_tiling.cpp:83 GenerateTiling(int N, int blockDim, uint8_t*). */
void GenerateTiling(int N, int blockDim, uint8_t *TilingHost);

/* Tiling autotuner (replaces the fixed host tiling of svd_tiling.cpp:11-66,
 * SVDTiling / initTCubeTiling, which sets one 1024^3 matmul tile for every
 * shape).  paco_autotune times the candidate configurations of the
 * single-matrix path on a synthetic M x N matrix (the persistent panel kernel
 * or the two-kernel row/column passes, rows per CTA of a panel, the tcgen05
 * or SIMT engine for the large products, the last columns on one
 * thread-block cluster or on the panel kernel), keeps the fastest for (M, N) in a
 * process-wide table that every later call of that shape uses, and returns
 * out[0] = chosen candidate, out[1] = its ms per SVD, out[2] = ms of the
 * defaults, out[3] = candidates tried.  It allocates its own device buffers
 * and synchronizes `stream`.  cfg[4] = {persistent (0/1), rows per CTA
 * (4..256), tcgen05 products (0/1), last columns kept off the cluster kernel
 * (0/1)}: paco_tune_get returns the entry in
 * use for (M, N) (the defaults {1, 16, 1, 0} if none), paco_tune_set stores
 * one (for example a choice saved by an earlier process). */
int paco_autotune(int M, int N, void *stream, double out[4]);
int paco_tune_get(int M, int N, int cfg[4]);
int paco_tune_set(int M, int N, const int cfg[4]);

/* QR-first reduction for tall matrices (no counterpart in the reference,
 * which lists it as future work, README.md:22): A = Q R, the SVD pipeline on
 * the N x N factor R, U = Q blockdiag(U_R, I).  It applies to shapes with
 * M > N and N >= 1024 whose QR blocks fit one thread-block cluster (M up to
 * about 13,000); mode 0 = off, 1 = on, 2 = automatic (on when M >= 1.6 N, the
 * default), -1 = query the mode, -2 = query whether calls of this shape take
 * the QR-first path now (1) or not (0).  paco_autotune times both choices for
 * such shapes.  Returns the mode stored (or the answer), -1 for an invalid
 * argument. */
int paco_tune_qr(int M, int N, int mode);

/* One field of the tuning entry for (M, N): which = 0 persistent panel
 * kernel (0/1), 1 rows per CTA of a panel (4..256), 2 tcgen05 products (0/1),
 * 3 last columns kept off the cluster kernel (0/1), 4 reflectors per
 * compact-WY block when U and V are formed (64 or 128; 0 = 128), 5 columns per
 * QR block (32 or 64; 0 = 64), 6 matrices per lockstep group of
 * paco_svd_multi (1..8; 0 = 4), 7 the QR-first mode of paco_tune_qr, 8 the
 * two-stage reduction (dense -> band -> bidiagonal by bulge chasing) with
 * band width 32 or 64, 0 off (the default; used for N >= 1024 when its
 * chasing kernel holds the band, and then before QR-first).  value -1
 * queries.  Returns the value stored or queried, -1 for an invalid
 * argument.  paco_autotune times fields 0-5, 7 and 8 for one shape;
 * paco_autotune_multi times field 6 (2, 4, 8) on `count` synthetic matrices
 * of the shape, then for tall shapes the other QR-first choice with that
 * group size (out as paco_autotune's, out[0] = the group size chosen).
 * paco_multi_group, when set, overrides field 6 for every shape. */
int paco_tune_param(int M, int N, int which, int value);
int paco_autotune_multi(int count, int M, int N, void *stream, double out[4]);

/* Buffer sizes in bytes of main.cpp:33-43, in this order:
 * [0] U M*M, [1] A M*N, [2] Vt N*N, [3] d N, [4] e N-1, [5] tauq N,
 * [6] taup N-1, [7] qt 2*N*N, [8] wt 2*N*N, [9] tiling, [10] idx 16*N*u32,
 * [11] workspace (this library's, replaces the 40*32 B soft-sync area). */
void paco_buffer_sizes(int M, int N, size_t out[12]);

/* Workspace bytes needed by upper_bidiagonalization and svd_DC. */
size_t paco_workspace_size(int M, int N);

/* Stage 1: Golub-Kahan Householder upper bidiagonalization of a (M x N).
 * a is overwritten with the Householder vectors (d on the diagonal, e on the
 * superdiagonal); d[N], e[N-1], tauq[N], taup[N-1] are written; u (M x M)
 * and vt (N x N) are formed explicitly (no pre-zeroing needed), so that
 * A = U * B * Vt.  Reflector convention of upper_bidiagonalization.cpp:182-218
 * (d_i, e_i >= 0 unless the reflected part is exactly zero).
 * Replaces upper_bidiagonalization.cpp:967
 *   upper_bidiagonalization(M, N, a, u, vt, d, e, tauq, taup, workspace). */
int upper_bidiagonalization(int M, int N, float *a, float *u, float *vt, float *d,
                            float *e, float *tauq, float *taup, void *workspace,
                            void *stream);

/* Stage 2: bidiagonal divide and conquer on (d, e).  On return d holds the
 * singular values in descending order, u[:, :N] <- u[:, :N] * Q and
 * vt <- W^T * vt.  a (M x N) is used as scratch (destroyed); qt, wt (2*N*N
 * floats each) and idx (16*N uint32) are scratch; tiling is the device copy
 * of the GenerateTiling blob.
 * Replaces svd.cpp:2105 svd_DC(M, N, a, u, vt, d, e, qt, wt, idx, workspace, tiling). */
int svd_DC(int M, int N, float *a, float *u, float *vt, float *d, float *e, float *qt,
           float *wt, uint32_t *idx, void *workspace, const uint8_t *tiling, void *stream);

/* Synchronizes `stream` and returns the first device-side error recorded in
 * `workspace` since the last call (then clears it).  *info receives detail. */
int paco_sync_status(void *workspace, void *stream, int *info);

/* Device-buffer one-shot SVD (both stages, the flow of main.cpp:56-174 on
 * device memory): A (M x N, destroyed), U (M x M), Vt (N x N), sigma (N,
 * descending).  ws must hold paco_svd_workspace_size(M, N) bytes; all the
 * intermediate buffers of main.cpp live in it.  Asynchronous on `stream`. */
size_t paco_svd_workspace_size(int M, int N);
int paco_svd(int M, int N, float *A, float *U, float *Vt, float *sigma, void *ws,
             size_t ws_bytes, void *stream);

/* Thin-U form of paco_svd: U is M x N, the first N left singular vectors
 * (A = U diag(sigma) Vt), where the reference always forms the M x M U
 * (main.cpp:33,173).  The reflectors are applied to [I; 0] (or, for a tall
 * matrix on the QR-first path, to [U_R; 0]) instead of forming M x M
 * products: for M = 2N about a third of the formation's multiply-adds and
 * half of U's memory.  Same workspace (paco_svd_workspace_size) and rules as
 * paco_svd. */
int paco_svd_thin(int M, int N, float *A, float *U, float *Vt, float *sigma, void *ws,
                  size_t ws_bytes, void *stream);

/* Host-buffer SVD through a reusable context (device buffers and pinned
 * staging allocated once): copies A to the device, runs both stages, copies
 * U, Vt, sigma back, synchronizes.  The path svd_main takes (main.cpp:64-174). */
typedef struct paco_ctx paco_ctx;
int paco_ctx_create(int M, int N, paco_ctx **out);
int paco_ctx_svd_host(paco_ctx *ctx, const float *A, float *U, float *Vt, float *sigma);
void paco_ctx_destroy(paco_ctx *ctx);

/* Allocation-free SVD (no counterpart in the reference) for callers that
 * cannot call cudaMalloc: code running where a framework's caching allocator
 * owns all device memory, or real-time and embedded hosts that must not grow
 * their memory after start-up.  Same inputs and outputs as paco_svd (A is
 * destroyed), M <= 1024 and N <= 512 (larger shapes return
 * PACO_ERR_UNSUPPORTED).  All scratch lives in a 16 MiB device array inside
 * the library, which every GPU that loads the library holds until the process
 * exits; no device memory is allocated per call.  The first call on a device
 * looks up that array's address and keeps it for the life of the process, so
 * a device reset with cudaDeviceReset must not be followed by further calls
 * on that device.  Calls share the array: calls that overlap on the GPU, from
 * any stream or thread, race and must be serialized by the caller.  The call
 * synchronizes `stream` and returns the device status of the run
 * (PACO_ERR_INVALID_ARG when `stream` is being captured). */
int paco_svd_noalloc(int M, int N, float *A, float *U, float *Vt, float *sigma, void *stream);

/* Largest M (and so N) of a matrix of the batched form's one-CTA-per-matrix
 * kernels; larger matrices of one shape go to the multi-matrix form. */
#define PACO_BATCH_MAX_M 2048

/* Batched form (the reference runs one matrix per launch; this replaces a
 * host loop over main.cpp:126-158 for many independent small matrices).
 * Bytes of workspace paco_svd_batched needs for these shapes; 0 if a shape
 * is invalid (N < 1, M < N), or M > PACO_BATCH_MAX_M in a list whose shapes
 * are not all the same. */
size_t paco_batched_workspace_size(int count, const int *M, const int *N);

/* SVD of `count` independent row-major FP32 matrices in one persistent
 * launch: each CTA takes the next matrix (largest first) from a work queue
 * and runs bidiagonalization, divide and conquer and the back-transforms for
 * it.  When every matrix has one shape with M > PACO_BATCH_MAX_M the call is
 * paco_svd_multi (and paco_batched_workspace_size returns its workspace
 * size); other lists with such a matrix are PACO_ERR_UNSUPPORTED.
 * M, N and the pointer arrays are host arrays; A[b] (M x N), U[b]
 * (M x M), Vt[b] (N x N) and sigma[b] (N) are device buffers; A is read only.
 * `status` (device, count ints, may be null) receives each matrix's
 * PACO_* code.  Asynchronous on `stream`; the workspace and outputs must stay
 * alive until the stream has finished the call. */
int paco_svd_batched(int count, const int *M, const int *N, const float *const *A, float *const *U,
                     float *const *Vt, float *const *sigma, int *status, void *workspace, size_t ws_bytes,
                     void *stream);

/* Multi-matrix form for large matrices of one shape (a host loop over
 * main.cpp:126-158 in the reference, one matrix per launch): `count` SVDs
 * share the GPU in groups of k.  Stage 1 of a group runs in lockstep, each
 * persistent panel launch serving all k matrices with num_SMs / k CTAs each
 * (the column steps are latency-bound, so k matrices take little longer than
 * one); the divide-and-conquer runs of a group then proceed concurrently on
 * internal streams.  A[b] is read only; U[b] (M x M), Vt[b] (N x N),
 * sigma[b] (N) as paco_svd.  `status` (device, count ints, may be null)
 * receives each matrix's PACO_* code when its group has finished.
 * Asynchronous on `stream` (recorded as a CUDA graph per buffers on a
 * capturable stream); the workspace must stay alive until it has run. */
size_t paco_svd_multi_workspace_size(int count, int M, int N);
int paco_svd_multi(int count, int M, int N, const float *const *A, float *const *U, float *const *Vt,
                   float *const *sigma, int *status, void *workspace, size_t ws_bytes, void *stream);
/* Matrices per lockstep group of paco_svd_multi for every shape (1..8; 0 =
 * the shape's tuning entry, 4 by default); returns the previous setting.
 * Set it before computing workspace sizes. */
int paco_multi_group(int k);

/* Library version string. */
const char *paco_version(void);

/* Kernel timing (no counterpart in the reference, which is profiled with
 * msprof, myprof.sh:1-8): while enabled, every launch of the dominant
 * stage-1 kernel (the persistent panel kernel, or the row pass where that
 * one cannot launch) is bracketed by CUDA events on its stream.
 * paco_profile_read synchronizes on them and returns totals since the last
 * enable: out[0] = milliseconds, out[1] = launches, out[2] = bytes the
 * launches had to read (live row segments), out[3] = 1 for the persistent
 * panel kernel, 0 for the row pass.  Host-thread-local use only. */
void paco_profile_enable(int on);
void paco_profile_read(double out[4]);

/* Number of kernels this library has launched in the process so far (a
 * replay of a recorded CUDA graph counts the kernels the graph holds). */
unsigned long long paco_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* PACO_SVD_H */
