// C ABI of libpacosvd.so (declared in include/paco_svd.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "bdc.cuh"
#include "bidiag.cuh"
#include "qr.cuh"
#include "twostage.cuh"

namespace {

int device_sms()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
}

bool shape_ok(int M, int N) { return N >= 1 && M >= N && N <= PACO_MAX_N && (long)M * M < (1L << 40); }


struct SvdLayout {
    size_t ws, e, tauq, taup, qt, wt, idx, total;
};

SvdLayout svd_layout(int M, int N)
{
    SvdLayout L;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        size_t p = off;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    L.ws = take(std::max(bd_workspace_bytes(M, N), bdc_workspace_bytes(M, N)));
    L.e = take(sizeof(float) * N);
    L.tauq = take(sizeof(float) * N);
    L.taup = take(sizeof(float) * N);
    L.qt = take(sizeof(float) * 2 * nn);
    L.wt = take(sizeof(float) * 2 * nn);
    L.idx = take(sizeof(uint32_t) * 16 * (size_t)N);
    L.total = (off + 255) & ~(size_t)255;
    return L;
}

// QR-first layout (tall matrices): the N x N pipeline's layout first (its
// status block at offset 0 is the call's), then tau of the QR, R, U_R and the
// M x N stage-1 workspace that holds the QR factorization and the scratch of
// the products with M rows.
struct QrLayout {
    SvdLayout LR;
    size_t tau, ar, ur, bw, total;
};

QrLayout qr_layout(int M, int N)
{
    QrLayout Q;
    Q.LR = svd_layout(N, N);
    size_t off = Q.LR.total;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        size_t p = off;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    Q.tau = take(sizeof(float) * N);
    Q.ar = take(sizeof(float) * nn);
    Q.ur = take(sizeof(float) * nn);
    Q.bw = take(bd_workspace_bytes(M, N));
    Q.total = (off + 255) & ~(size_t)255;
    return Q;
}

// Shapes that may take the QR-first path (their workspace size covers it).
bool qr_possible(int M, int N) { return M > N && N >= 1024; }

// Two-stage path: the one-stage layout of (M, N) (its stage-1 workspace holds
// the band reduction, and is then reused by divide and conquer), the band and
// the chasing reflectors of both sides, sized for the widest band (64).
struct TsLayout {
    SvdLayout L;
    size_t band, rl, rr, total;
};

TsLayout ts_layout(int M, int N)
{
    TsLayout T;
    T.L = svd_layout(M, N);
    size_t off = T.L.total;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        size_t p = off;
        off += bytes;
        return p;
    };
    T.band = take(sizeof(float) * ts::band_floats(N, 64));
    T.rl = take(sizeof(float) * ts::refl_floats(N, 64));
    T.rr = take(sizeof(float) * ts::refl_floats(N, 64));
    T.total = (off + 255) & ~(size_t)255;
    return T;
}

// Shapes that may take the two-stage path (their workspace size covers it).
bool ts_possible(int M, int N) { return M >= N && N >= 1024; }

} // namespace

static unsigned long long g_launches = 0;
static int g_prof_on = 0;
void paco_count_launch() { g_launches++; }

int paco_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    return (dev >= 0 && dev < PACO_MAX_DEVICES) ? dev : 0;
}

// ------------------------------------------------ tiling autotuner state
// The reference fixes its tiling on the host (svd_tiling.cpp:11-66: one
// 1024^3 matmul tile and the leaf partition).  Here the shape-dependent
// choices of the single-matrix path are measured per (M, N) by
// paco_autotune and kept in a process-wide table; every later call of that
// shape reads its entry (other shapes use the defaults).  A change bumps a
// generation number so recorded CUDA graphs of older choices are re-recorded.
namespace {
struct TuneEntry {
    int M, N;
    PacoTune cfg;
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune;
unsigned g_tune_gen = 0;
const PacoTune kTuneDefault = {1, bd::RMIN_PER_BLOCK, 1, 0, 0, 0, 0, 0};

bool tune_valid(const PacoTune &t)
{
    return (t.persistent == 0 || t.persistent == 1) && (t.tc == 0 || t.tc == 1) && t.rows_per_cta >= 4 &&
           t.rows_per_cta <= 256 && (t.no_tail == 0 || t.no_tail == 1) && (t.wy == 0 || t.wy == 64 || t.wy == 128) &&
           (t.qb == 0 || t.qb == 32 || t.qb == 64) && t.mk >= 0 && t.mk <= PK_KMAX &&
           (t.ts == 0 || t.ts == 32 || t.ts == 64);
}

void tune_store(int M, int N, const PacoTune &cfg)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (TuneEntry &e : g_tune)
        if (e.M == M && e.N == N) {
            e.cfg = cfg;
            g_tune_gen++;
            return;
        }
    g_tune.push_back({M, N, cfg});
    g_tune_gen++;
}
}  // namespace

// QR-first choice per (M, N): 0 off, 1 on, 2 automatic (M >= 1.6 N), the default
namespace {
struct QrEntry {
    int M, N, mode;
};
std::vector<QrEntry> g_qr_modes;
}  // namespace

static int qr_mode_for(int M, int N)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const QrEntry &e : g_qr_modes)
        if (e.M == M && e.N == N) return e.mode;
    return 2;
}

static bool qr_chosen(int M, int N)
{
    if (!qr_possible(M, N)) return false;
    const int mode = qr_mode_for(M, N);
    if (mode == 0) return false;
    if (mode == 2 && (long)M * 10 < 16L * N) return false;
    return qr_fits(M, N);
}

PacoTune paco_tune_for(int M, int N)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const TuneEntry &e : g_tune)
        if (e.M == M && e.N == N) return e.cfg;
    return kTuneDefault;
}

// Two-stage reduction chosen for (M, N): the tuning entry's band width (0
// off, the default), a shape its workspace covers, and a band the chasing
// kernel holds.
static int ts_chosen(int M, int N)
{
    const int b = paco_tune_for(M, N).ts;
    return (b && ts_possible(M, N) && ts_fits(N, b)) ? b : 0;
}

// fills A with reproducible values uniform on [-1, 1) (a hash of the index)
__global__ void tune_fill(float *A, long n, unsigned seed)
{
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        unsigned x = (unsigned)t * 2654435761u ^ seed;
        x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
        A[t] = (float)(x >> 8) * (2.f / 16777216.f) - 1.f;
    }
}

__global__ void dev_status_begin(DevStatus *st, int stage)
{
    const int t = threadIdx.x;
    const bool keep = (stage == 2) && st->stage1_mark == PACO_STAGE1_MARK;
    __syncthreads();
    if (t < 60) st->counters[t] = 0;
    if (t == 0) {
        if (!keep) {
            st->code = 0;
            st->info = 0;
            st->secular_nonconv = 0;
            st->wait_timeouts = 0;
        }
        st->stage1_mark = (stage == 1) ? PACO_STAGE1_MARK : 0;
    }
}

extern "C" {

unsigned long long paco_launch_count(void) { return g_launches; }

// Byte offset, within the stage-1 workspace, of the phase timestamps written
// when PACO_PK_TRACE is set (a debugging aid; not part of the public header).
size_t paco_debug_trace_offset(int M, int N)
{
    BdWs w;
    char *base = (char *)(uintptr_t)(1u << 20); // any 256-byte aligned base
    bd_carve(base, M, N, &w);
    return (size_t)((char *)w.trace - base);
}

// Test hook (not part of the public header): one strided product
// C = alpha * opA * opB + beta * C on the SIMT engine (mode 0) or the tensor
// cores (mode 1; mode 2 keeps products without split-K off the persistent
// kernel), opA(m, k) = A[m * a_rs + k * a_cs], opB(k, n) = B[k * b_rs + n * b_cs].
// `ws` starts with the status block; the rest is GEMM scratch.  Synchronous.
size_t paco_debug_gemm_ws_bytes(int M, int N, int K)
{
    return 512 + sizeof(float) * std::max(gemm_tc_scratch_floats(M, N, K), (size_t)8 * M * N);
}

int paco_debug_gemm(int M, int N, int K, float alpha, const float *A, long a_rs, long a_cs, const float *B, long b_rs,
                    long b_cs, float beta, float *C, long ldc, int mode, void *ws, size_t ws_bytes, void *stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C || !ws || ws_bytes < paco_debug_gemm_ws_bytes(M, N, K))
        return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    DevStatus *st = (DevStatus *)ws;
    float *scr = (float *)((char *)ws + 512);
    bd_init_attrs();
    cudaMemsetAsync(st, 0, sizeof(DevStatus), s);
    cudaError_t err;
    if (mode == 1 || mode == 2) {  // 2: the one-tile-per-CTA kernel only
        const int prev = gemm_tc_set_persistent(mode == 1);
        err = gemm_tc_run(M, N, K, alpha, gop(A, a_rs, a_cs), gop(B, b_rs, b_cs), beta, C, ldc, scr, st, s);
        gemm_tc_set_persistent(prev);
    } else {
        err = gemm_run(M, N, K, alpha, gop(A, a_rs, a_cs), gop(B, b_rs, b_cs), beta, C, ldc,
                       std::min(8, std::max(1, K / 512)), scr, s);
    }
    if (err != cudaSuccess) return PACO_ERR_CUDA;
    return paco_sync_status(ws, stream, nullptr);
}

// Test hook (not part of the public header): byte offsets of the stage-1
// workspace fields, in the order of BdWs (st, W, Yt, X, ypart, tpart, cpart,
// rowbuf, inv_v0c, inv_v0r, sc, ctl, trace, bcA, bcB, Vp, T, gram, G1, G2,
// gscr, Vtmp, tcs), then the total; returns the number of values written.
int paco_debug_bd_layout(int M, int N, size_t out[24])
{
    BdWs w;
    char *base = (char *)(uintptr_t)(1u << 20);
    const size_t total = bd_carve(base, M, N, &w);
    const void *f[23] = {w.st, w.W, w.Yt, w.X, w.ypart, w.tpart, w.cpart, w.rowbuf, w.inv_v0c, w.inv_v0r, w.sc,
                         w.ctl, w.trace, w.bcA, w.bcB, w.Vp, w.T, w.gram, w.G1, w.G2, w.gscr, w.Vtmp, w.tcs};
    for (int k = 0; k < 23; k++) out[k] = f[k] ? (size_t)((const char *)f[k] - base) : total;
    out[23] = total;
    return 24;
}

// Test hook (not part of the public header): makes a bounded device-side
// wait run out and returns the status the library reports for it.
//   which 0: a tcgen05 kernel's mbarrier wait (one CTA holding tensor memory)
//   which 1: the persistent panel kernel's grid barrier (cooperative grid of
//            `ctas` CTAs whose barrier target is never reached)
// The waits give up after max_cycles SM cycles.  `ws` holds at least
// paco_debug_timeout_ws_bytes() bytes of device memory.  Synchronous.
size_t paco_debug_timeout_ws_bytes(void) { return 512 + sizeof(PkCtl); }

int paco_debug_wait_timeout(int which, long long max_cycles, int ctas, void *ws, void *stream)
{
    if (!ws || max_cycles <= 0 || (which != 0 && which != 1) || ctas < 1 || ctas > device_sms())
        return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    DevStatus *st = (DevStatus *)ws;
    PkCtl *ctl = (PkCtl *)((char *)ws + 512);
    if (cudaMemsetAsync(st, 0, sizeof(DevStatus), s) != cudaSuccess) return PACO_ERR_CUDA;
    const bool ok = which == 0 ? gemm_tc_debug_timeout(st, max_cycles, s)
                               : bd_pk_debug_timeout(ctl, st, ctas, max_cycles, s);
    if (!ok) {
        cudaGetLastError();
        return PACO_ERR_CUDA;
    }
    return paco_sync_status(ws, stream, nullptr);
}

// Test hook (not part of the public header): the iteration limit of the
// secular-equation solver (100 unless lowered; values below 1 restore it),
// for the single-matrix and the batched form.  Synchronous.
void paco_debug_secular_maxit(int n)
{
    if (n < 1) n = 100;
    bdc_set_sec_maxit(n);
    bt_set_sec_maxit(n);
}

const char *paco_version(void) { return "paco-svd-b200 1.0 (sm_100a)"; }

void paco_profile_enable(int on)
{
    g_prof_on = on != 0;
    bd_profile_enable(on);
}

void paco_profile_read(double out[4])
{
    if (out) bd_profile_read(out);
}

int getTilingSize(int N, int svdBlockNum)
{
    (void)svdBlockNum;
    if (N <= 0) return (int)sizeof(TilingHeader);
    return (int)sizeof(TilingHeader) + 8 * leaf_partition(N, nullptr, nullptr);
}

void GenerateTiling(int N, int blockDim, uint8_t *TilingHost)
{
    (void)blockDim;
    if (!TilingHost || N <= 0) return;
    TilingHeader h;
    memset(&h, 0, sizeof(h));
    h.magic = PACO_TILING_MAGIC;
    h.N = (uint32_t)N;
    h.nleaf = (uint32_t)leaf_partition(N, nullptr, nullptr);
    h.offset = sizeof(TilingHeader);
    h.version = 1;
    memcpy(TilingHost, &h, sizeof(h));
    int *s = (int *)malloc(sizeof(int) * h.nleaf), *e = (int *)malloc(sizeof(int) * h.nleaf);
    leaf_partition(N, s, e);
    uint32_t *lv = (uint32_t *)(TilingHost + sizeof(TilingHeader));
    for (uint32_t t = 0; t < h.nleaf; t++) { lv[2 * t] = (uint32_t)s[t]; lv[2 * t + 1] = (uint32_t)e[t]; }
    free(s);
    free(e);
}

size_t paco_workspace_size(int M, int N)
{
    if (!shape_ok(M, N)) return 0;
    return std::max(bd_workspace_bytes(M, N), bdc_workspace_bytes(M, N));
}

void paco_buffer_sizes(int M, int N, size_t out[12])
{
    if (!out) return;
    size_t m = M > 0 ? M : 0, n = N > 0 ? N : 0;
    out[0] = m * m * 4; out[1] = m * n * 4; out[2] = n * n * 4; out[3] = n * 4;
    out[4] = n > 0 ? (n - 1) * 4 : 0; out[5] = n * 4; out[6] = n > 0 ? (n - 1) * 4 : 0;
    out[7] = 2 * n * n * 4; out[8] = 2 * n * n * 4; out[9] = (size_t)getTilingSize(N, 1);
    out[10] = 16 * n * 4; out[11] = paco_workspace_size(M, N);
}

int upper_bidiagonalization(int M, int N, float *a, float *u, float *vt, float *d, float *e, float *tauq,
                            float *taup, void *workspace, void *stream)
{
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    if (!a || !u || !vt || !d || !tauq || !workspace || (N > 1 && (!e || !taup))) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    // a new factorization starts: clear and mark the device status block
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>((DevStatus *)workspace, 1);
    if (cudaGetLastError() != cudaSuccess) return PACO_ERR_CUDA;
    return bd_run(M, N, a, a, u, vt, d, e, tauq, taup, workspace, s, device_sms());
}

int svd_DC(int M, int N, float *a, float *u, float *vt, float *d, float *e, float *qt, float *wt, uint32_t *idx,
           void *workspace, const uint8_t *tiling, void *stream)
{
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    if (!a || !u || !vt || !d || !qt || !wt || !idx || !workspace || (N > 1 && !e)) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>((DevStatus *)workspace, 2);
    if (cudaGetLastError() != cudaSuccess) return PACO_ERR_CUDA;
    return bdc_run(M, N, a, u, vt, d, e, qt, wt, idx, workspace, tiling, s);
}

int paco_sync_status(void *workspace, void *stream, int *info)
{
    if (!workspace) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) {
        if (info) *info = (int)err;
        return PACO_ERR_CUDA;
    }
    DevStatus st;
    if (cudaMemcpy(&st, workspace, sizeof(int) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return PACO_ERR_CUDA;
    int zero[4] = {0, 0, 0, 0};
    cudaMemcpy(workspace, zero, sizeof(zero), cudaMemcpyHostToDevice);
    if (info) *info = st.code ? st.info : st.secular_nonconv;
    if (st.code) return st.code;
    if (st.secular_nonconv) return PACO_ERR_NONCONVERGENCE;
    return PACO_OK;
}

size_t paco_svd_workspace_size(int M, int N)
{
    if (!shape_ok(M, N)) return 0;
    size_t one = svd_layout(M, N).total;
    if (qr_possible(M, N)) one = std::max(one, qr_layout(M, N).total);
    if (ts_possible(M, N)) one = std::max(one, ts_layout(M, N).total);
    return one;
}

int paco_tune_qr(int M, int N, int mode)
{
    if (!shape_ok(M, N) || mode < -2 || mode > 2) return -1;
    if (mode == -1) return qr_mode_for(M, N);
    if (mode == -2) return qr_chosen(M, N) ? 1 : 0;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        bool found = false;
        for (QrEntry &e : g_qr_modes)
            if (e.M == M && e.N == N) { e.mode = mode; found = true; }
        if (!found) g_qr_modes.push_back({M, N, mode});
        g_tune_gen++;
    }
    return mode;
}

// QR-first SVD of a tall matrix: A = Q R, the one-matrix pipeline on R
// (N x N), then U = Q blockdiag(U_R, I).  A is read only.
static int svd_direct_qr(int M, int N, const float *A, float *U, float *Vt, float *sigma, char *b,
                         const QrLayout &Q, void *stream, bool thin = false)
{
    cudaStream_t s = (cudaStream_t)stream;
    const SvdLayout &L = Q.LR;
    DevStatus *st = (DevStatus *)(b + L.ws);
    float *e = (float *)(b + L.e), *tq = (float *)(b + L.tauq), *tp = (float *)(b + L.taup);
    float *tau = (float *)(b + Q.tau), *AR = (float *)(b + Q.ar), *UR = (float *)(b + Q.ur);
    BdWs wq;
    bd_carve(b + Q.bw, M, N, &wq);
    wq.st = st;  // the QR phase reports into the call's status block
    if (!paco_tune_for(M, N).tc) wq.tcs = nullptr;
    bd_init_attrs();
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 1);
    bd_copy_in_launch(A, wq.W, M, N, wq.ldw, st, s);
    const PacoTune tn = paco_tune_for(M, N);
    int rc = qr_factor(wq, M, N, tau, s, tn.qb);
    if (rc) return rc;
    qr_extract_r_launch(wq, N, AR, s);
    rc = bd_run(N, N, AR, AR, UR, Vt, sigma, e, tq, tp, b + L.ws, s, device_sms());
    if (rc) return rc;
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 2);
    rc = bdc_run(N, N, AR, UR, Vt, sigma, e, (float *)(b + L.qt), (float *)(b + L.wt), (uint32_t *)(b + L.idx),
                 b + L.ws, nullptr, s);
    if (rc) return rc;
    return qr_form_u(wq, M, N, tau, UR, U, s, thin ? N : M, tn.wy);
}

// Two-stage SVD: A -> band (bandwidth b) -> bidiagonal by bulge chasing,
// U = Q1 (formed) times the left chasing reflectors, Vt = the right chasing
// reflectors times P1^T, then divide and conquer updates both.  A is
// destroyed (scratch), as on the one-stage path.
static int svd_direct_ts(int M, int N, float *A, float *U, float *Vt, float *sigma, char *b, const TsLayout &T,
                         int bw, void *stream, bool thin)
{
    cudaStream_t s = (cudaStream_t)stream;
    const SvdLayout &L = T.L;
    float *e = (float *)(b + L.e), *tq = (float *)(b + L.tauq), *tp = (float *)(b + L.taup);
    float *rl = (float *)(b + T.rl), *rr = (float *)(b + T.rr);
    BdWs w;
    bd_carve(b + L.ws, M, N, &w);
    DevStatus *st = w.st;
    const PacoTune tn = paco_tune_for(M, N);
    if (!tn.tc) w.tcs = nullptr;
    bd_init_attrs();
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 1);
    bd_copy_in_launch(A, w.W, M, N, w.ldw, st, s);
    int rc = ts_band_reduce(w, M, N, bw, tq, tp, s);
    if (!rc) rc = ts_chase(w, N, bw, (float *)(b + T.band), rl, rr, sigma, e, s);
    const long lu = thin ? N : M;
    if (!rc) rc = qr_form_u(w, M, N, tq, nullptr, U, s, (int)lu, tn.wy);
    if (!rc) rc = ts_form_p1t(w, N, bw, tp, A, Vt, s);
    if (!rc) rc = ts_apply(U, lu, N, M, 1, bw, rl, st, s);
    if (!rc) rc = ts_apply(Vt, N, N, N, 0, bw, rr, st, s);
    if (rc) return rc;
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 2);
    return bdc_run(M, N, A, U, Vt, sigma, e, (float *)(b + L.qt), (float *)(b + L.wt), (uint32_t *)(b + L.idx),
                   b + L.ws, nullptr, s, lu);
}

// One-stage SVD with the thin U (M x N): stage 1 forms H_0 ... H_{N-1} [I; 0]
// only, and stage 2 updates those N columns.
static int svd_direct_thin(int M, int N, float *A, float *U, float *Vt, float *sigma, char *b, const SvdLayout &L,
                           void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    float *e = (float *)(b + L.e), *tq = (float *)(b + L.tauq), *tp = (float *)(b + L.taup);
    DevStatus *st = (DevStatus *)(b + L.ws);
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 1);
    BdJob job = {M, N, A, A, U, Vt, sigma, e, tq, tp, b + L.ws, 1};
    int rc = bd_run_multi(1, &job, s, nullptr, device_sms());
    if (rc) return rc;
    paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(st, 2);
    return bdc_run(M, N, A, U, Vt, sigma, e, (float *)(b + L.qt), (float *)(b + L.wt), (uint32_t *)(b + L.idx),
                   b + L.ws, nullptr, s, N);
}

// Test hook (not part of the public header): the QR-first path's R factor
// (N x N, ld N, zeros below the diagonal) of A (M x N, M > N, N >= 1024) and,
// when Qout is not null, Q (M x M) explicitly; ws holds
// paco_svd_workspace_size(M, N) bytes.  Synchronous.
extern "C" int paco_debug_qr_r(int M, int N, const float *A, float *R, float *Qout, void *ws, size_t ws_bytes,
                               void *stream)
{
    if (!shape_ok(M, N) || !qr_possible(M, N) || !qr_fits(M, N) || !A || !R || !ws ||
        ws_bytes < paco_svd_workspace_size(M, N))
        return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    char *b = (char *)ws;
    const QrLayout Q = qr_layout(M, N);
    DevStatus *st = (DevStatus *)(b + Q.LR.ws);
    BdWs wq;
    bd_carve(b + Q.bw, M, N, &wq);
    wq.st = st;
    bd_init_attrs();
    cudaMemsetAsync(st, 0, sizeof(DevStatus), s);
    bd_copy_in_launch(A, wq.W, M, N, wq.ldw, st, s);
    int rc = qr_factor(wq, M, N, (float *)(b + Q.tau), s);
    if (rc) return rc;
    qr_extract_r_launch(wq, N, R, s);
    if (Qout) rc = qr_form_u(wq, M, N, (float *)(b + Q.tau), nullptr, Qout, s);  // Q (M x M) explicitly
    if (rc) return rc;
    return paco_sync_status(ws, stream, nullptr);
}

// Test hook (not part of the public header): stages 1 and 2 of the two-stage
// reduction of A (M x N, N >= 1024) with band width b: band (N x 3b, row i =
// columns i - b .. i + 2b - 1 of the band matrix; may be null) and the
// bidiagonal d (N), e (N - 1).  ws holds paco_svd_workspace_size(M, N) bytes.
// Synchronous.
extern "C" int paco_debug_ts(int M, int N, int b, const float *A, float *band, float *d, float *e, void *ws,
                             size_t ws_bytes, void *stream)
{
    if (!shape_ok(M, N) || !ts_possible(M, N) || !ts_fits(N, b) || !A || !d || !e || !ws ||
        ws_bytes < paco_svd_workspace_size(M, N))
        return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    char *p = (char *)ws;
    const TsLayout T = ts_layout(M, N);
    BdWs w;
    bd_carve(p + T.L.ws, M, N, &w);
    bd_init_attrs();
    cudaMemsetAsync(w.st, 0, sizeof(DevStatus), s);
    bd_copy_in_launch(A, w.W, M, N, w.ldw, w.st, s);
    int rc = ts_band_reduce(w, M, N, b, (float *)(p + T.L.tauq), (float *)(p + T.L.taup), s);
    float *bandp = (float *)(p + T.band);
    if (!rc) rc = ts_chase(w, N, b, bandp, (float *)(p + T.rl), (float *)(p + T.rr), d, e, s);
    if (rc) return rc;
    if (band) cudaMemcpyAsync(band, bandp, sizeof(float) * ts::band_floats(N, b), cudaMemcpyDeviceToDevice, s);
    return paco_sync_status(p + T.L.ws, stream, nullptr);
}

static int svd_direct(int M, int N, float *A, float *U, float *Vt, float *sigma, char *b, const SvdLayout &L,
                      void *stream)
{
    float *e = (float *)(b + L.e), *tq = (float *)(b + L.tauq), *tp = (float *)(b + L.taup);
    int rc = upper_bidiagonalization(M, N, A, U, Vt, sigma, e, tq, tp, b + L.ws, stream);
    if (rc) return rc;
    return svd_DC(M, N, A, U, Vt, sigma, e, (float *)(b + L.qt), (float *)(b + L.wt), (uint32_t *)(b + L.idx),
                  b + L.ws, nullptr, stream);
}

// The single-matrix SVD in the configuration of (M, N): the two-stage
// reduction when its tuning entry asks for it, QR-first for tall matrices when
// chosen, otherwise the one-stage pipeline.  b holds
// paco_svd_workspace_size(M, N) bytes.
static int svd_any(int M, int N, float *A, float *U, float *Vt, float *sigma, char *b, void *stream,
                   bool thin = false)
{
    if (const int bw = ts_chosen(M, N)) return svd_direct_ts(M, N, A, U, Vt, sigma, b, ts_layout(M, N), bw, stream, thin);
    if (qr_chosen(M, N)) return svd_direct_qr(M, N, A, U, Vt, sigma, b, qr_layout(M, N), stream, thin);
    if (thin) return svd_direct_thin(M, N, A, U, Vt, sigma, b, svd_layout(M, N), stream);
    return svd_direct(M, N, A, U, Vt, sigma, b, svd_layout(M, N), stream);
}

// The one-shot paths issue thousands of small launches per SVD; on a
// capturable stream a call is recorded once into a CUDA graph per key (shape,
// buffers, stream, tuning generation, profiling state) and replayed with a
// single cudaGraphLaunch afterwards.  PACO_GRAPHS=0 in the environment turns
// this off.  The cache is shared by host threads under a lock.
}  // extern "C"

namespace {
struct GraphEntry {
    std::vector<uintptr_t> key;
    cudaStream_t s;
    int prof;
    unsigned tune_gen;  // autotuner generation the graph was recorded under
    cudaGraphExec_t exec;
    int prof_run;
    unsigned long long kernels; // kernel launches recorded into the graph
};
std::vector<GraphEntry> g_graphs;
std::mutex g_graphs_mu;
bool graphs_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *v = getenv("PACO_GRAPHS");
        on = !(v && v[0] == '0');
    }
    return on != 0;
}

// Runs direct() (which enqueues the work on s and returns a PACO_* status)
// through the graph cache.
template <class F>
int run_cached(const std::vector<uintptr_t> &key, cudaStream_t s, F &&direct)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!graphs_enabled() || s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread ||
        cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return direct();
    std::lock_guard<std::mutex> lock(g_graphs_mu);
    for (GraphEntry &g : g_graphs) {
        if (g.key == key && g.s == s && g.prof == g_prof_on && g.tune_gen == g_tune_gen) {
            if (cudaGraphLaunch(g.exec, s) != cudaSuccess) return PACO_ERR_CUDA;
            bd_profile_replayed(g.prof_run);
            g_launches += g.kernels;
            return PACO_OK;
        }
    }
    bd_init_attrs();
    bdc_init_attrs();
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return direct();
    }
    const unsigned long long k0 = g_launches;
    int rc = direct();
    const unsigned long long kernels = g_launches - k0;
    g_launches = k0; // recorded, not yet run
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamEndCapture(s, &graph);
    if (rc || err != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : direct();
    }
    GraphEntry g;
    g.key = key; g.s = s; g.prof = g_prof_on; g.tune_gen = g_tune_gen;
    g.prof_run = g_prof_on ? bd_profile_last_graph_run() : -1;
    g.kernels = kernels;
    err = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return direct();
    }
    if (g_graphs.size() >= 16) {
        cudaGraphExecDestroy(g_graphs.front().exec);
        g_graphs.erase(g_graphs.begin());
    }
    g_graphs.push_back(g);
    if (cudaGraphLaunch(g.exec, s) != cudaSuccess) return PACO_ERR_CUDA;
    bd_profile_replayed(g.prof_run);
    g_launches += g.kernels;
    return PACO_OK;
}
}  // namespace

extern "C" {

int paco_svd(int M, int N, float *A, float *U, float *Vt, float *sigma, void *ws, size_t ws_bytes, void *stream)
{
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    if (!A || !U || !Vt || !sigma || !ws) return PACO_ERR_INVALID_ARG;
    if (ws_bytes < paco_svd_workspace_size(M, N)) return PACO_ERR_INVALID_ARG;
    char *b = (char *)ws;
    const std::vector<uintptr_t> key = {1, (uintptr_t)M, (uintptr_t)N, (uintptr_t)A, (uintptr_t)U, (uintptr_t)Vt,
                                        (uintptr_t)sigma, (uintptr_t)ws};
    return run_cached(key, (cudaStream_t)stream, [&]() { return svd_any(M, N, A, U, Vt, sigma, b, stream); });
}

int paco_svd_thin(int M, int N, float *A, float *U, float *Vt, float *sigma, void *ws, size_t ws_bytes,
                  void *stream)
{
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    if (!A || !U || !Vt || !sigma || !ws) return PACO_ERR_INVALID_ARG;
    if (ws_bytes < paco_svd_workspace_size(M, N)) return PACO_ERR_INVALID_ARG;
    char *b = (char *)ws;
    const std::vector<uintptr_t> key = {3, (uintptr_t)M, (uintptr_t)N, (uintptr_t)A, (uintptr_t)U, (uintptr_t)Vt,
                                        (uintptr_t)sigma, (uintptr_t)ws};
    return run_cached(key, (cudaStream_t)stream,
                      [&]() { return svd_any(M, N, A, U, Vt, sigma, b, stream, true); });
}

// ------------------------------------------------ multi-matrix form
// k SVDs of one large shape share the GPU: stage 1 of a group of k matrices
// runs in lockstep (each persistent panel launch serves all k, num_sms / k
// CTAs per matrix, so the latency of one column step is paid once for k
// matrices), then the k divide-and-conquer runs proceed concurrently on side
// streams.  Groups of k follow one another.  A is read only.
}  // extern "C"

namespace {
int g_multi_k = 0;  // matrices per lockstep group; 0 = automatic
std::mutex g_side_mu;
cudaStream_t g_side[64][PK_KMAX];

// Side streams of the current device, created once (outside stream capture).
cudaStream_t *side_streams()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_side_mu);
    if (!g_side[dev][0])
        for (auto &st : g_side[dev])
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    return g_side[dev];
}

int multi_group(int count, int M, int N)
{
    const int tuned = paco_tune_for(M, N).mk;
    const int k = g_multi_k > 0 ? g_multi_k : (tuned > 0 ? tuned : 4);
    return std::max(1, std::min({count, k, PK_KMAX}));
}

struct MultiLayout {
    SvdLayout L;
    size_t a_off, per, total;
    int k;
};

MultiLayout multi_layout(int count, int M, int N)
{
    MultiLayout m;
    m.L = svd_layout(M, N);
    m.a_off = m.L.total;  // the M x N scratch that replaces A (A stays read only)
    m.per = (m.a_off + sizeof(float) * (size_t)M * N + 255) & ~(size_t)255;
    if (qr_possible(M, N)) m.per = std::max(m.per, qr_layout(M, N).total);  // QR-first reads A only
    m.k = multi_group(count, M, N);
    m.total = m.per * m.k;
    return m;
}

struct StatusPtrs {
    DevStatus *st[PK_KMAX];
    int idx[PK_KMAX];
    int k;
};

// status[idx[j]] <- the PACO_* code of matrix j's run; its status block is cleared
__global__ void multi_status_k(StatusPtrs p, int *status)
{
    const int j = threadIdx.x;
    if (j >= p.k) return;
    DevStatus *st = p.st[j];
    int c = st->code;
    if (!c && st->secular_nonconv) c = PACO_ERR_NONCONVERGENCE;
    if (status) status[p.idx[j]] = c;
    st->code = 0;
    st->info = 0;
    st->secular_nonconv = 0;
    st->wait_timeouts = 0;
}

// The multi-matrix form with the QR-first reduction: per group, the QR of
// every matrix on its own side stream, stage 1 of the k factors R in lockstep,
// then per matrix (side streams) divide and conquer and U = Q blockdiag(U_R, I).
int svd_multi_qr(int count, int M, int N, const float *const *A, float *const *U, float *const *Vt,
                 float *const *sigma, int *status, char *ws, const MultiLayout &ml, cudaStream_t s,
                 cudaStream_t *side)
{
    cudaEvent_t *fe = bd_fork_events();
    const QrLayout Q = qr_layout(M, N);
    const SvdLayout &L = Q.LR;
    const bool tc = paco_tune_for(M, N).tc != 0;
    auto fork = [&](int k) {
        cudaEventRecord(fe[0], s);
        for (int j = 0; j < k; j++) cudaStreamWaitEvent(side[j], fe[0], 0);
    };
    auto join = [&](int k) {
        for (int j = 0; j < k; j++) {
            cudaEventRecord(fe[1 + j], side[j]);
            cudaStreamWaitEvent(s, fe[1 + j], 0);
        }
    };
    for (int g0 = 0; g0 < count; g0 += ml.k) {
        const int k = std::min(ml.k, count - g0);
        BdJob jobs[PK_KMAX];
        BdWs wq[PK_KMAX];
        StatusPtrs sp;
        sp.k = k;
        int rc = PACO_OK;
        for (int j = 0; j < k; j++) {
            char *b = ws + (size_t)j * ml.per;
            sp.st[j] = (DevStatus *)(b + L.ws);
            sp.idx[j] = g0 + j;
            paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(sp.st[j], 1);
            bd_carve(b + Q.bw, M, N, &wq[j]);
            wq[j].st = sp.st[j];
            if (!tc) wq[j].tcs = nullptr;
            float *AR = (float *)(b + Q.ar);
            jobs[j] = {N, N, AR, AR, (float *)(b + Q.ur), Vt[g0 + j], sigma[g0 + j], (float *)(b + L.e),
                       (float *)(b + L.tauq), (float *)(b + L.taup), b + L.ws};
        }
        fork(k);
        for (int j = 0; j < k && !rc; j++) {
            char *b = ws + (size_t)j * ml.per;
            bd_copy_in_launch(A[g0 + j], wq[j].W, M, N, wq[j].ldw, sp.st[j], side[j]);
            rc = qr_factor(wq[j], M, N, (float *)(b + Q.tau), side[j], paco_tune_for(M, N).qb);
            qr_extract_r_launch(wq[j], N, (float *)(b + Q.ar), side[j]);
        }
        join(k);
        if (rc) return rc;
        rc = bd_run_multi(k, jobs, s, side, device_sms());
        if (rc) return rc;
        fork(k);
        for (int j = 0; j < k && !rc; j++) {
            char *b = ws + (size_t)j * ml.per;
            paco_count_launch(), dev_status_begin<<<1, 64, 0, side[j]>>>(sp.st[j], 2);
            rc = bdc_run(N, N, jobs[j].a_out, jobs[j].u, Vt[g0 + j], sigma[g0 + j], jobs[j].e, (float *)(b + L.qt),
                         (float *)(b + L.wt), (uint32_t *)(b + L.idx), b + L.ws, nullptr, side[j]);
            if (!rc)
                rc = qr_form_u(wq[j], M, N, (float *)(b + Q.tau), jobs[j].u, U[g0 + j], side[j], M,
                               paco_tune_for(M, N).wy);
        }
        join(k);
        if (rc) return rc;
        paco_count_launch(), multi_status_k<<<1, 32, 0, s>>>(sp, status);
    }
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}

int svd_multi_direct(int count, int M, int N, const float *const *A, float *const *U, float *const *Vt,
                     float *const *sigma, int *status, char *ws, const MultiLayout &ml, cudaStream_t s)
{
    cudaStream_t *side = side_streams();
    if (!side) return PACO_ERR_CUDA;
    // kernel attributes before the first launch (the QR path's products come
    // before stage 1, which would set them otherwise)
    bd_init_attrs();
    bdc_init_attrs();
    cudaEvent_t *fe = bd_fork_events();
    const SvdLayout &L = ml.L;
    if (qr_chosen(M, N)) return svd_multi_qr(count, M, N, A, U, Vt, sigma, status, ws, ml, s, side);
    for (int g0 = 0; g0 < count; g0 += ml.k) {
        const int k = std::min(ml.k, count - g0);
        BdJob jobs[PK_KMAX];
        StatusPtrs sp;
        sp.k = k;
        for (int j = 0; j < k; j++) {
            char *b = ws + (size_t)j * ml.per;
            float *a = (float *)(b + ml.a_off);
            jobs[j] = {M, N, A[g0 + j], a, U[g0 + j], Vt[g0 + j], sigma[g0 + j], (float *)(b + L.e),
                       (float *)(b + L.tauq), (float *)(b + L.taup), b + L.ws};
            sp.st[j] = (DevStatus *)(b + L.ws);
            sp.idx[j] = g0 + j;
            paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(sp.st[j], 1);
        }
        int rc = bd_run_multi(k, jobs, s, side, device_sms());
        if (rc) return rc;
        if (k == 1) {
            paco_count_launch(), dev_status_begin<<<1, 64, 0, s>>>(sp.st[0], 2);
            char *b = ws;
            rc = bdc_run(M, N, jobs[0].a_out, U[g0], Vt[g0], sigma[g0], jobs[0].e, (float *)(b + L.qt),
                         (float *)(b + L.wt), (uint32_t *)(b + L.idx), b + L.ws, nullptr, s);
        } else {
            cudaEventRecord(fe[0], s);
            for (int j = 0; j < k && !rc; j++) {
                char *b = ws + (size_t)j * ml.per;
                cudaStreamWaitEvent(side[j], fe[0], 0);
                paco_count_launch(), dev_status_begin<<<1, 64, 0, side[j]>>>(sp.st[j], 2);
                rc = bdc_run(M, N, jobs[j].a_out, U[g0 + j], Vt[g0 + j], sigma[g0 + j], jobs[j].e,
                             (float *)(b + L.qt), (float *)(b + L.wt), (uint32_t *)(b + L.idx), b + L.ws, nullptr,
                             side[j]);
            }
            for (int j = 0; j < k; j++) {
                cudaEventRecord(fe[1 + j], side[j]);
                cudaStreamWaitEvent(s, fe[1 + j], 0);
            }
        }
        if (rc) return rc;
        paco_count_launch(), multi_status_k<<<1, 32, 0, s>>>(sp, status);
    }
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
}  // namespace

extern "C" {

size_t paco_svd_multi_workspace_size(int count, int M, int N)
{
    if (count < 1 || !shape_ok(M, N)) return 0;
    return multi_layout(count, M, N).total;
}

int paco_multi_group(int k)
{
    const int prev = g_multi_k;
    if (k >= 0 && k <= PK_KMAX) g_multi_k = k;
    return prev;
}

int paco_svd_multi(int count, int M, int N, const float *const *A, float *const *U, float *const *Vt,
                   float *const *sigma, int *status, void *workspace, size_t ws_bytes, void *stream)
{
    if (count < 1 || !A || !U || !Vt || !sigma || !workspace) return PACO_ERR_INVALID_ARG;
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    for (int b = 0; b < count; b++)
        if (!A[b] || !U[b] || !Vt[b] || !sigma[b]) return PACO_ERR_INVALID_ARG;
    const MultiLayout ml = multi_layout(count, M, N);
    if (ws_bytes < ml.total) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (!side_streams()) return PACO_ERR_CUDA;
    std::vector<uintptr_t> key = {2, (uintptr_t)count, (uintptr_t)M, (uintptr_t)N, (uintptr_t)ml.k,
                                  (uintptr_t)workspace, (uintptr_t)status};
    for (int b = 0; b < count; b++) {
        key.push_back((uintptr_t)A[b]);
        key.push_back((uintptr_t)U[b]);
        key.push_back((uintptr_t)Vt[b]);
        key.push_back((uintptr_t)sigma[b]);
    }
    return run_cached(key, s, [&]() {
        return svd_multi_direct(count, M, N, A, U, Vt, sigma, status, (char *)workspace, ml, s);
    });
}

// ------------------------------------------------ tiling autotuner

int paco_tune_get(int M, int N, int cfg[4])
{
    if (!cfg) return PACO_ERR_INVALID_ARG;
    const PacoTune t = paco_tune_for(M, N);
    cfg[0] = t.persistent; cfg[1] = t.rows_per_cta; cfg[2] = t.tc; cfg[3] = t.no_tail;
    return PACO_OK;
}

int paco_tune_set(int M, int N, const int cfg[4])
{
    if (!cfg || !shape_ok(M, N)) return PACO_ERR_INVALID_ARG;
    PacoTune t = paco_tune_for(M, N);  // the tile-shape fields stay as they are
    t.persistent = cfg[0]; t.rows_per_cta = cfg[1]; t.tc = cfg[2]; t.no_tail = cfg[3];
    if (!tune_valid(t)) return PACO_ERR_INVALID_ARG;
    tune_store(M, N, t);
    return PACO_OK;
}

int paco_tune_param(int M, int N, int which, int value)
{
    if (!shape_ok(M, N) || which < 0 || which > 8) return -1;
    if (which == 7) return paco_tune_qr(M, N, value);
    PacoTune t = paco_tune_for(M, N);
    int *f[9] = {&t.persistent, &t.rows_per_cta, &t.tc, &t.no_tail, &t.wy, &t.qb, &t.mk, nullptr, &t.ts};
    if (value == -1) return *f[which];
    *f[which] = value;
    if (!tune_valid(t)) return -1;
    tune_store(M, N, t);
    return value;
}

int paco_autotune_multi(int count, int M, int N, void *stream, double out[4])
{
    if (count < 2 || !shape_ok(M, N)) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int prev_global = g_multi_k;
    g_multi_k = 0;  // the per-shape entry decides during the trials
    PacoTune t0 = paco_tune_for(M, N);
    size_t wsb = 0;
    const int ks[] = {2, 4, 8};
    for (int k : ks) {
        PacoTune c = t0;
        c.mk = k;
        tune_store(M, N, c);
        wsb = std::max(wsb, multi_layout(count, M, N).total);
    }
    std::vector<float *> A(count, nullptr), U(count, nullptr), Vt(count, nullptr), sg(count, nullptr);
    char *ws = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaSuccess;
    for (int b = 0; b < count && !err; b++) {
        err = cudaMalloc(&A[b], sizeof(float) * (size_t)M * N);
        err = err ? err : cudaMalloc(&U[b], sizeof(float) * (size_t)M * M);
        err = err ? err : cudaMalloc(&Vt[b], sizeof(float) * (size_t)N * N);
        err = err ? err : cudaMalloc(&sg[b], sizeof(float) * N);
    }
    err = err ? err : cudaMalloc(&ws, wsb);
    err = err ? err : cudaEventCreate(&e0);
    err = err ? err : cudaEventCreate(&e1);
    int rc = err ? PACO_ERR_CUDA : PACO_OK;
    float best = 1e30f, first = 0.f;
    int bk = t0.mk > 0 ? t0.mk : 4, tried = 0;
    for (int b = 0; b < count && !rc; b++)
        paco_count_launch(), tune_fill<<<std::min(4096, ceil_div((long)M * N, 256)), 256, 0, s>>>(A[b], (long)M * N,
                                                                                                   777u + b);
    for (int k : ks) {
        if (rc || k > count) break;
        PacoTune c = t0;
        c.mk = k;
        tune_store(M, N, c);
        const MultiLayout ml = multi_layout(count, M, N);
        float tk = 1e30f;
        for (int rep = 0; rep < 2 && !rc; rep++) {
            cudaEventRecord(e0, s);
            int r = svd_multi_direct(count, M, N, A.data(), U.data(), Vt.data(), sg.data(), nullptr, ws, ml, s);
            cudaEventRecord(e1, s);
            if (r || cudaEventSynchronize(e1) != cudaSuccess) { rc = r ? r : PACO_ERR_CUDA; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tk = ms;  // the first run warms up
        }
        tried++;
        if (k == ks[0]) first = tk;
        if (tk < best) { best = tk; bk = k; }
    }
    PacoTune c = t0;
    c.mk = rc ? t0.mk : bk;
    tune_store(M, N, c);
    // the QR-first choice of the single-matrix tuning may not suit k matrices
    // in lockstep (their R factors stream less): time the other choice too
    if (!rc && qr_possible(M, N) && qr_fits(M, N)) {
        const int mode = qr_mode_for(M, N);
        const bool on = qr_chosen(M, N);
        paco_tune_qr(M, N, on ? 0 : 1);
        const MultiLayout ml = multi_layout(count, M, N);
        float tq = 1e30f;
        if (ml.total <= wsb) {
            for (int rep = 0; rep < 2 && !rc; rep++) {
                cudaEventRecord(e0, s);
                int r = svd_multi_direct(count, M, N, A.data(), U.data(), Vt.data(), sg.data(), nullptr, ws, ml, s);
                cudaEventRecord(e1, s);
                if (r || cudaEventSynchronize(e1) != cudaSuccess) { rc = r ? r : PACO_ERR_CUDA; break; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) tq = ms;
            }
            tried++;
        }
        if (!rc && tq < best) best = tq;
        else paco_tune_qr(M, N, mode);
    }
    g_multi_k = prev_global;
    if (out) { out[0] = bk; out[1] = best; out[2] = first; out[3] = tried; }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    for (int b = 0; b < count; b++) { cudaFree(A[b]); cudaFree(U[b]); cudaFree(Vt[b]); cudaFree(sg[b]); }
    cudaFree(ws);
    return rc;
}

int paco_autotune(int M, int N, void *stream, double out[4])
{
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t wsb = paco_svd_workspace_size(M, N);
    float *A0 = nullptr, *A = nullptr, *U = nullptr, *Vt = nullptr, *sg = nullptr;
    char *ws = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaSuccess;
    err = err ? err : cudaMalloc(&A0, sizeof(float) * (size_t)M * N);
    err = err ? err : cudaMalloc(&A, sizeof(float) * (size_t)M * N);
    err = err ? err : cudaMalloc(&U, sizeof(float) * (size_t)M * M);
    err = err ? err : cudaMalloc(&Vt, sizeof(float) * (size_t)N * N);
    err = err ? err : cudaMalloc(&sg, sizeof(float) * N);
    err = err ? err : cudaMalloc(&ws, wsb);
    err = err ? err : cudaEventCreate(&e0);
    err = err ? err : cudaEventCreate(&e1);
    int rc = err ? PACO_ERR_CUDA : PACO_OK;
    // candidates: the defaults first, then fewer / more rows per CTA, the
    // SIMT engine for the large products, the two-kernel row/column passes,
    // the last columns on the panel kernel; for tall shapes the best of them
    // is then also timed with the QR-first choice flipped, then with 64-
    // reflector WY blocks, the two-stage reduction (bands 32 and 64) and
    // 32-column QR blocks
    PacoTune cands[] = {{1, bd::RMIN_PER_BLOCK, 1, 0}, {1, 8, 1, 0}, {1, 32, 1, 0}, {1, bd::RMIN_PER_BLOCK, 0, 0},
                        {0, bd::RMIN_PER_BLOCK, 1, 0}, {1, bd::RMIN_PER_BLOCK, 1, 1}};
    const int mk0 = paco_tune_for(M, N).mk;  // the multi-matrix group size is tuned separately
    for (PacoTune &c : cands) c.mk = mk0;
    const int nc = (int)(sizeof(cands) / sizeof(cands[0]));
    float best = 1e30f, tdef = 0.f;
    int bi = 0, tried = 0;
    auto time_one = [&]() {
        float tk = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            cudaMemcpyAsync(A, A0, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToDevice, s);
            cudaEventRecord(e0, s);
            int r = svd_any(M, N, A, U, Vt, sg, ws, stream);
            cudaEventRecord(e1, s);
            if (r || cudaEventSynchronize(e1) != cudaSuccess) { rc = r ? r : PACO_ERR_CUDA; break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tk = std::min(tk, ms);  // the first run warms up
        }
        int info = 0;
        if (!rc && paco_sync_status(ws, stream, &info) != PACO_OK) tk = 1e30f;  // not a usable choice
        tried++;
        return tk;
    };
    if (!rc) {
        paco_count_launch(), tune_fill<<<std::min(4096, ceil_div((long)M * N, 256)), 256, 0, s>>>(A0, (long)M * N,
                                                                                                   12345u);
        for (int k = 0; k < nc && !rc; k++) {
            tune_store(M, N, cands[k]);
            const float tk = time_one();
            if (k == 0) tdef = tk;
            if (tk < best) { best = tk; bi = k; }
        }
        tune_store(M, N, cands[bi]);
        if (!rc && qr_possible(M, N) && qr_fits(M, N)) {
            const int mode = qr_mode_for(M, N);
            const bool on = qr_chosen(M, N);
            paco_tune_qr(M, N, on ? 0 : 1);
            const float tq = time_one();
            if (!rc && tq < best) best = tq;
            else paco_tune_qr(M, N, mode);
        }
        // tile shapes of the blocked products: 64-reflector WY blocks, 32-column QR blocks
        PacoTune t = paco_tune_for(M, N);
        const int wy_sizes[] = {64};
        for (int wy : wy_sizes) {
            if (rc) break;
            PacoTune c = t;
            c.wy = wy;
            tune_store(M, N, c);
            const float tw = time_one();
            if (!rc && tw < best) { best = tw; t = c; }
            else tune_store(M, N, t);
        }
        // the two-stage reduction, band 32 and 64
        for (int bwid : {32, 64}) {
            if (rc || !ts_possible(M, N) || !ts_fits(N, bwid)) continue;
            PacoTune c = t;
            c.ts = bwid;
            tune_store(M, N, c);
            const float tt = time_one();
            if (!rc && tt < best) { best = tt; t = c; }
            else tune_store(M, N, t);
        }
        if (!rc && !t.ts && qr_chosen(M, N)) {
            PacoTune c = t;
            c.qb = 32;
            tune_store(M, N, c);
            const float tb = time_one();
            if (!rc && tb < best) { best = tb; t = c; }
            else tune_store(M, N, t);
        }
    }
    if (out) { out[0] = bi; out[1] = best; out[2] = tdef; out[3] = tried; }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(A0); cudaFree(A); cudaFree(U); cudaFree(Vt); cudaFree(sg); cudaFree(ws);
    return rc;
}

// ------------------------------------------------ allocation-free entry point
// Scratch of paco_svd_noalloc: a file-scope device array, so the entry point
// needs no cudaMalloc.  It is part of the loaded module, so every GPU that
// loads the library holds these bytes until the process exits.
#define PACO_NOALLOC_MAX_M 1024
#define PACO_NOALLOC_MAX_N 512
#define PACO_NOALLOC_BYTES (16u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[PACO_NOALLOC_BYTES];

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_addr[64]; // device address of the array, per device ordinal
}  // namespace

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name only stands in for the symbol, so the address is looked up
// once per device, with that device current, and cached.
static int noalloc_scratch(void **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PACO_ERR_CUDA;
    if (dev < 0 || dev >= 64) return PACO_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return PACO_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return PACO_OK;
}

int paco_svd_noalloc(int M, int N, float *A, float *U, float *Vt, float *sigma, void *stream)
{
    if (N < 1 || M < N) return PACO_ERR_INVALID_ARG;
    if (M > PACO_NOALLOC_MAX_M || N > PACO_NOALLOC_MAX_N) return PACO_ERR_UNSUPPORTED;
    if (!A || !U || !Vt || !sigma) return PACO_ERR_INVALID_ARG;
    // the call ends by synchronizing the stream, which a stream capture forbids
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t)stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        return PACO_ERR_INVALID_ARG;
    }
    if (cs != cudaStreamCaptureStatusNone) return PACO_ERR_INVALID_ARG;
    SvdLayout L = svd_layout(M, N);
    if (L.total > PACO_NOALLOC_BYTES) return PACO_ERR_UNSUPPORTED;
    void *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // the status block and counters at the start of the scratch are cleared by
    // the stages themselves; everything else is written before it is read
    rc = svd_direct(M, N, A, U, Vt, sigma, (char *)scratch, L, stream);
    if (rc) return rc;
    int info = 0;
    return paco_sync_status((char *)scratch + L.ws, stream, &info);
}

struct paco_ctx {
    int M, N;
    float *A, *U, *Vt, *sigma;
    void *ws;
    size_t ws_bytes;
    cudaStream_t stream;
};

int paco_ctx_create(int M, int N, paco_ctx **out)
{
    if (!out) return PACO_ERR_INVALID_ARG;
    *out = nullptr;
    if (!shape_ok(M, N)) return (N >= 1 && M >= N) ? PACO_ERR_UNSUPPORTED : PACO_ERR_INVALID_ARG;
    paco_ctx *c = (paco_ctx *)calloc(1, sizeof(paco_ctx));
    c->M = M; c->N = N;
    c->ws_bytes = paco_svd_workspace_size(M, N);
    cudaError_t err = cudaSuccess;
    err = err ? err : cudaMalloc(&c->A, sizeof(float) * (size_t)M * N);
    err = err ? err : cudaMalloc(&c->U, sizeof(float) * (size_t)M * M);
    err = err ? err : cudaMalloc(&c->Vt, sizeof(float) * (size_t)N * N);
    err = err ? err : cudaMalloc(&c->sigma, sizeof(float) * N);
    err = err ? err : cudaMalloc(&c->ws, c->ws_bytes);
    err = err ? err : cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        paco_ctx_destroy(c);
        return PACO_ERR_CUDA;
    }
    *out = c;
    return PACO_OK;
}

int paco_ctx_svd_host(paco_ctx *c, const float *A, float *U, float *Vt, float *sigma)
{
    if (!c || !A) return PACO_ERR_INVALID_ARG;
    const int M = c->M, N = c->N;
    cudaStream_t s = c->stream;
    if (cudaMemcpyAsync(c->A, A, sizeof(float) * (size_t)M * N, cudaMemcpyHostToDevice, s)) return PACO_ERR_CUDA;
    int rc = paco_svd(M, N, c->A, c->U, c->Vt, c->sigma, c->ws, c->ws_bytes, s);
    if (rc) return rc;
    if (U && cudaMemcpyAsync(U, c->U, sizeof(float) * (size_t)M * M, cudaMemcpyDeviceToHost, s)) return PACO_ERR_CUDA;
    if (Vt && cudaMemcpyAsync(Vt, c->Vt, sizeof(float) * (size_t)N * N, cudaMemcpyDeviceToHost, s))
        return PACO_ERR_CUDA;
    if (sigma && cudaMemcpyAsync(sigma, c->sigma, sizeof(float) * N, cudaMemcpyDeviceToHost, s)) return PACO_ERR_CUDA;
    SvdLayout L = svd_layout(M, N);
    int info = 0;
    return paco_sync_status((char *)c->ws + L.ws, s, &info);
}

void paco_ctx_destroy(paco_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->A); cudaFree(c->U); cudaFree(c->Vt); cudaFree(c->sigma); cudaFree(c->ws);
    if (c->stream) cudaStreamDestroy(c->stream);
    free(c);
}

} // extern "C"
