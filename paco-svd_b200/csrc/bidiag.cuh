// Stage-1 (bidiagonalization) constants, kernel arguments and workspace layout.
#pragma once

#include "common.cuh"
#include "gemm_tc.cuh"

namespace bd {
constexpr int NB = 32;             // panel width (reflectors per block update)
constexpr int RP_THREADS = 512;    // row-pass CTA size
constexpr int CP_THREADS = 256;    // column-pass CTA size (32 columns x 8 warps)
constexpr int RMAX = 8;            // max rows staged per TMA batch
constexpr int RB_CAP = 256;        // max row-pass CTAs (partial records)
constexpr int CB_CAP = 512;        // max column-pass CTAs (N/32)
constexpr int PR = 2 * NB + 8;     // floats per partial record
constexpr int RMIN_PER_BLOCK = 16; // rows per CTA of a panel unless the autotuner chose otherwise
constexpr int SPLITS = 8;          // split-K factor cap for the skinny V^T Q products
constexpr int PCAP = 512;          // CTA slots of a partial record (>= RB_CAP, CB_CAP)
constexpr int NBF = 128;           // reflectors per block update when U and V are formed
}  // namespace bd

struct StepScal {
    float t1[bd::NB];     // V_panel^T v        (column step)
    float t2[bd::NB];     // X_panel^T v
    float t3[bd::NB + 1]; // Y_panel^T u        (row step)
    float t4[bd::NB];     // U_panel u
    float x0col, x0row;   // pivots of the current reflectors
    float pad[5];
};

// Control words of the persistent panel kernel's grid barrier.
struct PkCtl {
    unsigned cnt;   // CTAs arrived at the current barrier
    unsigned gen;   // barrier generation, bumped by the last CTA
    unsigned abort; // set by a CTA whose bounded wait gave up
    unsigned pad[29];
};

struct BdArgs {
    int M, N;
    long ldw;
    DevStatus *st;
    float *W, *Yt, *X, *ypart, *tpart, *cpart, *rowbuf, *inv_v0c, *inv_v0r;
    StepScal *sc;
    float *d, *e, *tauq, *taup;
    unsigned long long *trace; // phase timestamps of one traced panel (or null)
    int trace_p0;
    float *bcA, *bcB; // broadcast slots of the persistent kernel's reflectors
};

// Arguments of one launch of the persistent panel kernel: the same panel of
// up to PK_KMAX matrices of one shape, G CTAs (and one barrier) per matrix.
constexpr int PK_KMAX = 8;
struct PkMulti {
    BdArgs a[PK_KMAX];
    PkCtl *ctl[PK_KMAX];
    unsigned cnt_base[PK_KMAX];  // barrier counter of each matrix before the launch
    int G;
};

struct BdWs {
    DevStatus *st;
    long ldw;
    float *W;      // M x ldw   working copy of A (row stride padded to 32 floats)
    float *Yt;     // NB x ldw  Y^T of the current panel
    float *X;      // M x NB    X of the current panel
    float *ypart;  // RB_CAP x ldw  per-CTA partial A^T x
    float *tpart;  // PR x PCAP, value-major: tpart[t * PCAP + cta]
    float *cpart;  // PR x PCAP
    float *rowbuf; // ldw       updated pivot row
    float *inv_v0c, *inv_v0r; // N each: 1/v0 of every reflector
    StepScal *sc;
    PkCtl *ctl;
    unsigned long long *trace; // NB+1 steps x 16 slots x 2 CTAs
    float *bcA, *bcB;          // PR each: pivot and panel entries of a reflector
    float *Vp;     // max(M,N) x NBF explicit reflector block (formation of U, V)
    float *T;      // NBF x NBF
    float *gram;   // NBF x NBF  Vp^T Vp
    float *G1, *G2;// NBF x max(M,N)
    float *gscr;   // SPLITS x NBF x max(M,N)  split-K partial products
    float *Vtmp;   // N x N  (V before the transpose into vt)
    float *tcs;    // tensor-core GEMM scratch (operand images, split-K partials); null when unused
    size_t tcs_floats;
};

// Lays the stage-1 buffers out in `base` (may be null to only measure);
// returns the bytes used.  The DevStatus block comes first.
static inline size_t bd_carve(void *base, int M, int N, BdWs *w)
{
    using namespace bd;
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = (off + 255) & ~(size_t)255;
        char *p = base ? (char *)base + off : nullptr;
        off += bytes;
        return p;
    };
    const long ldw = round_up(N, 32);
    const long mx = std::max(M, N);
    w->ldw = ldw;
    w->st = (DevStatus *)take(sizeof(DevStatus));
    w->W = (float *)take(sizeof(float) * (size_t)M * ldw);
    w->Yt = (float *)take(sizeof(float) * (size_t)NB * ldw);
    w->X = (float *)take(sizeof(float) * (size_t)M * NB);
    w->ypart = (float *)take(sizeof(float) * (size_t)RB_CAP * ldw);
    w->tpart = (float *)take(sizeof(float) * (size_t)PCAP * PR);
    w->cpart = (float *)take(sizeof(float) * (size_t)PCAP * PR);
    w->rowbuf = (float *)take(sizeof(float) * ldw);
    w->inv_v0c = (float *)take(sizeof(float) * N);
    w->inv_v0r = (float *)take(sizeof(float) * N);
    w->sc = (StepScal *)take(sizeof(StepScal));
    w->ctl = (PkCtl *)take(sizeof(PkCtl));
    w->trace = (unsigned long long *)take(sizeof(unsigned long long) * (NB + 1) * 16 * 2);
    w->bcA = (float *)take(sizeof(float) * PR);
    w->bcB = (float *)take(sizeof(float) * PR);
    w->Vp = (float *)take(sizeof(float) * (size_t)mx * NBF);
    w->T = (float *)take(sizeof(float) * NBF * NBF);
    w->gram = (float *)take(sizeof(float) * NBF * NBF);
    w->G1 = (float *)take(sizeof(float) * (size_t)NBF * mx);
    w->G2 = (float *)take(sizeof(float) * (size_t)NBF * mx);
    w->gscr = (float *)take(sizeof(float) * (size_t)SPLITS * NBF * mx);
    w->Vtmp = (float *)take(sizeof(float) * (size_t)N * N);
    // products sent to the tensor cores: G1 = Vp^T Q, G2 = T G1, Q -= Vp G2 and
    // the panel trailing update (matrices up to 1024 stay on the SIMT engine)
    const int shapes[4][3] = {{NBF, (int)mx, (int)mx}, {NBF, (int)mx, NBF}, {(int)mx, (int)mx, NBF}, {M, N, 2 * NB}};
    w->tcs_floats = mx > 1024 ? gemm_tc_scratch_for(shapes, 4) : 0;
    w->tcs = w->tcs_floats ? (float *)take(sizeof(float) * w->tcs_floats) : nullptr;
    return (off + 255) & ~(size_t)255;
}

// reflector of upper_bidiagonalization.cpp:182-218 from x0 and sigma = |x[1:]|^2
static __device__ __forceinline__ void make_reflector(float x0, float sigma, int len, float *beta, float *tau,
                                                      float *v0)
{
    if (len <= 1 || sigma == 0.f) {
        *beta = x0; *tau = 0.f; *v0 = 1.f;
        return;
    }
    float mu = sqrtf(x0 * x0 + sigma);
    float v = (x0 <= 0.f) ? x0 - mu : -sigma / (x0 + mu);
    *v0 = v;
    *tau = 2.f * v * v / (sigma + v * v);
    *beta = mu;
}

// Sums the per-CTA partial records rec[t * PCAP + cta] (cta < ncta) into
// out[t] for t < nval: one warp per value, all CTA slots loaded at once,
// summed in a fixed order.  Called by every thread of the CTA.
static __device__ __forceinline__ void reduce_records(const float *rec, int ncta, int nval, float *out)
{
    using namespace bd;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int t = warp; t < nval; t += nw) {
        float v[PCAP / 32];
#pragma unroll
        for (int k = 0; k < PCAP / 32; k++) {
            int c = lane + 32 * k;
            v[k] = (c < ncta) ? __ldcg(&rec[(long)t * PCAP + c]) : 0.f;
        }
        float sum = 0.f;
#pragma unroll
        for (int k = 0; k < PCAP / 32; k++) sum += v[k];
        sum = warp_sum(sum);
        if (lane == 0) out[t] = sum;
    }
    __syncthreads();
}

bool bd_panel_pk_launch(const BdArgs &a, PkCtl *ctl, int p0, int p1, int G, unsigned *cnt, cudaStream_t s);
bool bd_panel_pk_launch_multi(int k, const BdArgs *a, PkCtl *const *ctl, int p0, int p1, int G, unsigned *cnt,
                              cudaStream_t s);
// Test hook: a cooperative launch of G CTAs whose grid barrier never
// completes; its bounded waits give up after max_cycles.
bool bd_pk_debug_timeout(PkCtl *ctl, DevStatus *st, int G, long long max_cycles, cudaStream_t s);
// Cluster kernel for the last columns: its set-up (once, outside stream
// capture), the first panel boundary p from which the block A[p:, p:] goes to
// it (N when it never does), and that launch (false: not possible, the panels
// continue).
void bd_tail_init();
int bd_tail_start(int M, int N);
bool bd_tail_launch(const BdArgs &a, int p, cudaStream_t s);
void bd_pk_init_attrs();

size_t bd_workspace_bytes(int M, int N);
// Q[ro:ro+Lr, co:co+Lc] <- (I - Vp T' Vp^T) Q[...] with T' = T, or T^T when
// transT, for the nbp reflectors in w.Vp (T built from their Gram matrix).
cudaError_t apply_block_reflector_ex(const BdWs &w, float *Q, long ldq, long ro, int Lr, long co, int Lc, int nbp,
                                     const float *tau, bool transT, cudaStream_t s);
// X[ro:ro+Lr, co:co+Lc] <- X[...] (I - Vp T Vp^T), the nbp reflectors in w.Vp
// (rows of Vp = the Lc columns), T their forward triangular factor.
cudaError_t apply_block_reflector_right(const BdWs &w, float *X, long ldx, long ro, int Lr, long co, int Lc, int nbp,
                                        const float *tau, cudaStream_t s);
// w.Vp-style explicit block of the column reflectors [p0, p0 + nbp) stored in W.
void bd_column_vectors(const float *W, long ldw, int p0, int nbp, int Lp, float *Vp, cudaStream_t s);
// W (M x ldw, zero padded) <- a (M x N); non-finite entries are reported and replaced by 0.
void bd_copy_in_launch(const float *a, float *W, int M, int N, long ldw, DevStatus *st, cudaStream_t s);
void bd_profile_enable(int on);
void bd_profile_read(double out[4]);
int bd_profile_last_graph_run();
void bd_profile_replayed(int id);
void bd_init_attrs();
// One matrix of a stage-1 run.
struct BdJob {
    int M, N;
    const float *a_in;
    float *a_out, *u, *vt, *d, *e, *tauq, *taup;
    void *workspace;
    int thin;  // 1: u is the M x N thin U (ld N), U[:, :N] = H_0 ... H_{N-1} [I; 0]
};
// Stage 1 of k <= PK_KMAX matrices of one shape, the panels of all of them in
// lockstep (one persistent panel launch per panel serves every matrix); the
// cluster launches of their last columns run on side[0..k) (k > 1).
int bd_run_multi(int k, const BdJob *jobs, cudaStream_t s, cudaStream_t *side, int num_sms);
// Fork/join events of the side streams (1 + PK_KMAX), created on first use.
cudaEvent_t *bd_fork_events();
int bd_run(int M, int N, const float *a_in, float *a_out, float *u, float *vt, float *d, float *e, float *tauq,
           float *taup, void *workspace, cudaStream_t s, int num_sms);
