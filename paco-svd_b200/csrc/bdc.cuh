// Stage-2 (bidiagonal divide and conquer) layout and driver declarations.
#pragma once

#include "common.cuh"
#include "gemm_tc.cuh"

// Tiling blob written by GenerateTiling and read by svd_DC (replaces the
// SVDTiling + SVDSubmatrixInfo stack of svd_tiling.cpp:21-26, 83-130).
struct TilingHeader {
    uint32_t magic;   // 'PACO'
    uint32_t N;
    uint32_t nleaf;
    uint32_t offset;  // byte offset of the leaf array (32)
    uint32_t version; // 1
    uint32_t pad[3];
};
#define PACO_TILING_MAGIC 0x4F434150u

struct MergeMeta {
    int n, nc, nl, Lr, k, nrot, sq, pad;
    float orgnrm, tol, cns, sns;
};

struct RotEntry {
    int ra, rb;
    float c, s;
};

struct BdcWs {
    DevStatus *st;
    float *Us, *Vs;   // N x N: secular singular vectors of every merge (diagonal blocks)
    double *zsec;     // N: z of the secular problems
    RotEntry *rot;    // N: deflation rotations of every merge (indexed from its start)
    MergeMeta *meta;  // N: per-merge results, indexed by the merge's first column
    int *leaf_s, *leaf_e;        // leaves
    int *mg_s, *mg_m, *mg_e;     // merges of all levels, level after level
    int *perm;        // N: final descending order
    float *sig;       // N: sorted singular values
    float *tcs;       // tensor-core GEMM scratch of the final products; null when unused
    size_t tcs_floats;
};

static inline size_t bdc_carve(void *base, int M, int N, BdcWs *w)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = (off + 255) & ~(size_t)255;
        char *p = base ? (char *)base + off : nullptr;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    const int nleaf = N / 3 + 2;
    w->st = (DevStatus *)take(sizeof(DevStatus));
    w->Us = (float *)take(sizeof(float) * nn);
    w->Vs = (float *)take(sizeof(float) * nn);
    w->zsec = (double *)take(sizeof(double) * N);
    w->rot = (RotEntry *)take(sizeof(RotEntry) * N);
    w->meta = (MergeMeta *)take(sizeof(MergeMeta) * N);
    w->leaf_s = (int *)take(sizeof(int) * nleaf);
    w->leaf_e = (int *)take(sizeof(int) * nleaf);
    w->mg_s = (int *)take(sizeof(int) * nleaf);
    w->mg_m = (int *)take(sizeof(int) * nleaf);
    w->mg_e = (int *)take(sizeof(int) * nleaf);
    w->perm = (int *)take(sizeof(int) * N);
    w->sig = (float *)take(sizeof(float) * N);
    const int shapes[2][3] = {{M, N, N}, {N, N, N}};
    w->tcs_floats = std::max(M, N) > 1024 ? gemm_tc_scratch_for(shapes, 2) : 0;
    w->tcs = w->tcs_floats ? (float *)take(sizeof(float) * w->tcs_floats) : nullptr;
    return (off + 255) & ~(size_t)255;
}

// Leaf partition of svd_tiling.cpp:83-130 (host and device agree on it).
__host__ __device__ inline int leaf_partition(int N, int *starts, int *ends)
{
    if (N <= 0) return 0;
    if (N <= 2) {
        if (starts) { starts[0] = 0; ends[0] = N; }
        return 1;
    }
    int total = N / 3 + 1, rem = N % 3;
    if (starts) {
        for (int i = 0; i < total - 2; i++) { starts[i] = 3 * i; ends[i] = 3 * i + 3; }
        int i = total - 2;
        starts[i] = 3 * i;
        ends[i] = 3 * i + (rem == 0 ? 2 : 3);
        i = total - 1;
        if (rem == 0) { starts[i] = 3 * i - 1; ends[i] = 3 * i; }
        else if (rem == 1) { starts[i] = 3 * i; ends[i] = 3 * i + 1; }
        else { starts[i] = 3 * i; ends[i] = 3 * i + 2; }
    }
    return total;
}

size_t bdc_workspace_bytes(int M, int N);
void bdc_init_attrs();
// Secular-solver iteration limit of the single-matrix (bdc.cu) and batched
// (batched.cu) kernels; a test hook that forces the non-convergence report.
void bdc_set_sec_maxit(int n);
void bt_set_sec_maxit(int n);
// u holds U with ldu floats per row (ldu = M for the M x M U; N for the thin
// M x N U of paco_svd_thin); only its first N columns are read and written.
int bdc_run(int M, int N, float *a, float *u, float *vt, float *d, float *e, float *qt, float *wt, uint32_t *idx,
            void *workspace, const uint8_t *tiling, cudaStream_t s, long ldu = 0);
