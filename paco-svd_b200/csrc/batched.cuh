// Batched SVD of many small matrices (batched.cu): launch constants, the
// work items, and the layouts of the per-matrix area and of the per-CTA
// divide-and-conquer slot in the batched workspace.
#pragma once

#include "bdc_dev.cuh"

namespace bt {
constexpr int T_SWEEP = 512;            // threads of kernels 1 and 3
constexpr int W_SWEEP = T_SWEEP / 32;
constexpr int T_BDC = 256;              // threads of kernel 2 (the bdc bodies assume 256)
constexpr int KSMALL = 32;              // merges up to this k solve a secular root per thread
}  // namespace bt

struct BtItem {
    int M, N, index, pad;
    const float *A;
    float *U, *Vt, *sigma;
    size_t moff;  // byte offset of the matrix's area in the arena
};

// per-matrix area, alive from kernel 1 to kernel 3
struct BtMat {
    float *W;  // M x ldw: Householder vectors, d on the diagonal, e on the superdiagonal
    long ldw;
    float *d, *e, *tauq, *taup;
    float *QT, *WT;  // N x N (ld N): Q^T and W^T of the divide and conquer
    int *perm;       // N: descending order of the singular values
    float *sig;      // N: sorted singular values
    int *code;       // PACO_* status of the matrix
};

__host__ __device__ static size_t bt_mat_carve(char *base, int M, int N, BtMat *m)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = (off + 255) & ~(size_t)255;
        char *p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    m->ldw = (N + 3) & ~3;
    m->W = (float *)take(sizeof(float) * (size_t)M * m->ldw);
    m->d = (float *)take(sizeof(float) * N);
    m->e = (float *)take(sizeof(float) * N);
    m->tauq = (float *)take(sizeof(float) * N);
    m->taup = (float *)take(sizeof(float) * N);
    m->QT = (float *)take(sizeof(float) * nn);
    m->WT = (float *)take(sizeof(float) * nn);
    m->perm = (int *)take(sizeof(int) * N);
    m->sig = (float *)take(sizeof(float) * N);
    m->code = (int *)take(sizeof(int));
    return (off + 255) & ~(size_t)255;
}

// divide-and-conquer scratch of one CTA of kernel 2
struct BtBdcSlot {
    float *ST, *GT;  // N x N gather targets
    int *idx;        // 16 N: idxq, f, l, dsig, zhat, srow
    float *diff;     // N x N: d_j^2 - sigma_i^2 of the secular roots
    BdcWs bw;        // perm and sig are pointed at the matrix's area per matrix
};

__host__ __device__ static size_t bt_bdc_carve(char *base, int N, BtBdcSlot *s)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = (off + 255) & ~(size_t)255;
        char *p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    const int nleaf = N / 3 + 2;
    s->ST = (float *)take(sizeof(float) * nn);
    s->GT = (float *)take(sizeof(float) * nn);
    s->idx = (int *)take(sizeof(int) * 16 * (size_t)N);
    s->diff = (float *)take(sizeof(float) * nn);
    BdcWs &w = s->bw;
    w.st = (DevStatus *)take(sizeof(DevStatus));
    w.Us = (float *)take(sizeof(float) * nn);
    w.Vs = (float *)take(sizeof(float) * nn);
    w.zsec = (double *)take(sizeof(double) * N);
    w.rot = (RotEntry *)take(sizeof(RotEntry) * N);
    w.meta = (MergeMeta *)take(sizeof(MergeMeta) * N);
    w.leaf_s = (int *)take(sizeof(int) * nleaf);
    w.leaf_e = (int *)take(sizeof(int) * nleaf);
    w.mg_s = (int *)take(sizeof(int) * nleaf);
    w.mg_m = (int *)take(sizeof(int) * nleaf);
    w.mg_e = (int *)take(sizeof(int) * nleaf);
    w.perm = nullptr;
    w.sig = nullptr;
    w.tcs = nullptr;
    w.tcs_floats = 0;
    return (off + 255) & ~(size_t)255;
}
