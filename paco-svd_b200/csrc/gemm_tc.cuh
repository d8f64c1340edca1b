// FP32 products on the 5th-generation tensor cores (tcgen05, sm_100a) through
// a 3xTF32 split, for the large GEMMs of the pipeline (formation of U and V,
// the panel trailing update, the final U*Q and W^T*Vt products).  Operands use
// the same strided/gathered GemmOp addressing as the SIMT engine of gemm.cuh.
#pragma once

#include "gemm.cuh"

// Floats of scratch gemm_tc_run needs for an M x N x K product (operand
// images plus split-K partials).
size_t gemm_tc_scratch_floats(int M, int N, int K);

// True unless PACO_TC=0 is set in the environment.
bool gemm_tc_enabled();

// Sets the kernel attributes (dynamic shared memory); call once per device
// outside stream capture.
void gemm_tc_init_attrs();

// C = alpha * opA * opB + beta * C on the tensor cores; scratch holds
// gemm_tc_scratch_floats(M, N, K) floats.  A bounded wait that gives up
// records PACO_ERR_TIMEOUT in st.
// With lim (a device int), the product is limited to M' = min(M, *lim) rows
// and K' = min(K, *lim): opA rows and k beyond it read as 0 and C's rows
// beyond it are left as they are.  A limited product must not be split-K.
cudaError_t gemm_tc_run(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C, long ldc,
                        float *scratch, DevStatus *st, cudaStream_t s, const int *lim = nullptr);

// Products without split-K run on the persistent kernel (one CTA per SM
// walking the tiles) unless this is set to 0 (or PACO_TC_PERSISTENT=0);
// returns the previous setting.
int gemm_tc_set_persistent(int on);

// Tensor-core product when it is enabled, tc_scratch holds enough floats and
// the product is large enough to pay for the operand packing; otherwise the
// SIMT engine (with its own split-K scratch).
cudaError_t gemm_any(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C, long ldc,
                     int splits, float *simt_scratch, float *tc_scratch, size_t tc_floats, DevStatus *st,
                     cudaStream_t s);

// Scratch floats covering every product gemm_any may send to the tensor cores
// for the given list of shapes (max over them); 0 when the tensor-core path
// is not used for any of them.
size_t gemm_tc_scratch_for(const int (*shapes)[3], int n);

// Test hook: a kernel holding tensor memory whose mbarrier wait never
// completes; the wait gives up after max_cycles (PACO_ERR_TIMEOUT in st) and
// the tensor memory is freed before the CTA exits.
bool gemm_tc_debug_timeout(DevStatus *st, long long max_cycles, cudaStream_t s);
