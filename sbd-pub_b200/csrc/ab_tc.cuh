// Tensor-core (tcgen05) contraction of the dense alpha-beta path (see ab_tc.cu).
#pragma once

#include "tpb_common.cuh"

namespace sbdtpb {

int ab_tc_setup(sbd_tpb_handle *h);
// E[n][j] (FP32, label-major, n < npq, j < M) from the gathered hi/lo tiles already in d_ab_work.
int ab_tc_gemm(sbd_tpb_handle *h, const float *unused_D, float *E, size_t M);
// Gathers D = sum s_b C[Ja, Jb] straight into the tiled BF16 hi/lo layout.
int ab_tc_gather(sbd_tpb_handle *h, const float *C, size_t M);
// Bytes of the tiled hi/lo operand plus the FP32 result E.
size_t ab_tc_work_bytes(sbd_tpb_handle *h);
// Fused path (ab.tc_fused_stages > 0): E straight from C, the A tiles built in shared memory.
int ab_tc_fused(sbd_tpb_handle *h, const float *C, float *E, size_t M);
// Bytes of E alone (the fused path's work array).
size_t ab_tc_fused_work_bytes(sbd_tpb_handle *h);
// Reads and clears the kernel's bounded-wait status; error status if a wait expired.
int ab_tc_check(sbd_tpb_handle *h);

}  // namespace sbdtpb
