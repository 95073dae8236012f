// Declarations shared by the tensor-core update's host code and the
// mixed-precision LU driver.
#pragma once

#include <cuda.h>

#include "tc_gemm.cuh"

namespace b200la
{
// TMA map of a K-major operand: `rows` rows of `k` elements, row stride `ld`
// elements, boxes of one 128-byte K slice x box_rows rows, 128B swizzle.
int make_kmajor_map(CUtensorMap* map, const void* base, int kind, int64_t rows, int64_t k, int64_t ld,
    int box_rows);

// C[m x n] -= A B^T on the tensor cores (k_tc_update_persistent, or
// k_tc_update with B200LA_TC_PERSISTENT=0).  FP8 operands need the inverse
// power-of-two scales of their rows (inv_sa[m], inv_sb[n]).  max_ctas > 0
// caps the persistent grid (leaving SMs to kernels on other streams).
// place_cluster > 1 launches the persistent grid as clusters of that many
// CTAs (placement only: the CTAs do not talk), one cluster fewer than fit
// the device at once, so that whole GPCs hold the update and one GPC stays
// free for a cluster launched beside it.
int enqueue_tc_update(int kind, bool split3, const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& as,
    const CUtensorMap& bs, float* c, int64_t ldc, int m, int n, int k, DeviceStatus* st, cudaStream_t s,
    const float* inv_sa = nullptr, const float* inv_sb = nullptr, int max_ctas = 0, int place_cluster = 0);
}  // namespace b200la
