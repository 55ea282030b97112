// Split-precision GETT: FP64 operands sliced into int8 pieces with a shared
// power-of-two scale per row (Ozaki scheme), products on the tcgen05 tensor
// pipe with INT32 accumulation in TMEM, exact per-level sums recombined in FP64.
#pragma once
#include <cuda_runtime.h>
#include "kernels.cuh"

namespace ccqb {

constexpr int MAX_SLICES = 7;

struct SplitSizes {
    long long a_elems;   // max M * Kpad over split GETTs
    long long b_elems;   // max N * Kpad
    long long mn;        // max M + N (row scales)
};

struct SplitWorkspace {
    signed char *a = nullptr;   // slices of A, K-major, [slice][M][Kpad]
    signed char *b = nullptr;   // slices of B, K-major, [slice][N][Kpad]
    int *ea = nullptr;          // per-row exponents of A
    int *eb = nullptr;          // per-row exponents of B
    int *err = nullptr;         // set by a kernel whose bounded wait expired
    long long cap_a = 0, cap_b = 0, cap_mn = 0;
    int slices = 0;
};

void split_reserve(SplitWorkspace &w, SplitSizes s, int nslices);
void split_free(SplitWorkspace &w);
// Runs one GETT in split precision; returns the number of kernels launched.
// persistent: one CTA per SM over all output tiles, epilogue overlapped with
// the next tile's MMAs (else one CTA per output tile).
int split_gett(SplitWorkspace &w, const GettArgs &g, int a_kmajor, int b_kmajor, int nslices, cudaStream_t s,
               int persistent = 0);
int split_launch_count(const GettArgs &g, int nslices);
// Large enough for the tensor-core split path (else FP64 DMMA).
bool split_eligible(const GettArgs &g);
// Nonzero when a split kernel gave up waiting (pipeline stall).
int split_error(const SplitWorkspace &w);

}  // namespace ccqb
