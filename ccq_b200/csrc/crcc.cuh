// CR-CC(2,3) device kernels of libccq_b200 (sm_100a).
//
//  crdiag  : Hbar(CCSD) one-body diagonal (the left Jacobi denominators of
//            left_jacobi_update, src/update_lcc.f90:208-280, and D_B of
//            crcc23), the two-body diagonals h[p,q,p,q] (D_C) and the
//            three-body sums of cal_d3 (src/mm_correct.f90:346-481, D_D),
//            from T1-dressed and bare integrals and T2.
//  crcc_sum: sum over the unique triples of one spin block of
//            l3 * M3 / D for the four denominators A-D
//            (src/mm_correct.f90:110-338).
//  lenergy : sqrt(sum LH^2) + E_cor (calculate_left_energy,
//            src/energy.f90:103-136).
#pragma once
#include <cuda_runtime.h>

namespace ccqb {

struct CrDiagArgs {
    const double *FA, *FB, *VAA, *VAB, *VBB;   // T1-dressed, full active range n
    const double *VAA0, *VAB0, *VBB0;          // bare
    const double *T2A, *T2B, *T2C;             // [oa][oa][va][va], [oa][ob][va][vb], [ob][ob][vb][vb]
    double *HDA, *HDB;                         // [n]
    double *H2AA, *H2AB, *H2BB;                // [n][n]: h[p,q,p,q] (H2AB: p alpha, q beta)
    double *W1[4], *W2[4];                     // [n][n][n]
    int n, oa, ob, va, vb;
    int w1d_e0;  // first beta virtual (relative) summed in the beta-beta-beta three-body term
};

struct CrccArgs {
    const double *M, *L;   // one spin block, [i0][i1][i2][a0][a1][a2]
    int dims[6];
    int spin[3];           // spin of i_k / a_k (alpha first)
    int off[2];            // first virtual (full range) per spin: oa, ob
    int n;
    const double *fd[2];   // bare Fock diagonals
    const double *hd[2];   // Hbar one-body diagonals
    const double *h2aa, *h2ab, *h2bb;
    const double *w1[4], *w2[4];
    double *e23;           // four sums, accumulated
    long long total;
    // triples already iterated in an active space (CC(t;3)) are left out of the sums:
    // those with an occupied index >= act_occ_lo and a virtual index (full range) < act_vir_hi;
    // act_occ_lo = n leaves none out
    int act_occ_lo, act_vir_hi;
};

void launch_crdiag(const CrDiagArgs &a, cudaStream_t s);
void launch_crcc_sum(const CrccArgs &a, cudaStream_t s);
void launch_lenergy(const double *norm, const double *ecor, double *out, cudaStream_t s);

}  // namespace ccqb
