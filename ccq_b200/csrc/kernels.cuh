// Device kernels of libccq_b200 (sm_100a).
//
//  gett_f64     : GEMM over strided/permuted tensor views (GETT) in FP64 on the
//                 DMMA tensor pipe (mma.sync m16n8k8 f64).  Operand addresses
//                 come from per-mode offset tables, so a permuted slice of a
//                 resident tensor is read in place: this fuses the reference's
//                 reorder_shift / reorder_stripe + egemm + sum_stripe triple
//                 (src/cc/reorder_stripe.f90, src/dgemm.f90) into one kernel.
//  assemble     : residual gather of a spin block from permuted views, Jacobi
//                 step and antisymmetric fill (src/cc/t*_update.f90 tails).
//  diis_*       : ring residuum, B matrix, bordered solve and extrapolation
//                 (src/diis.F90).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ccqb {

// message returned by ccq_b200_last_error() on this thread
void set_last_error(const char *msg);

constexpr int MAXR = 8;        // max tensor rank (T4 blocks)
constexpr int MAX_TERMS = 65536; // max views gathered by one assemble

// One (A, B, K, alpha) term of a grouped GETT: several contractions that add
// into the same output view run as one launch, so the output is read and
// written once instead of once per contraction.
struct GettSeg {
    const double *A, *B;
    const int *offA_m, *offA_k, *offB_n, *offB_k;
    int K;
    double alpha;
};

struct GettArgs {
    const double *A;
    const double *B;
    double *C;
    const int *offA_m, *offA_k, *offB_n, *offB_k, *offC_m, *offC_n;
    int M, N, K;
    double alpha;
    int beta;       // 0: overwrite, 1: accumulate
    int kchunk;     // K range handled by one blockIdx.z (split-K, atomic epilogue)
    int c_nfast;    // 1: output contiguous along n (write-out walks n), 0: along m
    // 16-byte paths, set by the host only where the tables pair up contiguous,
    // 16-byte aligned elements: vec_a / vec_b for m- (n-) major operand loads,
    // vec_c for the output write-out along its fast mode
    int vec_a, vec_b, vec_c;
    const GettSeg *segs;  // grouped launch: nseg terms (A, B, tables, K, alpha above unused)
    int nseg;
    int tile;       // 0: tile family by shape (gett_f64_family); 1: 64 x 64 tiles; 2: skinny tiles;
                    // 3: small-K FMA kernel (whole K per launch, kchunk ignored);
                    // 4: 64 x 64 tiles with a 3-stage operand pipeline;
                    // 5: skinny tiles with a 2-stage ring (more CTAs per SM);
                    // 6: register-direct small-K kernel (whole K per launch, kchunk ignored)
};

constexpr int MAXG = 4;  // antisymmetric axis groups per source view

// One permuted view read by the assemble step.  Axis j of the source holds
// target axis src[j]; groups list source axes stored only for increasing
// indices (the source is antisymmetric in them), read sorted with sign.
struct AsmTerm {
    const double *p;
    double coef;
    int zstride[MAXR];
    signed char src[MAXR];
    signed char gpos[MAXG][MAXR];
    signed char glen[MAXG];
    signed char ng;
    signed char rank;
};

struct AsmArgs {
    double *T;
    int rank;                 // 2 * level
    int level;
    int dims[MAXR];
    int tstride[MAXR];
    int spin[MAXR];           // 0 alpha, 1 beta per axis
    int runstart[MAXR];       // 1 if this axis starts a same-spin run within its half
    const double *fdiag[2];   // denominator diagonals (active range): Fock, or Hbar for mode 2
    int nocc[2];
    double shift;
    int mode;                 // 0 jacobi, 1 copy, 2 left jacobi (shift - *ecor, sum of R^2 into *norm)
    const double *ecor;       // mode 2: correlation energy subtracted from the denominators
    double *norm;             // mode 2: accumulates nperm * R^2 (every stored element's LH^2)
    int nterms;
    const AsmTerm *terms;
    int nperm;                // orbit permutations of a canonical element
    const signed char *perm;  // nperm x rank axis maps
    const signed char *psign; // nperm signs
    long long total;          // number of canonical elements
    // canonical elements are enumerated run by run (a run = same-spin axes of one
    // half); run r covers axes [run_axis0[r], run_axis0[r] + run_len[r]) and has
    // run_count[r] increasing tuples stored at combos + run_off[r]
    int nruns;
    int run_axis0[MAXR], run_len[MAXR], run_count[MAXR], run_off[MAXR];
    const unsigned char *combos;
    int off32;                // every offset (terms, T, canonical index) fits in 32 bits
    int nplain;               // terms [0, nplain) read plain views (no sorted groups); the rest sorted
    // active-space triples (mode 0 only): an element is kept when at least one occupied index is
    // >= act_occ_lo and at least one virtual index is < act_vir_hi[spin]; the others are set to zero
    int act;
    int act_occ_lo;
    int act_vir_hi[2];
};

// FP64 GETT.  Tile family by output shape: 0 = 64 x 64 tiles; 1 = skinny rows
// (M <= 32), 2 = skinny columns (N <= 32, run transposed).  kchunk is the K
// range of one split-K slice that launch_gett_f64 expects in GettArgs::kchunk
// (more than one slice adds into C atomically, so C must start at zero).
int gett_f64_family(long long M, long long N);
int gett_f64_kchunk(long long M, long long N, long long K);
// Sets the shared-memory limits of the skinny kernels; call once before the
// first launch (outside stream capture).
cudaError_t gett_f64_prepare();
// Loads the code of the iteration's kernels now (lazy module loading would
// load each at its first launch, possibly in the middle of a solve).
cudaError_t preload_kernels(int diis_space);
void launch_gett_f64(const GettArgs &a, int a_kmajor, int b_kmajor, cudaStream_t s);
void launch_zero_view(double *C, const int *offm, const int *offn, int M, int N, cudaStream_t s);
void launch_assemble(const AsmArgs &a, cudaStream_t s);

// Batched launches over the contexts of many independent solves (one plan operation of every
// context at once).  owner[i] is the context of entry i; entries of contexts with active[owner[i]]
// zero do nothing.  GETTs: 64 x 64 tiles, split into K slices of the entry's kchunk (slices add into
// C atomically: zero it first), tstart[i] = first tile of entry i (tiles = all tiles); assembles: cstart[i] = first chunk of ASM_CHUNK canonical elements of entry i.
struct BatchCopy {
    double *dst;
    const double *src;   // null: zero dst
    long long n;
};
constexpr int ASM_CHUNK = 512;   // canonical elements per block of a batched assemble (256 threads x 2)
void launch_gett_f64_batched(const GettArgs *args, const int *tstart, int n, int tiles, const int *owner,
                             const int *active, int a_kmajor, int b_kmajor, cudaStream_t s);
void launch_assemble_batched(const AsmArgs *args, const long long *cstart, int n, long long chunks, int rank,
                             const int *owner, const int *active, cudaStream_t s);
void launch_copy_batched(const BatchCopy *cp, int n, const int *owner, const int *active, cudaStream_t s);
// zero the output views of the entries (before split-K slices add into them)
void launch_zero_views_batched(const GettArgs *args, int n, const int *owner, const int *active, cudaStream_t s);
void launch_fill(double *p, double v, long long n, cudaStream_t s);
void launch_f2c4(const double *f, double *out, long long n, cudaStream_t s);
void launch_sqdiff(const double *a, const double *b, long long n, double *out, cudaStream_t s);

// ccq's compressed CCSDt T3 (get_t_sizes_act): geometry of its ten sub-blocks inside the full T3
// blocks of a T vector, and the gather / scatter between the two (csrc/ccsdt_layout.cu)
struct T3ActGeom {
    long long t12 = 0;              // T1 + T2 elements (the same in both layouts)
    long long sub_off[11] = {};     // sub-block offsets within the compressed T3 part
    int block[10] = {};             // 0..3: T3A..T3D
    int lo[10][6] = {}, n[10][6] = {};   // sub-range start (0-based in the full block's axis) and extent
    long long full_off[4] = {};     // T3A..T3D offsets in the full T vector
    int fn[4][6] = {};              // full block extents (Fortran axis order)
    long long n_act = 0;            // compressed T3 elements
    long long t3_begin = 0, t3_end = 0;   // T3 range of the full T vector
};
void t3act_geometry(long long froz, long long occ_a, long long occ_b, long long orbs, long long act_occ_b,
                    long long act_unocc_a, T3ActGeom &g);
void launch_t3act_gather(const T3ActGeom &g, const double *tvec, double *cvec, cudaStream_t s);
void launch_t3act_scatter(const T3ActGeom &g, const double *cvec, double *tvec, cudaStream_t s);
void launch_diis_gram(const double *ring, long long stride, int ds, long long n, double *gram, cudaStream_t s);
void launch_diis_solve(double *gram, int ds, double *coef, int *info, cudaStream_t s);
void launch_diis_extrap(const double *ring, long long stride, int ds, long long n, const double *coef, double *t,
                        cudaStream_t s);

}  // namespace ccqb
