// Split-precision GETT on the tcgen05 tensor pipe (Ozaki scheme with int8 slices).
//
// A row r of an FP64 operand (read in place through its GETT offset tables) is
// scaled by 2^-e_r so that |x| < 1, then cut into S int8 slices
//     x 2^-e_r = s_1 2^-6 + s_2 2^-13 + ... + s_S 2^(-6-7(S-1)),  |s_t| <= 64.
// Products of slices are exact in INT32.  The kernel accumulates, for every
// level L = i + j (i, j slice indices, L <= S + 1), D_L = sum_k A_i B_j^T in
// its own TMEM accumulator; the epilogue recombines
//     C = alpha 2^(e_m + e_n - 12) sum_L D_L 2^(-7 (L - 2))
// in FP64 and scatters through the GETT's output offset table.  Dropped
// higher levels bound the error by ~S 2^(-7S-5) K max|A_m| max|B_n|.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

#include "split.cuh"

namespace ccqb {

namespace {

constexpr int TM = 128;        // rows of the output tile (TMEM lanes)
constexpr int BKB = 64;        // K bytes per pipeline stage (SWIZZLE_64B atom width)
constexpr long long kWaitLimit = 1LL << 26;

// ---------------------------------------------------------------------------
// slicing
// ---------------------------------------------------------------------------
// One warp per row: exponent from the row maximum, then S int8 slices written
// K-major into out[t][row][kp] (kp = padded K, zeros beyond K).
__global__ void slice_rows_kernel(const double *base, const int *offr, const int *offk, int R, int K, int Kp, int S,
                                  signed char *out, long long slice_stride, int *expo) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < R; r += nwarps) {
        const double *row = base + offr[r];
        double mx = 0.0;
        for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(row[offk[k]]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        int e = 0;
        if (mx > 0.0) frexp(mx, &e);   // mx = f 2^e, f in [0.5, 1)
        if (lane == 0) expo[r] = e;
        double scale = ldexp(1.0, -e);
        signed char *dst = out + (long long)r * Kp;
        for (int k = lane; k < Kp; k += 32) {
            double x = k < K ? row[offk[k]] * scale : 0.0;
            double t = x * 64.0;
            for (int q = 0; q < S; ++q) {
                double s = rint(t);
                dst[q * slice_stride + k] = (signed char)s;
                t = (t - s) * 128.0;
            }
        }
    }
}

// K-major rows with K <= 512: the row stays in registers (4 consecutive k per
// lane and 128-wide chunk), one pass over memory, slices stored as packed words.
__global__ void __launch_bounds__(256) slice_rows_reg_kernel(const double *base, const int *offr, const int *offk,
                                                             int R, int K, int Kp, int S, signed char *out,
                                                             long long slice_stride, int *expo) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nch = (Kp + 127) / 128;
    for (int r = warp; r < R; r += nwarps) {
        const double *row = base + offr[r];
        double xv[16];
        double mx = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                int k = 128 * j + 4 * lane + u;
                double x = (j < nch && k < K) ? row[offk[k]] : 0.0;
                xv[4 * j + u] = x;
                mx = fmax(mx, fabs(x));
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        int e = 0;
        if (mx > 0.0) frexp(mx, &e);
        if (lane == 0) expo[r] = e;
        const double scale = ldexp(1.0, -e);
        signed char *dst = out + (long long)r * Kp;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int k0 = 128 * j + 4 * lane;
            if (j >= nch || k0 >= Kp) continue;
            double t[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) t[u] = xv[4 * j + u] * scale * 64.0;
            for (int q = 0; q < S; ++q) {
                unsigned word = 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    double sv = rint(t[u]);
                    word |= ((unsigned)(int)sv & 0xFFu) << (8 * u);
                    t[u] = (t[u] - sv) * 128.0;
                }
                *reinterpret_cast<unsigned *>(dst + q * slice_stride + k0) = word;
            }
        }
    }
}

// Rows contiguous in memory (consecutive r -> consecutive addresses): a CTA
// takes 32 rows, reads them 32 at a time (coalesced), reduces the row maxima in
// shared memory, then slices 64-wide K chunks through a shared-memory tile so
// that every row's K-major int8 bytes are written as contiguous 64 B segments.
constexpr int SR = 32;    // rows per CTA
constexpr int SK = 64;    // K per chunk
__global__ void __launch_bounds__(256) slice_rows_tiled_kernel(const double *base, const int *offr, const int *offk,
                                                               int R, int K, int Kp, int S, signed char *out,
                                                               long long slice_stride, int *expo) {
    __shared__ double red[8][SR];
    __shared__ int esh[SR];
    __shared__ __align__(16) signed char tile[MAX_SLICES][SR][SK];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int r0 = blockIdx.x * SR; r0 < R; r0 += gridDim.x * SR) {
        const int r = r0 + lane;
        const bool rin = r < R;
        const long long orow = rin ? offr[r] : 0;
        double mx = 0.0;
        if (rin)
            for (int k = w; k < K; k += 8) mx = fmax(mx, fabs(base[orow + offk[k]]));
        red[w][lane] = mx;
        __syncthreads();
        if (w == 0) {
            double m = red[0][lane];
            for (int q = 1; q < 8; ++q) m = fmax(m, red[q][lane]);
            int e = 0;
            if (m > 0.0) frexp(m, &e);
            esh[lane] = e;
            if (rin) expo[r] = e;
        }
        __syncthreads();
        const double scale = ldexp(1.0, -esh[lane]);
        for (int k0 = 0; k0 < Kp; k0 += SK) {
            for (int j = 0; j < SK / 8; ++j) {
                int kk = w + 8 * j;
                int k = k0 + kk;
                double x = (rin && k < K) ? base[orow + offk[k]] * scale : 0.0;
                double t = x * 64.0;
                for (int q = 0; q < S; ++q) {
                    double sv = rint(t);
                    tile[q][lane][kk] = (signed char)sv;
                    t = (t - sv) * 128.0;
                }
            }
            __syncthreads();
            // write-out: each row's 64 bytes per slice, as 16 words of 4 bytes
            for (int idx = threadIdx.x; idx < S * SR * (SK / 4); idx += blockDim.x) {
                int q = idx / (SR * (SK / 4));
                int rem = idx % (SR * (SK / 4));
                int rr = rem / (SK / 4), wd = rem % (SK / 4);
                if (r0 + rr < R && k0 + wd * 4 < Kp) {
                    const int *src = reinterpret_cast<const int *>(&tile[q][rr][wd * 4]);
                    int *dst = reinterpret_cast<int *>(out + q * slice_stride + (long long)(r0 + rr) * Kp + k0 + wd * 4);
                    *dst = *src;
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes));
}
// Bounded wait on a phase parity; returns false when the limit is hit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    unsigned a = smem_u32(bar);
    for (long long it = 0; it < kWaitLimit; ++it) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity));
        if (ok) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ uint64_t smem_desc_sw64(const void *p) {
    // K-major, SWIZZLE_64B: 8-row atoms of 64 B, stride between atoms 512 B.
    uint64_t addr = smem_u32(p);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;           // start address [0,14)
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;         // stride byte offset [32,46)
    d |= (uint64_t)1 << 46;                  // descriptor version (sm100)
    d |= (uint64_t)4 << 61;                  // layout: SWIZZLE_64B
    return d;
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

// x * 2^n, correctly rounded: a multiply by the power of two built from its exponent bits
// when 2^n is a normal double, else the library ldexp
__device__ __forceinline__ double scale2(double x, int n) {
    if (n >= -1022 && n <= 1023) return x * __longlong_as_double((long long)(n + 1023) << 52);
    return ldexp(x, n);
}

template <int NT>
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

struct SplitArgs {
    double *C;
    const int *offC_m, *offC_n;
    const int *ea, *eb;
    int M, N, K, Kp;
    double alpha;
    int beta;
    int c_nfast;
    int *err;
};

// One CTA per 128 x NT output tile; warp 0 lane 0 issues TMA, warp 1 lane 0
// issues MMAs, all four warps read TMEM in the epilogue.
template <int S, int NT, int STAGES>
__global__ void __launch_bounds__(128, 2)
    split_gett_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, SplitArgs p) {
    constexpr int A_BYTES = TM * BKB;           // one slice tile of A
    constexpr int B_BYTES = NT * BKB;
    constexpr int STAGE = S * (A_BYTES + B_BYTES);
    constexpr int NLEV = S;                     // levels 2..S+1
    constexpr int TCOLS = (NLEV * NT <= 32) ? 32 : (NLEV * NT <= 64) ? 64 : (NLEV * NT <= 128) ? 128
                          : (NLEV * NT <= 256) ? 256 : 512;
    static_assert(NLEV * NT <= 512, "TMEM capacity");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + STAGES * STAGE);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    __shared__ int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * NT;
    const int ktiles = p.Kp / BKB;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer
        for (int kt = 0; kt < ktiles; ++kt) {
            int s = kt % STAGES;
            if (kt >= STAGES && !mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1)) {
                abort_flag = 1;
                break;
            }
            unsigned char *st = smem + s * STAGE;
            mbar_expect_tx(&full[s], STAGE);
            tma_load_3d(st, &ta, &full[s], kt * BKB, m0, 0);
            tma_load_3d(st + S * A_BYTES, &tb, &full[s], kt * BKB, n0, 0);
        }
        // drain: every issued copy has landed before the CTA can exit
        for (int kt = (ktiles > STAGES ? ktiles - STAGES : 0); kt < ktiles; ++kt)
            if (!mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1)) abort_flag = 1;
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: instruction descriptor S32 <- S8 x S8, K-major A and B
        const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                               ((uint32_t)(TM >> 4) << 24);
        bool ok = true;
        for (int kt = 0; kt < ktiles && ok; ++kt) {
            int s = kt % STAGES;
            if (!mbar_wait(&full[s], (kt / STAGES) & 1)) {
                abort_flag = 1;
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            unsigned char *st = smem + s * STAGE;
#pragma unroll
            for (int kk = 0; kk < BKB / 32; ++kk) {
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    uint64_t da = smem_desc_sw64(st + i * A_BYTES) + (uint64_t)(kk * 32 >> 4);
#pragma unroll
                    for (int j = 0; j < S - i; ++j) {
                        uint64_t db = smem_desc_sw64(st + S * A_BYTES + j * B_BYTES) + (uint64_t)(kk * 32 >> 4);
                        int lev = i + j;   // level L - 2
                        // the first product of each level (i = 0) at the first K step initialises it
                        uint32_t acc = (kt > 0 || kk > 0 || i > 0) ? 1u : 0u;
                        umma_i8(tmem + (uint32_t)(lev * NT), da, db, idesc, acc);
                    }
                }
            }
            umma_commit(&empty[s]);
        }
        umma_commit(done);
    }
    __syncwarp();
    // epilogue: every thread owns one TMEM lane (output row)
    bool good = mbar_wait(done, 0);
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    __syncthreads();
    if (!good || abort_flag) {
        if (threadIdx.x == 0) atomicExch(p.err, 1);
    } else {
        // Stage 64 output columns at a time in shared memory (the pipeline buffers
        // are free once every MMA has completed), then write them out along C's
        // contiguous mode with all reads of a batch in flight before its writes.
        constexpr int CW = 64;
        double (*Cs)[CW + 1] = reinterpret_cast<double (*)[CW + 1]>(smem);
        int *eas = reinterpret_cast<int *>(smem + TM * (CW + 1) * sizeof(double));
        int *ebs = eas + TM;
        long long *oms = reinterpret_cast<long long *>(ebs + NT);   // output row offsets (-1: outside)
        long long *ons = oms + TM;                                   // output column offsets
        const int row = warp * 32 + lane;
        for (int t = threadIdx.x; t < TM; t += blockDim.x) {
            bool in = m0 + t < p.M;
            eas[t] = in ? p.ea[m0 + t] : 0;
            oms[t] = in ? (long long)p.offC_m[m0 + t] : -1;
        }
        for (int t = threadIdx.x; t < NT; t += blockDim.x) {
            bool in = n0 + t < p.N;
            ebs[t] = in ? p.eb[n0 + t] : 0;
            ons[t] = in ? (long long)p.offC_n[n0 + t] : -1;
        }
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += CW) {
#pragma unroll
            for (int c0 = 0; c0 < CW; c0 += 32) {
                double val[32];
#pragma unroll
                for (int q = 0; q < 32; ++q) val[q] = 0.0;
#pragma unroll
                for (int lev = NLEV - 1; lev >= 0; --lev) {
                    int v[32];
                    tmem_ld32<NT>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(lev * NT + cb + c0), v);
                    const double w = ldexp(1.0, -7 * lev);
#pragma unroll
                    for (int q = 0; q < 32; ++q) val[q] += (double)v[q] * w;
                }
#pragma unroll
                for (int q = 0; q < 32; ++q) Cs[row][c0 + q] = val[q];
            }
            __syncthreads();
            const int tid = threadIdx.x;
#pragma unroll 1
            for (int p0 = 0; p0 < TM * CW / 128; p0 += 16) {
                double *cp[16];
                double cv[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    int idx = (p0 + u) * 128 + tid;
                    int ml, nl;
                    if (p.c_nfast) {
                        nl = idx % CW;
                        ml = idx / CW;
                    } else {
                        ml = idx % TM;
                        nl = idx / TM;
                    }
                    long long om = oms[ml], on = ons[cb + nl];
                    cp[u] = (om >= 0 && on >= 0) ? p.C + om + on : nullptr;
                    cv[u] = p.alpha * scale2(Cs[ml][nl], eas[ml] + ebs[cb + nl] - 12);
                }
                double old[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) old[u] = (cp[u] && p.beta) ? *cp[u] : 0.0;
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    if (cp[u]) *cp[u] = old[u] + cv[u];
            }
            __syncthreads();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// named barriers of the persistent kernel's epilogue warps (barrier 0 is __syncthreads):
// 1 and 2 for the two halves (128 threads each), 3 for all eight warps
__device__ __forceinline__ void epi_sync_half(int h) {
    if (h == 0)
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
    else
        asm volatile("bar.sync 2, 128;\n" ::: "memory");
}
__device__ __forceinline__ void epi_sync_all() { asm volatile("bar.sync 3, 256;\n" ::: "memory"); }

// Persistent variant: one CTA per SM walks the output tiles.  Warp 0 lane 0
// issues the TMA loads of a STAGES-deep ring, warp 1 lane 0 issues the MMAs of
// a tile into one of two TMEM accumulator sets, and warps 2-9 drain the other
// set (level recombination, scaling, scattered beta write) while the next tile
// is multiplied: the epilogue of tile t overlaps the MMAs of tile t + 1.
// Barriers: full/empty per ring stage; accf[b] (MMA -> epilogue, committed by
// tcgen05) and acce[b] (epilogue -> MMA, 256 arrivals) per accumulator set.
// Every wait is bounded; a timeout sets a shared abort flag that every role
// checks before its next wait, and the host reads the error word.
template <int S, int NT, int STAGES>
struct Persist {
    static constexpr int A_BYTES = TM * BKB, B_BYTES = NT * BKB;
    static constexpr int STAGE = S * (A_BYTES + B_BYTES);
    static constexpr int BUFC = S * NT;   // TMEM columns of one accumulator set (levels 2..S+1)
    static constexpr int CW = 32;         // output columns per epilogue pass
    static constexpr int CS_BYTES = 2 * TM * (CW + 1) * 8;   // one staging tile per epilogue half
    static constexpr int TAB_BYTES = TM * 4 + NT * 4 + TM * 8 + NT * 8;
    static constexpr int BAR_BYTES = (2 * STAGES + 5) * 8 + 16;
    static constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE + CS_BYTES + TAB_BYTES + BAR_BYTES;
    static_assert(2 * BUFC <= 512, "two accumulator sets must fit in TMEM");
    static_assert(STAGE % 1024 == 0 && A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "swizzle atom alignment");
    static_assert((TM * 4 + NT * 4) % 8 == 0 && CS_BYTES % 8 == 0, "table alignment");
};

template <int S, int NT, int STAGES>
__global__ void __launch_bounds__(320, 1)
    split_gett_persistent(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, SplitArgs p) {
    using P = Persist<S, NT, STAGES>;
    constexpr int CW = P::CW;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    double (*Cs)[CW + 1] = reinterpret_cast<double (*)[CW + 1]>(smem + STAGES * P::STAGE);
    int *eas = reinterpret_cast<int *>(smem + STAGES * P::STAGE + P::CS_BYTES);
    int *ebs = eas + TM;
    long long *oms = reinterpret_cast<long long *>(ebs + NT);   // output row offsets (-1: outside)
    long long *ons = oms + TM;                                   // output column offsets
    uint64_t *full = reinterpret_cast<uint64_t *>(ons + NT);
    uint64_t *empty = full + STAGES;
    uint64_t *accf = empty + STAGES;
    uint64_t *acce = accf + 2;
    uint64_t *fin = acce + 2;   // the MMA issuer's last commit: all its MMAs have completed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(fin + 1);
    __shared__ volatile int abort_flag;
    __shared__ volatile int epi_stop;   // written by epilogue thread 0 only, read by all eight warps after a barrier

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = (p.M + TM - 1) / TM, nt = (p.N + NT - 1) / NT;
    const int ntiles = mt * nt;
    const int ktiles = p.Kp / BKB;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 256);
        }
        mbar_init(fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // producer: the k-tiles of every tile of this CTA, through the ring
            long long kc = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x) {
                const int m0 = (tile % mt) * TM, n0 = (tile / mt) * NT;
                for (int kt = 0; kt < ktiles; ++kt, ++kc) {
                    const int s = (int)(kc % STAGES);
                    if (kc >= STAGES && !mbar_wait(&empty[s], (unsigned)(((kc / STAGES) - 1) & 1))) abort_flag = 1;
                    if (abort_flag) break;
                    unsigned char *st = smem + s * P::STAGE;
                    mbar_expect_tx(&full[s], P::STAGE);
                    tma_load_3d(st, &ta, &full[s], kt * BKB, m0, 0);
                    tma_load_3d(st + S * P::A_BYTES, &tb, &full[s], kt * BKB, n0, 0);
                }
            }
            // every issued copy lands before the CTA can exit
            for (long long q = kc > STAGES ? kc - STAGES : 0; q < kc; ++q)
                if (!mbar_wait(&full[q % STAGES], (unsigned)((q / STAGES) & 1))) abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: S32 <- S8 x S8, K-major A and B, M = 128, N = NT
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                                   ((uint32_t)(TM >> 4) << 24);
            long long kc = 0;
            int tl = 0;
            for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x, ++tl) {
                const int b = tl & 1, u = tl >> 1;
                // the epilogue has drained this accumulator set (its previous use)
                if (u > 0 && !mbar_wait(&acce[b], (unsigned)((u - 1) & 1))) {
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n");
                const uint32_t tacc = tmem + (uint32_t)(b * P::BUFC);
                bool ok = true;
                for (int kt = 0; kt < ktiles; ++kt, ++kc) {
                    const int s = (int)(kc % STAGES);
                    if (abort_flag || !mbar_wait(&full[s], (unsigned)((kc / STAGES) & 1))) {
                        abort_flag = 1;
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n");
                    unsigned char *st = smem + s * P::STAGE;
#pragma unroll
                    for (int kk = 0; kk < BKB / 32; ++kk) {
#pragma unroll
                        for (int i = 0; i < S; ++i) {
                            const uint64_t da = smem_desc_sw64(st + i * P::A_BYTES) + (uint64_t)(kk * 32 >> 4);
#pragma unroll
                            for (int j = 0; j < S - i; ++j) {
                                const uint64_t db =
                                    smem_desc_sw64(st + S * P::A_BYTES + j * P::B_BYTES) + (uint64_t)(kk * 32 >> 4);
                                // the first product of each level at the tile's first K step initialises it
                                const uint32_t acc = (kt > 0 || kk > 0 || i > 0) ? 1u : 0u;
                                umma_i8(tacc + (uint32_t)((i + j) * NT), da, db, idesc, acc);
                            }
                        }
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) break;
                umma_commit(&accf[b]);
            }
            // TMEM is released below only after every MMA this thread issued has completed
            umma_commit(fin);
            if (!mbar_wait(fin, 0)) abort_flag = 1;
        }
    } else {
        // epilogue: warps 2-9.  Warp w reads TMEM lanes 32 (w % 4) .. + 31 (its quadrant); the two
        // warps of a quadrant split the tile's 32-column chunks (half h takes chunks h, h + 2, ...)
        const int q = warp & 3, row = q * 32 + lane, et = threadIdx.x - 64, h = et >> 7, eh = et & 127;
        double (*Ch)[CW + 1] = Cs + h * TM;
        int tl = 0;
        // the eight warps leave the tile loop together: the stop decision is taken by one thread
        // and published through a barrier, never read from abort_flag by each thread on its own
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++tl) {
            const int b = tl & 1, u = tl >> 1;
            if (et == 0) {
                const bool ok = !abort_flag && mbar_wait(&accf[b], (unsigned)(u & 1));
                if (!ok) abort_flag = 1;
                epi_stop = ok ? 0 : 1;
            }
            epi_sync_all();
            if (epi_stop) break;
            // the phase has completed (thread 0 saw it): this returns at once and orders this thread's reads
            mbar_wait(&accf[b], (unsigned)(u & 1));
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            const int m0 = (tile % mt) * TM, n0 = (tile / mt) * NT;
            for (int t = et; t < TM; t += 256) {
                const bool in = m0 + t < p.M;
                eas[t] = in ? p.ea[m0 + t] : 0;
                oms[t] = in ? (long long)p.offC_m[m0 + t] : -1;
            }
            for (int t = et; t < NT; t += 256) {
                const bool in = n0 + t < p.N;
                ebs[t] = in ? p.eb[n0 + t] : 0;
                ons[t] = in ? (long long)p.offC_n[n0 + t] : -1;
            }
            epi_sync_all();   // tables in
            const uint32_t tacc = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * P::BUFC);
#pragma unroll 1
            for (int cb = h * CW; cb < NT; cb += 2 * CW) {
                double val[32];
#pragma unroll
                for (int c = 0; c < 32; ++c) val[c] = 0.0;
#pragma unroll
                for (int lev = S - 1; lev >= 0; --lev) {
                    int v[32];
                    tmem_ld32<NT>(tacc + (uint32_t)(lev * NT + cb), v);
                    const double w = ldexp(1.0, -7 * lev);
#pragma unroll
                    for (int c = 0; c < 32; ++c) val[c] += (double)v[c] * w;
                }
                if (cb + 2 * CW >= NT) {
                    // this thread's reads of the set are complete: release it to the MMA warp
                    asm volatile("tcgen05.fence::before_thread_sync;\n");
                    mbar_arrive(&acce[b]);
                }
                epi_sync_half(h);   // this half's previous write-out has finished reading Ch
#pragma unroll
                for (int c = 0; c < 32; ++c) Ch[row][c] = val[c];
                epi_sync_half(h);
#pragma unroll 1
                for (int p0 = 0; p0 < TM * CW / 128; p0 += 8) {
                    double *cp[8];
                    double cv[8];
#pragma unroll
                    for (int uu = 0; uu < 8; ++uu) {
                        const int idx = (p0 + uu) * 128 + eh;
                        int ml, nl;
                        if (p.c_nfast) {
                            nl = idx % CW;
                            ml = idx / CW;
                        } else {
                            ml = idx % TM;
                            nl = idx / TM;
                        }
                        const long long om = oms[ml], on = ons[cb + nl];
                        cp[uu] = (om >= 0 && on >= 0) ? p.C + om + on : nullptr;
                        cv[uu] = p.alpha * scale2(Ch[ml][nl], eas[ml] + ebs[cb + nl] - 12);
                    }
                    double old[8];
#pragma unroll
                    for (int uu = 0; uu < 8; ++uu) old[uu] = (cp[uu] && p.beta) ? *cp[uu] : 0.0;
#pragma unroll
                    for (int uu = 0; uu < 8; ++uu)
                        if (cp[uu]) *cp[uu] = old[uu] + cv[uu];
                }
            }
            epi_sync_all();   // tables and staging tiles are free for the next tile
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n");
    __syncthreads();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
    if (threadIdx.x == 0 && abort_flag) atomicExch(p.err, 1);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn get_encode() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeFn)p;
    });
    if (!fn) throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
    return fn;
}

// 3-D map over int8 slices [S][rows][Kp]; box (64 B, tile rows, S).
CUtensorMap make_map(signed char *base, long long rows, long long Kp, int S, int box_rows) {
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)S};
    cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)(Kp * rows)};
    cuuint32_t box[3] = {(cuuint32_t)BKB, (cuuint32_t)box_rows, (cuuint32_t)S};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed");
    return m;
}

template <int S, int NT, int STAGES>
void launch_split_persistent(const CUtensorMap &ta, const CUtensorMap &tb, const SplitArgs &a, cudaStream_t s) {
    const int tiles = ((a.M + TM - 1) / TM) * ((a.N + NT - 1) / NT);
    int dev = 0, sms = 0;   // SM count of the current device (one CTA per SM)
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms < 1) sms = 148;
    const int grid = std::min(tiles, sms);
    split_gett_persistent<S, NT, STAGES><<<grid, 320, Persist<S, NT, STAGES>::SMEM, s>>>(ta, tb, a);
}

template <int S, int NT, int STAGES>
void launch_split(const CUtensorMap &ta, const CUtensorMap &tb, const SplitArgs &a, cudaStream_t s) {
    constexpr int STAGE = S * (TM * BKB + NT * BKB);
    size_t smem = (size_t)STAGES * STAGE + 1024 + 256;
    dim3 grid((a.M + TM - 1) / TM, (a.N + NT - 1) / NT);
    split_gett_kernel<S, NT, STAGES><<<grid, 128, smem, s>>>(ta, tb, a);
}

int tile_n(int S) { return S <= 2 ? 128 : 64; }

template <int S, int NT, int STAGES>
void set_smem_attr() {
    constexpr int STAGE = S * (TM * BKB + NT * BKB);
    size_t smem = (size_t)STAGES * STAGE + 1024 + 256;
    if (cudaFuncSetAttribute(split_gett_kernel<S, NT, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        throw std::runtime_error("cannot enable large shared memory for the split kernel");
}

template <int S, int NT, int STAGES>
void set_persist_attr() {
    if (cudaFuncSetAttribute(split_gett_persistent<S, NT, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Persist<S, NT, STAGES>::SMEM) != cudaSuccess)
        throw std::runtime_error("cannot enable large shared memory for the persistent split kernel");
}

}  // namespace

void split_reserve(SplitWorkspace &w, SplitSizes sz, int nslices) {
    auto need = [&](long long a, long long b, long long mn) {
        return a * nslices > w.cap_a || b * nslices > w.cap_b || mn > w.cap_mn || nslices > w.slices;
    };
    if (!need(sz.a_elems, sz.b_elems, sz.mn) && w.err) return;
    split_free(w);
    long long ca = std::max(sz.a_elems, 1LL) * nslices, cb = std::max(sz.b_elems, 1LL) * nslices;
    if (cudaMalloc(&w.a, ca) != cudaSuccess || cudaMalloc(&w.b, cb) != cudaSuccess ||
        cudaMalloc(&w.ea, sizeof(int) * std::max(sz.mn, 1LL)) != cudaSuccess ||
        cudaMalloc(&w.eb, sizeof(int) * std::max(sz.mn, 1LL)) != cudaSuccess ||
        cudaMalloc(&w.err, sizeof(int)) != cudaSuccess) {
        split_free(w);
        throw std::runtime_error("split workspace allocation failed");
    }
    cudaMemset(w.err, 0, sizeof(int));
    set_smem_attr<2, 128, 3>();
    set_smem_attr<3, 64, 2>();
    set_smem_attr<4, 64, 2>();
    set_persist_attr<2, 128, 4>();
    set_persist_attr<3, 64, 3>();
    set_persist_attr<4, 64, 3>();
    w.cap_a = ca;
    w.cap_b = cb;
    w.cap_mn = sz.mn;
    w.slices = nslices;
}

void split_free(SplitWorkspace &w) {
    if (w.a) cudaFree(w.a);
    if (w.b) cudaFree(w.b);
    if (w.ea) cudaFree(w.ea);
    if (w.eb) cudaFree(w.eb);
    if (w.err) cudaFree(w.err);
    w = SplitWorkspace{};
}

bool split_eligible(const GettArgs &g) {
    // enough 128 x 128 tiles to fill the GPU and enough K to amortise slicing.
    // Measured on the CCSDT contractions: the K = 256 ring terms (gathered
    // operands, scattered beta = 1 output) and the M = 64 terms run slower
    // sliced than on the DMMA pipe; the K >= 496 ladder terms run 1.2-2.5x faster.
    long long tiles = ((g.M + 127LL) / 128) * ((g.N + 127LL) / 128);
    return g.M >= 256 && g.N >= 256 && g.K >= 320 && tiles >= 64;
}

int split_launch_count(const GettArgs &, int) { return 3; }

int split_error(const SplitWorkspace &w) {
    int h = 0;
    if (w.err) cudaMemcpy(&h, w.err, sizeof(int), cudaMemcpyDeviceToHost);
    return h;
}

void slice_operand(const double *base, const int *offr, const int *offk, int R, int K, int Kp, int S, signed char *out,
                   long long stride, int *expo, bool kmajor, cudaStream_t s) {
    if (kmajor && Kp <= 512) {
        int blocks = (int)std::min<long long>(((long long)R * 32 + 255) / 256, 148 * 32);
        slice_rows_reg_kernel<<<blocks, 256, 0, s>>>(base, offr, offk, R, K, Kp, S, out, stride, expo);
    } else if (kmajor) {
        int blocks = (int)std::min<long long>(((long long)R * 32 + 255) / 256, 148 * 16);
        slice_rows_kernel<<<blocks, 256, 0, s>>>(base, offr, offk, R, K, Kp, S, out, stride, expo);
    } else {
        int blocks = (int)std::min<long long>((R + SR - 1) / SR, 148 * 8);
        slice_rows_tiled_kernel<<<blocks, 256, 0, s>>>(base, offr, offk, R, K, Kp, S, out, stride, expo);
    }
}

int split_gett(SplitWorkspace &w, const GettArgs &g, int a_kmajor, int b_kmajor, int S, cudaStream_t s,
               int persistent) {
    if (S < 2 || S > 4) throw std::runtime_error("split GETT supports 2..4 slices");
    long long Kp = ((long long)g.K + BKB - 1) / BKB * BKB;
    long long Mr = g.M, Nr = g.N;
    if (Mr * Kp * S > w.cap_a || Nr * Kp * S > w.cap_b || Mr > w.cap_mn || Nr > w.cap_mn)
        throw std::runtime_error("split workspace too small");
    slice_operand(g.A, g.offA_m, g.offA_k, g.M, g.K, (int)Kp, S, w.a, Mr * Kp, w.ea, a_kmajor != 0, s);
    slice_operand(g.B, g.offB_n, g.offB_k, g.N, g.K, (int)Kp, S, w.b, Nr * Kp, w.eb, b_kmajor != 0, s);
    CUtensorMap ta = make_map(w.a, Mr, Kp, S, TM);
    CUtensorMap tb = make_map(w.b, Nr, Kp, S, tile_n(S));
    SplitArgs a{g.C, g.offC_m, g.offC_n, w.ea, w.eb, g.M, g.N, g.K, (int)Kp, g.alpha, g.beta, g.c_nfast, w.err};
    if (persistent) {
        switch (S) {
            case 2: launch_split_persistent<2, 128, 4>(ta, tb, a, s); break;
            case 3: launch_split_persistent<3, 64, 3>(ta, tb, a, s); break;
            case 4: launch_split_persistent<4, 64, 3>(ta, tb, a, s); break;
        }
        return 3;
    }
    switch (S) {
        case 2: launch_split<2, 128, 3>(ta, tb, a, s); break;
        case 3: launch_split<3, 64, 2>(ta, tb, a, s); break;
        case 4: launch_split<4, 64, 2>(ta, tb, a, s); break;
    }
    return 3;
}

}  // namespace ccqb
