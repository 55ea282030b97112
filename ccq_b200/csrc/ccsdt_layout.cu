// ccq's compressed T vector of active-space CCSDt (get_t_sizes_act,
// src/utils/cc_utils.f90:560-630) and the full-block T vector this engine keeps
// (get_t_sizes, :479-559).
//
// ccq stores the active triples as ten rectangular sub-blocks of the four T3
// spin blocks, each a slice of the block's own axes in the block's own axis
// order (the declarations of t3A .. t3D in src/cc_opt_ccsdt/*_update_opt.f,
// e.g. t2B0000_update_opt.f:48-57).  With N0 = froz, N1 = occ_a, N2 = occ_b,
// N3 = orbs, M1 = act_occ_b and M2 = act_unocc_a (1-based Fortran ranges):
//
//   t3A  (N1+1:N3, N1+1:N3, N1+1:M2, N0+1:N1, N0+1:N1, M1+1:N1)   of t3a
//   t3B1 (N2+1:N3, N1+1:N3, N1+1:M2, N0+1:N2, N0+1:N1, M1+1:N1)   of t3b
//   t3B2 (N2+1:M2, M2+1:N3, M2+1:N3, M1+1:N2, N0+1:M1, N0+1:M1)
//   t3B3 (N2+1:M2, M2+1:N3, M2+1:N3, N0+1:N2, N0+1:N1, M1+1:N1)
//   t3B4 (N2+1:N3, N1+1:N3, N1+1:M2, M1+1:N2, N0+1:M1, N0+1:M1)
//   t3C1 (N2+1:N3, N2+1:M2, N1+1:N3, N0+1:N2, M1+1:N2, N0+1:N1)   of t3c
//   t3C2 (M2+1:N3, M2+1:N3, N1+1:M2, N0+1:M1, N0+1:M1, M1+1:N1)
//   t3C3 (M2+1:N3, M2+1:N3, N1+1:M2, N0+1:N2, M1+1:N2, N0+1:N1)
//   t3C4 (N2+1:N3, N2+1:M2, N1+1:N3, N0+1:M1, N0+1:M1, M1+1:N1)
//   t3D  (N2+1:N3, N2+1:N3, N2+1:M2, N0+1:N2, N0+1:N2, M1+1:N2)   of t3d
//
// Compressing copies those slices out of the full blocks; expanding writes each
// compressed element back at its position and at every position its
// antisymmetry relates to it (the same-spin axis groups of the block), so the
// full block is whole again and zero outside the active triples.  T1 and T2 are
// the same in both layouts.  Host code: these run at the boundary only.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/ccq_b200.h"
#include "kernels.cuh"

namespace {

struct Range {
    long long lo, hi;   // 1-based inclusive Fortran bounds lo..hi (empty when hi < lo)
    long long n() const { return hi >= lo ? hi - lo + 1 : 0; }
};

struct Sub {
    int block;           // 0..3: t3a..t3d
    Range r[6];
};

struct Layout {
    long long N0, N1, N2, N3, M1, M2;
    Range full[4][6];
    std::vector<Sub> subs;
    long long t12 = 0;                 // T1 + T2 elements
    long long full_off[4] = {0, 0, 0, 0};   // offsets of T3A..T3D in the full vector
    long long full_size = 0, act_size = 0;

    Layout(const ccq_b200_dims &d, long long m1, long long m2) {
        N0 = d.froz;
        N1 = d.occ_a;
        N2 = d.occ_b;
        N3 = d.orbs;
        M1 = m1;
        M2 = m2;
        const Range va{N1 + 1, N3}, vb{N2 + 1, N3}, oa{N0 + 1, N1}, ob{N0 + 1, N2};
        const Range t3[4][6] = {{va, va, va, oa, oa, oa}, {vb, va, va, ob, oa, oa},
                                {vb, vb, va, ob, ob, oa}, {vb, vb, vb, ob, ob, ob}};
        std::memcpy(full, t3, sizeof(full));
        const long long noa = N1 - N0, nob = N2 - N0, nva = N3 - N1, nvb = N3 - N2;
        t12 = noa * nva + nob * nvb + noa * noa * nva * nva + noa * nob * nva * nvb + nob * nob * nvb * nvb;
        long long off = t12;
        for (int b = 0; b < 4; ++b) {
            full_off[b] = off;
            long long s = 1;
            for (int k = 0; k < 6; ++k) s *= full[b][k].n();
            off += s;
        }
        full_size = off;
        const Range avA{N1 + 1, M2}, avB{N2 + 1, M2}, iv{M2 + 1, N3}, aoA{M1 + 1, N1}, aoB{M1 + 1, N2},
            io{N0 + 1, M1};
        subs = {
            {0, {va, va, avA, oa, oa, aoA}},   // t3A
            {1, {vb, va, avA, ob, oa, aoA}},   // t3B1
            {1, {avB, iv, iv, aoB, io, io}},   // t3B2
            {1, {avB, iv, iv, ob, oa, aoA}},   // t3B3
            {1, {vb, va, avA, aoB, io, io}},   // t3B4
            {2, {vb, avB, va, ob, aoB, oa}},   // t3C1
            {2, {iv, iv, avA, io, io, aoA}},   // t3C2
            {2, {iv, iv, avA, ob, aoB, oa}},   // t3C3
            {2, {vb, avB, va, io, io, aoA}},   // t3C4
            {3, {vb, vb, avB, ob, ob, aoB}},   // t3D
        };
        act_size = t12;
        for (auto &s : subs) {
            long long n = 1;
            for (int k = 0; k < 6; ++k) n *= s.r[k].n();
            act_size += n;
        }
    }
    // column-major offset of Fortran indices x[0..5] in full block b
    long long full_index(int b, const long long *x) const {
        long long o = 0, st = 1;
        for (int k = 0; k < 6; ++k) {
            o += (x[k] - full[b][k].lo) * st;
            st *= full[b][k].n();
        }
        return full_off[b] + o;
    }
};

bool valid(const ccq_b200_dims *d, int64_t m1, int64_t m2) {
    const bool ok = d && d->froz >= 0 && d->occ_a >= d->froz && d->occ_b >= d->froz && d->orbs >= d->occ_a &&
                    d->orbs >= d->occ_b && m1 >= d->froz && m1 <= d->occ_b && m2 >= d->occ_a && m2 <= d->orbs;
    if (!ok) ccqb::set_last_error("CCSDt layout: froz <= act_occ_b <= occ_b and occ_a <= act_unocc_a <= orbs");
    return ok;
}

int bad_length() {
    ccqb::set_last_error("CCSDt layout: vector lengths do not match the full and compressed T vectors");
    return CCQ_B200_EINVAL;
}

// same-spin axis groups of each full block: {axes of a run of equal spins}
const int kGroups[4][4][3] = {
    {{0, 1, 2}, {3, 4, 5}, {-1, -1, -1}, {-1, -1, -1}},   // t3a(a,b,c,i,j,k): all alpha
    {{1, 2, -1}, {4, 5, -1}, {-1, -1, -1}, {-1, -1, -1}}, // t3b(c_b,b,a,k_b,j,i): (b,a), (j,i) alpha
    {{0, 1, -1}, {3, 4, -1}, {-1, -1, -1}, {-1, -1, -1}}, // t3c(c_b,b_b,a,k_b,j_b,i): (c,b), (k,j) beta
    {{0, 1, 2}, {3, 4, 5}, {-1, -1, -1}, {-1, -1, -1}},   // t3d: all beta
};

template <typename F>
void for_each_sub_element(const Layout &L, F f) {
    long long pos = L.t12;
    for (auto &s : L.subs) {
        long long n = 1;
        for (int k = 0; k < 6; ++k) n *= s.r[k].n();
        long long x[6];
        for (long long e = 0; e < n; ++e) {
            long long r = e;
            for (int k = 0; k < 6; ++k) {
                x[k] = s.r[k].lo + r % s.r[k].n();
                r /= s.r[k].n();
            }
            f(s, x, pos + e);
        }
        pos += n;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Device side: the compressed T3 part of a DIIS vector gathered from, and
// scattered back into, the full T3 blocks of a resident T vector.  One thread
// per compressed element; a thread decodes its sub-block and coordinates from
// the ten sub-block geometries (no tables).  The scatter writes every
// antisymmetric copy; elements reached from several compressed positions get
// the same value from each.
// ---------------------------------------------------------------------------
namespace ccqb {

void t3act_geometry(long long froz, long long occ_a, long long occ_b, long long orbs, long long act_occ_b,
                    long long act_unocc_a, T3ActGeom &g) {
    const ccq_b200_dims dims{froz, occ_a, occ_b, orbs};
    const Layout L(dims, act_occ_b, act_unocc_a);
    g.t12 = L.t12;
    long long off = 0;
    for (int s = 0; s < 10; ++s) {
        const Sub &u = L.subs[s];
        g.sub_off[s] = off;
        g.block[s] = u.block;
        long long n = 1;
        for (int k = 0; k < 6; ++k) {
            g.lo[s][k] = (int)(u.r[k].lo - L.full[u.block][k].lo);
            g.n[s][k] = (int)u.r[k].n();
            n *= u.r[k].n();
        }
        off += n;
    }
    g.sub_off[10] = off;
    g.n_act = off;
    for (int b = 0; b < 4; ++b) {
        g.full_off[b] = L.full_off[b];
        for (int k = 0; k < 6; ++k) g.fn[b][k] = (int)L.full[b][k].n();
    }
    g.t3_begin = L.full_off[0];
    g.t3_end = L.full_size;
}

}  // namespace ccqb

namespace {

// the sub-block of compressed element p (sub_off is increasing; empty sub-blocks are passed over) and
// its coordinates in the full block
__device__ __forceinline__ int t3act_decode(const ccqb::T3ActGeom &g, long long p, int x[6]) {
    int s = 0;
    while (s < 9 && p >= g.sub_off[s + 1]) ++s;
    long long e = p - g.sub_off[s];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        x[k] = g.lo[s][k] + (int)(e % g.n[s][k]);
        e /= g.n[s][k];
    }
    return g.block[s];
}

__device__ __forceinline__ long long t3act_full(const ccqb::T3ActGeom &g, int b, const int x[6]) {
    long long o = 0, st = 1;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        o += (long long)x[k] * st;
        st *= g.fn[b][k];
    }
    return g.full_off[b] + o;
}

__global__ void t3act_gather_kernel(ccqb::T3ActGeom g, const double *tvec, double *cvec) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.n_act;
         p += (long long)gridDim.x * blockDim.x) {
        int x[6];
        const int b = t3act_decode(g, p, x);
        cvec[p] = tvec[t3act_full(g, b, x)];
    }
}

__global__ void t3act_scatter_kernel(ccqb::T3ActGeom g, const double *cvec, double *tvec) {
    // permutations of a group of three (with parity); a group of two uses the first two
    const int p3[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 1, 0}, {1, 2, 0}, {2, 0, 1}};
    const int s3[6] = {1, -1, -1, -1, 1, 1};
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.n_act;
         p += (long long)gridDim.x * blockDim.x) {
        int x[6];
        const int b = t3act_decode(g, p, x);
        const double v = cvec[p];
        // same-spin axis groups: t3a, t3d (0,1,2),(3,4,5); t3b (1,2),(4,5); t3c (0,1),(3,4)
        const bool three = b == 0 || b == 3;
        const int g0 = b == 1 ? 1 : 0, g1 = b == 1 ? 4 : 3;
        const int np = three ? 6 : 2, len = three ? 3 : 2;
        for (int u = 0; u < np; ++u)
            for (int w = 0; w < np; ++w) {
                int y[6] = {x[0], x[1], x[2], x[3], x[4], x[5]};
                for (int k = 0; k < len; ++k) {
                    y[g0 + k] = x[g0 + p3[u][k]];
                    y[g1 + k] = x[g1 + p3[w][k]];
                }
                tvec[t3act_full(g, b, y)] = s3[u] * s3[w] * v;
            }
    }
}

int layout_grid(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

namespace ccqb {

void launch_t3act_gather(const T3ActGeom &g, const double *tvec, double *cvec, cudaStream_t s) {
    if (g.n_act) t3act_gather_kernel<<<layout_grid(g.n_act), 256, 0, s>>>(g, tvec, cvec);
}

void launch_t3act_scatter(const T3ActGeom &g, const double *cvec, double *tvec, cudaStream_t s) {
    cudaMemsetAsync(tvec + g.t3_begin, 0, sizeof(double) * (size_t)(g.t3_end - g.t3_begin), s);
    if (g.n_act) t3act_scatter_kernel<<<layout_grid(g.n_act), 256, 0, s>>>(g, cvec, tvec);
}

}  // namespace ccqb

extern "C" {

int64_t ccq_b200_t_size_act(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a) {
    if (!valid(dims, act_occ_b, act_unocc_a)) return CCQ_B200_EINVAL;
    return Layout(*dims, act_occ_b, act_unocc_a).act_size;
}

int ccq_b200_t_compress(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a, const double *t_full,
                        int64_t n_full, double *t_act, int64_t n_act) {
    if (!t_full || !t_act) {
        ccqb::set_last_error("CCSDt layout: null vector");
        return CCQ_B200_EINVAL;
    }
    if (!valid(dims, act_occ_b, act_unocc_a)) return CCQ_B200_EINVAL;
    const Layout L(*dims, act_occ_b, act_unocc_a);
    if (n_full != L.full_size || n_act != L.act_size) return bad_length();
    std::memcpy(t_act, t_full, sizeof(double) * (size_t)L.t12);
    for_each_sub_element(L, [&](const Sub &s, const long long *x, long long p) {
        t_act[p] = t_full[L.full_index(s.block, x)];
    });
    return 0;
}

int ccq_b200_t_expand(const ccq_b200_dims *dims, int64_t act_occ_b, int64_t act_unocc_a, const double *t_act,
                      int64_t n_act, double *t_full, int64_t n_full) {
    if (!t_full || !t_act) {
        ccqb::set_last_error("CCSDt layout: null vector");
        return CCQ_B200_EINVAL;
    }
    if (!valid(dims, act_occ_b, act_unocc_a)) return CCQ_B200_EINVAL;
    const Layout L(*dims, act_occ_b, act_unocc_a);
    if (n_full != L.full_size || n_act != L.act_size) return bad_length();
    std::memcpy(t_full, t_act, sizeof(double) * (size_t)L.t12);
    std::memset(t_full + L.t12, 0, sizeof(double) * (size_t)(L.full_size - L.t12));
    for_each_sub_element(L, [&](const Sub &s, const long long *x, long long p) {
        const double v = t_act[p];
        // every permutation within the block's same-spin axis groups, with its parity
        const int(*g)[3] = kGroups[s.block];
        int len[2];
        for (int q = 0; q < 2; ++q) len[q] = g[q][2] >= 0 ? 3 : 2;
        static const int p3[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 1, 0}, {1, 2, 0}, {2, 0, 1}};
        static const int s3[6] = {1, -1, -1, -1, 1, 1};
        static const int p2[2][3] = {{0, 1, 2}, {1, 0, 2}};
        static const int s2[2] = {1, -1};
        const int n0 = len[0] == 3 ? 6 : 2, n1 = len[1] == 3 ? 6 : 2;
        for (int u = 0; u < n0; ++u)
            for (int w = 0; w < n1; ++w) {
                long long y[6];
                for (int k = 0; k < 6; ++k) y[k] = x[k];
                const int *pu = len[0] == 3 ? p3[u] : p2[u];
                const int *pw = len[1] == 3 ? p3[w] : p2[w];
                for (int k = 0; k < len[0]; ++k) y[g[0][k]] = x[g[0][pu[k]]];
                for (int k = 0; k < len[1]; ++k) y[g[1][k]] = x[g[1][pw[k]]];
                const int sg = (len[0] == 3 ? s3[u] : s2[u]) * (len[1] == 3 ? s3[w] : s2[w]);
                t_full[L.full_index(s.block, y)] = sg * v;
            }
    });
    return 0;
}

}  // extern "C"
