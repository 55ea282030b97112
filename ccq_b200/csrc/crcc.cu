// CR-CC(2,3) kernels; see crcc.cuh for the role of each.
#include "crcc.cuh"

namespace ccqb {

namespace {

// element of a C-order rank-4 array with extents (n1, n2, n3) for the last three axes
__device__ __forceinline__ double at4(const double *p, int a, int b, int c, int d, int n1, int n2, int n3) {
    return __ldg(p + ((static_cast<long long>(a) * n1 + b) * n2 + c) * n3 + d);
}

// Hbar one-body diagonal h(p,p) of one spin (sigma = 0 alpha, 1 beta), full-range p:
//   occupied  h(i,i) = f~(i,i) + 1/2 sum_{m e f} <im||ef> t(ef,im)
//   virtual   h(a,a) = f~(a,a) - 1/2 sum_{m n f} <mn||af> t(af,mn)
// with the spin sums written out on the stored blocks.
__device__ double hbar1(const CrDiagArgs &g, int sigma, int p) {
    const int n = g.n, oa = g.oa, ob = g.ob, va = g.va, vb = g.vb;
    double s = 0.0;
    if (sigma == 0) {
        s = __ldg(g.FA + static_cast<long long>(p) * n + p);
        if (p < oa) {
            const int i = p;
            double x = 0.0, y = 0.0;
            for (int m = 0; m < oa; ++m)
                for (int e = 0; e < va; ++e)
                    for (int f = 0; f < va; ++f)
                        x += at4(g.VAA0, i, m, oa + e, oa + f, n, n, n) * at4(g.T2A, i, m, e, f, oa, va, va);
            for (int m = 0; m < ob; ++m)
                for (int e = 0; e < va; ++e)
                    for (int f = 0; f < vb; ++f)
                        y += at4(g.VAB0, i, m, oa + e, ob + f, n, n, n) * at4(g.T2B, i, m, e, f, ob, va, vb);
            s += 0.5 * x + y;
        } else {
            const int a = p - oa;
            double x = 0.0, y = 0.0;
            for (int m = 0; m < oa; ++m)
                for (int q = 0; q < oa; ++q)
                    for (int f = 0; f < va; ++f)
                        x += at4(g.VAA0, m, q, p, oa + f, n, n, n) * at4(g.T2A, m, q, a, f, oa, va, va);
            for (int m = 0; m < oa; ++m)
                for (int q = 0; q < ob; ++q)
                    for (int f = 0; f < vb; ++f)
                        y += at4(g.VAB0, m, q, p, ob + f, n, n, n) * at4(g.T2B, m, q, a, f, ob, va, vb);
            s -= 0.5 * x + y;
        }
    } else {
        s = __ldg(g.FB + static_cast<long long>(p) * n + p);
        if (p < ob) {
            const int i = p;
            double x = 0.0, y = 0.0;
            for (int m = 0; m < ob; ++m)
                for (int e = 0; e < vb; ++e)
                    for (int f = 0; f < vb; ++f)
                        x += at4(g.VBB0, i, m, ob + e, ob + f, n, n, n) * at4(g.T2C, i, m, e, f, ob, vb, vb);
            for (int m = 0; m < oa; ++m)
                for (int e = 0; e < va; ++e)
                    for (int f = 0; f < vb; ++f)
                        y += at4(g.VAB0, m, i, oa + e, ob + f, n, n, n) * at4(g.T2B, m, i, e, f, ob, va, vb);
            s += 0.5 * x + y;
        } else {
            const int a = p - ob;
            double x = 0.0, y = 0.0;
            for (int m = 0; m < ob; ++m)
                for (int q = 0; q < ob; ++q)
                    for (int f = 0; f < vb; ++f)
                        x += at4(g.VBB0, m, q, p, ob + f, n, n, n) * at4(g.T2C, m, q, a, f, ob, vb, vb);
            for (int m = 0; m < oa; ++m)
                for (int q = 0; q < ob; ++q)
                    for (int f = 0; f < va; ++f)
                        y += at4(g.VAB0, m, q, oa + f, p, n, n, n) * at4(g.T2B, m, q, f, a, ob, va, vb);
            s -= 0.5 * x + y;
        }
    }
    return s;
}

// Hbar two-body diagonal h[p,q,p,q] for a same-spin pair (sigma), full-range p, q:
//   occ-occ  v~[ijij] + 1/2 sum_{ef} <ij||ef> t(ef,ij)
//   vir-vir  v~[abab] + 1/2 sum_{mn} <mn||ab> t(ab,mn)
//   vir-occ  v~[aiai] - sum_{nf} <in||af> t(af,in)   (symmetric: h[i,a,i,a] = h[a,i,a,i])
__device__ double hbar2_same(const CrDiagArgs &g, int sigma, int p, int q) {
    const int n = g.n;
    const int o = sigma ? g.ob : g.oa, v = sigma ? g.vb : g.va;
    const double *V = sigma ? g.VBB : g.VAA;
    const double *V0 = sigma ? g.VBB0 : g.VAA0;
    const double *T = sigma ? g.T2C : g.T2A;
    if (p < o && q >= o) {
        const int t = p;
        p = q;
        q = t;
    }
    double s = at4(V, p, q, p, q, n, n, n);
    if (p < o && q < o) {
        double x = 0.0;
        for (int e = 0; e < v; ++e)
            for (int f = 0; f < v; ++f) x += at4(V0, p, q, o + e, o + f, n, n, n) * at4(T, p, q, e, f, o, v, v);
        s += 0.5 * x;
    } else if (p >= o && q >= o) {
        double x = 0.0;
        for (int m = 0; m < o; ++m)
            for (int k = 0; k < o; ++k) x += at4(V0, m, k, p, q, n, n, n) * at4(T, m, k, p - o, q - o, o, v, v);
        s += 0.5 * x;
    } else {
        // p virtual (a), q occupied (i)
        const int a = p - o, i = q;
        double x = 0.0, y = 0.0;
        for (int k = 0; k < o; ++k)
            for (int f = 0; f < v; ++f) x += at4(V0, i, k, p, o + f, n, n, n) * at4(T, i, k, a, f, o, v, v);
        if (sigma == 0) {
            for (int k = 0; k < g.ob; ++k)
                for (int f = 0; f < g.vb; ++f)
                    y += at4(g.VAB0, i, k, p, g.ob + f, n, n, n) * at4(g.T2B, i, k, a, f, g.ob, g.va, g.vb);
        } else {
            for (int k = 0; k < g.oa; ++k)
                for (int f = 0; f < g.va; ++f)
                    y += at4(g.VAB0, k, i, g.oa + f, p, n, n, n) * at4(g.T2B, k, i, f, a, g.ob, g.va, g.vb);
        }
        s -= x + y;
    }
    return s;
}

// h[p,q,p,q] for p alpha, q beta (full range)
__device__ double hbar2_ab(const CrDiagArgs &g, int p, int q) {
    const int n = g.n, oa = g.oa, ob = g.ob, va = g.va, vb = g.vb;
    double s = at4(g.VAB, p, q, p, q, n, n, n);
    double x = 0.0;
    if (p < oa && q < ob) {
        for (int e = 0; e < va; ++e)
            for (int f = 0; f < vb; ++f)
                x += at4(g.VAB0, p, q, oa + e, ob + f, n, n, n) * at4(g.T2B, p, q, e, f, ob, va, vb);
        s += x;
    } else if (p >= oa && q >= ob) {
        for (int m = 0; m < oa; ++m)
            for (int k = 0; k < ob; ++k)
                x += at4(g.VAB0, m, k, p, q, n, n, n) * at4(g.T2B, m, k, p - oa, q - ob, ob, va, vb);
        s += x;
    } else if (p >= oa) {
        // alpha virtual a = p, beta occupied i = q
        for (int k = 0; k < oa; ++k)
            for (int f = 0; f < vb; ++f)
                x += at4(g.VAB0, k, q, p, ob + f, n, n, n) * at4(g.T2B, k, q, p - oa, f, ob, va, vb);
        s -= x;
    } else {
        // alpha occupied i = p, beta virtual a = q
        for (int k = 0; k < ob; ++k)
            for (int f = 0; f < va; ++f)
                x += at4(g.VAB0, p, k, oa + f, q, n, n, n) * at4(g.T2B, p, k, f, q - ob, ob, va, vb);
        s -= x;
    }
    return s;
}

// three-body sums of cal_d3, full-range indices; zero outside their index ranges
//   W1A[x][p][q] = sum_e <pq||xe> t(xe,pq)  x alpha vir, p q alpha occ        (d3a1)
//   W1B           x alpha vir, p alpha occ, q beta occ, e beta                (d3b1)
//   W1C           x beta vir,  p alpha occ, q beta occ, e alpha               (d3c1)
//   W1D           x beta vir,  p q beta occ, e beta from w1d_e0               (d3d1)
//   W2A[x][z][y] = sum_m <ym||xz> t(xz,ym)  x z alpha vir, y alpha occ        (-d3a2)
//   W2B           x alpha, z beta vir, y alpha occ, m beta                     (-d3b2)
//   W2C           x alpha, z beta vir, y beta occ, m alpha                     (-d3c2)
//   W2D           x z beta vir, y beta occ                                     (-d3d2)
__device__ double w1(const CrDiagArgs &g, int c, int x, int p, int q) {
    const int n = g.n, oa = g.oa, ob = g.ob, va = g.va, vb = g.vb;
    double s = 0.0;
    switch (c) {
        case 0:
            if (x < oa || p >= oa || q >= oa) return 0.0;
            for (int e = 0; e < va; ++e)
                s += at4(g.VAA0, p, q, x, oa + e, n, n, n) * at4(g.T2A, p, q, x - oa, e, oa, va, va);
            return s;
        case 1:
            if (x < oa || p >= oa || q >= ob) return 0.0;
            for (int e = 0; e < vb; ++e)
                s += at4(g.VAB0, p, q, x, ob + e, n, n, n) * at4(g.T2B, p, q, x - oa, e, ob, va, vb);
            return s;
        case 2:
            if (x < ob || p >= oa || q >= ob) return 0.0;
            for (int e = 0; e < va; ++e)
                s += at4(g.VAB0, p, q, oa + e, x, n, n, n) * at4(g.T2B, p, q, e, x - ob, ob, va, vb);
            return s;
        default:
            if (x < ob || p >= ob || q >= ob) return 0.0;
            for (int e = g.w1d_e0; e < vb; ++e)
                s += at4(g.VBB0, p, q, x, ob + e, n, n, n) * at4(g.T2C, p, q, x - ob, e, ob, vb, vb);
            return s;
    }
}

__device__ double w2(const CrDiagArgs &g, int c, int x, int z, int y) {
    const int n = g.n, oa = g.oa, ob = g.ob, va = g.va, vb = g.vb;
    double s = 0.0;
    switch (c) {
        case 0:
            if (x < oa || z < oa || y >= oa) return 0.0;
            for (int m = 0; m < oa; ++m)
                s += at4(g.VAA0, y, m, x, z, n, n, n) * at4(g.T2A, y, m, x - oa, z - oa, oa, va, va);
            return s;
        case 1:
            if (x < oa || z < ob || y >= oa) return 0.0;
            for (int m = 0; m < ob; ++m)
                s += at4(g.VAB0, y, m, x, z, n, n, n) * at4(g.T2B, y, m, x - oa, z - ob, ob, va, vb);
            return s;
        case 2:
            if (x < oa || z < ob || y >= ob) return 0.0;
            for (int m = 0; m < oa; ++m)
                s += at4(g.VAB0, m, y, x, z, n, n, n) * at4(g.T2B, m, y, x - oa, z - ob, ob, va, vb);
            return s;
        default:
            if (x < ob || z < ob || y >= ob) return 0.0;
            for (int m = 0; m < ob; ++m)
                s += at4(g.VBB0, y, m, x, z, n, n, n) * at4(g.T2C, y, m, x - ob, z - ob, ob, vb, vb);
            return s;
    }
}

__global__ void crdiag_kernel(CrDiagArgs g) {
    const long long n = g.n, n2 = n * n, n3 = n2 * n;
    const long long total = 2 * n + 3 * n2 + 8 * n3;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        long long r = t;
        if (r < 2 * n) {
            const int sigma = (int)(r / n), p = (int)(r % n);
            (sigma ? g.HDB : g.HDA)[p] = hbar1(g, sigma, p);
            continue;
        }
        r -= 2 * n;
        if (r < 3 * n2) {
            const int w = (int)(r / n2);
            const int p = (int)((r % n2) / n), q = (int)(r % n);
            double v = 0.0;
            if (w == 1) {
                v = hbar2_ab(g, p, q);
            } else if (p != q) {
                v = hbar2_same(g, w == 0 ? 0 : 1, p, q);
            }
            (w == 0 ? g.H2AA : (w == 1 ? g.H2AB : g.H2BB))[r % n2] = v;
            continue;
        }
        r -= 3 * n2;
        const int w = (int)(r / n3);
        const long long e = r % n3;
        const int i0 = (int)(e / n2), i1 = (int)((e / n) % n), i2 = (int)(e % n);
        if (w < 4)
            g.W1[w][e] = w1(g, w, i0, i1, i2);
        else
            g.W2[w - 4][e] = w2(g, w - 4, i0, i1, i2);
    }
}

__device__ __forceinline__ double h2pair(const CrccArgs &a, int s1, int p, int s2, int q) {
    const long long n = a.n;
    if (s1 == 0 && s2 == 0) return __ldg(a.h2aa + p * n + q);
    if (s1 == 1 && s2 == 1) return __ldg(a.h2bb + p * n + q);
    return s1 == 0 ? __ldg(a.h2ab + p * n + q) : __ldg(a.h2ab + q * n + p);
}

__device__ __forceinline__ int w1case(int sx, int sp, int sq) {
    if (sx == 0 && sp == 0 && sq == 0) return 0;
    if (sx == 0 && sp == 0 && sq == 1) return 1;
    if (sx == 1 && sp == 0 && sq == 1) return 2;
    if (sx == 1 && sp == 1 && sq == 1) return 3;
    return -1;
}

__device__ __forceinline__ int w2case(int sx, int sz, int sy) {
    if (sx == 0 && sz == 0 && sy == 0) return 0;
    if (sx == 0 && sz == 1 && sy == 0) return 1;
    if (sx == 0 && sz == 1 && sy == 1) return 2;
    if (sx == 1 && sz == 1 && sy == 1) return 3;
    return -1;
}

__global__ void __launch_bounds__(256) crcc_sum_kernel(CrccArgs a) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const long long n = a.n, n2 = n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.total;
         t += (long long)gridDim.x * blockDim.x) {
        int x[6];
        long long r = t;
        for (int d = 5; d >= 0; --d) {
            x[d] = (int)(r % a.dims[d]);
            r /= a.dims[d];
        }
        // unique triples: increasing indices within each same-spin run
        bool canon = true;
        for (int k = 0; k < 2; ++k)
            if (a.spin[k] == a.spin[k + 1] && (x[k] >= x[k + 1] || x[3 + k] >= x[4 + k])) canon = false;
        if (!canon) continue;
        int po[3], pv[3], s[3];
        for (int k = 0; k < 3; ++k) {
            s[k] = a.spin[k];
            po[k] = x[k];
            pv[k] = a.off[s[k]] + x[3 + k];
        }
        // crcc23's active-space skip (src/mm_correct.f90:131,190,244,300)
        if (max(po[0], max(po[1], po[2])) >= a.act_occ_lo && min(pv[0], min(pv[1], pv[2])) < a.act_vir_hi)
            continue;
        const double lm = __ldg(a.L + t) * __ldg(a.M + t);
        double da = 0.0, db = 0.0;
        for (int k = 0; k < 3; ++k) {
            da += __ldg(a.fd[s[k]] + po[k]) - __ldg(a.fd[s[k]] + pv[k]);
            db += __ldg(a.hd[s[k]] + po[k]) - __ldg(a.hd[s[k]] + pv[k]);
        }
        double dc = db;
        for (int k = 0; k < 3; ++k)
            for (int l = k + 1; l < 3; ++l)
                dc -= h2pair(a, s[k], po[k], s[l], po[l]) + h2pair(a, s[k], pv[k], s[l], pv[l]);
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) dc += h2pair(a, s[k], pv[k], s[l], po[l]);
        double dd = dc;
        for (int k = 0; k < 3; ++k)
            for (int p = 0; p < 3; ++p)
                for (int q = p + 1; q < 3; ++q) {
                    const int c = w1case(s[k], s[p], s[q]);
                    if (c >= 0) dd += __ldg(a.w1[c] + (pv[k] * n + po[p]) * n + po[q]);
                }
        for (int p = 0; p < 3; ++p)
            for (int q = p + 1; q < 3; ++q)
                for (int k = 0; k < 3; ++k) {
                    const int c = w2case(s[p], s[q], s[k]);
                    if (c >= 0) dd += __ldg(a.w2[c] + (pv[p] * n + pv[q]) * n + po[k]);
                }
        (void)n2;
        acc[0] += lm / da;
        acc[1] += lm / db;
        acc[2] += lm / dc;
        acc[3] += lm / dd;
    }
    __shared__ double red[4][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < 4; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        atomicAdd(a.e23 + threadIdx.x, v);
    }
}

__global__ void lenergy_kernel(const double *norm, const double *ecor, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *out = sqrt(*norm) + *ecor;
}

}  // namespace

void launch_crdiag(const CrDiagArgs &a, cudaStream_t s) {
    const long long n = a.n;
    const long long total = 2 * n + 3 * n * n + 8 * n * n * n;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    crdiag_kernel<<<(int)blocks, 256, 0, s>>>(a);
}

void launch_crcc_sum(const CrccArgs &a, cudaStream_t s) {
    long long blocks = (a.total + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    crcc_sum_kernel<<<(int)blocks, 256, 0, s>>>(a);
}

void launch_lenergy(const double *norm, const double *ecor, double *out, cudaStream_t s) {
    lenergy_kernel<<<1, 32, 0, s>>>(norm, ecor, out);
}

}  // namespace ccqb
