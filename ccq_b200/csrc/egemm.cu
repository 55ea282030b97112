// dgemm.f90 call surface on host arrays (level-1 boundary of include/ccq_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ccq_b200.h"
#include "kernels.cuh"
#include "split.cuh"

namespace {

std::mutex g_mu;
struct Staging {
    double *a = nullptr, *b = nullptr, *c = nullptr;
    int *tab = nullptr;
    size_t ca = 0, cb = 0, cc = 0, ct = 0;
    cudaStream_t s = nullptr;
    int device = -1;
} g_st;

int grow(void **p, size_t *cap, size_t bytes) {
    if (*cap >= bytes) return 0;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, bytes) != cudaSuccess) return CCQ_B200_ENOMEM;
    *cap = bytes;
    return 0;
}

// C(k2,k1) = sum_k B(k3idx,k2idx) A(k3idx,k1idx), column-major host arrays.
int egemm_impl(long long k1, long long k2, long long k3, const double *A, const double *B, double *C) {
    if (k1 < 0 || k2 < 0 || k3 < 0 || (k1 * k2 > 0 && !C) || (k1 * k3 > 0 && !A) || (k2 * k3 > 0 && !B))
        return CCQ_B200_EINVAL;
    if (k1 > INT32_MAX || k2 > INT32_MAX || k3 > INT32_MAX || k1 * k3 > INT32_MAX || k2 * k3 > INT32_MAX ||
        k1 * k2 > INT32_MAX)
        return CCQ_B200_ERANGE;
    if (k1 == 0 || k2 == 0) return 0;
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CCQ_B200_ENODEV;
    if (g_st.device != dev) {
        g_st = Staging();
        g_st.device = dev;
        if (cudaStreamCreateWithFlags(&g_st.s, cudaStreamNonBlocking) != cudaSuccess) return CCQ_B200_ECUDA;
    }
    size_t na = (size_t)(k1 * k3), nb = (size_t)(k2 * k3), nc = (size_t)(k1 * k2);
    size_t nt = (size_t)(2 * k1 + 2 * k2 + 2 * k3);
    int r = 0;
    if ((r = grow((void **)&g_st.a, &g_st.ca, sizeof(double) * std::max<size_t>(na, 1)))) return r;
    if ((r = grow((void **)&g_st.b, &g_st.cb, sizeof(double) * std::max<size_t>(nb, 1)))) return r;
    if ((r = grow((void **)&g_st.c, &g_st.cc, sizeof(double) * nc))) return r;
    if ((r = grow((void **)&g_st.tab, &g_st.ct, sizeof(int) * nt))) return r;
    std::vector<int> t(nt);
    int *am = t.data(), *ak = am + k1, *bn = ak + k3, *bk = bn + k2, *cm = bk + k3, *cn = cm + k1;
    for (long long i = 0; i < k1; ++i) {
        am[i] = (int)(i * k3);
        cm[i] = (int)(i * k2);
    }
    for (long long i = 0; i < k2; ++i) {
        bn[i] = (int)(i * k3);
        cn[i] = (int)i;
    }
    for (long long i = 0; i < k3; ++i) ak[i] = bk[i] = (int)i;
    cudaStream_t s = g_st.s;
    if (na) cudaMemcpyAsync(g_st.a, A, sizeof(double) * na, cudaMemcpyHostToDevice, s);
    if (nb) cudaMemcpyAsync(g_st.b, B, sizeof(double) * nb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(g_st.tab, t.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s);
    int *d = g_st.tab;
    ccqb::GettArgs g{};
    g.A = g_st.a;
    g.B = g_st.b;
    g.C = g_st.c;
    g.offA_m = d;
    g.offA_k = d + k1;
    g.offB_n = d + k1 + k3;
    g.offB_k = d + k1 + k3 + k2;
    g.offC_m = d + k1 + 2 * k3 + k2;
    g.offC_n = d + 2 * k1 + 2 * k3 + k2;
    g.M = (int)k1;
    g.N = (int)k2;
    g.K = (int)k3;
    g.alpha = 1.0;
    g.beta = 0;
    g.c_nfast = 1;
    // 16-byte operand / output paths: rows of A, B (C) start on even elements
    g.vec_a = g.vec_b = (k3 % 2 == 0);
    g.vec_c = (k2 % 2 == 0);
    g.kchunk = ccqb::gett_f64_kchunk(k1, k2, k3);
    if (ccqb::gett_f64_prepare() != cudaSuccess) return CCQ_B200_ECUDA;
    if (k3 == 0 || (k3 + g.kchunk - 1) / g.kchunk > 1) cudaMemsetAsync(g_st.c, 0, sizeof(double) * nc, s);
    if (k3 > 0) ccqb::launch_gett_f64(g, 1, 1, s);
    cudaMemcpyAsync(C, g_st.c, sizeof(double) * nc, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return CCQ_B200_ECUDA;
    if (cudaGetLastError() != cudaSuccess) return CCQ_B200_ECUDA;
    return 0;
}

ccqb::SplitWorkspace g_split;

// Split-precision egemm (same layout as egemm_impl), nslices int8 slices.
int egemm_split_impl(long long k1, long long k2, long long k3, const double *A, const double *B, double *C, int S,
                     int persistent) {
    if (k1 <= 0 || k2 <= 0 || k3 <= 0 || !A || !B || !C || S < 2 || S > 4) return CCQ_B200_EINVAL;
    if (k1 > INT32_MAX || k2 > INT32_MAX || k3 > INT32_MAX || k1 * k3 > INT32_MAX || k2 * k3 > INT32_MAX ||
        k1 * k2 > INT32_MAX)
        return CCQ_B200_ERANGE;
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CCQ_B200_ENODEV;
    if (g_st.device != dev) {
        g_st = Staging();
        g_st.device = dev;
        if (cudaStreamCreateWithFlags(&g_st.s, cudaStreamNonBlocking) != cudaSuccess) return CCQ_B200_ECUDA;
    }
    size_t na = (size_t)(k1 * k3), nb = (size_t)(k2 * k3), nc = (size_t)(k1 * k2);
    size_t nt = (size_t)(2 * k1 + 2 * k2 + 2 * k3);
    int rc = 0;
    if ((rc = grow((void **)&g_st.a, &g_st.ca, sizeof(double) * na))) return rc;
    if ((rc = grow((void **)&g_st.b, &g_st.cb, sizeof(double) * nb))) return rc;
    if ((rc = grow((void **)&g_st.c, &g_st.cc, sizeof(double) * nc))) return rc;
    if ((rc = grow((void **)&g_st.tab, &g_st.ct, sizeof(int) * nt))) return rc;
    std::vector<int> t(nt);
    int *am = t.data(), *ak = am + k1, *bn = ak + k3, *bk = bn + k2, *cm = bk + k3, *cn = cm + k1;
    for (long long i = 0; i < k1; ++i) {
        am[i] = (int)(i * k3);
        cm[i] = (int)(i * k2);
    }
    for (long long i = 0; i < k2; ++i) {
        bn[i] = (int)(i * k3);
        cn[i] = (int)i;
    }
    for (long long i = 0; i < k3; ++i) ak[i] = bk[i] = (int)i;
    cudaStream_t s = g_st.s;
    cudaMemcpyAsync(g_st.a, A, sizeof(double) * na, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(g_st.b, B, sizeof(double) * nb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(g_st.tab, t.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s);
    int *d = g_st.tab;
    ccqb::GettArgs g{};
    g.A = g_st.a;
    g.B = g_st.b;
    g.C = g_st.c;
    g.offA_m = d;
    g.offA_k = d + k1;
    g.offB_n = d + k1 + k3;
    g.offB_k = d + k1 + k3 + k2;
    g.offC_m = d + k1 + 2 * k3 + k2;
    g.offC_n = d + 2 * k1 + 2 * k3 + k2;
    g.M = (int)k1;
    g.N = (int)k2;
    g.K = (int)k3;
    g.alpha = 1.0;
    g.beta = 0;
    g.c_nfast = 1;
    g.kchunk = (int)k3;
    g.c_nfast = 1;
    try {
        long long kp = (k3 + 63) / 64 * 64;
        ccqb::split_reserve(g_split, ccqb::SplitSizes{k1 * kp, k2 * kp, std::max(k1, k2)}, S);
        ccqb::split_gett(g_split, g, 1, 1, S, s, persistent);
    } catch (const std::exception &) {
        return CCQ_B200_ECUDA;
    }
    cudaMemcpyAsync(C, g_st.c, sizeof(double) * nc, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return CCQ_B200_ECUDA;
    if (cudaGetLastError() != cudaSuccess) return CCQ_B200_ECUDA;
    if (ccqb::split_error(g_split)) return CCQ_B200_ECUDA;
    return 0;
}

}  // namespace

extern "C" {

int ccq_b200_egemm_split(int64_t k1, int64_t k2, int64_t k3, const double *A, const double *B, double *C,
                         int64_t nslices) {
    return egemm_split_impl(k1, k2, k3, A, B, C, (int)nslices, 0);
}

int ccq_b200_egemm_split_kernel(int64_t k1, int64_t k2, int64_t k3, const double *A, const double *B, double *C,
                                int64_t nslices, int64_t persistent) {
    return egemm_split_impl(k1, k2, k3, A, B, C, (int)nslices, persistent ? 1 : 0);
}


int ccq_b200_egemm(int64_t k1, int64_t k2, int64_t k3, const double *A, const double *B, double *C) {
    return egemm_impl(k1, k2, k3, A, B, C);
}

// egemm1: C(k1) = A(k3,k1)^T B(k3)  ==  egemm with k2 = 1 and B as a column.
int ccq_b200_egemm1(int64_t k1, int64_t k3, const double *A, const double *B, double *C) {
    return egemm_impl(k1, 1, k3, A, B, C);
}

// egemm2: C(k2) = B(k3,k2)^T A(k3)  ==  egemm with k1 = 1.
int ccq_b200_egemm2(int64_t k2, int64_t k3, const double *A, const double *B, double *C) {
    return egemm_impl(1, k2, k3, A, B, C);
}

void egemm_(const int64_t *k1, const int64_t *k2, const int64_t *k3, const double *A, const double *B, double *C) {
    if (egemm_impl(*k1, *k2, *k3, A, B, C) != 0) {
        fprintf(stderr, "egemm: ccq_b200 device GEMM failed\n");
        exit(1);
    }
}
void egemm1_(const int64_t *k1, const int64_t *k3, const double *A, const double *B, double *C) {
    if (egemm_impl(*k1, 1, *k3, A, B, C) != 0) {
        fprintf(stderr, "egemm1: ccq_b200 device GEMV failed\n");
        exit(1);
    }
}
void egemm2_(const int64_t *k2, const int64_t *k3, const double *A, const double *B, double *C) {
    if (egemm_impl(1, *k2, *k3, A, B, C) != 0) {
        fprintf(stderr, "egemm2: ccq_b200 device GEMV failed\n");
        exit(1);
    }
}

}  // extern "C"
