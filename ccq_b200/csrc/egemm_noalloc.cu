// egemm on caller-owned device buffers with no device allocation at all.
//
// The regular egemm entry points stage host arrays through device buffers that
// the library allocates (and grows) itself.  Some hosts of this library cannot
// let it do that: an application whose device memory is entirely carved up by
// its own pool allocator (a framework's caching allocator, or a Fortran driver
// that reserves HBM for its T vectors up front), or a time-critical loop where
// cudaMalloc/cudaFree would synchronise the device and stall other streams.
// For them, ccq_b200_egemm_dev_noalloc takes device pointers for A, B and C and
// keeps the only scratch it needs -- the GETT offset tables -- in the
// fixed-size file-scope array below, which exists once per GPU that loads the
// library and lives until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ccq_b200.h"
#include "kernels.cuh"

namespace {

// Largest k1, k2, k3 accepted: six int32 tables of this length (1.5 MiB).
constexpr long long kNoAllocMaxDim = 65536;
constexpr int kTables = 6;

static __device__ __align__(256) int g_noalloc_tables[kTables * kNoAllocMaxDim];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
int *g_table_addr[kMaxDevices] = {nullptr};

// Host code only sees a stand-in for g_noalloc_tables; its device address is
// looked up once per device with that device current.
int table_address(int **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CCQ_B200_ENODEV;
    if (dev < 0 || dev >= kMaxDevices) return CCQ_B200_ENODEV;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_table_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_tables) != cudaSuccess || !p) return CCQ_B200_ECUDA;
        g_table_addr[dev] = static_cast<int *>(p);
    }
    *out = g_table_addr[dev];
    return 0;
}

// Offset tables of C(k2,k1) = B(k3,k2)^T A(k3,k1) in column-major storage,
// region r of the array holding table r.
__global__ void fill_egemm_tables(int *t, int k1, int k2, int k3) {
    const long long L = kNoAllocMaxDim;
    int n = max(k1, max(k2, k3));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < k1) {
            t[0 * L + i] = i * k3;   // A rows (m)
            t[4 * L + i] = i * k2;   // C rows (m)
        }
        if (i < k3) {
            t[1 * L + i] = i;        // A contraction index
            t[3 * L + i] = i;        // B contraction index
        }
        if (i < k2) {
            t[2 * L + i] = i * k3;   // B columns (n)
            t[5 * L + i] = i;        // C columns (n)
        }
    }
}

}  // namespace

extern "C" int ccq_b200_egemm_dev_noalloc(int64_t k1, int64_t k2, int64_t k3, const double *A, const double *B,
                                          double *C, void *stream) {
    if (k1 < 0 || k2 < 0 || k3 < 0) return CCQ_B200_EINVAL;
    if (k1 > kNoAllocMaxDim || k2 > kNoAllocMaxDim || k3 > kNoAllocMaxDim) return CCQ_B200_ERANGE;
    if (k1 * k3 > INT32_MAX || k2 * k3 > INT32_MAX || k1 * k2 > INT32_MAX) return CCQ_B200_ERANGE;
    if (k1 == 0 || k2 == 0) return 0;
    if (!C || (k3 > 0 && (!A || !B))) return CCQ_B200_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // a launch error pending from earlier work on this thread is not this call's
    (void)cudaGetLastError();
    int *t = nullptr;
    int rc = table_address(&t);
    if (rc) return rc;
    const long long L = kNoAllocMaxDim;
    const long long chunk = ccqb::gett_f64_kchunk(k1, k2, k3);
    if (ccqb::gett_f64_prepare() != cudaSuccess) return CCQ_B200_ECUDA;
    // split-K partial sums are added atomically into C, which must start at zero
    if (k3 == 0 || (k3 + chunk - 1) / chunk > 1) {
        if (cudaMemsetAsync(C, 0, sizeof(double) * (size_t)(k1 * k2), s) != cudaSuccess) return CCQ_B200_ECUDA;
    }
    if (k3 == 0) return cudaGetLastError() == cudaSuccess ? 0 : CCQ_B200_ECUDA;
    long long nmax = k1 > k2 ? (k1 > k3 ? k1 : k3) : (k2 > k3 ? k2 : k3);
    fill_egemm_tables<<<(int)((nmax + 255) / 256), 256, 0, s>>>(t, (int)k1, (int)k2, (int)k3);
    ccqb::GettArgs g{};
    g.A = A;
    g.B = B;
    g.C = C;
    g.offA_m = t + 0 * L;
    g.offA_k = t + 1 * L;
    g.offB_n = t + 2 * L;
    g.offB_k = t + 3 * L;
    g.offC_m = t + 4 * L;
    g.offC_n = t + 5 * L;
    g.M = (int)k1;
    g.N = (int)k2;
    g.K = (int)k3;
    g.alpha = 1.0;
    g.beta = 0;
    g.c_nfast = 1;
    // 16-byte operand / output paths: 16-byte aligned bases, rows starting on even elements
    auto al16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    g.vec_a = k3 % 2 == 0 && al16(A);
    g.vec_b = k3 % 2 == 0 && al16(B);
    g.vec_c = k2 % 2 == 0 && al16(C);
    g.kchunk = (int)chunk;
    ccqb::launch_gett_f64(g, 1, 1, s);
    return cudaGetLastError() == cudaSuccess ? 0 : CCQ_B200_ECUDA;
}
