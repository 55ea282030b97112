// FCIDUMP integral reader: the unique one- and two-electron integrals of a
// FCIDUMP file expanded into ccq's dense e1int(n,n) and e2int(n,n,n,n)
// (Fortran order, physicist <ij|ab> = chemist (ia|jb)), on the host or
// straight into device memory.
//
// Follows the reference's reader:
//   header       get_fcidump (src/parser.f90:260-313): lines up to the first
//                one containing "END"; NORB and NELEC by parse_key_val
//                (src/utils/utils.F90:416-462): the value runs from the "="
//                after the key to the next comma; the END line itself is not
//                parsed
//   integrals    load_fcidump (src/integrals.f90:93-210): records
//                "val i a j b" read list-directed (a record may continue on
//                the next line; whatever follows the fifth value on its line
//                is skipped; reading stops at the end of the file or at the
//                first record that does not parse)
//   orbital order  the orbitals are renumbered by the energies of the
//                "val i 0 0 0" records, ascending, ties in file order
//                (insertion_rank, src/external/ranking.f90:84-141); orbitals
//                without such a record count as energy 0
//   expansion    i a j b all nonzero: the eight real-orbital permutations of
//                (ia|jb) into e2int; i a nonzero, j = b = 0: e1int(i,a) and
//                e1int(a,i); all zero: nuclear repulsion; records are applied
//                in file order, so a later record overwrites an earlier one
//                at the same element
// Differences: a header without "END" or an index outside 1..NORB is an error
// here (the reference loops forever or writes out of bounds).
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ccq_b200.h"
#include "kernels.cuh"

namespace {

struct FciRecord {
    double val;
    int i, a, j, b;   // 1-based as in the file (0 = absent)
};

struct FciFile {
    long long norb = -1, nelec = -1;
    std::vector<FciRecord> recs;
};

struct FciError : std::runtime_error {
    int code;
    FciError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// parse_key_val + list-directed integer read of the value
bool key_value(const std::string &line, const char *key, long long *out) {
    size_t k = line.find(key);
    if (k == std::string::npos) return false;
    size_t comma = line.find(',', k);
    size_t eq = line.find('=', k);
    if (eq == std::string::npos || (comma != std::string::npos && eq > comma))
        throw FciError(CCQ_B200_EINVAL, std::string("FCIDUMP header: no '=' after ") + key);
    std::string val = line.substr(eq + 1, comma == std::string::npos ? std::string::npos : comma - eq - 1);
    const char *p = val.c_str();
    while (*p && isspace((unsigned char)*p)) ++p;
    char *end = nullptr;
    long long v = strtoll(p, &end, 10);
    if (end == p) throw FciError(CCQ_B200_EINVAL, std::string("FCIDUMP header: bad value of ") + key);
    *out = v;
    return true;
}

// list-directed tokens of one record: blanks and commas separate values
void split_tokens(const std::string &line, std::vector<std::string> &tok) {
    tok.clear();
    size_t i = 0, n = line.size();
    while (i < n) {
        while (i < n && (isspace((unsigned char)line[i]) || line[i] == ',')) ++i;
        size_t s = i;
        while (i < n && !isspace((unsigned char)line[i]) && line[i] != ',') ++i;
        if (i > s) tok.push_back(line.substr(s, i - s));
    }
}

bool parse_real(std::string t, double *v) {
    for (auto &ch : t)
        if (ch == 'D' || ch == 'd') ch = 'E';
    char *end = nullptr;
    *v = strtod(t.c_str(), &end);
    return end != t.c_str() && *end == '\0';
}

bool parse_int(const std::string &t, int *v) {
    char *end = nullptr;
    long long x = strtoll(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != '\0' || x < -2147483647LL || x > 2147483647LL) return false;
    *v = (int)x;
    return true;
}

FciFile read_fcidump(const char *path, bool records) {
    std::ifstream in(path);
    if (!in) throw FciError(CCQ_B200_EINVAL, std::string("FCIDUMP file not found: ") + path);
    FciFile f;
    std::string line;
    bool ended = false;
    while (std::getline(in, line)) {
        if (line.find("END") != std::string::npos) {
            ended = true;
            break;
        }
        key_value(line, "NORB", &f.norb);
        key_value(line, "NELEC", &f.nelec);
    }
    if (!ended) throw FciError(CCQ_B200_EINVAL, "FCIDUMP header has no END line");
    if (!records) return f;
    std::vector<std::string> tok, acc;
    while (true) {
        acc.clear();
        bool eof = false;
        while (acc.size() < 5) {
            if (!std::getline(in, line)) {
                eof = true;
                break;
            }
            split_tokens(line, tok);
            acc.insert(acc.end(), tok.begin(), tok.end());
        }
        if (eof) break;
        FciRecord r;
        if (!parse_real(acc[0], &r.val) || !parse_int(acc[1], &r.i) || !parse_int(acc[2], &r.a) ||
            !parse_int(acc[3], &r.j) || !parse_int(acc[4], &r.b))
            break;
        f.recs.push_back(r);
    }
    return f;
}

// new index (0-based) of every original orbital: stable ascending rank of the orbital energies
std::vector<int> orbital_order(const FciFile &f, int n) {
    std::vector<double> eig(n, 0.0);
    for (const auto &r : f.recs)
        if (r.i != 0 && r.a + r.j + r.b == 0) {
            if (r.i < 1 || r.i > n) throw FciError(CCQ_B200_EINVAL, "FCIDUMP orbital index outside 1..NORB");
            eig[r.i - 1] = r.val;
        }
    std::vector<int> rank(n);
    std::iota(rank.begin(), rank.end(), 0);
    std::stable_sort(rank.begin(), rank.end(), [&](int x, int y) { return eig[x] < eig[y]; });
    std::vector<int> inv(n);
    for (int k = 0; k < n; ++k) inv[rank[k]] = k;
    return inv;
}

__host__ __device__ inline long long e2pos(long long n, int i, int j, int a, int b) {
    return i + n * (j + n * (a + n * (long long)b));
}

// the eight positions of (ia|jb) in e2int (Fortran order), renumbered indices
__host__ __device__ inline void eight(long long n, int i, int a, int j, int b, long long (&p)[8]) {
    p[0] = e2pos(n, i, j, a, b);
    p[1] = e2pos(n, j, i, b, a);
    p[2] = e2pos(n, a, b, i, j);
    p[3] = e2pos(n, b, a, j, i);
    p[4] = e2pos(n, a, j, i, b);
    p[5] = e2pos(n, b, i, j, a);
    p[6] = e2pos(n, i, b, a, j);
    p[7] = e2pos(n, j, a, b, i);
}

struct Expanded {
    std::vector<double> val;
    std::vector<int> idx;   // 4 renumbered 0-based indices (i, a, j, b) per two-body record
    double enuc = 0.0;
};

// one- and zero-body records applied on the host; two-body records renumbered and checked
Expanded expand(const FciFile &f, int n, double *e1) {
    std::vector<int> inv = orbital_order(f, n);
    std::fill(e1, e1 + (size_t)n * n, 0.0);
    Expanded x;
    for (const auto &r : f.recs) {
        auto ok = [&](int q) { return q >= 1 && q <= n; };
        if (r.i != 0 && r.a != 0 && r.j != 0 && r.b != 0) {
            if (!ok(r.i) || !ok(r.a) || !ok(r.j) || !ok(r.b))
                throw FciError(CCQ_B200_EINVAL, "FCIDUMP orbital index outside 1..NORB");
            x.val.push_back(r.val);
            x.idx.insert(x.idx.end(), {inv[r.i - 1], inv[r.a - 1], inv[r.j - 1], inv[r.b - 1]});
        } else if (r.i != 0 && r.a != 0 && r.j + r.b == 0) {
            if (!ok(r.i) || !ok(r.a)) throw FciError(CCQ_B200_EINVAL, "FCIDUMP orbital index outside 1..NORB");
            const int i = inv[r.i - 1], a = inv[r.a - 1];
            e1[i + (size_t)n * a] = r.val;
            e1[a + (size_t)n * i] = r.val;
        } else if (r.i + r.a + r.j + r.b == 0) {
            x.enuc = r.val;
        }
    }
    return x;
}

// Device expansion, last record wins: pass 1 marks every element with the
// highest record number that writes it, pass 2 lets only that record store.
__global__ void fci_owner_kernel(const int *idx, long long nrec, long long n, int *owner) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
         r += (long long)gridDim.x * blockDim.x) {
        long long p[8];
        eight(n, idx[4 * r], idx[4 * r + 1], idx[4 * r + 2], idx[4 * r + 3], p);
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicMax(owner + p[q], (int)r);
    }
}

__global__ void fci_store_kernel(const int *idx, const double *val, long long nrec, long long n, const int *owner,
                                 double *e2) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
         r += (long long)gridDim.x * blockDim.x) {
        long long p[8];
        eight(n, idx[4 * r], idx[4 * r + 1], idx[4 * r + 2], idx[4 * r + 3], p);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (owner[p[q]] == (int)r) e2[p[q]] = val[r];
    }
}

int norb_checked(const FciFile &f, int64_t norb) {
    if (norb < 1 || norb > 4096) throw FciError(CCQ_B200_EINVAL, "FCIDUMP: norb out of range");
    if (f.norb >= 0 && f.norb != norb)
        throw FciError(CCQ_B200_EINVAL, "FCIDUMP: NORB of the header differs from the orbital count asked for");
    return (int)norb;
}

int fci_fail(const FciError &e) {
    ccqb::set_last_error(e.what());
    return e.code;
}

}  // namespace

extern "C" int ccq_b200_fcidump_header(const char *path, int64_t *norb, int64_t *nelec) {
    try {
        if (!path || !norb || !nelec) throw FciError(CCQ_B200_EINVAL, "fcidump_header: null argument");
        FciFile f = read_fcidump(path, false);
        *norb = f.norb;
        *nelec = f.nelec;
        return 0;
    } catch (const FciError &e) {
        return fci_fail(e);
    } catch (const std::exception &e) {
        return fci_fail(FciError(CCQ_B200_EINVAL, e.what()));
    }
}

extern "C" int ccq_b200_fcidump_read(const char *path, int64_t norb, double *e1, double *e2, double *enuc) {
    try {
        if (!path || !e1 || !e2 || !enuc) throw FciError(CCQ_B200_EINVAL, "fcidump_read: null argument");
        FciFile f = read_fcidump(path, true);
        const int n = norb_checked(f, norb);
        Expanded x = expand(f, n, e1);
        const long long nn = n;
        std::fill(e2, e2 + nn * nn * nn * nn, 0.0);
        for (size_t r = 0; r < x.val.size(); ++r) {
            long long p[8];
            eight(nn, x.idx[4 * r], x.idx[4 * r + 1], x.idx[4 * r + 2], x.idx[4 * r + 3], p);
            for (int q = 0; q < 8; ++q) e2[p[q]] = x.val[r];
        }
        *enuc = x.enuc;
        return 0;
    } catch (const FciError &e) {
        return fci_fail(e);
    } catch (const std::exception &e) {
        return fci_fail(FciError(CCQ_B200_EINVAL, e.what()));
    }
}

extern "C" int ccq_b200_fcidump_read_device(const char *path, int64_t norb, double *e1, double *e2_dev,
                                            double *enuc, void *stream) {
    int *d_idx = nullptr, *d_owner = nullptr;
    double *d_val = nullptr;
    auto release = [&]() {
        cudaFree(d_idx);
        cudaFree(d_owner);
        cudaFree(d_val);
    };
    try {
        if (!path || !e1 || !e2_dev || !enuc) throw FciError(CCQ_B200_EINVAL, "fcidump_read_device: null argument");
        FciFile f = read_fcidump(path, true);
        const int n = norb_checked(f, norb);
        Expanded x = expand(f, n, e1);
        const long long nn = n, n4 = nn * nn * nn * nn;
        const long long nrec = (long long)x.val.size();
        if (nrec > 2147483647LL) throw FciError(CCQ_B200_ERANGE, "FCIDUMP: more than 2^31 two-body records");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        auto ck = [](cudaError_t e, const char *what) {
            if (e != cudaSuccess)
                throw FciError(e == cudaErrorMemoryAllocation ? CCQ_B200_ENOMEM : CCQ_B200_ECUDA,
                               std::string(what) + ": " + cudaGetErrorString(e));
        };
        ck(cudaMemsetAsync(e2_dev, 0, sizeof(double) * n4, s), "memset e2");
        if (nrec > 0) {
            ck(cudaMalloc(&d_idx, sizeof(int) * 4 * nrec), "cudaMalloc idx");
            ck(cudaMalloc(&d_val, sizeof(double) * nrec), "cudaMalloc val");
            ck(cudaMalloc(&d_owner, sizeof(int) * n4), "cudaMalloc owner");
            ck(cudaMemcpyAsync(d_idx, x.idx.data(), sizeof(int) * 4 * nrec, cudaMemcpyHostToDevice, s), "copy idx");
            ck(cudaMemcpyAsync(d_val, x.val.data(), sizeof(double) * nrec, cudaMemcpyHostToDevice, s), "copy val");
            ck(cudaMemsetAsync(d_owner, 0xff, sizeof(int) * n4, s), "memset owner");
            const int blocks = (int)std::min<long long>((nrec + 255) / 256, 148 * 16);
            fci_owner_kernel<<<blocks, 256, 0, s>>>(d_idx, nrec, nn, d_owner);
            ck(cudaGetLastError(), "fci_owner_kernel");
            fci_store_kernel<<<blocks, 256, 0, s>>>(d_idx, d_val, nrec, nn, d_owner, e2_dev);
            ck(cudaGetLastError(), "fci_store_kernel");
        }
        ck(cudaStreamSynchronize(s), "synchronize");
        release();
        *enuc = x.enuc;
        return 0;
    } catch (const FciError &e) {
        release();
        return fci_fail(e);
    } catch (const std::exception &e) {
        release();
        return fci_fail(FciError(CCQ_B200_EINVAL, e.what()));
    }
}
