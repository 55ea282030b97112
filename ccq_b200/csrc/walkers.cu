// FCIQMC walker files for externally corrected CC (calc_type=CADFCIQMC): the
// CI coefficients of the walker list, intermediately normalised, and their
// cluster analysis into T1..T4 in ccq's t_vec and T4 block layouts.
//
// Follows the reference:
//   records      parse_fciqmc_c3 (src/ext_cor/ext_cor.f90:146-283) and
//                process_fciqmc_c4 (src/ext_cor/contract_t4.f90:12-125):
//                "c_id coef occ_1 .. occ_m" read list-directed, m = nel -
//                2 froz spin orbitals numbered from the first unfrozen one
//                (shift_occ_list, src/external/excitations.f90:498-517), odd
//                numbers alpha and even beta (get_excitation_spin_integrate,
//                :206-261); reading ends at the end of the file or at the
//                first record that does not parse
//   sign         excitation_sign_qmc (:442-495): the excitation is applied as
//                the pairs (from_k -> to_k), alpha pairs first, each list
//                ascending; the parity of the occupied orbitals passed gives
//                the sign between the determinant and the excitation
//                operator a+_{t1} .. a+_{tn} a_{fn} .. a_{f1}
//   C            level 0 is the normalisation (coef_norm), levels 1-3 are
//                stored (a repeated determinant keeps its last value), level
//                4 contributions of repeated determinants add up (each record
//                is contracted separately in process_fciqmc_c4), higher
//                levels are skipped; every C is divided by coef_norm
//   T            T = ln(1 + C) projected on each excitation rank: T1 = C1,
//                T2, T3 on every excitation (cluster_analysis_up_t3,
//                src/ext_cor/cluster_analysis.f90:10-258), T4 likewise on
//                every quadruple, C4 entering only where the file has one
//                (the C4 projection of process_fciqmc_c4 plus the products
//                of T1..T3 of drive_t4_contraction, contract_t4.f90:241-479)
//
// The cluster expansion is evaluated with one formula for every rank and spin
// case: T(X) = sum over the set partitions pi of the excitation X into
// number-conserving sub-excitations of (-1)^(k-1) (k-1)! sgn(pi) prod_b C(b),
// k = |pi|, sgn(pi) the parity of re-sorting the holes and particles of the
// blocks into X's order (orbital order: alpha before beta, then by index).
//
// Differences: the reference determinant here is the CC reference (alpha
// orbitals 1..occ_a, beta 1..occ_b); the reference uses spin orbitals
// 1..nel, the same for singlets and doublets.  A record naming an orbital
// outside the basis, an orbital twice, or changing Ms is an error here.
#include <algorithm>
#include <array>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ccq_b200.h"
#include "kernels.cuh"

namespace {

struct WError : std::runtime_error {
    int code;
    WError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

struct Orb {
    int spin;  // 0 alpha, 1 beta
    int idx;   // occupied: from the first unfrozen orbital; virtual: from the first virtual of its spin
};

// sizes of the active space
struct Space {
    int o[2], v[2];
};

// one partition of the hole and particle positions 0..n-1 of an excitation
struct Pattern {
    int k;
    double coef;                  // (-1)^(k-1) (k-1)! sgn
    std::vector<std::pair<int, int>> blocks;   // (hole mask, particle mask)
};

int parity(const std::vector<int> &seq) {
    int inv = 0;
    for (size_t a = 0; a < seq.size(); ++a)
        for (size_t b = a + 1; b < seq.size(); ++b)
            if (seq[a] > seq[b]) ++inv;
    return inv & 1;
}

void gen_patterns(int hleft, int pleft, std::vector<std::pair<int, int>> &cur, std::vector<Pattern> &out) {
    if (!hleft) {
        Pattern p;
        p.k = (int)cur.size();
        p.blocks = cur;
        std::vector<int> hs, ps;
        for (auto &b : cur)
            for (int q = 0; q < 4; ++q) {
                if (b.first >> q & 1) hs.push_back(q);
            }
        for (auto &b : cur)
            for (int q = 0; q < 4; ++q) {
                if (b.second >> q & 1) ps.push_back(q);
            }
        double f = 1.0;
        for (int q = 2; q < p.k; ++q) f *= q;
        const int sg = parity(hs) ^ parity(ps);
        p.coef = ((p.k - 1) & 1 ? -f : f) * (sg ? -1.0 : 1.0);
        out.push_back(p);
        return;
    }
    const int h0 = __builtin_ctz(hleft);
    const int rest = hleft & ~(1 << h0);
    for (int s = rest;; s = (s - 1) & rest) {
        const int hb = (1 << h0) | s;
        const int sz = __builtin_popcount(hb);
        for (int q = pleft;; q = (q - 1) & pleft) {
            if (__builtin_popcount(q) == sz) {
                cur.push_back({hb, q});
                gen_patterns(hleft & ~hb, pleft & ~q, cur, out);
                cur.pop_back();
            }
            if (q == 0) break;
        }
        if (s == 0) break;
    }
}

struct PatternTables {
    std::vector<Pattern> pats[5];
    PatternTables() {
        for (int m = 1; m <= 4; ++m) {
            std::vector<std::pair<int, int>> cur;
            gen_patterns((1 << m) - 1, (1 << m) - 1, cur, pats[m]);
        }
    }
};

// built once, on first use, by whichever thread gets there first (a function-local
// static is initialised exactly once even when several threads read walker files)
const std::vector<Pattern> &patterns(int n) {
    static const PatternTables tables;
    return tables.pats[n];
}

// dense spin block of rank m with nb beta electrons: [o_a..][o_b..][v_a..][v_b..], C order
struct Blocks {
    Space sp;
    std::vector<double> c[4][4];   // rank 1..3, nb 0..rank
    std::map<std::array<int16_t, 9>, double> c4;

    size_t size(int m, int nb) const {
        size_t s = 1;
        for (int q = 0; q < m; ++q) s *= (size_t)(q < m - nb ? sp.o[0] : sp.o[1]);
        for (int q = 0; q < m; ++q) s *= (size_t)(q < m - nb ? sp.v[0] : sp.v[1]);
        return s;
    }
    // h, p sorted alpha first
    static size_t index(const Space &sp, int m, const Orb *h, const Orb *p) {
        size_t x = 0;
        for (int q = 0; q < m; ++q) x = x * (size_t)sp.o[h[q].spin] + (size_t)h[q].idx;
        for (int q = 0; q < m; ++q) x = x * (size_t)sp.v[p[q].spin] + (size_t)p[q].idx;
        return x;
    }
    static std::array<int16_t, 9> key(int nb, const Orb *h, const Orb *p) {
        std::array<int16_t, 9> k{};
        k[0] = (int16_t)nb;
        for (int q = 0; q < 4; ++q) {
            k[1 + q] = (int16_t)h[q].idx;
            k[5 + q] = (int16_t)p[q].idx;
        }
        return k;
    }
    double get(int m, const Orb *h, const Orb *p) const {
        int nb = 0;
        for (int q = 0; q < m; ++q) nb += h[q].spin;
        if (m <= 3) return c[m][nb][index(sp, m, h, p)];
        auto it = c4.find(key(nb, h, p));
        return it == c4.end() ? 0.0 : it->second;
    }
};

// T of one excitation (holes h, particles p, n <= 4, both sorted alpha first)
double cluster_t(const Blocks &B, int n, const Orb *h, const Orb *p) {
    double t = 0.0;
    for (const Pattern &pt : patterns(n)) {
        double prod = pt.coef;
        for (auto &b : pt.blocks) {
            Orb bh[4], bp[4];
            int m = 0, mp = 0, na = 0, nap = 0;
            for (int q = 0; q < n; ++q)
                if (b.first >> q & 1) {
                    bh[m++] = h[q];
                    na += h[q].spin == 0;
                }
            for (int q = 0; q < n; ++q)
                if (b.second >> q & 1) {
                    bp[mp++] = p[q];
                    nap += p[q].spin == 0;
                }
            if (na != nap) {
                prod = 0.0;
                break;
            }
            prod *= B.get(m, bh, bp);
            if (prod == 0.0) break;
        }
        t += prod;
    }
    return t;
}

// every canonical excitation of rank m with nb beta electrons: f(h, p)
template <class F>
void each_canonical(const Space &sp, int m, int nb, F f) {
    const int na = m - nb;
    Orb h[4], p[4];
    // increasing index lists of length len from 0..lim-1
    auto first = [](int *x, int len, int lim) {
        for (int q = 0; q < len; ++q) x[q] = q;
        return len <= lim;
    };
    auto next = [](int *x, int len, int lim) {
        int q = len - 1;
        while (q >= 0 && x[q] == lim - len + q) --q;
        if (q < 0) return false;
        ++x[q];
        for (int r = q + 1; r < len; ++r) x[r] = x[r - 1] + 1;
        return true;
    };
    int ha[4], hb[4], pa[4], pb[4];
    if (!first(ha, na, sp.o[0]) || !first(hb, nb, sp.o[1]) || !first(pa, na, sp.v[0]) || !first(pb, nb, sp.v[1]))
        return;
    do {
        do {
            do {
                do {
                    for (int q = 0; q < na; ++q) {
                        h[q] = {0, ha[q]};
                        p[q] = {0, pa[q]};
                    }
                    for (int q = 0; q < nb; ++q) {
                        h[na + q] = {1, hb[q]};
                        p[na + q] = {1, pb[q]};
                    }
                    f(h, p);
                } while (next(pb, nb, sp.v[1]));
                first(pb, nb, sp.v[1]);
            } while (next(pa, na, sp.v[0]));
            first(pa, na, sp.v[0]);
        } while (next(hb, nb, sp.o[1]));
        first(hb, nb, sp.o[1]);
    } while (next(ha, na, sp.o[0]));
}

// writes v at every antisymmetric copy of the canonical excitation (h, p) into a dense block
void fill_copies(double *blk, const Space &sp, int m, int nb, const Orb *h, const Orb *p, double v) {
    const int na = m - nb;
    // positions within the alpha holes, beta holes, alpha particles and beta particles
    std::vector<int> a0, a1, a2, a3;
    for (int q = 0; q < na; ++q) a0.push_back(q), a2.push_back(q);
    for (int q = 0; q < nb; ++q) a1.push_back(q), a3.push_back(q);
    do {
        do {
            do {
                do {
                    Orb hh[4], pp[4];
                    for (int q = 0; q < na; ++q) {
                        hh[q] = h[a0[q]];
                        pp[q] = p[a2[q]];
                    }
                    for (int q = 0; q < nb; ++q) {
                        hh[na + q] = h[na + a1[q]];
                        pp[na + q] = p[na + a3[q]];
                    }
                    const int sg = parity(a0) ^ parity(a1) ^ parity(a2) ^ parity(a3);
                    blk[Blocks::index(sp, m, hh, pp)] = sg ? -v : v;
                } while (std::next_permutation(a3.begin(), a3.end()));
            } while (std::next_permutation(a2.begin(), a2.end()));
        } while (std::next_permutation(a1.begin(), a1.end()));
    } while (std::next_permutation(a0.begin(), a0.end()));
}

// list-directed tokens: blanks and commas separate values
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

bool parse_int(const std::string &t, long long *v) {
    char *end = nullptr;
    *v = strtoll(t.c_str(), &end, 10);
    return end != t.c_str() && *end == '\0';
}

struct Counts {
    double c_hf = 0.0;
    long long records = 0, quadruples = 0, higher = 0;
};

Counts read_walkers(const char *path, int froz, int occ_a, int occ_b, int orbs, int nel, Blocks &B) {
    std::ifstream in(path);
    if (!in) throw WError(CCQ_B200_EINVAL, std::string("walker file not found: ") + path);
    const Space &sp = B.sp;
    const int m = nel - 2 * froz;
    if (m <= 0) throw WError(CCQ_B200_EINVAL, "walkers: nel - 2 froz must be positive");
    const int nso = 2 * orbs;
    // reference occupancy over spin orbitals 1..nso (odd alpha, even beta)
    std::vector<char> ref(nso + 1, 0);
    for (int s = 1; s <= occ_a; ++s) ref[2 * s - 1] = 1;
    for (int s = 1; s <= occ_b; ++s) ref[2 * s] = 1;
    Counts cnt;
    std::vector<std::string> tok, acc;
    std::string line;
    std::vector<char> occ(nso + 1);
    while (true) {
        acc.clear();
        bool eof = false;
        while ((int)acc.size() < m + 2) {
            if (!std::getline(in, line)) {
                eof = true;
                break;
            }
            split_tokens(line, tok);
            acc.insert(acc.end(), tok.begin(), tok.end());
        }
        if (eof) break;
        long long cid = 0;
        double coef = 0.0;
        if (!parse_int(acc[0], &cid) || !parse_real(acc[1], &coef)) break;
        std::fill(occ.begin(), occ.end(), 0);
        for (int s = 1; s <= 2 * froz; ++s) occ[s] = 1;
        bool bad = false;
        for (int q = 0; q < m; ++q) {
            long long x = 0;
            if (!parse_int(acc[2 + q], &x)) {
                bad = true;
                break;
            }
            x += 2 * froz;
            if (x < 2 * froz + 1 || x > nso)
                throw WError(CCQ_B200_EINVAL, "walkers: record " + std::to_string(cnt.records + 1) +
                                                  " names a spin orbital outside the basis");
            if (occ[x]) throw WError(CCQ_B200_EINVAL, "walkers: record " + std::to_string(cnt.records + 1) +
                                                          " names a spin orbital twice");
            occ[x] = 1;
        }
        if (bad) break;
        ++cnt.records;
        // holes and particles, ascending spin-orbital numbers
        std::vector<int> from, to;
        for (int x = 1; x <= nso; ++x) {
            if (ref[x] && !occ[x]) from.push_back(x);
            if (!ref[x] && occ[x]) to.push_back(x);
        }
        const int lvl = (int)from.size();
        if (lvl > 4) {
            ++cnt.higher;
            continue;
        }
        // alpha pairs first (excitation_sign_qmc's from_spin / to_spin)
        std::vector<int> fs, ts;
        for (int x : from)
            if (x & 1) fs.push_back(x);
        for (int x : to)
            if (x & 1) ts.push_back(x);
        const int nfa = (int)fs.size();
        if (nfa != (int)ts.size())
            throw WError(CCQ_B200_EINVAL, "walkers: record " + std::to_string(cnt.records) + " changes Ms");
        for (int x : from)
            if (!(x & 1)) fs.push_back(x);
        for (int x : to)
            if (!(x & 1)) ts.push_back(x);
        std::vector<char> tmp(ref);
        int occ_sum = 0;
        for (int k = 0; k < lvl; ++k) {
            for (int x = 1; x < fs[k]; ++x) occ_sum += tmp[x];
            tmp[fs[k]] = 0;
            for (int x = 1; x < ts[k]; ++x) occ_sum += tmp[x];
            tmp[ts[k]] = 1;
        }
        const double c = (occ_sum & 1) ? -coef : coef;
        if (lvl == 0) {
            cnt.c_hf = c;
            continue;
        }
        Orb h[4], p[4];
        for (int k = 0; k < lvl; ++k) {
            const int sf = (fs[k] & 1) ? 0 : 1, st = (ts[k] & 1) ? 0 : 1;
            const int spf = (fs[k] + 1) / 2, spt = (ts[k] + 1) / 2;   // spatial, 1-based
            h[k] = {sf, spf - froz - 1};
            p[k] = {st, spt - (st ? occ_b : occ_a) - 1};
        }
        const int nb = lvl - nfa;
        if (lvl <= 3) {
            B.c[lvl][nb][Blocks::index(sp, lvl, h, p)] = c;
        } else {
            B.c4[Blocks::key(nb, h, p)] += c;
        }
    }
    if (cnt.c_hf == 0.0)
        throw WError(CCQ_B200_EINVAL, "walkers: the Hartree-Fock coefficient is not in the file");
    for (int lv = 1; lv <= 3; ++lv)
        for (int nb = 0; nb <= lv; ++nb)
            for (double &x : B.c[lv][nb]) x /= cnt.c_hf;
    for (auto &kv : B.c4) kv.second /= cnt.c_hf;
    cnt.quadruples = (long long)B.c4.size();
    return cnt;
}

int w_fail(const WError &e) {
    ccqb::set_last_error(e.what());
    return e.code;
}

}  // namespace

extern "C" int ccq_b200_walkers_read(const char *path, const ccq_b200_dims *dims, int64_t nel, int64_t with_sd,
                                     double *t_vec, int64_t t_size, double *t4, int64_t t4_size, double *info) {
    try {
        if (!path || !dims || !t_vec) throw WError(CCQ_B200_EINVAL, "walkers_read: null argument");
        const int froz = (int)dims->froz, occ_a = (int)dims->occ_a, occ_b = (int)dims->occ_b, orbs = (int)dims->orbs;
        if (froz < 0 || occ_b < froz || occ_a < occ_b || orbs < occ_a || orbs > 4096)
            throw WError(CCQ_B200_EINVAL, "walkers_read: bad dims");
        if (nel != occ_a + occ_b) throw WError(CCQ_B200_EINVAL, "walkers_read: nel must be occ_a + occ_b");
        Blocks B;
        B.sp = Space{{occ_a - froz, occ_b - froz}, {orbs - occ_a, orbs - occ_b}};
        for (int m = 1; m <= 3; ++m)
            for (int nb = 0; nb <= m; ++nb) B.c[m][nb].assign(B.size(m, nb), 0.0);
        // t_vec: T1A T1B T2A T2B T2C T3A..T3D; T4 blocks T4A..T4E
        int64_t need = 0, need4 = 0;
        for (int m = 1; m <= 3; ++m)
            for (int nb = 0; nb <= m; ++nb) need += (int64_t)B.size(m, nb);
        {
            size_t s4 = 0;
            for (int nb = 0; nb <= 4; ++nb) {
                size_t s = 1;
                for (int q = 0; q < 4; ++q) s *= (size_t)(q < 4 - nb ? B.sp.o[0] : B.sp.o[1]);
                for (int q = 0; q < 4; ++q) s *= (size_t)(q < 4 - nb ? B.sp.v[0] : B.sp.v[1]);
                s4 += s;
            }
            need4 = (int64_t)s4;
        }
        if (t_size != need) throw WError(CCQ_B200_EINVAL, "walkers_read: t_size must be the T1..T3 size");
        if (t4 && t4_size != need4) throw WError(CCQ_B200_EINVAL, "walkers_read: t4_size must be the T4 size");
        Counts cnt = read_walkers(path, froz, occ_a, occ_b, orbs, (int)nel, B);
        std::fill(t_vec, t_vec + t_size, 0.0);
        size_t off = 0;
        for (int m = 1; m <= 3; ++m)
            for (int nb = 0; nb <= m; ++nb) {
                double *blk = t_vec + off;
                off += B.size(m, nb);
                if (m < 3 && !with_sd) continue;
                each_canonical(B.sp, m, nb, [&](const Orb *h, const Orb *p) {
                    const double v = cluster_t(B, m, h, p);
                    if (v != 0.0) fill_copies(blk, B.sp, m, nb, h, p, v);
                });
            }
        if (t4) {
            std::fill(t4, t4 + t4_size, 0.0);
            size_t o4 = 0;
            for (int nb = 0; nb <= 4; ++nb) {
                double *blk = t4 + o4;
                size_t s = 1;
                for (int q = 0; q < 4; ++q) s *= (size_t)(q < 4 - nb ? B.sp.o[0] : B.sp.o[1]);
                for (int q = 0; q < 4; ++q) s *= (size_t)(q < 4 - nb ? B.sp.v[0] : B.sp.v[1]);
                o4 += s;
                each_canonical(B.sp, 4, nb, [&](const Orb *h, const Orb *p) {
                    const double v = cluster_t(B, 4, h, p);
                    if (v != 0.0) fill_copies(blk, B.sp, 4, nb, h, p, v);
                });
            }
        }
        if (info) {
            info[0] = cnt.c_hf;
            info[1] = (double)cnt.records;
            info[2] = (double)cnt.quadruples;
            info[3] = (double)cnt.higher;
        }
        return 0;
    } catch (const WError &e) {
        return w_fail(e);
    } catch (const std::exception &e) {
        return w_fail(WError(CCQ_B200_EINVAL, e.what()));
    }
}
