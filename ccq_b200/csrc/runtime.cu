// Host runtime of libccq_b200: plan instantiation, resident device state,
// ccq's iteration step and the C ABI declared in include/ccq_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ccq_b200.h"
#include "crcc.cuh"
#include "kernels.cuh"
#include "plans_embedded.h"
#include "split.cuh"

using namespace ccqb;

namespace {

thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess)                                                                    \
            throw Error(e_ == cudaErrorMemoryAllocation ? CCQ_B200_ENOMEM : CCQ_B200_ECUDA,       \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                         \
    } while (0)

int fail(const Error &e) {
    g_last_error = e.what();
    return e.code;
}

}  // namespace

void ccqb::set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

namespace {

// ---------------------------------------------------------------------------
// plan text
// ---------------------------------------------------------------------------
struct AxisSpec {
    std::string label, size, start;
};
struct ViewSpec {
    std::string buf;
    std::vector<AxisSpec> axes;
};

ViewSpec parse_view(const std::string &tok) {
    ViewSpec v;
    size_t lb = tok.find('[');
    if (lb == std::string::npos || tok.back() != ']') throw Error(CCQ_B200_EPLAN, "bad view " + tok);
    v.buf = tok.substr(0, lb);
    std::string body = tok.substr(lb + 1, tok.size() - lb - 2);
    if (!body.empty()) {
        std::stringstream ss(body);
        std::string a;
        while (std::getline(ss, a, ',')) {
            AxisSpec ax;
            ax.start = "0";
            size_t at = a.find('@');
            if (at != std::string::npos) {
                ax.start = a.substr(at + 1);
                a = a.substr(0, at);
            }
            size_t c = a.find(':');
            if (c == std::string::npos) throw Error(CCQ_B200_EPLAN, "bad axis " + a);
            ax.label = a.substr(0, c);
            ax.size = a.substr(c + 1);
            v.axes.push_back(ax);
        }
    }
    return v;
}

enum OpKind { OP_GETT, OP_ASM, OP_COPY, OP_ZERO, OP_PHASE, OP_CRDIAG, OP_LENERGY, OP_CRCC };

struct Op {
    OpKind kind;
    // GETT
    double alpha = 1.0;
    int beta = 0;
    ViewSpec c, a, b;
    std::string tag;
    std::vector<std::vector<std::string>> restrict_groups;   // R= annotation
    // active-space filters of the output index modes (CCSDt): a table keeps a tuple only if it passes
    // every filter of its mode
    struct ModeFilter {
        int mode = 0;                      // 0: the M mode (labels of A and C), 1: the N mode (B and C)
        bool any = true;                   // true: some label active; false: no label active
        std::vector<std::string> labels;
        std::vector<long long> lo, hi;     // label active iff lo <= value < hi
    };
    std::vector<ModeFilter> filters;
    // ASSEMBLE
    std::string block, mode;
    std::vector<std::pair<double, ViewSpec>> terms;
    // COPY / ZERO / PHASE
    std::string arg0, arg1;
    // instantiated
    GettArgs g{};
    int akm = 1, bkm = 1;
    bool zero_first = false;
    bool split = false;        // eligible for split precision
    long long mnk[3] = {0, 0, 0};
    bool skip = false;         // member of a grouped GETT run by a later op
    double group_flops = 0.0;  // FLOPs of a grouped launch (leader only)
    int group_size = 0;
    int split_choice = -1;     // -1 by shape (split_eligible); autotuned: 0 DMMA, 1 per-tile split kernel, 2 persistent
    int split_ws = 0;          // slicing workspace of a split GETT (0: the context's first; see split_pool)
    bool frozen = false;       // in a T3 / T4 phase of an externally corrected solve: not run
    std::vector<size_t> group_ops;   // every op of a grouped launch (leader only; members are skipped)
    std::vector<int> hcm, hcn; // output offset tables (grouping key)
    AsmArgs asmargs{};
    CrccArgs crcc{};           // CRCC: one spin block's four-denominator sums
};

struct BufSpec {
    std::string name, kind;
    std::vector<std::string> dims;
    std::vector<std::vector<int>> groups;   // antisymmetric axis groups (G= annotation)
};

std::vector<std::string> split_str(const std::string &s, char sep) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string x;
    while (std::getline(ss, x, sep))
        if (!x.empty()) out.push_back(x);
    return out;
}

struct Plan {
    std::string method;
    std::vector<BufSpec> bufs;
    std::vector<Op> ops;
};

Plan parse_plan(const char *text) {
    Plan p;
    std::stringstream in(text);
    std::string line;
    std::getline(in, line);
    {
        std::stringstream ls(line);
        std::string w;
        ls >> w >> p.method;
        if (w != "PLAN") throw Error(CCQ_B200_EPLAN, "plan header");
    }
    while (std::getline(in, line)) {
        std::stringstream ls(line);
        std::string w;
        ls >> w;
        if (w == "BUF") {
            BufSpec b;
            int nd;
            ls >> b.name >> b.kind >> nd;
            for (int i = 0; i < nd; ++i) {
                std::string d;
                ls >> d;
                b.dims.push_back(d);
            }
            std::string ann;
            if (ls >> ann) {
                if (ann.rfind("G=", 0) != 0) throw Error(CCQ_B200_EPLAN, "bad buffer annotation " + ann);
                for (auto &g : split_str(ann.substr(2), ';')) {
                    std::vector<int> axes;
                    for (auto &a : split_str(g, ',')) axes.push_back(std::stoi(a));
                    b.groups.push_back(axes);
                }
            }
            p.bufs.push_back(b);
        } else if (w == "OPS") {
            continue;
        } else if (w == "GETT") {
            Op o;
            o.kind = OP_GETT;
            std::string c, a, b;
            ls >> o.alpha >> o.beta >> c >> a >> b;
            std::string w2;
            while (ls >> w2) {
                if (w2.rfind("R=", 0) == 0) {
                    for (auto &g : split_str(w2.substr(2), ';')) o.restrict_groups.push_back(split_str(g, ','));
                } else {
                    o.tag = w2;
                }
            }
            o.c = parse_view(c);
            o.a = parse_view(a);
            o.b = parse_view(b);
            p.ops.push_back(o);
        } else if (w == "ASSEMBLE") {
            Op o;
            o.kind = OP_ASM;
            int nt;
            ls >> o.block >> o.mode >> nt;
            for (int i = 0; i < nt; ++i) {
                std::getline(in, line);
                std::stringstream ts(line);
                std::string tw, vv;
                double coef;
                ts >> tw >> coef >> vv;
                if (tw != "TERM") throw Error(CCQ_B200_EPLAN, "TERM expected");
                o.terms.push_back({coef, parse_view(vv)});
            }
            p.ops.push_back(o);
        } else if (w == "CRDIAG" || w == "LENERGY" || w == "CRCC") {
            Op o;
            o.kind = w == "CRDIAG" ? OP_CRDIAG : (w == "LENERGY" ? OP_LENERGY : OP_CRCC);
            ls >> o.arg0;
            p.ops.push_back(o);
        } else if (w == "COPY" || w == "ZERO" || w == "PHASE") {
            Op o;
            o.kind = w == "COPY" ? OP_COPY : (w == "ZERO" ? OP_ZERO : OP_PHASE);
            ls >> o.arg0 >> o.arg1;
            p.ops.push_back(o);
        } else if (w == "END") {
            break;
        } else if (!w.empty()) {
            throw Error(CCQ_B200_EPLAN, "unknown plan line: " + line);
        }
    }
    return p;
}

const char *find_plan(const std::string &calc_type, bool rhf) {
    // plan file names: the calc_type, with CR-CC(2,3) stored as CRCC23
    std::string key = (calc_type == "CR-CC(2,3)" ? std::string("CRCC23") : calc_type) + (rhf ? "_rhf" : "");
    for (int i = 0; ccqb_plans[i].name; ++i)
        if (key == ccqb_plans[i].name) return ccqb_plans[i].text;
    return nullptr;
}

struct DevBuf {
    double *ptr = nullptr;
    std::vector<long long> shape, stride;
    long long numel = 0;
    std::vector<std::vector<int>> groups;
};

}  // namespace

struct ccq_b200_ctx {
    std::string calc_type;
    int rhf = 0;
    double shift = 0.0;
    int ds = 5;
    long long oa, ob, va, vb, n, froz;
    std::map<std::string, long long> size;
    Plan plan;
    std::map<std::string, DevBuf> bufs;
    std::vector<void *> owned;
    double *tvec = nullptr;
    long long t_size = 0, vec_size = 0;
    long long vec_full = 0, vec_t12 = 0;   // DIIS vector sizes: the method's and T1 + T2 only
    double *ring = nullptr;
    double *scratch = nullptr;  // residuum / gram / coef
    int *dinfo = nullptr;
    double *fdiag_a = nullptr, *fdiag_b = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    double iter_ms = 0.0;
    // per-op profiling (eager sweeps only): events around every launch
    int profile = 0;
    std::vector<cudaEvent_t> pev;
    double prof_ms[4] = {0, 0, 0, 0};       // gett_f64, gett_split, assemble, other
    double prof_flops[4] = {0, 0, 0, 0};
    long long prof_launch[4] = {0, 0, 0, 0};
    size_t energy_op = 0;
    // CR-CC(2,3) plans: the CC sweep and energy end at the 'crcc' marker; the
    // left solve and the triples corrections follow in their own phases
    size_t cc_end = 0, lambda_op = 0, lenergy_op = 0, triples_op = 0;
    bool has_crcc = false;
    double *lvec = nullptr, *lring = nullptr;
    long long l_size = 0;
    CrDiagArgs crd{};
    cudaGraphExec_t lgexec = nullptr;
    // graph capture as a DAG: independent contractions on side streams
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> opev;
    cudaEvent_t cap_ev = nullptr;
    long long t_dev = 0;        // t_vec elements resident on the device (T1+T2 for CCSD-level methods)
    bool trace_init = false;    // stage times of context creation on stderr
    std::chrono::steady_clock::time_point t_init0;
    double *hpin = nullptr;     // pinned host slots for an iteration's results (E, residuum, DIIS info)
    int64_t async_iter = 0;     // iteration launched by iterate_async, 0 when none is pending
    double flops = 0.0;
    long long launches = 0;
    double sweep_ms = 0.0;
    int precision = CCQ_B200_PREC_FP64;
    int nslices = 4;
    int use_graph = 0;
    cudaGraphExec_t gexec = nullptr;
    int device = 0;
    long long act_occ_b = -1, act_unocc_a = -1;   // CCSDt: the active space the plan was restricted to
    // CCSDt: DIIS runs over ccq's compressed T vector (T1, T2 and the active T3 sub-blocks of
    // get_t_sizes_act), gathered from the full blocks after each sweep and scattered back after an
    // extrapolation
    bool cdiis = false;
    T3ActGeom geom{};
    double *cvec = nullptr;
    SplitWorkspace split{};
    // further slicing workspaces: split GETTs take them in turn, so that a split GETT is a node of the sweep's
    // dependency graph (waiting only for the previous user of its workspace) instead of a barrier
    std::vector<SplitWorkspace> split_pool;
    // host round trip of ccq_b200_iterate_host: each t_vec block is copied to host_out as soon as its
    // last write of the sweep is done (copy stream cstream, joined into the sweep's stream at its end)
    double *host_out = nullptr;
    cudaGraphExec_t gexec_host = nullptr;
    double *gexec_host_ptr = nullptr;
    // a DIIS iteration's host round trip: the sweep reads the input but copies nothing out (the
    // extrapolation rewrites every block); the whole extrapolated vector then goes to diis_out
    cudaGraphExec_t gexec_hin = nullptr;
    double *diis_out = nullptr;
    // ... and with host_in set (pinned input, dependency-graph sweep), the t_vec is copied in block by block on
    // istream inside the graph: an operation waits only for the copies of the blocks it reads
    const double *host_in = nullptr;
    const double *gexec_host_in = nullptr;
    cudaStream_t istream = nullptr;
    // when host_in is mapped into the device's address space (host_in_dev), the T3 blocks are read there at
    // their canonical elements only (sorted occupied and virtual indices within each same-spin run) by a
    // copy-mode assemble per block, which also writes every antisymmetric image on the device
    const double *host_in_dev = nullptr;
    std::map<std::string, AsmArgs> cin_args;   // per block read this way
    AsmTerm *cin_terms = nullptr;               // device: one term per such block
    long long cin_h2d = 0;                      // bytes the captured host round trip reads from host_in
    long long io_h2d = 0, io_d2h = 0;           // bytes of the last host round trip
    cudaStream_t cstream = nullptr;
    cudaEvent_t cjoin = nullptr;
    std::vector<cudaEvent_t> cev;
    std::vector<std::pair<size_t, std::string>> out_after;   // (op index, block) of every block's last write
    bool out_ready = false;

    // Device memory comes from the device's stream-ordered pool (on this context's stream): the memory of
    // a closed context goes back to the pool and a new context takes it from there, instead of a driver
    // unmap and map per buffer (a CR-CC(2,3) context created after another was freed spent 1.3 s in
    // cudaMalloc; this pool keeps up to kPoolKeep bytes of freed memory for the process).
    void *dalloc(size_t bytes) {
        void *p = nullptr;
        CK(cudaMallocAsync(&p, bytes ? bytes : 8, stream));
        owned.push_back(p);
        // touched once here: the first write to fresh device memory is slow (a 538 MB DIIS ring slot first
        // written at the first DIIS step cost 30-60 ms inside an iteration); the buffer is also filled by
        // copies and kernels on other streams, so the allocation completes now
        CK(cudaMemsetAsync(p, 0, bytes ? bytes : 8, stream));
        CK(cudaStreamSynchronize(stream));
        return p;
    }
    ~ccq_b200_ctx() {
        // every stream of this context is idle before its memory goes back to the pool
        if (stream) cudaStreamSynchronize(stream);
        for (auto st : side) cudaStreamSynchronize(st);
        if (cstream) cudaStreamSynchronize(cstream);
        if (istream) cudaStreamSynchronize(istream);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (lgexec) cudaGraphExecDestroy(lgexec);
        if (gexec_host) cudaGraphExecDestroy(gexec_host);
        if (gexec_hin) cudaGraphExecDestroy(gexec_hin);
        for (auto e : cev) cudaEventDestroy(e);
        if (cjoin) cudaEventDestroy(cjoin);
        if (cstream) cudaStreamDestroy(cstream);
        if (istream) cudaStreamDestroy(istream);
        for (auto e : opev) cudaEventDestroy(e);
        if (cap_ev) cudaEventDestroy(cap_ev);
        for (auto st : side) cudaStreamDestroy(st);
        split_free(split);
        for (auto &w : split_pool) split_free(w);
        if (hpin) cudaFreeHost(hpin);
        if (stream) {
            for (void *p : owned) cudaFreeAsync(p, stream);
            cudaStreamSynchronize(stream);
        }
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev2) cudaEventDestroy(ev2);
        for (auto e : pev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

long long tok(const ccq_b200_ctx *c, const std::string &s) {
    auto it = c->size.find(s);
    if (it == c->size.end()) throw Error(CCQ_B200_EPLAN, "unknown size token " + s);
    return it->second;
}

struct Resolved {
    double *base;
    std::map<std::string, long long> stride;   // per label
    std::map<std::string, long long> extent;
    std::vector<std::string> order;            // labels in axis order (first occurrence)
};

Resolved resolve(ccq_b200_ctx *c, const ViewSpec &v) {
    auto it = c->bufs.find(v.buf);
    if (it == c->bufs.end()) throw Error(CCQ_B200_EPLAN, "unknown buffer " + v.buf);
    const DevBuf &b = it->second;
    if (b.shape.size() != v.axes.size()) throw Error(CCQ_B200_EPLAN, "rank mismatch for " + v.buf);
    Resolved r;
    long long off = 0;
    for (size_t d = 0; d < v.axes.size(); ++d) {
        const AxisSpec &a = v.axes[d];
        long long st = tok(c, a.start);
        long long ex = tok(c, a.size);
        if (st + ex > b.shape[d]) throw Error(CCQ_B200_EPLAN, "view exceeds buffer " + v.buf);
        off += st * b.stride[d];
        if (!r.stride.count(a.label)) {
            r.order.push_back(a.label);
            r.stride[a.label] = 0;
            r.extent[a.label] = ex;
        }
        r.stride[a.label] += b.stride[d];
    }
    r.base = b.ptr + off;
    return r;
}

bool has(const Resolved &r, const std::string &l) { return r.stride.count(l) > 0; }

// Offset tables of one index mode (labels, last fastest) for views x and y.
// Restricted groups (label lists) are enumerated for increasing values only.
void build_table(const std::vector<std::string> &labels, const std::map<std::string, long long> &extent,
                 const Resolved &x, const Resolved *y, const std::vector<std::vector<std::string>> &groups,
                 const std::vector<const Op::ModeFilter *> &filters, std::vector<int> &tx, std::vector<int> &ty) {
    tx.clear();
    ty.clear();
    std::vector<std::vector<int>> gidx;   // positions in `labels` of each group's members, in group order
    for (auto &g : groups) {
        std::vector<int> pos;
        for (auto &l : g) {
            auto it = std::find(labels.begin(), labels.end(), l);
            if (it != labels.end()) pos.push_back((int)(it - labels.begin()));
        }
        if (pos.size() == g.size()) gidx.push_back(pos);
    }
    // each filter's labels as positions in `labels`
    struct F {
        bool any;
        std::vector<int> pos;
        std::vector<long long> lo, hi;
    };
    std::vector<F> fl;
    for (auto *f : filters) {
        F q{f->any, {}, f->lo, f->hi};
        for (auto &l : f->labels) {
            auto it = std::find(labels.begin(), labels.end(), l);
            if (it == labels.end()) throw Error(CCQ_B200_EPLAN, "filter label " + l + " not in its index mode");
            q.pos.push_back((int)(it - labels.begin()));
        }
        fl.push_back(q);
    }
    const size_t nd = labels.size();
    std::vector<long long> idx(nd, 0), ev(nd), sx(nd), sy(nd, 0);
    long long total = 1;
    for (size_t d = 0; d < nd; ++d) {
        ev[d] = extent.at(labels[d]);
        sx[d] = x.stride.at(labels[d]);
        if (y) sy[d] = y->stride.at(labels[d]);
        total *= ev[d];
    }
    if (total == 0) return;
    tx.reserve((size_t)total);
    if (y) ty.reserve((size_t)total);
    if (gidx.empty() && fl.empty()) {
        // a plain product of the labels' ranges: expanded label by label (the last one fastest),
        // the same order as the enumeration below, without per-tuple checks
        long long mx = 0, my = 0;
        for (size_t d = 0; d < nd; ++d) {
            mx += (ev[d] - 1) * sx[d];
            my += (ev[d] - 1) * sy[d];
        }
        if (mx > INT32_MAX || my > INT32_MAX) throw Error(CCQ_B200_ERANGE, "view offset beyond int32");
        tx.assign(1, 0);
        if (y) ty.assign(1, 0);
        for (size_t d = 0; d < nd; ++d) {
            const size_t cur = tx.size();
            std::vector<int> nx(cur * (size_t)ev[d]), ny(y ? cur * (size_t)ev[d] : 0);
            for (size_t j = 0; j < cur; ++j)
                for (long long i = 0; i < ev[d]; ++i) {
                    nx[j * ev[d] + i] = tx[j] + (int)(i * sx[d]);
                    if (y) ny[j * ev[d] + i] = ty[j] + (int)(i * sy[d]);
                }
            tx.swap(nx);
            if (y) ty.swap(ny);
        }
        return;
    }
    bool more = true;
    while (more) {
        bool ok = true;
        for (auto &g : gidx)
            for (size_t q = 1; q < g.size(); ++q)
                if (idx[g[q]] <= idx[g[q - 1]]) ok = false;
        for (auto &f : fl) {
            bool hit = false;
            for (size_t q = 0; q < f.pos.size(); ++q)
                hit = hit || (idx[f.pos[q]] >= f.lo[q] && idx[f.pos[q]] < f.hi[q]);
            if (hit != f.any) ok = false;
        }
        if (ok) {
            long long ox = 0, oy = 0;
            for (size_t d = 0; d < nd; ++d) {
                ox += idx[d] * sx[d];
                oy += idx[d] * sy[d];
            }
            if (ox > INT32_MAX || oy > INT32_MAX) throw Error(CCQ_B200_ERANGE, "view offset beyond int32");
            tx.push_back((int)ox);
            if (y) ty.push_back((int)oy);
        }
        more = false;
        for (int d = (int)nd - 1; d >= 0; --d) {
            if (++idx[d] < ev[d]) {
                more = true;
                break;
            }
            idx[d] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Active-space CCSDt at its own cost.  ccq's CCSDt keeps only the triples with
// at least one active occupied and one active virtual index (spatial orbitals
// above act_occ_b, up to act_unocc_a; src/parser.f90:495-499,
// src/utils/cc_utils.f90:560-630).  The residual terms of a T3 block (the Z
// buffers its Jacobi assemble reads) are then needed only on the elements whose
// occupied labels hold an active index and whose virtual labels hold one: a set
// that every permutation of the labels keeps, so the assemble's permuted and
// sorted reads of an active triple stay inside it.  Each GETT that writes such a
// Z keeps only those elements through filters on its output offset tables.  The
// labels of one kind (occupied or virtual) may sit in both output modes; then
// "some label active" is the disjoint union of "some M label active" and "no M
// label active, some N label active", so a contraction becomes at most four
// GETTs (usually one or two), each with filtered M and N tables.
// ---------------------------------------------------------------------------
struct ActiveSpace {
    long long occ_lo = 0;          // occupied index (from froz) >= occ_lo is active, both spins
    long long vir_hi[2] = {0, 0};  // virtual index (from occ of the spin) < vir_hi[spin] is active
};

void restrict_to_active(ccq_b200_ctx *c, const ActiveSpace &as) {
    std::map<std::string, int> t3z;   // Z buffers read only by T3 Jacobi assembles
    for (auto &o : c->plan.ops)
        if (o.kind == OP_ASM && o.block.size() == 3 && o.block[1] == '3' && o.mode == "jacobi")
            for (auto &t : o.terms)
                if (t.second.buf[0] == 'Z') t3z[t.second.buf] = 1;
    for (auto &o : c->plan.ops) {
        if (o.kind == OP_GETT) {
            t3z.erase(o.a.buf);
            t3z.erase(o.b.buf);
        }
        if (o.kind == OP_ASM && !(o.block.size() == 3 && o.block[1] == '3' && o.mode == "jacobi"))
            for (auto &t : o.terms) t3z.erase(t.second.buf);
    }
    const long long full_o[2] = {c->oa, c->ob}, full_v[2] = {c->va, c->vb};
    auto has_label = [](const ViewSpec &v, const std::string &l) {
        for (auto &ax : v.axes)
            if (ax.label == l) return true;
        return false;
    };
    std::vector<Op> ops;
    for (auto &o : c->plan.ops) {
        if (o.kind != OP_GETT || !t3z.count(o.c.buf)) {
            ops.push_back(o);
            continue;
        }
        // output labels by kind and index mode, with their active ranges
        struct L {
            std::string name;
            long long lo, hi;
        };
        std::vector<L> side[2][2];   // [occ/vir][M/N]
        bool ok = true;
        for (auto &ax : o.c.axes) {
            const std::string &z = ax.size;
            const int mode = has_label(o.a, ax.label) ? 0 : 1;
            if (z == "oa" || z == "ob") {
                const long long n = full_o[z == "ob"];
                side[0][mode].push_back({ax.label, std::min(as.occ_lo, n), n});
            } else if (z == "va" || z == "vb") {
                side[1][mode].push_back({ax.label, 0, std::min(as.vir_hi[z == "vb"], full_v[z == "vb"])});
            } else {
                ok = false;
            }
        }
        if (!ok || (side[0][0].empty() && side[0][1].empty()) || (side[1][0].empty() && side[1][1].empty())) {
            ops.push_back(o);
            continue;
        }
        auto filt = [](int mode, bool any, const std::vector<L> &ls) {
            Op::ModeFilter f;
            f.mode = mode;
            f.any = any;
            for (auto &l : ls) {
                f.labels.push_back(l.name);
                f.lo.push_back(l.lo);
                f.hi.push_back(l.hi);
            }
            return f;
        };
        // the pieces of one kind: lists of filters whose conjunction is a disjoint part of "some active"
        auto pieces = [&](const std::vector<L> *sd) {
            std::vector<std::vector<Op::ModeFilter>> out;
            if (sd[1].empty()) out.push_back({filt(0, true, sd[0])});
            else if (sd[0].empty()) out.push_back({filt(1, true, sd[1])});
            else {
                out.push_back({filt(0, true, sd[0])});
                out.push_back({filt(0, false, sd[0]), filt(1, true, sd[1])});
            }
            return out;
        };
        for (auto &po : pieces(side[0]))
            for (auto &pv : pieces(side[1])) {
                Op q = o;
                q.filters = po;
                q.filters.insert(q.filters.end(), pv.begin(), pv.end());
                ops.push_back(q);
            }
    }
    c->plan.ops = ops;
}

// The T3 Jacobi assembles hold the triples outside the active space at zero (and gather only the
// active ones); CR-CC(2,3) contexts (CC(t;3)) skip the active triples in the correction instead.
void apply_active_masks(ccq_b200_ctx *c, long long act_occ_b, long long act_unocc_a) {
    const long long occ_a = c->froz + c->oa, occ_b = c->froz + c->ob;
    for (auto &o : c->plan.ops) {
        if (o.kind == OP_CRCC) {
            // CC(t;3): the correction covers the triples outside the active space
            o.crcc.act_occ_lo = (int)(act_occ_b - c->froz);
            o.crcc.act_vir_hi = (int)(act_unocc_a - c->froz);
            continue;
        }
        if (o.kind != OP_ASM || o.block[1] != '3' || o.asmargs.mode != 0) continue;
        AsmArgs &a = o.asmargs;
        // spatial orbitals above act_occ_b (occupied) and up to act_unocc_a (virtual) are active,
        // for both spins; indices here count from froz (occupied) and from occ (virtual)
        a.act = 1;
        a.act_occ_lo = (int)(act_occ_b - c->froz);
        a.act_vir_hi[0] = (int)(act_unocc_a - occ_a);
        a.act_vir_hi[1] = (int)(act_unocc_a - occ_b);
    }
}

// The device's default memory pool keeps up to kPoolKeep bytes of freed memory for this process (its
// release threshold; a property of this process's pool, not of the GPU), set once per device.
constexpr uint64_t kPoolKeep = 16ull << 30;

void keep_pool_memory(int dev) {
    static std::once_flag once[64];
    if (dev < 0 || dev >= 64) return;
    std::call_once(once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = kPoolKeep;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
}

void trace_stamp(const ccq_b200_ctx *c, const char *what) {
    if (!c->trace_init) return;
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - c->t_init0).count();
    fprintf(stderr, "ccq_b200_init %-14s %8.2f ms\n", what, ms);
}

void instantiate(ccq_b200_ctx *c) {
    // ---- buffers -----------------------------------------------------------
    // amplitude blocks T1..T3 live in t_vec at get_t_sizes offsets
    static const char *tv_order[] = {"T1A", "T1B", "T2A", "T2B", "T2C", "T3A", "T3B", "T3C", "T3D"};
    std::map<std::string, long long> tv_off;
    long long off = 0;
    std::map<std::string, std::vector<std::string>> bdims;
    for (auto &b : c->plan.bufs) bdims[b.name] = b.dims;
    for (auto *nm : tv_order) {
        auto it = bdims.find(nm);
        if (it == bdims.end()) throw Error(CCQ_B200_EPLAN, std::string("plan lacks block ") + nm);
        long long ne = 1;
        for (auto &d : it->second) ne *= tok(c, d);
        tv_off[nm] = off;
        off += ne;
    }
    c->t_size = off;
    // CR-CC(2,3) solves CCSD; its DIIS vector is T1 + T2 (the T3 slots stay zero)
    c->vec_size = (c->calc_type == "CCSD" || c->calc_type == "CR-CC(2,3)") ? tv_off["T3A"] : c->t_size;
    if (c->cdiis) {
        if (c->geom.t12 != tv_off["T3A"] || c->geom.t3_end != c->t_size)
            throw Error(CCQ_B200_EPLAN, "CCSDt layout does not match the plan's T vector");
        c->vec_size = c->geom.t12 + c->geom.n_act;
        c->cvec = (double *)c->dalloc(sizeof(double) * std::max(c->vec_size, 1LL));
    }
    c->vec_full = c->vec_size;
    c->vec_t12 = tv_off["T3A"];
    // left amplitudes (L1A..L2C) share the T1/T2 layout in their own vector
    std::map<std::string, long long> lv_off;
    {
        static const char *lv_order[] = {"L1A", "L1B", "L2A", "L2B", "L2C"};
        long long lo = 0;
        for (auto *nm : lv_order) {
            auto it = bdims.find(nm);
            if (it == bdims.end()) continue;
            long long ne = 1;
            for (auto &d : it->second) ne *= tok(c, d);
            lv_off[nm] = lo;
            lo += ne;
        }
        c->l_size = lo;
        if (lo) {
            c->lvec = (double *)c->dalloc(sizeof(double) * lo);
            c->lring = (double *)c->dalloc(sizeof(double) * (size_t)(c->ds + 1) * lo);
            CK(cudaMemsetAsync(c->lvec, 0, sizeof(double) * lo, c->stream));
        }
    }
    // CCSD-level methods never touch the T3 slots of t_vec: they stay on the host side of the
    // boundary (zeros in get_t), and only T1 + T2 are resident
    c->t_dev = (c->calc_type == "CCSD" || c->calc_type == "CR-CC(2,3)") ? tv_off["T3A"] : c->t_size;
    c->tvec = (double *)c->dalloc(sizeof(double) * c->t_dev);
    CK(cudaMemsetAsync(c->tvec, 0, sizeof(double) * c->t_dev, c->stream));

    // work buffers: one arena, each phase packs its Z/X buffers from offset 0
    std::map<std::string, std::string> first_phase;
    {
        std::string phase = "init";
        auto note = [&](const ViewSpec &v) {
            if (!first_phase.count(v.buf)) first_phase[v.buf] = phase;
            else if (first_phase[v.buf] != phase && (v.buf[0] == 'Z' || v.buf[0] == 'X'))
                throw Error(CCQ_B200_EPLAN, "work buffer used across phases: " + v.buf);
        };
        for (auto &o : c->plan.ops) {
            if (o.kind == OP_PHASE) phase = o.arg0 + "#" + std::to_string(&o - &c->plan.ops[0]);
            if (o.kind == OP_GETT) {
                note(o.c);
                note(o.a);
                note(o.b);
            }
            if (o.kind == OP_ASM)
                for (auto &t : o.terms) note(t.second);
        }
    }
    {
        // work buffers live in a shared arena: each must be overwritten before it is read
        std::map<std::string, int> written;
        auto work = [](const std::string &b) { return !b.empty() && (b[0] == 'Z' || b[0] == 'X'); };
        for (auto &o : c->plan.ops) {
            if (o.kind == OP_PHASE) written.clear();
            if (o.kind == OP_GETT) {
                for (auto *v : {&o.a, &o.b})
                    if (work(v->buf) && !written.count(v->buf))
                        throw Error(CCQ_B200_EPLAN, v->buf + " read before written");
                if (work(o.c.buf)) {
                    if (o.beta && !written.count(o.c.buf))
                        throw Error(CCQ_B200_EPLAN, o.c.buf + " accumulated before written");
                    written[o.c.buf] = 1;
                }
            }
            if (o.kind == OP_ASM)
                for (auto &t : o.terms)
                    if (work(t.second.buf) && !written.count(t.second.buf))
                        throw Error(CCQ_B200_EPLAN, t.second.buf + " read by assemble before written");
        }
    }
    std::map<std::string, long long> phase_fill;
    std::map<std::string, long long> work_off;
    long long arena = 0;
    for (auto &b : c->plan.bufs) {
        if (b.kind != "work") continue;
        long long ne = 1;
        for (auto &d : b.dims) ne *= tok(c, d);
        ne = (ne + 31) / 32 * 32;
        std::string ph = first_phase.count(b.name) ? first_phase[b.name] : "unused";
        work_off[b.name] = phase_fill[ph];
        phase_fill[ph] += ne;
        arena = std::max(arena, phase_fill[ph]);
    }
    {
        // consecutive phases take alternate halves of a doubled arena (up to 16 GiB), so that a phase's
        // contractions need not wait for the previous phase's assemble to finish reading its work buffers
        // (CCQ_B200_ARENA_SINGLE set: one shared region)
        std::vector<std::pair<long long, std::string>> order;
        for (auto &kv : phase_fill) {
            const size_t h = kv.first.rfind('#');
            order.push_back({h == std::string::npos ? -1LL : std::atoll(kv.first.c_str() + h + 1), kv.first});
        }
        std::sort(order.begin(), order.end());
        if (order.size() >= 2 && sizeof(double) * 2 * arena <= (16LL << 30) && !getenv("CCQ_B200_ARENA_SINGLE")) {
            std::map<std::string, int> parity;
            for (size_t k = 0; k < order.size(); ++k) parity[order[k].second] = (int)(k & 1);
            for (auto &b : c->plan.bufs) {
                if (b.kind != "work") continue;
                const std::string ph = first_phase.count(b.name) ? first_phase[b.name] : "unused";
                if (parity[ph]) work_off[b.name] += arena;
            }
            arena *= 2;
        }
    }
    double *arena_ptr = (double *)c->dalloc(sizeof(double) * std::max(arena, 1LL));
    for (auto &b : c->plan.bufs) {
        DevBuf d;
        for (auto &x : b.dims) d.shape.push_back(tok(c, x));
        d.stride.assign(d.shape.size(), 1);
        for (int i = (int)d.shape.size() - 2; i >= 0; --i) d.stride[i] = d.stride[i + 1] * d.shape[i + 1];
        d.numel = 1;
        for (auto s : d.shape) d.numel *= s;
        d.groups = b.groups;
        if (tv_off.count(b.name)) {
            d.ptr = tv_off[b.name] < c->t_dev ? c->tvec + tv_off[b.name] : nullptr;
        } else if (lv_off.count(b.name)) {
            d.ptr = c->lvec + lv_off[b.name];
        } else if (b.kind == "work") {
            d.ptr = arena_ptr + work_off[b.name];
        } else {
            d.ptr = (double *)c->dalloc(sizeof(double) * std::max(d.numel, 1LL));
            CK(cudaMemsetAsync(d.ptr, 0, sizeof(double) * std::max(d.numel, 1LL), c->stream));
        }
        c->bufs[b.name] = d;
    }
    for (auto &b : c->plan.bufs)
        if (b.kind == "ones") launch_fill(c->bufs.at(b.name).ptr, 1.0, std::max(c->bufs.at(b.name).numel, 1LL), c->stream);
    trace_stamp(c, "buffers");

    // ---- operations ----------------------------------------------------------
    std::vector<int> itab;
    struct Pend {
        size_t op;
        size_t am, ak, bn, bk, cm, cn;
    };
    std::vector<Pend> pend;
    std::vector<AsmTerm> hterms;
    std::vector<signed char> hperm, hsign;
    std::vector<unsigned char> hcomb;
    struct PendA {
        size_t op, t0, p0;
    };
    std::vector<PendA> penda;
    c->flops = 0.0;
    c->cc_end = c->plan.ops.size();
    for (size_t i = 0; i < c->plan.ops.size(); ++i) {
        Op &o = c->plan.ops[i];
        if (o.kind == OP_PHASE && o.arg0 == "energy") c->energy_op = i;
        if (o.kind == OP_PHASE && o.arg0 == "crcc") {
            c->cc_end = i;
            c->has_crcc = true;
        }
        if (o.kind == OP_PHASE && o.arg0 == "lambda") c->lambda_op = i;
        if (o.kind == OP_PHASE && o.arg0 == "lenergy") c->lenergy_op = i;
        if (o.kind == OP_PHASE && o.arg0 == "triplesA") c->triples_op = i;
        if (o.kind == OP_CRCC) {
            const std::string x = o.arg0;
            if (x.size() != 1 || x[0] < 'A' || x[0] > 'D') throw Error(CCQ_B200_EPLAN, "CRCC block " + x);
            const DevBuf &M = c->bufs.at("M3" + x), &L = c->bufs.at("L3" + x);
            if (M.shape != L.shape || M.shape.size() != 6) throw Error(CCQ_B200_EPLAN, "CRCC block shapes");
            CrccArgs &r = o.crcc;
            r.M = M.ptr;
            r.L = L.ptr;
            r.total = M.numel;
            for (int d = 0; d < 6; ++d) r.dims[d] = (int)M.shape[d];
            const int nb = x[0] - 'A';
            for (int k = 0; k < 3; ++k) r.spin[k] = k < 3 - nb ? 0 : 1;
            r.off[0] = (int)c->oa;
            r.off[1] = (int)c->ob;
            r.n = (int)c->n;
            r.fd[0] = c->fdiag_a;
            r.fd[1] = c->fdiag_b;
            r.hd[0] = c->bufs.at("HDA").ptr;
            r.hd[1] = c->bufs.at("HDB").ptr;
            r.h2aa = c->bufs.at("H2AA").ptr;
            r.h2ab = c->bufs.at("H2AB").ptr;
            r.h2bb = c->bufs.at("H2BB").ptr;
            for (int q = 0; q < 4; ++q) {
                r.w1[q] = c->bufs.at(std::string("W1") + char('A' + q)).ptr;
                r.w2[q] = c->bufs.at(std::string("W2") + char('A' + q)).ptr;
            }
            r.e23 = c->bufs.at("E23").ptr;
            r.act_occ_lo = (int)c->n;
            r.act_vir_hi = 0;
        }
        if (o.kind == OP_CRDIAG) {
            CrDiagArgs &g = c->crd;
            g.FA = c->bufs.at("FA").ptr;
            g.FB = c->bufs.at("FB").ptr;
            g.VAA = c->bufs.at("VAA").ptr;
            g.VAB = c->bufs.at("VAB").ptr;
            g.VBB = c->bufs.at("VBB").ptr;
            g.VAA0 = c->bufs.at("VAA0").ptr;
            g.VAB0 = c->bufs.at("VAB0").ptr;
            g.VBB0 = c->bufs.at("VBB0").ptr;
            g.T2A = c->bufs.at("T2A").ptr;
            g.T2B = c->bufs.at("T2B").ptr;
            g.T2C = c->bufs.at("T2C").ptr;
            g.HDA = c->bufs.at("HDA").ptr;
            g.HDB = c->bufs.at("HDB").ptr;
            g.H2AA = c->bufs.at("H2AA").ptr;
            g.H2AB = c->bufs.at("H2AB").ptr;
            g.H2BB = c->bufs.at("H2BB").ptr;
            for (int q = 0; q < 4; ++q) {
                g.W1[q] = c->bufs.at(std::string("W1") + char('A' + q)).ptr;
                g.W2[q] = c->bufs.at(std::string("W2") + char('A' + q)).ptr;
            }
            g.n = (int)c->n;
            g.oa = (int)c->oa;
            g.ob = (int)c->ob;
            g.va = (int)c->va;
            g.vb = (int)c->vb;
            // cal_d3's beta-beta-beta term sums e = occ_a + 2 .. orbs (src/mm_correct.f90:455-463):
            // beta virtuals from relative index occ_a - occ_b + 1
            g.w1d_e0 = (int)std::max(0LL, c->oa + 1 - c->ob);
        }
        if (o.kind == OP_GETT) {
            Resolved C = resolve(c, o.c), A = resolve(c, o.a), B = resolve(c, o.b);
            std::vector<std::string> ml, nl, kl;
            std::map<std::string, long long> ext;
            for (auto &l : A.order) {
                ext[l] = A.extent[l];
                if (has(C, l) && !has(B, l)) ml.push_back(l);
                else if (has(B, l) && !has(C, l)) kl.push_back(l);
                else throw Error(CCQ_B200_EPLAN, "label " + l + " of A must be in exactly one of B, C");
            }
            for (auto &l : B.order) {
                ext[l] = B.extent[l];
                if (has(C, l) && !has(A, l)) nl.push_back(l);
                else if (!has(A, l)) throw Error(CCQ_B200_EPLAN, "dangling label " + l);
            }
            for (auto &l : C.order) {
                if (!has(A, l) && !has(B, l)) throw Error(CCQ_B200_EPLAN, "output label not produced: " + l);
                if (C.extent[l] != ext[l]) throw Error(CCQ_B200_EPLAN, "extent mismatch for label " + l);
            }
            for (auto &l : kl)
                if (B.extent[l] != A.extent[l]) throw Error(CCQ_B200_EPLAN, "extent mismatch for label " + l);
            // Order each mode's labels so that the tensor dominating that mode's traffic is
            // walked along its contiguous axis: C for the small-K updates of large
            // outputs, the operands otherwise (the last label of a mode varies fastest).
            {
                auto prod = [&](const std::vector<std::string> &v) {
                    double x = 1;
                    for (auto &l : v) x *= (double)ext[l];
                    return x;
                };
                double Mx = prod(ml), Nx = prod(nl), Kx = prod(kl);
                auto by = [&](std::vector<std::string> &v, const Resolved &X) {
                    std::stable_sort(v.begin(), v.end(), [&](const std::string &a, const std::string &b) {
                        return X.stride.at(a) > X.stride.at(b);
                    });
                };
                double tC = Mx * Nx * (o.beta ? 2.0 : 1.0);
                // large-K contractions are operand bound (and may run split, whose
                // slicers read rows along the operand's contiguous axis)
                bool opnd = Kx >= 256;
                if (!opnd && tC >= Mx * Kx) by(ml, C); else by(ml, A);
                if (!opnd && tC >= Nx * Kx) by(nl, C); else by(nl, B);
                if (Mx >= Nx) by(kl, A); else by(kl, B);
            }
            // restriction groups: each must lie entirely in one index mode
            double kscale = 1.0;
            for (auto &g : o.restrict_groups) {
                auto in = [&](const std::vector<std::string> &lst) {
                    for (auto &l : g)
                        if (std::find(lst.begin(), lst.end(), l) == lst.end()) return false;
                    return true;
                };
                if (in(kl)) {
                    for (size_t q = 2; q <= g.size(); ++q) kscale *= (double)q;
                } else if (!in(ml) && !in(nl)) {
                    throw Error(CCQ_B200_EPLAN, "restriction group spans index modes");
                }
                for (auto &l : g)
                    if (ext[l] != ext[g[0]]) throw Error(CCQ_B200_EPLAN, "restriction group with unequal extents");
            }
            std::vector<int> am, ak, bn, bk, cm, cn;
            std::vector<const Op::ModeFilter *> fm, fn;
            for (auto &f : o.filters) (f.mode == 0 ? fm : fn).push_back(&f);
            build_table(ml, ext, A, &C, o.restrict_groups, fm, am, cm);
            build_table(kl, ext, A, &B, o.restrict_groups, {}, ak, bk);
            build_table(nl, ext, B, &C, o.restrict_groups, fn, bn, cn);
            o.hcm = cm;
            o.hcn = cn;
            if (ml.empty()) { am.assign(1, 0); cm.assign(1, 0); }
            if (nl.empty()) { bn.assign(1, 0); cn.assign(1, 0); }
            if (kl.empty()) { ak.assign(1, 0); bk.assign(1, 0); }
            Pend p{i, itab.size(), 0, 0, 0, 0, 0};
            itab.insert(itab.end(), am.begin(), am.end());
            p.ak = itab.size();
            itab.insert(itab.end(), ak.begin(), ak.end());
            p.bn = itab.size();
            itab.insert(itab.end(), bn.begin(), bn.end());
            p.bk = itab.size();
            itab.insert(itab.end(), bk.begin(), bk.end());
            p.cm = itab.size();
            itab.insert(itab.end(), cm.begin(), cm.end());
            p.cn = itab.size();
            itab.insert(itab.end(), cn.begin(), cn.end());
            pend.push_back(p);
            long long M = (long long)am.size(), N = (long long)bn.size(), K = (long long)ak.size();
            if (M > INT32_MAX || N > INT32_MAX || K > INT32_MAX || (N + 63) / 64 > 65535)
                throw Error(CCQ_B200_ERANGE, "GETT too large");
            o.mnk[0] = M;
            o.mnk[1] = N;
            o.mnk[2] = K;
            c->flops += 2.0 * M * N * K;
            auto kmajor = [](const Resolved &X, const std::vector<std::string> &mm, const std::vector<std::string> &kk) {
                long long sk = kk.empty() ? (1LL << 40) : X.stride.at(kk.back());
                long long sm = mm.empty() ? (1LL << 40) : X.stride.at(mm.back());
                return sk <= sm ? 1 : 0;
            };
            o.akm = kmajor(A, ml, kl);
            o.bkm = kmajor(B, nl, kl);
            {
                long long sn = nl.empty() ? (1LL << 40) : C.stride.at(nl.back());
                long long sm = ml.empty() ? (1LL << 40) : C.stride.at(ml.back());
                o.g.c_nfast = sn <= sm ? 1 : 0;
            }
            o.g.A = A.base;
            o.g.B = B.base;
            o.g.C = C.base;
            {
                // 16-byte paths: the walked table pairs up contiguous elements, every
                // element the pair starts at is even (16-byte aligned with the base)
                auto paired = [](const std::vector<int> &w, const std::vector<int> &other, const double *base) {
                    if (w.size() < 2 || w.size() % 2 || (reinterpret_cast<uintptr_t>(base) & 15)) return 0;
                    for (size_t i = 0; i < w.size(); i += 2)
                        if (w[i + 1] != w[i] + 1 || (w[i] & 1)) return 0;
                    for (int x : other)
                        if (x & 1) return 0;
                    return 1;
                };
                o.g.vec_a = o.akm ? paired(ak, am, A.base) : paired(am, ak, A.base);
                o.g.vec_b = o.bkm ? paired(bk, bn, B.base) : paired(bn, bk, B.base);
                o.g.vec_c = o.g.c_nfast ? paired(cn, cm, C.base) : paired(cm, cn, C.base);
            }
            o.g.M = (int)M;
            o.g.N = (int)N;
            o.g.K = (int)K;
            o.g.alpha = o.alpha * kscale;
            o.g.beta = o.beta;
            long long chunk = gett_f64_kchunk(M, N, K);
            o.g.kchunk = (int)chunk;
            o.zero_first = (K + chunk - 1) / chunk > 1 && o.beta == 0;
            if (K == 0) o.g.kchunk = 16;
            o.split = o.tag.size() > 2 && o.tag[0] == 'T' && (o.tag[1] == '3' || o.tag[1] == '4');
        } else if (o.kind == OP_ASM) {
            auto it = c->bufs.find(o.block);
            if (it == c->bufs.end()) throw Error(CCQ_B200_EPLAN, "assemble target " + o.block);
            const DevBuf &T = it->second;
            AsmArgs &a = o.asmargs;
            int level = o.block[1] - '0';
            int nb = (int)(strchr("ABCDE", o.block[2]) - "ABCDE");
            a.level = level;
            a.rank = 2 * level;
            if (a.rank > MAXR || (int)T.shape.size() != a.rank) throw Error(CCQ_B200_EPLAN, "block rank");
            std::vector<int> spins(level);
            for (int k = 0; k < level; ++k) spins[k] = k < level - nb ? 0 : 1;
            a.total = 1;
            for (int d = 0; d < a.rank; ++d) {
                a.dims[d] = (int)T.shape[d];
                a.tstride[d] = (int)T.stride[d];
                a.spin[d] = spins[d % level];
                a.runstart[d] = (d % level == 0) || spins[d % level] != spins[d % level - 1];
                a.total *= T.shape[d];
            }
            a.T = T.ptr;
            a.fdiag[0] = c->fdiag_a;
            a.fdiag[1] = c->fdiag_b;
            a.nocc[0] = (int)c->oa;
            a.nocc[1] = (int)c->ob;
            a.shift = c->shift;
            if (o.mode == "jacobi") {
                a.mode = 0;
            } else if (o.mode == "copy") {
                a.mode = 1;
            } else if (o.mode == "ljacobi") {
                // left Jacobi step: Hbar one-body diagonal, shift - E_cor, sum of LH^2 into LN
                a.mode = 2;
                a.fdiag[0] = c->bufs.at("HDA").ptr;
                a.fdiag[1] = c->bufs.at("HDB").ptr;
                a.ecor = c->bufs.at("ECOR").ptr;
                a.norm = c->bufs.at("LN").ptr;
            } else {
                throw Error(CCQ_B200_EPLAN, "assemble mode " + o.mode);
            }
            std::vector<std::string> target;
            for (int k = 0; k < level; ++k) target.push_back("i" + std::to_string(k));
            for (int k = 0; k < level; ++k) target.push_back("a" + std::to_string(k));
            PendA pa{i, hterms.size(), hperm.size()};
            // 32-bit offsets when the block, every source buffer and the element count fit
            bool off32 = T.numel < (1LL << 31);
            for (auto &t : o.terms) {
                Resolved V = resolve(c, t.second);
                const DevBuf &src = c->bufs.at(t.second.buf);
                off32 = off32 && src.numel < (1LL << 31);
                AsmTerm at{};
                at.p = V.base;
                at.coef = t.first;
                if (V.order.size() != (size_t)a.rank || t.second.axes.size() != (size_t)a.rank)
                    throw Error(CCQ_B200_EPLAN, "assemble term rank");
                at.rank = (signed char)a.rank;
                for (int j = 0; j < a.rank; ++j) {
                    const std::string &lab = t.second.axes[j].label;
                    auto it = std::find(target.begin(), target.end(), lab);
                    if (it == target.end() || V.extent[lab] != a.dims[it - target.begin()])
                        throw Error(CCQ_B200_EPLAN, "assemble term does not cover " + lab + " of " + o.block);
                    at.src[j] = (signed char)(it - target.begin());
                    at.zstride[j] = (int)src.stride[j];
                }
                if (src.groups.size() > (size_t)MAXG) throw Error(CCQ_B200_EPLAN, "too many antisymmetric groups");
                at.ng = (signed char)src.groups.size();
                for (size_t g = 0; g < src.groups.size(); ++g) {
                    at.glen[g] = (signed char)src.groups[g].size();
                    for (size_t q = 0; q < src.groups[g].size(); ++q) at.gpos[g][q] = (signed char)src.groups[g][q];
                }
                {
                    // A group read sorted with sign whose axes all hold indices of one same-spin run of the
                    // block: a canonical element's indices increase along that run, so the sort is the same
                    // for every element. It is applied here (axes reassigned, sign into the coefficient)
                    // and the term becomes a plain view, read without a per-element sort.
                    std::vector<int> run_of(a.rank);
                    int r = -1;
                    for (int d = 0; d < a.rank; ++d) {
                        if (a.runstart[d]) ++r;
                        run_of[d] = r;
                    }
                    bool fixed = at.ng > 0;
                    for (int g = 0; g < at.ng && fixed; ++g)
                        for (int q = 1; q < at.glen[g]; ++q)
                            fixed = fixed && run_of[at.src[at.gpos[g][q]]] == run_of[at.src[at.gpos[g][0]]];
                    if (fixed) {
                        for (int g = 0; g < at.ng; ++g) {
                            std::vector<int> ax(at.gpos[g], at.gpos[g] + at.glen[g]);
                            std::sort(ax.begin(), ax.end());
                            std::vector<int> tg;
                            for (int x : ax) tg.push_back(at.src[x]);
                            int inv = 0;
                            for (size_t u = 0; u < tg.size(); ++u)
                                for (size_t w = u + 1; w < tg.size(); ++w) inv += tg[w] < tg[u];
                            if (inv & 1) at.coef = -at.coef;
                            std::sort(tg.begin(), tg.end());
                            for (size_t u = 0; u < ax.size(); ++u) at.src[ax[u]] = (signed char)tg[u];
                        }
                        at.ng = 0;
                    }
                }
                hterms.push_back(at);
            }
            a.nterms = (int)o.terms.size();
            if (a.nterms > MAX_TERMS) throw Error(CCQ_B200_EPLAN, "too many assemble terms");
            a.off32 = off32 ? 1 : 0;
            {
                // plain views (no antisymmetric group of two or more axes) ahead of the sorted ones
                auto plain = [](const AsmTerm &x) {
                    for (int g = 0; g < x.ng; ++g)
                        if (x.glen[g] > 1) return false;
                    return true;
                };
                auto first = hterms.begin() + (long)pa.t0;
                auto mid = std::stable_partition(first, hterms.end(), plain);
                a.nplain = (int)(mid - first);
            }
            // orbit permutations: within same-spin runs of each half
            std::vector<std::vector<int>> runs;
            for (int half = 0; half < 2; ++half) {
                int d = half * level;
                while (d < (half + 1) * level) {
                    int e = d + 1;
                    while (e < (half + 1) * level && spins[e % level] == spins[d % level]) ++e;
                    std::vector<int> r;
                    for (int q = d; q < e; ++q) r.push_back(q);
                    runs.push_back(r);
                    d = e;
                }
            }
            std::vector<std::vector<std::pair<std::vector<int>, int>>> rp;
            for (auto &r : runs) {
                std::vector<int> p(r.size());
                for (size_t q = 0; q < r.size(); ++q) p[q] = (int)q;
                std::vector<std::pair<std::vector<int>, int>> lst;
                do {
                    int sg = 1;
                    for (size_t x = 0; x < p.size(); ++x)
                        for (size_t y = x + 1; y < p.size(); ++y)
                            if (p[y] < p[x]) sg = -sg;
                    lst.push_back({p, sg});
                } while (std::next_permutation(p.begin(), p.end()));
                rp.push_back(lst);
            }
            std::vector<size_t> cur(rp.size(), 0);
            int np = 0;
            while (true) {
                std::vector<signed char> P(a.rank);
                int sg = 1;
                for (size_t r = 0; r < runs.size(); ++r) {
                    auto &pr = rp[r][cur[r]];
                    sg *= pr.second;
                    for (size_t q = 0; q < runs[r].size(); ++q) P[runs[r][q]] = (signed char)runs[r][pr.first[q]];
                }
                hperm.insert(hperm.end(), P.begin(), P.end());
                hsign.push_back((signed char)sg);
                ++np;
                size_t r = 0;
                while (r < rp.size() && ++cur[r] == rp[r].size()) cur[r++] = 0;
                if (r == rp.size()) break;
            }
            a.nperm = np;
            // canonical enumeration tables: increasing tuples of every run
            a.nruns = (int)runs.size();
            a.total = 1;
            for (size_t r = 0; r < runs.size(); ++r) {
                int L = (int)runs[r].size(), n = a.dims[runs[r][0]];
                if (n > 255) throw Error(CCQ_B200_ERANGE, "orbital extent above 255");
                a.run_axis0[r] = runs[r][0];
                a.run_len[r] = L;
                a.run_off[r] = (int)hcomb.size();
                std::vector<int> t(L);
                for (int l = 0; l < L; ++l) t[l] = l;
                int cnt = 0;
                if (L <= n) {
                    while (true) {
                        for (int l = 0; l < L; ++l) hcomb.push_back((unsigned char)t[l]);
                        ++cnt;
                        int l = L - 1;
                        while (l >= 0 && t[l] == n - L + l) --l;
                        if (l < 0) break;
                        ++t[l];
                        for (int q = l + 1; q < L; ++q) t[q] = t[q - 1] + 1;
                    }
                }
                a.run_count[r] = cnt;
                a.total *= cnt;
            }
            penda.push_back(pa);
        }
    }
    int *dtab = (int *)c->dalloc(sizeof(int) * std::max<size_t>(itab.size(), 1));
    CK(cudaMemcpyAsync(dtab, itab.data(), sizeof(int) * itab.size(), cudaMemcpyHostToDevice, c->stream));
    for (auto &p : pend) {
        Op &o = c->plan.ops[p.op];
        o.g.offA_m = dtab + p.am;
        o.g.offA_k = dtab + p.ak;
        o.g.offB_n = dtab + p.bn;
        o.g.offB_k = dtab + p.bk;
        o.g.offC_m = dtab + p.cm;
        o.g.offC_n = dtab + p.cn;
    }
    if (c->trace_init)
        fprintf(stderr, "ccq_b200_init table entries %zu, ops %zu, assemble terms %zu\n", itab.size(),
                c->plan.ops.size(), hterms.size());
    trace_stamp(c, "op tables");
    // Group small-K contractions that add into the same Z buffer with the same output tables (the
    // same split of Z's axes between the two operands; a writer whose tables match with the operands
    // exchanged is exchanged): one launch per group at the position of its last member.  Their
    // operands are not modified later in the phase (work buffers of one phase never share memory,
    // amplitudes change only in the closing assemble) and Z is only read by that assemble, so moving
    // the earlier members later is safe.  Every write into Z adds, except the first one executed,
    // which overwrites: the overwrite flag follows the new order.  With active-space filters (an op
    // split into pieces that must share one flag) only consecutive writers group, keeping the flags.
    {
        std::vector<GettSeg> hsegs;
        std::vector<std::pair<size_t, size_t>> leaders;
        auto groupable = [&](const Op &o) {
            return o.kind == OP_GETT && o.g.M > 0 && o.g.N > 0 && o.g.K > 0 && o.g.K < 256 && !o.zero_first &&
                   (o.g.K + o.g.kchunk - 1) / o.g.kchunk == 1 && o.c.buf[0] == 'Z' && !o.frozen;
        };
        bool any_filter = false;
        for (auto &o : c->plan.ops) any_filter = any_filter || !o.filters.empty();
        // 0: no match, 1: same tables, 2: tables of the exchanged operands
        auto match = [&](const Op &q, const Op &f) {
            if (q.g.C != f.g.C) return 0;
            if (q.hcm == f.hcm && q.hcn == f.hcn && q.g.c_nfast == f.g.c_nfast) return 1;
            if (!any_filter && q.hcm == f.hcn && q.hcn == f.hcm) return 2;
            return 0;
        };
        size_t b = 0;
        while (b < c->plan.ops.size()) {
            size_t e = b + 1;
            while (e < c->plan.ops.size() && c->plan.ops[e].kind != OP_PHASE) ++e;
            std::map<std::string, std::vector<size_t>> writers;
            for (size_t i = b; i < e; ++i) {
                Op &o = c->plan.ops[i];
                if (o.kind == OP_GETT && o.c.buf[0] == 'Z') writers[o.c.buf].push_back(i);
            }
            for (auto &wz : writers) {
                auto &lst = wz.second;
                // classes of mutually matching groupable writers (consecutive runs only with filters)
                std::vector<std::vector<std::pair<size_t, int>>> cls;   // (op, 1 same / 2 exchanged vs first)
                std::vector<std::pair<size_t, int>> run;
                for (size_t q = 0; q < lst.size(); ++q) {
                    Op &o = c->plan.ops[lst[q]];
                    if (!groupable(o)) {
                        if (any_filter && !run.empty()) {
                            cls.push_back(run);
                            run.clear();
                        }
                        continue;
                    }
                    if (any_filter) {
                        if (!run.empty() && match(o, c->plan.ops[run[0].first]) != 1) {
                            cls.push_back(run);
                            run.clear();
                        }
                        run.push_back({lst[q], 1});
                        continue;
                    }
                    bool placed = false;
                    for (auto &cl : cls) {
                        const int m = match(o, c->plan.ops[cl[0].first]);
                        if (m) {
                            cl.push_back({lst[q], m});
                            placed = true;
                            break;
                        }
                    }
                    if (!placed) cls.push_back({{lst[q], 1}});
                }
                if (!run.empty()) cls.push_back(run);
                bool regrouped = false;
                for (auto &cl : cls) {
                    if (cl.size() < 2) continue;
                    regrouped = true;
                    Op &lead = c->plan.ops[cl.back().first];
                    const int lead_m = cl.back().second;
                    size_t off = hsegs.size();
                    double fl = 0.0;
                    for (auto &mm : cl) {
                        Op &m = c->plan.ops[mm.first];
                        // orientation relative to the leader: exchange A and B where it differs
                        if (mm.second == lead_m)
                            hsegs.push_back(GettSeg{m.g.A, m.g.B, m.g.offA_m, m.g.offA_k, m.g.offB_n, m.g.offB_k,
                                                    m.g.K, m.g.alpha});
                        else
                            hsegs.push_back(GettSeg{m.g.B, m.g.A, m.g.offB_n, m.g.offB_k, m.g.offA_m, m.g.offA_k,
                                                    m.g.K, m.g.alpha});
                        fl += 2.0 * m.mnk[0] * m.mnk[1] * m.mnk[2];
                        if (&m != &lead) m.skip = true;
                    }
                    for (auto &mm : cl) {
                        const Op &m = c->plan.ops[mm.first];
                        const bool same = mm.second == lead_m;
                        lead.g.vec_a = lead.g.vec_a && (same ? m.g.vec_a && m.akm == lead.akm
                                                             : m.g.vec_b && m.bkm == lead.akm);
                        lead.g.vec_b = lead.g.vec_b && (same ? m.g.vec_b && m.bkm == lead.bkm
                                                             : m.g.vec_a && m.akm == lead.bkm);
                    }
                    lead.g.beta = c->plan.ops[cl[0].first].beta;
                    lead.g.nseg = (int)cl.size();
                    for (auto &mm : cl) lead.group_ops.push_back(mm.first);
                    lead.group_flops = fl;
                    lead.group_size = (int)cl.size();
                    leaders.push_back({cl.back().first, off});
                }
                if (!regrouped || any_filter) continue;
                // the first write executed into Z overwrites it, the others add
                bool first = true;
                for (size_t i : lst) {
                    Op &o = c->plan.ops[i];
                    if (o.skip || o.frozen || o.g.M == 0 || o.g.N == 0) continue;
                    o.beta = first ? 0 : 1;
                    o.g.beta = o.beta;
                    o.zero_first = !o.g.segs && o.group_ops.empty() && o.beta == 0 &&
                                   (o.g.K + o.g.kchunk - 1) / o.g.kchunk > 1;
                    first = false;
                }
            }
            b = e;
        }
        if (!hsegs.empty()) {
            GettSeg *dsegs = (GettSeg *)c->dalloc(sizeof(GettSeg) * hsegs.size());
            CK(cudaMemcpyAsync(dsegs, hsegs.data(), sizeof(GettSeg) * hsegs.size(), cudaMemcpyHostToDevice,
                               c->stream));
            for (auto &l : leaders) c->plan.ops[l.first].g.segs = dsegs + l.second;
        }
    }
    trace_stamp(c, "grouping");
    AsmTerm *dterms = (AsmTerm *)c->dalloc(sizeof(AsmTerm) * std::max<size_t>(hterms.size(), 1));
    CK(cudaMemcpyAsync(dterms, hterms.data(), sizeof(AsmTerm) * hterms.size(), cudaMemcpyHostToDevice, c->stream));
    signed char *dperm = (signed char *)c->dalloc(std::max<size_t>(hperm.size(), 1));
    signed char *dsign = (signed char *)c->dalloc(std::max<size_t>(hsign.size(), 1));
    CK(cudaMemcpyAsync(dperm, hperm.data(), hperm.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dsign, hsign.data(), hsign.size(), cudaMemcpyHostToDevice, c->stream));
    unsigned char *dcomb = (unsigned char *)c->dalloc(std::max<size_t>(hcomb.size(), 1));
    CK(cudaMemcpyAsync(dcomb, hcomb.data(), hcomb.size(), cudaMemcpyHostToDevice, c->stream));
    {
        size_t signs_before = 0;
        for (auto &p : penda) {
            c->plan.ops[p.op].asmargs.combos = dcomb;
            Op &o = c->plan.ops[p.op];
            o.asmargs.terms = dterms + p.t0;
            o.asmargs.perm = dperm + p.p0;
            o.asmargs.psign = dsign + signs_before;
            signs_before += o.asmargs.nperm;
        }
    }
    // ring and scratch
    c->ring = (double *)c->dalloc(sizeof(double) * (size_t)(c->ds + 1) * std::max(c->vec_size, 1LL));
    c->scratch = (double *)c->dalloc(sizeof(double) * 512);
    c->dinfo = (int *)c->dalloc(sizeof(int) * 4);
    CK(cudaStreamSynchronize(c->stream));
}

// the op runs on the split-precision kernel in this context's current mode
bool use_split(const ccq_b200_ctx *c, const Op &o) {
    if (c->precision != CCQ_B200_PREC_SPLIT || !o.split) return false;
    return o.split_choice >= 0 ? o.split_choice >= 1 : split_eligible(o.g);
}

// persistent split kernel (one CTA per SM, overlapped epilogue) unless tuned to the per-tile one
int split_persistent(const Op &o) { return o.split_choice == 1 ? 0 : 1; }

// split GETTs of a sweep rotate over this many slicing workspaces when one takes at most kSplitPoolBytes
constexpr int kSplitPool = 3;
constexpr long long kSplitPoolBytes = 1LL << 30;

SplitWorkspace &split_ws(ccq_b200_ctx *c, const Op &o) {
    return o.split_ws > 0 && o.split_ws <= (int)c->split_pool.size() ? c->split_pool[o.split_ws - 1] : c->split;
}

int op_class(const ccq_b200_ctx *c, const Op &o) {
    if (o.kind == OP_GETT) return use_split(c, o) ? 1 : 0;
    if (o.kind == OP_ASM) return 2;
    return 3;
}

void run_op(ccq_b200_ctx *c, Op &o, cudaStream_t st) {
    if (o.frozen) return;
    switch (o.kind) {
        case OP_GETT:
            if (o.skip || o.g.M == 0 || o.g.N == 0) break;
            if (o.zero_first) {
                launch_zero_view(o.g.C, o.g.offC_m, o.g.offC_n, o.g.M, o.g.N, st);
                ++c->launches;
            }
            if (o.g.K == 0) {
                if (!o.beta) {
                    launch_zero_view(o.g.C, o.g.offC_m, o.g.offC_n, o.g.M, o.g.N, st);
                    ++c->launches;
                }
                break;
            }
            if (use_split(c, o)) {
                c->launches += split_gett(split_ws(c, o), o.g, o.akm, o.bkm, c->nslices, st, split_persistent(o));
            } else {
                launch_gett_f64(o.g, o.akm, o.bkm, st);
                ++c->launches;
            }
            break;
        case OP_ASM:
            launch_assemble(o.asmargs, st);
            ++c->launches;
            break;
        case OP_COPY: {
            DevBuf &d = c->bufs.at(o.arg0);
            DevBuf &s = c->bufs.at(o.arg1);
            if (d.numel != s.numel) throw Error(CCQ_B200_EPLAN, "COPY size mismatch");
            CK(cudaMemcpyAsync(d.ptr, s.ptr, sizeof(double) * d.numel, cudaMemcpyDeviceToDevice, st));
            break;
        }
        case OP_ZERO: {
            DevBuf &d = c->bufs.at(o.arg0);
            CK(cudaMemsetAsync(d.ptr, 0, sizeof(double) * std::max(d.numel, 1LL), st));
            break;
        }
        case OP_PHASE:
            break;
        case OP_CRDIAG:
            launch_crdiag(c->crd, st);
            ++c->launches;
            break;
        case OP_LENERGY:
            launch_lenergy(c->bufs.at("LN").ptr, c->bufs.at("ECOR").ptr, c->bufs.at("EL").ptr, st);
            ++c->launches;
            break;
        case OP_CRCC:
            launch_crcc_sum(o.crcc, st);
            ++c->launches;
            break;
    }
}

// ops[from, to) issued for stream capture as a DAG.  Every GETT waits only for
// the GETTs it reads from, the last overwrite of its output and the earlier
// readers of that output; beta = 1 writers of one buffer do not wait for each
// other (their epilogues add with reductions).  Jacobi and copy assembles,
// buffer copies and zeroing are nodes of the same kind (they overwrite their
// output), so an assemble overlaps the next block's contractions that do not
// read it.  The rest (split GETTs, whose slicing shares one workspace, and the
// left-solve and CR-CC(2,3) kernels that accumulate scalars) is a barrier on
// the capturing stream.  Independent contractions then run on side
// streams at the same time.
// every t_vec block resident on the device, and the last sweep op that writes it
void prepare_copy_out(ccq_b200_ctx *c) {
    if (c->out_ready) return;
    c->out_after.clear();
    for (auto &b : c->plan.bufs) {
        if (b.kind != "amp") continue;
        const DevBuf &d = c->bufs.at(b.name);
        if (!d.ptr || d.ptr < c->tvec || d.ptr >= c->tvec + c->t_dev) continue;
        size_t last = (size_t)-1;
        for (size_t i = 0; i < c->cc_end; ++i) {
            const Op &o = c->plan.ops[i];
            if ((o.kind == OP_ASM && o.block == b.name) || (o.kind == OP_COPY && o.arg0 == b.name)) last = i;
        }
        c->out_after.push_back({last, b.name});
    }
    if (!c->cstream) {
        CK(cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->cjoin, cudaEventDisableTiming));
    }
    if (c->cev.size() < c->out_after.size()) {
        for (size_t k = c->cev.size(); k < c->out_after.size(); ++k) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            c->cev.push_back(e);
        }
    }
    c->out_ready = true;
}

// Copy-mode assembles reading the T3 blocks of the mapped host t_vec at their canonical elements (built
// before a sweep with host_in is captured); cin_h2d counts the bytes that then cross the host link.
void prepare_copy_in(ccq_b200_ctx *c) {
    c->cin_args.clear();
    c->cin_h2d = sizeof(double) * c->t_dev;
    if (!c->host_in || !c->host_in_dev) return;
    auto source = [&](const std::string &name) -> const Op * {
        for (size_t i = 0; i < c->cc_end; ++i) {
            const Op &o = c->plan.ops[i];
            if (o.kind == OP_ASM && o.block == name && (o.asmargs.mode == 0 || o.asmargs.mode == 1)) return &o;
        }
        return nullptr;
    };
    std::vector<AsmTerm> terms;
    std::vector<std::string> names;
    for (auto &b : c->plan.bufs) {
        if (b.kind != "amp") continue;
        const DevBuf &d = c->bufs.at(b.name);
        if (!d.ptr || d.ptr < c->tvec || d.ptr >= c->tvec + c->t_dev || d.shape.size() != 6) continue;
        const Op *src = source(b.name);
        if (!src) continue;
        AsmTerm t{};
        t.p = c->host_in_dev + (d.ptr - c->tvec);
        t.coef = 1.0;
        t.rank = 6;
        for (int j = 0; j < 6; ++j) {
            t.src[j] = (signed char)j;
            t.zstride[j] = src->asmargs.tstride[j];
        }
        terms.push_back(t);
        names.push_back(b.name);
    }
    if (terms.empty()) return;
    if (!c->cin_terms) {
        size_t cap = 0;
        for (auto &b : c->plan.bufs) cap += b.kind == "amp";
        c->cin_terms = (AsmTerm *)c->dalloc(sizeof(AsmTerm) * std::max<size_t>(cap, 1));
    }
    CK(cudaMemcpy(c->cin_terms, terms.data(), sizeof(AsmTerm) * terms.size(), cudaMemcpyHostToDevice));
    for (size_t k = 0; k < names.size(); ++k) {
        AsmArgs a = source(names[k])->asmargs;
        a.mode = 1;
        a.nterms = 1;
        a.nplain = 1;
        a.terms = c->cin_terms + k;
        a.act = 0;
        a.ecor = nullptr;
        a.norm = nullptr;
        c->cin_args[names[k]] = a;
        const DevBuf &d = c->bufs.at(names[k]);
        c->cin_h2d -= sizeof(double) * (d.numel - a.total);   // only the canonical elements cross
    }
}

void copy_block_out(ccq_b200_ctx *c, size_t k, cudaStream_t after) {
    const DevBuf &d = c->bufs.at(c->out_after[k].second);
    CK(cudaEventRecord(c->cev[k], after));
    CK(cudaStreamWaitEvent(c->cstream, c->cev[k], 0));
    CK(cudaMemcpyAsync(c->host_out + (d.ptr - c->tvec), d.ptr, sizeof(double) * d.numel, cudaMemcpyDeviceToHost,
                       c->cstream));
}

// copies of the blocks whose last write is op i (after it has been issued on stream st)
void copy_out_after(ccq_b200_ctx *c, size_t i, cudaStream_t st) {
    if (!c->host_out || c->plan.ops[i].frozen) return;
    for (size_t k = 0; k < c->out_after.size(); ++k)
        if (c->out_after[k].first == i) copy_block_out(c, k, st);
}

// blocks the sweep does not write (held fixed) go at its end; then the copy stream joins st
void copy_out_finish(ccq_b200_ctx *c, cudaStream_t st) {
    if (!c->host_out) return;
    for (size_t k = 0; k < c->out_after.size(); ++k)
        if (c->out_after[k].first == (size_t)-1 || c->plan.ops[c->out_after[k].first].frozen) copy_block_out(c, k, st);
    CK(cudaEventRecord(c->cjoin, c->cstream));
    CK(cudaStreamWaitEvent(st, c->cjoin, 0));
}

void run_ops_dag(ccq_b200_ctx *c, size_t from, size_t to) {
    // side streams of the captured dependency graph (CCQ_B200_DAG_STREAMS, 1..32, default 10: CCSDT-40
    // split 13.63 / 12.81 / 12.51 / 12.55 ms per iteration with 3 / 6 / 10 / 16)
    static const int NSIDE = [] {
        const char *e = getenv("CCQ_B200_DAG_STREAMS");
        const int v = e ? atoi(e) : 10;
        return v >= 1 && v <= 32 ? v : 10;
    }();
    if (c->side.empty()) {
        c->side.resize(NSIDE);
        for (auto &st : c->side) CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->cap_ev, cudaEventDisableTiming));
    }
    if (c->opev.size() < c->plan.ops.size()) {
        size_t old = c->opev.size();
        c->opev.resize(c->plan.ops.size(), nullptr);
        for (size_t i = old; i < c->opev.size(); ++i) CK(cudaEventCreateWithFlags(&c->opev[i], cudaEventDisableTiming));
    }
    struct BufState {
        std::vector<size_t> writers, full, readers;
    };
    std::map<std::string, BufState> st;
    std::vector<size_t> pending;
    // CCQ_B200_DAG_SERIAL set: assembles, copies and zeroing are barriers (the earlier schedule, for comparison)
    const bool serial_nodes = getenv("CCQ_B200_DAG_SERIAL") != nullptr;
    cudaEvent_t gate = c->cap_ev;   // the last barrier (or the capture's start)
    CK(cudaEventRecord(gate, c->stream));
    int rr = 0;
    std::vector<long long> last_on(NSIDE, -1);   // last node issued on each side stream since the last barrier
    static const bool round_robin = getenv("CCQ_B200_DAG_ROUND_ROBIN") != nullptr;
    auto join = [&]() {
        for (size_t j : pending) CK(cudaStreamWaitEvent(c->stream, c->opev[j], 0));
        pending.clear();
        st.clear();
        std::fill(last_on.begin(), last_on.end(), -1LL);
    };
    if (c->host_in && from == 0) {
        // the t_vec from the host, one node per amplitude block in t_vec order (T1, T2, then the T3 blocks)
        // that the block's readers wait for (pseudo-op index ops.size() + k)
        std::vector<std::pair<long long, std::string>> blk;
        for (auto &b : c->plan.bufs) {
            if (b.kind != "amp") continue;
            const DevBuf &d = c->bufs.at(b.name);
            if (d.ptr && d.ptr >= c->tvec && d.ptr < c->tvec + c->t_dev) blk.push_back({d.ptr - c->tvec, b.name});
        }
        std::sort(blk.begin(), blk.end());
        const size_t base = c->plan.ops.size();
        if (c->opev.size() < base + blk.size() + 1) {
            size_t old = c->opev.size();
            c->opev.resize(base + blk.size() + 1, nullptr);
            for (size_t i = old; i < c->opev.size(); ++i)
                CK(cudaEventCreateWithFlags(&c->opev[i], cudaEventDisableTiming));
        }
        if (!c->istream) CK(cudaStreamCreateWithFlags(&c->istream, cudaStreamNonBlocking));
        CK(cudaStreamWaitEvent(c->istream, gate, 0));
        // every element of [0, t_dev) once: block k covers up to the next block's start
        long long lo = 0;
        for (size_t k = 0; k < blk.size(); ++k) {
            const long long hi = k + 1 < blk.size() ? blk[k + 1].first : c->t_dev;
            auto ca = c->cin_args.find(blk[k].second);
            if (ca != c->cin_args.end()) {
                // canonical elements from the mapped host block, antisymmetric images written on the device
                launch_assemble(ca->second, c->istream);
                const long long end = blk[k].first + c->bufs.at(blk[k].second).numel;
                if (lo < blk[k].first)
                    CK(cudaMemcpyAsync(c->tvec + lo, c->host_in + lo, sizeof(double) * (blk[k].first - lo),
                                       cudaMemcpyHostToDevice, c->istream));
                if (end < hi)
                    CK(cudaMemcpyAsync(c->tvec + end, c->host_in + end, sizeof(double) * (hi - end),
                                       cudaMemcpyHostToDevice, c->istream));
            } else {
                CK(cudaMemcpyAsync(c->tvec + lo, c->host_in + lo, sizeof(double) * (hi - lo), cudaMemcpyHostToDevice,
                                   c->istream));
            }
            lo = hi;
            CK(cudaEventRecord(c->opev[base + k], c->istream));
            st[blk[k].second].writers.assign(1, base + k);
            st[blk[k].second].full.assign(1, base + k);
            pending.push_back(base + k);
        }
        if (blk.empty()) {
            CK(cudaMemcpyAsync(c->tvec, c->host_in, sizeof(double) * c->t_dev, cudaMemcpyHostToDevice, c->istream));
            CK(cudaEventRecord(c->opev[base], c->istream));
            pending.push_back(base);
        }
    }
    for (size_t i = from; i < to; ++i) {
        Op &o = c->plan.ops[i];
        if (o.kind == OP_PHASE || o.frozen) continue;
        if (o.kind == OP_GETT && (o.skip || o.g.M == 0 || o.g.N == 0)) continue;
        // Jacobi / copy assembles, buffer copies and zeroing are nodes too: each reads its term
        // buffers (and its own block) and overwrites one buffer
        const bool plain_node = !serial_nodes && ((o.kind == OP_ASM && o.asmargs.mode != 2) ||
                                                  o.kind == OP_COPY || o.kind == OP_ZERO);
        // a split GETT is a barrier only while every split GETT shares one slicing workspace
        const bool splitop = o.kind == OP_GETT && use_split(c, o);
        const bool barrier = (o.kind != OP_GETT && !plain_node) || (splitop && c->split_pool.empty());
        if (barrier) {
            join();
            run_op(c, o, c->stream);
            CK(cudaEventRecord(c->opev[i], c->stream));
            gate = c->opev[i];
            copy_out_after(c, i, c->stream);
            continue;
        }
        std::vector<size_t> deps;
        auto add = [&](const std::vector<size_t> &v) { deps.insert(deps.end(), v.begin(), v.end()); };
        std::vector<std::string> ins;
        std::string out;
        bool overwrite = true;
        if (o.kind == OP_GETT) {
            ins = {o.a.buf, o.b.buf};
            for (size_t m : o.group_ops) {
                ins.push_back(c->plan.ops[m].a.buf);
                ins.push_back(c->plan.ops[m].b.buf);
            }
            out = o.c.buf;
            // a grouped launch carries the beta of its first member (g.beta), not its own
            overwrite = !o.g.beta || o.zero_first || o.g.K == 0;
        } else if (o.kind == OP_ASM) {
            for (auto &t : o.terms) ins.push_back(t.second.buf);
            ins.push_back(o.block);
            out = o.block;
        } else if (o.kind == OP_COPY) {
            ins = {o.arg1};
            out = o.arg0;
        } else {
            out = o.arg0;
        }
        // the Z/X work buffers of different block phases share one arena: an access also waits for
        // every earlier access to a buffer whose memory overlaps
        auto alias_deps = [&](const std::string &nm) {
            auto it = c->bufs.find(nm);
            if (it == c->bufs.end() || !it->second.ptr) return;
            const double *lo = it->second.ptr, *hi = lo + std::max(it->second.numel, 1LL);
            for (auto &kv : st) {
                if (kv.first == nm) continue;
                auto jt = c->bufs.find(kv.first);
                if (jt == c->bufs.end() || !jt->second.ptr) continue;
                const double *l2 = jt->second.ptr, *h2 = l2 + std::max(jt->second.numel, 1LL);
                if (l2 < hi && lo < h2) {
                    add(kv.second.writers);
                    add(kv.second.readers);
                    add(kv.second.full);
                }
            }
        };
        for (auto &b : ins) {
            add(st[b].writers);
            alias_deps(b);
        }
        alias_deps(out);
        // the slicing workspace of a split GETT: wait for its previous user
        const std::string wsname = splitop ? "@split" + std::to_string(o.split_ws) : std::string();
        if (splitop) {
            add(st[wsname].writers);
            add(st[wsname].readers);
        }
        BufState &cs = st[out];
        add(cs.readers);
        add(overwrite ? cs.writers : cs.full);
        std::sort(deps.begin(), deps.end());
        deps.erase(std::unique(deps.begin(), deps.end()), deps.end());
        // a captured stream orders its operations, so the stream chosen adds an edge from its last node:
        // take the stream whose last node is the latest of this node's dependencies (a true edge), else
        // the stream whose last node is the oldest (round robin when CCQ_B200_DAG_ROUND_ROBIN is set)
        int si = rr++ % NSIDE;
        if (!round_robin) {
            int best = -1;
            for (int q = 0; q < NSIDE; ++q)
                if (last_on[q] >= 0 && std::binary_search(deps.begin(), deps.end(), (size_t)last_on[q]) &&
                    (best < 0 || last_on[q] > last_on[best]))
                    best = q;
            if (best < 0)
                for (int q = 0; q < NSIDE; ++q)
                    if (best < 0 || last_on[q] < last_on[best]) best = q;
            si = best;
        }
        last_on[si] = (long long)i;
        cudaStream_t sd = c->side[si];
        CK(cudaStreamWaitEvent(sd, gate, 0));
        for (size_t d : deps) CK(cudaStreamWaitEvent(sd, c->opev[d], 0));
        run_op(c, o, sd);
        CK(cudaEventRecord(c->opev[i], sd));
        copy_out_after(c, i, sd);
        pending.push_back(i);
        if (splitop) {
            st[wsname].writers.assign(1, i);
            st[wsname].readers.clear();
        }
        for (auto &b : ins) st[b].readers.push_back(i);
        if (overwrite) {
            cs.writers.assign(1, i);
            cs.full.assign(1, i);
            cs.readers.clear();
        } else {
            cs.writers.push_back(i);
        }
    }
    join();
    CK(cudaGetLastError());
}

void run_ops(ccq_b200_ctx *c, size_t from, size_t to) {
    bool prof = c->profile != 0;
    if (prof && c->pev.size() < 2 * c->plan.ops.size()) {
        for (auto e : c->pev) cudaEventDestroy(e);
        c->pev.assign(2 * c->plan.ops.size(), nullptr);
        for (auto &e : c->pev) CK(cudaEventCreate(&e));
    }
    for (size_t i = from; i < to; ++i) {
        Op &o = c->plan.ops[i];
        if (prof) CK(cudaEventRecord(c->pev[2 * i], c->stream));
        run_op(c, o, c->stream);
        if (prof) CK(cudaEventRecord(c->pev[2 * i + 1], c->stream));
        copy_out_after(c, i, c->stream);
    }
    CK(cudaGetLastError());
    if (prof) {
        CK(cudaStreamSynchronize(c->stream));
        const char *dump = getenv("CCQ_B200_PROFILE_DUMP");
        FILE *df = dump ? fopen(dump, "a") : nullptr;
        for (size_t i = from; i < to; ++i) {
            Op &o = c->plan.ops[i];
            if (o.kind == OP_PHASE || (o.kind == OP_GETT && o.skip)) continue;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->pev[2 * i], c->pev[2 * i + 1]));
            int k = op_class(c, o);
            c->prof_ms[k] += ms;
            c->prof_launch[k] += 1;
            const double fl = o.group_size ? o.group_flops : 2.0 * o.mnk[0] * o.mnk[1] * o.mnk[2];
            if (o.kind == OP_GETT) c->prof_flops[k] += fl;
            if (df) {
                if (o.kind == OP_GETT)
                    // ... tile choice (0: by shape), shape family (0: 64 x 64, 1/2: skinny rows/columns)
                    fprintf(df, "%zu GETT %d %s %lld %lld %lld %d %d %d %.6f %d %.6e %d %d\n", i, k, o.tag.c_str(),
                            o.mnk[0], o.mnk[1], o.mnk[2], o.akm, o.bkm, o.beta, ms, o.group_size, fl, o.g.tile,
                            gett_f64_family(o.g.M, o.g.N));
                else if (o.kind == OP_ASM)
                    fprintf(df, "%zu ASM %d %s %d %.6f\n", i, k, o.block.c_str(), o.asmargs.nterms, ms);
                else
                    fprintf(df, "%zu OTHER %d %s %.6f\n", i, k, o.arg0.c_str(), ms);
            }
        }
        if (df) fclose(df);
    }
}

void sweep(ccq_b200_ctx *c) {
    // with host_out set, the captured graph also holds the copy-out of every finished block
    if (c->host_out) prepare_copy_out(c);
    cudaGraphExec_t &ge = c->host_out ? c->gexec_host : (c->host_in ? c->gexec_hin : c->gexec);
    if (c->use_graph && !c->profile) {
        if (!ge) {
            if (c->host_out || c->host_in) prepare_copy_in(c);
            cudaGraph_t g;
            long long l0 = c->launches;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            try {
                if (c->use_graph == 2)
                    run_ops(c, 0, c->cc_end);
                else
                    run_ops_dag(c, 0, c->cc_end);
                copy_out_finish(c, c->stream);
            } catch (...) {
                cudaStreamEndCapture(c->stream, &g);
                throw;
            }
            CK(cudaStreamEndCapture(c->stream, &g));
            CK(cudaGraphInstantiate(&ge, g, 0));
            CK(cudaGraphDestroy(g));
            c->launches = l0 + (c->launches - l0);
        }
        CK(cudaGraphLaunch(ge, c->stream));
    } else {
        run_ops(c, 0, c->cc_end);
        copy_out_finish(c, c->stream);
    }
}


// every captured graph of the context (kernel arguments, op flags and copy targets are recorded in them)
void drop_graphs(ccq_b200_ctx *c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->lgexec) cudaGraphExecDestroy(c->lgexec);
    if (c->gexec_host) cudaGraphExecDestroy(c->gexec_host);
    if (c->gexec_hin) cudaGraphExecDestroy(c->gexec_hin);
    c->gexec = c->lgexec = c->gexec_host = c->gexec_hin = nullptr;
    c->gexec_host_ptr = nullptr;
    c->gexec_host_in = nullptr;
    c->out_ready = false;
}

long long count_sweep_launches(ccq_b200_ctx *c) {
    long long n = 0;
    for (size_t i = 0; i < c->cc_end; ++i) {
        const Op &o = c->plan.ops[i];
        if (o.frozen) continue;
        if (o.kind == OP_GETT && o.g.M && o.g.N && !o.skip) {
            if (o.zero_first || o.g.K == 0) ++n;
            if (o.g.K)
                n += use_split(c, o)
                         ? split_launch_count(o.g, c->nslices) : 1;
        } else if (o.kind == OP_ASM) {
            ++n;
        }
    }
    return n;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int ccq_b200_last_error(char *buf, int64_t len) {
    if (!buf || len <= 0) return CCQ_B200_EINVAL;
    snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
    return 0;
}

static int init_impl(const ccq_b200_dims *dims, const char *calc_type, const double *f_a, const double *f_b,
                     const double *v_aa, const double *v_ab, const double *v_bb, int64_t rhf, double shift,
                     int64_t diis_space, ccq_b200_ctx **out, bool rowmajor, int64_t act_occ_b,
                     int64_t act_unocc_a);

int ccq_b200_init(const ccq_b200_dims *dims, const char *calc_type, const double *f_a, const double *f_b,
                  const double *v_aa, const double *v_ab, const double *v_bb, int64_t rhf, double shift,
                  int64_t diis_space, ccq_b200_ctx **out) {
    return init_impl(dims, calc_type, f_a, f_b, v_aa, v_ab, v_bb, rhf, shift, diis_space, out, false, -1, -1);
}

int ccq_b200_init_rowmajor(const ccq_b200_dims *dims, const char *calc_type, const double *f_a, const double *f_b,
                           const double *v_aa, const double *v_ab, const double *v_bb, int64_t rhf, double shift,
                           int64_t diis_space, ccq_b200_ctx **out) {
    return init_impl(dims, calc_type, f_a, f_b, v_aa, v_ab, v_bb, rhf, shift, diis_space, out, true, -1, -1);
}

int ccq_b200_init_ex(const ccq_b200_dims *dims, const char *calc_type, const ccq_b200_init_opts *opts,
                     const double *f_a, const double *f_b, const double *v_aa, const double *v_ab,
                     const double *v_bb, int64_t rhf, double shift, int64_t diis_space, ccq_b200_ctx **out) {
    if (!opts) return fail(Error(CCQ_B200_EINVAL, "null options"));
    return init_impl(dims, calc_type, f_a, f_b, v_aa, v_ab, v_bb, rhf, shift, diis_space, out, opts->rowmajor != 0,
                     opts->act_occ_b, opts->act_unocc_a);
}

static int init_impl(const ccq_b200_dims *dims, const char *calc_type, const double *f_a, const double *f_b,
                     const double *v_aa, const double *v_ab, const double *v_bb, int64_t rhf, double shift,
                     int64_t diis_space, ccq_b200_ctx **out, bool rowmajor, int64_t act_occ_b,
                     int64_t act_unocc_a) {
    ccq_b200_ctx *c = nullptr;
    try {
        if (!dims || !calc_type || !f_a || !f_b || !v_aa || !v_ab || !v_bb || !out)
            throw Error(CCQ_B200_EINVAL, "null argument");
        *out = nullptr;
        if (diis_space < 1 || diis_space > 12) throw Error(CCQ_B200_EINVAL, "diis_space must be in 1..12");
        long long fr = dims->froz, oa = dims->occ_a - fr, ob = dims->occ_b - fr;
        long long va = dims->orbs - dims->occ_a, vb = dims->orbs - dims->occ_b, n = dims->orbs - fr;
        if (fr < 0 || oa < 1 || ob < 1 || va < 1 || vb < 1)
            throw Error(CCQ_B200_EINVAL, "invalid dimensions (need at least one occupied and virtual per spin)");
        std::string ct(calc_type);
        // CCSDt: the CCSDT plan restricted to ccq's active space (src/parser.f90:380-388)
        const bool active = ct == "CCSDt";
        if (active) {
            if (act_occ_b < fr || act_occ_b > dims->occ_b || act_unocc_a < dims->occ_a || act_unocc_a > dims->orbs)
                throw Error(CCQ_B200_EINVAL, "CCSDt: froz <= act_occ_b <= occ_b and occ_a <= act_unocc_a <= orbs");
            ct = "CCSDT";
        } else if (act_occ_b >= 0 || act_unocc_a >= 0) {
            throw Error(CCQ_B200_EINVAL, "an active space is given only with calc_type CCSDt");
        }
        if (ct != "CCSD" && ct != "CCSDT" && ct != "CCSDTQ" && ct != "CR-CC(2,3)")
            throw Error(CCQ_B200_EINVAL, "calc_type must be CCSD, CCSDT, CCSDt, CCSDTQ or CR-CC(2,3)");
        if (rhf && oa != ob) throw Error(CCQ_B200_EINVAL, "rhf requires occ_a == occ_b");
        const char *text = find_plan(ct, rhf != 0);
        if (!text) throw Error(CCQ_B200_EPLAN, "no plan for " + ct);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(CCQ_B200_ENODEV, "no CUDA device");
        c = new ccq_b200_ctx();
        // CCQ_B200_TRACE_INIT=1: stage times of context creation on stderr
        c->trace_init = getenv("CCQ_B200_TRACE_INIT") != nullptr;
        c->t_init0 = std::chrono::steady_clock::now();
        CK(cudaGetDevice(&c->device));
        keep_pool_memory(c->device);
        CK(gett_f64_prepare());
        CK(preload_kernels((int)diis_space));
        c->calc_type = ct;
        c->rhf = rhf != 0;
        c->shift = shift;
        c->ds = (int)diis_space;
        c->oa = oa;
        c->ob = ob;
        c->va = va;
        c->vb = vb;
        c->n = n;
        c->froz = fr;
        c->size = {{"oa", oa}, {"ob", ob}, {"va", va}, {"vb", vb}, {"n", n}, {"1", 1}, {"0", 0}, {"4", 4}};
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CK(cudaMallocHost(&c->hpin, 4 * sizeof(double)));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        CK(cudaEventCreate(&c->ev2));
        auto stamp = [&](const char *what) { trace_stamp(c, what); };
        stamp("stream/events");
        c->plan = parse_plan(text);
        if (active) {
            ActiveSpace as;
            as.occ_lo = act_occ_b - fr;
            as.vir_hi[0] = act_unocc_a - dims->occ_a;
            as.vir_hi[1] = act_unocc_a - dims->occ_b;
            restrict_to_active(c, as);
            c->act_occ_b = act_occ_b;
            c->act_unocc_a = act_unocc_a;
            t3act_geometry(fr, dims->occ_a, dims->occ_b, dims->orbs, act_occ_b, act_unocc_a, c->geom);
            c->cdiis = true;
        }
        stamp("parse");
        // host-side integral preparation
        long long orbs = dims->orbs;
        std::vector<double> FA(n * n), FB(n * n);
        // element (p, q) of f and (p, q, r, s) of v: column-major (Fortran) arrays, or row-major ones
        // (ccq_b200_init_rowmajor)
        auto F2 = [&](const double *x, long long p, long long q) {
            return rowmajor ? x[q + orbs * p] : x[p + orbs * q];
        };
        for (long long p = 0; p < n; ++p)
            for (long long q = 0; q < n; ++q) {
                FA[p * n + q] = F2(f_a, p + fr, q + fr);
                FB[p * n + q] = F2(f_b, p + fr, q + fr);
            }
        std::vector<double> HA(FA), HB(FB);
        auto V = [&](const double *x, long long p, long long q, long long r, long long s) {
            return rowmajor ? x[s + n * (r + n * (q + n * p))] : x[p + n * (q + n * (r + n * s))];
        };
        for (long long p = 0; p < n; ++p)
            for (long long q = 0; q < n; ++q) {
                double a = 0, b = 0;
                for (long long i = 0; i < oa; ++i) a += V(v_aa, p, i, q, i);
                for (long long i = 0; i < ob; ++i) a += V(v_ab, p, i, q, i);
                for (long long i = 0; i < ob; ++i) b += V(v_bb, p, i, q, i);
                for (long long i = 0; i < oa; ++i) b += V(v_ab, i, p, i, q);
                HA[p * n + q] -= a;
                HB[p * n + q] -= b;
            }
        std::vector<double> da(n), db(n);
        for (long long p = 0; p < n; ++p) {
            da[p] = FA[p * n + p];
            db[p] = FB[p * n + p];
        }
        c->fdiag_a = (double *)c->dalloc(sizeof(double) * n);
        c->fdiag_b = (double *)c->dalloc(sizeof(double) * n);
        CK(cudaMemcpy(c->fdiag_a, da.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->fdiag_b, db.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        stamp("host prep");
        instantiate(c);
        CK(cudaStreamSynchronize(c->stream));
        stamp("instantiate");
        auto up = [&](const char *name, const std::vector<double> &h) {
            DevBuf &d = c->bufs.at(name);
            if ((size_t)d.numel != h.size()) throw Error(CCQ_B200_EPLAN, std::string("size of ") + name);
            CK(cudaMemcpy(d.ptr, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
        };
        up("FA0", FA);
        up("FB0", FB);
        up("HA0", HA);
        up("HB0", HB);
        // two-electron blocks: the column-major arrays go up as they are (staged in the
        // dressed buffer of the same size, which the first dressing overwrites) and
        // are reordered to [p][q][r][s] on the device
        // (row-major arrays are already [p][q][r][s] and go straight into place)
        auto up4 = [&](const char *name, const char *stage, const double *f) {
            DevBuf &d = c->bufs.at(name);
            DevBuf &st = c->bufs.at(stage);
            const long long ne = n * n * n * n;
            if (d.numel != ne || st.numel != ne) throw Error(CCQ_B200_EPLAN, std::string("size of ") + name);
            if (rowmajor) {
                CK(cudaMemcpyAsync(d.ptr, f, sizeof(double) * ne, cudaMemcpyHostToDevice, c->stream));
                return;
            }
            CK(cudaMemcpyAsync(st.ptr, f, sizeof(double) * ne, cudaMemcpyHostToDevice, c->stream));
            launch_f2c4(st.ptr, d.ptr, n, c->stream);
        };
        up4("VAA0", "VAA", v_aa);
        up4("VAB0", "VAB", v_ab);
        up4("VBB0", "VBB", v_bb);
        // this context's stream only: contexts created by other host threads keep running
        CK(cudaStreamSynchronize(c->stream));
        if (active) apply_active_masks(c, act_occ_b, act_unocc_a);
        stamp("upload");
        *out = c;
        return 0;
    } catch (const Error &e) {
        delete c;
        return fail(e);
    } catch (const std::exception &e) {
        delete c;
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_sizes(const ccq_b200_ctx *c, int64_t *t_size, int64_t *vec_size) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    if (t_size) *t_size = c->t_size;
    if (vec_size) *vec_size = c->vec_size;
    return 0;
}

int ccq_b200_set_t(ccq_b200_ctx *c, const double *t, int64_t n) {
    try {
        if (!c || !t || n != c->t_size) throw Error(CCQ_B200_EINVAL, "set_t: size must equal t_size");
        CK(cudaMemcpyAsync(c->tvec, t, sizeof(double) * c->t_dev, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_get_t(const ccq_b200_ctx *c, double *t, int64_t n) {
    try {
        if (!c || !t || n != c->t_size) throw Error(CCQ_B200_EINVAL, "get_t: size must equal t_size");
        CK(cudaMemcpyAsync(t, c->tvec, sizeof(double) * c->t_dev, cudaMemcpyDeviceToHost, c->stream));
        if (c->t_dev < n) std::fill(t + c->t_dev, t + n, 0.0);
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_block(ccq_b200_ctx *c, const char *name, double *host, int64_t n, int64_t to_device) {
    try {
        if (!c || !name || !host) throw Error(CCQ_B200_EINVAL, "block: null argument");
        std::string nm(name);
        if (nm.size() != 3 || nm[0] != 'T') throw Error(CCQ_B200_EINVAL, "block: amplitude block name expected");
        auto it = c->bufs.find(nm);
        if (it == c->bufs.end()) throw Error(CCQ_B200_EINVAL, "block: unknown block " + nm);
        if (n != it->second.numel) throw Error(CCQ_B200_EINVAL, "block: size mismatch");
        if (!it->second.ptr) throw Error(CCQ_B200_EINVAL, "block: " + nm + " is not resident for " + c->calc_type);
        CK(cudaMemcpyAsync(to_device ? (void *)it->second.ptr : (void *)host,
                           to_device ? (const void *)host : (const void *)it->second.ptr, sizeof(double) * n,
                           to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

// ---- checkpoint / restart -------------------------------------------------------
// File: "CCQB200C" | int64 version, froz, oa, ob, va, vb, rhf, ds, t_dev, vec_size,
// nblocks, with_ring, iteration | double state[8] | char calc_type[32] | t_vec
// (t_dev doubles) | per amplitude block outside t_vec: char name[8], int64 numel,
// doubles | ring ((ds+1) vec_size doubles) when with_ring | "CKPTEND!" int64 bytes.
// Copies go through one pinned staging buffer in 64 MiB pieces.

namespace {

constexpr char kCkptMagic[8] = {'C', 'C', 'Q', 'B', '2', '0', '0', 'C'};
constexpr char kCkptEnd[8] = {'C', 'K', 'P', 'T', 'E', 'N', 'D', '!'};
constexpr long long kCkptVersion = 1;
constexpr size_t kStage = 64ull << 20;

struct CkptHead {
    long long version, froz, oa, ob, va, vb, rhf, ds, t_dev, vec_size, nblocks, with_ring, iteration;
    double state[8];
    char calc_type[32];
};

std::vector<std::pair<std::string, const DevBuf *>> outside_blocks(const ccq_b200_ctx *c) {
    std::vector<std::pair<std::string, const DevBuf *>> out;
    for (auto &b : c->plan.bufs)
        if (b.kind == "amp") {
            const DevBuf &d = c->bufs.at(b.name);
            if (d.ptr && (d.ptr < c->tvec || d.ptr >= c->tvec + c->t_dev)) out.push_back({b.name, &d});
        }
    return out;
}

struct Pinned {
    void *p = nullptr;
    Pinned() { CK(cudaMallocHost(&p, kStage)); }
    ~Pinned() { cudaFreeHost(p); }
};

void write_all(FILE *f, const void *p, size_t n, long long &total) {
    if (n && fwrite(p, 1, n, f) != n) throw Error(CCQ_B200_EINVAL, "checkpoint: write failed");
    total += (long long)n;
}

void read_all(FILE *f, void *p, size_t n) {
    if (n && fread(p, 1, n, f) != n) throw Error(CCQ_B200_EINVAL, "checkpoint: file truncated");
}

void dev_to_file(ccq_b200_ctx *c, FILE *f, const double *src, long long n, Pinned &st, long long &total) {
    const long long per = (long long)(kStage / sizeof(double));
    for (long long o = 0; o < n; o += per) {
        const long long k = std::min(per, n - o);
        CK(cudaMemcpyAsync(st.p, src + o, sizeof(double) * k, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        write_all(f, st.p, sizeof(double) * k, total);
    }
}

void file_to_dev(ccq_b200_ctx *c, FILE *f, double *dst, long long n, Pinned &st) {
    const long long per = (long long)(kStage / sizeof(double));
    for (long long o = 0; o < n; o += per) {
        const long long k = std::min(per, n - o);
        read_all(f, st.p, sizeof(double) * k);
        CK(cudaMemcpyAsync(dst + o, st.p, sizeof(double) * k, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
}

CkptHead read_head(FILE *f) {
    char magic[8];
    read_all(f, magic, 8);
    if (memcmp(magic, kCkptMagic, 8) != 0) throw Error(CCQ_B200_EINVAL, "checkpoint: not a checkpoint file");
    CkptHead h;
    read_all(f, &h, sizeof(h));
    if (h.version != kCkptVersion) throw Error(CCQ_B200_EINVAL, "checkpoint: unknown version");
    h.calc_type[31] = '\0';
    return h;
}

struct FileCloser {
    FILE *f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};

}  // namespace

int ccq_b200_checkpoint_save(ccq_b200_ctx *c, const char *path, int64_t with_ring, int64_t iteration,
                             const double *state) {
    try {
        if (!c || !path) throw Error(CCQ_B200_EINVAL, "checkpoint_save: null argument");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "checkpoint_save: an iteration is pending");
        CK(cudaSetDevice(c->device));
        CK(cudaStreamSynchronize(c->stream));
        auto blocks = outside_blocks(c);
        CkptHead h{};
        h.version = kCkptVersion;
        h.froz = c->froz;
        h.oa = c->oa;
        h.ob = c->ob;
        h.va = c->va;
        h.vb = c->vb;
        h.rhf = c->rhf;
        h.ds = c->ds;
        h.t_dev = c->t_dev;
        h.vec_size = c->vec_size;
        h.nblocks = (long long)blocks.size();
        h.with_ring = with_ring ? 1 : 0;
        h.iteration = iteration;
        for (int k = 0; k < 8; ++k) h.state[k] = state ? state[k] : 0.0;
        snprintf(h.calc_type, sizeof(h.calc_type), "%s", c->calc_type.c_str());
        // write next to the target and rename at the end: a crash never leaves a torn checkpoint
        const std::string tmp = std::string(path) + ".part";
        FileCloser fc{fopen(tmp.c_str(), "wb")};
        if (!fc.f) throw Error(CCQ_B200_EINVAL, std::string("checkpoint_save: cannot open ") + tmp);
        Pinned st;
        long long total = 0;
        write_all(fc.f, kCkptMagic, 8, total);
        write_all(fc.f, &h, sizeof(h), total);
        dev_to_file(c, fc.f, c->tvec, c->t_dev, st, total);
        for (auto &b : blocks) {
            char nm[8] = {0};
            snprintf(nm, sizeof(nm), "%s", b.first.c_str());
            long long n = b.second->numel;
            write_all(fc.f, nm, 8, total);
            write_all(fc.f, &n, sizeof(n), total);
            dev_to_file(c, fc.f, b.second->ptr, n, st, total);
        }
        if (with_ring) dev_to_file(c, fc.f, c->ring, (long long)(c->ds + 1) * c->vec_size, st, total);
        write_all(fc.f, kCkptEnd, 8, total);
        total += (long long)sizeof(total);
        write_all(fc.f, &total, sizeof(total), total);
        if (fclose(fc.f) != 0) {
            fc.f = nullptr;
            throw Error(CCQ_B200_EINVAL, "checkpoint_save: close failed");
        }
        fc.f = nullptr;
        if (rename(tmp.c_str(), path) != 0) throw Error(CCQ_B200_EINVAL, "checkpoint_save: rename failed");
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_checkpoint_info(const char *path, int64_t *dims, int64_t *iteration, int64_t *with_ring,
                             double *state, char *calc_type, int64_t len) {
    try {
        if (!path) throw Error(CCQ_B200_EINVAL, "checkpoint_info: null path");
        FileCloser fc{fopen(path, "rb")};
        if (!fc.f) throw Error(CCQ_B200_EINVAL, std::string("Restart file not found: ") + path);
        CkptHead h = read_head(fc.f);
        if (dims) {
            const long long d[9] = {h.froz, h.oa, h.ob, h.va, h.vb, h.rhf, h.ds, h.t_dev, h.vec_size};
            for (int k = 0; k < 9; ++k) dims[k] = d[k];
        }
        if (iteration) *iteration = h.iteration;
        if (with_ring) *with_ring = h.with_ring;
        if (state)
            for (int k = 0; k < 8; ++k) state[k] = h.state[k];
        if (calc_type && len > 0) snprintf(calc_type, (size_t)len, "%s", h.calc_type);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_checkpoint_load(ccq_b200_ctx *c, const char *path, int64_t *iteration, double *state,
                             int64_t *with_ring) {
    try {
        if (!c || !path) throw Error(CCQ_B200_EINVAL, "checkpoint_load: null argument");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "checkpoint_load: an iteration is pending");
        CK(cudaSetDevice(c->device));
        FileCloser fc{fopen(path, "rb")};
        if (!fc.f) throw Error(CCQ_B200_EINVAL, std::string("Restart file not found: ") + path);
        CkptHead h = read_head(fc.f);
        auto blocks = outside_blocks(c);
        if (std::string(h.calc_type) != c->calc_type || h.froz != c->froz || h.oa != c->oa || h.ob != c->ob ||
            h.va != c->va || h.vb != c->vb || h.rhf != c->rhf || h.t_dev != c->t_dev || h.vec_size != c->vec_size ||
            h.nblocks != (long long)blocks.size())
            throw Error(CCQ_B200_EINVAL, "checkpoint_load: the file belongs to another system or method");
        if (h.with_ring && h.ds != c->ds) throw Error(CCQ_B200_EINVAL, "checkpoint_load: diis_space differs");
        // the size trailer first: a truncated file is refused before any device state changes
        long long expect = 8 + (long long)sizeof(CkptHead) + 8 * h.t_dev + 16;   // magic, head, t_vec, trailer
        for (auto &b : blocks) expect += 16 + 8 * b.second->numel;
        if (h.with_ring) expect += 8 * (h.ds + 1) * h.vec_size;
        if (fseek(fc.f, 0, SEEK_END) != 0 || ftell(fc.f) != expect)
            throw Error(CCQ_B200_EINVAL, "checkpoint_load: file size does not match its header");
        if (fseek(fc.f, expect - 16, SEEK_SET) != 0) throw Error(CCQ_B200_EINVAL, "checkpoint_load: seek failed");
        char endm[8];
        long long total = 0;
        read_all(fc.f, endm, 8);
        read_all(fc.f, &total, 8);
        if (memcmp(endm, kCkptEnd, 8) != 0 || total != expect) throw Error(CCQ_B200_EINVAL, "checkpoint_load: bad trailer");
        if (fseek(fc.f, 8 + (long)sizeof(CkptHead), SEEK_SET) != 0)
            throw Error(CCQ_B200_EINVAL, "checkpoint_load: seek failed");
        Pinned st;
        file_to_dev(c, fc.f, c->tvec, c->t_dev, st);
        for (auto &b : blocks) {
            char nm[8];
            long long n = 0;
            read_all(fc.f, nm, 8);
            read_all(fc.f, &n, 8);
            nm[7] = '\0';
            if (b.first != nm || n != b.second->numel) throw Error(CCQ_B200_EINVAL, "checkpoint_load: block mismatch");
            file_to_dev(c, fc.f, b.second->ptr, n, st);
        }
        if (h.with_ring) file_to_dev(c, fc.f, c->ring, (long long)(h.ds + 1) * h.vec_size, st);
        if (iteration) *iteration = h.iteration;
        if (with_ring) *with_ring = h.with_ring;
        if (state)
            for (int k = 0; k < 8; ++k) state[k] = h.state[k];
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_update(ccq_b200_ctx *c) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        CK(cudaSetDevice(c->device));
        run_ops(c, 0, c->energy_op);
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_energy(ccq_b200_ctx *c, double *e) {
    try {
        if (!c || !e) throw Error(CCQ_B200_EINVAL, "null argument");
        CK(cudaSetDevice(c->device));
        run_ops(c, c->energy_op, c->cc_end);
        CK(cudaMemcpyAsync(e, c->bufs.at("E").ptr, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e2) {
        return fail(e2);
    } catch (const std::exception &e2) {
        return fail(Error(CCQ_B200_EINVAL, e2.what()));
    }
}

// One jacobi_iter step split in two: the launch enqueues the sweep, the ring
// write, the residuum and (on schedule) DIIS, and copies the results to pinned
// host slots; the finish waits for them.  Many contexts on their own streams
// can be launched before any is waited for.
// After the sweep of iteration iter: the DIIS ring write, residuum, the extrapolation every
// diis_space + 1 iterations, and the energy / residuum / DIIS status copied to the pinned slots.
static void post_sweep(ccq_b200_ctx *c, int64_t iter, cudaStream_t st) {
    const int ds = c->ds;
    const long long vs = c->vec_size;
    auto slot = [&](long long it) {
        long long q = it % (ds + 1);
        return q == 0 ? ds + 1 : q;
    };
    double *cur = c->ring + (slot(iter) - 1) * vs;
    const bool packed = c->cdiis && vs > c->vec_t12;   // CCSDt's compressed DIIS vector (not while T3 is held)
    if (packed) {
        CK(cudaMemcpyAsync(cur, c->tvec, sizeof(double) * c->vec_t12, cudaMemcpyDeviceToDevice, st));
        launch_t3act_gather(c->geom, c->tvec, cur + c->vec_t12, st);
        c->launches += 1;
    } else {
        CK(cudaMemcpyAsync(cur, c->tvec, sizeof(double) * vs, cudaMemcpyDeviceToDevice, st));
    }
    const double *prev = iter == 1 ? nullptr : c->ring + (slot(iter - 1) - 1) * vs;
    launch_sqdiff(prev, cur, vs, c->scratch, st);
    c->launches += 1;
    const int diis = (iter % (ds + 1)) == 0;
    if (diis) {
        launch_diis_gram(c->ring, vs, ds, vs, c->scratch + 8, st);
        launch_diis_solve(c->scratch + 8, ds, c->scratch + 8 + 169, c->dinfo, st);
        if (packed) {
            launch_diis_extrap(c->ring, vs, ds, vs, c->scratch + 8 + 169, c->cvec, st);
            CK(cudaMemcpyAsync(c->tvec, c->cvec, sizeof(double) * c->vec_t12, cudaMemcpyDeviceToDevice, st));
            launch_t3act_scatter(c->geom, c->cvec + c->vec_t12, c->tvec, st);
            c->launches += 2;
        } else {
            launch_diis_extrap(c->ring, vs, ds, vs, c->scratch + 8 + 169, c->tvec, st);
        }
        c->launches += 3;
        // the extrapolation rewrote T1 .. T3: the host copy is taken (again)
        if (double *dst = c->host_out ? c->host_out : c->diis_out)
            CK(cudaMemcpyAsync(dst, c->tvec, sizeof(double) * c->t_dev, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaEventRecord(c->ev2, st));
    CK(cudaMemcpyAsync(c->hpin, c->bufs.at("E").ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->hpin + 1, c->scratch, sizeof(double), cudaMemcpyDeviceToHost, st));
    c->hpin[2] = 0.0;
    if (diis) CK(cudaMemcpyAsync(c->hpin + 2, c->dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
}

static void iterate_launch(ccq_b200_ctx *c, int64_t iter) {
    CK(cudaSetDevice(c->device));
    c->launches = 0;
    CK(cudaEventRecord(c->ev0, c->stream));
    sweep(c);
    CK(cudaEventRecord(c->ev1, c->stream));
    c->launches = count_sweep_launches(c);
    post_sweep(c, iter, c->stream);
    c->async_iter = iter;
}

static void iterate_finish(ccq_b200_ctx *c, double *e_cor, double *res, int64_t *did_diis) {
    const int64_t iter = c->async_iter;
    if (iter < 1) throw Error(CCQ_B200_EINVAL, "iterate_wait: no iteration was launched");
    c->async_iter = 0;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->sweep_ms = ms;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev2));
    c->iter_ms = ms;
    const int diis = (iter % (c->ds + 1)) == 0;
    int info = 0;
    memcpy(&info, c->hpin + 2, sizeof(int));
    if (diis && info != 0) throw Error(CCQ_B200_ESINGULAR, "calc_diis: DIIS error in DGESV");
    if (c->precision == CCQ_B200_PREC_SPLIT) {
        bool expired = split_error(c->split) != 0;
        for (auto &w : c->split_pool) expired = expired || split_error(w) != 0;
        if (expired) throw Error(CCQ_B200_ECUDA, "split GETT pipeline wait expired");
    }
    if (e_cor) *e_cor = c->hpin[0];
    if (res) *res = std::sqrt(std::sqrt(c->hpin[1]));
    if (did_diis) *did_diis = diis;
}

int ccq_b200_iterate_host(ccq_b200_ctx *c, int64_t iter, const double *t_in, double *t_out, int64_t n,
                          double *e_cor, double *res, int64_t *did_diis) {
    try {
        if (!c || iter < 1 || !t_in || !t_out) throw Error(CCQ_B200_EINVAL, "iterate_host: bad argument");
        if (n != c->t_size) throw Error(CCQ_B200_EINVAL, "iterate_host: size must equal t_size");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "iterate_host: an iteration is pending");
        CK(cudaSetDevice(c->device));
        auto host_ptr = [](const void *p, const void **dev) {
            cudaPointerAttributes pa{};
            const bool r = cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
            cudaGetLastError();
            if (dev) *dev = r ? pa.devicePointer : nullptr;
            return r;
        };
        const void *in_dev = nullptr;
        const bool pinned = host_ptr(t_out, nullptr);
        // pinned input and a dependency-graph sweep: the input blocks are copied inside the graph, each
        // operation waiting only for the blocks it reads; else the whole t_vec is copied first
        const bool in_graph = pinned && host_ptr(t_in, &in_dev) && c->use_graph == 1 && !c->profile;
        if (!in_graph)
            CK(cudaMemcpyAsync(c->tvec, t_in, sizeof(double) * c->t_dev, cudaMemcpyHostToDevice, c->stream));
        if (!pinned) {
            // pageable memory cannot take asynchronous copies inside a captured sweep: copy after it
            iterate_launch(c, iter);
            iterate_finish(c, e_cor, res, did_diis);
            CK(cudaMemcpy(t_out, c->tvec, sizeof(double) * c->t_dev, cudaMemcpyDeviceToHost));
            c->io_h2d = c->io_d2h = (long long)sizeof(double) * c->t_dev;
            if (c->t_dev < n) std::fill(t_out + c->t_dev, t_out + n, 0.0);
            return 0;
        }
        const double *in_ptr = in_graph ? t_in : nullptr;
        if (c->gexec_host_ptr != t_out || c->gexec_host_in != in_ptr) {
            // the copy sources and targets are part of the captured graph
            if (c->gexec_host) cudaGraphExecDestroy(c->gexec_host);
            if (c->gexec_hin) cudaGraphExecDestroy(c->gexec_hin);
            c->gexec_host = c->gexec_hin = nullptr;
            c->gexec_host_ptr = t_out;
            c->gexec_host_in = in_ptr;
        }
        // a DIIS iteration copies nothing out during the sweep: the extrapolation after it rewrites every
        // block, and the extrapolated vector is copied out whole
        const bool diis_it = (iter % (c->ds + 1)) == 0;
        c->host_out = diis_it ? nullptr : t_out;
        c->diis_out = diis_it ? t_out : nullptr;
        c->host_in = in_ptr;
        c->host_in_dev = in_graph ? (const double *)in_dev : nullptr;
        try {
            iterate_launch(c, iter);
        } catch (...) {
            c->host_out = c->diis_out = nullptr;
            c->host_in = nullptr;
            throw;
        }
        c->host_out = c->diis_out = nullptr;
        c->host_in = nullptr;
        iterate_finish(c, e_cor, res, did_diis);
        // bytes across the host link: the input (canonical T3 elements when read in the graph) and the
        // whole vector out (block by block during the sweep, or after the extrapolation of a DIIS step)
        c->io_h2d = in_graph ? c->cin_h2d : (long long)sizeof(double) * c->t_dev;
        c->io_d2h = (long long)sizeof(double) * c->t_dev;
        if (c->t_dev < n) std::fill(t_out + c->t_dev, t_out + n, 0.0);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_io_bytes(ccq_b200_ctx *c, int64_t *h2d, int64_t *d2h) {
    if (!c || !h2d || !d2h) return fail(Error(CCQ_B200_EINVAL, "null argument"));
    *h2d = c->io_h2d;
    *d2h = c->io_d2h;
    return 0;
}

int ccq_b200_iterate(ccq_b200_ctx *c, int64_t iter, double *e_cor, double *res, int64_t *did_diis) {
    try {
        if (!c || iter < 1) throw Error(CCQ_B200_EINVAL, "iterate: bad argument");
        iterate_launch(c, iter);
        iterate_finish(c, e_cor, res, did_diis);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_iterate_async(ccq_b200_ctx *c, int64_t iter) {
    try {
        if (!c || iter < 1) throw Error(CCQ_B200_EINVAL, "iterate_async: bad argument");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "iterate_async: the previous iteration was not waited for");
        iterate_launch(c, iter);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_iterate_wait(ccq_b200_ctx *c, double *e_cor, double *res, int64_t *did_diis) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        iterate_finish(c, e_cor, res, did_diis);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

// ---- CR-CC(2,3): left CCSD and the triples corrections ----------------------

static void need_crcc(const ccq_b200_ctx *c) {
    if (!c->has_crcc) throw Error(CCQ_B200_EINVAL, "context was not created with calc_type CR-CC(2,3)");
}

int ccq_b200_lambda_init(ccq_b200_ctx *c, double e_cor) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        need_crcc(c);
        CK(cudaSetDevice(c->device));
        CK(cudaMemcpy(c->bufs.at("ECOR").ptr, &e_cor, sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemsetAsync(c->lvec, 0, sizeof(double) * c->l_size, c->stream));
        CK(cudaMemsetAsync(c->lring, 0, sizeof(double) * (size_t)(c->ds + 1) * c->l_size, c->stream));
        run_ops(c, c->cc_end, c->lambda_op);
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_lambda_iterate(ccq_b200_ctx *c, int64_t iter, double *e_left, double *res, int64_t *did_diis) {
    try {
        if (!c || iter < 1) throw Error(CCQ_B200_EINVAL, "lambda_iterate: bad argument");
        need_crcc(c);
        CK(cudaSetDevice(c->device));
        CK(cudaEventRecord(c->ev0, c->stream));
        if (c->use_graph && !c->profile) {
            if (!c->lgexec) {
                cudaGraph_t g;
                CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    if (c->use_graph == 2)
                        run_ops(c, c->lambda_op, c->triples_op);
                    else
                        run_ops_dag(c, c->lambda_op, c->triples_op);
                } catch (...) {
                    cudaStreamEndCapture(c->stream, &g);
                    throw;
                }
                CK(cudaStreamEndCapture(c->stream, &g));
                CK(cudaGraphInstantiate(&c->lgexec, g, 0));
                CK(cudaGraphDestroy(g));
            }
            CK(cudaGraphLaunch(c->lgexec, c->stream));
        } else {
            run_ops(c, c->lambda_op, c->triples_op);
        }
        CK(cudaEventRecord(c->ev1, c->stream));
        // ring, residuum and DIIS on the lambda vector (jacobi_iter on l_vec, src/solve_cc.f90:175-269)
        const int ds = c->ds;
        const long long vs = c->l_size;
        auto slot = [&](long long it) {
            long long q = it % (ds + 1);
            return q == 0 ? ds + 1 : q;
        };
        double *cur = c->lring + (slot(iter) - 1) * vs;
        CK(cudaMemcpyAsync(cur, c->lvec, sizeof(double) * vs, cudaMemcpyDeviceToDevice, c->stream));
        const double *prev = iter == 1 ? nullptr : c->lring + (slot(iter - 1) - 1) * vs;
        launch_sqdiff(prev, cur, vs, c->scratch, c->stream);
        const int diis = (iter % (ds + 1)) == 0;
        if (diis) {
            launch_diis_gram(c->lring, vs, ds, vs, c->scratch + 8, c->stream);
            launch_diis_solve(c->scratch + 8, ds, c->scratch + 8 + 169, c->dinfo, c->stream);
            launch_diis_extrap(c->lring, vs, ds, vs, c->scratch + 8 + 169, c->lvec, c->stream);
        }
        CK(cudaEventRecord(c->ev2, c->stream));
        double hs[2];
        int info = 0;
        CK(cudaMemcpyAsync(&hs[0], c->bufs.at("EL").ptr, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(&hs[1], c->scratch, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (diis) CK(cudaMemcpyAsync(&info, c->dinfo, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->sweep_ms = ms;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev2));
        c->iter_ms = ms;
        if (diis && info != 0) throw Error(CCQ_B200_ESINGULAR, "calc_diis: DIIS error in DGESV");
        if (e_left) *e_left = hs[0];
        if (res) *res = std::sqrt(std::sqrt(hs[1]));
        if (did_diis) *did_diis = diis;
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_crcc23(ccq_b200_ctx *c, double *e) {
    try {
        if (!c || !e) throw Error(CCQ_B200_EINVAL, "null argument");
        need_crcc(c);
        CK(cudaSetDevice(c->device));
        CK(cudaEventRecord(c->ev0, c->stream));
        CK(cudaMemsetAsync(c->bufs.at("E23").ptr, 0, 4 * sizeof(double), c->stream));
        run_ops(c, c->triples_op, c->plan.ops.size());
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaMemcpyAsync(e, c->bufs.at("E23").ptr, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->sweep_ms = ms;
        return 0;
    } catch (const Error &e2) {
        return fail(e2);
    } catch (const std::exception &e2) {
        return fail(Error(CCQ_B200_EINVAL, e2.what()));
    }
}

int ccq_b200_get_l(ccq_b200_ctx *c, double *l_vec, int64_t n) {
    try {
        if (!c || !l_vec) throw Error(CCQ_B200_EINVAL, "null argument");
        need_crcc(c);
        if (n != c->l_size) throw Error(CCQ_B200_EINVAL, "l_vec length must be the T1 + T2 size");
        CK(cudaSetDevice(c->device));
        CK(cudaMemcpyAsync(l_vec, c->lvec, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

// ---- autotuner ------------------------------------------------------------------
// One eager sweep in which every contraction is timed in each candidate
// configuration (64 x 64 / skinny DMMA tiles or the small-K FMA kernel,
// split-K chunk, and in split mode int8 slices or DMMA), writing into scratch so that the sweep's own data stay intact; the op
// then runs once for real in the fastest configuration.  The amplitudes are
// restored afterwards, so tuning does not count as an iteration.

static bool split_capable(const GettArgs &g) {
    long long tiles = ((g.M + 127LL) / 128) * ((g.N + 127LL) / 128);
    return g.M >= 64 && g.N >= 64 && g.K >= 256 && tiles >= 64;
}

struct TuneCfg {
    int tile, kchunk, split;
};

static float time_cfg(ccq_b200_ctx *c, Op &o, const TuneCfg &t, double *scratch, int reps) {
    GettArgs g = o.g;
    g.C = scratch;
    g.tile = t.tile;
    g.kchunk = t.kchunk;
    const bool zf = !g.segs && g.beta == 0 && (g.K + t.kchunk - 1) / t.kchunk > 1;
    auto run = [&]() {
        if (t.split) {
            split_gett(c->split, g, o.akm, o.bkm, c->nslices, c->stream, t.split == 2);
        } else {
            if (zf) launch_zero_view(g.C, g.offC_m, g.offC_n, g.M, g.N, c->stream);
            launch_gett_f64(g, o.akm, o.bkm, c->stream);
        }
    };
    run();
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < reps; ++r) run();
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    return ms / reps;
}

int ccq_b200_autotune(ccq_b200_ctx *c, int64_t reps, double *ms_default, double *ms_tuned) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "autotune: an iteration is pending");
        if (reps < 1) reps = 3;
        CK(cudaSetDevice(c->device));
        CK(cudaStreamSynchronize(c->stream));
        // amplitude state to restore: t_vec and the amplitude blocks outside it
        std::vector<std::pair<double *, long long>> keep;
        keep.push_back({c->tvec, c->t_dev});
        for (auto &b : c->plan.bufs)
            if (b.kind == "amp") {
                const DevBuf &d = c->bufs.at(b.name);
                if (d.ptr && (d.ptr < c->tvec || d.ptr >= c->tvec + c->t_dev)) keep.push_back({d.ptr, d.numel});
            }
        long long nkeep = 0, nscr = 1;
        for (auto &k : keep) nkeep += k.second;
        for (size_t i = 0; i < c->cc_end; ++i) {
            const Op &o = c->plan.ops[i];
            if (o.kind == OP_GETT) nscr = std::max(nscr, c->bufs.at(o.c.buf).numel);
        }
        double *backup = nullptr, *scratch = nullptr;
        CK(cudaMalloc(&backup, sizeof(double) * std::max(nkeep, 1LL)));
        CK(cudaMalloc(&scratch, sizeof(double) * nscr));
        auto release = [&]() {
            cudaFree(backup);
            cudaFree(scratch);
        };
        double t0 = 0.0, t1 = 0.0;
        // every candidate's time, one line each, when CCQ_B200_TUNE_DUMP names a file
        const char *dpath = getenv("CCQ_B200_TUNE_DUMP");
        FILE *dump = dpath ? fopen(dpath, "a") : nullptr;
        struct DumpCloser {
            FILE *&f;
            ~DumpCloser() {
                if (f) fclose(f);
            }
        } dump_closer{dump};
        try {
            long long off = 0;
            for (auto &k : keep) {
                CK(cudaMemcpyAsync(backup + off, k.first, sizeof(double) * k.second, cudaMemcpyDeviceToDevice,
                                   c->stream));
                off += k.second;
            }
            for (size_t i = 0; i < c->cc_end; ++i) {
                Op &o = c->plan.ops[i];
                if (o.kind != OP_GETT || o.skip || o.frozen || o.g.M == 0 || o.g.N == 0 || o.g.K == 0) {
                    run_op(c, o, c->stream);
                    continue;
                }
                const long long M = o.g.M, N = o.g.N, K = o.g.K;
                std::vector<TuneCfg> cand;
                const TuneCfg cur{o.g.tile, o.g.kchunk, use_split(c, o) ? (split_persistent(o) ? 2 : 1) : 0};
                cand.push_back(cur);
                std::vector<int> tiles = {1};
                if (std::min(M, N) <= 32) {
                    tiles.push_back(2);
                    tiles.push_back(5);
                }
                for (int tl : tiles) {
                    std::vector<long long> ch;
                    if (o.g.segs) {
                        ch.push_back(o.g.kchunk);
                    } else {
                        const long long c0 = o.g.kchunk;
                        for (long long x : {c0, K, 2 * c0, c0 / 2, c0 / 4})
                            ch.push_back(std::max(16LL, std::min(K + 15 - (K + 15) % 16, (x + 15) / 16 * 16)));
                    }
                    for (long long x : ch) {
                        TuneCfg t{tl, (int)x, 0};
                        bool dup = false;
                        for (auto &q : cand) dup = dup || (q.tile == t.tile && q.kchunk == t.kchunk && q.split == 0);
                        if (!dup) cand.push_back(t);
                    }
                }
                // small-K FMA kernel and register-direct DMMA kernel: whole K per launch
                if (K <= 128) cand.push_back(TuneCfg{3, o.g.segs ? o.g.kchunk : (int)((K + 15) / 16 * 16), 0});
                if (K <= 64) cand.push_back(TuneCfg{6, o.g.segs ? o.g.kchunk : (int)((K + 15) / 16 * 16), 0});
                // split precision: DMMA, the per-tile and the persistent int8 kernel
                if (c->precision == CCQ_B200_PREC_SPLIT && o.split && (split_capable(o.g) || cur.split))
                    for (int v : {0, 1, 2})
                        if (v != cur.split) cand.push_back(TuneCfg{0, o.g.kchunk, v});
                float best = 1e30f;
                TuneCfg pick = cur;
                for (size_t q = 0; q < cand.size(); ++q) {
                    const float ms = time_cfg(c, o, cand[q], scratch, (int)reps);
                    if (dump)
                        fprintf(dump, "%zu %s %lld %lld %lld tile=%d kchunk=%d split=%d %.6f\n", i, o.tag.c_str(), M, N,
                                K, cand[q].tile, cand[q].kchunk, cand[q].split, ms);
                    if (q == 0) t0 += ms;
                    if (ms < best) {
                        best = ms;
                        pick = cand[q];
                    }
                }
                t1 += best;
                o.g.tile = pick.tile;
                o.g.kchunk = pick.kchunk;
                o.zero_first = !o.g.segs && o.beta == 0 && (o.g.K + pick.kchunk - 1) / pick.kchunk > 1;
                if (c->precision == CCQ_B200_PREC_SPLIT && o.split) o.split_choice = pick.split;
                run_op(c, o, c->stream);
            }
            off = 0;
            for (auto &k : keep) {
                CK(cudaMemcpyAsync(k.first, backup + off, sizeof(double) * k.second, cudaMemcpyDeviceToDevice,
                                   c->stream));
                off += k.second;
            }
            CK(cudaStreamSynchronize(c->stream));
        } catch (...) {
            cudaStreamSynchronize(c->stream);
            release();
            throw;
        }
        release();
        drop_graphs(c);
        if (ms_default) *ms_default = t0;
        if (ms_tuned) *ms_tuned = t1;
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_set_external(ccq_b200_ctx *c, int64_t on) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        if (c->calc_type != "CCSDT" && c->calc_type != "CCSDTQ")
            throw Error(CCQ_B200_EINVAL, "set_external: a CCSDT or CCSDTQ context is required");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "set_external: an iteration is pending");
        // every operation of the T3 / T4 phases (their contractions, gathers and rhf copies)
        std::string phase;
        for (auto &o : c->plan.ops) {
            if (o.kind == OP_PHASE) {
                phase = o.arg0;
                continue;
            }
            if (&o - &c->plan.ops[0] >= (long)c->cc_end) break;
            o.frozen = on && phase.size() >= 2 && phase[0] == 'T' && (phase[1] == '3' || phase[1] == '4');
        }
        // DIIS over T1 + T2 (src/solve_cc.f90:66-72 with run%ext_cor)
        c->vec_size = on ? c->vec_t12 : c->vec_full;
        drop_graphs(c);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_set_active(ccq_b200_ctx *c, int64_t act_occ_b, int64_t act_unocc_a) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        if (c->calc_type != "CCSDT" && !c->has_crcc)
            throw Error(CCQ_B200_EINVAL, "set_active: a CCSDT or CR-CC(2,3) context is required");
        const long long occ_a = c->froz + c->oa, occ_b = c->froz + c->ob, orbs = occ_a + c->va;
        if (act_occ_b < c->froz || act_occ_b > occ_b || act_unocc_a < occ_a || act_unocc_a > orbs)
            throw Error(CCQ_B200_EINVAL, "set_active: froz <= act_occ_b <= occ_b and occ_a <= act_unocc_a <= orbs");
        if (c->act_occ_b >= 0 && (act_occ_b != c->act_occ_b || act_unocc_a != c->act_unocc_a))
            throw Error(CCQ_B200_EINVAL, "set_active: a CCSDt context keeps the active space it was created with");
        apply_active_masks(c, act_occ_b, act_unocc_a);
        // kernel arguments are recorded in the captured graphs
        drop_graphs(c);
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_force_tile(ccq_b200_ctx *c, int64_t tile) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    if (tile < 0 || tile > 6) return fail(Error(CCQ_B200_EINVAL, "force_tile: 0..6"));
    for (auto &o : c->plan.ops) {
        if (o.kind != OP_GETT || o.g.K == 0) continue;
        o.g.tile = (int)tile;
        if (o.g.segs) continue;
        // the small-K kernel takes the whole K range in one launch; the others the shape's split-K
        o.g.kchunk = (tile == 3 || tile == 6) ? (o.g.K + 15) / 16 * 16 : gett_f64_kchunk(o.g.M, o.g.N, o.g.K);
        o.zero_first = (o.g.K + o.g.kchunk - 1) / o.g.kchunk > 1 && o.beta == 0;
    }
    drop_graphs(c);
    return 0;
}

int ccq_b200_set_precision(ccq_b200_ctx *c, int64_t mode, int64_t nslices) {
    try {
        if (!c) throw Error(CCQ_B200_EINVAL, "null context");
        if (mode != CCQ_B200_PREC_FP64 && mode != CCQ_B200_PREC_SPLIT) throw Error(CCQ_B200_EINVAL, "precision mode");
        if (mode == CCQ_B200_PREC_SPLIT && (nslices < 2 || nslices > MAX_SLICES))
            throw Error(CCQ_B200_EINVAL, "nslices out of range");
        if (c->async_iter) throw Error(CCQ_B200_EINVAL, "set_precision: an iteration is pending");
        if (mode == CCQ_B200_PREC_SPLIT) {
            CK(cudaSetDevice(c->device));
            CK(cudaStreamSynchronize(c->stream));
            long long ma = 0, mb = 0, mc = 0;
            for (auto &o : c->plan.ops)
                if (o.kind == OP_GETT && o.split) {
                    ma = std::max(ma, o.mnk[0] * ((o.mnk[2] + 63) / 64 * 64));
                    mb = std::max(mb, o.mnk[1] * ((o.mnk[2] + 63) / 64 * 64));
                    mc = std::max(mc, std::max(o.mnk[0], o.mnk[1]));
                }
            const SplitSizes sz{ma, mb, mc};
            split_reserve(c->split, sz, (int)nslices);
            // kSplitPool workspaces in turn when they are small (else one, and split GETTs stay barriers)
            const long long bytes = (ma + mb) * nslices + 8 * mc;
            const int pool = bytes <= kSplitPoolBytes ? kSplitPool : 1;
            for (auto &w : c->split_pool) split_free(w);
            c->split_pool.assign(pool - 1, SplitWorkspace{});
            for (auto &w : c->split_pool) split_reserve(w, sz, (int)nslices);
            int k = 0;
            for (auto &o : c->plan.ops)
                if (o.kind == OP_GETT && o.split) o.split_ws = (k++) % pool;
        }
        drop_graphs(c);
        c->precision = (int)mode;
        c->nslices = (int)nslices;
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

int ccq_b200_use_graph(ccq_b200_ctx *c, int64_t enable) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    if (enable < 0 || enable > 2) return fail(Error(CCQ_B200_EINVAL, "use_graph: 0, 1 or 2"));
    if ((int)enable != c->use_graph) {
        drop_graphs(c);
    }
    c->use_graph = (int)enable;
    return 0;
}

int ccq_b200_stats(const ccq_b200_ctx *c, int64_t *launches, double *flops, double *sweep_ms) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    if (launches) *launches = c->launches;
    if (flops) *flops = c->flops;
    if (sweep_ms) *sweep_ms = c->sweep_ms;
    return 0;
}

int ccq_b200_timing(const ccq_b200_ctx *c, double *sweep_ms, double *iter_ms) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    if (sweep_ms) *sweep_ms = c->sweep_ms;
    if (iter_ms) *iter_ms = c->iter_ms;
    return 0;
}

int ccq_b200_profile(ccq_b200_ctx *c, int64_t enable) {
    if (!c) return fail(Error(CCQ_B200_EINVAL, "null context"));
    c->profile = enable != 0;
    for (int k = 0; k < 4; ++k) {
        c->prof_ms[k] = 0;
        c->prof_flops[k] = 0;
        c->prof_launch[k] = 0;
    }
    return 0;
}

int ccq_b200_profile_get(const ccq_b200_ctx *c, int64_t kind, double *ms, double *flops, int64_t *launches) {
    if (!c || kind < 0 || kind > 3) return fail(Error(CCQ_B200_EINVAL, "profile_get: bad argument"));
    if (ms) *ms = c->prof_ms[kind];
    if (flops) *flops = c->prof_flops[kind];
    if (launches) *launches = c->prof_launch[kind];
    return 0;
}

int ccq_b200_free(ccq_b200_ctx *c) {
    delete c;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched iterations of many independent contexts (C ABI ccq_b200_batch_*).
// Every context of a batch runs the same plan (same calc_type, rhf and diis_space, on one device),
// so operation k of every context is launched together: one GETT launch over the output tiles of
// all contexts' k-th contraction (64 x 64 tiles, whole K), one assemble launch over all their
// canonical elements, one launch for their buffer copies.  A device flag per context switches off
// the contexts that have converged.  Each context keeps its own amplitudes, ring and DIIS; only the
// per-context DIIS steps after the sweep are launched one context at a time.
// ---------------------------------------------------------------------------
struct BatchGett {
    int akm = 1, bkm = 1, n = 0, tiles = 0;
    GettArgs *args = nullptr;
    int *tstart = nullptr, *owner = nullptr;
    int nzero = 0;                      // entries whose split-K slices need a zeroed output
    GettArgs *zargs = nullptr;
    int *zowner = nullptr;
};

struct BatchStep {
    std::vector<BatchGett> gett;          // one launch per operand-orientation class
    int asm_rank = 0, asm_n = 0;
    long long asm_chunks = 0;
    AsmArgs *asm_args = nullptr;
    long long *asm_cstart = nullptr;
    int *asm_owner = nullptr;
    int ncopy = 0;
    BatchCopy *copies = nullptr;
    int *copy_owner = nullptr;
    std::vector<std::pair<int, GettArgs>> kzero;   // K = 0 contractions with beta = 0: zero the view
};

struct ccq_b200_batch {
    std::vector<ccq_b200_ctx *> ctx;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<BatchStep> steps;
    int *active_d = nullptr, *active_h = nullptr;
    std::vector<void *> owned;
    long long launches = 0;
    double sweep_ms = 0.0;

    template <typename T>
    T *upload(const std::vector<T> &h) {
        void *p = nullptr;
        CK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(h.size(), 1)));
        owned.push_back(p);
        if (!h.empty()) CK(cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
        return static_cast<T *>(p);
    }
    ~ccq_b200_batch() {
        for (void *p : owned) cudaFree(p);
        if (active_h) cudaFreeHost(active_h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" int ccq_b200_batch_create(ccq_b200_ctx *const *ctxs, int64_t n, ccq_b200_batch **out) {
    ccq_b200_batch *b = nullptr;
    try {
        if (!ctxs || n < 1 || !out) throw Error(CCQ_B200_EINVAL, "batch_create: bad argument");
        *out = nullptr;
        b = new ccq_b200_batch();
        for (int64_t j = 0; j < n; ++j) {
            ccq_b200_ctx *c = ctxs[j];
            if (!c) throw Error(CCQ_B200_EINVAL, "batch_create: null context");
            const ccq_b200_ctx *c0 = ctxs[0];
            if (c->device != c0->device || c->calc_type != c0->calc_type || c->rhf != c0->rhf || c->ds != c0->ds ||
                c->plan.ops.size() != c0->plan.ops.size() || c->cc_end != c0->cc_end)
                throw Error(CCQ_B200_EINVAL, "batch_create: contexts must share device, calc_type, rhf and diis_space");
            if (c->cdiis || c->async_iter) throw Error(CCQ_B200_EINVAL, "batch_create: unsupported context state");
            b->ctx.push_back(c);
        }
        b->device = ctxs[0]->device;
        CK(cudaSetDevice(b->device));
        CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&b->ev0));
        CK(cudaEventCreate(&b->ev1));
        CK(cudaMallocHost(&b->active_h, sizeof(int) * n));
        std::vector<int> ones(n, 1);
        b->active_d = b->upload(ones);
        const ccq_b200_ctx *c0 = ctxs[0];
        for (size_t i = 0; i < c0->cc_end; ++i) {
            BatchStep stp;
            const OpKind kind = c0->plan.ops[i].kind;
            std::map<std::pair<int, int>, std::vector<std::pair<int, GettArgs>>> cls;
            std::vector<AsmArgs> aa;
            std::vector<long long> cs;
            std::vector<int> aow;
            std::vector<BatchCopy> cp;
            std::vector<int> cow;
            for (int64_t j = 0; j < n; ++j) {
                ccq_b200_ctx *c = b->ctx[j];
                const Op &o = c->plan.ops[i];
                if (o.kind != kind) throw Error(CCQ_B200_EPLAN, "batch_create: plans differ");
                if (o.frozen) continue;
                switch (o.kind) {
                    case OP_GETT: {
                        if (o.skip || o.g.M == 0 || o.g.N == 0) break;
                        if (o.g.K == 0) {
                            if (!o.beta) stp.kzero.push_back({(int)j, o.g});
                            break;
                        }
                        GettArgs g = o.g;
                        if (g.nseg == 0 && (g.kchunk <= 0 || g.kchunk > g.K)) g.kchunk = g.K;
                        cls[{o.akm, o.bkm}].push_back({(int)j, g});
                        break;
                    }
                    case OP_ASM: {
                        if (stp.asm_rank && o.asmargs.rank != stp.asm_rank)
                            throw Error(CCQ_B200_EPLAN, "batch_create: assemble ranks differ");
                        stp.asm_rank = o.asmargs.rank;
                        cs.push_back(stp.asm_chunks);
                        stp.asm_chunks += (o.asmargs.total + ASM_CHUNK - 1) / ASM_CHUNK;
                        aa.push_back(o.asmargs);
                        aow.push_back((int)j);
                        break;
                    }
                    case OP_COPY: {
                        const DevBuf &d = c->bufs.at(o.arg0), &sbuf = c->bufs.at(o.arg1);
                        if (d.numel != sbuf.numel) throw Error(CCQ_B200_EPLAN, "COPY size mismatch");
                        cp.push_back({d.ptr, sbuf.ptr, d.numel});
                        cow.push_back((int)j);
                        break;
                    }
                    case OP_ZERO: {
                        const DevBuf &d = c->bufs.at(o.arg0);
                        cp.push_back({d.ptr, nullptr, std::max(d.numel, 1LL)});
                        cow.push_back((int)j);
                        break;
                    }
                    case OP_PHASE:
                        break;
                    default:
                        throw Error(CCQ_B200_EPLAN, "batch: plan operation without a batched kernel");
                }
            }
            for (auto &kv : cls) {
                BatchGett bg;
                bg.akm = kv.first.first;
                bg.bkm = kv.first.second;
                std::vector<GettArgs> args, zargs;
                std::vector<int> ts, ow, zow;
                for (auto &e : kv.second) {
                    const GettArgs &g = e.second;
                    const long long nz = g.nseg > 0 ? 1 : (g.K + g.kchunk - 1) / g.kchunk;
                    ts.push_back(bg.tiles);
                    bg.tiles += (int)(((g.M + 63) / 64) * ((g.N + 63) / 64) * nz);
                    args.push_back(g);
                    ow.push_back(e.first);
                    if (nz > 1 && !g.beta) {
                        zargs.push_back(g);
                        zow.push_back(e.first);
                    }
                }
                bg.n = (int)args.size();
                bg.args = b->upload(args);
                bg.tstart = b->upload(ts);
                bg.owner = b->upload(ow);
                if (!zargs.empty()) {
                    bg.nzero = (int)zargs.size();
                    bg.zargs = b->upload(zargs);
                    bg.zowner = b->upload(zow);
                }
                stp.gett.push_back(bg);
            }
            if (!aa.empty()) {
                stp.asm_n = (int)aa.size();
                stp.asm_args = b->upload(aa);
                stp.asm_cstart = b->upload(cs);
                stp.asm_owner = b->upload(aow);
            }
            if (!cp.empty()) {
                stp.ncopy = (int)cp.size();
                stp.copies = b->upload(cp);
                stp.copy_owner = b->upload(cow);
            }
            b->steps.push_back(std::move(stp));
        }
        *out = b;
        return 0;
    } catch (const Error &e) {
        delete b;
        return fail(e);
    } catch (const std::exception &e) {
        delete b;
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

extern "C" int ccq_b200_batch_iterate(ccq_b200_batch *b, int64_t iter, const int64_t *active, double *e_cor, double *res,
                           int64_t *did_diis) {
    try {
        if (!b || iter < 1 || !active) throw Error(CCQ_B200_EINVAL, "batch_iterate: bad argument");
        CK(cudaSetDevice(b->device));
        const int n = (int)b->ctx.size();
        for (int j = 0; j < n; ++j) b->active_h[j] = active[j] ? 1 : 0;
        CK(cudaMemcpyAsync(b->active_d, b->active_h, sizeof(int) * n, cudaMemcpyHostToDevice, b->stream));
        CK(cudaEventRecord(b->ev0, b->stream));
        long long launches = 0;
        for (auto &stp : b->steps) {
            for (auto &kz : stp.kzero)
                if (active[kz.first]) {
                    launch_zero_view(kz.second.C, kz.second.offC_m, kz.second.offC_n, kz.second.M, kz.second.N,
                                     b->stream);
                    ++launches;
                }
            for (auto &g : stp.gett) {
                if (g.nzero) {
                    launch_zero_views_batched(g.zargs, g.nzero, g.zowner, b->active_d, b->stream);
                    ++launches;
                }
                launch_gett_f64_batched(g.args, g.tstart, g.n, g.tiles, g.owner, b->active_d, g.akm, g.bkm, b->stream);
                ++launches;
            }
            if (stp.asm_n) {
                launch_assemble_batched(stp.asm_args, stp.asm_cstart, stp.asm_n, stp.asm_chunks, stp.asm_rank,
                                        stp.asm_owner, b->active_d, b->stream);
                ++launches;
            }
            if (stp.ncopy) {
                launch_copy_batched(stp.copies, stp.ncopy, stp.copy_owner, b->active_d, b->stream);
                ++launches;
            }
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(b->ev1, b->stream));
        for (int j = 0; j < n; ++j) {
            if (!active[j]) continue;
            ccq_b200_ctx *c = b->ctx[j];
            c->launches = 0;
            post_sweep(c, iter, b->stream);
            launches += c->launches;
        }
        CK(cudaStreamSynchronize(b->stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        b->sweep_ms = ms;
        b->launches = launches;
        const int diis = (iter % (b->ctx[0]->ds + 1)) == 0;
        for (int j = 0; j < n; ++j) {
            if (!active[j]) continue;
            ccq_b200_ctx *c = b->ctx[j];
            int info = 0;
            memcpy(&info, c->hpin + 2, sizeof(int));
            if (diis && info != 0) throw Error(CCQ_B200_ESINGULAR, "calc_diis: DIIS error in DGESV");
            if (e_cor) e_cor[j] = c->hpin[0];
            if (res) res[j] = std::sqrt(std::sqrt(c->hpin[1]));
            if (did_diis) did_diis[j] = diis;
        }
        return 0;
    } catch (const Error &e) {
        return fail(e);
    } catch (const std::exception &e) {
        return fail(Error(CCQ_B200_EINVAL, e.what()));
    }
}

extern "C" int ccq_b200_batch_stats(const ccq_b200_batch *b, int64_t *launches, double *sweep_ms) {
    if (!b) return fail(Error(CCQ_B200_EINVAL, "null batch"));
    if (launches) *launches = b->launches;
    if (sweep_ms) *sweep_ms = b->sweep_ms;
    return 0;
}

extern "C" int ccq_b200_batch_free(ccq_b200_batch *b) {
    delete b;
    return 0;
}


