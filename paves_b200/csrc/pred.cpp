// pred.cpp — host-side predicate compiler.
//
// The ABI hands over every query's predicate as a slice of the concatenated
// FvGpuPredNode / children / IN-value arrays (layout: engine.cpp:1232-1282,
// GpuConcat::build; node semantics: engine.cpp:397-431, FvPred::eval_node).
// Here each query's tree is walked from its root, bounds-checked, and
// re-serialized in post-order with n-ary AND/OR folded into binary steps so
// the device evaluates it with a 64-bit bit stack. Identical predicates in a
// batch share one program (and therefore one bitmap).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <unordered_map>

#include "index.h"

namespace pv {

namespace {

struct Walker {
    const FvGpuPredNode *nodes;
    int nnodes;
    const int32_t *children;
    int nchildren;
    const double *invals;
    int ninvals;
    int ncols;
    std::vector<PredInsn> out;
    std::vector<double> consts;
    int budget;  // guards against cyclic child references
    int depth = 0, maxdepth = 0;
    const char *err = nullptr;

    void push_depth(int d) {
        depth += d;
        if (depth > maxdepth) maxdepth = depth;
    }

    bool emit(int ni, int level) {
        if (ni < 0 || ni >= nnodes) { err = "predicate child index out of range"; return false; }
        if (--budget < 0) { err = "predicate tree is cyclic or too large"; return false; }
        if (level > 60) { err = "predicate tree deeper than 60 levels"; return false; }
        const FvGpuPredNode &n = nodes[ni];
        PredInsn in;
        memset(&in, 0, sizeof(in));
        in.kind = n.kind;
        switch (n.kind) {
            case FV_NODE_CMP:
                if (n.col < 0 || n.col >= ncols) { err = "predicate column out of range"; return false; }
                if (n.op < FV_CMP_LT || n.op > FV_CMP_NE) { err = "bad comparison operator"; return false; }
                in.col = n.col;
                in.op = n.op;
                in.value = n.value;
                out.push_back(in);
                push_depth(1);
                return true;
            case FV_NODE_IN: {
                if (n.col < 0 || n.col >= ncols) { err = "predicate column out of range"; return false; }
                if (n.nvalues < 0 || n.val0 < 0 || (int64_t)n.val0 + n.nvalues > ninvals) {
                    err = "IN value range out of bounds";
                    return false;
                }
                in.col = n.col;
                in.n = n.nvalues;
                in.val0 = (int32_t)consts.size();
                for (int i = 0; i < n.nvalues; i++) consts.push_back(invals[n.val0 + i]);
                out.push_back(in);
                push_depth(1);
                return true;
            }
            case FV_NODE_AND:
            case FV_NODE_OR: {
                if (n.nchildren < 0 || n.child0 < 0 ||
                    (int64_t)n.child0 + n.nchildren > nchildren) {
                    err = "child range out of bounds";
                    return false;
                }
                if (n.nchildren == 0) {
                    // empty AND is true, empty OR is false (engine.cpp:418-425)
                    in.n = 0;
                    out.push_back(in);
                    push_depth(1);
                    return true;
                }
                if (!emit(children[n.child0], level + 1)) return false;
                for (int i = 1; i < n.nchildren; i++) {
                    if (!emit(children[n.child0 + i], level + 1)) return false;
                    in.n = 2;
                    out.push_back(in);
                    push_depth(-1);
                }
                return true;
            }
            case FV_NODE_NOT:
                if (n.nchildren < 1 || n.child0 < 0 || n.child0 >= nchildren) {
                    err = "NOT without child";
                    return false;
                }
                if (!emit(children[n.child0], level + 1)) return false;
                in.n = 1;
                out.push_back(in);
                return true;
            default:
                err = "unknown predicate node kind";
                return false;
        }
    }
};

// ---- range form: a program that is an AND of comparisons and IN lists
// becomes one PV_NODE_RANGE instruction (see common.cuh). Comparisons on
// one column merge into one interval; IN lists of integers in [0, 64)
// become a bit mask; anything else (OR, NOT, NE, other IN lists) keeps the
// stack program.
struct Term {
    int col;
    bool mask;
    uint64_t bits;
    double lo, hi;
    bool lo_open, hi_open;
};

bool small_int(double v) { return v >= 0.0 && v < 64.0 && (double)(int)v == v; }

bool to_range(const std::vector<PredInsn> &prog, const std::vector<double> &consts,
              std::vector<PredInsn> &out, std::vector<double> &outc) {
    struct Conj {
        bool ok;
        std::vector<Term> t;
    };
    const double inf = HUGE_VAL;
    std::vector<Conj> st;
    for (const PredInsn &in : prog) {
        switch (in.kind) {
            case FV_NODE_CMP: {
                Term t{in.col, false, 0, -inf, inf, false, false};
                const double c = in.value;
                switch (in.op) {
                    case FV_CMP_LT: t.hi = c; t.hi_open = true; break;
                    case FV_CMP_LE: t.hi = c; break;
                    case FV_CMP_GT: t.lo = c; t.lo_open = true; break;
                    case FV_CMP_GE: t.lo = c; break;
                    case FV_CMP_EQ: t.lo = c; t.hi = c; break;
                    default: return false;  // NE is true for no NaN but not an interval
                }
                st.push_back({true, {t}});
                break;
            }
            case FV_NODE_IN: {
                Term t{in.col, true, 0, 0.0, 0.0, false, false};
                bool all_small = true;
                for (int j = 0; j < in.n; j++) {
                    const double v = consts[in.val0 + j];
                    if (small_int(v)) t.bits |= 1ull << (int)v;
                    else all_small = false;
                }
                if (!all_small) {
                    // one distinct value is an interval [v, v]
                    bool same = in.n > 0;
                    for (int j = 1; j < in.n && same; j++)
                        same = consts[in.val0 + j] == consts[in.val0];
                    if (!same) return false;
                    const double v = consts[in.val0];
                    t = Term{in.col, false, 0, v, v, false, false};
                }
                st.push_back({true, {t}});
                break;
            }
            case FV_NODE_AND:
                if (in.n == 0) {
                    st.push_back({true, {}});
                } else {
                    if (st.size() < 2) return false;
                    Conj b = st.back();
                    st.pop_back();
                    Conj &a = st.back();
                    a.ok = a.ok && b.ok;
                    a.t.insert(a.t.end(), b.t.begin(), b.t.end());
                }
                break;
            default:
                return false;  // OR, NOT
        }
    }
    if (st.size() != 1 || !st[0].ok) return false;
    // merge per column: one interval and one mask at most
    std::vector<Term> terms;
    for (const Term &t : st[0].t) {
        Term *m = nullptr;
        for (Term &u : terms)
            if (u.col == t.col && u.mask == t.mask) m = &u;
        if (!m) {
            terms.push_back(t);
            continue;
        }
        if (t.mask) {
            m->bits &= t.bits;
            continue;
        }
        if (t.lo != t.lo || m->lo != m->lo || t.hi != t.hi || m->hi != m->hi) {
            m->lo = m->hi = NAN;  // a NaN bound fails every row
            continue;
        }
        if (t.lo > m->lo) { m->lo = t.lo; m->lo_open = t.lo_open; }
        else if (t.lo == m->lo) m->lo_open = m->lo_open || t.lo_open;
        if (t.hi < m->hi) { m->hi = t.hi; m->hi_open = t.hi_open; }
        else if (t.hi == m->hi) m->hi_open = m->hi_open || t.hi_open;
    }
    if ((int)terms.size() > PV_RANGE_MAX_TERMS) return false;
    PredInsn r;
    memset(&r, 0, sizeof(r));
    r.kind = PV_NODE_RANGE;
    r.n = (int32_t)terms.size();
    r.val0 = 0;
    out.assign(1, r);
    outc.clear();
    for (Term t : terms) {
        // open bounds become closed ones: on doubles lo < v is lo' <= v with
        // lo' the next double up (v < hi likewise); an open +inf lower or
        // -inf upper bound admits nothing (NaN)
        if (!t.mask && t.lo_open) {
            t.lo = t.lo == HUGE_VAL ? NAN : nextafter(t.lo, HUGE_VAL);
            t.lo_open = false;
        }
        if (!t.mask && t.hi_open) {
            t.hi = t.hi == -HUGE_VAL ? NAN : nextafter(t.hi, -HUGE_VAL);
            t.hi_open = false;
        }
        const int meta = t.col | (t.mask ? PV_TERM_MASK : 0);
        outc.push_back((double)meta);
        if (t.mask) {
            double b;
            memcpy(&b, &t.bits, 8);
            outc.push_back(b);
        } else {
            outc.push_back(t.lo);
            outc.push_back(t.hi);
        }
    }
    return true;
}

// Structural hash and equality of node trees, straight from the ABI arrays
// (no allocation): identical predicates in different slices of the
// concatenated arrays are found before any program is built. hash returns
// false on anything the walker would reject; such queries take the walker,
// which reports the error.
struct TreeView {
    const FvGpuPredNode *nodes;
    int nnodes;
    const int32_t *children;
    int nchildren;
    const double *invals;
    int ninvals;

    static uint64_t mix(uint64_t h, uint64_t v) {
        h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        return h;
    }
    static uint64_t bits(double v) {
        uint64_t b;
        memcpy(&b, &v, 8);
        return b;
    }
    bool child_range(const FvGpuPredNode &n) const {
        return n.nchildren >= 0 && n.child0 >= 0 && (int64_t)n.child0 + n.nchildren <= nchildren;
    }
    bool hash(int ni, int level, int &budget, uint64_t &h) const {
        if (ni < 0 || ni >= nnodes || --budget < 0 || level > 60) return false;
        const FvGpuPredNode &n = nodes[ni];
        h = mix(h, (uint64_t)(uint32_t)n.kind);
        switch (n.kind) {
            case FV_NODE_CMP:
                h = mix(mix(mix(h, (uint64_t)(uint32_t)n.col), (uint64_t)(uint32_t)n.op), bits(n.value));
                return true;
            case FV_NODE_IN:
                if (n.nvalues < 0 || n.val0 < 0 || (int64_t)n.val0 + n.nvalues > ninvals) return false;
                h = mix(mix(h, (uint64_t)(uint32_t)n.col), (uint64_t)(uint32_t)n.nvalues);
                for (int i = 0; i < n.nvalues; i++) h = mix(h, bits(invals[n.val0 + i]));
                return true;
            case FV_NODE_AND:
            case FV_NODE_OR:
            case FV_NODE_NOT: {
                const int nc = n.kind == FV_NODE_NOT ? 1 : n.nchildren;
                if (n.kind == FV_NODE_NOT ? (n.nchildren < 1 || n.child0 < 0 || n.child0 >= nchildren)
                                          : !child_range(n))
                    return false;
                h = mix(h, (uint64_t)(uint32_t)nc);
                for (int i = 0; i < nc; i++)
                    if (!hash(children[n.child0 + i], level + 1, budget, h)) return false;
                return true;
            }
            default:
                return false;
        }
    }
    // a and b were both hashed successfully
    bool equal(int a, int b, int level) const {
        if (a == b) return true;
        if (level > 60) return false;
        const FvGpuPredNode &x = nodes[a], &y = nodes[b];
        if (x.kind != y.kind) return false;
        switch (x.kind) {
            case FV_NODE_CMP:
                return x.col == y.col && x.op == y.op && bits(x.value) == bits(y.value);
            case FV_NODE_IN:
                if (x.col != y.col || x.nvalues != y.nvalues) return false;
                for (int i = 0; i < x.nvalues; i++)
                    if (bits(invals[x.val0 + i]) != bits(invals[y.val0 + i])) return false;
                return true;
            default: {
                const int nx = x.kind == FV_NODE_NOT ? 1 : x.nchildren;
                const int ny = y.kind == FV_NODE_NOT ? 1 : y.nchildren;
                if (nx != ny) return false;
                for (int i = 0; i < nx; i++)
                    if (!equal(children[x.child0 + i], children[y.child0 + i], level + 1))
                        return false;
                return true;
            }
        }
    }
};

}  // namespace

// Compiles the per-query predicates of a batch. Returns 0, or -1 + errbuf.
int compile_predicates(int nq, const int32_t *proot, size_t proot_stride,
                       const FvGpuPredNode *nodes, int nnodes,
                       const int32_t *children, int nchildren,
                       const double *invals, int ninvals, int ncols,
                       PredBatch &pb, char *errbuf, size_t errlen) {
    pb.insns.clear();
    pb.progs.clear();
    pb.consts.clear();
    pb.qprog.assign(nq, -1);
    pb.cols_used.clear();
    if ((nnodes > 0 && !nodes) || (nchildren > 0 && !children) || (ninvals > 0 && !invals)) {
        snprintf(errbuf, errlen, "gpu: predicate array is NULL");
        return -1;
    }
    std::unordered_map<std::string, int> seen;
    // structurally identical trees (the same root included) share one
    // program without re-walking: an open-addressing table of
    // (hash, representative root, program)
    const TreeView tv{nodes, nnodes, children, nchildren, invals, ninvals};
    struct Rep {
        uint64_t h;
        int32_t root;
        int pid;
    };
    size_t tsize = 16;
    while (tsize < 2 * (size_t)nq) tsize <<= 1;
    std::vector<Rep> reps(tsize, Rep{0, -1, -1});
    for (int q = 0; q < nq; q++) {
        int32_t root = *(const int32_t *)((const char *)proot + (size_t)q * proot_stride);
        if (root < 0) continue;
        if (root >= nnodes) {
            snprintf(errbuf, errlen, "gpu: query %d predicate root %d out of range (nnodes=%d)",
                     q, root, nnodes);
            return -1;
        }
        uint64_t h = 0;
        int hb = 4 * nnodes + 16;
        const bool hashed = tv.hash(root, 0, hb, h);
        size_t slot = (size_t)(h ^ (h >> 29)) & (tsize - 1);
        if (hashed) {
            int hit = -1;
            for (; reps[slot].root >= 0; slot = (slot + 1) & (tsize - 1))
                if (reps[slot].h == h && tv.equal(reps[slot].root, root, 0)) {
                    hit = reps[slot].pid;
                    break;
                }
            if (hit >= 0) {
                pb.qprog[q] = hit;
                continue;
            }
        }
        Walker w{nodes, nnodes, children, nchildren, invals, ninvals, ncols, {}, {}, 4 * nnodes + 16};
        if (!w.emit(root, 0)) {
            snprintf(errbuf, errlen, "gpu: query %d: %s", q, w.err);
            return -1;
        }
        if (w.maxdepth > 63) {
            snprintf(errbuf, errlen, "gpu: query %d predicate needs a stack deeper than 63", q);
            return -1;
        }
        {
            std::vector<PredInsn> ri;
            std::vector<double> rc;
            if (to_range(w.out, w.consts, ri, rc)) {
                w.out.swap(ri);
                w.consts.swap(rc);
            }
        }
        // canonical bytes: instructions with constants inlined
        std::string sig;
        int32_t colmask = 0;
        for (const PredInsn &in : w.out) {
            PredInsn c = in;
            c.val0 = 0;
            sig.append((const char *)&c, sizeof(c));
            if (in.kind == FV_NODE_IN)
                sig.append((const char *)&w.consts[in.val0], sizeof(double) * in.n);
            if (in.kind == FV_NODE_CMP || in.kind == FV_NODE_IN) colmask |= (int32_t)(1u << (in.col & 31));
            if (in.kind == PV_NODE_RANGE) {
                sig.append((const char *)w.consts.data(), sizeof(double) * w.consts.size());
                for (size_t j = 0, k = 0; k < (size_t)in.n; k++) {
                    const int meta = (int)w.consts[j];
                    colmask |= (int32_t)(1u << ((meta & 0xFFFF) & 31));
                    j += (meta & PV_TERM_MASK) ? 2 : 3;
                }
            }
        }
        auto it = seen.find(sig);
        int pid;
        if (it != seen.end()) {
            pid = it->second;
        } else {
            pid = (int)pb.progs.size();
            PredProg pg;
            pg.insn0 = (int32_t)pb.insns.size();
            pg.ninsn = (int32_t)w.out.size();
            int32_t cbase = (int32_t)pb.consts.size();
            for (PredInsn in : w.out) {
                if (in.kind == FV_NODE_IN || in.kind == PV_NODE_RANGE) in.val0 += cbase;
                pb.insns.push_back(in);
            }
            pb.consts.insert(pb.consts.end(), w.consts.begin(), w.consts.end());
            pb.progs.push_back(pg);
            pb.cols_used.push_back(colmask);
            seen.emplace(std::move(sig), pid);
        }
        if (hashed) reps[slot] = Rep{h, root, pid};  // the free slot the probe stopped at
        pb.qprog[q] = pid;
    }
    return 0;
}

}  // namespace pv
