// pred.cpp — host-side predicate compiler.
//
// The ABI hands over every query's predicate as a slice of the concatenated
// FvGpuPredNode / children / IN-value arrays (layout: engine.cpp:1232-1282,
// GpuConcat::build; node semantics: engine.cpp:397-431, FvPred::eval_node).
// Here each query's tree is walked from its root, bounds-checked, and
// re-serialized in post-order with n-ary AND/OR folded into binary steps so
// the device evaluates it with a 64-bit bit stack. Identical predicates in a
// batch share one program (and therefore one bitmap).
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
    // identical roots map to the same program without re-walking
    std::unordered_map<int32_t, int> by_root;
    for (int q = 0; q < nq; q++) {
        int32_t root = *(const int32_t *)((const char *)proot + (size_t)q * proot_stride);
        if (root < 0) continue;
        if (root >= nnodes) {
            snprintf(errbuf, errlen, "gpu: query %d predicate root %d out of range (nnodes=%d)",
                     q, root, nnodes);
            return -1;
        }
        auto br = by_root.find(root);
        if (br != by_root.end()) {
            pb.qprog[q] = br->second;
            continue;
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
                if (in.kind == FV_NODE_IN) in.val0 += cbase;
                pb.insns.push_back(in);
            }
            pb.consts.insert(pb.consts.end(), w.consts.begin(), w.consts.end());
            pb.progs.push_back(pg);
            pb.cols_used.push_back(colmask);
            seen.emplace(std::move(sig), pid);
        }
        by_root.emplace(root, pid);
        pb.qprog[q] = pid;
    }
    return 0;
}

}  // namespace pv
