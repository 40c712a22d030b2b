// brute.cu — batched filtered top-K: staging, launch sequence, results.
//
// Replaces fv_gpu_brute_batch and its host paths (gpu_engine.cu:1776-2336).
// One call: compile the batch's predicates on the host (pred.cpp), pack
// queries + predicate programs into one pinned buffer and copy it with a
// single H2D transfer, then on the index's stream
//   bitmap_kernel  -> one packed bitmap per distinct predicate
//   scan           -> per-CTA top-K lists + grid-wide bounds
//   merge_kernel   -> FvHit [nq][topb], counts, truncation flags
// and one D2H transfer of the packed results. Spans, need_eval and dedup
// are accepted for ABI compatibility; the scan evaluates the full
// predicate through the bitmap, which selects exactly the rows the driver
// spans would (a covering driver equals its predicate's match set,
// engine.cpp:464-599) and cannot produce duplicates.
#include <string.h>

#include <algorithm>

#include "index.h"
#include "paves_ext.h"
#include "pv_internal.h"

namespace pv {

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int brute_prepare(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                  DevBatch &db, size_t extra_bytes, char *errbuf, size_t errlen) {
    const size_t qbytes = (size_t)nq * g->dpad * 4;
    const int P = (int)pb.progs.size();
    db.nq = nq;
    db.P = P;
    db.ninsns = (int)pb.insns.size();
    db.nconsts = (int)pb.consts.size();
    db.off_q = 0;
    db.off_qprog = al256(qbytes);
    db.off_progs = db.off_qprog + al256((size_t)nq * 4);
    db.off_insns = db.off_progs + al256((size_t)P * sizeof(PredProg) + 8);
    db.off_consts = db.off_insns + al256(pb.insns.size() * sizeof(PredInsn) + 8);
    db.off_extra = db.off_consts + al256(pb.consts.size() * 8 + 8);
    db.bytes = db.off_extra + al256(extra_bytes);
    PV_CUDA_OK(db.stage_h->ensure(db.bytes), errbuf, errlen);
    PV_CUDA_OK(db.stage_d->ensure(db.bytes), errbuf, errlen);
    char *h = db.stage_h->as<char>();
    float *hq = (float *)(h + db.off_q);
    if (g->dpad == g->dim) {
        memcpy(hq, queries, qbytes);
    } else {
        for (int q = 0; q < nq; q++) {
            memcpy(hq + (size_t)q * g->dpad, queries + (size_t)q * g->dim, (size_t)g->dim * 4);
            memset(hq + (size_t)q * g->dpad + g->dim, 0, (size_t)(g->dpad - g->dim) * 4);
        }
    }
    db.q_amax = pv_integral_amax(queries, (uint64_t)nq * g->dim);
    memcpy(h + db.off_qprog, pb.qprog.data(), (size_t)nq * 4);
    if (P) memcpy(h + db.off_progs, pb.progs.data(), (size_t)P * sizeof(PredProg));
    if (!pb.insns.empty())
        memcpy(h + db.off_insns, pb.insns.data(), pb.insns.size() * sizeof(PredInsn));
    if (!pb.consts.empty()) memcpy(h + db.off_consts, pb.consts.data(), pb.consts.size() * 8);
    // one range-form program with well-formed terms: the lean bitmap kernel
    db.one_range = false;
    if (P == 1 && pb.progs[0].ninsn == 1 && pb.progs[0].insn0 >= 0 &&
        pb.progs[0].insn0 < (int)pb.insns.size() &&
        pb.insns[pb.progs[0].insn0].kind == PV_NODE_RANGE) {
        const PredInsn &r = pb.insns[pb.progs[0].insn0];
        bool ok = r.n >= 1 && r.n <= PV_RANGE_MAX_TERMS;
        int ci = r.val0;
        const int nc = (int)pb.consts.size();
        for (int k = 0; k < r.n && ok; k++) {
            ok = ci >= 0 && ci + 2 <= nc;
            if (!ok) break;
            const int meta = (int)pb.consts[ci];
            const bool mask = meta & PV_TERM_MASK;
            ok = (meta & 0xFFFF) < g->ncols && (mask || ci + 3 <= nc);
            ci += mask ? 2 : 3;
        }
        db.one_range = ok;
    }
    // sparse route: one filter shared by the whole batch whose matches are
    // bounded by a small count (the scan then reads only those rows)
    db.sparse_bound = 0;
    if (P == 1 && !g->sorted_cols.empty()) {
        bool all = true;
        for (int q = 0; q < nq && all; q++) all = pb.qprog[q] == 0;
        if (all) {
            const uint64_t b = prog_upper_bound(g, pb.insns.data() + pb.progs[0].insn0,
                                                pb.progs[0].ninsn, pb.consts.data());
            // (the route holds one key per query and listed row: 128 MB at most)
            if (b <= sparse_limit(g->count) && (uint64_t)nq * b <= (1ull << 24))
                db.sparse_bound = b;
        }
    }
    return 0;
}

int brute_upload(FvGpuIndex *g, DevBatch &db, char *errbuf, size_t errlen) {
    PV_CUDA_OK(cudaMemcpyAsync(db.stage_d->p, db.stage_h->p, db.bytes, cudaMemcpyHostToDevice,
                               g->stream),
               errbuf, errlen);
    return 0;
}

// Device-side work of one batch: inputs already resident in db.stage_d.
int brute_launch(FvGpuIndex *g, DevBatch &db, uint32_t topb, int mode, FvHit *d_out,
                 uint32_t *d_cnt, uint8_t *d_trunc, char *errbuf, size_t errlen,
                 cudaEvent_t *ev, bool bitmaps_ready, cudaEvent_t bm_done) {
    const int nq = db.nq, P = db.P;
    char *d = db.stage_d->as<char>();
    const float *d_q = (const float *)(d + db.off_q);
    const int32_t *d_qprog = (const int32_t *)(d + db.off_qprog);
    const PredProg *d_progs = (const PredProg *)(d + db.off_progs);
    const PredInsn *d_insns = (const PredInsn *)(d + db.off_insns);
    const double *d_consts = (const double *)(d + db.off_consts);
    const uint64_t bm_words = (g->count + 31) / 32;
    ScanScratch &s = g->scan;

    if (ev) cudaEventRecord(ev[0], g->stream);
    if (bitmaps_ready) {
        // the caller launched the bitmaps of this batch
    } else if (db.counts_on_device && P > 0) {
        PV_CUDA_OK(s.bitmaps.ensure((size_t)P * bm_words * 4), errbuf, errlen);
        PV_CUDA_OK(s.popcnt.ensure((size_t)P * 8), errbuf, errlen);
        g->launches++;
        PV_CUDA_OK(launch_bitmaps_capped(g->d_cols, g->count, d_insns, d_progs, d_consts,
                                         (const int *)(d + db.off_counts), P, db.ninsns,
                                         db.nconsts, s.bitmaps.as<uint32_t>(), bm_words,
                                         s.popcnt.as<unsigned long long>(), g->sm_count,
                                         g->stream, g->ncols),
                   errbuf, errlen);
    } else if (P > 0) {
        PV_CUDA_OK(s.bitmaps.ensure((size_t)P * bm_words * 4), errbuf, errlen);
        PV_CUDA_OK(s.popcnt.ensure((size_t)P * 8), errbuf, errlen);
        g->launches++;
        PV_CUDA_OK(launch_bitmaps(g->d_cols, g->count, d_insns, d_progs, d_consts, P,
                                  s.bitmaps.as<uint32_t>(), bm_words,
                                  s.popcnt.as<unsigned long long>(), g->sm_count, g->stream,
                                  db.ninsns, db.nconsts, g->ncols, db.one_range),
                   errbuf, errlen);
    } else {
        PV_CUDA_OK(s.popcnt.ensure(8), errbuf, errlen);
    }
    // this batch's bitmap kernel is the last launch on the stream (query
    // prep may run beside it): launched here, or by a caller that says so
    // by asking for bm_done
    const bool bm_launched =
        !db.counts_on_device && P > 0 && (!bitmaps_ready || bm_done != nullptr);
    const bool sparse_route = db.sparse_bound > 0 && !db.counts_on_device && topb <= 1024;
    const bool low_tc_route =
        !sparse_route && mode == 1 && tc_supported(g) && tc_superset(g, topb, db.q_amax) > 0;
    const bool exact_tc_route = !sparse_route && !low_tc_route && mode == PV_MODE_EXACT &&
                                nq >= PV_EXACT_TC_MIN_NQ && tf32_supported(g) &&
                                tf32_superset(g, topb, db.q_amax) > 0;
    // bm_done: the bitmaps are complete once query prep, run beside them,
    // completes (tensor-core routes), else at once in stream order
    if (bm_done && !(low_tc_route || exact_tc_route))
        PV_CUDA_OK(cudaEventRecord(bm_done, g->stream), errbuf, errlen);
    g->last_sparse = 0;
    g->last_exact_tc = 0;
    if (sparse_route) {
        g->last_sparse = 1;
        // the matching rows on the tensor cores, when the mode scans there
        const bool low_tc = mode == 1 && tc_supported(g) && tc_superset(g, topb, db.q_amax) > 0;
        const bool exact_tc = mode == PV_MODE_EXACT && nq >= PV_EXACT_TC_MIN_NQ &&
                              tf32_supported(g) && tf32_superset(g, topb, db.q_amax) > 0;
        if ((low_tc || exact_tc) && db.sparse_bound >= PV_SPARSE_TC_MIN_ROWS) {
            if (sparse_tc_launch(g, db, topb, db.sparse_bound, exact_tc, d_out, d_cnt, d_trunc,
                                 ev, errbuf, errlen))
                return -1;
            g->last_exact_tc = exact_tc ? 1 : 0;
            if (ev) cudaEventRecord(ev[4], g->stream);
            return 0;
        }
        g->tc_err = nullptr;
        g->tc_unc = nullptr;
        if (ev) cudaEventRecord(ev[1], g->stream);
        if (sparse_launch(g, db, topb, db.sparse_bound, d_out, d_cnt, d_trunc, errbuf, errlen))
            return -1;
        if (ev) {
            cudaEventRecord(ev[2], g->stream);
            cudaEventRecord(ev[3], g->stream);
            cudaEventRecord(ev[4], g->stream);
        }
        return 0;
    }
    if (low_tc_route) {
        // a staged batch with its counts on the device (the stream's graphs)
        // may mark itself lazy: then it has no bitmaps (see stream.cu)
        TcLazy lz{(const int *)(d + db.off_counts) + 3, d_progs, d_insns, d_consts,
                  db.nconsts};
        if (launch_scan_tc(g, nq, db.q_amax, d_q, d_qprog, s.bitmaps.as<uint32_t>(), bm_words,
                           s.popcnt.as<unsigned long long>(), topb, d_out, d_cnt, d_trunc, ev,
                           errbuf, errlen, db.counts_on_device ? &lz : nullptr, false, nullptr,
                           bm_launched, bm_done))
            return -1;
        if (ev) cudaEventRecord(ev[4], g->stream);
        return 0;
    }
    if (exact_tc_route) {
        TcLazy lz{(const int *)(d + db.off_counts) + 3, d_progs, d_insns, d_consts,
                  db.nconsts};
        if (launch_scan_tc(g, nq, db.q_amax, d_q, d_qprog, s.bitmaps.as<uint32_t>(), bm_words,
                           s.popcnt.as<unsigned long long>(), topb, d_out, d_cnt, d_trunc, ev,
                           errbuf, errlen, db.counts_on_device ? &lz : nullptr, true, nullptr,
                           bm_launched, bm_done))
            return -1;
        g->last_exact_tc = 1;
        if (ev) cudaEventRecord(ev[4], g->stream);
        return 0;
    }
    g->tc_err = nullptr;
    g->tc_unc = nullptr;

    ScanPlan pl;
    // query tiles of 32-64 take the register-blocked kernel (FP32-pipe
    // bound), small tiles the bandwidth-bound one
    const bool tiled = plan_scan_f32t(g->count, g->dpad, nq, (int)topb, g->sm_count, pl);
    if (!tiled && !plan_scan_f32(g->count, g->dpad, nq, (int)topb, g->sm_count, pl)) {
        snprintf(errbuf, errlen, "gpu: dimension %d not supported by the scan", g->dim);
        return -1;
    }
    PV_CUDA_OK(s.tau.ensure((size_t)nq * 8), errbuf, errlen);
    PV_CUDA_OK(s.part.ensure((size_t)nq * pl.grow * topb * 8), errbuf, errlen);
    PV_CUDA_OK(s.part_cnt.ensure((size_t)nq * pl.grow * 4), errbuf, errlen);
    PV_CUDA_OK(cudaMemsetAsync(s.tau.p, 0xFF, (size_t)nq * 8, g->stream), errbuf, errlen);

    ScanF32Args a;
    a.vecs = g->d_vecs;
    a.nrows = g->count;
    a.dpad = g->dpad;
    a.queries = d_q;
    a.nq = nq;
    a.bitmaps = s.bitmaps.as<uint32_t>();
    a.bm_words = bm_words;
    a.qprog = d_qprog;
    a.K = (int)topb;
    a.S = pl.S;
    a.CB = pl.CB;
    a.rows_per_cta = pl.rows_per_cta;
    a.grow = pl.grow;
    a.qtiles = pl.qtiles;
    a.tau = s.tau.as<unsigned long long>();
    a.part = s.part.as<uint64_t>();
    a.part_cnt = s.part_cnt.as<uint32_t>();
    if (ev) cudaEventRecord(ev[1], g->stream);
    g->launches += 2;  // scan + merge
    PV_CUDA_OK(tiled ? launch_scan_f32t(a, pl, g->stream) : launch_scan_f32(a, pl, g->stream),
               errbuf, errlen);
    if (ev) {
        cudaEventRecord(ev[2], g->stream);
        cudaEventRecord(ev[3], g->stream);
    }
    PV_CUDA_OK(launch_merge(a.part, a.part_cnt, pl.grow, (int)topb, pl, a.tau, d_qprog,
                            s.popcnt.as<unsigned long long>(), g->count, nq, d_out, d_cnt,
                            d_trunc, g->stream),
               errbuf, errlen);
    if (ev) cudaEventRecord(ev[4], g->stream);
    return 0;
}

}  // namespace pv

using namespace pv;

extern "C" int fv_gpu_tile_variant_qt(int dim) {
    if (dim <= 0) return 0;
    return scan_f32_max_qt(dim);
}

extern "C" int fv_gpu_brute_batch(FvGpuIndex *g, int nq, const float *queries,
                                  const FvGpuQueryDesc *qd, const uint8_t *dedup,
                                  const FvGpuPredNode *nodes, int nnodes,
                                  const int32_t *children, int nchildren,
                                  const double *invals, int ninvals, const FvGpuSpan *spans,
                                  int nspans_total, const uint64_t *spanoff, int nspanoff,
                                  uint32_t topb, FvHit *out, uint32_t *out_cnt,
                                  uint8_t *truncated, char *errbuf, size_t errlen) {
    (void)dedup;
    (void)spans;
    (void)spanoff;
    (void)nspanoff;
    if (!g || nq < 1 || nq > FV_GPU_MAX_BATCH || topb == 0 || topb > FV_GPU_MAX_TOPB ||
        nspans_total > FV_GPU_MAX_SPANS * nq || !queries || !qd || !out || !out_cnt ||
        !truncated) {
        if (errbuf && errlen)
            snprintf(errbuf, errlen, "gpu: bad brute batch (nq=%d topb=%u)", nq, topb);
        return -1;
    }
    std::lock_guard<std::mutex> lk(g->mu);
    PV_CUDA_OK(cudaSetDevice(g->device), errbuf, errlen);
    PredBatch pb;
    if (compile_predicates(nq, &qd[0].proot, sizeof(FvGpuQueryDesc), nodes, nnodes, children,
                           nchildren, invals, ninvals, g->ncols, pb, errbuf, errlen) != 0)
        return -1;
    return brute_run_host(g, nq, queries, pb, topb, FV_GPU_PREC_FP32 == g->precision ? 0 : 1,
                          out, out_cnt, truncated, errbuf, errlen);
}

namespace pv {

// Re-runs exactly the queries whose reduced-precision superset the last TC
// merge could not certify (a full per-CTA list may have dropped a member of
// it) and writes their results over the caller's out / out_cnt / truncated
// (stride topb). Call after the batch's results were copied out: the re-run
// reuses the index's staging buffers.
int tc_redo_uncertain(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                      uint32_t topb, FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                      char *errbuf, size_t errlen) {
    g->last_uncertain = 0;
    if (!g->tc_unc) return 0;
    std::vector<uint8_t> unc((size_t)nq);
    PV_CUDA_OK(cudaMemcpyAsync(unc.data(), g->tc_unc, (size_t)nq, cudaMemcpyDeviceToHost,
                               g->stream),
               errbuf, errlen);
    PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    g->tc_unc = nullptr;
    return redo_flagged(g, nq, queries, pb, topb, unc.data(), out, out_cnt, truncated, errbuf,
                        errlen);
}

int redo_flagged(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                 uint32_t topb, const uint8_t *unc, FvHit *out, uint32_t *out_cnt,
                 uint8_t *truncated, char *errbuf, size_t errlen) {
    g->last_uncertain = 0;
    std::vector<int> idx;
    for (int q = 0; q < nq; q++)
        if (unc[q]) idx.push_back(q);
    g->last_uncertain = (int)idx.size();
    if (idx.empty()) return 0;
    const int n = (int)idx.size(), dim = g->dim;
    std::vector<float> sq((size_t)n * dim);
    PredBatch sub = pb;
    for (int i = 0; i < n; i++) {
        memcpy(&sq[(size_t)i * dim], queries + (size_t)idx[i] * dim, sizeof(float) * dim);
        sub.qprog[i] = pb.qprog[idx[i]];
    }
    sub.qprog.resize(n);
    std::vector<FvHit> so((size_t)n * topb);
    std::vector<uint32_t> sc(n);
    std::vector<uint8_t> st(n);
    const int launches = g->launches, nunc = n, took_tc = g->last_exact_tc;
    if (brute_run_host(g, n, sq.data(), sub, topb, PV_MODE_SIMT, so.data(), sc.data(),
                       st.data(), errbuf, errlen))
        return -1;
    g->launches += launches;
    g->last_uncertain = nunc;
    g->last_exact_tc = took_tc;  // the batch's own route
    for (int i = 0; i < n; i++) {
        const int q = idx[i];
        memcpy(out + (size_t)q * topb, &so[(size_t)i * topb], sizeof(FvHit) * sc[i]);
        out_cnt[q] = sc[i];
        truncated[q] = st[i];
    }
    return 0;
}

int brute_run_host(FvGpuIndex *g, int nq, const float *queries, const PredBatch &pb,
                   uint32_t topb, int mode, FvHit *out, uint32_t *out_cnt, uint8_t *truncated,
                   char *errbuf, size_t errlen) {
    g->launches = 0;
    DevBatch db;
    db.stage_h = &g->scan.stage_h;
    db.stage_d = &g->scan.stage_d;
    if (brute_prepare(g, nq, queries, pb, db, 0, errbuf, errlen)) return -1;
    const size_t hit_bytes = (size_t)nq * topb * sizeof(FvHit);
    const size_t off_cnt = al256(hit_bytes);
    const size_t off_tr = off_cnt + al256((size_t)nq * 4);
    const size_t obytes = off_tr + al256((size_t)nq);
    PV_CUDA_OK(g->scan.out_d.ensure(obytes), errbuf, errlen);
    PV_CUDA_OK(g->scan.out_h.ensure(obytes + 256), errbuf, errlen);  // + the watchdog word
    char *od = g->scan.out_d.as<char>();
    if (brute_upload(g, db, errbuf, errlen)) return -1;
    cudaEventRecord(g->ev0, g->stream);
    if (brute_launch(g, db, topb, mode, (FvHit *)od, (uint32_t *)(od + off_cnt),
                     (uint8_t *)(od + off_tr), errbuf, errlen, nullptr))
        return -1;
    cudaEventRecord(g->ev1, g->stream);
    PV_CUDA_OK(cudaMemcpyAsync(g->scan.out_h.p, od, obytes, cudaMemcpyDeviceToHost, g->stream),
               errbuf, errlen);
    tc_watchdog_enqueue(g, (int *)(g->scan.out_h.as<char>() + obytes));
    PV_CUDA_OK(cudaStreamSynchronize(g->stream), errbuf, errlen);
    if (check_tc_watchdog(g, errbuf, errlen)) return -1;
    cudaEventElapsedTime(&g->last_kernel_ms, g->ev0, g->ev1);
    const char *oh = g->scan.out_h.as<char>();
    const uint32_t *cnt = (const uint32_t *)(oh + off_cnt);
    for (int q = 0; q < nq; q++) {
        uint32_t c = cnt[q] > topb ? topb : cnt[q];
        memcpy(out + (size_t)q * topb, oh + (size_t)q * topb * sizeof(FvHit), c * sizeof(FvHit));
        out_cnt[q] = c;
    }
    memcpy(truncated, oh + off_tr, (size_t)nq);
    return tc_redo_uncertain(g, nq, queries, pb, topb, out, out_cnt, truncated, errbuf, errlen);
}

}  // namespace pv
