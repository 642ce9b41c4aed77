// Host side of the batched solver: problem upload, the autotuner that picks
// the thread-group size and operator format per size bucket, and the single
// persistent launch that solves the whole batch.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../../include/trlx.h"
#include "batched.h"

using trlb::batched::Params;
using trlb::batched::Problem;

struct trlx_batch {
    int nprob = 0;
    bool stencil = false;            // created from 5-point stencil data
    std::vector<Problem> probs;      // host copy (offsets)
    std::vector<int> L;              // stencil grid sides
    std::vector<long long> diag_off;
    // device arrays
    Problem *d_probs = nullptr;
    int *d_order = nullptr;
    double *d_diag = nullptr;
    long long *d_rp = nullptr;
    int *d_col = nullptr;
    double *d_val = nullptr;
    double *d_start = nullptr;
    double *d_basis = nullptr;
    size_t basis_doubles = 0;
    double *d_evec = nullptr;
    size_t evec_doubles = 0;
    double *d_eval = nullptr, *d_res = nullptr;
    int *d_info = nullptr;
    unsigned *d_queue = nullptr;
    int ned_alloc = 0, maxlan_alloc = 0;
    // autotuned configuration (per bucket: threads, format)
    bool tuned = false;
    int tuned_maxlan = 0;
    int bucket_threads[3] = {1024, 512, 256};
    int bucket_format[3] = {0, 0, 0};
    int cta = 1024;
    double tune_seconds = 0.0;
    // The solve's launch sequence (queue reset + the persistent kernel),
    // captured once as a CUDA graph per distinct launch configuration and
    // replayed on the batch's own stream.
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    Params graph_params{};
    int graph_blocks = 0;
    int graph_launches = 0;  // replays of the current graph
};

namespace {

// Size buckets (rows): [0] > 32768, [1] (8192, 32768], [2] <= 8192.
int bucket_of(int n) { return n > 32768 ? 0 : (n > 8192 ? 1 : 2); }

template <class X>
int upload(const std::vector<X> &h, X **d) {
    if (h.empty()) return 0;
    if (cudaMalloc(reinterpret_cast<void **>(d), sizeof(X) * h.size()) != cudaSuccess) {
        cudaGetLastError();
        return -5;
    }
    return cudaMemcpy(*d, h.data(), sizeof(X) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1001;
}

int sms() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

// (Re)allocate basis, outputs and per-problem offsets for ned / maxlan.
int prepare(trlx_batch *b, int ned, int maxlan) {
    if (b->ned_alloc == ned && b->maxlan_alloc == maxlan && b->d_basis) return 0;
    cudaFree(b->d_basis);
    cudaFree(b->d_evec);
    cudaFree(b->d_eval);
    cudaFree(b->d_res);
    cudaFree(b->d_info);
    b->d_basis = b->d_evec = b->d_eval = b->d_res = nullptr;
    b->d_info = nullptr;
    size_t boff = 0, eoff = 0;
    for (auto &p : b->probs) {
        p.basis_off = (long long)boff;
        p.evec_off = (long long)eoff;
        boff += (size_t)(maxlan + 1) * p.ld;
        eoff += (size_t)ned * p.n;
    }
    b->basis_doubles = boff;
    b->evec_doubles = eoff;
    if (cudaMalloc(&b->d_basis, sizeof(double) * boff) != cudaSuccess ||
        cudaMalloc(&b->d_evec, sizeof(double) * eoff) != cudaSuccess ||
        cudaMalloc(&b->d_eval, sizeof(double) * (size_t)b->nprob * ned) != cudaSuccess ||
        cudaMalloc(&b->d_res, sizeof(double) * (size_t)b->nprob * ned) != cudaSuccess ||
        cudaMalloc(&b->d_info, sizeof(int) * 4 * (size_t)b->nprob) != cudaSuccess) {
        cudaGetLastError();
        return -5;
    }
    cudaFree(b->d_probs);
    b->d_probs = nullptr;
    int rc = upload(b->probs, &b->d_probs);
    if (rc) return rc;
    b->ned_alloc = ned;
    b->maxlan_alloc = maxlan;
    return 0;
}

Params base_params(trlx_batch *b, const trlx_batch_options *o) {
    Params P;
    std::memset(&P, 0, sizeof P);  // padding too: launch configurations are compared bytewise
    P.nprob = b->nprob;
    P.ned = o->ned;
    P.maxlan = o->maxlan;
    P.lohi = o->lohi;
    P.restart = o->restart;
    P.maxmv = o->maxmv;
    P.tol = o->tol;
    P.seed = o->seed;
    P.probs = b->d_probs;
    P.order = b->d_order;
    P.diag = b->d_diag;
    P.row_ptr = b->d_rp;
    P.col = b->d_col;
    P.val = b->d_val;
    P.start = b->d_start;
    P.basis = b->d_basis;
    P.evec = b->d_evec;
    P.eval = b->d_eval;
    P.res = b->d_res;
    P.info_out = b->d_info;
    P.queue = b->d_queue;
    return P;
}

// CSR arrays (5-point Laplacian + diagonal) for the problems listed; fills
// the problems' rp/ent offsets.  Used when a stencil batch is tuned or run in
// CSR format.
int build_csr(trlx_batch *b, const std::vector<double> &hdiag) {
    std::vector<long long> rp;
    std::vector<int> col;
    std::vector<double> val;
    size_t rows = 0;
    for (int p = 0; p < b->nprob; ++p) rows += (size_t)b->L[p] * b->L[p];
    rp.reserve(rows + b->nprob);
    col.reserve(5 * rows);
    val.reserve(5 * rows);
    for (int p = 0; p < b->nprob; ++p) {
        const int L = b->L[p], n = L * L;
        Problem &pr = b->probs[p];
        pr.rp_off = (long long)rp.size();
        pr.ent_off = (long long)col.size();
        long long e = 0;
        for (int i = 0; i < n; ++i) {
            rp.push_back(e);
            const int ix = i % L, iy = i / L;
            auto put = [&](int j, double v) {
                col.push_back(j);
                val.push_back(v);
                ++e;
            };
            if (iy > 0) put(i - L, -1.0);
            if (ix > 0) put(i - 1, -1.0);
            put(i, 4.0 + hdiag[b->diag_off[p] + i]);
            if (ix < L - 1) put(i + 1, -1.0);
            if (iy < L - 1) put(i + L, -1.0);
        }
        rp.push_back(e);
    }
    int rc = upload(rp, &b->d_rp);
    if (!rc) rc = upload(col, &b->d_col);
    if (!rc) rc = upload(val, &b->d_val);
    return rc;
}

// One persistent launch: SMs x resident CTAs of P.cta threads.  The queue
// reset and the launch are one CUDA graph, captured the first time a launch
// configuration is seen and replayed while it stays the same.
int run(trlx_batch *b, Params P, int nsm) {
    int min_threads = P.cta;
    for (int f = 0; f < P.nphases; ++f) min_threads = std::min(min_threads, P.phase_threads[f]);
    // Sets the kernel's shared-memory attribute before any capture.
    const int blocks = nsm * trlb::batched::max_blocks_per_sm(min_threads, P.maxlan, P.cta);
    if (!b->stream && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return -1001;
    const bool same = b->graph && b->graph_blocks == blocks && std::memcmp(&b->graph_params, &P, sizeof P) == 0;
    if (!same) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) return -1001;
        cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned) * 4, b->stream);
        const int rc = trlb::batched::launch(P, blocks, b->stream);
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc || ce != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc ? rc : -1001;
        }
        const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            b->graph = nullptr;
            cudaGetLastError();
            return -1001;
        }
        b->graph_params = P;
        b->graph_blocks = blocks;
        b->graph_launches = 0;
    }
    if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return -1001;
    b->graph_launches++;
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? 0 : -1001;
}

}  // namespace

extern "C" {

int trlx_batch_create_stencil5(int nprob, const int *L, const double *const *diag, trlx_batch **out) {
    if (nprob <= 0 || !L || !diag || !out) return -1;
    auto *b = new trlx_batch();
    b->nprob = nprob;
    b->stencil = true;
    b->L.assign(L, L + nprob);
    std::vector<double> hdiag;
    for (int p = 0; p < nprob; ++p) {
        if (L[p] < 4) {
            delete b;
            return -1;
        }
        Problem pr{};
        pr.n = L[p] * L[p];
        pr.L = L[p];
        pr.ld = (pr.n + 31) / 32 * 32;
        pr.diag_off = (long long)hdiag.size();
        pr.start_off = -1;
        b->diag_off.push_back(pr.diag_off);
        hdiag.insert(hdiag.end(), diag[p], diag[p] + pr.n);
        b->probs.push_back(pr);
    }
    int rc = upload(hdiag, &b->d_diag);
    // CSR form of the same operators, for the autotuner's format choice.
    if (!rc) rc = build_csr(b, hdiag);
    std::vector<int> order(nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->probs[a].n > b->probs[c].n; });
    if (!rc) rc = upload(order, &b->d_order);
    if (!rc && cudaMalloc(&b->d_queue, sizeof(unsigned) * 4) != cudaSuccess) rc = -5;
    if (rc) {
        trlx_batch_destroy(b);
        return rc;
    }
    *out = b;
    return 0;
}

int trlx_batch_set_start(trlx_batch *b, const double *const *start) {
    if (!b || !start) return -1;
    std::vector<double> h;
    for (int p = 0; p < b->nprob; ++p) {
        if (start[p]) {
            b->probs[p].start_off = (long long)h.size();
            h.insert(h.end(), start[p], start[p] + b->probs[p].n);
        } else {
            b->probs[p].start_off = -1;
        }
    }
    cudaFree(b->d_start);
    b->d_start = nullptr;
    int rc = upload(h, &b->d_start);
    if (rc) return rc;
    if (b->d_probs) {
        cudaFree(b->d_probs);
        b->d_probs = nullptr;
        rc = upload(b->probs, &b->d_probs);
    }
    return rc;
}

void trlx_batch_default_options(trlx_batch_options *o) {
    if (!o) return;
    o->ned = 8;
    o->maxlan = 32;
    o->lohi = -1;
    o->restart = 1;
    o->maxmv = 100000;
    o->tol = 1e-8;
    o->seed = 0x3243F6A8885A308Dull;
    o->threads = 0;
    o->format = -1;
    o->cta_threads = 0;
}

// Whether groups of th threads fit a CTA of cta threads: a valid split
// (cta, cta / 2 or cta / 4) whose cta / th groups each get their shared
// state and dense workspace for maxlan.
static bool split_fits(int maxlan, int th, int cta) {
    if (th != cta && th != cta / 2 && th != cta / 4) return false;
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    return trlb::batched::smem_bytes(maxlan, th, cta) <= (size_t)optin;
}

int trlx_batch_autotune(trlx_batch *b, const trlx_batch_options *o, trlx_batch_config *best) {
    if (!b || !o) return -1;
    if (o->maxlan < 4 || o->maxlan > 64 || o->ned < 1 || o->ned >= o->maxlan) return -1;
    int rc = prepare(b, o->ned, o->maxlan);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int nsm = sms();
    // Problems per bucket in solve order (largest first).
    std::vector<int> order(b->nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->probs[a].n > b->probs[c].n; });
    double total = 0.0;
    // Per CTA size and bucket: the fastest split and format on the sample,
    // and that time scaled to the whole bucket.
    const int ctas[2] = {1024, 512};
    double best_t[2][3] = {{0, 0, 0}, {0, 0, 0}};
    int best_th[2][3] = {{1024, 512, 256}, {512, 256, 128}}, best_fmt[2][3] = {{0, 0, 0}, {0, 0, 0}};
    bool cta_ok[2] = {o->cta_threads == 0 || o->cta_threads == 1024, o->cta_threads == 0 || o->cta_threads == 512};
    for (int bk = 0; bk < 3; ++bk) {
        std::vector<int> members;
        for (int q : order)
            if (bucket_of(b->probs[q].n) == bk) members.push_back(q);
        if (members.empty()) continue;
        // A sample that fills the machine with the smallest groups once.
        const int want = std::min<int>((int)members.size(), nsm * 4);
        std::vector<int> sample;
        for (int k = 0; k < want; ++k) sample.push_back(members[(size_t)k * members.size() / want]);
        int *d_sample = nullptr;
        if (upload(sample, &d_sample)) return -5;
        for (int ci = 0; ci < 2; ++ci) {
            if (!cta_ok[ci]) continue;
            const int cta = ctas[ci];
            double bt = 1e30;
            for (int fmt = 0; fmt < 2; ++fmt) {
                for (int th : {cta, cta / 2, cta / 4}) {
                    if (!split_fits(o->maxlan, th, cta)) continue;
                    Params P = base_params(b, o);
                    P.order = d_sample;
                    P.format = fmt;
                    P.cta = cta;
                    P.nphases = 1;
                    P.phase_threads[0] = th;
                    P.phase_begin[0] = 0;
                    P.phase_end[0] = (int)sample.size();
                    P.maxmv = std::min(o->maxmv, 4 * o->maxlan);  // a bounded slice of the solve
                    cudaEventRecord(e0);
                    if (run(b, P, nsm)) {
                        cudaFree(d_sample);
                        return -1001;
                    }
                    cudaEventRecord(e1);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    total += ms * 1e-3;
                    if (ms < bt) {
                        bt = ms;
                        best_th[ci][bk] = th;
                        best_fmt[ci][bk] = fmt;
                    }
                }
            }
            if (bt >= 1e30) cta_ok[ci] = false;  // no split of this CTA fits
            best_t[ci][bk] = bt * (double)members.size() / (double)sample.size();
        }
        cudaFree(d_sample);
    }
    int ci = 0;
    if (cta_ok[1] && (!cta_ok[0] || best_t[1][0] + best_t[1][1] + best_t[1][2] <
                                        best_t[0][0] + best_t[0][1] + best_t[0][2]))
        ci = 1;
    b->cta = ctas[ci];
    for (int k = 0; k < 3; ++k) {
        b->bucket_threads[k] = best_th[ci][k];
        b->bucket_format[k] = best_fmt[ci][k];
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tuned = true;
    b->tuned_maxlan = o->maxlan;
    b->tune_seconds = total;
    if (best) {
        for (int k = 0; k < 3; ++k) {
            best->bucket_threads[k] = b->bucket_threads[k];
            best->bucket_format[k] = b->bucket_format[k];
        }
        best->tune_seconds = total;
        best->cta_threads = b->cta;
    }
    return 0;
}

int trlx_batch_solve(trlx_batch *b, const trlx_batch_options *o, double *eval, double *res, int *info,
                     trlx_batch_config *used) {
    if (!b || !o) return -1;
    if (o->maxlan < 4 || o->maxlan > 64 || o->ned < 1 || o->ned >= o->maxlan) return -1;
    int rc = prepare(b, o->ned, o->maxlan);
    if (rc) return rc;
    if (o->threads == 0 && (!b->tuned || b->tuned_maxlan != o->maxlan)) {
        rc = trlx_batch_autotune(b, o, nullptr);
        if (rc) return rc;
    }
    // CTA size: the caller's, else the one a forced group size implies
    // (128-thread groups exist only in 512-thread CTAs), else the tuned one.
    int cta = o->cta_threads;
    if (!cta) cta = o->threads ? (o->threads == 128 ? 512 : 1024) : b->cta;
    if (cta != 1024 && cta != 512) return -1;
    // Phases follow the buckets (largest problems first).  One format per
    // launch: the one most problems' buckets prefer.
    int cnt[3] = {0, 0, 0};
    for (auto &p : b->probs) cnt[bucket_of(p.n)]++;
    Params P = base_params(b, o);
    int fmt_votes[2] = {0, 0};
    int th_of[3] = {cta, cta, cta};
    int pos = 0;
    P.nphases = 0;
    for (int bk = 0; bk < 3; ++bk) {
        if (!cnt[bk]) continue;
        int th = o->threads ? o->threads : (cta == b->cta ? b->bucket_threads[bk] : cta);
        if (!split_fits(o->maxlan, th, cta)) return -1;
        th_of[bk] = th;
        fmt_votes[o->format >= 0 ? o->format : b->bucket_format[bk]] += cnt[bk];
        P.phase_threads[P.nphases] = th;
        P.phase_begin[P.nphases] = pos;
        P.phase_end[P.nphases] = pos + cnt[bk];
        pos += cnt[bk];
        P.nphases++;
    }
    P.cta = cta;
    P.format = o->format >= 0 ? o->format : (fmt_votes[1] > fmt_votes[0] ? 1 : 0);
    if (P.format == 0 && !b->stencil) P.format = 1;
    rc = run(b, P, sms());
    if (rc) return rc;
    if (eval) cudaMemcpy(eval, b->d_eval, sizeof(double) * (size_t)b->nprob * o->ned, cudaMemcpyDeviceToHost);
    if (res) cudaMemcpy(res, b->d_res, sizeof(double) * (size_t)b->nprob * o->ned, cudaMemcpyDeviceToHost);
    if (info) cudaMemcpy(info, b->d_info, sizeof(int) * 4 * (size_t)b->nprob, cudaMemcpyDeviceToHost);
    if (used) {
        for (int k = 0; k < 3; ++k) {
            used->bucket_threads[k] = th_of[k];
            used->bucket_format[k] = P.format;
        }
        used->tune_seconds = b->tune_seconds;
        used->cta_threads = cta;
        used->graph_replays = b->graph_launches;
    }
    return 0;
}

int trlx_batch_eigenvectors(trlx_batch *b, int prob, double *out) {
    if (!b || prob < 0 || prob >= b->nprob || !out || !b->d_evec) return -1;
    const Problem &p = b->probs[prob];
    return cudaMemcpy(out, b->d_evec + p.evec_off, sizeof(double) * (size_t)b->ned_alloc * p.n, cudaMemcpyDefault) ==
                   cudaSuccess
               ? 0
               : -1001;
}

int trlx_batch_size(const trlx_batch *b, int prob) {
    if (!b || prob < 0 || prob >= b->nprob) return -1;
    return b->probs[prob].n;
}

void trlx_batch_destroy(trlx_batch *b) {
    if (!b) return;
    cudaFree(b->d_probs);
    cudaFree(b->d_order);
    cudaFree(b->d_diag);
    cudaFree(b->d_rp);
    cudaFree(b->d_col);
    cudaFree(b->d_val);
    cudaFree(b->d_start);
    cudaFree(b->d_basis);
    cudaFree(b->d_evec);
    cudaFree(b->d_eval);
    cudaFree(b->d_res);
    cudaFree(b->d_info);
    cudaFree(b->d_queue);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
