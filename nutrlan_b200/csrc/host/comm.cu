// Host-callback and NCCL communicators, and the C API around them.
#include "comm.h"

#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "../../../include/trlx.h"

namespace trlb {
namespace {

// ---- host callback ----------------------------------------------------------
class HostComm : public Comm {
   public:
    HostComm(int nranks, int r, trlx_allreduce_fn fn, void *ctx) : fn_(fn), ctx_(ctx) {
        size = nranks;
        rank = r;
    }
    ~HostComm() override {
        if (pin_) cudaFreeHost(pin_);
    }

    int sum_device(double *d, size_t n, cudaStream_t st) override {
        if (n == 0) return 0;
        if (!grow(n)) return -1001;
        if (cudaMemcpyAsync(pin_, d, n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return -1001;
        if (fn_(pin_, (long long)n, kOpSum, ctx_) != 0) return -1010;
        if (cudaMemcpyAsync(d, pin_, n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return -1001;
        return 0;
    }
    int reduce_host(double *h, size_t n, int op) override {
        if (n == 0) return 0;
        return fn_(h, (long long)n, op, ctx_) == 0 ? 0 : -1010;
    }
    // Every (sender, receiver) pair owns a segment of one board of all
    // messages; a rank fills its own segments, the others stay zero, and one
    // sum over the ranks delivers every message (x + 0 = x exactly).
    int exchange(const double *send, const std::vector<long> &soff, double *recv, const std::vector<long> &roff,
                 const std::vector<long> &counts, cudaStream_t st) override {
        std::vector<long> bo(counts.size() + 1, 0);
        for (size_t k = 0; k < counts.size(); ++k) bo[k + 1] = bo[k] + counts[k];
        const size_t total = (size_t)bo.back();
        if (total == 0) return 0;
        if (!grow(total)) return -1001;
        std::memset(pin_, 0, total * sizeof(double));
        for (int q = 0; q < size; ++q) {
            const long c = soff[q + 1] - soff[q];
            if (c > 0 &&
                cudaMemcpyAsync(pin_ + bo[(size_t)rank * size + q], send + soff[q], c * sizeof(double),
                                cudaMemcpyDeviceToHost, st) != cudaSuccess)
                return -1001;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) return -1001;
        if (fn_(pin_, (long long)total, kOpSum, ctx_) != 0) return -1010;
        for (int p = 0; p < size; ++p) {
            const long c = roff[p + 1] - roff[p];
            if (c > 0 &&
                cudaMemcpyAsync(recv + roff[p], pin_ + bo[(size_t)p * size + rank], c * sizeof(double),
                                cudaMemcpyHostToDevice, st) != cudaSuccess)
                return -1001;
        }
        return cudaStreamSynchronize(st) == cudaSuccess ? 0 : -1001;
    }

   private:
    bool grow(size_t n) {
        if (n <= cap_) return true;
        if (pin_) cudaFreeHost(pin_);
        pin_ = nullptr;
        cap_ = 0;
        if (cudaMallocHost(&pin_, n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            pin_ = nullptr;
            return false;
        }
        cap_ = n;
        return true;
    }
    trlx_allreduce_fn fn_;
    void *ctx_;
    double *pin_ = nullptr;
    size_t cap_ = 0;
};

// ---- NCCL, resolved at run time ------------------------------------------------
struct NcclApi {
    decltype(&ncclGetUniqueId) get_unique_id = nullptr;
    decltype(&ncclCommInitRank) init_rank = nullptr;
    decltype(&ncclCommDestroy) destroy = nullptr;
    decltype(&ncclAllReduce) all_reduce = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclGroupStart) group_start = nullptr;
    decltype(&ncclGroupEnd) group_end = nullptr;
    decltype(&ncclGetErrorString) error_string = nullptr;
    bool ok = false;
};

const NcclApi &nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *names[] = {std::getenv("TRLX_NCCL_LIB"), "libnccl.so.2", "libnccl.so"};
        void *h = nullptr;
        for (const char *nm : names)
            if (nm && (h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return;
        auto sym = [&](auto &f, const char *name) {
            f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(h, name));
            return f != nullptr;
        };
        api.ok = sym(api.get_unique_id, "ncclGetUniqueId") && sym(api.init_rank, "ncclCommInitRank") &&
                 sym(api.destroy, "ncclCommDestroy") && sym(api.all_reduce, "ncclAllReduce") &&
                 sym(api.send, "ncclSend") && sym(api.recv, "ncclRecv") &&
                 sym(api.group_start, "ncclGroupStart") && sym(api.group_end, "ncclGroupEnd") &&
                 sym(api.error_string, "ncclGetErrorString");
    });
    return api;
}

int nccl_check(ncclResult_t r, const char *what) {
    if (r == ncclSuccess) return 0;
    std::fprintf(stderr, "TRLAN-B200: %s failed: %s\n", what, nccl().error_string(r));
    return -1010;
}

class NcclComm : public Comm {
   public:
    NcclComm(int nranks, int r, ncclComm_t c) : comm_(c) {
        size = nranks;
        rank = r;
    }
    ~NcclComm() override {
        if (tmp_) cudaFree(tmp_);
        if (comm_) nccl().destroy(comm_);
    }
    int sum_device(double *d, size_t n, cudaStream_t st) override {
        if (n == 0) return 0;
        return nccl_check(nccl().all_reduce(d, d, n, ncclDouble, ncclSum, comm_, st), "ncclAllReduce");
    }
    int reduce_host(double *h, size_t n, int op) override {
        if (n == 0) return 0;
        if (n > cap_) {
            if (tmp_) cudaFree(tmp_);
            tmp_ = nullptr;
            cap_ = 0;
            if (cudaMalloc(&tmp_, n * sizeof(double)) != cudaSuccess) return -1001;
            cap_ = n;
        }
        const ncclRedOp_t o = op == kOpMax ? ncclMax : (op == kOpMin ? ncclMin : ncclSum);
        if (cudaMemcpy(tmp_, h, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return -1001;
        if (int e = nccl_check(nccl().all_reduce(tmp_, tmp_, n, ncclDouble, o, comm_, 0), "ncclAllReduce"))
            return e;
        return cudaMemcpy(h, tmp_, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1001;
    }
    int exchange(const double *send, const std::vector<long> &soff, double *recv, const std::vector<long> &roff,
                 const std::vector<long> &, cudaStream_t st) override {
        if (int e = nccl_check(nccl().group_start(), "ncclGroupStart")) return e;
        int err = 0;
        for (int p = 0; p < size && !err; ++p) {
            if (p == rank) continue;
            const long sc = soff[p + 1] - soff[p], rc = roff[p + 1] - roff[p];
            if (sc > 0) err = nccl_check(nccl().send(send + soff[p], sc, ncclDouble, p, comm_, st), "ncclSend");
            if (!err && rc > 0)
                err = nccl_check(nccl().recv(recv + roff[p], rc, ncclDouble, p, comm_, st), "ncclRecv");
        }
        const int e2 = nccl_check(nccl().group_end(), "ncclGroupEnd");
        return err ? err : e2;
    }

   private:
    ncclComm_t comm_;
    double *tmp_ = nullptr;
    size_t cap_ = 0;
};

}  // namespace
}  // namespace trlb

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
extern "C" int trlx_comm_create_host(int nranks, int rank, trlx_allreduce_fn fn, void *ctx, trlx_comm **out) {
    if (!out || !fn || nranks < 1 || rank < 0 || rank >= nranks) return -1;
    *out = new trlx_comm{new trlb::HostComm(nranks, rank, fn, ctx)};
    return 0;
}

extern "C" int trlx_comm_nccl_id(unsigned char id[128]) {
    static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id is 128 bytes");
    if (!id) return -1;
    const auto &api = trlb::nccl();
    if (!api.ok) return -1011;
    ncclUniqueId u;
    if (int e = trlb::nccl_check(api.get_unique_id(&u), "ncclGetUniqueId")) return e;
    std::memcpy(id, u.internal, sizeof(u.internal));
    return 0;
}

extern "C" int trlx_comm_create_nccl(int nranks, int rank, const unsigned char id[128], trlx_comm **out) {
    if (!out || !id || nranks < 1 || rank < 0 || rank >= nranks) return -1;
    const auto &api = trlb::nccl();
    if (!api.ok) return -1011;
    ncclUniqueId u;
    std::memcpy(u.internal, id, sizeof(u.internal));
    ncclComm_t c = nullptr;
    if (int e = trlb::nccl_check(api.init_rank(&c, nranks, u, rank), "ncclCommInitRank")) return e;
    *out = new trlx_comm{new trlb::NcclComm(nranks, rank, c)};
    return 0;
}

extern "C" int trlx_comm_rank(const trlx_comm *c) { return c && c->impl ? c->impl->rank : -1; }
extern "C" int trlx_comm_size(const trlx_comm *c) { return c && c->impl ? c->impl->size : -1; }

extern "C" int trlx_comm_allreduce(trlx_comm *c, double *buf, long long count, int op) {
    if (!c || !c->impl || (count > 0 && !buf) || count < 0 || op < TRLX_SUM || op > TRLX_MIN) return -1;
    return c->impl->reduce_host(buf, (size_t)count, op);
}

extern "C" void trlx_comm_destroy(trlx_comm *c) {
    if (!c) return;
    delete c->impl;
    delete c;
}

extern "C" int trlx_init_info_comm(trl_info *info, trlx_comm *comm, int nloc, int mxlan, int lohi, int ned,
                                   double tol, int restart, int maxmv) {
    if (!info || !comm || !comm->impl || nloc < 0) return -1;
    trl_init_info(info, nloc, mxlan, lohi, ned, tol, restart, maxmv, NULL);
    double tot = (double)nloc;
    if (int e = comm->impl->reduce_host(&tot, 1, trlb::kOpSum)) return e;
    info->ntot = (int)tot;
    if (maxmv <= 0) info->maxmv = std::min(std::max(info->ntot, 1000), 1000 * ned);
    info->my_pe = comm->impl->rank;
    info->npes = comm->impl->size;
    info->mpicomp = comm;
    return 0;
}
