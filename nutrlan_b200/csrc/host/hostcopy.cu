// Pipelined host <-> device copies through pinned staging buffers.
//
// The copy is cut into chunks of at most kChunk bytes (whole rows when a
// row fits, else pieces of one row).  Host-to-device: the copy threads fill
// staging buffer c % kRing from the user's memory, the DMA of that buffer is
// queued, and the threads move on to the next buffer while the link works.
// Device-to-host: kRing DMAs are queued up front; as each lands, the threads
// drain its buffer into the user's memory and the buffer's next DMA is
// queued.  A per-buffer event says when a buffer may be refilled or read.
#include "hostcopy.h"

#include <sched.h>

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace trlb {
namespace {

constexpr size_t kChunk = size_t(16) << 20;  // bytes per staging buffer
constexpr int kRing = 4;                     // staging buffers
constexpr size_t kDirect = size_t(4) << 20;  // smaller copies go straight to the driver

// `rows` rows of `len` bytes between two pitched regions, addressed as one
// flat range of rows*len bytes.
struct Block {
    char *dst;
    size_t dp;
    const char *src;
    size_t sp;
    size_t len;
};

void copy_range(const Block &B, size_t a, size_t b) {
    while (a < b) {
        const size_t r = a / B.len, o = a - r * B.len;
        const size_t n = std::min(B.len - o, b - a);
        std::memcpy(B.dst + r * B.dp + o, B.src + r * B.sp + o, n);
        a += n;
    }
}

int copy_threads() {
    if (const char *s = std::getenv("TRLX_COPY_THREADS")) {
        const int v = std::atoi(s);
        if (v >= 1 && v <= 64) return v;
    }
    cpu_set_t set;
    int ncpu = 0;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) ncpu = CPU_COUNT(&set);
    if (ncpu <= 0) ncpu = (int)std::thread::hardware_concurrency();
    // Draining pinned buffers into pageable memory while the link fills the
    // next ones takes about 12 threads to keep up with 55 GB/s on a 16-core
    // host (8 threads: 38 GB/s, 4: 26 GB/s); a quarter of the cores is left
    // to the rest of the process.
    return std::max(1, std::min(12, ncpu - ncpu / 4));
}

// A fixed team of threads that split one Block copy between them; the
// calling thread takes part 0 and returns when every part is done.
class Team {
  public:
    explicit Team(int n) : n_(n) {
        for (int i = 1; i < n; ++i) th_.emplace_back([this, i] { loop(i); });
    }
    ~Team() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void run(const Block &B, size_t total) {
        if (n_ == 1 || total < (size_t(1) << 20)) {
            copy_range(B, 0, total);
            return;
        }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = B;
            total_ = total;
            left_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        part(0);
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return left_ == 0; });
    }

  private:
    void part(int i) {
        const size_t per = ((total_ + n_ - 1) / n_ + 63) / 64 * 64;
        const size_t a = std::min(total_, per * i), b = std::min(total_, a + per);
        copy_range(job_, a, b);
    }
    void loop(int i) {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            part(i);
            std::lock_guard<std::mutex> g(m_);
            if (--left_ == 0) done_.notify_one();
        }
    }
    const int n_;
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    Block job_{};
    size_t total_ = 0;
    int left_ = 0;
    unsigned long gen_ = 0;
    bool stop_ = false;
};

// One staged copy at a time per process (the link is shared anyway).
struct Stager {
    std::mutex m;
    char *buf = nullptr;
    Team *team = nullptr;
    bool ensure() {
        if (!buf) {
            if (cudaHostAlloc(reinterpret_cast<void **>(&buf), kChunk * kRing, cudaHostAllocPortable) !=
                cudaSuccess) {
                cudaGetLastError();
                buf = nullptr;
                return false;
            }
        }
        if (!team) team = new Team(copy_threads());
        return true;
    }
    void release() {
        if (buf) cudaFreeHost(buf);
        buf = nullptr;
        delete team;
        team = nullptr;
    }
};

// Never destroyed: freeing pinned memory or joining threads during static
// destruction at process exit would race with the CUDA runtime's teardown.
Stager &stager() {
    static Stager *s = new Stager;
    return *s;
}

bool pageable(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

cudaError_t dma(char *dev, size_t dp, char *pin, size_t nr, size_t len, bool h2d, cudaStream_t st) {
    if (nr == 1)
        return h2d ? cudaMemcpyAsync(dev, pin, len, cudaMemcpyHostToDevice, st)
                   : cudaMemcpyAsync(pin, dev, len, cudaMemcpyDeviceToHost, st);
    return h2d ? cudaMemcpy2DAsync(dev, dp, pin, len, len, nr, cudaMemcpyHostToDevice, st)
               : cudaMemcpy2DAsync(pin, len, dev, dp, len, nr, cudaMemcpyDeviceToHost, st);
}

}  // namespace

cudaError_t host_copy_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows,
                         cudaMemcpyKind kind, cudaStream_t st) {
    if (width == 0 || rows == 0) return cudaSuccess;
    const bool h2d = kind == cudaMemcpyHostToDevice;
    if (!h2d && kind != cudaMemcpyDeviceToHost) return cudaErrorInvalidMemcpyDirection;
    const void *host = h2d ? src : dst;
    Stager &S = stager();
    std::unique_lock<std::mutex> lock(S.m, std::defer_lock);
    bool staged = width * rows >= kDirect && pageable(host);
    if (staged) {
        lock.lock();
        staged = S.ensure();
    }
    if (!staged) {
        cudaError_t e = rows == 1 ? cudaMemcpyAsync(dst, src, width, kind, st)
                                  : cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    }

    char *dev = static_cast<char *>(h2d ? dst : const_cast<void *>(src));
    const size_t devp = h2d ? dpitch : spitch;
    char *hst = static_cast<char *>(h2d ? const_cast<void *>(src) : dst);
    const size_t hp = h2d ? spitch : dpitch;
    const bool whole = width <= kChunk;
    const size_t rpc = whole ? kChunk / width : 1;                   // rows per chunk
    const size_t cpr = whole ? 1 : (width + kChunk - 1) / kChunk;    // chunks per row
    const size_t nchunks = whole ? (rows + rpc - 1) / rpc : rows * cpr;
    struct Piece {
        size_t r0, nr, off, len;
    };
    auto piece = [&](size_t c) -> Piece {
        if (whole) {
            const size_t r0 = c * rpc;
            return {r0, std::min(rpc, rows - r0), 0, width};
        }
        const size_t off = (c % cpr) * kChunk;
        return {c / cpr, 1, off, std::min(kChunk, width - off)};
    };
    auto pin = [&](size_t c) { return S.buf + (c % kRing) * kChunk; };

    cudaEvent_t ev[kRing] = {};
    cudaError_t err = cudaSuccess;
    int nev = 0;
    for (; nev < kRing && err == cudaSuccess; ++nev) err = cudaEventCreateWithFlags(&ev[nev], cudaEventDisableTiming);
    if (err != cudaSuccess) --nev;
    std::vector<bool> queued(kRing, false);
    auto enqueue = [&](size_t c) {
        const Piece p = piece(c);
        const int k = (int)(c % kRing);
        cudaError_t e = dma(dev + p.r0 * devp + p.off, devp, pin(c), p.nr, p.len, h2d, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], st);
        queued[k] = e == cudaSuccess;
        return e;
    };
    if (err == cudaSuccess && h2d) {
        for (size_t c = 0; c < nchunks && err == cudaSuccess; ++c) {
            const int k = (int)(c % kRing);
            if (queued[k]) err = cudaEventSynchronize(ev[k]);
            if (err != cudaSuccess) break;
            const Piece p = piece(c);
            S.team->run(Block{pin(c), p.len, hst + p.r0 * hp + p.off, hp, p.len}, p.nr * p.len);
            err = enqueue(c);
        }
    } else if (err == cudaSuccess) {
        for (size_t c = 0; c < nchunks && c < (size_t)kRing && err == cudaSuccess; ++c) err = enqueue(c);
        for (size_t c = 0; c < nchunks && err == cudaSuccess; ++c) {
            const int k = (int)(c % kRing);
            err = cudaEventSynchronize(ev[k]);
            queued[k] = false;
            if (err != cudaSuccess) break;
            const Piece p = piece(c);
            S.team->run(Block{hst + p.r0 * hp + p.off, hp, pin(c), p.len, p.len}, p.nr * p.len);
            if (c + kRing < nchunks) err = enqueue(c + kRing);
        }
    }
    // Every queued DMA has finished before the buffers are handed to the
    // next copy (also on the error path).
    for (int k = 0; k < nev; ++k) {
        if (queued[k]) {
            cudaError_t e = cudaEventSynchronize(ev[k]);
            if (err == cudaSuccess) err = e;
        }
        cudaEventDestroy(ev[k]);
    }
    return err;
}

void release_staging() {
    Stager &S = stager();
    std::lock_guard<std::mutex> g(S.m);
    S.release();
}

}  // namespace trlb
