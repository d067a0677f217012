// sbf_server.cu -- request server over a resident filter: continuous
// batching of insert and query requests.  No reference counterpart (the
// reference is a library with one caller per filter).
//
// Requests (a buffer of records: reads to query or sequences to insert) are
// queued in arrival order.  A worker thread forms each batch from the
// longest run of queued requests of the same operation that fits the batch
// cap, admits it when the device staging ring (the memory budget) has room
// and fewer than max_inflight batches are on the GPU, and launches it as one
// ragged pass over all its records: copies on an upload stream, the kernel
// on a compute stream, query results on a download stream, so the copies of
// one batch overlap the kernels of the batches around it.  A batch's ranges
// are uploaded as the clients gave them, in one copy, and rebased by a small
// kernel.  Batches run their kernels in arrival order on one stream,
// so every query sees exactly the inserts that arrived before it: results
// equal one-request-at-a-time execution.  A completion thread waits for
// each batch's last event in launch order, stamps its requests, frees their
// ring space and wakes waiters.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_expand.h"
#include "sbf_host.h"
#include "sbf_internal.h"
#include "sbf_ragged.h"

using namespace sbf;

namespace sbf {

bool is_pinned(const void* p);

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

constexpr uint64_t kAlign = 256;
constexpr uint64_t kDirectBytes = 256 << 10;  // pinned spans at least this size skip the gather

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Operations: 0 insert, 1 query (one byte per window), 2 query with
// bit-packed results, 3 query returning per-record counts only (two uint64
// per record: valid windows, positive windows; computed in the query
// kernel's epilogue, no hit bytes written).  Bit-packed requests start at
// multiples of 32 bytes of the batch, so each request's bits start on a word
// boundary.
constexpr int kOpInsert = 0, kOpQuery = 1, kOpQueryBits = 2, kOpQueryCounts = 3;
// Flag on any operation: the request body is 2-bit dense-packed DNA (32
// symbols per little-endian uint64, the reference's dense format,
// dense_packed.hpp:36-50) and its ranges count symbols.  The batch is
// unpacked to bytes on the GPU, so a quarter of the bytes cross PCIe.
constexpr int kOpDense = 0x10;
int base_op(int op) { return op & 0xF; }
bool is_dense(int op) { return (op & kOpDense) != 0; }
uint64_t result_bytes(int op, uint64_t windows, uint64_t records) {
    op = base_op(op);
    return op == kOpQueryBits     ? (windows + 31) / 32 * 4
           : op == kOpQuery       ? windows
           : op == kOpQueryCounts ? records * 16
                                  : 0;
}
// Device bytes of a batch's result region.
uint64_t out_region(int op, uint64_t seq_bytes, uint64_t records) {
    op = base_op(op);
    return op == kOpInsert ? 0 : align_up(op == kOpQueryCounts ? records * 16 : seq_bytes, kAlign);
}
// Packed words holding symbols [lo, hi).
uint64_t dense_words(uint64_t lo, uint64_t hi) { return hi > lo ? (hi + 31) / 32 - lo / 32 : 0; }

// FIFO ring allocator: regions are released in allocation order.  The
// live regions occupy [tail, head) when head > tail and wrap around the end
// of the ring otherwise; a region never straddles the end.
struct Ring {
    uint64_t cap = 0, head = 0;
    std::deque<std::pair<uint64_t, uint64_t>> live;  // (offset, bytes), oldest first
    bool alloc(uint64_t bytes, uint64_t* off) {
        if (bytes == 0) bytes = 1;
        if (bytes > cap) return false;
        if (live.empty()) {
            *off = 0;
        } else {
            const uint64_t tail = live.front().first;
            if (head > tail) {
                if (cap - head >= bytes)
                    *off = head;
                else if (tail >= bytes)
                    *off = 0;
                else
                    return false;
            } else if (head < tail) {
                if (tail - head < bytes) return false;
                *off = head;
            } else {
                return false;  // head == tail with live regions: full
            }
        }
        live.emplace_back(*off, bytes);
        head = *off + bytes;
        return true;
    }
    // Undoes the newest allocation (head restored to `old_head`).
    void undo_back(uint64_t old_head) {
        live.pop_back();
        head = old_head;
    }
    void release_front() { live.pop_front(); }
};

}  // namespace

struct SrvRequest {
    uint64_t ticket = 0;
    int op = 0;  // 0 insert, 1 query
    const uint8_t* base = nullptr;
    const DevRange* ranges = nullptr;  // host, offsets relative to base
    uint64_t n = 0;
    uint64_t lo = 0, hi = 0;  // byte span [lo, hi) of base
    uint8_t* out = nullptr;
    bool pinned = false;  // sequence span is in pinned memory
    double t_arrival = 0, t_done = 0;
    uint64_t windows = 0;
    int status = SBF_OK;
    bool done = false;
};

struct SrvBatch {
    int op = 0;
    std::vector<SrvRequest*> reqs;
    std::vector<uint64_t> req_off;  // each request's first byte in the batch
    std::vector<uint64_t> req_rec;  // each request's first record in the batch
    uint64_t seq_bytes = 0, n_ranges = 0;
    uint64_t packed_bytes = 0;  // dense batches: staged packed words
    uint64_t dev_off = 0, dev_bytes = 0, pin_off = 0, pin_bytes = 0;
    // Byte-result queries expanded on the host: the downloaded bits, the
    // last res_bytes of the batch's pinned region.
    uint64_t res_bytes = 0;
    bool complete = false;
    int status = SBF_OK;
    cudaEvent_t ev_up = nullptr, ev_comp = nullptr, ev_done = nullptr;
};

// In-place rebase of a batch's ranges, copied as the client gave them:
// ranges [dst, dst + n) (one request's) get `delta` added to their offsets.
struct FixEntry {
    uint64_t dst, n;
    int64_t delta;
};

// Dense batches: request e's symbols [sym0, sym0 + n_sym) of the packed
// words starting at word src_word are written as bytes at dst.  The batch's
// work is cut into segments of kUnpackSeg symbols; entry e's segments are
// the global segments [seg0, seg0 + ceil(n_sym / kUnpackSeg)).
constexpr uint64_t kUnpackSeg = 8192;
struct UnpackEntry {
    uint64_t src_word, sym0, n_sym, dst, seg0;
};

// A-C-T-G for codes 0-3 (DnaAlphabet, Alphabet.cuh:132-141).  CTAs take the
// batch's segments grid-strided, so many small requests and a few large
// ones spread over the grid alike.
__global__ void unpack_dense_kernel(const uint64_t* packed, const UnpackEntry* tab,
                                    uint32_t n_tab, uint64_t n_segs, uint8_t* seq) {
    for (uint64_t g = blockIdx.x; g < n_segs; g += gridDim.x) {
        // The entry holding segment g (last entry with seg0 <= g).
        uint32_t lo = 0, hi = n_tab;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (tab[mid].seg0 <= g)
                lo = mid;
            else
                hi = mid;
        }
        const UnpackEntry u = tab[lo];
        const uint64_t t0 = (g - u.seg0) * kUnpackSeg;
        const uint64_t t1 = t0 + kUnpackSeg < u.n_sym ? t0 + kUnpackSeg : u.n_sym;
        for (uint64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
            const uint64_t sym = u.sym0 + t;
            const uint32_t code =
                static_cast<uint32_t>(packed[u.src_word + sym / 32] >> (2 * (sym % 32))) & 3u;
            seq[u.dst + t] = static_cast<uint8_t>(0x47544341u >> (8 * code));
        }
    }
}

__global__ void rebase_ranges_kernel(DevRange* rng, const FixEntry* tab, uint32_t n_tab) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t e = warp; e < n_tab; e += warps) {
        const FixEntry t = tab[e];
        for (uint64_t j = lane; j < t.n; j += 32)
            rng[t.dst + j].offset =
                static_cast<uint64_t>(static_cast<int64_t>(rng[t.dst + j].offset) + t.delta);
    }
}

struct Server {
    sbf_filter* f = nullptr;
    sbf_server_config cfg{};
    // Byte-result queries (op 1) download one bit per window and the
    // completion thread expands them into the requests' buffers with this
    // pool (null: bytes are downloaded).
    std::unique_ptr<ExpandPool> pool;
    bool expands(int op) const { return pool != nullptr && base_op(op) == kOpQuery; }
    // Requests start on 32-byte boundaries of the batch where results are
    // bit-packed (so each request's bits start on a word), else 16.
    uint64_t pad(int op) const { return base_op(op) == kOpQueryBits || expands(op) ? 32 : 16; }
    uint8_t* pinned_results(const SrvBatch* b) const {
        return h_ring + b->pin_off + b->pin_bytes - b->res_bytes;
    }
    cudaStream_t up = nullptr, comp = nullptr, down = nullptr;
    uint8_t* d_ring = nullptr;
    uint8_t* h_ring = nullptr;
    unsigned int* d_ctl = nullptr;  // [0] work-queue counter, [2..9] counts
    Ring dring, hring;
    RaggedGraph graph[2];

    std::mutex mu;
    std::condition_variable cv;
    std::deque<SrvRequest*> pending;
    std::deque<SrvBatch*> inflight;   // admitted, in order (ring release order)
    std::deque<SrvBatch*> launched;   // launched, awaiting completion, in order
    std::vector<cudaEvent_t> events;  // free events
    std::unordered_map<uint64_t, std::unique_ptr<SrvRequest>> reqs;
    uint64_t next_ticket = 1;
    uint32_t inflight_batches = 0;
    bool stop = false;
    int fatal = SBF_OK;
    std::string fatal_msg;
    std::thread worker, completer;

    // Statistics since the last reset.
    std::vector<double> latencies;
    uint64_t n_batches = 0, n_batched_reqs = 0, q_windows = 0, i_windows = 0, n_reqs = 0;
    double t_first = 0, t_last = 0;
    double busy_s = 0, admit_wait_s = 0, slot_wait_s = 0;

    void run();
    void finish();
    int launch(SrvBatch* b);
    void complete(SrvBatch* b, int status);
};

void Server::complete(SrvBatch* b, int status) {
    std::lock_guard<std::mutex> lk(mu);
    const double t = now_s();
    for (SrvRequest* r : b->reqs) {
        r->t_done = t;
        r->status = status;
        r->done = true;
        latencies.push_back(t - r->t_arrival);
        (base_op(r->op) != kOpInsert ? q_windows : i_windows) += r->windows;
        ++n_reqs;
        if (t_first == 0 || r->t_arrival < t_first) t_first = r->t_arrival;
        t_last = std::max(t_last, t);
    }
    ++n_batches;
    n_batched_reqs += b->reqs.size();
    b->complete = true;
    for (cudaEvent_t ev : {b->ev_up, b->ev_comp, b->ev_done})
        if (ev) events.push_back(ev);
    b->ev_up = b->ev_comp = b->ev_done = nullptr;
    --inflight_batches;
    // Ring space is released in batch order.
    while (!inflight.empty() && inflight.front()->complete) {
        SrvBatch* x = inflight.front();
        inflight.pop_front();
        dring.release_front();
        hring.release_front();
        delete x;
    }
    cv.notify_all();
}

// Completion thread: waits for each launched batch's last event in launch
// order and completes it; no stream ever waits on host work.
void Server::finish() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv.wait(lk, [&] {
            return !launched.empty() || (stop && pending.empty() && inflight_batches == 0);
        });
        if (launched.empty()) break;
        SrvBatch* b = launched.front();
        launched.pop_front();
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(b->ev_done);
        if (e != cudaSuccess) {
            b->status = cuda_fail(e, "cudaEventSynchronize(batch)");
            std::lock_guard<std::mutex> g(mu);
            if (fatal == SBF_OK) {
                fatal = b->status;
                fatal_msg = sbf_last_error_message();
            }
        } else if (b->status == SBF_OK && expands(b->op)) {
            // Downloaded bits -> each request's result bytes.
            std::vector<ExpandItem> items;
            items.reserve(b->reqs.size());
            for (size_t i = 0; i < b->reqs.size(); ++i) {
                SrvRequest* r = b->reqs[i];
                if (r->windows)
                    items.push_back(ExpandItem{
                        reinterpret_cast<const uint32_t*>(pinned_results(b) + b->req_off[i] / 8),
                        static_cast<uint8_t*>(r->out), r->windows});
            }
            pool->run_items(items.data(), items.size());
        }
        complete(b, b->status);
        lk.lock();
    }
}

void Server::run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        const double w0 = now_s();
        const bool had_work = !pending.empty();
        cv.wait(lk, [&] {
            return (stop && pending.empty()) ||
                   (!pending.empty() && inflight_batches < cfg.max_inflight);
        });
        if (had_work) slot_wait_s += now_s() - w0;
        if (pending.empty()) {
            if (stop) break;
            continue;
        }
        // The longest same-operation run of queued requests within the caps.
        auto* b = new SrvBatch();
        b->op = pending.front()->op;
        const bool dense = is_dense(b->op);
        uint64_t seq = 0, nr = 0, gather = 0, packed = 0;
        size_t take = 0;
        for (SrvRequest* r : pending) {
            if (r->op != b->op) break;
            if (cfg.max_batch_requests && take >= cfg.max_batch_requests) break;
            const uint64_t span = align_up(r->hi - r->lo, pad(r->op));
            if (take > 0 && (seq + span > cfg.max_batch_bytes ||
                             (nr + r->n) * sizeof(DevRange) > cfg.max_batch_bytes))
                break;
            seq += span;
            nr += r->n;
            // Bytes staged for the request: its span, or its packed words.
            const uint64_t staged = dense ? dense_words(r->lo, r->hi) * 8 : span;
            packed += dense ? staged : 0;
            if (!(r->pinned && staged >= kDirectBytes)) gather += staged;
            ++take;
        }
        const uint64_t n_tiles = seq / kTileKmers + 2;
        const uint64_t unpack_tab = dense ? align_up(take * sizeof(UnpackEntry), kAlign) : 0;
        const uint64_t dev_bytes = align_up(seq, kAlign) + out_region(b->op, seq, nr) +
                                   align_up(nr * sizeof(DevRange), kAlign) +
                                   align_up(n_tiles * 4, kAlign) +
                                   align_up(take * sizeof(FixEntry), kAlign) +
                                   (dense ? align_up(packed, kAlign) : 0) + unpack_tab;
        const uint64_t res_bytes = expands(b->op) ? align_up(seq / 8 + 64, kAlign) : 0;
        const uint64_t pin_bytes = align_up(nr * sizeof(DevRange), kAlign) +
                                   align_up(take * sizeof(FixEntry), kAlign) + unpack_tab +
                                   align_up(gather, kAlign) + res_bytes;
        // Admission: wait for ring space (completions free it).
        for (;;) {
            uint64_t doff = 0, poff = 0;
            const uint64_t old_head = dring.head;
            if (dring.alloc(dev_bytes, &doff)) {
                if (hring.alloc(pin_bytes, &poff)) {
                    b->dev_off = doff;
                    b->pin_off = poff;
                    break;
                }
                dring.undo_back(old_head);
            }
            if (inflight_batches == 0) {
                // Cannot happen for admitted sizes; fail the requests.
                fatal = SBF_ERR_RESOURCE;
                fatal_msg = "batch does not fit the server's staging";
                break;
            }
            const double a0 = now_s();
            cv.wait(lk);
            admit_wait_s += now_s() - a0;
        }
        if (fatal != SBF_OK) {
            for (size_t i = 0; i < take; ++i) {
                pending.front()->status = fatal;
                pending.front()->done = true;
                pending.pop_front();
            }
            delete b;
            cv.notify_all();
            continue;
        }
        b->dev_bytes = dev_bytes;
        b->pin_bytes = pin_bytes;
        b->res_bytes = res_bytes;
        b->seq_bytes = seq;
        b->n_ranges = nr;
        b->packed_bytes = packed;
        for (size_t i = 0; i < take; ++i) {
            b->reqs.push_back(pending.front());
            pending.pop_front();
        }
        inflight.push_back(b);
        ++inflight_batches;
        for (cudaEvent_t* ev : {&b->ev_up, &b->ev_comp, &b->ev_done}) {
            *ev = events.back();
            events.pop_back();
        }
        lk.unlock();
        const double l0 = now_s();
        const int s = launch(b);
        const double l1 = now_s();
        if (s != SBF_OK) {
            {
                std::lock_guard<std::mutex> g(mu);
                if (fatal == SBF_OK) {
                    fatal = s;
                    fatal_msg = sbf_last_error_message();
                }
            }
            // Nothing of this batch may still be queued on the streams that
            // read its ring space: wait for them before releasing it.
            cudaStreamSynchronize(up);
            cudaStreamSynchronize(comp);
            cudaStreamSynchronize(down);
            complete(b, s);
            lk.lock();
        } else {
            lk.lock();
            launched.push_back(b);
            cv.notify_all();
        }
        busy_s += l1 - l0;
    }
}

int Server::launch(SrvBatch* b) {
    const bool query = base_op(b->op) != kOpInsert;
    const bool expand = expands(b->op);
    const bool bits = base_op(b->op) == kOpQueryBits || expand;
    const bool tally = base_op(b->op) == kOpQueryCounts;
    uint8_t* dbase = d_ring + b->dev_off;
    uint8_t* d_seq = dbase;
    uint8_t* d_out = query ? dbase + align_up(b->seq_bytes, kAlign) : nullptr;
    auto* d_rng = reinterpret_cast<DevRange*>(dbase + align_up(b->seq_bytes, kAlign) +
                                              out_region(b->op, b->seq_bytes, b->n_ranges));
    auto* d_tile = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(d_rng) +
                                               align_up(b->n_ranges * sizeof(DevRange), kAlign));
    auto* d_fix = reinterpret_cast<FixEntry*>(
        reinterpret_cast<uint8_t*>(d_tile) + align_up((b->seq_bytes / kTileKmers + 2) * 4, kAlign));
    const bool dense = is_dense(b->op);
    const uint64_t unpack_tab = dense ? align_up(b->reqs.size() * sizeof(UnpackEntry), kAlign) : 0;
    uint8_t* d_packed =
        reinterpret_cast<uint8_t*>(d_fix) + align_up(b->reqs.size() * sizeof(FixEntry), kAlign);
    auto* d_unpack =
        reinterpret_cast<UnpackEntry*>(d_packed + (dense ? align_up(b->packed_bytes, kAlign) : 0));
    auto* h_rng = reinterpret_cast<DevRange*>(h_ring + b->pin_off);
    auto* h_fix = reinterpret_cast<FixEntry*>(h_ring + b->pin_off +
                                              align_up(b->n_ranges * sizeof(DevRange), kAlign));
    auto* h_unpack = reinterpret_cast<UnpackEntry*>(
        reinterpret_cast<uint8_t*>(h_fix) + align_up(b->reqs.size() * sizeof(FixEntry), kAlign));
    uint8_t* h_gather = reinterpret_cast<uint8_t*>(h_unpack) + unpack_tab;
    uint64_t o = 0, k = 0, g = 0, pw = 0, n_segs = 0;
    uint32_t n_fix = 0, n_unpack = 0;
    // Consecutive gathered requests are one copy (into the sequence region,
    // or into the packed-word region for dense batches).
    uint8_t* run_base = dense ? d_packed : d_seq;
    uint64_t run_dev = 0, run_pin = 0, run_bytes = 0;
    auto flush_run = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        if (run_bytes)
            e = cudaMemcpyAsync(run_base + run_dev, h_gather + run_pin, run_bytes,
                                cudaMemcpyHostToDevice, up);
        run_bytes = 0;
        return e;
    };
    cudaError_t e;
    b->req_off.resize(b->reqs.size());
    b->req_rec.resize(b->reqs.size());
    for (size_t i = 0; i < b->reqs.size(); ++i) {
        SrvRequest* r = b->reqs[i];
        const uint64_t span = r->hi - r->lo;
        const uint64_t padded = align_up(span, pad(r->op));
        b->req_off[i] = o;
        b->req_rec[i] = k;
        if (r->n) {
            // One bulk copy of the client's ranges; offsets are rebased on the GPU.
            std::memcpy(h_rng + k, r->ranges, r->n * sizeof(DevRange));
            h_fix[n_fix++] =
                FixEntry{k, r->n, static_cast<int64_t>(o) - static_cast<int64_t>(r->lo)};
            k += r->n;
        }
        if (dense) {
            // Packed words of symbols [lo, hi), unpacked to d_seq + o.
            const uint64_t nw = dense_words(r->lo, r->hi);
            const uint8_t* src = r->base + (r->lo / 32) * 8;
            if (nw) {
                h_unpack[n_unpack++] = UnpackEntry{pw, r->lo % 32, span, o, n_segs};
                n_segs += (span + kUnpackSeg - 1) / kUnpackSeg;
                if (r->pinned && nw * 8 >= kDirectBytes) {
                    e = flush_run();
                    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(batch)");
                    e = cudaMemcpyAsync(d_packed + pw * 8, src, nw * 8, cudaMemcpyHostToDevice, up);
                    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(request)");
                } else {
                    std::memcpy(h_gather + g, src, nw * 8);
                    if (run_bytes == 0) {
                        run_dev = pw * 8;
                        run_pin = g;
                    }
                    run_bytes = (g + nw * 8) - run_pin;
                    g += nw * 8;
                }
                pw += nw;
            }
        } else if (r->pinned && padded >= kDirectBytes) {
            e = flush_run();
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(batch)");
            e = cudaMemcpyAsync(d_seq + o, r->base + r->lo, span, cudaMemcpyHostToDevice, up);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(request)");
        } else {
            std::memcpy(h_gather + g, r->base + r->lo, span);
            if (run_bytes == 0) {
                run_dev = o;
                run_pin = g;
            }
            run_bytes = (g + padded) - run_pin;
            g += padded;
        }
        o += padded;
    }
    e = flush_run();
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(batch)");
    if (k) {
        e = cudaMemcpyAsync(d_rng, h_rng, k * sizeof(DevRange), cudaMemcpyHostToDevice, up);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(ranges)");
        e = cudaMemcpyAsync(d_fix, h_fix, n_fix * sizeof(FixEntry), cudaMemcpyHostToDevice, up);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(rebase table)");
    }
    if (n_unpack) {
        e = cudaMemcpyAsync(d_unpack, h_unpack, n_unpack * sizeof(UnpackEntry),
                            cudaMemcpyHostToDevice, up);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(unpack table)");
    }
    if ((e = cudaEventRecord(b->ev_up, up)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = cudaStreamWaitEvent(comp, b->ev_up, 0)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamWaitEvent");
    // The unpack and the rebase run on the compute stream: the upload stream
    // carries only copies, so it never waits for SMs held by the previous
    // batch's kernel.
    if (n_unpack) {
        const unsigned blocks =
            static_cast<unsigned>(std::min<uint64_t>(n_segs, static_cast<uint64_t>(f->sms) * 8));
        unpack_dense_kernel<<<blocks, 256, 0, comp>>>(reinterpret_cast<const uint64_t*>(d_packed),
                                                      d_unpack, n_unpack, n_segs, d_seq);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "unpack_dense_kernel");
    }
    if (n_fix) {
        const unsigned blocks = std::min<unsigned>((n_fix * 32 + 255) / 256, 1024);
        rebase_ranges_kernel<<<blocks, 256, 0, comp>>>(d_rng, d_fix, n_fix);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "rebase_ranges_kernel");
    }
    if (k) {
        TileParams p =
            ragged_params(f, query, d_seq, b->seq_bytes, d_rng, k, d_tile, tally ? nullptr : d_out,
                          d_ctl, reinterpret_cast<unsigned long long*>(d_ctl + 2) + (query ? 2 : 0),
                          bits);
        if (tally) {
            // (valid, positive) pairs per record, accumulated by the kernel.
            if ((e = cudaMemsetAsync(d_out, 0, k * 16, comp)) != cudaSuccess)
                return cuda_fail(e, "cudaMemsetAsync");
            p.rec_valid = reinterpret_cast<unsigned long long*>(d_out);
            p.rec_pos = p.rec_valid + 1;
            p.rec_shift = 1;
        }
        const int rc = cfg.use_graph
                           ? ragged_graph_launch(f, graph[query ? 1 : 0], query, p, 0, comp)
                           : ragged_launch(f, query, p, 0, comp);
        if (rc != SBF_OK) return rc;
    } else if (query && !tally && b->seq_bytes) {
        if ((e = cudaMemsetAsync(d_out, 0, b->seq_bytes, comp)) != cudaSuccess)
            return cuda_fail(e, "cudaMemsetAsync");
    }
    if (!query) {
        if ((e = cudaEventRecord(b->ev_done, comp)) != cudaSuccess)
            return cuda_fail(e, "cudaEventRecord");
        return SBF_OK;
    }
    if ((e = cudaEventRecord(b->ev_comp, comp)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = cudaStreamWaitEvent(down, b->ev_comp, 0)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamWaitEvent");
    for (size_t i = 0; i < b->reqs.size(); ++i) {
        SrvRequest* r = b->reqs[i];
        if (tally ? r->n == 0 : r->windows == 0) continue;
        const uint64_t src = tally ? b->req_rec[i] * 16 : bits ? b->req_off[i] / 8 : b->req_off[i];
        void* dst = expand ? static_cast<void*>(pinned_results(b) + src) : r->out;
        const uint64_t bytes = expand ? (r->windows + 31) / 32 * 4
                                      : result_bytes(b->op, r->windows, r->n);
        if ((e = cudaMemcpyAsync(dst, d_out + src, bytes, cudaMemcpyDeviceToHost, down)) !=
            cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(hits)");
    }
    if ((e = cudaEventRecord(b->ev_done, down)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    return SBF_OK;
}

}  // namespace sbf

struct sbf_server {
    sbf::Server s;
};

extern "C" double sbf_server_now(void) { return now_s(); }

extern "C" int sbf_server_create(sbf_filter_t* f, const sbf_server_config* config,
                                 sbf_server_t** out) {
    if (!f || !out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    *out = nullptr;
    if (const int bs = f->require_byte_symbols("the request server"); bs != SBF_OK) return bs;
    sbf_server_config c{};
    if (config) c = *config;
    if (c.staging_bytes == 0) c.staging_bytes = uint64_t{16} << 30;
    if (c.max_batch_bytes == 0) c.max_batch_bytes = uint64_t{256} << 20;
    if (c.pinned_bytes == 0) c.pinned_bytes = uint64_t{1} << 30;
    if (c.max_inflight == 0) c.max_inflight = 16;
    if (c.staging_bytes < (uint64_t{1} << 20) || c.pinned_bytes < (uint64_t{1} << 20))
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "server staging and pinned budgets must be >= 1 MiB");
    c.max_batch_bytes =
        std::min<uint64_t>({c.max_batch_bytes, c.staging_bytes / 4, c.pinned_bytes / 4});
    auto* h = new sbf_server();
    Server& s = h->s;
    s.f = f;
    s.cfg = c;
    s.dring.cap = c.staging_bytes;
    s.hring.cap = c.pinned_bytes;
    cudaError_t e;
    int rc = SBF_OK;
    do {
        if ((e = cudaStreamCreateWithFlags(&s.up, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&s.comp, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&s.down, cudaStreamNonBlocking)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaStreamCreate");
            break;
        }
        if ((e = cudaMalloc(&s.d_ring, c.staging_bytes)) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(SBF_ERR_RESOURCE, "cannot allocate %llu bytes of server staging",
                           static_cast<unsigned long long>(c.staging_bytes));
            break;
        }
        if ((e = cudaMallocHost(&s.h_ring, c.pinned_bytes)) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(SBF_ERR_RESOURCE, "cannot allocate %llu bytes of pinned staging",
                           static_cast<unsigned long long>(c.pinned_bytes));
            break;
        }
        if ((e = cudaMalloc(&s.d_ctl, 64)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMalloc");
            break;
        }
        if ((e = cudaMemset(s.d_ctl, 0, 64)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemset");
            break;
        }
        for (uint32_t i = 0; i < 3 * (c.max_inflight + 1) && rc == SBF_OK; ++i) {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
                rc = cuda_fail(e, "cudaEventCreate");
            else
                s.events.push_back(ev);
        }
    } while (false);
    if (rc != SBF_OK) {
        sbf_server_destroy(h);
        return rc;
    }
    if (const int t = host_expand_threads(); t > 0) {
        try {
            s.pool = std::make_unique<ExpandPool>(t);
        } catch (...) {
            s.pool.reset();  // no host threads to be had: download bytes
        }
    }
    try {
        s.worker = std::thread([&s] { s.run(); });
        s.completer = std::thread([&s] { s.finish(); });
    } catch (...) {
        // Nothing is queued yet, so destroy only joins what did start.
        sbf_server_destroy(h);
        return set_error(SBF_ERR_RESOURCE, "cannot start the server threads");
    }
    *out = h;
    return SBF_OK;
}

extern "C" int sbf_server_submit(sbf_server_t* h, int op, const char* base,
                                 const sbf_record_range* ranges, uint64_t n, uint8_t* out,
                                 uint64_t out_len, double arrival, uint64_t* ticket) {
    if (!h || !ticket) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    Server& s = h->s;
    if ((op & ~(kOpDense | 0xF)) != 0 || base_op(op) > kOpQueryCounts)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "op must be 0 (insert), 1 (query), 2 (query, bit-packed) or 3 (query, "
                         "per-record counts), optionally with 0x10 (dense-packed input)");
    if (is_dense(op) && s.f->alphabet != SBF_ALPHABET_DNA)
        return set_error(SBF_ERR_INVALID_ARGUMENT, "dense-packed requests need the DNA alphabet");
    if (n && (!ranges || !base)) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    auto r = std::make_unique<SrvRequest>();
    r->op = op;
    r->base = reinterpret_cast<const uint8_t*>(base);
    r->ranges = reinterpret_cast<const DevRange*>(ranges);
    r->n = n;
    if (n) {
        for (uint64_t i = 1; i < n; ++i)
            if (ranges[i].sequence_offset <
                ranges[i - 1].sequence_offset + ranges[i - 1].sequence_bytes)
                return set_error(SBF_ERR_INVALID_ARGUMENT,
                                 "request ranges must be ordered and non-overlapping");
        r->lo = ranges[0].sequence_offset;
        r->hi = std::max(r->lo, ranges[n - 1].sequence_offset + ranges[n - 1].sequence_bytes);
    }
    const uint64_t span = r->hi - r->lo;
    r->windows = span >= s.f->k ? span - s.f->k + 1 : 0;
    const bool has_result =
        base_op(op) == kOpQueryCounts ? n > 0 : (base_op(op) != kOpInsert && r->windows > 0);
    if (has_result && (!out || out_len < result_bytes(op, r->windows, n)))
        return set_error(SBF_ERR_INVALID_ARGUMENT, "query output span is too small");
    if (align_up(span, s.pad(op)) > s.cfg.max_batch_bytes || n * sizeof(DevRange) > s.cfg.max_batch_bytes)
        return set_error(SBF_ERR_INVALID_ARGUMENT,
                         "request of %llu bytes exceeds the server's batch cap of %llu bytes",
                         static_cast<unsigned long long>(span),
                         static_cast<unsigned long long>(s.cfg.max_batch_bytes));
    r->out = out;
    r->pinned = span && is_pinned(base + (is_dense(op) ? (r->lo / 32) * 8 : r->lo));
    r->t_arrival = arrival > 0 ? arrival : now_s();
    std::lock_guard<std::mutex> lk(s.mu);
    if (s.fatal != SBF_OK)
        return set_error(s.fatal, "server stopped after an error: %s", s.fatal_msg.c_str());
    r->ticket = s.next_ticket++;
    *ticket = r->ticket;
    s.pending.push_back(r.get());
    s.reqs.emplace(r->ticket, std::move(r));
    s.cv.notify_all();
    return SBF_OK;
}

extern "C" int sbf_server_wait(sbf_server_t* h, uint64_t ticket, double timeout_s,
                               sbf_server_request_info* info) {
    if (!h) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.reqs.find(ticket);
    if (it == s.reqs.end()) return set_error(SBF_ERR_INVALID_ARGUMENT, "unknown ticket");
    SrvRequest* r = it->second.get();
    auto ready = [&] { return r->done; };
    if (timeout_s > 0) {
        if (!s.cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
            return set_error(SBF_ERR_RESOURCE, "request %llu not complete within the timeout",
                             static_cast<unsigned long long>(ticket));
    } else {
        s.cv.wait(lk, ready);
    }
    if (info) {
        info->status = r->status;
        info->latency_s = r->t_done - r->t_arrival;
        info->windows = r->windows;
        info->arrival_s = r->t_arrival;
        info->done_s = r->t_done;
    }
    const int st = r->status;
    s.reqs.erase(it);
    if (st != SBF_OK) return set_error(st, "request failed: %s", s.fatal_msg.c_str());
    return SBF_OK;
}

extern "C" int sbf_server_drain(sbf_server_t* h) {
    if (!h) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    s.cv.wait(lk, [&] { return s.pending.empty() && s.inflight_batches == 0; });
    for (auto it = s.reqs.begin(); it != s.reqs.end();) {
        if (it->second->done)
            it = s.reqs.erase(it);
        else
            ++it;
    }
    if (s.fatal != SBF_OK) return set_error(s.fatal, "server error: %s", s.fatal_msg.c_str());
    return SBF_OK;
}

extern "C" int sbf_server_get_stats(sbf_server_t* h, int reset, sbf_server_stats* out) {
    if (!h || !out) return set_error(SBF_ERR_INVALID_ARGUMENT, "null pointer");
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    std::vector<double> l = s.latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
        if (l.empty()) return 0.0;
        const size_t i = std::min(l.size() - 1, static_cast<size_t>(q * (l.size() - 1) + 0.5));
        return l[i];
    };
    double sum = 0;
    for (double x : l) sum += x;
    *out = sbf_server_stats{};
    out->requests = s.n_reqs;
    out->batches = s.n_batches;
    out->query_windows = s.q_windows;
    out->insert_windows = s.i_windows;
    out->wall_s = s.t_last > s.t_first ? s.t_last - s.t_first : 0;
    out->p50_s = pct(0.50);
    out->p99_s = pct(0.99);
    out->p999_s = pct(0.999);
    out->max_s = l.empty() ? 0 : l.back();
    out->mean_s = l.empty() ? 0 : sum / l.size();
    out->mean_batch_requests =
        s.n_batches ? static_cast<double>(s.n_batched_reqs) / s.n_batches : 0;
    out->worker_busy_s = s.busy_s;
    out->admission_wait_s = s.admit_wait_s;
    out->slot_wait_s = s.slot_wait_s;
    if (reset) {
        s.latencies.clear();
        s.n_batches = s.n_batched_reqs = s.q_windows = s.i_windows = s.n_reqs = 0;
        s.t_first = s.t_last = 0;
        s.busy_s = s.admit_wait_s = s.slot_wait_s = 0;
    }
    return SBF_OK;
}

extern "C" void sbf_server_destroy(sbf_server_t* h) {
    if (!h) return;
    Server& s = h->s;
    {
        std::lock_guard<std::mutex> lk(s.mu);
        s.stop = true;
        s.cv.notify_all();
    }
    if (s.worker.joinable()) {
        // The worker drains the queue before it exits.
        std::unique_lock<std::mutex> lk(s.mu);
        s.cv.wait(lk, [&] { return s.pending.empty() && s.inflight_batches == 0; });
        lk.unlock();
        s.worker.join();
    }
    if (s.completer.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s.mu);
            s.cv.notify_all();
        }
        s.completer.join();
    }
    if (s.up) cudaStreamSynchronize(s.up);
    if (s.comp) cudaStreamSynchronize(s.comp);
    if (s.down) cudaStreamSynchronize(s.down);
    for (auto& g : s.graph) ragged_graph_release(g);
    for (cudaEvent_t ev : s.events) cudaEventDestroy(ev);
    if (s.d_ring) cudaFree(s.d_ring);
    if (s.h_ring) cudaFreeHost(s.h_ring);
    if (s.d_ctl) cudaFree(s.d_ctl);
    if (s.up) cudaStreamDestroy(s.up);
    if (s.comp) cudaStreamDestroy(s.comp);
    if (s.down) cudaStreamDestroy(s.down);
    delete h;
}
