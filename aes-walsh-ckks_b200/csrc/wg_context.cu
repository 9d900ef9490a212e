// Context construction: the host tables (wg_tables.cpp) uploaded once into device-resident
// buffers, per-stream scratch and the switching-key registry.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>

#include "wg_internal.hpp"
#include "wg_ntt.cuh"
#include "wg_ring.hpp"
#include "wg_tables.hpp"

namespace wg {

static bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s) cudaStreamIsCapturing(s, &cs);
    return cs != cudaStreamCaptureStatusNone;
}

std::atomic<uint64_t> g_stage_calls{0}, g_stage_bytes{0}, g_stage_wait_ns{0};

void stage_stats(uint64_t* calls, uint64_t* bytes, uint64_t* wait_ns) {
    *calls = g_stage_calls.load();
    *bytes = g_stage_bytes.load();
    *wait_ns = g_stage_wait_ns.load();
}

void* BatchBuffers::stage(const Context& c, const void* data, size_t bytes, cudaStream_t s) {
    const size_t off = reserve(c, bytes, s);
    std::memcpy(h_ring + off, data, bytes);
    return commit(off, bytes, s);
}

size_t BatchBuffers::reserve(const Context& c, size_t bytes, cudaStream_t s) {
    g_stage_calls.fetch_add(1, std::memory_order_relaxed);
    g_stage_bytes.fetch_add(bytes, std::memory_order_relaxed);
    if (capturing(s))
        fail(kRuntime, "batched calls cannot be captured into a graph (their staging is reused); use wg_batch_plan_*");
    const size_t need = (std::max<size_t>(bytes, 1) + 255) & ~size_t{255};
    if (need > ring_bytes) {
        // grow: everything queued on the stream may still read the old device ring
        check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(s), "staging ring resize");
        for (Flight& f : flights) spare_events.push_back(f.done);
        flights.clear();
        cudaFree(d_ring);
        cudaFreeHost(h_ring);
        d_ring = h_ring = nullptr;
        ring_bytes = 0;
        const size_t cap = std::max<size_t>(need * 2, size_t{64} << 20);
        if (cudaMalloc((void**)&d_ring, cap) != cudaSuccess || cudaMallocHost((void**)&h_ring, cap) != cudaSuccess) {
            cudaGetLastError();
            fail(kNoMemory, "staging ring allocation failed");
        }
        ring_bytes = cap;
        head = 0;
    }
    // wait for the uploads whose host bytes this region still holds (ring_place: the newest
    // overlapping one, which completes every older one too; all of them are then released)
    size_t wait = 0;
    const size_t begin = ring_place(head, ring_bytes, need, flights, &wait);
    head = begin;
    if (wait > 0) {
        const auto t0 = std::chrono::steady_clock::now();
        check_cuda(cudaEventSynchronize(flights[wait - 1].done), "staging ring wait");
        g_stage_wait_ns.fetch_add(
            (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count(),
            std::memory_order_relaxed);
        for (size_t k = 0; k < wait; ++k) {
            spare_events.push_back(flights.front().done);
            flights.pop_front();
        }
    }
    return begin;
}

void* BatchBuffers::commit(size_t begin, size_t bytes, cudaStream_t s) {
    const size_t need = (std::max<size_t>(bytes, 1) + 255) & ~size_t{255};
    const size_t end = begin + need;
    check_cuda(cudaMemcpyAsync(d_ring + begin, h_ring + begin, bytes, cudaMemcpyHostToDevice, s), "staging upload");
    cudaEvent_t ev = nullptr;
    if (!spare_events.empty()) {
        ev = spare_events.back();
        spare_events.pop_back();
    } else {
        check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    }
    check_cuda(cudaEventRecord(ev, s), "staging event");
    flights.push_back({begin, end, ev});
    head = end;
    return d_ring + begin;
}

uint64_t* BatchBuffers::arena(const Context& c, size_t words, cudaStream_t s) {
    if (words <= arena_words) return d_arena;
    if (capturing(s)) fail(kRuntime, "batched scratch must be sized (one uncaptured call) before graph capture");
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    // the smaller arena may still be in use by work queued on this stream (the only user of
    // this stream's arena); other streams keep running
    check_cuda(cudaStreamSynchronize(s), "batched scratch resize");
    cudaFree(d_arena);
    d_arena = nullptr;
    arena_words = 0;
    if (cudaMalloc(&d_arena, words * 8) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "batched scratch allocation failed");
    }
    arena_words = words;
    return d_arena;
}

void BatchBuffers::release() {
    for (Flight& f : flights) {
        cudaEventSynchronize(f.done);
        cudaEventDestroy(f.done);
    }
    flights.clear();
    for (cudaEvent_t e : spare_events) cudaEventDestroy(e);
    spare_events.clear();
    cudaFree(d_ring);
    cudaFreeHost(h_ring);
    cudaFree(d_arena);
    d_ring = h_ring = nullptr;
    d_arena = nullptr;
    ring_bytes = 0;
}

BatchBuffers& Context::batch_buffers(cudaStream_t s) {
    std::lock_guard<std::mutex> g(ws_mutex);
    auto it = batches.find(s);
    if (it != batches.end()) return it->second;
    if (capturing(s)) fail(kRuntime, "batched buffers for this stream must be reserved before graph capture");
    return batches[s];
}

// bytes cached by the chunk caches of every context of the process
static std::atomic<size_t> chunk_cache_total{0};

void* Context::take_chunk(size_t bytes, cudaStream_t s, size_t* got) {
    if (capturing(s)) return nullptr;  // no dependency on work outside a capture
    std::lock_guard<std::mutex> g(chunk_mutex);
    auto it = chunk_cache.lower_bound(bytes);
    if (it == chunk_cache.end() || it->first > 2 * bytes) return nullptr;
    const CachedChunk ch = it->second;
    chunk_cache.erase(it);
    chunk_cache_bytes -= ch.bytes;
    chunk_cache_total -= ch.bytes;
    check_cuda(cudaStreamWaitEvent(s, ch.done, 0), "chunk reuse");
    chunk_events.push_back(ch.done);
    *got = ch.bytes;
    return ch.p;
}

void Context::give_chunk(void* p, size_t bytes, cudaStream_t s) {
    std::lock_guard<std::mutex> g(chunk_mutex);
    if (capturing(s) || chunk_cache_total.load() + bytes > kChunkCacheBytes) {
        cudaFreeAsync(p, s);
        return;
    }
    cudaEvent_t ev = nullptr;
    if (!chunk_events.empty()) {
        ev = chunk_events.back();
        chunk_events.pop_back();
    } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(p, s);
        return;
    }
    if (cudaEventRecord(ev, s) != cudaSuccess) {
        cudaGetLastError();
        chunk_events.push_back(ev);
        cudaFreeAsync(p, s);
        return;
    }
    chunk_cache.emplace(bytes, CachedChunk{p, bytes, ev});
    chunk_cache_bytes += bytes;
    chunk_cache_total += bytes;
}

void Context::trim(cudaStream_t s) {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    {
        std::lock_guard<std::mutex> g(ws_mutex);
        if (capturing(s)) fail(kRuntime, "trim: the stream is capturing a graph");
        auto bi = batches.find(s);
        if (bi != batches.end()) {
            check_cuda(cudaStreamSynchronize(s), "trim");
            bi->second.release();
            batches.erase(bi);
        }
        auto wi = workspaces.find(s);
        if (wi != workspaces.end()) {
            check_cuda(cudaStreamSynchronize(s), "trim");
            cudaFree(wi->second.base);
            workspaces.erase(wi);
        }
    }
    std::lock_guard<std::mutex> g(chunk_mutex);
    for (auto& kv : chunk_cache) {
        cudaEventSynchronize(kv.second.done);
        cudaFree(kv.second.p);
        chunk_events.push_back(kv.second.done);
    }
    chunk_cache.clear();
    chunk_cache_total -= chunk_cache_bytes;
    chunk_cache_bytes = 0;
    // the stream-ordered pool keeps freed blocks up to its release threshold: hand them back
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
}

Context::~Context() {
    chunk_cache_total -= chunk_cache_bytes;
    for (auto& kv : chunk_cache) {
        cudaFree(kv.second.p);
        cudaEventDestroy(kv.second.done);
    }
    for (cudaEvent_t ev : chunk_events) cudaEventDestroy(ev);
    for (auto& kv : consts) {
        cudaFree(kv.second.d);
        cudaEventDestroy(kv.second.ready);
    }
    for (auto& kv : keys) cudaFree(kv.second.d_data);
    for (auto& kv : workspaces) cudaFree(kv.second.base);
    for (auto& kv : batches) kv.second.release();
    cudaFree(d_modup);
    cudaFree(d_mod);
    cudaFree(d_tw);
    cudaFree(d_tables);
}

size_t Context::workspace_words() const {
    // the largest switch plus room for a permuted copy of a ciphertext (conjugation) and the
    // rescale remainders
    return keyswitch_workspace_words(*this, nq - 1) + 4 * nq * N;
}

uint64_t* Context::workspace(cudaStream_t s) {
    std::lock_guard<std::mutex> g(ws_mutex);
    auto it = workspaces.find(s);
    if (it != workspaces.end()) return it->second.base;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (s) cudaStreamIsCapturing(s, &cs);
    if (cs != cudaStreamCaptureStatusNone)
        fail(kRuntime, "workspace for this stream must be reserved (wg_ctx_reserve) before graph capture");
    Workspace w;
    w.words = workspace_words();
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (cudaMalloc(&w.base, w.words * 8) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "workspace allocation failed");
    }
    workspaces.emplace(s, w);
    return w.base;
}

const KeyEntry& Context::key(int kind, int64_t rotation) const {
    auto it = keys.find({kind, rotation});
    if (it == keys.end()) fail(kRuntime, "switching key is unavailable");
    return it->second;
}

Context* create_context(uint64_t N, const uint64_t* q, size_t nq, const uint64_t* p, size_t np, size_t dnum,
                        int device) {
    if (N < 1024 || N > 65536 || (N & (N - 1))) fail(kInvalid, "ring degree must be a power of two in [2^10, 2^16]");
    if (nq == 0 || np == 0) fail(kInvalid, "hybrid key switching needs at least one Q and one P modulus");
    if (np > (size_t)16) fail(kInvalid, "at most 16 P moduli are supported");
    if (dnum == 0 || dnum > nq) fail(kInvalid, "invalid hybrid key-switch partition count");
    for (size_t i = 0; i < nq + np; ++i) {
        const uint64_t m = i < nq ? q[i] : p[i - nq];
        if (m >= (uint64_t{1} << 62) || m < 3 || (m - 1) % (2 * N)) fail(kInvalid, "moduli must be primes 1 mod 2N below 2^62");
    }
    if ((nq + dnum - 1) / dnum > 16) fail(kInvalid, "digit width above 16 limbs is not supported");
    auto c = std::make_unique<Context>();
    c->device = device;
    c->N = N;
    c->logN = __builtin_ctzll(N);
    c->nq = nq;
    c->np = np;
    c->dnum = dnum;
    c->alpha = (nq + dnum - 1) / dnum;
    c->q.assign(q, q + nq);
    c->p.assign(p, p + np);
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    {
        // The batched operations draw their temporaries from this process's stream-ordered
        // pool; let it keep up to 8 GiB across synchronisations instead of unmapping and
        // remapping it around every event wait.
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t cur = 0;
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur);
            uint64_t want = uint64_t{8} << 30;
            if (cur < want) cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &want);
        }
        cudaGetLastError();
    }
    HostTables H = build_tables(N, q, nq, p, np, dnum);
    c->mods = H.mods;
    const size_t nm = nq + np;

    // Upload.
    auto dev_alloc = [&](void** ptr, size_t bytes) {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            fail(kNoMemory, "device allocation failed while building the context");
        }
    };
    dev_alloc((void**)&c->d_mod, nm * sizeof(Modulus));
    dev_alloc((void**)&c->d_tw, H.tw.size() * 8);
    c->tables_words = H.words.size() + 1;
    dev_alloc((void**)&c->d_tables, c->tables_words * 8);
    check_cuda(cudaMemcpy(c->d_mod, c->mods.data(), nm * sizeof(Modulus), cudaMemcpyHostToDevice), "upload moduli");
    {
        // interleaved (w, Shoup w) pairs per modulus and direction, as the NTT kernels read them
        std::vector<ntt::TwPair> pairs(nm * 2 * N);
        for (size_t i = 0; i < nm; ++i) ntt::interleave_twiddles(N, H.tw.data() + i * 4 * N, pairs.data() + i * 2 * N);
        check_cuda(cudaMemcpy(c->d_tw, pairs.data(), pairs.size() * sizeof(ntt::TwPair), cudaMemcpyHostToDevice),
                   "upload twiddles");
    }
    check_cuda(cudaMemcpy(c->d_tables, H.words.data(), H.words.size() * 8, cudaMemcpyHostToDevice),
               "upload tables");
    const uint64_t* T = c->d_tables;
    c->modup.resize(nq);
    for (size_t level = 0; level < nq; ++level) {
        for (size_t part = 0; part < H.modup[level].size(); ++part) {
            const ModUpOffsets& o = H.modup[level][part];
            ModUpDesc d;
            d.src_count = o.src_count;
            d.dst_count = o.dst_count;
            d.src_first = o.src_first;
            d.pad = 0;
            d.qhat_inv = T + o.qhat_inv;
            d.qhat_inv_s = T + o.qhat_inv_s;
            d.src_inv = reinterpret_cast<const double*>(T + o.src_inv);
            d.qhat = T + o.qhat;
            d.qhat_s = T + o.qhat_s;
            d.corr = T + o.corr;
            d.dst_limb = reinterpret_cast<const int*>(T + o.dst_limb);
            d.dst_mod = reinterpret_cast<const int*>(T + o.dst_mod);
            c->modup[level].push_back(d);
        }
    }
    c->fold_inv.resize(nq);
    c->fold_inv_s.resize(nq);
    for (size_t level = 0; level < nq; ++level) {
        c->fold_inv[level] = T + H.fold_inv[level];
        c->fold_inv_s[level] = T + H.fold_inv_s[level];
    }
    {
        std::vector<ModUpDesc> flat(nq * dnum);
        for (size_t level = 0; level < nq; ++level)
            for (size_t part = 0; part < c->modup[level].size(); ++part) flat[level * dnum + part] = c->modup[level][part];
        dev_alloc((void**)&c->d_modup, flat.size() * sizeof(ModUpDesc));
        check_cuda(cudaMemcpy(c->d_modup, flat.data(), flat.size() * sizeof(ModUpDesc), cudaMemcpyHostToDevice),
                   "upload ModUp descriptors");
    }
    c->rs_host_off.assign(nq, 0);
    for (size_t d = 1; d < nq; ++d) {
        c->rs_host_off[d] = c->rs_host.size();
        c->rs_host.insert(c->rs_host.end(), H.words.begin() + H.rescale[d], H.words.begin() + H.rescale[d] + 4 * d);
    }
    c->rs_one_s.assign(nq, nullptr);
    c->rs_inv_p.assign(nq, nullptr);
    c->rs_inv_p_s.assign(nq, nullptr);
    c->rs_half.assign(nq, nullptr);
    for (size_t d = 1; d < nq; ++d) {
        c->rs_one_s[d] = T + H.rescale[d];
        c->rs_inv_p[d] = T + H.rescale[d] + d;
        c->rs_inv_p_s[d] = T + H.rescale[d] + 2 * d;
        c->rs_half[d] = T + H.rescale[d] + 3 * d;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        c->sm_count = sms;
    cudaGetLastError();
    ntt_autotune(*c);
    return c.release();
}

}  // namespace wg
