// Batched execution: one launch per pipeline stage over every ciphertext, limb and digit of a
// batch, whatever their levels.
//
// Each stage reads a table of small jobs (pointers, modulus index, constants) from device
// memory; block (x, y + 65535 z) runs tile x of job y.  All tables of a call are built on the
// host, staged in pinned memory and uploaded with one copy, so a batched key switch over 64
// ciphertexts is 7-8 launches (12-13 with the NTT steps unfused) instead of that many per
// ciphertext.
// Arithmetic is shared with the single-ciphertext path (wg_keyswitch.cuh, wg_arith.cuh), so
// results are identical.
#include <algorithm>
#include <cstring>
#include <memory>
#include <optional>

#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"

namespace wg {
using namespace bk;

// ------------------------------------------------------------------------------------------
// Job-table staging
// ------------------------------------------------------------------------------------------
void JobTable::upload(Context& c, cudaStream_t s) {
    WG_SPAN("upload");
    base = c.batch_buffers(s).stage(c, bytes.data(), bytes.size(), s);
}

// ------------------------------------------------------------------------------------------
// Batched key switch
// ------------------------------------------------------------------------------------------
struct KsPlan {
    const NttJob* intt_in;
    int n_intt_in;
    const ModUpJob* modup;
    int n_modup;
    const NttJob* ntt_digits;
    int n_ntt_digits;
    const MacGroupJob* mac;
    int n_mac;
    const NttJob* intt_p;
    int n_intt_p;
    const ModDownJob* moddown;
    int n_moddown;
    const NttJob* ntt_contrib;
    int n_ntt_contrib;
    const CombineJob* combine;
    int n_combine;
    const GatherJob* gather;
    int n_gather;
    const NttEpiJob* contrib_epi;  // fused: forward row phase of the contributions + combine
    int n_contrib_epi;
    double contrib_epi_bytes;
    double mac_bytes, modup_bytes, moddown_bytes, combine_bytes;
    bool fused;   // ModUp / ModDown fused with the NTT column phases (Context::ntt_fusion)
    int max_src;  // widest digit (fused ModUp shared memory)
};

size_t batch_keyswitch_words(const Context& c, const KsItem* items, size_t n) {
    size_t w = 0;
    for (size_t i = 0; i < n; ++i) w += keyswitch_workspace_words(c, items[i].level);
    return w;
}

static KsPlan plan_keyswitch(const Context& c, const KsItem* items, size_t n, uint64_t* ws, JobTable& t) {
    const size_t N = c.N, K = c.np, nq = c.nq;
    std::vector<NttJob> intt_in, ntt_digits, intt_p, ntt_contrib;
    std::vector<ModUpJob> modup;
    std::vector<MacGroupJob> mac;
    std::vector<ModDownJob> moddown;
    std::vector<CombineJob> combine;
    std::vector<GatherJob> gather;
    std::vector<NttEpiJob> contrib_epi;
    KsPlan p{};
    p.fused = c.fuse(2 * n);  // the ModDown launch has two jobs per switch
    // MAC groups: consecutive switches with the same key, level and digit layout (up to
    // kMacGroup), one job per QP limb; [group_begin, it) is the open group
    size_t group_begin = 0;
    std::vector<uint64_t*> group_digits, group_acc;
    auto close_group = [&](size_t end) {
        if (end == group_begin) return;
        const KsItem& g = items[group_begin];
        const size_t L = g.level + 1, T = L + K, B = c.parts_at(g.level);
        for (size_t i = 0; i < T; ++i) {
            MacGroupJob jb{};
            jb.key = g.key->d_data;
            jb.part_stride = T * N;
            jb.L = (int)L;
            jb.K = (int)K;
            jb.parts = (int)B;
            jb.alpha = (int)c.alpha;
            jb.key_level = (int)g.key->key_level;
            jb.i = (int)i;
            jb.n = (int)(end - group_begin);
            for (size_t k = group_begin; k < end; ++k) {
                jb.key_term[k - group_begin] = items[k].key_term;
                jb.digits[k - group_begin] = group_digits[k - group_begin];
                jb.acc[k - group_begin] = group_acc[k - group_begin];
            }
            mac.push_back(jb);
        }
        p.mac_bytes += 8.0 * N * T * (2.0 * B + (double)(end - group_begin) * (B + 2.0));
        group_begin = end;
        group_digits.clear();
        group_acc.clear();
    };
    for (size_t it = 0; it < n; ++it) {
        const KsItem& x = items[it];
        const size_t level = x.level, L = level + 1, T = L + K, B = c.parts_at(level);
        if (level >= nq) fail(kInvalid, "batched keyswitch: invalid ciphertext level");
        if (x.key->key_level < level) fail(kRuntime, "keyswitch: switch key level is below ciphertext level");
        if (x.key->parts < B) fail(kRuntime, "keyswitch: insufficient key partitions");
        uint64_t* coeff = ws;
        uint64_t* digits = coeff + L * N;
        uint64_t* acc = digits + B * T * N;
        uint64_t* contrib = acc + 2 * T * N;
        ws += keyswitch_workspace_words(c, level);
        for (size_t l = 0; l < L; ++l) intt_in.push_back({x.key_term + l * N, coeff + l * N, (int)l, 0});
        for (size_t j = 0; j < B; ++j) {
            modup.push_back({c.d_modup + level * c.dnum + j, coeff, digits + j * T * N});
            const ModUpDesc& d = c.modup[level][j];
            p.max_src = std::max(p.max_src, d.src_count);
            p.modup_bytes += 8.0 * N * (d.src_count + d.dst_count);
            const size_t s0 = j * c.alpha, s1 = std::min(s0 + c.alpha, L);
            for (size_t l = 0; l < T; ++l) {
                if (l >= s0 && l < s1) continue;
                uint64_t* ptr = digits + j * T * N + l * N;
                ntt_digits.push_back({ptr, ptr, (int)(l < L ? l : nq + (l - L)), 0});
            }
        }
        if (it > group_begin) {
            const KsItem& g = items[group_begin];
            if (it - group_begin == (size_t)kMacGroup || g.key != x.key || g.level != x.level) close_group(it);
        }
        group_digits.push_back(digits);
        group_acc.push_back(acc);
        for (int poly = 0; poly < 2; ++poly)
            for (size_t pi = 0; pi < K; ++pi) {
                uint64_t* ptr = acc + (poly * T + L + pi) * N;
                intt_p.push_back({ptr, ptr, (int)(nq + pi), 0});
            }
        for (int poly = 0; poly < 2; ++poly) {
            moddown.push_back({acc + (poly * T + L) * N, contrib + poly * L * N, c.fold_inv[level],
                               c.fold_inv_s[level], (int)L, 0});
            if (!p.fused)
                for (size_t qi = 0; qi < L; ++qi) {
                    uint64_t* ptr = contrib + (poly * L + qi) * N;
                    ntt_contrib.push_back({ptr, ptr, (int)qi, 0});
                }
        }
        p.moddown_bytes += 8.0 * N * 2.0 * (K + L);
        const bool gal = x.galois != 0;
        for (size_t qi = 0; qi < L; ++qi) {
            uint64_t* bo = gal ? acc + T * N : x.b;
            uint64_t* ao = gal ? acc : x.a;
            if (p.fused) {
                // a: accumulator poly 0, contribution limbs [0, L); b: poly 1, [L, 2L)
                contrib_epi.push_back({contrib + qi * N, acc + qi * N, x.a_in ? x.a_in + qi * N : nullptr,
                                       ao + qi * N, (uint64_t)x.a_add, 0, (int)qi, kEpiCombine});
                contrib_epi.push_back({contrib + (L + qi) * N, acc + (T + qi) * N,
                                       x.b_in ? x.b_in + qi * N : nullptr, bo + qi * N, (uint64_t)x.b_add, 0,
                                       (int)qi, kEpiCombine});
            } else {
                combine.push_back(
                    {acc, contrib, x.b_in, x.a_in, bo, ao, (int)L, (int)K, (int)qi, x.b_add, x.a_add, 0});
            }
            if (gal)
                gather.push_back({acc + T * N + qi * N, acc + qi * N, x.b + qi * N, x.a + qi * N, x.galois});
        }
        p.combine_bytes += 8.0 * N * L * (x.b_add + x.a_add + 6.0) + (gal ? 8.0 * N * L * 4.0 : 0.0);
    }
    close_group(n);
    p.intt_in = t.add(intt_in);
    p.n_intt_in = (int)intt_in.size();
    p.modup = t.add(modup);
    p.n_modup = (int)modup.size();
    p.ntt_digits = t.add(ntt_digits);
    p.n_ntt_digits = (int)ntt_digits.size();
    p.mac = t.add(mac);
    p.n_mac = (int)mac.size();
    p.intt_p = t.add(intt_p);
    p.n_intt_p = (int)intt_p.size();
    p.moddown = t.add(moddown);
    p.n_moddown = (int)moddown.size();
    p.ntt_contrib = t.add(ntt_contrib);
    p.n_ntt_contrib = (int)ntt_contrib.size();
    p.combine = t.add(combine);
    p.n_combine = (int)combine.size();
    p.gather = t.add(gather);
    p.n_gather = (int)gather.size();
    p.contrib_epi = t.add(contrib_epi);
    p.n_contrib_epi = (int)contrib_epi.size();
    p.contrib_epi_bytes = ntt_epilogue_bytes(contrib_epi, N);
    return p;
}

static void run_keyswitch(const Context& c, const KsPlan& p, const JobTable& t, cudaStream_t s) {
    const size_t N = c.N;
    if (p.fused) {
        // inverse row phase -> [inverse column phase, ModUp, forward column phase] -> forward
        // row phase; the same around ModDown (wg_ksfuse.cu)
        ntt_jobs_phase(c, t.at(p.intt_in), p.n_intt_in, false, false, s);
        modup_ntt_jobs(c, t.at(p.modup), p.n_modup, p.max_src, p.modup_bytes, s);
        ntt_jobs_phase(c, t.at(p.ntt_digits), p.n_ntt_digits, true, false, s);
        {
            Probe probe(kClsKeyMac, p.mac_bytes, s);
            kb_mac_group<<<grid_for(c, p.n_mac), kT, 0, s>>>(t.at(p.mac), p.n_mac, c.d_mod, (int)c.nq, N);
        }
        ntt_jobs_phase(c, t.at(p.intt_p), p.n_intt_p, false, false, s);
        moddown_ntt_jobs(c, t.at(p.moddown), p.n_moddown, p.moddown_bytes, s);
        ntt_rows_epilogue_jobs(c, t.at(p.contrib_epi), p.n_contrib_epi, p.contrib_epi_bytes, s);
        if (p.n_gather) {
            Probe probe(kClsCombine, 8.0 * N * 4.0 * p.n_gather, s);
            kb_gather<<<grid_for(c, p.n_gather), kT, 0, s>>>(t.at(p.gather), p.n_gather, c.logN);
        }
        check_cuda(cudaGetLastError(), "batched keyswitch launch");
        return;
    }
    ntt_jobs(c, t.at(p.intt_in), p.n_intt_in, false, s);
    {
        Probe probe(kClsModUp, p.modup_bytes, s);
        kb_modup<<<grid_for(c, p.n_modup), kT, 0, s>>>(t.at(p.modup), p.n_modup, c.d_mod, N);
    }
    ntt_jobs(c, t.at(p.ntt_digits), p.n_ntt_digits, true, s);
    {
        Probe probe(kClsKeyMac, p.mac_bytes, s);
        kb_mac_group<<<grid_for(c, p.n_mac), kT, 0, s>>>(t.at(p.mac), p.n_mac, c.d_mod, (int)c.nq, N);
    }
    ntt_jobs(c, t.at(p.intt_p), p.n_intt_p, false, s);
    {
        Probe probe(kClsModDown, p.moddown_bytes, s);
        kb_moddown<<<grid_for(c, p.n_moddown), kT, 0, s>>>(t.at(p.moddown), p.n_moddown, c.d_mod, (int)c.nq,
                                                            (int)c.np, N);
    }
    ntt_jobs(c, t.at(p.ntt_contrib), p.n_ntt_contrib, true, s);
    {
        Probe probe(kClsCombine, p.combine_bytes, s);
        kb_combine<<<grid_for(c, p.n_combine), kT, 0, s>>>(t.at(p.combine), p.n_combine, c.d_mod, N);
        if (p.n_gather) kb_gather<<<grid_for(c, p.n_gather), kT, 0, s>>>(t.at(p.gather), p.n_gather, c.logN);
    }
    check_cuda(cudaGetLastError(), "batched keyswitch launch");
}

void batch_keyswitch(Context& c, const KsItem* items, size_t n, cudaStream_t s) {
    WG_SPAN("keyswitch");
    if (n == 0) return;
    uint64_t* ws = c.batch_buffers(s).arena(c, batch_keyswitch_words(c, items, n), s);
    JobTable t;
    KsPlan p = plan_keyswitch(c, items, n, ws, t);
    t.upload(c, s);
    run_keyswitch(c, p, t, s);
}

// ------------------------------------------------------------------------------------------
// Batched mul + relin + rescale + rotate
// ------------------------------------------------------------------------------------------
// A planned pipeline: the job-table image and the launch sequence that reads it.
struct PipelinePlan {
    JobTable t;
    const TensorJob* jt = nullptr;
    int nt = 0;
    std::optional<RescaleJobs> rescale;
    KsPlan p1{}, p2{};
    bool rotate = false;
    double tb = 0;
};

// Arena: c2 per ciphertext, rescale remainders, then the larger of the two key-switch batches.
static size_t pipeline_words(const Context& c, size_t count, const size_t* levels, const uint64_t* galois,
                             size_t* c2_out, size_t* rem_out) {
    const size_t N = c.N;
    std::vector<KsItem> relin_items(count), rot_items;
    size_t c2_words = 0, rem_words = 0;
    for (size_t i = 0; i < count; ++i) {
        c2_words += (levels[i] + 1) * N;
        rem_words += 2 * levels[i] * N;
        relin_items[i].level = levels[i];
        if (galois[i]) {
            KsItem it;
            it.level = levels[i] - 1;
            rot_items.push_back(it);
        }
    }
    const size_t ks1 = batch_keyswitch_words(c, relin_items.data(), count);
    const size_t ks2 = batch_keyswitch_words(c, rot_items.data(), rot_items.size());
    if (c2_out) *c2_out = c2_words;
    if (rem_out) *rem_out = rem_words;
    return c2_words + rem_words + std::max(ks1, ks2);
}

static void plan_pipeline(const Context& c, PipelinePlan& P, size_t count, const size_t* levels,
                          uint64_t* const* xb, uint64_t* const* xa, const uint64_t* const* yb,
                          const uint64_t* const* ya, const uint64_t* galois, const KeyEntry* relin,
                          const KeyEntry* const* rot_keys, uint64_t* arena) {
    const size_t N = c.N;
    size_t c2_words = 0, rem_words = 0;
    pipeline_words(c, count, levels, galois, &c2_words, &rem_words);
    uint64_t* c2base = arena;
    uint64_t* rembase = c2base + c2_words;
    uint64_t* ksbase = rembase + rem_words;
    std::vector<KsItem> relin_items(count), rot_items;
    std::vector<TensorJob> tensor;
    RescaleJobs& rs = P.rescale.emplace();
    uint64_t* c2p = c2base;
    uint64_t* remp = rembase;
    for (size_t i = 0; i < count; ++i) {
        const size_t lv = levels[i], L = lv + 1;
        for (size_t l = 0; l < L; ++l)
            tensor.push_back({xb[i] + l * N, xa[i] + l * N, yb[i] + l * N, ya[i] + l * N, c2p + l * N, (int)l, 0});
        KsItem& ri = relin_items[i];
        ri.level = lv;
        ri.key_term = c2p;
        ri.key = relin;
        ri.b_in = xb[i];
        ri.a_in = xa[i];
        ri.b = xb[i];
        ri.a = xa[i];
        ri.b_add = 1;
        ri.a_add = 1;
        ri.galois = 0;
        c2p += L * N;
        for (int poly = 0; poly < 2; ++poly) {
            rs.add(poly ? xa[i] : xb[i], lv, remp);
            remp += lv * N;
        }
        if (galois[i]) {
            KsItem it;
            it.level = lv - 1;
            it.key_term = xa[i];
            it.key = rot_keys[i];
            it.b_in = xb[i];
            it.a_in = xa[i];
            it.b = xb[i];
            it.a = xa[i];
            it.b_add = 1;
            it.a_add = 0;
            it.galois = galois[i];
            rot_items.push_back(it);
        }
        P.tb += 8.0 * N * (lv + 1) * 7.0;
    }
    P.jt = P.t.add(tensor);
    P.nt = (int)tensor.size();
    rs.plan(c, P.t);
    P.p1 = plan_keyswitch(c, relin_items.data(), count, ksbase, P.t);
    P.p2 = plan_keyswitch(c, rot_items.data(), rot_items.size(), ksbase, P.t);
    P.rotate = !rot_items.empty();
}

static void launch_pipeline(const Context& c, const PipelinePlan& P, cudaStream_t s) {
    const JobTable& t = P.t;
    {
        Probe probe(kClsElementwise, P.tb, s);
        kb_tensor<<<grid_wide(c, P.nt), kT, 0, s>>>(t.at(P.jt), P.nt, c.d_mod);
    }
    run_keyswitch(c, P.p1, t, s);
    P.rescale->run(c, t, s);
    if (P.rotate) run_keyswitch(c, P.p2, t, s);
    check_cuda(cudaGetLastError(), "batched pipeline launch");
}

void batch_mul_relin_rescale_rotate(Context& c, size_t count, const size_t* levels, uint64_t* const* xb,
                                    uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                                    const int64_t* rots, const uint64_t* galois, const KeyEntry* relin,
                                    const KeyEntry* const* rot_keys, cudaStream_t s) {
    (void)rots;
    if (count == 0) return;
    uint64_t* arena = c.batch_buffers(s).arena(c, pipeline_words(c, count, levels, galois, nullptr, nullptr), s);
    PipelinePlan P;
    plan_pipeline(c, P, count, levels, xb, xa, yb, ya, galois, relin, rot_keys, arena);
    P.t.upload(c, s);
    launch_pipeline(c, P, s);
}

// ------------------------------------------------------------------------------------------
// Graph-captured batch plan
// ------------------------------------------------------------------------------------------
BatchGraph::~BatchGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_jobs);
    cudaFree(d_arena);
}

BatchGraph* batch_graph_create(Context& c, size_t count, const size_t* levels, uint64_t* const* xb,
                               uint64_t* const* xa, const uint64_t* const* yb, const uint64_t* const* ya,
                               const uint64_t* galois, const KeyEntry* relin, const KeyEntry* const* rot_keys) {
    if (count == 0) fail(kInvalid, "batch plan: empty batch");
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    std::unique_ptr<BatchGraph> g(new BatchGraph);
    const size_t words = pipeline_words(c, count, levels, galois, nullptr, nullptr);
    if (cudaMalloc(&g->d_arena, words * 8) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "batch plan: scratch allocation failed");
    }
    PipelinePlan P;
    plan_pipeline(c, P, count, levels, xb, xa, yb, ya, galois, relin, rot_keys, g->d_arena);
    if (cudaMalloc(&g->d_jobs, std::max<size_t>(P.t.bytes.size(), 16)) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "batch plan: job-table allocation failed");
    }
    check_cuda(cudaMemcpy(g->d_jobs, P.t.bytes.data(), P.t.bytes.size(), cudaMemcpyHostToDevice), "job upload");
    P.t.base = g->d_jobs;
    cudaStream_t ps = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking), "stream");
    uint64_t before[kClsCount], after[kClsCount];
    probe_counts(before);
    check_cuda(cudaStreamBeginCapture(ps, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        launch_pipeline(c, P, ps);
    } catch (...) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(ps, &junk);
        if (junk) cudaGraphDestroy(junk);
        cudaStreamDestroy(ps);
        cudaGetLastError();
        throw;
    }
    const cudaError_t ec = cudaStreamEndCapture(ps, &g->graph);
    probe_counts(after);
    cudaStreamDestroy(ps);
    check_cuda(ec, "end capture");
    check_cuda(cudaGraphInstantiate(&g->exec, g->graph, 0), "graph instantiate");
    for (int k = 0; k < kClsCount; ++k) g->launches[k] = after[k] - before[k];
    return g.release();
}

void batch_graph_launch(BatchGraph& g, cudaStream_t s) {
    check_cuda(cudaGraphLaunch(g.exec, s), "graph launch");
    probe_add(g.launches);
}

}  // namespace wg
