// Rotation, conjugation and relinearisation switching keys generated on the device.
//
// Reference: generate_rotation_key_hybrid (src/ckks/context/rotation_key_generation.cpp:92-199),
// generate_conjugation_key_hybrid (src/ckks/context/conjugation_key_generation.cpp:63-167) and
// encrypt_rlk_hybrid (src/ckks/context/relinearization_key_generation.cpp:131-199, which
// encrypts P s^2 with ckks_encrypt_custom_eval: the same form with x = s^2, y = s).
// For each non-empty part of the hybrid decomposition (alpha = ceil(L / dnum) Q limbs each) and
// every QP limb m:
//     b = [limb in the part] (P mod m) x + e - a y,   then a and b times fold_m * 2^64 (mod m)
// with (x, y) = (s, pi_{-r}(s)) for a rotation by r and (conj(s), s) for the conjugation, x and y
// the NTTs of the secret's images, `a` uniform in the evaluation domain and `e` one small integer
// polynomial per part (the same integers in every limb) after its NTT.  fold_m is P^-1 mod q for
// Q limbs and (P / p_j)^-1 mod p_j for P limbs (ckks_fold_hybrid_switch_key_constants) and 2^64
// the Montgomery radix (ckks_convert_switch_key_to_montgomery_inplace); the reference multiplies
// by the two constants one after the other, which gives the same canonical residue as one
// multiplication by their product.
//
// The mask and the noise may come from the caller (then the key is a pure function of its
// inputs and matches the reference's construction residue for residue), or be drawn on the
// device: `a` uniform modulo each limb from SplitMix64 (Steele, Lea and Flood, 2014) over a
// per-key stream, with rejection; `e` the rounded Box-Muller normal of standard deviation sigma,
// cut at 12 sigma.  SplitMix64 is a statistical generator, not a cryptographic one (the reference
// draws with std::mt19937_64, also not cryptographic): a production key generator feeds its own
// randomness through `a` and `e`.
#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/walsh_gpu.h"
#include "wg_batch.hpp"
#include "wg_batch_kernels.cuh"
#include "wg_internal.hpp"

namespace wg {
using namespace bk;

namespace {

struct SecretJob {
    const int8_t* src;
    uint64_t* dst;
    int mod, pad;
};

struct NoiseJob {
    const int64_t* src;
    uint64_t* dst;
    int mod, pad;
};

struct UniformJob {
    uint64_t* dst;
    uint64_t stream;
    int mod, pad;
};

struct AssembleJob {
    const uint64_t* a_in;
    const uint64_t* x;
    const uint64_t* y;
    const uint64_t* e;
    uint64_t* a_out;
    uint64_t* b_out;
    uint64_t pm;  // P mod m on the part's own Q limbs, 0 elsewhere
    uint64_t c;   // fold constant times the Montgomery radix, mod m
    int mod, square;  // square: x times x (relinearisation key)
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// small signed integers (secret coefficients) as canonical residues
__global__ void __launch_bounds__(kT) kb_secret_limbs(const SecretJob* jobs, int n, const Modulus* mods) {
    const SecretJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    const int v = j->src[k];
    j->dst[k] = v >= 0 ? (uint64_t)v % q : (q - (uint64_t)(-v) % q) % q;
}

// reduce_i64_mod_q of the noise integers
__global__ void __launch_bounds__(kT) kb_noise_limbs(const NoiseJob* jobs, int n, const Modulus* mods) {
    const NoiseJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    const int64_t v = j->src[k];
    j->dst[k] = v >= 0 ? (uint64_t)v % q : (q - (uint64_t)(-(v + 1)) % q - 1) % q;
}

// uniform residues mod q: the low bits(q) bits of successive SplitMix64 outputs of the
// coefficient's counter, first one below q (at most 64 draws; each is accepted with probability
// above 1/2, and the last resort reduces)
__global__ void __launch_bounds__(kT) kb_uniform(const UniformJob* jobs, int n, const Modulus* mods, uint64_t seed) {
    const UniformJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const uint64_t q = mods[j->mod].q;
    const int bits = 64 - __clzll((long long)q);
    const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    uint64_t ctr = seed ^ (j->stream * 0xD1B54A32D192ED03ull) ^ ((uint64_t)k << 7);
    uint64_t v = 0;
    for (int t = 0; t < 64; ++t) {
        v = splitmix64(ctr + (uint64_t)t) & mask;
        if (v < q) break;
    }
    j->dst[k] = v < q ? v : v % q;
}

// rounded normal noise of standard deviation sigma, cut at 12 sigma
__global__ void __launch_bounds__(kT) kb_gauss(int64_t* out, size_t count, uint64_t seed, uint64_t stream,
                                               double sigma) {
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    if (k >= count) return;
    const uint64_t base = seed ^ (stream * 0x9E6C63D0676A9A99ull) ^ ((uint64_t)k << 9);
    const uint64_t r1 = splitmix64(base), r2 = splitmix64(base + 1);
    const double u1 = ((double)(r1 >> 11) + 1.0) * 0x1p-53;  // (0, 1]
    const double u2 = (double)(r2 >> 11) * 0x1p-53;          // [0, 1)
    double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2) * sigma;
    const double cut = 12.0 * sigma;
    z = z > cut ? cut : (z < -cut ? -cut : z);
    out[k] = llrint(z);
}

__global__ void __launch_bounds__(kT) kb_key_assemble(const AssembleJob* jobs, int n, const Modulus* mods) {
    const AssembleJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->mod];
    const uint64_t q = m.q;
    const uint64_t a = j->a_in[k];
    const uint64_t xv = j->square ? barrett_mul(j->x[k], j->x[k], m) : j->x[k];
    uint64_t b = j->pm ? barrett_mul(xv, j->pm, m) : 0;
    b = add_mod(b, j->e[k], q);
    b = sub_mod(b, barrett_mul(a, j->y[k], m), q);
    j->b_out[k] = barrett_mul(b, j->c, m);
    j->a_out[k] = barrett_mul(a, j->c, m);
}

struct EncryptJob {
    uint64_t* b;          // out
    const uint64_t* a;    // mask (evaluation form)
    const uint64_t* pt;   // plaintext (evaluation form)
    const uint64_t* e;    // noise limb (evaluation form)
    const uint64_t* s;    // secret limb (evaluation form)
    int mod, pad;
};

// ckks_encrypt_custom_eval: b = pt + e - a s
__global__ void __launch_bounds__(kT) kb_encrypt(const EncryptJob* jobs, int n, const Modulus* mods) {
    const EncryptJob* j = job_of(jobs, n);
    if (!j) return;
    const size_t k = (size_t)blockIdx.x * kT + threadIdx.x;
    const Modulus m = mods[j->mod];
    const uint64_t q = m.q;
    j->b[k] = sub_mod(add_mod(j->pt[k], j->e[k], q), barrett_mul(j->a[k], j->s[k], m), q);
}

uint64_t inv_mod(uint64_t a, uint64_t m) { return host::powmod(a % m, m - 2, m); }  // m prime

// apply_automorphism_to_secret: coefficient i moves to i * index mod 2N, negated past N
std::vector<int8_t> automorph_secret(const int8_t* s, size_t N, uint64_t index) {
    std::vector<int8_t> y(N, 0);
    for (size_t i = 0; i < N; ++i) {
        const size_t m = (size_t)(((unsigned __int128)i * index) % (2 * N));
        y[m >= N ? m - N : m] = m >= N ? (int8_t)-s[i] : s[i];
    }
    return y;
}

template <class Job, class Kernel>
void run_jobs(Context& c, const std::vector<Job>& jobs, Kernel kernel, double bytes_per_job, cudaStream_t s) {
    if (jobs.empty()) return;
    JobTable t;
    const Job* j = t.add(jobs);
    t.upload(c, s);
    Probe probe(kClsElementwise, bytes_per_job * (double)jobs.size(), s);
    kernel<<<grid_for(c, jobs.size()), kT, 0, s>>>(t.at(j), (int)jobs.size(), c.d_mod);
    check_cuda(cudaGetLastError(), "key generation");
}

// Shape of a key: the moduli of its limbs (table indices), per limb P mod m (used on the own Q
// limbs of a part) and the fold-and-radix constant, the parts' own Q limb ranges.
struct KeyShape {
    std::vector<int> mods;
    std::vector<uint64_t> pm, cst;
    std::vector<std::pair<size_t, size_t>> ranges;
    size_t key_level = 0;
};

uint64_t radix_mod(uint64_t m) { return (uint64_t)(((unsigned __int128)1 << 64) % m); }

// every Q limb and P limb, the context's hybrid parts (ckks_fold_hybrid_switch_key_constants
// over all P moduli)
KeyShape full_shape(const Context& c) {
    KeyShape k;
    const size_t L = c.nq, K = c.np;
    for (size_t i = 0; i < L + K; ++i) {
        const uint64_t m = i < L ? c.q[i] : c.p[i - L];
        uint64_t prod = 1, phat = 1;
        for (size_t j = 0; j < K; ++j) {
            prod = host::mulmod(prod, c.p[j] % m, m);
            if (i >= L && j != i - L) phat = host::mulmod(phat, c.p[j] % m, m);
        }
        k.mods.push_back((int)i);  // P limbs follow the Q limbs in the modulus table
        k.pm.push_back(prod);
        k.cst.push_back(host::mulmod(i < L ? inv_mod(prod, m) : inv_mod(phat, m), radix_mod(m), m));
    }
    for (size_t part = 0; part < c.parts_at(L - 1); ++part)
        k.ranges.push_back({part * c.alpha, std::min((part + 1) * c.alpha, L)});
    k.key_level = L - 1;
    return k;
}

// the compact level-0 key over (q0, p0) (generate_secret_key_switch_key_q0p0_hybrid: the
// plaintext is the source times p0 on q0, folded over {q0} and {p0} alone)
KeyShape q0p0_shape(const Context& c) {
    KeyShape k;
    const uint64_t q0 = c.q[0], p0 = c.p[0];
    k.mods = {0, (int)c.nq};
    k.pm = {p0 % q0, 0};
    k.cst = {host::mulmod(inv_mod(p0 % q0, q0), radix_mod(q0), q0), radix_mod(p0)};
    k.ranges = {{0, 1}};
    k.key_level = 0;
    return k;
}

// b = P x + e - a y per part and limb (x squared limb by limb when `square`), then a and b
// times the limb's constant; returns the device key [part][a|b][limbs][N]
KeyEntry build_key(Context& c, const KeyShape& k, const std::vector<int8_t>& x, const std::vector<int8_t>& y,
                   bool square, const uint64_t* a_host, const int64_t* e_host, uint64_t key_seed, double sigma,
                   uint64_t* out_host, cudaStream_t s) {
    const size_t N = c.N, T = k.mods.size(), parts = k.ranges.size();
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    // device scratch: x, y limbs [2][T][N], mask [parts][T][N], noise limbs [parts][T][N], the
    // noise integers [parts][N] and the secrets' bytes [2][N]
    const size_t limb_words = T * N;
    const size_t words = 2 * limb_words + 2 * parts * limb_words + parts * N + (2 * N + 7) / 8;
    uint64_t* ws = nullptr;
    if (cudaMallocAsync((void**)&ws, words * 8, s) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "wg_keygen: scratch allocation failed");
    }
    uint64_t* dx = ws;
    uint64_t* dy = dx + limb_words;
    uint64_t* da = dy + limb_words;
    uint64_t* de = da + parts * limb_words;
    int64_t* dei = reinterpret_cast<int64_t*>(de + parts * limb_words);
    int8_t* dsec = reinterpret_cast<int8_t*>(dei + parts * N);
    const size_t key_words = parts * 2 * limb_words;
    KeyEntry entry;
    entry.parts = parts;
    entry.key_level = k.key_level;
    if (cudaMalloc((void**)&entry.d_data, key_words * 8) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(ws, s);
        fail(kNoMemory, "wg_keygen: key allocation failed");
    }
    try {
        check_cuda(cudaMemcpyAsync(dsec, x.data(), N, cudaMemcpyHostToDevice, s), "wg_keygen upload");
        check_cuda(cudaMemcpyAsync(dsec + N, y.data(), N, cudaMemcpyHostToDevice, s), "wg_keygen upload");
        if (a_host) {
            check_cuda(cudaMemcpyAsync(da, a_host, parts * limb_words * 8, cudaMemcpyHostToDevice, s), "wg_keygen upload");
            check_cuda(cudaMemcpyAsync(dei, e_host, parts * N * 8, cudaMemcpyHostToDevice, s), "wg_keygen upload");
        }
        std::vector<SecretJob> sec;
        std::vector<NttJob> ntt;
        for (size_t i = 0; i < T; ++i) {
            sec.push_back({dsec, dx + i * N, k.mods[i], 0});
            sec.push_back({dsec + N, dy + i * N, k.mods[i], 0});
            ntt.push_back({dx + i * N, dx + i * N, k.mods[i], 0});
            ntt.push_back({dy + i * N, dy + i * N, k.mods[i], 0});
        }
        std::vector<UniformJob> uni;
        std::vector<NoiseJob> noise;
        for (size_t part = 0; part < parts; ++part)
            for (size_t i = 0; i < T; ++i) {
                uni.push_back({da + (part * T + i) * N, (uint64_t)(part * T + i), k.mods[i], 0});
                noise.push_back({dei + part * N, de + (part * T + i) * N, k.mods[i], 0});
                ntt.push_back({de + (part * T + i) * N, de + (part * T + i) * N, k.mods[i], 0});
            }
        run_jobs(c, sec, kb_secret_limbs, 9.0 * N, s);
        if (!a_host) {
            JobTable t;
            const UniformJob* j = t.add(uni);
            t.upload(c, s);
            {
                Probe probe(kClsElementwise, 8.0 * N * uni.size(), s);
                kb_uniform<<<grid_for(c, uni.size()), kT, 0, s>>>(t.at(j), (int)uni.size(), c.d_mod, key_seed);
            }
            const size_t count = parts * N;
            kb_gauss<<<(unsigned)((count + kT - 1) / kT), kT, 0, s>>>(dei, count, key_seed, 0x5EEDull, sigma);
            check_cuda(cudaGetLastError(), "wg_keygen sampling");
        }
        run_jobs(c, noise, kb_noise_limbs, 16.0 * N, s);
        {
            JobTable t;
            const NttJob* j = t.add(ntt);
            t.upload(c, s);
            ntt_jobs(c, t.at(j), (int)ntt.size(), true, s);
        }
        std::vector<AssembleJob> asm_jobs;
        for (size_t part = 0; part < parts; ++part) {
            const size_t s0 = k.ranges[part].first, s1 = k.ranges[part].second;
            uint64_t* key_a = entry.d_data + (part * 2 + 0) * limb_words;
            uint64_t* key_b = entry.d_data + (part * 2 + 1) * limb_words;
            for (size_t i = 0; i < T; ++i) {
                AssembleJob jb;
                jb.a_in = da + (part * T + i) * N;
                jb.x = dx + i * N;
                jb.y = dy + i * N;
                jb.e = de + (part * T + i) * N;
                jb.a_out = key_a + i * N;
                jb.b_out = key_b + i * N;
                jb.pm = (i >= s0 && i < s1) ? k.pm[i] : 0;
                jb.c = k.cst[i];
                jb.mod = k.mods[i];
                jb.square = square ? 1 : 0;
                asm_jobs.push_back(jb);
            }
        }
        run_jobs(c, asm_jobs, kb_key_assemble, 48.0 * N, s);
        if (out_host)
            check_cuda(cudaMemcpyAsync(out_host, entry.d_data, key_words * 8, cudaMemcpyDeviceToHost, s),
                       "wg_keygen download");
        check_cuda(cudaFreeAsync(ws, s), "wg_keygen scratch");
        ws = nullptr;
        check_cuda(cudaStreamSynchronize(s), "wg_keygen");
    } catch (...) {
        if (ws) cudaFreeAsync(ws, s);
        cudaStreamSynchronize(s);
        cudaFree(entry.d_data);
        throw;
    }
    return entry;
}

void install_key(Context& c, int kind, int64_t r, const KeyEntry& entry) {
    auto it = c.keys.find({kind, r});
    if (it != c.keys.end()) {
        cudaFree(it->second.d_data);
        it->second = entry;
    } else {
        c.keys.emplace(std::make_pair(kind, r), entry);
    }
}

void check_ternary(const int8_t* s, size_t N, const char* what) {
    if (!s) throw std::invalid_argument(std::string("wg_keygen: null ") + what);
    for (size_t i = 0; i < N; ++i)
        if (s[i] < -1 || s[i] > 1) throw std::invalid_argument(std::string("wg_keygen: ") + what + " must be ternary");
}

}  // namespace

void keygen_switch_key(Context& c, int kind, int64_t rotation, const int8_t* secret, const uint64_t* a_host,
                       const int64_t* e_host, uint64_t seed, double sigma, uint64_t* out_host, cudaStream_t s) {
    if (kind != WG_KEY_ROTATION && kind != WG_KEY_CONJ && kind != WG_KEY_RELIN)
        throw std::invalid_argument("wg_keygen: only rotation, conjugation and relinearisation keys are generated");
    check_ternary(secret, c.N, "secret");
    if (!a_host != !e_host) throw std::invalid_argument("wg_keygen: give both the mask and the noise, or neither");
    if (!a_host && !(sigma > 0.0 && sigma < 1e6)) throw std::invalid_argument("wg_keygen: invalid noise deviation");
    const size_t N = c.N, slots = N / 2;
    int64_t r = 0;
    if (kind == WG_KEY_ROTATION) {
        r = rotation % (int64_t)slots;
        if (r < 0) r += (int64_t)slots;
        if (r == 0) throw std::invalid_argument("wg_keygen: zero rotation needs no key");
    }
    // (x, y): b = P x + e - a y
    std::vector<int8_t> x, y;
    if (kind == WG_KEY_ROTATION) {
        x.assign(secret, secret + N);
        // rotation_automorphism_index(N, -r) = 5^(slots - r) mod 2N
        y = automorph_secret(secret, N, host::powmod(5, (uint64_t)((int64_t)slots - r) % slots, 2 * N));
    } else if (kind == WG_KEY_RELIN) {
        x.assign(secret, secret + N);  // squared limb by limb in the evaluation domain
        y.assign(secret, secret + N);
    } else {
        x = automorph_secret(secret, N, 2 * N - 1);
        y.assign(secret, secret + N);
    }
    // distinct streams per key (kind, rotation) so that keys of one seed differ
    const uint64_t key_seed = seed ^ ((uint64_t)kind << 56) ^ ((uint64_t)r * 0xA24BAED4963EE407ull);
    const KeyEntry entry = build_key(c, full_shape(c), x, y, kind == WG_KEY_RELIN, a_host, e_host, key_seed, sigma,
                                     out_host, s);
    install_key(c, kind, r, entry);
}

void keygen_secret_switch(Context& c, int kind, const int8_t* source, const int8_t* target, const uint64_t* a_host,
                          const int64_t* e_host, uint64_t seed, double sigma, uint64_t* out_host, cudaStream_t s) {
    if (kind != WG_KEY_DENSE_TO_SPARSE && kind != WG_KEY_SPARSE_TO_DENSE)
        throw std::invalid_argument("wg_keygen: secret switches are dense-to-sparse or sparse-to-dense");
    check_ternary(source, c.N, "source secret");
    check_ternary(target, c.N, "target secret");
    if (!a_host != !e_host) throw std::invalid_argument("wg_keygen: give both the mask and the noise, or neither");
    if (!a_host && !(sigma > 0.0 && sigma < 1e6)) throw std::invalid_argument("wg_keygen: invalid noise deviation");
    const std::vector<int8_t> x(source, source + c.N), y(target, target + c.N);
    const uint64_t key_seed = seed ^ ((uint64_t)kind << 56) ^ 0x3C6EF372FE94F82Bull;
    const KeyShape k = kind == WG_KEY_DENSE_TO_SPARSE ? q0p0_shape(c) : full_shape(c);
    const KeyEntry entry = build_key(c, k, x, y, false, a_host, e_host, key_seed, sigma, out_host, s);
    install_key(c, kind, 0, entry);
}

void encrypt_symmetric(Context& c, size_t count, size_t level, const uint64_t* const* pts, const int8_t* secret,
                       const uint64_t* a_host, const int64_t* e_host, uint64_t seed, double sigma,
                       uint64_t* const* out_b, uint64_t* const* out_a, cudaStream_t s) {
    if (count == 0) return;
    if (level >= c.nq) throw std::invalid_argument("ckks_encrypt: invalid level");
    check_ternary(secret, c.N, "secret");
    if (!a_host != !e_host) throw std::invalid_argument("wg_encrypt: give both the mask and the noise, or neither");
    if (!a_host && !(sigma > 0.0 && sigma < 1e6)) throw std::invalid_argument("wg_encrypt: invalid noise deviation");
    const size_t N = c.N, L = level + 1;
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice");
    constexpr size_t kChunk = 128;  // ciphertexts per pass (bounds the noise scratch)
    const size_t chunk = std::min(count, kChunk);
    // scratch: secret limbs [L][N], noise limbs [chunk][L][N], noise integers [chunk][N], secret bytes
    const size_t words = L * N + chunk * L * N + chunk * N + (N + 7) / 8;
    uint64_t* ws = nullptr;
    if (cudaMallocAsync((void**)&ws, words * 8, s) != cudaSuccess) {
        cudaGetLastError();
        fail(kNoMemory, "wg_encrypt: scratch allocation failed");
    }
    uint64_t* ds = ws;
    uint64_t* de = ds + L * N;
    int64_t* dei = reinterpret_cast<int64_t*>(de + chunk * L * N);
    int8_t* dsec = reinterpret_cast<int8_t*>(dei + chunk * N);
    try {
        check_cuda(cudaMemcpyAsync(dsec, secret, N, cudaMemcpyHostToDevice, s), "wg_encrypt upload");
        std::vector<SecretJob> sec;
        std::vector<NttJob> sntt;
        for (size_t l = 0; l < L; ++l) {
            sec.push_back({dsec, ds + l * N, (int)l, 0});
            sntt.push_back({ds + l * N, ds + l * N, (int)l, 0});
        }
        run_jobs(c, sec, kb_secret_limbs, 9.0 * N, s);
        {
            JobTable t;
            const NttJob* j = t.add(sntt);
            t.upload(c, s);
            ntt_jobs(c, t.at(j), (int)sntt.size(), true, s);
        }
        for (size_t c0 = 0; c0 < count; c0 += chunk) {
            const size_t nc = std::min(chunk, count - c0);
            std::vector<UniformJob> uni;
            std::vector<NoiseJob> noise;
            std::vector<NttJob> entt;
            std::vector<EncryptJob> enc;
            for (size_t i = 0; i < nc; ++i)
                for (size_t l = 0; l < L; ++l) {
                    uni.push_back({out_a[c0 + i] + l * N, (uint64_t)((c0 + i) * L + l), (int)l, 0});
                    noise.push_back({dei + i * N, de + (i * L + l) * N, (int)l, 0});
                    entt.push_back({de + (i * L + l) * N, de + (i * L + l) * N, (int)l, 0});
                    enc.push_back({out_b[c0 + i] + l * N, out_a[c0 + i] + l * N, pts[c0 + i] + l * N,
                                   de + (i * L + l) * N, ds + l * N, (int)l, 0});
                }
            if (a_host) {
                for (size_t i = 0; i < nc; ++i)
                    check_cuda(cudaMemcpyAsync(out_a[c0 + i], a_host + (c0 + i) * L * N, L * N * 8,
                                               cudaMemcpyHostToDevice, s), "wg_encrypt upload");
                check_cuda(cudaMemcpyAsync(dei, e_host + c0 * N, nc * N * 8, cudaMemcpyHostToDevice, s),
                           "wg_encrypt upload");
            } else {
                const uint64_t key_seed = seed ^ 0x6A09E667F3BCC909ull ^ ((uint64_t)level << 48);
                JobTable t;
                const UniformJob* j = t.add(uni);
                t.upload(c, s);
                {
                    Probe probe(kClsElementwise, 8.0 * N * uni.size(), s);
                    kb_uniform<<<grid_for(c, uni.size()), kT, 0, s>>>(t.at(j), (int)uni.size(), c.d_mod, key_seed);
                }
                kb_gauss<<<(unsigned)((nc * N + kT - 1) / kT), kT, 0, s>>>(dei, nc * N, key_seed, (uint64_t)c0 + 1,
                                                                          sigma);
                check_cuda(cudaGetLastError(), "wg_encrypt sampling");
            }
            run_jobs(c, noise, kb_noise_limbs, 16.0 * N, s);
            {
                JobTable t;
                const NttJob* j = t.add(entt);
                t.upload(c, s);
                ntt_jobs(c, t.at(j), (int)entt.size(), true, s);
            }
            run_jobs(c, enc, kb_encrypt, 40.0 * N, s);
            // the next chunk's uploads and draws reuse the noise scratch only after this one
            // has been consumed (stream order)
        }
        check_cuda(cudaFreeAsync(ws, s), "wg_encrypt scratch");
        ws = nullptr;
        check_cuda(cudaStreamSynchronize(s), "wg_encrypt");
    } catch (...) {
        if (ws) cudaFreeAsync(ws, s);
        cudaStreamSynchronize(s);
        throw;
    }
}

}  // namespace wg
