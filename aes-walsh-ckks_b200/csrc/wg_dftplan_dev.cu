// Bootstrapping DFT plans built on the context's device: the host generates each stage's
// diagonals (wg_dftplan.cpp), the device encodes them into QP plaintexts in Montgomery form
// straight into the stage's diagonal store.
//
// Reference: encode_sparse_dft_stage, src/ckks/operations/bootstrap/ckks_bootstrap_dft.cpp:
// 777-892.  A term's diagonal is repeated periodically from the active slots to all N/2 slots,
// rotated right by its giant-step offset (index rounded down to a multiple of the baby-step
// count), encoded at the stage's plaintext scale over the Q limbs of the stage's level followed
// by the P limbs, transformed to evaluation form and converted to Montgomery form: the same
// FP64 encoder steps as the reference's (encode_slots_custom_basis_rotated :53-96), so the
// residues are the reference's.
#include <memory>
#include <vector>

#include "wg_batch.hpp"
#include "wg_dftplan.hpp"
#include "wg_internal.hpp"

namespace wg {

std::vector<LtStage*> dft_plan_create(Context& c, const dft::Literal& lit, cudaStream_t s) {
    const std::vector<dft::Stage> stages = dft::generate_plan(lit, c.N, c.q);
    const size_t N = c.N, full = N / 2;
    std::vector<LtStage*> made;
    try {
        for (const dft::Stage& st : stages) {
            std::vector<uint64_t> idx(st.indices.begin(), st.indices.end());
            LtStage* ls = lt_stage_create(c, st.level, idx.size(), idx.data(), nullptr, st.baby, st.slots,
                                          st.rescale_after);
            made.push_back(ls);
            lt_stage_set_plaintext_scale(*ls, st.plaintext_scale);
            const size_t T = st.level + 1 + c.np;
            std::vector<int> mods;
            for (size_t l = 0; l <= st.level; ++l) mods.push_back((int)l);
            for (size_t pi = 0; pi < c.np; ++pi) mods.push_back((int)(c.nq + pi));
            uint64_t* base = lt_stage_data(*ls);
            // encode in chunks of terms (the encoder's scratch is 16 N bytes per plaintext)
            constexpr size_t kChunk = 64;
            std::vector<double> re(kChunk * full), im(kChunk * full);
            std::vector<uint64_t*> outs(kChunk);
            for (size_t t0 = 0; t0 < idx.size(); t0 += kChunk) {
                const size_t n = std::min(kChunk, idx.size() - t0);
                for (size_t k = 0; k < n; ++k) {
                    const size_t term = t0 + k;
                    const std::vector<dft::cplx>& d = st.diagonals[term];
                    const size_t active = d.size();
                    const size_t rot = (idx[term] / st.baby) * st.baby;
                    for (size_t i = 0; i < full; ++i) {
                        const size_t src = ((i + full - rot) & (full - 1)) % active;
                        re[k * full + i] = d[src].real();
                        im[k * full + i] = d[src].imag();
                    }
                    outs[k] = base + term * T * N;
                }
                encode_slots_device_basis(c, n, mods, st.plaintext_scale, re.data(), im.data(), outs.data(), true,
                                          true, s);
            }
        }
    } catch (...) {
        for (LtStage* ls : made) lt_stage_destroy(ls);
        throw;
    }
    return made;
}

}  // namespace wg
