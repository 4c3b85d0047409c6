// Prints the engine's constant tables as JSON, for the test that pins them to
// the reference's source text (tests/test_reference_constants.py).  Host code
// only: it calls the engine's __host__ __device__ constexpr tables and its
// stochastic-rounding hash, and launches nothing, so it runs without a GPU.
// stdin: a count, then that many "key seed" pairs to hash.
#include <cstdio>

#include "../simlab_b200/csrc/d3q27.h"
#include "../simlab_b200/csrc/lbm_device.cuh"

int main() {
    std::printf("{\"d3q19\": {\"c\": [");
    for (int i = 0; i < 19; i++) std::printf("%s[%d, %d, %d]", i ? ", " : "", lbm::CX(i), lbm::CY(i), lbm::CZ(i));
    std::printf("], \"opp\": [");
    for (int i = 0; i < 19; i++) std::printf("%s%d", i ? ", " : "", lbm::OPP(i));
    std::printf("], \"weight\": [");
    for (int i = 0; i < 19; i++) std::printf("%s%.17g", i ? ", " : "", lbm::WD(i));
    std::printf("], \"record\": {\"RS\": %u, \"R_MASK\": %u, \"R_CELL\": %u, \"R_Q\": %u, \"R_FPOST\": %u, \"R_MACRO\": %u, \"R_FT\": %u}",
                lbm::RS, lbm::R_MASK, lbm::R_CELL, lbm::R_Q, lbm::R_FPOST, lbm::R_MACRO, lbm::R_FT);
    std::printf(", \"fp16_scale\": %.17g}, \"step_seed_mul\": %u", (double)lbm::FP16_SCALE, lbm::STEP_SEED_MUL);
    std::printf(", \"d3q27\": {\"c\": [");
    for (int i = 0; i < 27; i++) std::printf("%s[%d, %d, %d]", i ? ", " : "", lbm27::CX(i), lbm27::CY(i), lbm27::CZ(i));
    std::printf("], \"opp\": [");
    for (int i = 0; i < 27; i++) std::printf("%s%d", i ? ", " : "", lbm27::OPP27(i));
    std::printf("], \"slot\": [");
    for (int i = 0; i < 27; i++) std::printf("%s%d", i ? ", " : "", lbm27::SLOT(i));
    std::printf("], \"weight\": [");
    for (int i = 0; i < 27; i++) std::printf("%s%.17g", i ? ", " : "", lbm27::WD(i));
    std::printf("], \"record\": {\"RS\": %u, \"R_MASK\": %u, \"R_CELL\": %u, \"R_Q\": %u, \"R_FT\": %u, \"MW\": %u, \"T_FLUID\": %u, "
                "\"T_SOLID\": %u, \"T_FACE\": %u, \"T_GHOST\": %u, \"T_RESTRICT\": %u}",
                lbm27::RS, lbm27::R_MASK, lbm27::R_CELL, lbm27::R_Q, lbm27::R_FT, lbm27::MW, lbm27::T_FLUID, lbm27::T_SOLID,
                lbm27::T_FACE, lbm27::T_GHOST, lbm27::T_RESTRICT);
    std::printf(", \"seed\": {\"src_mul\": %u, \"mw_mul\": %u}}", lbm27::SEED_SRC_MUL, lbm27::SEED_MW_MUL);
    unsigned n = 0;
    if (std::scanf("%u", &n) != 1) n = 0;
    std::printf(", \"sr_hash\": [");
    for (unsigned k = 0; k < n; k++) {
        unsigned key = 0, seed = 0;
        if (std::scanf("%u %u", &key, &seed) != 2) break;
        std::printf("%s[%u, %u, %u]", k ? ", " : "", key, seed, lbm::sr_hash(key, seed));
    }
    std::printf("]}\n");
    return 0;
}
