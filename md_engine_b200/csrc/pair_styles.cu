// The per-site pair kernel's forms for the pair evaluators beyond LJ/cut and
// WCA -- force-shifted LJ (FixLJCutFS.cu, PairEvaluatorLJFS.h), CHARMM LJ
// with 1-4 parameters (FixLJCHARMM.cu, PairEvaluatorCHARMM.h), TICG
// (FixTICG.cu, PairEvaluatorTICG.h) -- and for the damped shifted force
// charge term (FixChargePairDSF.cu, ChargeEvaluatorDSF.h) with any of them;
// compiled apart from pair.cu so that the two build in parallel.
#include "pair_kernel.cuh"

namespace mdx {
namespace pk {

namespace {

template <int T>
int styles_kind(const PairArgs &A, const PairArgs *tab, int nrep, int lj, int ck, bool vir, bool energy, bool acc,
                cudaStream_t st) {
    switch (lj * 3 + ck) {
        case 0 * 3 + 2: launch_t<T, 0, 2>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 1 * 3 + 2: launch_t<T, 1, 2>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 2 * 3 + 2: launch_t<T, 2, 2>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 3 * 3 + 0: launch_t<T, 3, 0>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 3 * 3 + 1: launch_t<T, 3, 1>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 3 * 3 + 2: launch_t<T, 3, 2>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 4 * 3 + 0: launch_t<T, 4, 0>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 4 * 3 + 1: launch_t<T, 4, 1>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 4 * 3 + 2: launch_t<T, 4, 2>(A, tab, nrep, vir, energy, acc, st); return 0;
        case 5 * 3 + 0: launch_t<T, 5, 0>(A, tab, nrep, vir, energy, acc, st); return 0;
    }
    set_error(MDX_ERR_UNSUPPORTED, "pair evaluator %d with charge evaluator %d is not built", lj, ck);
    return MDX_ERR_UNSUPPORTED;
}

}  // namespace

int pair_launch_styles(const PairArgs &A, const PairArgs *tab, int nrep, int team, int lj, int ck, bool vir,
                       bool energy, bool acc, cudaStream_t st) {
    switch (team) {
        case 1: return styles_kind<1>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 2: return styles_kind<2>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 4: return styles_kind<4>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 8: return styles_kind<8>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 16: return styles_kind<16>(A, tab, nrep, lj, ck, vir, energy, acc, st);
        case 32: return styles_kind<32>(A, tab, nrep, lj, ck, vir, energy, acc, st);
    }
    set_error(MDX_ERR_ARG, "team size %d not in {1,2,4,8,16,32}", team);
    return MDX_ERR_ARG;
}

}  // namespace pk
}  // namespace mdx
