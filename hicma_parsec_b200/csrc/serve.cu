// One serving request through the C ABI: generate -> band fix / auto-tune ->
// factor -> log-likelihood, on a descriptor that lives only for the call.
//
// No counterpart in the reference, whose driver stops at the factor
// (hicma_parsec/testing_dpotrf.c:830-903); the steps before the factorization
// follow that driver: STARSH_gen (:459-470), rank gather and statistics
// (:476-500), band auto-tuning and regeneration (:531-575), HiCMA_dpotrf_L
// (:783-789).  Host code only: every step is a public entry point of the
// library, so the result is the one a caller making the same calls gets.
#include <algorithm>
#include <string>
#include <vector>

#include "tlr_internal.h"

extern "C" int hicma_tlr_serve_loglik(hicma_tlr_ctx *ctx, const hicma_tlr_problem *prob, int N, int NB,
                                      double acc, int maxrank, int autoband, const double *y, double *loglik,
                                      double *logdet, double *x, int *band) {
    if (!ctx || !prob || !y || !loglik || !logdet || N <= 0 || NB <= 0 || acc <= 0.0) {
        tlr::tlr_set_error("invalid argument: serve_loglik arguments");
        return HICMA_TLR_ERR_ARG;
    }
    if (N % NB != 0) {
        tlr::tlr_set_error("invalid argument: N must be a multiple of NB");
        return HICMA_TLR_ERR_ARG;
    }
    const int NT = N / NB;
    const int cap = maxrank > 0 ? maxrank : std::min(NB / 2 - 1, 200);
    if (cap < 1) {
        tlr::tlr_set_error("invalid argument: NB too small for a low-rank tile");
        return HICMA_TLR_ERR_ARG;
    }
    hicma_tlr_desc *A = nullptr;
    int rc = hicma_tlr_desc_create(ctx, N, NB, cap, 1, &A);
    if (rc) return rc;
    std::vector<int> gen((size_t)NT * NT), G((size_t)NT * NT);
    int info = 0, b = 1;
    rc = hicma_tlr_generate(ctx, HICMA_TLR_LOWER, A, gen.data(), prob, nullptr, acc, cap, 1, 0, &info);
    if (!rc) rc = hicma_tlr_rank_gather(ctx, A, G.data(), 1);
    if (!rc) {
        if (info != 0) {
            // tiles the rank rule rejected (rank -1) become dense: widen the band over them
            b = 2;
            for (int m = 1; m < NT; ++m)
                for (int n = 0; n < m; ++n)
                    if (gen[(size_t)n * NT + m] < 0) b = std::max(b, m - n + 1);
        } else if (autoband) {
            b = std::max(b, hicma_tlr_band_autotune(G.data(), NT, NB, 0));
        }
        b = std::min(b, NT);
        if (b > 1) rc = hicma_tlr_band_regenerate(ctx, HICMA_TLR_LOWER, A, prob, b);
    }
    int finfo = 0;
    if (!rc) {
        int la = -1, two = 0;
        double cpt[6] = {0};
        finfo = hicma_tlr_dpotrf_L(ctx, HICMA_TLR_LOWER, A, nullptr, acc, 0, cap, &la, b, NB, cap, 0, &two,
                                   nullptr, nullptr, cpt, 0);
        if (finfo < 0) rc = finfo;
    }
    if (!rc && finfo == 0) rc = hicma_tlr_loglik(ctx, A, y, loglik, logdet, x);
    if (band) *band = b;
    const std::string err = rc ? hicma_tlr_last_error() : "";
    hicma_tlr_desc_destroy(A);
    if (rc) {
        tlr::tlr_set_error(err.c_str());
        return rc;
    }
    return finfo;
}
