/*
 * Per-configuration drop-in library, named like the reference's
 * lib/libmsm_{curve}_{c}_{alpha}_{debug}.so (core/src/msm.rs:101-112; curve
 * bn254 or bls12381 as in core/src/msm/xmake.lua's target list), whose
 * window size and target window count are fixed at build time exactly as the
 * reference's Makefile.msm bakes MSM_WINDOW_SIZE / MSM_TARGET_WINDOWS /
 * MSM_DEBUG into each of its 2,880 targets.  It exports the reference's two
 * symbols (core/src/msm/src/msm.h:4-11) and forwards to libimpeller_msm.so,
 * where the window size is a runtime parameter.
 */
#include "impeller_msm.h"

#ifndef MSM_WINDOW_SIZE
#error "MSM_WINDOW_SIZE must be defined"
#endif
#ifndef MSM_TARGET_WINDOWS
#error "MSM_TARGET_WINDOWS must be defined"
#endif
#ifndef MSM_DEBUG
#define MSM_DEBUG 0
#endif
#ifndef MSM_CURVE_ID
#define MSM_CURVE_ID IMPELLER_CURVE_BN254
#endif

cudaError_t msm(void *const *buffers, unsigned long *buffer_sizes, unsigned long long len,
                unsigned int batch_per_run, unsigned int parts, unsigned int stage_scalers,
                unsigned int stage_points, unsigned int num_cards, const unsigned int *cards,
                unsigned int const *const *h_points, unsigned int batches,
                unsigned int const *const *h_scaler_batch, unsigned int *const *h_result) {
    return impeller_msm_cfg_curve(MSM_CURVE_ID, MSM_WINDOW_SIZE, MSM_TARGET_WINDOWS, MSM_DEBUG, buffers,
                                  buffer_sizes, len, batch_per_run, parts, stage_scalers, stage_points, num_cards,
                                  cards, h_points, batches, h_scaler_batch, h_result);
}

cudaError_t msm_precompute(unsigned long long len, unsigned int *const *h_points, unsigned int max_cards) {
    return impeller_msm_precompute_cfg_curve(MSM_CURVE_ID, MSM_WINDOW_SIZE, MSM_TARGET_WINDOWS, len, h_points,
                                             max_cards);
}
