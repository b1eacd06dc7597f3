/*
 * C ABI of the B200 number-theoretic transform (BN254 Fr and the other
 * 8-limb fields), a drop-in for the reference's NTT library.
 *
 * The reference loads lib/libntt.so (core/src/ntt.rs:23, 98-106), built from
 * core/src/ntt/src/ntt.cu for one field chosen at build time (NTT_FIELD,
 * default bn254_fr, core/src/ntt/xmake.lua:1-12), and binds the five symbols
 * of core/src/ntt/src/ntt.h:5-16.  libimpeller_msm.so exports the same five
 * symbols for BN254 Fr (the default field), plus field-selecting variants.
 *
 * Layout (the reference's): a field element is 8 little-endian u32 limbs in
 * Montgomery form (R = 2^256); a polynomial is `len` elements.  PolyPtr is the
 * reference's view of a possibly rotated or sliced device array
 * (core/src/common/iter/src/iter.cuh:12-18, core/src/poly_ptr.rs:5-11):
 * logical element i lives at ptr[(start + i) mod whole_len] with
 * start = len - rotate when rotate != 0, else offset.
 */
#ifndef IMPELLER_NTT_H
#define IMPELLER_NTT_H

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct PolyPtr {
    unsigned int *ptr;
    size_t len;
    size_t rotate;
    size_t offset;
    size_t whole_len;
} PolyPtr;

/* core/src/common/slice/poly_slice.h:4-12: element i of a slice maps to
 * (begin + i) mod len of the underlying polynomial. */
typedef struct PolySlice {
    unsigned long long begin, slice_len, len;
} PolySlice;

/* Fields (the reference's NTT_FIELD values with 8 limbs). */
#define IMPELLER_NTT_BN254_FR 0
#define IMPELLER_NTT_BN254_FQ 1
#define IMPELLER_NTT_BLS12381_FR 2

/* In-place forward NTT of x (len = 2^log_len, natural order in and out):
 * X[k] = sum_j x[j] w^(j k), twiddle[i] = w^i for i < len / 2 on the device
 * (ssip_precompute makes it).  Asynchronous on `stream`.  The two
 * max_threads_*_log arguments are the reference's launch-shape knobs; they
 * are checked (at most 10) and do not change the result.
 * Replaces ntt.h:6 (core/src/ntt/src/ssip_ntt.cuh:500-567). */
cudaError_t ssip_ntt(PolyPtr x, const unsigned int *twiddle, unsigned int log_len, cudaStream_t stream,
                     const unsigned int max_threads_stage1_log, const unsigned int max_threads_stage2_log);

/* twiddle[i] = unit^i for i < len, host arrays (unit: one element).
 * Blocking.  (The reference names the second argument log_len but passes
 * the table length, core/src/ntt.rs:226-231.)  Replaces ntt.h:9. */
cudaError_t ssip_precompute(unsigned int *twiddle, unsigned int len, const unsigned int *unit);

/* The same transform as ssip_ntt with twiddles recomputed on the device from
 * omegas[i] = w^(2^i) (32 elements, device) instead of a len/2 table: extra
 * device memory is a constant 192 KiB (three 2048-entry power tables), not
 * proportional to len.  pq / pq_deg are the reference's small-root table
 * (gen_pq_omegas); they are checked for consistency of pq_deg and are not
 * otherwise read.  Replaces ntt.h:12 (core/src/ntt/src/recompute_ntt.cuh:364-439). */
cudaError_t recompute_ntt(PolyPtr x, const unsigned int *pq_d, unsigned int pq_deg, const unsigned int *omegas_d,
                          unsigned int log_len, cudaStream_t stream, const unsigned int max_threads_stage1_log,
                          const unsigned int max_threads_stage2_log);

/* Host tables for recompute_ntt: pq[i] = (unit^(len >> pq_deg))^i for
 * i < 2^(pq_deg-1), omegas[i] = unit^(2^i) for i < 32.  Blocking (computed
 * on the current device).  Replaces ntt.h:15 (precompute.cuh:100-125). */
void gen_pq_omegas(unsigned int *pq, unsigned int *omegas, unsigned int pq_deg, unsigned int len, unsigned int *unit);

/* poly[i] *= powers[poly_slice->to_origin(i) mod power_num] for i < poly.len
 * (device arrays).  Asynchronous.  Replaces ntt.h:18
 * (core/src/ntt/src/distribute_powers.cuh:5-19). */
cudaError_t distribute_powers(PolyPtr poly, const unsigned int *powers, unsigned long long power_num,
                              cudaStream_t stream, const PolySlice *poly_slice);

/* The same five operations on a chosen field (IMPELLER_NTT_*). */
cudaError_t impeller_ntt(int field, PolyPtr x, const unsigned int *twiddle, unsigned int log_len,
                         cudaStream_t stream);
cudaError_t impeller_ntt_precompute(int field, unsigned int *twiddle, unsigned int len, const unsigned int *unit);
cudaError_t impeller_ntt_recompute(int field, PolyPtr x, const unsigned int *omegas_d, unsigned int log_len,
                                   cudaStream_t stream);
cudaError_t impeller_ntt_gen_pq_omegas(int field, unsigned int *pq, unsigned int *omegas, unsigned int pq_deg,
                                       unsigned int len, const unsigned int *unit);
cudaError_t impeller_ntt_distribute_powers(int field, PolyPtr poly, const unsigned int *powers,
                                           unsigned long long power_num, cudaStream_t stream,
                                           const PolySlice *poly_slice);

/* Kernel launches one ssip_ntt of 2^log_len elements makes (passes plus the
 * reordering pass). */
unsigned int impeller_ntt_launches(unsigned int log_len);

#ifdef __cplusplus
}
#endif

#endif
