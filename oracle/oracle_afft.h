/* Test infrastructure (oracle): additive-FFT engine declarations. */
#ifndef SCRS_ORACLE_AFFT_H
#define SCRS_ORACLE_AFFT_H

#include "oracle_internal.h"

#define AFFT_MAX_TRANSFORM_SIZE 65536u /* scrs/src/afft/transform.rs:13 */
#define AFFT_TARGETED_MAX_MISSING 5u   /* scrs/src/afft/decoder.rs:578 */

typedef struct {
    size_t size;
    size_t log_size;
    uint16_t* factors; /* heap layout, root at index 1 */
    uint16_t derivative_factors[16];
} afft_plan;

typedef struct {
    size_t k, m, n, L;
    size_t padded_k;
    size_t transform_size;
    afft_plan interp;
    afft_plan transform;
} afft_profile;

int afft_plan_init(afft_plan* plan, size_t size);
void afft_plan_free(afft_plan* plan);
void afft_forward(const afft_plan* plan, uint16_t* values);
void afft_inverse(const afft_plan* plan, uint16_t* values);
void afft_forward_bytes(const afft_plan* p, uint8_t* rows, size_t L);
void afft_inverse_bytes(const afft_plan* p, uint8_t* rows, size_t L);
void afft_forward_bytes_trunc_range(const afft_plan* p, uint8_t* rows, size_t L, size_t active,
                                    size_t rs, size_t re);
void afft_forward_bytes_high_coset_range(const afft_plan* p, uint8_t* rows, size_t L, size_t rs,
                                         size_t re);
void afft_inverse_truncated_bytes(const afft_plan* p, uint8_t* rows, size_t L, size_t active);
void afft_derivative_bytes(const afft_plan* p, const uint8_t* coeffs, size_t L, uint8_t* deriv);

int afft_profile_init(afft_profile* pr, size_t k, size_t m, size_t L);
void afft_profile_free(afft_profile* pr);
void afft_encode_blocked(const afft_profile* p, const uint8_t* data, uint8_t* repairs,
                         size_t width, int fused);
void afft_encode(const afft_profile* p, const uint8_t* data, uint8_t* repairs);
void afft_locator_evaluations(const uint8_t* known, size_t ts, uint16_t* values,
                              uint16_t* derivatives);
void afft_systematic_locator(const afft_profile* p, uint16_t* products, uint16_t* derivs);
void afft_finalize(const afft_profile* p, const uint8_t* have, const uint8_t* payloads,
                   uint8_t* out);

#endif
