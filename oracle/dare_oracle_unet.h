/*
 * dare_oracle_unet.h -- CPU restatement of the learned linear preconditioner
 * (TEST INFRASTRUCTURE ONLY; see dare_oracle_unet.c).
 *
 * Parameters are FP32, layer after layer (enc0, enc1, enc2, enc3, dec3, dec2,
 * dec1, dec0), each [27][cout][cin].  Vectors are over the internal cells,
 * ordinal (i*n1 + j)*n2 + k; activations [cell][channel].
 */
#ifndef DARE_ORACLE_UNET_H_
#define DARE_ORACLE_UNET_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int64_t dor_unet_num_params(void);
/* z = u + U(u); acts (optional) receives S0, P1, S1, P2, S2, P3, E3 back to back. */
int dor_unet_forward(const int n[3], const float* w, const double* u, int bf16, double* z, double* acts);
/* mean over pairs of ||N(r_b) - e_b||^2 / ||e_b||^2 and its gradient (num_params doubles, may be NULL). */
int dor_unet_loss_grad(const int n[3], const float* w, const double* r, const double* e, int count, int bf16,
                       double* loss, double* grad);

#ifdef __cplusplus
}
#endif
#endif
