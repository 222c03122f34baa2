/*
 * libsemisim_b200 - training kernels of the learned sweep predictor (b200m_*).
 *
 * No counterpart in the reference (it has no learned component).  These run the network's
 * forward pass with saved activations, its backward pass and Adam on the GPU, on device
 * buffers the caller owns (any allocator: the training driver in
 * semiconductor_devices_simulator_b200/learned.py uses PyTorch tensors).  All pointers are
 * device pointers; `stream` is a cudaStream_t (null: the legacy default stream).
 *
 * Sizes: MI = 48 features, MH = 128 hidden units (3 layers), MO = 8 outputs (3 used).
 *   P     FP32 parameters [nparam]: W1 [MH][MI], b1 [MH], W2 [MH][MH], b2, W3, b3,
 *         W4 [MO][MH] (rows 3-7 zero), b4 [MO]
 *   Wb    BF16 weight pack [nwb] (W1, W2, W3, W4), bias FP32 [nbias] (b1 | b2 | b3 | b4)
 *   X     BF16 features [B][MI];  Y FP32 outputs [B][MO];  T FP32 targets [B][3]
 *   Z     FP32 pre-activations [3][B][MH];  H BF16 activations [3][B][MH]
 *   dZ    BF16 scratch [3][B][MH];  dY BF16 scratch [B][MO];  G FP32 gradient [nparam]
 * Every call returns 1, or 0 when the launch failed.
 */
#ifndef SEMISIM_B200_LEARNED_H
#define SEMISIM_B200_LEARNED_H

#ifdef __cplusplus
extern "C" {
#endif

/* nparam, nwb, nbias of the network */
int b200m_mlp_sizes(int *nparam, int *nwb, int *nbias);
/* features of every node of the current instance's device from two solutions x1 (now)
   and x0 (one step back), the extrapolation ratio s and the step's contact voltage
   changes dv4 (host array of 4, volts): X [N][48] BF16 */
int b200m_seed_features(const double *psi1, const double *phin1, const double *phip1, const double *psi0,
                        const double *phin0, const double *phip0, double s, const double *dv4, void *X,
                        void *stream);
/* Wb and bias from P */
int b200m_mlp_pack(const float *P, void *Wb, float *bias, void *stream);
/* forward of B rows with saved activations */
int b200m_mlp_forward(const void *X, int B, const void *Wb, const float *bias, float *Y, float *Z, void *H,
                      void *stream);
/* gradient of the mean squared error over B x 3 added into G (zero it first); the loss
   added into *loss (device float) */
int b200m_mlp_backward(const void *X, int B, const void *Wb, const float *Y, const float *T, const float *Z,
                       const void *H, void *dZ, void *dY, float *G, float *loss, void *stream);
/* one Adam step (step count t >= 1, betas 0.9 / 0.999, eps 1e-8) on P, moments M and V;
   refreshes Wb and bias */
int b200m_mlp_adam(float *P, const float *G, float *M, float *V, float lr, int t, void *Wb, float *bias,
                   void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SEMISIM_B200_LEARNED_H */
