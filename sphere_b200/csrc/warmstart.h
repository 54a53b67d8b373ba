// Learned warm start of the Darcy pressure solve (warmstart.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sphb {

struct WarmStart;

// Darcy fields the network reads, ghost-padded (nx+2)(ny+2)(nz+2) doubles,
// and the cells the solve may change (interior, x fastest, 1 = free).
struct WSDarcyInputs {
    const double *p;      // previous solution
    const double *phi, *dphi;
    const unsigned char *free;
};

// nullptr when the device cannot run the tensor-core kernels.  use_net =
// false keeps only the extrapolation (no network, no training).
WarmStart *ws_create(int nx, int ny, int nz, uint64_t seed, int train_solves, bool use_net);
void ws_destroy(WarmStart *w);
// Prediction for this solve: guess = p + free * (the change extrapolated
// from the last solves + the network's correction), on the interior cells
// of the padded guess array; the first solve's guess is p.
// With a network, guess_base (when not null) receives the extrapolation
// alone, so the solve can start from whichever candidate is best.
cudaError_t ws_predict(WarmStart *w, const WSDarcyInputs &in, double *guess, double *guess_base,
                       cudaStream_t st);
// After a solve: while the training budget lasts, Adam steps towards the
// part of the solve's change (p_star - p_prev) that the extrapolation of
// the last prediction missed; then records the change (for the next
// extrapolation and as a network input) and the running scales.
cudaError_t ws_train(WarmStart *w, const double *p_prev, const double *p_star, cudaStream_t st);
int ws_trained(const WarmStart *w);
int ws_predictions(const WarmStart *w);
int ws_error(WarmStart *w, cudaStream_t st);
float ws_last_loss(WarmStart *w, cudaStream_t st);

// test hooks on host arrays: parameters of layer 0..2 (w: [27][16 out][16 in],
// b: [16]), forward of already-normalised 4-channel inputs, and the
// gradients of the mean squared error over free cells
int ws_set_params(WarmStart *w, int layer, const float *wt, const float *b);
int ws_get_params(WarmStart *w, int layer, float *wt, float *b);
int ws_forward_host(WarmStart *w, const float *x3, float *out);
int ws_gradients_host(WarmStart *w, const float *x3, const float *target,
                      const unsigned char *free, float *dw, float *db);

}  // namespace sphb
