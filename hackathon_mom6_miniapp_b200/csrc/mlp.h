// mlp.h -- the barotropic surrogate network (k_mlp.cu): a 175-256-256-2 MLP
// with GELU, BF16 weights and activations, FP32 accumulation on the tcgen05
// tensor cores, FP32 master weights trained with Adam.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace mom6b {

constexpr int kMlpIn = 175;     // 5 x 5 stencil x 7 channels
constexpr int kMlpInPad = 176;  // padded to the MMA K step (16)
constexpr int kMlpHidden = 256;
constexpr int kMlpOut = 2;
constexpr int kMlpChannels = 7; // eta, ubt, vbt, forcing u, forcing v, depth, f

// Flat parameter layout (fp32 master copy, gradients and Adam moments):
// W1 [256][176], b1 [256], W2 [256][256], b2 [256], W3 [2][256], b3 [2].
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpInPad;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kOffB3 + kMlpOut;

// Inputs of one barotropic call, the channels the features read.
struct BtInputs {
    const double *eta, *ubt, *vbt;
};

// The grid quantities the surrogate kernels read.
struct SurGrid {
    Dims D;
    const double *IareaT, *Datu, *Datv, *cor;   // 2-D metrics (cor: CoriolisBu)
    double depth;                               // flat bottom depth [m]
    double dt_total;                            // dtbt * nstep of one barotropic call
    int iu0, iu1, jv0, jv1;                     // transport ranges (serial: is..ie-1, js..je-1)
};

// Features of B sampled columns (cells of the compute domain picked by a
// hash of (seed, sample)) into X [B][176] and XT [176][B], and each sample's
// stencil amplitude into amp [B]; norm holds the 7 inverse channel stds.  The
// dynamic channels (eta, ubt, vbt) are divided by the amplitude, floored by a
// tenth of their RMS over the domain (reduced into gacc, 2 doubles).
cudaError_t launch_sur_features_train(const SurGrid& g, const BtInputs& in, const float* norm,
                                      double* gacc, int B, uint64_t seed, __nv_bfloat16* X,
                                      __nv_bfloat16* XT, float* amp, cudaStream_t s);
// Targets of the same samples: the substep-averaged transports divided by
// their stds (norm[7], norm[8]) and by the sample's amplitude.
cudaError_t launch_sur_targets(const SurGrid& g, const double* uh_avg, const double* vh_avg,
                               const float* norm, const float* amp, int B, uint64_t seed,
                               float* Y, cudaStream_t s);
// Features (and amplitudes) of every compute cell, row (j - js) * nx + (i - is).
cudaError_t launch_sur_features_all(const SurGrid& g, const BtInputs& in, const float* norm,
                                    double* gacc, __nv_bfloat16* X, float* amp, cudaStream_t s);
// eta_out = eta_in - dt_total IareaT div(U, V) in FP64 from the predicted
// transports (outputs times target std times amplitude), and the averaged
// velocities U / Datu, V / Datv.
cudaError_t launch_sur_advance(const SurGrid& g, const float* outi, const float* norm,
                               const float* amp, const double* eta_in, double* eta_out,
                               double* u_av, double* v_av, cudaStream_t s);
// Error of the predicted transports (outi, all compute cells) against the
// substep-averaged transports of the plain btstep: adds sum (pred - true)^2
// and sum true^2 over both components and the compute domain to acc[0], acc[1].
cudaError_t launch_sur_transport_err(const SurGrid& g, const float* outi, const float* norm,
                                     const float* amp, const double* uh_avg,
                                     const double* vh_avg, double* acc, cudaStream_t s);
// Relative L2 difference of two 2-D fields over the compute domain: writes
// sum (a - b)^2 and sum b^2 to acc[0], acc[1] (acc zeroed first).
cudaError_t launch_sur_diff(const Dims& D, const double* a, const double* b, double* acc,
                            cudaStream_t s);

class Mlp {
public:
    Mlp() = default;
    ~Mlp();
    // batch: the largest training batch; seed: weight initialisation
    cudaError_t init(int batch, uint64_t seed, cudaStream_t s);
    // host copies of the fp32 parameters (kMlpParams floats)
    cudaError_t get_params(float* host) const;
    cudaError_t set_params(const float* host);
    // One training step on a batch whose features X (bf16 [B][176]), XT
    // ([176][B]) and targets Y (fp32 [B][2]) are in the object's buffers:
    // forward, loss, backward, Adam.  Returns the loss (before the update)
    // through *loss_dev (device float), no host synchronisation.
    cudaError_t train_step(int B, float lr, cudaStream_t s);
    // Gradient of the loss on the current batch without an update (into the
    // object's gradient buffer).
    cudaError_t gradients(int B, cudaStream_t s);
    cudaError_t grads_to_host(float* host, cudaStream_t s) const;
    // Forward of n rows of Xin (bf16 [n][176], tensor map built by
    // prepare_inference) into out (fp32 [n][2]).
    cudaError_t prepare_inference(int n);
    cudaError_t predict(int n, cudaStream_t s);

    // batch buffers (training)
    __nv_bfloat16 *X = nullptr, *XT = nullptr;  // [B][176], [176][B]
    float* Y = nullptr;                          // targets [B][2]
    float* amp = nullptr;                        // stencil amplitudes of the batch [B]
    double* gacc = nullptr;                      // domain sums of the amplitude floor [2]
    float* out = nullptr;                        // outputs [B][2]
    float* loss = nullptr;                       // [1]: loss of the last train step
    int* err = nullptr;                          // tensor-core wait failures
    // inference buffers
    __nv_bfloat16* Xi = nullptr;                 // [n][176]
    float* outi = nullptr;                       // [n][2]
    float* ampi = nullptr;                       // stencil amplitudes [n]
    int ni_cap = 0;
    int B_cap = 0;
    int64_t steps = 0;                           // Adam steps taken
    // normalisation: feature channel std and target std (host and device)
    float feat_std[kMlpChannels] = {1, 1, 1, 1, 1, 1, 1};
    float targ_std[kMlpOut] = {1, 1};
    float* d_norm = nullptr;                     // [7 feature inverse stds, 2 target stds]
    int launches = 0;

private:
    cudaError_t bf16_copies(cudaStream_t s);
    cudaError_t forward(int B, bool keep, cudaStream_t s);
    cudaError_t backward(int B, cudaStream_t s);
    cudaError_t make_maps(int B);
    int map_B = 0;
    float *P = nullptr, *G = nullptr, *Mo = nullptr, *Vo = nullptr;
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W2Tb = nullptr;
    float* W3r = nullptr;                         // bf16-rounded W3 as fp32
    float *Z1 = nullptr, *Z2 = nullptr;           // pre-activations [B][256]
    __nv_bfloat16 *H1 = nullptr, *H1T = nullptr, *H2 = nullptr;
    __nv_bfloat16 *dZ2 = nullptr, *dZ2T = nullptr, *dZ1T = nullptr;
    float* part = nullptr;                        // split-K partials
    float* bpart = nullptr;                       // per-block partials of the output layer
    __nv_bfloat16* H1i = nullptr;                 // inference hidden [n][256]
    CUtensorMap mX, mH1, mdZ2, mdZ2T, mdZ1T;              // A operands (box 64 x 128)
    CUtensorMap mW1, mW2, mW2T, mH1T_B, mXT_B;            // B operands (box 64 x N)
    CUtensorMap mXi, mH1i;
    bool maps_ok = false, imaps_ok = false;
};

} // namespace mom6b
