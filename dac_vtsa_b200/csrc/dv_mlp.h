// dv_mlp.h -- the learned Newton predictor's network object, shared by dv_mlp.cu and the integrator.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "dacvtsa.h"

namespace dv {
namespace mlp {

// Architecture: NIN inputs (NFEAT used, the rest zero) -> NH -> NH -> NH (tanh) -> NOUT outputs (NOUT_USED
// used).  All widths are multiples of 16 (tcgen05 K and N granularity).
constexpr int NIN = 112, NH = 128, NOUT = 16, NOUT_USED = 6, NFEAT = 97;
constexpr int NB = 4096;       // training batch (samples)
constexpr int NSPLIT = 8;      // K splits of the weight-gradient products (NB / NSPLIT samples each)
// parameter vector (fp32): W1 [NH x NIN], b1 [NH], W2 [NH x NH], b2, W3 [NH x NH], b3, W4 [NOUT x NH], b4 [NOUT]
constexpr int64_t OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
                  OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH * NH, OFF_W4 = OFF_B3 + NH,
                  OFF_B4 = OFF_W4 + NOUT * NH, NPARAM = OFF_B4 + NOUT;
// normalisation constants (doubles): [0,6) level scales, [6,12) spatial-difference scales, [12] scale of
// the solver-unit features, [13,19) output scale per variable, [19] target clip
constexpr int NNORM = DV_MLP_NNORM;
}  // namespace mlp
}  // namespace dv

struct dv_mlp {
    // fp32 master parameters, their gradient and Adam moments (device)
    float *P = nullptr, *G = nullptr, *Mo = nullptr, *Vo = nullptr;
    // bf16 operand copies in panel layout: forward W (rows = outputs) and transposed W (rows = inputs)
    __nv_bfloat16 *W1 = nullptr, *W2 = nullptr, *W3 = nullptr, *W4 = nullptr;
    __nv_bfloat16 *W2t = nullptr, *W3t = nullptr, *W4t = nullptr;
    double* norm = nullptr;                     // device copy of the normalisation constants
    double norm_h[dv::mlp::NNORM];
    // recorded training samples: features (panel layout, cap rows) and raw targets [cap][8]
    __nv_bfloat16* Xs = nullptr;
    float* Ts = nullptr;
    int64_t cap = 0, count = 0;
    // training batch buffers
    __nv_bfloat16 *Xb = nullptr, *Xbt = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr, *H1t = nullptr,
                  *H2t = nullptr, *H3t = nullptr, *D4 = nullptr, *D4t = nullptr, *D3 = nullptr, *D2 = nullptr,
                  *D1 = nullptr, *D3t = nullptr, *D2t = nullptr, *D1t = nullptr;
    float *Tb = nullptr, *part = nullptr, *bpart = nullptr, *lossp = nullptr;
    // inference buffers (rows = cells rounded up to 128), sized by dv_mlp_reserve
    int64_t inf_rows = 0;
    __nv_bfloat16 *Xi = nullptr, *Ha = nullptr, *Hb = nullptr;
    float* Oi = nullptr;
    int* d_err = nullptr;
    int64_t adam_t = 0;
    float* h_loss = nullptr;                    // pinned: loss partials of the last step
};

namespace dv {
namespace mlp {
// Inputs of the feature kernel for one implicit stage: the two latest states A (at t_A) and B (at
// t_A - dt_ab) and the right-hand side fA at A; the stage's target time is t_A + dt_tgt.
struct StageInputs {
    int32_t Nr, Nth, Nz;
    int64_t nc;
    const double* A;
    const double* B;
    const double* fA;
    const double* atol7;
    double rtol, dt_tgt, dt_ab, h;
    int32_t stage, step_code;
};
// Features of every cell into the inference buffer, forward pass, and pred[v*nc + c] += the network's
// correction (scaled) for the 6 cell unknowns, truncated to >= 0.1 max(ytr, 0) for c and q.
int predict(dv_mlp* net, const StageInputs& in, const double* ytr, double* pred, cudaStream_t s);
// Features of cells first + j*stride (j < cnt) into sample rows net->count + j.
int record_features(dv_mlp* net, const StageInputs& in, int64_t first, int64_t stride, int64_t cnt, cudaStream_t s);
// Targets (z* - z_ext)/s of the same cells into rows net->count + j; then net->count += cnt.
int record_targets(dv_mlp* net, const StageInputs& in, const double* zstar, const double* zext, int64_t first,
                   int64_t stride, int64_t cnt, cudaStream_t s);
}  // namespace mlp
}  // namespace dv
