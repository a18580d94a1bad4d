// dv_mlp.cu -- the learned Newton predictor: a per-cell network whose BF16 products run on the sm_100a
// tensor cores (tcgen05.mma, FP32 accumulation in tensor memory), with its own forward, backward and
// Adam kernels.
//
// The reference starts every implicit stage from an extrapolation (core/solver.py:420 for stage 1,
// :432/:435 for stage 2): a straight line through the two latest states to the stage's time.  The
// network adds a per-cell correction to that line, predicted from the cell's and its six face
// neighbours' states at those two levels, the right-hand side at the latest level, the step-size
// ratio, the stage and the cycle step.  It is trained on stage solutions the plain solver itself
// produced; the integrator starts Newton from whichever of the two guesses has the smaller scaled
// residual, so the unchanged Newton tolerance decides the converged state in both cases.
//
// Products (all M = 128 rows per CTA, N <= 128 columns, K in chunks of 64 staged through a two-deep
// shared-memory ring by cp.async, one elected thread issuing the MMAs and committing to an mbarrier):
//   forward   H1 = tanh(X W1^T + b1), H2, H3 likewise, O = H3 W4^T + b4
//   backward  D4 = dL/dO, D3 = (D4 W4) * (1 - H3^2), D2 = (D3 W3) * (1 - H2^2), D1 = (D2 W2) * (1 - H1^2)
//             dW4^T = H3^T D4, dW3 = D3^T H2, dW2 = D2^T H1, dW1 = D1^T X (K = samples, split over CTAs)
// Every activation and gradient is written in both panel layouts (rows = samples for the next forward /
// backward product, rows = features for the weight-gradient product).
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include "dv_internal.h"
#include "dv_mlp.h"
#include "dv_umma.cuh"

using bf16 = __nv_bfloat16;

namespace dv {
namespace mlp {

using namespace dv::umma;

enum { E_TANH = 0, E_OUT = 1, E_LOSS = 2, E_DTANH = 3, E_PART = 4 };

struct GemmP {
    const bf16* A;
    int64_t ra;           // rows of A's panel layout
    const bf16* B;
    int64_t rb;           // rows of B's panel layout (rows 0..N-1 used)
    int N;                // 16..128, multiple of 16
    int kpanels;          // K / 8 handled by one CTA (even)
    int split;            // 1: blockIdx.x selects a K range (weight gradients); 0: an M tile
    int mode;
    int64_t rows_valid;   // rows at or beyond this are written as zero and carry no loss
    const float* bias;
    bf16* orm;            // output, panel layout with rows = samples (orm_r rows)
    int64_t orm_r;
    bf16* ofm;            // output, panel layout with rows = features (ofm_r rows), K = samples
    int64_t ofm_r;
    float* of;            // fp32 output (E_OUT rows x ldf; E_PART partials)
    int64_t ldf;
    const bf16* hd;       // E_DTANH: activation (panel layout, rows = samples, hd_r rows)
    int64_t hd_r;
    const float* tgt;     // E_LOSS: targets [rows][8]
    float dscale;         // E_LOSS: dL/dO = dscale * (O - target)
    float* lossp;         // E_LOSS: per-CTA sum of squared errors
    float* bsum;          // E_LOSS / E_DTANH: per-CTA column sums of the written gradient [grid][N]
    int* err;
};

constexpr int KCH = 8;                         // panels per staged K chunk (64 columns)
constexpr uint32_t STAGE_A = KCH * 128 * 16;   // 16 KB
constexpr uint32_t STAGE_B = KCH * 128 * 16;   // 16 KB (N <= 128)
constexpr uint32_t GEMM_SMEM = 2 * (STAGE_A + STAGE_B);
// allocation with a guard band: a descriptor whose leading and stride offsets were read the other way
// round (row groups 2 KB apart) still addresses only memory of this CTA
constexpr uint32_t GEMM_SMEM_ALLOC = GEMM_SMEM + 65536;

__device__ __forceinline__ float bf2f(bf16 x) { return __bfloat162float(x); }

__global__ void __launch_bounds__(128) k_gemm(GemmP g) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_s;
    __shared__ float red[4][16];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int N = g.N;
    const int64_t m0 = g.split ? 0 : (int64_t)blockIdx.x * 128;
    const int64_t kp0 = g.split ? (int64_t)blockIdx.x * g.kpanels : 0;
    const int nch = (g.kpanels + KCH - 1) / KCH;
    const uint32_t sb = smem_u32(smem);
    const uint32_t sA[2] = {sb, sb + STAGE_A};
    const uint32_t sB[2] = {sb + 2 * STAGE_A, sb + 2 * STAGE_A + STAGE_B};
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    if (warp == 0) tmem_alloc(smem_u32(&tmem_s), ncols);
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_s;
    const uint32_t idesc = idesc_bf16_m128(N);

    auto load = [&](int c, int s) {
        const int pc = min(KCH, g.kpanels - c * KCH);
        const int64_t kp = kp0 + (int64_t)c * KCH;
        for (int idx = tid; idx < pc * 128; idx += 128) {
            const int p = idx >> 7, r = idx & 127;
            cp_async16(sA[s] + p * 2048 + r * 16, g.A + ((kp + p) * g.ra + m0 + r) * 8);
        }
        for (int idx = tid; idx < pc * N; idx += 128) {
            const int p = idx / N, r = idx - p * N;
            cp_async16(sB[s] + p * (N * 16) + r * 16, g.B + ((kp + p) * g.rb + r) * 8);
        }
        cp_async_commit();
    };
    bool ok = true;
    load(0, 0);
    for (int c = 0; c < nch; ++c) {
        const int s = c & 1;
        if (c + 1 < nch) {
            if (c >= 1 && !mbar_wait(s ? bar0 : bar1, (uint32_t)(((c - 1) >> 1) & 1))) ok = false;
            load(c + 1, s ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
            const int pc = min(KCH, g.kpanels - c * KCH);
            for (int q = 0; q < pc / 2; ++q) {
                const uint64_t da = sdesc(sA[s] + q * 2 * 2048, 2048, 128);
                const uint64_t db = sdesc(sB[s] + q * 2 * (N * 16), N * 16, 128);
                mma_bf16(tmem, da, db, idesc, (c > 0 || q > 0) ? 1u : 0u);
            }
            mma_commit(s ? bar1 : bar0);
        }
    }
    const int last = nch - 1;
    if (!mbar_wait((last & 1) ? bar1 : bar0, (uint32_t)((last >> 1) & 1))) ok = false;
    ok = __syncthreads_and(ok ? 1 : 0) != 0;     // one verdict for the whole CTA (the epilogue has barriers)
    fence_after_sync();
    if (!ok) {
        atomicOr(g.err, 8);
        // the products may still run: give them one more bounded wait before the memory is released
        mbar_wait((last & 1) ? bar1 : bar0, (uint32_t)((last >> 1) & 1));
    }
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    const int64_t row = m0 + tid;
    float lsum = 0.0f;
    for (int c0 = 0; c0 < N && ok; c0 += 16) {
        float v[16];
        tmem_ld16(trow + c0, v);
        if (g.mode == E_PART) {
            float* o = g.of + ((int64_t)blockIdx.x * 128 + tid) * N + c0;
#pragma unroll
            for (int i = 0; i < 16; ++i) o[i] = v[i];
            continue;
        }
        if (g.mode == E_OUT) {
            if (row < g.rows_valid) {
                float* o = g.of + row * g.ldf + c0;
#pragma unroll
                for (int i = 0; i < 16; ++i) o[i] = v[i] + g.bias[c0 + i];
            }
            continue;
        }
        const bool live = row < g.rows_valid;
        float w[16];
        if (g.mode == E_TANH) {
#pragma unroll
            for (int i = 0; i < 16; ++i) w[i] = live ? tanhf(v[i] + g.bias[c0 + i]) : 0.0f;
        } else if (g.mode == E_DTANH) {
            const uint4* hp0 = reinterpret_cast<const uint4*>(g.hd + pidx(row, c0, g.hd_r));
            const uint4* hp1 = reinterpret_cast<const uint4*>(g.hd + pidx(row, c0 + 8, g.hd_r));
            uint4 hv[2] = {*hp0, *hp1};
            const bf16* hb = reinterpret_cast<const bf16*>(hv);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float h = bf2f(hb[i]);
                w[i] = live ? v[i] * (1.0f - h * h) : 0.0f;
            }
        } else {   // E_LOSS
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = c0 + i;
                float d = 0.0f;
                if (live && n < NOUT_USED) d = (v[i] + g.bias[n]) - g.tgt[row * 8 + n];
                lsum += d * d;
                w[i] = g.dscale * d;
            }
        }
        bf16 wb[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) wb[i] = __float2bfloat16_rn(w[i]);
        if (g.orm) {
            *reinterpret_cast<uint4*>(g.orm + pidx(row, c0, g.orm_r)) = *reinterpret_cast<const uint4*>(wb);
            *reinterpret_cast<uint4*>(g.orm + pidx(row, c0 + 8, g.orm_r)) = *reinterpret_cast<const uint4*>(wb + 8);
        }
        if (g.ofm) {
#pragma unroll
            for (int i = 0; i < 16; ++i) g.ofm[pidx(c0 + i, row, g.ofm_r)] = wb[i];
        }
        if (g.bsum) {   // column sums of the bf16-rounded gradient, in a fixed order
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float x = bf2f(wb[i]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0) red[warp][i] = x;
            }
            __syncthreads();
            if (tid < 16)
                g.bsum[(int64_t)blockIdx.x * N + c0 + tid] = ((red[0][tid] + red[1][tid]) + red[2][tid]) + red[3][tid];
            __syncthreads();
        }
    }
    if (g.mode == E_LOSS && g.lossp) {
        float x = lsum;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        __syncthreads();
        if (lane == 0) red[warp][0] = x;
        __syncthreads();
        if (tid == 0) g.lossp[blockIdx.x] = ((red[0][0] + red[1][0]) + red[2][0]) + red[3][0];
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

static int gemm(const GemmP& g, int grid, cudaStream_t s) {
    DV_CUDA(dv::allow_dyn_smem((const void*)k_gemm));
    DV_LAUNCH(dv::K_MLP, s, k_gemm<<<grid, 128, GEMM_SMEM_ALLOC, s>>>(g));
    return launch_ok("k_gemm");
}

// ------------------------------------------------------------------------------------ features
__device__ __forceinline__ double fasinh(double x) { return asinh(x); }

// Feature row of cell c (see the file comment): levels, spatial differences at A, changes A - B at the
// seven stencil points and dt_tgt f(A) in the solver's error-scale units of the cell, the extrapolation
// ratio, log10 h, the stage, the cycle step one-hot and a constant 1.
__device__ void cell_features(const StageInputs& in, const double* __restrict__ nrm, int64_t c, float* f) {
    const int k = (int)(c % in.Nz);
    const int64_t rr = c / in.Nz;
    const int j = (int)(rr % in.Nth);
    const int i = (int)(rr / in.Nth);
    const int64_t nc = in.nc;
    int64_t nb[7];
    nb[0] = c;
    nb[1] = k > 0 ? c - 1 : c;
    nb[2] = k < in.Nz - 1 ? c + 1 : c;
    nb[3] = i > 0 ? c - (int64_t)in.Nth * in.Nz : c;
    nb[4] = i < in.Nr - 1 ? c + (int64_t)in.Nth * in.Nz : c;
    const int jm = j > 0 ? j - 1 : in.Nth - 1, jp = j < in.Nth - 1 ? j + 1 : 0;
    nb[5] = ((int64_t)i * in.Nth + jm) * in.Nz + k;
    nb[6] = ((int64_t)i * in.Nth + jp) * in.Nz + k;
    const double ts = nrm[12];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        const double a0 = in.A[v * nc + c];
        const double sc = in.atol7[v] + in.rtol * fabs(a0);
        f[v] = (float)fasinh(a0 / nrm[v]);
#pragma unroll
        for (int p = 1; p < 7; ++p) f[6 + (p - 1) * 6 + v] = (float)fasinh((in.A[v * nc + nb[p]] - a0) / nrm[6 + v]);
#pragma unroll
        for (int p = 0; p < 7; ++p) {
            const int64_t q = v * nc + nb[p];
            f[42 + p * 6 + v] = (float)fasinh((in.A[q] - in.B[q]) / sc / ts);
        }
        f[84 + v] = (float)fasinh(in.dt_tgt * in.fA[v * nc + c] / sc / ts);
    }
    f[90] = (float)fmin(in.dt_tgt / in.dt_ab, 10.0);
    f[91] = (float)(log10(in.h) / 4.0);
    f[92] = (float)in.stage;
#pragma unroll
    for (int q = 0; q < 4; ++q) f[93 + q] = in.step_code == q ? 1.0f : 0.0f;
}

__global__ void k_features(StageInputs in, const double* __restrict__ nrm, int64_t first, int64_t stride,
                           int64_t cnt, bf16* __restrict__ X, int64_t xr, int64_t row0) {
    const int64_t jj = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= cnt) return;
    const int64_t c = first + jj * stride;
    float f[NIN];
#pragma unroll
    for (int q = 0; q < NIN; ++q) f[q] = 0.0f;
    cell_features(in, nrm, c, f);
    const int64_t row = row0 + jj;
#pragma unroll
    for (int p = 0; p < NIN / 8; ++p) {
        bf16 wb[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) wb[q] = __float2bfloat16_rn(f[p * 8 + q]);
        *reinterpret_cast<uint4*>(X + pidx(row, p * 8, xr)) = *reinterpret_cast<const uint4*>(wb);
    }
}

// The network's correction of the extrapolated start, per cell and variable, in units of that
// cell's extrapolated increment |z_ext - A| plus 1 % of the error scale s: the extrapolation error
// grows with the local rate of change (fronts, blowdown) and vanishes in quiet stages, so a target
// in fixed error-scale units would give the network a constant error floor that quiet stages, where
// the extrapolation is already close, cannot afford.
__device__ __forceinline__ double increment_unit(double zext, double a, double sc) { return fabs(zext - a) + 1e-2 * sc; }

// pred[v][c] = max(pred + out * oscale_v * unit, 0.1 max(ytr, 0)) (the floor for c and q only).
// Corrections smaller than nrm[20] increment units are not applied: where the extrapolation is
// already close (most cells of most stages, within a few percent of the increment) the network's
// own error is of the same size, and leaving those cells alone keeps its gain at the fronts.
__global__ void k_apply(StageInputs in, const double* __restrict__ nrm, const float* __restrict__ O,
                        const double* __restrict__ ytr, double* __restrict__ pred) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= in.nc) return;
    const double gate = nrm[20];
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        const int64_t q = v * in.nc + c;
        const double sc = in.atol7[v] + in.rtol * fabs(in.A[q]);
        const double corr = (double)O[c * NOUT + v] * nrm[13 + v];
        if (fabs(corr) < gate) continue;
        double z = pred[q] + corr * increment_unit(pred[q], in.A[q], sc);
        if (v < 5) z = fmax(z, 0.1 * fmax(ytr[q], 0.0));
        pred[q] = z;
    }
}

__global__ void k_targets(StageInputs in, const double* __restrict__ zs, const double* __restrict__ ze, int64_t first,
                          int64_t stride, int64_t cnt, float* __restrict__ T, int64_t row0) {
    const int64_t jj = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= cnt) return;
    const int64_t c = first + jj * stride;
    float* t = T + (row0 + jj) * 8;
#pragma unroll
    for (int v = 0; v < 6; ++v) {
        const int64_t q = v * in.nc + c;
        const double sc = in.atol7[v] + in.rtol * fabs(in.A[q]);
        t[v] = (float)((zs[q] - ze[q]) / increment_unit(ze[q], in.A[q], sc));
    }
    t[6] = 1.0f;
    t[7] = 0.0f;
}

// ------------------------------------------------------------------------------------ training
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Batch rows j < NB: sample idx(j) (a hash of seed, step and j, or j itself when seed < 0) copied in
// both layouts, targets scaled by the output scales and clipped.
__global__ void k_gather(const bf16* __restrict__ Xs, int64_t cap, const float* __restrict__ Ts, int64_t count,
                         int64_t seed, int64_t step, const double* __restrict__ nrm, bf16* __restrict__ Xb,
                         bf16* __restrict__ Xbt, float* __restrict__ Tb) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)NB * (NIN / 8)) return;
    const int64_t j = t / (NIN / 8);
    const int p = (int)(t - j * (NIN / 8));
    const int64_t s = seed < 0 ? j : (int64_t)(mix64((uint64_t)seed * 0x9e3779b97f4a7c15ull + (uint64_t)step * 1000003ull +
                                                     (uint64_t)j) % (uint64_t)count);
    const uint4 v = *reinterpret_cast<const uint4*>(Xs + pidx(s, p * 8, cap));
    *reinterpret_cast<uint4*>(Xb + pidx(j, p * 8, NB)) = v;
    const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
    for (int q = 0; q < 8; ++q) Xbt[pidx(p * 8 + q, j, NIN)] = e[q];
    if (p == 0) {
        const double clip = nrm[19];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            float x = q < NOUT_USED ? (float)fmax(-clip, fmin(clip, (double)Ts[s * 8 + q] / nrm[13 + q])) : 0.0f;
            Tb[j * 8 + q] = x;
        }
    }
}

// Gradient of parameter q: the weight-gradient partials (or the bias column sums) summed in CTA order.
__device__ float param_grad(int64_t q, const float* __restrict__ part, const float* __restrict__ bsum) {
    // part: [4 products][NSPLIT][128][128] ; bsum: [4 layers][NB/128][128]
    const int64_t PS = (int64_t)NSPLIT * 128 * 128, TB = NB / 128;
    float g = 0.0f;
    int layer = -1, m = 0, n = 0, nn = 0;
    bool bias = false;
    if (q < OFF_B1) { layer = 0; m = (int)(q / NIN); n = (int)(q % NIN); nn = NIN; }
    else if (q < OFF_W2) { layer = 0; bias = true; n = (int)(q - OFF_B1); nn = NH; }
    else if (q < OFF_B2) { layer = 1; m = (int)((q - OFF_W2) / NH); n = (int)((q - OFF_W2) % NH); nn = NH; }
    else if (q < OFF_W3) { layer = 1; bias = true; n = (int)(q - OFF_B2); nn = NH; }
    else if (q < OFF_B3) { layer = 2; m = (int)((q - OFF_W3) / NH); n = (int)((q - OFF_W3) % NH); nn = NH; }
    else if (q < OFF_W4) { layer = 2; bias = true; n = (int)(q - OFF_B3); nn = NH; }
    else if (q < OFF_B4) {   // W4[o][h] = dW4^T[h][o]
        layer = 3;
        const int o = (int)((q - OFF_W4) / NH), h = (int)((q - OFF_W4) % NH);
        m = h; n = o; nn = NOUT;
    } else { layer = 3; bias = true; n = (int)(q - OFF_B4); nn = NOUT; }
    if (bias) {
        const int w = layer == 3 ? NOUT : NH;
        for (int64_t b = 0; b < TB; ++b) g += bsum[layer * TB * 128 + b * w + n];
    } else {
        for (int sp = 0; sp < NSPLIT; ++sp) g += part[layer * PS + ((int64_t)sp * 128 + m) * nn + n];
    }
    return g;
}

__global__ void k_collect_grad(const float* __restrict__ part, const float* __restrict__ bsum, float* __restrict__ G) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < NPARAM) G[q] = param_grad(q, part, bsum);
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ Mo, float* __restrict__ Vo,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= NPARAM) return;
    const float g = G[q];
    const float m = b1 * Mo[q] + (1.0f - b1) * g;
    const float v = b2 * Vo[q] + (1.0f - b2) * g * g;
    Mo[q] = m;
    Vo[q] = v;
    P[q] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// bf16 operand copies of the fp32 parameters: W (rows = outputs) and W^T (rows = inputs) panels
__global__ void k_pack_weights(const float* __restrict__ P, bf16* W1, bf16* W2, bf16* W3, bf16* W4, bf16* W2t, bf16* W3t,
                               bf16* W4t) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < (int64_t)NH * NIN) {
        const int m = (int)(q / NIN), n = (int)(q % NIN);
        W1[pidx(m, n, NH)] = __float2bfloat16_rn(P[OFF_W1 + q]);
    }
    if (q < (int64_t)NH * NH) {
        const int m = (int)(q / NH), n = (int)(q % NH);
        const bf16 a = __float2bfloat16_rn(P[OFF_W2 + q]), b = __float2bfloat16_rn(P[OFF_W3 + q]);
        W2[pidx(m, n, NH)] = a;
        W2t[pidx(n, m, NH)] = a;
        W3[pidx(m, n, NH)] = b;
        W3t[pidx(n, m, NH)] = b;
    }
    if (q < (int64_t)NOUT * NH) {
        const int o = (int)(q / NH), h = (int)(q % NH);
        const bf16 a = __float2bfloat16_rn(P[OFF_W4 + q]);
        W4[pidx(o, h, NOUT)] = a;
        W4t[pidx(h, o, NH)] = a;
    }
}

static unsigned g1(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

static int pack(dv_mlp* net, cudaStream_t s) {
    // one thread per entry of the largest matrix (W2, W3: NH x NH)
    const int64_t most = std::max<int64_t>((int64_t)NH * NIN, std::max<int64_t>((int64_t)NH * NH, (int64_t)NOUT * NH));
    DV_LAUNCH(dv::K_MLP, s, k_pack_weights<<<g1(most), 256, 0, s>>>(net->P, net->W1, net->W2, net->W3, net->W4, net->W2t,
                                                                     net->W3t, net->W4t));
    return launch_ok("k_pack_weights");
}

static GemmP base(dv_mlp* net) {
    GemmP g;
    memset(&g, 0, sizeof g);
    g.err = net->d_err;
    return g;
}

// Forward + backward of one batch (rows of Xb/Xbt/Tb); leaves the gradient in net->G and the loss
// partials in net->lossp.
static int grad_batch(dv_mlp* net, int64_t rows_valid, cudaStream_t s) {
    const int TB = NB / 128;
    GemmP g = base(net);
    g.rows_valid = rows_valid;
    // H1 = tanh(X W1^T + b1)
    g.A = net->Xb; g.ra = NB; g.B = net->W1; g.rb = NH; g.N = NH; g.kpanels = NIN / 8; g.mode = E_TANH;
    g.bias = net->P + OFF_B1; g.orm = net->H1; g.orm_r = NB; g.ofm = net->H1t; g.ofm_r = NH;
    DV_TRY(gemm(g, TB, s));
    g.A = net->H1; g.B = net->W2; g.kpanels = NH / 8; g.bias = net->P + OFF_B2; g.orm = net->H2; g.ofm = net->H2t;
    DV_TRY(gemm(g, TB, s));
    g.A = net->H2; g.B = net->W3; g.bias = net->P + OFF_B3; g.orm = net->H3; g.ofm = net->H3t;
    DV_TRY(gemm(g, TB, s));
    // O = H3 W4^T + b4 ; D4 = dscale (O - T)
    g.A = net->H3; g.B = net->W4; g.rb = NOUT; g.N = NOUT; g.mode = E_LOSS; g.bias = net->P + OFF_B4;
    g.orm = net->D4; g.orm_r = NB; g.ofm = net->D4t; g.ofm_r = NOUT; g.tgt = net->Tb;
    g.dscale = 2.0f / (float)((double)rows_valid * NOUT_USED);
    g.lossp = net->lossp; g.bsum = net->bpart + 3 * TB * 128;
    DV_TRY(gemm(g, TB, s));
    // D3 = (D4 W4) (1 - H3^2) ; D2 ; D1
    GemmP d = base(net);
    d.rows_valid = rows_valid;
    d.mode = E_DTANH; d.N = NH; d.orm_r = NB; d.ofm_r = NH; d.hd_r = NB;
    d.A = net->D4; d.ra = NB; d.B = net->W4t; d.rb = NH; d.kpanels = NOUT / 8; d.hd = net->H3;
    d.orm = net->D3; d.ofm = net->D3t; d.bsum = net->bpart + 2 * TB * 128;
    DV_TRY(gemm(d, TB, s));
    d.A = net->D3; d.B = net->W3t; d.kpanels = NH / 8; d.hd = net->H2; d.orm = net->D2; d.ofm = net->D2t;
    d.bsum = net->bpart + 1 * TB * 128;
    DV_TRY(gemm(d, TB, s));
    d.A = net->D2; d.B = net->W2t; d.hd = net->H1; d.orm = net->D1; d.ofm = net->D1t; d.bsum = net->bpart;
    DV_TRY(gemm(d, TB, s));
    // weight gradients: K = samples split over NSPLIT CTAs each
    const int64_t PS = (int64_t)NSPLIT * 128 * 128;
    GemmP w = base(net);
    w.split = 1; w.mode = E_PART; w.kpanels = NB / 8 / NSPLIT;
    w.A = net->D1t; w.ra = NH; w.B = net->Xbt; w.rb = NIN; w.N = NIN; w.of = net->part;
    DV_TRY(gemm(w, NSPLIT, s));
    w.A = net->D2t; w.B = net->H1t; w.rb = NH; w.N = NH; w.of = net->part + PS;
    DV_TRY(gemm(w, NSPLIT, s));
    w.A = net->D3t; w.B = net->H2t; w.of = net->part + 2 * PS;
    DV_TRY(gemm(w, NSPLIT, s));
    w.A = net->H3t; w.B = net->D4t; w.rb = NOUT; w.N = NOUT; w.of = net->part + 3 * PS;
    DV_TRY(gemm(w, NSPLIT, s));
    DV_LAUNCH(dv::K_MLP, s, k_collect_grad<<<g1(NPARAM), 256, 0, s>>>(net->part, net->bpart, net->G));
    return launch_ok("k_collect_grad");
}

static int forward_rows(dv_mlp* net, const bf16* X, int64_t rows, int64_t rows_valid, float* out, cudaStream_t s) {
    const int grid = (int)(rows / 128);
    GemmP g = base(net);
    g.rows_valid = rows_valid;
    g.A = X; g.ra = rows; g.B = net->W1; g.rb = NH; g.N = NH; g.kpanels = NIN / 8; g.mode = E_TANH;
    g.bias = net->P + OFF_B1; g.orm = net->Ha; g.orm_r = rows;
    DV_TRY(gemm(g, grid, s));
    g.A = net->Ha; g.B = net->W2; g.kpanels = NH / 8; g.bias = net->P + OFF_B2; g.orm = net->Hb;
    DV_TRY(gemm(g, grid, s));
    g.A = net->Hb; g.B = net->W3; g.bias = net->P + OFF_B3; g.orm = net->Ha;
    DV_TRY(gemm(g, grid, s));
    g.A = net->Ha; g.B = net->W4; g.rb = NOUT; g.N = NOUT; g.mode = E_OUT; g.bias = net->P + OFF_B4; g.orm = nullptr;
    g.of = out; g.ldf = NOUT;
    return gemm(g, grid, s);
}

int predict(dv_mlp* net, const StageInputs& in, const double* ytr, double* pred, cudaStream_t s) {
    const int64_t rows = (in.nc + 127) / 128 * 128;
    if (rows > net->inf_rows) {
        set_error("dv_mlp: inference buffers smaller than the model (call dv_mlp_reserve)");
        return DV_ERR_ARG;
    }
    DV_LAUNCH(dv::K_MLP, s, k_features<<<g1(in.nc, 128), 128, 0, s>>>(in, net->norm, 0, 1, in.nc, net->Xi, rows, 0));
    DV_CUDA(cudaGetLastError());
    DV_TRY(forward_rows(net, net->Xi, rows, in.nc, net->Oi, s));
    DV_LAUNCH(dv::K_MLP, s, k_apply<<<g1(in.nc), 256, 0, s>>>(in, net->norm, net->Oi, ytr, pred));
    return launch_ok("k_apply");
}

int record_features(dv_mlp* net, const StageInputs& in, int64_t first, int64_t stride, int64_t cnt, cudaStream_t s) {
    if (net->count + cnt > net->cap) return DV_OK;
    DV_LAUNCH(dv::K_MLP, s, k_features<<<g1(cnt, 128), 128, 0, s>>>(in, net->norm, first, stride, cnt, net->Xs, net->cap,
                                                                      net->count));
    return launch_ok("k_features");
}

int record_targets(dv_mlp* net, const StageInputs& in, const double* zstar, const double* zext, int64_t first,
                   int64_t stride, int64_t cnt, cudaStream_t s) {
    if (net->count + cnt > net->cap) return DV_OK;
    DV_LAUNCH(dv::K_MLP, s, k_targets<<<g1(cnt), 256, 0, s>>>(in, zstar, zext, first, stride, cnt, net->Ts, net->count));
    DV_CUDA(cudaGetLastError());
    net->count += cnt;
    return DV_OK;
}

}  // namespace mlp
}  // namespace dv

using namespace dv;
using namespace dv::mlp;

namespace {
template <class T>
int dalloc(T** p, int64_t n) {
    if (cudaMalloc((void**)p, sizeof(T) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "cudaMalloc(mlp)");
    return cudaMemset(*p, 0, sizeof(T) * (size_t)std::max<int64_t>(n, 1)) == cudaSuccess ? DV_OK
                                                                                       : cuda_fail(cudaGetLastError(), "cudaMemset(mlp)");
}
void bf16_round_host(const float* x, int64_t n, std::vector<uint16_t>& out) {
    out.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        uint32_t u;
        memcpy(&u, &x[i], 4);
        const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);   // round to nearest even (finite inputs)
        out[i] = (uint16_t)(r >> 16);
    }
}
}  // namespace

extern "C" {

int dv_mlp_create(int64_t sample_capacity, uint64_t seed, dv_mlp** out) {
    std::lock_guard<std::recursive_mutex> lk_(dv::capture_mutex());
    if (!out || sample_capacity < 0) { set_error("dv_mlp_create: bad argument"); return DV_ERR_ARG; }
    dv_mlp* n = new dv_mlp();
    n->cap = (sample_capacity + NB - 1) / NB * NB;
    int rc = DV_OK;
    const int64_t TB = NB / 128;
    auto A = [&](auto** p, int64_t cnt) { if (rc == DV_OK) rc = dalloc(p, cnt); };
    A(&n->P, NPARAM); A(&n->G, NPARAM); A(&n->Mo, NPARAM); A(&n->Vo, NPARAM);
    A(&n->W1, (int64_t)NH * NIN); A(&n->W2, (int64_t)NH * NH); A(&n->W3, (int64_t)NH * NH); A(&n->W4, (int64_t)NOUT * NH);
    A(&n->W2t, (int64_t)NH * NH); A(&n->W3t, (int64_t)NH * NH); A(&n->W4t, (int64_t)NOUT * NH);
    A(&n->norm, NNORM);
    A(&n->Xs, std::max<int64_t>(n->cap, NB) * NIN); A(&n->Ts, std::max<int64_t>(n->cap, NB) * 8);
    A(&n->Xb, (int64_t)NB * NIN); A(&n->Xbt, (int64_t)NB * NIN); A(&n->Tb, (int64_t)NB * 8);
    for (bf16** p : {&n->H1, &n->H2, &n->H3, &n->H1t, &n->H2t, &n->H3t, &n->D3, &n->D2, &n->D1, &n->D3t, &n->D2t, &n->D1t})
        A(p, (int64_t)NB * NH);
    A(&n->D4, (int64_t)NB * NOUT); A(&n->D4t, (int64_t)NB * NOUT);
    A(&n->part, 4LL * NSPLIT * 128 * 128); A(&n->bpart, 4LL * TB * 128); A(&n->lossp, TB);
    A(&n->d_err, 1);
    if (rc == DV_OK && cudaMallocHost((void**)&n->h_loss, sizeof(float) * TB) != cudaSuccess)
        rc = cuda_fail(cudaGetLastError(), "cudaMallocHost(mlp)");
    if (rc != DV_OK) { dv_mlp_destroy(n); return rc; }
    // initial parameters: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) hidden weights, zero biases, zero output
    // layer (the untrained network predicts no correction: the plain extrapolation)
    std::vector<float> P(NPARAM, 0.0f);
    uint64_t st = seed * 0x9e3779b97f4a7c15ull + 1;
    auto uni = [&]() {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int64_t off, int64_t cnt, double fan) {
        const double a = 1.0 / std::sqrt(fan);
        for (int64_t i = 0; i < cnt; ++i) P[off + i] = (float)((2.0 * uni() - 1.0) * a);
    };
    fill(OFF_W1, (int64_t)NH * NIN, NFEAT);
    fill(OFF_W2, (int64_t)NH * NH, NH);
    fill(OFF_W3, (int64_t)NH * NH, NH);
    double nrm[NNORM] = {0.02, 0.5, 40.0, 1.0, 5.0, 1e7, 2e-3, 5e-2, 4.0, 0.1, 0.5, 1e6, 10.0,
                         1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 8.0};
    rc = dv_mlp_set_params(n, P.data(), NPARAM, nrm, NNORM);
    if (rc != DV_OK) { dv_mlp_destroy(n); return rc; }
    *out = n;
    return DV_OK;
}

int dv_mlp_destroy(dv_mlp* n) {
    std::lock_guard<std::recursive_mutex> lk_(dv::capture_mutex());
    if (!n) return DV_OK;
    void* ptrs[] = {n->P, n->G, n->Mo, n->Vo, n->W1, n->W2, n->W3, n->W4, n->W2t, n->W3t, n->W4t, n->norm, n->Xs, n->Ts,
                    n->Xb, n->Xbt, n->H1, n->H2, n->H3, n->H1t, n->H2t, n->H3t, n->D4, n->D4t, n->D3, n->D2, n->D1,
                    n->D3t, n->D2t, n->D1t, n->Tb, n->part, n->bpart, n->lossp, n->Xi, n->Ha, n->Hb, n->Oi, n->d_err};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (n->h_loss) cudaFreeHost(n->h_loss);
    delete n;
    return DV_OK;
}

int dv_mlp_reserve(dv_mlp* n, int64_t ncell) {
    if (!n || ncell <= 0) { set_error("dv_mlp_reserve: bad argument"); return DV_ERR_ARG; }
    const int64_t rows = (ncell + 127) / 128 * 128;
    if (rows <= n->inf_rows) return DV_OK;
    for (void* p : {(void*)n->Xi, (void*)n->Ha, (void*)n->Hb, (void*)n->Oi})
        if (p) cudaFree(p);
    n->Xi = n->Ha = n->Hb = nullptr;
    n->Oi = nullptr;
    n->inf_rows = 0;
    int rc = dalloc(&n->Xi, rows * NIN);
    if (rc == DV_OK) rc = dalloc(&n->Ha, rows * NH);
    if (rc == DV_OK) rc = dalloc(&n->Hb, rows * NH);
    if (rc == DV_OK) rc = dalloc(&n->Oi, rows * NOUT);
    if (rc == DV_OK) n->inf_rows = rows;
    return rc;
}

int dv_mlp_set_params(dv_mlp* n, const float* params, int64_t nparams, const double* norm, int32_t nnorm) {
    if (!n || !params || nparams != NPARAM || (norm && nnorm != NNORM)) {
        set_error("dv_mlp_set_params: expected DV_MLP_NPARAM parameters and DV_MLP_NNORM constants");
        return DV_ERR_ARG;
    }
    DV_CUDA(cudaMemcpy(n->P, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
    DV_CUDA(cudaMemset(n->Mo, 0, sizeof(float) * NPARAM));
    DV_CUDA(cudaMemset(n->Vo, 0, sizeof(float) * NPARAM));
    n->adam_t = 0;
    if (norm) {
        memcpy(n->norm_h, norm, sizeof(double) * NNORM);
        DV_CUDA(cudaMemcpy(n->norm, norm, sizeof(double) * NNORM, cudaMemcpyHostToDevice));
    }
    DV_TRY(pack(n, 0));
    DV_CUDA(cudaDeviceSynchronize());
    return DV_OK;
}

int dv_mlp_get_params(const dv_mlp* n, float* params, double* norm) {
    if (!n || !params) { set_error("dv_mlp_get_params: null argument"); return DV_ERR_ARG; }
    DV_CUDA(cudaMemcpy(params, n->P, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    if (norm) memcpy(norm, n->norm_h, sizeof(double) * NNORM);
    return DV_OK;
}

int64_t dv_mlp_sample_count(const dv_mlp* n) { return n ? n->count : -1; }

int dv_mlp_get_samples(const dv_mlp* n, int64_t first, int64_t count, float* X, float* T) {
    if (!n || first < 0 || count < 0 || first + count > n->count || (!X && !T)) {
        set_error("dv_mlp_get_samples: bad argument");
        return DV_ERR_ARG;
    }
    if (count == 0) return DV_OK;
    if (X) {        // the store is in panels of 8 features: copy each panel's rows, then transpose
        std::vector<uint16_t> pan((size_t)count * 8);
        for (int p = 0; p < NIN / 8; ++p) {
            DV_CUDA(cudaMemcpy(pan.data(), n->Xs + pidx(first, p * 8, n->cap), sizeof(uint16_t) * pan.size(),
                               cudaMemcpyDeviceToHost));
            for (int64_t r = 0; r < count; ++r)
                for (int q = 0; q < 8; ++q) {
                    const uint32_t bits = (uint32_t)pan[(size_t)r * 8 + q] << 16;
                    float v;
                    memcpy(&v, &bits, sizeof v);
                    X[(size_t)r * NIN + p * 8 + q] = v;
                }
        }
    }
    if (T) DV_CUDA(cudaMemcpy(T, n->Ts + first * 8, sizeof(float) * (size_t)count * 8, cudaMemcpyDeviceToHost));
    return DV_OK;
}

int dv_mlp_clear_samples(dv_mlp* n) {
    if (!n) { set_error("null argument"); return DV_ERR_ARG; }
    n->count = 0;
    return DV_OK;
}

// Forward pass of rows of host features (row-major fp32, rounded to bf16) -> outputs [rows][NOUT].
int dv_mlp_forward_host(dv_mlp* n, const float* X, int64_t rows, float* out) {
    if (!n || !X || !out || rows <= 0) { set_error("dv_mlp_forward_host: bad argument"); return DV_ERR_ARG; }
    const int64_t R = (rows + 127) / 128 * 128;
    DV_TRY(dv_mlp_reserve(n, R));
    std::vector<uint16_t> xb;
    bf16_round_host(X, rows * NIN, xb);
    std::vector<uint16_t> panel((size_t)R * NIN, 0);
    for (int64_t r = 0; r < rows; ++r)
        for (int k = 0; k < NIN; ++k) panel[pidx(r, k, R)] = xb[r * NIN + k];
    DV_CUDA(cudaMemcpy(n->Xi, panel.data(), panel.size() * 2, cudaMemcpyHostToDevice));
    DV_TRY(forward_rows(n, n->Xi, R, rows, n->Oi, 0));
    DV_CUDA(cudaMemcpy(out, n->Oi, sizeof(float) * rows * NOUT, cudaMemcpyDeviceToHost));
    int e = 0;
    DV_CUDA(cudaMemcpy(&e, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { set_error("dv_mlp: a tensor-core product's completion wait timed out"); return DV_ERR_CUDA; }
    return DV_OK;
}

// One tensor-core product D [M][N] = A [M][K] B[N][K]^T of host fp32 matrices rounded to BF16 (M a
// multiple of 128, N a multiple of 16 up to 128, K a multiple of 16), FP32 result: the check of the
// product kernel itself.  Allocates its device buffers.
int dv_mlp_gemm_host(int32_t M, int32_t N, int32_t K, const float* A, const float* B, float* D) {
    if (M <= 0 || M % 128 || N < 16 || N > 128 || N % 16 || K <= 0 || K % 16 || !A || !B || !D) {
        set_error("dv_mlp_gemm_host: M multiple of 128, N in 16..128 multiple of 16, K multiple of 16");
        return DV_ERR_ARG;
    }
    std::vector<uint16_t> ab, bb;
    bf16_round_host(A, (int64_t)M * K, ab);
    bf16_round_host(B, (int64_t)N * K, bb);
    std::vector<uint16_t> ap((size_t)M * K), bp((size_t)N * K);
    for (int64_t r = 0; r < M; ++r)
        for (int k = 0; k < K; ++k) ap[pidx(r, k, M)] = ab[r * K + k];
    for (int64_t r = 0; r < N; ++r)
        for (int k = 0; k < K; ++k) bp[pidx(r, k, N)] = bb[r * K + k];
    bf16 *dA = nullptr, *dB = nullptr;
    float *dD = nullptr, *dz = nullptr;
    int* derr = nullptr;
    int rc = DV_OK;
    if (cudaMalloc((void**)&dA, ap.size() * 2) != cudaSuccess || cudaMalloc((void**)&dB, bp.size() * 2) != cudaSuccess ||
        cudaMalloc((void**)&dD, sizeof(float) * (size_t)M * N) != cudaSuccess ||
        cudaMalloc((void**)&dz, sizeof(float) * N) != cudaSuccess || cudaMalloc((void**)&derr, sizeof(int)) != cudaSuccess)
        rc = cuda_fail(cudaGetLastError(), "cudaMalloc(gemm check)");
    if (rc == DV_OK) {
        cudaMemcpy(dA, ap.data(), ap.size() * 2, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, bp.data(), bp.size() * 2, cudaMemcpyHostToDevice);
        cudaMemset(dz, 0, sizeof(float) * N);
        cudaMemset(derr, 0, sizeof(int));
        GemmP g;
        memset(&g, 0, sizeof g);
        g.A = dA; g.ra = M; g.B = dB; g.rb = N; g.N = N; g.kpanels = K / 8; g.mode = E_OUT; g.rows_valid = M;
        g.bias = dz; g.of = dD; g.ldf = N; g.err = derr;
        rc = gemm(g, M / 128, 0);
        if (rc == DV_OK && cudaDeviceSynchronize() != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "k_gemm");
        int e = 0;
        if (rc == DV_OK) cudaMemcpy(&e, derr, sizeof(int), cudaMemcpyDeviceToHost);
        if (rc == DV_OK && e) { set_error("dv_mlp: a tensor-core product's completion wait timed out"); rc = DV_ERR_CUDA; }
        if (rc == DV_OK) cudaMemcpy(D, dD, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost);
    }
    for (void* q : {(void*)dA, (void*)dB, (void*)dD, (void*)dz, (void*)derr})
        if (q) cudaFree(q);
    return rc;
}

// Gradient of the batch loss mean((O - T)^2) over the used outputs for host features X [rows][NIN] and
// targets T [rows][8] (already scaled; rows <= DV_MLP_BATCH), into grad [DV_MLP_NPARAM]; *loss = the mean.
int dv_mlp_gradient_host(dv_mlp* n, const float* X, const float* T, int64_t rows, float* grad, double* loss) {
    if (!n || !X || !T || !grad || rows <= 0 || rows > NB) { set_error("dv_mlp_gradient_host: bad argument"); return DV_ERR_ARG; }
    std::vector<uint16_t> xb;
    bf16_round_host(X, rows * NIN, xb);
    std::vector<uint16_t> rm((size_t)NB * NIN, 0), fm((size_t)NB * NIN, 0);
    std::vector<float> tb((size_t)NB * 8, 0.0f);
    for (int64_t r = 0; r < rows; ++r) {
        for (int k = 0; k < NIN; ++k) {
            rm[pidx(r, k, NB)] = xb[r * NIN + k];
            fm[pidx(k, r, NIN)] = xb[r * NIN + k];
        }
        for (int k = 0; k < 8; ++k) tb[r * 8 + k] = T[r * 8 + k];
    }
    DV_CUDA(cudaMemcpy(n->Xb, rm.data(), rm.size() * 2, cudaMemcpyHostToDevice));
    DV_CUDA(cudaMemcpy(n->Xbt, fm.data(), fm.size() * 2, cudaMemcpyHostToDevice));
    DV_CUDA(cudaMemcpy(n->Tb, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice));
    DV_TRY(grad_batch(n, rows, 0));
    DV_CUDA(cudaMemcpy(grad, n->G, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    std::vector<float> lp(NB / 128);
    DV_CUDA(cudaMemcpy(lp.data(), n->lossp, sizeof(float) * lp.size(), cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (float x : lp) s += x;
    if (loss) *loss = s / ((double)rows * NOUT_USED);
    int e = 0;
    DV_CUDA(cudaMemcpy(&e, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { set_error("dv_mlp: a tensor-core product's completion wait timed out"); return DV_ERR_CUDA; }
    return DV_OK;
}

// Adam on the recorded samples: `steps` batches of DV_MLP_BATCH samples drawn (with replacement, by a
// hash of seed, step and row) from the recorded set; the output scales are set first from the recorded
// targets (RMS per variable) unless keep_scales.  loss_hist (host, `steps` entries) receives each
// batch's mean loss when non-NULL.
int dv_mlp_train(dv_mlp* n, int32_t steps, float lr, uint64_t seed, int32_t keep_scales, float* loss_hist, void* stream) {
    if (!n || steps < 0) { set_error("dv_mlp_train: bad argument"); return DV_ERR_ARG; }
    if (n->count < NB) { set_error("dv_mlp_train: fewer recorded samples than one batch"); return DV_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    if (!keep_scales) {
        std::vector<float> T((size_t)n->count * 8);
        DV_CUDA(cudaMemcpyAsync(T.data(), n->Ts, sizeof(float) * T.size(), cudaMemcpyDeviceToHost, s));
        DV_CUDA(cudaStreamSynchronize(s));
        for (int v = 0; v < NOUT_USED; ++v) {
            double ss = 0.0;
            for (int64_t r = 0; r < n->count; ++r) ss += (double)T[r * 8 + v] * T[r * 8 + v];
            n->norm_h[13 + v] = std::max(std::sqrt(ss / (double)n->count), 1e-6);
        }
        DV_CUDA(cudaMemcpyAsync(n->norm, n->norm_h, sizeof(double) * NNORM, cudaMemcpyHostToDevice, s));
    }
    const int TB = NB / 128;
    for (int it = 0; it < steps; ++it) {
        DV_LAUNCH(dv::K_MLP, s, k_gather<<<g1((int64_t)NB * (NIN / 8)), 256, 0, s>>>(n->Xs, n->cap, n->Ts, n->count,
                                                                                    (int64_t)(seed & 0x7fffffffffffll),
                                                                                    n->adam_t, n->norm, n->Xb, n->Xbt, n->Tb));
        DV_CUDA(cudaGetLastError());
        DV_TRY(grad_batch(n, NB, s));
        n->adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, (float)n->adam_t), c2 = 1.0f - std::pow(b2, (float)n->adam_t);
        DV_LAUNCH(dv::K_MLP, s, k_adam<<<g1(NPARAM), 256, 0, s>>>(n->P, n->G, n->Mo, n->Vo, lr, b1, b2, 1e-8f, c1, c2));
        DV_CUDA(cudaGetLastError());
        DV_TRY(pack(n, s));
        if (loss_hist) {
            DV_CUDA(cudaMemcpyAsync(n->h_loss, n->lossp, sizeof(float) * TB, cudaMemcpyDeviceToHost, s));
            DV_CUDA(cudaStreamSynchronize(s));
            double t = 0.0;
            for (int b = 0; b < TB; ++b) t += n->h_loss[b];
            loss_hist[it] = (float)(t / ((double)NB * NOUT_USED));
        }
    }
    DV_CUDA(cudaStreamSynchronize(s));
    int e = 0;
    DV_CUDA(cudaMemcpy(&e, n->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { set_error("dv_mlp: a tensor-core product's completion wait timed out"); return DV_ERR_CUDA; }
    return DV_OK;
}

}  // extern "C"
