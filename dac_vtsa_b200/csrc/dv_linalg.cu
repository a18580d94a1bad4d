// dv_linalg.cu -- preconditioner (block-pentadiagonal LU along z) and Krylov vector kernels.
//
// The reference preconditions GMRES with a SuperLU factorisation of M = I - d h J restricted to
// theta sectors (+ the innermost rings fully coupled), core/solver.py:334-337 and
// core/jacobian.py:50-69,88-91.  Here M is partitioned into z-planes: a partition is either one
// theta sector (mode theta_block: cells (i, j, k) for all rings i of sector j, plus the wall
// node (j, k)) or a whole cross-section (mode full).  Inside a partition every coupling of the
// stencil is kept: within a plane (r, and theta in full mode) and between planes k-2..k+2 (the
// MUSCL z+-2 reach).  The partition matrix is block-pentadiagonal in z with dense nb x nb
// blocks, factorised by block Gaussian elimination:
//   L2_k = A(k,k-2) Uinv_{k-2}
//   L1_k = (A(k,k-1) - L2_k U1_{k-2}) Uinv_{k-1}
//   D_k  = A(k,k) - L1_k U1_{k-1} - L2_k U2_{k-2},      Uinv_k = D_k^-1 (Gauss-Jordan, partial pivoting)
//   U1_k = A(k,k+1) - L1_k U2_{k-1},                    U2_k = A(k,k+2)
// and applied by one forward and one backward sweep along z (one CTA per partition).
#include <algorithm>
#include "dv_internal.h"
#include "dv_physics.cuh"

namespace dv {

struct PcGeom {
    int Nr, Nth, Nz, wall, mode, nb, nparts;
    int64_t nc;
};

static __device__ __forceinline__ int64_t pc_glob(const PcGeom& g, int part, int k, int l) {
    const int64_t offw = (int64_t)DV_NV * g.nc;
    if (g.mode == 0) {   // theta sector `part`
        if (l < DV_NV * g.Nr) {
            int i = l / DV_NV, v = l % DV_NV;
            return (int64_t)v * g.nc + ((int64_t)i * g.Nth + part) * g.Nz + k;
        }
        return offw + (int64_t)part * g.Nz + k;
    }
    if (l < DV_NV * g.Nr * g.Nth) {
        int pos = l / DV_NV, v = l % DV_NV;
        return (int64_t)v * g.nc + (int64_t)pos * g.Nz + k;
    }
    return offw + (int64_t)(l - DV_NV * g.Nr * g.Nth) * g.Nz + k;
}

// local index of (cell (i, j), var v) / wall (j) inside its partition; part of column j
static __device__ __forceinline__ int pc_local(const PcGeom& g, int i, int j, int v) {
    if (g.mode == 0) return (v < DV_NV) ? i * DV_NV + v : DV_NV * g.Nr;
    return (v < DV_NV) ? (i * g.Nth + j) * DV_NV + v : DV_NV * g.Nr * g.Nth + j;
}

// ---------------------------------------------------------------- assembly of I - dh J
// blocks: [part][Nz][5][nb*nb] column-major, slot d+2 holds A(k, k+d).
__global__ void k_pc_zero(double* __restrict__ A, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        A[q] = 0.0;
}

__global__ void k_pc_scatter(PcGeom g, const double* __restrict__ J, double dh, double* __restrict__ A) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    const int slot = blockIdx.y;
    const int k = (int)(c % g.Nz);
    const int64_t rj = c / g.Nz;
    const int j = (int)(rj % g.Nth), i = (int)(rj / g.Nth);
    int ni = i, nj = j, nk = k;
    bool ok = true;
    switch (slot) {
        case 0: break;
        case 1: nk = k - 1; ok = nk >= 0; break;
        case 2: nk = k + 1; ok = nk < g.Nz; break;
        case 3: nk = k - 2; ok = nk >= 0; break;
        case 4: nk = k + 2; ok = nk < g.Nz; break;
        case 5: ni = i - 1; ok = ni >= 0; break;
        case 6: ni = i + 1; ok = ni < g.Nr; break;
        case 7: ok = g.Nth > 1 && g.mode == 1; nj = (j == 0) ? g.Nth - 1 : j - 1; break;
        default: ok = g.Nth > 1 && g.mode == 1; nj = (j == g.Nth - 1) ? 0 : j + 1; break;
    }
    if (!ok) return;
    const int part = (g.mode == 0) ? j : 0;
    const int d = nk - k;
    const int nb = g.nb;
    double* B = A + (((int64_t)part * g.Nz + k) * 5 + (d + 2)) * (int64_t)nb * nb;
    const bool row_wall_ok = g.wall && i == g.Nr - 1;
    const bool col_wall_ok = g.wall && ni == g.Nr - 1;
    for (int rv = 0; rv < DV_NB; ++rv) {
        if (rv == DV_NV && !row_wall_ok) continue;
        const int lr = pc_local(g, i, j, rv);
        for (int cv = 0; cv < DV_NB; ++cv) {
            if (cv == DV_NV && !col_wall_ok) continue;
            const int lc = pc_local(g, ni, nj, cv);
            const double jv = J[((int64_t)(slot * DV_NB + rv) * DV_NB + cv) * g.nc + c];
            double val = -dh * jv;
            if (slot == 0 && rv == cv) val += 1.0;
            B[(int64_t)lc * nb + lr] = val;
        }
    }
}

// ---------------------------------------------------------------- CTA-level dense kernels
// C = beta C + alpha A B  (nb x nb, column-major, generic pointers); 256 threads, 32x32 tiles.
static __device__ void cta_gemm(int nb, double alpha, const double* A, const double* B, double beta, double* C,
                                double* shA, double* shB) {
    const int tid = threadIdx.x;
    const int tr = tid % 32, tc4 = (tid / 32) * 4;
    for (int ti = 0; ti < nb; ti += 32) {
        for (int tj = 0; tj < nb; tj += 32) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int kk = 0; kk < nb; kk += 32) {
                for (int q = tid; q < 1024; q += blockDim.x) {
                    int r = q % 32, cc = q / 32;
                    int gr = ti + r, gk = kk + cc;
                    shA[cc * 32 + r] = (gr < nb && gk < nb) ? A[(int64_t)gk * nb + gr] : 0.0;
                    int gk2 = kk + r, gc = tj + cc;
                    shB[cc * 32 + r] = (gk2 < nb && gc < nb) ? B[(int64_t)gc * nb + gk2] : 0.0;
                }
                __syncthreads();
#pragma unroll 8
                for (int q = 0; q < 32; ++q) {
                    double a = shA[q * 32 + tr];
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] += a * shB[(tc4 + u) * 32 + q];
                }
                __syncthreads();
            }
            const int gr = ti + tr;
            if (gr < nb) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    int gc = tj + tc4 + u;
                    if (gc < nb) {
                        double* cp = C + (int64_t)gc * nb + gr;
                        *cp = (beta == 0.0) ? alpha * acc[u] : beta * (*cp) + alpha * acc[u];
                    }
                }
            }
        }
    }
    __syncthreads();
}

static __device__ void cta_copy(int64_t n, const double* src, double* dst) {
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) dst[q] = src[q];
    __syncthreads();
}

// In-place inverse of D (nb x nb, column-major) using W (nb x 2nb scratch).  Returns 1 if a zero /
// non-finite pivot was met (the pivot is then replaced by 1 so the factorisation stays finite).
static __device__ int cta_inverse(int nb, double* D, double* W, double* red_v, int* red_i) {
    const int tid = threadIdx.x;
    const int64_t n2 = (int64_t)nb * nb;
    for (int64_t q = tid; q < 2 * n2; q += blockDim.x) {
        int64_t col = q / nb, row = q % nb;
        W[q] = (col < nb) ? D[q] : ((col - nb) == row ? 1.0 : 0.0);
    }
    __syncthreads();
    int bad = 0;
    for (int pc = 0; pc < nb; ++pc) {
        // pivot search (rows pc..nb-1 of column pc)
        double best = -1.0;
        int bi = pc;
        for (int r = pc + tid; r < nb; r += blockDim.x) {
            double v = fabs(W[(int64_t)pc * nb + r]);
            if (v > best || (v == best && r < bi)) { best = v; bi = r; }
        }
        red_v[tid] = best;
        red_i[tid] = bi;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (tid < s) {
                double ov = red_v[tid + s];
                int oi = red_i[tid + s];
                if (ov > red_v[tid] || (ov == red_v[tid] && oi < red_i[tid])) { red_v[tid] = ov; red_i[tid] = oi; }
            }
            __syncthreads();
        }
        const int pr = red_i[0];
        const double pmax = red_v[0];
        __syncthreads();
        if (pr != pc) {
            for (int c = pc + tid; c < 2 * nb; c += blockDim.x) {
                double a = W[(int64_t)c * nb + pc];
                W[(int64_t)c * nb + pc] = W[(int64_t)c * nb + pr];
                W[(int64_t)c * nb + pr] = a;
            }
        }
        __syncthreads();
        double piv = W[(int64_t)pc * nb + pc];
        if (!(pmax > 0.0) || !isfinite(piv)) {
            bad = 1;
            piv = 1.0;
        }
        const double inv = 1.0 / piv;
        __syncthreads();
        for (int c = pc + 1 + tid; c < 2 * nb; c += blockDim.x) W[(int64_t)c * nb + pc] *= inv;
        __syncthreads();
        const int64_t ncols = 2 * nb - (pc + 1);
        for (int64_t q = tid; q < ncols * nb; q += blockDim.x) {
            int c = pc + 1 + (int)(q / nb);
            int r = (int)(q % nb);
            if (r == pc) continue;
            double fr = W[(int64_t)pc * nb + r];
            if (fr != 0.0) W[(int64_t)c * nb + r] -= fr * W[(int64_t)c * nb + pc];
        }
        __syncthreads();
    }
    for (int64_t q = tid; q < n2; q += blockDim.x) D[q] = W[n2 + q];
    __syncthreads();
    return bad;
}

// One CTA per partition: sequential block elimination along z.
__global__ void __launch_bounds__(256) k_pc_factor(PcGeom g, double* __restrict__ A, double* __restrict__ work,
                                                   int* __restrict__ info, int use_smem) {
    extern __shared__ double dsm[];
    __shared__ double shA[1024], shB[1024];
    __shared__ double red_v[256];
    __shared__ int red_i[256];
    const int part = blockIdx.x;
    const int nb = g.nb;
    const int64_t n2 = (int64_t)nb * nb;
    double* base = A + (int64_t)part * g.Nz * 5 * n2;
    double* T = work + (int64_t)part * 4 * n2;          // temp block
    double* W = use_smem ? dsm : (T + n2);             // 2*n2 Gauss-Jordan scratch
    int bad = 0;
    for (int k = 0; k < g.Nz; ++k) {
        double* Ak = base + (int64_t)k * 5 * n2;
        double* Am2 = Ak;
        double* Am1 = Ak + n2;
        double* A0 = Ak + 2 * n2;
        double* Ap1 = Ak + 3 * n2;
        double* Uinv_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 2) * n2 : nullptr;
        double* U1_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 3) * n2 : nullptr;
        double* U2_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 4) * n2 : nullptr;
        double* Uinv_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 2) * n2 : nullptr;
        double* U1_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 3) * n2 : nullptr;
        double* U2_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 4) * n2 : nullptr;
        if (k >= 2) {                                   // L2 = A(k,k-2) Uinv_{k-2}
            cta_gemm(nb, 1.0, Am2, Uinv_2, 0.0, T, shA, shB);
            cta_copy(n2, T, Am2);
            cta_gemm(nb, -1.0, Am2, U1_2, 1.0, Am1, shA, shB);   // A(k,k-1) -= L2 U1_{k-2}
            cta_gemm(nb, -1.0, Am2, U2_2, 1.0, A0, shA, shB);    // D -= L2 U2_{k-2}
        }
        if (k >= 1) {                                   // L1 = (...) Uinv_{k-1}
            cta_gemm(nb, 1.0, Am1, Uinv_1, 0.0, T, shA, shB);
            cta_copy(n2, T, Am1);
            cta_gemm(nb, -1.0, Am1, U1_1, 1.0, A0, shA, shB);    // D -= L1 U1_{k-1}
            cta_gemm(nb, -1.0, Am1, U2_1, 1.0, Ap1, shA, shB);   // U1 = A(k,k+1) - L1 U2_{k-1}
        }
        bad |= cta_inverse(nb, A0, W, red_v, red_i);
    }
    if (threadIdx.x == 0) info[part] = bad;
}

// x = diag(1/sc) M^-1 diag(sc) b  for all partitions (one CTA each, 256 threads, 4 threads per row).
__global__ void __launch_bounds__(256) k_pc_apply(PcGeom g, const double* __restrict__ A, const double* __restrict__ b,
                                                  const double* __restrict__ sc, double* __restrict__ x) {
    extern __shared__ double xs[];                  // [Nz][nb]
    const int part = blockIdx.x;
    const int nb = g.nb;
    const int64_t n2 = (int64_t)nb * nb;
    const double* base = A + (int64_t)part * g.Nz * 5 * n2;
    const int tid = threadIdx.x;
    const int lane4 = tid & 3;
    const int rows_per_pass = blockDim.x / 4;
    for (int64_t q = tid; q < (int64_t)g.Nz * nb; q += blockDim.x) {
        int k = (int)(q / nb), l = (int)(q % nb);
        int64_t gi = pc_glob(g, part, k, l);
        xs[q] = sc ? b[gi] * sc[gi] : b[gi];
    }
    __syncthreads();
    // forward: z_k = b_k - L1_k z_{k-1} - L2_k z_{k-2}
    for (int k = 1; k < g.Nz; ++k) {
        const double* L1 = base + ((int64_t)k * 5 + 1) * n2;
        const double* L2 = base + ((int64_t)k * 5 + 0) * n2;
        const double* z1 = xs + (int64_t)(k - 1) * nb;
        const double* z2 = (k >= 2) ? xs + (int64_t)(k - 2) * nb : nullptr;
        for (int r0 = 0; r0 < nb; r0 += rows_per_pass) {
            int r = r0 + tid / 4;
            double acc = 0.0;
            if (r < nb) {
                for (int c = lane4; c < nb; c += 4) {
                    acc += L1[(int64_t)c * nb + r] * z1[c];
                    if (z2) acc += L2[(int64_t)c * nb + r] * z2[c];
                }
            }
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            if (r < nb && lane4 == 0) xs[(int64_t)k * nb + r] -= acc;
        }
        __syncthreads();
    }
    // backward: x_k = Uinv_k (z_k - U1_k x_{k+1} - U2_k x_{k+2}); tmp held in registers then written
    for (int k = g.Nz - 1; k >= 0; --k) {
        const double* Ui = base + ((int64_t)k * 5 + 2) * n2;
        const double* U1 = base + ((int64_t)k * 5 + 3) * n2;
        const double* U2 = base + ((int64_t)k * 5 + 4) * n2;
        const double* x1 = (k + 1 < g.Nz) ? xs + (int64_t)(k + 1) * nb : nullptr;
        const double* x2 = (k + 2 < g.Nz) ? xs + (int64_t)(k + 2) * nb : nullptr;
        double* zk = xs + (int64_t)k * nb;
        if (x1) {
            for (int r0 = 0; r0 < nb; r0 += rows_per_pass) {
                int r = r0 + tid / 4;
                double acc = 0.0;
                if (r < nb) {
                    for (int c = lane4; c < nb; c += 4) {
                        acc += U1[(int64_t)c * nb + r] * x1[c];
                        if (x2) acc += U2[(int64_t)c * nb + r] * x2[c];
                    }
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                __syncthreads();
                if (r < nb && lane4 == 0) zk[r] -= acc;
            }
            __syncthreads();
        }
        // x_k = Uinv_k zk  (rows computed into registers, written after a barrier)
        double outv[8];
        int nout = 0;
        for (int r0 = 0; r0 < nb; r0 += rows_per_pass) {
            int r = r0 + tid / 4;
            double acc = 0.0;
            if (r < nb)
                for (int c = lane4; c < nb; c += 4) acc += Ui[(int64_t)c * nb + r] * zk[c];
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            if (nout < 8) outv[nout] = acc;
            ++nout;
        }
        __syncthreads();
        nout = 0;
        for (int r0 = 0; r0 < nb; r0 += rows_per_pass) {
            int r = r0 + tid / 4;
            if (r < nb && lane4 == 0 && nout < 8) zk[r] = outv[nout];
            ++nout;
        }
        __syncthreads();
    }
    for (int64_t q = tid; q < (int64_t)g.Nz * nb; q += blockDim.x) {
        int k = (int)(q / nb), l = (int)(q % nb);
        int64_t gi = pc_glob(g, part, k, l);
        x[gi] = sc ? xs[q] / sc[gi] : xs[q];
    }
}

static PcGeom geom_of(const dv_model* m, int mode) {
    PcGeom g;
    g.Nr = m->p.Nr;
    g.Nth = m->p.Nth;
    g.Nz = m->p.Nz;
    g.wall = m->p.wall_on;
    g.mode = (m->p.Nth > 1 && mode == 0) ? 0 : 1;
    g.nc = m->nc;
    if (g.mode == 0) {
        g.nb = DV_NV * g.Nr + (g.wall ? 1 : 0);
        g.nparts = g.Nth;
    } else {
        g.nb = DV_NV * g.Nr * g.Nth + (g.wall ? g.Nth : 0);
        g.nparts = 1;
    }
    return g;
}

static int smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

int precond_factor(dv_model* m, const double* J, double dh, int mode, cudaStream_t s) {
    PcGeom g = geom_of(m, mode);
    if (g.nb > m->pc_cap_nb || g.nparts > m->pc_cap_parts) {
        set_error("preconditioner partition larger than the workspace allocated at model creation");
        return DV_ERR_ARG;
    }
    if (g.nb > 8 * 64) {
        set_error("preconditioner block size above the supported 512 (use theta_block)");
        return DV_ERR_UNSUPPORTED;
    }
    const int64_t n2 = (int64_t)g.nb * g.nb;
    const int64_t total = (int64_t)g.nparts * g.Nz * 5 * n2;
    k_pc_zero<<<std::min<int64_t>((total + 255) / 256, 4096), 256, 0, s>>>(m->d_pc, total);
    dim3 grid((unsigned)((m->nc + 127) / 128), DV_NSLOT);
    k_pc_scatter<<<grid, 128, 0, s>>>(g, J, dh, m->d_pc);
    const size_t static_smem = (2 * 1024 + 256) * sizeof(double) + 256 * sizeof(int);
    size_t need = (size_t)2 * n2 * sizeof(double);
    int use_smem = (need + static_smem) <= (size_t)smem_optin() ? 1 : 0;
    size_t dyn = use_smem ? need : 0;
    if (use_smem) DV_CUDA(cudaFuncSetAttribute(k_pc_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    k_pc_factor<<<g.nparts, 256, dyn, s>>>(g, m->d_pc, m->d_pc_work, m->d_pc_info, use_smem);
    DV_CUDA(cudaGetLastError());
    m->pc_mode = g.mode;
    m->pc_nb = g.nb;
    m->pc_nparts = g.nparts;
    m->pc_ready = 1;
    return DV_OK;
}

int precond_apply(dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s) {
    if (!m->pc_ready) {
        set_error("preconditioner applied before it was factorised");
        return DV_ERR_ARG;
    }
    PcGeom g = geom_of(m, m->pc_mode == 0 ? 0 : 1);
    size_t dyn = (size_t)g.Nz * g.nb * sizeof(double);
    if (dyn > 48 * 1024) DV_CUDA(cudaFuncSetAttribute(k_pc_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    if (dyn > (size_t)smem_optin()) {
        set_error("preconditioner sweep vector exceeds shared memory");
        return DV_ERR_UNSUPPORTED;
    }
    k_pc_apply<<<g.nparts, 256, dyn, s>>>(g, m->d_pc, b, sc, x);
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

}  // namespace dv
