// dv_linalg.cu -- preconditioner: block-pentadiagonal LU of I - dh J along z, and its sweep.
//
// The reference preconditions GMRES with a SuperLU factorisation of M = I - d h J restricted to
// theta sectors (+ the innermost rings fully coupled), core/solver.py:334-337 and
// core/jacobian.py:50-69,88-91.  Here M is partitioned into z-planes: a partition is either one
// theta sector (mode 0: cells (i, j, k) for all rings i of sector j, plus the wall node (j, k)),
// a whole cross-section (mode 1), or, in mode 2, the innermost ring of every sector as one
// partition plus rings 1.. of each sector (with its wall node) as the others: the inner ring's
// theta couplings stay in the preconditioner, which the reference keeps for its innermost rings.
// Inside a partition every coupling of the
// stencil is kept: within a plane (r, and theta in full mode) and between planes k-2..k+2 (the
// MUSCL z+-2 reach).  The partition matrix is block-pentadiagonal in z with dense nb x nb blocks
// (row-major, leading dimension ld >= nb, zero padded), factorised by block Gaussian elimination:
//   L2_k = A(k,k-2) Uinv_{k-2}
//   L1_k = (A(k,k-1) - L2_k U1_{k-2}) Uinv_{k-1}
//   D_k  = A(k,k) - L1_k U1_{k-1} - L2_k U2_{k-2},      Uinv_k = D_k^-1 (Gauss-Jordan, partial pivoting)
//   U1_k = A(k,k+1) - L1_k U2_{k-1},                    U2_k = A(k,k+2)
// Stored per plane k: slot 0 L2_k, slot 1 L1_k, slot 2 Uinv_k, slot 3 -Uinv_k U1_k, slot 4 -Uinv_k U2_k,
// so that both sweeps are one fused GEMV per plane:
//   forward  z_k = b_k - L1_k z_{k-1} - L2_k z_{k-2}
//   backward x_k = Uinv_k z_k + (-Uinv_k U1_k) x_{k+1} + (-Uinv_k U2_k) x_{k+2}
// Twisted form (Nz >= 8, both kernels in shared memory): the same recurrences run top-down over
// planes 0..zs-1 and, mirrored, bottom-up over planes Nz-1..zs+2 at the same time (a cluster of
// two CTAs per partition); the separator planes zs, zs+1 (zs = (Nz-2)/2) take the Schur
// contributions of both sides, and their 2 nb x 2 nb system is inverted by blocks.  Half the
// sequential plane chain of the one-directional form, for the same matrix.
#include <algorithm>
#include <vector>
#include <type_traits>
#include "dv_internal.h"
#include "dv_physics.cuh"

namespace dv {

struct PcGeom {
    int Nr, Nth, Nz, wall, mode, nb, nparts, ld;
    int rg, tg;            // mode 3: ring groups per sector (rings 1..Nr-1), theta groups of the core ring
    int zs;                // twisted factorisation: separator planes zs, zs+1 (0: one direction, top-down)
    int ncv;               // cell unknowns (6 per cell) of the partition; nb - ncv wall nodes follow
    int64_t nc, bs;        // bs: block stride in doubles (nb*ld rounded up to even: 16-byte multiple)
    // self-checks of the kernels: factor storage (entries; < 0: unchecked), state length, error word
    int64_t cap, nstate;
    int* err;
};

// Error word bit of an index that fell outside its storage (the access is skipped, not made).
#define PC_ERR_RANGE 32
static __device__ __forceinline__ bool pc_range_ok(const PcGeom& g, int64_t first, int64_t count) {
    if (g.cap < 0 || (first >= 0 && first + count <= g.cap)) return true;
    if (g.err) atomicOr(g.err, PC_ERR_RANGE);
    return false;
}

// Mode 3 (mode 2 split for large cross-sections): contiguous groups of n items in G groups, the
// first n % G groups one item larger.  Ring groups cover rings 1..Nr-1 of a sector (the wall node
// goes with the outermost, smallest group); theta groups cover the sectors of the core ring.
static __host__ __device__ __forceinline__ void pc_group(int n, int G, int gi, int& a0, int& a1) {
    const int base = n / G, extra = n % G;
    a0 = gi * base + (gi < extra ? gi : extra);
    a1 = a0 + base + (gi < extra ? 1 : 0);
}
static __host__ __device__ __forceinline__ int pc_group_of(int n, int G, int t) {
    const int base = n / G, extra = n % G;
    return (t < extra * (base + 1)) ? t / (base + 1) : extra + (t - extra * (base + 1)) / base;
}

// Geometry as seen by one partition: nb and ncv of that partition (ld, bs and strides stay the
// largest partition's).  Mode 2: parts 0..Nth-1 are sectors (rings 1..Nr-1 + wall), part Nth the core.
// Mode 3: part j*rg + gi is ring group gi of sector j (+ the wall in the last group), part
// Nth*rg + h theta group h of the core ring.
static __host__ __device__ __forceinline__ PcGeom pc_part(const PcGeom& g, int part) {
    PcGeom q = g;
    if (g.mode == 2) {
        if (part == g.Nth) { q.ncv = DV_NV * g.Nth; q.nb = q.ncv; }
        else { q.ncv = DV_NV * (g.Nr - 1); q.nb = q.ncv + (g.wall ? 1 : 0); }
    } else if (g.mode == 3) {
        int a0, a1;
        if (part >= g.Nth * g.rg) {
            pc_group(g.Nth, g.tg, part - g.Nth * g.rg, a0, a1);
            q.ncv = DV_NV * (a1 - a0);
            q.nb = q.ncv;
        } else {
            const int gi = part % g.rg;
            pc_group(g.Nr - 1, g.rg, gi, a0, a1);
            q.ncv = DV_NV * (a1 - a0);
            q.nb = q.ncv + ((g.wall && gi == g.rg - 1) ? 1 : 0);
        }
    }
    return q;
}

// partition of the cell unknowns of cell (i, j)
static __host__ __device__ __forceinline__ int pc_part_of(const PcGeom& g, int i, int j) {
    if (g.mode == 0) return j;
    if (g.mode == 2) return (i == 0) ? g.Nth : j;
    if (g.mode == 3)
        return (i == 0) ? g.Nth * g.rg + pc_group_of(g.Nth, g.tg, j) : j * g.rg + pc_group_of(g.Nr - 1, g.rg, i - 1);
    return 0;
}

#define PC_SMEM_NB 56      // largest block the shared-memory factorisation keeps resident (9 blocks)

// leading dimension of the stored blocks: nb rounded up to 16, so a row is a whole number of
// 16-column groups that the sweep's 8 lanes read as 16-byte column pairs
static inline int pc_ld(int nb) { return (nb + 15) / 16 * 16; }

// leading dimension of the blocks the factorisation keeps in shared memory: nb rounded up to 4 and
// made == 4 (mod 8), so the 8 rows of a DMMA A fragment (and the 4 rows of a B fragment) start on
// different 8-bank groups; without that padding when nine blocks would not fit
static inline int pc_lds(int nb, size_t budget) {
    const int l4 = (nb + 3) / 4 * 4;
    const int l = (l4 % 8 == 0) ? l4 + 4 : l4;
    return (size_t)9 * nb * l * sizeof(double) <= budget ? l : l4;
}

static __host__ __device__ __forceinline__ int64_t pc_glob(const PcGeom& g, int part, int k, int l) {
    const int64_t offw = (int64_t)DV_NV * g.nc;
    if (g.mode == 3) {
        int a0, a1;
        if (part >= g.Nth * g.rg) {             // core theta group: (sector j, var v) of ring 0
            pc_group(g.Nth, g.tg, part - g.Nth * g.rg, a0, a1);
            const int j = a0 + l / DV_NV, v = l % DV_NV;
            return (int64_t)v * g.nc + (int64_t)j * g.Nz + k;
        }
        const int j = part / g.rg, gi = part % g.rg;
        pc_group(g.Nr - 1, g.rg, gi, a0, a1);
        if (l < DV_NV * (a1 - a0)) {            // rings 1 + a0 .. 1 + a1 - 1 of sector j
            const int i = 1 + a0 + l / DV_NV, v = l % DV_NV;
            return (int64_t)v * g.nc + ((int64_t)i * g.Nth + j) * g.Nz + k;
        }
        return offw + (int64_t)j * g.Nz + k;
    }
    if (g.mode == 2) {
        if (part == g.Nth) {                    // core: (sector j, var v) of ring 0
            const int j = l / DV_NV, v = l % DV_NV;
            return (int64_t)v * g.nc + (int64_t)j * g.Nz + k;
        }
        if (l < DV_NV * (g.Nr - 1)) {           // sector `part`, rings 1..Nr-1
            const int i = 1 + l / DV_NV, v = l % DV_NV;
            return (int64_t)v * g.nc + ((int64_t)i * g.Nth + part) * g.Nz + k;
        }
        return offw + (int64_t)part * g.Nz + k;
    }
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

// local index of (cell (i, j), var v) / wall (j) inside its partition
static __host__ __device__ __forceinline__ int pc_local(const PcGeom& g, int i, int j, int v) {
    if (g.mode == 3) {
        int a0, a1;
        if (v == DV_NV) {                       // the wall node follows the cells of the outer group
            pc_group(g.Nr - 1, g.rg, g.rg - 1, a0, a1);
            return DV_NV * (a1 - a0);
        }
        if (i == 0) {
            pc_group(g.Nth, g.tg, pc_group_of(g.Nth, g.tg, j), a0, a1);
            return (j - a0) * DV_NV + v;
        }
        pc_group(g.Nr - 1, g.rg, pc_group_of(g.Nr - 1, g.rg, i - 1), a0, a1);
        return (i - 1 - a0) * DV_NV + v;
    }
    if (g.mode == 2) {
        if (v == DV_NV) return DV_NV * (g.Nr - 1);
        return (i == 0) ? j * DV_NV + v : (i - 1) * DV_NV + v;
    }
    if (g.mode == 0) return (v < DV_NV) ? i * DV_NV + v : DV_NV * g.Nr;
    return (v < DV_NV) ? (i * g.Nth + j) * DV_NV + v : DV_NV * g.Nr * g.Nth + j;
}

// The z-couplings A(k, k+-1), A(k, k+-2) only connect a cell to itself in another plane: they are
// block diagonal with 6x6 cell blocks (and 1x1 wall entries).  First index / size of the block of l:
static __device__ __forceinline__ void pc_cellblock(const PcGeom& g, int l, int& b0, int& bsz) {
    if (l < g.ncv) { b0 = (l / DV_NV) * DV_NV; bsz = DV_NV; }
    else { b0 = l; bsz = 1; }
}

// ---------------------------------------------------------------- assembly of I - dh J
// blocks: [part][Nz][5][bs] row-major (B[row*ld + col]); slot d+2 holds A(k, k+d).
__global__ void k_pc_zero(double* __restrict__ A, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        A[q] = 0.0;
}

__global__ void k_pc_to_f32(const double* __restrict__ A, float* __restrict__ B, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        B[q] = (float)A[q];
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
        case 7: ok = g.Nth > 1 && g.mode != 0; nj = (j == 0) ? g.Nth - 1 : j - 1; break;
        default: ok = g.Nth > 1 && g.mode != 0; nj = (j == g.Nth - 1) ? 0 : j + 1; break;
    }
    const int part = pc_part_of(g, i, j);
    if (!ok || pc_part_of(g, ni, nj) != part) return;      // coupling across partitions: dropped
    const int d = nk - k;
    const int64_t boff = (((int64_t)part * g.Nz + k) * 5 + (d + 2)) * g.bs;
    if (part >= g.nparts || !pc_range_ok(g, boff, g.bs)) {
        if (part >= g.nparts && g.err) atomicOr(g.err, PC_ERR_RANGE);
        return;
    }
    double* B = A + boff;
    const int pnb = pc_part(g, part).nb;
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
            if (lr >= pnb || lc >= pnb) {
                if (g.err) atomicOr(g.err, PC_ERR_RANGE);
                continue;
            }
            B[(int64_t)lr * g.ld + lc] = val;
        }
    }
}

// ---------------------------------------------------------------- shared-memory dense kernels (row-major)
// 256 threads as a 16 x 16 grid; thread (ty, tx) owns rows ty + 16a and columns tx + 16b (a, b < 4),
// i.e. a 4 x 4 register tile of any nb <= 64 matrix.  No integer division in the inner loops.
#define SM_T 16
#define SM_R 4

// D = A B + D on the FP64 tensor cores: one 8x8x4 product per warp instruction.  Fragments
// (lane = 4 g + t): a = A[g][t], b = B[t][g], d = D[g][2t .. 2t+1].
static __device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// C = beta C + alpha A B (row-major in shared memory, leading dimension ld, nb <= 64, alpha = +-1):
// 8x8 output tiles spread over the warps, each accumulated by DMMA over k in steps of 4; entries
// beyond nb read as zero and are not written.  (Accumulating all of a warp's tiles together
// measured slower on B200: 5.8 us against 3.7 us for nb = 48.)
static __device__ void sm_gemm(int nb, int ld, double alpha, const double* A, const double* B, double beta,
                               double* C) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int nt = (nb + 7) >> 3;
    for (int tile = warp; tile < nt * nt; tile += nw) {
        const int ti = tile / nt, tj = tile - ti * nt;
        const int r = 8 * ti + g;                 // row of A and C held by this lane
        const int cb = 8 * tj + g;                // column of B in the b fragment
        const int c0 = 8 * tj + 2 * t4;           // columns of C in the d fragment
        double d0 = 0.0, d1 = 0.0;
        for (int kk = 0; kk < nb; kk += 4) {
            const int ka = kk + t4;
            const double a = (r < nb && ka < nb) ? alpha * A[r * ld + ka] : 0.0;
            const double b = (ka < nb && cb < nb) ? B[ka * ld + cb] : 0.0;
            dmma_884(d0, d1, a, b);
        }
        if (r < nb) {
            double* cp = C + r * ld + c0;
            if (c0 < nb) cp[0] = (beta == 0.0) ? d0 : beta * cp[0] + d0;
            if (c0 + 1 < nb) cp[1] = (beta == 0.0) ? d1 : beta * cp[1] + d1;
        }
    }
    __syncthreads();
}

// C = beta C + alpha Bd X with Bd block diagonal (cell blocks); all three in shared memory with
// leading dimension ld.
static __device__ void sm_bd_left(const PcGeom& g, int ld, double alpha, const double* Bd, const double* X,
                                  double beta, double* C) {
    const int nb = g.nb;
    const int tx = threadIdx.x % SM_T, ty = threadIdx.x / SM_T;
#pragma unroll
    for (int a = 0; a < SM_R; ++a) {
        const int r = ty + SM_T * a;
        if (r >= nb) continue;
        int b0, bsz;
        pc_cellblock(g, r, b0, bsz);
#pragma unroll
        for (int b = 0; b < SM_R; ++b) {
            const int c = tx + SM_T * b;
            if (c >= nb) continue;
            double acc = 0.0;
            for (int q = b0; q < b0 + bsz; ++q) acc += Bd[r * ld + q] * X[q * ld + c];
            double* cp = C + r * ld + c;
            *cp = (beta == 0.0) ? alpha * acc : beta * (*cp) + alpha * acc;
        }
    }
    __syncthreads();
}

// C = beta C + alpha X Bd with Bd block diagonal (any memory space, leading dimension ldb); X and C
// in shared memory with leading dimension ld.
static __device__ void sm_bd_right(const PcGeom& g, int ld, double alpha, const double* X, const double* Bd,
                                   int ldb, double beta, double* C) {
    const int nb = g.nb;
    const int tx = threadIdx.x % SM_T, ty = threadIdx.x / SM_T;
#pragma unroll
    for (int b = 0; b < SM_R; ++b) {
        const int c = tx + SM_T * b;
        if (c >= nb) continue;
        int b0, bsz;
        pc_cellblock(g, c, b0, bsz);
#pragma unroll
        for (int a = 0; a < SM_R; ++a) {
            const int r = ty + SM_T * a;
            if (r >= nb) continue;
            double acc = 0.0;
            for (int q = b0; q < b0 + bsz; ++q) acc += X[r * ld + q] * Bd[q * ldb + c];
            double* cp = C + r * ld + c;
            *cp = (beta == 0.0) ? alpha * acc : beta * (*cp) + alpha * acc;
        }
    }
    __syncthreads();
}

// In-place Gauss-Jordan inverse (row-major, nb <= 64) with partial pivoting; returns 1 on a zero /
// non-finite pivot (replaced by 1 so the factors stay finite; reported through the info flag).
// In-place Gauss-Jordan inverse with partial pivoting of the nb x nb block *A (shared memory, nb <=
// 64, 256 threads), ping-ponging between *A and *B (same size).  Thread t updates column t % 64 on
// the rows congruent to t / 64 modulo 4 (coalesced row accesses, broadcast column-k reads); the
// threads of column k+1 also keep the running maxima of its new entries (rows > k), so the next
// pivot is known after the one barrier of the step.  The pivot is the largest |entry|, the
// smallest row index among equal ones.  The row interchanges are undone at the end by a single
// column gather.  On return *A holds the inverse (the pointers may have been exchanged).
static __device__ int sm_inverse_unb(int nb, int ld, double*& A, double*& B, int* perm, int* idx, double* pv, int* pi) {
    const int tid = threadIdx.x;
    const int cc = tid & 63, rq = tid >> 6;
    constexpr int RPT = 16;                       // rows per thread for nb <= 64
    int bad = 0;
    if (cc == 0) {                                // column 0: partial maxima per row group
        double best = -1.0;
        int bi = nb;
        for (int i = rq; i < nb; i += 4) {
            const double v = fabs(A[i * ld]);
            if (v > best) { best = v; bi = i; }
        }
        pv[rq] = best;
        pi[rq] = bi;
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        const double* cpv = pv + 4 * (k & 1);
        const int* cpi = pi + 4 * (k & 1);
        double best = cpv[0];
        int p = cpi[0];
#pragma unroll
        for (int q = 1; q < 4; ++q)
            if (cpv[q] > best || (cpv[q] == best && cpi[q] < p)) { best = cpv[q]; p = cpi[q]; }
        if (tid == 0) perm[k] = p;
        double piv = A[p * ld + k];
        if (!(fabs(piv) > 0.0) || !isfinite(piv)) { bad = 1; piv = 1.0; }
        const double inv = 1.0 / piv;
        if (cc < nb) {
            const double pr = ((cc == k) ? 1.0 : A[p * ld + cc]) * inv;     // scaled pivot row
            const bool nextcol = (cc == k + 1);
            double nbest = -1.0;
            int nbi = nb;
#pragma unroll
            for (int a = 0; a < RPT; ++a) {
                const int i = rq + 4 * a;
                if (i >= nb) break;
                double val;
                if (i == k) {
                    val = pr;
                } else {
                    const int src = (i == p) ? k : i;                      // rows k and p exchanged
                    const double fc = A[src * ld + k];                     // old column k
                    val = ((cc == k) ? 0.0 : A[src * ld + cc]) - fc * pr;
                }
                B[i * ld + cc] = val;
                if (nextcol && i > k) {
                    const double v = fabs(val);
                    if (v > nbest) { nbest = v; nbi = i; }
                }
            }
            if (nextcol) {
                pv[4 * ((k + 1) & 1) + rq] = nbest;
                pi[4 * ((k + 1) & 1) + rq] = nbi;
            }
        }
        __syncthreads();
        double* t = A; A = B; B = t;
    }
    if (tid == 0) {                               // the row interchanges, undone as column interchanges
        for (int c = 0; c < nb; ++c) idx[c] = c;
        for (int k = nb - 1; k >= 0; --k) {
            const int q = perm[k], t = idx[k];
            idx[k] = idx[q];
            idx[q] = t;
        }
    }
    __syncthreads();
    if (cc < nb)
        for (int i = rq; i < nb; i += 4) B[i * ld + cc] = A[i * ld + idx[cc]];
    __syncthreads();
    double* t = A; A = B; B = t;
    return bad;
}

// Blocked Gauss-Jordan inverse with partial pivoting of the nb x nb block *A (shared memory, nb <=
// 64, 256 threads, leading dimension ld); *B (same size) is scratch.  Columns are processed in
// panels of 8: the pivot steps of a panel run on a small column-major copy of its columns (one
// barrier per step, the next pivot found by the warp that updates its column), then the panel's
// row interchanges are applied to the other columns, the panel's pivot rows are set aside and the
// other columns receive the panel's combined transformation as one rank-8 DMMA update:
//   x <- [x with the pivot rows zeroed] + Panel * x(pivot rows).
// The pivot is the largest |entry|, the smallest row index among equal ones.  The row
// interchanges are undone at the end by one column gather.  On return *A holds the inverse (the
// pointers may have been exchanged).
static __device__ int sm_inverse_blk(int nb, int ld, double*& A, double*& B, int* perm, int* idx, int* pi) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* P0 = B;                               // panel copies: [8][nb] column-major, ping-pong
    double* P1 = B + nb * 8;
    double* Bs = B + 2 * nb * 8;                  // the panel's pivot rows: [8][ld] (fits: see sm_inverse)
    int bad = 0;
    for (int j0 = 0; j0 < nb; j0 += 8) {
        const int jb = min(8, nb - j0);
        for (int q = tid; q < nb * 8; q += blockDim.x) {       // panel copy
            const int cq = q / nb, i = q - cq * nb;
            P0[q] = (cq < jb) ? A[i * ld + j0 + cq] : 0.0;
        }
        if (warp == 0) {                          // pivot of the panel's first column
            double best = -1.0;
            int bi = nb;
            for (int i = j0 + lane; i < nb; i += 32) {
                const double v = fabs(A[i * ld + j0]);
                if (v > best) { best = v; bi = i; }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) pi[0] = bi;
        }
        __syncthreads();
        double* Pc = P0;
        double* Pn = P1;
        for (int kq = 0; kq < jb; ++kq) {         // pivot steps of the panel: warp w updates column w
            const int k = j0 + kq;
            const int p = pi[kq & 1];
            if (tid == 0) perm[k] = p;
            double piv = Pc[kq * nb + p];
            if (!(fabs(piv) > 0.0) || !isfinite(piv)) { bad = 1; piv = 1.0; }
            const double inv = 1.0 / piv;
            const int cq = warp;
            double best = -1.0;
            int bi = nb;
            if (cq < jb) {
                const double pr = ((cq == kq) ? 1.0 : Pc[cq * nb + p]) * inv;
                for (int i = lane; i < nb; i += 32) {
                    double val;
                    if (i == k) {
                        val = pr;
                    } else {
                        const int src = (i == p) ? k : i;
                        val = ((cq == kq) ? 0.0 : Pc[cq * nb + src]) - Pc[kq * nb + src] * pr;
                    }
                    Pn[cq * nb + i] = val;
                    if (cq == kq + 1 && i > k) {
                        const double v = fabs(val);
                        if (v > best) { best = v; bi = i; }
                    }
                }
            }
            if (cq == kq + 1) {                   // the next pivot (warp-uniform branch)
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const double ov = __shfl_down_sync(0xffffffffu, best, off);
                    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
                }
                if (lane == 0) pi[(kq + 1) & 1] = bi;
            }
            __syncthreads();
            double* t = Pc; Pc = Pn; Pn = t;
        }
        if (tid < nb && (tid < j0 || tid >= j0 + jb)) {    // the panel's row interchanges elsewhere
            const int c = tid;
            for (int kq = 0; kq < jb; ++kq) {
                const int k = j0 + kq, p = perm[k];
                if (p != k) {
                    const double t = A[k * ld + c];
                    A[k * ld + c] = A[p * ld + c];
                    A[p * ld + c] = t;
                }
            }
        }
        __syncthreads();
        for (int q = tid; q < 8 * ld; q += blockDim.x) {   // set the pivot rows aside
            const int kq = q / ld, c = q - kq * ld;
            double v = 0.0;
            if (kq < jb && c < nb && (c < j0 || c >= j0 + jb)) {
                v = A[(j0 + kq) * ld + c];
                A[(j0 + kq) * ld + c] = 0.0;
            }
            Bs[q] = v;
        }
        __syncthreads();
        {                                         // other columns += Panel * Bs; panel columns <- Panel
            const int g = lane >> 2, t4 = lane & 3;
            const int nt = (nb + 7) >> 3;
            for (int tile = warp; tile < nt * nt; tile += (int)(blockDim.x >> 5)) {
                const int ti = tile / nt, tj = tile - ti * nt;
                const int r = 8 * ti + g, cb = 8 * tj + g, c0 = 8 * tj + 2 * t4;
                double d0 = 0.0, d1 = 0.0;
#pragma unroll
                for (int kk = 0; kk < 8; kk += 4) {
                    const double a = (r < nb && kk + t4 < jb) ? Pc[(kk + t4) * nb + r] : 0.0;
                    const double b = (cb < nb) ? Bs[(kk + t4) * ld + cb] : 0.0;
                    dmma_884(d0, d1, a, b);
                }
                if (r < nb) {
                    double* cp = A + r * ld;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int c = c0 + e;
                        if (c >= nb) continue;
                        if (c >= j0 && c < j0 + jb) cp[c] = Pc[(c - j0) * nb + r];
                        else cp[c] += (e == 0) ? d0 : d1;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (tid == 0) {                               // the row interchanges, undone as column interchanges
        for (int c = 0; c < nb; ++c) idx[c] = c;
        for (int k = nb - 1; k >= 0; --k) {
            const int q = perm[k], t = idx[k];
            idx[k] = idx[q];
            idx[q] = t;
        }
    }
    __syncthreads();
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int i = q / nb, c = q - i * nb;
        B[i * ld + c] = A[i * ld + idx[c]];
    }
    __syncthreads();
    double* t = A; A = B; B = t;
    return bad;
}

// Inverse of the nb x nb block *A: blocked when *B can hold the panel copies and pivot rows.
static __device__ int sm_inverse(int nb, int ld, double*& A, double*& B, int* perm, int* idx, double* pv, int* pi) {
    if (16 * nb + 8 * ld <= nb * ld) return sm_inverse_blk(nb, ld, A, B, perm, idx, pi);
    return sm_inverse_unb(nb, ld, A, B, perm, idx, pv, pi);
}

// rows x columns < nb of a block, global (leading dimension ld) <-> shared memory (lds); the
// padding columns keep the zeros they were given.  256 threads, nb <= PC_SMEM_NB: thread t moves
// the entries t + 256 i (row-major over nb x nb), i < CP_K, stepping (row, column) without a
// division; cp_in issues all of its global loads before the first shared store, so one copy
// costs one L2 round trip.
#define CP_K 13                                  // 13 * 256 >= 56 * 56
static __device__ void cp_in(int nb, int ld, int lds, const double* __restrict__ src, double* __restrict__ dst) {
    const int dr = 256 / nb, dc = 256 - dr * nb;
    int r = threadIdx.x / nb, c = threadIdx.x - r * nb;
    double v[CP_K];
    int off[CP_K];
#pragma unroll
    for (int i = 0; i < CP_K; ++i) {
        off[i] = (r < nb) ? r * lds + c : -1;
        v[i] = (r < nb) ? src[r * ld + c] : 0.0;
        r += dr;
        c += dc;
        if (c >= nb) { c -= nb; ++r; }
    }
#pragma unroll
    for (int i = 0; i < CP_K; ++i)
        if (off[i] >= 0) dst[off[i]] = v[i];
}
static __device__ void cp_out(int nb, int ld, int lds, const double* __restrict__ src, double* __restrict__ dst) {
    const int dr = 256 / nb, dc = 256 - dr * nb;
    int r = threadIdx.x / nb, c = threadIdx.x - r * nb;
#pragma unroll
    for (int i = 0; i < CP_K; ++i) {
        if (r < nb) dst[r * ld + c] = src[r * lds + c];
        r += dr;
        c += dc;
        if (c >= nb) { c -= nb; ++r; }
    }
}

// ---------------------------------------------------------------- clusters of two CTAs
static __device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
static __device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// a value in the shared memory of CTA `rank` of this cluster, at the address of *p in this CTA
static __device__ __forceinline__ double ld_peer_cta(const double* p, uint32_t rank) {
    uint32_t ra;
    double v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(smem_u32(p)), "r"(rank));
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
    return v;
}
static __device__ __forceinline__ int ld_peer_cta(const int* p, uint32_t rank) {
    uint32_t ra;
    int v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(smem_u32(p)), "r"(rank));
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(ra) : "memory");
    return v;
}

// One CTA per partition (TW: per direction of a partition, a cluster of two), every working block
// resident in shared memory (nb <= PC_SMEM_NB).  The elimination runs in the CTA's local plane
// frame: rank 0 top-down over planes 0..zs-1, rank 1 bottom-up over planes Nz-1..zs+2, local
// slot sl of local plane t being global slot 4 - sl of plane Nz-1-t for rank 1.  TW: after its n
// planes each rank also forms the multipliers of the separator planes n, n+1 and their Schur contributions Q = -(couplings through
// the eliminated planes); rank 0 adds both ranks' Q to the separator blocks (read through
// distributed shared memory) and stores the inverse of the 2 nb x 2 nb separator matrix
// S = [S11 S12; S21 S22] by blocks (Dm = S11^-1, Dn = (S22 - S21 Dm S12)^-1):
//   plane zs:   slot 2 Sinv11 = Dm + Dm S12 Dn S21 Dm,  slot 3 Sinv12 = -Dm S12 Dn
//   plane zs+1: slot 1 Sinv21 = -Dn S21 Dm,             slot 2 Sinv22 = Dn
// so that the sweep solves the separator in two independent stages.
template <bool TW>
__global__ void __launch_bounds__(256) k_pc_factor_smem(PcGeom gin, double* __restrict__ A, int* __restrict__ info, int lds) {
    const int rank = TW ? (int)(blockIdx.x & 1u) : 0;
    const int part = TW ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const PcGeom g = pc_part(gin, part);
    extern __shared__ __align__(128) double dsm[];
    __shared__ int perm[64], idx[64];
    __shared__ double pv[8];
    __shared__ int pi[8];
    __shared__ int qoff[4], sbad;
    const int nb = g.nb, ld = g.ld;
    const int n2 = nb * lds;                   // one shared-memory block
    const int Nz = g.Nz;
    const int n = TW ? (rank == 0 ? g.zs : Nz - g.zs - 2) : Nz;
    double* buf[9];
    for (int q = 0; q < 9; ++q) buf[q] = dsm + (int64_t)q * n2;
    double *S0 = buf[0], *S1 = buf[1], *S2 = buf[2], *S3 = buf[3], *T = buf[4];
    double *Ui1 = buf[5], *Ui2 = buf[6], *U11 = buf[7], *U12 = buf[8];
    for (int64_t q = threadIdx.x; q < 9 * (int64_t)n2; q += blockDim.x) dsm[q] = 0.0;   // zero padding columns
    __syncthreads();
    double* base = A + (int64_t)part * Nz * 5 * g.bs;
    // block (local plane t, local slot sl)
    auto B = [&](int t, int sl) -> double* {
        const int P = (rank == 0) ? t : Nz - 1 - t;
        const int64_t off = ((int64_t)P * 5 + ((rank == 0) ? sl : 4 - sl)) * g.bs;
        // outside the partition's planes or the storage: recorded, and the partition's first block
        // stands in (the factors are then wrong and the error word says so)
        if (P < 0 || P >= Nz || !pc_range_ok(g, (int64_t)part * Nz * 5 * g.bs + off, g.bs)) return base;
        return base + off;
    };
    int bad = 0;
    for (int k = 0; k < n; ++k) {
        if (k >= 2) cp_in(nb, ld, lds, B(k, 0), S0);
        if (k >= 1) cp_in(nb, ld, lds, B(k, 1), S1);
        cp_in(nb, ld, lds, B(k, 2), S2);
        cp_in(nb, ld, lds, B(k, 3), S3);
        __syncthreads();
        if (k >= 2) {
            double* U2_2 = B(k - 2, 4);                                        // A(k-2, k), block diagonal
            sm_bd_left(g, lds, 1.0, S0, Ui2, 0.0, T);                               // L2 = A(k,k-2) Uinv_{k-2}
            double* t = S0; S0 = T; T = t;
            sm_gemm(nb, lds, -1.0, S0, U12, 1.0, S1);                           // A(k,k-1) -= L2 U1_{k-2}
            sm_bd_right(g, lds, -1.0, S0, U2_2, ld, 1.0, S2);                           // D -= L2 U2_{k-2}
            sm_bd_right(g, lds, -1.0, Ui2, U2_2, ld, 0.0, T);                           // -Uinv_{k-2} U2_{k-2}
            cp_out(nb, ld, lds, T, U2_2);                                             // (U2_{k-2} is not needed again)
            __syncthreads();
        }
        if (k >= 1) {
            const double* U2_1 = B(k - 1, 4);                                  // A(k-1, k+1), block diagonal
            if (k == 1) sm_bd_left(g, lds, 1.0, S1, Ui1, 0.0, T);                  // L1 = A(1,0) Uinv_0
            else sm_gemm(nb, lds, 1.0, S1, Ui1, 0.0, T);                        // L1 = (...) Uinv_{k-1}
            double* t = S1; S1 = T; T = t;
            sm_gemm(nb, lds, -1.0, S1, U11, 1.0, S2);                           // D -= L1 U1_{k-1}
            sm_bd_right(g, lds, -1.0, S1, U2_1, ld, 1.0, S3);                           // U1 = A(k,k+1) - L1 U2_{k-1}
        }
        bad |= sm_inverse(nb, lds, S2, T, perm, idx, pv, pi);              // (T: ping-pong buffer)
        sm_gemm(nb, lds, -1.0, S2, S3, 0.0, T);                                 // -Uinv_k U1_k
        if (k >= 2) cp_out(nb, ld, lds, S0, B(k, 0));
        if (k >= 1) cp_out(nb, ld, lds, S1, B(k, 1));
        cp_out(nb, ld, lds, S2, B(k, 2));
        cp_out(nb, ld, lds, T, B(k, 3));
        __syncthreads();
        // rotate: Uinv_{k-2} <- Uinv_{k-1} <- Uinv_k ; U1 likewise; freed blocks become S2 / S3
        double* fi = Ui2; Ui2 = Ui1; Ui1 = S2; S2 = fi;
        double* fu = U12; U12 = U11; U11 = S3; S3 = fu;
    }
    if constexpr (!TW) {
        // slot 4 of the last two planes: U2_k = A(k, k+2) = 0 for k >= Nz-2 (zeroed at assembly)
        if (threadIdx.x == 0) info[part] = bad;
    } else {
        // separator plane n: coupled to planes n-2 and n-1
        cp_in(nb, ld, lds, B(n, 0), S0);                                             // A(n, n-2)
        cp_in(nb, ld, lds, B(n, 1), S1);                                             // A(n, n-1)
        __syncthreads();
        double* U2_2 = B(n - 2, 4);                                            // A(n-2, n)
        double* U2_1 = B(n - 1, 4);                                            // A(n-1, n+1)
        sm_bd_left(g, lds, 1.0, S0, Ui2, 0.0, T);                                   // L2_n = A(n,n-2) Uinv_{n-2}
        { double* t = S0; S0 = T; T = t; }
        sm_gemm(nb, lds, -1.0, S0, U12, 1.0, S1);                               // A(n,n-1) - L2 U1_{n-2}
        sm_bd_right(g, lds, -1.0, S0, U2_2, ld, 0.0, S2);                               // Q(n,n) = -L2 U2_{n-2}
        sm_bd_right(g, lds, -1.0, Ui2, U2_2, ld, 0.0, T);                               // -Uinv_{n-2} U2_{n-2}
        cp_out(nb, ld, lds, T, U2_2);
        __syncthreads();
        sm_gemm(nb, lds, 1.0, S1, Ui1, 0.0, T);                                 // L1_n = (...) Uinv_{n-1}
        { double* t = S1; S1 = T; T = t; }
        sm_gemm(nb, lds, -1.0, S1, U11, 1.0, S2);                               // Q(n,n) -= L1 U1_{n-1}
        sm_bd_right(g, lds, -1.0, S1, U2_1, ld, 0.0, S3);                               // Q(n,n+1) = -L1 U2_{n-1}
        cp_out(nb, ld, lds, S0, B(n, 0));
        cp_out(nb, ld, lds, S1, B(n, 1));
        __syncthreads();
        // separator plane n+1: coupled to plane n-1 only
        cp_in(nb, ld, lds, B(n + 1, 0), S0);                                         // A(n+1, n-1)
        __syncthreads();
        sm_bd_left(g, lds, 1.0, S0, Ui1, 0.0, T);                                   // L2_{n+1} = A(n+1,n-1) Uinv_{n-1}
        { double* t = S0; S0 = T; T = t; }
        double* Q10 = Ui2;                                                     // (Uinv_{n-2}, U1_{n-2}: done)
        double* Q11 = U12;
        sm_gemm(nb, lds, -1.0, S0, U11, 0.0, Q10);                              // Q(n+1,n) = -L2 U1_{n-1}
        sm_bd_right(g, lds, -1.0, S0, U2_1, ld, 0.0, Q11);                              // Q(n+1,n+1) = -L2 U2_{n-1}
        sm_bd_right(g, lds, -1.0, Ui1, U2_1, ld, 0.0, T);                               // -Uinv_{n-1} U2_{n-1}
        cp_out(nb, ld, lds, T, U2_1);
        cp_out(nb, ld, lds, S0, B(n + 1, 0));
        if (threadIdx.x == 0) {
            qoff[0] = (int)(S2 - dsm);
            qoff[1] = (int)(S3 - dsm);
            qoff[2] = (int)(Q10 - dsm);
            qoff[3] = (int)(Q11 - dsm);
            sbad = bad;
        }
        __syncthreads();
        cluster_sync_all();                                                    // both ranks hold Q
        // rank 0: S = A_sep + Q(rank 0) + Q(rank 1); rank 1's local block (a, b) is separator (1-a, 1-b)
        double* Sb[4] = {S2, S3, Q10, Q11};                                    // separator (0,0) (0,1) (1,0) (1,1)
        if (rank == 0) {
            int ro[4];
            for (int q = 0; q < 4; ++q) ro[q] = ld_peer_cta(&qoff[3 - q], 1u);
            const double* Ab[4] = {B(n, 2), B(n, 3), B(n + 1, 1), B(n + 1, 2)};
            for (int q = 0; q < 4; ++q)
                for (int r = threadIdx.x >> 5; r < nb; r += blockDim.x >> 5)
                    for (int c = threadIdx.x & 31; c < nb; c += 32) {
                        const int es = r * lds + c;
                        Sb[q][es] = (Ab[q][r * ld + c] + Sb[q][es]) + ld_peer_cta(dsm + ro[q] + es, 1u);
                    }
            if (threadIdx.x == 0) bad |= ld_peer_cta(&sbad, 1u);
        }
        __syncthreads();
        cluster_sync_all();                                                    // rank 1's blocks have been read
        if (rank == 0) {
            double *S11 = Sb[0], *S12 = Sb[1], *S21 = Sb[2], *S22 = Sb[3];
            double* Xn = S0;                                                   // free: S0, S1, Ui1, U11 (+ T)
            double* Y = S1;
            bad |= sm_inverse(nb, lds, S11, T, perm, idx, pv, pi);             // Dm = S11^-1
            sm_gemm(nb, lds, -1.0, S11, S12, 0.0, Xn);                          // Xn = -Dm S12
            sm_gemm(nb, lds, 1.0, S21, S11, 0.0, Y);                            // Y = S21 Dm
            sm_gemm(nb, lds, 1.0, S21, Xn, 1.0, S22);                           // S22 - S21 Dm S12
            bad |= sm_inverse(nb, lds, S22, T, perm, idx, pv, pi);             // Dn = Sinv22
            sm_gemm(nb, lds, 1.0, Xn, S22, 0.0, S12);                           // Sinv12 = Xn Dn
            sm_gemm(nb, lds, -1.0, S22, Y, 0.0, S21);                           // Sinv21 = -Dn Y
            sm_gemm(nb, lds, -1.0, S12, Y, 1.0, S11);                           // Sinv11 = Dm - Sinv12 Y
            cp_out(nb, ld, lds, S11, B(n, 2));
            cp_out(nb, ld, lds, S12, B(n, 3));
            cp_out(nb, ld, lds, S21, B(n + 1, 1));
            cp_out(nb, ld, lds, S22, B(n + 1, 2));
            if (threadIdx.x == 0) info[part] = bad;
        }
    }
}

// ---------------------------------------------------------------- global-memory fallback (large blocks)
// C = beta C + alpha A B, row-major (leading dimension ld) in global memory; 256 threads, 32x32 tiles.
static __device__ void cta_gemm(int nb, int ld, double alpha, const double* A, const double* B, double beta,
                                double* C, double* shA, double* shB) {
    const int tid = threadIdx.x;
    const int tc = tid % 32, tr4 = (tid / 32) * 4;
    for (int ti = 0; ti < nb; ti += 32) {
        for (int tj = 0; tj < nb; tj += 32) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int kk = 0; kk < nb; kk += 32) {
                for (int q = tid; q < 1024; q += blockDim.x) {
                    int r = q / 32, cc = q % 32;
                    int gr = ti + r, gk = kk + cc;
                    shA[r * 32 + cc] = (gr < nb && gk < nb) ? A[(int64_t)gr * ld + gk] : 0.0;
                    int gk2 = kk + r, gc = tj + cc;
                    shB[r * 32 + cc] = (gk2 < nb && gc < nb) ? B[(int64_t)gk2 * ld + gc] : 0.0;
                }
                __syncthreads();
#pragma unroll 8
                for (int q = 0; q < 32; ++q) {
                    double b = shB[q * 32 + tc];
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] += shA[(tr4 + u) * 32 + q] * b;
                }
                __syncthreads();
            }
            const int gc = tj + tc;
            if (gc < nb) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    int gr = ti + tr4 + u;
                    if (gr < nb) {
                        double* cp = C + (int64_t)gr * ld + gc;
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

// Gauss-Jordan inverse of the row-major D (leading dimension ld) through an augmented scratch W
// (nb x 2nb, column-major over the augmented matrix).  Reading D column-major inverts D^T; the
// inverse of the transpose is the transpose of the inverse, so writing back the same way yields
// the row-major inverse.
static __device__ int cta_inverse(int nb, int ld, double* D, double* W, double* red_v, int* red_i) {
    const int tid = threadIdx.x;
    const int64_t n2 = (int64_t)nb * nb;
    for (int64_t q = tid; q < 2 * n2; q += blockDim.x) {
        int64_t col = q / nb, row = q % nb;
        W[q] = (col < nb) ? D[col * ld + row] : ((col - nb) == row ? 1.0 : 0.0);
    }
    __syncthreads();
    int bad = 0;
    for (int pc = 0; pc < nb; ++pc) {
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
    for (int64_t q = tid; q < n2; q += blockDim.x) {
        int64_t col = q / nb, row = q % nb;
        D[col * ld + row] = W[n2 + q];
    }
    __syncthreads();
    return bad;
}

__global__ void __launch_bounds__(256) k_pc_factor_glob(PcGeom gin, double* __restrict__ A, double* __restrict__ work,
                                                        int* __restrict__ info, int use_smem) {
    const PcGeom g = pc_part(gin, (int)blockIdx.x);
    extern __shared__ double dsm[];
    __shared__ double shA[1024], shB[1024];
    __shared__ double red_v[256];
    __shared__ int red_i[256];
    const int part = blockIdx.x;
    const int nb = g.nb, ld = g.ld;
    const int64_t n2 = (int64_t)nb * ld;
    const int64_t bs = g.bs;
    if (!pc_range_ok(g, (int64_t)part * g.Nz * 5 * bs, (int64_t)g.Nz * 5 * bs)) return;   // geometry beyond the storage
    double* base = A + (int64_t)part * g.Nz * 5 * bs;
    const int64_t n2w = (int64_t)gin.nb * ld;          // workspace stride: the largest partition's block
    double* T = work + (int64_t)part * 4 * n2w;
    double* W = use_smem ? dsm : (T + n2w);
    int bad = 0;
    for (int k = 0; k < g.Nz; ++k) {
        double* Ak = base + (int64_t)k * 5 * bs;
        double* Am2 = Ak;
        double* Am1 = Ak + bs;
        double* A0 = Ak + 2 * bs;
        double* Ap1 = Ak + 3 * bs;
        double* Uinv_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 2) * bs : nullptr;
        double* U1_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 3) * bs : nullptr;
        double* U2_1 = (k >= 1) ? base + ((int64_t)(k - 1) * 5 + 4) * bs : nullptr;
        double* Uinv_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 2) * bs : nullptr;
        double* U1_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 3) * bs : nullptr;
        double* U2_2 = (k >= 2) ? base + ((int64_t)(k - 2) * 5 + 4) * bs : nullptr;
        if (k >= 2) {
            cta_gemm(nb, ld, 1.0, Am2, Uinv_2, 0.0, T, shA, shB);
            cta_copy(n2, T, Am2);
            cta_gemm(nb, ld, -1.0, Am2, U1_2, 1.0, Am1, shA, shB);
            cta_gemm(nb, ld, -1.0, Am2, U2_2, 1.0, A0, shA, shB);
        }
        if (k >= 1) {
            cta_gemm(nb, ld, 1.0, Am1, Uinv_1, 0.0, T, shA, shB);
            cta_copy(n2, T, Am1);
            cta_gemm(nb, ld, -1.0, Am1, U1_1, 1.0, A0, shA, shB);
            cta_gemm(nb, ld, -1.0, Am1, U2_1, 1.0, Ap1, shA, shB);
        }
        bad |= cta_inverse(nb, ld, A0, W, red_v, red_i);
    }
    // fused-sweep form: slot 3 <- -Uinv_k U1_k, slot 4 <- -Uinv_k U2_k
    for (int k = 0; k < g.Nz; ++k) {
        double* Ak = base + (int64_t)k * 5 * bs;
        for (int slot = 3; slot <= 4; ++slot) {
            cta_gemm(nb, ld, -1.0, Ak + 2 * bs, Ak + slot * bs, 0.0, T, shA, shB);
            cta_copy(n2, T, Ak + slot * bs);
        }
    }
    if (threadIdx.x == 0) info[part] = bad;
}

// ---------------------------------------------------------------- sweeps
static __device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
static __device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait: false after `limit` polls (~2^22 by default; each poll may itself suspend briefly)
static __device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit = 1 << 22) {
    for (int it = 0; it < limit; ++it)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// Self-test of the bounded wait: an mbarrier that nothing arrives at, waited on by one warp with
// `polls` polls; the timeout sets bit 1 of *err exactly as in the sweep, and the kernel returns.
__global__ void k_selftest_mbar(int polls, int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    const bool arrived = mbar_wait(smem_u32(&bar), 0u, polls);
    __syncwarp();
    if (threadIdx.x == 0) {
        if (!arrived) atomicOr(err, 1);
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
    }
}

int selftest_mbar_timeout(int polls, int* err, cudaStream_t s) {
    k_selftest_mbar<<<1, 32, 0, s>>>(polls, err);
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

// Plane frame of one elimination direction.  TW = false: planes 0..Nz-1 top-down (the whole
// partition).  TW = true (twisted factorisation, a cluster of two CTAs per partition): rank 0
// eliminates planes 0..zs-1 top-down, rank 1 planes Nz-1..zs+2 bottom-up, and the separator
// planes zs, zs+1 take both ranks' contributions and an explicit inverse of their own.  In its
// local frame each rank sees planes
// t = 0, 1, .. (global gp(t)) with slot sl holding the coupling to local plane t + sl - 2, which is
// global slot gs(sl): bottom-up, A(t, t-1) local is A(p, p+1) global, and so on.  The local
// eliminated planes are 0..n-1; local n and n+1 are the separator planes.
struct PcFrame {
    int rank, n, Nz;
    __device__ __forceinline__ int gp(int t) const { return rank == 0 ? t : Nz - 1 - t; }
    __device__ __forceinline__ int gs(int sl) const { return rank == 0 ? sl : 4 - sl; }
};

// x = diag(1/sc) M^-1 diag(sc) b for all partitions: one CTA (256 threads; 8 lanes per group, two
// rows per group) per partition, or per direction of a partition (TW).  The factor blocks of the
// next planes stream into an NBUF-deep shared ring (cp.async.bulk with an mbarrier) while the
// current plane is swept.  NJ = ld / 16: lane l reads the column pairs (2l + 16j, 2l + 16j + 1),
// j < NJ, of a block row and of the solution plane with 16-byte loads (8-byte for FP32 blocks),
// a fixed, fully unrolled batch; padding columns hold zeros.
// Stages of one CTA (local frame):
//   F(t), t = 1..n-1:   z_t = b_t - L1_t z_{t-1} - L2_t z_{t-2}                  (slots 0, 1)
//   TW only:
//   X:                  p_n = b_n - L1_n z_{n-1} - L2_n z_{n-2},  p_{n+1} = b_{n+1} - L2_{n+1} z_{n-1}
//                       (b of the separator read by rank 0 only); the two ranks' p are summed
//                       through distributed shared memory into r
//   C0, C1:             the separator (both ranks; r_m, r_m1: global planes zs, zs+1)
//                       x of local plane n + i = [Sinv blocks of that plane] [r_m; r_m1]
//   B(t), t = n-1..0:   x_t = Uinv_t z_t + (-Uinv_t U1_t) x_{t+1} + (-Uinv_t U2_t) x_{t+2}  (slots 2..4)
// Without TW the backward stages run t = Nz-1..0 (couplings beyond the last plane are absent).
#define PA_THREADS 256
#define PA_LANES 8
#define PA_IO 8            // entries per thread whose loads the prologue / epilogue batch
template <int NJ, int NBUF, typename TS, bool TW>
__global__ void __launch_bounds__(PA_THREADS) k_pc_apply(PcGeom gin, const TS* __restrict__ A,
                                                         const double* __restrict__ b, const double* __restrict__ sc,
                                                         double* __restrict__ x, int* __restrict__ err, PaFuse F) {
    pdl_wait();                                // (launched programmatically inside the GMRES graph)
    pdl_trigger();
    if (F.stop && *F.stop) {                   // an Arnoldi step after the solve stopped: a zero direction
        if (blockIdx.x == 0 && threadIdx.x == 0 && F.out) *F.out = 0.0;
        return;                                // (every CTA of the grid returns here: no barrier is left open)
    }
    extern __shared__ __align__(128) double dsm[];
    __shared__ __align__(8) uint64_t bars[NBUF];
    constexpr int LD = NJ * 2 * PA_LANES;
    const int rank = TW ? (int)(blockIdx.x & 1u) : 0;
    const int part = TW ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const PcGeom g = pc_part(gin, part);
    const int nb = g.nb, Nz = g.Nz;
    const int tid = threadIdx.x;
    const int64_t bs = g.bs;
    const PcFrame fr{rank, TW ? (rank == 0 ? g.zs : Nz - g.zs - 2) : Nz, Nz};
    const int n = fr.n;
    double* xs = dsm;                          // [Nz][LD] local planes: b, then z (forward, in place); r on the separator
    double* xb = xs + (int64_t)Nz * LD;        // [Nz][LD]: x (backward sweep); padding columns zero
    double* xch = xb + (int64_t)Nz * LD;       // [2][LD]: this rank's partial right-hand sides of the separator (TW)
    TS* buf0 = reinterpret_cast<TS*>(xch + 2 * LD);   // NBUF ring buffers of [3 bs]
    const TS* base = A + (int64_t)part * Nz * 5 * bs;
    const int S = TW ? 2 * n + 2 : 2 * Nz - 1;
    // local planes whose b this CTA reads and whose x it writes
    const int nio = TW ? (rank == 0 ? n + 2 : n) : Nz;
    auto blk = [&](int t, int sl) -> const TS* { return base + ((int64_t)fr.gp(t) * 5 + fr.gs(sl)) * bs; };
    // the stage's copies: one contiguous run of slots, plus (TW stage X) one more block
    auto issue = [&](int s, uint32_t dst, uint32_t bar) {
        const uint32_t b1 = (uint32_t)(bs * sizeof(TS));
        const TS* src;
        uint32_t nblk;
        const TS* src2 = nullptr;
        if (s < n - 1) {                                   // F(t): slots 0, 1
            src = (fr.rank == 0) ? blk(s + 1, 0) : blk(s + 1, 1);
            nblk = 2;
        } else if (TW && s == n - 1) {                     // X: plane n slots 0, 1; plane n+1 slot 0
            src = (fr.rank == 0) ? blk(n, 0) : blk(n, 1);
            nblk = 2;
            src2 = blk(n + 1, 0);
        } else if (TW && s <= n + 1) {                     // C(i): the separator plane's two Sinv blocks
            const int P = fr.gp(n + (s - n));
            src = base + ((int64_t)P * 5 + (P == g.zs ? 2 : 1)) * bs;
            nblk = 2;
        } else {                                           // B(t): slots 2..4
            const int t = TW ? n - 1 - (s - (n + 2)) : Nz - 1 - (s - (Nz - 1));
            src = (fr.rank == 0) ? blk(t, 2) : blk(t, 4);
            nblk = 3;
        }
        const uint32_t tot = (nblk + (src2 ? 1u : 0u)) * b1;
        // a copy from outside the factor storage is not issued (its stage then times out)
        if (!pc_range_ok(g, (int64_t)(src - A), (int64_t)nblk * bs) || (src2 && !pc_range_ok(g, (int64_t)(src2 - A), bs)))
            return;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tot) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(dst), "l"(src), "r"(nblk * b1), "r"(bar) : "memory");
        if (src2)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         ::"r"(dst + nblk * b1), "l"(src2), "r"(b1), "r"(bar) : "memory");
    };
    if (tid == 0) {
        for (int q = 0; q < NBUF; ++q) mbar_init(smem_u32(&bars[q]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int rh = (nb + 1) >> 1;              // rows per half: a group of 8 lanes takes rows r0 and r0 + rh
    // the thread that issues the ring's copies and the warp that polls their mbarriers: the last warp
    // when it has no rows (nb <= 56), so neither the copy issue nor the poll is on the row warps' path
    // to the next barrier; that warp then takes no part in the prologue either
    const int issuer = (rh <= PA_THREADS / PA_LANES - 32 / PA_LANES) ? PA_THREADS - 32 : 0;
    const int pollw = issuer / 32;
    const int nthr = issuer ? issuer : PA_THREADS;   // threads that load b and clear xb
    if (tid == issuer)                           // the first NBUF stages are in flight from the start
        for (int q = 0; q < NBUF && q < S; ++q) issue(q, smem_u32(buf0 + (int64_t)q * 3 * bs), smem_u32(&bars[q]));
    const int fcol = F.V ? *F.col : 0;
    const double fscale = F.V ? *F.scale : 0.0;
    const double* __restrict__ src = F.V ? ((fcol == 0) ? F.src0 : F.src1) : b;
    // b (or the basis vector to normalise) into xs: PA_IO entries per thread at a time, all their
    // loads issued before the first use
    for (int q0 = (tid < nthr) ? tid : Nz * LD; q0 < Nz * LD; q0 += PA_IO * nthr) {
        int64_t gi[PA_IO];
        double bv[PA_IO], sv[PA_IO];
#pragma unroll
        for (int u = 0; u < PA_IO; ++u) {
            const int q = q0 + u * nthr;
            const int t = q / LD, l = q - t * LD;
            bool in = q < Nz * LD && l < nb && t < nio;
            gi[u] = in ? pc_glob(g, part, fr.gp(t), l) : -1;
            if (in && (gi[u] < 0 || gi[u] >= g.nstate)) {
                if (g.err) atomicOr(g.err, PC_ERR_RANGE);
                in = false;
                gi[u] = -1;
            }
            bv[u] = in ? src[gi[u]] : 0.0;
            sv[u] = (in && sc) ? sc[gi[u]] : 1.0;
        }
#pragma unroll
        for (int u = 0; u < PA_IO; ++u) {
            const int q = q0 + u * nthr;
            if (q >= Nz * LD) break;
            double v = 0.0;
            if (gi[u] >= 0) {
                double x0 = bv[u];
                if (F.V) {                       // normalise the basis vector on the way in
                    x0 = fscale * x0;
                    F.V[(int64_t)fcol * F.ldv + gi[u]] = x0;
                }
                v = sc ? x0 * sv[u] : x0;
            }
            xs[q] = v;
        }
    }
    for (int q = tid; q < Nz * LD && tid < nthr; q += nthr) xb[q] = 0.0;
    __syncthreads();
    const int lane = tid % PA_LANES;
    const int grp = tid / PA_LANES;
    const int r0 = grp, r1 = grp + rh;
    const bool act0 = r0 < rh, act1 = act0 && r1 < nb;
    int issued = (S < NBUF) ? S : NBUF;        // stages whose copies have been issued
    int bi = 0, pb = NBUF - 1;                 // this stage's ring buffer, the previous stage's
    uint32_t par = 0;
    // one block times one solution plane for both rows of the group (the vector loads are shared)
    using TS2 = typename std::conditional<std::is_same<TS, float>::value, float2, double2>::type;
    auto dot2 = [&](const TS* M, const double* v, double& acc0, double& acc1) {
        const TS2* ma = reinterpret_cast<const TS2*>(M + r0 * LD) + lane;
        const TS2* mb = reinterpret_cast<const TS2*>(M + (act1 ? r1 : r0) * LD) + lane;
        const double2* vp = reinterpret_cast<const double2*>(v) + lane;
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const double2 vv = vp[PA_LANES * j];
            const TS2 a = ma[PA_LANES * j], c = mb[PA_LANES * j];
            acc0 += (double)a.x * vv.x;
            acc1 += (double)c.x * vv.x;
            acc0 += (double)a.y * vv.y;
            acc1 += (double)c.y * vv.y;
        }
    };
    auto reduce = [&](double& acc0, double& acc1) {
#pragma unroll
        for (int off = PA_LANES / 2; off > 0; off >>= 1) {
            acc0 += __shfl_xor_sync(0xffffffffu, acc0, off, PA_LANES);
            acc1 += __shfl_xor_sync(0xffffffffu, acc1, off, PA_LANES);
        }
    };
    auto put = [&](double* row, double a0, double a1) {
        if (lane == 0 && act0) {
            row[r0] = a0;
            if (act1) row[r1] = a1;
        }
    };
    // One barrier per stage: it publishes the previous stage's rows and frees its buffer, which is
    // refilled right after it.  Forward rows overwrite b_t by z_t in xs (each row reads and writes
    // only its own entry of plane t); backward rows go to xb, as every row reads all of z_t.  Warp
    // `pollw` alone polls the copy's mbarrier; the barrier carries its answer to the others.
    auto stage = [&](int s) -> bool {
        TS* buf = buf0 + (int64_t)bi * 3 * bs;
        const bool arrived = ((tid >> 5) == pollw) ? mbar_wait(smem_u32(&bars[bi]), par) : true;
        if (!__syncthreads_and(arrived)) {       // uniform decision: no thread is left at a barrier
            if (tid == 0) atomicOr(err, 1);
            return false;
        }
        if (s >= 1 && s - 1 + NBUF < S) {        // the previous stage's buffer is free: refill it
            if (tid == issuer) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(s - 1 + NBUF, smem_u32(buf0 + (int64_t)pb * 3 * bs), smem_u32(&bars[pb]));
            }
            issued = s + NBUF;
        }
        const int64_t oL2 = (fr.rank == 0) ? 0 : bs, oL1 = (fr.rank == 0) ? bs : 0;
        double a0 = 0.0, a1 = 0.0;
        if (s < n - 1) {                                       // F(t)
            const int t = s + 1;
            double* row = xs + (int64_t)t * LD;
            double b0 = 0.0, b1 = 0.0;                         // this plane's b, read ahead of the products
            if (lane == 0 && act0) {
                b0 = row[r0];
                if (act1) b1 = row[r1];
            }
            if (act0) {
                dot2(buf + oL1, xs + (int64_t)(t - 1) * LD, a0, a1);
                if (t >= 2) dot2(buf + oL2, xs + (int64_t)(t - 2) * LD, a0, a1);
            }
            reduce(a0, a1);
            if (lane == 0 && act0) {
                row[r0] = b0 - a0;
                if (act1) row[r1] = b1 - a1;
            }
        } else if (TW && s == n - 1) {                         // X: partial right-hand sides of the separator
            if (act0) {
                dot2(buf + oL1, xs + (int64_t)(n - 1) * LD, a0, a1);
                dot2(buf + oL2, xs + (int64_t)(n - 2) * LD, a0, a1);
            }
            reduce(a0, a1);
            if (lane == 0 && act0) {
                xch[r0] = xs[(int64_t)n * LD + r0] - a0;
                if (act1) xch[r1] = xs[(int64_t)n * LD + r1] - a1;
            }
            a0 = a1 = 0.0;
            if (act0) dot2(buf + 2 * bs, xs + (int64_t)(n - 1) * LD, a0, a1);
            reduce(a0, a1);
            if (lane == 0 && act0) {
                xch[LD + r0] = xs[(int64_t)(n + 1) * LD + r0] - a0;
                if (act1) xch[LD + r1] = xs[(int64_t)(n + 1) * LD + r1] - a1;
            }
        } else if (TW && s <= n + 1) {                         // C(i): both ranks solve the separator
            const int t = n + (s - n);
            const int lz0 = (fr.rank == 0) ? n : n + 1;        // local plane of global zs
            if (act0) {
                dot2(buf, xs + (int64_t)lz0 * LD, a0, a1);
                dot2(buf + bs, xs + (int64_t)(2 * n + 1 - lz0) * LD, a0, a1);
            }
            reduce(a0, a1);
            put(xb + (int64_t)t * LD, a0, a1);
        } else {                                               // B(t)
            const int t = TW ? n - 1 - (s - (n + 2)) : Nz - 1 - (s - (Nz - 1));
            const int lim = TW ? n + 2 : Nz;
            const int64_t oU = (fr.rank == 0) ? 0 : 2 * bs, oW2 = (fr.rank == 0) ? 2 * bs : 0;
            if (act0) {
                dot2(buf + oU, xs + (int64_t)t * LD, a0, a1);
                if (t + 1 < lim) dot2(buf + bs, xb + (int64_t)(t + 1) * LD, a0, a1);
                if (t + 2 < lim) dot2(buf + oW2, xb + (int64_t)(t + 2) * LD, a0, a1);
            }
            reduce(a0, a1);
            put(xb + (int64_t)t * LD, a0, a1);
        }
        pb = bi;
        if (++bi == NBUF) {
            bi = 0;
            par ^= 1u;
        }
        return true;
    };
    bool ok = true;
    int s = 0;
    const int s_x = TW ? n : S;                  // stages before the exchange
    for (; s < s_x && ok; ++s) ok = stage(s);
    if constexpr (TW) {
        __syncthreads();                         // this rank's partials are in xch
        cluster_sync_all();                      // ... and the other rank's (both ranks always arrive)
        if (ok) {
            const uint32_t other = (uint32_t)(fr.rank ^ 1);
            for (int q = tid; q < 2 * LD; q += blockDim.x) {
                const int c = q / LD, l = q - c * LD;   // separator plane zs + c, row l
                if (l >= nb) continue;
                // plane zs + c is slot c of rank 0's xch and slot 1 - c of rank 1's; the sum is
                // taken in the same order on both ranks, so both hold the same r
                const double* q0 = xch + c * LD + l;
                const double* q1 = xch + (1 - c) * LD + l;
                const double p0 = (fr.rank == 0) ? *q0 : ld_peer_cta(q0, other);
                const double p1 = (fr.rank == 0) ? ld_peer_cta(q1, other) : *q1;
                xs[(int64_t)(n + ((fr.rank == 0) ? c : 1 - c)) * LD + l] = p0 + p1;
            }
        }
        __syncthreads();
    }
    for (; s < S && ok; ++s) ok = stage(s);
    const int s_fail = ok ? S : s - 1;           // first stage whose data was not consumed
    __syncthreads();                             // the last stage's rows
    double ss = 0.0;
    if (!ok) {                                   // drain copies still in flight (bounded) and leave x untouched
        if (tid == 0)
            for (int s2 = s_fail; s2 < issued; ++s2)
                mbar_wait(smem_u32(&bars[s2 % NBUF]), (uint32_t)((s2 / NBUF) & 1));
    } else {                                     // x out, PA_IO entries per thread at a time
        for (int q0 = tid; q0 < Nz * LD; q0 += PA_IO * PA_THREADS) {
            int64_t gi[PA_IO];
            double sv[PA_IO];
#pragma unroll
            for (int u = 0; u < PA_IO; ++u) {
                const int q = q0 + u * PA_THREADS;
                const int t = q / LD, l = q - t * LD;
                bool in = q < Nz * LD && l < nb && t < nio;
                gi[u] = in ? pc_glob(g, part, fr.gp(t), l) : -1;
                if (in && (gi[u] < 0 || gi[u] >= g.nstate)) {
                    if (g.err) atomicOr(g.err, PC_ERR_RANGE);
                    in = false;
                    gi[u] = -1;
                }
                sv[u] = (in && sc) ? sc[gi[u]] : 1.0;
            }
#pragma unroll
            for (int u = 0; u < PA_IO; ++u) {
                if (gi[u] < 0) continue;
                const int q = q0 + u * PA_THREADS;
                const double xv = sc ? xb[q] / sv[u] : xb[q];
                x[gi[u]] = xv;
                ss += xv * xv;
            }
        }
    }
    if (F.out) {                                 // rms of the result: per-CTA partial, last CTA finishes
        __shared__ double wsum[PA_THREADS / 32];
        __shared__ bool last;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, off);
        if ((tid & 31) == 0) wsum[tid >> 5] = ss;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < PA_THREADS / 32; ++w) t += wsum[w];
            F.part[blockIdx.x] = t;
            __threadfence();
            last = (atomicAdd(F.ticket, 1u) == gridDim.x - 1);
        }
        __syncthreads();
        if (last && tid == 0) {
            __threadfence();
            *F.out = sqrt(sum_partials(F.part, (int)gridDim.x, 1) / (double)F.n);
            *F.ticket = 0u;
        }
    }
    if constexpr (TW) cluster_sync_all();        // the other rank has finished reading this CTA's xch
}

// Sweep for partitions too large for the shared-memory pipeline: same fused stages, operands read
// from global memory (L2).
template <typename TS>
__global__ void __launch_bounds__(512) k_pc_apply_glob(PcGeom gin, const TS* __restrict__ A,
                                                       const double* __restrict__ b, const double* __restrict__ sc,
                                                       double* __restrict__ x, double* __restrict__ xs_all) {
    __shared__ double tv[512];
    const int part = blockIdx.x;
    const PcGeom g = pc_part(gin, part);
    const int nb = g.nb, ld = g.ld;
    const int tid = threadIdx.x;
    const int64_t bs = g.bs;
    double* xs = xs_all + (int64_t)part * g.Nz * ld;
    if (!pc_range_ok(g, (int64_t)part * g.Nz * 5 * bs, (int64_t)g.Nz * 5 * bs)) return;   // geometry beyond the storage
    const TS* base = A + (int64_t)part * g.Nz * 5 * bs;
    for (int64_t q = tid; q < (int64_t)g.Nz * nb; q += blockDim.x) {
        int k = (int)(q / nb), l = (int)(q % nb);
        int64_t gi = pc_glob(g, part, k, l);
        xs[(int64_t)k * ld + l] = sc ? b[gi] * sc[gi] : b[gi];
    }
    __syncthreads();
    const int S = 2 * g.Nz - 1;
    for (int s = 0; s < S; ++s) {
        const bool fwd = s < g.Nz - 1;
        const int k = fwd ? s + 1 : g.Nz - 1 - (s - (g.Nz - 1));
        const TS* Ak = base + (int64_t)k * 5 * bs;
        const TS* M0 = fwd ? Ak + bs : Ak + 2 * bs;
        const double* v0 = fwd ? xs + (int64_t)(k - 1) * ld : xs + (int64_t)k * ld;
        const TS* M1 = fwd ? ((k >= 2) ? Ak : nullptr) : ((k + 1 < g.Nz) ? Ak + 3 * bs : nullptr);
        const double* v1 = fwd ? ((k >= 2) ? xs + (int64_t)(k - 2) * ld : nullptr)
                               : ((k + 1 < g.Nz) ? xs + (int64_t)(k + 1) * ld : nullptr);
        const TS* M2 = (!fwd && k + 2 < g.Nz) ? Ak + 4 * bs : nullptr;
        const double* v2 = (!fwd && k + 2 < g.Nz) ? xs + (int64_t)(k + 2) * ld : nullptr;
        for (int r = tid; r < nb; r += blockDim.x) {
            double acc = 0.0;
            for (int c = 0; c < nb; ++c) acc += (double)M0[(int64_t)r * ld + c] * v0[c];
            if (M1) for (int c = 0; c < nb; ++c) acc += (double)M1[(int64_t)r * ld + c] * v1[c];
            if (M2) for (int c = 0; c < nb; ++c) acc += (double)M2[(int64_t)r * ld + c] * v2[c];
            tv[r] = fwd ? xs[(int64_t)k * ld + r] - acc : acc;
        }
        __syncthreads();
        for (int r = tid; r < nb; r += blockDim.x) xs[(int64_t)k * ld + r] = tv[r];
        __syncthreads();
    }
    for (int64_t q = tid; q < (int64_t)g.Nz * nb; q += blockDim.x) {
        int k = (int)(q / nb), l = (int)(q % nb);
        int64_t gi = pc_glob(g, part, k, l);
        x[gi] = sc ? xs[(int64_t)k * ld + l] / sc[gi] : xs[(int64_t)k * ld + l];
    }
}

// Largest partition of mode 3 the shared-memory kernels take at their tuned size.
#define PC_SPLIT_NB 48

static PcGeom geom_of_params(const dv_step_params& p, int mode) {
    PcGeom g;
    g.Nr = p.Nr;
    g.Nth = p.Nth;
    g.Nz = p.Nz;
    g.wall = p.wall_on;
    g.rg = g.tg = 1;
    g.cap = -1;
    g.nstate = (int64_t)DV_NV * p.Nr * p.Nth * p.Nz + (p.wall_on ? (int64_t)p.Nth * p.Nz : 0);
    g.err = nullptr;
    // mode 3 is the split form of mode 2 (a factorisation records it as the mode it used): derive it again
    if (mode == 3) mode = 2;
    // mode 2 needs a second ring and a second sector; below that it is mode 0 (or 1 for one sector)
    if (mode == 2 && (p.Nr < 2 || p.Nth < 2)) mode = 0;
    g.mode = (p.Nth > 1 && (mode == 0 || mode == 2)) ? mode : 1;
    g.nc = (int64_t)p.Nr * p.Nth * p.Nz;
    static const bool split_ok = [] {
        const char* e = getenv("DVTSA_PC_SPLIT");
        return !(e && e[0] == '0');
    }();
    if (g.mode == 2 && split_ok && std::max(DV_NV * (g.Nr - 1) + (g.wall ? 1 : 0), DV_NV * g.Nth) > PC_SMEM_NB) {
        // too large for the shared-memory kernels: split the sectors into ring groups and the core
        // ring into theta groups of at most PC_SPLIT_NB unknowns (mode 3)
        g.mode = 3;
        auto nb_ring = [&](int G) {
            int worst = 0;
            for (int gi = 0; gi < G; ++gi) {
                int a0, a1;
                pc_group(g.Nr - 1, G, gi, a0, a1);
                worst = std::max(worst, DV_NV * (a1 - a0) + ((g.wall && gi == G - 1) ? 1 : 0));
            }
            return worst;
        };
        g.rg = 1;
        while (g.rg < g.Nr - 1 && nb_ring(g.rg) > PC_SPLIT_NB) ++g.rg;
        g.tg = 1;
        while (g.tg < g.Nth && DV_NV * ((g.Nth + g.tg - 1) / g.tg) > PC_SPLIT_NB) ++g.tg;
        g.nb = std::max(nb_ring(g.rg), DV_NV * ((g.Nth + g.tg - 1) / g.tg));
        g.ncv = g.nb;
        g.nparts = g.Nth * g.rg + g.tg;
        g.ld = pc_ld(g.nb);
        g.bs = (((int64_t)g.nb * g.ld + 1) / 2) * 2;
        g.zs = 0;
        return g;
    }
    if (g.mode == 0) {
        g.nb = DV_NV * g.Nr + (g.wall ? 1 : 0);
        g.ncv = DV_NV * g.Nr;
        g.nparts = g.Nth;
    } else if (g.mode == 2) {
        const int nb_sector = DV_NV * (g.Nr - 1) + (g.wall ? 1 : 0), nb_core = DV_NV * g.Nth;
        g.nb = std::max(nb_sector, nb_core);
        g.ncv = g.nb;                       // per-partition values come from pc_part
        g.nparts = g.Nth + 1;
    } else {
        g.nb = DV_NV * g.Nr * g.Nth + (g.wall ? g.Nth : 0);
        g.ncv = DV_NV * g.Nr * g.Nth;
        g.nparts = 1;
    }
    g.ld = pc_ld(g.nb);
    g.bs = (((int64_t)g.nb * g.ld + 1) / 2) * 2;
    g.zs = 0;
    return g;
}

static PcGeom geom_of(const dv_model* m, int mode) {
    PcGeom g = geom_of_params(m->p, mode);
    g.cap = m->pc_doubles;
    g.err = m->d_err;
    return g;
}

void precond_capacity(const dv_step_params& p, int* cap_nb, int* cap_parts, int64_t* pc_need, int64_t* work_need) {
    int nb = 0, parts = 0;
    int64_t need = 0;
    for (int mode : {0, 1, 2}) {
        const PcGeom g = geom_of_params(p, mode);
        if (g.mode == 1 && g.nb > 512) continue;       // whole cross-sections only up to 512 unknowns
        nb = std::max(nb, g.nb);
        parts = std::max(parts, g.nparts);
        need = std::max(need, precond_doubles(g.nb, g.nparts, g.Nz));
    }
    *cap_nb = nb;
    *cap_parts = parts;
    *pc_need = need;
    *work_need = precond_work_doubles(nb, parts, p.Nz);
}

// Host check of the partition maps of a geometry (tests): every (partition, plane, local index) maps
// to an unknown inside the state, each unknown exactly once, and the inverse map (cell / wall ->
// partition, local index) agrees.  Returns the number of violations.
int64_t precond_check_maps(const dv_step_params& p, int mode, int* nparts_out, int* nb_out) {
    const PcGeom g = geom_of_params(p, mode);
    const int64_t nc = g.nc, offw = (int64_t)DV_NV * nc, n = offw + (g.wall ? (int64_t)g.Nth * g.Nz : 0);
    std::vector<int> seen(n, 0);
    int64_t bad = 0;
    for (int part = 0; part < g.nparts; ++part) {
        const PcGeom q = pc_part(g, part);
        if (q.nb > g.nb || q.ncv > q.nb || q.nb < 1) ++bad;
        for (int k = 0; k < g.Nz; ++k)
            for (int l = 0; l < q.nb; ++l) {
                const int64_t gi = pc_glob(q, part, k, l);
                if (gi < 0 || gi >= n) { ++bad; continue; }
                seen[gi] += 1;
            }
    }
    for (int64_t u = 0; u < n; ++u)
        if (seen[u] != 1) ++bad;
    for (int i = 0; i < g.Nr; ++i)
        for (int j = 0; j < g.Nth; ++j)
            for (int k = 0; k < g.Nz; ++k) {
                const int part = pc_part_of(g, i, j);
                if (part < 0 || part >= g.nparts) { ++bad; continue; }
                const PcGeom q = pc_part(g, part);
                const int64_t cell = ((int64_t)i * g.Nth + j) * g.Nz + k;
                for (int v = 0; v < DV_NV; ++v) {
                    const int l = pc_local(g, i, j, v);
                    if (l < 0 || l >= q.ncv || pc_glob(q, part, k, l) != v * nc + cell) ++bad;
                }
                if (g.wall && i == g.Nr - 1) {
                    const int l = pc_local(g, i, j, DV_NV);
                    if (l < q.ncv || l >= q.nb || pc_glob(q, part, k, l) != offw + (int64_t)j * g.Nz + k) ++bad;
                }
            }
    *nparts_out = g.nparts;
    *nb_out = g.nb;
    return bad;
}

int precond_partitions(const dv_model* m, int* mode, int* zs, int* nb_out, int cap) {
    if (!m->pc_ready) return 0;
    const PcGeom g = geom_of(m, m->pc_mode);
    *mode = g.mode;
    *zs = m->pc_zs;
    for (int q = 0; q < g.nparts && q < cap; ++q) nb_out[q] = pc_part(g, q).nb;
    return g.nparts;
}

// the geometry the current factors were computed with
static PcGeom geom_factored(const dv_model* m) {
    PcGeom g = geom_of(m, m->pc_mode);
    g.zs = m->pc_zs;
    return g;
}

static int smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

int64_t precond_doubles(int nb, int nparts, int Nz) {
    const int ld = pc_ld(nb);
    return (int64_t)nparts * Nz * 5 * ((((int64_t)nb * ld + 1) / 2) * 2);
}

int64_t precond_work_doubles(int nb, int nparts, int Nz) {
    const int ld = pc_ld(nb);
    return std::max((int64_t)nparts * 4 * (int64_t)nb * ld, (int64_t)nparts * Nz * (int64_t)ld);
}

// a launch of `kern` as clusters of two CTAs (grid = 2 x partitions)
template <typename... KArgs, typename... Args>
static cudaError_t launch_pair(void (*kern)(KArgs...), unsigned grid, unsigned block, size_t dyn, cudaStream_t s,
                               bool pdl, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 2 : 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

static size_t apply_smem(const PcGeom& g, int nbuf, size_t tsize);
static bool apply_fusable(const PcGeom& g, size_t tsize);
static size_t pc_tsize(const dv_model* m);

// Twisted factorisation: the top-down and bottom-up eliminations run at the same time and meet at
// the separator planes zs, zs+1, which halves the sequential plane chain of the factorisation and
// of both sweeps.  Taken when each direction keeps at least three planes and both kernels run from
// shared memory; DVTSA_PC_TWIST=0 keeps the one-directional form.
static int pc_twist_zs(const PcGeom& g, size_t tsize, bool factor_smem) {
    const char* e = getenv("DVTSA_PC_TWIST");
    if (e && e[0] == '0') return 0;
    if (g.Nz < 8 || !factor_smem || !apply_fusable(g, tsize)) return 0;
    return (g.Nz - 2) / 2;
}

int precond_factor(dv_model* m, const double* J, double dh, int mode, cudaStream_t s) {
    PcGeom g = geom_of(m, mode);
    if (g.nb > m->pc_cap_nb || g.nparts > m->pc_cap_parts) {
        set_error("preconditioner partition larger than the workspace allocated at model creation");
        return DV_ERR_ARG;
    }
    if (g.nb > 512) {
        set_error("preconditioner block size above the supported 512 (use theta_block)");
        return DV_ERR_UNSUPPORTED;
    }
    const int64_t total = (int64_t)g.nparts * g.Nz * 5 * g.bs;
    DV_LAUNCH(dv::K_PC_FACTOR, s, k_pc_zero<<<std::min<int64_t>((total + 255) / 256, 4096), 256, 0, s>>>(m->d_pc, total));
    dim3 grid((unsigned)((m->nc + 127) / 128), DV_NSLOT);
    DV_LAUNCH(dv::K_PC_FACTOR, s, k_pc_scatter<<<grid, 128, 0, s>>>(g, J, dh, m->d_pc));
    const int optin = smem_optin();
    const size_t budget = (size_t)optin - 2048;             // static shared memory of the kernel
    const int lds = pc_lds(g.nb, budget);
    const size_t dyn = (size_t)9 * g.nb * lds * sizeof(double);
    const bool factor_smem = g.nb <= PC_SMEM_NB && dyn <= budget;
    g.zs = pc_twist_zs(g, pc_tsize(m), factor_smem);
    if (factor_smem && g.zs > 0) {
        if (dyn > 48 * 1024)
            DV_CUDA(allow_dyn_smem((const void*)k_pc_factor_smem<true>));
        DV_LAUNCH(dv::K_PC_FACTOR, s,
                  DV_CUDA(launch_pair(k_pc_factor_smem<true>, 2u * g.nparts, 256u, dyn, s, false, g, m->d_pc, m->d_pc_info,
                                      lds)));
    } else if (factor_smem) {
        if (dyn > 48 * 1024)
            DV_CUDA(allow_dyn_smem((const void*)k_pc_factor_smem<false>));
        DV_LAUNCH(dv::K_PC_FACTOR, s, k_pc_factor_smem<false><<<g.nparts, 256, dyn, s>>>(g, m->d_pc, m->d_pc_info, lds));
    } else {
        const size_t static_smem = (2 * 1024 + 256) * sizeof(double) + 256 * sizeof(int);
        size_t need = (size_t)2 * g.nb * g.nb * sizeof(double);
        int use_smem = (need + static_smem) <= (size_t)optin ? 1 : 0;
        size_t dyn = use_smem ? need : 0;
        if (use_smem && dyn > 48 * 1024)
            DV_CUDA(allow_dyn_smem((const void*)k_pc_factor_glob));
        DV_LAUNCH(dv::K_PC_FACTOR, s, k_pc_factor_glob<<<g.nparts, 256, dyn, s>>>(g, m->d_pc, m->d_pc_work, m->d_pc_info, use_smem));
    }
    if (m->pc_fp32) {               // the sweep streams an FP32 copy of the factors
        const int64_t tot = (int64_t)g.nparts * g.Nz * 5 * g.bs;
        DV_LAUNCH(dv::K_PC_FACTOR, s, k_pc_to_f32<<<std::min<int64_t>((tot + 255) / 256, 4096), 256, 0, s>>>(m->d_pc, m->d_pc32, tot));
    }
    DV_CUDA(cudaGetLastError());
    m->pc_mode = g.mode;
    m->pc_nb = g.nb;
    m->pc_nparts = g.nparts;
    m->pc_zs = g.zs;
    m->pc_ready = 1;
    return DV_OK;
}

// shared memory of the sweep with an NBUF-deep ring: solution planes, one plane of scratch, buffers
// shared memory of the sweep with an NBUF-deep ring of factor blocks stored as `tsize`-byte values
static size_t apply_smem(const PcGeom& g, int nbuf, size_t tsize) {
    return sizeof(double) * (size_t)(2 * (int64_t)g.Nz * g.ld + 2 * g.ld) + tsize * (size_t)((int64_t)nbuf * 3 * g.bs);
}

static size_t pc_tsize(const dv_model* m) { return m->pc_fp32 ? sizeof(float) : sizeof(double); }

// ring depth: three stages in flight when they fit in shared memory, else two
static int apply_nbuf(const PcGeom& g, size_t tsize, int want = 0) {
    const bool three = apply_smem(g, 3, tsize) <= (size_t)smem_optin();
    return (three && want != 2) ? 3 : 2;
}

template <int NJ, int NBUF, typename TS, bool TW>
static void launch_apply_tw(const PcGeom& g, dv_model* m, const TS* A, const double* b, const double* sc, double* x,
                            cudaStream_t s, const PaFuse& F, bool count) {
    const size_t dyn = apply_smem(g, NBUF, sizeof(TS));
    auto kern = k_pc_apply<NJ, NBUF, TS, TW>;
    if (dyn > 48 * 1024) allow_dyn_smem((const void*)kern);
    if (count) prof_begin(dv::K_PC_APPLY, s);
    if (TW) launch_pair(kern, 2u * g.nparts, PA_THREADS, dyn, s, F.pdl, g, A, b, sc, x, m->d_err, F);
    else kern<<<g.nparts, PA_THREADS, dyn, s>>>(g, A, b, sc, x, m->d_err, F);
    if (count) prof_end(dv::K_PC_APPLY, s);
}

template <int NJ, int NBUF, typename TS>
static void launch_apply_k(const PcGeom& g, dv_model* m, const TS* A, const double* b, const double* sc, double* x,
                           cudaStream_t s, const PaFuse& F, bool count) {
    if (g.zs > 0) launch_apply_tw<NJ, NBUF, TS, true>(g, m, A, b, sc, x, s, F, count);
    else launch_apply_tw<NJ, NBUF, TS, false>(g, m, A, b, sc, x, s, F, count);
}

template <int NJ>
static void launch_apply_nj(const PcGeom& g, dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s,
                            const PaFuse& F, bool count) {
    if (m->pc_fp32) {               // factors stored in FP32 (mixed-precision Krylov), products in FP64
        if (apply_nbuf(g, sizeof(float), m->tune.sweep_nbuf) == 3) launch_apply_k<NJ, 3, float>(g, m, m->d_pc32, b, sc, x, s, F, count);
        else launch_apply_k<NJ, 2, float>(g, m, m->d_pc32, b, sc, x, s, F, count);
    } else {
        if (apply_nbuf(g, sizeof(double), m->tune.sweep_nbuf) == 3) launch_apply_k<NJ, 3, double>(g, m, m->d_pc, b, sc, x, s, F, count);
        else launch_apply_k<NJ, 2, double>(g, m, m->d_pc, b, sc, x, s, F, count);
    }
}

static void launch_apply(const PcGeom& g, dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s,
                         const PaFuse& F, bool count) {
    switch (g.ld / (2 * PA_LANES)) {
        case 1: launch_apply_nj<1>(g, m, b, sc, x, s, F, count); break;
        case 2: launch_apply_nj<2>(g, m, b, sc, x, s, F, count); break;
        case 3: launch_apply_nj<3>(g, m, b, sc, x, s, F, count); break;
        default: launch_apply_nj<4>(g, m, b, sc, x, s, F, count); break;
    }
}

int precond_apply(dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s) {
    if (!m->pc_ready) {
        set_error("preconditioner applied before it was factorised");
        return DV_ERR_ARG;
    }
    PcGeom g = geom_factored(m);
    if (precond_apply_fusable(m)) {
        launch_apply(g, m, b, sc, x, s, PaFuse(), true);
    } else {
        if (m->pc_fp32) {
            DV_LAUNCH(dv::K_PC_APPLY, s, k_pc_apply_glob<float><<<g.nparts, 512, 0, s>>>(g, m->d_pc32, b, sc, x, m->d_pc_work));
        } else {
            DV_LAUNCH(dv::K_PC_APPLY, s, k_pc_apply_glob<double><<<g.nparts, 512, 0, s>>>(g, m->d_pc, b, sc, x, m->d_pc_work));
        }
    }
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

static bool apply_fusable(const PcGeom& g, size_t tsize) {
    return g.nb <= 64 && g.ld % (2 * PA_LANES) == 0 && apply_smem(g, 2, tsize) <= (size_t)smem_optin();
}

bool precond_apply_fusable(dv_model* m) { return apply_fusable(geom_factored(m), pc_tsize(m)); }

int precond_apply_capture(dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s,
                          const PaFuse& F) {
    PcGeom g = geom_factored(m);
    if (precond_apply_fusable(m)) {
        launch_apply(g, m, b, sc, x, s, F, false);    // attributes were set by an earlier precond_apply
    } else {
        if (F.V || F.out) {
            set_error("fused sweep requested for a partition the shared-memory sweep does not take");
            return DV_ERR_ARG;
        }
        if (m->pc_fp32) k_pc_apply_glob<float><<<g.nparts, 512, 0, s>>>(g, m->d_pc32, b, sc, x, m->d_pc_work);
        else k_pc_apply_glob<double><<<g.nparts, 512, 0, s>>>(g, m->d_pc, b, sc, x, m->d_pc_work);
    }
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

// ---------------------------------------------------------------- FP32 assembled-Jacobian operator
// Mixed-precision Krylov: the GMRES operator u -> (v - dh J v)/s, v = u s, with J the FP32 block
// Jacobian (the same difference quotients as the FD Jacobian, rounded), products and sums in FP32;
// replaces the FP64 finite-difference matvec (core/solver.py:196-203) inside GMRES.  One thread per
// cell computes its six rows and, for an outer-ring cell, its wall node's row.  Blocks known to be
// structurally zero (loading rows of neighbour slots, the wall row of inner cells) are not read.
__global__ void __launch_bounds__(256) k_spmv32(int Nr, int Nth, int Nz, int wall, const float* __restrict__ J,
                                                const double* __restrict__ u, const double* __restrict__ sc,
                                                double dh, const double* __restrict__ dh_dev, double* __restrict__ out) {
    const int64_t nc = (int64_t)Nr * Nth * Nz;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const double dhv = dh_dev ? dh_dev[1] : dh;
    const int k = (int)(c % Nz);
    const int64_t rr = c / Nz;
    const int j = (int)(rr % Nth);
    const int i = (int)(rr / Nth);
    const bool outer_wall = wall && i == Nr - 1;
    const int64_t offw = (int64_t)DV_NV * nc;
    float acc[DV_NB];
#pragma unroll
    for (int r = 0; r < DV_NB; ++r) acc[r] = 0.0f;
#pragma unroll
    for (int slot = 0; slot < DV_NSLOT; ++slot) {
        int ni = i, nj = j, nk = k;
        bool ok = true;
        switch (slot) {
            case 0: break;
            case 1: nk = k - 1; ok = nk >= 0; break;
            case 2: nk = k + 1; ok = nk < Nz; break;
            case 3: nk = k - 2; ok = nk >= 0; break;
            case 4: nk = k + 2; ok = nk < Nz; break;
            case 5: ni = i - 1; ok = ni >= 0; break;
            case 6: ni = i + 1; ok = ni < Nr; break;
            case 7: ok = Nth > 1; nj = (j == 0) ? Nth - 1 : j - 1; break;
            default: ok = Nth > 1; nj = (j == Nth - 1) ? 0 : j + 1; break;
        }
        if (!ok) continue;
        const int64_t cn = ((int64_t)ni * Nth + nj) * Nz + nk;
        const float* Js = J + (int64_t)slot * DV_NB * DV_NB * nc + c;
#pragma unroll
        for (int cv = 0; cv < DV_NV; ++cv) {
            const int64_t q = (int64_t)cv * nc + cn;
            const float x = (float)(u[q] * sc[q]);
#pragma unroll
            for (int rv = 0; rv < DV_NV; ++rv) {
                if ((rv == 3 || rv == 4) && slot != 0) continue;
                acc[rv] = fmaf(Js[(int64_t)(rv * DV_NB + cv) * nc], x, acc[rv]);
            }
            if (outer_wall && slot == 0) acc[DV_NV] = fmaf(Js[(int64_t)(DV_NV * DV_NB + cv) * nc], x, acc[DV_NV]);
        }
        if (wall && ni == Nr - 1) {      // the neighbour's wall node (column 6)
            const int64_t q = offw + (int64_t)nj * Nz + nk;
            const float x = (float)(u[q] * sc[q]);
            if (slot == 0) {
#pragma unroll
                for (int rv = 0; rv < DV_NV; ++rv) {
                    if (rv == 3 || rv == 4) continue;
                    acc[rv] = fmaf(Js[(int64_t)(rv * DV_NB + DV_NV) * nc], x, acc[rv]);
                }
            }
            if (outer_wall && (slot == 0 || slot == 1 || slot == 2 || slot == 7 || slot == 8))
                acc[DV_NV] = fmaf(Js[(int64_t)(DV_NV * DV_NB + DV_NV) * nc], x, acc[DV_NV]);
        }
    }
#pragma unroll
    for (int rv = 0; rv < DV_NV; ++rv) {
        const int64_t q = (int64_t)rv * nc + c;
        out[q] = (u[q] * sc[q] - dhv * (double)acc[rv]) / sc[q];
    }
    if (outer_wall) {
        const int64_t q = offw + (int64_t)j * Nz + k;
        out[q] = (u[q] * sc[q] - dhv * (double)acc[DV_NV]) / sc[q];
    }
}

int launch_spmv32(dv_model* m, const double* u, const double* sc, double dh, const double* dh_dev, double* out,
                  cudaStream_t s, bool count) {
    const dv_step_params& p = m->p;
    const int bl = (m->tune.spmv_block == 64 || m->tune.spmv_block == 256) ? m->tune.spmv_block : 128;
    const unsigned grid = (unsigned)((m->nc + bl - 1) / bl);
    if (count) {
        DV_LAUNCH(dv::K_SPMV, s, k_spmv32<<<grid, bl, 0, s>>>(p.Nr, p.Nth, p.Nz, p.wall_on, m->d_J32, u, sc, dh, dh_dev, out));
    } else {
        k_spmv32<<<grid, bl, 0, s>>>(p.Nr, p.Nth, p.Nz, p.wall_on, m->d_J32, u, sc, dh, dh_dev, out);
    }
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

}  // namespace dv
