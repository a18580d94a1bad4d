// dv_solver.cu -- Newton-Krylov stage solve, adaptive 2-stage implicit RK integrator, C ABI.
//
// Control flow mirrors the reference exactly (core/solver.py); the arithmetic runs on the GPU
// (dv_kernels.cu, dv_linalg.cu and the vector kernels below) and the host reads back a few
// scalars per Krylov iteration to take the same branch decisions.
#include <atomic>
#include <map>
#include <mutex>
#include <unordered_map>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#include "dv_internal.h"
#include "dv_mlp.h"

#include <utility>
#include "dv_physics.cuh"

namespace dv {

static thread_local std::string g_err;

// ---------------------------------------------------------------- buffer pool
namespace {
struct PoolKey {
    int dev;          // -1: pinned host memory
    size_t bytes;
    bool operator<(const PoolKey& o) const { return dev != o.dev ? dev < o.dev : bytes < o.bytes; }
};
std::mutex g_pool_mu;
std::map<PoolKey, std::vector<void*>> g_pool_free;
std::unordered_map<void*, PoolKey> g_pool_live;
int64_t g_pool_cached = 0;

cudaError_t pool_get(void** p, size_t bytes, bool host) {
    *p = nullptr;
    int dev = -1;
    if (!host) {
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
    }
    const PoolKey k{dev, bytes};
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto it = g_pool_free.find(k);
        if (it != g_pool_free.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            g_pool_cached -= (int64_t)bytes;
            g_pool_live[*p] = k;
            return cudaSuccess;
        }
    }
    cudaError_t e = host ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool_live[*p] = k;
    return cudaSuccess;
}

void pool_put(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pool_live.find(p);
    if (it == g_pool_live.end()) return;       // not pool memory: never happens for handle buffers
    g_pool_free[it->second].push_back(p);
    g_pool_cached += (int64_t)it->second.bytes;
    g_pool_live.erase(it);
}
}  // namespace

cudaError_t pool_malloc(void** p, size_t bytes) { return pool_get(p, bytes, false); }
cudaError_t pool_malloc_host(void** p, size_t bytes) { return pool_get(p, bytes, true); }
void pool_free(void* p) { pool_put(p); }
void pool_free_host(void* p) { pool_put(p); }

bool pdl_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_PDL");
        v = (e && e[0] == '1') ? 1 : 0;
    }
    return v == 1;
}

std::recursive_mutex& capture_mutex() {
    static std::recursive_mutex mu;
    return mu;
}

cudaError_t allow_dyn_smem(const void* func) {
    static std::mutex mu;
    static std::vector<std::pair<int, const void*>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (const auto& d : done)
        if (d.first == dev && d.second == func) return cudaSuccess;
    int optin = 0;
    cudaFuncAttributes fa;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess ||
        (e = cudaFuncGetAttributes(&fa, func)) != cudaSuccess)
        return e;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e == cudaSuccess) done.emplace_back(dev, func);
    return e;
}
void set_error(const std::string& m) { g_err = m; }

// ---------------------------------------------------------------- launch accounting / profiler
struct ProfSlot {
    int64_t launches = 0, timed = 0;
    double ms = 0.0;
};
static ProfSlot g_prof[K_NKIND];
static std::atomic<int64_t> g_launches{0};   // launches of every thread (models run concurrently)
static bool g_prof_on = false;
struct Pending {
    int kind;
    cudaEvent_t a, b;
};
static std::vector<Pending> g_pending;
static std::vector<cudaEvent_t> g_free_ev;
static cudaEvent_t g_open_ev = nullptr;

static cudaEvent_t ev_get() {
    if (!g_free_ev.empty()) {
        cudaEvent_t e = g_free_ev.back();
        g_free_ev.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(int kind, cudaStream_t s) {
    ++g_launches;
    ++g_prof[kind].launches;
    if (!g_prof_on) return;
    g_open_ev = ev_get();
    cudaEventRecord(g_open_ev, s);
}

void count_launch(int kind) {
    ++g_launches;
    ++g_prof[kind].launches;
}

void count_launches(int kind, int64_t n) {
    g_launches += n;
    g_prof[kind].launches += n;
}

void prof_end(int kind, cudaStream_t s) {
    if (!g_prof_on || !g_open_ev) return;
    cudaEvent_t b = ev_get();
    cudaEventRecord(b, s);
    g_pending.push_back({kind, g_open_ev, b});
    g_open_ev = nullptr;
    if (g_pending.size() > 8192) {      // bound the pool: wait for the oldest and fold them in
        cudaEventSynchronize(g_pending.back().b);
        prof_flush();
    }
}

void prof_flush() {
    size_t keep = 0;
    for (size_t q = 0; q < g_pending.size(); ++q) {
        Pending& p = g_pending[q];
        if (cudaEventQuery(p.b) == cudaSuccess) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.a, p.b);
            g_prof[p.kind].ms += ms;
            g_prof[p.kind].timed += 1;
            g_free_ev.push_back(p.a);
            g_free_ev.push_back(p.b);
        } else {
            g_pending[keep++] = p;
        }
    }
    g_pending.resize(keep);
    cudaGetLastError();
}
int cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string("CUDA error ") + cudaGetErrorString(e) + " in " + what;
    return DV_ERR_CUDA;
}

// ---------------------------------------------------------------- vector kernels
#define VB 256
static unsigned vgrid(int64_t n) {
    int64_t b = (n + VB - 1) / VB;
    return (unsigned)(b < 1024 ? (b < 1 ? 1 : b) : 1024);
}

__global__ void k_scale(int64_t nc, int64_t n, const double* __restrict__ z, const double* __restrict__ atol7,
                        double rtol, double* __restrict__ s) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int v = (int)(i / nc);
        if (v > DV_NV) v = DV_NV;
        s[i] = atol7[v] + rtol * fabs(z[i]);
    }
}

// out = a*x + b*y   (y may be null)
__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = y ? a * x[i] + b * y[i] : a * x[i];
}

// out = x + a*y  (numpy  x + a * y)
__global__ void k_xpay(int64_t n, const double* __restrict__ x, double a, const double* __restrict__ y,
                       double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = x[i] + a * y[i];
}

// out = num / den (den may be null), with an optional sign: out = sgn * num / den
__global__ void k_div(int64_t n, double sgn, const double* __restrict__ num, const double* __restrict__ den,
                      double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (sgn < 0 ? -num[i] : num[i]) / den[i];
}

__global__ void k_mul(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

// positivity truncation of gas concentrations and loadings (core/solver.py:99-108): i < npos
__global__ void k_truncate(int64_t n, int64_t npos, const double* __restrict__ z, double lam, const double* __restrict__ dz,
                           double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = z[i] + lam * dz[i];
        if (i < npos) v = npmax(v, 0.1 * npmax(z[i], 0.0));
        out[i] = v;
    }
}

// truncation of a prediction: out = max(x, 0.1 max(y, 0)) on i < npos, else x
__global__ void k_truncate_to(int64_t n, int64_t npos, const double* __restrict__ x, const double* __restrict__ y,
                              double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = x[i];
        if (i < npos) v = npmax(v, 0.1 * npmax(y[i], 0.0));
        out[i] = v;
    }
}

// partial sums of (a/b)^2 (b null: a^2); non-finite terms propagate
__global__ void k_sumsq(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double sh[VB];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = b ? a[i] / b[i] : a[i];
        acc += v * v;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = VB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// k_sumsq then k_finish in one launch: the block that finishes last (ticket) sums the partials
// with k_finish's own strided loop and tree, so the result is the same to the bit
__global__ void k_sumsq_finish(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ part, unsigned* ticket, int mode, double* __restrict__ out) {
    __shared__ double sh[VB];
    __shared__ bool last;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = b ? a[i] / b[i] : a[i];
        acc += v * v;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = VB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sh[0];
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    acc = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) acc += ((volatile const double*)part)[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = VB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double v = sh[0];
        if (mode == 0) v = sqrt(v / (double)n);
        else if (mode == 1) v = fmax(1.0, sqrt(v / (double)n));
        else if (mode == 2) v = sqrt(v);
        out[0] = v;
        *ticket = 0u;
    }
}

// out[slot] = mode 0: sqrt(sum/n); 1: max(1, sqrt(sum/n)); 2: sqrt(sum) ; 3: sum
__global__ void k_finish(int nparts, const double* __restrict__ part, double n, int mode, double* __restrict__ out) {
    __shared__ double sh[VB];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = VB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double v = sh[0];
        if (mode == 0) v = sqrt(v / n);
        else if (mode == 1) v = fmax(1.0, sqrt(v / n));
        else if (mode == 2) v = sqrt(v);
        out[0] = v;
    }
}

// partial dots: part[blk][q] = sum_i V[q][i] w[i] (q < m), part[blk][m] = sum w^2
__global__ void k_dots(int64_t n, int m, const double* __restrict__ V, int64_t ldv, const double* __restrict__ w,
                       double* __restrict__ part) {
    __shared__ double sh[VB];
    for (int q = 0; q <= m; ++q) {
        const double* a = (q < m) ? V + q * ldv : w;
        double acc = 0.0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            acc += a[i] * w[i];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s = VB / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(int64_t)blockIdx.x * (m + 1) + q] = sh[0];
        __syncthreads();
    }
}

__global__ void k_dots_finish(int nblk, int m1, const double* __restrict__ part, double* __restrict__ out) {
    int q = blockIdx.x;
    __shared__ double sh[VB];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc += part[(int64_t)b * m1 + q];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = VB / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sh[0];
}

// w -= sum_q h[q] V[q]
__global__ void k_orth_update(int64_t n, int m, const double* __restrict__ V, int64_t ldv, const double* __restrict__ h,
                              double* __restrict__ w) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < m; ++q) acc += h[q] * V[q * ldv + i];
        w[i] -= acc;
    }
}

// x = sum_q y[q] V[q]  (y from host, passed by value through a small device buffer)
__global__ void k_combine(int64_t n, int m, const double* __restrict__ V, int64_t ldv, const double* __restrict__ y,
                          double* __restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < m; ++q) acc += y[q] * V[q * ldv + i];
        x[i] = acc;
    }
}

// conservation sums: out[0..3] = W R (species moles + energy), out[4..7] = W s (core/residual.py:146-168).
// Grid-stride over cells; each block sums its eight values, the last block to finish adds the
// block sums in block order (deterministic) and resets the ticket.
__global__ void __launch_bounds__(VB) k_cons(dv_step_params p, const double* __restrict__ R,
                                             const double* __restrict__ s, double* __restrict__ part,
                                             unsigned* ticket, double* __restrict__ out) {
    __shared__ double sh[VB / 32][8];
    __shared__ bool last;
    const int64_t nc = (int64_t)p.Nr * p.Nth * p.Nz, nw = p.wall_on ? (int64_t)p.Nth * p.Nz : 0;
    const int64_t ncz = (int64_t)p.Nth * p.Nz;
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const double V = p.V[(int)(c / ncz)];
#pragma unroll
        for (int which = 0; which < 2; ++which) {
            const double* x = which ? s : R;
#pragma unroll
            for (int m = 0; m < DV_NG; ++m) {
                double v = p.eps_t * V * x[m * nc + c];
                if (m < DV_NA) v += p.rho_b * V * x[(DV_NG + m) * nc + c];
                acc[which * 4 + m] += v;
            }
            acc[which * 4 + DV_NG] += V * x[(int64_t)(DV_NG + DV_NA) * nc + c];      // e block
        }
    }
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
        acc[DV_NG] += p.wall_C * R[(int64_t)DV_NV * nc + w];
        acc[4 + DV_NG] += p.wall_C * s[(int64_t)DV_NV * nc + w];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        double v = acc[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) sh[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double t = 0.0;
        for (int w2 = 0; w2 < VB / 32; ++w2) t += sh[w2][threadIdx.x];
        part[(int64_t)blockIdx.x * 8 + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last && threadIdx.x < 8) {
        __threadfence();
        out[threadIdx.x] = sum_partials(part + threadIdx.x, (int)gridDim.x, 8);
    }
    if (last && threadIdx.x == 0) *ticket = 0u;
}

// Balance projection (no reference counterpart).  The conserved quantity an unknown belongs to
// (rows of W): species k for c_k and, for k < DV_NA, the loading q_k; 3 for e and the wall.
__device__ __forceinline__ int cons_quantity(int64_t i, int64_t nc) {
    const int64_t blk = i / nc;
    return blk < DV_NG ? (int)blk : (blk < DV_NG + DV_NA ? (int)(blk - DV_NG) : DV_NG);
}

// Basis direction b_q of the projection, in scaled variables (u = b / s): a relative change of the
// species' concentrations and loadings (b = z, keeps them positive), an additive change of one error
// scale for the energy and wall unknowns (b = s); 0 outside quantity q.
__global__ void k_cons_basis(int64_t nc, int64_t n, int q, const double* __restrict__ z, const double* __restrict__ s,
                             double* __restrict__ u) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int w = cons_quantity(i, nc);
    u[i] = (w != q) ? 0.0 : (q < DV_NG ? z[i] / s[i] : 1.0);
}

// z += sum_q lam_q b_q
__global__ void k_cons_shift(int64_t nc, int64_t n, double l0, double l1, double l2, double l3,
                             const double* __restrict__ s, double* __restrict__ z) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int w = cons_quantity(i, nc);
    const double l = w == 0 ? l0 : (w == 1 ? l1 : (w == 2 ? l2 : l3));
    z[i] = (w < DV_NG) ? z[i] * (1.0 + l) : z[i] + l * s[i];
}

// Solve G lam = rhs (4 x 4, row-major) over the quantities with active[q]; lam = 0 elsewhere.
// Gaussian elimination with partial pivoting; false if the active system is singular.
static bool solve_small(const double* G, const double* rhs, const bool* active, double* lam) {
    int idx[4], k = 0;
    for (int q = 0; q < 4; ++q) {
        lam[q] = 0.0;
        if (active[q]) idx[k++] = q;
    }
    double A[4][5];
    for (int a = 0; a < k; ++a) {
        for (int b = 0; b < k; ++b) A[a][b] = G[idx[a] * 4 + idx[b]];
        A[a][k] = rhs[idx[a]];
    }
    for (int c = 0; c < k; ++c) {
        int piv = c;
        for (int a = c + 1; a < k; ++a)
            if (std::fabs(A[a][c]) > std::fabs(A[piv][c])) piv = a;
        if (!(std::fabs(A[piv][c]) > 0.0)) return false;
        if (piv != c)
            for (int b = 0; b <= k; ++b) std::swap(A[c][b], A[piv][b]);
        for (int a = c + 1; a < k; ++a) {
            const double f = A[a][c] / A[c][c];
            for (int b = c; b <= k; ++b) A[a][b] -= f * A[c][b];
        }
    }
    for (int c = k - 1; c >= 0; --c) {
        double v = A[c][k];
        for (int b = c + 1; b < k; ++b) v -= A[c][b] * lam[idx[b]];
        lam[idx[c]] = v / A[c][c];
        if (!std::isfinite(lam[idx[c]])) return false;
    }
    return true;
}

static unsigned cons_grid(int64_t nc) {
    const int64_t b = (nc + VB - 1) / VB;
    return (unsigned)(b < 1 ? 1 : (b > 64 ? 64 : b));
}

// err scale: sc = atol + rtol max(|y|, |z|)  (core/solver.py:461)
__global__ void k_err_scale(int64_t nc, int64_t n, const double* __restrict__ y, const double* __restrict__ z,
                            const double* __restrict__ atol7, double rtol, double* __restrict__ sc) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int v = (int)(i / nc);
        if (v > DV_NV) v = DV_NV;
        sc[i] = atol7[v] + rtol * npmax(fabs(y[i]), fabs(z[i]));
    }
}

// y3 = y + h (w1 f_n + w2 f1 + w3 f2);  out = z2 - y3   (core/solver.py:456-460)
__global__ void k_err_vec(int64_t n, const double* __restrict__ y, const double* __restrict__ z2, double h, double w1,
                          const double* __restrict__ fn, double w2, const double* __restrict__ f1, double w3,
                          const double* __restrict__ f2, double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double y3 = y[i] + h * (w1 * fn[i] + w2 * f1[i] + w3 * f2[i]);
        out[i] = z2[i] - y3;
    }
}

// ---------------------------------------------------------------- device GMRES state
// Everything scipy's gmres loop keeps between Arnoldi steps, on the device, so a CUDA graph can run
// the loop without the host (see gmres_graph).  The first four doubles are written by the host
// before each launch; the matvec kernels read t and dh from them.
constexpr int GM_KMAX = 30;
struct GmDev {
    double t, dh, rtol, atol;
    double bn2, atol_eff, ptol, presid, scale, rnorm;
    int col, done, skip, iters, info, ncomb, pad0, pad1;
    double H[GM_KMAX * (GM_KMAX + 1)], S[GM_KMAX + 1], gc[GM_KMAX], gs[GM_KMAX], y[GM_KMAX + 1];
};
static size_t gm_state_bytes() { return sizeof(GmDev); }

// ---------------------------------------------------------------- workspace
// Test aid: with DVTSA_FILL=<byte>[,<mask>] in the environment, newly allocated workspaces are
// filled with that byte (mask bits: 1 model, 2 Krylov workspace, 4 integrator, 8 pinned host
// buffers; default all).  A result that changes with the byte reads memory nothing wrote.
static void debug_fill(void* p, size_t bytes, int group, bool host = false) {
    const char* e = getenv("DVTSA_FILL");
    if (!e || !p) return;
    int byte = 0, mask = 15;
    if (sscanf(e, "%i,%i", &byte, &mask) < 1) return;
    if (!(mask & group)) return;
    if (host) memset(p, byte & 0xff, bytes);
    else cudaMemset(p, byte & 0xff, bytes);
}

int work_alloc(Work& W, int64_t n, int kdim, int64_t jac_doubles) {
    W.n = n;
    W.kdim = kdim;
    W.nparts = 1024;
    auto A = [&](double** p, int64_t cnt) { return pool_malloc((void**)p, sizeof(double) * (size_t)cnt); };
    if (A(&W.V, (kdim + 1) * n) || A(&W.w, n) || A(&W.u, n) || A(&W.x, n) || A(&W.r, n) || A(&W.b, n) ||
        A(&W.s, n) || A(&W.z, n) || A(&W.f, n) || A(&W.R, n) || A(&W.dz, n) || A(&W.zt, n) || A(&W.ft, n) ||
        A(&W.Rt, n) || A(&W.tmp, n) || A(&W.best, n) || A(&W.part, (int64_t)W.nparts * (kdim + 2)) ||
        A(&W.scal, 32) || A(&W.hbuf, 4 * (kdim + 2)) || A(&W.ybuf, kdim + 2) || A(&W.J, jac_doubles) ||
        A(&W.vin, n) || A(&W.wout, n) || A(&W.apart, 4096) || pool_malloc(&W.gm, gm_state_bytes()) != cudaSuccess ||
        pool_malloc((void**)&W.tickets, 16 * sizeof(unsigned)) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "cudaMalloc(Krylov workspace)");
    if (pool_malloc_host(&W.gm_host, 256) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaMallocHost");
    if (pool_malloc_host((void**)&W.hpin, sizeof(double) * 4 * (kdim + 8)) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "cudaMallocHost");
    {
        const size_t d = sizeof(double);
        std::pair<double*, int64_t> bufs[] = {{W.V, (kdim + 1) * n}, {W.w, n}, {W.u, n}, {W.x, n}, {W.r, n}, {W.b, n},
                                              {W.s, n}, {W.z, n}, {W.f, n}, {W.R, n}, {W.dz, n}, {W.zt, n}, {W.ft, n},
                                              {W.Rt, n}, {W.tmp, n}, {W.best, n},
                                              {W.part, (int64_t)W.nparts * (kdim + 2)}, {W.scal, 32},
                                              {W.hbuf, 4 * (kdim + 2)}, {W.ybuf, kdim + 2}, {W.J, jac_doubles},
                                              {W.vin, n}, {W.wout, n}};
        for (auto& b : bufs) debug_fill(b.first, d * (size_t)b.second, 2);
        debug_fill(W.gm, gm_state_bytes(), 2);
        debug_fill(W.gm_host, 256, 8, true);
        debug_fill(W.hpin, d * 4 * (kdim + 8), 8, true);
        debug_fill(W.apart, d * 4096, 2);
    }
    if (cudaMemset(W.tickets, 0, 16 * sizeof(unsigned)) != cudaSuccess)   // ticket counters start at zero
        return cuda_fail(cudaGetLastError(), "cudaMemset(tickets)");
    return DV_OK;
}

void work_free(Work& W) {
    if (W.gm_exec) cudaGraphExecDestroy(W.gm_exec);
    if (W.gm_graph) cudaGraphDestroy(W.gm_graph);
    if (W.gm_cs) cudaStreamDestroy(W.gm_cs);
    double* ptrs[] = {W.V, W.w, W.u, W.x, W.r, W.b, W.s, W.z, W.f, W.R, W.dz, W.zt, W.ft, W.Rt, W.tmp, W.best,
                      W.part, W.scal, W.hbuf, W.ybuf, W.J, W.vin, W.wout, W.apart};
    for (double* p : ptrs) pool_free(p);
    pool_free(W.gm);
    pool_free(W.tickets);
    pool_free_host(W.hpin);
    pool_free_host(W.gm_host);
    W = Work();
}

// reductions returning host values (synchronise)
static int rms_ratio_dev(Work& W, int64_t n, const double* a, const double* b, int mode, double* dst, cudaStream_t s) {
    unsigned g = vgrid(n);
    DV_LAUNCH(dv::K_VECTOR, s, k_sumsq_finish<<<g, VB, 0, s>>>(n, a, b, W.part, W.tickets + 6, mode, dst));
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

static int fetch(Work& W, const double* dev, int cnt, double* host, cudaStream_t s) {
    DV_CUDA(cudaMemcpyAsync(W.hpin, dev, sizeof(double) * cnt, cudaMemcpyDeviceToHost, s));
    DV_CUDA(cudaStreamSynchronize(s));
    memcpy(host, W.hpin, sizeof(double) * cnt);
    if (g_prof_on && !g_pending.empty()) prof_flush();
    return DV_OK;
}

static int rms_ratio(Work& W, int64_t n, const double* a, const double* b, double* out, cudaStream_t s) {
    int rc = rms_ratio_dev(W, n, a, b, 0, W.scal + 8, s);
    if (rc) return rc;
    return fetch(W, W.scal + 8, 1, out, s);
}




// LAPACK dlartg (3.10+): c, s, r with [c s; -s c] [f; g] = [r; 0]
static void lartg(double f, double g, double& c, double& s, double& r) {
    const double safmin = std::numeric_limits<double>::min();
    const double safmax = 1.0 / safmin;
    const double rtmin = std::sqrt(safmin), rtmax = std::sqrt(safmax / 2);
    double f1 = std::fabs(f), g1 = std::fabs(g);
    if (g == 0.0) {
        c = 1.0; s = 0.0; r = f;
    } else if (f == 0.0) {
        c = 0.0; s = std::copysign(1.0, g); r = g1;
    } else if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        double d = std::sqrt(f * f + g * g);
        c = f1 / d;
        r = std::copysign(d, f);
        s = g / r;
    } else {
        double u = std::min(safmax, std::max(safmin, std::max(f1, g1)));
        double fs = f / u, gs = g / u;
        double d = std::sqrt(fs * fs + gs * gs);
        c = std::fabs(fs) / d;
        r = std::copysign(d, f);
        s = gs / r;
        r *= u;
    }
}

// Operator of the Newton linear system in scaled variables, right-preconditioned:
// AP(w) = matvec(prec(w)), prec(r) = M^-1 (r s) / s, matvec(u) = (v - dh (f(z + sig v) - f)/sig)/s.
struct Op {
    dv_model* m;
    double t, dh;
    const double* z;
    const double* f;
    const double* s;
    int64_t n;
};

static int apply_AP(Work& W, const Op& op, const double* w, double* out, cudaStream_t st) {
    DV_TRY(precond_apply(op.m, w, op.s, W.u, st));                      // u = prec(w)
    DV_TRY(rms_ratio_dev(W, op.n, W.u, nullptr, 0, W.scal + 0, st));   // scal[0] = rms(u)
    if (op.m->op32) return launch_spmv32(op.m, W.u, op.s, op.dh, nullptr, out, st);
    DV_TRY(launch_matvec(op.m, op.t, op.z, W.u, op.s, op.f, op.dh, W.scal, out, st));
    return DV_OK;
}

// out = b - A u for a correction u in scaled variables (the GMRES operator without the preconditioner)
static int op_residual(Work& W, const Op& op, const double* b, const double* u, double* out, cudaStream_t st) {
    DV_TRY(rms_ratio_dev(W, op.n, u, nullptr, 0, W.scal + 0, st));     // scal[0] = rms(u): the FD step
    if (op.m->op32) DV_TRY(launch_spmv32(op.m, u, op.s, op.dh, nullptr, out, st));
    else DV_TRY(launch_matvec(op.m, op.t, op.z, u, op.s, op.f, op.dh, W.scal, out, st));
    DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<vgrid(op.n), VB, 0, st>>>(op.n, 1.0, b, -1.0, out, out));
    return DV_OK;
}

// scipy.sparse.linalg.gmres(AP, b, rtol, atol, restart=kdim, maxiter=1) with M = identity
// (scipy/sparse/linalg/_isolve/iterative.py); x written to W.x.  Returns info (0 = converged).
static int gmres(Work& W, const Op& op, const double* b, double rtol, double atol, int kdim, int* info,
                 int64_t* inner, cudaStream_t st) {
    const int64_t n = op.n;
    double bn2;
    DV_TRY(rms_ratio_dev(W, n, b, nullptr, 2, W.scal + 9, st));
    DV_TRY(fetch(W, W.scal + 9, 1, &bn2, st));
    const double atol_eff = std::max(atol, rtol * bn2);
    *info = 0;
    if (bn2 == 0.0 || bn2 < atol_eff) {       // ||r0|| < atol with x0 = 0: x = 0, u = prec(x) = 0, r = b
        DV_CUDA(cudaMemsetAsync(W.x, 0, sizeof(double) * n, st));
        DV_CUDA(cudaMemsetAsync(W.u, 0, sizeof(double) * n, st));
        if (b != W.r) DV_CUDA(cudaMemcpyAsync(W.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        return DV_OK;
    }
    double ptol = bn2 * std::min(1.0, atol_eff / bn2);
    const double eps = std::numeric_limits<double>::epsilon();
    const int64_t ldv = n;
    DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<vgrid(n), VB, 0, st>>>(n, 1.0 / bn2, b, 0.0, nullptr, W.V));      // v0 = r / ||r||
    std::vector<double> H((size_t)kdim * (kdim + 1), 0.0), S(kdim + 1, 0.0), gc(kdim), gs(kdim);
    auto h = [&](int col, int k) -> double& { return H[(size_t)col * (kdim + 1) + k]; };
    S[0] = bn2;
    bool breakdown = false;
    int col = 0;
    double presid = 0.0;
    const unsigned g = vgrid(n);
    for (col = 0; col < kdim; ++col) {
        double* w = W.V + (col + 1) * ldv;
        DV_TRY(apply_AP(W, op, W.V + col * ldv, w, st));
        // classical Gram-Schmidt, twice (orthogonality equivalent to scipy's modified GS)
        const int m = col + 1;
        DV_LAUNCH(dv::K_VECTOR, st, k_dots<<<g, VB, 0, st>>>(n, m, W.V, ldv, w, W.part));
        DV_LAUNCH(dv::K_VECTOR, st, k_dots_finish<<<m + 1, VB, 0, st>>>((int)g, m + 1, W.part, W.hbuf));
        DV_LAUNCH(dv::K_VECTOR, st, k_orth_update<<<g, VB, 0, st>>>(n, m, W.V, ldv, W.hbuf, w));
        DV_LAUNCH(dv::K_VECTOR, st, k_dots<<<g, VB, 0, st>>>(n, m, W.V, ldv, w, W.part));
        DV_LAUNCH(dv::K_VECTOR, st, k_dots_finish<<<m + 1, VB, 0, st>>>((int)g, m + 1, W.part, W.hbuf + (kdim + 2)));
        DV_LAUNCH(dv::K_VECTOR, st, k_orth_update<<<g, VB, 0, st>>>(n, m, W.V, ldv, W.hbuf + (kdim + 2), w));
        DV_TRY(rms_ratio_dev(W, n, w, nullptr, 2, W.hbuf + 2 * (kdim + 2), st));
        DV_CUDA(cudaGetLastError());
        std::vector<double> hh(2 * (kdim + 2) + 1);
        DV_CUDA(cudaMemcpyAsync(W.hpin, W.hbuf, sizeof(double) * (2 * (kdim + 2) + 1), cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
        memcpy(hh.data(), W.hpin, sizeof(double) * hh.size());
        const double h0 = std::sqrt(hh[m]);          // ||w|| before orthogonalisation
        for (int k = 0; k <= col; ++k) h(col, k) = hh[k] + hh[(kdim + 2) + k];
        const double h1 = hh[2 * (kdim + 2)];
        h(col, col + 1) = h1;
        if (h1 <= eps * h0 || !(h1 == h1)) {
            h(col, col + 1) = 0.0;
            breakdown = true;
        } else {
            DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0 / h1, w, 0.0, nullptr, w));
        }
        for (int k = 0; k < col; ++k) {
            double c = gc[k], s = gs[k];
            double n0 = h(col, k), n1 = h(col, k + 1);
            h(col, k) = c * n0 + s * n1;
            h(col, k + 1) = -s * n0 + c * n1;
        }
        double c, s, mag;
        lartg(h(col, col), h(col, col + 1), c, s, mag);
        gc[col] = c;
        gs[col] = s;
        h(col, col) = mag;
        h(col, col + 1) = 0.0;
        double tmp = -s * S[col];
        S[col] = c * S[col];
        S[col + 1] = tmp;
        presid = std::fabs(tmp);
        *inner += 1;
        if (!(presid == presid)) break;
        if (presid <= ptol || breakdown) break;
    }
    if (col == kdim) col = kdim - 1;
    if (h(col, col) == 0.0) S[col] = 0.0;
    std::vector<double> y(col + 1);
    for (int k = 0; k <= col; ++k) y[k] = S[k];
    for (int k = col; k > 0; --k) {
        if (y[k] != 0.0) {
            y[k] /= h(k, k);
            double tmp = y[k];
            for (int q = 0; q < k; ++q) y[q] -= tmp * h(k, q);
        }
    }
    if (y[0] != 0.0) y[0] /= h(0, 0);
    memcpy(W.hpin, y.data(), sizeof(double) * (col + 1));
    DV_CUDA(cudaMemcpyAsync(W.ybuf, W.hpin, sizeof(double) * (col + 1), cudaMemcpyHostToDevice, st));
    DV_LAUNCH(dv::K_VECTOR, st, k_combine<<<g, VB, 0, st>>>(n, col + 1, W.V, ldv, W.ybuf, W.x));
    // true residual r = b - AP x
    DV_TRY(apply_AP(W, op, W.x, W.r, st));
    DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, b, -1.0, W.r, W.r));
    double rnorm;
    DV_TRY(rms_ratio_dev(W, n, W.r, nullptr, 2, W.scal + 10, st));
    DV_TRY(fetch(W, W.scal + 10, 1, &rnorm, st));
    *info = (rnorm <= atol_eff) ? 0 : 1;
    return DV_OK;
}


static int check_device_error(dv_model* m);
static void clear_device_error(dv_model* m);

// the model's device error word: bit 1 a preconditioner sweep's bulk-copy wait timed out, bit 4 a
// grid barrier of a cooperative kernel (Gram-Schmidt, the FD matvec) timed out
static const char* device_error_text(int e) {
    if (e & 32) return "a preconditioner index fell outside its storage (the access was skipped)";
    if (e & 1) return "a bounded device wait (preconditioner bulk copy) timed out";
    if (e & 4) return "a bounded device wait (GMRES grid barrier) timed out";
    return "a bounded device wait timed out";
}

// ---------------------------------------------------------------- device-driven GMRES
// The loop of gmres() above as a CUDA graph: the pre-loop kernels, a conditional WHILE node whose
// body is one Arnoldi step (normalise the previous basis vector, precondition, FD matvec, two
// classical Gram-Schmidt passes, Givens update and the stopping test on the device), and the
// post-loop least-squares solve, combination and true-residual check.  Same kernels and the same
// arithmetic in the same order as gmres(), so the same bits, without a host round trip per step.

__device__ __forceinline__ double std_max_d(double a, double b) { return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double std_min_d(double a, double b) { return (b < a) ? b : a; }   // std::min

// LAPACK dlartg (3.10+), as lartg() above
__device__ void lartg_d(double f, double g, double& c, double& s, double& r) {
    const double safmin = 2.2250738585072014e-308;          // smallest normal double
    const double safmax = 1.0 / safmin;
    const double rtmin = sqrt(safmin), rtmax = sqrt(safmax / 2);
    double f1 = fabs(f), g1 = fabs(g);
    if (g == 0.0) {
        c = 1.0; s = 0.0; r = f;
    } else if (f == 0.0) {
        c = 0.0; s = copysign(1.0, g); r = g1;
    } else if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        double d = sqrt(f * f + g * g);
        c = f1 / d;
        r = copysign(d, f);
        s = g / r;
    } else {
        double u = std_min_d(safmax, std_max_d(safmin, std_max_d(f1, g1)));
        double fs = f / u, gs = g / u;
        double d = sqrt(fs * fs + gs * gs);
        c = fabs(fs) / d;
        r = copysign(d, f);
        s = gs / r;
        r *= u;
    }
}

__global__ void k_gm_init(GmDev* st, const double* __restrict__ scal, int kdim, cudaGraphConditionalHandle hnd,
                          unsigned* bar) {
    if (threadIdx.x == 0 && bar) {              // barrier words of k_cgs_fused: no arrivals pending
        bar[0] = 0u;
        bar[2] = 0u;
    }
    for (int q = threadIdx.x; q < kdim * (kdim + 1); q += blockDim.x) st->H[q] = 0.0;
    for (int q = threadIdx.x; q <= kdim; q += blockDim.x) st->S[q] = 0.0;
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double bn2 = scal[9];
    const double atol_eff = std_max_d(st->atol, st->rtol * bn2);
    bool skip = (bn2 == 0.0);
    double ptol = 0.0;
    if (!skip) {
        ptol = bn2 * std_min_d(1.0, atol_eff / bn2);
        if (bn2 < atol_eff) skip = true;
    }
    st->bn2 = bn2;
    st->atol_eff = atol_eff;
    st->ptol = ptol;
    st->info = 0;
    st->skip = skip;
    st->done = skip;
    st->col = 0;
    st->iters = 0;
    st->ncomb = 0;
    st->presid = 0.0;
    st->scale = skip ? 0.0 : 1.0 / bn2;      // v0 = r / ||r||
    st->S[0] = bn2;
    cudaGraphSetConditional(hnd, skip ? 0u : 1u);
}

// V[col] = src * scale (src = b for the first vector, else the orthogonalised operator output) and
// its copy vin, the preconditioner's input
__global__ void k_gm_norm(int64_t n, const GmDev* __restrict__ st, const double* __restrict__ b,
                          const double* __restrict__ wout, double* __restrict__ V, int64_t ldv,
                          double* __restrict__ vin) {
    const int col = st->col;
    const double sc = st->scale;
    const double* src = (col == 0) ? b : wout;
    double* v = V + (int64_t)col * ldv;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = sc * src[i];
        v[i] = x;
        vin[i] = x;
    }
}

__global__ void k_dots_gm(int64_t n, const GmDev* __restrict__ st, const double* __restrict__ V, int64_t ldv,
                          const double* __restrict__ w, double* __restrict__ part) {
    __shared__ double sh[VB];
    const int m = st->col + 1;
    for (int q = 0; q <= m; ++q) {
        const double* a = (q < m) ? V + q * ldv : w;
        double acc = 0.0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            acc += a[i] * w[i];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s2 = VB / 2; s2 > 0; s2 >>= 1) {
            if (threadIdx.x < s2) sh[threadIdx.x] += sh[threadIdx.x + s2];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(int64_t)blockIdx.x * (m + 1) + q] = sh[0];
        __syncthreads();
    }
}

__global__ void k_dots_finish_gm(int nblk, const GmDev* __restrict__ st, const double* __restrict__ part,
                                 double* __restrict__ out) {
    const int m1 = st->col + 2;
    const int q = blockIdx.x;
    if (q >= m1) return;
    __shared__ double sh[VB];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc += part[(int64_t)b * m1 + q];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = VB / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) sh[threadIdx.x] += sh[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sh[0];
}

__global__ void k_orth_update_gm(int64_t n, const GmDev* __restrict__ st, const double* __restrict__ V, int64_t ldv,
                                 const double* __restrict__ h, double* __restrict__ w) {
    const int m = st->col + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < m; ++q) acc += h[q] * V[q * ldv + i];
        w[i] -= acc;
    }
}

// Hessenberg column, Givens rotations, residual estimate and the stopping test of gmres().  One
// thread.  The rotated entry k + 1 of the new column is carried to the next rotation in a register
// and the loads (hh, the stored rotations) go through restrict pointers, so they run ahead of the
// chain of rotations instead of each waiting behind the previous entry's store.
__device__ void gm_givens(GmDev* st, const double* __restrict__ hh, int kdim, cudaGraphConditionalHandle hnd) {
    const double eps = 2.220446049250313e-16;                 // double epsilon
    const int col = st->col;
    const int m = col + 1;
    double* __restrict__ Hc = st->H + (int64_t)col * (kdim + 1);      // column col of H
    const double* __restrict__ gcs = st->gc;
    const double* __restrict__ gss = st->gs;
    const double h0 = sqrt(hh[m]);
    const double h1 = hh[2 * (kdim + 2)];
    const double S_col = st->S[col], ptol = st->ptol;         // loaded with the column, ahead of their use
    const int iters = st->iters;
    bool breakdown = false;
    if (h1 <= eps * h0 || !(h1 == h1)) breakdown = true;      // the subdiagonal entry is taken as 0
    else st->scale = 1.0 / h1;
    double carry = hh[0] + hh[(kdim + 2)];                     // entry k of the column, rotated by 0..k-1
    for (int k = 0; k < col; ++k) {
        const double c = gcs[k], s2 = gss[k];
        const double n0 = carry, n1 = hh[k + 1] + hh[(kdim + 2) + k + 1];
        Hc[k] = c * n0 + s2 * n1;
        carry = -s2 * n0 + c * n1;
    }
    double c, s2, mag;
    lartg_d(carry, breakdown ? 0.0 : h1, c, s2, mag);
    st->gc[col] = c;
    st->gs[col] = s2;
    Hc[col] = mag;
    Hc[col + 1] = 0.0;
    double tmp = -s2 * S_col;
    st->S[col] = c * S_col;
    st->S[col + 1] = tmp;
    const double presid = fabs(tmp);
    st->presid = presid;
    st->iters = iters + 1;
    const bool stop = !(presid == presid) || presid <= ptol || breakdown || col + 1 == kdim;
    if (!stop) st->col = col + 1;
    st->done = stop;
    cudaGraphSetConditional(hnd, stop ? 0u : 1u);
}

__global__ void k_gm_givens(GmDev* st, const double* __restrict__ hh, int kdim, cudaGraphConditionalHandle hnd) {
    if (threadIdx.x == 0) gm_givens(st, hh, kdim, hnd);
}

// ---- fused classical Gram-Schmidt of the graph body (three kernels per Arnoldi step)
// Warp sums of the first cnt entries of acc into out[q] (lane 0).  Each entry is the same butterfly
// over the 32 lanes; they run eight at a time, side by side (one uniform branch per eight), so the
// sums wait on about five shuffle latencies per eight entries instead of five per entry.
__device__ __forceinline__ void warp_sums(const double (&acc)[GM_KMAX + 1], int cnt, int lane, double* out) {
#pragma unroll
    for (int q0 = 0; q0 <= GM_KMAX; q0 += 8) {
        if (q0 < cnt) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = (q0 + u <= GM_KMAX) ? acc[q0 + u] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] += __shfl_xor_sync(0xffffffffu, v[u], off);
            if (lane == 0)
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (q0 + u < cnt) out[q0 + u] = v[u];
        }
    }
}

// Block sums of the first cnt entries of acc (VB threads) into part[blockIdx.x * GM_PS + q];
// returns true in the block that finished last (after the other blocks' partials are visible).
constexpr int GM_PS = GM_KMAX + 2;      // partial stride per block
constexpr int GM_PREFIX = 4;            // Arnoldi steps of the GMRES graph ahead of its WHILE node
__device__ __forceinline__ bool gm_block_partials(const double (&acc)[GM_KMAX + 1], int cnt, double* part,
                                                  unsigned* ticket) {
    __shared__ double sm[VB / 32][GM_PS];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    warp_sums(acc, cnt, lane, sm[wid]);
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
        double t = 0.0;
        for (int w2 = 0; w2 < VB / 32; ++w2) t += sm[w2][threadIdx.x];
        part[(int64_t)blockIdx.x * GM_PS + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// out[q] = sum over blocks of part[.. q], q < cnt, in block order (called by the last block)
__device__ __forceinline__ void gm_finish_partials(const double* part, int cnt, double* out, unsigned* ticket) {
    if ((int)threadIdx.x < cnt) {
        out[threadIdx.x] = sum_partials(part + threadIdx.x, (int)gridDim.x, GM_PS);
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// pass 1: out[q] = V_q . w (q < m) and out[m] = w . w, m = col + 1
__global__ void __launch_bounds__(VB) k_cgs_dots(int64_t n, const GmDev* __restrict__ st, const double* __restrict__ V,
                                                 int64_t ldv, const double* __restrict__ w, double* __restrict__ part,
                                                 unsigned* ticket, double* __restrict__ out) {
    if (st->done) return;                  // a step after the solve stopped
    const int m = st->col + 1;
    double acc[GM_KMAX + 1];
#pragma unroll
    for (int q = 0; q <= GM_KMAX; ++q) acc[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int q = 0; q <= GM_KMAX; ++q) {
            if (q < m) acc[q] += V[q * ldv + i] * wi;
            else if (q == m) acc[q] += wi * wi;
        }
    }
    if (gm_block_partials(acc, m + 1, part, ticket)) gm_finish_partials(part, m + 1, out, ticket);
}

// w -= sum_q h[q] V_q, then pass 2: out[q] = V_q . w (q < m)
__global__ void __launch_bounds__(VB) k_cgs_orth_dots(int64_t n, const GmDev* __restrict__ st,
                                                      const double* __restrict__ V, int64_t ldv,
                                                      const double* __restrict__ h, double* __restrict__ w,
                                                      double* __restrict__ part, unsigned* ticket,
                                                      double* __restrict__ out) {
    if (st->done) return;                  // a step after the solve stopped
    const int m = st->col + 1;
    double acc[GM_KMAX + 1];
#pragma unroll
    for (int q = 0; q <= GM_KMAX; ++q) acc[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double o = 0.0;
        for (int q = 0; q < m; ++q) o += h[q] * V[q * ldv + i];
        const double wi = w[i] - o;
        w[i] = wi;
#pragma unroll
        for (int q = 0; q < GM_KMAX; ++q)
            if (q < m) acc[q] += V[q * ldv + i] * wi;
    }
    if (gm_block_partials(acc, m, part, ticket)) gm_finish_partials(part, m, out, ticket);
}

// w -= sum_q h2[q] V_q, ||w|| into hh[2 (kdim+2)], then the Givens update and stopping test
__global__ void __launch_bounds__(VB) k_cgs_orth_norm(int64_t n, GmDev* st, const double* __restrict__ V, int64_t ldv,
                                                      double* __restrict__ hh, double* __restrict__ w,
                                                      double* __restrict__ part, unsigned* ticket, int kdim,
                                                      cudaGraphConditionalHandle hnd) {
    if (st->done) return;                  // a step after the solve stopped
    const int m = st->col + 1;
    const double* h2 = hh + (kdim + 2);
    double acc[GM_KMAX + 1];
    acc[0] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double o = 0.0;
        for (int q = 0; q < m; ++q) o += h2[q] * V[q * ldv + i];
        const double wi = w[i] - o;
        w[i] = wi;
        acc[0] += wi * wi;
    }
    if (gm_block_partials(acc, 1, part, ticket)) {
        if (threadIdx.x == 0) {
            hh[2 * (kdim + 2)] = sqrt(sum_partials(part, (int)gridDim.x, GM_PS));
            *ticket = 0u;
            gm_givens(st, hh, kdim, hnd);
        }
    }
}

// ---- CGS2 of one Arnoldi step in a single cooperative launch (grid_sync_bounded: dv_internal.h)

// this block's sums of the first cnt entries of acc into part[blockIdx.x * GM_PS + q]
__device__ __forceinline__ void gm_store_partials(const double (&acc)[GM_KMAX + 1], int cnt, double* part) {
    __shared__ double sm[VB / 32][GM_PS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    warp_sums(acc, cnt, lane, sm[wid]);
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
        double t = 0.0;
        for (int w2 = 0; w2 < VB / 32; ++w2) t += sm[w2][threadIdx.x];
        part[(int64_t)blockIdx.x * GM_PS + threadIdx.x] = t;
    }
}

// The grid's per-block partials of entries q < cnt, copied into this block's shared memory by all
// its threads at once (one round of L2 loads), for a finish that then adds them in block order from
// shared memory: the same additions in the same order as sum_partials, without one L2 round trip
// per block.  Grids of more than CG_MAXB blocks finish with sum_partials.
constexpr int CG_MAXB = 160;
__device__ __forceinline__ void stage_partials(const double* part, int cnt, double (*ps)[GM_PS]) {
    const int nb = (int)gridDim.x;
    for (int i = threadIdx.x; i < nb * cnt; i += blockDim.x) {
        const int b = i / cnt, q = i - b * cnt;
        ps[b][q] = __ldcg(part + (int64_t)b * GM_PS + q);
    }
    __syncthreads();
}
__device__ __forceinline__ double finish_partials(const double* part, int q, double (*ps)[GM_PS]) {
    if (gridDim.x > CG_MAXB) return sum_partials(part + q, (int)gridDim.x, GM_PS);
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += ps[b][q];
    return t;
}

// k_cgs_dots + k_cgs_orth_dots + k_cgs_orth_norm in one launch, with the same block partition and
// the same summation order (so the same results): the two global sums between the passes are
// grid barriers instead of kernel boundaries, and every block sums the partials itself in block
// order.  Each pass has its own partials (a fast block never overwrites what a slow one reads).
// hh receives h (pass 1, with w.w at hh[m]), h2 (pass 2) and ||w|| (pass 3); the last block of
// pass 3 runs the Givens update and the stopping test.  bar: [0] arrivals, [1] generation,
// [2] pass-3 ticket.
__global__ void __launch_bounds__(VB) k_cgs_fused(int64_t n, GmDev* st, const double* __restrict__ V, int64_t ldv,
                                                  double* __restrict__ hh, double* __restrict__ w,
                                                  double* __restrict__ part, unsigned* bar, int kdim,
                                                  cudaGraphConditionalHandle hnd, int* err) {
    if (st->done) return;                  // a step after the solve stopped (uniform over the grid)
    const int m = st->col + 1;
    __shared__ double hs[GM_KMAX + 1];
    __shared__ double ps[CG_MAXB][GM_PS];
    __shared__ bool last;
    const bool staged = gridDim.x <= CG_MAXB;     // grid-uniform
    const int64_t pstride = (int64_t)gridDim.x * GM_PS;
    double* part1 = part;
    double* part2 = part + pstride;
    double* part3 = part + 2 * pstride;
    double acc[GM_KMAX + 1];
    // pass 1: V_q . w (q < m) and w . w
#pragma unroll
    for (int q = 0; q <= GM_KMAX; ++q) acc[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int q = 0; q <= GM_KMAX; ++q) {
            if (q < m) acc[q] += V[q * ldv + i] * wi;
            else if (q == m) acc[q] += wi * wi;
        }
    }
    gm_store_partials(acc, m + 1, part1);
    grid_sync_bounded(bar, bar + 1, err);
    if (staged) stage_partials(part1, m + 1, ps);
    if ((int)threadIdx.x <= m) {
        const double t = finish_partials(part1, threadIdx.x, ps);
        hs[threadIdx.x] = t;
        if (blockIdx.x == 0) hh[threadIdx.x] = t;
    }
    __syncthreads();
    // pass 2: w -= sum_q h[q] V_q, then V_q . w
#pragma unroll
    for (int q = 0; q <= GM_KMAX; ++q) acc[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double o = 0.0;
        for (int q = 0; q < m; ++q) o += hs[q] * V[q * ldv + i];
        const double wi = w[i] - o;
        w[i] = wi;
#pragma unroll
        for (int q = 0; q < GM_KMAX; ++q)
            if (q < m) acc[q] += V[q * ldv + i] * wi;
    }
    gm_store_partials(acc, m, part2);
    grid_sync_bounded(bar, bar + 1, err);
    if (staged) stage_partials(part2, m, ps);
    if ((int)threadIdx.x < m) {
        const double t = finish_partials(part2, threadIdx.x, ps);
        hs[threadIdx.x] = t;
        if (blockIdx.x == 0) hh[(kdim + 2) + threadIdx.x] = t;
    }
    __syncthreads();
    // pass 3: w -= sum_q h2[q] V_q, ||w||
    acc[0] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double o = 0.0;
        for (int q = 0; q < m; ++q) o += hs[q] * V[q * ldv + i];
        const double wi = w[i] - o;
        w[i] = wi;
        acc[0] += wi * wi;
    }
    gm_store_partials(acc, 1, part3);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(bar + 2, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last) {                                 // block-uniform
        __threadfence();
        if (staged) stage_partials(part3, 1, ps);
        if (threadIdx.x == 0) {
            hh[2 * (kdim + 2)] = sqrt(finish_partials(part3, 0, ps));
            bar[2] = 0u;
            gm_givens(st, hh, kdim, hnd);
        }
    }
}

// Self-test of the bounded grid barrier: a cooperative pair of blocks of which block 1 returns
// without arriving; block 0's wait gives up after `polls` polls and sets bit 4 of *err exactly as
// in k_cgs_fused, and the kernel returns.
__global__ void k_selftest_grid(int polls, unsigned* bar, int* err) {
    if (blockIdx.x != 0) return;
    grid_sync_bounded(bar, bar + 1, err, polls);
}

// least squares by back substitution (as in gmres()); ybuf = y, ncomb = its length
__global__ void k_gm_solve(GmDev* st, double* __restrict__ ybuf, int kdim) {
    if (threadIdx.x != 0) return;
    if (st->skip) {
        st->ncomb = 0;
        return;
    }
    const int col = st->col;
    double* H = st->H;
    auto h = [&](int c, int k) -> double& { return H[c * (kdim + 1) + k]; };
    double* S = st->S;
    if (h(col, col) == 0.0) S[col] = 0.0;
    double* y = st->y;
    for (int k = 0; k <= col; ++k) y[k] = S[k];
    for (int k = col; k > 0; --k) {
        if (y[k] != 0.0) {
            y[k] /= h(k, k);
            double tmp = y[k];
            for (int q = 0; q < k; ++q) y[q] -= tmp * h(k, q);
        }
    }
    if (y[0] != 0.0) y[0] /= h(0, 0);
    for (int k = 0; k <= col; ++k) ybuf[k] = y[k];
    st->ncomb = col + 1;
}

__global__ void k_combine_gm(int64_t n, const GmDev* __restrict__ st, const double* __restrict__ V, int64_t ldv,
                             const double* __restrict__ y, double* __restrict__ x) {
    const int m = st->ncomb;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < m; ++q) acc += y[q] * V[q * ldv + i];
        x[i] = acc;
    }
}

__global__ void k_gm_info(GmDev* st, const double* __restrict__ scal) {
    if (threadIdx.x != 0) return;
    const double rnorm = scal[10];
    st->rnorm = rnorm;
    st->info = st->skip ? 0 : ((rnorm <= st->atol_eff) ? 0 : 1);
}

// Host view of the results read back after a graph run.
struct GmHost {
    double args[4];               // t, dh, rtol, atol
    int res[6];                   // col, done, skip, iters, info, ncomb
    int err;                      // the model's device error word, read back with the results
};

// Arnoldi steps captured ahead of the WHILE node: GM_PREFIX, or DVTSA_GMRES_PREFIX=<0..8> from the
// environment (read once per process; a tuning knob: more steps save WHILE relaunches of long
// solves, but lengthen every graph launch on the host and run empty steps in short solves)
static int gmres_prefix() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_GMRES_PREFIX");
        v = GM_PREFIX;
        if (e && e[0] >= '0' && e[0] <= '8' && e[1] == 0) v = e[0] - '0';
    }
    return v;
}

// Arnoldi steps per pass through the WHILE body: the model's tuning, else DVTSA_GMRES_BODY=<1|2> from
// the environment (read once per process), else 2.  Each pass costs a device-side relaunch; a second
// step after the stop returns at once (the sweep sees the stop flag, the operator a zero direction).
static int gmres_body(const dv_model* m) {
    if (m->tune.gmres_body == 1 || m->tune.gmres_body == 2) return m->tune.gmres_body;
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_GMRES_BODY");
        v = (e && e[0] == '1' && e[1] == 0) ? 1 : 2;
    }
    return v;
}

// DVTSA_GMRES_COOP=0 keeps the three-kernel CGS2 in the GMRES graph (read once per process)
static bool gmres_coop_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_GMRES_COOP");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// The GMRES operator's launches inside the graph: the FP64 finite-difference matvec (three residual
// kernels) or, with the mixed-precision operator, one FP32 assembled-Jacobian product.
static int op_capture(dv_model* m, Work& W, const double* dargs, double* out, cudaStream_t c) {
    if (m->op32) return launch_spmv32(m, W.u, W.s, 0.0, dargs, out, c, false);
    return matvec_capture(m, dargs, W.z, W.u, W.s, W.f, W.scal, out, c, W.tickets + 11);
}
static void op_count(const dv_model* m, int64_t* cnt) {
    if (m->op32) cnt[K_SPMV] += 1;
    else cnt[K_MATVEC] += matvec_capture_kernels();
}

// A capture that another host thread invalidated (for instance by the first launch of a kernel,
// which loads it into the context while this thread captures): gm_build tries again.
static constexpr int GM_CAPTURE_RETRY = 1000;

static int gm_build_once(dv_model* m, Work& W, int kdim) {
    if (W.gm_exec) { cudaGraphExecDestroy(W.gm_exec); W.gm_exec = nullptr; }
    if (W.gm_graph) { cudaGraphDestroy(W.gm_graph); W.gm_graph = nullptr; }
    if (!W.gm_cs) DV_CUDA(cudaStreamCreateWithFlags(&W.gm_cs, cudaStreamNonBlocking));
    cudaStream_t body_cs = nullptr;
    DV_CUDA(cudaStreamCreateWithFlags(&body_cs, cudaStreamNonBlocking));
    GmDev* st = (GmDev*)W.gm;
    const double* dargs = (const double*)st;              // t, dh
    const int64_t n = W.n, ldv = n;
    const unsigned g = vgrid(n);
    cudaStream_t cs = W.gm_cs;
    int64_t fixed[K_NKIND] = {0}, iter[K_NKIND] = {0};
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    cudaGraph_t cg = nullptr;
    cudaGraphConditionalHandle hnd = 0;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaStreamCaptureStatus cst;
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hnd, cg, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        // pre: ||b||, loop state
        k_sumsq_finish<<<g, VB, 0, cs>>>(n, W.b, nullptr, W.part, W.tickets + 6, 2, W.scal + 9);
        k_gm_init<<<1, VB, 0, cs>>>(st, W.scal, kdim, hnd, W.tickets + 8);
        fixed[K_VECTOR] += 2;
    }
    const bool fused = precond_apply_fusable(m);
    // the cooperative CGS2 kernel takes at most one block per SM (all of them must be resident)
    static bool coop_ok = true;               // cleared if the CUDA driver refuses a cooperative node
    int nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned gc = std::min<unsigned>(g, (unsigned)std::max(nsm, 1));
    const bool coop = coop_ok && gmres_coop_enabled();
    bool coop_failed = false;
    // One Arnoldi step of the fused form: sweep with normalisation prologue and rms epilogue,
    // matvec, CGS2 in three kernels; every kernel returns at once when st->done is set.
    auto arnoldi_step = [&](cudaStream_t c) -> int {
        PaFuse F;
        F.col = &st->col;
        F.scale = &st->scale;
        F.src0 = W.b;
        F.src1 = W.wout;
        F.V = W.V;
        F.ldv = ldv;
        F.part = W.apart;
        F.ticket = W.tickets + 0;
        F.out = W.scal + 0;
        F.n = n;
        F.stop = &st->done;
        F.pdl = pdl_enabled();
        int rc = precond_apply_capture(m, W.vin, W.s, W.u, c, F);
        if (rc == DV_OK) rc = op_capture(m, W, dargs, W.wout, c);
        if (coop) {                          // CGS2 as one cooperative launch (co-resident blocks)
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(gc);
            cfg.blockDim = dim3(VB);
            cfg.stream = c;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeCooperative;
            at[0].val.cooperative = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            if (cudaLaunchKernelEx(&cfg, k_cgs_fused, n, st, (const double*)W.V, ldv, W.hbuf, W.wout, W.part,
                                   W.tickets + 8, kdim, hnd, m->d_err) != cudaSuccess)
                coop_failed = true;
        } else {
            k_cgs_dots<<<g, VB, 0, c>>>(n, st, W.V, ldv, W.wout, W.part, W.tickets + 1, W.hbuf);
            k_cgs_orth_dots<<<g, VB, 0, c>>>(n, st, W.V, ldv, W.hbuf, W.wout, W.part, W.tickets + 2,
                                             W.hbuf + (kdim + 2));
            k_cgs_orth_norm<<<g, VB, 0, c>>>(n, st, W.V, ldv, W.hbuf, W.wout, W.part, W.tickets + 3, kdim, hnd);
        }
        return rc;
    };
    const int ncgs = coop ? 1 : 3;           // launches of the CGS2 part of a step
    // The first GM_PREFIX steps are plain nodes ahead of the WHILE node: every solve takes at least
    // two steps and most take five or more, and each pass through the WHILE body costs a device-side
    // relaunch (~20 us on B200) that a plain node does not; a step after the stop returns at once.
    const int prefix = fused ? std::min(m->tune.gmres_prefix >= 0 ? m->tune.gmres_prefix : gmres_prefix(), kdim) : 0;
    const int body_steps = fused ? gmres_body(m) : 1;        // Arnoldi steps per pass through the WHILE body
    if (e == cudaSuccess) {
        for (int q = 0; q < prefix && e == cudaSuccess; ++q) {
            if (arnoldi_step(cs) != DV_OK) e = cudaErrorUnknown;
            fixed[K_PC_APPLY] += 1;
            op_count(m, fixed);
            fixed[K_VECTOR] += ncgs;
        }
        if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, &deps, &ndeps);
    }
    cudaGraphNode_t cnode = nullptr;
    cudaGraph_t body = nullptr;
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp);
        if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(body_cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        // body: one Arnoldi step
        int rc = DV_OK;
        if (fused) {
            for (int q = 0; q < body_steps && rc == DV_OK; ++q) {
                rc = arnoldi_step(body_cs);
                iter[K_PC_APPLY] += 1;
                op_count(m, iter);
                iter[K_VECTOR] += ncgs;
            }
        } else {
            k_gm_norm<<<g, VB, 0, body_cs>>>(n, st, W.b, W.wout, W.V, ldv, W.vin);
            iter[K_VECTOR] += 1;
            rc = precond_apply_capture(m, W.vin, W.s, W.u, body_cs);
            iter[K_PC_APPLY] += 1;
            k_sumsq<<<g, VB, 0, body_cs>>>(n, W.u, nullptr, W.part);
            k_finish<<<1, VB, 0, body_cs>>>((int)g, W.part, (double)n, 0, W.scal + 0);
            iter[K_VECTOR] += 2;
            if (rc == DV_OK) rc = op_capture(m, W, dargs, W.wout, body_cs);
            op_count(m, iter);
            for (int pass = 0; pass < 2; ++pass) {
                double* hb = W.hbuf + pass * (kdim + 2);
                k_dots_gm<<<g, VB, 0, body_cs>>>(n, st, W.V, ldv, W.wout, W.part);
                k_dots_finish_gm<<<kdim + 2, VB, 0, body_cs>>>((int)g, st, W.part, hb);
                k_orth_update_gm<<<g, VB, 0, body_cs>>>(n, st, W.V, ldv, hb, W.wout);
            }
            k_sumsq<<<g, VB, 0, body_cs>>>(n, W.wout, nullptr, W.part);
            k_finish<<<1, VB, 0, body_cs>>>((int)g, W.part, (double)n, 2, W.hbuf + 2 * (kdim + 2));
            k_gm_givens<<<1, 32, 0, body_cs>>>(st, W.hbuf, kdim, hnd);
            iter[K_VECTOR] += 9;
        }
        cudaGraph_t tmp = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(body_cs, &tmp);
        e = (rc != DV_OK) ? cudaErrorUnknown : e2;
    }
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
        // post: y, x = V y, true residual r = b - AP x
        k_gm_solve<<<1, 32, 0, cs>>>(st, W.ybuf, kdim);
        k_combine_gm<<<g, VB, 0, cs>>>(n, st, W.V, ldv, W.ybuf, W.x);
        fixed[K_VECTOR] += 2;
        int rc;
        if (fused) {
            PaFuse F;
            F.part = W.apart;
            F.ticket = W.tickets + 4;
            F.out = W.scal + 0;
            F.n = n;
            F.pdl = pdl_enabled();
            rc = precond_apply_capture(m, W.x, W.s, W.u, cs, F);
        } else {
            rc = precond_apply_capture(m, W.x, W.s, W.u, cs);
            k_sumsq<<<g, VB, 0, cs>>>(n, W.u, nullptr, W.part);
            k_finish<<<1, VB, 0, cs>>>((int)g, W.part, (double)n, 0, W.scal + 0);
            fixed[K_VECTOR] += 2;
        }
        fixed[K_PC_APPLY] += 1;
        if (rc == DV_OK) rc = op_capture(m, W, dargs, W.r, cs);
        op_count(m, fixed);
        k_axpby<<<g, VB, 0, cs>>>(n, 1.0, W.b, -1.0, W.r, W.r);
        k_sumsq_finish<<<g, VB, 0, cs>>>(n, W.r, nullptr, W.part, W.tickets + 6, 2, W.scal + 10);
        k_gm_info<<<1, 32, 0, cs>>>(st, W.scal);
        fixed[K_VECTOR] += 3;
        if (rc != DV_OK) e = cudaErrorUnknown;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t e3 = cudaStreamEndCapture(cs, &graph);     // always end the capture
    if (e == cudaSuccess) e = e3;
    cudaStreamDestroy(body_cs);
    if (coop_failed) {                        // build again with the three-kernel CGS2
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        coop_ok = false;
        return gm_build_once(m, W, kdim);
    }
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (e == cudaErrorStreamCaptureInvalidated) return GM_CAPTURE_RETRY;
        return cuda_fail(e, "building the GMRES graph");
    }
    W.gm_graph = graph;
    DV_CUDA(cudaGraphInstantiate(&W.gm_exec, graph, 0));
    W.gm_kdim = kdim;
    W.gm_mode = m->pc_mode;
    W.gm_nb = m->pc_nb;
    W.gm_nparts = m->pc_nparts;
    W.gm_zs = m->pc_zs;
    W.gm_prefix = prefix;
    W.gm_fp32 = m->pc_fp32;
    W.gm_op32 = m->op32;
    W.gm_tuned = m->tune.gmres_prefix;
    W.gm_body = body_steps;
    for (int k = 0; k < K_NKIND; ++k) {
        W.gm_fixed[k] = fixed[k];
        W.gm_iter[k] = iter[k];
    }
    return DV_OK;
}

static int gm_build(dv_model* m, Work& W, int kdim) {
    std::lock_guard<std::recursive_mutex> lk(capture_mutex());
    for (int attempt = 0; attempt < 16; ++attempt) {
        const int rc = gm_build_once(m, W, kdim);
        if (rc != GM_CAPTURE_RETRY) return rc;
        std::this_thread::sleep_for(std::chrono::microseconds(200 << std::min(attempt, 6)));
    }
    return cuda_fail(cudaErrorStreamCaptureInvalidated, "building the GMRES graph (capture invalidated 16 times)");
}

// gmres() run by the graph; same contract.  b, op.z, op.f, op.s must be the workspace's own
// vectors (the graph is built on their addresses).
static int gmres_graph(Work& W, const Op& op, const double* b, double rtol, double atol, int kdim, int* info,
                       int64_t* inner, cudaStream_t st) {
    dv_model* m = op.m;
    if (!W.gm_exec || W.gm_kdim != kdim || W.gm_mode != m->pc_mode || W.gm_nb != m->pc_nb ||
        W.gm_nparts != m->pc_nparts || W.gm_fp32 != m->pc_fp32 || W.gm_zs != m->pc_zs ||
        W.gm_op32 != m->op32 || W.gm_tuned != m->tune.gmres_prefix ||
        (precond_apply_fusable(m) && W.gm_body != gmres_body(m)))
        DV_TRY(gm_build(m, W, kdim));
    GmHost* hst = (GmHost*)W.gm_host;
    hst->args[0] = op.t;
    hst->args[1] = op.dh;
    hst->args[2] = rtol;
    hst->args[3] = atol;
    GmDev* dev = (GmDev*)W.gm;
    DV_CUDA(cudaMemcpyAsync(dev, hst->args, sizeof(hst->args), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaGraphLaunch(W.gm_exec, st));
    DV_CUDA(cudaMemcpyAsync(hst->res, &dev->col, sizeof(hst->res), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(&hst->err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return DV_OK;
}

// Results of the last gmres_graph launch, once the stream has been synchronised.
static int gmres_graph_collect(Work& W, dv_model* m, int* info, int64_t* inner) {
    GmHost* hst = (GmHost*)W.gm_host;
    const int iters = hst->res[3], skip = hst->res[2];
    *info = hst->res[4];
    *inner += iters;
    m->nfev += iters + (skip ? 0 : 1);
    const int looped = (std::max(iters - W.gm_prefix, 0) + W.gm_body - 1) / std::max(W.gm_body, 1);   // WHILE passes
    for (int k = 0; k < K_NKIND; ++k) count_launches(k, W.gm_fixed[k] + W.gm_iter[k] * looped);
    if (g_prof_on && !g_pending.empty()) prof_flush();
    if (hst->err != 0) {                  // (read back with the results: no extra round trip)
        set_error(device_error_text(hst->err));
        hst->err = 0;
        clear_device_error(m);
        return DV_ERR_CUDA;
    }
    return DV_OK;
}

// DVTSA_GMRES_GRAPH=0 in the environment runs GMRES host-driven (read once per process; for tools
// that want plain kernel launches, such as a kernel-by-kernel profiler).
static bool gmres_graph_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("DVTSA_GMRES_GRAPH");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// The graph when it applies; the host-driven loop while launches are being profiled one by one.
// With *pending set on return the graph is still running: call gmres_graph_collect after the
// next synchronisation of the stream.
static int gmres_start(Work& W, const Op& op, const double* b, double rtol, double atol, int kdim, int* info,
                       int64_t* inner, bool* pending, cudaStream_t st) {
    *pending = false;
    if (g_prof_on || !gmres_graph_enabled() || b != W.b || op.z != W.z || op.f != W.f || op.s != W.s ||
        kdim > GM_KMAX)
        return gmres(W, op, b, rtol, atol, kdim, info, inner, st);
    DV_TRY(gmres_graph(W, op, b, rtol, atol, kdim, info, inner, st));
    *pending = true;
    return DV_OK;
}

static int gmres_any(Work& W, const Op& op, const double* b, double rtol, double atol, int kdim, int* info,
                     int64_t* inner, cudaStream_t st) {
    bool pending = false;
    DV_TRY(gmres_start(W, op, b, rtol, atol, kdim, info, inner, &pending, st));
    if (!pending) return DV_OK;
    DV_CUDA(cudaStreamSynchronize(st));
    return gmres_graph_collect(W, op.m, info, inner);
}

}  // namespace dv
// ================================================================== Newton-Krylov stage solve
namespace dv {

struct NewtonCtx {
    dv_model* m;
    Work* W;
    const double* atol7;
    int64_t n, npos;
    dv_newton_opts o;
    dv_newton_result* res;
    int64_t* gm_counter;      // GMRES iterations counted towards the Jacobian-refresh rule
};

static int refresh_J(NewtonCtx& C, double t, const double* z, double dh, cudaStream_t st) {
    // fc = rhs(t, zc); J = jac(t, zc, fc); factor(J, h) with h = dh / D (core/solver.py:350-356)
    Work& W = *C.W;
    DV_TRY(launch_rhs(C.m, t, z, W.tmp, nullptr, st));
    DV_TRY(launch_fd_jacobian(C.m, t, z, W.tmp, W.J, st));
    C.m->nfev += C.m->ncolours;
    if (C.m->op32) {
        DV_TRY(launch_fd_jacobian32(C.m, t, z, W.tmp, C.m->d_J32, st));
        C.m->nfev += C.m->ncolours;
    }
    const double D = (2.0 - std::sqrt(2.0)) / 2.0;
    const double h = dh / D;
    DV_TRY(precond_factor(C.m, W.J, D * h, C.o.precond_mode, st));
    return DV_OK;
}

// newton_krylov (core/solver.py:154-294) on the GPU.  z written to `zout`.
static int newton_krylov(NewtonCtx& C, double t, const double* z0, const double* rhs_known, double dh, double* zout,
                         cudaStream_t st) {
    Work& W = *C.W;
    dv_model* m = C.m;
    const int64_t n = C.n;
    const unsigned g = vgrid(n);
    dv_newton_result& r = *C.res;
    r.ok = 0;
    r.iters = 0;
    r.rate = 0.0;
    r.refreshed = 0;
    const double kappa = C.o.kappa, rtol = C.o.rtol;
    auto scale = [&](const double* z, double* s) { DV_LAUNCH(dv::K_VECTOR, st, k_scale<<<g, VB, 0, st>>>(m->nc, n, z, C.atol7, rtol, s)); };
    auto stage = [&](const double* z, double* f, double* R) -> int {
        // f = rhs(z); R = z - dh f - rhs_known
        DV_TRY(launch_rhs(m, t, z, f, nullptr, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, z, -dh, f, R));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, R, -1.0, rhs_known, R));
        return DV_OK;
    };
    auto pnorm = [&](const double* RR, const double* ss, double* out) -> int {
        DV_TRY(precond_apply(m, RR, nullptr, W.tmp, st));
        return rms_ratio(W, n, W.tmp, ss, out, st);
    };
    auto copy = [&](const double* a, double* b) { DV_CUDA(cudaMemcpyAsync(b, a, sizeof(double) * n, cudaMemcpyDeviceToDevice, st)); return DV_OK; };
    auto cons_ok = [&](const double* R, const double* z, bool* ok) -> int {
        if (C.o.cons_tol <= 0.0) { *ok = true; return DV_OK; }
        scale(z, W.tmp);
        DV_LAUNCH(dv::K_VECTOR, st, k_cons<<<cons_grid(m->nc), VB, 0, st>>>(m->p, R, W.tmp, W.apart, W.tickets + 5, W.scal));
        DV_CUDA(cudaGetLastError());
        double v[8];
        DV_TRY(fetch(W, W.scal, 8, v, st));
        *ok = true;
        for (int q = 0; q < 4; ++q)
            if (!(std::fabs(v[q]) <= C.o.cons_tol * v[4 + q])) *ok = false;
        return DV_OK;
    };

    // Balance projection of a converged stage solution W.z whose balances are not closed: the
    // correction z += sum_q lam_q b_q, one direction per conserved quantity (k_cons_basis), with
    // W A B lam = -W R (A = I - dh J applied to each b_q by the finite-difference operator), closes
    // the linearised balances exactly; the state moves by about |W R| / |W z| relative, far below
    // the tolerance.  Recomputes f and R at the new state; *okp = balances closed after it.
    auto project = [&](bool* okp) -> int {
        *okp = false;
        if (4 * (W.kdim + 2) < 40) return DV_OK;    // hbuf too small for the 40 sums
        double* H = W.hbuf;                  // 5 x 8 balance sums (free outside GMRES)
        DV_TRY(rms_ratio_dev(W, n, W.z, W.s, 1, W.scal + 1, st));       // the FD step's max(1, rms(z/s))
        for (int q = 0; q < 4; ++q) {
            DV_LAUNCH(dv::K_VECTOR, st, k_cons_basis<<<g, VB, 0, st>>>(m->nc, n, q, W.z, W.s, W.dz));
            DV_TRY(rms_ratio_dev(W, n, W.dz, nullptr, 0, W.scal + 0, st));
            DV_TRY(launch_matvec(m, t, W.z, W.dz, W.s, W.f, dh, W.scal, W.r, st));     // (A b_q) / s
            DV_LAUNCH(dv::K_VECTOR, st, k_mul<<<g, VB, 0, st>>>(n, W.r, W.s, W.w));
            DV_LAUNCH(dv::K_VECTOR, st, k_cons<<<cons_grid(m->nc), VB, 0, st>>>(m->p, W.w, W.s, W.apart,
                                                                                  W.tickets + 5, H + 8 * q));
        }
        DV_LAUNCH(dv::K_VECTOR, st, k_cons<<<cons_grid(m->nc), VB, 0, st>>>(m->p, W.R, W.s, W.apart, W.tickets + 5,
                                                                              H + 32));
        m->nfev += 4;
        double h[40];
        DV_TRY(fetch(W, H, 40, h, st));
        double G[16], rhs[4], lam[4];
        bool active[4];
        for (int q = 0; q < 4; ++q) {
            rhs[q] = -h[32 + q];
            active[q] = std::fabs(h[8 * q + q]) > 1e-12 * h[32 + 4 + q];     // quantity present
            for (int b = 0; b < 4; ++b) G[q * 4 + b] = h[8 * b + q];         // row q: W_q (A b_b)
        }
        // a quantity whose closure would need more than a small correction (a species whose
        // inventory is at its absolute-tolerance floor, such as N2 under vacuum) leaves the system
        bool solved = false;
        for (int pass = 0; pass < 4 && !solved; ++pass) {
            if (!solve_small(G, rhs, active, lam)) return DV_OK;
            solved = true;
            for (int q = 0; q < 4; ++q)
                if (active[q] && !(std::fabs(lam[q]) <= (q < DV_NG ? 1e-2 : 1.0))) {
                    active[q] = false;
                    solved = false;
                }
        }
        if (!solved) return DV_OK;
        DV_LAUNCH(dv::K_VECTOR, st, k_cons_shift<<<g, VB, 0, st>>>(m->nc, n, lam[0], lam[1], lam[2], lam[3], W.s, W.z));
        DV_TRY(stage(W.z, W.f, W.R));
        return cons_ok(W.R, W.z, okp);
    };

    // An unclosed stage returns its best converged state (by rms(R/s), as the reference does); with
    // the balance projection on, the quantities that can be closed are closed on that state first.
    auto return_best = [&]() -> int {
        if (!C.o.balance_projection) return copy(W.best, zout);
        DV_TRY(copy(W.best, W.z));
        scale(W.z, W.s);
        DV_TRY(stage(W.z, W.f, W.R));
        bool okp = false;
        DV_TRY(project(&okp));
        return copy(W.z, zout);
    };

    auto cons_eval = [&](const double* v) -> bool {
        if (C.o.cons_tol <= 0.0) return true;
        bool ok = true;
        for (int q = 0; q < 4; ++q)
            if (!(std::fabs(v[q]) <= C.o.cons_tol * v[4 + q])) ok = false;
        return ok;
    };
    // Queue the evaluation of the full Newton step from the GMRES solution W.x: dz, the trial point
    // at lam = 1 with its stage residual, and the scalars the host tests (rms(dz), rms(R/s), the
    // preconditioned norm, the step length, the balance sums); copy them into W.hpin[16..47].
    auto speculate = [&]() -> int {
        DV_TRY(precond_apply(m, W.x, W.s, W.u, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_mul<<<g, VB, 0, st>>>(n, W.u, W.s, W.dz));
        DV_TRY(rms_ratio_dev(W, n, W.dz, nullptr, 0, W.scal + 11, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_truncate<<<g, VB, 0, st>>>(n, C.npos, W.z, 1.0, W.dz, W.zt));
        DV_TRY(stage(W.zt, W.ft, W.Rt));
        DV_TRY(rms_ratio_dev(W, n, W.Rt, W.s, 0, W.scal + 12, st));
        DV_TRY(precond_apply(m, W.Rt, nullptr, W.tmp, st));
        DV_TRY(rms_ratio_dev(W, n, W.tmp, W.s, 0, W.scal + 13, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.zt, -1.0, W.z, W.r));
        DV_TRY(rms_ratio_dev(W, n, W.r, W.s, 0, W.scal + 14, st));
        if (C.o.cons_tol > 0.0) {
            scale(W.zt, W.w);
            // into scal[16..23]: scal[0..1] still feed the matvec of a GMRES rerun after a refresh
            DV_LAUNCH(dv::K_VECTOR, st, k_cons<<<cons_grid(m->nc), VB, 0, st>>>(m->p, W.Rt, W.w, W.apart, W.tickets + 5,
                                                                                  W.scal + 16));
        }
        DV_CUDA(cudaMemcpyAsync(W.hpin + 16, W.scal, sizeof(double) * 32, cudaMemcpyDeviceToHost, st));
        return DV_OK;
    };

    DV_TRY(copy(z0, W.z));
    DV_TRY(stage(W.z, W.f, W.R));
    scale(W.z, W.s);
    // rms(R/s) and the preconditioned norm of R, queued into scal[24..25]: they come back with the
    // first iteration's speculated scalars (one synchronisation fewer per stage solve and per
    // norm); a non-finite rms then returns z0 as before, with the counters of that iteration undone
    DV_TRY(rms_ratio_dev(W, n, W.R, W.s, 0, W.scal + 24, st));
    DV_TRY(precond_apply(m, W.R, nullptr, W.tmp, st));
    DV_TRY(rms_ratio_dev(W, n, W.tmp, W.s, 0, W.scal + 25, st));
    double rn = 0.0, pn = 0.0;
    const int64_t nfev0 = m->nfev;
    double step_prev = -1.0;     // < 0 : None
    int polish = 0;
    bool have_best = false;
    double best_rn = 0.0;
    bool new_lu = false;
    bool projected = false;      // the balance projection was tried in this solve
    int it = -1;
    const double sqrt_n = std::sqrt((double)n);
    while (it + 1 < C.o.max_iter + polish) {
        ++it;
        scale(W.z, W.s);
        DV_LAUNCH(dv::K_VECTOR, st, k_div<<<g, VB, 0, st>>>(n, -1.0, W.R, W.s, W.b));                    // b = -R/s
        DV_TRY(rms_ratio_dev(W, n, W.z, W.s, 1, W.scal + 1, st));           // zs = max(1, rms(z/s))
        Op op{m, t, dh, W.z, W.f, W.s, n};
        const double floor_ = (polish ? 1e-4 : 0.1 * kappa) * sqrt_n;
        int info = 0;
        int64_t inner = 0;
        bool pending = false;
        DV_TRY(gmres_start(W, op, W.b, polish ? 1e-3 : C.o.eta, floor_, C.o.krylov_dim, &info, &inner, &pending, st));
        // the full step (lam = 1) and every norm the host tests next, queued behind GMRES, read
        // back with one synchronisation (same kernels and inputs as evaluating them one by one)
        DV_TRY(speculate());
        DV_CUDA(cudaStreamSynchronize(st));
        if (pending) DV_TRY(gmres_graph_collect(W, m, &info, &inner));
        if (it == 0) {                                       // the norms queued before the loop
            rn = W.hpin[16 + 24];
            pn = W.hpin[16 + 25];
            if (!std::isfinite(rn)) {
                m->nfev = nfev0;
                DV_TRY(copy(z0, zout));
                r.rate = INFINITY;
                return DV_OK;
            }
        }
        bool spec_ok = true;
        if (polish) r.gmres_polish += inner;
        else { r.gmres_iters += inner; if (C.gm_counter) *C.gm_counter += inner; }
        if (info != 0 && C.o.allow_refresh && !new_lu && !polish) {
            spec_ok = false;                                 // factors change: the speculation is void
            m->nfev -= 1;                                    // (its residual evaluation is not counted)
            DV_TRY(refresh_J(C, t, W.z, dh, st));
            new_lu = true;
            r.refreshed = 1;
            r.jac_refresh_in_newton += 1;
            DV_TRY(pnorm(W.R, W.s, &pn));
            int64_t inner2 = 0;
            DV_TRY(gmres_any(W, op, W.b, C.o.eta, floor_, C.o.krylov_dim, &info, &inner2, st));
            r.gmres_iters += inner2;
            if (C.gm_counter) *C.gm_counter += inner2;
        }
        // polish: further restart cycles until the polish tolerance (1e-3 of ||b||) or the cycle
        // limit.  Each cycle solves A P^-1 x_c = b0 - A P^-1 (x_1 + .. x_c-1), the linear residual
        // of the summed solution recomputed from it (the speculation queued behind the first cycle
        // reused the GMRES residual vector, and is void anyway); the Newton step is then formed
        // from x = sum x_c, as from a single cycle's solution.
        const int pcyc = std::min(std::max(C.o.polish_cycles, 1), 8);
        if (polish && info != 0 && pcyc > 1) {
            spec_ok = false;
            m->nfev -= 1;
            DV_LAUNCH(dv::K_VECTOR, st, k_div<<<g, VB, 0, st>>>(n, -1.0, W.R, W.s, W.tmp));   // b0 = -R/s
            double bn0 = 0.0;
            DV_TRY(rms_ratio(W, n, W.tmp, nullptr, &bn0, st));
            DV_TRY(copy(W.x, W.dz));                          // dz: the summed solution x
            for (int cyc = 1; cyc < pcyc && info != 0; ++cyc) {
                DV_TRY(precond_apply(m, W.dz, W.s, W.u, st));       // u = P^-1 x
                DV_TRY(op_residual(W, op, W.tmp, W.u, W.b, st));    // b = b0 - A u
                double rk = 0.0;
                DV_TRY(rms_ratio(W, n, W.b, nullptr, &rk, st));
                if (!(rk > 1e-3 * bn0) || !std::isfinite(rk)) break;
                int64_t inner2 = 0;
                DV_TRY(gmres_any(W, op, W.b, std::min(1.0, 1e-3 * bn0 / rk), floor_, C.o.krylov_dim, &info,
                                 &inner2, st));
                r.gmres_polish += inner2;
                m->nfev += 1;                                 // the residual's operator product
                DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.dz, 1.0, W.x, W.dz));
            }
            DV_TRY(copy(W.dz, W.x));
            DV_TRY(copy(W.tmp, W.b));
        }
        if (!spec_ok) {
            DV_TRY(speculate());
            DV_CUDA(cudaStreamSynchronize(st));
        }
        const double* sv = W.hpin + 16;                      // speculated scalars (see speculate)
        // dz = prec(w) * s
        const double dzn = sv[11];
        if (!std::isfinite(dzn)) {
            DV_TRY(copy(z0, zout));
            r.iters = it + 1;
            r.rate = INFINITY;
            return DV_OK;
        }
        double lam = 1.0, rn_try = 0.0, pn_try = INFINITY;
        for (int ls = 0; ls < 4; ++ls) {
            if (ls == 0) {                                   // lam = 1: already evaluated
                rn_try = sv[12];
                pn_try = std::isfinite(rn_try) ? sv[13] : INFINITY;
            } else {
                DV_LAUNCH(dv::K_VECTOR, st, k_truncate<<<g, VB, 0, st>>>(n, C.npos, W.z, lam, W.dz, W.zt));
                DV_TRY(stage(W.zt, W.ft, W.Rt));
                DV_TRY(rms_ratio(W, n, W.Rt, W.s, &rn_try, st));
                if (std::isfinite(rn_try)) DV_TRY(pnorm(W.Rt, W.s, &pn_try));
                else pn_try = INFINITY;
            }
            if (std::isfinite(pn_try) && (pn_try <= (1.0 - 1e-4 * lam) * pn || ls == 3)) break;
            lam *= 0.5;
        }
        if (!std::isfinite(pn_try)) {
            DV_TRY(copy(z0, zout));
            r.iters = it + 1;
            r.rate = INFINITY;
            return DV_OK;
        }
        // step = rms((z_try - z)/s)
        double step;
        if (lam == 1.0) {
            step = sv[14];
        } else {
            DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.zt, -1.0, W.z, W.tmp));
            DV_TRY(rms_ratio(W, n, W.tmp, W.s, &step, st));
        }
        const bool cons_spec = (lam == 1.0);
        // accept the trial point (copies, not pointer swaps: the GMRES graph is built on these addresses)
        DV_TRY(copy(W.zt, W.z));
        DV_TRY(copy(W.ft, W.f));
        DV_TRY(copy(W.Rt, W.R));
        rn = rn_try;
        pn = pn_try;
        const double rate = (step_prev < 0.0) ? 0.0 : step / std::max(step_prev, 1e-300);
        const bool sp = step_prev >= 0.0;
        const bool converged = (lam == 1.0 && step <= kappa && (info == 0 || sp)) ||
                               (sp && lam == 1.0 && info == 0 && rate < 1.0 && rate / (1.0 - rate) * step <= kappa) ||
                               pn <= kappa;
        if (converged) {
            if (!have_best || rn < best_rn) {
                have_best = true;
                best_rn = rn;
                DV_TRY(copy(W.z, W.best));
            }
            bool ok;
            if (cons_spec) ok = cons_eval(sv + 16);
            else DV_TRY(cons_ok(W.R, W.z, &ok));
            if (ok) {
                DV_TRY(copy(W.z, zout));
                r.ok = 1; r.iters = it + 1; r.rate = rate;
                return DV_OK;
            }
            if (C.o.balance_projection && !projected) {
                projected = true;
                bool okp = false;
                DV_TRY(project(&okp));
                if (okp) {
                    r.balance_projected += 1;
                    DV_TRY(copy(W.z, zout));
                    r.ok = 1; r.iters = it + 1; r.rate = rate;
                    return DV_OK;
                }
                // not closed: the reference's polish continues from the (projected) state
                scale(W.z, W.s);
                DV_TRY(rms_ratio(W, n, W.R, W.s, &rn, st));
                DV_TRY(pnorm(W.R, W.s, &pn));
            }
            if (polish < (C.o.max_polish > 0 ? C.o.max_polish : 2)) {
                polish += 1;
                step_prev = -1.0;
                continue;
            }
            r.balance_unclosed += 1;
            DV_TRY(return_best());
            r.ok = 1; r.iters = it + 1; r.rate = rate;
            return DV_OK;
        }
        if (have_best) {
            r.balance_unclosed += 1;
            DV_TRY(return_best());
            r.ok = 1; r.iters = it + 1; r.rate = rate;
            return DV_OK;
        }
        if (sp && lam == 1.0 && info == 0) {
            const int left = C.o.max_iter - it - 1;
            if (it >= 2 && (rate >= 1.0 || std::pow(rate, left) / (1.0 - rate) * step > kappa * 1e3)) {
                DV_TRY(copy(W.z, zout));
                r.ok = 0; r.iters = it + 1; r.rate = rate;
                return DV_OK;
            }
        }
        step_prev = step;
    }
    DV_TRY(copy(W.z, zout));
    r.ok = 0;
    r.iters = it + 1;
    r.rate = 1.0;
    return DV_OK;
}

}  // namespace dv

namespace dv {
// newton_modified (core/solver.py:111-151): Newton iterations with the stored factors as the
// Jacobian, dz = -M^-1 R; positivity truncation; accepted on the contraction estimate
// rate / (1 - rate) |dz| <= kappa (never on the first iterate), then the conservation check of
// the next residual.  One synchronisation per iteration (the host takes the branch decisions).
static int newton_modified(dv_model* m, double t, const double* z0, const double* rhs_known, double dh, int max_iter,
                           double kappa, double fail_rate, double cons_tol, double rtol, double* zout, bool* ok,
                           int* iters, double* rate, cudaStream_t st) {
    Work& W = *m->W;
    const int64_t n = m->n;
    const int64_t npos = (int64_t)(DV_NG + DV_NA) * m->nc;
    const unsigned g = vgrid(n);
    auto copy = [&](const double* a, double* b) {
        return cudaMemcpyAsync(b, a, sizeof(double) * n, cudaMemcpyDeviceToDevice, st) == cudaSuccess
                   ? DV_OK : cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
    };
    auto finish = [&](const double* z, bool good, int it) -> int {
        DV_TRY(copy(z, zout));
        *ok = good;
        *iters = it;
        return DV_OK;
    };
    DV_TRY(copy(z0, W.z));
    double nrm_prev = -1.0;
    *rate = 0.0;
    bool done = false;
    for (int it = 0; it < max_iter + 2; ++it) {
        DV_TRY(launch_rhs(m, t, W.z, W.f, nullptr, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.z, -dh, W.f, W.R));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.R, -1.0, rhs_known, W.R));
        double rr = 0.0;
        DV_TRY(rms_ratio(W, n, W.R, nullptr, &rr, st));
        if (!std::isfinite(rr)) {
            *rate = INFINITY;
            return finish(z0, false, it);
        }
        if (done) {                                  // converged in the step norm: the balances
            bool cok = true;
            DV_LAUNCH(dv::K_VECTOR, st, k_scale<<<g, VB, 0, st>>>(m->nc, n, W.z, m->d_atol7, rtol, W.tmp));
            DV_LAUNCH(dv::K_VECTOR, st, k_cons<<<cons_grid(m->nc), VB, 0, st>>>(m->p, W.R, W.tmp, W.apart,
                                                                                  W.tickets + 5, W.scal));
            double v[8];
            DV_TRY(fetch(W, W.scal, 8, v, st));
            for (int q = 0; q < 4; ++q)
                if (!(std::fabs(v[q]) <= cons_tol * v[4 + q])) cok = false;
            if (cok || it >= max_iter + 1) return finish(W.z, true, it);
        } else if (it >= max_iter) {
            break;
        }
        DV_TRY(precond_apply(m, W.R, nullptr, W.dz, st));                    // z_new = z - M^-1 R
        DV_LAUNCH(dv::K_VECTOR, st, k_truncate<<<g, VB, 0, st>>>(n, npos, W.z, -1.0, W.dz, W.zt));
        DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<g, VB, 0, st>>>(n, 1.0, W.zt, -1.0, W.z, W.r));
        DV_LAUNCH(dv::K_VECTOR, st, k_scale<<<g, VB, 0, st>>>(m->nc, n, W.zt, m->d_atol7, rtol, W.s));
        double nrm = 0.0;
        DV_TRY(rms_ratio(W, n, W.r, W.s, &nrm, st));
        DV_TRY(copy(W.zt, W.z));
        if (!std::isfinite(nrm)) {
            *rate = INFINITY;
            return finish(z0, false, it + 1);
        }
        if (done) continue;
        // no acceptance on the first iterate: a stale factorisation can give a small update while the
        // residual is still large; the rate estimate needs two iterates
        if (nrm_prev >= 0.0) {
            *rate = nrm / std::max(nrm_prev, 1e-300);
            if (*rate >= fail_rate) return finish(W.z, false, it + 1);
            if (*rate / (1.0 - *rate) * nrm <= kappa) {
                if (cons_tol <= 0.0) return finish(W.z, true, it + 1);
                done = true;
            }
        } else if (nrm < 1e-8) {
            if (cons_tol <= 0.0) {
                *rate = 0.0;
                return finish(W.z, true, it + 1);
            }
            done = true;
        }
        nrm_prev = nrm;
    }
    return finish(W.z, false, max_iter);
}
}  // namespace dv

// ================================================================== integrator (TRBDF2, core/solver.py:297-511)
namespace dv {

static const double GAMMA_ = 2.0 - 1.4142135623730951;        // 2 - sqrt 2 (np.sqrt(2.0))
static const double D_ = GAMMA_ / 2.0;
static const double C1_ = 1.0 / (GAMMA_ * (2.0 - GAMMA_));
static const double C2_ = (1.0 - GAMMA_) * (1.0 - GAMMA_) / (GAMMA_ * (2.0 - GAMMA_));
static const double W1_ = (3.0 * GAMMA_ - 1.0) / (6.0 * GAMMA_);
static const double W2_ = 1.0 / (6.0 * GAMMA_ * (1.0 - GAMMA_));
static const double W3_ = (2.0 - 3.0 * GAMMA_) / (6.0 * (1.0 - GAMMA_));
static const double G_SD_ = 1.0 - 1.0 / 1.4142135623730951;
static const double SW1_ = (3.0 * G_SD_ - 1.0) / (6.0 * G_SD_);
static const double SW2_ = 1.0 / (6.0 * G_SD_ * (1.0 - G_SD_));
static const double SW3_ = (2.0 - 3.0 * G_SD_) / (6.0 * (1.0 - G_SD_));

// out = y + a * ((z1 - y) / dh)       (SDIRK2 stage-2 right-hand side, core/solver.py:430-431)
__global__ void k_sd_rhs2(int64_t n, const double* __restrict__ y, const double* __restrict__ z1, double dh, double a,
                          double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = y[i] + a * ((z1[i] - y[i]) / dh);
}
// out = truncate(y + (z1 - y)/c, y)    (stage-2 predictor, core/solver.py:432,435)
__global__ void k_pred2(int64_t n, int64_t npos, const double* __restrict__ y, const double* __restrict__ z1, double c,
                        double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = y[i] + (z1[i] - y[i]) / c;
        if (i < npos) v = npmax(v, 0.1 * npmax(y[i], 0.0));
        out[i] = v;
    }
}
// out = (z2 - y) / h
__global__ void k_slope(int64_t n, const double* __restrict__ y, const double* __restrict__ z2, double h,
                        double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (z2[i] - y[i]) / h;
}

// Start of a stage solve: keep cand (the network's guess) when its scaled residual is no larger than
// that of alt (the extrapolation), else overwrite it with alt; count which one was taken.
__global__ void k_pick(int64_t n, const double* __restrict__ r, const double* __restrict__ alt, double* __restrict__ cand,
                       int64_t* __restrict__ cnt) {
    const bool keep = r[0] <= r[1];
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[keep ? 0 : 1] += 1;
    if (keep) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        cand[i] = alt[i];
}

}  // namespace dv

struct dv_integrator {
    dv_model* m;
    dv_solver_opts o;
    int64_t n;
    double *y, *fn, *slope, *z1, *z2, *f1, *f2, *rhs1, *rhs2, *pred, *ev, *es, *d_g;   // device vectors
    double* h_g;                  // pinned: 3 x DV_NACC accumulator rates
    int* h_err;                   // pinned: the model's device error word, read with the error norm
    double acc[DV_NACC], gn[DV_NACC];
    double t, t_end, h, h_cap, h_lu, log_refactor;
    bool have_J, have_lu, fresh, have_slope, started;
    bool j32_fresh;               // the FP32 operator Jacobian was taken at the current state
    int jac_age;
    int64_t gm;                   // GMRES iterations (non-polish) since start
    dv_step_report rep;
    // learned Newton predictor (dv_integrator_set_predictor)
    dv_mlp* mlp;
    int pred_on, rec_stride, step_code;
    double *yprev, *zext;         // state before the last accepted step; the extrapolated guess
    double h_prev;                // size of the last accepted step
    bool have_prev;               // yprev and h_prev hold the step before the current state
    int64_t *d_pick, *h_pick;     // [0] network guess chosen, [1] extrapolation chosen (device; pinned copy)
    int mode;                     // Newton mode: 0 krylov, 1 hybrid, 2 modified (TRBDF2.mode)
};

namespace dv {
// The predictor's inputs for one stage: latest level A (at the stage's start), the one before it B,
// f(A), and the stage's time offsets.
static mlp::StageInputs stage_inputs(const dv_integrator* g, const double* A, const double* B, const double* fA,
                                     double dt_tgt, double dt_ab, double h, int stage) {
    mlp::StageInputs in;
    const dv_model* m = g->m;
    in.Nr = m->p.Nr;
    in.Nth = m->p.Nth;
    in.Nz = m->p.Nz;
    in.nc = m->nc;
    in.A = A;
    in.B = B;
    in.fA = fA;
    in.atol7 = m->d_atol7;
    in.rtol = g->o.rtol;
    in.dt_tgt = dt_tgt;
    in.dt_ab = dt_ab;
    in.h = h;
    in.stage = stage;
    in.step_code = g->step_code;
    return in;
}

// Predicted start of a stage: g->pred holds the extrapolation on entry.  With recording on, the
// features of every rec_stride-th cell are stored (targets follow once the stage converged); with the
// network on, g->pred becomes the network's guess or stays the extrapolation, whichever has the smaller
// scaled stage residual (two residual evaluations, no host synchronisation).  Returns whether the
// extrapolation was saved in g->zext (a fallback exists).
static int predict_stage(dv_integrator* g, const mlp::StageInputs& in, double t, const double* rhs_known, double dh,
                         int64_t first, int64_t cnt, bool* saved, cudaStream_t st) {
    *saved = false;
    if (!g->mlp || (!g->pred_on && g->rec_stride <= 0)) return DV_OK;
    dv_model* m = g->m;
    Work& W = *m->W;
    const int64_t n = g->n;
    const unsigned gr = vgrid(n);
    DV_CUDA(cudaMemcpyAsync(g->zext, g->pred, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    *saved = true;
    if (g->rec_stride > 0) DV_TRY(mlp::record_features(g->mlp, in, first, g->rec_stride, cnt, st));
    if (!g->pred_on) return DV_OK;
    DV_TRY(mlp::predict(g->mlp, in, in.stage == 0 ? in.A : in.B, g->pred, st));
    // each start is judged by its simplified Newton correction ||M^-1 R / s||, the distance to the
    // stage solution that the Newton iteration measures progress by: the raw ||R / s|| is dominated
    // by the stiff pressure couplings, where a state error far below tolerance leaves a large residual
    const double* cands[2] = {g->pred, g->zext};
    for (int q = 0; q < 2; ++q) {
        DV_TRY(launch_stage_residual(m, t, cands[q], dh, rhs_known, W.Rt, st));
        DV_TRY(precond_apply(m, W.Rt, nullptr, W.tmp, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_scale<<<gr, VB, 0, st>>>(m->nc, n, cands[q], m->d_atol7, g->o.rtol, W.w));
        DV_TRY(rms_ratio_dev(W, n, W.tmp, W.w, 0, W.scal + 26 + q, st));
    }
    m->nfev += 2;
    DV_LAUNCH(dv::K_VECTOR, st, k_pick<<<gr, VB, 0, st>>>(n, W.scal + 26, g->zext, g->pred, g->d_pick));
    DV_CUDA(cudaGetLastError());
    return DV_OK;
}

// A bounded device wait that gave up leaves a flag in the model; surface it as an error.
// One implicit stage (TRBDF2._solve_stage, core/solver.py:339-368) from g->pred: modified Newton first
// in the hybrid (at most 4 iterations, rate limit 0.5) and modified (max_newton_iter, 0.9) modes, and
// Newton-Krylov otherwise or when the hybrid attempt fails.  With the learned predictor, a failure
// from the network's start is repeated from the extrapolation (g->zext, saved by predict_stage).
// `no` carries the step's refresh permission (the reference's self._fresh, set before stage 1).
static int solve_stage(dv_integrator* g, const dv_newton_opts& no, double ts, const double* rhs, double dh, bool saved,
                       double* out, bool* ok_out, double* rate_out, cudaStream_t st) {
    dv_model* m = g->m;
    Work& W = *m->W;
    dv_step_report& R = g->rep;
    const int64_t n = g->n, npos = (int64_t)(DV_NG + DV_NA) * m->nc;
    *ok_out = false;
    *rate_out = INFINITY;
    const double* starts[2] = {g->pred, (saved && g->pred_on) ? g->zext : nullptr};
    for (int attempt = 0; attempt < 2 && starts[attempt]; ++attempt) {
        dv_newton_opts o = no;
        if (attempt == 1) {
            R.pred_retry += 1;
            o.allow_refresh = g->fresh ? 0 : 1;
        }
        if (g->mode != 0) {
            bool okm = false;
            int it = 0;
            double rate = 0.0;
            DV_TRY(newton_modified(m, ts, starts[attempt], rhs, dh, g->mode == 2 ? o.max_iter : 4, o.kappa,
                                   g->mode == 2 ? 0.9 : 0.5, o.cons_tol, o.rtol, out, &okm, &it, &rate, st));
            R.newton_iters += it;
            if (okm || g->mode == 2) {
                *ok_out = okm;
                *rate_out = rate;
                if (okm) return DV_OK;
                continue;
            }
            R.modified_fail += 1;
        }
        dv_newton_result r;
        memset(&r, 0, sizeof r);
        NewtonCtx C{m, &W, m->d_atol7, n, npos, o, &r, &g->gm};
        DV_TRY(newton_krylov(C, ts, starts[attempt], rhs, dh, out, st));
        R.n_krylov += 1;
        R.newton_iters += r.iters;
        R.gmres_iters += r.gmres_iters;
        R.gmres_polish += r.gmres_polish;
        R.balance_unclosed += r.balance_unclosed;
        R.balance_projected += r.balance_projected;
        R.jac_refresh_in_newton += r.jac_refresh_in_newton;
        if (r.ok) R.krylov_ok += 1; else R.krylov_fail += 1;
        if (r.refreshed) {                // Jacobian and factors were replaced inside the stage
            R.n_jac += 1;
            R.n_lu += 1;
            g->h_lu = dh / D_;
            g->jac_age = 0;
            g->fresh = true;
        }
        *ok_out = r.ok != 0;
        *rate_out = r.ok ? 0.0 : r.rate;
        if (r.ok) return DV_OK;
    }
    return DV_OK;
}

// After a reported timeout nothing of the abandoned wait is in flight (the caller synchronised):
// clear the error word and the ticket counters the abandoned reduction or barrier left behind, so
// the model's next call starts clean.
static void clear_device_error(dv_model* m) {
    cudaMemset(m->d_err, 0, sizeof(int));
    if (m->W && m->W->tickets) cudaMemset(m->W->tickets, 0, 16 * sizeof(unsigned));
    cudaDeviceSynchronize();
}

static int check_device_error(dv_model* m) {
    int e = 0;
    DV_CUDA(cudaMemcpy(&e, m->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e != 0) {
        set_error(device_error_text(e));
        clear_device_error(m);
        return DV_ERR_CUDA;
    }
    return DV_OK;
}
}  // namespace dv
using namespace dv;

namespace {
// time `reps` back-to-back runs of fn on stream s (CUDA events), microseconds per run
template <class F>
static int time_us(cudaStream_t s, int reps, F&& fn, double* out) {
    cudaEvent_t a, b;
    DV_CUDA(cudaEventCreate(&a));
    DV_CUDA(cudaEventCreate(&b));
    int rc = fn();                                   // warm-up (attributes, graph build)
    if (rc == DV_OK) rc = cudaEventRecord(a, s) == cudaSuccess ? DV_OK : DV_ERR_CUDA;
    for (int r = 0; r < reps && rc == DV_OK; ++r) rc = fn();
    if (rc == DV_OK) rc = cudaEventRecord(b, s) == cudaSuccess ? DV_OK : DV_ERR_CUDA;
    if (rc == DV_OK) rc = cudaEventSynchronize(b) == cudaSuccess ? DV_OK : DV_ERR_CUDA;
    float ms = 0.0f;
    if (rc == DV_OK) cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *out = 1e3 * ms / std::max(reps, 1);
    return rc;
}

}  // namespace

extern "C" {

int dv_abi_version(void) { return DV_ABI_VERSION; }

int dv_selftest_wait_timeout(int32_t polls, int32_t* bits) {
    if (!bits || polls < 1) { set_error("dv_selftest_wait_timeout: null bits or polls < 1"); return DV_ERR_ARG; }
    int* d = nullptr;                          // [0] error word, [1..3] barrier words
    DV_CUDA(cudaMalloc((void**)&d, 4 * sizeof(int)));
    int rc = DV_OK;
    cudaError_t e = cudaMemset(d, 0, 4 * sizeof(int));
    if (e == cudaSuccess) rc = selftest_mbar_timeout(polls, d, 0);
    if (e == cudaSuccess && rc == DV_OK) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2);
        cfg.blockDim = dim3(32);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, k_selftest_grid, (int)polls, (unsigned*)(d + 1), d);
    }
    int h = 0;
    if (e == cudaSuccess && rc == DV_OK) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (rc != DV_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "dv_selftest_wait_timeout");
    *bits = h;
    return DV_OK;
}

int dv_model_set_tuning(dv_model* m, const dv_tuning* t) {
    if (!m || !t || t->gmres_prefix < -1 || t->gmres_prefix > 8 || (t->sweep_nbuf != 0 && t->sweep_nbuf != 2 &&
        t->sweep_nbuf != 3) || (t->spmv_block != 0 && t->spmv_block != 64 && t->spmv_block != 128 &&
        t->spmv_block != 256) || (t->fdjac_block != 0 && t->fdjac_block != 64 && t->fdjac_block != 128) ||
        t->gmres_body < 0 || t->gmres_body > 2) {
        set_error("dv_model_set_tuning: parameter outside its candidates");
        return DV_ERR_ARG;
    }
    m->tune = *t;
    return DV_OK;
}

int dv_model_get_tuning(const dv_model* m, dv_tuning* t) {
    if (!m || !t) { set_error("null argument"); return DV_ERR_ARG; }
    *t = m->tune;
    return DV_OK;
}

int dv_autotune(dv_model* m, double t, const double* y, double dh, int32_t reps, dv_tuning* best, double* times_us,
                int32_t ntimes, void* stream) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    if (!m || !y || !best || reps < 1 || dh <= 0.0) { set_error("dv_autotune: bad argument"); return DV_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    Work& W = *m->W;
    const int64_t n = m->n;
    double tm[DV_TUNE_NTIMES];
    for (double& v : tm) v = 0.0;
    const dv_tuning saved = m->tune;
    dv_tuning tu = m->tune;
    const int mode = m->pc_ready ? m->pc_mode : 2;
    DV_TRY(launch_rhs(m, t, y, W.f, nullptr, st));
    // FD Jacobian block size
    const int fj[2] = {64, 128};
    double bestv = INFINITY;
    for (int q = 0; q < 2; ++q) {
        m->tune.fdjac_block = fj[q];
        DV_TRY(time_us(st, reps, [&] { return launch_fd_jacobian(m, t, y, W.f, W.J, st); }, &tm[q]));
        if (tm[q] < bestv) { bestv = tm[q]; tu.fdjac_block = fj[q]; }
    }
    m->tune.fdjac_block = tu.fdjac_block;
    DV_TRY(precond_factor(m, W.J, dh, mode, st));
    // sweep ring depth (the shared-memory sweep only)
    DV_CUDA(cudaMemcpyAsync(W.b, W.f, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    if (precond_apply_fusable(m)) {
        bestv = INFINITY;
        for (int q = 0; q < 2; ++q) {
            m->tune.sweep_nbuf = 2 + q;
            DV_TRY(time_us(st, reps, [&] { return precond_apply(m, W.b, nullptr, W.x, st); }, &tm[2 + q]));
            if (tm[2 + q] < bestv) { bestv = tm[2 + q]; tu.sweep_nbuf = 2 + q; }
        }
        m->tune.sweep_nbuf = tu.sweep_nbuf;
    }
    // FP32 Jacobian product block size
    DV_TRY(launch_fd_jacobian32(m, t, y, W.f, m->d_J32, st));
    DV_LAUNCH(dv::K_VECTOR, st, k_scale<<<vgrid(n), VB, 0, st>>>(m->nc, n, y, m->d_atol7, 1e-4, W.s));
    const int sb[3] = {64, 128, 256};
    bestv = INFINITY;
    for (int q = 0; q < 3; ++q) {
        m->tune.spmv_block = sb[q];
        DV_TRY(time_us(st, reps, [&] { return launch_spmv32(m, W.b, W.s, dh, nullptr, W.r, st); }, &tm[4 + q]));
        if (tm[4 + q] < bestv) { bestv = tm[4 + q]; tu.spmv_block = sb[q]; }
    }
    m->tune.spmv_block = tu.spmv_block;
    // GMRES prefix: whole stage solves z - dh f(t, z) = y from the explicit Euler guess
    DV_LAUNCH(dv::K_VECTOR, st, k_xpay<<<vgrid(n), VB, 0, st>>>(n, y, dh, W.f, W.zt));
    double* z0 = nullptr;
    double* zo = nullptr;
    DV_CUDA(cudaMalloc((void**)&z0, sizeof(double) * n));
    DV_CUDA(cudaMalloc((void**)&zo, sizeof(double) * n));
    DV_CUDA(cudaMemcpyAsync(z0, W.zt, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    dv_newton_opts no;
    no.max_iter = 7;
    no.krylov_dim = 30;
    no.allow_refresh = 0;
    no.precond_mode = mode;
    no.kappa = 0.01;
    no.eta = 1e-2;
    no.rtol = 1e-4;
    no.cons_tol = 0.0;
    no.max_polish = 2;
    no.polish_cycles = 1;
    no.balance_projection = 0;
    no.pad_ = 0;
    bestv = INFINITY;
    int rc = DV_OK;
    const int64_t nfev0 = m->nfev;
    for (int q = 0; q < 5 && rc == DV_OK; ++q) {
        m->tune.gmres_prefix = 2 * q;
        rc = time_us(st, std::max(1, reps / 10), [&] {
            dv_newton_result r;
            memset(&r, 0, sizeof r);
            NewtonCtx C{m, &W, m->d_atol7, n, (int64_t)(DV_NG + DV_NA) * m->nc, no, &r, nullptr};
            return newton_krylov(C, t + dh, z0, y, dh, zo, st);
        }, &tm[7 + q]);
        if (rc == DV_OK && tm[7 + q] < bestv) { bestv = tm[7 + q]; tu.gmres_prefix = 2 * q; }
    }
    m->tune.gmres_prefix = tu.gmres_prefix;
    bestv = INFINITY;
    for (int q = 0; q < 2 && rc == DV_OK; ++q) {          // steps per WHILE pass, with the chosen prefix
        m->tune.gmres_body = 1 + q;
        rc = time_us(st, std::max(1, reps / 10), [&] {
            dv_newton_result r;
            memset(&r, 0, sizeof r);
            NewtonCtx C{m, &W, m->d_atol7, n, (int64_t)(DV_NG + DV_NA) * m->nc, no, &r, nullptr};
            return newton_krylov(C, t + dh, z0, y, dh, zo, st);
        }, &tm[12 + q]);
        if (rc == DV_OK && tm[12 + q] < bestv) { bestv = tm[12 + q]; tu.gmres_body = 1 + q; }
    }
    m->nfev = nfev0;
    cudaFree(z0);
    cudaFree(zo);
    if (rc != DV_OK) { m->tune = saved; return rc; }
    m->tune = tu;
    *best = tu;
    if (times_us)
        for (int q = 0; q < ntimes && q < DV_TUNE_NTIMES; ++q) times_us[q] = tm[q];
    return check_device_error(m);
}

int dv_model_flag_wait_timeout(dv_model* m, int32_t bits) {
    if (!m || bits <= 0) { set_error("dv_model_flag_wait_timeout: bad argument"); return DV_ERR_ARG; }
    DV_CUDA(cudaMemcpy(m->d_err, &bits, sizeof(int), cudaMemcpyHostToDevice));
    return DV_OK;
}

int dv_profile_enable(int32_t on) {
    cudaDeviceSynchronize();
    prof_flush();
    for (auto& q : g_prof) q = ProfSlot();
    g_prof_on = on != 0;
    return DV_OK;
}

int dv_profile_read(int32_t kind, int64_t* launches, int64_t* timed, double* total_ms) {
    if (kind < 0 || kind >= K_NKIND) { set_error("dv_profile_read: bad kernel kind"); return DV_ERR_ARG; }
    DV_CUDA(cudaDeviceSynchronize());
    prof_flush();
    if (launches) *launches = g_prof[kind].launches;
    if (timed) *timed = g_prof[kind].timed;
    if (total_ms) *total_ms = g_prof[kind].ms;
    return DV_OK;
}

int64_t dv_launch_count(void) { return g_launches.load(); }
size_t dv_step_params_size(void) { return sizeof(dv_step_params); }

int64_t dv_pool_cached_bytes(void) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    return g_pool_cached;
}

int dv_pool_release(void) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    std::lock_guard<std::mutex> lk(g_pool_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : g_pool_free) {
        if (kv.first.dev >= 0) cudaSetDevice(kv.first.dev);
        for (void* q : kv.second) {
            if (kv.first.dev < 0) cudaFreeHost(q);
            else cudaFree(q);
        }
    }
    cudaSetDevice(cur);
    g_pool_free.clear();
    g_pool_cached = 0;
    return launch_ok("dv_pool_release");
}

size_t dv_struct_size(const char* name) {
    if (!name) return 0;
    const std::string n(name);
    if (n == "dv_newton_opts") return sizeof(dv_newton_opts);
    if (n == "dv_newton_result") return sizeof(dv_newton_result);
    if (n == "dv_solver_opts") return sizeof(dv_solver_opts);
    if (n == "dv_step_report") return sizeof(dv_step_report);
    if (n == "dv_tuning") return sizeof(dv_tuning);
    return 0;
}
const char* dv_last_error(void) { return g_err.c_str(); }

int dv_device_count(int* n) {
    if (!n) return DV_ERR_ARG;
    cudaError_t e = cudaGetDeviceCount(n);
    if (e != cudaSuccess) {
        *n = 0;
        cudaGetLastError();
    }
    return DV_OK;
}

int dv_model_set_krylov_fp32(dv_model* m, int32_t mask) {
    if (!m || mask < 0 || mask > 3) { set_error("dv_model_set_krylov_fp32: mask must be 0..3"); return DV_ERR_ARG; }
    const int f = (mask & DV_KRYLOV_FP32_FACTORS) ? 1 : 0;
    if (m->pc_fp32 != f) {
        m->pc_fp32 = f;
        m->pc_ready = 0;                // the next dv_precond_factor builds the copy the sweep reads
    }
    m->op32 = (mask & DV_KRYLOV_FP32_OPERATOR) ? 1 : 0;
    return DV_OK;
}

int dv_model_destroy(dv_model* m) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    if (!m) return DV_OK;
    void* ptrs[] = {m->d_aux, m->d_rec, m->d_split, m->d_diag, m->d_acc, m->d_pc, m->d_pc32, m->d_J32, m->d_pc_work, m->d_pc_piv, m->d_pc_info, m->d_atol7,
                    m->d_err};
    cudaDeviceSynchronize();              // no work in flight still uses the buffers the pool keeps
    for (void* q : ptrs) pool_free(q);
    if (m->W) {
        work_free(*m->W);
        delete m->W;
    }
    delete m;
    return DV_OK;
}

int dv_model_create(const dv_step_params* p, const double* feed_flux, const double* n_nom, const double* coverage,
                    dv_model** out) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    if (!p || !out || !feed_flux || !n_nom || !coverage) { set_error("null argument"); return DV_ERR_ARG; }
    if (p->Nr < 1 || p->Nth < 1 || p->Nz < 1 || p->Nr > DV_MAX_NR || p->Nth == 2) {
        set_error("grid dimensions outside the supported range (1 <= Nr <= 64, Ntheta != 2)");
        return DV_ERR_ARG;
    }
    dv_model* m = new dv_model();
    memset(m, 0, sizeof(dv_model));
    m->p = *p;
    m->nc = (int64_t)p->Nr * p->Nth * p->Nz;
    m->nw = p->wall_on ? (int64_t)p->Nth * p->Nz : 0;
    m->n = DV_NV * m->nc + m->nw;
    m->rl = rec_layout(*p);
    m->jac_doubles = (int64_t)DV_NSLOT * DV_NB * DV_NB * m->nc;
    const int64_t nf = (int64_t)p->Nr * p->Nth, nwall = (int64_t)p->Nth * p->Nz;
    int nb_sector = DV_NV * p->Nr + (p->wall_on ? 1 : 0);
    int nb_full = DV_NV * p->Nr * p->Nth + (p->wall_on ? p->Nth : 0);
    bool full_ok = nb_full <= 512;
    // mode 2 (innermost ring of all sectors as one partition + rings 1.. per sector): Nth + 1 parts
    const int nb_ring = (p->Nr >= 2 && p->Nth >= 2)
                            ? std::max(DV_NV * (p->Nr - 1) + (p->wall_on ? 1 : 0), DV_NV * p->Nth) : 0;
    m->pc_cap_nb = std::max(full_ok ? std::max(nb_full, nb_sector) : nb_sector, nb_ring);
    m->pc_cap_parts = p->Nth + 1;
    int64_t pc_need = std::max(precond_doubles(nb_sector, p->Nth, p->Nz),
                               full_ok ? precond_doubles(nb_full, 1, p->Nz) : (int64_t)0);
    if (nb_ring) pc_need = std::max(pc_need, precond_doubles(nb_ring, p->Nth + 1, p->Nz));
    {   // the split partitions (mode 3) that large cross-sections use instead of mode 2
        int cnb = 0, cparts = 0;
        int64_t cneed = 0, cwork = 0;
        precond_capacity(*p, &cnb, &cparts, &cneed, &cwork);
        m->pc_cap_nb = std::max(m->pc_cap_nb, cnb);
        m->pc_cap_parts = std::max(m->pc_cap_parts, cparts);
        pc_need = std::max(pc_need, cneed);
    }
    int64_t work_need = precond_work_doubles(m->pc_cap_nb, m->pc_cap_parts, p->Nz);
    m->pc_doubles = pc_need;
    const int64_t rec_n = std::max<int64_t>(m->rl.total, m->n);
    bool fail = pool_malloc((void**)&m->d_aux, sizeof(double) * (2 * nf + nwall)) != cudaSuccess ||
                pool_malloc((void**)&m->d_rec, sizeof(double) * rec_n) != cudaSuccess ||
                pool_malloc((void**)&m->d_split, sizeof(double) * split_doubles(*p)) != cudaSuccess ||
                pool_malloc((void**)&m->d_diag, sizeof(double) * m->rl.total) != cudaSuccess ||
                pool_malloc((void**)&m->d_acc, sizeof(double) * DV_NACC) != cudaSuccess ||
                pool_malloc((void**)&m->d_pc, sizeof(double) * pc_need) != cudaSuccess ||
                pool_malloc((void**)&m->d_pc32, sizeof(float) * pc_need) != cudaSuccess ||
                pool_malloc((void**)&m->d_J32, sizeof(float) * m->jac_doubles) != cudaSuccess ||
                pool_malloc((void**)&m->d_pc_work, sizeof(double) * work_need) != cudaSuccess ||
                pool_malloc((void**)&m->d_pc_piv, sizeof(int) * (size_t)m->pc_cap_parts * m->pc_cap_nb) != cudaSuccess ||
                pool_malloc((void**)&m->d_pc_info, sizeof(int) * (size_t)m->pc_cap_parts) != cudaSuccess ||
                pool_malloc((void**)&m->d_atol7, sizeof(double) * DV_NB) != cudaSuccess ||
                pool_malloc((void**)&m->d_err, sizeof(int)) != cudaSuccess;
    if (fail) {
        int rc = cuda_fail(cudaGetLastError(), "cudaMalloc(model workspace)");
        dv_model_destroy(m);
        return rc;
    }
    debug_fill(m->d_rec, sizeof(double) * rec_n, 1);
    debug_fill(m->d_split, sizeof(double) * split_doubles(*p), 1);
    debug_fill(m->d_diag, sizeof(double) * m->rl.total, 1);
    debug_fill(m->d_acc, sizeof(double) * DV_NACC, 1);
    debug_fill(m->d_pc, sizeof(double) * pc_need, 1);
    debug_fill(m->d_pc32, sizeof(float) * pc_need, 1);
    debug_fill(m->d_J32, sizeof(float) * m->jac_doubles, 1);
    debug_fill(m->d_pc_work, sizeof(double) * work_need, 1);
    debug_fill(m->d_pc_piv, sizeof(int) * (size_t)m->pc_cap_parts * m->pc_cap_nb, 1);
    debug_fill(m->d_pc_info, sizeof(int) * (size_t)m->pc_cap_parts, 1);
    m->W = new Work();
    int rc = work_alloc(*m->W, m->n, 30, m->jac_doubles);
    if (rc != DV_OK) {
        dv_model_destroy(m);
        return rc;
    }
    cudaMemcpy(m->d_aux, feed_flux, sizeof(double) * nf, cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_aux + nf, n_nom, sizeof(double) * nf, cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_aux + 2 * nf, coverage, sizeof(double) * nwall, cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_atol7, p->atol, sizeof(double) * DV_NB, cudaMemcpyHostToDevice);
    m->aux.feed_flux = m->d_aux;
    m->aux.n_nom = m->d_aux + nf;
    m->aux.cov = m->d_aux + 2 * nf;
    cudaMemset(m->d_rec, 0, sizeof(double) * rec_n);
    cudaMemset(m->d_err, 0, sizeof(int));
    int32_t ncol = 0;
    std::vector<int64_t> colour((size_t)m->n);
    rc = dv_colour_columns(p->Nr, p->Nth, p->Nz, p->wall_on, colour.data(), &ncol);
    if (rc != DV_OK) {
        dv_model_destroy(m);
        return rc;
    }
    m->ncolours = ncol;
    m->tune.gmres_prefix = -1;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        dv_model_destroy(m);
        return cuda_fail(e, "dv_model_create");
    }
    *out = m;
    return DV_OK;
}

int dv_model_sizes(const dv_model* m, int64_t* n_core, int64_t* ncell, int64_t* n_wall, int64_t* jac_doubles,
                   int64_t* diag_doubles) {
    if (!m) return DV_ERR_ARG;
    if (n_core) *n_core = m->n;
    if (ncell) *ncell = m->nc;
    if (n_wall) *n_wall = m->nw;
    if (jac_doubles) *jac_doubles = m->jac_doubles;
    if (diag_doubles) *diag_doubles = m->rl.total;
    return DV_OK;
}

int64_t dv_model_nfev(const dv_model* m) { return m ? m->nfev : -1; }

int dv_rhs(dv_model* m, double t, const double* y, double* f, double* acc, void* stream) {
    if (!m || !y || !f) { set_error("null argument"); return DV_ERR_ARG; }
    return launch_rhs(m, t, y, f, acc, (cudaStream_t)stream);
}

int dv_stage_residual(dv_model* m, double t, const double* y, double gamma_h, const double* rhs_known, double* R,
                      void* stream) {
    if (!m || !y || !rhs_known || !R) { set_error("null argument"); return DV_ERR_ARG; }
    return launch_stage_residual(m, t, y, gamma_h, rhs_known, R, (cudaStream_t)stream);
}

int dv_rhs_diag(dv_model* m, double t, const double* y, double* diag, void* stream) {
    if (!m || !y || !diag) { set_error("null argument"); return DV_ERR_ARG; }
    return launch_diag(m, t, y, diag, (cudaStream_t)stream);
}

int dv_outlet_row(dv_model* m, double t, const double* y, double c_feed_co2, double* row, void* stream) {
    if (!m || !y || !row) { set_error("null argument"); return DV_ERR_ARG; }
    return launch_outlet(m, t, y, c_feed_co2, row, (cudaStream_t)stream);
}

int dv_fd_jacobian(dv_model* m, double t, const double* y, const double* f0, double* J, void* stream) {
    if (!m || !y || !f0 || !J) { set_error("null argument"); return DV_ERR_ARG; }
    m->nfev += m->ncolours;
    return launch_fd_jacobian(m, t, y, f0, J, (cudaStream_t)stream);
}

int dv_precond_factor(dv_model* m, const double* J, double dh, int32_t mode, void* stream) {
    if (!m || !J) { set_error("null argument"); return DV_ERR_ARG; }
    return precond_factor(m, J, dh, mode, (cudaStream_t)stream);
}

int dv_precond_partitions(const dv_model* m, int32_t* mode, int32_t* zs, int32_t* nb, int32_t cap, int32_t* nparts) {
    if (!m || !mode || !zs || !nparts || (cap > 0 && !nb)) { set_error("null argument"); return DV_ERR_ARG; }
    int md = -1, z = 0;
    std::vector<int> tmp(std::max(cap, 0));
    *nparts = precond_partitions(m, &md, &z, tmp.data(), cap);
    *mode = md;
    *zs = z;
    for (int q = 0; q < cap && q < *nparts; ++q) nb[q] = tmp[q];
    return DV_OK;
}

int dv_precond_check_maps(const dv_step_params* p, int32_t mode, int32_t* nparts, int32_t* nb, int64_t* violations) {
    if (!p || !nparts || !nb || !violations) { set_error("null argument"); return DV_ERR_ARG; }
    int np = 0, b = 0;
    *violations = precond_check_maps(*p, mode, &np, &b);
    *nparts = np;
    *nb = b;
    return DV_OK;
}

int dv_precond_solve(dv_model* m, const double* b, double* x, void* stream) {
    if (!m || !b || !x) { set_error("null argument"); return DV_ERR_ARG; }
    return precond_apply(m, b, nullptr, x, (cudaStream_t)stream);
}

int dv_newton_stage(dv_model* m, double t, const double* z0, const double* rhs_known, double dh, const dv_newton_opts* o,
                    double* z_out, dv_newton_result* r, void* stream) {
    if (!m || !z0 || !rhs_known || !o || !z_out || !r) { set_error("null argument"); return DV_ERR_ARG; }
    if (!m->pc_ready) { set_error("dv_newton_stage needs a factorised preconditioner"); return DV_ERR_ARG; }
    if (o->krylov_dim < 1 || o->krylov_dim > m->W->kdim) { set_error("krylov_dim outside 1..30"); return DV_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    memset(r, 0, sizeof(*r));
    NewtonCtx C{m, m->W, m->d_atol7, m->n, DV_NG * m->nc + DV_NA * m->nc, *o, r, nullptr};
    if (m->op32) {                     // FP32 operator Jacobian at z0
        Work& W = *m->W;
        DV_TRY(launch_rhs(m, t, z0, W.tmp, nullptr, st));
        DV_TRY(launch_fd_jacobian32(m, t, z0, W.tmp, m->d_J32, st));
        m->nfev += 1 + m->ncolours;
    }
    int rc = newton_krylov(C, t, z0, rhs_known, dh, z_out, st);
    cudaStreamSynchronize(st);
    if (rc == DV_OK) rc = check_device_error(m);
    return rc;
}

// ------------------------------------------------------------------ integrator
int dv_integrator_destroy(dv_integrator* g) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    if (!g) return DV_OK;
    double* ptrs[] = {g->y, g->fn, g->slope, g->z1, g->z2, g->f1, g->f2, g->rhs1, g->rhs2, g->pred, g->ev, g->es, g->d_g,
                      g->yprev, g->zext};
    cudaDeviceSynchronize();              // no work in flight still uses the buffers the pool keeps
    for (double* q : ptrs) pool_free(q);
    pool_free(g->d_pick);
    pool_free_host(g->h_pick);
    pool_free_host(g->h_g);
    pool_free_host(g->h_err);
    delete g;
    return DV_OK;
}

int dv_integrator_create(dv_model* m, const dv_solver_opts* o, dv_integrator** out) {
    std::lock_guard<std::recursive_mutex> lk_(capture_mutex());
    if (!m || !o || !out) { set_error("null argument"); return DV_ERR_ARG; }
    if (o->scheme != 0 && o->scheme != 1) { set_error("scheme must be 0 (sdirk2) or 1 (trbdf2)"); return DV_ERR_ARG; }
    dv_integrator* g = new dv_integrator();
    memset(g, 0, sizeof(dv_integrator));
    g->m = m;
    g->o = *o;
    g->n = m->n;
    g->log_refactor = std::log(o->refactor_ratio);
    if (o->newton_mode < 0 || o->newton_mode > 2) {
        delete g;
        set_error("newton_mode must be 0 (krylov), 1 (hybrid) or 2 (modified)");
        return DV_ERR_ARG;
    }
    // modified Newton needs exact factors; with partitioned (approximate) ones it keeps the Krylov
    // fallback (core/solver.py:328-329)
    g->mode = (o->newton_mode == 2 && o->precond_mode != 1) ? 1 : o->newton_mode;
    m->op32 = (o->krylov_fp32 & DV_KRYLOV_FP32_OPERATOR) ? 1 : 0;
    if (m->pc_fp32 != ((o->krylov_fp32 & DV_KRYLOV_FP32_FACTORS) ? 1 : 0)) {   // factors rebuilt in the requested storage
        m->pc_fp32 = (o->krylov_fp32 & DV_KRYLOV_FP32_FACTORS) ? 1 : 0;
        m->pc_ready = 0;
    }
    double** vecs[] = {&g->y, &g->fn, &g->slope, &g->z1, &g->z2, &g->f1, &g->f2, &g->rhs1, &g->rhs2, &g->pred, &g->ev, &g->es};
    for (double** v : vecs) {
        if (pool_malloc((void**)v, sizeof(double) * g->n) != cudaSuccess) {
            int rc = cuda_fail(cudaGetLastError(), "cudaMalloc(integrator)");
            dv_integrator_destroy(g);
            return rc;
        }
    }
    if (pool_malloc((void**)&g->d_g, sizeof(double) * 3 * DV_NACC) != cudaSuccess ||
        pool_malloc_host((void**)&g->h_g, sizeof(double) * 3 * DV_NACC) != cudaSuccess ||
        pool_malloc_host((void**)&g->h_err, sizeof(int)) != cudaSuccess) {
        int rc = cuda_fail(cudaGetLastError(), "cudaMalloc(integrator)");
        dv_integrator_destroy(g);
        return rc;
    }
    for (double** v : vecs) debug_fill(*v, sizeof(double) * g->n, 4);
    debug_fill(g->d_g, sizeof(double) * 3 * DV_NACC, 4);
    debug_fill(g->h_g, sizeof(double) * 3 * DV_NACC, 8, true);
    debug_fill(g->h_err, sizeof(int), 8, true);
    *out = g;
    return DV_OK;
}

int dv_integrator_start(dv_integrator* g, const double* y0, double t_end, void* stream) {
    if (!g || !y0) { set_error("null argument"); return DV_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    g->t = 0.0;
    g->t_end = t_end;
    DV_CUDA(cudaMemcpyAsync(g->y, y0, sizeof(double) * g->n, cudaMemcpyDefault, st));
    DV_TRY(launch_rhs(g->m, 0.0, g->y, g->fn, g->d_g, st));
    DV_CUDA(cudaMemcpyAsync(g->h_g, g->d_g, sizeof(double) * DV_NACC, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    memcpy(g->gn, g->h_g, sizeof(double) * DV_NACC);
    memset(g->acc, 0, sizeof(g->acc));
    g->h = std::min(std::min(g->o.h_init, g->o.h_max), t_end);
    g->have_J = g->have_lu = g->fresh = g->have_slope = false;
    g->have_prev = false;
    g->j32_fresh = false;
    if (g->d_pick) DV_CUDA(cudaMemsetAsync(g->d_pick, 0, 2 * sizeof(int64_t), st));
    g->jac_age = 0;
    g->h_cap = INFINITY;
    g->h_lu = 0.0;
    g->gm = 0;
    memset(&g->rep, 0, sizeof(g->rep));
    g->rep.nfev = g->m->nfev;
    g->started = true;
    return DV_OK;
}

const double* dv_integrator_y(const dv_integrator* g) { return g ? g->y : nullptr; }

int dv_integrator_copy_y(const dv_integrator* g, double* dst, void* stream) {
    if (!g || !dst) { set_error("null argument"); return DV_ERR_ARG; }
    DV_CUDA(cudaMemcpyAsync(dst, g->y, sizeof(double) * g->n, cudaMemcpyDefault, (cudaStream_t)stream));
    DV_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return DV_OK;
}

int dv_integrator_set_predictor(dv_integrator* g, dv_mlp* net, int32_t predict, int32_t record_stride,
                                int32_t step_code) {
    if (!g || record_stride < 0 || step_code < 0 || step_code > 3) {
        set_error("dv_integrator_set_predictor: bad argument");
        return DV_ERR_ARG;
    }
    if (!net) {
        g->mlp = nullptr;
        g->pred_on = 0;
        g->rec_stride = 0;
        return DV_OK;
    }
    DV_TRY(dv_mlp_reserve(net, g->m->nc));
    if (!g->yprev) {
        if (pool_malloc((void**)&g->yprev, sizeof(double) * g->n) != cudaSuccess ||
            pool_malloc((void**)&g->zext, sizeof(double) * g->n) != cudaSuccess ||
            pool_malloc((void**)&g->d_pick, 2 * sizeof(int64_t)) != cudaSuccess ||
            pool_malloc_host((void**)&g->h_pick, 2 * sizeof(int64_t)) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "cudaMalloc(predictor)");
        DV_CUDA(cudaMemset(g->d_pick, 0, 2 * sizeof(int64_t)));
        g->h_pick[0] = g->h_pick[1] = 0;
        g->have_prev = false;
    }
    g->mlp = net;
    g->pred_on = predict ? 1 : 0;
    g->rec_stride = record_stride;
    g->step_code = step_code;
    return DV_OK;
}

int dv_integrator_advance(dv_integrator* g, double t_target, dv_step_report* rep, void* stream) {
    if (!g || !rep) { set_error("null argument"); return DV_ERR_ARG; }
    if (!g->started) { set_error("dv_integrator_advance before dv_integrator_start"); return DV_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    dv_model* m = g->m;
    Work& W = *m->W;
    const int64_t n = g->n;
    const unsigned gr = vgrid(n);
    const int64_t npos = (int64_t)(DV_NG + DV_NA) * m->nc;
    const bool sd = g->o.scheme == 0;
    const double c_mid = sd ? G_SD_ : GAMMA_;
    dv_step_report& R = g->rep;
    const int64_t nfev0 = m->nfev;
    const int64_t nfev_base = R.nfev;
    auto sync_nfev = [&]() { R.nfev = nfev_base + (m->nfev - nfev0); };
    dv_newton_opts no;
    no.max_iter = g->o.max_newton_iter;
    no.krylov_dim = 30;
    no.precond_mode = g->o.precond_mode;
    no.kappa = g->o.newton_kappa;
    no.eta = 1e-2;
    no.rtol = g->o.rtol;
    no.cons_tol = g->o.conservation_tol;
    no.max_polish = g->o.max_polish;
    no.polish_cycles = g->o.polish_cycles;
    no.balance_projection = g->o.balance_projection;
    no.pad_ = 0;
    while (g->t < g->t_end * (1.0 - 1e-12)) {
        const int64_t gm0 = g->gm;
        if (R.n_steps + R.n_reject + R.n_newton_fail > g->o.max_steps) {
            sync_nfev();
            *rep = R;
            char buf[160];
            snprintf(buf, sizeof buf, "too many steps at t=%.4gs", g->t);
            set_error(buf);
            return DV_ERR_STEPS;
        }
        const double h_desired = g->h;
        double h = std::min(std::min(g->h, g->o.h_max), t_target - g->t);
        const bool truncated = h < h_desired * (1.0 - 1e-9);
        if (h < 1e-10 * std::max(1.0, g->t_end)) {
            sync_nfev();
            *rep = R;
            char buf[160];
            snprintf(buf, sizeof buf, "step size underflow (h=%.3e) at t=%.6gs", h, g->t);
            set_error(buf);
            return DV_ERR_UNDERFLOW;
        }
        g->h = h;
        if (!g->have_J || g->jac_age >= g->o.jacobian_max_age) {
            DV_TRY(launch_fd_jacobian(m, g->t, g->y, g->fn, W.J, st));
            m->nfev += m->ncolours;
            R.n_jac += 1;
            g->have_J = true;
            g->jac_age = 0;
            g->fresh = true;
            g->have_lu = false;
        }
        if (!g->have_lu || std::fabs(std::log(h / g->h_lu)) > (g->mode == 2 ? 0.35 : g->log_refactor)) {
            DV_TRY(precond_factor(m, W.J, D_ * h, g->o.precond_mode, st));
            g->h_lu = h;
            R.n_lu += 1;
            g->have_lu = true;
        }
        const double dh = D_ * h;
        if (m->op32 && !g->j32_fresh) {    // FP32 operator Jacobian at the step's start state
            DV_TRY(launch_fd_jacobian32(m, g->t, g->y, g->fn, m->d_J32, st));
            m->nfev += m->ncolours;
            g->j32_fresh = true;
        }
        // ---- stage 1
        if (sd) {
            DV_CUDA(cudaMemcpyAsync(g->rhs1, g->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        } else {
            DV_LAUNCH(dv::K_VECTOR, st, k_xpay<<<gr, VB, 0, st>>>(n, g->y, dh, g->fn, g->rhs1));
        }
        if (g->have_slope) {
            DV_LAUNCH(dv::K_VECTOR, st, k_xpay<<<gr, VB, 0, st>>>(n, g->y, c_mid * h, g->slope, g->pred));
            DV_LAUNCH(dv::K_VECTOR, st, k_truncate_to<<<gr, VB, 0, st>>>(n, npos, g->pred, g->y, g->pred));
        } else {
            DV_CUDA(cudaMemcpyAsync(g->pred, g->y, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        // learned predictor (off unless dv_integrator_set_predictor attached a network)
        const bool use_net = g->mlp && g->have_prev;
        const int64_t stride = g->rec_stride > 0 ? g->rec_stride : 1;
        mlp::StageInputs in1{};
        bool saved1 = false;
        const int64_t first1 = (R.n_steps * 2 + R.n_reject * 5 + R.n_newton_fail * 3) % stride;
        const int64_t cnt1 = (m->nc - first1 + stride - 1) / stride;
        if (use_net) {
            in1 = stage_inputs(g, g->y, g->yprev, g->fn, c_mid * h, g->h_prev, h, 0);
            DV_TRY(predict_stage(g, in1, g->t + c_mid * h, g->rhs1, dh, first1, cnt1, &saved1, st));
        }
        no.allow_refresh = g->fresh ? 0 : 1;          // self._fresh = fresh (set before stage 1)
        bool ok = false;
        double r1 = 0.0, r2 = 0.0;
        DV_TRY(solve_stage(g, no, g->t + c_mid * h, g->rhs1, dh, saved1, g->z1, &ok, &r1, st));
        if (ok && saved1 && g->rec_stride > 0)
            DV_TRY(mlp::record_targets(g->mlp, in1, g->z1, g->zext, first1, g->rec_stride, cnt1, st));
        if (ok) {
            if (sd) {
                DV_LAUNCH(dv::K_VECTOR, st, k_sd_rhs2<<<gr, VB, 0, st>>>(n, g->y, g->z1, dh, (1.0 - G_SD_) * h, g->rhs2));
            } else {
                DV_LAUNCH(dv::K_VECTOR, st, k_axpby<<<gr, VB, 0, st>>>(n, C1_, g->z1, -C2_, g->y, g->rhs2));
            }
            DV_LAUNCH(dv::K_VECTOR, st, k_pred2<<<gr, VB, 0, st>>>(n, npos, g->y, g->z1, c_mid, g->pred));
            mlp::StageInputs in2{};
            bool saved2 = false;
            const int64_t first2 = (first1 + 1) % stride;
            const int64_t cnt2 = (m->nc - first2 + stride - 1) / stride;
            if (g->mlp) {      // levels z1 (with f(z1) from stage 1's last Newton iterate) and y
                in2 = stage_inputs(g, g->z1, g->y, W.f, (1.0 - c_mid) * h, c_mid * h, h, 1);
                DV_TRY(predict_stage(g, in2, g->t + h, g->rhs2, dh, first2, cnt2, &saved2, st));
            }
            DV_TRY(solve_stage(g, no, g->t + h, g->rhs2, dh, saved2, g->z2, &ok, &r2, st));
            if (ok && saved2 && g->rec_stride > 0)
                DV_TRY(mlp::record_targets(g->mlp, in2, g->z2, g->zext, first2, g->rec_stride, cnt2, st));
        }
        if (!ok) {
            R.n_newton_fail += 1;
            if (!g->fresh) {
                g->have_J = false;
            } else {
                g->h_cap = std::min(g->h_cap, 0.5 * h);
                g->h = h * 0.3;
                g->have_lu = false;
            }
            continue;
        }
        // ---- error estimate filtered by M^-1 (core/solver.py:454-469)
        DV_TRY(launch_rhs(m, g->t + c_mid * h, g->z1, g->f1, g->d_g + DV_NACC, st));
        DV_TRY(launch_rhs(m, g->t + h, g->z2, g->f2, g->d_g + 2 * DV_NACC, st));
        if (sd) {
            DV_LAUNCH(dv::K_VECTOR, st, k_err_vec<<<gr, VB, 0, st>>>(n, g->y, g->z2, h, SW1_, g->fn, SW2_, g->f1, SW3_, g->f2, g->ev));
        } else {
            DV_LAUNCH(dv::K_VECTOR, st, k_err_vec<<<gr, VB, 0, st>>>(n, g->y, g->z2, h, W1_, g->fn, W2_, g->f1, W3_, g->f2, g->ev));
        }
        DV_TRY(precond_apply(m, g->ev, nullptr, g->ev, st));
        DV_LAUNCH(dv::K_VECTOR, st, k_err_scale<<<gr, VB, 0, st>>>(m->nc, n, g->y, g->z2, m->d_atol7, g->o.rtol, g->es));
        // the accumulator rates of both stages and the device error word come back with the error
        // norm (one synchronisation)
        DV_CUDA(cudaMemcpyAsync(g->h_g + DV_NACC, g->d_g + DV_NACC, sizeof(double) * 2 * DV_NACC,
                                cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaMemcpyAsync(g->h_err, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        double en;
        DV_TRY(rms_ratio(W, n, g->ev, g->es, &en, st));
        if (!std::isfinite(en)) en = 1e6;
        R.err_norm = en;
        if (en > 1.0) {
            R.n_reject += 1;
            g->h = h * std::max(0.2, 0.9 * std::pow(en, -1.0 / 3.0));
            continue;
        }
        // ---- accept
        const double* g1 = g->h_g + DV_NACC;
        const double* g2 = g->h_g + 2 * DV_NACC;
        for (int q = 0; q < DV_NACC; ++q) {
            if (sd) {
                g->acc[q] = g->acc[q] + h * ((1.0 - G_SD_) * g1[q] + G_SD_ * g2[q]);
            } else {
                double acc_g = g->acc[q] + D_ * h * (g->gn[q] + g1[q]);
                g->acc[q] = C1_ * acc_g - C2_ * g->acc[q] + D_ * h * g2[q];
            }
        }
        DV_LAUNCH(dv::K_VECTOR, st, k_slope<<<gr, VB, 0, st>>>(n, g->y, g->z2, h, g->slope));
        g->have_slope = true;
        if (g->yprev) {            // keep the state before this step for the predictor's second level
            double* old_prev = g->yprev;
            g->yprev = g->y;
            g->y = g->z2;
            g->z2 = old_prev;
            g->have_prev = true;
            g->h_prev = h;
        } else {
            std::swap(g->y, g->z2);
        }
        std::swap(g->fn, g->f2);
        memcpy(g->gn, g2, sizeof(double) * DV_NACC);
        g->t = g->t + h;
        R.n_steps += 1;
        g->j32_fresh = false;
        g->jac_age += 1;
        g->fresh = false;
        if ((g->mode == 2 && std::max(r1, r2) > 0.5) || g->gm - gm0 > g->o.gmres_refresh)
            g->jac_age = g->o.jacobian_max_age;       // stale Jacobian / factors: refresh next step
        double fac = (en < 1e-8) ? 4.0 : std::min(4.0, std::max(0.2, 0.9 * std::pow(en, -1.0 / 3.0)));
        if (1.0 <= fac && fac < 1.25) fac = 1.0;
        double hn = truncated ? std::max(h * fac, h_desired) : h * fac;
        g->h_cap *= 1.15;
        g->h = std::min(hn, g->h_cap);
        R.t = g->t;
        R.h_used = h;
        memcpy(R.acc, g->acc, sizeof(g->acc));
        sync_nfev();
        if (g->d_pick) DV_CUDA(cudaMemcpyAsync(g->h_pick, g->d_pick, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
        if (g->d_pick) {
            R.pred_net = g->h_pick[0];
            R.pred_extrap = g->h_pick[1];
        }
        *rep = R;
        if (*g->h_err != 0) {                 // (read with the error norm; the rest of the step has no wait)
            set_error(device_error_text(*g->h_err));
            *g->h_err = 0;
            clear_device_error(m);
            return DV_ERR_CUDA;
        }
        return DV_OK;
    }
    R.t = g->t;
    sync_nfev();
    *rep = R;
    return DV_OK;
}

}  // extern "C"
