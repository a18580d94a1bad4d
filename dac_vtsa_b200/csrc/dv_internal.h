// dv_internal.h -- model handle and launchers shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include <string>
#include "dacvtsa.h"

namespace dv {

void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
// DV_OK after a successful launch, else the launch error as DV_ERR_CUDA.
inline int launch_ok(const char* what) {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DV_OK : cuda_fail(e, what);
}

// Dynamic shared memory above 48 KB for kernel `func`: its attribute is raised once per device, to
// the most the kernel can take, under a lock.  Models of different sizes launch the same kernel with
// different amounts from several host threads (an ensemble); setting the attribute to each launch's
// own amount would let one thread lower it under another's launch.
cudaError_t allow_dyn_smem(const void* func);

// Held while a GMRES graph is captured and while handles are created or destroyed (device memory
// allocated or freed, device-wide synchronisations): models driven from several host threads then
// never allocate, free or synchronise the device in the middle of another thread's stream capture.
std::recursive_mutex& capture_mutex();

// Buffer pool of the handles' device and pinned host memory: a destroyed handle's buffers are kept
// per (device, size) and handed to the next handle that asks for the same size, so the reference's
// pattern of one model and one integrator per cycle step allocates once per shape instead of every
// step.  pool_free / pool_free_host take only memory from pool_malloc / pool_malloc_host; the
// caller makes sure no work in flight still uses it (handle destruction synchronises the device).
cudaError_t pool_malloc(void** p, size_t bytes);
cudaError_t pool_malloc_host(void** p, size_t bytes);
void pool_free(void* p);
void pool_free_host(void* p);

// Launch accounting: every kernel launch of the library goes through DV_LAUNCH, which counts it per
// kind and, when profiling is on (dv_profile_enable), brackets it with CUDA events on its stream.
enum KernelKind { K_RESIDUAL = 0, K_MATVEC = 1, K_FDJAC = 2, K_PC_FACTOR = 3, K_PC_APPLY = 4, K_VECTOR = 5,
                  K_MLP = 6, K_SPMV = 7, K_NKIND = 8 };
void prof_begin(int kind, cudaStream_t s);
void prof_end(int kind, cudaStream_t s);
void prof_flush();
// Count one launch of `kind` without the profiler's events (for code that must not create any).
void count_launch(int kind);
void count_launches(int kind, int64_t n);
#define DV_LAUNCH(kind, stream, ...)      \
    do {                                  \
        dv::prof_begin(kind, stream);     \
        __VA_ARGS__;                      \
        dv::prof_end(kind, stream);       \
    } while (0)

#ifndef DV_TRY
#define DV_TRY(x)                     \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != DV_OK) return rc_; \
    } while (0)
#endif

#define DV_CUDA(call)                                      \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return dv::cuda_fail(e_, #call); \
    } while (0)

struct Work {
    int64_t n = 0;
    int kdim = 0;
    double *V = nullptr, *w = nullptr, *u = nullptr, *x = nullptr, *r = nullptr, *b = nullptr, *s = nullptr;
    double *z = nullptr, *f = nullptr, *R = nullptr, *dz = nullptr, *zt = nullptr, *ft = nullptr, *Rt = nullptr;
    double *tmp = nullptr, *best = nullptr;
    double *part = nullptr, *scal = nullptr, *hbuf = nullptr, *ybuf = nullptr;
    double* hpin = nullptr;       // pinned host mirror of small results
    double* J = nullptr;          // Jacobian storage used by in-stage refreshes
    int nparts = 0;
    // device-driven GMRES: one CUDA graph per workspace (built at first use), its device state
    double *vin = nullptr, *wout = nullptr;   // normalised basis vector in / operator output
    unsigned* tickets = nullptr;              // ticket counters of the fused reductions (zeroed)
    double* apart = nullptr;                  // per-CTA partials of the fused sweep's reduction
    void* gm = nullptr;                       // device GMRES state
    void* gm_host = nullptr;                  // pinned host mirror of it
    cudaGraph_t gm_graph = nullptr;
    cudaGraphExec_t gm_exec = nullptr;
    cudaStream_t gm_cs = nullptr;             // capture stream
    int gm_kdim = 0, gm_mode = -1, gm_nb = 0, gm_nparts = 0, gm_fp32 = -1, gm_zs = -1, gm_op32 = -1, gm_tuned = -2;
    int gm_prefix = 0;                        // Arnoldi steps captured ahead of the WHILE node
    int gm_body = 1;                          // Arnoldi steps per pass through the WHILE body
    int64_t gm_fixed[K_NKIND] = {}, gm_iter[K_NKIND] = {};   // launches per graph run: fixed + per iteration
};
int work_alloc(Work& W, int64_t n, int kdim, int64_t jac_doubles);

#ifdef __CUDACC__
// Programmatic dependent launch (sm_90+): a kernel launched with programmatic stream serialisation
// may start while its predecessor in the stream is still running; pdl_wait() blocks until that
// predecessor has completed and its writes are visible, so it comes before the kernel's first read
// of anything its predecessors wrote.  pdl_trigger() lets this kernel's own programmatic dependent
// be scheduled now (its blocks then wait in pdl_wait()).  Both return at once in a kernel launched
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Grid-wide barrier of a cooperative launch: one thread per block arrives on *cnt, the last one
// resets it and advances *gen; the others poll *gen at most `limit` times and then set bit 4 of
// *err and go on (the host reports the error; no thread waits forever).
__device__ __forceinline__ void grid_sync_bounded(unsigned* cnt, unsigned* gen, int* err, int limit = 1 << 24) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vg = gen;
        const unsigned g0 = *vg;
        __threadfence();
        if (atomicAdd(cnt, 1u) == gridDim.x - 1) {
            *cnt = 0u;
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            for (int it = 0; *vg == g0; ++it) {
                if (it > limit) {
                    atomicOr(err, 4);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}
// sum of p[b * stride], b < nb, in index order: the deterministic finish of per-block partials
// written by other SMs (volatile loads: never served from this SM's L1)
__device__ __forceinline__ double sum_partials(const double* p, int nb, int64_t stride) {
    double t = 0.0;
    for (int b = 0; b < nb; ++b) t += ((volatile const double*)p)[(int64_t)b * stride];
    return t;
}
#endif
void work_free(Work& W);

struct DevAux {
    const double* feed_flux;
    const double* n_nom;
    const double* cov;
};

// Diagnostics / record layout offsets (doubles) within one record buffer.
struct RecLayout {
    int64_t T, P, y, qstar, uz, ur, uth, bnd, Qj, Qa, Qw, Rb, Qhx, total;
};
RecLayout rec_layout(const dv_step_params& p);
// Doubles of the split residual's scratch (per-cell properties + per-face fluxes).
int64_t split_doubles(const dv_step_params& p);

}  // namespace dv

struct dv_model {
    dv_step_params p;
    int64_t nc, nw, n;              // cells, wall unknowns, n_core
    double* d_aux;                  // feed_flux | n_nom | cov
    dv::DevAux aux;
    dv::RecLayout rl;
    double* d_rec;                  // internal record scratch (accumulators)
    double* d_split;                // per-cell properties and per-face fluxes of the split residual
    double* d_diag;                 // diagnostics record of the outlet summary (dv_outlet_row)
    double* d_acc;                  // DV_NACC
    int64_t nfev;
    int64_t jac_doubles;
    // preconditioner: block-pentadiagonal LU along z per partition
    int pc_mode, pc_nparts, pc_nb, pc_ready;
    int pc_zs;                      // twisted factorisation: first separator plane (0: top-down only)
    int pc_fp32;                    // sweep reads an FP32 copy of the factors (mixed-precision Krylov)
    float* d_pc32;                  // that copy, same layout as d_pc
    int op32;                       // GMRES operator = FP32 assembled Jacobian d_J32 (mixed-precision Krylov)
    float* d_J32;                   // [DV_NSLOT][DV_NB][DV_NB][ncell] (allocated on first use)
    int pc_cap_nb, pc_cap_parts;
    double* d_pc;                   // [parts][Nz][5][nb*nb]
    int64_t pc_doubles;             // entries allocated for d_pc (and d_pc32)
    double* d_pc_work;              // [parts][2][nb*nb] factorisation scratch
    int* d_pc_piv;                  // [parts][nb] pivot work
    int* d_pc_info;                 // [parts] singular-pivot flags
    int* d_err;                     // device error word (bounded waits that gave up)
    dv::Work* W;                    // Krylov / Newton workspace (allocated at creation)
    double* d_atol7;                // per-block absolute tolerances (device)
    int ncolours;                   // colours of the Jacobian pattern (counts RHS-equivalents)
    dv_tuning tune;                 // launch parameters (dv_model_set_tuning / dv_autotune)
};

namespace dv {
// residual family (dv_kernels.cu, -fmad=false)
int launch_rhs(dv_model* m, double t, const double* y, double* f, double* acc, cudaStream_t s);
int launch_stage_residual(dv_model* m, double t, const double* y, double gamma_h, const double* rhs_known,
                          double* R, cudaStream_t s);
int launch_diag(dv_model* m, double t, const double* y, double* diag, cudaStream_t s);
// Outlet summary of state y into row (DV_OUTLET_N doubles, device), via the diagnostics in m->d_diag.
int launch_outlet(dv_model* m, double t, const double* y, double c_feed, double* row, cudaStream_t s);
// out = (v - dh (f(z + sig v) - f0)/sig)/s with v = u*s, sig = SQRT_EPS*scal[1]/scal[0] (scal on device)
int launch_matvec(dv_model* m, double t, const double* z, const double* u, const double* sc, const double* f0,
                  double dh, const double* scal, double* out, cudaStream_t s);
int launch_fd_jacobian(dv_model* m, double t, const double* y, const double* f0, double* J, cudaStream_t s);
// The same difference quotients rounded to FP32 (the mixed-precision Krylov operator's Jacobian).
int launch_fd_jacobian32(dv_model* m, double t, const double* y, const double* f0, float* J, cudaStream_t s);
// Assembled-Jacobian operator of the Newton system in scaled variables, FP32 products and sums:
// out = (v - dh J v)/s with v = u s and J the FP32 block Jacobian m->d_J32; dh read from dh_dev when
// non-null (graph capture), else dh.
int launch_spmv32(dv_model* m, const double* u, const double* sc, double dh, const double* dh_dev, double* out,
                  cudaStream_t s, bool count = true);
// linear algebra (dv_linalg.cu)
int precond_factor(dv_model* m, const double* J, double dh, int mode, cudaStream_t s);
int64_t precond_doubles(int nb, int nparts, int Nz);
// Partition mode, twisted separator plane and block size of every partition of the current factors
// (nb_out up to cap entries); returns the number of partitions (0 before the first factorisation).
int precond_partitions(const dv_model* m, int* mode, int* zs, int* nb_out, int cap);
// Host check of a geometry's partition maps (number of violations; 0 = consistent).
int64_t precond_check_maps(const dv_step_params& p, int mode, int* nparts, int* nb);
// Largest block, partition count and storage over the partition modes a model of p can factorise.
void precond_capacity(const dv_step_params& p, int* cap_nb, int* cap_parts, int64_t* pc_need, int64_t* work_need);
int64_t precond_work_doubles(int nb, int nparts, int Nz);
// x = diag(1/sc) M^-1 diag(sc) b  (sc may be NULL: plain solve)
int precond_apply(dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s);
// Work the shared-memory sweep can do on the side when it runs in the GMRES graph.  Prologue (V
// non-null): the input is src = (*col == 0 ? src0 : src1) scaled by *scale, and is also stored to
// V[*col].  Epilogue (out non-null): *out = sqrt(sum x^2 / n) over the result, reduced through
// per-CTA partials `part` and a ticket counter (the last CTA sums them in CTA order).
struct PaFuse {
    const int* col = nullptr;
    const double* scale = nullptr;
    const double* src0 = nullptr;
    const double* src1 = nullptr;
    double* V = nullptr;
    int64_t ldv = 0;
    double* part = nullptr;
    unsigned* ticket = nullptr;
    double* out = nullptr;
    int64_t n = 0;
    const int* stop = nullptr;        // when *stop != 0 at launch: write *out = 0 and do nothing else
    bool pdl = false;                 // launch with programmatic stream serialisation (inside the GMRES graph)
};
// Programmatic dependent launches inside the GMRES graph: off unless DVTSA_PDL=1 (read once;
// measured 2 % slower on the 8x8x32 heating window, bit-identical results).
bool pdl_enabled();
bool precond_apply_fusable(dv_model* m);
// bounded-wait self-test: one sweep-style mbarrier wait that nothing completes (bit 1 of *err)
int selftest_mbar_timeout(int polls, int* err, cudaStream_t s);
// The same launches without launch accounting or attribute changes, for stream capture (the
// attributes are set by an earlier precond_apply).  Returns the number of kernels launched.
int precond_apply_capture(dv_model* m, const double* b, const double* sc, double* x, cudaStream_t s,
                          const PaFuse& F = PaFuse());
// FD matvec of the split residual for stream capture: t and gh are read from dargs[0..1] (device).
// With `bar` (two zeroed barrier words) the three phases run as one cooperative launch.
int matvec_capture(dv_model* m, const double* dargs, const double* z, const double* u, const double* sc,
                   const double* f0, const double* scal, double* out, cudaStream_t s, unsigned* bar = nullptr);
// Kernels one matvec_capture with `bar` launched (1 cooperative, or the 3 of the split residual).
int matvec_capture_kernels();
}  // namespace dv
