/*
 * ORACLE -- BENCH / TEST INFRASTRUCTURE ONLY.  Nothing in the product (opensol_b200/) links, loads or calls this
 * file; bench.py's reference-replay leg and tests/ do, to time open_sol's own GPU step on the same grid.
 *
 * Reference-kernel replay of open_sol's 2D E_z GPU step (the cupy backend, which this image cannot run): the
 * reference's two RawKernels (update_h_kernel / update_e_kernel, open_sol/physics/em/solvers/
 * fdtd_ez_2d_kernels.py:23-122) are compiled unchanged from the reference tree into a cubin by
 * oracle/make_ref_replay.py and loaded here with the driver API; the launch sequence of one step follows
 * FDTDEngine2D_Ez.advance (fdtd_ez_2d.py:71-119) and _fixed_block (fdtd_2d_base.py:558-599):
 *
 *   H graph: update_h_kernel on (32, 8, 1) blocks, then one CPML psi launch per active side (h rows);
 *   E graph: update_e_kernel, then one CPML psi launch per active side (e rows);
 *   eager:   the line source's scaled-profile add at t + dt/2 (core/sources.py:221-229), skipped when its float32
 *            value is 0;
 *   eager, every sample_interval steps: per flux monitor one phase launch and two complex128 line accumulations
 *            (physics/em/monitors.py:22-34,203-238).
 *
 * The cupy ElementwiseKernels among them (the CPML psi update + apply, boundaries.py:27-37; the scaled-profile add,
 * core/sources.py:146-154; the DFT phase and line accumulation, monitors.py:22-34,84-90) are restated below as plain
 * kernels with one thread per element of the (possibly strided) view, as cupy's elementwise launches index them.
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define REPLAY_MAX_SIDES 4
#define REPLAY_MAX_MONITORS 8
#define ELEMENTWISE_THREADS 128

typedef struct {
    int axis;                 /* 0: an x side (psi (npml, ny)), 1: a y side (psi (nx, npml)) */
    int npml;
    int e_row0, h_row0;       /* first grid row of the side's e / h rows */
    float sign;               /* +1 for x sides, -1 for y sides */
    const float *b_e, *a_e, *inv_e, *b_h, *a_h, *inv_h;   /* (npml,) rows */
    float *psi_e, *psi_h;
} ReplaySide;

typedef struct {
    int normal_axis;          /* 0: a line along y at x-cell `position`; 1: along x at y-cell `position` */
    int position, lo, hi, nf;
    const double *omega;      /* (nf,) 2 pi f */
    double dt_m;              /* dt * sample_interval */
    float2 *phases;           /* (nf,) complex64 scratch */
    double2 *e_acc, *h_acc;   /* (nf, hi - lo) complex128 */
} ReplayMonitor;

typedef struct {
    int nx, ny;
    float *ez, *hx, *hy;
    const float *ca, *cb, *da, *db;
    const float *inv_dx_e, *inv_dx_h, *inv_dy_e, *inv_dy_h;
    int n_sides;
    ReplaySide sides[REPLAY_MAX_SIDES];
    int src_axis, src_position, src_lo, src_hi;   /* src_axis -1: no source */
    const float *profile;
    int n_monitors;
    ReplayMonitor monitors[REPLAY_MAX_MONITORS];
    int sample_interval;
} ReplayConfig;

typedef struct {
    ReplayConfig cfg;
    CUmodule module;
    CUfunction update_h, update_e;
    cudaStream_t stream;
    cudaGraphExec_t h_exec, e_exec;
    cudaEvent_t start, stop;
    const float *zero_partner;   /* the real-only engine's partner arrays: the field itself, cos 1, sin 0 */
} Replay;

static char replay_error[512];

extern "C" const char *replay_ez2d_last_error(void) { return replay_error; }

#define CUDA_OK(call)                                                                                           \
    do {                                                                                                        \
        cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess) {                                                                                \
            snprintf(replay_error, sizeof replay_error, "%s: %s", #call, cudaGetErrorString(e_));               \
            return 1;                                                                                           \
        }                                                                                                       \
    } while (0)
#define CU_OK(call)                                                                                             \
    do {                                                                                                        \
        CUresult r_ = (call);                                                                                   \
        if (r_ != CUDA_SUCCESS) {                                                                               \
            const char *s_ = NULL;                                                                              \
            cuGetErrorString(r_, &s_);                                                                          \
            snprintf(replay_error, sizeof replay_error, "%s: %s", #call, s_ ? s_ : "?");                        \
            return 1;                                                                                           \
        }                                                                                                       \
    } while (0)

/* psi = b psi + a (f_hi - f_lo) inv; field += sign coefficient psi over one side's (rows x line) view. */
__global__ void replay_cpml_psi(int axis, int npml, int nx, int ny, int row0, int shift_hi, int shift_lo,
                                const float *b, const float *a, const float *inv, float sign,
                                const float *source, const float *coefficient, float *psi, float *field) {
    const long long n = axis == 0 ? (long long)npml * ny : (long long)nx * npml;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        int i, j, r;
        if (axis == 0) {
            r = (int)(e / ny);
            j = (int)(e % ny);
            i = row0 + r;
        } else {
            i = (int)(e / npml);
            r = (int)(e % npml);
            j = row0 + r;
        }
        const long long idx = (long long)i * ny + j;
        const long long step = axis == 0 ? ny : 1;
        const float f_hi = source[idx + shift_hi * step], f_lo = source[idx + shift_lo * step];
        const float value = b[r] * psi[e] + a[r] * (f_hi - f_lo) * inv[r];
        psi[e] = value;
        field[idx] += sign * coefficient[idx] * value;
    }
}

/* target += (float)(scale * profile) on the source line. */
__global__ void replay_add_scaled_profile(float *target, long long stride, const float *profile, float scale, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) target[c * stride] += scale * profile[c];
}

/* ph = complex64(cos(-omega t) dt_m, sin(-omega t) dt_m), the phase evaluated in float64. */
__global__ void replay_dft_phase(const double *omega, double t, double dt_m, float2 *ph, int nf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) {
        const double p = -omega[f] * t;
        ph[f] = make_float2((float)(cos(p) * dt_m), (float)(sin(p) * dt_m));
    }
}

/* acc[f, c] += complex128(ph[f]) * (double)line[c]. */
__global__ void replay_dft_accumulate(const float *line, long long stride, const float2 *ph, double2 *acc, int nf,
                                      int n) {
    const long long total = (long long)nf * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(e / n), c = (int)(e % n);
        const double v = (double)line[c * stride];
        const float2 p = ph[f];
        double2 a = acc[e];
        a.x += (double)p.x * v;
        a.y += (double)p.y * v;
        acc[e] = a;
    }
}

static unsigned elementwise_blocks(long long n) {
    long long b = (n + ELEMENTWISE_THREADS - 1) / ELEMENTWISE_THREADS;
    return (unsigned)(b < 1 ? 1 : (b > 65535LL * 64 ? 65535LL * 64 : b));
}

static int launch_update_h(Replay *r) {
    ReplayConfig *c = &r->cfg;
    int periodic = 0;
    float one = 1.0f, zero = 0.0f;
    const float *partner = c->ez;
    void *args[] = {&c->ez, &c->hx, &c->hy, &c->da, &c->db, &c->inv_dx_h, &c->inv_dy_h, &c->nx, &c->ny,
                    &periodic, &periodic, &partner, &one, &zero, &one, &zero};
    CU_OK(cuLaunchKernel(r->update_h, (c->ny + 31) / 32, (c->nx + 7) / 8, 1, 32, 8, 1, 0, (CUstream)r->stream, args,
                         NULL));
    return 0;
}

static int launch_update_e(Replay *r) {
    ReplayConfig *c = &r->cfg;
    int periodic = 0;
    float one = 1.0f, zero = 0.0f;
    const float *hx_partner = c->hx, *hy_partner = c->hy;
    void *args[] = {&c->ez, &c->hx, &c->hy, &c->ca, &c->cb, &c->inv_dx_e, &c->inv_dy_e, &c->nx, &c->ny,
                    &periodic, &periodic, &hx_partner, &hy_partner, &one, &zero, &one, &zero};
    CU_OK(cuLaunchKernel(r->update_e, (c->ny + 31) / 32, (c->nx + 7) / 8, 1, 32, 8, 1, 0, (CUstream)r->stream, args,
                         NULL));
    return 0;
}

/* kind 0: h rows (source E_z, coefficient db, field H_y / H_x); kind 1: e rows (source H_y / H_x, cb, E_z). */
static int launch_cpml(Replay *r, int kind) {
    ReplayConfig *c = &r->cfg;
    for (int s = 0; s < c->n_sides; ++s) {
        ReplaySide *side = &c->sides[s];
        const long long n = side->axis == 0 ? (long long)side->npml * c->ny : (long long)c->nx * side->npml;
        if (kind == 0) {   /* h rows r: f_hi = E_z[r + 1], f_lo = E_z[r] */
            float *field = side->axis == 0 ? c->hy : c->hx;
            replay_cpml_psi<<<elementwise_blocks(n), ELEMENTWISE_THREADS, 0, r->stream>>>(
                side->axis, side->npml, c->nx, c->ny, side->h_row0, 1, 0, side->b_h, side->a_h, side->inv_h,
                side->sign, c->ez, c->db, side->psi_h, field);
        } else {           /* e rows r: f_hi = H[r], f_lo = H[r - 1] */
            const float *source = side->axis == 0 ? c->hy : c->hx;
            replay_cpml_psi<<<elementwise_blocks(n), ELEMENTWISE_THREADS, 0, r->stream>>>(
                side->axis, side->npml, c->nx, c->ny, side->e_row0, 0, -1, side->b_e, side->a_e, side->inv_e,
                side->sign, source, c->cb, side->psi_e, c->ez);
        }
        CUDA_OK(cudaGetLastError());
    }
    return 0;
}

static int capture(Replay *r, int kind, cudaGraphExec_t *exec) {
    cudaGraph_t graph;
    CUDA_OK(cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
    int bad = kind == 0 ? launch_update_h(r) : launch_update_e(r);
    if (!bad) bad = launch_cpml(r, kind);
    cudaError_t end = cudaStreamEndCapture(r->stream, &graph);
    if (bad) return 1;
    CUDA_OK(end);
    CUDA_OK(cudaGraphInstantiate(exec, graph, 0));
    CUDA_OK(cudaGraphDestroy(graph));
    return 0;
}

extern "C" int replay_ez2d_create(const char *cubin_path, const ReplayConfig *cfg, void **out) {
    *out = NULL;
    if (cfg->n_sides > REPLAY_MAX_SIDES || cfg->n_monitors > REPLAY_MAX_MONITORS || cfg->sample_interval < 1) {
        snprintf(replay_error, sizeof replay_error, "replay: unsupported configuration");
        return 1;
    }
    CUDA_OK(cudaFree(0));   /* the primary context current, shared with the caller's runtime allocations */
    Replay *r = (Replay *)calloc(1, sizeof(Replay));
    r->cfg = *cfg;
    if (cuModuleLoad(&r->module, cubin_path) != CUDA_SUCCESS) {
        snprintf(replay_error, sizeof replay_error, "replay: cannot load %s", cubin_path);
        free(r);
        return 1;
    }
    CU_OK(cuModuleGetFunction(&r->update_h, r->module, "update_h_kernel"));
    CU_OK(cuModuleGetFunction(&r->update_e, r->module, "update_e_kernel"));
    CUDA_OK(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreate(&r->start));
    CUDA_OK(cudaEventCreate(&r->stop));
    /* the reference's first step of a key runs eagerly (module load outside the capture), later ones replay */
    if (launch_update_h(r) || launch_cpml(r, 0) || launch_update_e(r) || launch_cpml(r, 1)) return 1;
    CUDA_OK(cudaStreamSynchronize(r->stream));
    if (capture(r, 0, &r->h_exec) || capture(r, 1, &r->e_exec)) return 1;
    *out = r;
    return 0;
}

/* Reset fields, psi and spectra to zero (the caller's buffers) on the replay stream. */
extern "C" int replay_ez2d_reset(void *handle) {
    Replay *r = (Replay *)handle;
    ReplayConfig *c = &r->cfg;
    const size_t cells = (size_t)c->nx * c->ny * sizeof(float);
    CUDA_OK(cudaMemsetAsync(c->ez, 0, cells, r->stream));
    CUDA_OK(cudaMemsetAsync(c->hx, 0, cells, r->stream));
    CUDA_OK(cudaMemsetAsync(c->hy, 0, cells, r->stream));
    for (int s = 0; s < c->n_sides; ++s) {
        const ReplaySide *side = &c->sides[s];
        const size_t n = (side->axis == 0 ? (size_t)side->npml * c->ny : (size_t)c->nx * side->npml) * sizeof(float);
        CUDA_OK(cudaMemsetAsync(side->psi_e, 0, n, r->stream));
        CUDA_OK(cudaMemsetAsync(side->psi_h, 0, n, r->stream));
    }
    for (int m = 0; m < c->n_monitors; ++m) {
        const ReplayMonitor *mon = &c->monitors[m];
        const size_t n = (size_t)mon->nf * (mon->hi - mon->lo) * sizeof(double2);
        CUDA_OK(cudaMemsetAsync(mon->e_acc, 0, n, r->stream));
        CUDA_OK(cudaMemsetAsync(mon->h_acc, 0, n, r->stream));
    }
    CUDA_OK(cudaStreamSynchronize(r->stream));
    return 0;
}

/* Steps first_step .. first_step + n_steps - 1: source_values[k] = float32 amplitude * s(t + dt/2) of step k,
 * sample_times = the engine clock after each DFT-sampled step, in order.  *ms = device time of the whole run
 * (events on the replay stream). */
extern "C" int replay_ez2d_run(void *handle, int first_step, int n_steps, const float *source_values,
                               const double *sample_times, float *ms) {
    Replay *r = (Replay *)handle;
    ReplayConfig *c = &r->cfg;
    int q = 0;
    CUDA_OK(cudaEventRecord(r->start, r->stream));
    for (int k = 0; k < n_steps; ++k) {
        CUDA_OK(cudaGraphLaunch(r->h_exec, r->stream));
        CUDA_OK(cudaGraphLaunch(r->e_exec, r->stream));
        if (c->src_axis >= 0 && source_values[k] != 0.0f) {
            const int n = c->src_hi - c->src_lo;
            float *target = c->src_axis == 0 ? c->ez + (long long)c->src_lo * c->ny + c->src_position
                                             : c->ez + (long long)c->src_position * c->ny + c->src_lo;
            const long long stride = c->src_axis == 0 ? c->ny : 1;
            replay_add_scaled_profile<<<(n + ELEMENTWISE_THREADS - 1) / ELEMENTWISE_THREADS, ELEMENTWISE_THREADS, 0,
                                        r->stream>>>(target, stride, c->profile, source_values[k], n);
        }
        if ((first_step + k + 1) % c->sample_interval == 0) {
            const double t = sample_times[q++];
            for (int m = 0; m < c->n_monitors; ++m) {
                ReplayMonitor *mon = &c->monitors[m];
                const int n = mon->hi - mon->lo;
                const float *e_line, *h_line;
                long long stride;
                if (mon->normal_axis == 0) {
                    e_line = c->ez + (long long)mon->position * c->ny + mon->lo;
                    h_line = c->hy + (long long)mon->position * c->ny + mon->lo;
                    stride = 1;
                } else {
                    e_line = c->ez + (long long)mon->lo * c->ny + mon->position;
                    h_line = c->hx + (long long)mon->lo * c->ny + mon->position;
                    stride = c->ny;
                }
                replay_dft_phase<<<1, 32 * ((mon->nf + 31) / 32), 0, r->stream>>>(mon->omega, t, mon->dt_m,
                                                                                  mon->phases, mon->nf);
                const long long total = (long long)mon->nf * n;
                replay_dft_accumulate<<<elementwise_blocks(total), ELEMENTWISE_THREADS, 0, r->stream>>>(
                    e_line, stride, mon->phases, mon->e_acc, mon->nf, n);
                replay_dft_accumulate<<<elementwise_blocks(total), ELEMENTWISE_THREADS, 0, r->stream>>>(
                    h_line, stride, mon->phases, mon->h_acc, mon->nf, n);
            }
        }
    }
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaEventRecord(r->stop, r->stream));
    CUDA_OK(cudaEventSynchronize(r->stop));
    CUDA_OK(cudaEventElapsedTime(ms, r->start, r->stop));
    return 0;
}

extern "C" void replay_ez2d_destroy(void *handle) {
    Replay *r = (Replay *)handle;
    if (!r) return;
    cudaStreamSynchronize(r->stream);
    cudaGraphExecDestroy(r->h_exec);
    cudaGraphExecDestroy(r->e_exec);
    cudaEventDestroy(r->start);
    cudaEventDestroy(r->stop);
    cudaStreamDestroy(r->stream);
    cuModuleUnload(r->module);
    free(r);
}
