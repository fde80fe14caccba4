// 2D E_z-polarisation FDTD engine for sm_100a: device state, launch planning and the os_fdtd2d_* C ABI.
//
// The default path (fdtd2d_tb.cuh) advances T Yee steps per launch: an interior kernel (4 columns per thread, 128-bit
// loads, no CPML) plus a general kernel for the CPML slabs and grid edges, both reading one field buffer set and
// writing the other; then, when the launch crossed DFT sample steps, the staged-DFT kernel.  The per-half-step kernels
// of fdtd2d_kernels.cuh (one thread per cell, fields updated in place) remain selectable as variant 0 and serve as
// the plain reference of the same arithmetic.  The arithmetic of every cell follows open_sol's evaluation order
// (fdtd_ez_2d_kernels.py:23-122, boundaries.py:27-37, core/sources.py:146-154) and the files are compiled with
// -fmad=false, so each product and sum is rounded on its own as on the CPU: results are bit-identical to open_sol's
// CPU backend.  The CPML corrections of a cell are applied in FACES order (x sides, then y sides), as open_sol's one
// launch per side does.
#include "common.cuh"

#include <functional>
#include "fdtd2d_kernels.cuh"
#include "fdtd2d_tb.cuh"
#include "fdtd2d_interior.cuh"
#include "fdtd2d_hz.cuh"
#include "fdtd2d_hz2.cuh"
#include "fdtd2d_frame.cuh"

#include <algorithm>

#include <vector>
#include <memory>
#include <mutex>
#include <cstring>

namespace os {

struct LineSource2D {
    int32_t axis, position, lo, hi;
    DeviceArray<float> profile;
};

struct FluxLine2D {
    int32_t normal_axis, position, lo, hi, nf;
    DeviceArray<double> e_acc, h_acc;   // (nf, n) complex128 as double pairs
    DeviceArray<float> stage;           // (TB_MAX_T, 2, n) samples of one launch
};

// Field probes: one component of one cell recorded after every step.  rows holds, per probe, `capacity` floats
// indexed by the step (n_step after the step - 1); a probe added at step s has rows from s on.
constexpr int OS_MAX_PROBES = 8;
struct ProbeSet {
    int32_t n;
    int32_t ix[OS_MAX_PROBES], iy[OS_MAX_PROBES], comp[OS_MAX_PROBES];
    int64_t start[OS_MAX_PROBES];
};

// +x plane-wave TFSF box (TFSFSource): the 1D incident line and the side coefficients, all float32 as computed by
// the host.
struct Tfsf2D {
    int32_t x0, x1, y0, y1, aux_x0, aux_n, source_index;
    float coef_h[4], coef_e[4], mur_lo, mur_hi;
    DeviceArray<float> aux_ez, aux_hy, aux_coef_h, aux_coef_e;   // H_z boxes: aux_ez = incident E_y, aux_hy = H_z
};

// Drude (kind 0) or Lorentz (kind 1) pole on a cell box: drive (box, pole drive x cell mask) and its state.
struct Pole2D {
    int32_t kind, i0, i1, j0, j1;
    int32_t comp = 0;                   // field of an H_z engine's face set: 0 E_x (hi-y faces), 1 E_y (hi-x faces)
    float damping, restoring;
    DeviceArray<float> drive, a, b;     // Drude: a = J; Lorentz: a = P, b = dP
};

struct DftMap2D {                       // field-map running DFT (DFTMonitor)
    int32_t x0, y0, ds, mx, my, nf;     // first sampled cell, stride, samples per axis, frequencies
    bool hz;                            // H_z engine: H_z, E_x, E_y maps (E at the cell centres), two phase tables
    DeviceArray<float> acc;             // E_z: (nf, mx, my); H_z: (3, nf, mx, my); complex64 as float pairs
};

}  // namespace os

struct OsFdtd2D {
    OsGrid2D grid{};
    cudaStream_t stream = nullptr;        // the stream every call enqueues on
    cudaStream_t own_stream = nullptr;    // created with the handle, destroyed with it
    cudaStream_t side_stream = nullptr;   // the border kernel runs here, overlapping the interior kernel
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaEvent_t ev_handoff = nullptr;     // orders the next stream after the previous one (os_fdtd2d_set_stream)
    bool timed = false;
    os::DeviceArray<float> ez[2], hx[2], hy[2];   // double-buffered fields; `cur` is the live set
    int cur = 0;
    os::DeviceArray<float> ca, cb, da, db;
    float da_uniform = 1.0f, db_uniform = 0.0f;
    bool has_ca = false, has_dadb = false, has_cb = false, has_spacings = false;
    os::DeviceArray<float> inv_dx_e, inv_dx_h, inv_dy_e, inv_dy_h;
    os::DeviceArray<float> cpml_rows[4];   // per side: b_e, a_e, inv_e, b_h, a_h, inv_h (6 * npml)
    os::DeviceArray<float> psi_e[2][4], psi_h[2][4];
    // scratch states of the frame's intermediate steps in a blocked launch (E_z engines; allocated at creation)
    os::DeviceArray<float> sez[2], shx[2], shy[2], spsi_e[2][4], spsi_h[2][4];
    bool cpml_set[4] = {false, false, false, false};
    std::vector<float> host_inv[4];       // inv_dx_e, inv_dx_h, inv_dy_e, inv_dy_h (host copies: interior check)
    int32_t variant = 1;                  // 0: per-half-step kernels, 1: temporally blocked
    int32_t steps_per_launch = 3;         // T of the blocked kernels
    int32_t tile_rows = 0;                // rows per interior tile (0: chosen from the grid, interior_rows)
    int32_t gen_tile_rows = 16;           // rows per general tile
    int64_t launches = 0;                 // kernels launched by the last advance
    bool profiling = false;               // bracket every kernel with events (os_fdtd2d_kernel_times)
    int64_t stall_probe_ns = 0;           // test hook of the bounded waits (os_fdtd2d_set_stall_probe)
    std::vector<cudaEvent_t> prof_events; // pool, grown on demand
    std::vector<int> prof_kind;           // kind of each recorded pair: 0 interior, 1 general, 2 DFT, 3 per-step
    size_t prof_used = 0;
    std::vector<std::unique_ptr<os::LineSource2D>> lines;
    std::vector<std::unique_ptr<os::FluxLine2D>> fluxes;
    std::vector<std::unique_ptr<os::DftMap2D>> maps;   // field-map DFTs (E_z engines), after the flux lines in a
                                                       // chunk's phase table
    std::vector<std::unique_ptr<os::Tfsf2D>> tfsf;   // plane-wave boxes (E_z engines; their value rows follow the
                                                     // line sources' in a chunk's value table)
    std::vector<std::unique_ptr<os::Pole2D>> poles;   // dispersive poles (E_z engines), in add order
    os::DeviceArray<float> jz_total;      // (nx, ny) summed Drude J on drude_box
    int32_t drude_box[4] = {0, 0, 0, 0};  // union box of the Drude poles (i0, i1, j0, j1); empty when i1 == i0
    float inv_dt = 0.0f;                  // float32 1 / dt of the Lorentz corrections
    os::ProbeSet probes{};                // field probes (recorded after every step)
    os::DeviceArray<float> probe_rows;    // (OS_MAX_PROBES, probe_capacity) values by step
    os::DeviceArray<float> probe_stage;   // (OS_MAX_PROBES, TB_MAX_T, 2) the probes' cells at each step of a launch
    int64_t probe_capacity = 0;           // rows per probe
    int64_t sample_interval = 1;
    int64_t n_step = 0;
    os::DeviceArray<int32_t> err;         // set by a kernel whose bounded wait ran out
    os::DeviceArray<float> line_values;   // (n_lines, n_steps) of the current chunk
    os::DeviceArray<float> phases;        // per monitor (n_samples, nf, 2) of the current chunk
    int device = 0;
    // H_z polarisation (os_fdtd2d_hz_create): ez / hx / hy hold H_z / E_x / E_y, ca / cb the E_x face coefficients
    int32_t polarization = 0;             // 0 E_z, 1 H_z
    os::DeviceArray<float> ca_y, cb_y;    // E_y face coefficients (coefficient form)
    os::DeviceArray<float> eps_cell;      // eps_r per cell (lossless form: face coefficients evaluated in the kernel)
    os::DeviceArray<float> shares;        // lower_x, upper_x (nx each), lower_y, upper_y (ny each)
    bool hz_eps = false;                  // lossless form active
    float dt_hz = 0.0f, eps0_hz = 0.0f;   // dt and eps0 of the lossless form
    int32_t hz_rows = 0;                  // rows per CTA of the fused step kernel (0: chosen per grid)
    int sm_count = 148;                   // multiprocessors of the device (launch sizing)
};

namespace os {

static int bind_device(OsFdtd2D *h) {
    OS_CUDA(cudaSetDevice(h->device));
    return OS_OK;
}

static size_t cells(const OsFdtd2D *h) { return (size_t)h->grid.nx * (size_t)h->grid.ny; }

// Synchronise the handle's stream and report a kernel whose bounded wait ran out (the flag is cleared).
static int sync_and_check(OsFdtd2D *h) {
    OS_CUDA(cudaStreamSynchronize(h->stream));
    int32_t flag = 0;
    OS_CUDA(cudaMemcpy(&flag, h->err.ptr, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag) {
        OS_CUDA(cudaMemset(h->err.ptr, 0, sizeof(int32_t)));
        set_error("a staged row did not arrive within the bounded wait: the fields of the last advance are invalid");
        return OS_ERR_CUDA;
    }
    return OS_OK;
}

static int zero_state(OsFdtd2D *h) {
    const size_t n = cells(h);
    const int c = h->cur;
    OS_CUDA(cudaMemsetAsync(h->ez[c].ptr, 0, n * sizeof(float), h->stream));
    OS_CUDA(cudaMemsetAsync(h->hx[c].ptr, 0, n * sizeof(float), h->stream));
    OS_CUDA(cudaMemsetAsync(h->hy[c].ptr, 0, n * sizeof(float), h->stream));
    for (int s = 0; s < 4; ++s) {
        if (h->psi_e[c][s].ptr) OS_CUDA(cudaMemsetAsync(h->psi_e[c][s].ptr, 0, h->psi_e[c][s].bytes(), h->stream));
        if (h->psi_h[c][s].ptr) OS_CUDA(cudaMemsetAsync(h->psi_h[c][s].ptr, 0, h->psi_h[c][s].bytes(), h->stream));
    }
    for (auto &f : h->fluxes) {
        OS_CUDA(cudaMemsetAsync(f->e_acc.ptr, 0, f->e_acc.bytes(), h->stream));
        OS_CUDA(cudaMemsetAsync(f->h_acc.ptr, 0, f->h_acc.bytes(), h->stream));
    }
    for (auto &d : h->maps) OS_CUDA(cudaMemsetAsync(d->acc.ptr, 0, d->acc.bytes(), h->stream));
    for (auto &t : h->tfsf) {
        OS_CUDA(cudaMemsetAsync(t->aux_ez.ptr, 0, t->aux_ez.bytes(), h->stream));
        OS_CUDA(cudaMemsetAsync(t->aux_hy.ptr, 0, t->aux_hy.bytes(), h->stream));
    }
    for (auto &q : h->poles) {
        OS_CUDA(cudaMemsetAsync(q->a.ptr, 0, q->a.bytes(), h->stream));
        if (q->b.ptr) OS_CUDA(cudaMemsetAsync(q->b.ptr, 0, q->b.bytes(), h->stream));
    }
    if (h->jz_total.ptr) OS_CUDA(cudaMemsetAsync(h->jz_total.ptr, 0, h->jz_total.bytes(), h->stream));
    for (int k = 0; k < h->probes.n; ++k) h->probes.start[k] = 0;   // rows recorded again from step 0
    h->n_step = 0;
    return OS_OK;
}

static Ez2DParams make_params(const OsFdtd2D *h) {
    Ez2DParams p{};
    p.nx = h->grid.nx;
    p.ny = h->grid.ny;
    p.periodic_x = h->grid.periodic_x;
    p.periodic_y = h->grid.periodic_y;
    p.npml = h->grid.npml;
    p.ez = h->ez[h->cur].ptr;
    p.hx = h->hx[h->cur].ptr;
    p.hy = h->hy[h->cur].ptr;
    p.ca = h->has_ca ? h->ca.ptr : nullptr;
    p.cb = h->cb.ptr;
    p.da = h->has_dadb ? h->da.ptr : nullptr;
    p.db = h->has_dadb ? h->db.ptr : nullptr;
    p.da_uniform = h->da_uniform;
    p.db_uniform = h->db_uniform;
    p.inv_dx_e = h->inv_dx_e.ptr;
    p.inv_dx_h = h->inv_dx_h.ptr;
    p.inv_dy_e = h->inv_dy_e.ptr;
    p.inv_dy_h = h->inv_dy_h.ptr;
    p.cpml_mask = 0;
    const int npml = h->grid.npml;
    for (int s = 0; s < 4; ++s) {
        if (!(h->grid.cpml_sides & (1 << s))) continue;
        p.cpml_mask |= 1 << s;
        const float *rows = h->cpml_rows[s].ptr;
        p.b_e[s] = rows;
        p.a_e[s] = rows + npml;
        p.inv_e[s] = rows + 2 * npml;
        p.b_h[s] = rows + 3 * npml;
        p.a_h[s] = rows + 4 * npml;
        p.inv_h[s] = rows + 5 * npml;
        p.psi_e[s] = h->psi_e[h->cur][s].ptr;
        p.psi_h[s] = h->psi_h[h->cur][s].ptr;
    }
    p.n_lines = (int32_t)h->lines.size();
    for (size_t l = 0; l < h->lines.size(); ++l) {
        p.lines[l].axis = h->lines[l]->axis;
        p.lines[l].position = h->lines[l]->position;
        p.lines[l].lo = h->lines[l]->lo;
        p.lines[l].hi = h->lines[l]->hi;
        p.lines[l].profile = h->lines[l]->profile.ptr;
    }
    return p;
}

// Entry points of one polarisation refuse a handle of the other.
static int require_hz(const OsFdtd2D *h, const char *fn) {
    OS_CHECK(h, OS_ERR_INVALID, "%s: null handle", fn);
    OS_CHECK(h->polarization == 1, OS_ERR_STATE, "%s: the handle is an E_z engine (os_fdtd2d_create)", fn);
    return OS_OK;
}
static int require_ez(const OsFdtd2D *h, const char *fn) {
    OS_CHECK(h, OS_ERR_INVALID, "%s: null handle", fn);
    OS_CHECK(h->polarization == 0, OS_ERR_STATE, "%s: the handle is an H_z engine (os_fdtd2d_hz_create)", fn);
    return OS_OK;
}

}  // namespace os

using namespace os;

static int create_2d(const OsGrid2D *grid, int32_t polarization, OsFdtd2D **out) {
    OS_CHECK(grid && out, OS_ERR_INVALID, "os_fdtd2d_create: null argument");
    *out = nullptr;
    const OsGrid2D g = *grid;
    OS_CHECK(g.nx >= 1 && g.ny >= 1, OS_ERR_INVALID, "os_fdtd2d_create: grid %d x %d has no cells", g.nx, g.ny);
    OS_CHECK((int64_t)g.nx * g.ny < ((int64_t)1 << 40), OS_ERR_INVALID, "os_fdtd2d_create: grid too large");
    OS_CHECK(g.nx <= 65535 * EZ2D_BLOCK_Y, OS_ERR_INVALID, "os_fdtd2d_create: nx = %d exceeds %d", g.nx,
             65535 * EZ2D_BLOCK_Y);
    OS_CHECK((g.cpml_sides & ~15) == 0, OS_ERR_INVALID, "os_fdtd2d_create: cpml_sides %d has bits beyond the 2D faces",
             g.cpml_sides);
    OS_CHECK(!(g.periodic_x && (g.cpml_sides & 3)) && !(g.periodic_y && (g.cpml_sides & 12)), OS_ERR_INVALID,
             "periodic/bloch BCs must be paired: a periodic axis has no CPML side");
    for (int axis = 0; axis < 2; ++axis) {
        const int n = axis == 0 ? g.nx : g.ny;
        const int layers = ((g.cpml_sides >> (2 * axis)) & 1) + ((g.cpml_sides >> (2 * axis + 1)) & 1);
        if (layers) {
            OS_CHECK(g.npml >= 1, OS_ERR_INVALID, "cpml_npml must be an integer >= 1 with a cpml face, got %d", g.npml);
            OS_CHECK(n >= layers * g.npml + 2, OS_ERR_INVALID,
                     "%c axis: %d cells cannot hold %d CPML layer(s) of %d cells plus the 2 unstretched rows; it "
                     "needs at least %d cells", axis == 0 ? 'x' : 'y', n, layers, g.npml, layers * g.npml + 2);
        }
    }
    std::unique_ptr<OsFdtd2D> h(new OsFdtd2D());
    h->grid = g;
    h->device = g.device;
    OS_TRY(bind_device(h.get()));
    OS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    OS_CUDA(cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking));
    OS_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    OS_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    OS_CUDA(cudaEventCreateWithFlags(&h->ev_handoff, cudaEventDisableTiming));
    h->stream = h->own_stream;
    OS_CUDA(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device));
    OS_CUDA(cudaEventCreate(&h->ev_start));
    OS_CUDA(cudaEventCreate(&h->ev_stop));
    const size_t n = cells(h.get());
    h->polarization = polarization;
    for (int b = 0; b < 2; ++b) {
        OS_TRY(h->ez[b].alloc(n));
        OS_TRY(h->hx[b].alloc(n));
        OS_TRY(h->hy[b].alloc(n));
        if (polarization == 0) {
            OS_TRY(h->sez[b].alloc(n));
            OS_TRY(h->shx[b].alloc(n));
            OS_TRY(h->shy[b].alloc(n));
        }
    }
    for (int s = 0; s < 4; ++s) {
        if (!(g.cpml_sides & (1 << s))) continue;
        const size_t slab = (s < 2 ? (size_t)g.ny : (size_t)g.nx) * (size_t)g.npml;
        for (int b = 0; b < 2; ++b) {
            OS_TRY(h->psi_e[b][s].alloc(slab));
            OS_TRY(h->psi_h[b][s].alloc(slab));
            if (polarization == 0) {
                OS_TRY(h->spsi_e[b][s].alloc(slab));
                OS_TRY(h->spsi_h[b][s].alloc(slab));
            }
        }
        OS_TRY(h->cpml_rows[s].alloc(6 * (size_t)g.npml));
    }
    OS_TRY(h->err.alloc(1));
    OS_CUDA(cudaMemsetAsync(h->err.ptr, 0, sizeof(int32_t), h->stream));
    OS_TRY(zero_state(h.get()));   // queued on the handle's stream; every later use is ordered behind it
    *out = h.release();
    return OS_OK;
}

extern "C" int os_fdtd2d_create(const OsGrid2D *grid, OsFdtd2D **out) { return create_2d(grid, 0, out); }

extern "C" int os_fdtd2d_destroy(OsFdtd2D *h) {
    if (!h) return OS_OK;
    cudaSetDevice(h->device);
    // The device arrays go to the pool, to be handed out again once the work queued so far on the handle's streams
    // (its own, the side stream, and a caller's stream it is set to, which the caller keeps alive while the handle
    // uses it) has finished; no cudaFree, which would wait for the whole device.
    {
        cudaStream_t streams[3] = {h->own_stream, h->side_stream, h->stream};
        const int n_streams = (h->stream && h->stream != h->own_stream) ? 3 : 2;
        PoolEvents *ev = pool_events(streams, n_streams);
        auto give = [&](auto &a) { a.give_to_pool(ev); };
        for (int b = 0; b < 2; ++b) {
            give(h->ez[b]), give(h->hx[b]), give(h->hy[b]);
            give(h->sez[b]), give(h->shx[b]), give(h->shy[b]);
            for (int sd = 0; sd < 4; ++sd) {
                give(h->psi_e[b][sd]), give(h->psi_h[b][sd]);
                give(h->spsi_e[b][sd]), give(h->spsi_h[b][sd]);
            }
        }
        give(h->ca), give(h->cb), give(h->da), give(h->db), give(h->ca_y), give(h->cb_y);
        give(h->eps_cell), give(h->shares);
        give(h->inv_dx_e), give(h->inv_dx_h), give(h->inv_dy_e), give(h->inv_dy_h);
        for (int sd = 0; sd < 4; ++sd) give(h->cpml_rows[sd]);
        for (auto &l : h->lines) give(l->profile);
        for (auto &f : h->fluxes) give(f->e_acc), give(f->h_acc), give(f->stage);
        for (auto &d : h->maps) give(d->acc);
        for (auto &t : h->tfsf) give(t->aux_ez), give(t->aux_hy), give(t->aux_coef_h), give(t->aux_coef_e);
        for (auto &q : h->poles) give(q->drive), give(q->a), give(q->b);
        give(h->jz_total);
        give(h->probe_rows), give(h->probe_stage);
        give(h->err), give(h->line_values), give(h->phases);
        pool_events_done(ev);
    }
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    if (h->side_stream) cudaStreamSynchronize(h->side_stream);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev_handoff) cudaEventDestroy(h->ev_handoff);
    cudaStream_t stream = h->own_stream, side = h->side_stream;
    delete h;   // frees the device arrays
    if (stream) cudaStreamDestroy(stream);
    if (side) cudaStreamDestroy(side);
    return OS_OK;
}

extern "C" int os_fdtd2d_set_spacings(OsFdtd2D *h, const float *inv_dx_e, const float *inv_dx_h,
                                      const float *inv_dy_e, const float *inv_dy_h) {
    OS_CHECK(h && inv_dx_e && inv_dx_h && inv_dy_e && inv_dy_h, OS_ERR_INVALID, "os_fdtd2d_set_spacings: null argument");
    OS_TRY(bind_device(h));
    OS_TRY(upload(h->inv_dx_e, inv_dx_e, h->grid.nx, h->stream));
    OS_TRY(upload(h->inv_dx_h, inv_dx_h, h->grid.nx, h->stream));
    OS_TRY(upload(h->inv_dy_e, inv_dy_e, h->grid.ny, h->stream));
    OS_TRY(upload(h->inv_dy_h, inv_dy_h, h->grid.ny, h->stream));
    h->host_inv[0].assign(inv_dx_e, inv_dx_e + h->grid.nx);
    h->host_inv[1].assign(inv_dx_h, inv_dx_h + h->grid.nx);
    h->host_inv[2].assign(inv_dy_e, inv_dy_e + h->grid.ny);
    h->host_inv[3].assign(inv_dy_h, inv_dy_h + h->grid.ny);
    h->has_spacings = true;
    return OS_OK;
}

extern "C" int os_fdtd2d_set_materials(OsFdtd2D *h, const float *eps_r, const float *sigma_e, const float *mu_r,
                                       const float *sigma_m, float dt, float eps0, float mu0) {
    OS_TRY(require_ez(h, "os_fdtd2d_set_materials"));
    OS_CHECK(eps_r, OS_ERR_INVALID, "os_fdtd2d_set_materials: eps_r is required");
    OS_TRY(bind_device(h));
    const size_t n = cells(h);
    OS_TRY(h->cb.alloc(n));
    // eps_r / sigma_e (and mu_r / sigma_m) are staged in temporary device arrays that go to the pool behind the
    // coefficient kernels (no host wait: jobs are set up while others run); ca is only kept for a lossy grid.
    DeviceArray<float> eps_dev, sigma_dev, mu_dev, sm_dev;
    OS_TRY(upload(eps_dev, eps_r, n, h->stream));
    if (sigma_e) {
        OS_TRY(upload(sigma_dev, sigma_e, n, h->stream));
        OS_TRY(h->ca.alloc(n));
    }
    const int threads = 256;
    const unsigned blocks = (unsigned)((n + threads - 1) / threads);
    ez2d_e_coefficients_kernel<<<blocks, threads, 0, h->stream>>>(eps_dev.ptr, sigma_dev.ptr, dt, eps0, n,
                                                                  sigma_e ? h->ca.ptr : nullptr, h->cb.ptr);
    OS_CUDA(cudaGetLastError());
    h->has_ca = sigma_e != nullptr;
    h->has_cb = true;
    if (mu_r || sigma_m) {
        if (mu_r) OS_TRY(upload(mu_dev, mu_r, n, h->stream));
        if (sigma_m) OS_TRY(upload(sm_dev, sigma_m, n, h->stream));
        OS_TRY(h->da.alloc(n));
        OS_TRY(h->db.alloc(n));
        ez2d_h_coefficients_kernel<<<blocks, threads, 0, h->stream>>>(mu_dev.ptr, sm_dev.ptr, dt, mu0, n, h->da.ptr,
                                                                      h->db.ptr);
        OS_CUDA(cudaGetLastError());
        h->has_dadb = true;
    } else {
        // vacuum permeability: da = (1 - 0) / 1, db = (dt / mu0) / 1 (fdtd_ez_2d_kernels.py:335-340)
        const float mu = 1.0f * mu0;
        const float k = (0.0f * dt) / (2.0f * mu);
        const float denom = 1.0f + k;
        h->da_uniform = (1.0f - k) / denom;
        h->db_uniform = (dt / mu) / denom;
        h->has_dadb = false;
    }
    give_after(h->stream, eps_dev, sigma_dev, mu_dev, sm_dev);
    return OS_OK;
}

extern "C" int os_fdtd2d_set_coefficients(OsFdtd2D *h, const float *ca, const float *cb, const float *da,
                                          const float *db, float da_uniform, float db_uniform) {
    OS_TRY(require_ez(h, "os_fdtd2d_set_coefficients"));
    OS_CHECK(cb, OS_ERR_INVALID, "os_fdtd2d_set_coefficients: cb is required");
    OS_CHECK((da == nullptr) == (db == nullptr), OS_ERR_INVALID, "os_fdtd2d_set_coefficients: pass both da and db or neither");
    OS_TRY(bind_device(h));
    const size_t n = cells(h);
    OS_TRY(upload(h->cb, cb, n, h->stream));
    h->has_cb = true;
    h->has_ca = ca != nullptr;
    if (ca) OS_TRY(upload(h->ca, ca, n, h->stream));
    h->has_dadb = da != nullptr;
    if (da) {
        OS_TRY(upload(h->da, da, n, h->stream));
        OS_TRY(upload(h->db, db, n, h->stream));
    }
    h->da_uniform = da_uniform;
    h->db_uniform = db_uniform;
    return OS_OK;
}

extern "C" int os_fdtd2d_read_cb(OsFdtd2D *h, float *cb) {
    OS_TRY(require_ez(h, "os_fdtd2d_read_cb"));
    OS_CHECK(cb, OS_ERR_INVALID, "os_fdtd2d_read_cb: null argument");
    OS_CHECK(h->has_cb, OS_ERR_STATE, "os_fdtd2d_read_cb: coefficients are not set");
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(cb, h->cb.ptr, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// H_z polarisation: the same handle with H_z / E_x / E_y in the three field buffer sets.

extern "C" int os_fdtd2d_hz_create(const OsGrid2D *grid, OsFdtd2D **out) { return create_2d(grid, 1, out); }

extern "C" int os_fdtd2d_hz_set_materials(OsFdtd2D *h, const float *eps_xx, const float *eps_yy,
                                          const float *sigma_e, const float *mu_r, const float *sigma_m,
                                          const float *lower_x, const float *upper_x, const float *lower_y,
                                          const float *upper_y, float dt, float eps0, float mu0) {
    OS_TRY(require_hz(h, "os_fdtd2d_hz_set_materials"));
    OS_CHECK(eps_xx && eps_yy && lower_x && upper_x && lower_y && upper_y, OS_ERR_INVALID,
             "os_fdtd2d_hz_set_materials: eps_xx, eps_yy and the face shares are required");
    OS_TRY(bind_device(h));
    const size_t n = cells(h);
    const int nx = h->grid.nx, ny = h->grid.ny;
    // Lossless form: no sigma_e (or all zero), eps_xx = eps_yy with every eps_r > 0 and finite, vacuum permeability;
    // then k = 0 and the denominators are exactly 1, so cb = dt / (face eps_r * eps0) is evaluated in the step kernel.
    bool lossless = true;
    if (sigma_e)
        for (size_t c = 0; c < n && lossless; ++c) lossless = sigma_e[c] == 0.0f;
    bool eps_form = lossless && !mu_r && !sigma_m && std::memcmp(eps_xx, eps_yy, n * sizeof(float)) == 0;
    for (size_t c = 0; c < n && eps_form; ++c) eps_form = eps_xx[c] > 0.0f && eps_xx[c] <= 3.0e38f;
    std::vector<float> shares(2 * (size_t)nx + 2 * (size_t)ny);
    std::memcpy(shares.data(), lower_x, nx * sizeof(float));
    std::memcpy(shares.data() + nx, upper_x, nx * sizeof(float));
    std::memcpy(shares.data() + 2 * nx, lower_y, ny * sizeof(float));
    std::memcpy(shares.data() + 2 * nx + ny, upper_y, ny * sizeof(float));
    OS_TRY(upload(h->shares, shares.data(), shares.size(), h->stream));
    DeviceArray<float> exx, eyy, sig, mu_dev, sm_dev;   // staging, to the pool behind the kernels that read them
    OS_TRY(upload(exx, eps_xx, n, h->stream));
    OS_TRY(upload(eyy, eps_yy, n, h->stream));
    if (sigma_e && !lossless) OS_TRY(upload(sig, sigma_e, n, h->stream));
    OS_TRY(h->cb.alloc(n));
    OS_TRY(h->cb_y.alloc(n));
    if (!lossless) {
        OS_TRY(h->ca.alloc(n));
        OS_TRY(h->ca_y.alloc(n));
    }
    const float *sh = h->shares.ptr;
    const dim3 block(EZ2D_BLOCK_X, EZ2D_BLOCK_Y);
    const dim3 grid_dim((unsigned)((ny + block.x - 1) / block.x), (unsigned)((nx + block.y - 1) / block.y));
    hz2d_face_coefficients_kernel<<<grid_dim, block, 0, h->stream>>>(
        exx.ptr, eyy.ptr, sig.ptr, sh, sh + nx, sh + 2 * nx, sh + 2 * nx + ny, nx, ny, h->grid.periodic_x,
        h->grid.periodic_y, dt, eps0, lossless ? nullptr : h->ca.ptr, h->cb.ptr, lossless ? nullptr : h->ca_y.ptr,
        h->cb_y.ptr);
    OS_CUDA(cudaGetLastError());
    h->has_ca = !lossless;
    h->has_cb = true;
    h->hz_eps = eps_form;
    h->dt_hz = dt;
    h->eps0_hz = eps0;
    if (eps_form) {
        OS_TRY(h->eps_cell.alloc(n));
        OS_CUDA(cudaMemcpyAsync(h->eps_cell.ptr, exx.ptr, n * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    }
    if (mu_r || sigma_m) {
        if (mu_r) OS_TRY(upload(mu_dev, mu_r, n, h->stream));
        if (sigma_m) OS_TRY(upload(sm_dev, sigma_m, n, h->stream));
        OS_TRY(h->da.alloc(n));
        OS_TRY(h->db.alloc(n));
        const unsigned blocks = (unsigned)((n + 255) / 256);
        ez2d_h_coefficients_kernel<<<blocks, 256, 0, h->stream>>>(mu_dev.ptr, sm_dev.ptr, dt, mu0, n, h->da.ptr,
                                                                  h->db.ptr);
        OS_CUDA(cudaGetLastError());
        h->has_dadb = true;
    } else {
        // vacuum permeability: da = (1 - 0) / 1, db = (dt / mu0) / 1 (fdtd_ez_2d_kernels.py:335-340)
        const float mu = 1.0f * mu0;
        const float k = (0.0f * dt) / (2.0f * mu);
        const float denom = 1.0f + k;
        h->da_uniform = (1.0f - k) / denom;
        h->db_uniform = (dt / mu) / denom;
        h->has_dadb = false;
    }
    give_after(h->stream, exx, eyy, sig, mu_dev, sm_dev);
    return OS_OK;
}

extern "C" int os_fdtd2d_hz_read_cb(OsFdtd2D *h, float *cb_x, float *cb_y) {
    OS_TRY(require_hz(h, "os_fdtd2d_hz_read_cb"));
    OS_CHECK(cb_x && cb_y, OS_ERR_INVALID, "os_fdtd2d_hz_read_cb: null argument");
    OS_CHECK(h->has_cb, OS_ERR_STATE, "os_fdtd2d_hz_read_cb: materials are not set");
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(cb_x, h->cb.ptr, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaMemcpyAsync(cb_y, h->cb_y.ptr, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd2d_hz_form(OsFdtd2D *h, int32_t *lossless_form) {
    OS_TRY(require_hz(h, "os_fdtd2d_hz_form"));
    OS_CHECK(lossless_form, OS_ERR_INVALID, "os_fdtd2d_hz_form: null argument");
    *lossless_form = h->hz_eps ? 1 : 0;
    return OS_OK;
}

extern "C" int os_fdtd2d_set_cpml_side(OsFdtd2D *h, int32_t side, const float *b_e, const float *a_e,
                                       const float *inv_e, const float *b_h, const float *a_h, const float *inv_h) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_cpml_side: null handle");
    int s = -1;
    for (int k = 0; k < 4; ++k)
        if (side == (1 << k)) s = k;
    OS_CHECK(s >= 0, OS_ERR_INVALID, "os_fdtd2d_set_cpml_side: side %d is not one OS_SIDE_* bit of a 2D face", side);
    OS_CHECK(h->grid.cpml_sides & side, OS_ERR_INVALID, "os_fdtd2d_set_cpml_side: side %d is not a CPML face", side);
    OS_CHECK(b_e && a_e && inv_e && b_h && a_h && inv_h, OS_ERR_INVALID, "os_fdtd2d_set_cpml_side: null row");
    OS_TRY(bind_device(h));
    const size_t npml = (size_t)h->grid.npml;
    const float *rows[6] = {b_e, a_e, inv_e, b_h, a_h, inv_h};
    for (int r = 0; r < 6; ++r)
        OS_CUDA(cudaMemcpyAsync(h->cpml_rows[s].ptr + r * npml, rows[r], npml * sizeof(float), cudaMemcpyHostToDevice,
                                h->stream));
    h->cpml_set[s] = true;
    return OS_OK;
}

extern "C" int os_fdtd2d_add_line_source(OsFdtd2D *h, int32_t axis, int32_t position, int32_t lo, int32_t hi,
                                         const float *profile, int32_t *source_id) {
    OS_CHECK(h && profile, OS_ERR_INVALID, "os_fdtd2d_add_line_source: null argument");
    OS_CHECK(axis == 0 || axis == 1, OS_ERR_INVALID, "LineSource axis must be 'x' or 'y', got %d", axis);
    OS_CHECK(h->lines.size() < (size_t)OS_MAX_LINES_2D, OS_ERR_INVALID, "at most %d line sources per engine",
             OS_MAX_LINES_2D);
    const int n_along = axis == 0 ? h->grid.nx : h->grid.ny;
    const int n_across = axis == 0 ? h->grid.ny : h->grid.nx;
    OS_CHECK(0 <= lo && lo < hi && hi <= n_along, OS_ERR_INVALID,
             "LineSource span must be a half-open cell range lo < hi inside the grid, got (%d, %d)", lo, hi);
    OS_CHECK(0 <= position && position < n_across, OS_ERR_INVALID, "LineSource position %d outside the grid", position);
    OS_TRY(bind_device(h));
    std::unique_ptr<LineSource2D> src(new LineSource2D());
    src->axis = axis;
    src->position = position;
    src->lo = lo;
    src->hi = hi;
    OS_TRY(upload(src->profile, profile, (size_t)(hi - lo), h->stream));
    if (source_id) *source_id = (int32_t)h->lines.size();
    h->lines.push_back(std::move(src));
    return OS_OK;
}

extern "C" int os_fdtd2d_set_line_profile(OsFdtd2D *h, int32_t source_id, const float *profile) {
    OS_CHECK(h && profile, OS_ERR_INVALID, "os_fdtd2d_set_line_profile: null argument");
    OS_CHECK(source_id >= 0 && (size_t)source_id < h->lines.size(), OS_ERR_INVALID, "no line source %d", source_id);
    OS_TRY(bind_device(h));
    LineSource2D &src = *h->lines[source_id];
    OS_TRY(upload(src.profile, profile, (size_t)(src.hi - src.lo), h->stream));
    return OS_OK;
}

extern "C" int os_fdtd2d_add_flux_line(OsFdtd2D *h, int32_t normal_axis, int32_t position, int32_t lo, int32_t hi,
                                       int32_t nf, int32_t *monitor_id) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_add_flux_line: null handle");
    OS_CHECK(normal_axis == 0 || normal_axis == 1, OS_ERR_INVALID, "FluxMonitor axis must be 'x' or 'y'");
    const int n_along = normal_axis == 0 ? h->grid.ny : h->grid.nx;
    const int n_across = normal_axis == 0 ? h->grid.nx : h->grid.ny;
    OS_CHECK(0 <= lo && lo < hi && hi <= n_along, OS_ERR_INVALID,
             "FluxMonitor span must be a half-open cell range lo < hi, got (%d, %d)", lo, hi);
    OS_CHECK(0 <= position && position < n_across, OS_ERR_INVALID, "FluxMonitor position %d outside the grid",
             position);
    OS_CHECK(nf >= 1, OS_ERR_INVALID, "monitor frequencies must be a non-empty list");
    OS_CHECK(h->fluxes.size() < (size_t)TB_MAX_MONS, OS_ERR_INVALID, "at most %d flux lines per engine", TB_MAX_MONS);
    OS_TRY(bind_device(h));
    std::unique_ptr<FluxLine2D> m(new FluxLine2D());
    m->normal_axis = normal_axis;
    m->position = position;
    m->lo = lo;
    m->hi = hi;
    m->nf = nf;
    const size_t n = (size_t)nf * (size_t)(hi - lo) * 2;
    OS_TRY(m->e_acc.alloc(n));
    OS_TRY(m->h_acc.alloc(n));
    OS_TRY(m->stage.alloc((size_t)TB_MAX_T * 2 * (size_t)(hi - lo)));
    OS_CUDA(cudaMemsetAsync(m->e_acc.ptr, 0, m->e_acc.bytes(), h->stream));
    OS_CUDA(cudaMemsetAsync(m->h_acc.ptr, 0, m->h_acc.bytes(), h->stream));
    if (monitor_id) *monitor_id = (int32_t)h->fluxes.size();
    h->fluxes.push_back(std::move(m));
    return OS_OK;
}

extern "C" int os_fdtd2d_set_sample_interval(OsFdtd2D *h, int64_t sample_interval) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_sample_interval: null handle");
    OS_CHECK(sample_interval >= 1, OS_ERR_INVALID, "sample_interval must be >= 1, got %lld", (long long)sample_interval);
    h->sample_interval = sample_interval;
    return OS_OK;
}

namespace os {

// Event pair around one kernel launch when profiling (kind: 0 interior, 1 general, 2 DFT, 3 per-step kernels).
static int prof_begin(OsFdtd2D *h, int kind, cudaStream_t stream) {
    if (!h->profiling) return OS_OK;
    while (h->prof_events.size() < 2 * (h->prof_used + 1)) {
        cudaEvent_t e;
        OS_CUDA(cudaEventCreate(&e));
        h->prof_events.push_back(e);
    }
    if (h->prof_kind.size() < h->prof_used + 1) h->prof_kind.resize(h->prof_used + 1);
    h->prof_kind[h->prof_used] = kind;
    OS_CUDA(cudaEventRecord(h->prof_events[2 * h->prof_used], stream));
    return OS_OK;
}

static int prof_end(OsFdtd2D *h, cudaStream_t stream) {
    if (!h->profiling) return OS_OK;
    OS_CUDA(cudaEventRecord(h->prof_events[2 * h->prof_used + 1], stream));
    h->prof_used += 1;
    return OS_OK;
}

struct Rect {
    int r0, r1, c0, c1;
};

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Tiles of one kernel: rectangles cut into tile_w x tile_rows output tiles (one warp each).
static void set_tiles(TBParams &q, const std::vector<Rect> &rects, int tile_w, int tile_rows) {
    q.n_rects = 0;
    int first = 0;
    for (const Rect &r : rects) {
        if (r.r1 <= r.r0 || r.c1 <= r.c0) continue;
        TBRect &t = q.rects[q.n_rects++];
        t.r0 = r.r0;
        t.r1 = r.r1;
        t.c0 = r.c0;
        t.c1 = r.c1;
        t.tiles_c = (r.c1 - r.c0 + tile_w - 1) / tile_w;
        t.first_tile = first;
        first += t.tiles_c * ((r.r1 - r.r0 + tile_rows - 1) / tile_rows);
    }
    q.tile_w = tile_w;
    q.tile_rows = tile_rows;
    q.n_tiles = first;
}

static bool constant_over(const std::vector<float> &v, int a, int b, float *value) {
    if (a < 0 || b > (int)v.size() || a >= b) return false;
    for (int k = a; k < b; ++k)
        if (v[k] != v[a]) return false;
    *value = v[a];
    return true;
}

// The interior rectangle (cells whose T-step dependency cone avoids the CPML slabs and the non-periodic edges) and the
// border rectangles around it.  Interior rows need i0 - T >= npml + 1 and i1 - 1 + T <= nx - npml - 2 on a CPML x
// axis; columns likewise with the 4-column left halo of the 128-bit loads.
// Rows per interior tile when the choice is left to the plan (tile_rows 0), for one or several interior rectangles
// (rows x columns) sharing a launch: each warp streams its tile's rows one after the other and blocks of 4 warps
// run in waves of 4 per SM, so the launch takes about (whole waves) x (tile rows + the 2 T cone rows + 4 rows of
// pipeline start).  The height in 8..128 that minimises that (the taller one on a tie).
static int wave_rows(int sm_count, int T, const std::vector<std::pair<int, int>> &rects) {
    const int64_t slots = (int64_t)sm_count * 4;
    int best = 128;
    int64_t best_cost = -1;
    for (int R = 128; R >= 8; R -= 4) {
        int64_t tiles = 0;
        for (const auto &rc : rects) tiles += (int64_t)((rc.first + R - 1) / R) * ((rc.second + 119) / 120);
        const int64_t blocks = (tiles + TB_WARPS - 1) / TB_WARPS;
        const int64_t waves = (blocks + slots - 1) / slots;
        const int64_t cost = waves * (R + 2 * T + 4);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = R;
        }
    }
    return best;
}

static int interior_rows(const OsFdtd2D *h, int T, int rows, int cols, int rows_override = 0) {
    if (rows_override > 0) return rows_override;
    if (h->tile_rows > 0) return h->tile_rows;
    if (rows <= 0 || cols <= 0) return 128;
    return wave_rows(h->sm_count, T, {{rows, cols}});
}

// The interior rectangle of the blocked kernels (rows [r0, r1), columns [c0, c1)), or false when there is none.
static bool interior_rect(const OsFdtd2D *h, int T, Rect &in);

static void plan_tiles(const OsFdtd2D *h, int T, TBParams &interior, TBParams &general, bool &has_interior,
                       int rows_override = 0) {
    const OsGrid2D &g = h->grid;
    const int npml = g.npml;
    const bool cx = (g.cpml_sides & 3) != 0, cy = (g.cpml_sides & 12) != 0;
    Rect in{0, g.nx, 0, g.ny};
    if (!g.periodic_x) {
        in.r0 = cx ? npml + 1 + T : g.nx;
        in.r1 = cx ? g.nx - npml - 1 - T : 0;
    }
    if (!g.periodic_y) {
        in.c0 = cy ? round_up(npml + 1 + 4, 4) : g.ny;
        in.c1 = cy ? g.ny - npml - 1 - T : 0;
    }
    // a row length that is not a multiple of 4 staggers the rows' 16-byte alignment: the interior kernel copies
    // each row window from the boundary before it, which a periodic y (a window wrapping into two copies) does not
    // allow
    has_interior = h->variant == 1 && in.r1 > in.r0 && in.c1 > in.c0 && (g.ny % 4 == 0 || !g.periodic_y) &&
                   !h->has_dadb && h->da_uniform == 1.0f;
    // uniform curl spacings over the interior's dependency cone (rows [r0 - T, r1 + T), columns [c0 - 4, c1 + T));
    // the columns a tile loads beyond its cone feed no output and may be anything
    if (has_interior) {
        const int ra = g.periodic_x ? 0 : in.r0 - T, rb = g.periodic_x ? g.nx : in.r1 + T;
        const int ca = g.periodic_y ? 0 : in.c0 - 4, cbnd = g.periodic_y ? g.ny : in.c1 + T;
        has_interior = constant_over(h->host_inv[0], ra, rb, &interior.s_inv_dx_e) &&
                       constant_over(h->host_inv[1], ra, rb, &interior.s_inv_dx_h) &&
                       constant_over(h->host_inv[2], ca, cbnd, &interior.s_inv_dy_e) &&
                       constant_over(h->host_inv[3], ca, cbnd, &interior.s_inv_dy_h);
    }
    std::vector<Rect> border;
    if (!has_interior) {
        border.push_back(Rect{0, g.nx, 0, g.ny});
        set_tiles(interior, {}, 120, interior_rows(h, T, 0, 0, rows_override));
    } else {
        border.push_back(Rect{0, in.r0, 0, g.ny});
        border.push_back(Rect{in.r1, g.nx, 0, g.ny});
        border.push_back(Rect{in.r0, in.r1, 0, in.c0});
        border.push_back(Rect{in.r0, in.r1, in.c1, g.ny});
        set_tiles(interior, {in}, 120, interior_rows(h, T, in.r1 - in.r0, in.c1 - in.c0, rows_override));
    }
    set_tiles(general, border, 32 - 2 * T, h->gen_tile_rows);
}

static bool interior_rect(const OsFdtd2D *h, int T, Rect &in) {
    TBParams a{}, b{};
    bool has = false;
    plan_tiles(h, T, a, b, has, 128);
    if (!has || !a.n_tiles) return false;
    in = Rect{a.rects[0].r0, a.rects[0].r1, a.rects[0].c0, a.rects[0].c1};
    return true;
}

static void fill_common(const OsFdtd2D *h, TBParams &q) {
    const OsGrid2D &g = h->grid;
    q.nx = g.nx;
    q.ny = g.ny;
    q.px = g.periodic_x;
    q.py = g.periodic_y;
    q.npml = g.npml;
    q.cpml_mask = g.cpml_sides;
    q.cb = h->cb.ptr;
    q.ca = h->has_ca ? h->ca.ptr : nullptr;
    q.da = h->has_dadb ? h->da.ptr : nullptr;
    q.db = h->has_dadb ? h->db.ptr : nullptr;
    q.da_u = h->da_uniform;
    q.db_u = h->db_uniform;
    q.inv_dx_e = h->inv_dx_e.ptr;
    q.inv_dx_h = h->inv_dx_h.ptr;
    q.inv_dy_e = h->inv_dy_e.ptr;
    q.inv_dy_h = h->inv_dy_h.ptr;
    for (int s = 0; s < 4; ++s) q.cpml_rows[s] = h->cpml_rows[s].ptr;
    q.n_lines = (int32_t)h->lines.size();
    for (size_t l = 0; l < h->lines.size(); ++l) {
        q.lines[l].axis = h->lines[l]->axis;
        q.lines[l].position = h->lines[l]->position;
        q.lines[l].lo = h->lines[l]->lo;
        q.lines[l].hi = h->lines[l]->hi;
        q.lines[l].profile = h->lines[l]->profile.ptr;
    }
    q.line_values = h->line_values.ptr;
    q.n_mons = (int32_t)h->fluxes.size();
    for (size_t k = 0; k < h->fluxes.size(); ++k) {
        q.mons[k].normal_axis = h->fluxes[k]->normal_axis;
        q.mons[k].position = h->fluxes[k]->position;
        q.mons[k].lo = h->fluxes[k]->lo;
        q.mons[k].hi = h->fluxes[k]->hi;
        q.mons[k].stage = h->fluxes[k]->stage.ptr;
    }
    q.m = h->sample_interval;
    q.err = h->err.ptr;
    q.stall_probe_ns = h->stall_probe_ns;
}

template <int T, bool CA, bool PX, bool PY, bool VEC>
static int launch_interior(OsFdtd2D *h, const TBParams &q) {
    const size_t smem = (size_t)TB_WARPS * ip_warp_smem_bytes(T, CA);
    static bool attr_set = false;   // one flag per instantiation
    if (!attr_set) {
        OS_CUDA(cudaFuncSetAttribute(ez2d_interior_kernel<T, CA, PX, PY, VEC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    const dim3 blocks((unsigned)((q.n_tiles + TB_WARPS - 1) / TB_WARPS)), threads(TB_WARPS * 32);
    ez2d_interior_kernel<T, CA, PX, PY, VEC><<<blocks, threads, smem, h->stream>>>(q);
    return OS_OK;
}

// ny % 4 == 0 selects the aligned kernels; a row length that is not a multiple of 4 only ever has an interior with a
// non-periodic y (plan_tiles)
template <int T, bool CA>
static int launch_interior_ca(OsFdtd2D *h, const TBParams &q) {
    const bool px = h->grid.periodic_x != 0, py = h->grid.periodic_y != 0, vec = h->grid.ny % 4 == 0;
    if (!vec) return px ? launch_interior<T, CA, true, false, false>(h, q) : launch_interior<T, CA, false, false, false>(h, q);
    if (px && py) return launch_interior<T, CA, true, true, true>(h, q);
    if (px) return launch_interior<T, CA, true, false, true>(h, q);
    if (py) return launch_interior<T, CA, false, true, true>(h, q);
    return launch_interior<T, CA, false, false, true>(h, q);
}

template <int T>
static int launch_interior_any(OsFdtd2D *h, const TBParams &q) {
    return h->has_ca ? launch_interior_ca<T, true>(h, q) : launch_interior_ca<T, false>(h, q);
}

// The staging slot of frame step k (1..T) of a launch with the sample mask of `q` (-1: not a staging step).
static void set_frame_slots(EzFrameParams &f, const TBParams &q, int k) {
    f.sample_slot = ((q.sample_mask >> (k - 1)) & 1u) ? __builtin_popcount(q.sample_mask & ((1u << (k - 1)) - 1u)) : -1;
}

// Parameters of frame step k (1..T) of one blocked launch of T steps from buffer set in_set to out_set: the region
// is the grid minus the interior rectangle `in` (NULL: none) shrunk by T - k cells on each non-periodic side; it
// reads the state of step k - 1 (the input set for k = 1, else a scratch set) and writes that of step k (a scratch
// set, the output set for k = T).  `q` carries the launch's sources, monitors, sample mask and first value column.
static EzFrameParams make_frame_params(const OsFdtd2D *h, int T, int k, const TBParams &q, const Rect *in, int in_set,
                                       int out_set) {
    const OsGrid2D &g = h->grid;
    EzFrameParams f{};
    f.nx = g.nx, f.ny = g.ny, f.px = g.periodic_x, f.py = g.periodic_y, f.npml = g.npml;
    f.cpml_mask = g.cpml_sides;
    f.ca = q.ca, f.cb = q.cb, f.da = q.da, f.db = q.db, f.da_u = q.da_u, f.db_u = q.db_u;
    f.inv_dx_e = q.inv_dx_e, f.inv_dx_h = q.inv_dx_h, f.inv_dy_e = q.inv_dy_e, f.inv_dy_h = q.inv_dy_h;
    const bool from_io = k == 1, to_io = k == T;
    const int src = (k - 2) % 2, dst = (k - 1) % 2;
    f.ez_in = from_io ? h->ez[in_set].ptr : h->sez[src].ptr;
    f.hx_in = from_io ? h->hx[in_set].ptr : h->shx[src].ptr;
    f.hy_in = from_io ? h->hy[in_set].ptr : h->shy[src].ptr;
    f.ez_out = to_io ? h->ez[out_set].ptr : h->sez[dst].ptr;
    f.hx_out = to_io ? h->hx[out_set].ptr : h->shx[dst].ptr;
    f.hy_out = to_io ? h->hy[out_set].ptr : h->shy[dst].ptr;
    for (int sd = 0; sd < 4; ++sd) {
        f.cpml_rows[sd] = q.cpml_rows[sd];
        f.psi_e_in[sd] = from_io ? h->psi_e[in_set][sd].ptr : h->spsi_e[src][sd].ptr;
        f.psi_h_in[sd] = from_io ? h->psi_h[in_set][sd].ptr : h->spsi_h[src][sd].ptr;
        f.psi_e_out[sd] = to_io ? h->psi_e[out_set][sd].ptr : h->spsi_e[dst][sd].ptr;
        f.psi_h_out[sd] = to_io ? h->psi_h[out_set][sd].ptr : h->spsi_h[dst][sd].ptr;
    }
    f.n_lines = q.n_lines;
    for (int l = 0; l < q.n_lines; ++l) f.lines[l] = q.lines[l];
    f.line_values = q.line_values;
    f.values_stride = q.values_stride;
    f.k_col = q.k0 + (k - 1);
    f.n_mons = q.n_mons;
    for (int m = 0; m < q.n_mons; ++m) f.mons[m] = q.mons[m];
    set_frame_slots(f, q, k);
    Rect sh{0, 0, 0, 0};
    if (in) {
        f.in_r0 = in->r0, f.in_r1 = in->r1, f.in_c0 = in->c0, f.in_c1 = in->c1;
        const int w = T - k;
        sh = *in;
        if (!g.periodic_x) sh.r0 += w, sh.r1 -= w;
        if (!g.periodic_y) sh.c0 += w, sh.c1 -= w;
    }
    Rect region[4];
    int n_region = 0;
    if (sh.r1 > sh.r0 && sh.c1 > sh.c0) {
        region[n_region++] = Rect{0, sh.r0, 0, g.ny};
        region[n_region++] = Rect{sh.r1, g.nx, 0, g.ny};
        region[n_region++] = Rect{sh.r0, sh.r1, 0, sh.c0};
        region[n_region++] = Rect{sh.r0, sh.r1, sh.c1, g.ny};
    } else {
        region[n_region++] = Rect{0, g.nx, 0, g.ny};
    }
    f.n_rects = 0;
    f.first[0] = 0;
    for (int r = 0; r < n_region; ++r) {
        const Rect &rc = region[r];
        if (rc.r1 <= rc.r0 || rc.c1 <= rc.c0) continue;
        const int n = f.n_rects++;
        f.r0[n] = rc.r0, f.r1[n] = rc.r1, f.c0[n] = rc.c0, f.c1[n] = rc.c1;
        f.first[n + 1] = f.first[n] + (int64_t)(rc.r1 - rc.r0) * (rc.c1 - rc.c0);
    }
    return f;
}

// Blocks of 256 threads (one per cell) of a frame step launch.
static int64_t frame_blocks(const EzFrameParams &f) { return (f.first[f.n_rects] + 255) / 256; }

// The frame of one blocked launch of T steps: T single-step launches of ez2d_frame_step_kernel on stream `s`.
// `tmpl` (NULL: built here) holds the launch's T step parameters for its buffer parity, made by make_frame_params
// from the same plan; only the value column and the sample slot of each step are set here from `q`.
static int launch_frame_chain(OsFdtd2D *h, int T, const TBParams &q, const Rect *in, cudaStream_t s,
                              const EzFrameParams *tmpl) {
    for (int k = 1; k <= T; ++k) {
        EzFrameParams f = tmpl ? tmpl[k - 1] : make_frame_params(h, T, k, q, in, h->cur, h->cur ^ 1);
        f.line_values = q.line_values;
        f.values_stride = q.values_stride;
        f.k_col = q.k0 + (k - 1);
        set_frame_slots(f, q, k);
        if (f.first[f.n_rects] == 0) continue;
        OS_TRY(prof_begin(h, 1, s));
        ez2d_frame_step_kernel<<<(unsigned)frame_blocks(f), 256, 0, s>>>(f);
        OS_TRY(prof_end(h, s));
        h->launches += 1;
    }
    return OS_OK;
}

// One blocked launch: the border (general) kernel forks onto the side stream and overlaps the interior kernel; both
// read the same input buffers and write disjoint cells of the output buffers, and the main stream waits for both.
template <int T>
static int launch_tb(OsFdtd2D *h, const TBParams &interior, const TBParams &general, bool has_interior,
                     const EzFrameParams *frame_tmpl = nullptr) {
    const dim3 threads(TB_WARPS * 32);
    const bool run_interior = has_interior && interior.n_tiles;
    // profiling: no fork, so that each event pair times one kernel alone (shares as in a serialised launch list)
    const bool fork = run_interior && general.n_tiles && !h->profiling;
    cudaStream_t gstream = fork ? h->side_stream : h->stream;
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_fork, h->stream));
        OS_CUDA(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    }
    if (general.n_tiles && h->variant == 1) {
        // the frame: one single-step launch per step over the shrinking band around the interior
        Rect in{};
        if (run_interior) in = Rect{interior.rects[0].r0, interior.rects[0].r1, interior.rects[0].c0,
                                    interior.rects[0].c1};
        OS_TRY(launch_frame_chain(h, T, general, run_interior ? &in : nullptr, gstream, frame_tmpl));
    } else if (general.n_tiles) {
        const dim3 blocks((unsigned)((general.n_tiles + TB_WARPS - 1) / TB_WARPS));
        OS_TRY(prof_begin(h, 1, gstream));
        if (h->has_ca) ez2d_tb_kernel<T, 1, true, true><<<blocks, threads, 0, gstream>>>(general);
        else ez2d_tb_kernel<T, 1, true, false><<<blocks, threads, 0, gstream>>>(general);
        OS_TRY(prof_end(h, gstream));
        h->launches += 1;
    }
    if (run_interior) {
        OS_TRY(prof_begin(h, 0, h->stream));
        OS_TRY(launch_interior_any<T>(h, interior));
        OS_TRY(prof_end(h, h->stream));
        h->launches += 1;
    }
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_join, h->side_stream));
        OS_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

static int launch_tb_any(OsFdtd2D *h, int T, const TBParams &interior, const TBParams &general, bool has_interior,
                         const EzFrameParams *frame_tmpl = nullptr) {
    switch (T) {
        case 1: return launch_tb<1>(h, interior, general, has_interior, frame_tmpl);
        case 2: return launch_tb<2>(h, interior, general, has_interior, frame_tmpl);
        case 3: return launch_tb<3>(h, interior, general, has_interior, frame_tmpl);
        default: return launch_tb<4>(h, interior, general, has_interior, frame_tmpl);
    }
}

// Input / output buffer sets of one launch from buffer `in` to buffer `out`.
static void bind_buffers(OsFdtd2D *h, TBParams &q, int in, int out) {
    q.ez_in = h->ez[in].ptr;
    q.hx_in = h->hx[in].ptr;
    q.hy_in = h->hy[in].ptr;
    q.ez_out = h->ez[out].ptr;
    q.hx_out = h->hx[out].ptr;
    q.hy_out = h->hy[out].ptr;
    for (int s = 0; s < 4; ++s) {
        q.psi_e_in[s] = h->psi_e[in][s].ptr;
        q.psi_h_in[s] = h->psi_h[in][s].ptr;
        q.psi_e_out[s] = h->psi_e[out][s].ptr;
        q.psi_h_out[s] = h->psi_h[out][s].ptr;
    }
}

// Temporally blocked chunk: launches of T steps (a shorter last one), buffers swapped after each.  `values` and
// `phase_table` are the chunk's device tables (source values, DFT phases).
// Floats of a chunk's phase table: per flux line, then per field map, (n_samples, nf) complex64 phases.
static size_t phase_floats_of(const OsFdtd2D *h, int64_t n_samples) {
    size_t n = 0;
    for (auto &f : h->fluxes) n += (size_t)n_samples * f->nf * 2;
    for (auto &d : h->maps) n += (size_t)n_samples * d->nf * 2 * (d->hz ? 2 : 1);
    return n;
}

// The field maps' DFT of sample q, from the E_z of buffer set `set` (the state right after the sample step).
static int fold_maps(OsFdtd2D *h, const float *ez, int64_t q, int64_t first_sample, int64_t n_samples,
                     const float *phase_table) {
    size_t offset = 0;
    for (auto &f : h->fluxes) offset += (size_t)n_samples * f->nf * 2;
    for (auto &d : h->maps) {
        const float *ph = phase_table + offset + (size_t)(q - first_sample) * d->nf * 2;
        const int64_t total = (int64_t)d->nf * d->mx * d->my;
        OS_TRY(prof_begin(h, 2, h->stream));
        if (d->hz) {   // E-time phases, then the H_z phases at t - dt/2
            const float *ph_h = ph + (size_t)n_samples * d->nf * 2;
            const int c = h->cur;
            hz2d_dft_map_kernel<<<(unsigned)((total + 255) / 256), 256, 0, h->stream>>>(
                h->ez[c].ptr, h->hx[c].ptr, h->hy[c].ptr, h->grid.nx, h->grid.ny, h->grid.periodic_x,
                h->grid.periodic_y, d->x0, d->y0, d->ds, d->mx, d->my, d->nf, ph, ph_h, d->acc.ptr);
        } else {
            ez2d_dft_map_kernel<<<(unsigned)((total + 255) / 256), 256, 0, h->stream>>>(
                ez, h->grid.ny, d->x0, d->y0, d->ds, d->mx, d->my, d->nf, ph, d->acc.ptr);
        }
        OS_TRY(prof_end(h, h->stream));
        h->launches += 1;
        offset += (size_t)n_samples * d->nf * 2 * (d->hz ? 2 : 1);
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// The probes' values after step `row` + 1 from the buffer set `set` (FieldProbe.record at t_full,
// fdtd_2d_base.py:481-487).  One warp.
__global__ void ez2d_probe_kernel(ProbeSet ps, const float *f0, const float *f1, const float *f2, int ny, float *rows,
                                  int64_t capacity, int64_t row) {
    const int k = threadIdx.x;
    if (k >= ps.n || row < ps.start[k]) return;
    const float *f = ps.comp[k] == 0 ? f0 : ps.comp[k] == 1 ? f1 : f2;
    rows[(size_t)k * capacity + row] = f[(size_t)ps.ix[k] * ny + ps.iy[k]];
}

static int record_probes(OsFdtd2D *h) {
    const int c = h->cur;
    OS_TRY(prof_begin(h, 2, h->stream));
    ez2d_probe_kernel<<<1, 32, 0, h->stream>>>(h->probes, h->ez[c].ptr, h->hx[c].ptr, h->hy[c].ptr, h->grid.ny,
                                                h->probe_rows.ptr, h->probe_capacity, h->n_step - 1);
    OS_TRY(prof_end(h, h->stream));
    h->launches += 1;
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// The probes' values after steps n0 + 1 .. n0 + T of a blocked launch, from the cells the launch's kernels staged
// (slot s - 1 of step s: E_z, then the tangential H: H_y of a cell staged as an x-normal line, H_x as a y-normal
// one).  Thread k * TB_MAX_T + s: probe k, step s + 1.
__global__ void ez2d_probe_staged_kernel(ProbeSet ps, const float *stage, float *rows, int64_t capacity, int64_t n0,
                                         int T) {
    const int k = threadIdx.x / TB_MAX_T, s = threadIdx.x % TB_MAX_T;
    if (k >= ps.n || s >= T) return;
    const int64_t row = n0 + s;
    if (row < ps.start[k]) return;
    rows[(size_t)k * capacity + row] = stage[((size_t)k * TB_MAX_T + s) * 2 + (ps.comp[k] == 0 ? 0 : 1)];
}

static int record_probes_staged(OsFdtd2D *h, int T, int64_t n0) {
    OS_TRY(prof_begin(h, 2, h->stream));
    ez2d_probe_staged_kernel<<<1, OS_MAX_PROBES * TB_MAX_T, 0, h->stream>>>(h->probes, h->probe_stage.ptr,
                                                                             h->probe_rows.ptr, h->probe_capacity,
                                                                             n0, T);
    OS_TRY(prof_end(h, h->stream));
    h->launches += 1;
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// The field probes as monitors of the blocked E_z kernels, after the flux lines: each probe's cell is a staged line of
// one cell (E_z and H_y probes x-normal, whose stage holds E_z then H_y; H_x probes y-normal, E_z then H_x).  A launch
// with probes marks every step as a staging step, so the kernels stage step s in slot s - 1 and the flux lines' DFT
// reads its sample steps' slots from there.
static bool probes_fit_mons(const OsFdtd2D *h) {
    return h->probe_stage.ptr && h->fluxes.size() + (size_t)h->probes.n <= (size_t)TB_MAX_MONS;
}
static void add_probe_mons(const OsFdtd2D *h, TBParams &q) {
    for (int k = 0; k < h->probes.n; ++k) {
        TBMon &M = q.mons[q.n_mons++];
        const bool hx = h->probes.comp[k] == 1;
        M.normal_axis = hx ? 1 : 0;
        M.position = hx ? h->probes.iy[k] : h->probes.ix[k];
        M.lo = hx ? h->probes.ix[k] : h->probes.iy[k];
        M.hi = M.lo + 1;
        M.stage = h->probe_stage.ptr + (size_t)k * TB_MAX_T * 2;
    }
}

// Room for the probes' rows of the next n_steps steps: the rows grow by doubling, the recorded ones copied over on
// the handle's stream and the old block given to the pool behind that copy.
static int reserve_probe_rows(OsFdtd2D *h, int64_t n_steps) {
    if (h->probes.n == 0) return OS_OK;
    const int64_t need = h->n_step + n_steps;
    if (need <= h->probe_capacity) return OS_OK;
    const int64_t cap = std::max<int64_t>(need, std::max<int64_t>(1024, 2 * h->probe_capacity));
    DeviceArray<float> grown;
    OS_TRY(grown.alloc((size_t)OS_MAX_PROBES * (size_t)cap));
    if (h->probe_capacity > 0 && h->n_step > 0)
        OS_CUDA(cudaMemcpy2DAsync(grown.ptr, (size_t)cap * sizeof(float), h->probe_rows.ptr,
                                  (size_t)h->probe_capacity * sizeof(float), (size_t)h->n_step * sizeof(float),
                                  OS_MAX_PROBES, cudaMemcpyDeviceToDevice, h->stream));
    give_after(h->stream, h->probe_rows);
    std::swap(h->probe_rows.ptr, grown.ptr);
    std::swap(h->probe_rows.count, grown.count);
    std::swap(h->probe_rows.capacity, grown.capacity);
    std::swap(h->probe_rows.cls, grown.cls);
    h->probe_capacity = cap;
    return OS_OK;
}

static int advance_blocked(OsFdtd2D *h, int64_t n_steps, int64_t first_sample, int64_t n_samples,
                           const float *values, const float *phase_table) {
    const int64_t m = h->sample_interval;
    const bool staged_probes = h->probes.n > 0 && probes_fit_mons(h);
    // The plan of a launch depends only on its length T (the full steps_per_launch, or a shorter last one): tiles,
    // coefficients, sources, monitors, and the frame steps' regions for both buffer parities.  Each launch then only
    // sets its buffers, first step and sample mask.
    struct LaunchPlan {
        int T = 0;
        TBParams interior{}, general{};
        bool has_interior = false;
        std::vector<EzFrameParams> frame[2];   // [input buffer set][step - 1]
    };
    LaunchPlan plans[TB_MAX_T + 1];   // by T
    auto plan_for = [&](int T) -> LaunchPlan & {
        LaunchPlan &pl = plans[T];
        if (pl.T == T) return pl;
        pl = LaunchPlan{};
        pl.T = T;
        plan_tiles(h, T, pl.interior, pl.general, pl.has_interior);
        fill_common(h, pl.interior);
        fill_common(h, pl.general);
        if (staged_probes) add_probe_mons(h, pl.interior), add_probe_mons(h, pl.general);
        if (h->variant == 1 && pl.general.n_tiles) {
            const bool run_interior = pl.has_interior && pl.interior.n_tiles;
            const Rect box = run_interior ? Rect{pl.interior.rects[0].r0, pl.interior.rects[0].r1,
                                                 pl.interior.rects[0].c0, pl.interior.rects[0].c1}
                                          : Rect{0, 0, 0, 0};
            for (int par = 0; par < 2; ++par)
                for (int k = 1; k <= T; ++k)
                    pl.frame[par].push_back(
                        make_frame_params(h, T, k, pl.general, run_interior ? &box : nullptr, par, par ^ 1));
        }
        return pl;
    };
    int64_t k = 0;
    while (k < n_steps) {
        int T = (int)std::min<int64_t>(h->steps_per_launch, n_steps - k);
        // field maps read E_z between launches: a launch ends on every sample step; field probes are staged by the
        // launch's kernels at every step (one step per launch when they do not fit among the monitors)
        if (!h->maps.empty()) T = (int)std::min<int64_t>(T, m - h->n_step % m);
        if (h->probes.n && !staged_probes) T = 1;
        LaunchPlan &pl = plan_for(T);
        TBParams interior = pl.interior, general = pl.general;
        const int in = h->cur, out = h->cur ^ 1;
        for (TBParams *q : {&interior, &general}) {
            bind_buffers(h, *q, in, out);
            q->line_values = values;
            q->values_stride = n_steps;
            q->k0 = k;
            q->n0 = h->n_step;
            q->q_first = h->n_step / m + 1;
            q->sample_mask = 0;
            for (int st = 1; st <= T; ++st)
                if ((h->n_step + st) % m == 0) q->sample_mask |= 1u << (st - 1);
            if (h->fluxes.empty()) q->sample_mask = 0;
            if (staged_probes) q->sample_mask = (1u << T) - 1u;   // every step staged (slot s - 1)
        }
        OS_TRY(launch_tb_any(h, T, interior, general, pl.has_interior,
                             pl.frame[in].empty() ? nullptr : pl.frame[in].data()));
        h->cur = out;
        // DFT samples taken inside this launch, accumulated in sample order
        const int64_t q_lo = h->n_step / m + 1, q_hi = (h->n_step + T) / m;
        if (!h->fluxes.empty() && q_hi >= q_lo) {
            size_t offset = 0;
            for (auto &f : h->fluxes) {
                const float *ph = phase_table + offset + (size_t)(q_lo - first_sample) * f->nf * 2;
                const int n = f->hi - f->lo;
                const int total = n * f->nf;
                OS_TRY(prof_begin(h, 2, h->stream));
                // sample q_lo is step q_lo * m of the run: its slot, then every m-th, when every step was staged
                const int slot0 = staged_probes ? (int)(q_lo * m - h->n_step - 1) : 0;
                const int stride = staged_probes ? (int)m : 1;
                ez2d_flux_staged_kernel<<<(total + 255) / 256, 256, 0, h->stream>>>(
                    f->stage.ptr, n, f->nf, (int)(q_hi - q_lo + 1), slot0, stride, ph, f->e_acc.ptr, f->h_acc.ptr);
                OS_TRY(prof_end(h, h->stream));
                h->launches += 1;
                offset += (size_t)n_samples * f->nf * 2;
            }
            OS_CUDA(cudaGetLastError());
        }
        if (staged_probes) OS_TRY(record_probes_staged(h, T, h->n_step));
        h->n_step += T;
        k += T;
        if (!h->maps.empty() && h->n_step % m == 0)
            OS_TRY(fold_maps(h, h->ez[h->cur].ptr, h->n_step / m, first_sample, n_samples, phase_table));
        if (h->probes.n && !staged_probes) OS_TRY(record_probes(h));
    }
    return OS_OK;
}

// The poles' J / P updates from E^n (fdtd_ez_2d.py:318-345): the Drude total zeroed on the union box when several
// Drude poles add into it, each Drude pole in add order, then each Lorentz pole.
static int pole_updates(OsFdtd2D *h) {
    const int ny = h->grid.ny, c = h->cur;
    int n_drude = 0;
    for (auto &q : h->poles) n_drude += q->kind == 0;
    const int32_t *u = h->drude_box;
    if (n_drude > 1)
        OS_CUDA(cudaMemset2DAsync(h->jz_total.ptr + (size_t)u[0] * ny + u[2], (size_t)ny * sizeof(float), 0,
                                  (size_t)(u[3] - u[2]) * sizeof(float), (size_t)(u[1] - u[0]), h->stream));
    for (int pass = 0; pass < 2; ++pass)
        for (auto &q : h->poles) {
            if (q->kind != pass) continue;
            const int64_t cells = (int64_t)(q->i1 - q->i0) * (q->j1 - q->j0);
            const unsigned blocks = (unsigned)((cells + 255) / 256);
            if (q->kind == 0)
                ez2d_drude_j_kernel<<<blocks, 256, 0, h->stream>>>(h->ez[c].ptr, ny, q->i0, q->i1, q->j0, q->j1,
                                                                   q->damping, q->drive.ptr, q->a.ptr,
                                                                   h->jz_total.ptr, n_drude == 1);
            else
                ez2d_lorentz_p_kernel<<<blocks, 256, 0, h->stream>>>(h->ez[c].ptr, ny, q->i0, q->i1, q->j0, q->j1,
                                                                     q->damping, q->restoring, q->drive.ptr, q->a.ptr,
                                                                     q->b.ptr);
            h->launches += 1;
        }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// The E corrections after the E update (fdtd_ez_2d.py:347-358): Drude on the union box, then each Lorentz pole.
static int pole_corrections(OsFdtd2D *h) {
    const int ny = h->grid.ny, c = h->cur;
    const int32_t *u = h->drude_box;
    if (u[1] > u[0]) {
        const int64_t cells = (int64_t)(u[1] - u[0]) * (u[3] - u[2]);
        ez2d_pole_correct_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(
            h->ez[c].ptr, ny, u[0], u[1], u[2], u[3], h->cb.ptr, h->jz_total.ptr, nullptr, 0.0f);
        h->launches += 1;
    }
    for (auto &q : h->poles) {
        if (q->kind != 1) continue;
        const int64_t cells = (int64_t)(q->i1 - q->i0) * (q->j1 - q->j0);
        ez2d_pole_correct_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(
            h->ez[c].ptr, ny, q->i0, q->i1, q->j0, q->j1, h->cb.ptr, nullptr, q->b.ptr, h->inv_dt);
        h->launches += 1;
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// H_z engine: J / P of every pole face set from E^n (fdtd_hz_2d.py:286-309), every Drude set in add order, then every
// Lorentz one; the drive array carries drive x face weight.
static int hz_pole_updates(OsFdtd2D *h) {
    const int ny = h->grid.ny, c = h->cur;
    for (int pass = 0; pass < 2; ++pass)
        for (auto &q : h->poles) {
            if (q->kind != pass) continue;
            const float *e = q->comp == 0 ? h->hx[c].ptr : h->hy[c].ptr;
            const int64_t cells = (int64_t)(q->i1 - q->i0) * (q->j1 - q->j0);
            const unsigned blocks = (unsigned)((cells + 255) / 256);
            if (q->kind == 0)
                ez2d_drude_j_kernel<<<blocks, 256, 0, h->stream>>>(e, ny, q->i0, q->i1, q->j0, q->j1, q->damping,
                                                                   q->drive.ptr, q->a.ptr, nullptr, 0);
            else
                ez2d_lorentz_p_kernel<<<blocks, 256, 0, h->stream>>>(e, ny, q->i0, q->i1, q->j0, q->j1, q->damping,
                                                                     q->restoring, q->drive.ptr, q->a.ptr, q->b.ptr);
            h->launches += 1;
        }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// H_z engine: the E corrections after the E update (fdtd_hz_2d.py:311-325), face set by face set: Drude
// E -= cb J (written E - (cb * 1) J, the same bits), then Lorentz E -= cb inv_dt dP, cb of the set's faces.
static int hz_pole_corrections(OsFdtd2D *h) {
    const int ny = h->grid.ny, c = h->cur;
    for (int pass = 0; pass < 2; ++pass)
        for (auto &q : h->poles) {
            if (q->kind != pass) continue;
            float *e = q->comp == 0 ? h->hx[c].ptr : h->hy[c].ptr;
            const float *cb = q->comp == 0 ? h->cb.ptr : h->cb_y.ptr;
            const int64_t cells = (int64_t)(q->i1 - q->i0) * (q->j1 - q->j0);
            ez2d_pole_correct_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, h->stream>>>(
                e, ny, q->i0, q->i1, q->j0, q->j1, cb, nullptr, q->kind == 0 ? q->a.ptr : q->b.ptr,
                q->kind == 0 ? 1.0f : h->inv_dt);
            h->launches += 1;
        }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// Per-half-step chunk (variant 0): H kernel, E kernel, DFT of sample steps; fields updated in place.
static int advance_per_step(OsFdtd2D *h, int64_t n_steps, int64_t first_sample, int64_t n_samples,
                            const float *values, const float *phase_table) {
    const int64_t m = h->sample_interval;
    Ez2DParams p = make_params(h);
    Ez2DParams p_no_lines = p;
    p_no_lines.n_lines = 0;
    const dim3 block(EZ2D_BLOCK_X, EZ2D_BLOCK_Y);
    const dim3 grid((unsigned)((h->grid.ny + block.x - 1) / block.x), (unsigned)((h->grid.nx + block.y - 1) / block.y));
    for (int64_t k = 0; k < n_steps; ++k) {
        OS_TRY(prof_begin(h, 3, h->stream));
        ez2d_h_kernel<<<grid, block, 0, h->stream>>>(p);
        for (auto &t : h->tfsf) {   // TFSFSource.inject_h after the H update (fdtd_ez_2d.py:85-88)
            const int side = std::max(t->x1 - t->x0, t->y1 - t->y0);
            ez2d_tfsf_h_kernel<<<(side + 255) / 256, 256, 0, h->stream>>>(
                p.hx, p.hy, t->aux_ez.ptr, t->x0, t->x1, t->y0, t->y1, t->aux_x0, h->grid.ny, t->coef_h[0],
                t->coef_h[1], t->coef_h[2], t->coef_h[3]);
            ez2d_tfsf_aux_h_kernel<<<(t->aux_n + 255) / 256, 256, 0, h->stream>>>(t->aux_ez.ptr, t->aux_coef_h.ptr,
                                                                                   t->aux_hy.ptr, t->aux_n);
            h->launches += 2;
        }
        if (h->poles.empty()) {
            ez2d_e_kernel<<<grid, block, 0, h->stream>>>(p, values, n_steps, k);
        } else {
            // poles (fdtd_ez_2d.py:263-358): J / P from E^n, the E update (its sources held back), the pole
            // corrections, then the line sources
            OS_TRY(pole_updates(h));
            ez2d_e_kernel<<<grid, block, 0, h->stream>>>(p_no_lines, values, n_steps, k);
            OS_TRY(pole_corrections(h));
            if (p.n_lines) ez2d_line_inject_kernel<<<grid, block, 0, h->stream>>>(p, values, n_steps, k);
            h->launches += 1;
        }
        for (size_t b = 0; b < h->tfsf.size(); ++b) {   // TFSFSource.inject_e at t + dt/2 (fdtd_ez_2d.py:92-99)
            Tfsf2D &t = *h->tfsf[b];
            ez2d_tfsf_e_kernel<<<(t.y1 - t.y0 + 255) / 256, 256, 0, h->stream>>>(
                p.ez, t.aux_hy.ptr, t.x0, t.x1, t.y0, t.y1, t.aux_x0, h->grid.ny, t.coef_e[0], t.coef_e[1]);
            // this step's source value: row n_lines + b of the chunk's value table
            const float *value = values + (h->lines.size() + b) * (size_t)n_steps + (size_t)k;
            ez2d_tfsf_aux_e_kernel<<<1, 256, 0, h->stream>>>(t.aux_ez.ptr, t.aux_hy.ptr, t.aux_n, t.aux_coef_e.ptr,
                                                             t.source_index, value, t.mur_lo, t.mur_hi);
            h->launches += 2;
        }
        OS_TRY(prof_end(h, h->stream));
        h->launches += 2;
        h->n_step += 1;
        if (!h->fluxes.empty() && h->n_step % m == 0) {
            const int64_t q = h->n_step / m;
            size_t offset = 0;
            for (auto &f : h->fluxes) {
                const float *ph = phase_table + offset + (size_t)(q - first_sample) * f->nf * 2;
                const int n = f->hi - f->lo;
                const int total = n * f->nf;
                ez2d_flux_kernel<<<(total + 255) / 256, 256, 0, h->stream>>>(
                    p.ez, f->normal_axis == 0 ? p.hy : p.hx, h->grid.ny, f->normal_axis, f->position, f->lo, n,
                    f->nf, ph, f->e_acc.ptr, f->h_acc.ptr);
                h->launches += 1;
                offset += (size_t)n_samples * f->nf * 2;
            }
        }
        if (!h->maps.empty() && h->n_step % m == 0)
            OS_TRY(fold_maps(h, p.ez, h->n_step / m, first_sample, n_samples, phase_table));
        if (h->probes.n) OS_TRY(record_probes(h));
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// Parameters of the H_z kernels: inputs from buffer set `in`, outputs to `out` (the same set for the in-place
// per-half-step kernels).
static Hz2DParams make_hz_params(const OsFdtd2D *h, int in, int out) {
    Hz2DParams p{};
    p.nx = h->grid.nx;
    p.ny = h->grid.ny;
    p.px = h->grid.periodic_x;
    p.py = h->grid.periodic_y;
    p.npml = h->grid.npml;
    p.hz_in = h->ez[in].ptr;
    p.ex_in = h->hx[in].ptr;
    p.ey_in = h->hy[in].ptr;
    p.hz_out = h->ez[out].ptr;
    p.ex_out = h->hx[out].ptr;
    p.ey_out = h->hy[out].ptr;
    p.ca_x = h->has_ca ? h->ca.ptr : nullptr;
    p.cb_x = h->cb.ptr;
    p.ca_y = h->has_ca ? h->ca_y.ptr : nullptr;
    p.cb_y = h->cb_y.ptr;
    p.da = h->has_dadb ? h->da.ptr : nullptr;
    p.db = h->has_dadb ? h->db.ptr : nullptr;
    p.da_u = h->da_uniform;
    p.db_u = h->db_uniform;
    p.eps = h->eps_cell.ptr;
    p.dt = h->dt_hz;
    p.eps0 = h->eps0_hz;
    const int nx = h->grid.nx, ny = h->grid.ny;
    p.lo_x = h->shares.ptr;
    p.up_x = h->shares.ptr ? h->shares.ptr + nx : nullptr;
    p.lo_y = h->shares.ptr ? h->shares.ptr + 2 * nx : nullptr;
    p.up_y = h->shares.ptr ? h->shares.ptr + 2 * nx + ny : nullptr;
    p.ixe = h->inv_dx_e.ptr;
    p.ixh = h->inv_dx_h.ptr;
    p.iye = h->inv_dy_e.ptr;
    p.iyh = h->inv_dy_h.ptr;
    const int npml = h->grid.npml;
    for (int s = 0; s < 4; ++s) {
        if (!(h->grid.cpml_sides & (1 << s))) continue;
        p.cpml_mask |= 1 << s;
        const float *rows = h->cpml_rows[s].ptr;
        p.b_e[s] = rows;
        p.a_e[s] = rows + npml;
        p.inv_e[s] = rows + 2 * npml;
        p.b_h[s] = rows + 3 * npml;
        p.a_h[s] = rows + 4 * npml;
        p.inv_h[s] = rows + 5 * npml;
        p.psi_e_in[s] = h->psi_e[in][s].ptr;
        p.psi_h_in[s] = h->psi_h[in][s].ptr;
        p.psi_e_out[s] = h->psi_e[out][s].ptr;
        p.psi_h_out[s] = h->psi_h[out][s].ptr;
    }
    p.n_lines = (int32_t)h->lines.size();
    for (size_t l = 0; l < h->lines.size(); ++l) {
        p.lines[l].axis = h->lines[l]->axis;
        p.lines[l].position = h->lines[l]->position;
        p.lines[l].lo = h->lines[l]->lo;
        p.lines[l].hi = h->lines[l]->hi;
        p.lines[l].profile = h->lines[l]->profile.ptr;
    }
    return p;
}

// The fused H_z step's split: the interior box (every H_z / E_x / E_y update plain, columns in groups of 4) and the
// border rectangles around it.
struct HzPlan {
    bool interior = false;
    int ia = 0, ib = 0, jc0 = 0, jc1 = 0;
    HzBorderRects rects{};
};

static HzPlan hz_plan(const OsFdtd2D *h) {
    HzPlan q;
    const int nx = h->grid.nx, ny = h->grid.ny, npml = h->grid.npml, sides = h->grid.cpml_sides;
    // rows [ia, ib) own, row ib the halo: no CPML row among H_z rows ia..ib and E_y rows ia..ib-1, no grid edge
    q.ia = (sides & 1) ? npml + 1 : 1;
    q.ib = (sides & 2) ? nx - npml - 2 : nx - 2;
    int c0 = (sides & 4) ? npml + 1 : 1;
    c0 = (c0 + 3) / 4 * 4;
    const int cmax = (sides & 8) ? ny - npml - 2 : ny - 2;   // the halo column jc1 <= cmax
    q.jc0 = c0;
    q.jc1 = cmax > c0 ? c0 + (cmax - c0) / 4 * 4 : c0;
    q.interior = q.ib > q.ia && q.jc1 > q.jc0;
    int n = 0;
    auto add = [&](int r0, int r1, int cc0, int cc1) {
        if (r1 <= r0 || cc1 <= cc0) return;
        q.rects.r0[n] = r0, q.rects.r1[n] = r1, q.rects.c0[n] = cc0, q.rects.c1[n] = cc1;
        ++n;
    };
    if (q.interior) {
        add(0, q.ia, 0, ny);
        add(q.ib, nx, 0, ny);
        add(q.ia, q.ib, 0, q.jc0);
        add(q.ia, q.ib, q.jc1, ny);
    } else {
        add(0, nx, 0, ny);
    }
    q.rects.n = n;
    q.rects.first[0] = 0;
    for (int k = 0; k < n; ++k)
        q.rects.first[k + 1] =
            q.rects.first[k] + (int64_t)(q.rects.r1[k] - q.rects.r0[k]) * (q.rects.c1[k] - q.rects.c0[k]);
    return q;
}

// Rows per CTA of the interior kernel: about four waves of CTAs over the device's resident slots, 8..64 rows.
static int hz_rows_per_cta(const OsFdtd2D *h, const HzPlan &q) {
    if (h->hz_rows > 0) return h->hz_rows;
    const int64_t warps = (q.jc1 - q.jc0 + 127) / 128;
    const int64_t ctas_x = (warps + HZ_THREADS / 32 - 1) / (HZ_THREADS / 32);
    const int64_t want_ctas = (int64_t)h->sm_count * 6 * 4;
    int64_t rows = ((int64_t)(q.ib - q.ia) * ctas_x + want_ctas - 1) / want_ctas;
    rows = std::max<int64_t>(8, std::min<int64_t>(64, rows));
    return (int)rows;
}

// One fused H_z step: the border kernel forks onto the side stream and overlaps the interior kernel (TMA-staged rows
// for the lossless form on a row length that keeps the copies 16-byte aligned, direct loads otherwise); both read the
// same input buffers and write disjoint cells of the output buffers, and the main stream waits for both.
static int launch_hz_step(OsFdtd2D *h, const HzPlan &q, Hz2DParams p) {
    const bool vec = h->grid.ny % 4 == 0;
    const int64_t border_cells = q.rects.first[q.rects.n];
    const bool fork = q.interior && border_cells > 0 && !h->profiling;   // profiling: each kernel timed alone
    cudaStream_t bstream = fork ? h->side_stream : h->stream;
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_fork, h->stream));
        OS_CUDA(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    }
    if (border_cells > 0) {
        const unsigned blocks = (unsigned)((border_cells + 255) / 256);
        OS_TRY(prof_begin(h, 1, bstream));
        if (h->hz_eps) hz2d_border_kernel<true><<<blocks, 256, 0, bstream>>>(p, q.rects);
        else hz2d_border_kernel<false><<<blocks, 256, 0, bstream>>>(p, q.rects);
        OS_TRY(prof_end(h, bstream));
        h->launches += 1;
    }
    if (q.interior) {
        p.ia = q.ia, p.ib = q.ib, p.jc0 = q.jc0, p.jc1 = q.jc1;
        p.rows_per_cta = hz_rows_per_cta(h, q);
        const int warps = (q.jc1 - q.jc0 + 127) / 128;
        const dim3 grid((unsigned)((warps + HZ_THREADS / 32 - 1) / (HZ_THREADS / 32)),
                        (unsigned)((q.ib - q.ia + p.rows_per_cta - 1) / p.rows_per_cta));
        int32_t *err = h->err.ptr;
        OS_TRY(prof_begin(h, 0, h->stream));
        if (h->hz_eps && vec) {
            hz2d_interior_kernel<true, true, true>
                <<<grid, HZ_THREADS, (HZ_THREADS / 32) * hz_warp_smem_bytes(), h->stream>>>(p, err);
        } else if (h->hz_eps) {
            hz2d_interior_kernel<true, false, false><<<grid, HZ_THREADS, 0, h->stream>>>(p, err);
        } else if (vec) {
            hz2d_interior_kernel<false, true, false><<<grid, HZ_THREADS, 0, h->stream>>>(p, err);
        } else {
            hz2d_interior_kernel<false, false, false><<<grid, HZ_THREADS, 0, h->stream>>>(p, err);
        }
        OS_TRY(prof_end(h, h->stream));
        h->launches += 1;
    }
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_join, h->side_stream));
        OS_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    }
    return OS_OK;
}

// The two-step H_z launch's split: the interior box of hz2d_interior2_kernel (the single-step box less one row and four
// columns on each side, so that its two-step cone holds plain updates only) and the border's two regions: step 1 over
// the grid minus the box shrunk by one cell (its step-1 state, which step 2 reads around every cell it updates, goes to
// the scratch set), step 2 over the grid minus the box.
struct HzPlan2 {
    bool interior = false;
    int ia = 0, ib = 0, jc0 = 0, jc1 = 0;
    HzBorderRects rects1{}, rects2{};
};

// The grid minus rows [r0, r1) x columns [c0, c1) as up to four rectangles (the whole grid when the box is empty).
static HzBorderRects hz_frame_rects(const OsFdtd2D *h, int r0, int r1, int c0, int c1) {
    const int nx = h->grid.nx, ny = h->grid.ny;
    HzBorderRects q{};
    int n = 0;
    auto add = [&](int a0, int a1, int b0, int b1) {
        if (a1 <= a0 || b1 <= b0) return;
        q.r0[n] = a0, q.r1[n] = a1, q.c0[n] = b0, q.c1[n] = b1;
        ++n;
    };
    if (r1 > r0 && c1 > c0) {
        add(0, r0, 0, ny);
        add(r1, nx, 0, ny);
        add(r0, r1, 0, c0);
        add(r0, r1, c1, ny);
    } else {
        add(0, nx, 0, ny);
    }
    q.n = n;
    q.first[0] = 0;
    for (int k = 0; k < n; ++k)
        q.first[k + 1] = q.first[k] + (int64_t)(q.r1[k] - q.r0[k]) * (q.c1[k] - q.c0[k]);
    for (int k = n; k < 4; ++k) q.first[k + 1] = q.first[n];
    return q;
}

static HzPlan2 hz_plan2(const OsFdtd2D *h) {
    const HzPlan q1 = hz_plan(h);
    HzPlan2 q;
    q.ia = q1.ia + 1;
    q.ib = q1.ib - 1;
    q.jc0 = q1.jc0 + 4;
    q.jc1 = q1.jc1 - 4;
    // the kernel's form: ca = 1 and uniform da / db (no conductivity, no magnetic cells; cb from the stored arrays),
    // rows a multiple of 4 cells (TMA-staged windows)
    q.interior = q1.interior && q.ib > q.ia && q.jc1 > q.jc0 && !h->has_ca && !h->has_dadb && h->grid.ny % 4 == 0;
    if (q.interior) {
        q.rects1 = hz_frame_rects(h, q.ia + 1, q.ib - 1, q.jc0 + 1, q.jc1 - 1);
        q.rects2 = hz_frame_rects(h, q.ia, q.ib, q.jc0, q.jc1);
    }
    return q;
}

// Two fused H_z steps from set `in` to set `out` (p.k_step: the first step's column of the source tables): the
// border's two single steps through the scratch set on the side stream, the interior's two-step kernel on the main
// stream; they write disjoint cells of the output set.
// Field probes after the first step of a two-step H_z launch, a state no buffer holds inside the box: a cell outside
// the box shrunk by one (the region the border's first step covers) is read from the scratch set that step wrote; a
// cell inside it (plain: no CPML row, edge or wrap in reach) is stepped here from the launch's input set with the
// border's per-cell functions (no psi written: none of them is in a CPML layer), its faces' cb from the stored
// arrays (the two-step launch needs no ca).  `p` holds the first step's inputs and value column; `row` is the step's
// row in the probe rows.  Thread k: probe k.
__global__ void hz2d_probe_mid_kernel(const Hz2DParams p, ProbeSet ps, int i0, int i1, int j0, int j1,
                                      const float *shz, const float *sex, const float *sey, float *rows,
                                      int64_t capacity, int64_t row) {
    const int k = threadIdx.x;
    if (k >= ps.n || row < ps.start[k]) return;
    const int i = ps.ix[k], j = ps.iy[k], comp = ps.comp[k];
    const size_t idx = (size_t)i * p.ny + j;
    float v;
    if (!(i >= i0 && i < i1 && j >= j0 && j < j1)) {
        v = (comp == 0 ? shz : comp == 1 ? sex : sey)[idx];
    } else {
        float exo, eyo, sx, sy;
        const float hz = hz2d_hz_at(p, i, j, false, exo, eyo);
        if (comp == 0) {
            v = hz;
        } else if (comp == 1) {
            const float up = hz2d_hz_at(p, i, j + 1, false, sx, sy);
            v = hz2d_ex_at(p, i, j, exo, 1.0f, __ldg(p.cb_x + idx), hz, up);
        } else {
            const float up = hz2d_hz_at(p, i + 1, j, false, sx, sy);
            v = hz2d_ey_at(p, i, j, eyo, 1.0f, __ldg(p.cb_y + idx), hz, up);
        }
    }
    rows[(size_t)k * capacity + row] = v;
}

static int launch_hz_step2(OsFdtd2D *h, const HzPlan2 &q, const Hz2DParams &p) {
    const bool fork = !h->profiling;   // profiling: each kernel timed alone
    cudaStream_t bstream = fork ? h->side_stream : h->stream;
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_fork, h->stream));
        OS_CUDA(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
    }
    Hz2DParams b1 = p, b2 = p;
    b1.hz_out = h->sez[0].ptr, b1.ex_out = h->shx[0].ptr, b1.ey_out = h->shy[0].ptr;
    b2.hz_in = h->sez[0].ptr, b2.ex_in = h->shx[0].ptr, b2.ey_in = h->shy[0].ptr;
    b2.k_step = p.k_step + 1;
    for (int sd = 0; sd < 4; ++sd) {
        if (!(p.cpml_mask & (1 << sd))) continue;
        b1.psi_e_out[sd] = h->spsi_e[0][sd].ptr, b1.psi_h_out[sd] = h->spsi_h[0][sd].ptr;
        b2.psi_e_in[sd] = h->spsi_e[0][sd].ptr, b2.psi_h_in[sd] = h->spsi_h[0][sd].ptr;
    }
    const Hz2DParams *bp[2] = {&b1, &b2};
    const HzBorderRects *br[2] = {&q.rects1, &q.rects2};
    for (int st = 0; st < 2; ++st) {
        const int64_t cells_b = br[st]->first[br[st]->n];
        if (cells_b <= 0) continue;
        OS_TRY(prof_begin(h, 1, bstream));
        if (h->hz_eps) hz2d_border_kernel<true><<<(unsigned)((cells_b + 255) / 256), 256, 0, bstream>>>(*bp[st], *br[st]);
        else hz2d_border_kernel<false><<<(unsigned)((cells_b + 255) / 256), 256, 0, bstream>>>(*bp[st], *br[st]);
        OS_TRY(prof_end(h, bstream));
        h->launches += 1;
    }
    Hz2DParams pi = p;
    pi.ia = q.ia, pi.ib = q.ib, pi.jc0 = q.jc0, pi.jc1 = q.jc1;
    {
        const int64_t warps = (q.jc1 - q.jc0 + HZ2_OUT - 1) / HZ2_OUT;
        const int64_t ctas_x = (warps + HZ_THREADS / 32 - 1) / (HZ_THREADS / 32);
        const int64_t want = (int64_t)h->sm_count * 4 * 4;   // about four waves of four CTAs per SM
        int64_t rows = h->hz_rows > 0 ? h->hz_rows : ((int64_t)(q.ib - q.ia) * ctas_x + want - 1) / want;
        pi.rows_per_cta = (int32_t)std::max<int64_t>(h->hz_rows > 0 ? 1 : 16, std::min<int64_t>(128, rows));
    }
    const dim3 grid((unsigned)((q.jc1 - q.jc0 + HZ2_OUT * (HZ_THREADS / 32) - 1) / (HZ2_OUT * (HZ_THREADS / 32))),
                    (unsigned)((q.ib - q.ia + pi.rows_per_cta - 1) / pi.rows_per_cta));
    OS_TRY(prof_begin(h, 0, h->stream));
    hz2d_interior2_kernel<<<grid, HZ_THREADS, (HZ_THREADS / 32) * hz2_warp_smem_bytes(), h->stream>>>(pi, h->err.ptr);
    OS_TRY(prof_end(h, h->stream));
    h->launches += 1;
    if (fork) {
        OS_CUDA(cudaEventRecord(h->ev_join, h->side_stream));
        OS_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    }
    if (h->probes.n) {   // the first step's values (the second's are read from the output set after the launch)
        OS_TRY(prof_begin(h, 2, h->stream));
        hz2d_probe_mid_kernel<<<1, 32, 0, h->stream>>>(b1, h->probes, q.ia + 1, q.ib - 1, q.jc0 + 1, q.jc1 - 1,
                                                       h->sez[0].ptr, h->shx[0].ptr, h->shy[0].ptr,
                                                       h->probe_rows.ptr, h->probe_capacity, h->n_step);
        OS_TRY(prof_end(h, h->stream));
        h->launches += 1;
        OS_CUDA(cudaGetLastError());
    }
    return OS_OK;
}

// H_z chunk: variant 0 launches the in-place H and E kernels per step, otherwise one fused step kernel per step
// (buffers swapped after each), or with steps_per_launch 2 two steps per launch wherever the next step is not a
// sampled one (the flux lines and field maps are sampled after every sample step, so a sample step ends a launch);
// field probes record the first step of a two-step launch with hz2d_probe_mid_kernel and the second from the output.
static int advance_hz(OsFdtd2D *h, int64_t n_steps, int64_t first_sample, int64_t n_samples, const float *values,
                      const float *phase_table) {
    const int64_t m = h->sample_interval;
    const int nx = h->grid.nx, ny = h->grid.ny;
    const dim3 cell_block(EZ2D_BLOCK_X, EZ2D_BLOCK_Y);
    const dim3 cell_grid((unsigned)((ny + cell_block.x - 1) / cell_block.x),
                         (unsigned)((nx + cell_block.y - 1) / cell_block.y));
    const HzPlan plan = hz_plan(h);
    const bool per_half = h->variant == 0 || !h->tfsf.empty() || !h->poles.empty();
    const bool sampled = !h->fluxes.empty() || !h->maps.empty();
    HzPlan2 plan2;
    const bool two = !per_half && h->steps_per_launch == 2 && h->sez[0].ptr && (plan2 = hz_plan2(h)).interior;
    for (int64_t k = 0; k < n_steps; ++k) {
        const int in = h->cur, out = per_half ? h->cur : h->cur ^ 1;
        Hz2DParams p = make_hz_params(h, in, out);
        p.line_values = values;
        p.values_stride = n_steps;
        p.k_step = k;
        int64_t advanced = 1;
        if (two && k + 1 < n_steps && !(sampled && (h->n_step + 1) % m == 0)) {   // steps k and k + 1 in one launch
            OS_TRY(launch_hz_step2(h, plan2, p));
            advanced = 2;
            k += 1;
        } else if (per_half) {   // a TFSF box and the poles act between the half steps
            OS_TRY(prof_begin(h, 3, h->stream));
            hz2d_h_kernel<<<cell_grid, cell_block, 0, h->stream>>>(p);
            for (auto &t : h->tfsf) {   // TFSFSourceHz.inject_magnetic (fdtd_hz_2d.py:160-163)
                hz2d_tfsf_h_kernel<<<(t->y1 - t->y0 + 255) / 256, 256, 0, h->stream>>>(
                    h->ez[in].ptr, t->aux_ez.ptr, t->x0, t->x1, t->y0, t->y1, t->aux_x0, ny, t->coef_h[0],
                    t->coef_h[1]);
                // aux_hz[k] += coef[k - 1] (aux_ey[k] - aux_ey[k - 1]), k >= 1
                ez2d_tfsf_aux_h_kernel<<<(t->aux_n + 255) / 256, 256, 0, h->stream>>>(
                    t->aux_ez.ptr, t->aux_coef_h.ptr, t->aux_hy.ptr + 1, t->aux_n);
                h->launches += 2;
            }
            if (h->poles.empty()) {
                hz2d_e_kernel<<<cell_grid, cell_block, 0, h->stream>>>(p);
            } else {
                // poles (fdtd_hz_2d.py:233-284): J / P from E^n, the E update (its sheets held back), the pole
                // corrections, then the sheets
                Hz2DParams p_no_lines = p;
                p_no_lines.n_lines = 0;
                OS_TRY(hz_pole_updates(h));
                hz2d_e_kernel<<<cell_grid, cell_block, 0, h->stream>>>(p_no_lines);
                OS_TRY(hz_pole_corrections(h));
                if (p.n_lines) {
                    hz2d_line_inject_kernel<<<cell_grid, cell_block, 0, h->stream>>>(p);
                    h->launches += 1;
                }
            }
            for (size_t b = 0; b < h->tfsf.size(); ++b) {   // TFSFSourceHz.inject_electric (fdtd_hz_2d.py:171-174)
                Tfsf2D &t = *h->tfsf[b];
                const int side = std::max(t.x1 - t.x0, t.y1 - t.y0);
                hz2d_tfsf_e_kernel<<<(side + 255) / 256, 256, 0, h->stream>>>(
                    h->hx[in].ptr, h->hy[in].ptr, t.aux_hy.ptr, t.x0, t.x1, t.y0, t.y1, t.aux_x0, ny, t.coef_e[0],
                    t.coef_e[1], t.coef_e[2], t.coef_e[3]);
                // aux_ey[a] += ce[a] (aux_hz[a + 1] - aux_hz[a]), the soft source, the Mur ends
                const float *value = values + (h->lines.size() + b) * (size_t)n_steps + (size_t)k;
                ez2d_tfsf_aux_e_kernel<<<1, 256, 0, h->stream>>>(t.aux_ez.ptr, t.aux_hy.ptr + 1, t.aux_n,
                                                                 t.aux_coef_e.ptr, t.source_index, value, t.mur_lo,
                                                                 t.mur_hi);
                h->launches += 2;
            }
            OS_TRY(prof_end(h, h->stream));
            h->launches += 2;
        } else {
            OS_TRY(launch_hz_step(h, plan, p));
        }
        h->cur = out;
        h->n_step += advanced;
        if (!h->maps.empty() && h->n_step % m == 0)
            OS_TRY(fold_maps(h, nullptr, h->n_step / m, first_sample, n_samples, phase_table));
        if (h->probes.n) OS_TRY(record_probes(h));
        if (!h->fluxes.empty() && h->n_step % m == 0) {
            const int64_t q = h->n_step / m;
            size_t offset = 0;
            for (auto &f : h->fluxes) {
                const float *ph = phase_table + offset + (size_t)(q - first_sample) * f->nf * 2;
                const int n = f->hi - f->lo;
                const int total = n * f->nf;
                // E_y on the hi-x faces for a line normal to x, E_x on the hi-y faces for one normal to y; H_z
                OS_TRY(prof_begin(h, 2, h->stream));
                ez2d_flux_kernel<<<(total + 255) / 256, 256, 0, h->stream>>>(
                    f->normal_axis == 0 ? h->hy[h->cur].ptr : h->hx[h->cur].ptr, h->ez[h->cur].ptr, ny,
                    f->normal_axis, f->position, f->lo, n, f->nf, ph, f->e_acc.ptr, f->h_acc.ptr);
                OS_TRY(prof_end(h, h->stream));
                h->launches += 1;
                offset += (size_t)n_samples * f->nf * 2;
            }
        }
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// Argument and state checks shared by the advance entry points (`fn` names the caller in messages).
static int check_advance(const OsFdtd2D *h, const char *fn, int64_t n_steps, const float *line_values,
                         int64_t first_sample, int64_t n_samples, const float *phases) {
    OS_CHECK(h, OS_ERR_INVALID, "%s: null handle", fn);
    OS_CHECK(n_steps >= 0, OS_ERR_INVALID, "n_steps must be >= 0, got %lld", (long long)n_steps);
    OS_CHECK(h->has_cb && h->has_spacings, OS_ERR_STATE, "%s: coefficients and spacings must be set", fn);
    for (int s = 0; s < 4; ++s)
        OS_CHECK(!(h->grid.cpml_sides & (1 << s)) || h->cpml_set[s], OS_ERR_STATE,
                 "%s: CPML side %d has no recursion rows", fn, 1 << s);
    if (n_steps == 0) return OS_OK;
    OS_CHECK((h->lines.empty() && h->tfsf.empty()) || line_values, OS_ERR_INVALID, "%s: line_values is required", fn);
    const int64_t m = h->sample_interval;
    const int64_t q_first = h->n_step / m + 1, q_last = (h->n_step + n_steps) / m;
    if ((!h->fluxes.empty() || !h->maps.empty()) && q_last >= q_first) {
        OS_CHECK(phases && first_sample <= q_first && first_sample + n_samples - 1 >= q_last, OS_ERR_INVALID,
                 "%s: the phase table covers samples [%lld, %lld), the chunk needs [%lld, %lld]", fn,
                 (long long)first_sample, (long long)(first_sample + n_samples), (long long)q_first,
                 (long long)q_last);
    }
    return OS_OK;
}

// The chunk's kernels between the start/stop timing events, reading the given device tables.
static int run_chunk(OsFdtd2D *h, int64_t n_steps, int64_t first_sample, int64_t n_samples, const float *values,
                     const float *phase_table) {
    OS_CUDA(cudaEventRecord(h->ev_start, h->stream));
    // a TFSF box or a pole acts between the H and E updates of every step: the per-half-step kernels run them
    const int rc = h->polarization == 1 ? advance_hz(h, n_steps, first_sample, n_samples, values, phase_table)
                   : (h->variant == 0 || !h->tfsf.empty() || !h->poles.empty())
                       ? advance_per_step(h, n_steps, first_sample, n_samples, values, phase_table)
                       : advance_blocked(h, n_steps, first_sample, n_samples, values, phase_table);
    if (rc != OS_OK) return rc;
    OS_CUDA(cudaEventRecord(h->ev_stop, h->stream));
    h->timed = true;
    return OS_OK;
}

}  // namespace os

extern "C" int os_fdtd2d_hz_plan(OsFdtd2D *h, int64_t *interior_cells, int64_t *border_cells) {
    OS_TRY(require_hz(h, "os_fdtd2d_hz_plan"));
    OS_CHECK(interior_cells && border_cells, OS_ERR_INVALID, "os_fdtd2d_hz_plan: null argument");
    if (h->steps_per_launch == 2 && h->sez[0].ptr) {   // the two-step box (border: the cells outside it)
        const HzPlan2 q = hz_plan2(h);
        if (q.interior) {
            *interior_cells = (int64_t)(q.ib - q.ia) * (q.jc1 - q.jc0);
            *border_cells = q.rects2.first[q.rects2.n];
            return OS_OK;
        }
    }
    const HzPlan q = hz_plan(h);
    *interior_cells = q.interior ? (int64_t)(q.ib - q.ia) * (q.jc1 - q.jc0) : 0;
    *border_cells = q.rects.first[q.rects.n];
    return OS_OK;
}

extern "C" int os_fdtd2d_advance(OsFdtd2D *h, int64_t n_steps, const float *line_values, int64_t first_sample,
                                 int64_t n_samples, const float *phases) {
    OS_TRY(check_advance(h, "os_fdtd2d_advance", n_steps, line_values, first_sample, n_samples, phases));
    h->launches = 0;
    h->prof_used = 0;
    if (n_steps == 0) return OS_OK;
    OS_TRY(bind_device(h));
    const size_t value_rows = h->lines.size() + h->tfsf.size();   // line sources, then TFSF boxes
    if (value_rows) OS_TRY(upload(h->line_values, line_values, value_rows * (size_t)n_steps, h->stream));
    const size_t phase_floats = phase_floats_of(h, n_samples);
    if (phase_floats && phases) OS_TRY(upload(h->phases, phases, phase_floats, h->stream));
    OS_TRY(reserve_probe_rows(h, n_steps));
    return run_chunk(h, n_steps, first_sample, n_samples, h->line_values.ptr, h->phases.ptr);
}

// ---------------------------------------------------------------------------------------------------------------
// Allocation-free advance.  os_fdtd2d_advance stages a chunk's source-value and DFT-phase tables in grow-only
// device buffers of the handle, which allocate on the first chunk and whenever a chunk outgrows them (cudaFree +
// cudaMalloc; cudaFree waits for the whole device).  Callers that must not allocate at that point -- a serving loop
// whose jobs share one GPU on several streams, where a device-wide wait in one job stalls the others, or a job
// admitted under a fixed memory budget that must not grow after admission -- use os_fdtd2d_advance_noalloc, which
// stages the same tables in this fixed file-scope array instead.  Nothing in it has to start at zero: every call
// copies its tables in before its kernels read them and the kernels read no float beyond what was copied.  The array
// is one per device and per process, so calls whose device work can overlap (different streams with no ordering
// between them) race on it; calls on one stream, or ordered by events, are safe.
static __device__ __align__(256) float g_noalloc_scratch[OS_FDTD_NOALLOC_MAX_FLOATS];

namespace os {

// Device address of g_noalloc_scratch on the current device, looked up once per device (the first lookup may load
// the module onto the device, so the first call for a device belongs before any stream capture).  The cached address
// belongs to the device's primary context as it was at the lookup: a process that resets the device
// (cudaDeviceReset) or tears its primary context down must not call os_fdtd2d_advance_noalloc on it afterwards; the
// engines of that context are gone with it anyway.
static int noalloc_scratch(int device, float **out) {
    static std::mutex mu;
    static float *addr[OS_FDTD_MAX_DEVICES] = {};
    OS_CHECK(device >= 0 && device < OS_FDTD_MAX_DEVICES, OS_ERR_INVALID,
             "os_fdtd2d_advance_noalloc: device %d is outside [0, %d)", device, OS_FDTD_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void *p = nullptr;
        OS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        OS_CHECK(p && ((uintptr_t)p & 255) == 0, OS_ERR_CUDA,
                 "os_fdtd2d_advance_noalloc: the scratch array is not 256-byte aligned on device %d", device);
        addr[device] = (float *)p;
    }
    *out = addr[device];
    return OS_OK;
}

}  // namespace os

extern "C" int os_fdtd2d_advance_noalloc(OsFdtd2D *h, int64_t n_steps, const float *line_values,
                                         int64_t first_sample, int64_t n_samples, const float *phases) {
    using namespace os;
    OS_TRY(check_advance(h, "os_fdtd2d_advance_noalloc", n_steps, line_values, first_sample, n_samples, phases));
    OS_CHECK(!h->profiling, OS_ERR_STATE,
             "os_fdtd2d_advance_noalloc: profiling is on (its event pool grows on demand); turn it off first");
    OS_CHECK(h->probes.n == 0 || h->n_step + n_steps <= h->probe_capacity, OS_ERR_STATE,
             "os_fdtd2d_advance_noalloc: the field probes' rows would have to grow; advance with os_fdtd2d_advance");
    // tables: line values at float 0, phases at the next 64-float (256-byte) boundary.  Step and sample counts are
    // bounded before they multiply anything, so no product below can wrap around.
    const size_t value_rows = h->lines.size() + h->tfsf.size();
    size_t sample_floats = 0;   // phase floats per DFT sample, over every flux line and field map
    for (auto &f : h->fluxes) sample_floats += (size_t)f->nf * 2;
    for (auto &d : h->maps) sample_floats += (size_t)d->nf * 2 * (d->hz ? 2 : 1);
    OS_CHECK(value_rows == 0 || n_steps <= (int64_t)(OS_FDTD_NOALLOC_MAX_FLOATS / value_rows), OS_ERR_INVALID,
             "os_fdtd2d_advance_noalloc: %lld steps of %zu source rows exceed the fixed scratch of %d floats; advance "
             "fewer steps per call", (long long)n_steps, value_rows, OS_FDTD_NOALLOC_MAX_FLOATS);
    const bool with_phases = n_steps > 0 && n_samples > 0 && phases;   // uploaded only when given, as advance does
    OS_CHECK(!with_phases || sample_floats == 0 ||
                 n_samples <= (int64_t)(OS_FDTD_NOALLOC_MAX_FLOATS / sample_floats), OS_ERR_INVALID,
             "os_fdtd2d_advance_noalloc: %lld DFT samples of %zu phase floats exceed the fixed scratch of %d floats; "
             "advance fewer steps per call", (long long)n_samples, sample_floats, OS_FDTD_NOALLOC_MAX_FLOATS);
    const size_t value_floats = n_steps > 0 ? value_rows * (size_t)n_steps : 0;
    const size_t phase_floats = with_phases ? (size_t)n_samples * sample_floats : 0;
    const size_t phase_offset = (value_floats + 63) / 64 * 64;
    const size_t need = phase_floats ? phase_offset + phase_floats : value_floats;
    OS_CHECK(need <= (size_t)OS_FDTD_NOALLOC_MAX_FLOATS, OS_ERR_INVALID,
             "os_fdtd2d_advance_noalloc: the chunk's tables need %zu floats (%zu source values + %zu phase floats), "
             "the fixed scratch holds %d; advance fewer steps per call",
             need, value_floats, phase_floats, OS_FDTD_NOALLOC_MAX_FLOATS);
    h->launches = 0;
    h->prof_used = 0;
    if (n_steps == 0) return OS_OK;
    OS_TRY(bind_device(h));
    float *scratch = nullptr;
    OS_TRY(noalloc_scratch(h->device, &scratch));
    if (value_floats)
        OS_CUDA(cudaMemcpyAsync(scratch, line_values, value_floats * sizeof(float), cudaMemcpyHostToDevice,
                                h->stream));
    if (phase_floats)
        OS_CUDA(cudaMemcpyAsync(scratch + phase_offset, phases, phase_floats * sizeof(float),
                                cudaMemcpyHostToDevice, h->stream));
    return run_chunk(h, n_steps, first_sample, n_samples, scratch, scratch + phase_offset);
}

extern "C" int os_fdtd2d_set_stall_probe(OsFdtd2D *h, int64_t wait_ns) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_stall_probe: null handle");
    OS_CHECK(wait_ns >= 0 && wait_ns <= (int64_t)TB_WAIT_NS, OS_ERR_INVALID,
             "os_fdtd2d_set_stall_probe: the wait must be within [0, %llu] ns", (unsigned long long)TB_WAIT_NS);
    h->stall_probe_ns = wait_ns;
    return OS_OK;
}

extern "C" int os_fdtd2d_configure(OsFdtd2D *h, int32_t variant, int32_t steps_per_launch, int32_t tile_rows) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_configure: null handle");
    OS_CHECK(variant >= 0 && variant <= 2, OS_ERR_INVALID,
             "variant must be 0 (per half step), 1 (blocked) or 2 (blocked, general kernel only)");
    OS_CHECK(steps_per_launch >= 1 && steps_per_launch <= TB_MAX_T, OS_ERR_INVALID,
             "steps_per_launch must be in [1, %d], got %d", TB_MAX_T, steps_per_launch);
    if (h->polarization == 1) {
        // H_z: variant 0 per-half-step kernels, 1 the fused step kernel with tile_rows rows per CTA (0: per grid);
        // steps_per_launch 2: the interior box advances two steps per launch (hz2d_interior2_kernel) where it applies
        OS_CHECK(variant <= 1 && (steps_per_launch == 1 || steps_per_launch == 2) && tile_rows >= 0, OS_ERR_INVALID,
                 "an H_z engine takes variant 0 or 1, steps_per_launch 1 or 2 and tile_rows >= 0, got %d, %d, %d",
                 variant, steps_per_launch, tile_rows);
        if (steps_per_launch == 2 && !h->sez[0].ptr) {   // the border's step-1 state (made here, not in an advance)
            OS_TRY(bind_device(h));
            const size_t n = cells(h);
            OS_TRY(h->sez[0].alloc(n));
            OS_TRY(h->shx[0].alloc(n));
            OS_TRY(h->shy[0].alloc(n));
            const OsGrid2D &g = h->grid;
            for (int sd = 0; sd < 4; ++sd) {
                if (!(g.cpml_sides & (1 << sd))) continue;
                const size_t slab = (sd < 2 ? (size_t)g.ny : (size_t)g.nx) * (size_t)g.npml;
                OS_TRY(h->spsi_e[0][sd].alloc(slab));
                OS_TRY(h->spsi_h[0][sd].alloc(slab));
            }
        }
        h->variant = variant;
        h->steps_per_launch = steps_per_launch;
        h->hz_rows = tile_rows;
        return OS_OK;
    }
    OS_CHECK(tile_rows >= 0, OS_ERR_INVALID, "tile_rows must be >= 0 (0: chosen from the grid), got %d", tile_rows);
    h->variant = variant;
    h->steps_per_launch = steps_per_launch;
    h->tile_rows = tile_rows;
    return OS_OK;
}

extern "C" int os_fdtd2d_autotune(OsFdtd2D *h, int32_t steps_per_launch, const int32_t *candidates,
                                  int32_t n_candidates, int32_t repeats, int32_t *best_rows, float *best_ms) {
    OS_TRY(require_ez(h, "os_fdtd2d_autotune"));
    OS_CHECK(candidates && n_candidates > 0 && best_rows && best_ms, OS_ERR_INVALID,
             "os_fdtd2d_autotune: null argument or no candidates");
    OS_CHECK(steps_per_launch >= 1 && steps_per_launch <= TB_MAX_T, OS_ERR_INVALID,
             "steps_per_launch must be in [1, %d]", TB_MAX_T);
    OS_CHECK(h->has_cb && h->has_spacings, OS_ERR_STATE, "os_fdtd2d_autotune: coefficients and spacings must be set");
    OS_TRY(bind_device(h));
    const int saved_rows = h->tile_rows;
    const bool saved_prof = h->profiling;
    h->profiling = false;
    cudaEvent_t t0, t1;
    OS_CUDA(cudaEventCreate(&t0));
    OS_CUDA(cudaEventCreate(&t1));
    float best = -1.0f;
    int best_r = saved_rows;
    int rc = OS_OK;
    // candidates are timed in interleaved rounds and each keeps its fastest round, so that a slow spell of the
    // device during one candidate's trial does not decide the choice
    constexpr int kRounds = 3;
    for (int c_all = 0; c_all < kRounds * n_candidates && rc == OS_OK; ++c_all) {
        const int c = c_all % n_candidates;
        if (candidates[c] < 1) continue;
        h->tile_rows = candidates[c];
        TBParams interior{}, general{};
        bool has_interior = false;
        plan_tiles(h, steps_per_launch, interior, general, has_interior);
        for (TBParams *q : {&interior, &general}) {
            fill_common(h, *q);
            q->n_lines = 0;       // sources and monitors do not change the timing of a trial launch
            q->n_mons = 0;
            q->sample_mask = 0;
            // trial launches read the live buffers and write the idle ones, which are never swapped in
            bind_buffers(h, *q, h->cur, h->cur ^ 1);
        }
        for (int w = 0; w < (c_all < n_candidates ? 2 : 1) && rc == OS_OK; ++w)
            rc = launch_tb_any(h, steps_per_launch, interior, general, has_interior);
        if (rc != OS_OK) break;
        if (cudaEventRecord(t0, h->stream) != cudaSuccess) { rc = OS_ERR_CUDA; break; }
        for (int k = 0; k < std::max(1, repeats) && rc == OS_OK; ++k)
            rc = launch_tb_any(h, steps_per_launch, interior, general, has_interior);
        if (rc != OS_OK) break;
        float ms = 0.0f;
        if (cudaEventRecord(t1, h->stream) != cudaSuccess || cudaEventSynchronize(t1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, t0, t1) != cudaSuccess) {
            rc = os::cuda_status(cudaGetLastError(), "os_fdtd2d_autotune timing");
            break;
        }
        ms /= std::max(1, repeats);
        if (best < 0.0f || ms < best) {
            best = ms;
            best_r = candidates[c];
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    h->profiling = saved_prof;
    h->tile_rows = rc == OS_OK ? best_r : saved_rows;
    if (rc != OS_OK) return rc;
    *best_rows = best_r;
    *best_ms = best;
    return OS_OK;
}

extern "C" int os_fdtd2d_plan_info(OsFdtd2D *h, int32_t steps_per_launch, int64_t *interior_cells,
                                   int64_t *interior_tiles, int64_t *general_tiles) {
    OS_TRY(require_ez(h, "os_fdtd2d_plan_info"));
    OS_CHECK(interior_cells && interior_tiles && general_tiles, OS_ERR_INVALID, "os_fdtd2d_plan_info: null argument");
    OS_CHECK(steps_per_launch >= 1 && steps_per_launch <= TB_MAX_T, OS_ERR_INVALID,
             "steps_per_launch must be in [1, %d]", TB_MAX_T);
    OS_CHECK(h->has_spacings, OS_ERR_STATE, "os_fdtd2d_plan_info: spacings are not set");
    TBParams interior{}, general{};
    bool has_interior = false;
    plan_tiles(h, steps_per_launch, interior, general, has_interior);
    int64_t cells_in = 0;
    if (has_interior)
        for (int r = 0; r < interior.n_rects; ++r)
            cells_in += (int64_t)(interior.rects[r].r1 - interior.rects[r].r0) *
                        (int64_t)(interior.rects[r].c1 - interior.rects[r].c0);
    *interior_cells = cells_in;
    *interior_tiles = has_interior ? interior.n_tiles : 0;
    *general_tiles = general.n_tiles;
    return OS_OK;
}

extern "C" int os_fdtd2d_set_profiling(OsFdtd2D *h, int32_t on) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_profiling: null handle");
    h->profiling = on != 0;
    return OS_OK;
}

extern "C" int os_fdtd2d_kernel_times(OsFdtd2D *h, int32_t kind, double *total_ms, int64_t *launches) {
    OS_CHECK(h && total_ms && launches, OS_ERR_INVALID, "os_fdtd2d_kernel_times: null argument");
    OS_TRY(bind_device(h));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    OS_CUDA(cudaStreamSynchronize(h->side_stream));
    double total = 0.0;
    int64_t count = 0;
    for (size_t k = 0; k < h->prof_used; ++k) {
        if (h->prof_kind[k] != kind) continue;
        float ms = 0.0f;
        OS_CUDA(cudaEventElapsedTime(&ms, h->prof_events[2 * k], h->prof_events[2 * k + 1]));
        total += ms;
        count += 1;
    }
    *total_ms = total;
    *launches = count;
    return OS_OK;
}

extern "C" int os_fdtd2d_launch_count(OsFdtd2D *h, int64_t *launches) {
    OS_CHECK(h && launches, OS_ERR_INVALID, "os_fdtd2d_launch_count: null argument");
    *launches = h->launches;
    return OS_OK;
}

extern "C" int os_fdtd2d_step_count(OsFdtd2D *h, int64_t *n_step) {
    OS_CHECK(h && n_step, OS_ERR_INVALID, "os_fdtd2d_step_count: null argument");
    *n_step = h->n_step;
    return OS_OK;
}

extern "C" int os_fdtd2d_read_flux_spectra(OsFdtd2D *h, int32_t monitor_id, double *e_spectra, double *h_spectra) {
    OS_CHECK(h && e_spectra && h_spectra, OS_ERR_INVALID, "os_fdtd2d_read_flux_spectra: null argument");
    OS_CHECK(monitor_id >= 0 && (size_t)monitor_id < h->fluxes.size(), OS_ERR_INVALID, "no flux monitor %d", monitor_id);
    OS_TRY(bind_device(h));
    FluxLine2D &f = *h->fluxes[monitor_id];
    OS_CUDA(cudaMemcpyAsync(e_spectra, f.e_acc.ptr, f.e_acc.bytes(), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaMemcpyAsync(h_spectra, f.h_acc.ptr, f.h_acc.bytes(), cudaMemcpyDeviceToHost, h->stream));
    OS_TRY(sync_and_check(h));
    return OS_OK;
}

extern "C" int os_fdtd2d_add_dft_map(OsFdtd2D *h, int32_t x_start, int32_t x_stop, int32_t y_start, int32_t y_stop,
                                     int32_t downsample, int32_t nf, int32_t *map_id) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_add_dft_map: null handle");
    OS_CHECK(0 <= x_start && x_start < x_stop && x_stop <= h->grid.nx && 0 <= y_start && y_start < y_stop &&
                 y_stop <= h->grid.ny,
             OS_ERR_INVALID, "DFTMonitor box [%d, %d) x [%d, %d) must be a non-empty box inside the %d x %d grid",
             x_start, x_stop, y_start, y_stop, h->grid.nx, h->grid.ny);
    OS_CHECK(downsample >= 1, OS_ERR_INVALID, "DFTMonitor downsample must be an int >= 1, got %d", downsample);
    OS_CHECK(nf >= 1, OS_ERR_INVALID, "monitor frequencies must be a non-empty list");
    OS_TRY(bind_device(h));
    std::unique_ptr<DftMap2D> d(new DftMap2D());
    // dft_sample_slice (monitors.py:152-155): every ds-th cell from the middle of the first ds-cell block
    d->ds = downsample;
    d->x0 = x_start + std::min(downsample, x_stop - x_start) / 2;
    d->y0 = y_start + std::min(downsample, y_stop - y_start) / 2;
    d->mx = (x_stop - d->x0 + downsample - 1) / downsample;
    d->my = (y_stop - d->y0 + downsample - 1) / downsample;
    d->nf = nf;
    d->hz = h->polarization == 1;
    OS_TRY(d->acc.alloc((size_t)nf * d->mx * d->my * 2 * (d->hz ? 3 : 1)));
    OS_CUDA(cudaMemsetAsync(d->acc.ptr, 0, d->acc.bytes(), h->stream));
    if (map_id) *map_id = (int32_t)h->maps.size();
    h->maps.push_back(std::move(d));
    return OS_OK;
}

extern "C" int os_fdtd2d_add_tfsf(OsFdtd2D *h, int32_t x0, int32_t x1, int32_t y0, int32_t y1, int32_t aux_cells,
                                  int32_t aux_x0, int32_t source_index, const float *coef_h, const float *coef_e,
                                  float mur_lo, float mur_hi, const float *aux_coef_h, const float *aux_coef_e,
                                  int32_t *tfsf_id) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_add_tfsf: null handle");
    OS_CHECK(coef_h && coef_e && aux_coef_h && aux_coef_e, OS_ERR_INVALID, "os_fdtd2d_add_tfsf: null argument");
    OS_CHECK(1 <= x0 && x0 < x1 && x1 < h->grid.nx && 1 <= y0 && y0 < y1 && y1 < h->grid.ny, OS_ERR_INVALID,
             "TFSF box [%d, %d) x [%d, %d) must keep one scattered-field cell on every side of the %d x %d grid", x0,
             x1, y0, y1, h->grid.nx, h->grid.ny);
    OS_CHECK(aux_x0 >= 1 && aux_x0 + (x1 - x0) < aux_cells && 1 <= source_index && source_index < aux_cells - 1,
             OS_ERR_INVALID, "TFSF incident line of %d cells cannot hold the box at %d and the source at %d",
             aux_cells, aux_x0, source_index);
    OS_CHECK(h->tfsf.size() < 4, OS_ERR_INVALID, "at most 4 TFSF boxes per engine");
    OS_CHECK(h->lines.size() + h->tfsf.size() < (size_t)OS_MAX_LINES_2D, OS_ERR_INVALID,
             "at most %d line sources and TFSF boxes per engine", OS_MAX_LINES_2D);
    OS_TRY(bind_device(h));
    std::unique_ptr<Tfsf2D> t(new Tfsf2D());
    t->x0 = x0, t->x1 = x1, t->y0 = y0, t->y1 = y1;
    t->aux_n = aux_cells, t->aux_x0 = aux_x0, t->source_index = source_index;
    for (int k = 0; k < 4; ++k) t->coef_h[k] = coef_h[k];
    for (int k = 0; k < 4; ++k) t->coef_e[k] = coef_e[k];
    t->mur_lo = mur_lo, t->mur_hi = mur_hi;
    OS_TRY(t->aux_ez.alloc((size_t)aux_cells));
    OS_TRY(t->aux_hy.alloc((size_t)aux_cells));
    OS_CUDA(cudaMemsetAsync(t->aux_ez.ptr, 0, t->aux_ez.bytes(), h->stream));
    OS_CUDA(cudaMemsetAsync(t->aux_hy.ptr, 0, t->aux_hy.bytes(), h->stream));
    OS_TRY(upload(t->aux_coef_h, aux_coef_h, (size_t)aux_cells - 1, h->stream));
    OS_TRY(upload(t->aux_coef_e, aux_coef_e, (size_t)aux_cells, h->stream));
    if (tfsf_id) *tfsf_id = (int32_t)h->tfsf.size();
    h->tfsf.push_back(std::move(t));
    return OS_OK;
}

extern "C" int os_fdtd2d_add_pole(OsFdtd2D *h, int32_t kind, int32_t i0, int32_t i1, int32_t j0, int32_t j1,
                                  float damping, float restoring, const float *drive, float inv_dt, int32_t *pole_id) {
    OS_TRY(require_ez(h, "os_fdtd2d_add_pole"));
    OS_CHECK(drive, OS_ERR_INVALID, "os_fdtd2d_add_pole: null drive");
    OS_CHECK(kind == 0 || kind == 1, OS_ERR_INVALID, "pole kind must be 0 (Drude) or 1 (Lorentz), got %d", kind);
    OS_CHECK(0 <= i0 && i0 < i1 && i1 <= h->grid.nx && 0 <= j0 && j0 < j1 && j1 <= h->grid.ny, OS_ERR_INVALID,
             "pole box [%d, %d) x [%d, %d) outside the %d x %d grid", i0, i1, j0, j1, h->grid.nx, h->grid.ny);
    OS_CHECK(h->poles.size() < 32, OS_ERR_INVALID, "at most 32 poles per engine");
    OS_TRY(bind_device(h));
    std::unique_ptr<Pole2D> q(new Pole2D());
    q->kind = kind, q->i0 = i0, q->i1 = i1, q->j0 = j0, q->j1 = j1;
    q->damping = damping, q->restoring = restoring;
    const size_t n = (size_t)(i1 - i0) * (size_t)(j1 - j0);
    OS_TRY(upload(q->drive, drive, n, h->stream));
    OS_TRY(q->a.alloc(n));
    OS_CUDA(cudaMemsetAsync(q->a.ptr, 0, q->a.bytes(), h->stream));
    if (kind == 1) {
        OS_TRY(q->b.alloc(n));
        OS_CUDA(cudaMemsetAsync(q->b.ptr, 0, q->b.bytes(), h->stream));
        h->inv_dt = inv_dt;
    } else {
        if (!h->jz_total.ptr) {
            OS_TRY(h->jz_total.alloc(cells(h)));
            OS_CUDA(cudaMemsetAsync(h->jz_total.ptr, 0, h->jz_total.bytes(), h->stream));
        }
        int32_t *u = h->drude_box;
        if (u[1] == u[0]) u[0] = i0, u[1] = i1, u[2] = j0, u[3] = j1;
        else u[0] = std::min(u[0], i0), u[1] = std::max(u[1], i1), u[2] = std::min(u[2], j0), u[3] = std::max(u[3], j1);
    }
    if (pole_id) *pole_id = (int32_t)h->poles.size();
    h->poles.push_back(std::move(q));
    return OS_OK;
}

extern "C" int os_fdtd2d_hz_add_pole(OsFdtd2D *h, int32_t kind, int32_t component, int32_t i0, int32_t i1, int32_t j0,
                                     int32_t j1, float damping, float restoring, const float *drive, float inv_dt,
                                     int32_t *pole_id) {
    OS_TRY(require_hz(h, "os_fdtd2d_hz_add_pole"));
    OS_CHECK(drive, OS_ERR_INVALID, "os_fdtd2d_hz_add_pole: null drive");
    OS_CHECK(kind == 0 || kind == 1, OS_ERR_INVALID, "pole kind must be 0 (Drude) or 1 (Lorentz), got %d", kind);
    OS_CHECK(component == 0 || component == 1, OS_ERR_INVALID, "pole component must be 0 (E_x) or 1 (E_y), got %d",
             component);
    OS_CHECK(0 <= i0 && i0 < i1 && i1 <= h->grid.nx && 0 <= j0 && j0 < j1 && j1 <= h->grid.ny, OS_ERR_INVALID,
             "pole box [%d, %d) x [%d, %d) outside the %d x %d grid", i0, i1, j0, j1, h->grid.nx, h->grid.ny);
    OS_CHECK(h->poles.size() < 64, OS_ERR_INVALID, "at most 64 pole face sets per engine");
    OS_TRY(bind_device(h));
    std::unique_ptr<Pole2D> q(new Pole2D());
    q->kind = kind, q->comp = component, q->i0 = i0, q->i1 = i1, q->j0 = j0, q->j1 = j1;
    q->damping = damping, q->restoring = restoring;
    const size_t n = (size_t)(i1 - i0) * (size_t)(j1 - j0);
    OS_TRY(upload(q->drive, drive, n, h->stream));
    OS_TRY(q->a.alloc(n));
    OS_CUDA(cudaMemsetAsync(q->a.ptr, 0, q->a.bytes(), h->stream));
    if (kind == 1) {
        OS_TRY(q->b.alloc(n));
        OS_CUDA(cudaMemsetAsync(q->b.ptr, 0, q->b.bytes(), h->stream));
        h->inv_dt = inv_dt;
    }
    if (pole_id) *pole_id = (int32_t)h->poles.size();
    h->poles.push_back(std::move(q));
    return OS_OK;
}

extern "C" int os_fdtd2d_add_probe(OsFdtd2D *h, int32_t ix, int32_t iy, int32_t component, int32_t *probe_id) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_add_probe: null handle");
    OS_CHECK(0 <= ix && ix < h->grid.nx && 0 <= iy && iy < h->grid.ny, OS_ERR_INVALID,
             "field probe cell (%d, %d) outside the %d x %d grid", ix, iy, h->grid.nx, h->grid.ny);
    OS_CHECK(component >= 0 && component <= 2, OS_ERR_INVALID, "unknown field component %d", component);
    OS_CHECK(h->probes.n < OS_MAX_PROBES, OS_ERR_INVALID, "at most %d field probes per engine", OS_MAX_PROBES);
    if (!h->probe_stage.ptr) {
        OS_TRY(bind_device(h));
        OS_TRY(h->probe_stage.alloc((size_t)OS_MAX_PROBES * TB_MAX_T * 2));
    }
    const int k = h->probes.n++;
    h->probes.ix[k] = ix, h->probes.iy[k] = iy, h->probes.comp[k] = component;
    h->probes.start[k] = h->n_step;
    if (probe_id) *probe_id = k;
    return OS_OK;
}

extern "C" int os_fdtd2d_read_probe(OsFdtd2D *h, int32_t probe_id, float *values, int64_t max_values,
                                    int64_t *n_values) {
    OS_CHECK(h && n_values, OS_ERR_INVALID, "os_fdtd2d_read_probe: null argument");
    OS_CHECK(probe_id >= 0 && probe_id < h->probes.n, OS_ERR_INVALID, "no field probe %d", probe_id);
    const int64_t start = h->probes.start[probe_id];
    const int64_t n = std::max<int64_t>(0, h->n_step - start);
    *n_values = n;
    if (n == 0 || !values) return OS_OK;   // values NULL: the count only
    OS_CHECK(max_values >= n, OS_ERR_INVALID, "os_fdtd2d_read_probe: room for %lld values, %lld recorded",
             (long long)max_values, (long long)n);
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(values, h->probe_rows.ptr + (size_t)probe_id * h->probe_capacity + start,
                            (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_TRY(sync_and_check(h));
    return OS_OK;
}

extern "C" int os_fdtd2d_read_dft_map(OsFdtd2D *h, int32_t map_id, float *spectra) {
    OS_CHECK(h && spectra, OS_ERR_INVALID, "os_fdtd2d_read_dft_map: null argument");
    OS_CHECK(map_id >= 0 && (size_t)map_id < h->maps.size(), OS_ERR_INVALID, "no field-map monitor %d", map_id);
    OS_TRY(bind_device(h));
    DftMap2D &d = *h->maps[map_id];
    OS_CUDA(cudaMemcpyAsync(spectra, d.acc.ptr, d.acc.bytes(), cudaMemcpyDeviceToHost, h->stream));
    OS_TRY(sync_and_check(h));
    return OS_OK;
}

static float *component_ptr(OsFdtd2D *h, int32_t component) {
    switch (component) {
        case OS_EZ: return h->ez[h->cur].ptr;
        case OS_HX: return h->hx[h->cur].ptr;
        case OS_HY: return h->hy[h->cur].ptr;
        default: return nullptr;
    }
}

extern "C" int os_fdtd2d_read_field(OsFdtd2D *h, int32_t component, float *out) {
    OS_CHECK(h && out, OS_ERR_INVALID, "os_fdtd2d_read_field: null argument");
    float *src = component_ptr(h, component);
    OS_CHECK(src, OS_ERR_INVALID, "os_fdtd2d_read_field: unknown component %d", component);
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(out, src, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_TRY(sync_and_check(h));
    return OS_OK;
}

extern "C" int os_fdtd2d_write_field(OsFdtd2D *h, int32_t component, const float *in) {
    OS_CHECK(h && in, OS_ERR_INVALID, "os_fdtd2d_write_field: null argument");
    float *dst = component_ptr(h, component);
    OS_CHECK(dst, OS_ERR_INVALID, "os_fdtd2d_write_field: unknown component %d", component);
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(dst, in, cells(h) * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd2d_reset(OsFdtd2D *h) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_reset: null handle");
    OS_TRY(bind_device(h));
    return zero_state(h);
}

extern "C" int os_fdtd2d_synchronize(OsFdtd2D *h) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_synchronize: null handle");
    OS_TRY(bind_device(h));
    return sync_and_check(h);
}

extern "C" int os_fdtd2d_set_stream(OsFdtd2D *h, void *cuda_stream) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_stream: null handle");
    OS_TRY(bind_device(h));
    cudaStream_t next = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
    if (next != h->stream) {
        // the new stream waits on the device for the work queued so far on the old one (no host wait)
        OS_CUDA(cudaEventRecord(h->ev_handoff, h->stream));
        OS_CUDA(cudaStreamWaitEvent(next, h->ev_handoff, 0));
        h->stream = next;
    }
    return OS_OK;
}

extern "C" int os_fdtd2d_last_advance_ms(OsFdtd2D *h, float *ms) {
    OS_CHECK(h && ms, OS_ERR_INVALID, "os_fdtd2d_last_advance_ms: null argument");
    *ms = 0.0f;
    if (!h->timed) return OS_OK;
    OS_TRY(bind_device(h));
    OS_CUDA(cudaEventSynchronize(h->ev_stop));
    OS_CUDA(cudaEventElapsedTime(ms, h->ev_start, h->ev_stop));
    return OS_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// Batched advance of several simulations on one device: every T steps one border launch and one interior launch per
// template configuration cover the tiles of all of them (a warp finds its simulation in a prefix table of tile
// counts), and one launch folds the DFT samples of all their flux lines.  Each simulation's arithmetic is exactly
// that of os_fdtd2d_advance, so its results are the same alone and in the batch.  The per-launch parameters of the
// whole call are built on the host into one page-locked block and reach the device in one copy.
struct OsFdtd2DBatch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;          // the frame steps run here, overlapping the interior launches
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool timed = false;
    struct Staging {                   // page-locked staging of one call's launch parameters
        unsigned char *host = nullptr;
        size_t capacity = 0;
        cudaEvent_t copied = nullptr;  // its copy to the device has run
        bool pending = false;
    };
    static constexpr int kStaging = 4; // calls in flight before one waits for an earlier call's copy
    Staging staging[kStaging];
    int next_staging = 0;
    os::DeviceArray<unsigned char> dev;
    int64_t launches = 0;
};

namespace os {

struct BatchGroup {                    // one kernel launch of a batched step: jobs sharing a template configuration
    int kind;                          // 0 interior, 1 general
    bool ca, px, py, vec;              // vec: ny % 4 == 0 (interior groups)
    std::vector<TBParams> params;
    std::vector<int> tile_start{0};
    size_t params_off = 0, tiles_off = 0;
};

struct FrameStep {                     // one frame step of a batched blocked launch: the jobs' regions
    std::vector<EzFrameParams> params;
    std::vector<int32_t> block_start{0};   // 256-thread blocks per job, cumulative
    size_t params_off = 0, starts_off = 0;
};

struct BatchLaunch {
    int T;
    std::vector<FrameStep> frames;     // steps 1..T
    std::vector<BatchGroup> groups;
    std::vector<FluxBatchItem> items;
    int max_item_cells = 0;
    size_t items_off = 0;
};

static BatchGroup &batch_group(BatchLaunch &L, int kind, bool ca, bool px, bool py, bool vec) {
    for (auto &g : L.groups)
        if (g.kind == kind && g.ca == ca && g.px == px && g.py == py && g.vec == vec) return g;
    L.groups.push_back(BatchGroup{kind, ca, px, py, vec, {}, {0}, 0, 0});
    return L.groups.back();
}

template <int T, bool CA, bool PX, bool PY, bool VEC>
static int launch_interior_batch(cudaStream_t s, const TBParams *jobs, const int *tiles, int n_jobs, int total) {
    const size_t smem = (size_t)TB_WARPS * ip_warp_smem_bytes(T, CA) + (size_t)TB_WARPS * sizeof(TBParams);
    static bool attr_set = false;
    if (!attr_set) {
        OS_CUDA(cudaFuncSetAttribute(ez2d_interior_batch_kernel<T, CA, PX, PY, VEC>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
    }
    ez2d_interior_batch_kernel<T, CA, PX, PY, VEC>
        <<<(unsigned)((total + TB_WARPS - 1) / TB_WARPS), TB_WARPS * 32, smem, s>>>(jobs, tiles, n_jobs);
    return OS_OK;
}

template <int T, bool CA>
static int launch_interior_batch_ca(cudaStream_t s, const BatchGroup &g, const TBParams *jobs, const int *tiles,
                                    int n, int total) {
    if (!g.vec) {
        return g.px ? launch_interior_batch<T, CA, true, false, false>(s, jobs, tiles, n, total)
                    : launch_interior_batch<T, CA, false, false, false>(s, jobs, tiles, n, total);
    }
    if (g.px && g.py) return launch_interior_batch<T, CA, true, true, true>(s, jobs, tiles, n, total);
    if (g.px) return launch_interior_batch<T, CA, true, false, true>(s, jobs, tiles, n, total);
    if (g.py) return launch_interior_batch<T, CA, false, true, true>(s, jobs, tiles, n, total);
    return launch_interior_batch<T, CA, false, false, true>(s, jobs, tiles, n, total);
}

template <int T>
static int launch_group(cudaStream_t s, const BatchGroup &g, const unsigned char *dev) {
    const TBParams *jobs = reinterpret_cast<const TBParams *>(dev + g.params_off);
    const int *tiles = reinterpret_cast<const int *>(dev + g.tiles_off);
    const int n = (int)g.params.size(), total = g.tile_start.back();
    if (!total) return OS_OK;
    if (g.kind == 1) {
        const dim3 blocks((unsigned)((total + TB_WARPS - 1) / TB_WARPS));
        if (g.ca) ez2d_tb_batch_kernel<T, 1, true, true><<<blocks, TB_WARPS * 32, 0, s>>>(jobs, tiles, n);
        else ez2d_tb_batch_kernel<T, 1, true, false><<<blocks, TB_WARPS * 32, 0, s>>>(jobs, tiles, n);
        return OS_OK;
    }
    return g.ca ? launch_interior_batch_ca<T, true>(s, g, jobs, tiles, n, total)
                : launch_interior_batch_ca<T, false>(s, g, jobs, tiles, n, total);
}

static int launch_group_any(int T, cudaStream_t s, const BatchGroup &g, const unsigned char *dev) {
    switch (T) {
        case 1: return launch_group<1>(s, g, dev);
        case 2: return launch_group<2>(s, g, dev);
        case 3: return launch_group<3>(s, g, dev);
        default: return launch_group<4>(s, g, dev);
    }
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace os

extern "C" int os_fdtd2d_batch_create(int32_t device, OsFdtd2DBatch **out) {
    OS_CHECK(out, OS_ERR_INVALID, "os_fdtd2d_batch_create: null argument");
    *out = nullptr;
    std::unique_ptr<OsFdtd2DBatch> b(new OsFdtd2DBatch());
    b->device = device;
    OS_CUDA(cudaSetDevice(device));
    OS_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    OS_CUDA(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
    OS_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    OS_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    for (auto &st : b->staging) OS_CUDA(cudaEventCreateWithFlags(&st.copied, cudaEventDisableTiming));
    OS_CUDA(cudaEventCreate(&b->ev_start));
    OS_CUDA(cudaEventCreate(&b->ev_stop));
    *out = b.release();
    return OS_OK;
}

extern "C" int os_fdtd2d_batch_destroy(OsFdtd2DBatch *b) {
    if (!b) return OS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->side) cudaStreamSynchronize(b->side);
    for (auto &st : b->staging) {
        if (st.host) cudaFreeHost(st.host);
        if (st.copied) cudaEventDestroy(st.copied);
    }
    if (b->ev_start) cudaEventDestroy(b->ev_start);
    if (b->ev_stop) cudaEventDestroy(b->ev_stop);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    cudaStream_t s = b->stream, side = b->side;
    delete b;
    if (s) cudaStreamDestroy(s);
    if (side) cudaStreamDestroy(side);
    return OS_OK;
}

extern "C" int os_fdtd2d_batch_stream(OsFdtd2DBatch *b, void **stream) {
    OS_CHECK(b && stream, OS_ERR_INVALID, "os_fdtd2d_batch_stream: null argument");
    *stream = (void *)b->stream;
    return OS_OK;
}

extern "C" int os_fdtd2d_batch_advance(OsFdtd2DBatch *b, OsFdtd2D *const *handles, int32_t n_jobs, int64_t n_steps,
                                       const float *const *line_values, const int64_t *first_samples,
                                       const int64_t *n_samples, const float *const *phases) {
    using namespace os;
    OS_CHECK(b && (n_jobs == 0 || (handles && line_values && first_samples && n_samples && phases)), OS_ERR_INVALID,
             "os_fdtd2d_batch_advance: null argument");
    OS_CHECK(n_jobs >= 0 && n_steps >= 0, OS_ERR_INVALID, "os_fdtd2d_batch_advance: negative count");
    b->launches = 0;
    if (n_jobs == 0 || n_steps == 0) return OS_OK;
    const int T = handles[0]->steps_per_launch;
    for (int32_t q = 0; q < n_jobs; ++q) {
        OsFdtd2D *h = handles[q];
        OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_batch_advance: job %d has no handle", q);
        OS_TRY(require_ez(h, "os_fdtd2d_batch_advance"));
        OS_TRY(check_advance(h, "os_fdtd2d_batch_advance", n_steps, line_values[q], first_samples[q], n_samples[q],
                             phases[q]));
        OS_CHECK(h->device == b->device, OS_ERR_INVALID, "os_fdtd2d_batch_advance: job %d is on device %d, the batch on "
                 "%d", q, h->device, b->device);
        OS_CHECK(h->variant != 0 && h->steps_per_launch == T, OS_ERR_INVALID,
                 "os_fdtd2d_batch_advance: every job needs the blocked kernels with the same steps per launch (%d)", T);
        OS_CHECK(h->stream == b->stream, OS_ERR_STATE,
                 "os_fdtd2d_batch_advance: job %d is not on the batch stream (os_fdtd2d_set_stream with "
                 "os_fdtd2d_batch_stream)", q);
        OS_CHECK(!h->profiling, OS_ERR_STATE, "os_fdtd2d_batch_advance: job %d has profiling on", q);
        OS_CHECK(h->maps.empty() && h->probes.n == 0 && h->tfsf.empty() && h->poles.empty(), OS_ERR_STATE,
                 "os_fdtd2d_batch_advance: job %d has field-map monitors, field probes, a TFSF box or poles (advance "
                 "it with os_fdtd2d_advance)", q);
    }
    OS_CUDA(cudaSetDevice(b->device));
    // every job's own tables, in its own buffers, as os_fdtd2d_advance uploads them
    for (int32_t q = 0; q < n_jobs; ++q) {
        OsFdtd2D *h = handles[q];
        h->launches = 0;
        h->prof_used = 0;
        if (!h->lines.empty()) OS_TRY(upload(h->line_values, line_values[q], h->lines.size() * (size_t)n_steps,
                                             b->stream));
        size_t phase_floats = 0;
        for (auto &f : h->fluxes) phase_floats += (size_t)n_samples[q] * f->nf * 2;
        if (!h->fluxes.empty() && phase_floats && phases[q])
            OS_TRY(upload(h->phases, phases[q], phase_floats, b->stream));
    }
    // plans of the full-T launches and of the shorter last one, per job
    const int64_t n_launch = (n_steps + T - 1) / T;
    const int T_last = (int)(n_steps - (n_launch - 1) * T);
    struct Plan {
        TBParams interior{}, general{};
        bool has_interior = false;
    };
    // one tile height for the jobs that leave it to the plan, chosen for all their interior tiles together (a large
    // batch gets tall tiles, the last few jobs short ones)
    int batch_rows = 0;
    {
        std::vector<std::pair<int, int>> rects;
        for (int32_t q = 0; q < n_jobs; ++q) {
            Rect in{};
            if (handles[q]->tile_rows == 0 && interior_rect(handles[q], T, in))
                rects.push_back({in.r1 - in.r0, in.c1 - in.c0});
        }
        if (!rects.empty()) batch_rows = wave_rows(handles[0]->sm_count, T, rects);
    }
    std::vector<Plan> plan_full(n_jobs), plan_last(n_jobs);
    for (int32_t q = 0; q < n_jobs; ++q) {
        const int rows = handles[q]->tile_rows > 0 ? 0 : batch_rows;
        plan_tiles(handles[q], T, plan_full[q].interior, plan_full[q].general, plan_full[q].has_interior, rows);
        plan_tiles(handles[q], T_last, plan_last[q].interior, plan_last[q].general, plan_last[q].has_interior, rows);
        for (Plan *pl : {&plan_full[q], &plan_last[q]}) {
            fill_common(handles[q], pl->interior);
            fill_common(handles[q], pl->general);
        }
    }
    std::vector<BatchLaunch> launches((size_t)n_launch);
    for (int64_t l = 0; l < n_launch; ++l) {
        BatchLaunch &L = launches[(size_t)l];
        L.T = l + 1 < n_launch ? T : T_last;
        L.frames.resize((size_t)L.T);
        for (int32_t q = 0; q < n_jobs; ++q) {
            OsFdtd2D *h = handles[q];
            const Plan &pl = l + 1 < n_launch ? plan_full[q] : plan_last[q];
            const int in = (h->cur + (int)(l & 1)) & 1, out = in ^ 1;
            const int64_t m = h->sample_interval, n0 = h->n_step + l * T;
            uint32_t mask = 0;
            for (int st = 1; st <= L.T; ++st)
                if ((n0 + st) % m == 0) mask |= 1u << (st - 1);
            if (h->fluxes.empty()) mask = 0;
            if (h->variant == 1 && pl.general.n_tiles) {
                // the frame: one batched single-step launch per step over the jobs' shrinking bands
                TBParams base = pl.general;
                bind_buffers(h, base, in, out);
                base.line_values = h->line_values.ptr;
                base.values_stride = n_steps;
                base.k0 = l * T;
                base.sample_mask = mask;
                const bool run_interior = pl.has_interior && pl.interior.n_tiles;
                const Rect box = run_interior ? Rect{pl.interior.rects[0].r0, pl.interior.rects[0].r1,
                                                     pl.interior.rects[0].c0, pl.interior.rects[0].c1}
                                              : Rect{0, 0, 0, 0};
                for (int k = 1; k <= L.T; ++k) {
                    const EzFrameParams f = make_frame_params(h, L.T, k, base, run_interior ? &box : nullptr, in, out);
                    if (!f.first[f.n_rects]) continue;
                    FrameStep &fs = L.frames[(size_t)(k - 1)];
                    fs.params.push_back(f);
                    fs.block_start.push_back(fs.block_start.back() + (int32_t)frame_blocks(f));
                }
            }
            for (int kind = 1; kind >= 0; --kind) {
                const TBParams &base = kind == 0 ? pl.interior : pl.general;
                if (kind == 0 && !pl.has_interior) continue;
                if (kind == 1 && h->variant == 1) continue;   // advanced by the frame steps above
                if (!base.n_tiles) continue;
                BatchGroup &g = batch_group(L, kind, h->has_ca, kind == 0 && h->grid.periodic_x,
                                            kind == 0 && h->grid.periodic_y, kind == 0 && h->grid.ny % 4 == 0);
                g.params.push_back(base);
                TBParams &p = g.params.back();
                bind_buffers(h, p, in, out);
                p.line_values = h->line_values.ptr;
                p.values_stride = n_steps;
                p.k0 = l * T;
                p.n0 = n0;
                p.q_first = n0 / m + 1;
                p.sample_mask = mask;
                g.tile_start.push_back(g.tile_start.back() + p.n_tiles);
            }
            const int64_t q_lo = n0 / m + 1, q_hi = (n0 + L.T) / m;
            if (!h->fluxes.empty() && q_hi >= q_lo) {
                size_t offset = 0;
                for (auto &f : h->fluxes) {
                    FluxBatchItem it{};
                    it.stage = f->stage.ptr;
                    it.phases = h->phases.ptr + offset + (size_t)(q_lo - first_samples[q]) * f->nf * 2;
                    it.e_acc = f->e_acc.ptr;
                    it.h_acc = f->h_acc.ptr;
                    it.n = f->hi - f->lo;
                    it.nf = f->nf;
                    it.n_q = (int)(q_hi - q_lo + 1);
                    L.items.push_back(it);
                    L.max_item_cells = std::max(L.max_item_cells, it.n * it.nf);
                    offset += (size_t)n_samples[q] * f->nf * 2;
                }
            }
        }
    }
    // one page-locked block for the whole call, one copy to the device
    size_t total = 0;
    for (auto &L : launches) {
        for (auto &fs : L.frames) {
            if (fs.params.empty()) continue;
            fs.params_off = total = align_up(total, 16);
            total += fs.params.size() * sizeof(EzFrameParams);
            fs.starts_off = total = align_up(total, 16);
            total += fs.block_start.size() * sizeof(int32_t);
        }
        for (auto &g : L.groups) {
            g.params_off = total = align_up(total, 16);
            total += g.params.size() * sizeof(TBParams);
            g.tiles_off = total = align_up(total, 16);
            total += g.tile_start.size() * sizeof(int);
        }
        L.items_off = total = align_up(total, 16);
        total += L.items.size() * sizeof(FluxBatchItem);
    }
    // a ring of staging blocks: a call waits only for the copy of the call kStaging calls back
    OsFdtd2DBatch::Staging &st = b->staging[b->next_staging];
    b->next_staging = (b->next_staging + 1) % OsFdtd2DBatch::kStaging;
    if (st.pending) {
        OS_CUDA(cudaEventSynchronize(st.copied));
        st.pending = false;
    }
    if (total > st.capacity) {   // grown by doubling: cudaFreeHost waits for the device
        if (st.host) OS_CUDA(cudaFreeHost(st.host));
        st.host = nullptr;
        st.capacity = 0;
        const size_t want = std::max(total, (size_t)2 * b->dev.capacity + ((size_t)1 << 20));
        OS_CUDA(cudaHostAlloc((void **)&st.host, want, cudaHostAllocPortable));
        st.capacity = want;
    }
    unsigned char *const host = st.host;
    for (auto &L : launches) {
        for (auto &fs : L.frames) {
            if (fs.params.empty()) continue;
            memcpy(host + fs.params_off, fs.params.data(), fs.params.size() * sizeof(EzFrameParams));
            memcpy(host + fs.starts_off, fs.block_start.data(), fs.block_start.size() * sizeof(int32_t));
        }
        for (auto &g : L.groups) {
            memcpy(host + g.params_off, g.params.data(), g.params.size() * sizeof(TBParams));
            memcpy(host + g.tiles_off, g.tile_start.data(), g.tile_start.size() * sizeof(int));
        }
        if (!L.items.empty()) memcpy(host + L.items_off, L.items.data(), L.items.size() * sizeof(FluxBatchItem));
    }
    // one device block, rewritten by each call's copy behind the previous call's launches on the stream
    OS_TRY(b->dev.alloc(total > b->dev.capacity ? std::max(total, 2 * b->dev.capacity) : total, b->stream));
    OS_CUDA(cudaMemcpyAsync(b->dev.ptr, host, total, cudaMemcpyHostToDevice, b->stream));
    OS_CUDA(cudaEventRecord(st.copied, b->stream));
    st.pending = true;
    OS_CUDA(cudaEventRecord(b->ev_start, b->stream));
    for (auto &L : launches) {
        // the frame steps fork onto the side stream and overlap the interior launches (disjoint cells; both read
        // only the launch's input state), the stream waits for them before the DFT fold
        bool fork = false;
        for (auto &fs : L.frames) fork = fork || !fs.params.empty();
        if (fork) {
            OS_CUDA(cudaEventRecord(b->ev_fork, b->stream));
            OS_CUDA(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
        }
        for (auto &fs : L.frames) {
            if (fs.params.empty()) continue;
            ez2d_frame_step_batch_kernel<<<(unsigned)fs.block_start.back(), 256, 0, b->side>>>(
                reinterpret_cast<const EzFrameParams *>(b->dev.ptr + fs.params_off),
                reinterpret_cast<const int32_t *>(b->dev.ptr + fs.starts_off), (int)fs.params.size());
            b->launches += 1;
        }
        for (auto &g : L.groups) {
            if (g.kind != 1) continue;
            OS_TRY(launch_group_any(L.T, b->stream, g, b->dev.ptr));
            b->launches += 1;
        }
        for (auto &g : L.groups) {
            if (g.kind != 0) continue;
            OS_TRY(launch_group_any(L.T, b->stream, g, b->dev.ptr));
            b->launches += 1;
        }
        if (fork) {
            OS_CUDA(cudaEventRecord(b->ev_join, b->side));
            OS_CUDA(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
        }
        if (!L.items.empty()) {
            const dim3 grid((unsigned)((L.max_item_cells + 255) / 256), (unsigned)L.items.size());
            ez2d_flux_staged_batch_kernel<<<grid, 256, 0, b->stream>>>(
                reinterpret_cast<const FluxBatchItem *>(b->dev.ptr + L.items_off));
            b->launches += 1;
        }
    }
    OS_CUDA(cudaGetLastError());
    OS_CUDA(cudaEventRecord(b->ev_stop, b->stream));
    b->timed = true;
    for (int32_t q = 0; q < n_jobs; ++q) {
        OsFdtd2D *h = handles[q];
        h->cur = (h->cur + (int)(n_launch & 1)) & 1;
        h->n_step += n_steps;
    }
    return OS_OK;
}

extern "C" int os_fdtd2d_batch_last_ms(OsFdtd2DBatch *b, float *ms, int64_t *launches) {
    OS_CHECK(b && ms && launches, OS_ERR_INVALID, "os_fdtd2d_batch_last_ms: null argument");
    OS_CHECK(b->timed, OS_ERR_STATE, "os_fdtd2d_batch_last_ms: no batched advance yet");
    OS_CUDA(cudaSetDevice(b->device));
    OS_CUDA(cudaEventSynchronize(b->ev_stop));
    OS_CUDA(cudaEventElapsedTime(ms, b->ev_start, b->ev_stop));
    *launches = b->launches;
    return OS_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// Discrete adjoint of a 2D E_z simulation (fdtd2d_adjoint.cuh): checkpoints of the forward state, recomputation of a
// segment from its checkpoint with the per-step kernels (bit-identical to every other kernel choice) while the E of
// the design box is recorded, then the transposed steps backward through the segment.
#include "fdtd2d_adjoint.cuh"

struct OsAdjoint2D {
    OsFdtd2D *h = nullptr;
    int32_t bi0 = 0, bi1 = 0, bj0 = 0, bj1 = 0;
    int32_t n_slots = 0, seg_steps = 0;
    size_t slot_floats = 0;
    os::DeviceArray<float> ckpt;                       // n_slots x (ez, hx, hy, psi_e sides, psi_h sides)
    os::DeviceArray<float> le[2], lhx[2], lhy[2];
    os::DeviceArray<float> lpe[2][4], lph[2][4];
    int e_par = 0;                                     // live parity of lambda_E and the psi adjoints
    // Backward pipeline: the recomputation of segment s (engine stream) records E over the box into rec[s & 1] while
    // the transposed sweep of segment s + 1 (adjoint stream) reads rec[(s + 1) & 1]; ev_rec[b] marks a recording into
    // rec[b] done, ev_swept[b] a sweep of rec[b] done (the next recording into it waits for that).
    os::DeviceArray<float> rec[2];                     // (seg_steps + 1) x box each
    os::DeviceArray<double> grad;                      // box
    os::DeviceArray<float> values, src_e, src_h;
    os::DeviceArray<int32_t> src_row;                  // per step of the segment: row of its adjoint source, or -1
    cudaStream_t adj_stream = nullptr;
    cudaEvent_t ev_rec[2] = {nullptr, nullptr}, ev_swept[2] = {nullptr, nullptr};
    bool swept_pending[2] = {false, false};
    cudaGraphExec_t rec_graph[2] = {nullptr, nullptr};           // full-length recomputation, per rec buffer
    cudaGraphExec_t sweep_graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // per rec buffer and parity
    int sweep_monitor[2][2] = {{-1, -1}, {-1, -1}};
    int64_t graph_launches = 0;
};

namespace os {

static size_t adj_box(const OsAdjoint2D *a) { return (size_t)(a->bi1 - a->bi0) * (size_t)(a->bj1 - a->bj0); }

// (device pointer, floats) of every piece of one checkpoint in slot order
static void adj_pieces(OsAdjoint2D *a, std::vector<std::pair<float *, size_t>> &out) {
    OsFdtd2D *h = a->h;
    const size_t n = cells(h);
    const int c = h->cur;
    out.clear();
    out.push_back({h->ez[c].ptr, n});
    out.push_back({h->hx[c].ptr, n});
    out.push_back({h->hy[c].ptr, n});
    for (int s = 0; s < 4; ++s) {
        if (h->psi_e[c][s].ptr) out.push_back({h->psi_e[c][s].ptr, h->psi_e[c][s].count});
        if (h->psi_h[c][s].ptr) out.push_back({h->psi_h[c][s].ptr, h->psi_h[c][s].count});
    }
}

static Ez2DAdjParams adj_params(OsAdjoint2D *a) {
    OsFdtd2D *h = a->h;
    Ez2DAdjParams p{};
    p.nx = h->grid.nx;
    p.ny = h->grid.ny;
    p.px = h->grid.periodic_x;
    p.py = h->grid.periodic_y;
    p.npml = h->grid.npml;
    p.cpml_mask = h->grid.cpml_sides;
    p.ca = h->has_ca ? h->ca.ptr : nullptr;
    p.cb = h->cb.ptr;
    p.da = h->has_dadb ? h->da.ptr : nullptr;
    p.db = h->has_dadb ? h->db.ptr : nullptr;
    p.da_u = h->da_uniform;
    p.db_u = h->db_uniform;
    p.ixe = h->inv_dx_e.ptr;
    p.ixh = h->inv_dx_h.ptr;
    p.iye = h->inv_dy_e.ptr;
    p.iyh = h->inv_dy_h.ptr;
    const int npml = h->grid.npml;
    for (int s = 0; s < 4; ++s) {
        if (!(h->grid.cpml_sides & (1 << s))) continue;
        const float *rows = h->cpml_rows[s].ptr;
        p.b_e[s] = rows;
        p.a_e[s] = rows + npml;
        p.inv_e[s] = rows + 2 * npml;
        p.b_h[s] = rows + 3 * npml;
        p.a_h[s] = rows + 4 * npml;
        p.inv_h[s] = rows + 5 * npml;
    }
    p.bi0 = a->bi0;
    p.bi1 = a->bi1;
    p.bj0 = a->bj0;
    p.bj1 = a->bj1;
    p.grad = a->grad.ptr;
    return p;
}

}  // namespace os

extern "C" int os_fdtd2d_adjoint_create(OsFdtd2D *h, int32_t box_i0, int32_t box_i1, int32_t box_j0, int32_t box_j1,
                                        int32_t n_slots, int32_t segment_steps, OsAdjoint2D **out) {
    using namespace os;
    OS_CHECK(h && out, OS_ERR_INVALID, "os_fdtd2d_adjoint_create: null argument");
    OS_TRY(require_ez(h, "os_fdtd2d_adjoint_create"));
    *out = nullptr;
    OS_CHECK(h->tfsf.empty() && h->poles.empty(), OS_ERR_STATE,
             "os_fdtd2d_adjoint_create: the adjoint does not transpose a TFSF box or a dispersive pole");
    OS_CHECK(h->has_cb && h->has_spacings, OS_ERR_STATE, "os_fdtd2d_adjoint_create: coefficients and spacings first");
    OS_CHECK(0 <= box_i0 && box_i0 < box_i1 && box_i1 <= h->grid.nx && 0 <= box_j0 && box_j0 < box_j1 &&
                 box_j1 <= h->grid.ny, OS_ERR_INVALID, "os_fdtd2d_adjoint_create: design box outside the grid");
    OS_CHECK(n_slots >= 1 && segment_steps >= 1, OS_ERR_INVALID, "os_fdtd2d_adjoint_create: bad checkpoint layout");
    std::unique_ptr<OsAdjoint2D> a(new OsAdjoint2D());
    a->h = h;
    a->bi0 = box_i0;
    a->bi1 = box_i1;
    a->bj0 = box_j0;
    a->bj1 = box_j1;
    a->n_slots = n_slots;
    a->seg_steps = segment_steps;
    OS_TRY(bind_device(h));
    std::vector<std::pair<float *, size_t>> pieces;
    adj_pieces(a.get(), pieces);
    for (auto &pc : pieces) a->slot_floats += pc.second;
    OS_TRY(a->ckpt.alloc(a->slot_floats * (size_t)n_slots));
    const size_t n = cells(h);
    for (int b = 0; b < 2; ++b) {
        OS_TRY(a->le[b].alloc(n));
        OS_TRY(a->lhx[b].alloc(n));
        OS_TRY(a->lhy[b].alloc(n));
        for (int s = 0; s < 4; ++s) {
            if (!(h->grid.cpml_sides & (1 << s))) continue;
            OS_TRY(a->lpe[b][s].alloc(h->psi_e[0][s].count));
            OS_TRY(a->lph[b][s].alloc(h->psi_h[0][s].count));
        }
    }
    for (auto &r : a->rec) OS_TRY(r.alloc((size_t)(segment_steps + 1) * adj_box(a.get())));
    OS_TRY(a->grad.alloc(adj_box(a.get())));
    OS_CUDA(cudaStreamCreateWithFlags(&a->adj_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        OS_CUDA(cudaEventCreateWithFlags(&a->ev_rec[b], cudaEventDisableTiming));
        OS_CUDA(cudaEventCreateWithFlags(&a->ev_swept[b], cudaEventDisableTiming));
    }
    *out = a.release();
    return OS_OK;
}

extern "C" int os_fdtd2d_adjoint_destroy(OsAdjoint2D *a) {
    if (!a) return OS_OK;
    cudaSetDevice(a->h->device);
    cudaStreamSynchronize(a->h->stream);
    if (a->adj_stream) cudaStreamSynchronize(a->adj_stream);
    for (int b = 0; b < 2; ++b) {
        if (a->rec_graph[b]) cudaGraphExecDestroy(a->rec_graph[b]);
        for (cudaGraphExec_t g : a->sweep_graph[b])
            if (g) cudaGraphExecDestroy(g);
        if (a->ev_rec[b]) cudaEventDestroy(a->ev_rec[b]);
        if (a->ev_swept[b]) cudaEventDestroy(a->ev_swept[b]);
    }
    if (a->adj_stream) cudaStreamDestroy(a->adj_stream);
    delete a;
    return OS_OK;
}

extern "C" int os_fdtd2d_adjoint_save(OsAdjoint2D *a, int32_t slot) {
    using namespace os;
    OS_CHECK(a && slot >= 0 && slot < a->n_slots, OS_ERR_INVALID, "os_fdtd2d_adjoint_save: no slot %d", slot);
    OS_TRY(bind_device(a->h));
    std::vector<std::pair<float *, size_t>> pieces;
    adj_pieces(a, pieces);
    float *dst = a->ckpt.ptr + (size_t)slot * a->slot_floats;
    for (auto &pc : pieces) {
        OS_CUDA(cudaMemcpyAsync(dst, pc.first, pc.second * sizeof(float), cudaMemcpyDeviceToDevice, a->h->stream));
        dst += pc.second;
    }
    return OS_OK;
}

extern "C" int os_fdtd2d_adjoint_reset(OsAdjoint2D *a) {
    using namespace os;
    OS_CHECK(a, OS_ERR_INVALID, "os_fdtd2d_adjoint_reset: null handle");
    OS_TRY(bind_device(a->h));
    cudaStream_t s = a->h->stream;
    for (int b = 0; b < 2; ++b) {
        for (DeviceArray<float> *d : {&a->le[b], &a->lhx[b], &a->lhy[b]})
            OS_CUDA(cudaMemsetAsync(d->ptr, 0, d->bytes(), s));
        for (int q = 0; q < 4; ++q) {
            if (a->lpe[b][q].ptr) OS_CUDA(cudaMemsetAsync(a->lpe[b][q].ptr, 0, a->lpe[b][q].bytes(), s));
            if (a->lph[b][q].ptr) OS_CUDA(cudaMemsetAsync(a->lph[b][q].ptr, 0, a->lph[b][q].bytes(), s));
        }
    }
    OS_CUDA(cudaMemsetAsync(a->grad.ptr, 0, a->grad.bytes(), s));
    a->e_par = 0;
    // the adjoint stream's next sweep must also follow these zeroings and every earlier sweep: one wait on the engine
    // stream, which a sweep's own wait for its recording orders anyway; earlier sweeps are joined here
    for (int b = 0; b < 2; ++b) {
        if (a->swept_pending[b]) OS_CUDA(cudaStreamWaitEvent(s, a->ev_swept[b], 0));
        a->swept_pending[b] = false;
    }
    return OS_OK;
}

extern "C" int os_fdtd2d_adjoint_segment(OsAdjoint2D *a, int32_t slot, int64_t step0, int32_t n_steps,
                                         const float *line_values, int32_t monitor_id, int32_t n_sources,
                                         const int32_t *source_steps, const float *source_e, const float *source_h) {
    using namespace os;
    OS_CHECK(a && slot >= 0 && slot < a->n_slots, OS_ERR_INVALID, "os_fdtd2d_adjoint_segment: no slot %d", slot);
    OsFdtd2D *h = a->h;
    OS_CHECK(n_steps >= 1 && n_steps <= a->seg_steps, OS_ERR_INVALID,
             "os_fdtd2d_adjoint_segment: %d steps, the segment holds at most %d", n_steps, a->seg_steps);
    OS_CHECK(h->lines.empty() || line_values, OS_ERR_INVALID, "os_fdtd2d_adjoint_segment: line_values is required");
    OS_CHECK(monitor_id >= 0 && monitor_id < (int32_t)h->fluxes.size(), OS_ERR_INVALID,
             "os_fdtd2d_adjoint_segment: no monitor %d", monitor_id);
    OS_CHECK(n_sources == 0 || (source_steps && source_e && source_h), OS_ERR_INVALID,
             "os_fdtd2d_adjoint_segment: adjoint sources are required");
    for (int32_t q = 0; q < n_sources; ++q)
        OS_CHECK(source_steps[q] >= 0 && source_steps[q] < n_steps && (q == 0 || source_steps[q] > source_steps[q - 1]),
                 OS_ERR_INVALID, "os_fdtd2d_adjoint_segment: source steps must be increasing within the segment");
    OS_TRY(bind_device(h));
    cudaStream_t s = h->stream, as = a->adj_stream;
    const int rb = slot & 1;   // the record buffer of this segment
    const size_t box = adj_box(a);
    // ---- engine stream: recompute the segment from its checkpoint, recording E over the box into rec[rb]
    if (a->swept_pending[rb]) OS_CUDA(cudaStreamWaitEvent(s, a->ev_swept[rb], 0));   // its last reader is done
    {
        std::vector<std::pair<float *, size_t>> pieces;
        adj_pieces(a, pieces);
        const float *src = a->ckpt.ptr + (size_t)slot * a->slot_floats;
        for (auto &pc : pieces) {
            OS_CUDA(cudaMemcpyAsync(pc.first, src, pc.second * sizeof(float), cudaMemcpyDeviceToDevice, s));
            src += pc.second;
        }
    }
    if (!h->lines.empty()) {   // the values of the whole segment length, so a captured body reads them in place
        OS_TRY(a->values.alloc(h->lines.size() * (size_t)a->seg_steps));
        OS_CUDA(cudaMemcpyAsync(a->values.ptr, line_values, h->lines.size() * (size_t)n_steps * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    }
    auto recompute = [&](int32_t steps) -> int {
        const int box_blocks = (int)((box + 255) / 256);
        Ez2DParams p = make_params(h);
        const dim3 block(EZ2D_BLOCK_X, EZ2D_BLOCK_Y);
        const dim3 grid((unsigned)((h->grid.ny + block.x - 1) / block.x),
                        (unsigned)((h->grid.nx + block.y - 1) / block.y));
        float *rec = a->rec[rb].ptr;
        ez2d_record_box_kernel<<<box_blocks, 256, 0, s>>>(p.ez, h->grid.ny, a->bi0, a->bi1, a->bj0, a->bj1, rec);
        for (int32_t k = 0; k < steps; ++k) {   // the E kernel records the box of its own step
            ez2d_h_kernel<<<grid, block, 0, s>>>(p);
            ez2d_e_kernel<<<grid, block, 0, s>>>(p, a->values.ptr, steps, k, rec + (size_t)(k + 1) * box, a->bi0,
                                                 a->bi1, a->bj0, a->bj1);
        }
        return OS_OK;
    };
    // a full-length segment replays a captured graph (its arguments are the same for every segment using rec[rb])
    auto run_captured = [&](cudaStream_t stream, cudaGraphExec_t &exec, const std::function<int()> &body) -> int {
        if (!exec) {
            cudaGraph_t g = nullptr;
            OS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const int rc = body();
            const cudaError_t end = cudaStreamEndCapture(stream, &g);
            if (rc != OS_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            OS_CUDA(end);
            const cudaError_t inst = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            OS_CUDA(inst);
        }
        OS_CUDA(cudaGraphLaunch(exec, stream));
        a->graph_launches += 1;
        return OS_OK;
    };
    if (n_steps == a->seg_steps) OS_TRY(run_captured(s, a->rec_graph[rb], [&] { return recompute(n_steps); }));
    else OS_TRY(recompute(n_steps));
    OS_CUDA(cudaEventRecord(a->ev_rec[rb], s));
    // ---- adjoint stream: the transposed steps backward over rec[rb], the monitor's DFT samples as sources
    OS_CUDA(cudaStreamWaitEvent(as, a->ev_rec[rb], 0));
    const FluxLine2D &mon = *h->fluxes[monitor_id];
    const int n_line = mon.hi - mon.lo;
    {   // source rows and the per-step row table
        std::vector<int32_t> rows((size_t)a->seg_steps, -1);
        for (int32_t q = 0; q < n_sources; ++q) rows[(size_t)source_steps[q]] = q;
        OS_TRY(a->src_row.alloc((size_t)a->seg_steps));
        OS_CUDA(cudaMemcpyAsync(a->src_row.ptr, rows.data(), rows.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                as));
        OS_TRY(a->src_e.alloc((size_t)a->seg_steps * n_line));
        OS_TRY(a->src_h.alloc((size_t)a->seg_steps * n_line));
        if (n_sources) {
            OS_CUDA(cudaMemcpyAsync(a->src_e.ptr, source_e, (size_t)n_sources * n_line * sizeof(float),
                                    cudaMemcpyHostToDevice, as));
            OS_CUDA(cudaMemcpyAsync(a->src_h.ptr, source_h, (size_t)n_sources * n_line * sizeof(float),
                                    cudaMemcpyHostToDevice, as));
        }
        OS_CUDA(cudaStreamSynchronize(as));   // the host rows above are released on return
    }
    const int par = a->e_par;
    auto sweep = [&](int32_t steps) -> int {
        Ez2DAdjParams q = adj_params(a);
        const dim3 ablock(32, 8);
        const dim3 agrid((unsigned)((h->grid.ny + 31) / 32), (unsigned)((h->grid.nx + 7) / 8));
        const float *rec = a->rec[rb].ptr;
        int e = par;
        for (int32_t k = steps - 1; k >= 0; --k) {
            float *lh = mon.normal_axis == 0 ? a->lhy[0].ptr : a->lhx[0].ptr;
            ez2d_adj_source_kernel<<<(n_line + 127) / 128, 128, 0, as>>>(
                a->le[e].ptr, lh, h->grid.ny, mon.normal_axis, mon.position, mon.lo, n_line, a->src_row.ptr, k,
                a->src_e.ptr, a->src_h.ptr);
            q.le_in = a->le[e].ptr;
            q.lhx_in = a->lhx[0].ptr;
            q.lhy_in = a->lhy[0].ptr;
            q.lhx_out = a->lhx[1].ptr;
            q.lhy_out = a->lhy[1].ptr;
            for (int sd = 0; sd < 4; ++sd) {
                q.lpe_in[sd] = a->lpe[e][sd].ptr;
                q.lpe_out[sd] = a->lpe[e ^ 1][sd].ptr;
                q.lph_in[sd] = a->lph[e][sd].ptr;
                q.lph_out[sd] = a->lph[e ^ 1][sd].ptr;
            }
            q.e_next = rec + (size_t)(k + 1) * box;
            q.e_prev = rec + (size_t)k * box;
            ez2d_adj_e_kernel<<<agrid, ablock, 0, as>>>(q);
            q.lhx_in = a->lhx[1].ptr;
            q.lhy_in = a->lhy[1].ptr;
            q.lhx_out = a->lhx[0].ptr;
            q.lhy_out = a->lhy[0].ptr;
            q.le_out = a->le[e ^ 1].ptr;
            ez2d_adj_h_kernel<<<agrid, ablock, 0, as>>>(q);
            e ^= 1;
        }
        return OS_OK;
    };
    if (n_steps == a->seg_steps) {
        cudaGraphExec_t &exec = a->sweep_graph[rb][par];
        if (exec && a->sweep_monitor[rb][par] != monitor_id) {
            OS_CUDA(cudaGraphExecDestroy(exec));
            exec = nullptr;
        }
        a->sweep_monitor[rb][par] = monitor_id;
        OS_TRY(run_captured(as, exec, [&] { return sweep(n_steps); }));
    } else {
        OS_TRY(sweep(n_steps));
    }
    OS_CUDA(cudaEventRecord(a->ev_swept[rb], as));
    a->swept_pending[rb] = true;
    a->e_par = (par + (int)(n_steps & 1)) & 1;
    OS_CUDA(cudaGetLastError());
    h->n_step = step0 + n_steps;   // the live buffers hold the recomputed state at the segment's end
    return OS_OK;
}

extern "C" int os_fdtd2d_adjoint_gradient(OsAdjoint2D *a, double *out) {
    using namespace os;
    OS_CHECK(a && out, OS_ERR_INVALID, "os_fdtd2d_adjoint_gradient: null argument");
    OS_TRY(bind_device(a->h));
    OS_CUDA(cudaMemcpyAsync(out, a->grad.ptr, a->grad.bytes(), cudaMemcpyDeviceToHost, a->adj_stream));
    OS_CUDA(cudaStreamSynchronize(a->adj_stream));
    OS_CUDA(cudaStreamSynchronize(a->h->stream));
    return OS_OK;
}
