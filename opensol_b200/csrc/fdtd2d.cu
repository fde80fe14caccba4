// 2D E_z-polarisation FDTD engine for sm_100a: device state, step kernels and the os_fdtd2d_* C ABI.
//
// One Yee step = the H kernel (Yee H update with the H-row CPML psi recursion and correction fused in) followed by the
// E kernel (Yee E update, E-row CPML, then the soft line sources), and every sample_interval steps the line-DFT kernel.
// This is open_sol's step (open_sol/physics/em/solvers/fdtd_ez_2d.py:71-119) with its separate CPML and source
// launches folded into the two field passes.  The arithmetic of every cell follows the reference's evaluation order
// (fdtd_ez_2d_kernels.py:23-122, boundaries.py:27-37, core/sources.py:146-154) and the file is compiled with
// -fmad=false, so each product and sum is rounded on its own as on the CPU: results are bit-identical to open_sol's
// CPU backend.  The CPML corrections of a cell are applied in FACES order (x sides, then y sides), as open_sol's one
// launch per side does.
#include "common.cuh"
#include "fdtd2d_kernels.cuh"

#include <vector>
#include <memory>

namespace os {

struct LineSource2D {
    int32_t axis, position, lo, hi;
    DeviceArray<float> profile;
};

struct FluxLine2D {
    int32_t normal_axis, position, lo, hi, nf;
    DeviceArray<double> e_acc, h_acc;   // (nf, n) complex128 as double pairs
};

}  // namespace os

struct OsFdtd2D {
    OsGrid2D grid{};
    cudaStream_t stream = nullptr;        // the stream every call enqueues on
    cudaStream_t own_stream = nullptr;    // created with the handle, destroyed with it
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool timed = false;
    os::DeviceArray<float> ez, hx, hy;
    os::DeviceArray<float> ca, cb, da, db;
    float da_uniform = 1.0f, db_uniform = 0.0f;
    bool has_ca = false, has_dadb = false, has_cb = false, has_spacings = false;
    os::DeviceArray<float> inv_dx_e, inv_dx_h, inv_dy_e, inv_dy_h;
    os::DeviceArray<float> cpml_rows[4];   // per side: b_e, a_e, inv_e, b_h, a_h, inv_h (6 * npml)
    os::DeviceArray<float> psi_e[4], psi_h[4];
    bool cpml_set[4] = {false, false, false, false};
    std::vector<std::unique_ptr<os::LineSource2D>> lines;
    std::vector<std::unique_ptr<os::FluxLine2D>> fluxes;
    int64_t sample_interval = 1;
    int64_t n_step = 0;
    os::DeviceArray<float> line_values;   // (n_lines, n_steps) of the current chunk
    os::DeviceArray<float> phases;        // per monitor (n_samples, nf, 2) of the current chunk
    int device = 0;
};

namespace os {

static int bind_device(OsFdtd2D *h) {
    OS_CUDA(cudaSetDevice(h->device));
    return OS_OK;
}

static size_t cells(const OsFdtd2D *h) { return (size_t)h->grid.nx * (size_t)h->grid.ny; }

static int zero_state(OsFdtd2D *h) {
    const size_t n = cells(h);
    OS_CUDA(cudaMemsetAsync(h->ez.ptr, 0, n * sizeof(float), h->stream));
    OS_CUDA(cudaMemsetAsync(h->hx.ptr, 0, n * sizeof(float), h->stream));
    OS_CUDA(cudaMemsetAsync(h->hy.ptr, 0, n * sizeof(float), h->stream));
    for (int s = 0; s < 4; ++s) {
        if (h->psi_e[s].ptr) OS_CUDA(cudaMemsetAsync(h->psi_e[s].ptr, 0, h->psi_e[s].bytes(), h->stream));
        if (h->psi_h[s].ptr) OS_CUDA(cudaMemsetAsync(h->psi_h[s].ptr, 0, h->psi_h[s].bytes(), h->stream));
    }
    for (auto &f : h->fluxes) {
        OS_CUDA(cudaMemsetAsync(f->e_acc.ptr, 0, f->e_acc.bytes(), h->stream));
        OS_CUDA(cudaMemsetAsync(f->h_acc.ptr, 0, f->h_acc.bytes(), h->stream));
    }
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
    p.ez = h->ez.ptr;
    p.hx = h->hx.ptr;
    p.hy = h->hy.ptr;
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
        p.psi_e[s] = h->psi_e[s].ptr;
        p.psi_h[s] = h->psi_h[s].ptr;
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

}  // namespace os

using namespace os;

extern "C" int os_fdtd2d_create(const OsGrid2D *grid, OsFdtd2D **out) {
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
    h->stream = h->own_stream;
    OS_CUDA(cudaEventCreate(&h->ev_start));
    OS_CUDA(cudaEventCreate(&h->ev_stop));
    const size_t n = cells(h.get());
    OS_TRY(h->ez.alloc(n));
    OS_TRY(h->hx.alloc(n));
    OS_TRY(h->hy.alloc(n));
    for (int s = 0; s < 4; ++s) {
        if (!(g.cpml_sides & (1 << s))) continue;
        const size_t slab = (s < 2 ? (size_t)g.ny : (size_t)g.nx) * (size_t)g.npml;
        OS_TRY(h->psi_e[s].alloc(slab));
        OS_TRY(h->psi_h[s].alloc(slab));
        OS_TRY(h->cpml_rows[s].alloc(6 * (size_t)g.npml));
    }
    OS_TRY(zero_state(h.get()));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return OS_OK;
}

extern "C" int os_fdtd2d_destroy(OsFdtd2D *h) {
    if (!h) return OS_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    cudaStream_t stream = h->own_stream;
    delete h;   // frees the device arrays
    if (stream) cudaStreamDestroy(stream);
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
    h->has_spacings = true;
    return OS_OK;
}

extern "C" int os_fdtd2d_set_materials(OsFdtd2D *h, const float *eps_r, const float *sigma_e, const float *mu_r,
                                       const float *sigma_m, float dt, float eps0, float mu0) {
    OS_CHECK(h && eps_r, OS_ERR_INVALID, "os_fdtd2d_set_materials: eps_r is required");
    OS_TRY(bind_device(h));
    const size_t n = cells(h);
    OS_TRY(h->cb.alloc(n));
    // eps_r / sigma_e are staged in temporary device arrays (freed after the coefficient kernel has run); ca is only
    // kept for a lossy grid.
    DeviceArray<float> eps_dev, sigma_dev;
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
        DeviceArray<float> mu_dev, sm_dev;
        if (mu_r) OS_TRY(upload(mu_dev, mu_r, n, h->stream));
        if (sigma_m) OS_TRY(upload(sm_dev, sigma_m, n, h->stream));
        OS_TRY(h->da.alloc(n));
        OS_TRY(h->db.alloc(n));
        ez2d_h_coefficients_kernel<<<blocks, threads, 0, h->stream>>>(mu_dev.ptr, sm_dev.ptr, dt, mu0, n, h->da.ptr,
                                                                      h->db.ptr);
        OS_CUDA(cudaGetLastError());
        h->has_dadb = true;
        OS_CUDA(cudaStreamSynchronize(h->stream));   // the staging arrays are freed on return
    } else {
        // vacuum permeability: da = (1 - 0) / 1, db = (dt / mu0) / 1 (fdtd_ez_2d_kernels.py:335-340)
        const float mu = 1.0f * mu0;
        const float k = (0.0f * dt) / (2.0f * mu);
        const float denom = 1.0f + k;
        h->da_uniform = (1.0f - k) / denom;
        h->db_uniform = (dt / mu) / denom;
        h->has_dadb = false;
        OS_CUDA(cudaStreamSynchronize(h->stream));
    }
    return OS_OK;
}

extern "C" int os_fdtd2d_set_coefficients(OsFdtd2D *h, const float *ca, const float *cb, const float *da,
                                          const float *db, float da_uniform, float db_uniform) {
    OS_CHECK(h && cb, OS_ERR_INVALID, "os_fdtd2d_set_coefficients: cb is required");
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
    OS_CHECK(h && cb, OS_ERR_INVALID, "os_fdtd2d_read_cb: null argument");
    OS_CHECK(h->has_cb, OS_ERR_STATE, "os_fdtd2d_read_cb: coefficients are not set");
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(cb, h->cb.ptr, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
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

extern "C" int os_fdtd2d_advance(OsFdtd2D *h, int64_t n_steps, const float *line_values, int64_t first_sample,
                                 int64_t n_samples, const float *phases) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_advance: null handle");
    OS_CHECK(n_steps >= 0, OS_ERR_INVALID, "n_steps must be >= 0, got %lld", (long long)n_steps);
    OS_CHECK(h->has_cb && h->has_spacings, OS_ERR_STATE, "os_fdtd2d_advance: coefficients and spacings must be set");
    for (int s = 0; s < 4; ++s)
        OS_CHECK(!(h->grid.cpml_sides & (1 << s)) || h->cpml_set[s], OS_ERR_STATE,
                 "os_fdtd2d_advance: CPML side %d has no recursion rows", 1 << s);
    if (n_steps == 0) return OS_OK;
    OS_CHECK(h->lines.empty() || line_values, OS_ERR_INVALID, "os_fdtd2d_advance: line_values is required");
    const int64_t m = h->sample_interval;
    const int64_t q_first = h->n_step / m + 1, q_last = (h->n_step + n_steps) / m;
    if (!h->fluxes.empty() && q_last >= q_first) {
        OS_CHECK(phases && first_sample <= q_first && first_sample + n_samples - 1 >= q_last, OS_ERR_INVALID,
                 "os_fdtd2d_advance: the phase table covers samples [%lld, %lld), the chunk needs [%lld, %lld]",
                 (long long)first_sample, (long long)(first_sample + n_samples), (long long)q_first,
                 (long long)q_last);
    }
    OS_TRY(bind_device(h));
    if (!h->lines.empty()) OS_TRY(upload(h->line_values, line_values, h->lines.size() * (size_t)n_steps, h->stream));
    size_t phase_floats = 0;
    for (auto &f : h->fluxes) phase_floats += (size_t)n_samples * f->nf * 2;
    if (!h->fluxes.empty() && phase_floats && phases) OS_TRY(upload(h->phases, phases, phase_floats, h->stream));

    Ez2DParams p = make_params(h);
    const dim3 block(EZ2D_BLOCK_X, EZ2D_BLOCK_Y);
    const dim3 grid((unsigned)((h->grid.ny + block.x - 1) / block.x), (unsigned)((h->grid.nx + block.y - 1) / block.y));
    OS_CUDA(cudaEventRecord(h->ev_start, h->stream));
    for (int64_t k = 0; k < n_steps; ++k) {
        ez2d_h_kernel<<<grid, block, 0, h->stream>>>(p);
        ez2d_e_kernel<<<grid, block, 0, h->stream>>>(p, h->line_values.ptr, n_steps, k);
        h->n_step += 1;
        if (!h->fluxes.empty() && h->n_step % m == 0) {
            const int64_t q = h->n_step / m;
            size_t offset = 0;
            for (auto &f : h->fluxes) {
                const float *ph = h->phases.ptr + offset + (size_t)(q - first_sample) * f->nf * 2;
                const int n = f->hi - f->lo;
                const int total = n * f->nf;
                ez2d_flux_kernel<<<(total + 255) / 256, 256, 0, h->stream>>>(
                    h->ez.ptr, f->normal_axis == 0 ? h->hy.ptr : h->hx.ptr, h->grid.ny, f->normal_axis, f->position,
                    f->lo, n, f->nf, ph, f->e_acc.ptr, f->h_acc.ptr);
                offset += (size_t)n_samples * f->nf * 2;
            }
        }
    }
    OS_CUDA(cudaEventRecord(h->ev_stop, h->stream));
    OS_CUDA(cudaGetLastError());
    h->timed = true;
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
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

static float *component_ptr(OsFdtd2D *h, int32_t component) {
    switch (component) {
        case OS_EZ: return h->ez.ptr;
        case OS_HX: return h->hx.ptr;
        case OS_HY: return h->hy.ptr;
        default: return nullptr;
    }
}

extern "C" int os_fdtd2d_read_field(OsFdtd2D *h, int32_t component, float *out) {
    OS_CHECK(h && out, OS_ERR_INVALID, "os_fdtd2d_read_field: null argument");
    float *src = component_ptr(h, component);
    OS_CHECK(src, OS_ERR_INVALID, "os_fdtd2d_read_field: unknown component %d", component);
    OS_TRY(bind_device(h));
    OS_CUDA(cudaMemcpyAsync(out, src, cells(h) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
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
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd2d_set_stream(OsFdtd2D *h, void *cuda_stream) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd2d_set_stream: null handle");
    OS_TRY(bind_device(h));
    cudaStream_t next = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
    if (next != h->stream) {
        OS_CUDA(cudaStreamSynchronize(h->stream));
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
