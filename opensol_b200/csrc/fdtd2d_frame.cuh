// The frame of a temporally blocked 2D E_z launch, advanced one Yee step per launch.
//
// A blocked launch advances T steps.  The interior kernel writes the cells of the interior rectangle `in` at step
// n + T from the fields at step n alone.  The rest of the grid, the frame F, is advanced here by T single-step
// launches over shrinking regions: step k (1..T) updates R_k = the grid minus `in` shrunk by T - k cells on each
// non-periodic side, reading the state of step k - 1 (R_{k-1} contains every cell R_k reads) and writing that of
// step k.  Step T writes exactly F, into the output buffer set, beside the interior kernel's cells; steps 1..T-1 write
// scratch buffer sets.  Every cell of R_k is one thread: it updates its own H_x, H_y (with their CPML psi), takes the
// H_x left of it from the lane before (the thread of that cell) or, at a warp's first lane and a rectangle's first
// column, evaluates it again, evaluates again the H_y below it (their psi not stored), then updates E_z with its CPML
// psi, the line sources and, on a DFT sample step, stages the flux-line samples of the frame's own cells.  The arithmetic is that
// of ez2d_h_kernel / ez2d_e_kernel, in open_sol's order (fdtd_ez_2d_kernels.py:23-122, boundaries.py:27-37,
// 752-760, core/sources.py:221-229), so the results are the same bits as every other path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd2d_kernels.cuh"
#include "fdtd2d_tb.cuh"

struct EzFrameParams {
    int32_t nx, ny, px, py, npml, cpml_mask;
    const float *ez_in, *hx_in, *hy_in;
    float *ez_out, *hx_out, *hy_out;
    const float *ca, *cb, *da, *db;   // ca NULL: 1; da/db NULL: the uniform values
    float da_u, db_u;
    const float *inv_dx_e, *inv_dx_h, *inv_dy_e, *inv_dy_h;
    const float *cpml_rows[4];        // b_e, a_e, inv_e, b_h, a_h, inv_h (npml each)
    const float *psi_e_in[4], *psi_h_in[4];
    float *psi_e_out[4], *psi_h_out[4];
    int32_t n_lines;
    TBLine lines[TB_MAX_LINES];
    const float *line_values;         // (n_lines, values_stride); this step's column: k_col
    int64_t values_stride, k_col;
    int32_t n_mons;
    TBMon mons[TB_MAX_MONS];
    int32_t sample_slot;              // staging slot of this step, -1 when it is not a DFT sample step
    int32_t in_r0, in_r1, in_c0, in_c1;   // the interior rectangle (its cells are staged by the interior kernel)
    int32_t n_rects;                  // the region of this step: up to 4 rectangles
    int32_t r0[4], r1[4], c0[4], c1[4];
    int64_t first[5];                 // cell offsets of the rectangles
};
static_assert(sizeof(EzFrameParams) % 4 == 0, "EzFrameParams is copied as 32-bit words");

__device__ __forceinline__ float ezf_wrap_hi(float w) { return w * 1.0f + w * 0.0f; }

// The CPML side of an axis (lo_side: SX_LO or SY_LO; lo_side + 1 the hi side) whose H rows (lo: rows 0..npml-1,
// hi: n-npml-1..n-2) hold row r, with its slab row k; -1 when none.
__device__ __forceinline__ int ezf_h_side(int lo_side, int mask, int r, int n, int npml, int &k) {
    if (((mask >> lo_side) & 1) && r < npml) {
        k = r;
        return lo_side;
    }
    if (((mask >> (lo_side + 1)) & 1) && r >= n - npml - 1 && r <= n - 2) {
        k = r - (n - npml - 1);
        return lo_side + 1;
    }
    return -1;
}

// The same for the E rows (lo: rows 1..npml, hi: n-npml-1..n-2).
__device__ __forceinline__ int ezf_e_side(int lo_side, int mask, int r, int n, int npml, int &k) {
    if (((mask >> lo_side) & 1) && r >= 1 && r <= npml) {
        k = r - 1;
        return lo_side;
    }
    if (((mask >> (lo_side + 1)) & 1) && r >= n - npml - 1 && r <= n - 2) {
        k = r - (n - npml - 1);
        return lo_side + 1;
    }
    return -1;
}

// New H_x of face (i, j) (fdtd_ez_2d_kernels.py:41-44, y-side H-row CPML); the last face of an open y keeps its
// value.  psi written when `own`.
__device__ __forceinline__ float ezf_hx_at(const EzFrameParams &p, int i, int j, bool own) {
    const int ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    const float hx_old = __ldg(p.hx_in + idx);
    if (!(j < ny - 1 || p.py)) return hx_old;
    const float e = __ldg(p.ez_in + idx);
    const float da = p.da ? __ldg(p.da + idx) : p.da_u;
    const float db = p.db ? __ldg(p.db + idx) : p.db_u;
    const float e_up = j < ny - 1 ? __ldg(p.ez_in + idx + 1) : ezf_wrap_hi(__ldg(p.ez_in + (size_t)i * ny));
    float v = da * hx_old - db * (e_up - e) * __ldg(p.inv_dy_h + j);
    int k;
    const int s = ezf_h_side(SY_LO, p.cpml_mask, j, ny, npml, k);
    if (s >= 0) {
        const float *rows = p.cpml_rows[s];
        const size_t q_at = (size_t)i * npml + k;
        float q = __ldg(p.psi_h_in[s] + q_at) * rows[3 * npml + k];
        q += rows[4 * npml + k] * (__ldg(p.ez_in + idx + 1) - e) * rows[5 * npml + k];
        if (own) p.psi_h_out[s][q_at] = q;
        v += (-db) * q;
    }
    return v;
}

// New H_y of face (i, j) (fdtd_ez_2d_kernels.py:45-47, x-side H-row CPML); the last face of an open x keeps its value.
__device__ __forceinline__ float ezf_hy_at(const EzFrameParams &p, int i, int j, bool own) {
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    const float hy_old = __ldg(p.hy_in + idx);
    if (!(i < nx - 1 || p.px)) return hy_old;
    const float e = __ldg(p.ez_in + idx);
    const float da = p.da ? __ldg(p.da + idx) : p.da_u;
    const float db = p.db ? __ldg(p.db + idx) : p.db_u;
    const float e_up = i < nx - 1 ? __ldg(p.ez_in + idx + ny) : ezf_wrap_hi(__ldg(p.ez_in + j));
    float v = da * hy_old + db * (e_up - e) * __ldg(p.inv_dx_h + i);
    int k;
    const int s = ezf_h_side(SX_LO, p.cpml_mask, i, nx, npml, k);
    if (s >= 0) {
        const float *rows = p.cpml_rows[s];
        const size_t q_at = (size_t)k * ny + j;
        float q = __ldg(p.psi_h_in[s] + q_at) * rows[3 * npml + k];
        q += rows[4 * npml + k] * (__ldg(p.ez_in + idx + ny) - e) * rows[5 * npml + k];
        if (own) p.psi_h_out[s][q_at] = q;
        v += db * q;
    }
    return v;
}

// Cells of a step's region.
__device__ __forceinline__ int64_t ezf_cells(const EzFrameParams &p) {
    return p.n_rects == 1 ? p.first[1] : p.n_rects == 2 ? p.first[2] : p.n_rects == 3 ? p.first[3] : p.first[4];
}

// The step of the region's t-th cell.  Every lane of the warp calls it (the H_x hand-over is a warp shuffle); lanes
// with t >= ezf_cells(p) compute nothing.
__device__ __forceinline__ void ezf_cell(const EzFrameParams &p, int64_t t) {
    const bool valid = t < ezf_cells(p);
    if (!valid) t = 0;
    // the rectangle of this cell, selected without indexing the parameter arrays by a runtime value
    int k = 0;
    if (p.n_rects > 1 && t >= p.first[1]) k = 1;
    if (p.n_rects > 2 && t >= p.first[2]) k = 2;
    if (p.n_rects > 3 && t >= p.first[3]) k = 3;
    const int64_t first = k == 0 ? 0 : k == 1 ? p.first[1] : k == 2 ? p.first[2] : p.first[3];
    const int rr0 = k == 0 ? p.r0[0] : k == 1 ? p.r0[1] : k == 2 ? p.r0[2] : p.r0[3];
    const int cc0 = k == 0 ? p.c0[0] : k == 1 ? p.c0[1] : k == 2 ? p.c0[2] : p.c0[3];
    const int cc1 = k == 0 ? p.c1[0] : k == 1 ? p.c1[1] : k == 2 ? p.c1[2] : p.c1[3];
    const int64_t local = t - first;
    const int w = cc1 - cc0;
    int i, j;
    if (local < 0x7fffffff) {   // 32-bit division for every cell but those of a rectangle past 2^31 cells
        i = rr0 + (int)local / w, j = cc0 + (int)local % w;
    } else {
        i = rr0 + (int)(local / w), j = cc0 + (int)(local % w);
    }
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;

    // ---- H half step: this cell's faces (stored), the H_x left of it (the lane before's when that lane holds
    // cell (i, j - 1) of the same rectangle, else evaluated again) and the H_y below it (evaluated again)
    float hx_c = 0.0f, hy_c = 0.0f;
    if (valid) {
        hx_c = ezf_hx_at(p, i, j, true);
        hy_c = ezf_hy_at(p, i, j, true);
        p.hx_out[idx] = hx_c;
        p.hy_out[idx] = hy_c;
    }
    const float hx_lane_before = __shfl_up_sync(0xffffffffu, hx_c, 1);
    if (!valid) return;
    const float one = 1.0f, zero = 0.0f;
    float hy_dn = 0.0f, hx_left = 0.0f;
    if (i >= 1) hy_dn = ezf_hy_at(p, i - 1, j, false);
    else if (p.px) hy_dn = ezf_hy_at(p, nx - 1, j, false);
    if ((threadIdx.x & 31) != 0 && j > cc0) hx_left = hx_lane_before;   // thread t - 1: cell (i, j - 1)
    else if (j >= 1) hx_left = ezf_hx_at(p, i, j - 1, false);
    else if (p.py) hx_left = ezf_hx_at(p, i, ny - 1, false);

    // ---- E half step (fdtd_ez_2d_kernels.py:103-120), E-row CPML x then y sides, line sources
    float curl;
    if (i >= 1) curl = (hy_c - hy_dn) * __ldg(p.inv_dx_e + i);
    else if (p.px) curl = (hy_c - (hy_dn * one - hy_dn * zero)) * __ldg(p.inv_dx_e + i);
    else curl = hy_c * __ldg(p.inv_dx_e + i);
    if (j >= 1) curl -= (hx_c - hx_left) * __ldg(p.inv_dy_e + j);
    else if (p.py) curl -= (hx_c - (hx_left * one - hx_left * zero)) * __ldg(p.inv_dy_e + j);
    else curl -= hx_c * __ldg(p.inv_dy_e + j);
    const float cb = __ldg(p.cb + idx);
    const float ez_old = __ldg(p.ez_in + idx);
    float v = (p.ca ? __ldg(p.ca + idx) * ez_old : ez_old) + cb * curl;
    if (p.cpml_mask) {   // the E-row CPML of the x side holding row i, then of the y side holding column j
        int kr;
        const int sx = ezf_e_side(SX_LO, p.cpml_mask, i, nx, npml, kr);
        if (sx >= 0) {
            const float *rows = p.cpml_rows[sx];
            const size_t q_at = (size_t)kr * ny + j;
            float q = __ldg(p.psi_e_in[sx] + q_at) * rows[kr];
            q += rows[npml + kr] * (hy_c - hy_dn) * rows[2 * npml + kr];
            p.psi_e_out[sx][q_at] = q;
            v += cb * q;
        }
        const int sy = ezf_e_side(SY_LO, p.cpml_mask, j, ny, npml, kr);
        if (sy >= 0) {
            const float *rows = p.cpml_rows[sy];
            const size_t q_at = (size_t)i * npml + kr;
            float q = __ldg(p.psi_e_in[sy] + q_at) * rows[kr];
            q += rows[npml + kr] * (hx_c - hx_left) * rows[2 * npml + kr];
            p.psi_e_out[sy][q_at] = q;
            v += (-cb) * q;
        }
    }
    for (int l = 0; l < p.n_lines; ++l) {
        const TBLine &L = p.lines[l];
        const int along = L.axis == 0 ? i : j, across = L.axis == 0 ? j : i;
        if (across == L.position && along >= L.lo && along < L.hi) {
            const float value = p.line_values[(size_t)l * p.values_stride + p.k_col];
            if (value != 0.0f) v += value * L.profile[along - L.lo];
        }
    }
    p.ez_out[idx] = v;

    // ---- DFT sample of the frame's own cells (the interior kernel stages the interior's)
    if (p.sample_slot >= 0 && !(i >= p.in_r0 && i < p.in_r1 && j >= p.in_c0 && j < p.in_c1)) {
        const int slot = p.sample_slot;
        for (int m = 0; m < p.n_mons; ++m) {
            const TBMon &M = p.mons[m];
            const int n = M.hi - M.lo;
            if (M.normal_axis == 0) {
                if (i == M.position && j >= M.lo && j < M.hi) {
                    M.stage[(slot * 2) * n + (j - M.lo)] = v;
                    M.stage[(slot * 2 + 1) * n + (j - M.lo)] = hy_c;
                }
            } else if (j == M.position && i >= M.lo && i < M.hi) {
                M.stage[(slot * 2) * n + (i - M.lo)] = v;
                M.stage[(slot * 2 + 1) * n + (i - M.lo)] = hx_c;
            }
        }
    }
}

__global__ void __launch_bounds__(256) ez2d_frame_step_kernel(const EzFrameParams p) {
    ezf_cell(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// One frame step of several simulations in one launch.  Each block serves one job: job q owns blocks
// [block_start[q], block_start[q + 1]) and its cells in order; the block copies the job's parameters into shared
// memory once, so the per-cell code reads them from there.
__global__ void __launch_bounds__(256) ez2d_frame_step_batch_kernel(const EzFrameParams *__restrict__ jobs,
                                                                    const int32_t *__restrict__ block_start,
                                                                    int n_jobs) {
    __shared__ __align__(16) unsigned char smem[sizeof(EzFrameParams)];
    const int b = blockIdx.x;
    int lo = 0, hi = n_jobs - 1;   // the job q with block_start[q] <= b < block_start[q + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (block_start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const uint32_t *src = reinterpret_cast<const uint32_t *>(jobs + lo);
    uint32_t *dst = reinterpret_cast<uint32_t *>(smem);
    for (int w = threadIdx.x; w < (int)(sizeof(EzFrameParams) / 4); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    const EzFrameParams &p = *reinterpret_cast<const EzFrameParams *>(smem);
    ezf_cell(p, (int64_t)(b - block_start[lo]) * blockDim.x + threadIdx.x);
}
