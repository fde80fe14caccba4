// Device kernels of the 2D H_z-polarisation engine (H_z at cell centres, E_x on the hi-y faces, E_y on the hi-x
// faces).  Compiled with -fmad=false: every product and sum is rounded on its own, in the order of open_sol's CPU
// twins, so the results are bit-identical to the reference CPU backend:
//   H_z: curl = (E_x[j] - E_x[j-1]) iye[j] - (E_y[i] - E_y[i-1]) ixe[i] (the lo sample below row 0 is the wrapped
//        E * 1 - E * 0 on a periodic axis and absent otherwise), H_z = da H_z + db curl
//        (fdtd_hz_2d_kernels.py:28-91); then the cell-centre CPML rows, x sides (source E_y, H_z += (-db) psi) before
//        y sides (source E_x, H_z += db psi), psi = b psi + a (E[r] - E[r-1]) inv (boundaries.py:27-37,764-767);
//   E_x = ca_x E_x + cb_x (H_z[j+1] - H_z) iyh[j], E_y = ca_y E_y - cb_y (H_z[i+1] - H_z) ixh[i]; the last face of an
//        open axis is not updated, of a periodic one it reads H_z * 1 + H_z * 0 of row 0 (fdtd_hz_2d_kernels.py:94-174);
//        then the hi-face CPML rows, psi = b psi + a (H_z[r+1] - H_z[r]) inv, E_y += (-cb_y) psi on the x sides,
//        E_x += cb_x psi on the y sides (boundaries.py:769-772); then the tangential sheet sources in add order,
//        E += value * profile (physics/em/sources.py:469-480).
//
// Two kernel sets:
//   hz2d_h_kernel + hz2d_e_kernel: one thread per cell, one launch per half step, fields updated in place (the plain
//        form of the arithmetic, variant 0);
//   hz2d_step_kernel: one launch per Yee step reading one field / psi buffer set and writing the other.  A CTA owns a
//        strip of 128 columns and a run of rows; it streams down the rows computing H_z of row i (own columns plus
//        the one column right of the strip, from the old E only), then E_x of row i and E_y of row i - 1 from the new
//        H_z held in shared memory and registers, so each field is read and written once per step.  The CTA also
//        computes H_z of the row after its run (not stored) for the E_y of its last row.  With EPS (lossless, eps_xx
//        = eps_yy, uniform permeability) the face coefficients are not stored: cb = dt / (eps_face eps0) is evaluated
//        from one eps_r word per cell exactly as the coefficient kernel does (denominator 1 + 0 = 1), trading two
//        divisions for 8 bytes per cell.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd2d_kernels.cuh"

#define HZ_STRIP 128

struct Hz2DParams {
    int32_t nx, ny, px, py, npml, cpml_mask;
    const float *hz_in, *ex_in, *ey_in;
    float *hz_out, *ex_out, *ey_out;
    const float *ca_x, *cb_x, *ca_y, *cb_y;   // ca NULL: 1
    const float *da, *db;                     // NULL: the uniform values
    float da_u, db_u;
    const float *eps;                         // eps_r per cell (EPS kernels)
    const float *lo_x, *up_x, *lo_y, *up_y;   // face shares along x (nx,) and y (ny,) (EPS kernels)
    float dt, eps0;
    const float *ixe, *ixh, *iye, *iyh;
    const float *b_e[4], *a_e[4], *inv_e[4], *b_h[4], *a_h[4], *inv_h[4];
    const float *psi_e_in[4], *psi_h_in[4];
    float *psi_e_out[4], *psi_h_out[4];
    int32_t n_lines;
    LineSrcDev lines[OS_MAX_LINES_2D];
    const float *line_values;
    int64_t values_stride, k_step;
    int32_t rows_per_cta;
};

__device__ __forceinline__ float hz_wrap_lo(float w) { return w * 1.0f - w * 0.0f; }
__device__ __forceinline__ float hz_wrap_hi(float w) { return w * 1.0f + w * 0.0f; }

// Slab row of cell-centre row r on side s (lo: rows 1..npml, hi: n-npml-1..n-2), -1 outside.
__device__ __forceinline__ int hz_e_row(int s, int r, int n, int npml) {
    const int k = (s == SX_LO || s == SY_LO) ? r - 1 : r - (n - npml - 1);
    return (k >= 0 && k < npml) ? k : -1;
}

// Slab row of hi-face row r on side s (lo: rows 0..npml-1, hi: n-npml-1..n-2), -1 outside.
__device__ __forceinline__ int hz_h_row(int s, int r, int n, int npml) {
    const int k = (s == SX_LO || s == SY_LO) ? r : r - (n - npml - 1);
    return (k >= 0 && k < npml) ? k : -1;
}

// New H_z of cell (r, j) from the input buffers (r, j physical).  Returns the cell's own old E_x and E_y in ex_c /
// ey_c.  The CPML psi of the cell is written only when `own`.
__device__ __forceinline__ float hz2d_hz_at(const Hz2DParams &p, int r, int j, bool own, float &ex_c, float &ey_c) {
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)r * ny + j;
    ex_c = __ldg(p.ex_in + idx);
    ey_c = __ldg(p.ey_in + idx);
    float dex, dey;   // E[r] - E[r - 1] along y (E_x) and x (E_y); the bare sample when there is no lo neighbour
    if (j >= 1) dex = ex_c - __ldg(p.ex_in + idx - 1);
    else if (p.py) dex = ex_c - hz_wrap_lo(__ldg(p.ex_in + idx + ny - 1));
    else dex = ex_c;
    if (r >= 1) dey = ey_c - __ldg(p.ey_in + idx - ny);
    else if (p.px) dey = ey_c - hz_wrap_lo(__ldg(p.ey_in + (size_t)(nx - 1) * ny + j));
    else dey = ey_c;
    float curl = dex * __ldg(p.iye + j);
    curl -= dey * __ldg(p.ixe + r);
    const float da = p.da ? __ldg(p.da + idx) : p.da_u;
    const float db = p.db ? __ldg(p.db + idx) : p.db_u;
    float v = da * __ldg(p.hz_in + idx) + db * curl;
    if (p.cpml_mask) {
        for (int s = 0; s < 4; ++s) {
            if (!(p.cpml_mask & (1 << s))) continue;
            const bool xs = s < 2;
            const int k = hz_e_row(s, xs ? r : j, xs ? nx : ny, npml);
            if (k < 0) continue;
            const size_t q_at = xs ? (size_t)k * ny + j : (size_t)r * npml + k;
            float q = p.psi_e_in[s][q_at] * p.b_e[s][k];
            q += p.a_e[s][k] * (xs ? dey : dex) * p.inv_e[s][k];
            if (own) p.psi_e_out[s][q_at] = q;
            v += (xs ? -db : db) * q;
        }
    }
    return v;
}

// New E_x of face (r, j) given H_z (r, j) and the H_z difference operand: hz_up = H_z(r, j + 1), already the wrapped
// H_z * 1 + H_z * 0 of column 0 on a periodic y for j = ny - 1.  Writes psi when `own` (always, in practice).
__device__ __forceinline__ float hz2d_ex_at(const Hz2DParams &p, int r, int j, float ex_old, float ca, float cb,
                                            float h, float hz_up) {
    const int ny = p.ny, npml = p.npml;
    const float diff = hz_up - h;
    float v = ca * ex_old + cb * diff * p.iyh[j];
    if (p.cpml_mask & ((1 << SY_LO) | (1 << SY_HI))) {
        for (int s = SY_LO; s <= SY_HI; ++s) {
            if (!(p.cpml_mask & (1 << s))) continue;
            const int k = hz_h_row(s, j, ny, npml);
            if (k < 0) continue;
            const size_t q_at = (size_t)r * npml + k;
            float q = p.psi_h_in[s][q_at] * p.b_h[s][k];
            q += p.a_h[s][k] * diff * p.inv_h[s][k];
            p.psi_h_out[s][q_at] = q;
            v += cb * q;
        }
    }
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &L = p.lines[l];
        if (L.axis == 0 && L.position == j && r >= L.lo && r < L.hi) {
            const float value = p.line_values[(size_t)l * p.values_stride + p.k_step];
            if (value != 0.0f) v += value * L.profile[r - L.lo];
        }
    }
    return v;
}

// New E_y of face (r, j) given H_z (r, j) and hz_up = H_z(r + 1, j) (the wrapped form of row 0 for r = nx - 1).
__device__ __forceinline__ float hz2d_ey_at(const Hz2DParams &p, int r, int j, float ey_old, float ca, float cb,
                                            float h, float hz_up) {
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const float diff = hz_up - h;
    float v = ca * ey_old - cb * diff * p.ixh[r];
    if (p.cpml_mask & ((1 << SX_LO) | (1 << SX_HI))) {
        for (int s = SX_LO; s <= SX_HI; ++s) {
            if (!(p.cpml_mask & (1 << s))) continue;
            const int k = hz_h_row(s, r, nx, npml);
            if (k < 0) continue;
            const size_t q_at = (size_t)k * ny + j;
            float q = p.psi_h_in[s][q_at] * p.b_h[s][k];
            q += p.a_h[s][k] * diff * p.inv_h[s][k];
            p.psi_h_out[s][q_at] = q;
            v += (-cb) * q;
        }
    }
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &L = p.lines[l];
        if (L.axis == 1 && L.position == r && j >= L.lo && j < L.hi) {
            const float value = p.line_values[(size_t)l * p.values_stride + p.k_step];
            if (value != 0.0f) v += value * L.profile[j - L.lo];
        }
    }
    return v;
}

// ---------------------------------------------------------------------------------------------- per half step

__global__ void __launch_bounds__(EZ2D_BLOCK_X *EZ2D_BLOCK_Y) hz2d_h_kernel(const Hz2DParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    float ex_c, ey_c;
    const float v = hz2d_hz_at(p, i, j, true, ex_c, ey_c);
    p.hz_out[(size_t)i * p.ny + j] = v;
}

__global__ void __launch_bounds__(EZ2D_BLOCK_X *EZ2D_BLOCK_Y) hz2d_e_kernel(const Hz2DParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = p.nx, ny = p.ny;
    if (i >= nx || j >= ny) return;
    const size_t idx = (size_t)i * ny + j;
    const float *hz = p.hz_in;   // the updated H_z (in place)
    const float h = hz[idx];
    if (j < ny - 1 || p.py) {
        const float up = j < ny - 1 ? hz[idx + 1] : hz_wrap_hi(hz[(size_t)i * ny]);
        p.ex_out[idx] = hz2d_ex_at(p, i, j, p.ex_in[idx], p.ca_x ? p.ca_x[idx] : 1.0f, p.cb_x[idx], h, up);
    }
    if (i < nx - 1 || p.px) {
        const float up = i < nx - 1 ? hz[idx + ny] : hz_wrap_hi(hz[j]);
        p.ey_out[idx] = hz2d_ey_at(p, i, j, p.ey_in[idx], p.ca_y ? p.ca_y[idx] : 1.0f, p.cb_y[idx], h, up);
    }
}

// ---------------------------------------------------------------------------------------------- fused step

// cb of a lossless face from the two cells' eps_r and the face shares: the coefficient kernel's arithmetic with
// sigma = 0 (k = 0, denominator exactly 1).
__device__ __forceinline__ float hz_cb_lossless(float eps_self, float eps_partner, float lower, float upper, float dt,
                                                float eps0) {
    const float face = eps_self * lower + eps_partner * upper;
    return dt / (face * eps0);
}

template <bool EPS>
__global__ void __launch_bounds__(HZ_STRIP) hz2d_step_kernel(const Hz2DParams p) {
    __shared__ float s_hz[2][HZ_STRIP + 1];
    __shared__ float s_eps[2][HZ_STRIP + 1];
    const int t = threadIdx.x;
    const int j0 = blockIdx.x * HZ_STRIP;
    const int j = j0 + t;
    const int nx = p.nx, ny = p.ny;
    const int r0 = blockIdx.y * p.rows_per_cta;
    if (r0 >= nx) return;   // whole CTA
    const int r1 = min(nx, r0 + p.rows_per_cta);
    const bool active = j < ny;
    const int last_t = min(HZ_STRIP - 1, ny - 1 - j0);
    const int jh = (j0 + HZ_STRIP < ny) ? j0 + HZ_STRIP : (p.py ? 0 : -1);   // H_z column right of the strip
    const bool halo_thread = t == last_t && jh >= 0;
    const bool halo_row = p.px || r1 < nx;
    const int i_end = halo_row ? r1 : r1 - 1;
    const float lo_y = EPS && active ? p.lo_y[j] : 0.0f, up_y = EPS && active ? p.up_y[j] : 0.0f;
    const float iyh = active ? p.iyh[j] : 0.0f;
    (void)iyh;

    float hz_prev = 0.0f, ey_prev = 0.0f, eps_prev = 0.0f, ca_y_prev = 1.0f, cb_y_prev = 0.0f;
    for (int i = r0; i <= i_end; ++i) {
        const int r = i == nx ? 0 : i;   // physical row (i == nx only on a periodic x)
        const bool own_row = i < r1;
        const int b = i & 1;
        float h_new = 0.0f, ex_c = 0.0f, ey_c = 0.0f, eps_c = 0.0f;
        if (active) {
            h_new = hz2d_hz_at(p, r, j, own_row, ex_c, ey_c);
            const size_t idx = (size_t)r * ny + j;
            if (own_row) p.hz_out[idx] = h_new;
            if (EPS) eps_c = p.eps[idx];
            s_hz[b][t] = h_new;
            if (EPS) s_eps[b][t] = eps_c;
        }
        if (halo_thread) {
            float ex_h, ey_h;
            s_hz[b][t + 1] = hz2d_hz_at(p, r, jh, false, ex_h, ey_h);
            if (EPS) s_eps[b][t + 1] = p.eps[(size_t)r * ny + jh];
        }
        __syncthreads();
        if (active) {
            const size_t idx = (size_t)r * ny + j;
            float ca_x = 1.0f, cb_x = 0.0f, ca_y = 1.0f, cb_y = 0.0f;
            if (own_row) {
                // E_x of (r, j)
                if (j < ny - 1 || p.py) {
                    const float right = s_hz[b][t + 1];
                    const float up = j < ny - 1 ? right : hz_wrap_hi(right);
                    if (EPS) {
                        cb_x = hz_cb_lossless(eps_c, s_eps[b][t + 1], lo_y, up_y, p.dt, p.eps0);
                    } else {
                        ca_x = p.ca_x ? p.ca_x[idx] : 1.0f;
                        cb_x = p.cb_x[idx];
                    }
                    p.ex_out[idx] = hz2d_ex_at(p, r, j, ex_c, ca_x, cb_x, h_new, up);
                } else {
                    p.ex_out[idx] = ex_c;   // the last face of an open y is never updated
                }
            }
            // E_y of (i - 1, j)
            if (i > r0) {
                const int re = i - 1;
                const size_t ide = (size_t)re * ny + j;
                if (re < nx - 1 || p.px) {
                    const float up = re < nx - 1 ? h_new : hz_wrap_hi(h_new);
                    if (EPS) cb_y_prev = hz_cb_lossless(eps_prev, eps_c, p.lo_x[re], p.up_x[re], p.dt, p.eps0);
                    p.ey_out[ide] = hz2d_ey_at(p, re, j, ey_prev, ca_y_prev, cb_y_prev, hz_prev, up);
                } else {
                    p.ey_out[ide] = ey_prev;
                }
            }
            if (!EPS && own_row) {
                ca_y = p.ca_y ? p.ca_y[idx] : 1.0f;
                cb_y = p.cb_y[idx];
            }
            hz_prev = h_new;
            ey_prev = ey_c;
            eps_prev = eps_c;
            ca_y_prev = ca_y;
            cb_y_prev = cb_y;
        }
    }
    if (!halo_row && active) p.ey_out[(size_t)(r1 - 1) * ny + j] = ey_prev;   // the last face of an open x
}

// ---------------------------------------------------------------------------------------------- coefficients

// ca / cb of the E_x (hi-y) and E_y (hi-x) faces from the cell eps_xx, eps_yy, sigma_e and the face shares:
// face value = self * lower + partner * upper, partner = the next cell (wrapped on a periodic axis, the cell itself on
// the last face of an open one); eps = face * eps0, k = sigma dt / (2 eps), ca = (1 - k) / (1 + k),
// cb = (dt / eps) / (1 + k) (fdtd_hz_2d_kernels.py:196-248).  sigma NULL = 0; ca_x / ca_y NULL: not written.
__global__ void hz2d_face_coefficients_kernel(const float *__restrict__ eps_xx, const float *__restrict__ eps_yy,
                                              const float *__restrict__ sigma, const float *__restrict__ lo_x,
                                              const float *__restrict__ up_x, const float *__restrict__ lo_y,
                                              const float *__restrict__ up_y, int nx, int ny, int px, int py, float dt,
                                              float eps0, float *__restrict__ ca_x, float *__restrict__ cb_x,
                                              float *__restrict__ ca_y, float *__restrict__ cb_y) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const size_t idx = (size_t)i * ny + j;
    const int pj = j < ny - 1 ? j + 1 : (py ? 0 : j);
    const int pi = i < nx - 1 ? i + 1 : (px ? 0 : i);
    const size_t idx_x = (size_t)i * ny + pj, idx_y = (size_t)pi * ny + j;
    const float s_self = sigma ? sigma[idx] : 0.0f;
    {
        const float e = eps_xx[idx] * lo_y[j] + eps_xx[idx_x] * up_y[j];
        const float s = s_self * lo_y[j] + (sigma ? sigma[idx_x] : 0.0f) * up_y[j];
        const float eps = e * eps0;
        const float k = s * dt / (2.0f * eps);
        const float denom = 1.0f + k;
        if (ca_x) ca_x[idx] = (1.0f - k) / denom;
        cb_x[idx] = (dt / eps) / denom;
    }
    {
        const float e = eps_yy[idx] * lo_x[i] + eps_yy[idx_y] * up_x[i];
        const float s = s_self * lo_x[i] + (sigma ? sigma[idx_y] : 0.0f) * up_x[i];
        const float eps = e * eps0;
        const float k = s * dt / (2.0f * eps);
        const float denom = 1.0f + k;
        if (ca_y) ca_y[idx] = (1.0f - k) / denom;
        cb_y[idx] = (dt / eps) / denom;
    }
}
