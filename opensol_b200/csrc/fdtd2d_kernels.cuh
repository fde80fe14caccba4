// Device kernels of the 2D E_z engine.  Compiled with -fmad=false: every multiply and add below is rounded on its own,
// in the order open_sol's CPU twins evaluate it, so the results are bit-identical to the reference CPU backend.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define OS_MAX_LINES_2D 16
#define EZ2D_BLOCK_X 128
#define EZ2D_BLOCK_Y 2

struct LineSrcDev {
    int32_t axis, position, lo, hi;
    const float *profile;
};

// Everything one step of the E_z engine reads, passed by value (kernel parameter space).
struct Ez2DParams {
    int32_t nx, ny, periodic_x, periodic_y, npml, cpml_mask;
    float *ez, *hx, *hy;
    const float *ca, *cb, *da, *db;   // ca NULL: 1; da/db NULL: the uniform values
    float da_uniform, db_uniform;
    const float *inv_dx_e, *inv_dx_h, *inv_dy_e, *inv_dy_h;
    const float *b_e[4], *a_e[4], *inv_e[4], *b_h[4], *a_h[4], *inv_h[4];
    float *psi_e[4], *psi_h[4];
    int32_t n_lines;
    LineSrcDev lines[OS_MAX_LINES_2D];
};

// CPML side ids in open_sol FACES order.
enum { SX_LO = 0, SX_HI = 1, SY_LO = 2, SY_HI = 3 };

// H half step of cell (i, j): fdtd_ez_2d_kernels.py:37-48 (real-only engine: the periodic wrap reads
// ez * 1 + ez * 0, as the reference's partner term with wrap cos 1, sin 0), then the H-row CPML of the y sides on H_x
// and of the x sides on H_y (boundaries.py:27-37,752-755: psi = b psi + a (ez[r+1] - ez[r]) inv; hy += db psi,
// hx += (-db) psi).
__global__ void __launch_bounds__(EZ2D_BLOCK_X *EZ2D_BLOCK_Y) ez2d_h_kernel(const Ez2DParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    const float e = p.ez[idx];
    const float da = p.da ? p.da[idx] : p.da_uniform;
    const float db = p.db ? p.db[idx] : p.db_uniform;
    const float one = 1.0f, zero = 0.0f;

    // H_x (hi-y faces)
    if (j < ny - 1 || p.periodic_y) {
        const float e_up = j < ny - 1 ? p.ez[idx + 1] : p.ez[(size_t)i * ny] * one + p.ez[(size_t)i * ny] * zero;
        float v = da * p.hx[idx] - db * (e_up - e) * p.inv_dy_h[j];
        if ((p.cpml_mask & (1 << SY_LO)) && j < npml) {
            const int k = j;
            float *psi = p.psi_h[SY_LO] + (size_t)i * npml + k;
            float q = *psi * p.b_h[SY_LO][k];
            q += p.a_h[SY_LO][k] * (p.ez[idx + 1] - e) * p.inv_h[SY_LO][k];
            *psi = q;
            v += (-db) * q;
        } else if ((p.cpml_mask & (1 << SY_HI)) && j >= ny - npml - 1 && j < ny - 1) {
            const int k = j - (ny - npml - 1);
            float *psi = p.psi_h[SY_HI] + (size_t)i * npml + k;
            float q = *psi * p.b_h[SY_HI][k];
            q += p.a_h[SY_HI][k] * (p.ez[idx + 1] - e) * p.inv_h[SY_HI][k];
            *psi = q;
            v += (-db) * q;
        }
        p.hx[idx] = v;
    }
    // H_y (hi-x faces)
    if (i < nx - 1 || p.periodic_x) {
        const float e_up = i < nx - 1 ? p.ez[idx + ny] : p.ez[j] * one + p.ez[j] * zero;
        float v = da * p.hy[idx] + db * (e_up - e) * p.inv_dx_h[i];
        if ((p.cpml_mask & (1 << SX_LO)) && i < npml) {
            const int k = i;
            float *psi = p.psi_h[SX_LO] + (size_t)k * ny + j;
            float q = *psi * p.b_h[SX_LO][k];
            q += p.a_h[SX_LO][k] * (p.ez[idx + ny] - e) * p.inv_h[SX_LO][k];
            *psi = q;
            v += db * q;
        } else if ((p.cpml_mask & (1 << SX_HI)) && i >= nx - npml - 1 && i < nx - 1) {
            const int k = i - (nx - npml - 1);
            float *psi = p.psi_h[SX_HI] + (size_t)k * ny + j;
            float q = *psi * p.b_h[SX_HI][k];
            q += p.a_h[SX_HI][k] * (p.ez[idx + ny] - e) * p.inv_h[SX_HI][k];
            *psi = q;
            v += db * q;
        }
        p.hy[idx] = v;
    }
}

// E half step of cell (i, j): fdtd_ez_2d_kernels.py:103-120, then the E-row CPML x sides (ez += cb psi) and y sides
// (ez += (-cb) psi) (boundaries.py:757-760), then the soft line sources in add order (core/sources.py:221-229: skipped
// when the step's float32 value is 0, else ez += value * profile).
// rec (optional): the new E_z of the cells of box [bi0, bi1) x [bj0, bj1) is also written to rec, row by row (the
// adjoint's recomputation records the design box this way, in the step's own launch).
__global__ void __launch_bounds__(EZ2D_BLOCK_X *EZ2D_BLOCK_Y)
    ez2d_e_kernel(const Ez2DParams p, const float *__restrict__ line_values, int64_t n_steps, int64_t k_step,
                  float *__restrict__ rec = nullptr, int bi0 = 0, int bi1 = 0, int bj0 = 0, int bj1 = 0) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    const float one = 1.0f, zero = 0.0f;
    const float hy_c = p.hy[idx], hx_c = p.hx[idx];
    float curl;
    if (i >= 1) {
        curl = (hy_c - p.hy[idx - ny]) * p.inv_dx_e[i];
    } else if (p.periodic_x) {
        const size_t w = (size_t)(nx - 1) * ny + j;
        curl = (hy_c - (p.hy[w] * one - p.hy[w] * zero)) * p.inv_dx_e[i];
    } else {
        curl = hy_c * p.inv_dx_e[i];
    }
    if (j >= 1) {
        curl -= (hx_c - p.hx[idx - 1]) * p.inv_dy_e[j];
    } else if (p.periodic_y) {
        const size_t w = idx + ny - 1;
        curl -= (hx_c - (p.hx[w] * one - p.hx[w] * zero)) * p.inv_dy_e[j];
    } else {
        curl -= hx_c * p.inv_dy_e[j];
    }
    const float cb = p.cb[idx];
    const float ez_old = p.ez[idx];
    float v = (p.ca ? p.ca[idx] * ez_old : ez_old) + cb * curl;
    if ((p.cpml_mask & (1 << SX_LO)) && i >= 1 && i <= npml) {
        const int k = i - 1;
        float *psi = p.psi_e[SX_LO] + (size_t)k * ny + j;
        float q = *psi * p.b_e[SX_LO][k];
        q += p.a_e[SX_LO][k] * (hy_c - p.hy[idx - ny]) * p.inv_e[SX_LO][k];
        *psi = q;
        v += cb * q;
    } else if ((p.cpml_mask & (1 << SX_HI)) && i >= nx - npml - 1 && i <= nx - 2) {
        const int k = i - (nx - npml - 1);
        float *psi = p.psi_e[SX_HI] + (size_t)k * ny + j;
        float q = *psi * p.b_e[SX_HI][k];
        q += p.a_e[SX_HI][k] * (hy_c - p.hy[idx - ny]) * p.inv_e[SX_HI][k];
        *psi = q;
        v += cb * q;
    }
    if ((p.cpml_mask & (1 << SY_LO)) && j >= 1 && j <= npml) {
        const int k = j - 1;
        float *psi = p.psi_e[SY_LO] + (size_t)i * npml + k;
        float q = *psi * p.b_e[SY_LO][k];
        q += p.a_e[SY_LO][k] * (hx_c - p.hx[idx - 1]) * p.inv_e[SY_LO][k];
        *psi = q;
        v += (-cb) * q;
    } else if ((p.cpml_mask & (1 << SY_HI)) && j >= ny - npml - 1 && j <= ny - 2) {
        const int k = j - (ny - npml - 1);
        float *psi = p.psi_e[SY_HI] + (size_t)i * npml + k;
        float q = *psi * p.b_e[SY_HI][k];
        q += p.a_e[SY_HI][k] * (hx_c - p.hx[idx - 1]) * p.inv_e[SY_HI][k];
        *psi = q;
        v += (-cb) * q;
    }
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &s = p.lines[l];
        const int along = s.axis == 0 ? i : j, across = s.axis == 0 ? j : i;
        if (across == s.position && along >= s.lo && along < s.hi) {
            const float value = line_values[(size_t)l * n_steps + k_step];
            if (value != 0.0f) v += value * s.profile[along - s.lo];
        }
    }
    p.ez[idx] = v;
    if (rec && i >= bi0 && i < bi1 && j >= bj0 && j < bj1) rec[(size_t)(i - bi0) * (bj1 - bj0) + (j - bj0)] = v;
}

// Line DFT of a flux monitor at one sample (physics/em/monitors.py:45-46,84-90): acc[f, c] += complex128(phase_f) *
// (double)field, for E_z and the tangential H, one thread per (frequency, cell).  The products of a float phase and a
// float sample are exact in double, so the float64 running sums equal the reference's complex128 ones.
__global__ void ez2d_flux_kernel(const float *__restrict__ ez, const float *__restrict__ h_field, int ny,
                                 int normal_axis, int position, int lo, int n, int nf, const float *__restrict__ phases,
                                 double *__restrict__ e_acc, double *__restrict__ h_acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nf) return;
    const int f = t / n, c = t - f * n;
    const size_t cell = normal_axis == 0 ? (size_t)position * ny + (size_t)(lo + c) : (size_t)(lo + c) * ny + position;
    const double pr = (double)phases[2 * f], pi = (double)phases[2 * f + 1];
    const double e = (double)ez[cell], hv = (double)h_field[cell];
    const size_t a = ((size_t)f * n + c) * 2;
    e_acc[a] += pr * e;
    e_acc[a + 1] += pi * e;
    h_acc[a] += pr * hv;
    h_acc[a + 1] += pi * hv;
}

// Field-map DFT of E_z at one sample (DFTMonitor.update with _dft_accum_host, physics/em/monitors.py:36-37,281-311):
// acc[f, a, b] += phase_f * E_z[x0 + a ds, y0 + b ds] in complex64 arithmetic: the float sample taken as a complex
// number with imaginary part 0, the product's parts pr v - pi 0 and pr 0 + pi v, then the sum, each rounded to float.
// One thread per (frequency, sample).
__global__ void ez2d_dft_map_kernel(const float *__restrict__ ez, int ny, int x0, int y0, int ds, int mx, int my,
                                    int nf, const float *__restrict__ phases, float *__restrict__ acc) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per_f = (int64_t)mx * my;
    if (t >= per_f * nf) return;
    const int f = (int)(t / per_f);
    const int64_t c = t - (int64_t)f * per_f;
    const int a = (int)(c / my), b = (int)(c - (int64_t)a * my);
    const float v = ez[(size_t)(x0 + a * ds) * ny + (size_t)(y0 + b * ds)];
    const float pr = phases[2 * f], pi = phases[2 * f + 1], zero = 0.0f;
    const float re = pr * v - pi * zero, im = pr * zero + pi * v;
    acc[2 * t] = acc[2 * t] + re;
    acc[2 * t + 1] = acc[2 * t + 1] + im;
}

// Field-map DFT of the H_z engine at one sample (DFTMonitor.update for 'hz', physics/em/monitors.py:296-322, with
// _dft_accum_host and _dft_accum_pair_host :36-41): H_z at the cell with the phases of t - dt/2; E_x collocated to
// the cell centre as float(0.5) (E_x[x, y] + E_x[x, y - 1]) and E_y as float(0.5) (E_y[x, y] + E_y[x - 1, y]) with
// the E phases, the lo partner of row / column 0 the wrapped last face on a periodic axis, else the face itself
// (_centre_pairs, :156-167).  acc: (3, nf, mx, my) complex64 (H_z, E_x, E_y).  One thread per (frequency, sample).
__global__ void hz2d_dft_map_kernel(const float *__restrict__ hz, const float *__restrict__ ex,
                                    const float *__restrict__ ey, int nx, int ny, int px, int py, int x0, int y0,
                                    int ds, int mx, int my, int nf, const float *__restrict__ ph_e,
                                    const float *__restrict__ ph_h, float *__restrict__ acc) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per_f = (int64_t)mx * my, total = per_f * nf;
    if (t >= total) return;
    const int f = (int)(t / per_f);
    const int64_t c = t - (int64_t)f * per_f;
    const int a = (int)(c / my), b = (int)(c - (int64_t)a * my);
    const int x = x0 + a * ds, y = y0 + b * ds;
    const int y_lo = y >= 1 ? y - 1 : (py ? ny - 1 : 0), x_lo = x >= 1 ? x - 1 : (px ? nx - 1 : 0);
    const float half = 0.5f, zero = 0.0f;
    const float v[3] = {hz[(size_t)x * ny + y], half * (ex[(size_t)x * ny + y] + ex[(size_t)x * ny + y_lo]),
                        half * (ey[(size_t)x * ny + y] + ey[(size_t)x_lo * ny + y])};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float *ph = q == 0 ? ph_h : ph_e;
        const float pr = ph[2 * f], pi = ph[2 * f + 1];
        const float re = pr * v[q] - pi * zero, im = pr * zero + pi * v[q];
        const int64_t o = 2 * ((int64_t)q * total + t);
        acc[o] = acc[o] + re;
        acc[o + 1] = acc[o + 1] + im;
    }
}

// Soft line sources on E_z after the E update, as the E kernel's own loop adds them: for the per-step path of an
// engine whose pole corrections must come between the E update and the sources (fdtd_ez_2d.py:90-99).
__global__ void ez2d_line_inject_kernel(const Ez2DParams p, const float *__restrict__ line_values, int64_t n_steps,
                                        int64_t k_step) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const size_t idx = (size_t)i * p.ny + j;
    float v = p.ez[idx];
    bool hit = false;
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &s = p.lines[l];
        const int along = s.axis == 0 ? i : j, across = s.axis == 0 ? j : i;
        if (across == s.position && along >= s.lo && along < s.hi) {
            const float value = line_values[(size_t)l * n_steps + k_step];
            if (value != 0.0f) {
                v += value * s.profile[along - s.lo];
                hit = true;
            }
        }
    }
    if (hit) p.ez[idx] = v;
}

// ---- dispersive poles on a cell box [i0, i1) x [j0, j1) (fdtd_ez_2d_kernels.py:190-260, fdtd_ez_2d.py:318-358);
// box arrays (i1 - i0, j1 - j0), grid arrays (nx, ny).  drive = the pole's drive coefficient times the cell mask, so
// cells outside the material keep J = 0 / P = 0.
// Drude J^{n+1/2} = J + (damping J + drive E^n), then jz_total = J (store: one pole) or jz_total += J.
__global__ void ez2d_drude_j_kernel(const float *__restrict__ ez, int ny, int i0, int i1, int j0, int j1,
                                    float damping, const float *__restrict__ drive, float *__restrict__ jz,
                                    float *__restrict__ jz_total, int store) {
    const int w = j1 - j0;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)(i1 - i0) * w) return;
    const int i = i0 + (int)(t / w), j = j0 + (int)(t % w);
    const size_t g = (size_t)i * ny + j;
    const float jn = jz[t] + (damping * jz[t] + drive[t] * ez[g]);
    jz[t] = jn;
    if (jz_total) jz_total[g] = store ? jn : jz_total[g] + jn;   // NULL: per-pole corrections (H_z face sets)
}

// Lorentz in velocity form: dP += damping dP - restoring P^n + drive E^n, then P += dP.
__global__ void ez2d_lorentz_p_kernel(const float *__restrict__ ez, int ny, int i0, int i1, int j0, int j1,
                                      float damping, float restoring, const float *__restrict__ drive,
                                      float *__restrict__ pz, float *__restrict__ dpz) {
    const int w = j1 - j0;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)(i1 - i0) * w) return;
    const size_t g = (size_t)(i0 + (int)(t / w)) * ny + (j0 + (int)(t % w));
    const float dp = dpz[t] + (damping * dpz[t] - restoring * pz[t] + drive[t] * ez[g]);
    dpz[t] = dp;
    pz[t] = pz[t] + dp;
}

// E corrections after the E update: Drude E -= cb jz_total on the union box (dp NULL), Lorentz E -= (cb inv_dt) dP
// on the pole's box (dp = its box array).
__global__ void ez2d_pole_correct_kernel(float *__restrict__ ez, int ny, int i0, int i1, int j0, int j1,
                                         const float *__restrict__ cb, const float *__restrict__ jz_total,
                                         const float *__restrict__ dp, float inv_dt) {
    const int w = j1 - j0;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)(i1 - i0) * w) return;
    const size_t g = (size_t)(i0 + (int)(t / w)) * ny + (j0 + (int)(t % w));
    if (dp) ez[g] = ez[g] - cb[g] * inv_dt * dp[t];
    else ez[g] = ez[g] - cb[g] * jz_total[g];
}

// ---- +x plane-wave TFSF box (TFSFSource, physics/em/sources.py:35-52,72-186,334-350)
// Scattered / total-field H corrections after the H update: H_y on rows x0 - 1 (-) and x1 - 1 (+) from the incident
// E_z at the box's first / last column, H_x on columns y0 - 1 (+) and y1 - 1 (-) from the incident E_z of each row.
__global__ void ez2d_tfsf_h_kernel(float *__restrict__ hx, float *__restrict__ hy, const float *__restrict__ aux_ez,
                                   int x0, int x1, int y0, int y1, int aux_x0, int ny, float c_xlo, float c_xhi,
                                   float c_ylo, float c_yhi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < y1 - y0) {
        const int j = y0 + k;
        hy[(size_t)(x0 - 1) * ny + j] = hy[(size_t)(x0 - 1) * ny + j] - c_xlo * aux_ez[aux_x0];
        hy[(size_t)(x1 - 1) * ny + j] = hy[(size_t)(x1 - 1) * ny + j] + c_xhi * aux_ez[aux_x0 + (x1 - 1 - x0)];
    }
    if (k < x1 - x0) {
        const size_t row = (size_t)(x0 + k) * ny;
        const float incident = aux_ez[aux_x0 + k];
        hx[row + (y0 - 1)] = hx[row + (y0 - 1)] + c_ylo * incident;
        hx[row + (y1 - 1)] = hx[row + (y1 - 1)] - c_yhi * incident;
    }
}

// The incident line's H update: aux_hy[a] += coef[a] (aux_ez[a + 1] - aux_ez[a]), a < n - 1.
__global__ void ez2d_tfsf_aux_h_kernel(const float *__restrict__ aux_ez, const float *__restrict__ coef,
                                       float *__restrict__ aux_hy, int n) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < n - 1) aux_hy[a] = aux_hy[a] + coef[a] * (aux_ez[a + 1] - aux_ez[a]);
}

// Total-field E_z corrections after the E update: rows x0 (-) and x1 - 1 (+) from the incident H_y.
__global__ void ez2d_tfsf_e_kernel(float *__restrict__ ez, const float *__restrict__ aux_hy, int x0, int x1, int y0,
                                   int y1, int aux_x0, int ny, float c_xlo, float c_xhi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= y1 - y0) return;
    const int j = y0 + k;
    ez[(size_t)x0 * ny + j] = ez[(size_t)x0 * ny + j] - c_xlo * aux_hy[aux_x0 - 1];
    ez[(size_t)(x1 - 1) * ny + j] = ez[(size_t)(x1 - 1) * ny + j] + c_xhi * aux_hy[aux_x0 + (x1 - 1 - x0)];
}

// The incident line's E update (one block): aux_ez[a] += ce[a] (aux_hy[a] - aux_hy[a - 1]) for 0 < a < n - 1, the soft
// source value at aux cell `src`, then the Mur ends from the ends' values before the update.
__global__ void ez2d_tfsf_aux_e_kernel(float *__restrict__ aux_ez, const float *__restrict__ aux_hy, int n,
                                       const float *__restrict__ ce, int src, const float *__restrict__ value,
                                       float mur_lo, float mur_hi) {
    __shared__ float edge_old[4];
    if (threadIdx.x == 0) {
        edge_old[0] = aux_ez[0], edge_old[1] = aux_ez[1], edge_old[2] = aux_ez[n - 2], edge_old[3] = aux_ez[n - 1];
    }
    __syncthreads();
    for (int a = 1 + threadIdx.x; a < n - 1; a += blockDim.x) aux_ez[a] = aux_ez[a] + ce[a] * (aux_hy[a] - aux_hy[a - 1]);
    __syncthreads();
    if (threadIdx.x == 0) {
        aux_ez[src] = aux_ez[src] + *value;
        aux_ez[0] = edge_old[1] + mur_lo * (aux_ez[1] - edge_old[0]);
        aux_ez[n - 1] = edge_old[2] + mur_hi * (aux_ez[n - 2] - edge_old[3]);
    }
}

// H_z box (TFSFSourceHz, physics/em/sources.py:55-70,108-172,352-379): total-field H_z corrections after the H_z
// update on rows x0 (+, from the incident E_y below the box) and x1 - 1 (-); scattered-field E corrections after the
// E update: E_y on rows x0 - 1 (+) and x1 - 1 (-) from the incident H_z, E_x on columns y0 - 1 (-) and y1 - 1 (+).
__global__ void hz2d_tfsf_h_kernel(float *__restrict__ hz, const float *__restrict__ aux_ey, int x0, int x1, int y0,
                                   int y1, int aux_x0, int ny, float c_xlo, float c_xhi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= y1 - y0) return;
    const int j = y0 + k;
    hz[(size_t)x0 * ny + j] = hz[(size_t)x0 * ny + j] + c_xlo * aux_ey[aux_x0 - 1];
    hz[(size_t)(x1 - 1) * ny + j] = hz[(size_t)(x1 - 1) * ny + j] - c_xhi * aux_ey[aux_x0 + (x1 - 1 - x0)];
}

__global__ void hz2d_tfsf_e_kernel(float *__restrict__ ex, float *__restrict__ ey, const float *__restrict__ aux_hz,
                                   int x0, int x1, int y0, int y1, int aux_x0, int ny, float c_xlo, float c_xhi,
                                   float c_ylo, float c_yhi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < y1 - y0) {
        const int j = y0 + k;
        ey[(size_t)(x0 - 1) * ny + j] = ey[(size_t)(x0 - 1) * ny + j] + c_xlo * aux_hz[aux_x0];
        ey[(size_t)(x1 - 1) * ny + j] = ey[(size_t)(x1 - 1) * ny + j] - c_xhi * aux_hz[aux_x0 + (x1 - 1 - x0)];
    }
    if (k < x1 - x0) {
        const size_t row = (size_t)(x0 + k) * ny;
        const float incident = aux_hz[aux_x0 + k];
        ex[row + (y0 - 1)] = ex[row + (y0 - 1)] - c_ylo * incident;
        ex[row + (y1 - 1)] = ex[row + (y1 - 1)] + c_yhi * incident;
    }
}

// ca / cb from float32 eps_r, sigma_e (fdtd_ez_2d_kernels.py:314-332, T = float); sigma NULL = lossless (ca not
// written: it is 1).
__global__ void ez2d_e_coefficients_kernel(const float *__restrict__ eps_r, const float *__restrict__ sigma, float dt,
                                           float eps0, size_t n, float *__restrict__ ca, float *__restrict__ cb) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float eps = eps_r[t] * eps0;
    const float s = sigma ? sigma[t] : 0.0f;
    const float k = s * dt / (2.0f * eps);
    const float denom = 1.0f + k;
    if (ca) ca[t] = (1.0f - k) / denom;
    cb[t] = (dt / eps) / denom;
}

// da / db from float32 mu_r, sigma_m (fdtd_ez_2d_kernels.py:335-353); NULL arrays read 1 / 0.
__global__ void ez2d_h_coefficients_kernel(const float *__restrict__ mu_r, const float *__restrict__ sigma_m, float dt,
                                           float mu0, size_t n, float *__restrict__ da, float *__restrict__ db) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float mu = (mu_r ? mu_r[t] : 1.0f) * mu0;
    const float s = sigma_m ? sigma_m[t] : 0.0f;
    const float k = s * dt / (2.0f * mu);
    const float denom = 1.0f + k;
    da[t] = (1.0f - k) / denom;
    db[t] = (dt / mu) / denom;
}
