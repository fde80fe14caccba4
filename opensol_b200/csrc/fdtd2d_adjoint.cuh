// Discrete adjoint of the 2D E_z time step for sm_100a (no open_sol counterpart: open_sol has no FDTD adjoint).
//
// The forward step is linear in the state (E_z, H_x, H_y, the CPML psi of every side): H half step (Yee, then the
// H-row CPML: psi = b psi + a (E[r+1] - E[r]) inv, H += sign db psi), E half step (Yee, then the E-row CPML:
// psi = b psi + a (H[r] - H[r-1]) inv, E += sign cb psi), line injection, DFT sample; sign = +1 on the x sides (on
// H_y / E_z through H_y) and -1 on the y sides.  Its exact transpose, run backward in time, propagates the adjoint
// lambda of the state; these kernels evaluate it in gather form, one thread per cell, reading input buffers and
// writing output buffers so no thread reads a value another one has already rewritten:
//   ez2d_adj_e_kernel: transpose of the E half step: lambda_H += curl^T (cb lambda_E) + the psi paths, new psi
//                      adjoints, and the gradient term lambda_E (E^{n+1} - E^n) on the design box;
//   ez2d_adj_h_kernel: transpose of the H half step: lambda_E = ca lambda_E + curl^T (db lambda_H) + psi paths,
//                      lambda_H = da lambda_H on the updated faces.
// The edge rules follow the forward: no lo neighbour below row 0 of an open axis, the last H face of an open axis
// never updated, wrapped neighbours on a periodic axis.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct Ez2DAdjParams {
    int32_t nx, ny, px, py, npml, cpml_mask;
    const float *ca, *cb, *da, *db;   // ca NULL: 1; da/db NULL: the uniform values
    float da_u, db_u;
    const float *ixe, *ixh, *iye, *iyh;
    const float *b_e[4], *a_e[4], *inv_e[4], *b_h[4], *a_h[4], *inv_h[4];
    const float *le_in;
    float *le_out;
    const float *lhx_in, *lhy_in;
    float *lhx_out, *lhy_out;
    const float *lpe_in[4], *lph_in[4];
    float *lpe_out[4], *lph_out[4];
    int32_t bi0, bi1, bj0, bj1;       // design box [bi0, bi1) x [bj0, bj1)
    const float *e_next, *e_prev;     // E over the box after / before this step (box layout)
    double *grad;                     // box accumulator of lambda_E (E^{n+1} - E^n)
};

enum { ADJ_XLO = 0, ADJ_XHI = 1, ADJ_YLO = 2, ADJ_YHI = 3 };

// psi row of grid row r on side s for the E rows (lo: 1..npml, hi: n-npml-1..n-2), -1 outside.
__device__ __forceinline__ int adj_e_row(int s, int r, int n, int npml) {
    const int k = (s == ADJ_XLO || s == ADJ_YLO) ? r - 1 : r - (n - npml - 1);
    return (k >= 0 && k < npml) ? k : -1;
}

// psi row of grid row r on side s for the H rows (lo: 0..npml-1, hi: n-npml-1..n-2), -1 outside.
__device__ __forceinline__ int adj_h_row(int s, int r, int n, int npml) {
    const int k = (s == ADJ_XLO || s == ADJ_YLO) ? r : r - (n - npml - 1);
    return (k >= 0 && k < npml) ? k : -1;
}

// cb * lambda_E of cell (i, j)
__device__ __forceinline__ float adj_u(const Ez2DAdjParams &p, int i, int j) {
    const size_t c = (size_t)i * p.ny + j;
    return p.cb[c] * p.le_in[c];
}

// w = lambda_psi + sign cb lambda_E of the E-row psi of side s at cell (i, j) with slab row k
__device__ __forceinline__ float adj_we(const Ez2DAdjParams &p, int s, int k, int i, int j) {
    const bool xs = s < 2;
    const size_t q = xs ? (size_t)k * p.ny + j : (size_t)i * p.npml + k;
    return p.lpe_in[s][q] + (xs ? 1.0f : -1.0f) * adj_u(p, i, j);
}

__global__ void __launch_bounds__(256) ez2d_adj_e_kernel(const Ez2DAdjParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    const float u = adj_u(p, i, j);
    // lambda_H_y(i, j): E(i, j) reads H_y(i) with +ixe[i]; E(i + 1, j) reads it with -ixe[i + 1]
    float hy = p.lhy_in[idx] + u * p.ixe[i];
    if (i + 1 < nx) hy -= adj_u(p, i + 1, j) * p.ixe[i + 1];
    else if (p.px) hy -= adj_u(p, 0, j) * p.ixe[0];
    // lambda_H_x(i, j): E(i, j) reads H_x(j) with -iye[j]; E(i, j + 1) reads it with +iye[j + 1]
    float hx = p.lhx_in[idx] - u * p.iye[j];
    if (j + 1 < ny) hx += adj_u(p, i, j + 1) * p.iye[j + 1];
    else if (p.py) hx += adj_u(p, i, 0) * p.iye[0];
    for (int s = 0; s < 4; ++s) {
        if (!(p.cpml_mask & (1 << s))) continue;
        const bool xs = s < 2;
        const int r = xs ? i : j, n = xs ? nx : ny;
        const float *a = p.a_e[s], *inv = p.inv_e[s];
        int k = adj_e_row(s, r, n, npml);
        if (k >= 0) {   // this cell's own E-row psi: source H[r] (+), own new lambda_psi
            const float w = adj_we(p, s, k, i, j);
            const size_t q = xs ? (size_t)k * ny + j : (size_t)i * npml + k;
            p.lpe_out[s][q] = p.b_e[s][k] * w;
            if (xs) hy += a[k] * inv[k] * w;
            else hx += a[k] * inv[k] * w;
        }
        k = adj_e_row(s, r + 1, n, npml);
        if (k >= 0) {   // the next row's psi reads H[r] as its lo sample (-)
            const float w = xs ? adj_we(p, s, k, i + 1, j) : adj_we(p, s, k, i, j + 1);
            if (xs) hy -= a[k] * inv[k] * w;
            else hx -= a[k] * inv[k] * w;
        }
    }
    p.lhx_out[idx] = hx;
    p.lhy_out[idx] = hy;
    if (i >= p.bi0 && i < p.bi1 && j >= p.bj0 && j < p.bj1) {
        const size_t b = (size_t)(i - p.bi0) * (p.bj1 - p.bj0) + (j - p.bj0);
        p.grad[b] += (double)p.le_in[idx] * ((double)p.e_next[b] - (double)p.e_prev[b]);
    }
}

// db of cell c
__device__ __forceinline__ float adj_db(const Ez2DAdjParams &p, size_t c) { return p.db ? p.db[c] : p.db_u; }

// w = lambda_psi + sign db lambda_H of the H-row psi of side s at cell (i, j) with slab row k (lambda_H: the input
// of this kernel, i.e. the adjoint of H after its half step)
__device__ __forceinline__ float adj_wh(const Ez2DAdjParams &p, int s, int k, int i, int j) {
    const bool xs = s < 2;
    const size_t c = (size_t)i * p.ny + j;
    const size_t q = xs ? (size_t)k * p.ny + j : (size_t)i * p.npml + k;
    return xs ? p.lph_in[s][q] + 1.0f * adj_db(p, c) * p.lhy_in[c]
              : p.lph_in[s][q] + (-1.0f) * adj_db(p, c) * p.lhx_in[c];
}

__global__ void __launch_bounds__(256) ez2d_adj_h_kernel(const Ez2DAdjParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const int nx = p.nx, ny = p.ny, npml = p.npml;
    const size_t idx = (size_t)i * ny + j;
    float e = p.ca ? p.ca[idx] * p.le_in[idx] : p.le_in[idx];
    // H_x(i, j) = da H_x - db (E(j + 1) - E(j)) iyh[j]: E(j) gets +db iyh lambda
    const bool hx_updated = j < ny - 1 || p.py;
    if (hx_updated) e += adj_db(p, idx) * p.iyh[j] * p.lhx_in[idx];
    if (j >= 1) {
        const size_t c = idx - 1;
        e -= adj_db(p, c) * p.iyh[j - 1] * p.lhx_in[c];
    } else if (p.py) {
        const size_t c = idx + ny - 1;
        e -= adj_db(p, c) * p.iyh[ny - 1] * p.lhx_in[c];
    }
    // H_y(i, j) = da H_y + db (E(i + 1) - E(i)) ixh[i]: E(i) gets -db ixh lambda
    const bool hy_updated = i < nx - 1 || p.px;
    if (hy_updated) e -= adj_db(p, idx) * p.ixh[i] * p.lhy_in[idx];
    if (i >= 1) {
        const size_t c = idx - ny;
        e += adj_db(p, c) * p.ixh[i - 1] * p.lhy_in[c];
    } else if (p.px) {
        const size_t c = (size_t)(nx - 1) * ny + j;
        e += adj_db(p, c) * p.ixh[nx - 1] * p.lhy_in[c];
    }
    for (int s = 0; s < 4; ++s) {
        if (!(p.cpml_mask & (1 << s))) continue;
        const bool xs = s < 2;
        const int r = xs ? i : j, n = xs ? nx : ny;
        const float *a = p.a_h[s], *inv = p.inv_h[s];
        int k = adj_h_row(s, r, n, npml);
        if (k >= 0) {   // this cell's own H-row psi reads E[r] as its lo sample (-)
            const float w = adj_wh(p, s, k, i, j);
            const size_t q = xs ? (size_t)k * ny + j : (size_t)i * npml + k;
            p.lph_out[s][q] = p.b_h[s][k] * w;
            e -= a[k] * inv[k] * w;
        }
        k = adj_h_row(s, r - 1, n, npml);
        if (k >= 0) {   // the previous row's psi reads E[r] as its hi sample (+)
            const float w = xs ? adj_wh(p, s, k, i - 1, j) : adj_wh(p, s, k, i, j - 1);
            e += a[k] * inv[k] * w;
        }
    }
    p.le_out[idx] = e;
    const float da = p.da ? p.da[idx] : p.da_u;
    p.lhx_out[idx] = hx_updated ? da * p.lhx_in[idx] : p.lhx_in[idx];
    p.lhy_out[idx] = hy_updated ? da * p.lhy_in[idx] : p.lhy_in[idx];
}

// dJ/de and dJ/dh of the DFT sample of step k (row row_of_step[k] of de / dh, none when -1) added to lambda_E and
// lambda_H on a flux line (normal 0: x-cell `position`, H_y; normal 1: y-cell `position`, H_x).
__global__ void ez2d_adj_source_kernel(float *le, float *lh, int ny, int normal_axis, int position, int lo, int n,
                                       const int32_t *__restrict__ row_of_step, int k, const float *__restrict__ de_rows,
                                       const float *__restrict__ dh_rows) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int row = row_of_step[k];
    if (row < 0) return;
    const float *de = de_rows + (size_t)row * n, *dh = dh_rows + (size_t)row * n;
    const size_t cell = normal_axis == 0 ? (size_t)position * ny + (lo + c) : (size_t)(lo + c) * ny + position;
    le[cell] += de[c];
    lh[cell] += dh[c];
}

// E over the design box into a box-layout buffer.
__global__ void ez2d_record_box_kernel(const float *__restrict__ ez, int ny, int bi0, int bi1, int bj0, int bj1,
                                       float *__restrict__ out) {
    const int w = bj1 - bj0;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (bi1 - bi0) * w) return;
    const int i = bi0 + t / w, j = bj0 + t % w;
    out[t] = ez[(size_t)i * ny + j];
}
