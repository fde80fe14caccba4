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
//   hz2d_interior_kernel + hz2d_border_kernel (variant 1): per Yee step, both read one field / psi buffer set and
//        write the other.  The interior kernel covers the box where every update is the plain Yee one (no CPML row,
//        edge or wrap in reach): each warp streams a strip of 128 columns down its rows, 4 columns per lane, H_z of a
//        row then E_x of the row and E_y of the row below from registers and warp shuffles, so each field is read
//        and written once per step; in the lossless form (eps_xx = eps_yy, no sigma, vacuum permeability) the rows
//        arrive by TMA bulk copies into a per-warp ring and the face cb = dt / (face eps eps0) is evaluated from one
//        eps_r word per cell, exactly as the coefficient kernel evaluates it (denominator 1 + 0 = 1).  The border
//        kernel updates the frame around the box one thread per cell with the per-cell functions, evaluating the
//        two neighbouring new H_z its E_x / E_y read again from the old E.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd2d_kernels.cuh"
#include "fdtd2d_tb.cuh"

#define HZ_THREADS 128   // threads per CTA of the fused step; 4 columns each

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
    int32_t ia, ib, jc0, jc1;                 // interior box of the fused step: rows [ia, ib), columns [jc0, jc1)
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

// Sheet sources after the E update and the pole corrections (TangentialSheetCurrentSource.inject_electric at
// t + dt/2): E_x faces (i, position) for axis 0, E_y faces (position, j) for axis 1, each line in add order, a 0 value
// skipped; the same additions hz2d_ex_at / hz2d_ey_at make inside the E update.
__global__ void __launch_bounds__(EZ2D_BLOCK_X *EZ2D_BLOCK_Y) hz2d_line_inject_kernel(const Hz2DParams p) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= p.nx || j >= p.ny) return;
    const size_t idx = (size_t)i * p.ny + j;
    for (int axis = 0; axis < 2; ++axis) {
        float *e = axis == 0 ? p.ex_out : p.ey_out;
        float v = 0.0f;
        bool hit = false;
        for (int l = 0; l < p.n_lines; ++l) {
            const LineSrcDev &L = p.lines[l];
            if (L.axis != axis) continue;
            const int along = axis == 0 ? i : j, across = axis == 0 ? j : i;
            if (across != L.position || along < L.lo || along >= L.hi) continue;
            const float value = p.line_values[(size_t)l * p.values_stride + p.k_step];
            if (value == 0.0f) continue;
            if (!hit) v = e[idx], hit = true;
            v += value * L.profile[along - L.lo];
        }
        if (hit) e[idx] = v;
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

// four consecutive floats of a row (16-byte aligned when VEC)
template <bool VEC>
__device__ __forceinline__ void hz_ld4(const float *base, size_t idx, float (&v)[4]) {
    if (VEC) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(base + idx));
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = __ldg(base + idx + c);
    }
}

template <bool VEC>
__device__ __forceinline__ void hz_st4(float *base, size_t idx, const float (&v)[4]) {
    if (VEC) {
        *reinterpret_cast<float4 *>(base + idx) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) base[idx + c] = v[c];
    }
}

// ---- the fused step: an interior kernel and a border kernel per Yee step, both reading one field / psi buffer set
// and writing the other, over disjoint cells.
//
// The interior box (rows [ia, ib), columns [jc0, jc1), chosen by the host) holds the cells whose H_z, E_x and E_y
// updates, and those of the H_z one row below and one column right of the box, touch no CPML row, grid edge or wrap:
// there every cell takes the same plain expressions.  The border kernel covers the rest of the grid with the per-cell
// functions above.

// H_z of four plain cells from their old values (ex_left: E_x of the column left of the first).
__device__ __forceinline__ void hz_plain_h(const float (&hzo)[4], const float (&exo)[4], const float (&eyo)[4],
                                           const float (&eyp)[4], float ex_left, const float (&iye)[4], float ixe,
                                           const float (&da)[4], const float (&db)[4], float (&hn)[4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float dex = exo[c] - (c == 0 ? ex_left : exo[c - 1]);
        const float dey = eyo[c] - eyp[c];
        float curl = dex * iye[c];
        curl -= dey * ixe;
        hn[c] = da[c] * hzo[c] + db[c] * curl;
    }
}

// E_x of four plain faces and E_y of the four faces of the row below (lossless form: cb from eps; else coefficient
// arrays), then the sheet sources crossing them (added after E in add order, skipped for a 0 value).
template <bool EPS>
__device__ __forceinline__ void hz_plain_e(const Hz2DParams &p, float (&vx)[4], float (&vy)[4], int r, int re, int jt,
                                           bool do_x, bool do_y, const float (&hn)[4], const float (&exo)[4],
                                           const float (&ep)[4], float h_next, float e_next, const float (&lo_y)[4],
                                           const float (&up_y)[4], const float (&iyh)[4], const float (&hzp)[4],
                                           const float (&eyp)[4], const float (&epp)[4], const float (&cax)[4],
                                           const float (&cbx)[4], const float (&cay)[4], const float (&cby)[4]) {
    const float ixh = do_y ? __ldg(p.ixh + re) : 0.0f;
    const float lo_x = EPS && do_y ? __ldg(p.lo_x + re) : 0.0f, up_x = EPS && do_y ? __ldg(p.up_x + re) : 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float bx = EPS ? hz_cb_lossless(ep[c], c < 3 ? ep[c + 1] : e_next, lo_y[c], up_y[c], p.dt, p.eps0)
                             : cbx[c];
        const float dx = (c < 3 ? hn[c + 1] : h_next) - hn[c];
        vx[c] = (EPS ? 1.0f : cax[c]) * exo[c] + bx * dx * iyh[c];
        const float by = EPS ? hz_cb_lossless(epp[c], ep[c], lo_x, up_x, p.dt, p.eps0) : cby[c];
        const float dy = hn[c] - hzp[c];
        vy[c] = (EPS ? 1.0f : cay[c]) * eyp[c] - by * dy * ixh;
    }
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &L = p.lines[l];
        if (L.axis == 0) {   // E_x faces (i, position), i in [lo, hi)
            if (do_x && L.position >= jt && L.position < jt + 4 && r >= L.lo && r < L.hi) {
                const float value = p.line_values[(size_t)l * p.values_stride + p.k_step];
                if (value != 0.0f) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (jt + c == L.position) vx[c] += value * L.profile[r - L.lo];
                }
            }
        } else if (do_y && L.position == re && jt + 3 >= L.lo && jt < L.hi) {   // E_y faces (position, j)
            const float value = p.line_values[(size_t)l * p.values_stride + p.k_step];
            if (value != 0.0f) {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (jt + c >= L.lo && jt + c < L.hi) vy[c] += value * L.profile[jt + c - L.lo];
            }
        }
    }
}

// Row staging of the interior kernel (lossless form): lane 0 of each warp copies row windows of H_z, E_x, E_y and
// eps_r (the strip's 128 columns plus 4 on each side, clipped to the grid) into a per-warp ring of HZ_SLOTS slots by
// 1D bulk copies (cp.async.bulk, no multicast), HZ_AHEAD rows ahead of the row being consumed, each slot completing
// on its own mbarrier.  The lanes read their old values, the E_x left of their first column and (the strip's last
// lane) the halo column from shared memory.  A slot is refilled after the warp has read it (__syncwarp, then lane 0
// orders the reads before the copy engine's writes with fence.proxy.async).  Waits are bounded (tb_mbar_wait): one
// that runs out sets the engine's error flag, waits (bounded) for the copies still in flight and ends the warp.
#define HZ_AHEAD 3
#define HZ_SLOTS (HZ_AHEAD + 1)
#define HZ_WIN 136   // floats of one staged row window: 4 + 128 + 4 columns
__host__ __device__ constexpr int hz_warp_smem_bytes() { return HZ_SLOTS * 4 * HZ_WIN * 4 + HZ_SLOTS * 8; }

struct HzStage {
    float *ring;          // [slot][array: hz, ex, ey, eps][HZ_WIN]
    uint64_t *bar;        // [slot]
    int jw, c_lo, c_hi;   // window columns [c_lo, c_hi) of the grid at slot offset c_lo - (jw - 4)

    __device__ __forceinline__ float *slot(int s, int a) const { return ring + (s * 4 + a) * HZ_WIN; }

    // lane 0: copy row r into slot s
    __device__ __forceinline__ void issue(const Hz2DParams &p, int r, int s) const {
        const uint32_t bytes = (uint32_t)(c_hi - c_lo) * 4u;
        tb_mbar_expect_tx(bar + s, 4u * bytes);
        const size_t src = (size_t)r * p.ny + c_lo;
        const int off = c_lo - (jw - 4);
        tb_bulk_g2s(slot(s, 0) + off, p.hz_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 1) + off, p.ex_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 2) + off, p.ey_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 3) + off, p.eps + src, bytes, bar + s);
    }
};

// Interior kernel.  Each warp owns a strip of up to 128 columns of the box (lane l: columns jt .. jt + 3,
// jt = jw + 4 l) and walks the CTA's rows r0 .. r1 - 1 plus the halo row r1, with no barrier: row i gives H_z of
// row i from the old E (the strip's last lane also the halo column right of the strip), the next lane's first H_z /
// eps by warp shuffle, then E_x of row i and E_y of row i - 1.  STAGED (lossless form): rows through the TMA ring;
// otherwise 16-byte (VEC) or scalar loads from global memory.
template <bool EPS, bool VEC, bool STAGED>
__global__ void __launch_bounds__(HZ_THREADS, 6) hz2d_interior_kernel(const Hz2DParams p, int32_t *err) {
    extern __shared__ __align__(16) unsigned char hz_smem[];
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int jw = p.jc0 + (blockIdx.x * (HZ_THREADS / 32) + warp) * 128;
    if (jw >= p.jc1) return;   // whole warp (its barriers are never used)
    const int jt = jw + 4 * lane;
    const int ny = p.ny;
    const int r0 = p.ia + blockIdx.y * p.rows_per_cta;
    if (r0 >= p.ib) return;
    const int r1 = min(p.ib, r0 + p.rows_per_cta);
    const int j_end = min(jw + 128, p.jc1);             // the strip's columns [jw, j_end); halo column j_end
    const bool active = jt < j_end;
    const int last_lane = (j_end - 1 - jw) / 4;
    const bool halo_lane = lane == last_lane;

    HzStage st;
    if constexpr (STAGED) {
        unsigned char *mine = hz_smem + warp * hz_warp_smem_bytes();
        st.ring = reinterpret_cast<float *>(mine);
        st.bar = reinterpret_cast<uint64_t *>(mine + HZ_SLOTS * 4 * HZ_WIN * 4);
        st.jw = jw;
        st.c_lo = max(jw - 4, 0);
        st.c_hi = min(jw + 132, ny);
        if (lane == 0) {
            for (int s = 0; s < HZ_SLOTS; ++s) tb_mbar_init(st.bar + s, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            tb_fence_proxy_async();
            for (int i = r0; i <= min(r1, r0 + HZ_AHEAD); ++i) st.issue(p, i, (i - r0) % HZ_SLOTS);
        }
        __syncwarp();
    }

    float iye[4], iyh[4], lo_y[4], up_y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int jc = active ? jt + c : jw;
        iye[c] = __ldg(p.iye + jc);
        iyh[c] = __ldg(p.iyh + jc);
        lo_y[c] = EPS ? __ldg(p.lo_y + jc) : 0.0f;
        up_y[c] = EPS ? __ldg(p.up_y + jc) : 0.0f;
    }
    const float iye_h = __ldg(p.iye + j_end);
    float hzp[4] = {0.0f, 0.0f, 0.0f, 0.0f}, eyp[4] = {0.0f, 0.0f, 0.0f, 0.0f}, epp[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float ey_halo_prev = 0.0f;   // old E_y of the halo column, row below
    if (active) {
#pragma unroll
        for (int c = 0; c < 4; ++c) eyp[c] = __ldg(p.ey_in + (size_t)(r0 - 1) * ny + jt + c);
    }
    if (halo_lane) ey_halo_prev = __ldg(p.ey_in + (size_t)(r0 - 1) * ny + j_end);

    for (int i = r0; i <= r1; ++i) {
        const bool own_row = i < r1;
        const size_t row = (size_t)i * ny;
        float hzo[4] = {0.0f, 0.0f, 0.0f, 0.0f}, exo[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float eyo[4] = {0.0f, 0.0f, 0.0f, 0.0f}, ep[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float ex_left = 0.0f, hz_h = 0.0f, ex_h = 0.0f, ey_h = 0.0f, ep_h = 0.0f;
        if constexpr (STAGED) {
            const int k = i - r0, s = k % HZ_SLOTS;
            if (!tb_mbar_wait(st.bar + s, (uint32_t)((k / HZ_SLOTS) & 1))) {
                if (lane == 0) atomicExch(err, 1);
                for (int q = i; q <= min(r1, i + HZ_AHEAD); ++q) {   // copies still in flight, this row's included
                    const int kq = q - r0;
                    tb_mbar_wait(st.bar + kq % HZ_SLOTS, (uint32_t)((kq / HZ_SLOTS) & 1));
                }
                return;
            }
            if (active) {
                const int o = 4 + 4 * lane;
                const float4 a = *reinterpret_cast<const float4 *>(st.slot(s, 0) + o);
                const float4 bx = *reinterpret_cast<const float4 *>(st.slot(s, 1) + o);
                const float4 by = *reinterpret_cast<const float4 *>(st.slot(s, 2) + o);
                const float4 be = *reinterpret_cast<const float4 *>(st.slot(s, 3) + o);
                hzo[0] = a.x, hzo[1] = a.y, hzo[2] = a.z, hzo[3] = a.w;
                exo[0] = bx.x, exo[1] = bx.y, exo[2] = bx.z, exo[3] = bx.w;
                eyo[0] = by.x, eyo[1] = by.y, eyo[2] = by.z, eyo[3] = by.w;
                ep[0] = be.x, ep[1] = be.y, ep[2] = be.z, ep[3] = be.w;
                ex_left = st.slot(s, 1)[o - 1];
                if (halo_lane) {
                    hz_h = st.slot(s, 0)[o + 4];
                    ex_h = st.slot(s, 1)[o + 4];
                    ey_h = st.slot(s, 2)[o + 4];
                    ep_h = st.slot(s, 3)[o + 4];
                }
            }
            __syncwarp();
            if (lane == 0 && i + HZ_AHEAD + 1 <= r1) {
                tb_fence_proxy_async();
                st.issue(p, i + HZ_AHEAD + 1, s);
            }
        } else {
            if (active) {
                hz_ld4<VEC>(p.hz_in, row + jt, hzo);
                hz_ld4<VEC>(p.ex_in, row + jt, exo);
                hz_ld4<VEC>(p.ey_in, row + jt, eyo);
                if (EPS) hz_ld4<VEC>(p.eps, row + jt, ep);
                if (lane == 0) ex_left = __ldg(p.ex_in + row + jt - 1);
                if (halo_lane) {
                    hz_h = __ldg(p.hz_in + row + j_end);
                    ex_h = __ldg(p.ex_in + row + j_end);
                    ey_h = __ldg(p.ey_in + row + j_end);
                    if (EPS) ep_h = __ldg(p.eps + row + j_end);
                }
            }
            const float left = __shfl_up_sync(FULL, exo[3], 1);
            if (lane != 0) ex_left = left;
        }

        // H_z of the row and of the halo column
        const float ixe = __ldg(p.ixe + i);
        float da[4], db[4];
        float da_h = p.da_u, db_h = p.db_u;
        if (!EPS && p.da) {
            if (active) {
                hz_ld4<VEC>(p.da, row + jt, da);
                hz_ld4<VEC>(p.db, row + jt, db);
            } else {
#pragma unroll
                for (int c = 0; c < 4; ++c) da[c] = db[c] = 0.0f;
            }
            if (halo_lane) da_h = __ldg(p.da + row + j_end), db_h = __ldg(p.db + row + j_end);
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) da[c] = p.da_u, db[c] = p.db_u;
        }
        float hn[4];
        hz_plain_h(hzo, exo, eyo, eyp, ex_left, iye, ixe, da, db, hn);
        if (own_row && active) hz_st4<VEC>(p.hz_out, row + jt, hn);
        float h_halo = 0.0f;
        if (halo_lane) {
            const float dex = ex_h - exo[3];
            const float dey = ey_h - ey_halo_prev;
            float curl = dex * iye_h;
            curl -= dey * ixe;
            h_halo = da_h * hz_h + db_h * curl;
        }
        ey_halo_prev = ey_h;
        float h_next = __shfl_down_sync(FULL, hn[0], 1), e_next = EPS ? __shfl_down_sync(FULL, ep[0], 1) : 0.0f;
        if (halo_lane) h_next = h_halo, e_next = ep_h;

        // E_x of row i, E_y of row i - 1
        if (active) {
            float cax[4], cbx[4], cay[4], cby[4];
            const int re = i - 1;
            const bool do_y = i > r0;
            if (!EPS) {
                hz_ld4<VEC>(p.cb_x, row + jt, cbx);
                hz_ld4<VEC>(p.cb_y, (size_t)re * ny + jt, cby);
                if (p.ca_x) {
                    hz_ld4<VEC>(p.ca_x, row + jt, cax);
                    hz_ld4<VEC>(p.ca_y, (size_t)re * ny + jt, cay);
                } else {
#pragma unroll
                    for (int c = 0; c < 4; ++c) cax[c] = cay[c] = 1.0f;
                }
            }
            float vx[4], vy[4];
            hz_plain_e<EPS>(p, vx, vy, i, re, jt, own_row, do_y, hn, exo, ep, h_next, e_next, lo_y, up_y, iyh, hzp,
                            eyp, epp, cax, cbx, cay, cby);
            if (own_row) hz_st4<VEC>(p.ex_out, row + jt, vx);
            if (do_y) hz_st4<VEC>(p.ey_out, (size_t)re * ny + jt, vy);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            hzp[c] = hn[c];
            eyp[c] = eyo[c];
            epp[c] = ep[c];
        }
    }
}

// Border kernel: one thread per cell of the grid outside the interior box (up to four rectangles, rects[k] = rows
// [r0, r1) x columns [c0, c1), cell offsets in first[k]).  A thread updates its H_z, E_x and E_y; the new H_z of the
// cell right of it and of the cell above it, which its E_x / E_y read, it evaluates again from the old E (not stored).
struct HzBorderRects {
    int32_t n;
    int32_t r0[4], r1[4], c0[4], c1[4];
    int64_t first[5];
};

template <bool EPS>
__global__ void __launch_bounds__(256) hz2d_border_kernel(const Hz2DParams p, const HzBorderRects rects) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = rects.n == 1 ? rects.first[1] : rects.n == 2 ? rects.first[2]
                          : rects.n == 3 ? rects.first[3] : rects.first[4];
    if (t >= total) return;
    // the rectangle of this cell, selected without indexing the parameter arrays by a runtime value
    int k = 0;
    if (rects.n > 1 && t >= rects.first[1]) k = 1;
    if (rects.n > 2 && t >= rects.first[2]) k = 2;
    if (rects.n > 3 && t >= rects.first[3]) k = 3;
    const int64_t first = k == 0 ? 0 : k == 1 ? rects.first[1] : k == 2 ? rects.first[2] : rects.first[3];
    const int rr0 = k == 0 ? rects.r0[0] : k == 1 ? rects.r0[1] : k == 2 ? rects.r0[2] : rects.r0[3];
    const int cc0 = k == 0 ? rects.c0[0] : k == 1 ? rects.c0[1] : k == 2 ? rects.c0[2] : rects.c0[3];
    const int cc1 = k == 0 ? rects.c1[0] : k == 1 ? rects.c1[1] : k == 2 ? rects.c1[2] : rects.c1[3];
    const int64_t local = t - first;
    const int w = cc1 - cc0;
    const int i = rr0 + (int)(local / w), j = cc0 + (int)(local % w);
    const int nx = p.nx, ny = p.ny;
    const size_t idx = (size_t)i * ny + j;
    float exo, eyo, scratch_x, scratch_y;
    const float h = hz2d_hz_at(p, i, j, true, exo, eyo);
    p.hz_out[idx] = h;
    if (j < ny - 1 || p.py) {
        const int jn = j < ny - 1 ? j + 1 : 0;
        const float hn = hz2d_hz_at(p, i, jn, false, scratch_x, scratch_y);
        const float up = j < ny - 1 ? hn : hz_wrap_hi(hn);
        float ca = 1.0f, cb;
        if (EPS) {
            cb = hz_cb_lossless(__ldg(p.eps + idx), __ldg(p.eps + (size_t)i * ny + jn), __ldg(p.lo_y + j),
                                __ldg(p.up_y + j), p.dt, p.eps0);
        } else {
            ca = p.ca_x ? __ldg(p.ca_x + idx) : 1.0f;
            cb = __ldg(p.cb_x + idx);
        }
        p.ex_out[idx] = hz2d_ex_at(p, i, j, exo, ca, cb, h, up);
    } else {
        p.ex_out[idx] = exo;   // the last face of an open y is never updated
    }
    if (i < nx - 1 || p.px) {
        const int in = i < nx - 1 ? i + 1 : 0;
        const float hn = hz2d_hz_at(p, in, j, false, scratch_x, scratch_y);
        const float up = i < nx - 1 ? hn : hz_wrap_hi(hn);
        float ca = 1.0f, cb;
        if (EPS) {
            cb = hz_cb_lossless(__ldg(p.eps + idx), __ldg(p.eps + (size_t)in * ny + j), __ldg(p.lo_x + i),
                                __ldg(p.up_x + i), p.dt, p.eps0);
        } else {
            ca = p.ca_y ? __ldg(p.ca_y + idx) : 1.0f;
            cb = __ldg(p.cb_y + idx);
        }
        p.ey_out[idx] = hz2d_ey_at(p, i, j, eyo, ca, cb, h, up);
    } else {
        p.ey_out[idx] = eyo;   // the last face of an open x is never updated
    }
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
