// 3D Yee kernels for sm_100a: the H update and the E update of one step (CPML fused through per-axis row maps, the
// dipole injection fused into the E update) and the running DFT of the flux planes.
//
// Layout as open_sol's em_fdtd_3d (engine3d.py:4-12): fields (nx, ny, nz) float32, z contiguous, idx = (i ny + j) nz
// + k; E_x on the hi-x face, E_y on the hi-y face, E_z on the hi-z face of a cell; H on the edges; a uint16 material id
// per cell and small per-id tables.  Each thread owns one (j, k) column and streams along x over a chunk of planes,
// carrying the plane it loaded as the next (H) or previous (E) neighbour into the following iteration; a warp covers 32
// consecutive k, so every field access of a warp is one contiguous 128-byte row.
//
// Arithmetic: the evaluation order of update_h_3d / update_e_3d (physics/em3d/kernels3d.py:335-392,538-609) and its
// numpy twins (:451-463,640-661) for a Cartesian grid with one real field set (the radial factors are exactly 1 and
// are left out), compiled with -fmad=false: results equal the reference's numpy twins bit for bit.  A sample read
// across the hi edge of an axis is c F + s F with c = 1, s = 0, as the reference's wrap_load evaluates it; on a
// non-periodic axis the last row's inverse spacing is 0.  The missing lo H below row 0 of a non-periodic axis is 0.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mbarrier.cuh"

#define EM3D_EPS0F 8.8541878128e-12f

constexpr int EM3D_BZ = 32;            // threads along z (one warp)
constexpr int EM3D_BY = 8;             // warps along y
constexpr int EM3D_MAX_DIPOLES = 16;

struct Em3DCpmlAxis {
    const int32_t *rm_h, *rm_e;        // grid row -> psi row (-1 outside the layers)
    const float *b_h, *g_h, *b_e, *g_e;
    float *ph_first, *ph_second, *pe_first, *pe_second;       // psi read
    float *oph_first, *oph_second, *ope_first, *ope_second;   // psi written (the same arrays for an in-place step)
    int32_t nr;                        // psi rows of the axis (0: no CPML on it)
};

// A box of cells [i0, i1) x [j0, j1) x [k0, k1).
struct Em3DBox {
    int32_t i0, i1, j0, j1, k0, k1;
};

constexpr int EM3D_MAX_BOXES = 6;

struct Em3DParams {
    int32_t nx, ny, nz, px, py, pz;
    int32_t x_chunk;                   // x planes per block
    float *ex, *ey, *ez, *hx, *hy, *hz;        // the fields a kernel reads
    float *oex, *oey, *oez, *ohx, *ohy, *ohz;  // where it writes them (the same arrays for an in-place step)
    // em3d_h_kernel / em3d_e_kernel: the cells they update, as boxes; blockIdx.z runs over the boxes' x chunks
    // (zbase[b] = first z block of box b), blockIdx.x / y over the largest box's k / j extent
    int32_t n_boxes;
    Em3DBox boxes[EM3D_MAX_BOXES];
    int32_t zbase[EM3D_MAX_BOXES + 1];
    const uint16_t *mat;
    const float *t_ex, *t_ey, *t_ez, *t_sig;   // E tables per material id
    const float *t_da, *t_db;                  // H coefficients per material id
    int32_t h_uniform;                         // every id has da = da_u, db = db_u (mat is not read by H)
    float da_u, db_u;
    int32_t e_lossless;                        // every sigma_e is 0: ca = 1, cb = dt / eps
    int32_t n_ids;
    int32_t same_ok;                           // every face share is 0.5: t_same holds the same-id faces
    const float *t_same;                       // per component: ca (n_ids) then cb (n_ids)
    const float *iex, *iey, *iez, *ihx, *ihy, *ihz;
    const float *wlx, *wux, *wly, *wuy, *wlz, *wuz;
    float dt;
    Em3DCpmlAxis cpml[3];
    int32_t n_dip;
    int32_t dip_comp[EM3D_MAX_DIPOLES];
    int32_t dip_i[EM3D_MAX_DIPOLES];           // x plane of the dipole cell
    int32_t dip_o[EM3D_MAX_DIPOLES];           // in-plane offset j nz + k
    float dip_weight[EM3D_MAX_DIPOLES];
    const float *dip_values;                   // (n_dip, values_stride) float32 amplitude per step
    int64_t values_stride, k_step;
    int32_t *err;                              // set to 1 when a bounded wait of the staged kernel runs out
};

__device__ __forceinline__ float em3d_wrapped(float v) { return __fadd_rn(__fmul_rn(1.0f, v), __fmul_rn(0.0f, v)); }

// psi' = b psi + g difference, written to psi_out (psi_in itself for an in-place step); returns psi'.
__device__ __forceinline__ float em3d_psi(const float *psi_in, float *psi_out, size_t p, float b, float g,
                                          float difference) {
    const float value = b * psi_in[p] + g * difference;
    psi_out[p] = value;
    return value;
}

// ---------------------------------------------------------------------------------------------------- H update
// Thread (j, k) streams x-planes i0 .. i1 - 1.  The loads of plane i + 1 (its next plane, its y / z neighbours, its
// own H) are issued before plane i is computed, so every warp keeps two planes of loads in flight; fields the kernel
// only reads go through the read-only path.  In-plane offsets are 32-bit (ny nz < 2^31 is checked at create).
// The box of this block and its x chunk (boxes of em3d_h_kernel / em3d_e_kernel; blocks of BZ x BY threads along
// k and j).
template <int BZ, int BY>
__device__ __forceinline__ bool em3d_block_box(const Em3DParams &p, int &j, int &k, int &i0, int &i1) {
    int b = 0;
    while (b + 1 < p.n_boxes && (int)blockIdx.z >= p.zbase[b + 1]) ++b;
    const Em3DBox bx = p.boxes[b];
    k = bx.k0 + blockIdx.x * BZ + threadIdx.x;
    j = bx.j0 + blockIdx.y * BY + threadIdx.y;
    i0 = bx.i0 + ((int)blockIdx.z - p.zbase[b]) * p.x_chunk;
    i1 = min(bx.i1, i0 + p.x_chunk);
    return j < bx.j1 && k < bx.k1 && i0 < i1;
}

template <int BZ = EM3D_BZ, int BY = EM3D_BY>
__global__ void __launch_bounds__(BZ * BY) em3d_h_kernel(const Em3DParams p) {
    int j, k, i0, i1;
    if (!em3d_block_box<BZ, BY>(p, j, k, i0, i1)) return;
    const size_t sx = (size_t)p.ny * p.nz;
    const float *__restrict__ ex = p.ex;
    const float *__restrict__ ey = p.ey;
    const float *__restrict__ ez = p.ez;
    const float *hx = p.hx;   // H in, H out: the same arrays when the step runs in place
    const float *hy = p.hy;
    const float *hz = p.hz;
    float *ohx = p.ohx;
    float *ohy = p.ohy;
    float *ohz = p.ohz;
    const bool wy = j + 1 == p.ny, wz = k + 1 == p.nz;
    const int o = j * p.nz + k;
    const int oy = wy ? k : o + p.nz;             // hi y neighbour (row 0 across the edge)
    const int oz = wz ? j * p.nz : o + 1;         // hi z neighbour
    const float ihy = p.ihy[j], ihz = p.ihz[k];
    const int32_t ry = p.cpml[1].nr ? p.cpml[1].rm_h[j] : -1;
    const int32_t rz = p.cpml[2].nr ? p.cpml[2].rm_h[k] : -1;
    size_t b = (size_t)i0 * sx;                                   // plane i
    size_t bn = (size_t)(i0 + 1 < p.nx ? i0 + 1 : 0) * sx;        // plane i + 1 (plane 0 across the x edge)
    float ex0 = __ldg(ex + b + o), ey0 = __ldg(ey + b + o), ez0 = __ldg(ez + b + o);
    float exn = __ldg(ex + bn + o), eyn = __ldg(ey + bn + o), ezn = __ldg(ez + bn + o);
    float exy = __ldg(ex + b + oy), ezy = __ldg(ez + b + oy);
    float exz = __ldg(ex + b + oz), eyz = __ldg(ey + b + oz);
    float hx0 = hx[b + o], hy0 = hy[b + o], hz0 = hz[b + o];
    for (int i = i0; i < i1; ++i) {
        const bool more = i + 1 < i1;
        const size_t bnn = (size_t)(i + 2 < p.nx ? i + 2 : 0) * sx;   // plane i + 2
        float exn2 = 0.0f, eyn2 = 0.0f, ezn2 = 0.0f, exy2 = 0.0f, ezy2 = 0.0f, exz2 = 0.0f, eyz2 = 0.0f;
        float hx2 = 0.0f, hy2 = 0.0f, hz2 = 0.0f;
        if (more) {
            exn2 = __ldg(ex + bnn + o);
            eyn2 = __ldg(ey + bnn + o);
            ezn2 = __ldg(ez + bnn + o);
            exy2 = __ldg(ex + bn + oy);
            ezy2 = __ldg(ez + bn + oy);
            exz2 = __ldg(ex + bn + oz);
            eyz2 = __ldg(ey + bn + oz);
            hx2 = hx[bn + o];
            hy2 = hy[bn + o];
            hz2 = hz[bn + o];
        }
        const bool wx = i + 1 == p.nx;
        const float dez_y = (wy ? em3d_wrapped(ezy) : ezy) - ez0;
        const float dey_z = (wz ? em3d_wrapped(eyz) : eyz) - ey0;
        const float dex_z = (wz ? em3d_wrapped(exz) : exz) - ex0;
        const float dez_x = (wx ? em3d_wrapped(ezn) : ezn) - ez0;
        const float dey_x = (wx ? em3d_wrapped(eyn) : eyn) - ey0;
        const float dex_y = (wy ? em3d_wrapped(exy) : exy) - ex0;
        float da, db;
        if (p.h_uniform) {
            da = p.da_u;
            db = p.db_u;
        } else {
            const uint16_t m = p.mat[b + o];
            da = p.t_da[m];
            db = p.t_db[m];
        }
        const float ihx = p.ihx[i];
        float vx = da * hx0 - db * (dez_y * ihy - dey_z * ihz);
        float vy = da * hy0 - db * (dex_z * ihz - dez_x * ihx);
        float vz = da * hz0 - db * (dey_x * ihx - dex_y * ihy);
        if (p.cpml[0].nr) {
            const int32_t r = p.cpml[0].rm_h[i];
            if (r >= 0) {   // x layers: H_y from E_z (+), H_z from E_y (-)
                const Em3DCpmlAxis &c = p.cpml[0];
                const size_t q = (size_t)r * sx + o;
                vy += db * em3d_psi(c.ph_first, c.oph_first, q, c.b_h[r], c.g_h[r], dez_x);
                vz -= db * em3d_psi(c.ph_second, c.oph_second, q, c.b_h[r], c.g_h[r], dey_x);
            }
        }
        if (ry >= 0) {   // y layers: H_x from E_z (-), H_z from E_x (+)
            const Em3DCpmlAxis &c = p.cpml[1];
            const size_t q = ((size_t)i * c.nr + ry) * p.nz + k;
            vx -= db * em3d_psi(c.ph_first, c.oph_first, q, c.b_h[ry], c.g_h[ry], dez_y);
            vz += db * em3d_psi(c.ph_second, c.oph_second, q, c.b_h[ry], c.g_h[ry], dex_y);
        }
        if (rz >= 0) {   // z layers: H_x from E_y (+), H_y from E_x (-)
            const Em3DCpmlAxis &c = p.cpml[2];
            const size_t q = ((size_t)i * p.ny + j) * c.nr + rz;
            vx += db * em3d_psi(c.ph_first, c.oph_first, q, c.b_h[rz], c.g_h[rz], dey_z);
            vy -= db * em3d_psi(c.ph_second, c.oph_second, q, c.b_h[rz], c.g_h[rz], dex_z);
        }
        ohx[b + o] = vx;
        ohy[b + o] = vy;
        ohz[b + o] = vz;
        ex0 = exn;
        ey0 = eyn;
        ez0 = ezn;
        exn = exn2;
        eyn = eyn2;
        ezn = ezn2;
        exy = exy2;
        ezy = ezy2;
        exz = exz2;
        eyz = eyz2;
        hx0 = hx2;
        hy0 = hy2;
        hz0 = hz2;
        b = bn;
        bn = bnn;
    }
}

// ---------------------------------------------------------------------------------------------------- E update
// ca, cb of the face between cells a and b (face_coefficients, kernels3d.py:61-82; b = a on the last row of a
// non-periodic axis).
__device__ __forceinline__ void em3d_face(const Em3DParams &p, const float *t_eps, uint16_t ia, uint16_t ib, float wa,
                                          float wb, float &ca, float &cb) {
    float ea = t_eps[ia], eb = t_eps[ib];
    if (ea < 0.0f && eb < 0.0f) {
        ca = 0.0f;
        cb = 0.0f;
        return;
    }
    float sa = 0.0f, sb = 0.0f;
    if (!p.e_lossless) {
        sa = p.t_sig[ia];
        sb = p.t_sig[ib];
    }
    if (ea < 0.0f) {
        ea = eb;
        sa = sb;
    } else if (eb < 0.0f) {
        eb = ea;
        sb = sa;
    }
    const float eps = (wa * ea + wb * eb) * EM3D_EPS0F;
    if (p.e_lossless) {   // sigma 0: loss 0, den 1, so ca = 1 and cb = dt / eps exactly
        ca = 1.0f;
        cb = p.dt / eps;
        return;
    }
    const float sig = wa * sa + wb * sb;
    const float loss = sig * p.dt / (2.0f * eps);
    const float den = 1.0f + loss;
    ca = (1.0f - loss) / den;
    cb = (p.dt / eps) / den;
}

// The same with the table of faces between two cells of one material id (t_same: per component ca then cb per id,
// computed by em3d_face with the grid's uniform shares 0.5 / 0.5, so the values are the formula's own).
__device__ __forceinline__ void em3d_face_fast(const Em3DParams &p, int comp, const float *t_eps, uint16_t ia,
                                               uint16_t ib, float wa, float wb, float &ca, float &cb) {
    if (p.same_ok && ia == ib) {
        ca = p.t_same[(2 * comp) * p.n_ids + ia];
        cb = p.t_same[(2 * comp + 1) * p.n_ids + ia];
        return;
    }
    em3d_face(p, t_eps, ia, ib, wa, wb, ca, cb);
}

// F0 - F[lo neighbour]: the wrapped sample on a periodic axis, F0 itself below row 0 of an open axis.
__device__ __forceinline__ float em3d_lo_diff(float f0, float lo, bool first_row, int periodic) {
    if (!first_row) return f0 - lo;
    return periodic ? f0 - em3d_wrapped(lo) : f0;
}

template <int BZ = EM3D_BZ, int BY = EM3D_BY>
__global__ void __launch_bounds__(BZ * BY, 4) em3d_e_kernel(const Em3DParams p) {
    int j, k, i0, i1;
    if (!em3d_block_box<BZ, BY>(p, j, k, i0, i1)) return;
    const size_t sx = (size_t)p.ny * p.nz;
    const float *__restrict__ hx = p.hx;
    const float *__restrict__ hy = p.hy;
    const float *__restrict__ hz = p.hz;
    const float *ex = p.ex;   // E in, E out: the same arrays when the step runs in place
    const float *ey = p.ey;
    const float *ez = p.ez;
    float *oex = p.oex;
    float *oey = p.oey;
    float *oez = p.oez;
    const uint16_t *__restrict__ mat = p.mat;
    const bool fy = j == 0, fz = k == 0;
    const int o = j * p.nz + k;
    const int oym = fy ? (p.ny - 1) * p.nz + k : o - p.nz;   // lo y neighbour (last row across the edge)
    const int ozm = fz ? j * p.nz + p.nz - 1 : o - 1;
    // hi partners of the E_y / E_z faces (the cell itself on the last row of an open axis)
    const int oyp = j + 1 < p.ny ? o + p.nz : (p.py ? k : o);
    const int ozp = k + 1 < p.nz ? o + 1 : (p.pz ? j * p.nz : o);
    const float iey = p.iey[j], iez = p.iez[k];
    const float wly = p.wly[j], wuy = p.wuy[j], wlz = p.wlz[k], wuz = p.wuz[k];
    const int32_t ry = p.cpml[1].nr ? p.cpml[1].rm_e[j] : -1;
    const int32_t rz = p.cpml[2].nr ? p.cpml[2].rm_e[k] : -1;
    auto partner_plane = [&](int i) -> size_t {   // plane of the hi-x partner of plane i
        return (size_t)(i + 1 < p.nx ? i + 1 : (p.px ? 0 : i)) * sx;
    };
    size_t b = (size_t)i0 * sx;
    const size_t bm = (size_t)(i0 > 0 ? i0 - 1 : p.nx - 1) * sx;   // plane i - 1 (wrapped for i = 0)
    float hy_m = __ldg(hy + bm + o), hz_m = __ldg(hz + bm + o);
    float hx0 = __ldg(hx + b + o), hy0 = __ldg(hy + b + o), hz0 = __ldg(hz + b + o);
    float hx_y = __ldg(hx + b + oym), hz_y = __ldg(hz + b + oym);
    float hx_z = __ldg(hx + b + ozm), hy_z = __ldg(hy + b + ozm);
    float ex0 = ex[b + o], ey0 = ey[b + o], ez0 = ez[b + o];
    uint16_t m0 = __ldg(mat + b + o), mx = __ldg(mat + partner_plane(i0) + o);
    uint16_t my = __ldg(mat + b + oyp), mz = __ldg(mat + b + ozp);
    for (int i = i0; i < i1; ++i) {
        const bool more = i + 1 < i1;
        const size_t bn = (size_t)(i + 1) * sx;   // plane i + 1 (only read when more)
        float hx2 = 0.0f, hy2 = 0.0f, hz2 = 0.0f, hx_y2 = 0.0f, hz_y2 = 0.0f, hx_z2 = 0.0f, hy_z2 = 0.0f;
        float ex2 = 0.0f, ey2 = 0.0f, ez2 = 0.0f;
        uint16_t mx2 = 0, my2 = 0, mz2 = 0;
        if (more) {
            hx2 = __ldg(hx + bn + o);
            hy2 = __ldg(hy + bn + o);
            hz2 = __ldg(hz + bn + o);
            hx_y2 = __ldg(hx + bn + oym);
            hz_y2 = __ldg(hz + bn + oym);
            hx_z2 = __ldg(hx + bn + ozm);
            hy_z2 = __ldg(hy + bn + ozm);
            ex2 = ex[bn + o];
            ey2 = ey[bn + o];
            ez2 = ez[bn + o];
            mx2 = __ldg(mat + partner_plane(i + 1) + o);
            my2 = __ldg(mat + bn + oyp);
            mz2 = __ldg(mat + bn + ozp);
        }
        const bool fx = i == 0;
        const float dhz_y = em3d_lo_diff(hz0, hz_y, fy, p.py);
        const float dhy_z = em3d_lo_diff(hy0, hy_z, fz, p.pz);
        const float dhx_z = em3d_lo_diff(hx0, hx_z, fz, p.pz);
        const float dhz_x = em3d_lo_diff(hz0, hz_m, fx, p.px);
        const float dhy_x = em3d_lo_diff(hy0, hy_m, fx, p.px);
        const float dhx_y = em3d_lo_diff(hx0, hx_y, fy, p.py);
        float ca, cbx, cby, cbz;
        em3d_face_fast(p, 0, p.t_ex, m0, mx, p.wlx[i], p.wux[i], ca, cbx);
        const float iex = p.iex[i];
        float vx = ca * ex0 + cbx * (dhz_y * iey - dhy_z * iez);
        em3d_face_fast(p, 1, p.t_ey, m0, my, wly, wuy, ca, cby);
        float vy = ca * ey0 + cby * (dhx_z * iez - dhz_x * iex);
        em3d_face_fast(p, 2, p.t_ez, m0, mz, wlz, wuz, ca, cbz);
        float vz = ca * ez0 + cbz * (dhy_x * iex - dhx_y * iey);
        if (p.cpml[0].nr) {
            const int32_t r = p.cpml[0].rm_e[i];
            if (r >= 0) {   // x layers: E_y from H_z (-), E_z from H_y (+)
                const Em3DCpmlAxis &c = p.cpml[0];
                const size_t q = (size_t)r * sx + o;
                vy -= cby * em3d_psi(c.pe_first, c.ope_first, q, c.b_e[r], c.g_e[r], dhz_x);
                vz += cbz * em3d_psi(c.pe_second, c.ope_second, q, c.b_e[r], c.g_e[r], dhy_x);
            }
        }
        if (ry >= 0) {   // y layers: E_x from H_z (+), E_z from H_x (-)
            const Em3DCpmlAxis &c = p.cpml[1];
            const size_t q = ((size_t)i * c.nr + ry) * p.nz + k;
            vx += cbx * em3d_psi(c.pe_first, c.ope_first, q, c.b_e[ry], c.g_e[ry], dhz_y);
            vz -= cbz * em3d_psi(c.pe_second, c.ope_second, q, c.b_e[ry], c.g_e[ry], dhx_y);
        }
        if (rz >= 0) {   // z layers: E_x from H_y (-), E_y from H_x (+)
            const Em3DCpmlAxis &c = p.cpml[2];
            const size_t q = ((size_t)i * p.ny + j) * c.nr + rz;
            vx -= cbx * em3d_psi(c.pe_first, c.ope_first, q, c.b_e[rz], c.g_e[rz], dhy_z);
            vy += cby * em3d_psi(c.pe_second, c.ope_second, q, c.b_e[rz], c.g_e[rz], dhx_z);
        }
        // dipoles (DipoleSource3D.inject, sources3d.py:69-75): E += FP32(s(t + dt/2)) * weight after the update
        for (int d = 0; d < p.n_dip; ++d) {
            if (p.dip_o[d] != o || p.dip_i[d] != i) continue;
            const float add = p.dip_values[d * p.values_stride + p.k_step] * p.dip_weight[d];
            if (p.dip_comp[d] == 0) vx = vx + add;
            else if (p.dip_comp[d] == 1) vy = vy + add;
            else vz = vz + add;
        }
        oex[b + o] = vx;
        oey[b + o] = vy;
        oez[b + o] = vz;
        hy_m = hy0;
        hz_m = hz0;
        hx0 = hx2;
        hy0 = hy2;
        hz0 = hz2;
        hx_y = hx_y2;
        hz_y = hz_y2;
        hx_z = hx_z2;
        hy_z = hy_z2;
        ex0 = ex2;
        ey0 = ey2;
        ez0 = ez2;
        m0 = (i + 1 < p.nx) ? mx : m0;   // the next plane's own id (mx is it whenever i + 1 < nx)
        mx = mx2;
        my = my2;
        mz = mz2;
        b = bn;
    }
}

// ---------------------------------------------------------------------------------------------------- fused step
// One whole Yee step (H then E) of the cells of box `in` -- every cell but the outermost layer of each axis, where a
// sample would cross the grid edge -- in one pass that reads E^n, H^{n-1/2} and the CPML psi once and writes E^{n+1},
// H^{n+1/2} and psi' once: two field sets and two psi sets, read one, write the other, swapped after each step.  A
// block is a 32 x TY tile of (k, j) columns streaming a chunk of x planes; lane 0 of each warp is the column k0 - 1
// and warp 0 the row j0 - 1, whose H the tile's E update needs: they compute H only (the halo, never stored; a halo
// cell in a CPML layer reads the old psi and stores nothing).  Per plane every thread updates H of its column, then E
// takes H^{n+1/2} of the k - 1 neighbour from the next lower lane (a shuffle), of the j - 1 neighbour through shared
// memory (double-buffered by plane parity, one barrier per plane) and of the i - 1 plane from the thread's own
// previous iteration (the chunk starts one plane early, with H only).  The arithmetic of every cell, CPML terms
// included, is em3d_h_kernel's and em3d_e_kernel's term for term, so the results are those of the two-kernel step
// bit for bit.
constexpr int EM3D_FZ = 32;   // lanes along k (lane 0: the halo column)

template <int TY, int MINB>
__global__ void __launch_bounds__(EM3D_FZ * TY, MINB) em3d_fused_kernel(const Em3DParams p, const Em3DBox in) {
    __shared__ float s_hz[2][TY][EM3D_FZ];
    __shared__ float s_hx[2][TY][EM3D_FZ];
    const int lane = threadIdx.x, w = threadIdx.y;
    const int kk = in.k0 - 1 + (int)blockIdx.x * (EM3D_FZ - 1) + lane;
    const int jj = in.j0 - 1 + (int)blockIdx.y * (TY - 1) + w;
    const bool e_thread = lane > 0 && w > 0;                    // not a halo lane or row
    const bool emit = e_thread && kk < in.k1 && jj < in.j1;     // stores its column's results
    // a column past the box computes a discarded copy of the box's last column (every address stays inside)
    const int k = min(kk, in.k1 - 1), j = min(jj, in.j1 - 1);
    const int i_first = in.i0 + (int)blockIdx.z * p.x_chunk;
    const int i_last = min(in.i1, i_first + p.x_chunk);
    const size_t sx = (size_t)p.ny * p.nz;
    const int o = j * p.nz + k;
    const int oy = o + p.nz, oz = o + 1;
    const float *__restrict__ ex = p.ex;
    const float *__restrict__ ey = p.ey;
    const float *__restrict__ ez = p.ez;
    const float *__restrict__ hx = p.hx;
    const float *__restrict__ hy = p.hy;
    const float *__restrict__ hz = p.hz;
    float *__restrict__ oex = p.oex;
    float *__restrict__ oey = p.oey;
    float *__restrict__ oez = p.oez;
    float *__restrict__ ohx = p.ohx;
    float *__restrict__ ohy = p.ohy;
    float *__restrict__ ohz = p.ohz;
    const uint16_t *__restrict__ mat = p.mat;
    const float ihy = p.ihy[j], ihz = p.ihz[k];
    const float iey = p.iey[j], iez = p.iez[k];
    const float wly = p.wly[j], wuy = p.wuy[j], wlz = p.wlz[k], wuz = p.wuz[k];
    // CPML rows of this column on y and z (-1: outside the layers)
    const int32_t ryh = p.cpml[1].nr ? p.cpml[1].rm_h[j] : -1, rye = p.cpml[1].nr ? p.cpml[1].rm_e[j] : -1;
    const int32_t rzh = p.cpml[2].nr ? p.cpml[2].rm_h[k] : -1, rze = p.cpml[2].nr ? p.cpml[2].rm_e[k] : -1;
    // plane i = i_first - 1 (the halo plane), its loads
    int i = i_first - 1;
    size_t b = (size_t)i * sx;
    size_t bn = b + sx;
    float ex0 = __ldg(ex + b + o), ey0 = __ldg(ey + b + o), ez0 = __ldg(ez + b + o);
    float exn = __ldg(ex + bn + o), eyn = __ldg(ey + bn + o), ezn = __ldg(ez + bn + o);
    float exy = __ldg(ex + b + oy), ezy = __ldg(ez + b + oy);
    float exz = __ldg(ex + b + oz), eyz = __ldg(ey + b + oz);
    float hx0 = __ldg(hx + b + o), hy0 = __ldg(hy + b + o), hz0 = __ldg(hz + b + o);
    uint16_t m0 = __ldg(mat + b + o), mx = __ldg(mat + bn + o);
    uint16_t my = __ldg(mat + b + oy), mz = __ldg(mat + b + oz);
    float hy_m = 0.0f, hz_m = 0.0f;   // H^{n+1/2} of plane i - 1 of this column
    int par = 0;
    for (; i < i_last; ++i) {
        const bool more = i + 1 < i_last;
        const size_t bnn = bn + sx;
        float exn2 = 0.0f, eyn2 = 0.0f, ezn2 = 0.0f, exy2 = 0.0f, ezy2 = 0.0f, exz2 = 0.0f, eyz2 = 0.0f;
        float hx2 = 0.0f, hy2 = 0.0f, hz2 = 0.0f;
        uint16_t mx2 = 0, my2 = 0, mz2 = 0;
        if (more) {   // plane i + 1's loads (plane i + 2 <= i_last <= in.i1 <= nx - 1)
            exn2 = __ldg(ex + bnn + o);
            eyn2 = __ldg(ey + bnn + o);
            ezn2 = __ldg(ez + bnn + o);
            exy2 = __ldg(ex + bn + oy);
            ezy2 = __ldg(ez + bn + oy);
            exz2 = __ldg(ex + bn + oz);
            eyz2 = __ldg(ey + bn + oz);
            hx2 = __ldg(hx + bn + o);
            hy2 = __ldg(hy + bn + o);
            hz2 = __ldg(hz + bn + o);
            mx2 = __ldg(mat + bnn + o);
            my2 = __ldg(mat + bn + oy);
            mz2 = __ldg(mat + bn + oz);
        }
        const bool inside = i >= i_first;
        const bool store = emit && inside;
        // H^{n+1/2} of (i, j, k): em3d_h_kernel's update (no sample crosses the grid edge in the box)
        float da, db;
        if (p.h_uniform) {
            da = p.da_u;
            db = p.db_u;
        } else {
            da = p.t_da[m0];
            db = p.t_db[m0];
        }
        const float ihx = p.ihx[i];
        const float dez_y = ezy - ez0, dey_z = eyz - ey0, dex_z = exz - ex0, dez_x = ezn - ez0;
        const float dey_x = eyn - ey0, dex_y = exy - ex0;
        float vhx = da * hx0 - db * (dez_y * ihy - dey_z * ihz);
        float vhy = da * hy0 - db * (dex_z * ihz - dez_x * ihx);
        float vhz = da * hz0 - db * (dey_x * ihx - dex_y * ihy);
        const int32_t rxh = p.cpml[0].nr ? p.cpml[0].rm_h[i] : -1;
        if (rxh >= 0) {   // x layers: H_y from E_z (+), H_z from E_y (-)
            const Em3DCpmlAxis &c = p.cpml[0];
            const size_t q = (size_t)rxh * sx + o;
            const float f = c.b_h[rxh] * c.ph_first[q] + c.g_h[rxh] * dez_x;
            const float g = c.b_h[rxh] * c.ph_second[q] + c.g_h[rxh] * dey_x;
            if (store) {
                c.oph_first[q] = f;
                c.oph_second[q] = g;
            }
            vhy += db * f;
            vhz -= db * g;
        }
        if (ryh >= 0) {   // y layers: H_x from E_z (-), H_z from E_x (+)
            const Em3DCpmlAxis &c = p.cpml[1];
            const size_t q = ((size_t)i * c.nr + ryh) * p.nz + k;
            const float f = c.b_h[ryh] * c.ph_first[q] + c.g_h[ryh] * dez_y;
            const float g = c.b_h[ryh] * c.ph_second[q] + c.g_h[ryh] * dex_y;
            if (store) {
                c.oph_first[q] = f;
                c.oph_second[q] = g;
            }
            vhx -= db * f;
            vhz += db * g;
        }
        if (rzh >= 0) {   // z layers: H_x from E_y (+), H_y from E_x (-)
            const Em3DCpmlAxis &c = p.cpml[2];
            const size_t q = ((size_t)i * p.ny + j) * c.nr + rzh;
            const float f = c.b_h[rzh] * c.ph_first[q] + c.g_h[rzh] * dey_z;
            const float g = c.b_h[rzh] * c.ph_second[q] + c.g_h[rzh] * dex_z;
            if (store) {
                c.oph_first[q] = f;
                c.oph_second[q] = g;
            }
            vhx += db * f;
            vhy -= db * g;
        }
        if (store) {
            ohx[b + o] = vhx;
            ohy[b + o] = vhy;
            ohz[b + o] = vhz;
        }
        s_hz[par][w][lane] = vhz;
        s_hx[par][w][lane] = vhx;
        const float hy_z = __shfl_up_sync(0xffffffffu, vhy, 1);   // H^{n+1/2} of (i, j, k - 1)
        const float hx_z = __shfl_up_sync(0xffffffffu, vhx, 1);
        __syncthreads();
        if (e_thread && inside) {
            const float hz_y = s_hz[par][w - 1][lane];            // H^{n+1/2} of (i, j - 1, k)
            const float hx_y = s_hx[par][w - 1][lane];
            const float dhz_y = vhz - hz_y, dhy_z = vhy - hy_z, dhx_z = vhx - hx_z;
            const float dhz_x = vhz - hz_m, dhy_x = vhy - hy_m, dhx_y = vhx - hx_y;
            float ca, cbx, cby, cbz;
            const float iex = p.iex[i];
            em3d_face_fast(p, 0, p.t_ex, m0, mx, p.wlx[i], p.wux[i], ca, cbx);
            float vx = ca * ex0 + cbx * (dhz_y * iey - dhy_z * iez);
            em3d_face_fast(p, 1, p.t_ey, m0, my, wly, wuy, ca, cby);
            float vy = ca * ey0 + cby * (dhx_z * iez - dhz_x * iex);
            em3d_face_fast(p, 2, p.t_ez, m0, mz, wlz, wuz, ca, cbz);
            float vz = ca * ez0 + cbz * (dhy_x * iex - dhx_y * iey);
            const int32_t rxe = p.cpml[0].nr ? p.cpml[0].rm_e[i] : -1;
            if (rxe >= 0) {   // x layers: E_y from H_z (-), E_z from H_y (+)
                const Em3DCpmlAxis &c = p.cpml[0];
                const size_t q = (size_t)rxe * sx + o;
                const float f = c.b_e[rxe] * c.pe_first[q] + c.g_e[rxe] * dhz_x;
                const float g = c.b_e[rxe] * c.pe_second[q] + c.g_e[rxe] * dhy_x;
                if (emit) {
                    c.ope_first[q] = f;
                    c.ope_second[q] = g;
                }
                vy -= cby * f;
                vz += cbz * g;
            }
            if (rye >= 0) {   // y layers: E_x from H_z (+), E_z from H_x (-)
                const Em3DCpmlAxis &c = p.cpml[1];
                const size_t q = ((size_t)i * c.nr + rye) * p.nz + k;
                const float f = c.b_e[rye] * c.pe_first[q] + c.g_e[rye] * dhz_y;
                const float g = c.b_e[rye] * c.pe_second[q] + c.g_e[rye] * dhx_y;
                if (emit) {
                    c.ope_first[q] = f;
                    c.ope_second[q] = g;
                }
                vx += cbx * f;
                vz -= cbz * g;
            }
            if (rze >= 0) {   // z layers: E_x from H_y (-), E_y from H_x (+)
                const Em3DCpmlAxis &c = p.cpml[2];
                const size_t q = ((size_t)i * p.ny + j) * c.nr + rze;
                const float f = c.b_e[rze] * c.pe_first[q] + c.g_e[rze] * dhy_z;
                const float g = c.b_e[rze] * c.pe_second[q] + c.g_e[rze] * dhx_z;
                if (emit) {
                    c.ope_first[q] = f;
                    c.ope_second[q] = g;
                }
                vx -= cbx * f;
                vy += cby * g;
            }
            for (int d = 0; d < p.n_dip; ++d) {   // dipoles: E += FP32(s(t + dt/2)) * weight after the update
                if (p.dip_o[d] != o || p.dip_i[d] != i) continue;
                const float add = p.dip_values[d * p.values_stride + p.k_step] * p.dip_weight[d];
                if (p.dip_comp[d] == 0) vx = vx + add;
                else if (p.dip_comp[d] == 1) vy = vy + add;
                else vz = vz + add;
            }
            if (emit) {
                oex[b + o] = vx;
                oey[b + o] = vy;
                oez[b + o] = vz;
            }
        }
        hy_m = vhy;
        hz_m = vhz;
        ex0 = exn;
        ey0 = eyn;
        ez0 = ezn;
        exn = exn2;
        eyn = eyn2;
        ezn = ezn2;
        exy = exy2;
        ezy = ezy2;
        exz = exz2;
        eyz = eyz2;
        hx0 = hx2;
        hy0 = hy2;
        hz0 = hz2;
        m0 = mx;
        mx = mx2;
        my = my2;
        mz = mz2;
        b = bn;
        bn = bnn;
        par ^= 1;
    }
}

// ---------------------------------------------------------------------------------------------------- staged step
// em3d_fused_kernel with the planes staged in shared memory: each x plane of the block's tile arrives by tiled tensor
// copies (cp.async.bulk.tensor, one per array: the three E boxes of TY + 1 rows, the three H boxes of TY rows, the
// material-id box of TY + 1 rows; this GPU's own memory, no multicast) into a ring of EM3D_RING plane slots,
// EM3D_RING - 2 planes ahead of the plane being computed, completing on one mbarrier per slot; the threads read E, H
// and the material ids from shared memory instead of holding loads in flight.  Boxes start at row j0 - 1 and at the
// 16-byte boundary at or before column k0 - 1 (moved left where a box would pass the row end): 40 floats or 48 ids
// wide; rows past the grid are filled with zeros by the copy and read only by threads whose results are discarded.
// Needs nz a multiple of 8 and at least 48.  Warp 0 (the halo row, which computes no E) issues the copies of plane
// i + EM3D_RING - 1 into the slot of plane i - 1 after the plane's barrier, when no thread reads that slot any more.
// Every wait is bounded (2 s): a block whose wait runs out sets *err, waits (bounded) for its own copies in flight and
// returns; material ids are clamped below n_ids, so a stale slot never indexes past the tables.  Arithmetic and
// results: em3d_fused_kernel's, bit for bit.
constexpr int EM3D_RING = 4;
constexpr int EM3D_WF = 40;   // floats per field box row (160 B)
constexpr int EM3D_WM = 48;   // ids per material box row (96 B)

// Tensor maps of one staged launch: E and H components of the field set read (boxes of TY + 1 and TY rows), ids.
struct Em3DMaps {
    CUtensorMap e[3], h[3], m;
};

__host__ __device__ constexpr int em3d_round128(int bytes) { return (bytes + 127) / 128 * 128; }

template <int TY>
struct Em3DStageLayout {   // byte offsets inside one ring slot, every box on a 128-byte boundary
    static constexpr int e_bytes = em3d_round128((TY + 1) * EM3D_WF * 4);
    static constexpr int h_bytes = em3d_round128(TY * EM3D_WF * 4);
    static constexpr int m_bytes = em3d_round128((TY + 1) * EM3D_WM * 2);
    static constexpr int e_off = 0, h_off = 3 * e_bytes, m_off = h_off + 3 * h_bytes;
    static constexpr int slot = m_off + m_bytes;
    static constexpr uint32_t tx = (uint32_t)((TY + 1) * EM3D_WF * 4 * 3 + TY * EM3D_WF * 4 * 3 + (TY + 1) * EM3D_WM * 2);
};

template <int TY>
__host__ __device__ constexpr size_t em3d_staged_smem() {
    return (size_t)Em3DStageLayout<TY>::slot * EM3D_RING + 2 * 2 * TY * 32 * sizeof(float) + EM3D_RING * sizeof(uint64_t);
}

__device__ __forceinline__ void em3d_tensor_g2s(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                                uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(tb_smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(tb_smem_addr(bar))
        : "memory");
}

// The seven copies of one plane into one slot (warp 0; lane 0 arms the barrier first).
template <int TY>
__device__ __forceinline__ void em3d_issue_plane(const Em3DMaps &maps, unsigned char *slot, uint64_t *bar, int plane,
                                                 int j_row0, int ca, int cam, int lane) {
    using L = Em3DStageLayout<TY>;
    if (lane == 0) tb_mbar_expect_tx(bar, L::tx);
    __syncwarp();
    if (lane < 3) em3d_tensor_g2s(slot + L::e_off + lane * L::e_bytes, &maps.e[lane], ca, j_row0, plane, bar);
    else if (lane < 6) em3d_tensor_g2s(slot + L::h_off + (lane - 3) * L::h_bytes, &maps.h[lane - 3], ca, j_row0, plane,
                                       bar);
    else if (lane == 6) em3d_tensor_g2s(slot + L::m_off, &maps.m, cam, j_row0, plane, bar);
}

template <int TY, int MINB>
__global__ void __launch_bounds__(EM3D_FZ * TY, MINB)
    em3d_staged_kernel(const Em3DParams p, const Em3DBox in, const __grid_constant__ Em3DMaps maps) {
    using L = Em3DStageLayout<TY>;
    extern __shared__ __align__(128) unsigned char em3d_smem[];
    float(*s_hz)[TY][EM3D_FZ] = reinterpret_cast<float(*)[TY][EM3D_FZ]>(em3d_smem + L::slot * EM3D_RING);
    float(*s_hx)[TY][EM3D_FZ] = reinterpret_cast<float(*)[TY][EM3D_FZ]>(
        em3d_smem + L::slot * EM3D_RING + 2 * TY * EM3D_FZ * sizeof(float));
    uint64_t *bar = reinterpret_cast<uint64_t *>(em3d_smem + L::slot * EM3D_RING + 4 * TY * EM3D_FZ * sizeof(float));
    const int lane = threadIdx.x, w = threadIdx.y;
    const int k_lo = in.k0 - 1 + (int)blockIdx.x * (EM3D_FZ - 1);   // this tile's first column (the halo)
    const int j_row0 = in.j0 - 1 + (int)blockIdx.y * (TY - 1);      // its first row (the halo)
    const int kk = k_lo + lane, jj = j_row0 + w;
    const bool e_thread = lane > 0 && w > 0;
    const bool emit = e_thread && kk < in.k1 && jj < in.j1;
    const int k = min(kk, in.k1 - 1), j = min(jj, in.j1 - 1);
    const int i_first = in.i0 + (int)blockIdx.z * p.x_chunk;
    const int i_last = min(in.i1, i_first + p.x_chunk);
    const int ca = min(k_lo & ~3, p.nz - EM3D_WF);     // 16-byte window starts
    const int cam = min(k_lo & ~7, p.nz - EM3D_WM);
    const int r = j - j_row0;                          // this thread's row in the staged tile
    const int c0 = k - ca, m_c = k - cam;              // its column in the field / id windows
    const size_t sx = (size_t)p.ny * p.nz;
    const int o = j * p.nz + k;
    const int base = i_first - 1;                      // plane of ring position 0
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int q = 0; q < EM3D_RING; ++q) tb_mbar_init(bar + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tb_fence_proxy_async();
    }
    __syncthreads();
    if (w == 0)
        for (int q = 0; q < EM3D_RING && base + q <= i_last; ++q)
            em3d_issue_plane<TY>(maps, em3d_smem + q * L::slot, bar + q, base + q, j_row0, ca, cam, lane);
    const int n_issued_max = i_last - base + 1;        // planes base .. i_last are staged
    float *__restrict__ oex = p.oex;
    float *__restrict__ oey = p.oey;
    float *__restrict__ oez = p.oez;
    float *__restrict__ ohx = p.ohx;
    float *__restrict__ ohy = p.ohy;
    float *__restrict__ ohz = p.ohz;
    const float ihy = p.ihy[j], ihz = p.ihz[k];
    const float iey = p.iey[j], iez = p.iez[k];
    const float wly = p.wly[j], wuy = p.wuy[j], wlz = p.wlz[k], wuz = p.wuz[k];
    const int32_t ryh = p.cpml[1].nr ? p.cpml[1].rm_h[j] : -1, rye = p.cpml[1].nr ? p.cpml[1].rm_e[j] : -1;
    const int32_t rzh = p.cpml[2].nr ? p.cpml[2].rm_h[k] : -1, rze = p.cpml[2].nr ? p.cpml[2].rm_e[k] : -1;
    const uint16_t id_max = (uint16_t)(p.n_ids - 1);
    bool ok = tb_mbar_wait(bar, 0);                    // plane base
    float hy_m = 0.0f, hz_m = 0.0f;
    int par = 0;
    for (int i = base; i < i_last; ++i) {
        const int q = i - base;
        const unsigned char *cur = em3d_smem + (q % EM3D_RING) * L::slot;
        const unsigned char *nxt = em3d_smem + ((q + 1) % EM3D_RING) * L::slot;
        ok = tb_mbar_wait(bar + (q + 1) % EM3D_RING, (uint32_t)(((q + 1) / EM3D_RING) & 1)) && ok;
        const float *ce0 = reinterpret_cast<const float *>(cur + L::e_off);
        const float *ce1 = reinterpret_cast<const float *>(cur + L::e_off + L::e_bytes);
        const float *ce2 = reinterpret_cast<const float *>(cur + L::e_off + 2 * L::e_bytes);
        const float *ch = reinterpret_cast<const float *>(cur + L::h_off);
        const uint16_t *cm = reinterpret_cast<const uint16_t *>(cur + L::m_off);
        const int at = r * EM3D_WF + c0, below = at + EM3D_WF;   // (row r, col c0) and the row after it
        const float ex0 = ce0[at], ey0 = ce1[at], ez0 = ce2[at];
        const float exy = ce0[below], ezy = ce2[below];
        const float exz = ce0[at + 1], eyz = ce1[at + 1];
        const float eyn = reinterpret_cast<const float *>(nxt + L::e_off + L::e_bytes)[at];
        const float ezn = reinterpret_cast<const float *>(nxt + L::e_off + 2 * L::e_bytes)[at];
        const float hx0 = ch[at], hy0 = ch[L::h_bytes / 4 + at], hz0 = ch[2 * (L::h_bytes / 4) + at];
        const int m_at = r * EM3D_WM + m_c;
        const uint16_t m0 = min(cm[m_at], id_max);
        const bool inside = i >= i_first;
        const bool store = emit && inside;
        float da, db;
        if (p.h_uniform) {
            da = p.da_u;
            db = p.db_u;
        } else {
            da = p.t_da[m0];
            db = p.t_db[m0];
        }
        const float ihx = p.ihx[i];
        const float dez_y = ezy - ez0, dey_z = eyz - ey0, dex_z = exz - ex0, dez_x = ezn - ez0;
        const float dey_x = eyn - ey0, dex_y = exy - ex0;
        float vhx = da * hx0 - db * (dez_y * ihy - dey_z * ihz);
        float vhy = da * hy0 - db * (dex_z * ihz - dez_x * ihx);
        float vhz = da * hz0 - db * (dey_x * ihx - dex_y * ihy);
        const int32_t rxh = p.cpml[0].nr ? p.cpml[0].rm_h[i] : -1;
        if (rxh >= 0) {   // x layers: H_y from E_z (+), H_z from E_y (-)
            const Em3DCpmlAxis &c = p.cpml[0];
            const size_t qq = (size_t)rxh * sx + o;
            const float f = c.b_h[rxh] * c.ph_first[qq] + c.g_h[rxh] * dez_x;
            const float g = c.b_h[rxh] * c.ph_second[qq] + c.g_h[rxh] * dey_x;
            if (store) {
                c.oph_first[qq] = f;
                c.oph_second[qq] = g;
            }
            vhy += db * f;
            vhz -= db * g;
        }
        if (ryh >= 0) {   // y layers: H_x from E_z (-), H_z from E_x (+)
            const Em3DCpmlAxis &c = p.cpml[1];
            const size_t qq = ((size_t)i * c.nr + ryh) * p.nz + k;
            const float f = c.b_h[ryh] * c.ph_first[qq] + c.g_h[ryh] * dez_y;
            const float g = c.b_h[ryh] * c.ph_second[qq] + c.g_h[ryh] * dex_y;
            if (store) {
                c.oph_first[qq] = f;
                c.oph_second[qq] = g;
            }
            vhx -= db * f;
            vhz += db * g;
        }
        if (rzh >= 0) {   // z layers: H_x from E_y (+), H_y from E_x (-)
            const Em3DCpmlAxis &c = p.cpml[2];
            const size_t qq = ((size_t)i * p.ny + j) * c.nr + rzh;
            const float f = c.b_h[rzh] * c.ph_first[qq] + c.g_h[rzh] * dey_z;
            const float g = c.b_h[rzh] * c.ph_second[qq] + c.g_h[rzh] * dex_z;
            if (store) {
                c.oph_first[qq] = f;
                c.oph_second[qq] = g;
            }
            vhx += db * f;
            vhy -= db * g;
        }
        if (store) {
            ohx[(size_t)i * sx + o] = vhx;
            ohy[(size_t)i * sx + o] = vhy;
            ohz[(size_t)i * sx + o] = vhz;
        }
        s_hz[par][w][lane] = vhz;
        s_hx[par][w][lane] = vhx;
        const float hy_z = __shfl_up_sync(0xffffffffu, vhy, 1);
        const float hx_z = __shfl_up_sync(0xffffffffu, vhx, 1);
        if (__syncthreads_or(!ok)) {   // a wait ran out somewhere in the block: stop, after the copies in flight
            if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(p.err, 1);
            if (w == 0)   // positions q + 1 .. q + 2 may still be in flight (q + 3 is issued after this barrier)
                for (int qq = q + 1; qq < min(n_issued_max, q + EM3D_RING - 1); ++qq)
                    tb_mbar_wait(bar + qq % EM3D_RING, (uint32_t)((qq / EM3D_RING) & 1));
            return;
        }
        // no thread reads the slot of plane i - 1 any more: it takes plane i + EM3D_RING - 1
        if (w == 0 && q >= 1 && i + EM3D_RING - 1 <= i_last) {
            tb_fence_proxy_async();
            em3d_issue_plane<TY>(maps, em3d_smem + ((q - 1) % EM3D_RING) * L::slot, bar + (q - 1) % EM3D_RING,
                                 i + EM3D_RING - 1, j_row0, ca, cam, lane);
        }
        if (e_thread && inside) {
            const float hz_y = s_hz[par][w - 1][lane];
            const float hx_y = s_hx[par][w - 1][lane];
            const float dhz_y = vhz - hz_y, dhy_z = vhy - hy_z, dhx_z = vhx - hx_z;
            const float dhz_x = vhz - hz_m, dhy_x = vhy - hy_m, dhx_y = vhx - hx_y;
            const uint16_t mx = min(reinterpret_cast<const uint16_t *>(nxt + L::m_off)[m_at], id_max);
            const uint16_t my = min(cm[m_at + EM3D_WM], id_max);
            const uint16_t mz = min(cm[m_at + 1], id_max);
            float ca_, cbx, cby, cbz;
            const float iex = p.iex[i];
            em3d_face_fast(p, 0, p.t_ex, m0, mx, p.wlx[i], p.wux[i], ca_, cbx);
            float vx = ca_ * ex0 + cbx * (dhz_y * iey - dhy_z * iez);
            em3d_face_fast(p, 1, p.t_ey, m0, my, wly, wuy, ca_, cby);
            float vy = ca_ * ey0 + cby * (dhx_z * iez - dhz_x * iex);
            em3d_face_fast(p, 2, p.t_ez, m0, mz, wlz, wuz, ca_, cbz);
            float vz = ca_ * ez0 + cbz * (dhy_x * iex - dhx_y * iey);
            const int32_t rxe = p.cpml[0].nr ? p.cpml[0].rm_e[i] : -1;
            if (rxe >= 0) {
                const Em3DCpmlAxis &c = p.cpml[0];
                const size_t qq = (size_t)rxe * sx + o;
                const float f = c.b_e[rxe] * c.pe_first[qq] + c.g_e[rxe] * dhz_x;
                const float g = c.b_e[rxe] * c.pe_second[qq] + c.g_e[rxe] * dhy_x;
                if (emit) {
                    c.ope_first[qq] = f;
                    c.ope_second[qq] = g;
                }
                vy -= cby * f;
                vz += cbz * g;
            }
            if (rye >= 0) {
                const Em3DCpmlAxis &c = p.cpml[1];
                const size_t qq = ((size_t)i * c.nr + rye) * p.nz + k;
                const float f = c.b_e[rye] * c.pe_first[qq] + c.g_e[rye] * dhz_y;
                const float g = c.b_e[rye] * c.pe_second[qq] + c.g_e[rye] * dhx_y;
                if (emit) {
                    c.ope_first[qq] = f;
                    c.ope_second[qq] = g;
                }
                vx += cbx * f;
                vz -= cbz * g;
            }
            if (rze >= 0) {
                const Em3DCpmlAxis &c = p.cpml[2];
                const size_t qq = ((size_t)i * p.ny + j) * c.nr + rze;
                const float f = c.b_e[rze] * c.pe_first[qq] + c.g_e[rze] * dhy_z;
                const float g = c.b_e[rze] * c.pe_second[qq] + c.g_e[rze] * dhx_z;
                if (emit) {
                    c.ope_first[qq] = f;
                    c.ope_second[qq] = g;
                }
                vx -= cbx * f;
                vy += cby * g;
            }
            for (int d = 0; d < p.n_dip; ++d) {
                if (p.dip_o[d] != o || p.dip_i[d] != i) continue;
                const float add = p.dip_values[d * p.values_stride + p.k_step] * p.dip_weight[d];
                if (p.dip_comp[d] == 0) vx = vx + add;
                else if (p.dip_comp[d] == 1) vy = vy + add;
                else vz = vz + add;
            }
            if (emit) {
                oex[(size_t)i * sx + o] = vx;
                oey[(size_t)i * sx + o] = vy;
                oez[(size_t)i * sx + o] = vz;
            }
        }
        hy_m = vhy;
        hz_m = vhz;
        par ^= 1;
    }
    // the last staged plane (i_last) was waited in the last iteration; nothing is in flight
}

// ---------------------------------------------------------------------------------------------------- running DFT
// One (E, H) pair of a flux plane (PlaneFlux3D, monitors3d.py:42-113): E = mean of the two layers across the plane,
// H on the plane, complex128 sums acc += ph * sample (the line kernels of physics/em/monitors.py:84-96).
struct Em3DFluxPair {
    int32_t e_comp, h_comp, normal, edge;
    int32_t o[3], n[3];                // box of the pair's samples (n[normal] = 1, o[normal] ignored)
    int32_t nf;
    int32_t phase_offset;              // offset of the pair's monitor in one sample's phase row (floats)
    double *e_acc, *h_acc;             // (nf, n cells) complex128 as double pairs
};

__global__ void em3d_flux_kernel(const Em3DFluxPair *pairs, const float *ex, const float *ey, const float *ez,
                                 const float *hx, const float *hy, const float *hz, int ny, int nz,
                                 const float *phases) {
    const Em3DFluxPair q = pairs[blockIdx.y];
    const int cells = q.n[0] * q.n[1] * q.n[2];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    int ijk[3] = {c / (q.n[1] * q.n[2]), (c / q.n[2]) % q.n[1], c % q.n[2]};
    for (int a = 0; a < 3; ++a) ijk[a] += q.o[a];
    ijk[q.normal] = q.edge - 1;
    const size_t lower = ((size_t)ijk[0] * ny + ijk[1]) * nz + ijk[2];
    const size_t step = q.normal == 0 ? (size_t)ny * nz : (q.normal == 1 ? (size_t)nz : 1);
    const float *e = q.e_comp == 0 ? ex : (q.e_comp == 1 ? ey : ez);
    const float *h = q.h_comp == 0 ? hx : (q.h_comp == 1 ? hy : hz);
    const double mean = 0.5 * ((double)e[lower] + (double)e[lower + step]);
    const double hv = (double)h[lower];
    const float *ph = phases + q.phase_offset;
    for (int f = 0; f < q.nf; ++f) {
        const double pr = (double)ph[2 * f], pi = (double)ph[2 * f + 1];
        double2 *ea = reinterpret_cast<double2 *>(q.e_acc) + (size_t)f * cells + c;
        double2 *ha = reinterpret_cast<double2 *>(q.h_acc) + (size_t)f * cells + c;
        double2 v = *ea;
        v.x = v.x + pr * mean;
        v.y = v.y + pi * mean;
        *ea = v;
        double2 w = *ha;
        w.x = w.x + pr * hv;
        w.y = w.y + pi * hv;
        *ha = w;
    }
}

// ---------------------------------------------------------------------------------------------------- setup
// da, db per material id (edge_coefficients, kernels3d.py:44-54): mu = mu_r mu0, loss = sigma_m dt / (2 mu).
__global__ void em3d_h_tables_kernel(const float *t_mu, const float *t_sm, int n, float dt, float *t_da,
                                     float *t_db) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const float mu = t_mu[m] * 1.2566370614e-6f;
    const float loss = t_sm[m] * dt / (2.0f * mu);
    const float den = 1.0f + loss;
    t_da[m] = (1.0f - loss) / den;
    t_db[m] = (dt / mu) / den;
}

// cb of E component comp on the face of cell (i, j, k) (box_face_cb_3d for a one-cell box, kernels3d.py:745-779).
__global__ void em3d_face_cb_kernel(const Em3DParams p, int comp, int i, int j, int k, float *out) {
    const size_t sy = (size_t)p.nz, sx = (size_t)p.ny * p.nz;
    const size_t idx = (size_t)i * sx + (size_t)j * sy + k;
    size_t b;
    float wa, wb;
    const float *t;
    if (comp == 0) {
        b = i + 1 < p.nx ? idx + sx : (p.px ? idx - (size_t)(p.nx - 1) * sx : idx);
        wa = p.wlx[i];
        wb = p.wux[i];
        t = p.t_ex;
    } else if (comp == 1) {
        b = j + 1 < p.ny ? idx + sy : (p.py ? idx - (size_t)(p.ny - 1) * sy : idx);
        wa = p.wly[j];
        wb = p.wuy[j];
        t = p.t_ey;
    } else {
        b = k + 1 < p.nz ? idx + 1 : (p.pz ? idx - (size_t)(p.nz - 1) : idx);
        wa = p.wlz[k];
        wb = p.wuz[k];
        t = p.t_ez;
    }
    float ca, cb;
    em3d_face(p, t, p.mat[idx], p.mat[b], wa, wb, ca, cb);
    *out = cb;
}

// ca, cb of the faces between two cells of the same material id, per E component, with the uniform shares 0.5 / 0.5
// (the values em3d_face gives those faces; out: per component ca then cb, n_ids each).
__global__ void em3d_same_tables_kernel(const Em3DParams p, float *out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= p.n_ids) return;
    const float *t[3] = {p.t_ex, p.t_ey, p.t_ez};
    for (int comp = 0; comp < 3; ++comp) {
        float ca, cb;
        em3d_face(p, t[comp], (uint16_t)m, (uint16_t)m, 0.5f, 0.5f, ca, cb);
        out[(2 * comp) * p.n_ids + m] = ca;
        out[(2 * comp + 1) * p.n_ids + m] = cb;
    }
}
