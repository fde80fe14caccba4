/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Nothing in the product (opensol_b200/) links, loads or calls this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the reference results are compared with.
 *
 * Plain-C restatement of the two fused field updates of open_sol's 3D Yee engine (em_fdtd_3d, Cartesian grid, one
 * real field set, single-precision storage and arithmetic) on the CPU:
 *
 *   H update: open_sol/physics/em3d/kernels3d.py:335-392 (update_h_3d; numpy twin _update_h_host :451-463, CPML
 *             rows _cpml_h_rows :422-441), edge coefficients da / db of the lower cell's material id (:44-54, numpy
 *             _edge_tables :150-155);
 *   E update: kernels3d.py:538-609 (update_e_3d; numpy twin _update_e_host :640-661, CPML rows _cpml_e_rows
 *             :612-637), face coefficients ca / cb = the width-weighted mean of the two cells' table values with the
 *             PEC rules (:61-82, numpy _face_coefficients :158-185).
 *
 * Built twice: ORACLE_REAL = float (the single-precision engine's arithmetic) and ORACLE_REAL = double (the same
 * updates in float64, the 3D double-precision run the float32 results' error is stated against; open_sol's 3D engine
 * has no double stepper of its own).
 *
 * Every float32 operation is evaluated in the reference's order with no contraction (-ffp-contract=off), so the
 * results equal the reference's numpy twins bit for bit.  The reference's default numba twins compute da / db and
 * ca / cb in float64 and so differ from both in the last bits; the tests compare against them within a tolerance.
 * On a Cartesian grid the reference's radial factors are exactly 1 and are left out (a multiply by 1.0f is exact).
 * A non-periodic axis: the hi neighbour of the last row wraps (its inverse spacing is 0, kernels3d.py:117-125,
 * engine3d.py:191-196); the missing lo H of row 0 is 0 (the numpy twin's _lo_difference keeps the sample itself,
 * kernels3d.py:128-139).
 */
#include <stdint.h>
#include <stddef.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;
#define ORACLE_IS_FLOAT (sizeof(real) == sizeof(float))
/* vacuum constants rounded once to the arithmetic type (the float build uses the float literals) */
#define EPS0F (ORACLE_IS_FLOAT ? (real)8.8541878128e-12f : (real)8.8541878128e-12)
#define MU0F (ORACLE_IS_FLOAT ? (real)1.2566370614e-6f : (real)1.2566370614e-6)

typedef struct {
    int32_t nx, ny, nz;
    int32_t px, py, pz;                       /* periodic axes */
    real *ex, *ey, *ez, *hx, *hy, *hz;       /* (nx, ny, nz), z contiguous */
    const uint16_t *mat;                      /* material id per cell */
    const real *t_ex, *t_ey, *t_ez;          /* eps_r per id and E component (PEC id: -1) */
    const real *t_sig, *t_mu, *t_sm;         /* sigma_e, mu_r, sigma_m per id */
    const real *iex, *iey, *iez;             /* kappa-folded 1 / cell width (E curls) */
    const real *ihx, *ihy, *ihz;             /* kappa-folded 1 / hi-face spacing (H curls; last row 0 if open) */
    const real *wlx, *wux, *wly, *wuy, *wlz, *wuz;   /* hi-face shares of the lower / upper cell */
    real dt;
    /* CPML per axis (x, y, z) and kind: row map (grid row -> psi row or -1), b, gain per psi row, two psi arrays of
     * the axis' first and second component; nr = psi rows of the axis (0: no CPML on it) */
    int32_t nr[3];
    const int32_t *rm_h[3], *rm_e[3];
    const real *b_h[3], *g_h[3], *b_e[3], *g_e[3];
    real *ph_first[3], *ph_second[3], *pe_first[3], *pe_second[3];
} OracleEM3D;

static inline real wrapped(real v) { return 1.0f * v + 0.0f * v; }   /* c F + s F_partner with c = 1, s = 0 */

static inline real psi_step(real *psi, size_t p, real b, real g, real difference) {
    const real value = b * psi[p] + g * difference;
    psi[p] = value;
    return value;
}

static inline size_t psi_index(int axis, int32_t r, int i, int j, int k, int ny, int nz, const int32_t *nr) {
    if (axis == 0) return ((size_t)r * ny + j) * nz + k;
    if (axis == 1) return ((size_t)i * nr[1] + r) * nz + k;
    return ((size_t)i * ny + j) * nr[2] + r;
}

void oracle_em3d_update_h(OracleEM3D *s) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const size_t sy = (size_t)nz, sx = (size_t)ny * nz;
    const real dt = s->dt;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        const int wx = i + 1 == nx, ip = wx ? 0 : i + 1;
        const int32_t rx = s->nr[0] ? s->rm_h[0][i] : -1;
        for (int j = 0; j < ny; ++j) {
            const int wy = j + 1 == ny, jp = wy ? 0 : j + 1;
            const int32_t ry = s->nr[1] ? s->rm_h[1][j] : -1;
            for (int k = 0; k < nz; ++k) {
                const int wz = k + 1 == nz, kp = wz ? 0 : k + 1;
                const int32_t rz = s->nr[2] ? s->rm_h[2][k] : -1;
                const size_t idx = (size_t)i * sx + (size_t)j * sy + k;
                const uint16_t m = s->mat[idx];
                const real mu = s->t_mu[m] * MU0F;
                const real loss = s->t_sm[m] * dt / (2.0f * mu);
                const real den = 1.0f + loss;
                const real da = (1.0f - loss) / den;
                const real db = (dt / mu) / den;
                const real ex0 = s->ex[idx], ey0 = s->ey[idx], ez0 = s->ez[idx];
                const size_t ixp = (size_t)ip * sx + (size_t)j * sy + k;
                const size_t iyp = (size_t)i * sx + (size_t)jp * sy + k;
                const size_t izp = (size_t)i * sx + (size_t)j * sy + kp;
                const real ex_y = wy ? wrapped(s->ex[iyp]) : s->ex[iyp];
                const real ex_z = wz ? wrapped(s->ex[izp]) : s->ex[izp];
                const real ey_x = wx ? wrapped(s->ey[ixp]) : s->ey[ixp];
                const real ey_z = wz ? wrapped(s->ey[izp]) : s->ey[izp];
                const real ez_x = wx ? wrapped(s->ez[ixp]) : s->ez[ixp];
                const real ez_y = wy ? wrapped(s->ez[iyp]) : s->ez[iyp];
                const real dez_y = ez_y - ez0, dey_z = ey_z - ey0, dex_z = ex_z - ex0, dez_x = ez_x - ez0;
                const real dey_x = ey_x - ey0, dex_y = ex_y - ex0;
                real vx = da * s->hx[idx] - db * (dez_y * s->ihy[j] - dey_z * s->ihz[k]);
                real vy = da * s->hy[idx] - db * (dex_z * s->ihz[k] - dez_x * s->ihx[i]);
                real vz = da * s->hz[idx] - db * (dey_x * s->ihx[i] - dex_y * s->ihy[j]);
                if (rx >= 0) {   /* x layers: H_y from E_z (+), H_z from E_y (-) */
                    const size_t p = psi_index(0, rx, i, j, k, ny, nz, s->nr);
                    vy += db * psi_step(s->ph_first[0], p, s->b_h[0][rx], s->g_h[0][rx], dez_x);
                    vz -= db * psi_step(s->ph_second[0], p, s->b_h[0][rx], s->g_h[0][rx], dey_x);
                }
                if (ry >= 0) {   /* y layers: H_x from E_z (-), H_z from E_x (+) */
                    const size_t p = psi_index(1, ry, i, j, k, ny, nz, s->nr);
                    vx -= db * psi_step(s->ph_first[1], p, s->b_h[1][ry], s->g_h[1][ry], dez_y);
                    vz += db * psi_step(s->ph_second[1], p, s->b_h[1][ry], s->g_h[1][ry], dex_y);
                }
                if (rz >= 0) {   /* z layers: H_x from E_y (+), H_y from E_x (-) */
                    const size_t p = psi_index(2, rz, i, j, k, ny, nz, s->nr);
                    vx += db * psi_step(s->ph_first[2], p, s->b_h[2][rz], s->g_h[2][rz], dey_z);
                    vy -= db * psi_step(s->ph_second[2], p, s->b_h[2][rz], s->g_h[2][rz], dex_z);
                }
                s->hx[idx] = vx;
                s->hy[idx] = vy;
                s->hz[idx] = vz;
            }
        }
    }
}

/* ca, cb of the face between cells a and b (b = a on the last row of a non-periodic axis). */
static inline void face_coefficients(const OracleEM3D *s, const real *t_eps, size_t a, size_t b, real wa, real wb,
                                     real *ca, real *cb) {
    const uint16_t ia = s->mat[a], ib = s->mat[b];
    real ea = t_eps[ia], eb = t_eps[ib];
    real sa = s->t_sig[ia], sb = s->t_sig[ib];
    if (ea < 0.0f && eb < 0.0f) {
        *ca = 0.0f;
        *cb = 0.0f;
        return;
    }
    if (ea < 0.0f) {
        ea = eb;
        sa = sb;
    } else if (eb < 0.0f) {
        eb = ea;
        sb = sa;
    }
    const real eps = (wa * ea + wb * eb) * EPS0F;
    const real sig = wa * sa + wb * sb;
    const real loss = sig * s->dt / (2.0f * eps);
    const real den = 1.0f + loss;
    *ca = (1.0f - loss) / den;
    *cb = (s->dt / eps) / den;
}

/* F0 - F[lo neighbour] along an axis: the wrapped sample on a periodic axis, nothing below row 0 otherwise. */
static inline real lo_difference(real f0, const real *f, size_t lo_index, int first_row, int periodic) {
    if (!first_row) return f0 - f[lo_index];
    return periodic ? f0 - wrapped(f[lo_index]) : f0;
}

void oracle_em3d_update_e(OracleEM3D *s) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const size_t sy = (size_t)nz, sx = (size_t)ny * nz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        const int im = i == 0 ? nx - 1 : i - 1;
        const size_t bx = i + 1 < nx ? sx : (s->px ? (size_t)0 - (size_t)(nx - 1) * sx : 0);
        const int32_t rx = s->nr[0] ? s->rm_e[0][i] : -1;
        for (int j = 0; j < ny; ++j) {
            const int jm = j == 0 ? ny - 1 : j - 1;
            const size_t by = j + 1 < ny ? sy : (s->py ? (size_t)0 - (size_t)(ny - 1) * sy : 0);
            const int32_t ry = s->nr[1] ? s->rm_e[1][j] : -1;
            for (int k = 0; k < nz; ++k) {
                const int km = k == 0 ? nz - 1 : k - 1;
                const size_t bz = k + 1 < nz ? 1 : (s->pz ? (size_t)0 - (size_t)(nz - 1) : 0);
                const int32_t rz = s->nr[2] ? s->rm_e[2][k] : -1;
                const size_t idx = (size_t)i * sx + (size_t)j * sy + k;
                const size_t ixm = (size_t)im * sx + (size_t)j * sy + k;
                const size_t iym = (size_t)i * sx + (size_t)jm * sy + k;
                const size_t izm = (size_t)i * sx + (size_t)j * sy + km;
                const real hx0 = s->hx[idx], hy0 = s->hy[idx], hz0 = s->hz[idx];
                const real dhz_y = lo_difference(hz0, s->hz, iym, j == 0, s->py);
                const real dhy_z = lo_difference(hy0, s->hy, izm, k == 0, s->pz);
                const real dhx_z = lo_difference(hx0, s->hx, izm, k == 0, s->pz);
                const real dhz_x = lo_difference(hz0, s->hz, ixm, i == 0, s->px);
                const real dhy_x = lo_difference(hy0, s->hy, ixm, i == 0, s->px);
                const real dhx_y = lo_difference(hx0, s->hx, iym, j == 0, s->py);
                real ca, cbx, cby, cbz;
                face_coefficients(s, s->t_ex, idx, idx + bx, s->wlx[i], s->wux[i], &ca, &cbx);
                real vx = ca * s->ex[idx] + cbx * (dhz_y * s->iey[j] - dhy_z * s->iez[k]);
                face_coefficients(s, s->t_ey, idx, idx + by, s->wly[j], s->wuy[j], &ca, &cby);
                real vy = ca * s->ey[idx] + cby * (dhx_z * s->iez[k] - dhz_x * s->iex[i]);
                face_coefficients(s, s->t_ez, idx, idx + bz, s->wlz[k], s->wuz[k], &ca, &cbz);
                real vz = ca * s->ez[idx] + cbz * (dhy_x * s->iex[i] - dhx_y * s->iey[j]);
                if (rx >= 0) {   /* x layers: E_y from H_z (-), E_z from H_y (+) */
                    const size_t p = psi_index(0, rx, i, j, k, ny, nz, s->nr);
                    vy -= cby * psi_step(s->pe_first[0], p, s->b_e[0][rx], s->g_e[0][rx], dhz_x);
                    vz += cbz * psi_step(s->pe_second[0], p, s->b_e[0][rx], s->g_e[0][rx], dhy_x);
                }
                if (ry >= 0) {   /* y layers: E_x from H_z (+), E_z from H_x (-) */
                    const size_t p = psi_index(1, ry, i, j, k, ny, nz, s->nr);
                    vx += cbx * psi_step(s->pe_first[1], p, s->b_e[1][ry], s->g_e[1][ry], dhz_y);
                    vz -= cbz * psi_step(s->pe_second[1], p, s->b_e[1][ry], s->g_e[1][ry], dhx_y);
                }
                if (rz >= 0) {   /* z layers: E_x from H_y (-), E_y from H_x (+) */
                    const size_t p = psi_index(2, rz, i, j, k, ny, nz, s->nr);
                    vx -= cbx * psi_step(s->pe_first[2], p, s->b_e[2][rz], s->g_e[2][rz], dhy_z);
                    vy += cby * psi_step(s->pe_second[2], p, s->b_e[2][rz], s->g_e[2][rz], dhx_z);
                }
                s->ex[idx] = vx;
                s->ey[idx] = vy;
                s->ez[idx] = vz;
            }
        }
    }
}

/* cb of E component comp on the face of one cell (box_face_cb_3d, kernels3d.py:745-779, for a 1-cell box). */
real oracle_em3d_face_cb(const OracleEM3D *s, int comp, int i, int j, int k) {
    const size_t sy = (size_t)s->nz, sx = (size_t)s->ny * s->nz;
    const size_t idx = (size_t)i * sx + (size_t)j * sy + k;
    real ca, cb;
    if (comp == 0) {
        const size_t b = i + 1 < s->nx ? idx + sx : (s->px ? idx - (size_t)(s->nx - 1) * sx : idx);
        face_coefficients(s, s->t_ex, idx, b, s->wlx[i], s->wux[i], &ca, &cb);
    } else if (comp == 1) {
        const size_t b = j + 1 < s->ny ? idx + sy : (s->py ? idx - (size_t)(s->ny - 1) * sy : idx);
        face_coefficients(s, s->t_ey, idx, b, s->wly[j], s->wuy[j], &ca, &cb);
    } else {
        const size_t b = k + 1 < s->nz ? idx + 1 : (s->pz ? idx - (size_t)(s->nz - 1) : idx);
        face_coefficients(s, s->t_ez, idx, b, s->wlz[k], s->wuz[k], &ca, &cb);
    }
    return cb;
}
