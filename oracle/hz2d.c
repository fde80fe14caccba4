/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Nothing in the product (opensol_b200/) links, loads or calls this file;
 * only tests/ do, as the reference results are compared with.
 *
 * Plain-C restatement of open_sol's 2D H_z-polarisation FDTD time step on the CPU (H_z at cell centres, E_x on the
 * hi-y faces, E_y on the hi-x faces), float32 or float64 (-DORACLE_REAL=double), in the reference CPU twins' order:
 *
 *   H_z Yee update: open_sol/physics/em/solvers/fdtd_hz_2d_kernels.py:28-91 (update_hz_kernel and its numpy twin):
 *       curl = (E_x[j] - E_x[j-1]) iye[j] - (E_y[i] - E_y[i-1]) ixe[i]; the lo sample below row 0 wraps on a
 *       periodic axis (E * 1 - E * 0) and is 0 otherwise; H_z = da H_z + db curl;
 *   H_z CPML (CPMLSided.apply_hz, physics/em/boundaries.py:764-767, 732-750, 27-37): cell-centre rows, psi = b psi +
 *       a (E[r] - E[r-1]) inv with E_y on the x sides (correction sign -1) and E_x on the y sides (+1), H_z += sign
 *       db psi;
 *   E_x / E_y Yee update (update_exy_kernel, fdtd_hz_2d_kernels.py:94-174): E_x = ca_x E_x + cb_x (H_z[j+1] - H_z)
 *       iyh[j], E_y = ca_y E_y - cb_y (H_z[i+1] - H_z) ixh[i]; the last face of an open axis is never updated, of a
 *       periodic one it reads H_z * 1 + H_z * 0 of row 0;
 *   E CPML (CPMLSided.apply_exy, boundaries.py:769-772): hi-face rows, psi = b psi + a (H_z[r+1] - H_z[r]) inv,
 *       E_y += -cb_y psi on the x sides, E_x += cb_x psi on the y sides;
 *   sheet injection (TangentialSheetCurrentSource.inject_electric, physics/em/sources.py:469-480): E_x (axis 'x') or
 *       E_y (axis 'y') += FP32(amp s(t + dt/2)) * profile on the line's faces;
 *   DFT sample (FluxMonitor 'hz', physics/em/monitors.py:350-362): E_y (normal x) or E_x (normal y) and H_z on the line.
 */
#include <stdint.h>
#include <stddef.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

enum { SIDE_XLO = 0, SIDE_XHI = 1, SIDE_YLO = 2, SIDE_YHI = 3 };

typedef struct {
    int32_t nx, ny, periodic_x, periodic_y;
    real *hz, *ex, *ey;
    const real *ca_x, *cb_x, *ca_y, *cb_y, *da, *db;
    const real *inv_dx_e, *inv_dx_h, *inv_dy_e, *inv_dy_h;
    int32_t npml;
    int32_t cpml_active[4];
    const real *b_e[4], *a_e[4], *inv_e[4];
    const real *b_h[4], *a_h[4], *inv_h[4];
    real *psi_e[4], *psi_h[4];
} OracleHz2D;

typedef struct {
    int32_t axis, position, lo, hi;
    const float *profile;
    const float *values;
} OracleLineHz;

typedef struct {
    int32_t normal_axis, position, lo, hi, nf;
    double *e_acc, *h_acc;
    const float *phases;
    int64_t first_sample, n_samples;
} OracleFluxHz;

/* TFSFSourceHz (open_sol/physics/em/sources.py:55-70,352-379): the incident line holds E_y (aux_ey, hi faces) and
 * H_z (aux_hz, centres); coef_h[0..1] act on H_z rows x0 / x1 - 1, coef_e on E_y rows x0 - 1 / x1 - 1 and E_x columns
 * y0 - 1 / y1 - 1. */
typedef struct {
    int32_t x0, x1, y0, y1, aux_x0, aux_n, source_index;
    real coef_h[4], coef_e[4], mur_lo, mur_hi;
    real *aux_ey, *aux_hz;
    const real *aux_coef_h, *aux_coef_e;
    const float *values;
} OracleTfsfHz;

/* A Drude / Lorentz pole on one E face set (fdtd_hz_2d.py:441-472,547-570): comp 0 = E_x (hi-y faces), 1 = E_y
 * (hi-x faces); drive = the pole's drive coefficient times the face weight (the face average of its cell mask) on
 * the box, so faces outside the medium keep J = 0 / P = 0. */
typedef struct {
    int32_t kind, comp;                       /* kind 0 Drude, 1 Lorentz */
    int32_t i0, i1, j0, j1;                   /* face box */
    real damping, restoring;
    const real *drive;                        /* (box) drive x face weight */
    real *a, *b;                              /* Drude: a = J; Lorentz: a = P, b = dP (box) */
} OraclePoleHz;

/* _pole_updates (fdtd_hz_2d.py:286-309) from E^n: every Drude face set in add order, then every Lorentz one. */
static void hz_poles_update(const OracleHz2D *s, int32_t n_poles, const OraclePoleHz *poles)
{
    const size_t ny = (size_t)s->ny;
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < n_poles; ++q) {
            const OraclePoleHz *p = &poles[q];
            if (p->kind != pass) continue;
            const real *e = p->comp == 0 ? s->ex : s->ey;
            const int w = p->j1 - p->j0;
            for (int i = p->i0; i < p->i1; ++i)
                for (int j = p->j0; j < p->j1; ++j) {
                    const size_t t = (size_t)(i - p->i0) * w + (j - p->j0), g = (size_t)i * ny + j;
                    if (p->kind == 0) {
                        p->a[t] += p->damping * p->a[t] + p->drive[t] * e[g];
                    } else {
                        p->b[t] += p->damping * p->b[t] - p->restoring * p->a[t] + p->drive[t] * e[g];
                        p->a[t] += p->b[t];
                    }
                }
        }
}

/* _pole_corrections (fdtd_hz_2d.py:311-325): E -= cb J per Drude face set, then E -= cb inv_dt dP per Lorentz one,
 * cb of the face set (cb_x / cb_y). */
static void hz_poles_correct(const OracleHz2D *s, int32_t n_poles, const OraclePoleHz *poles, real inv_dt)
{
    const size_t ny = (size_t)s->ny;
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < n_poles; ++q) {
            const OraclePoleHz *p = &poles[q];
            if (p->kind != pass) continue;
            real *e = p->comp == 0 ? s->ex : s->ey;
            const real *cb = p->comp == 0 ? s->cb_x : s->cb_y;
            const int w = p->j1 - p->j0;
            for (int i = p->i0; i < p->i1; ++i)
                for (int j = p->j0; j < p->j1; ++j) {
                    const size_t t = (size_t)(i - p->i0) * w + (j - p->j0), g = (size_t)i * ny + j;
                    if (p->kind == 0) e[g] -= cb[g] * p->a[t];
                    else e[g] -= cb[g] * inv_dt * p->b[t];
                }
        }
}

/* inject_magnetic: H_z corrections from the incident E_y, then aux_hz[k] += coef[k - 1] (aux_ey[k] - aux_ey[k - 1]). */
static void tfsf_h(const OracleHz2D *s, const OracleTfsfHz *t)
{
    const size_t ny = (size_t)s->ny;
    for (int j = t->y0; j < t->y1; ++j) {
        s->hz[(size_t)t->x0 * ny + j] += t->coef_h[0] * t->aux_ey[t->aux_x0 - 1];
        s->hz[(size_t)(t->x1 - 1) * ny + j] -= t->coef_h[1] * t->aux_ey[t->aux_x0 + (t->x1 - 1 - t->x0)];
    }
    for (int k = 1; k < t->aux_n; ++k) t->aux_hz[k] += t->aux_coef_h[k - 1] * (t->aux_ey[k] - t->aux_ey[k - 1]);
}

/* inject_electric: E_y / E_x corrections from the incident H_z, then the incident E_y update (aux_ey[a] += ce[a]
 * (aux_hz[a + 1] - aux_hz[a])), the soft source and the Mur ends. */
static void tfsf_e(const OracleHz2D *s, const OracleTfsfHz *t, int64_t k)
{
    const size_t ny = (size_t)s->ny;
    for (int j = t->y0; j < t->y1; ++j) {
        s->ey[(size_t)(t->x0 - 1) * ny + j] += t->coef_e[0] * t->aux_hz[t->aux_x0];
        s->ey[(size_t)(t->x1 - 1) * ny + j] -= t->coef_e[1] * t->aux_hz[t->aux_x0 + (t->x1 - 1 - t->x0)];
    }
    for (int i = t->x0; i < t->x1; ++i) {
        const real incident = t->aux_hz[t->aux_x0 + (i - t->x0)];
        s->ex[(size_t)i * ny + (t->y0 - 1)] -= t->coef_e[2] * incident;
        s->ex[(size_t)i * ny + (t->y1 - 1)] += t->coef_e[3] * incident;
    }
    const int n = t->aux_n;
    const real old0 = t->aux_ey[0], old1 = t->aux_ey[1], old2 = t->aux_ey[n - 2], old3 = t->aux_ey[n - 1];
    for (int a = 1; a < n - 1; ++a) t->aux_ey[a] += t->aux_coef_e[a] * (t->aux_hz[a + 1] - t->aux_hz[a]);
    t->aux_ey[t->source_index] += (real)t->values[k];
    t->aux_ey[0] = old1 + t->mur_lo * (t->aux_ey[1] - old0);
    t->aux_ey[n - 1] = old2 + t->mur_hi * (t->aux_ey[n - 2] - old3);
}

static void update_hz(const OracleHz2D *s) {
    const int nx = s->nx, ny = s->ny;
    const real one = (real)1, zero = (real)0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            const size_t idx = (size_t)i * ny + j;
            real curl;
            if (j >= 1) {
                curl = (s->ex[idx] - s->ex[idx - 1]) * s->inv_dy_e[j];
            } else if (s->periodic_y) {
                const size_t w = idx + ny - 1;
                curl = (s->ex[idx] - (s->ex[w] * one - s->ex[w] * zero)) * s->inv_dy_e[j];
            } else {
                curl = s->ex[idx] * s->inv_dy_e[j];
            }
            if (i >= 1) {
                curl -= (s->ey[idx] - s->ey[idx - ny]) * s->inv_dx_e[i];
            } else if (s->periodic_x) {
                const size_t w = (size_t)(nx - 1) * ny + j;
                curl -= (s->ey[idx] - (s->ey[w] * one - s->ey[w] * zero)) * s->inv_dx_e[i];
            } else {
                curl -= s->ey[idx] * s->inv_dx_e[i];
            }
            s->hz[idx] = s->da[idx] * s->hz[idx] + s->db[idx] * curl;
        }
    }
}

static void update_exy(const OracleHz2D *s) {
    const int nx = s->nx, ny = s->ny;
    const real one = (real)1, zero = (real)0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            const size_t idx = (size_t)i * ny + j;
            const real h = s->hz[idx];
            if (j < ny - 1) {
                s->ex[idx] = s->ca_x[idx] * s->ex[idx] + s->cb_x[idx] * (s->hz[idx + 1] - h) * s->inv_dy_h[j];
            } else if (s->periodic_y) {
                const size_t w = (size_t)i * ny;
                s->ex[idx] = s->ca_x[idx] * s->ex[idx]
                             + s->cb_x[idx] * (s->hz[w] * one + s->hz[w] * zero - h) * s->inv_dy_h[j];
            }
            if (i < nx - 1) {
                s->ey[idx] = s->ca_y[idx] * s->ey[idx] - s->cb_y[idx] * (s->hz[idx + ny] - h) * s->inv_dx_h[i];
            } else if (s->periodic_x) {
                const size_t w = (size_t)j;
                s->ey[idx] = s->ca_y[idx] * s->ey[idx]
                             - s->cb_y[idx] * (s->hz[w] * one + s->hz[w] * zero - h) * s->inv_dx_h[i];
            }
        }
    }
}

static int side_first_row(int side, int kind_e, int n, int npml) {
    const int lo = (side == SIDE_XLO || side == SIDE_YLO);
    if (lo) return kind_e ? 1 : 0;
    return n - npml - 1;
}

/* One side's psi update and correction.  kind_e: the cell-centre rows on H_z (source E_y on x sides, E_x on y sides,
 * coefficient db, sign -1 on x / +1 on y, f_hi = src[r], f_lo = src[r - 1]); otherwise the hi-face rows on E (source
 * H_z, field E_y with -cb_y on x sides, E_x with +cb_x on y sides, f_hi = src[r + 1], f_lo = src[r]). */
static void cpml_side(const OracleHz2D *s, int side, int kind_e) {
    const int nx = s->nx, ny = s->ny, npml = s->npml;
    const int x_side = (side == SIDE_XLO || side == SIDE_XHI);
    const real sign = x_side ? (real)-1 : (real)1;
    const real *b = kind_e ? s->b_e[side] : s->b_h[side];
    const real *a = kind_e ? s->a_e[side] : s->a_h[side];
    const real *inv = kind_e ? s->inv_e[side] : s->inv_h[side];
    real *psi = kind_e ? s->psi_e[side] : s->psi_h[side];
    const real *src = kind_e ? (x_side ? s->ey : s->ex) : s->hz;
    real *field = kind_e ? s->hz : (x_side ? s->ey : s->ex);
    const real *coef = kind_e ? s->db : (x_side ? s->cb_y : s->cb_x);
    const int first = side_first_row(side, kind_e, x_side ? nx : ny, npml);
    const int up = kind_e ? 0 : 1, dn = kind_e ? -1 : 0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < (x_side ? npml : nx); ++i) {
        for (int j = 0; j < (x_side ? ny : npml); ++j) {
            const int k = x_side ? i : j;
            const int r = first + k;
            size_t cell, hi_cell, lo_cell;
            if (x_side) {
                cell = (size_t)r * ny + j;
                hi_cell = (size_t)(r + up) * ny + j;
                lo_cell = (size_t)(r + dn) * ny + j;
            } else {
                cell = (size_t)i * ny + r;
                hi_cell = (size_t)i * ny + (r + up);
                lo_cell = (size_t)i * ny + (r + dn);
            }
            const size_t p = x_side ? (size_t)k * ny + j : (size_t)i * npml + k;
            real q = psi[p] * b[k];
            q += a[k] * (src[hi_cell] - src[lo_cell]) * inv[k];
            psi[p] = q;
            field[cell] += sign * coef[cell] * q;
        }
    }
}

static void inject_line(const OracleHz2D *s, const OracleLineHz *line, int64_t k) {
    const float value = line->values[k];
    if (value == 0.0f) return;
    real *target = line->axis == 0 ? s->ex : s->ey;
    for (int c = line->lo; c < line->hi; ++c) {
        const size_t cell = line->axis == 0 ? (size_t)c * s->ny + line->position
                                            : (size_t)line->position * s->ny + c;
        const float add = value * line->profile[c - line->lo];
        target[cell] += (real)add;
    }
}

static void accumulate_flux(const OracleHz2D *s, OracleFluxHz *m, int64_t sample) {
    const int n = m->hi - m->lo;
    const float *ph = m->phases + (size_t)(sample - m->first_sample) * m->nf * 2;
    const real *e = m->normal_axis == 0 ? s->ey : s->ex;
    for (int f = 0; f < m->nf; ++f) {
        const double pr = (double)ph[2 * f], pi = (double)ph[2 * f + 1];
        for (int c = 0; c < n; ++c) {
            const size_t cell = m->normal_axis == 0 ? (size_t)m->position * s->ny + (m->lo + c)
                                                    : (size_t)(m->lo + c) * s->ny + m->position;
            const double ev = (double)e[cell], hv = (double)s->hz[cell];
            const size_t a = ((size_t)f * n + c) * 2;
            m->e_acc[a] += pr * ev;
            m->e_acc[a + 1] += pi * ev;
            m->h_acc[a] += pr * hv;
            m->h_acc[a + 1] += pi * hv;
        }
    }
}

/* One chunk of FDTDEngine2D_Hz.advance (fdtd_hz_2d.py:143-198, 233-284): H_z + CPML, TFSF H side, pole updates from
 * E^n, E_x / E_y + CPML, pole corrections, sheet sources, TFSF E side, flux samples. */
int oracle_hz2d_advance_full(OracleHz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines,
                             const OracleLineHz *lines, int32_t n_monitors, OracleFluxHz *monitors,
                             int64_t sample_interval, int32_t n_tfsf, const OracleTfsfHz *tfsf, int32_t n_poles,
                             const OraclePoleHz *poles, real inv_dt) {
    for (int64_t k = 0; k < n_steps; ++k) {
        update_hz(s);
        for (int side = 0; side < 4; ++side)
            if (s->cpml_active[side]) cpml_side(s, side, 1);
        for (int b = 0; b < n_tfsf; ++b) tfsf_h(s, &tfsf[b]);
        if (n_poles) hz_poles_update(s, n_poles, poles);
        update_exy(s);
        for (int side = 0; side < 4; ++side)
            if (s->cpml_active[side]) cpml_side(s, side, 0);
        if (n_poles) hz_poles_correct(s, n_poles, poles, inv_dt);
        for (int l = 0; l < n_lines; ++l) inject_line(s, &lines[l], k);
        for (int b = 0; b < n_tfsf; ++b) tfsf_e(s, &tfsf[b], k);
        const int64_t n_step = step0 + k + 1;
        if (n_monitors > 0 && n_step % sample_interval == 0) {
            const int64_t sample = n_step / sample_interval;
            for (int mi = 0; mi < n_monitors; ++mi) {
                OracleFluxHz *m = &monitors[mi];
                if (sample < m->first_sample || sample >= m->first_sample + m->n_samples) return -1;
                accumulate_flux(s, m, sample);
            }
        }
    }
    return 0;
}

int oracle_hz2d_advance_tfsf(OracleHz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines,
                             const OracleLineHz *lines, int32_t n_monitors, OracleFluxHz *monitors,
                             int64_t sample_interval, int32_t n_tfsf, const OracleTfsfHz *tfsf) {
    return oracle_hz2d_advance_full(s, step0, n_steps, n_lines, lines, n_monitors, monitors, sample_interval, n_tfsf,
                                    tfsf, 0, 0, (real)0);
}

int oracle_hz2d_advance(OracleHz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines, const OracleLineHz *lines,
                        int32_t n_monitors, OracleFluxHz *monitors, int64_t sample_interval) {
    return oracle_hz2d_advance_full(s, step0, n_steps, n_lines, lines, n_monitors, monitors, sample_interval, 0, 0,
                                    0, 0, (real)0);
}
