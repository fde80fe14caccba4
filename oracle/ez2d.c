/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Nothing in the product (opensol_b200/) links, loads or calls this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the reference results are compared with.
 *
 * Plain-C restatement of open_sol's 2D E_z-polarisation FDTD time step on the CPU, written to reproduce the
 * reference CPU backend's float32 (or float64, -DORACLE_REAL=double) arithmetic bit for bit:
 *   - Yee H update            open_sol/physics/em/solvers/fdtd_ez_2d_kernels.py:23-81   (update_h_kernel + numba twin)
 *   - Yee E update            open_sol/physics/em/solvers/fdtd_ez_2d_kernels.py:88-163  (update_e_kernel + numba twin)
 *   - CPML psi update+apply   open_sol/physics/em/boundaries.py:27-37 (numpy twin), sides in FACES order
 *                             (open_sol/core/constants.py:18), rows from cpml_side_rows (boundaries.py:570-576),
 *                             signs ez: x +, y - (boundaries.py:713-715), per-side views (boundaries.py:732-760)
 *   - step order              open_sol/physics/em/solvers/fdtd_ez_2d.py:71-119 (H, H CPML, E, E CPML, sources at
 *                             t + dt/2, n_step += 1, monitors every sample_interval steps: fdtd_2d_base.py:470-488)
 *   - soft line source        open_sol/core/sources.py:146-154,221-229 (target += scale * profile, skipped at 0)
 *   - line DFT accumulation   open_sol/physics/em/monitors.py:45-46 (complex128 += complex64 phase * (double)f)
 *   - dispersive poles        open_sol/physics/em/solvers/fdtd_ez_2d_kernels.py:190-260 (host twins), order of
 *                             fdtd_ez_2d.py:263-358: Drude J / Lorentz P from E^n before the E update (Drude poles
 *                             first, each kind in add order), the E corrections after the E update and its CPML
 *   - TFSF plane-wave box     open_sol/physics/em/sources.py:35-52 (host twins of the side corrections and the 1D
 *                             incident line), 334-350 (inject_h after the H update, inject_e after the E update); the
 *                             E-side corrections run after the line sources (open_sol: sources in add order, which
 *                             gives the same bits whenever no line source shares a cell with a box side)
 * Every float operation keeps the reference's evaluation order; build with -ffp-contract=off (no FMA contraction).
 * Rows are parallelised with OpenMP: each cell of a half step is independent, so the thread count never changes a
 * result.
 */
#include <stdint.h>
#include <stddef.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

/* CPML side order = open_sol FACES: x_lo, x_hi, y_lo, y_hi. */
enum { SIDE_XLO = 0, SIDE_XHI = 1, SIDE_YLO = 2, SIDE_YHI = 3 };

typedef struct {
    int32_t nx, ny, periodic_x, periodic_y;
    real *ez, *hx, *hy;                       /* (nx, ny) row-major, j fastest */
    const real *ca;                           /* NULL: ca = 1 everywhere */
    const real *cb;
    const real *da, *db;                      /* NULL: the uniform values below */
    real da_uniform, db_uniform;
    const real *inv_dx_e, *inv_dx_h;          /* (nx,) kappa folded */
    const real *inv_dy_e, *inv_dy_h;          /* (ny,) kappa folded */
    int32_t npml;
    int32_t cpml_active[4];
    const real *b_e[4], *a_e[4], *inv_e[4];   /* (npml,) per side: cell-centre rows */
    const real *b_h[4], *a_h[4], *inv_h[4];   /* (npml,) per side: hi-face rows */
    real *psi_e[4], *psi_h[4];                /* x sides (npml, ny), y sides (nx, npml) */
} OracleEz2D;

typedef struct {
    int32_t axis;          /* 'x' line (along x at y-cell position) = 0, 'y' line = 1 */
    int32_t position;
    int32_t lo, hi;        /* half-open span along the line */
    const float *profile;  /* (hi - lo,) calibrated float32 profile */
    const float *values;   /* (n_steps,) float32 amplitude * temporal(t + dt/2) of each step of the chunk */
} OracleLine;

typedef struct {
    int32_t normal_axis;   /* 0: normal x (line of constant x-cell: E_z, H_y), 1: normal y (E_z, H_x) */
    int32_t position;
    int32_t lo, hi;
    int32_t nf;
    double *e_acc, *h_acc; /* (nf, hi - lo) complex128 as (re, im) pairs */
    const float *phases;   /* (n_samples, nf) complex64 as (re, im) pairs, sample q at row q - first_sample */
    int64_t first_sample;
    int64_t n_samples;
} OracleFlux;

typedef struct {
    int32_t x0, x1, y0, y1, aux_x0, aux_n, source_index;
    real coef_h[4], coef_e[2], mur_lo, mur_hi;
    real *aux_ez, *aux_hy;                    /* (aux_n,) incident line: cell centres / hi faces */
    const real *aux_coef_h, *aux_coef_e;      /* (aux_n - 1,) / (aux_n,) */
    const float *values;                      /* (n_steps,) float32 soft-source value of each step of the chunk */
} OracleTfsf;

typedef struct {
    int32_t kind;                             /* 0 Drude, 1 Lorentz */
    int32_t i0, i1, j0, j1;                   /* cell box */
    real damping, restoring;
    const real *drive;                        /* (box) drive coefficient x cell mask */
    real *a, *b;                              /* Drude: a = J; Lorentz: a = P, b = dP (box) */
} OraclePole;

static inline real coef_or(const real *array, size_t idx, real uniform) { return array ? array[idx] : uniform; }

/* _pole_updates (fdtd_ez_2d.py:318-345) from E^n; jz_total is zeroed on drude_box first when several Drude poles
 * add into it (one pole stores J). */
static void poles_update(const OracleEz2D *s, int32_t n_poles, const OraclePole *poles, real *jz_total,
                         const int32_t *drude_box)
{
    const size_t ny = (size_t)s->ny;
    int n_drude = 0;
    for (int q = 0; q < n_poles; ++q) n_drude += poles[q].kind == 0;
    if (n_drude > 1)
        for (int i = drude_box[0]; i < drude_box[1]; ++i)
            for (int j = drude_box[2]; j < drude_box[3]; ++j) jz_total[(size_t)i * ny + j] = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < n_poles; ++q) {
            const OraclePole *p = &poles[q];
            if (p->kind != pass) continue;
            const int w = p->j1 - p->j0;
            for (int i = p->i0; i < p->i1; ++i)
                for (int j = p->j0; j < p->j1; ++j) {
                    const size_t t = (size_t)(i - p->i0) * w + (j - p->j0), g = (size_t)i * ny + j;
                    if (p->kind == 0) {
                        p->a[t] += p->damping * p->a[t] + p->drive[t] * s->ez[g];
                        jz_total[g] = n_drude == 1 ? p->a[t] : jz_total[g] + p->a[t];
                    } else {
                        p->b[t] += p->damping * p->b[t] - p->restoring * p->a[t] + p->drive[t] * s->ez[g];
                        p->a[t] += p->b[t];
                    }
                }
        }
}

/* _pole_corrections (fdtd_ez_2d.py:347-358). */
static void poles_correct(const OracleEz2D *s, int32_t n_poles, const OraclePole *poles, const real *jz_total,
                          const int32_t *drude_box, real inv_dt)
{
    const size_t ny = (size_t)s->ny;
    for (int i = drude_box[0]; i < drude_box[1]; ++i)
        for (int j = drude_box[2]; j < drude_box[3]; ++j) {
            const size_t g = (size_t)i * ny + j;
            s->ez[g] -= s->cb[g] * jz_total[g];
        }
    for (int q = 0; q < n_poles; ++q) {
        const OraclePole *p = &poles[q];
        if (p->kind != 1) continue;
        const int w = p->j1 - p->j0;
        for (int i = p->i0; i < p->i1; ++i)
            for (int j = p->j0; j < p->j1; ++j) {
                const size_t t = (size_t)(i - p->i0) * w + (j - p->j0), g = (size_t)i * ny + j;
                s->ez[g] -= s->cb[g] * inv_dt * p->b[t];
            }
    }
}

/* TFSFSource.inject_h: H_y / H_x side corrections from the incident E_z, then the incident H update. */
static void tfsf_h(const OracleEz2D *s, const OracleTfsf *t)
{
    const size_t ny = (size_t)s->ny;
    for (int j = t->y0; j < t->y1; ++j) {
        s->hy[(size_t)(t->x0 - 1) * ny + j] -= t->coef_h[0] * t->aux_ez[t->aux_x0];
        s->hy[(size_t)(t->x1 - 1) * ny + j] += t->coef_h[1] * t->aux_ez[t->aux_x0 + (t->x1 - 1 - t->x0)];
    }
    for (int i = t->x0; i < t->x1; ++i) {
        const real incident = t->aux_ez[t->aux_x0 + (i - t->x0)];
        s->hx[(size_t)i * ny + (t->y0 - 1)] += t->coef_h[2] * incident;
        s->hx[(size_t)i * ny + (t->y1 - 1)] -= t->coef_h[3] * incident;
    }
    for (int a = 0; a < t->aux_n - 1; ++a) t->aux_hy[a] += t->aux_coef_h[a] * (t->aux_ez[a + 1] - t->aux_ez[a]);
}

/* TFSFSource.inject_e: E_z side corrections from the incident H_y, then the incident E update with the soft source
 * and the Mur ends (from the ends' values before the update). */
static void tfsf_e(const OracleEz2D *s, const OracleTfsf *t, int64_t k)
{
    const size_t ny = (size_t)s->ny;
    for (int j = t->y0; j < t->y1; ++j) {
        s->ez[(size_t)t->x0 * ny + j] -= t->coef_e[0] * t->aux_hy[t->aux_x0 - 1];
        s->ez[(size_t)(t->x1 - 1) * ny + j] += t->coef_e[1] * t->aux_hy[t->aux_x0 + (t->x1 - 1 - t->x0)];
    }
    const int n = t->aux_n;
    const real old0 = t->aux_ez[0], old1 = t->aux_ez[1], old2 = t->aux_ez[n - 2], old3 = t->aux_ez[n - 1];
    for (int a = 1; a < n - 1; ++a) t->aux_ez[a] += t->aux_coef_e[a] * (t->aux_hy[a] - t->aux_hy[a - 1]);
    t->aux_ez[t->source_index] += (real)t->values[k];
    t->aux_ez[0] = old1 + t->mur_lo * (t->aux_ez[1] - old0);
    t->aux_ez[n - 1] = old2 + t->mur_hi * (t->aux_ez[n - 2] - old3);
}

static void update_h(const OracleEz2D *s)
{
    const int nx = s->nx, ny = s->ny;
    const real one = (real)1, zero = (real)0;   /* real-only engine: wrap cos 1, sin 0, partner = self */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            const size_t idx = (size_t)i * ny + j;
            const real e = s->ez[idx];
            const real da = coef_or(s->da, idx, s->da_uniform);
            const real db = coef_or(s->db, idx, s->db_uniform);
            if (j < ny - 1) {
                s->hx[idx] = da * s->hx[idx] - db * (s->ez[idx + 1] - e) * s->inv_dy_h[j];
            } else if (s->periodic_y) {
                const real wrap = s->ez[(size_t)i * ny] * one + s->ez[(size_t)i * ny] * zero;
                s->hx[idx] = da * s->hx[idx] - db * (wrap - e) * s->inv_dy_h[j];
            }
            if (i < nx - 1) {
                s->hy[idx] = da * s->hy[idx] + db * (s->ez[idx + ny] - e) * s->inv_dx_h[i];
            } else if (s->periodic_x) {
                const real wrap = s->ez[j] * one + s->ez[j] * zero;
                s->hy[idx] = da * s->hy[idx] + db * (wrap - e) * s->inv_dx_h[i];
            }
        }
    }
}

static void update_e(const OracleEz2D *s)
{
    const int nx = s->nx, ny = s->ny;
    const real one = (real)1, zero = (real)0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < ny; ++j) {
            const size_t idx = (size_t)i * ny + j;
            real curl;
            if (i >= 1) {
                curl = (s->hy[idx] - s->hy[idx - ny]) * s->inv_dx_e[i];
            } else if (s->periodic_x) {
                const size_t w = (size_t)(nx - 1) * ny + j;
                curl = (s->hy[idx] - (s->hy[w] * one - s->hy[w] * zero)) * s->inv_dx_e[i];
            } else {
                curl = s->hy[idx] * s->inv_dx_e[i];
            }
            if (j >= 1) {
                curl -= (s->hx[idx] - s->hx[idx - 1]) * s->inv_dy_e[j];
            } else if (s->periodic_y) {
                const size_t w = idx + ny - 1;
                curl -= (s->hx[idx] - (s->hx[w] * one - s->hx[w] * zero)) * s->inv_dy_e[j];
            } else {
                curl -= s->hx[idx] * s->inv_dy_e[j];
            }
            const real ca = coef_or(s->ca, idx, one);
            s->ez[idx] = ca * s->ez[idx] + s->cb[idx] * curl;
        }
    }
}

/* First row of a side's slab: lo E rows 1..npml, lo H rows 0..npml-1, hi E and H rows n-npml-1..n-2. */
static int side_first_row(int side, int kind_e, int n, int npml)
{
    const int lo = (side == SIDE_XLO || side == SIDE_YLO);
    if (lo) return kind_e ? 1 : 0;
    return n - npml - 1;
}

/* psi = b psi + a (f_hi - f_lo) inv; field += (sign coefficient) psi, one side; kind_e selects the E rows
 * (f_hi = src[r], f_lo = src[r - 1], coefficient cb, field ez) or the H rows (f_hi = src[r + 1], f_lo = src[r],
 * coefficient db, field hy on x sides / hx on y sides). */
static void cpml_side(const OracleEz2D *s, int side, int kind_e)
{
    const int nx = s->nx, ny = s->ny, npml = s->npml;
    const int x_side = (side == SIDE_XLO || side == SIDE_XHI);
    const real sign = x_side ? (real)1 : (real)-1;
    const real *b = kind_e ? s->b_e[side] : s->b_h[side];
    const real *a = kind_e ? s->a_e[side] : s->a_h[side];
    const real *inv = kind_e ? s->inv_e[side] : s->inv_h[side];
    real *psi = kind_e ? s->psi_e[side] : s->psi_h[side];
    const real *src = kind_e ? (x_side ? s->hy : s->hx) : s->ez;
    real *field = kind_e ? s->ez : (x_side ? s->hy : s->hx);
    const int first = side_first_row(side, kind_e, x_side ? nx : ny, npml);
    const int up = kind_e ? 0 : 1, dn = kind_e ? -1 : 0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < (x_side ? npml : nx); ++i) {
        for (int j = 0; j < (x_side ? ny : npml); ++j) {
            const int k = x_side ? i : j;                 /* slab row index along the graded axis */
            const int r = first + k;                      /* grid row along that axis */
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
            const real coefficient = kind_e ? s->cb[cell] : coef_or(s->db, cell, s->db_uniform);
            field[cell] += sign * coefficient * q;
        }
    }
}

static void inject_line(const OracleEz2D *s, const OracleLine *line, int64_t k)
{
    const float value = line->values[k];
    if (value == 0.0f) return;   /* a pulse past its float32 envelope: the reference skips the launch */
    for (int c = line->lo; c < line->hi; ++c) {
        const size_t cell = line->axis == 0 ? (size_t)c * s->ny + line->position
                                            : (size_t)line->position * s->ny + c;
        const float add = value * line->profile[c - line->lo];
        s->ez[cell] += (real)add;
    }
}

static void accumulate_flux(const OracleEz2D *s, OracleFlux *m, int64_t sample)
{
    const int n = m->hi - m->lo;
    const float *ph = m->phases + (size_t)(sample - m->first_sample) * m->nf * 2;
    const real *h = m->normal_axis == 0 ? s->hy : s->hx;
    for (int f = 0; f < m->nf; ++f) {
        const double pr = (double)ph[2 * f], pi = (double)ph[2 * f + 1];
        for (int c = 0; c < n; ++c) {
            const size_t cell = m->normal_axis == 0 ? (size_t)m->position * s->ny + (m->lo + c)
                                                    : (size_t)(m->lo + c) * s->ny + m->position;
            const double e = (double)s->ez[cell], hv = (double)h[cell];
            const size_t a = ((size_t)f * n + c) * 2;
            m->e_acc[a] += pr * e;
            m->e_acc[a + 1] += pi * e;
            m->h_acc[a] += pr * hv;
            m->h_acc[a + 1] += pi * hv;
        }
    }
}

/* Advance n_steps steps starting after engine step `step0` (the engine's n_step before the chunk).  Line source
 * values are indexed by the step within the chunk; monitors sample when (step0 + k + 1) % sample_interval == 0.
 * Returns 0, or -1 when a monitor's phase table does not cover a sample. */
int oracle_ez2d_advance_full(OracleEz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines, const OracleLine *lines,
                             int32_t n_monitors, OracleFlux *monitors, int64_t sample_interval, int32_t n_tfsf,
                             const OracleTfsf *tfsf, int32_t n_poles, const OraclePole *poles, real *jz_total,
                             const int32_t *drude_box, real inv_dt)
{
    for (int64_t k = 0; k < n_steps; ++k) {
        update_h(s);
        for (int side = 0; side < 4; ++side)
            if (s->cpml_active[side]) cpml_side(s, side, 0);
        for (int b = 0; b < n_tfsf; ++b) tfsf_h(s, &tfsf[b]);
        if (n_poles) poles_update(s, n_poles, poles, jz_total, drude_box);
        update_e(s);
        for (int side = 0; side < 4; ++side)
            if (s->cpml_active[side]) cpml_side(s, side, 1);
        if (n_poles) poles_correct(s, n_poles, poles, jz_total, drude_box, inv_dt);
        for (int l = 0; l < n_lines; ++l) inject_line(s, &lines[l], k);
        for (int b = 0; b < n_tfsf; ++b) tfsf_e(s, &tfsf[b], k);
        const int64_t n_step = step0 + k + 1;
        if (n_monitors > 0 && n_step % sample_interval == 0) {
            const int64_t sample = n_step / sample_interval;
            for (int mi = 0; mi < n_monitors; ++mi) {
                OracleFlux *m = &monitors[mi];
                if (sample < m->first_sample || sample >= m->first_sample + m->n_samples) return -1;
                accumulate_flux(s, m, sample);
            }
        }
    }
    return 0;
}

int oracle_ez2d_advance_tfsf(OracleEz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines, const OracleLine *lines,
                             int32_t n_monitors, OracleFlux *monitors, int64_t sample_interval, int32_t n_tfsf,
                             const OracleTfsf *tfsf)
{
    const int32_t no_box[4] = {0, 0, 0, 0};
    return oracle_ez2d_advance_full(s, step0, n_steps, n_lines, lines, n_monitors, monitors, sample_interval, n_tfsf,
                                    tfsf, 0, 0, 0, no_box, 0);
}

int oracle_ez2d_advance(OracleEz2D *s, int64_t step0, int64_t n_steps, int32_t n_lines, const OracleLine *lines,
                        int32_t n_monitors, OracleFlux *monitors, int64_t sample_interval)
{
    return oracle_ez2d_advance_tfsf(s, step0, n_steps, n_lines, lines, n_monitors, monitors, sample_interval, 0, 0);
}

int oracle_ez2d_real_size(void) { return (int)sizeof(real); }
