// Temporally blocked 2D E_z step kernels: one launch advances the whole grid by T Yee steps.
//
// Layout.  Fields are double-buffered (read set "in", write set "out", swapped per launch), so a launch has no
// read-after-write hazard between its warps and every warp works alone: no __syncthreads, no atomics.  The grid is
// cut into tiles; one warp owns one tile's outputs (a rectangle of rows x columns) and streams its rows in increasing
// i.  Thread `lane` holds C adjacent columns; neighbours across threads come by warp shuffle.
//
// Time skew.  While streaming, stage s (1..T) of the warp's pipeline computes step s of row r - s when row r is
// loaded: H^s[i] needs E^(s-1) at rows i and i+1, E^s[i] needs H^s at rows i and i-1 (fdtd_ez_2d_kernels.py:23-122),
// so every input of stage s is already in registers.  Each field is kept as two rows (this iteration's and the last
// one's) per stage; the iteration parity PH selects which array plays which role, so no register moves are needed.
// A tile loads T extra rows before and after its own rows and halo columns on both sides; the cells of that cone are
// recomputed redundantly (bit-identical, every cell being a pure function of the inputs).
//
// Two variants share the code.  The interior variant (GEN = false, C = 4, 128-bit loads) covers the cells whose whole
// dependency cone lies off the CPML slabs and grid edges: uniform curl spacings, da = 1, uniform db, cb (and ca for
// lossy cells) per cell.  The general variant (GEN = true, C = 1) covers the rest: per-row / per-column kappa-folded
// spacings, per-cell da/db, the non-periodic edge rules, and the CPML psi recursion (boundaries.py:27-37) whose state
// flows through the stages like the fields.  Periodic wraps are modular indices; where open_sol evaluates the wrapped
// neighbour as f * cos + f * sin with cos 1, sin 0 (a real-only engine) the same expression is evaluated, so even the
// signs of zeros match.
//
// Row staging (interior variant).  Rows are brought into a per-warp shared-memory ring by the copy engine: lane 0
// issues one 1D bulk copy (cp.async.bulk, TMA) per array and row segment, TB_AHEAD rows ahead of the row being
// consumed, completing on an mbarrier per ring slot; the fields of a row are read back once, the coefficient rows (cb,
// ca) are read by stages 1..T from a ring deep enough to keep them until stage T has used them.  The copies occupy no
// registers while in flight, so the loads of the next rows overlap T stages of arithmetic of several rows.  Before a
// slot is refilled the warp synchronises and lane 0 orders the lanes' reads before the copy engine's writes with
// fence.proxy.async.  Waits are bounded: a wait that runs out sets the engine's error flag and the warp stops.
//
// Sources and monitors.  Line sources are added after E and its CPML, per step, in add order, skipped when the step's
// float32 value is 0 (core/sources.py:221-229).  On a DFT sample step the owning warp copies the flux line's E_z and
// tangential H into a small staging buffer; a separate kernel accumulates the running DFTs in sample order
// (monitors.py:45-46), so the complex128 sums are exactly the reference's.
#pragma once

#include <cuda_runtime.h>
#include "mbarrier.cuh"
#include <stdint.h>

#define TB_MAX_LINES 16
#define TB_MAX_MONS 8
#define TB_MAX_RECTS 4
#define TB_WARPS 4
#define TB_MAX_T 4
#define TB_AHEAD 3                        // rows staged ahead of the row being consumed (interior variant)

struct TBLine {
    int32_t axis, position, lo, hi;   // axis 0: cells (i, position), i in [lo, hi); axis 1: cells (position, j)
    const float *profile;
};

struct TBMon {
    int32_t normal_axis, position, lo, hi;   // normal 0: cells (position, j); normal 1: cells (i, position)
    float *stage;                            // (samples of the launch, 2, hi - lo): E_z then the tangential H
};

struct TBRect {
    int32_t r0, r1, c0, c1;   // output rows [r0, r1), columns [c0, c1)
    int32_t tiles_c, first_tile;
};

struct TBParams {
    int32_t nx, ny, px, py, npml, cpml_mask;
    const float *ez_in, *hx_in, *hy_in;
    float *ez_out, *hx_out, *hy_out;
    const float *cb, *ca, *da, *db;   // ca NULL: 1; da/db NULL: da_u / db_u
    float da_u, db_u;
    const float *inv_dx_e, *inv_dx_h, *inv_dy_e, *inv_dy_h;
    float s_inv_dx_e, s_inv_dx_h, s_inv_dy_e, s_inv_dy_h;   // the bulk values (interior variant)
    const float *cpml_rows[4];                              // b_e, a_e, inv_e, b_h, a_h, inv_h (npml each)
    const float *psi_e_in[4], *psi_h_in[4];
    float *psi_e_out[4], *psi_h_out[4];
    int32_t n_lines;
    TBLine lines[TB_MAX_LINES];
    const float *line_values;   // (n_lines, values_stride)
    int64_t values_stride;
    int64_t k0;                 // column of this launch's first step in line_values
    int32_t n_mons;
    TBMon mons[TB_MAX_MONS];
    int64_t n0;                 // engine steps taken before this launch
    int64_t m;                  // DFT sample interval
    int64_t q_first;            // sample number of staging slot 0
    uint32_t sample_mask;       // bit s - 1: step s of this launch is a DFT sample step
    int32_t n_rects;
    TBRect rects[TB_MAX_RECTS];
    int32_t tile_w, tile_rows, n_tiles;
    int32_t *err;   // set to 1 when a bounded wait runs out (read by the host after the launch)
    // test hook of the bounded waits (0: off): warp 0 of block 0 of the interior kernel first waits on an mbarrier
    // that nothing completes, at most this many nanoseconds, and then gives up as a real wait does
    int64_t stall_probe_ns;
    int64_t reserved;
};

// Shared memory of one warp of the interior variant: field ring (TB_AHEAD + 1 slots x E, H_x, H_y rows), coefficient
// rings (T + TB_AHEAD + 1 slots of cb, and of ca when per-cell), one mbarrier per field slot.
__host__ __device__ constexpr int tb_field_slots() { return TB_AHEAD + 1; }
__host__ __device__ constexpr int tb_coef_slots(int T) { return T + TB_AHEAD + 1; }
__host__ __device__ constexpr int tb_warp_smem_bytes(int T, bool ca) {
    return (tb_field_slots() * 3 + tb_coef_slots(T) * (ca ? 2 : 1)) * 128 * 4 + tb_field_slots() * 8;
}

// a mod n for the few periods a stream index can be off (no integer division: the streams stay within a couple of
// periods of [0, n)).
__device__ __forceinline__ int tb_wrap(int a, int n) {
    while (a < 0) a += n;
    while (a >= n) a -= n;
    return a;
}

// open_sol's wrapped lo-side neighbour of a real-only engine: f * wrap_cos - f_partner * wrap_sin with cos 1, sin 0
// and partner = f (fdtd_ez_2d_kernels.py:109-118).
__device__ __forceinline__ float tb_lo_wrap(float f) {
    const float one = 1.0f, zero = 0.0f;
    return f * one - f * zero;
}

template <int T, int C, bool GEN>
struct TBState {
    float E[2][T + 1][C];
    float Hx[2][T + 1][C];
    float Hy[2][T + 1][C];
    // CPML psi (general variant): x-side psi of H_y / E_z rows, y-side psi of H_x / E_z columns
    float pxh[2][T + 1][GEN ? C : 1];
    float pxe[2][T + 1][GEN ? C : 1];
    float pyh[2][T + 1][GEN ? C : 1];
    float pye[2][T + 1][GEN ? C : 1];
};

// Per-thread column facts.  An interior thread's C columns are contiguous and aligned, so they share one base
// column, one in-grid flag and one wrap flag (only the first can be column 0); a mask holds which are outputs.
template <int C>
struct TBCols {
    int jp0;            // physical column of the first column (jp0 + c: the others, C > 1)
    int jps[1];         // physical column (C = 1: the general variant)
    bool in_grid0;      // the columns are real cells (false: outside a non-periodic grid)
    uint32_t own;       // bit c: column c is one of this tile's output columns
    bool wrap_lo0;      // the first column is column 0 of a periodic y axis
    float inv_y_h[C], inv_y_e[C];
    // y-side CPML (general variant): side (2 / 3) and slab index of the H and E column, -1 when none
    int yh_side[C], yh_k[C], ye_side[C], ye_k[C];
    __device__ __forceinline__ int jp(int c) const { return C == 1 ? jps[0] : jp0 + c; }
    __device__ __forceinline__ bool in_grid(int c) const { return in_grid0; }
    __device__ __forceinline__ bool owns(int c) const { return (own >> c) & 1u; }
    __device__ __forceinline__ bool wrap_lo(int c) const { return c == 0 && wrap_lo0; }
};

// Which x-side (rows) or y-side (columns) CPML slab holds H row / E row `g` along an axis of n cells, and its index.
__device__ __forceinline__ void tb_cpml_slot(int g, int n, int npml, bool lo_on, bool hi_on, int lo_side, int hi_side,
                                             int &h_side, int &h_k, int &e_side, int &e_k) {
    h_side = e_side = -1;
    h_k = e_k = 0;
    if (lo_on && g >= 0 && g < npml) { h_side = lo_side; h_k = g; }
    else if (hi_on && g >= n - npml - 1 && g <= n - 2) { h_side = hi_side; h_k = g - (n - npml - 1); }
    if (lo_on && g >= 1 && g <= npml) { e_side = lo_side; e_k = g - 1; }
    else if (hi_on && g >= n - npml - 1 && g <= n - 2) { e_side = hi_side; e_k = g - (n - npml - 1); }
}

template <int C>
__device__ __forceinline__ void tb_load_row(const float *__restrict__ src, size_t row_base, const TBCols<C> &cols,
                                            bool vec, float (&out)[C]) {
    if (C == 4 && vec) {
        if (cols.in_grid0) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(src + row_base + cols.jp(0)));
            out[0] = v.x;
            out[1] = v.y;
            out[2] = v.z;
            out[3] = v.w;
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) out[c] = 0.0f;
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; ++c) out[c] = cols.in_grid(c) ? __ldg(src + row_base + cols.jp(c)) : 0.0f;
    }
}

template <int T, int C, bool GEN, bool CA>
struct TBWarp {
    const TBParams &p;   // rare paths only (CPML rows, line and monitor records); hot values are copied below
    TBCols<C> cols;
    TBState<T, C, GEN> st;
    int i0, i1, r_begin, r_end;
    bool vec;
    // hot parameters in registers: reading them through `p` after a global store would reload them
    int nx, ny, npml, cpml_mask;
    bool px, py;
    const float *__restrict__ ez_in, *__restrict__ hx_in, *__restrict__ hy_in;
    float *ez_out, *hx_out, *hy_out;
    const float *__restrict__ cbp, *__restrict__ cap, *__restrict__ dap, *__restrict__ dbp;
    float da_u, db_u, s_inv_dx_e, s_inv_dx_h, s_inv_dy_e, s_inv_dy_h;
    const float *__restrict__ inv_dx_e, *__restrict__ inv_dx_h;
    uint32_t sample_mask;
    uint32_t line_mask;   // line sources whose cells can fall in this tile's cone
    uint32_t mon_mask;    // flux lines with cells among this tile's outputs
    // interior variant: this warp's staging ring
    static constexpr bool BULK = !GEN;
    float *sm_fields = nullptr, *sm_cb = nullptr, *sm_ca = nullptr;
    uint64_t *sm_bar = nullptr;
    int win0 = 0;          // first column of the 128-column window (stream coordinates)
    uint32_t row_bytes = 0;  // bytes one array's row window brings in
    int lane = 0;
    bool failed = false;

    __device__ __forceinline__ TBWarp(const TBParams &params)
        : p(params), nx(params.nx), ny(params.ny), npml(params.npml), cpml_mask(params.cpml_mask),
          px(params.px != 0), py(params.py != 0), ez_in(params.ez_in), hx_in(params.hx_in), hy_in(params.hy_in),
          ez_out(params.ez_out), hx_out(params.hx_out), hy_out(params.hy_out), cbp(params.cb), cap(params.ca),
          dap(params.da), dbp(params.db), da_u(params.da_u), db_u(params.db_u), s_inv_dx_e(params.s_inv_dx_e),
          s_inv_dx_h(params.s_inv_dx_h), s_inv_dy_e(params.s_inv_dy_e), s_inv_dy_h(params.s_inv_dy_h),
          inv_dx_e(params.inv_dx_e), inv_dx_h(params.inv_dx_h), sample_mask(params.sample_mask) {}

    __device__ __forceinline__ int phys_row(int i) const { return px ? tb_wrap(i, nx) : i; }

    // Bulk copies of one array's 128-column window of physical row rp into `dst` (lane 0).  The window wraps on a
    // periodic y axis (several segments when ny < 128); on a non-periodic axis the part beyond the grid is not copied
    // (those columns lie outside every output's cone).
    __device__ __forceinline__ void copy_window(float *dst, const float *src_row, uint64_t *bar) const {
        int remaining = 128, d = 0, col = py ? tb_wrap(win0, ny) : win0;
        while (remaining > 0 && col < ny) {
            const int len = min(remaining, ny - col);
            tb_bulk_g2s(dst + d, src_row + col, (uint32_t)len * 4u, bar);
            d += len;
            remaining -= len;
            if (!py) break;
            col = 0;
        }
    }

    __device__ __forceinline__ uint32_t window_bytes() const {
        uint32_t bytes = 0;
        int remaining = 128, col = py ? tb_wrap(win0, ny) : win0;
        while (remaining > 0 && col < ny) {
            const int len = min(remaining, ny - col);
            bytes += (uint32_t)len * 4u;
            remaining -= len;
            if (!py) break;
            col = 0;
        }
        return bytes;
    }

    // Lane 0: stage stream row R (fields into field slot, coefficients into coefficient slots).
    __device__ __forceinline__ void issue_row(int R) {
        const int k = R - r_begin;
        const int fs = k % tb_field_slots(), cs = k % tb_coef_slots(T);
        uint64_t *bar = sm_bar + fs;
        const size_t base = (size_t)phys_row(R) * (size_t)ny;
        tb_mbar_expect_tx(bar, row_bytes * (CA ? 5u : 4u));
        float *f = sm_fields + fs * 384;
        copy_window(f, ez_in + base, bar);
        copy_window(f + 128, hx_in + base, bar);
        copy_window(f + 256, hy_in + base, bar);
        copy_window(sm_cb + cs * 128, cbp + base, bar);
        if (CA) copy_window(sm_ca + cs * 128, cap + base, bar);
    }

    // All lanes: wait until stream row R has landed (R <= r_end), then read its fields into the stage-0 registers
    // (R > r_end: the slot's last row, long landed; the values feed no output).
    template <int PH>
    __device__ __forceinline__ bool take_row(int R) {
        const int k = R - r_begin;
        const int fs = k % tb_field_slots();
        if (R <= r_end && !tb_mbar_wait(sm_bar + fs, (uint32_t)((k / tb_field_slots()) & 1))) return false;
        const float *f = sm_fields + fs * 384 + lane * 4;
        const float4 e = *reinterpret_cast<const float4 *>(f);
        const float4 hx = *reinterpret_cast<const float4 *>(f + 128);
        const float4 hy = *reinterpret_cast<const float4 *>(f + 256);
        st.E[PH][0][0] = e.x; st.E[PH][0][1] = e.y; st.E[PH][0][2] = e.z; st.E[PH][0][3] = e.w;
        st.Hx[PH][0][0] = hx.x; st.Hx[PH][0][1] = hx.y; st.Hx[PH][0][2] = hx.z; st.Hx[PH][0][3] = hx.w;
        st.Hy[PH][0][0] = hy.x; st.Hy[PH][0][1] = hy.y; st.Hy[PH][0][2] = hy.z; st.Hy[PH][0][3] = hy.w;
        return true;
    }

    // Stage 0 of stream row r: fields (and psi^0 of CPML cells) from the input buffers.
    template <int PH>
    __device__ __forceinline__ void load_row(int r) {
        const int rp = phys_row(r);
        const size_t base = (size_t)rp * (size_t)ny;
        tb_load_row<C>(ez_in, base, cols, vec, st.E[PH][0]);
        tb_load_row<C>(hx_in, base, cols, vec, st.Hx[PH][0]);
        tb_load_row<C>(hy_in, base, cols, vec, st.Hy[PH][0]);
        // the coefficient rows of row r are first read by stage 1 of the next iteration: pull them into L1 now
        if (cols.in_grid0) {
            asm volatile("prefetch.global.L1 [%0];" ::"l"(cbp + base + cols.jp(0)));
            if (CA) asm volatile("prefetch.global.L1 [%0];" ::"l"(cap + base + cols.jp(0)));
        }
        if constexpr (GEN) {
            int xh_side, xh_k, xe_side, xe_k;
            tb_cpml_slot(rp, nx, npml, cpml_mask & 1, cpml_mask & 2, 0, 1, xh_side, xh_k, xe_side, xe_k);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const bool g = cols.in_grid(c);
                const int j = cols.jp(c);
                st.pxh[PH][0][c] = (g && xh_side >= 0) ? p.psi_h_in[xh_side][(size_t)xh_k * ny + j] : 0.0f;
                st.pxe[PH][0][c] = (g && xe_side >= 0) ? p.psi_e_in[xe_side][(size_t)xe_k * ny + j] : 0.0f;
                st.pyh[PH][0][c] = (g && cols.yh_side[c] >= 0)
                                       ? p.psi_h_in[cols.yh_side[c]][(size_t)rp * npml + cols.yh_k[c]] : 0.0f;
                st.pye[PH][0][c] = (g && cols.ye_side[c] >= 0)
                                       ? p.psi_e_in[cols.ye_side[c]][(size_t)rp * npml + cols.ye_k[c]] : 0.0f;
            }
        }
    }

    // Stage S of the iteration of stream row r: step S of row i = r - S.
    template <int PH, int S>
    __device__ __forceinline__ void stage(int r) {
        constexpr int Q = PH ^ 1;   // last iteration's arrays
        const int i = r - S;
        // The general variant skips rows outside the stream (its loads index global rows).  The interior variant
        // always computes: out-of-stream rows only read in-bounds ring slots and produce values no output uses, and
        // an unconditional pipeline keeps only one phase of the arrays alive across iterations.
        if (GEN && (i < r_begin || i > r_end)) return;
        const int ip = phys_row(i);
        const size_t base = (size_t)ip * (size_t)ny;

        float cb[C], ca[C], da[C], db[C];
        if constexpr (BULK) {
            const int cs = (i - r_begin + tb_coef_slots(T)) % tb_coef_slots(T);   // i >= r_begin - T
            const float4 v = *reinterpret_cast<const float4 *>(sm_cb + cs * 128 + lane * 4);
            cb[0] = v.x; cb[1] = v.y; cb[2] = v.z; cb[3] = v.w;
            if constexpr (CA) {
                const float4 w = *reinterpret_cast<const float4 *>(sm_ca + cs * 128 + lane * 4);
                ca[0] = w.x; ca[1] = w.y; ca[2] = w.z; ca[3] = w.w;
            }
        } else {
            tb_load_row<C>(cbp, base, cols, vec, cb);
            if constexpr (CA) {
                tb_load_row<C>(cap, base, cols, vec, ca);
            }
        }
        if constexpr (GEN) {
            if (dap) {
                tb_load_row<C>(dap, base, cols, vec, da);
                tb_load_row<C>(dbp, base, cols, vec, db);
            } else {
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    da[c] = da_u;
                    db[c] = db_u;
                }
            }
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) db[c] = db_u;
        }
        float inv_x_h, inv_x_e;
        int xh_side = -1, xh_k = 0, xe_side = -1, xe_k = 0;
        if constexpr (GEN) {
            inv_x_h = __ldg(inv_dx_h + ip);
            inv_x_e = __ldg(inv_dx_e + ip);
            tb_cpml_slot(ip, nx, npml, cpml_mask & 1, cpml_mask & 2, 0, 1, xh_side, xh_k, xe_side, xe_k);
        } else {
            inv_x_h = s_inv_dx_h;
            inv_x_e = s_inv_dx_e;
        }

        // ---- H^S of row i (fdtd_ez_2d_kernels.py:41-47, then the H-row CPML, boundaries.py:752-755)
        float hxn[C], hyn[C];
        const float e_right_last = __shfl_down_sync(0xffffffffu, st.E[Q][S - 1][0], 1);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float e = st.E[Q][S - 1][c];
            const float e_right = c < C - 1 ? st.E[Q][S - 1][c + 1] : e_right_last;
            const float e_up = st.E[PH][S - 1][c];
            const float hx_old = st.Hx[Q][S - 1][c];
            const float hy_old = st.Hy[Q][S - 1][c];
            const int j = cols.jp(c);
            // H_x: every column but the last of a non-periodic y axis (whose face is never updated)
            if (GEN && !py && j == ny - 1) {
                hxn[c] = hx_old;
            } else {
                float v;
                if constexpr (GEN) {
                    v = da[c] * hx_old - db[c] * (e_right - e) * cols.inv_y_h[c];
                    if (cols.yh_side[c] >= 0) {
                        const int sd = cols.yh_side[c], k = cols.yh_k[c];
                        const float *rows = p.cpml_rows[sd];
                        float q = st.pyh[Q][S - 1][c] * rows[3 * npml + k];
                        q += rows[4 * npml + k] * (e_right - e) * rows[5 * npml + k];
                        st.pyh[PH][S][c] = q;
                        v += (-db[c]) * q;
                    }
                } else {
                    v = hx_old - db[c] * (e_right - e) * s_inv_dy_h;
                }
                hxn[c] = v;
            }
            // H_y: every row but the last of a non-periodic x axis
            if (GEN && !px && ip == nx - 1) {
                hyn[c] = hy_old;
            } else {
                float v;
                if constexpr (GEN) {
                    v = da[c] * hy_old + db[c] * (e_up - e) * inv_x_h;
                    if (xh_side >= 0) {
                        const float *rows = p.cpml_rows[xh_side];
                        float q = st.pxh[Q][S - 1][c] * rows[3 * npml + xh_k];
                        q += rows[4 * npml + xh_k] * (e_up - e) * rows[5 * npml + xh_k];
                        st.pxh[PH][S][c] = q;
                        v += db[c] * q;
                    }
                } else {
                    v = hy_old + db[c] * (e_up - e) * inv_x_h;
                }
                hyn[c] = v;
            }
        }

        // ---- E^S of row i (fdtd_ez_2d_kernels.py:107-120), E-row CPML x then y sides, line sources
        const float hx_left_first = __shfl_up_sync(0xffffffffu, hxn[C - 1], 1);
        const bool wrap_row = px && ip == 0;   // row 0 of a periodic x axis: its lo neighbour is the last row
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const int j = cols.jp(c);
            float hx_left = c > 0 ? hxn[c - 1] : hx_left_first;
            float hy_down = st.Hy[Q][S][c];   // H_y^S of row i - 1
            float curl;
            if (GEN && !px && ip == 0) {
                curl = hyn[c] * inv_x_e;
            } else {
                if (wrap_row) hy_down = tb_lo_wrap(hy_down);
                curl = (hyn[c] - hy_down) * inv_x_e;
            }
            const float inv_y_e = GEN ? cols.inv_y_e[c] : s_inv_dy_e;
            if (GEN && !py && j == 0) {
                curl -= hxn[c] * inv_y_e;
            } else {
                if (cols.wrap_lo(c)) hx_left = tb_lo_wrap(hx_left);
                curl -= (hxn[c] - hx_left) * inv_y_e;
            }
            const float e_old = st.E[Q][S - 1][c];
            float v = (CA ? ca[c] * e_old : e_old) + cb[c] * curl;
            if constexpr (GEN) {
                if (xe_side >= 0) {
                    const float *rows = p.cpml_rows[xe_side];
                    float q = st.pxe[Q][S - 1][c] * rows[xe_k];
                    q += rows[npml + xe_k] * (hyn[c] - hy_down) * rows[2 * npml + xe_k];
                    st.pxe[PH][S][c] = q;
                    v += cb[c] * q;
                }
                if (cols.ye_side[c] >= 0) {
                    const int sd = cols.ye_side[c], k = cols.ye_k[c];
                    const float *rows = p.cpml_rows[sd];
                    float q = st.pye[Q][S - 1][c] * rows[k];
                    q += rows[npml + k] * (hxn[c] - hx_left) * rows[2 * npml + k];
                    st.pye[PH][S][c] = q;
                    v += (-cb[c]) * q;
                }
            }
            for (uint32_t lines = line_mask; lines; lines &= lines - 1) {
                const int l = __ffs(lines) - 1;
                const TBLine &L = p.lines[l];
                const int along = L.axis == 0 ? ip : j, across = L.axis == 0 ? j : ip;
                if (across == L.position && along >= L.lo && along < L.hi && cols.in_grid(c)) {
                    const float value = p.line_values[(size_t)l * p.values_stride + p.k0 + (S - 1)];
                    if (value != 0.0f) v += value * L.profile[along - L.lo];
                }
            }
            st.E[PH][S][c] = v;
            st.Hx[PH][S][c] = hxn[c];
            st.Hy[PH][S][c] = hyn[c];
        }

        // ---- DFT sample: the owner copies the flux lines' E_z and tangential H of this step
        if (mon_mask && ((sample_mask >> (S - 1)) & 1u) && i >= i0 && i < i1) {
            const int slot = __popc(sample_mask & ((1u << (S - 1)) - 1u));
            for (uint32_t mons = mon_mask; mons; mons &= mons - 1) {
                const int mi = __ffs(mons) - 1;
                const TBMon &M = p.mons[mi];
                const int n = M.hi - M.lo;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    if (!cols.owns(c)) continue;
                    const int j = cols.jp(c);
                    if (M.normal_axis == 0) {
                        if (ip == M.position && j >= M.lo && j < M.hi) {
                            M.stage[(slot * 2) * n + (j - M.lo)] = st.E[PH][S][c];
                            M.stage[(slot * 2 + 1) * n + (j - M.lo)] = hyn[c];
                        }
                    } else if (j == M.position && ip >= M.lo && ip < M.hi) {
                        M.stage[(slot * 2) * n + (ip - M.lo)] = st.E[PH][S][c];
                        M.stage[(slot * 2 + 1) * n + (ip - M.lo)] = hxn[c];
                    }
                }
            }
        }
    }

    // Outputs of stage T (row r - T) into the output buffers.
    template <int PH>
    __device__ __forceinline__ void store(int r) {
        const int i = r - T;
        if (i < i0 || i >= i1) return;
        const int ip = phys_row(i);
        const size_t base = (size_t)ip * (size_t)ny;
        if (C == 4 && vec && cols.own == 0xFu) {
            *reinterpret_cast<float4 *>(ez_out + base + cols.jp(0)) =
                make_float4(st.E[PH][T][0], st.E[PH][T][1], st.E[PH][T][2], st.E[PH][T][3]);
            *reinterpret_cast<float4 *>(hx_out + base + cols.jp(0)) =
                make_float4(st.Hx[PH][T][0], st.Hx[PH][T][1], st.Hx[PH][T][2], st.Hx[PH][T][3]);
            *reinterpret_cast<float4 *>(hy_out + base + cols.jp(0)) =
                make_float4(st.Hy[PH][T][0], st.Hy[PH][T][1], st.Hy[PH][T][2], st.Hy[PH][T][3]);
        } else if (cols.own) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (!cols.owns(c)) continue;
                ez_out[base + cols.jp(c)] = st.E[PH][T][c];
                hx_out[base + cols.jp(c)] = st.Hx[PH][T][c];
                hy_out[base + cols.jp(c)] = st.Hy[PH][T][c];
            }
        }
        if constexpr (GEN) {
            int xh_side, xh_k, xe_side, xe_k;
            tb_cpml_slot(ip, nx, npml, cpml_mask & 1, cpml_mask & 2, 0, 1, xh_side, xh_k, xe_side, xe_k);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (!cols.owns(c)) continue;
                const int j = cols.jp(c);
                if (xh_side >= 0) p.psi_h_out[xh_side][(size_t)xh_k * ny + j] = st.pxh[PH][T][c];
                if (xe_side >= 0) p.psi_e_out[xe_side][(size_t)xe_k * ny + j] = st.pxe[PH][T][c];
                if (cols.yh_side[c] >= 0)
                    p.psi_h_out[cols.yh_side[c]][(size_t)ip * npml + cols.yh_k[c]] = st.pyh[PH][T][c];
                if (cols.ye_side[c] >= 0)
                    p.psi_e_out[cols.ye_side[c]][(size_t)ip * npml + cols.ye_k[c]] = st.pye[PH][T][c];
            }
        }
    }

    template <int PH, int S>
    __device__ __forceinline__ void stages_from(int r) {
        if constexpr (S <= T) {
            stage<PH, S>(r);
            if constexpr (S == 1 && !BULK) {
                // stage 1 was the last reader of last iteration's stage-0 row: prefetch row r + 1 into it
                if (r + 1 <= r_end) load_row<PH ^ 1>(r + 1);
            }
            stages_from<PH, S + 1>(r);
        }
    }

    template <int PH>
    __device__ __forceinline__ void iteration(int r) {
        if constexpr (BULK) {
            if (!take_row<PH>(r)) {
                failed = true;
                return;
            }
        }
        stages_from<PH, 1>(r);
        store<PH>(r);
        if constexpr (BULK) {
            // the field slot of row r and the coefficient slot of row r - T are free: refill with row r + AHEAD + 1
            __syncwarp();
            if (lane == 0 && r + TB_AHEAD + 1 <= r_end) {
                tb_fence_proxy_async();
                issue_row(r + TB_AHEAD + 1);
            }
        }
    }

    // After a failed wait: wait (bounded) for the copies still in flight so none lands after the warp has left.
    __device__ __forceinline__ void drain(int r_from) {
        for (int R = r_from; R <= min(r_end, r_from + TB_AHEAD); ++R) {
            const int k = R - r_begin;
            tb_mbar_wait(sm_bar + k % tb_field_slots(), (uint32_t)((k / tb_field_slots()) & 1));
        }
    }
};

template <int T, int C, bool GEN, bool CA>
__device__ __forceinline__ void ez2d_tb_tile(const TBParams &p, int w, unsigned char *tb_smem) {
    const int lane = threadIdx.x & 31;
    if (w >= p.n_tiles) return;   // whole warps leave together (the shuffles below need all 32 lanes)
    int rect = 0;
    for (int q = 1; q < p.n_rects; ++q)
        if (w >= p.rects[q].first_tile) rect = q;
    const TBRect R = p.rects[rect];
    const int t = w - R.first_tile;
    const int tc = t % R.tiles_c, tr = t / R.tiles_c;
    const int j0 = R.c0 + tc * p.tile_w, j1 = min(j0 + p.tile_w, R.c1);

    TBWarp<T, C, GEN, CA> W(p);
    W.i0 = R.r0 + tr * p.tile_rows;
    W.i1 = min(W.i0 + p.tile_rows, R.r1);
    W.r_begin = p.px ? W.i0 - T : max(0, W.i0 - T);
    W.r_end = p.px ? W.i1 - 1 + T : min(p.nx - 1, W.i1 - 1 + T);
    W.vec = (C == 4) && (p.ny % 4 == 0);
    constexpr int HL = C == 1 ? T : 4;
    // Line sources that can reach this tile's cone, flux lines with cells among its outputs (usually none).
    {
        const int cone_c0 = j0 - HL, cone_c1 = j0 - HL + 32 * C;   // loaded columns (stream coordinates)
        uint32_t lm = 0, mm = 0;
        for (int l = 0; l < p.n_lines; ++l) {
            const TBLine &L = p.lines[l];
            bool hit;
            if (p.px || p.py) {
                hit = true;   // wrapped coordinates: keep the per-cell test
            } else if (L.axis == 0) {   // cells (i, position), i in [lo, hi)
                hit = L.position >= cone_c0 && L.position < cone_c1 && L.hi > W.r_begin && L.lo <= W.r_end;
            } else {                    // cells (position, j)
                hit = L.position >= W.r_begin && L.position <= W.r_end && L.hi > cone_c0 && L.lo < cone_c1;
            }
            if (hit) lm |= 1u << l;
        }
        for (int q = 0; q < p.n_mons; ++q) {
            const TBMon &M = p.mons[q];
            const bool hit = M.normal_axis == 0
                                 ? (M.position >= W.i0 && M.position < W.i1 && M.hi > j0 && M.lo < j1)
                                 : (M.position >= j0 && M.position < j1 && M.hi > W.i0 && M.lo < W.i1);
            if (hit) mm |= 1u << q;
        }
        W.line_mask = lm;
        W.mon_mask = p.sample_mask ? mm : 0u;
    }
    {
        const int jl0 = j0 - HL + lane * C;   // first loaded column of this thread (stream coordinates)
        W.cols.in_grid0 = p.py || (jl0 >= 0 && jl0 < p.ny);
        W.cols.jp0 = p.py ? tb_wrap(jl0, p.ny) : jl0;
        W.cols.wrap_lo0 = p.py && W.cols.jp0 == 0;
        W.cols.own = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const int jl = jl0 + c;
            if (jl >= j0 && jl < j1) W.cols.own |= 1u << c;
            const int jpc = p.py ? tb_wrap(jl, p.ny) : jl;
            if (c == 0) W.cols.jps[0] = jpc;
            const bool g = p.py || (jl >= 0 && jl < p.ny);
            const int jc = g ? jpc : 0;
            if (GEN) {
                W.cols.inv_y_h[c] = __ldg(p.inv_dy_h + jc);
                W.cols.inv_y_e[c] = __ldg(p.inv_dy_e + jc);
                tb_cpml_slot(g ? jc : -1, p.ny, p.npml, p.cpml_mask & 4, p.cpml_mask & 8, 2, 3, W.cols.yh_side[c],
                             W.cols.yh_k[c], W.cols.ye_side[c], W.cols.ye_k[c]);
            } else {
                W.cols.inv_y_h[c] = W.cols.inv_y_e[c] = 0.0f;
                W.cols.yh_side[c] = W.cols.ye_side[c] = -1;
                W.cols.yh_k[c] = W.cols.ye_k[c] = 0;
            }
        }
    }
    // Pipeline registers start at 0 (a non-periodic first row reads no H_y below it; the rest is outside the cone).
#pragma unroll
    for (int ph = 0; ph < 2; ++ph)
#pragma unroll
        for (int s = 0; s <= T; ++s)
#pragma unroll
            for (int c = 0; c < C; ++c) {
                W.st.E[ph][s][c] = W.st.Hx[ph][s][c] = W.st.Hy[ph][s][c] = 0.0f;
                if (GEN) W.st.pxh[ph][s][c] = W.st.pxe[ph][s][c] = W.st.pyh[ph][s][c] = W.st.pye[ph][s][c] = 0.0f;
            }
    W.lane = lane;
    if constexpr (!GEN) {
        unsigned char *mine = tb_smem + (threadIdx.x >> 5) * tb_warp_smem_bytes(T, CA);
        W.sm_fields = reinterpret_cast<float *>(mine);
        W.sm_cb = W.sm_fields + tb_field_slots() * 384;
        W.sm_ca = W.sm_cb + tb_coef_slots(T) * 128;
        W.sm_bar = reinterpret_cast<uint64_t *>(W.sm_cb + tb_coef_slots(T) * 128 * (CA ? 2 : 1));
        W.win0 = j0 - 4;
        W.row_bytes = W.window_bytes();
        if (lane == 0) {
            for (int q = 0; q < tb_field_slots(); ++q) tb_mbar_init(W.sm_bar + q, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            tb_fence_proxy_async();   // the copy engine sees the initialised barriers
            for (int R = W.r_begin; R <= min(W.r_end, W.r_begin + TB_AHEAD); ++R) W.issue_row(R);
        }
        __syncwarp();
    } else {
        W.template load_row<0>(W.r_begin);
    }
    const int r_last = W.r_end + T;
    for (int r = W.r_begin; r <= r_last; r += 2) {
        W.template iteration<0>(r);
        if (W.failed) {
            if (lane == 0) atomicExch(p.err, 1);
            W.drain(r);
            return;
        }
        if (r + 1 <= r_last) {
            W.template iteration<1>(r + 1);
            if (W.failed) {
                if (lane == 0) atomicExch(p.err, 1);
                W.drain(r + 1);
                return;
            }
        }
    }
}

template <int T, int C, bool GEN, bool CA>
__global__ void __launch_bounds__(TB_WARPS * 32) ez2d_tb_kernel(const TBParams p) {
    extern __shared__ __align__(16) unsigned char tb_smem[];
    ez2d_tb_tile<T, C, GEN, CA>(p, blockIdx.x * TB_WARPS + (threadIdx.x >> 5), tb_smem);
}

// Several simulations in one launch (as ez2d_interior_batch_kernel).
template <int T, int C, bool GEN, bool CA>
__global__ void __launch_bounds__(TB_WARPS * 32) ez2d_tb_batch_kernel(const TBParams *__restrict__ jobs,
                                                                   const int *__restrict__ tile_start, int n_jobs) {
    extern __shared__ __align__(16) unsigned char tb_smem[];
    const int g = blockIdx.x * TB_WARPS + (threadIdx.x >> 5);
    if (g >= tile_start[n_jobs]) return;
    int job = 0;
    while (job + 1 < n_jobs && g >= tile_start[job + 1]) ++job;
    ez2d_tb_tile<T, C, GEN, CA>(jobs[job], g - tile_start[job], tb_smem);
}

// Running DFTs of one flux line from the staged samples of one launch, in sample order (monitors.py:45-46,84-90):
// sample q of the launch in staging slot slot0 + q * slot_stride (0 and 1 when only the sample steps were staged;
// the first sample step's slot and the sample interval when every step was).
__device__ __forceinline__ void ez2d_flux_staged(int t, const float *__restrict__ stage, int n, int nf, int n_q,
                                                 int slot0, int slot_stride, const float *__restrict__ phases,
                                                 double *__restrict__ e_acc, double *__restrict__ h_acc) {
    if (t >= n * nf) return;
    const int f = t / n, c = t - f * n;
    const size_t a = ((size_t)f * n + c) * 2;
    double er = e_acc[a], ei = e_acc[a + 1], hr = h_acc[a], hi = h_acc[a + 1];
    for (int q = 0; q < n_q; ++q) {
        const double pr = (double)phases[((size_t)q * nf + f) * 2], pi = (double)phases[((size_t)q * nf + f) * 2 + 1];
        const size_t slot = (size_t)(slot0 + q * slot_stride);
        const double e = (double)stage[(slot * 2) * n + c], hv = (double)stage[(slot * 2 + 1) * n + c];
        er += pr * e;
        ei += pi * e;
        hr += pr * hv;
        hi += pi * hv;
    }
    e_acc[a] = er;
    e_acc[a + 1] = ei;
    h_acc[a] = hr;
    h_acc[a + 1] = hi;
}

__global__ void ez2d_flux_staged_kernel(const float *__restrict__ stage, int n, int nf, int n_q, int slot0,
                                        int slot_stride, const float *__restrict__ phases, double *__restrict__ e_acc,
                                        double *__restrict__ h_acc) {
    ez2d_flux_staged(blockIdx.x * blockDim.x + threadIdx.x, stage, n, nf, n_q, slot0, slot_stride, phases, e_acc,
                     h_acc);
}

// One flux line of one simulation in a batched launch.
struct FluxBatchItem {
    const float *stage;
    const float *phases;
    double *e_acc, *h_acc;
    int32_t n, nf, n_q, pad;
};

__global__ void ez2d_flux_staged_batch_kernel(const FluxBatchItem *__restrict__ items) {
    const FluxBatchItem it = items[blockIdx.y];
    ez2d_flux_staged(blockIdx.x * blockDim.x + threadIdx.x, it.stage, it.n, it.nf, it.n_q, 0, 1, it.phases, it.e_acc,
                     it.h_acc);
}
