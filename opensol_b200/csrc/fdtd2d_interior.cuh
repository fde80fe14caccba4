// Interior kernel of the temporally blocked 2D E_z step (the cells whose T-step dependency cone avoids the CPML slabs
// and the non-periodic grid edges; fdtd2d_tb.cuh has the general kernel and the shared plumbing).
//
// One warp streams one tile of 120 output columns (128 loaded: 4 halo columns on each side, enough for T <= 4) and
// tile_rows output rows, T steps per launch, with the time-skewed register pipeline described in fdtd2d_tb.cuh.  Rows
// arrive in a per-warp shared-memory ring by 1D bulk copies (TMA) TB_AHEAD rows ahead.  A thread holds 4 adjacent
// columns as two float2 pairs and does the arithmetic with the packed sm_100 operations __fadd2_rn / __fmul2_rn: each
// lane of a packed operation is rounded on its own exactly like the scalar __fadd_rn / __fmul_rn, so the results are
// the same bits as open_sol's float32 evaluation (x - y is evaluated as x + (-y), which IEEE defines identically).
// One exception is kept out: the code generator merges a packed multiply into a following packed add (a packed fused
// multiply-add, one rounding instead of two, even from explicit .rn PTX), so every add whose operand is a product is
// done per lane with the scalar __fadd_rn, which is never merged.  Multiplies and the adds of plain differences stay
// packed.  The periodic wraps are compile-time (PX, PY): a non-periodic axis costs nothing.
#pragma once

#include "fdtd2d_tb.cuh"

// Floats of one staged row window in shared memory: the 128 columns plus room for a copy that starts up to 3 floats
// before them (rounded down to a 16-byte boundary when the row length is not a multiple of 4) and is rounded up to
// 16 bytes.
#define IP_ROW 136

// Shared memory of one warp of the interior kernel: field ring (TB_AHEAD + 1 slots x E, H_x, H_y windows),
// coefficient rings (T + TB_AHEAD + 1 slots of cb, and of ca when per-cell), one mbarrier per field slot.
__host__ __device__ constexpr int ip_warp_smem_bytes(int T, bool ca) {
    return (tb_field_slots() * 3 + tb_coef_slots(T) * (ca ? 2 : 1)) * IP_ROW * 4 + tb_field_slots() * 8;
}

// packed add / subtract: only for operands that are not products (see above)
__device__ __forceinline__ float2 ip_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 ip_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
// per-lane add / subtract of a product: two separately rounded scalar operations, never merged with the multiply
__device__ __forceinline__ float2 ip_add_p(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 ip_sub_p(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, -b.x), __fadd_rn(a.y, -b.y));
}

template <int T, bool CA, bool PX, bool PY, bool VEC, bool HELD>
struct IPWarp {
    const TBParams &p;
    // tile
    int i0, i1, r_begin, r_end, j0, j1;
    int lane, jl0, jp0;
    uint32_t own;          // bit c: column jl0 + c is an output column
    bool in_grid0;         // the 4 columns are real cells
    bool wrap_lo0;         // PY: the first column is column 0 (its lo neighbour is the wrapped last column)
    uint32_t line_mask, mon_mask, sample_mask;
    int nx, ny;
    static constexpr bool vec = VEC;   // ny % 4 == 0: every row window starts 16-byte aligned (float4 reads, stores)
    float2 db2, ixh2, ixe2, iyh2, iye2;
    float *ez_out, *hx_out, *hy_out;
    const float *__restrict__ ez_in, *__restrict__ hx_in, *__restrict__ hy_in, *__restrict__ cbp, *__restrict__ cap;
    // HELD: the grid sizes, array pointers and bulk coefficients above are copied into registers once per tile (the
    // one-grid kernel, whose p is its kernel parameter); otherwise they are read from p where they are used (the
    // batched kernel, whose p is the warp's copy in shared memory), which keeps fewer registers live in the row loop
    __device__ __forceinline__ int gnx() const { if constexpr (HELD) return nx; else return p.nx; }
    __device__ __forceinline__ int gny() const { if constexpr (HELD) return ny; else return p.ny; }
    __device__ __forceinline__ float2 pair(float2 held, float v) const {
        if constexpr (HELD) return held;
        else return make_float2(v, v);
    }
    template <typename P>
    __device__ __forceinline__ P ptr(P held, P v) const {
        if constexpr (HELD) return held;
        else return v;
    }
    // staging ring
    float *sm_fields, *sm_cb, *sm_ca;
    uint64_t *sm_bar;
    uint32_t row_bytes;
    bool failed = false;
    // pipeline: [parity][stage][pair]
    float2 E[2][T + 1][2], Hx[2][T + 1][2], Hy[2][T + 1][2];

    __device__ __forceinline__ IPWarp(const TBParams &params) : p(params) {}

    __device__ __forceinline__ int phys_row(int i) const { return PX ? tb_wrap(i, gnx()) : i; }

    // Offset (0..3 floats) of row R's first window column behind the 16-byte boundary its copy starts on (0 when
    // ny % 4 == 0; the host plans an interior on a row length that is not a multiple of 4 only for a non-periodic y).
    __device__ __forceinline__ int row_off(int R) const {
        // (row * ny + j0 - 4) mod 4 in 32-bit arithmetic: a wrapped product keeps its value mod 4
        return vec ? 0 : (int)(((uint32_t)phys_row(R) * (uint32_t)gny() + (uint32_t)j0) & 3u);
    }

    // Bulk copies of one row window (columns j0 - 4 .., 128 of them, clipped to the grid) into dst; returns the
    // bytes.  A row that does not start 16-byte aligned is copied from the boundary before it, rounded up to 16
    // bytes (the data then starts at dst + row_off).
    __device__ __forceinline__ uint32_t window(float *dst, const float *src_row, uint64_t *bar, bool issue) const {
        if constexpr (!VEC) {
            const int col = j0 - 4;
            const int len = min(128, gny() - col);
            const int off = (int)(((uintptr_t)(src_row + col) >> 2) & 3u);
            const uint32_t bytes = (uint32_t)((len + off + 3) & ~3) * 4u;
            if (issue) tb_bulk_g2s(dst, src_row + col - off, bytes, bar);
            return bytes;
        }
        uint32_t bytes = 0;
        const int ny = gny();
        int remaining = 128, d = 0, col = PY ? tb_wrap(j0 - 4, ny) : j0 - 4;
        while (remaining > 0 && col < ny) {
            const int len = min(remaining, ny - col);
            if (issue) tb_bulk_g2s(dst + d, src_row + col, (uint32_t)len * 4u, bar);
            bytes += (uint32_t)len * 4u;
            d += len;
            remaining -= len;
            if (!PY) break;
            col = 0;
        }
        return bytes;
    }

    // lane 0: stage stream row R
    __device__ __forceinline__ void issue_row(int R) {
        const int k = R - r_begin;
        const int fs = k % tb_field_slots(), cs = k % tb_coef_slots(T);
        uint64_t *bar = sm_bar + fs;
        const size_t base = (size_t)phys_row(R) * (size_t)gny();
        const float *e_in = ptr(ez_in, p.ez_in);
        // every array of the row has the same alignment (the arrays start 256-byte aligned), so the same byte count
        const uint32_t bytes = vec ? row_bytes : window(nullptr, e_in + base, nullptr, false);
        tb_mbar_expect_tx(bar, bytes * (CA ? 5u : 4u));
        float *f = sm_fields + fs * (3 * IP_ROW);
        window(f, e_in + base, bar, true);
        window(f + IP_ROW, ptr(hx_in, p.hx_in) + base, bar, true);
        window(f + 2 * IP_ROW, ptr(hy_in, p.hy_in) + base, bar, true);
        window(sm_cb + cs * IP_ROW, ptr(cbp, p.cb) + base, bar, true);
        if (CA) window(sm_ca + cs * IP_ROW, ptr(cap, p.ca) + base, bar, true);
    }

    // The lane's four floats of a staged window: q = window + 4 lane (16-byte aligned), off = the row's offset
    // (row_off).  An aligned row is one 16-byte read; otherwise two aligned 16-byte reads (conflict-free, where four
    // scalar reads at a 16-byte lane stride would hit each bank four times) and a shift by the offset, which is the
    // same for the whole warp.
    __device__ __forceinline__ float4 ld_win(const float *q, int off) const {
        const float4 a = *reinterpret_cast<const float4 *>(q);
        if constexpr (VEC) {
            return a;
        } else {
            const float4 b = *reinterpret_cast<const float4 *>(q + 4);
            switch (off) {
                case 0: return a;
                case 1: return make_float4(a.y, a.z, a.w, b.x);
                case 2: return make_float4(a.z, a.w, b.x, b.y);
                default: return make_float4(a.w, b.x, b.y, b.z);
            }
        }
    }

    template <int PH>
    __device__ __forceinline__ bool take_row(int R) {
        const int k = R - r_begin;
        const int fs = k % tb_field_slots();
        if (R <= r_end && !tb_mbar_wait(sm_bar + fs, (uint32_t)((k / tb_field_slots()) & 1))) return false;
        const float *f = sm_fields + fs * (3 * IP_ROW) + lane * 4;
        float4 e, hx, hy;
        if constexpr (VEC) {
            e = ld_win(f, 0);
            hx = ld_win(f + IP_ROW, 0);
            hy = ld_win(f + 2 * IP_ROW, 0);
        } else {   // the three windows of a row share its offset: one shift for all
            const float4 a0 = *reinterpret_cast<const float4 *>(f), b0 = *reinterpret_cast<const float4 *>(f + 4);
            const float4 a1 = *reinterpret_cast<const float4 *>(f + IP_ROW);
            const float4 b1 = *reinterpret_cast<const float4 *>(f + IP_ROW + 4);
            const float4 a2 = *reinterpret_cast<const float4 *>(f + 2 * IP_ROW);
            const float4 b2 = *reinterpret_cast<const float4 *>(f + 2 * IP_ROW + 4);
            switch (row_off(R)) {
                case 0: e = a0, hx = a1, hy = a2; break;
                case 1:
                    e = make_float4(a0.y, a0.z, a0.w, b0.x), hx = make_float4(a1.y, a1.z, a1.w, b1.x);
                    hy = make_float4(a2.y, a2.z, a2.w, b2.x);
                    break;
                case 2:
                    e = make_float4(a0.z, a0.w, b0.x, b0.y), hx = make_float4(a1.z, a1.w, b1.x, b1.y);
                    hy = make_float4(a2.z, a2.w, b2.x, b2.y);
                    break;
                default:
                    e = make_float4(a0.w, b0.x, b0.y, b0.z), hx = make_float4(a1.w, b1.x, b1.y, b1.z);
                    hy = make_float4(a2.w, b2.x, b2.y, b2.z);
                    break;
            }
        }
        E[PH][0][0] = make_float2(e.x, e.y);
        E[PH][0][1] = make_float2(e.z, e.w);
        Hx[PH][0][0] = make_float2(hx.x, hx.y);
        Hx[PH][0][1] = make_float2(hx.z, hx.w);
        Hy[PH][0][0] = make_float2(hy.x, hy.y);
        Hy[PH][0][1] = make_float2(hy.z, hy.w);
        return true;
    }

    // Line sources of this tile's cone (rare): ez += value * profile on the line cells, per component.
    template <int S>
    __device__ __forceinline__ void inject(int ip, float2 (&ez)[2]) const {
        for (uint32_t lines = line_mask; lines; lines &= lines - 1) {
            const int l = __ffs(lines) - 1;
            const TBLine &L = p.lines[l];
            if (!in_grid0) continue;
            // the step's value is read only where this row holds a cell of the line
            bool hit = false;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int j = jp0 + c;
                const int along = L.axis == 0 ? ip : j, across = L.axis == 0 ? j : ip;
                hit = hit || (across == L.position && along >= L.lo && along < L.hi);
            }
            if (!hit) continue;
            const float value = p.line_values[(size_t)l * p.values_stride + p.k0 + (S - 1)];
            if (value == 0.0f) continue;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int j = jp0 + c;
                const int along = L.axis == 0 ? ip : j, across = L.axis == 0 ? j : ip;
                if (across == L.position && along >= L.lo && along < L.hi) {
                    float &v = (c & 1) ? ez[c >> 1].y : ez[c >> 1].x;
                    v = __fadd_rn(v, __fmul_rn(value, L.profile[along - L.lo]));
                }
            }
        }
    }

    template <int S>
    __device__ __forceinline__ void sample(int i, int ip, const float2 (&ez)[2], const float2 (&hxn)[2],
                                           const float2 (&hyn)[2]) const {
        const int slot = __popc(sample_mask & ((1u << (S - 1)) - 1u));
        for (uint32_t mons = mon_mask; mons; mons &= mons - 1) {
            const TBMon &M = p.mons[__ffs(mons) - 1];
            const int n = M.hi - M.lo;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (!((own >> c) & 1u)) continue;
                const int j = jp0 + c;
                const float e = (c & 1) ? ez[c >> 1].y : ez[c >> 1].x;
                if (M.normal_axis == 0) {
                    if (ip == M.position && j >= M.lo && j < M.hi) {
                        M.stage[(slot * 2) * n + (j - M.lo)] = e;
                        M.stage[(slot * 2 + 1) * n + (j - M.lo)] = (c & 1) ? hyn[c >> 1].y : hyn[c >> 1].x;
                    }
                } else if (j == M.position && ip >= M.lo && ip < M.hi) {
                    M.stage[(slot * 2) * n + (ip - M.lo)] = e;
                    M.stage[(slot * 2 + 1) * n + (ip - M.lo)] = (c & 1) ? hxn[c >> 1].y : hxn[c >> 1].x;
                }
            }
        }
    }

    // Step S of row i = r - S (every row of the stream window, see fdtd2d_tb.cuh).
    template <int PH, int S>
    __device__ __forceinline__ void stage(int r) {
        constexpr int Q = PH ^ 1;
        const int i = r - S;
        const int ip = phys_row(i);
        const int cs = (i - r_begin + tb_coef_slots(T)) % tb_coef_slots(T);
        const int co = lane * 4, off = row_off(i);
        const float4 cbv = ld_win(sm_cb + cs * IP_ROW + co, off);
        const float2 cb[2] = {make_float2(cbv.x, cbv.y), make_float2(cbv.z, cbv.w)};
        float2 ca[2];
        if constexpr (CA) {
            const float4 cav = ld_win(sm_ca + cs * IP_ROW + co, off);
            ca[0] = make_float2(cav.x, cav.y);
            ca[1] = make_float2(cav.z, cav.w);
        }
        const float2 db2 = pair(this->db2, p.db_u), ixh2 = pair(this->ixh2, p.s_inv_dx_h);
        const float2 iyh2 = pair(this->iyh2, p.s_inv_dy_h), ixe2 = pair(this->ixe2, p.s_inv_dx_e);
        const float2 iye2 = pair(this->iye2, p.s_inv_dy_e);
        const float2(&eq)[2] = E[Q][S - 1];    // E^(S-1) of row i
        const float2(&eu)[2] = E[PH][S - 1];   // E^(S-1) of row i + 1
        // ---- H^S (fdtd_ez_2d_kernels.py:41-47 with da = 1)
        const float e_right_last = __shfl_down_sync(0xffffffffu, eq[0].x, 1);
        const float2 eright[2] = {make_float2(eq[0].y, eq[1].x), make_float2(eq[1].y, e_right_last)};
        float2 hxn[2], hyn[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            hxn[k] = ip_sub_p(Hx[Q][S - 1][k], ip_mul(ip_mul(db2, ip_sub(eright[k], eq[k])), iyh2));
            hyn[k] = ip_add_p(Hy[Q][S - 1][k], ip_mul(ip_mul(db2, ip_sub(eu[k], eq[k])), ixh2));
        }
        // ---- E^S (fdtd_ez_2d_kernels.py:107-120)
        float hx_left_first = __shfl_up_sync(0xffffffffu, hxn[1].y, 1);
        if (PY && wrap_lo0) hx_left_first = tb_lo_wrap(hx_left_first);
        const float2 hxl[2] = {make_float2(hx_left_first, hxn[0].x), make_float2(hxn[0].y, hxn[1].x)};
        float2 hyd[2] = {Hy[Q][S][0], Hy[Q][S][1]};   // H_y^S of row i - 1
        if (PX && ip == 0) {
#pragma unroll
            for (int k = 0; k < 2; ++k) hyd[k] = make_float2(tb_lo_wrap(hyd[k].x), tb_lo_wrap(hyd[k].y));
        }
        float2 ez[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float2 curl = ip_sub_p(ip_mul(ip_sub(hyn[k], hyd[k]), ixe2), ip_mul(ip_sub(hxn[k], hxl[k]), iye2));
            ez[k] = ip_add_p(CA ? ip_mul(ca[k], eq[k]) : eq[k], ip_mul(cb[k], curl));
        }
        if (line_mask) inject<S>(ip, ez);
        if (mon_mask && ((sample_mask >> (S - 1)) & 1u) && i >= i0 && i < i1) sample<S>(i, ip, ez, hxn, hyn);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            E[PH][S][k] = ez[k];
            Hx[PH][S][k] = hxn[k];
            Hy[PH][S][k] = hyn[k];
        }
    }

    template <int PH>
    __device__ __forceinline__ void store(int r) {
        const int i = r - T;
        if (i < i0 || i >= i1) return;
        const size_t base = (size_t)phys_row(i) * (size_t)gny() + jp0;
        float *ez_out = ptr(this->ez_out, p.ez_out), *hx_out = ptr(this->hx_out, p.hx_out);
        float *hy_out = ptr(this->hy_out, p.hy_out);
        if (own == 0xFu && vec) {
            *reinterpret_cast<float4 *>(ez_out + base) =
                make_float4(E[PH][T][0].x, E[PH][T][0].y, E[PH][T][1].x, E[PH][T][1].y);
            *reinterpret_cast<float4 *>(hx_out + base) =
                make_float4(Hx[PH][T][0].x, Hx[PH][T][0].y, Hx[PH][T][1].x, Hx[PH][T][1].y);
            *reinterpret_cast<float4 *>(hy_out + base) =
                make_float4(Hy[PH][T][0].x, Hy[PH][T][0].y, Hy[PH][T][1].x, Hy[PH][T][1].y);
        } else if (own == 0xFu) {   // a misaligned row: four scalar stores per field, no per-column tests
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                ez_out[base + 2 * k] = E[PH][T][k].x, ez_out[base + 2 * k + 1] = E[PH][T][k].y;
                hx_out[base + 2 * k] = Hx[PH][T][k].x, hx_out[base + 2 * k + 1] = Hx[PH][T][k].y;
                hy_out[base + 2 * k] = Hy[PH][T][k].x, hy_out[base + 2 * k + 1] = Hy[PH][T][k].y;
            }
        } else if (own) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (!((own >> c) & 1u)) continue;
                ez_out[base + c] = (c & 1) ? E[PH][T][c >> 1].y : E[PH][T][c >> 1].x;
                hx_out[base + c] = (c & 1) ? Hx[PH][T][c >> 1].y : Hx[PH][T][c >> 1].x;
                hy_out[base + c] = (c & 1) ? Hy[PH][T][c >> 1].y : Hy[PH][T][c >> 1].x;
            }
        }
    }

    template <int PH, int S>
    __device__ __forceinline__ void stages_from(int r) {
        if constexpr (S <= T) {
            stage<PH, S>(r);
            stages_from<PH, S + 1>(r);
        }
    }

    template <int PH>
    __device__ __forceinline__ void iteration(int r) {
        if (!take_row<PH>(r)) {
            failed = true;
            return;
        }
        stages_from<PH, 1>(r);
        store<PH>(r);
        __syncwarp();
        if (lane == 0 && r + TB_AHEAD + 1 <= r_end) {
            tb_fence_proxy_async();
            issue_row(r + TB_AHEAD + 1);
        }
    }

    __device__ __forceinline__ void drain(int r_from) {
        for (int R = r_from; R <= min(r_end, r_from + TB_AHEAD); ++R) {
            const int k = R - r_begin;
            tb_mbar_wait(sm_bar + k % tb_field_slots(), (uint32_t)((k / tb_field_slots()) & 1));
        }
    }
};

// One warp's tile w of the interior plan p (tb_smem: the block's dynamic shared memory).
template <int T, bool CA, bool PX, bool PY, bool VEC, bool HELD>
__device__ __forceinline__ void ez2d_interior_tile(const TBParams &p, int w, unsigned char *tb_smem) {
    const int lane = threadIdx.x & 31;
    if (w >= p.n_tiles) return;   // whole warps leave together
    int rect = 0;
    for (int q = 1; q < p.n_rects; ++q)
        if (w >= p.rects[q].first_tile) rect = q;
    const TBRect R = p.rects[rect];
    const int t = w - R.first_tile;
    const int tc = t % R.tiles_c, tr = t / R.tiles_c;

    IPWarp<T, CA, PX, PY, VEC, HELD> W(p);
    W.lane = lane;
    W.nx = p.nx;
    W.ny = p.ny;
    W.j0 = R.c0 + tc * p.tile_w;
    W.j1 = min(W.j0 + p.tile_w, R.c1);
    W.i0 = R.r0 + tr * p.tile_rows;
    W.i1 = min(W.i0 + p.tile_rows, R.r1);
    W.r_begin = W.i0 - T;
    W.r_end = PX ? W.i1 - 1 + T : min(p.nx - 1, W.i1 - 1 + T);
    W.jl0 = W.j0 - 4 + lane * 4;
    W.jp0 = PY ? tb_wrap(W.jl0, p.ny) : W.jl0;
    W.in_grid0 = PY || (W.jl0 >= 0 && W.jl0 < p.ny);
    W.wrap_lo0 = PY && W.jp0 == 0;
    W.own = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (W.jl0 + c >= W.j0 && W.jl0 + c < W.j1) W.own |= 1u << c;
    W.db2 = make_float2(p.db_u, p.db_u);
    W.ixh2 = make_float2(p.s_inv_dx_h, p.s_inv_dx_h);
    W.ixe2 = make_float2(p.s_inv_dx_e, p.s_inv_dx_e);
    W.iyh2 = make_float2(p.s_inv_dy_h, p.s_inv_dy_h);
    W.iye2 = make_float2(p.s_inv_dy_e, p.s_inv_dy_e);
    W.ez_in = p.ez_in;
    W.hx_in = p.hx_in;
    W.hy_in = p.hy_in;
    W.cbp = p.cb;
    W.cap = p.ca;
    W.ez_out = p.ez_out;
    W.hx_out = p.hx_out;
    W.hy_out = p.hy_out;
    W.sample_mask = p.sample_mask;
    // line sources that can reach the cone, flux lines among the outputs
    {
        const int c0 = W.j0 - 4, c1 = W.j0 + 124;
        uint32_t lm = 0, mm = 0;
        for (int l = 0; l < p.n_lines; ++l) {
            const TBLine &L = p.lines[l];
            bool hit;
            if (PX || PY) hit = true;
            else if (L.axis == 0) hit = L.position >= c0 && L.position < c1 && L.hi > W.r_begin && L.lo <= W.r_end;
            else hit = L.position >= W.r_begin && L.position <= W.r_end && L.hi > c0 && L.lo < c1;
            if (hit) lm |= 1u << l;
        }
        for (int q = 0; q < p.n_mons; ++q) {
            const TBMon &M = p.mons[q];
            const bool hit = M.normal_axis == 0
                                 ? (M.position >= W.i0 && M.position < W.i1 && M.hi > W.j0 && M.lo < W.j1)
                                 : (M.position >= W.j0 && M.position < W.j1 && M.hi > W.i0 && M.lo < W.i1);
            if (hit) mm |= 1u << q;
        }
        W.line_mask = lm;
        W.mon_mask = p.sample_mask ? mm : 0u;
    }
#pragma unroll
    for (int ph = 0; ph < 2; ++ph)
#pragma unroll
        for (int s = 0; s <= T; ++s)
#pragma unroll
            for (int k = 0; k < 2; ++k) W.E[ph][s][k] = W.Hx[ph][s][k] = W.Hy[ph][s][k] = make_float2(0.0f, 0.0f);

    unsigned char *mine = tb_smem + (threadIdx.x >> 5) * ip_warp_smem_bytes(T, CA);
    W.sm_fields = reinterpret_cast<float *>(mine);
    W.sm_cb = W.sm_fields + tb_field_slots() * 3 * IP_ROW;
    W.sm_ca = W.sm_cb + tb_coef_slots(T) * IP_ROW;
    W.sm_bar = reinterpret_cast<uint64_t *>(W.sm_cb + tb_coef_slots(T) * IP_ROW * (CA ? 2 : 1));
    W.row_bytes = W.vec ? W.window(nullptr, nullptr, nullptr, false) : 0u;
    if (lane == 0) {
        for (int q = 0; q < tb_field_slots(); ++q) tb_mbar_init(W.sm_bar + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tb_fence_proxy_async();
        for (int Rr = W.r_begin; Rr <= min(W.r_end, W.r_begin + TB_AHEAD); ++Rr) W.issue_row(Rr);
    }
    __syncwarp();
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

template <int T, bool CA, bool PX, bool PY, bool VEC>
__global__ void __launch_bounds__(TB_WARPS * 32, 4) ez2d_interior_kernel(const TBParams p) {
    extern __shared__ __align__(16) unsigned char tb_smem[];
    if (p.stall_probe_ns && blockIdx.x == 0 && threadIdx.x < 32) {
        // test hook: a wait on an mbarrier that no copy and no thread ever completes, bounded like every real wait;
        // when it runs out the warp sets the error flag and leaves its tile unwritten, as a real timeout does (it has
        // issued no copy yet, so nothing is in flight)
        __shared__ uint64_t probe_bar;
        if (threadIdx.x == 0) {
            tb_mbar_init(&probe_bar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
        bool done = tb_mbar_try_wait(&probe_bar, 0);
        const uint64_t t0 = tb_globaltimer();
        while (!done && tb_globaltimer() - t0 <= (uint64_t)p.stall_probe_ns) done = tb_mbar_try_wait(&probe_bar, 0);
        if (!__all_sync(0xffffffffu, done)) {
            if (threadIdx.x == 0) atomicExch(p.err, 1);
            return;
        }
    }
    ez2d_interior_tile<T, CA, PX, PY, VEC, true>(p, blockIdx.x * TB_WARPS + (threadIdx.x >> 5), tb_smem);
}

// Several simulations in one launch: warp g runs tile g - tile_start[job] of jobs[job], tile_start ascending with
// tile_start[n_jobs] = the total (every job shares T and the template configuration).
static_assert(sizeof(TBParams) % 16 == 0, "TBParams is staged per warp in shared memory as 32-bit words");

template <int T, bool CA, bool PX, bool PY, bool VEC>
__global__ void __launch_bounds__(TB_WARPS * 32, 4) ez2d_interior_batch_kernel(const TBParams *__restrict__ jobs,
                                                                         const int *__restrict__ tile_start,
                                                                         int n_jobs) {
    extern __shared__ __align__(16) unsigned char tb_smem[];
    const int g = blockIdx.x * TB_WARPS + (threadIdx.x >> 5);
    if (g >= tile_start[n_jobs]) return;
    int job = 0;
    while (job + 1 < n_jobs && g >= tile_start[job + 1]) ++job;
    // the warp's job parameters into shared memory (after the block's staging rings): the tile code reads them
    // there, not from global memory
    TBParams *mine = reinterpret_cast<TBParams *>(tb_smem + TB_WARPS * ip_warp_smem_bytes(T, CA)) +
                     (threadIdx.x >> 5);
    const uint32_t *src = reinterpret_cast<const uint32_t *>(jobs + job);
    uint32_t *dst = reinterpret_cast<uint32_t *>(mine);
    for (int w = threadIdx.x & 31; w < (int)(sizeof(TBParams) / 4); w += 32) dst[w] = src[w];
    __syncwarp();
    ez2d_interior_tile<T, CA, PX, PY, VEC, false>(*mine, g - tile_start[job], tb_smem);
}
