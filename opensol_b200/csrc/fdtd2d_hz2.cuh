// Two-step interior kernel of the fused H_z step (no conductivity, no magnetic cells, rows a multiple of 4 cells): two
// Yee steps per launch for the cells of an interior box, reading field set a and writing set b, with every
// intermediate value in registers.
//
// The same warp strips, lanes and TMA row ring as hz2d_interior_kernel, and the same arithmetic term for term, in a
// skewed two-stage pipeline: while streaming row r, stage 1 makes step 1 of row r (H_z^1(r), E_x^1(r)) and E_y^1 of
// row r - 1; stage 2 makes step 2 one row behind (H_z^2(r - 1), E_x^2(r - 1), E_y^2(r - 2)).  A block streams rows
// r0 - 1 .. r1 + 1 and stores step 2 of its rows [r0, r1).  Step 2's columns need step 1 one column beyond the strip
// on each side: a warp holds 128 columns and stores the middle 120, its first and last lanes computing the halo
// columns with the same code as the rest.  The sheet sources of each step are added to the E values of that step,
// the halo columns' included.  The faces' cb are read from the
// stored coefficient arrays (hz2d_face_coefficients_kernel: with no conductivity the denominator is exactly 1, so
// they are the lossless form's dt / (face eps eps0) as well), staged with the fields, and kept for stage 2.  The host
// chooses the box so that every update in this cone is the plain one (no CPML row, edge or wrap): the single-step box
// less one row and four columns on each side.  Every wait is bounded (the ring's tb_mbar_wait).
#pragma once

#include "fdtd2d_hz.cuh"

// Sheet sources of step `k` on the lane's four E_x faces of row r (columns jt .. jt + 3; axis 0 lines: faces
// (r, position), r in [lo, hi)) and four E_y faces of row re (axis 1 lines: faces (position, j), j in [lo, hi)), added
// in line order after the update, a zero value skipped, as hz_plain_e adds them; each line is tested once per row.
__device__ __forceinline__ void hz2_src_x4(const Hz2DParams &p, int64_t k, int r, int jt, float (&v)[4]) {
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &L = p.lines[l];
        if (L.axis != 0 || L.position < jt || L.position >= jt + 4 || r < L.lo || r >= L.hi) continue;
        const float value = p.line_values[(size_t)l * p.values_stride + k];
        if (value == 0.0f) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (jt + c == L.position) v[c] += value * L.profile[r - L.lo];
    }
}
__device__ __forceinline__ void hz2_src_y4(const Hz2DParams &p, int64_t k, int re, int jt, float (&v)[4]) {
    for (int l = 0; l < p.n_lines; ++l) {
        const LineSrcDev &L = p.lines[l];
        if (L.axis != 1 || L.position != re || jt + 3 < L.lo || jt >= L.hi) continue;
        const float value = p.line_values[(size_t)l * p.values_stride + k];
        if (value == 0.0f) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (jt + c >= L.lo && jt + c < L.hi) v[c] += value * L.profile[jt + c - L.lo];
    }
}

// One plain H_z update: da H + db ((E_x - E_x left) iye - (E_y - E_y below) ixe).
__device__ __forceinline__ float hz2_h(float da, float db, float h, float ex, float ex_left, float ey, float ey_below,
                                       float iye, float ixe) {
    const float dex = ex - ex_left;
    const float dey = ey - ey_below;
    float curl = dex * iye;
    curl -= dey * ixe;
    return da * h + db * curl;
}

// Plain E_x (ca = 1): 1 E_x + cb (H_z right - H_z) iyh.
__device__ __forceinline__ float hz2_ex(float ex, float bx, float h, float h_right, float iyh) {
    const float dx = h_right - h;
    return 1.0f * ex + bx * dx * iyh;
}

// Plain E_y (ca = 1) of row re: 1 E_y - cb (H_z above - H_z) ixh.
__device__ __forceinline__ float hz2_ey(float ey, float by, float h, float h_above, float ixh) {
    const float dy = h_above - h;
    return 1.0f * ey - by * dy * ixh;
}

// Row staging of the two-step kernel: five arrays per row (H_z, E_x, E_y in, the stored face cb of E_x and of E_y),
// each a window of HZ_WIN columns from jw - 8 (clipped to the grid), in a per-warp ring of HZ_SLOTS slots by 1D bulk
// copies (cp.async.bulk, no multicast).
constexpr int HZ2_ARRAYS = 5;
constexpr int HZ2_OUT = 120;   // output columns of a warp strip: lanes 1..30 (lanes 0 and 31 are halo lanes)
__host__ __device__ constexpr int hz2_warp_smem_bytes() { return HZ_SLOTS * HZ2_ARRAYS * HZ_WIN * 4 + HZ_SLOTS * 8; }

struct Hz2Stage {
    float *ring;          // [slot][array][HZ_WIN]
    uint64_t *bar;        // [slot]
    int jw, c_lo, c_hi;   // window columns [c_lo, c_hi) of the grid at slot offset c_lo - (jw - 8)

    __device__ __forceinline__ float *slot(int s, int a) const { return ring + (s * HZ2_ARRAYS + a) * HZ_WIN; }

    // lane 0: copy row r into slot s
    __device__ __forceinline__ void issue(const Hz2DParams &p, int r, int s) const {
        const uint32_t bytes = (uint32_t)(c_hi - c_lo) * 4u;
        tb_mbar_expect_tx(bar + s, HZ2_ARRAYS * bytes);
        const size_t src = (size_t)r * p.ny + c_lo;
        const int off = c_lo - (jw - 8);
        tb_bulk_g2s(slot(s, 0) + off, p.hz_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 1) + off, p.ex_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 2) + off, p.ey_in + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 3) + off, p.cb_x + src, bytes, bar + s);
        tb_bulk_g2s(slot(s, 4) + off, p.cb_y + src, bytes, bar + s);
    }
};

// Lane l holds columns jw - 4 + 4 l .. + 3, the whole warp the same vector code: lanes 1..30 own the strip's 120
// output columns [jw, j_end); lane 0 (columns jw - 4 .. jw - 1) and the lane after the last output lane are halo
// lanes whose step-1 values at jw - 1 and j_end, j_end + 1 (and step-2 H_z at j_end) the output lanes read by
// shuffle; a halo lane's other values miss a neighbour and are never read.  Only output columns are stored.
__global__ void __launch_bounds__(HZ_THREADS, 4) hz2d_interior2_kernel(const Hz2DParams p, int32_t *err) {
    extern __shared__ __align__(16) unsigned char hz_smem[];
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int jw = p.jc0 + (blockIdx.x * (HZ_THREADS / 32) + warp) * HZ2_OUT;
    if (jw >= p.jc1) return;   // whole warp (its barriers are never used)
    const int jt = jw - 4 + 4 * lane;
    const int ny = p.ny;
    const int r0 = p.ia + blockIdx.y * p.rows_per_cta;
    if (r0 >= p.ib) return;
    const int r1 = min(p.ib, r0 + p.rows_per_cta);
    const int j_end = min(jw + HZ2_OUT, p.jc1);          // the strip's output columns [jw, j_end)
    const bool out_lane = jt >= jw && jt < j_end;
    const int R0 = r0 - 1, R1 = r1 + 1;                  // streamed rows R0 .. R1

    Hz2Stage st;
    {
        unsigned char *mine = hz_smem + warp * hz2_warp_smem_bytes();
        st.ring = reinterpret_cast<float *>(mine);
        st.bar = reinterpret_cast<uint64_t *>(mine + HZ_SLOTS * HZ2_ARRAYS * HZ_WIN * 4);
        st.jw = jw;
        st.c_lo = max(jw - 8, 0);
        st.c_hi = min(jw + 128, ny);
        if (lane == 0) {
            for (int s = 0; s < HZ_SLOTS; ++s) tb_mbar_init(st.bar + s, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            tb_fence_proxy_async();
            for (int R = R0; R <= min(R1, R0 + HZ_AHEAD); ++R) st.issue(p, R, (R - R0) % HZ_SLOTS);
        }
        __syncwarp();
    }

    float iye[4], iyh[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int jc = min(max(jt + c, 0), ny - 1);
        iye[c] = __ldg(p.iye + jc);
        iyh[c] = __ldg(p.iyh + jc);
    }
    const float da = p.da_u, db = p.db_u;

    // carried state (stage 1 of the previous row, stage 2 of the row before) and the face cb of earlier rows
    float ey0p[4] = {}, h1p[4] = {}, e1xp[4] = {}, e1ypp[4] = {}, h2p[4] = {};
    float cbxp[4] = {}, cbyp[4] = {}, cbypp[4] = {};   // cb of E_x of row r - 1, of E_y of rows r - 1 and r - 2
    {   // old E_y of row R0 - 1
        const size_t row = (size_t)(R0 - 1) * ny;
#pragma unroll
        for (int c = 0; c < 4; ++c) ey0p[c] = __ldg(p.ey_in + row + min(max(jt + c, 0), ny - 1));
    }
    const int o = 4 + 4 * lane;   // the lane's first column in a window (window column 0 = grid column jw - 8)

    for (int r = R0; r <= R1; ++r) {
        const int k = r - R0, s = k % HZ_SLOTS;
        if (!tb_mbar_wait(st.bar + s, (uint32_t)((k / HZ_SLOTS) & 1))) {
            if (lane == 0) atomicExch(err, 1);
            for (int q = r; q <= min(R1, r + HZ_AHEAD); ++q) {   // copies still in flight, this row's included
                const int kq = q - R0;
                tb_mbar_wait(st.bar + kq % HZ_SLOTS, (uint32_t)((kq / HZ_SLOTS) & 1));
            }
            return;
        }
        float hzo[4], exo[4], eyo[4], cbx[4], cby[4];
        {
            const float4 a = *reinterpret_cast<const float4 *>(st.slot(s, 0) + o);
            const float4 bx = *reinterpret_cast<const float4 *>(st.slot(s, 1) + o);
            const float4 by = *reinterpret_cast<const float4 *>(st.slot(s, 2) + o);
            const float4 cx = *reinterpret_cast<const float4 *>(st.slot(s, 3) + o);
            const float4 cy = *reinterpret_cast<const float4 *>(st.slot(s, 4) + o);
            hzo[0] = a.x, hzo[1] = a.y, hzo[2] = a.z, hzo[3] = a.w;
            exo[0] = bx.x, exo[1] = bx.y, exo[2] = bx.z, exo[3] = bx.w;
            eyo[0] = by.x, eyo[1] = by.y, eyo[2] = by.z, eyo[3] = by.w;
            cbx[0] = cx.x, cbx[1] = cx.y, cbx[2] = cx.z, cbx[3] = cx.w;
            cby[0] = cy.x, cby[1] = cy.y, cby[2] = cy.z, cby[3] = cy.w;
        }
        const float ex_l0 = st.slot(s, 1)[o - 1];   // old E_x left of the lane (lane 0: from the window)
        __syncwarp();
        if (lane == 0 && r + HZ_AHEAD + 1 <= R1) {
            tb_fence_proxy_async();
            st.issue(p, r + HZ_AHEAD + 1, s);
        }

        // ---- stage 1: step 1 of row r (H_z, E_x) and E_y of row r - 1
        const float ixe = __ldg(p.ixe + r);
        float h1[4];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            h1[c] = hz2_h(da, db, hzo[c], exo[c], c == 0 ? ex_l0 : exo[c - 1], eyo[c], ey0p[c], iye[c], ixe);
        const float h1_next = __shfl_down_sync(FULL, h1[0], 1);   // H_z^1 right of the lane (lane 31: unused)
        const int64_t k1 = p.k_step, k2 = p.k_step + 1;
        float e1x[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) e1x[c] = hz2_ex(exo[c], cbx[c], h1[c], c < 3 ? h1[c + 1] : h1_next, iyh[c]);
        if (p.n_lines) hz2_src_x4(p, k1, r, jt, e1x);
        float e1y[4] = {};
        if (r > R0) {   // E_y^1 of row r - 1 (rows r0 - 1 .. r1), with that row's stored cb
            const int re = r - 1;
            const float ixh = __ldg(p.ixh + re);
#pragma unroll
            for (int c = 0; c < 4; ++c) e1y[c] = hz2_ey(ey0p[c], cbyp[c], h1p[c], h1[c], ixh);
            if (p.n_lines) hz2_src_y4(p, k1, re, jt, e1y);
        }

        // ---- stage 2: step 2 of row r - 1 (H_z, E_x) and E_y of row r - 2
        float h2[4] = {};
        if (r >= r0 + 1) {
            const int rs = r - 1;
            const float ixe_s = __ldg(p.ixe + rs);
            const float e1x_left = __shfl_up_sync(FULL, e1xp[3], 1);   // lane 0: unused
#pragma unroll
            for (int c = 0; c < 4; ++c)
                h2[c] = hz2_h(da, db, h1p[c], e1xp[c], c == 0 ? e1x_left : e1xp[c - 1], e1y[c], e1ypp[c], iye[c],
                              ixe_s);
            const float h2_next = __shfl_down_sync(FULL, h2[0], 1);
            if (rs < r1 && out_lane) {   // rows r0 .. r1 - 1 are stored; row r1 is the halo of E_y
                float e2x[4];
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    e2x[c] = hz2_ex(e1xp[c], cbxp[c], h2[c], c < 3 ? h2[c + 1] : h2_next, iyh[c]);
                if (p.n_lines) hz2_src_x4(p, k2, rs, jt, e2x);
                const size_t row = (size_t)rs * ny + jt;
                hz_st4<true>(p.hz_out, row, h2);
                hz_st4<true>(p.ex_out, row, e2x);
            }
            if (r >= r0 + 2 && out_lane) {   // E_y^2 of row r - 2
                const int re = r - 2;
                const float ixh = __ldg(p.ixh + re);
                float e2y[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) e2y[c] = hz2_ey(e1ypp[c], cbypp[c], h2p[c], h2[c], ixh);
                if (p.n_lines) hz2_src_y4(p, k2, re, jt, e2y);
                hz_st4<true>(p.ey_out, (size_t)re * ny + jt, e2y);
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            ey0p[c] = eyo[c];
            h2p[c] = h2[c];
            h1p[c] = h1[c];
            e1xp[c] = e1x[c];
            e1ypp[c] = e1y[c];
            cbxp[c] = cbx[c];
            cbypp[c] = cbyp[c];
            cbyp[c] = cby[c];
        }
    }
}
