// Lean staged form of the fused 3D step (em3d_fused_kernel's one-pass schedule and arithmetic, bit for bit): H^{n+1/2}
// then E^{n+1} of every cell of box `in` (every cell but the outermost layer of each axis), reading field set a and
// CPML psi set a, writing set b.
//
// A thread owns four adjacent k cells (one 16-byte vector of each array), so a warp row covers a tile of 128 cells
// starting on a multiple of 4; lane 0 also computes H_x and H_y of the cell below the tile (the halo cell, never
// stored) for its E.  A block is TY warp rows along j; warp 0 is the halo row j0 - 1 (H only).  The block streams a
// chunk of x planes, starting one plane early (the halo plane, H only).  Each plane of the tile arrives in shared
// memory by tiled tensor copies (cp.async.bulk.tensor, this GPU's own memory, no multicast) into a ring of RING plane
// slots, every box starting 4 cells before the tile: per E component TY + 1 rows x 136 cells (the halo cell, the
// tile, lane 31's k + 1 neighbour; the row above for the j + 1 neighbour), per H component TY rows x 132, the
// material ids TY + 1 rows x 144 from the 8-id boundary at or before the box.  Boxes that pass an edge of the grid are zero-filled by the copy and feed only
// results that are discarded.  Warp 0 issues the copies of plane i + RING - 1 into the slot of plane i - 1 after the
// plane's barrier, when no thread reads that slot any more.
//
// Arithmetic: products and plain differences in packed FP32 pairs (__fmul2_rn, __fadd2_rn; x - y as x + (-y)), and
// every add or subtract with a product operand per lane with the scalar __fadd_rn, which the code generator never
// merges into a fused multiply-add: each lane rounds exactly like em3d_h_kernel's / em3d_e_kernel's scalar code.
// With CA1 (every face's ca is 1: no conductivity, no perfect conductor) ca * E is E itself and is not multiplied;
// with HU every id has the same H coefficients (da_u, db_u) and the ids are not read for H.
// Neighbours along k come from the next / previous lane (shuffles) or, for lane 31's k + 1, from the staged box; along
// j from the staged row above (E) or the row below's new H through shared memory (one barrier per plane); along x
// from the next slot (E) or the thread's previous plane (H).  The coefficients of a face between two cells of one id
// come from the same-id table (one load per component when the four cells and their partners share one id); any other
// face (a material boundary, or a grid with non-uniform shares) takes em3d_face.  CPML terms: a vector of psi per x or
// y layer row (16-byte loads and stores), per cell on the z layers (the cells' z rows packed one byte each in a
// register, the rows' coefficients in shared memory).  Per-plane scalars (inverse spacings, x CPML rows and
// coefficients, face shares) are staged in shared memory when the block starts.  Stores are one 16-byte vector per
// array when every thread of the warp stores all four of its cells or none, per cell otherwise (box edges).  The
// dipoles are not added here: em3d_dipole_kernel adds them after the step.
//
// The box is every cell but the outermost layer of the x and y axes; along z it also holds rows 0 and nz - 1 when z is
// not periodic: E of row 0 reads 0 as the H below it (em3d_lo_diff returns F itself; F - 0 is the same bits), H of
// row nz - 1 reads the wrapped sample of row 0 (one load by the thread holding that row), and the E_z face of row
// nz - 1 is the cell's own.
//
// Every wait is bounded (2 s): a block whose wait runs out sets *err, waits (bounded) for its own copies in flight and
// returns; ids read from a slot are clamped below n_ids.  Needs nz a multiple of 4 and at least 144, ny at least
// TY + 1 (a tensor map's box may not be larger than the array), at most EM3D_LEAN_MAX_ZROWS z CPML rows and chunks of
// at most EM3D_LEAN_MAX_PLANES - 1 planes.
#pragma once

#include "fdtd3d_kernels.cuh"

constexpr int EM3D_LV = 4;                     // cells per thread along k
constexpr int EM3D_LTILE = 32 * EM3D_LV;       // cells of a warp row (128)

// Boxes of one plane: E and ids TY + 1 rows, H TY rows from the tile's first row (its halo row j0 - 1); with NX (no
// exchange: every warp computes the H of the row below its own) one more row of each.
template <int TY, bool NX = false>
struct Em3DLeanLayout {   // byte offsets inside one ring slot, every box on a 128-byte boundary
    static constexpr int WE = 136, WH = 132, WM = 144;
    static constexpr int ER = TY + 1 + (NX ? 1 : 0), HR = TY + (NX ? 1 : 0), MR = ER;   // box rows
    static constexpr int e_bytes = em3d_round128(ER * WE * 4);
    static constexpr int h_bytes = em3d_round128(HR * WH * 4);
    static constexpr int m_bytes = em3d_round128(MR * WM * 2);
    static constexpr int e_off = 0, h_off = 3 * e_bytes, m_off = h_off + 3 * h_bytes;
    static constexpr int slot = m_off + m_bytes;
    static constexpr uint32_t tx = (uint32_t)(3 * ER * WE * 4 + 3 * HR * WH * 4 + MR * WM * 2);
    static constexpr int xch = NX ? 0 : 2 * TY * 128 * 4;   // one parity of one exchanged H component
};

constexpr int EM3D_LEAN_MAX_PLANES = 64;       // x planes of one block's chunk, the halo plane included
constexpr int EM3D_LEAN_MAX_ZROWS = 255;       // z CPML rows (one byte per cell row index, 0xff: none)

// Shared memory of one lean block, every region on a 16-byte boundary (the ring on 128): ring, exchanged H (two
// parities), mbarriers, z CPML coefficients (b_h, g_h, b_e, g_e per z row; 16-byte vectors of four rows), per-plane
// scalars, the tile's z inverse spacings (H then E).
template <int TY, int RING, bool NX = false>
struct Em3DLeanSmem {
    static constexpr size_t xch = Em3DLeanLayout<TY, NX>::slot * (size_t)RING;
    static constexpr size_t bars = xch + 2 * (size_t)Em3DLeanLayout<TY, NX>::xch;
    static constexpr size_t zc = bars + (RING * sizeof(uint64_t) + 15) / 16 * 16;
    __host__ __device__ static constexpr size_t plane(int z_rows) { return zc + 16 * (size_t)z_rows; }
    __host__ __device__ static constexpr size_t kz(int z_rows) { return plane(z_rows) + EM3D_LEAN_MAX_PLANES * 40; }
    __host__ __device__ static constexpr size_t bytes(int z_rows) { return kz(z_rows) + 2 * EM3D_LTILE * 4; }
};

template <int TY, int RING, bool NX = false>
__host__ __device__ constexpr size_t em3d_lean_smem(int z_rows) {
    return Em3DLeanSmem<TY, RING, NX>::bytes(z_rows);
}

// Tensor maps of one lean launch: E and H components of the field set read, ids.
struct Em3DLeanMaps {
    CUtensorMap e[3], h[3], m;
};

__device__ __forceinline__ float2 lp_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 lp_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 ls_add(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 ls_sub(float2 a, float2 b) {
    return make_float2(__fadd_rn(a.x, -b.x), __fadd_rn(a.y, -b.y));
}
__device__ __forceinline__ float2 lp_dup(float v) { return make_float2(v, v); }

__device__ __forceinline__ void lv_lds(const float *ptr, float2 (&v)[2]) {
    const float4 t = *reinterpret_cast<const float4 *>(ptr);
    v[0] = make_float2(t.x, t.y);
    v[1] = make_float2(t.z, t.w);
}
__device__ __forceinline__ void lv_ldg(const float *ptr, float2 (&v)[2]) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(ptr));
    v[0] = make_float2(t.x, t.y);
    v[1] = make_float2(t.z, t.w);
}
__device__ __forceinline__ float lv_get(const float2 (&v)[2], int c) {
    return c == 0 ? v[0].x : (c == 1 ? v[0].y : (c == 2 ? v[1].x : v[1].y));
}
__device__ __forceinline__ void lv_set(float2 (&v)[2], int c, float x) {
    if (c == 0) v[0].x = x;
    else if (c == 1) v[0].y = x;
    else if (c == 2) v[1].x = x;
    else v[1].y = x;
}
// store the cells of `mask` (bit c: cell c): one 16-byte store when all four
__device__ __forceinline__ void lv_st(float *ptr, const float2 (&v)[2], unsigned mask) {
    if (mask == 0xFu) {
        *reinterpret_cast<float4 *>(ptr) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
        return;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (mask & (1u << c)) ptr[c] = lv_get(v, c);
}
__device__ __forceinline__ uint32_t lv_id(uint2 m, int c) {
    const uint32_t w = c < 2 ? m.x : m.y;
    return (c & 1) ? (w >> 16) : (w & 0xffffu);
}

// The cells k .. k + 3 shifted by one: k + 1 .. k + 4 (next = cell k + 4) and k - 1 .. k + 2 (prev = cell k - 1).
__device__ __forceinline__ void lv_up(const float2 (&v)[2], float next, float2 (&out)[2]) {
    out[0] = make_float2(v[0].y, v[1].x);
    out[1] = make_float2(v[1].y, next);
}
__device__ __forceinline__ void lv_down(const float2 (&v)[2], float prev, float2 (&out)[2]) {
    out[0] = make_float2(prev, v[0].x);
    out[1] = make_float2(v[0].y, v[1].x);
}

// The seven copies of one plane into one slot (warp 0; lane 0 arms the barrier first).
template <int TY, bool NX>
__device__ __forceinline__ void em3d_lean_issue(const Em3DLeanMaps &maps, unsigned char *slot, uint64_t *bar,
                                                int plane, int j_row0, int ke, int km, int lane) {
    using L = Em3DLeanLayout<TY, NX>;
    if (lane == 0) tb_mbar_expect_tx(bar, L::tx);
    __syncwarp();
    if (lane < 3) em3d_tensor_g2s(slot + L::e_off + lane * L::e_bytes, &maps.e[lane], ke, j_row0, plane, bar);
    else if (lane < 6) em3d_tensor_g2s(slot + L::h_off + (lane - 3) * L::h_bytes, &maps.h[lane - 3], ke, j_row0, plane,
                                       bar);
    else if (lane == 6) em3d_tensor_g2s(slot + L::m_off, &maps.m, km, j_row0, plane, bar);
}

// ca, cb of the face between ids a and b on one axis (the same-id table when the ids match and every share is 0.5).
__device__ __forceinline__ void em3d_lean_face(const Em3DParams &p, const float *t_same, int comp, const float *t_eps,
                                               uint32_t a, uint32_t b, float wa, float wb, float &ca, float &cb) {
    if (p.same_ok && a == b) {
        ca = __ldg(t_same + (2 * comp) * p.n_ids + a);
        cb = __ldg(t_same + (2 * comp + 1) * p.n_ids + a);
        return;
    }
    em3d_face(p, t_eps, (uint16_t)a, (uint16_t)b, wa, wb, ca, cb);
}

// Per-plane scalars of one block's chunk, staged in shared memory at the start: inverse spacings, the x CPML rows
// and their coefficients, the x face shares.
struct Em3DLeanPlane {
    float ihx, iex, bh, gh, be, ge, wl, wu;
    int32_t rh, re;
};

// Store the cells of `mask` (bit c: cell c); vec: every thread of the warp stores all four cells or none.
__device__ __forceinline__ void lv_store(float *ptr, const float2 (&v)[2], unsigned mask, bool vec) {
    if (vec) {
        if (mask) *reinterpret_cast<float4 *>(ptr) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
        return;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (mask & (1u << c)) ptr[c] = lv_get(v, c);
}

template <int TY, int RING, int MINB, bool CA1, bool HU, bool EARLY, bool NX>
__global__ void __launch_bounds__(32 * TY, MINB)
    em3d_lean_kernel(const Em3DParams p, const Em3DBox in, const __grid_constant__ Em3DLeanMaps maps) {
    using L = Em3DLeanLayout<TY, NX>;
    extern __shared__ __align__(128) unsigned char em3d_lean_smem_buf[];
    unsigned char *const ring = em3d_lean_smem_buf;
    using S = Em3DLeanSmem<TY, RING, NX>;
    float *const s_hx = reinterpret_cast<float *>(ring + S::xch);   // [2][TY][128]
    float *const s_hz = s_hx + 2 * TY * 128;
    uint64_t *const bar = reinterpret_cast<uint64_t *>(ring + S::bars);
    float *const s_zc = reinterpret_cast<float *>(ring + S::zc);    // [4][nrz]
    Em3DLeanPlane *const s_plane = reinterpret_cast<Em3DLeanPlane *>(ring + S::plane(p.cpml[2].nr));
    float *const s_kz = reinterpret_cast<float *>(ring + S::kz(p.cpml[2].nr));   // [2][128]
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int kt0 = (in.k0 & ~3) + (int)blockIdx.x * EM3D_LTILE;  // the tile's first cell
    const int kv = kt0 + EM3D_LV * lane;                         // this thread's first cell (may be off the grid)
    const int ks = min(max(kv, 0), p.nz - EM3D_LV);              // the same, clamped: global addresses
    // the boxes' first row: the halo row below the tile's first output row
    const int j_row0 = in.j0 - 1 + (int)blockIdx.y * (NX ? TY : TY - 1);
    const int rb = NX ? w + 1 : w;                               // this warp's row in the boxes
    const int jj = j_row0 + rb;
    const int j = min(jj, in.j1 - 1);
    const int i_first = in.i0 + (int)blockIdx.z * p.x_chunk;
    const int i_last = min(in.i1, i_first + p.x_chunk);
    const int ke = kt0 - EM3D_LV;                                // box start, 4 cells before the tile
    const int km = ke & ~7;                                      // id box start (a multiple of 8)
    // cells stored by this thread (H and E alike): not the halo row, inside the box
    unsigned kmask = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (kv + c >= in.k0 && kv + c < in.k1) kmask |= 1u << c;
    if ((!NX && w == 0) || jj >= in.j1) kmask = 0;
    const bool vec = __all_sync(0xffffffffu, kmask == 0u || kmask == 0xFu);
    // the box reaches the z edges only on an open z axis: the thread holding row 0 / row nz - 1
    const bool first = in.k0 == 0 && kv == 0, last = in.k1 == p.nz && kv + EM3D_LV == p.nz;
    const size_t sx = (size_t)p.ny * p.nz;
    const int o = j * p.nz + ks;                                 // in-plane offset of the thread's vector
    const int at_e = rb * L::WE + EM3D_LV + EM3D_LV * lane;      // the vector in an E box row
    const int at_h = rb * L::WH + EM3D_LV + EM3D_LV * lane;
    const int at_m = rb * L::WM + (kt0 - km) + EM3D_LV * lane;
    const bool halo = lane == 0 && kt0 > 0;                      // lane 0 also computes H_x, H_y of cell kt0 - 1
    const int base = i_first - 1;
    if (tid == 0) {
        for (int q = 0; q < RING; ++q) tb_mbar_init(bar + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tb_fence_proxy_async();
    }
    for (int q = tid; q < i_last - base; q += 32 * TY) {   // planes base .. i_last - 1, the ones the loop steps
        const int i = base + q;
        Em3DLeanPlane pl;
        pl.ihx = p.ihx[i];
        pl.iex = p.iex[i];
        pl.wl = p.wlx[i];
        pl.wu = p.wux[i];
        pl.rh = p.cpml[0].nr ? p.cpml[0].rm_h[i] : -1;
        pl.re = p.cpml[0].nr ? p.cpml[0].rm_e[i] : -1;
        pl.bh = pl.rh >= 0 ? p.cpml[0].b_h[pl.rh] : 0.0f;
        pl.gh = pl.rh >= 0 ? p.cpml[0].g_h[pl.rh] : 0.0f;
        pl.be = pl.re >= 0 ? p.cpml[0].b_e[pl.re] : 0.0f;
        pl.ge = pl.re >= 0 ? p.cpml[0].g_e[pl.re] : 0.0f;
        s_plane[q] = pl;
    }
    for (int c = tid; c < EM3D_LTILE; c += 32 * TY) {
        const int kc = min(kt0 + c, p.nz - 1);
        s_kz[c] = p.ihz[kc];
        s_kz[EM3D_LTILE + c] = p.iez[kc];
    }
    const int nrz = p.cpml[2].nr;
    for (int r = tid; r < nrz; r += 32 * TY) {
        s_zc[r] = p.cpml[2].b_h[r];
        s_zc[nrz + r] = p.cpml[2].g_h[r];
        s_zc[2 * nrz + r] = p.cpml[2].b_e[r];
        s_zc[3 * nrz + r] = p.cpml[2].g_e[r];
    }
    __syncthreads();
    if (w == 0)
        for (int q = 0; q < RING && base + q <= i_last; ++q)
            em3d_lean_issue<TY, NX>(maps, ring + q * L::slot, bar + q, base + q, j_row0, ke, km, lane);
    const int n_issued_max = i_last - base + 1;
    // per-row and per-cell spacings; CPML rows of the row (y) and of the cells (z, one byte each, 0xff: none)
    const float2 ihy2 = lp_dup(p.ihy[j]), iey2 = lp_dup(p.iey[j]);
    uint32_t zrh = 0xffffffffu, zre = 0xffffffffu;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int kc = min(max(kv + c, 0), p.nz - 1);
        if (nrz) {
            const int32_t rh = p.cpml[2].rm_h[kc], re = p.cpml[2].rm_e[kc];
            if (rh >= 0) zrh = (zrh & ~(0xffu << (8 * c))) | ((uint32_t)rh << (8 * c));
            if (re >= 0) zre = (zre & ~(0xffu << (8 * c))) | ((uint32_t)re << (8 * c));
        }
    }
    const float ihz_h = p.ihz[max(kt0 - 1, 0)];
    const int32_t zr_h = nrz ? p.cpml[2].rm_h[max(kt0 - 1, 0)] : -1;
    // z rows r0 .. r0 + 3 on a multiple of 4 (and a multiple of 4 rows): one 16-byte psi vector for the four cells
    const bool zvh = nrz % 4 == 0 && (zrh & 3u) == 0 && zrh == (zrh & 0xffu) * 0x01010101u + 0x03020100u;
    const bool zve = nrz % 4 == 0 && (zre & 3u) == 0 && zre == (zre & 0xffu) * 0x01010101u + 0x03020100u;
    const int32_t ryh = p.cpml[1].nr ? p.cpml[1].rm_h[j] : -1, rye = p.cpml[1].nr ? p.cpml[1].rm_e[j] : -1;
    const float2 byh = lp_dup(ryh >= 0 ? p.cpml[1].b_h[ryh] : 0.0f), gyh = lp_dup(ryh >= 0 ? p.cpml[1].g_h[ryh] : 0.0f);
    const float2 bye = lp_dup(rye >= 0 ? p.cpml[1].b_e[rye] : 0.0f), gye = lp_dup(rye >= 0 ? p.cpml[1].g_e[rye] : 0.0f);
    // NX: the row below (j - 1): its inverse spacing and y CPML row (H map)
    const int jb = max(j - 1, 0);
    const float ihyb = NX ? p.ihy[jb] : 0.0f;
    const int32_t ryb = NX && p.cpml[1].nr ? p.cpml[1].rm_h[jb] : -1;
    const float byb = ryb >= 0 ? p.cpml[1].b_h[ryb] : 0.0f, gyb = ryb >= 0 ? p.cpml[1].g_h[ryb] : 0.0f;
    const uint32_t id_max = (uint32_t)(p.n_ids - 1);
    const float *__restrict__ t_same = p.t_same;
    float *__restrict__ oex = p.oex;
    float *__restrict__ oey = p.oey;
    float *__restrict__ oez = p.oez;
    float *__restrict__ ohx = p.ohx;
    float *__restrict__ ohy = p.ohy;
    float *__restrict__ ohz = p.ohz;
    bool ok = tb_mbar_wait(bar, 0);   // plane base
    float2 hy_m[2] = {}, hz_m[2] = {};   // H^{n+1/2} of plane i - 1
    int par = 0;
    int cs = 0, ns = 1;                  // ring slots of planes i and i + 1
    uint32_t nph = 0;                    // mbarrier phase parity of plane i + 1's slot
    size_t bo = (size_t)base * sx + o;   // the thread's vector in plane i
    for (int i = base; i < i_last; ++i, bo += sx) {
        const int q = i - base;
        const unsigned char *cur = ring + cs * L::slot;
        const unsigned char *nxt = ring + ns * L::slot;
        if (NX) {
            // every warp is done with plane i - 1 (and every wait so far succeeded): its slot takes plane
            // i + RING - 1 now, a whole plane before it is read
            if (__syncthreads_or(!ok)) {   // a wait ran out somewhere in the block: stop, after the copies in flight
                if (tid == 0) atomicExch(p.err, 1);
                if (w == 0)   // positions q (its wait ran out, maybe) .. q + RING - 2 may be in flight
                    for (int qq = q; qq < min(n_issued_max, q + RING - 1); ++qq)
                        tb_mbar_wait(bar + qq % RING, (uint32_t)((qq / RING) & 1));
                return;
            }
            if (w == 0 && q >= 1 && i + RING - 1 <= i_last) {
                const int ps = cs == 0 ? RING - 1 : cs - 1;
                tb_fence_proxy_async();
                em3d_lean_issue<TY, NX>(maps, ring + ps * L::slot, bar + ps, i + RING - 1, j_row0, ke, km, lane);
            }
        } else if (EARLY) {
            // every warp is done with plane i - 1: its slot takes plane i + RING - 1 now, a whole plane before it is
            // read
            __syncthreads();
            if (w == 0 && q >= 1 && i + RING - 1 <= i_last) {
                const int ps = cs == 0 ? RING - 1 : cs - 1;
                tb_fence_proxy_async();
                em3d_lean_issue<TY, NX>(maps, ring + ps * L::slot, bar + ps, i + RING - 1, j_row0, ke, km, lane);
            }
        }
        ok = tb_mbar_wait(bar + ns, nph) && ok;
        const Em3DLeanPlane pl = s_plane[q];
        const float *ce0 = reinterpret_cast<const float *>(cur + L::e_off);
        const float *ce1 = ce0 + L::e_bytes / 4;
        const float *ce2 = ce1 + L::e_bytes / 4;
        const float *ch = reinterpret_cast<const float *>(cur + L::h_off);
        const float *ne1 = reinterpret_cast<const float *>(nxt + L::e_off + L::e_bytes);
        const float *ne2 = ne1 + L::e_bytes / 4;
        const bool inside = i >= i_first;
        const unsigned smask = inside ? kmask : 0u;
        // ---- H^{n+1/2} of the thread's four cells
        float2 ex0[2], ey0[2], ez0[2], exy[2], ezy[2], eyn[2], ezn[2], hx0[2], hy0[2], hz0[2];
        lv_lds(ce0 + at_e, ex0);
        lv_lds(ce1 + at_e, ey0);
        lv_lds(ce2 + at_e, ez0);
        lv_lds(ce0 + at_e + L::WE, exy);
        lv_lds(ce2 + at_e + L::WE, ezy);
        lv_lds(ne1 + at_e, eyn);
        lv_lds(ne2 + at_e, ezn);
        lv_lds(ch + at_h, hx0);
        lv_lds(ch + L::h_bytes / 4 + at_h, hy0);
        lv_lds(ch + 2 * (L::h_bytes / 4) + at_h, hz0);
        float2 exk[2], eyk[2];   // E_x, E_y at k + 1 (across the hi z edge: the wrapped sample of row 0)
        float exn4 = ce0[at_e + 4], eyn4 = ce1[at_e + 4];
        if (last) {
            exn4 = em3d_wrapped(__ldg(p.ex + (bo - ks)));
            eyn4 = em3d_wrapped(__ldg(p.ey + (bo - ks)));
        }
        lv_up(ex0, exn4, exk);
        lv_up(ey0, eyn4, eyk);
        constexpr bool hu = HU;
        float2 dav[2], dbv[2];
        if (hu) {
            dav[0] = dav[1] = lp_dup(p.da_u);
            dbv[0] = dbv[1] = lp_dup(p.db_u);
        } else {
            const uint2 m0v = *reinterpret_cast<const uint2 *>(reinterpret_cast<const uint16_t *>(cur + L::m_off) +
                                                               at_m);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint32_t m = min(lv_id(m0v, c), id_max);
                lv_set(dav, c, __ldg(p.t_da + m));
                lv_set(dbv, c, __ldg(p.t_db + m));
            }
        }
        const float2 ihx2 = lp_dup(pl.ihx);
        float2 dez_y[2], dey_z[2], dex_z[2], dez_x[2], dey_x[2], dex_y[2];
        float2 vhx[2], vhy[2], vhz[2], ihz[2];
        lv_lds(s_kz + EM3D_LV * lane, ihz);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            dez_y[h] = lp_sub(ezy[h], ez0[h]);
            dey_z[h] = lp_sub(eyk[h], ey0[h]);
            dex_z[h] = lp_sub(exk[h], ex0[h]);
            dez_x[h] = lp_sub(ezn[h], ez0[h]);
            dey_x[h] = lp_sub(eyn[h], ey0[h]);
            dex_y[h] = lp_sub(exy[h], ex0[h]);
            vhx[h] = ls_sub(lp_mul(dav[h], hx0[h]),
                            lp_mul(dbv[h], ls_sub(lp_mul(dez_y[h], ihy2), lp_mul(dey_z[h], ihz[h]))));
            vhy[h] = ls_sub(lp_mul(dav[h], hy0[h]),
                            lp_mul(dbv[h], ls_sub(lp_mul(dex_z[h], ihz[h]), lp_mul(dez_x[h], ihx2))));
            vhz[h] = ls_sub(lp_mul(dav[h], hz0[h]),
                            lp_mul(dbv[h], ls_sub(lp_mul(dey_x[h], ihx2), lp_mul(dex_y[h], ihy2))));
        }
        if (pl.rh >= 0) {   // x layers: H_y from E_z (+), H_z from E_y (-)
            const Em3DCpmlAxis &c = p.cpml[0];
            const size_t qq = (size_t)pl.rh * sx + o;
            const float2 bb = lp_dup(pl.bh), gg = lp_dup(pl.gh);
            float2 pf[2], pg[2], f[2], g[2];
            lv_ldg(c.ph_first + qq, pf);
            lv_ldg(c.ph_second + qq, pg);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                f[h] = ls_add(lp_mul(bb, pf[h]), lp_mul(gg, dez_x[h]));
                g[h] = ls_add(lp_mul(bb, pg[h]), lp_mul(gg, dey_x[h]));
                vhy[h] = ls_add(vhy[h], lp_mul(dbv[h], f[h]));
                vhz[h] = ls_sub(vhz[h], lp_mul(dbv[h], g[h]));
            }
            lv_store(c.oph_first + qq, f, smask, vec);
            lv_store(c.oph_second + qq, g, smask, vec);
        }
        if (ryh >= 0) {   // y layers: H_x from E_z (-), H_z from E_x (+)
            const Em3DCpmlAxis &c = p.cpml[1];
            const size_t qq = ((size_t)i * c.nr + ryh) * p.nz + ks;
            float2 pf[2], pg[2], f[2], g[2];
            lv_ldg(c.ph_first + qq, pf);
            lv_ldg(c.ph_second + qq, pg);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                f[h] = ls_add(lp_mul(byh, pf[h]), lp_mul(gyh, dez_y[h]));
                g[h] = ls_add(lp_mul(byh, pg[h]), lp_mul(gyh, dex_y[h]));
                vhx[h] = ls_sub(vhx[h], lp_mul(dbv[h], f[h]));
                vhz[h] = ls_add(vhz[h], lp_mul(dbv[h], g[h]));
            }
            lv_store(c.oph_first + qq, f, smask, vec);
            lv_store(c.oph_second + qq, g, smask, vec);
        }
        if (zvh) {   // z layers, four consecutive rows: H_x from E_y (+), H_y from E_x (-)
            const Em3DCpmlAxis &c = p.cpml[2];
            const int r0 = (int)(zrh & 0xffu);
            const size_t qq = ((size_t)i * p.ny + j) * nrz + r0;
            float2 pf[2], pg[2], bz[2], gz[2], f[2], g[2];
            lv_ldg(c.ph_first + qq, pf);
            lv_ldg(c.ph_second + qq, pg);
            lv_lds(s_zc + r0, bz);
            lv_lds(s_zc + nrz + r0, gz);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                f[h] = ls_add(lp_mul(bz[h], pf[h]), lp_mul(gz[h], dey_z[h]));
                g[h] = ls_add(lp_mul(bz[h], pg[h]), lp_mul(gz[h], dex_z[h]));
                vhx[h] = ls_add(vhx[h], lp_mul(dbv[h], f[h]));
                vhy[h] = ls_sub(vhy[h], lp_mul(dbv[h], g[h]));
            }
            lv_store(c.oph_first + qq, f, smask, smask == 0u || smask == 0xFu);
            lv_store(c.oph_second + qq, g, smask, smask == 0u || smask == 0xFu);
        } else if (zrh != 0xffffffffu) {   // z layers, per cell
            const Em3DCpmlAxis &c = p.cpml[2];
            const size_t zb = ((size_t)i * p.ny + j) * nrz;
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const uint32_t r = (zrh >> (8 * cc)) & 0xffu;
                if (r == 0xffu) continue;
                const float bz = s_zc[r], gz = s_zc[nrz + r], db = lv_get(dbv, cc);
                const float f = __fadd_rn(__fmul_rn(bz, c.ph_first[zb + r]), __fmul_rn(gz, lv_get(dey_z, cc)));
                const float g = __fadd_rn(__fmul_rn(bz, c.ph_second[zb + r]), __fmul_rn(gz, lv_get(dex_z, cc)));
                if (smask & (1u << cc)) {
                    c.oph_first[zb + r] = f;
                    c.oph_second[zb + r] = g;
                }
                lv_set(vhx, cc, __fadd_rn(lv_get(vhx, cc), __fmul_rn(db, f)));
                lv_set(vhy, cc, __fadd_rn(lv_get(vhy, cc), -__fmul_rn(db, g)));
            }
        }
        lv_store(ohx + bo, vhx, smask, vec);
        lv_store(ohy + bo, vhy, smask, vec);
        lv_store(ohz + bo, vhz, smask, vec);
        float *const xhx = s_hx + par * TY * 128, *const xhz = s_hz + par * TY * 128;
        if constexpr (!NX) {
            *reinterpret_cast<float4 *>(xhx + w * 128 + EM3D_LV * lane) = make_float4(vhx[0].x, vhx[0].y, vhx[1].x,
                                                                                     vhx[1].y);
            *reinterpret_cast<float4 *>(xhz + w * 128 + EM3D_LV * lane) = make_float4(vhz[0].x, vhz[0].y, vhz[1].x,
                                                                                     vhz[1].y);
        }
        // H^{n+1/2} of cell k - 1 (lane - 1; lane 0: the halo cell kt0 - 1); below row 0 of the open z axis, 0:
        // F - 0 is F, em3d_lo_diff's value
        float hx_prev = __shfl_up_sync(0xffffffffu, vhx[1].y, 1);
        float hy_prev = __shfl_up_sync(0xffffffffu, vhy[1].y, 1);
        if (first) hx_prev = hy_prev = 0.0f;
        if (halo) {   // em3d_h_kernel's H_x and H_y of cell kt0 - 1 (its CPML psi read, not stored: its tile stores it)
            const int kh = kt0 - 1;
            const float ex_h = ce0[at_e - 1], ey_h = ce1[at_e - 1], ez_h = ce2[at_e - 1];
            const float dez_y_h = ce2[at_e - 1 + L::WE] - ez_h, dey_z_h = ey0[0].x - ey_h;
            const float dex_z_h = ex0[0].x - ex_h, dez_x_h = ne2[at_e - 1] - ez_h;
            float da = p.da_u, db = p.db_u;
            if (!hu) {
                const uint32_t m = min((uint32_t)reinterpret_cast<const uint16_t *>(cur + L::m_off)[at_m - 1], id_max);
                da = __ldg(p.t_da + m);
                db = __ldg(p.t_db + m);
            }
            float hx = da * ch[at_h - 1] - db * (dez_y_h * ihy2.x - dey_z_h * ihz_h);
            float hy = da * ch[L::h_bytes / 4 + at_h - 1] - db * (dex_z_h * ihz_h - dez_x_h * pl.ihx);
            if (pl.rh >= 0) {   // x layers: H_y from E_z (+)
                const size_t qq = (size_t)pl.rh * sx + (size_t)j * p.nz + kh;
                hy += db * (pl.bh * p.cpml[0].ph_first[qq] + pl.gh * dez_x_h);
            }
            if (ryh >= 0) {   // y layers: H_x from E_z (-)
                const size_t qq = ((size_t)i * p.cpml[1].nr + ryh) * p.nz + kh;
                hx -= db * (byh.x * p.cpml[1].ph_first[qq] + gyh.x * dez_y_h);
            }
            if (zr_h >= 0) {   // z layers: H_x from E_y (+), H_y from E_x (-)
                const size_t qq = ((size_t)i * p.ny + j) * nrz + zr_h;
                hx += db * (s_zc[zr_h] * p.cpml[2].ph_first[qq] + s_zc[nrz + zr_h] * dey_z_h);
                hy -= db * (s_zc[zr_h] * p.cpml[2].ph_second[qq] + s_zc[nrz + zr_h] * dex_z_h);
            }
            hx_prev = hx;
            hy_prev = hy;
        }
        float2 hzy[2], hxy[2];   // H^{n+1/2} of row j - 1 (H_z, H_x)
        if constexpr (NX) {   // evaluated here from the staged row below (its psi read, not stored)
            float2 exb[2], eyb[2], ezb[2], eynb[2], hxb0[2], hzb0[2], eykb[2];
            lv_lds(ce0 + at_e - L::WE, exb);
            lv_lds(ce1 + at_e - L::WE, eyb);
            lv_lds(ce2 + at_e - L::WE, ezb);
            lv_lds(ne1 + at_e - L::WE, eynb);
            lv_lds(ch + at_h - L::WH, hxb0);
            lv_lds(ch + 2 * (L::h_bytes / 4) + at_h - L::WH, hzb0);
            float eyn4b = ce1[at_e - L::WE + 4];
            if (last) eyn4b = em3d_wrapped(__ldg(p.ey + (bo - ks - p.nz)));
            lv_up(eyb, eyn4b, eykb);
            float2 dab[2], dbb[2];
            if (hu) {
                dab[0] = dab[1] = lp_dup(p.da_u);
                dbb[0] = dbb[1] = lp_dup(p.db_u);
            } else {
                const uint2 mbv = *reinterpret_cast<const uint2 *>(
                    reinterpret_cast<const uint16_t *>(cur + L::m_off) + at_m - L::WM);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t m = min(lv_id(mbv, c), id_max);
                    lv_set(dab, c, __ldg(p.t_da + m));
                    lv_set(dbb, c, __ldg(p.t_db + m));
                }
            }
            const float2 ihyb2 = lp_dup(ihyb);
            float2 dez_yb[2], dey_zb[2], dey_xb[2], dex_yb[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                dez_yb[h] = lp_sub(ez0[h], ezb[h]);
                dey_zb[h] = lp_sub(eykb[h], eyb[h]);
                dey_xb[h] = lp_sub(eynb[h], eyb[h]);
                dex_yb[h] = lp_sub(ex0[h], exb[h]);
                hxy[h] = ls_sub(lp_mul(dab[h], hxb0[h]),
                                lp_mul(dbb[h], ls_sub(lp_mul(dez_yb[h], ihyb2), lp_mul(dey_zb[h], ihz[h]))));
                hzy[h] = ls_sub(lp_mul(dab[h], hzb0[h]),
                                lp_mul(dbb[h], ls_sub(lp_mul(dey_xb[h], ihx2), lp_mul(dex_yb[h], ihyb2))));
            }
            if (pl.rh >= 0) {   // x layers: H_z from E_y (-)
                const size_t qq = (size_t)pl.rh * sx + (o - p.nz);
                const float2 bb = lp_dup(pl.bh), gg = lp_dup(pl.gh);
                float2 pg[2];
                lv_ldg(p.cpml[0].ph_second + qq, pg);
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    hzy[h] = ls_sub(hzy[h], lp_mul(dbb[h], ls_add(lp_mul(bb, pg[h]), lp_mul(gg, dey_xb[h]))));
            }
            if (ryb >= 0) {   // y layers: H_x from E_z (-), H_z from E_x (+)
                const size_t qq = ((size_t)i * p.cpml[1].nr + ryb) * p.nz + ks;
                const float2 bb = lp_dup(byb), gg = lp_dup(gyb);
                float2 pf[2], pg[2];
                lv_ldg(p.cpml[1].ph_first + qq, pf);
                lv_ldg(p.cpml[1].ph_second + qq, pg);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    hxy[h] = ls_sub(hxy[h], lp_mul(dbb[h], ls_add(lp_mul(bb, pf[h]), lp_mul(gg, dez_yb[h]))));
                    hzy[h] = ls_add(hzy[h], lp_mul(dbb[h], ls_add(lp_mul(bb, pg[h]), lp_mul(gg, dex_yb[h]))));
                }
            }
            if (zvh) {   // z layers, four consecutive rows: H_x from E_y (+)
                const int r0 = (int)(zrh & 0xffu);
                const size_t qq = ((size_t)i * p.ny + jb) * nrz + r0;
                float2 pf[2], bz[2], gz[2];
                lv_ldg(p.cpml[2].ph_first + qq, pf);
                lv_lds(s_zc + r0, bz);
                lv_lds(s_zc + nrz + r0, gz);
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    hxy[h] = ls_add(hxy[h], lp_mul(dbb[h], ls_add(lp_mul(bz[h], pf[h]), lp_mul(gz[h], dey_zb[h]))));
            } else if (zrh != 0xffffffffu) {   // z layers, per cell
                const size_t zb = ((size_t)i * p.ny + jb) * nrz;
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    const uint32_t r = (zrh >> (8 * cc)) & 0xffu;
                    if (r == 0xffu) continue;
                    const float f = __fadd_rn(__fmul_rn(s_zc[r], p.cpml[2].ph_first[zb + r]),
                                              __fmul_rn(s_zc[nrz + r], lv_get(dey_zb, cc)));
                    lv_set(hxy, cc, __fadd_rn(lv_get(hxy, cc), __fmul_rn(lv_get(dbb, cc), f)));
                }
            }
        } else {
            if (__syncthreads_or(!ok)) {   // a wait ran out somewhere in the block: stop, after the copies in flight
                if (tid == 0) atomicExch(p.err, 1);
                if (w == 0)
                    for (int qq = q + 1; qq < min(n_issued_max, q + RING - 1); ++qq)
                        tb_mbar_wait(bar + qq % RING, (uint32_t)((qq / RING) & 1));
                return;
            }
            // no thread reads the slot of plane i - 1 any more: it takes plane i + RING - 1
            if (!EARLY && w == 0 && q >= 1 && i + RING - 1 <= i_last) {
                const int ps = cs == 0 ? RING - 1 : cs - 1;
                tb_fence_proxy_async();
                em3d_lean_issue<TY, NX>(maps, ring + ps * L::slot, bar + ps, i + RING - 1, j_row0, ke, km, lane);
            }
            if (w > 0) {
                lv_lds(xhz + (w - 1) * 128 + EM3D_LV * lane, hzy);   // H^{n+1/2} of row j - 1, from the warp below
                lv_lds(xhx + (w - 1) * 128 + EM3D_LV * lane, hxy);
            }
        }
        if ((NX || w > 0) && inside) {
            // ---- E^{n+1} of the thread's four cells
            float2 hxk[2], hyk[2];
            lv_down(vhx, hx_prev, hxk);
            lv_down(vhy, hy_prev, hyk);
            const uint16_t *cm = reinterpret_cast<const uint16_t *>(cur + L::m_off);
            const uint16_t *nm = reinterpret_cast<const uint16_t *>(nxt + L::m_off);
            const uint2 m0v = *reinterpret_cast<const uint2 *>(cm + at_m);
            const uint2 mxv = *reinterpret_cast<const uint2 *>(nm + at_m);
            const uint2 myv = *reinterpret_cast<const uint2 *>(cm + at_m + L::WM);
            const uint32_t mze = last ? lv_id(m0v, 3) : cm[at_m + 4];   // the last row's E_z face: the cell itself
            float2 cax[2], cay[2], caz[2], cbx[2], cby[2], cbz[2];
            const uint32_t a = min(m0v.x & 0xffffu, id_max);
            const uint32_t rep = a | (a << 16);
            if (p.same_ok && m0v.x == rep && m0v.y == rep && mxv.x == rep && mxv.y == rep && myv.x == rep &&
                myv.y == rep && mze == a) {   // one id around all four cells
                cbx[0] = cbx[1] = lp_dup(__ldg(t_same + p.n_ids + a));
                cby[0] = cby[1] = lp_dup(__ldg(t_same + 3 * p.n_ids + a));
                cbz[0] = cbz[1] = lp_dup(__ldg(t_same + 5 * p.n_ids + a));
                if (!CA1) {
                    cax[0] = cax[1] = lp_dup(__ldg(t_same + a));
                    cay[0] = cay[1] = lp_dup(__ldg(t_same + 2 * p.n_ids + a));
                    caz[0] = caz[1] = lp_dup(__ldg(t_same + 4 * p.n_ids + a));
                }
            } else {
                const float wly = p.wly[j], wuy = p.wuy[j];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t m0 = min(lv_id(m0v, c), id_max), mx = min(lv_id(mxv, c), id_max);
                    const uint32_t my = min(lv_id(myv, c), id_max);
                    const uint32_t mz = min(c < 3 ? lv_id(m0v, c + 1) : mze, id_max);
                    const int kc = min(max(kv + c, 0), p.nz - 1);
                    float ca, cb;
                    em3d_lean_face(p, t_same, 0, p.t_ex, m0, mx, pl.wl, pl.wu, ca, cb);
                    lv_set(cax, c, ca);
                    lv_set(cbx, c, cb);
                    em3d_lean_face(p, t_same, 1, p.t_ey, m0, my, wly, wuy, ca, cb);
                    lv_set(cay, c, ca);
                    lv_set(cby, c, cb);
                    em3d_lean_face(p, t_same, 2, p.t_ez, m0, mz, p.wlz[kc], p.wuz[kc], ca, cb);
                    lv_set(caz, c, ca);
                    lv_set(cbz, c, cb);
                }
            }
            const float2 iex2 = lp_dup(pl.iex);
            float2 dhz_y[2], dhy_z[2], dhx_z[2], dhz_x[2], dhy_x[2], dhx_y[2], vx[2], vy[2], vz[2], iez[2];
            float2 ex0[2], ey0[2], ez0[2];   // E^n of the cells, read again from the slot
            lv_lds(s_kz + EM3D_LTILE + EM3D_LV * lane, iez);
            lv_lds(ce0 + at_e, ex0);
            lv_lds(ce1 + at_e, ey0);
            lv_lds(ce2 + at_e, ez0);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                dhz_y[h] = lp_sub(vhz[h], hzy[h]);
                dhy_z[h] = lp_sub(vhy[h], hyk[h]);
                dhx_z[h] = lp_sub(vhx[h], hxk[h]);
                dhz_x[h] = lp_sub(vhz[h], hz_m[h]);
                dhy_x[h] = lp_sub(vhy[h], hy_m[h]);
                dhx_y[h] = lp_sub(vhx[h], hxy[h]);
                const float2 bx = CA1 ? ex0[h] : lp_mul(cax[h], ex0[h]);
                const float2 by = CA1 ? ey0[h] : lp_mul(cay[h], ey0[h]);
                const float2 bz = CA1 ? ez0[h] : lp_mul(caz[h], ez0[h]);
                vx[h] = ls_add(bx, lp_mul(cbx[h], ls_sub(lp_mul(dhz_y[h], iey2), lp_mul(dhy_z[h], iez[h]))));
                vy[h] = ls_add(by, lp_mul(cby[h], ls_sub(lp_mul(dhx_z[h], iez[h]), lp_mul(dhz_x[h], iex2))));
                vz[h] = ls_add(bz, lp_mul(cbz[h], ls_sub(lp_mul(dhy_x[h], iex2), lp_mul(dhx_y[h], iey2))));
            }
            if (pl.re >= 0) {   // x layers: E_y from H_z (-), E_z from H_y (+)
                const Em3DCpmlAxis &c = p.cpml[0];
                const size_t qq = (size_t)pl.re * sx + o;
                const float2 bb = lp_dup(pl.be), gg = lp_dup(pl.ge);
                float2 pf[2], pg[2], f[2], g[2];
                lv_ldg(c.pe_first + qq, pf);
                lv_ldg(c.pe_second + qq, pg);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    f[h] = ls_add(lp_mul(bb, pf[h]), lp_mul(gg, dhz_x[h]));
                    g[h] = ls_add(lp_mul(bb, pg[h]), lp_mul(gg, dhy_x[h]));
                    vy[h] = ls_sub(vy[h], lp_mul(cby[h], f[h]));
                    vz[h] = ls_add(vz[h], lp_mul(cbz[h], g[h]));
                }
                lv_store(c.ope_first + qq, f, kmask, vec);
                lv_store(c.ope_second + qq, g, kmask, vec);
            }
            if (rye >= 0) {   // y layers: E_x from H_z (+), E_z from H_x (-)
                const Em3DCpmlAxis &c = p.cpml[1];
                const size_t qq = ((size_t)i * c.nr + rye) * p.nz + ks;
                float2 pf[2], pg[2], f[2], g[2];
                lv_ldg(c.pe_first + qq, pf);
                lv_ldg(c.pe_second + qq, pg);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    f[h] = ls_add(lp_mul(bye, pf[h]), lp_mul(gye, dhz_y[h]));
                    g[h] = ls_add(lp_mul(bye, pg[h]), lp_mul(gye, dhx_y[h]));
                    vx[h] = ls_add(vx[h], lp_mul(cbx[h], f[h]));
                    vz[h] = ls_sub(vz[h], lp_mul(cbz[h], g[h]));
                }
                lv_store(c.ope_first + qq, f, kmask, vec);
                lv_store(c.ope_second + qq, g, kmask, vec);
            }
            if (zve) {   // z layers, four consecutive rows: E_x from H_y (-), E_y from H_x (+)
                const Em3DCpmlAxis &c = p.cpml[2];
                const int r0 = (int)(zre & 0xffu);
                const size_t qq = ((size_t)i * p.ny + j) * nrz + r0;
                float2 pf[2], pg[2], bz[2], gz[2], f[2], g[2];
                lv_ldg(c.pe_first + qq, pf);
                lv_ldg(c.pe_second + qq, pg);
                lv_lds(s_zc + 2 * nrz + r0, bz);
                lv_lds(s_zc + 3 * nrz + r0, gz);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    f[h] = ls_add(lp_mul(bz[h], pf[h]), lp_mul(gz[h], dhy_z[h]));
                    g[h] = ls_add(lp_mul(bz[h], pg[h]), lp_mul(gz[h], dhx_z[h]));
                    vx[h] = ls_sub(vx[h], lp_mul(cbx[h], f[h]));
                    vy[h] = ls_add(vy[h], lp_mul(cby[h], g[h]));
                }
                lv_store(c.ope_first + qq, f, kmask, kmask == 0u || kmask == 0xFu);
                lv_store(c.ope_second + qq, g, kmask, kmask == 0u || kmask == 0xFu);
            } else if (zre != 0xffffffffu) {   // z layers, per cell
                const Em3DCpmlAxis &c = p.cpml[2];
                const size_t zb = ((size_t)i * p.ny + j) * nrz;
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    const uint32_t r = (zre >> (8 * cc)) & 0xffu;
                    if (r == 0xffu) continue;
                    const float bz = s_zc[2 * nrz + r], gz = s_zc[3 * nrz + r];
                    const float f = __fadd_rn(__fmul_rn(bz, c.pe_first[zb + r]), __fmul_rn(gz, lv_get(dhy_z, cc)));
                    const float g = __fadd_rn(__fmul_rn(bz, c.pe_second[zb + r]), __fmul_rn(gz, lv_get(dhx_z, cc)));
                    if (kmask & (1u << cc)) {
                        c.ope_first[zb + r] = f;
                        c.ope_second[zb + r] = g;
                    }
                    lv_set(vx, cc, __fadd_rn(lv_get(vx, cc), -__fmul_rn(lv_get(cbx, cc), f)));
                    lv_set(vy, cc, __fadd_rn(lv_get(vy, cc), __fmul_rn(lv_get(cby, cc), g)));
                }
            }
            lv_store(oex + bo, vx, kmask, vec);
            lv_store(oey + bo, vy, kmask, vec);
            lv_store(oez + bo, vz, kmask, vec);
        }
        hy_m[0] = vhy[0];
        hy_m[1] = vhy[1];
        hz_m[0] = vhz[0];
        hz_m[1] = vhz[1];
        par ^= 1;
        cs = ns;
        ns = ns + 1 == RING ? 0 : ns + 1;
        nph ^= ns == 0 ? 1u : 0u;
    }
    if constexpr (NX) {   // the last plane's wait is checked here
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(p.err, 1);
            if (w == 0)
                for (int qq = max(0, n_issued_max - RING); qq < n_issued_max; ++qq)
                    tb_mbar_wait(bar + qq % RING, (uint32_t)((qq / RING) & 1));
        }
    }
    // the last staged plane (i_last) was waited in the last iteration; nothing is in flight
}

// The dipoles of one step, in order (DipoleSource3D.inject, sources3d.py:69-75): E += FP32(s(t + dt/2)) * weight on
// the updated field, as em3d_e_kernel adds them at the end of a cell's update.  One thread.
__global__ void em3d_dipole_kernel(const Em3DParams p) {
    for (int d = 0; d < p.n_dip; ++d) {
        const float add = p.dip_values[d * p.values_stride + p.k_step] * p.dip_weight[d];
        float *f = p.dip_comp[d] == 0 ? p.oex : (p.dip_comp[d] == 1 ? p.oey : p.oez);
        const size_t at = (size_t)p.dip_i[d] * p.ny * p.nz + p.dip_o[d];
        f[at] = f[at] + add;
    }
}
