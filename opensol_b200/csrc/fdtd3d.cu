// 3D FDTD engine for sm_100a: device state, launches and the os_fdtd3d_* C ABI (replaces open_sol's FDTDEngine3D,
// physics/em3d/engine3d.py:157-554, for a Cartesian grid with one real field set and float32 fields).
//
// One Yee step follows the reference's own order (engine3d.py:497-554): H with its CPML, then E with its CPML and the
// dipole injection; on DFT sample steps em3d_flux_kernel accumulates every flux pair.  Four forms, bit-identical:
//   variant 3 (default): two field sets and two CPML psi sets, read one, write the other, swapped after every step;
//     em3d_lean_kernel (fdtd3d_lean.cuh) does H and E of every cell but the outermost x and y layers (and the z faces
//     too on an open z axis) in one pass over tensor-copy-staged planes, four cells a thread; the outer layers run
//     em3d_h_kernel, then em3d_e_kernel, per face in block shapes of their own; em3d_dipole_kernel adds the dipoles.
//     Rows of a multiple of 4 cells, at least 144; other grids run variant 0;
//   variant 0: em3d_h_kernel then em3d_e_kernel over the whole grid, in place on one field set;
//   variant 1: variant 3's schedule with em3d_fused_kernel, one cell a thread (every cell but the outermost layer of
//     each axis), the faces by the face kernels;
//   variant 2: variant 1 with each x plane of a tile staged in shared memory by tiled tensor copies
//     (em3d_staged_kernel).
// On 512^3: variant 3 71.7 G cell-updates/s (52 B of algorithmic traffic a cell-update: 0.57 of the measured copy
// bandwidth), variant 0 48.3 (two kernels re-reading the fields, ~76 B), variant 1 42.7, variant 2 46.4.
// A chunk of n steps is enqueued with no host synchronisation: per-step dipole amplitudes and per-sample DFT phases
// arrive as small tables computed on the host in float64 and rounded as open_sol rounds them.
#include "common.cuh"
#include "fdtd3d_kernels.cuh"
#include "fdtd3d_lean.cuh"

#include <algorithm>
#include <memory>
#include <vector>

struct OsFdtd3D {
    OsGrid3D grid{};
    int device = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool timed = false;
    os::DeviceArray<float> field[6];            // ex, ey, ez, hx, hy, hz
    os::DeviceArray<float> field2[6];           // the second field set of variant 1 (allocated on first use)
    int cur = 0;                                // the set holding the current state (0: field, 1: field2)
    int32_t variant = 3;                        // on 512^3: 71.7 G cell-updates/s; variant 0 48.3, 1 42.7, 2 46.4
    int32_t fused_config = -1;                  // launch shape of the fused form's kernel (speed only; -1: default)
    os::DeviceArray<uint16_t> mat;
    os::DeviceArray<float> tables;              // t_ex, t_ey, t_ez, t_sig, t_da, t_db (6 * n_ids)
    os::DeviceArray<float> same;                // same-id face ca, cb per component (6 * n_ids)
    int32_t n_ids = 0;
    bool same_ok = false;                       // every face share is 0.5
    bool has_materials = false, has_spacings = false;
    bool h_uniform = true, e_lossless = true;
    float da_u = 1.0f, db_u = 0.0f, dt = 0.0f;
    os::DeviceArray<float> rows;                // iex, iey, iez, ihx, ihy, ihz, wlx, wux, wly, wuy, wlz, wuz
    struct Cpml {
        int32_t nr = 0;
        os::DeviceArray<int32_t> rm;            // rm_e (n), rm_h (n)
        os::DeviceArray<float> coef;            // b_e, g_e, b_h, g_h (nr each)
        os::DeviceArray<float> psi;             // pe_first, pe_second, ph_first, ph_second
        os::DeviceArray<float> psi2;            // the second psi set of variant 1 (allocated on first use)
        size_t psi_count = 0;
    } cpml[3];
    struct Dipole {
        int32_t comp, i, o;                     // component, x plane, in-plane offset j nz + k
        float weight;
    };
    std::vector<Dipole> dipoles;
    std::vector<int32_t> monitor_nf;            // frequencies per flux monitor
    std::vector<Em3DFluxPair> pairs;            // host copy (pointers into acc)
    std::vector<std::unique_ptr<os::DeviceArray<double>>> acc;   // per pair: e then h accumulators
    os::DeviceArray<Em3DFluxPair> pairs_dev;
    bool pairs_dirty = false;
    int32_t max_pair_cells = 0;
    int64_t sample_interval = 1;
    int64_t n_step = 0;
    int64_t launches = 0;
    int32_t x_chunk = 64;
    os::DeviceArray<float> values;              // (n_dipoles, n_steps) of the current chunk
    os::DeviceArray<float> phases;              // (n_samples, sum nf, 2) of the current chunk
    os::DeviceArray<float> scratch;             // one float (face cb read-back)
    os::DeviceArray<int32_t> err;               // set by a staged kernel whose bounded wait ran out
    Em3DMaps maps[2][2];                        // staged form: tensor maps per field set read and tile height (8, 16)
    bool maps_ok[2][2] = {{false, false}, {false, false}};
    Em3DLeanMaps lean_maps[2][8];               // lean form: per field set read and launch configuration
    bool lean_maps_ok[2][8] = {};
    bool ca_one = true;                         // every face's ca is 1 (no conductivity, no perfect conductor)
};

namespace os {

static int bind3(OsFdtd3D *h) {
    OS_CUDA(cudaSetDevice(h->device));
    return OS_OK;
}

static size_t cells3(const OsFdtd3D *h) { return (size_t)h->grid.nx * h->grid.ny * h->grid.nz; }

// Component c (ex, ey, ez, hx, hy, hz) of field set `set`.
static float *fset(const OsFdtd3D *h, int set, int c) { return set ? h->field2[c].ptr : h->field[c].ptr; }

// x chunks of box b along x.
static int32_t box_chunks(const Em3DBox &b, int32_t x_chunk) {
    return b.i1 > b.i0 ? (b.i1 - b.i0 + x_chunk - 1) / x_chunk : 0;
}

// Boxes of em3d_h_kernel / em3d_e_kernel: one box, the whole grid.
static void whole_grid_boxes(const OsFdtd3D *h, Em3DParams &p) {
    const OsGrid3D &g = h->grid;
    p.n_boxes = 1;
    p.boxes[0] = Em3DBox{0, g.nx, 0, g.ny, 0, g.nz};
    p.zbase[0] = 0;
    p.zbase[1] = box_chunks(p.boxes[0], p.x_chunk);
}

static Em3DParams make_params3(const OsFdtd3D *h) {
    Em3DParams p{};
    const OsGrid3D &g = h->grid;
    p.nx = g.nx;
    p.ny = g.ny;
    p.nz = g.nz;
    p.px = g.periodic[0];
    p.py = g.periodic[1];
    p.pz = g.periodic[2];
    p.x_chunk = h->x_chunk;
    p.ex = p.oex = fset(h, h->cur, 0);
    p.ey = p.oey = fset(h, h->cur, 1);
    p.ez = p.oez = fset(h, h->cur, 2);
    p.hx = p.ohx = fset(h, h->cur, 3);
    p.hy = p.ohy = fset(h, h->cur, 4);
    p.hz = p.ohz = fset(h, h->cur, 5);
    whole_grid_boxes(h, p);
    p.mat = h->mat.ptr;
    p.err = h->err.ptr;
    const int n = h->n_ids;
    const float *t = h->tables.ptr;
    p.t_ex = t;
    p.t_ey = t + n;
    p.t_ez = t + 2 * n;
    p.t_sig = t + 3 * n;
    p.t_da = t + 4 * n;
    p.t_db = t + 5 * n;
    p.h_uniform = h->h_uniform;
    p.da_u = h->da_u;
    p.db_u = h->db_u;
    p.e_lossless = h->e_lossless;
    p.n_ids = h->n_ids;
    p.same_ok = h->same_ok && h->same.ptr;
    p.t_same = h->same.ptr;
    const float *r = h->rows.ptr;
    const size_t nx = g.nx, ny = g.ny, nz = g.nz;
    p.iex = r;
    p.iey = r + nx;
    p.iez = r + nx + ny;
    p.ihx = r + nx + ny + nz;
    p.ihy = p.ihx + nx;
    p.ihz = p.ihy + ny;
    p.wlx = p.ihz + nz;
    p.wux = p.wlx + nx;
    p.wly = p.wux + nx;
    p.wuy = p.wly + ny;
    p.wlz = p.wuy + ny;
    p.wuz = p.wlz + nz;
    p.dt = h->dt;
    for (int a = 0; a < 3; ++a) {
        const auto &c = h->cpml[a];
        Em3DCpmlAxis &q = p.cpml[a];
        q.nr = c.nr;
        if (!c.nr) continue;
        const size_t n_axis = a == 0 ? nx : (a == 1 ? ny : nz);
        q.rm_e = c.rm.ptr;
        q.rm_h = c.rm.ptr + n_axis;
        q.b_e = c.coef.ptr;
        q.g_e = c.coef.ptr + c.nr;
        q.b_h = c.coef.ptr + 2 * c.nr;
        q.g_h = c.coef.ptr + 3 * c.nr;
        float *psi = h->cur ? c.psi2.ptr : c.psi.ptr;
        q.pe_first = q.ope_first = psi;
        q.pe_second = q.ope_second = psi + c.psi_count;
        q.ph_first = q.oph_first = psi + 2 * c.psi_count;
        q.ph_second = q.oph_second = psi + 3 * c.psi_count;
    }
    p.n_dip = (int32_t)h->dipoles.size();
    for (size_t d = 0; d < h->dipoles.size(); ++d) {
        p.dip_comp[d] = h->dipoles[d].comp;
        p.dip_i[d] = h->dipoles[d].i;
        p.dip_o[d] = h->dipoles[d].o;
        p.dip_weight[d] = h->dipoles[d].weight;
    }
    return p;
}

static int zero_state3(OsFdtd3D *h) {
    h->cur = 0;
    for (auto &f : h->field) OS_CUDA(cudaMemsetAsync(f.ptr, 0, f.bytes(), h->stream));
    for (auto &c : h->cpml)
        if (c.psi.ptr) OS_CUDA(cudaMemsetAsync(c.psi.ptr, 0, c.psi.bytes(), h->stream));
    for (auto &a : h->acc) OS_CUDA(cudaMemsetAsync(a->ptr, 0, a->bytes(), h->stream));
    h->n_step = 0;
    return OS_OK;
}

// Launch grid of em3d_h_kernel / em3d_e_kernel with bz x by blocks over p's boxes.
static dim3 box_grid(const Em3DParams &p, int bz = EM3D_BZ, int by = EM3D_BY) {
    int32_t nj = 0, nk = 0;
    for (int b = 0; b < p.n_boxes; ++b) {
        nj = std::max(nj, p.boxes[b].j1 - p.boxes[b].j0);
        nk = std::max(nk, p.boxes[b].k1 - p.boxes[b].k0);
    }
    return dim3((unsigned)((nk + bz - 1) / bz), (unsigned)((nj + by - 1) / by), (unsigned)p.zbase[p.n_boxes]);
}

// variant 1's fused box: every cell but the outermost layer of each axis.
static Em3DBox fused_box(const OsFdtd3D *h) {
    const OsGrid3D &g = h->grid;
    return Em3DBox{1, g.nx - 1, 1, g.ny - 1, 1, g.nz - 1};
}

// variant 3's lean kernel: rows of a multiple of 4 cells (16-byte vectors), boxes no larger than the grid (the id box
// is 144 cells wide, the tallest 17 rows), z CPML rows that fit one byte.
static bool lean_ok(const OsFdtd3D *h) {
    return h->grid.nz % 4 == 0 && h->grid.nz >= Em3DLeanLayout<16>::WM && h->grid.ny >= 17 &&
           h->cpml[2].nr <= EM3D_LEAN_MAX_ZROWS;
}

// The step runs on two field sets (variants 1, 2; variant 3 where its kernel applies, else the in-place form).
static bool fused_active(const OsFdtd3D *h) {
    const OsGrid3D &g = h->grid;
    const bool form = h->variant == 1 || h->variant == 2 || (h->variant == 3 && lean_ok(h));
    return form && g.nx >= 3 && g.ny >= 3 && g.nz >= 3;
}

// variant 2 stages the planes by bulk copies: rows must start on 16-byte boundaries and hold the 48-id window.
static bool staged_active(const OsFdtd3D *h) {
    return fused_active(h) && h->variant == 2 && h->grid.nz % 8 == 0 && h->grid.nz >= EM3D_WM;
}

static bool lean_active(const OsFdtd3D *h) { return h->variant == 3 && fused_active(h); }

// The lean kernel's box: the fused box, and along a non-periodic z axis rows 0 and nz - 1 too (the z faces).
static Em3DBox lean_box(const OsFdtd3D *h) {
    Em3DBox b = fused_box(h);
    if (!h->grid.periodic[2]) {
        b.k0 = 0;
        b.k1 = h->grid.nz;
    }
    return b;
}

// A bounded wait of a staged kernel ran out: report it once (the flag is cleared) as OS_ERR_CUDA.
static int check_err3(OsFdtd3D *h) {
    int32_t flag = 0;
    OS_CUDA(cudaMemcpyAsync(&flag, h->err.ptr, sizeof(flag), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    if (flag) {
        OS_CUDA(cudaMemsetAsync(h->err.ptr, 0, sizeof(int32_t), h->stream));
        OS_CUDA(cudaStreamSynchronize(h->stream));
        OS_CHECK(false, OS_ERR_CUDA, "a 3D step kernel gave up waiting for its staged planes (2 s); the fields of "
                                     "that advance are not valid");
    }
    return OS_OK;
}

// The outermost layer around the fused box, in three launches of their own block shapes, each block streaming one x
// plane (a face holds one or two cells across, so short chunks give the launch its threads): 0 = the x faces (32 x 8
// blocks along k and j), 1 = the y faces (rows of 128 along k), 2 = the z faces (256 along j: one k per face).
enum { FACES_X = 0, FACES_Y = 1, FACES_Z = 2 };
static void face_boxes(const OsFdtd3D *h, Em3DParams &p, int which) {
    const OsGrid3D &g = h->grid;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Em3DBox xf[2] = {{0, 1, 0, ny, 0, nz}, {nx - 1, nx, 0, ny, 0, nz}};
    const Em3DBox yf[2] = {{1, nx - 1, 0, 1, 0, nz}, {1, nx - 1, ny - 1, ny, 0, nz}};
    const Em3DBox zf[2] = {{1, nx - 1, 1, ny - 1, 0, 1}, {1, nx - 1, 1, ny - 1, nz - 1, nz}};
    const Em3DBox *all = which == FACES_X ? xf : (which == FACES_Y ? yf : zf);
    p.x_chunk = 1;
    p.n_boxes = 0;
    p.zbase[0] = 0;
    for (int q = 0; q < 2; ++q) {
        const Em3DBox &b = all[q];
        p.boxes[p.n_boxes] = b;
        p.zbase[p.n_boxes + 1] = p.zbase[p.n_boxes] + box_chunks(b, p.x_chunk);
        ++p.n_boxes;
    }
}

// H (e = false) or E (e = true) of the face launches (the z faces unless the interior kernel covers them); returns
// the number of launches.
static int launch_faces(const OsFdtd3D *h, const Em3DParams (&f)[3], bool e, bool z_faces) {
    if (e) {
        em3d_e_kernel<32, 8><<<box_grid(f[0], 32, 8), dim3(32, 8), 0, h->stream>>>(f[0]);
        em3d_e_kernel<128, 1><<<box_grid(f[1], 128, 1), dim3(128, 1), 0, h->stream>>>(f[1]);
        if (z_faces) em3d_e_kernel<1, 256><<<box_grid(f[2], 1, 256), dim3(1, 256), 0, h->stream>>>(f[2]);
    } else {
        em3d_h_kernel<32, 8><<<box_grid(f[0], 32, 8), dim3(32, 8), 0, h->stream>>>(f[0]);
        em3d_h_kernel<128, 1><<<box_grid(f[1], 128, 1), dim3(128, 1), 0, h->stream>>>(f[1]);
        if (z_faces) em3d_h_kernel<1, 256><<<box_grid(f[2], 1, 256), dim3(1, 256), 0, h->stream>>>(f[2]);
    }
    return z_faces ? 3 : 2;
}

// Point the psi of p's CPML axes: read set `in`, write set `out`.
static void point_psi(const OsFdtd3D *h, Em3DParams &p, int in, int out) {
    for (int a = 0; a < 3; ++a) {
        const auto &c = h->cpml[a];
        if (!c.nr) continue;
        float *pi = in ? c.psi2.ptr : c.psi.ptr, *po = out ? c.psi2.ptr : c.psi.ptr;
        Em3DCpmlAxis &q = p.cpml[a];
        q.pe_first = pi;
        q.pe_second = pi + c.psi_count;
        q.ph_first = pi + 2 * c.psi_count;
        q.ph_second = pi + 3 * c.psi_count;
        q.ope_first = po;
        q.ope_second = po + c.psi_count;
        q.oph_first = po + 2 * c.psi_count;
        q.oph_second = po + 3 * c.psi_count;
    }
}

// em3d_fused_kernel configurations: (tile rows, blocks per SM the register budget is cut for).
constexpr int FUSED_CONFIGS = 5;
static int fused_rows(int config) { return config == 0 || config == 1 ? 16 : 8; }
static int fused_cfg(const OsFdtd3D *h) { return h->fused_config < 0 ? 3 : h->fused_config; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (the library does not link libcuda itself).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_tiled_fn(EncodeTiledFn *out) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        OS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
        OS_CHECK(ptr && q == cudaDriverEntryPointSuccess, OS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = (EncodeTiledFn)ptr;
    }
    *out = fn;
    return OS_OK;
}

// A map of one (nx, ny, nz) array, z contiguous, with boxes of box_k x box_j x 1 (zero fill outside the array).
static int encode_box(CUtensorMap *map, const void *base, CUtensorMapDataType type, size_t elem, const OsGrid3D &g,
                      uint32_t box_k, uint32_t box_j) {
    EncodeTiledFn fn;
    OS_TRY(encode_tiled_fn(&fn));
    const cuuint64_t dims[3] = {(cuuint64_t)g.nz, (cuuint64_t)g.ny, (cuuint64_t)g.nx};
    const cuuint64_t strides[2] = {(cuuint64_t)g.nz * elem, (cuuint64_t)g.ny * g.nz * elem};
    const cuuint32_t box[3] = {box_k, box_j, 1};
    const cuuint32_t element_strides[3] = {1, 1, 1};
    const CUresult r = fn(map, type, 3, const_cast<void *>(base), dims, strides, box, element_strides,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    OS_CHECK(r == CUDA_SUCCESS, OS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return OS_OK;
}

// The staged launch's maps for field set `set` and tile height ty (made once per handle).
static int staged_maps(OsFdtd3D *h, int set, int ty, const Em3DMaps **out) {
    const int t = ty == 16 ? 1 : 0;
    if (!h->maps_ok[set][t]) {
        Em3DMaps &m = h->maps[set][t];
        for (int c = 0; c < 3; ++c) {
            OS_TRY(encode_box(&m.e[c], fset(h, set, c), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->grid, EM3D_WF, ty + 1));
            OS_TRY(encode_box(&m.h[c], fset(h, set, 3 + c), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->grid, EM3D_WF,
                              ty));
        }
        OS_TRY(encode_box(&m.m, h->mat.ptr, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, h->grid, EM3D_WM, ty + 1));
        h->maps_ok[set][t] = true;
    }
    *out = &h->maps[set][t];
    return OS_OK;
}

// em3d_lean_kernel configurations (on 512^3): 0 = 16 tile rows, 3 ring slots, one block per SM (67.7 G
// cell-updates/s); 1 = 8 rows, 3 slots, two blocks per SM, each plane's copies issued after its exchange barrier
// (70.2); 2 (the default) = 1 with the copies issued at the top of the plane behind a second barrier, a whole plane
// ahead (71.7); 3 = 6 rows, 4 slots, two blocks per SM, early copies (58.3: fewer warps); 4 = 2 with no exchange:
// every warp computes H_x, H_z of the row below its own (8 output rows a block, one barrier per plane; 69.6: the
// extra H work costs more than the barrier and the halo warp it saves).
constexpr int LEAN_CONFIGS = 5;
static_assert(LEAN_CONFIGS <= 8, "lean map cache");

template <int TY, bool NX>
static int lean_maps(OsFdtd3D *h, int set, int config, const Em3DLeanMaps **out) {
    if (!h->lean_maps_ok[set][config]) {
        using L = Em3DLeanLayout<TY, NX>;
        Em3DLeanMaps &m = h->lean_maps[set][config];
        for (int c = 0; c < 3; ++c) {
            OS_TRY(encode_box(&m.e[c], fset(h, set, c), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->grid, L::WE, L::ER));
            OS_TRY(encode_box(&m.h[c], fset(h, set, 3 + c), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, h->grid, L::WH, L::HR));
        }
        OS_TRY(encode_box(&m.m, h->mat.ptr, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, h->grid, L::WM, L::MR));
        h->lean_maps_ok[set][config] = true;
    }
    *out = &h->lean_maps[set][config];
    return OS_OK;
}

template <int TY, int RING, int MINB, bool CA1, bool HU, bool EARLY, bool NX>
static int launch_lean_shape(OsFdtd3D *h, int set, int config, const Em3DParams &p, const Em3DBox &in,
                             cudaStream_t s) {
    static bool attr_set = false;   // per template instance; the attribute outlives the handle
    if (!attr_set) {
        OS_CUDA(cudaFuncSetAttribute(em3d_lean_kernel<TY, RING, MINB, CA1, HU, EARLY, NX>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)em3d_lean_smem<TY, RING, NX>(EM3D_LEAN_MAX_ZROWS)));
        attr_set = true;
    }
    const Em3DLeanMaps *maps = nullptr;
    OS_TRY((lean_maps<TY, NX>(h, set, config, &maps)));
    const dim3 grid((unsigned)((in.k1 - (in.k0 & ~3) + EM3D_LTILE - 1) / EM3D_LTILE),
                    (unsigned)(NX ? (in.j1 - in.j0 + TY - 1) / TY : (in.j1 - in.j0 + TY - 2) / (TY - 1)),
                    (unsigned)((in.i1 - in.i0 + p.x_chunk - 1) / p.x_chunk));
    em3d_lean_kernel<TY, RING, MINB, CA1, HU, EARLY, NX>
        <<<grid, dim3(32, TY), em3d_lean_smem<TY, RING, NX>(p.cpml[2].nr), s>>>(p, in, *maps);
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

template <bool CA1, bool HU>
static int launch_lean_ca(OsFdtd3D *h, int set, int config, const Em3DParams &p, const Em3DBox &in, cudaStream_t s) {
    switch (config) {
        case 0: return launch_lean_shape<16, 3, 1, CA1, HU, false, false>(h, set, config, p, in, s);
        case 1: return launch_lean_shape<8, 3, 2, CA1, HU, false, false>(h, set, config, p, in, s);
        case 3: return launch_lean_shape<6, 4, 2, CA1, HU, true, false>(h, set, config, p, in, s);
        case 4: return launch_lean_shape<8, 3, 2, CA1, HU, true, true>(h, set, config, p, in, s);
        default: return launch_lean_shape<8, 3, 2, CA1, HU, true, false>(h, set, config, p, in, s);
    }
}

// The lean kernel streams chunks of at most EM3D_LEAN_MAX_PLANES - 1 planes (its per-plane table).
static int launch_lean(OsFdtd3D *h, int set, Em3DParams p, const Em3DBox &in, cudaStream_t s) {
    const int config = h->fused_config < 0 ? 2 : h->fused_config % LEAN_CONFIGS;
    p.x_chunk = std::min<int32_t>(p.x_chunk, EM3D_LEAN_MAX_PLANES - 1);
    if (h->ca_one)
        return h->h_uniform ? launch_lean_ca<true, true>(h, set, config, p, in, s)
                            : launch_lean_ca<true, false>(h, set, config, p, in, s);
    return h->h_uniform ? launch_lean_ca<false, true>(h, set, config, p, in, s)
                        : launch_lean_ca<false, false>(h, set, config, p, in, s);
}

template <int TY, int MINB>
static int launch_staged_shape(dim3 grid, const Em3DParams &p, const Em3DBox &in, const Em3DMaps &maps,
                               cudaStream_t s) {
    constexpr size_t bytes = em3d_staged_smem<TY>();
    static bool attr_set = false;   // per template instance; the attribute outlives the handle
    if (!attr_set) {
        OS_CUDA(cudaFuncSetAttribute(em3d_staged_kernel<TY, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes));
        attr_set = true;
    }
    em3d_staged_kernel<TY, MINB><<<grid, dim3(EM3D_FZ, TY), bytes, s>>>(p, in, maps);
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

static int launch_staged(OsFdtd3D *h, int set, dim3 grid, const Em3DParams &p, const Em3DBox &in, cudaStream_t s) {
    const int config = fused_cfg(h);
    const Em3DMaps *maps = nullptr;
    OS_TRY(staged_maps(h, set, fused_rows(config), &maps));
    switch (config) {
        case 0: return launch_staged_shape<16, 1>(grid, p, in, *maps, s);
        case 1: return launch_staged_shape<16, 2>(grid, p, in, *maps, s);
        case 2: return launch_staged_shape<8, 2>(grid, p, in, *maps, s);
        case 3: return launch_staged_shape<8, 3>(grid, p, in, *maps, s);
        default: return launch_staged_shape<8, 4>(grid, p, in, *maps, s);
    }
}

static int launch_fused(int config, dim3 grid, const Em3DParams &p, const Em3DBox &in, cudaStream_t s) {
    switch (config) {
        case 0: em3d_fused_kernel<16, 1><<<grid, dim3(EM3D_FZ, 16), 0, s>>>(p, in); break;
        case 1: em3d_fused_kernel<16, 2><<<grid, dim3(EM3D_FZ, 16), 0, s>>>(p, in); break;
        case 2: em3d_fused_kernel<8, 2><<<grid, dim3(EM3D_FZ, 8), 0, s>>>(p, in); break;
        case 3: em3d_fused_kernel<8, 3><<<grid, dim3(EM3D_FZ, 8), 0, s>>>(p, in); break;
        default: em3d_fused_kernel<8, 4><<<grid, dim3(EM3D_FZ, 8), 0, s>>>(p, in); break;
    }
    OS_CUDA(cudaGetLastError());
    return OS_OK;
}

// Point p's inputs at set `in` and its outputs at set `out` (components from c0 to c0 + 2 of each, or all).
static void point_sets(const OsFdtd3D *h, Em3DParams &p, int e_in, int h_in, int e_out, int h_out) {
    p.ex = fset(h, e_in, 0);
    p.ey = fset(h, e_in, 1);
    p.ez = fset(h, e_in, 2);
    p.hx = fset(h, h_in, 3);
    p.hy = fset(h, h_in, 4);
    p.hz = fset(h, h_in, 5);
    p.oex = fset(h, e_out, 0);
    p.oey = fset(h, e_out, 1);
    p.oez = fset(h, e_out, 2);
    p.ohx = fset(h, h_out, 3);
    p.ohy = fset(h, h_out, 4);
    p.ohz = fset(h, h_out, 5);
}

}  // namespace os

using namespace os;

extern "C" int os_fdtd3d_create(const OsGrid3D *grid, OsFdtd3D **out) {
    OS_CHECK(grid && out, OS_ERR_INVALID, "os_fdtd3d_create: null argument");
    *out = nullptr;
    const OsGrid3D g = *grid;
    OS_CHECK(g.nx >= 1 && g.ny >= 1 && g.nz >= 1, OS_ERR_INVALID, "os_fdtd3d_create: grid %d x %d x %d has no cells",
             g.nx, g.ny, g.nz);
    OS_CHECK(g.ny <= 65535 * EM3D_BY && (int64_t)g.ny * g.nz < ((int64_t)1 << 31) &&
                 (int64_t)g.nx * g.ny * g.nz < ((int64_t)1 << 40), OS_ERR_INVALID,
             "os_fdtd3d_create: grid %d x %d x %d too large", g.nx, g.ny, g.nz);
    std::unique_ptr<OsFdtd3D> h(new OsFdtd3D());
    h->grid = g;
    h->device = g.device;
    OS_TRY(bind3(h.get()));
    OS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    OS_CUDA(cudaEventCreate(&h->ev_start));
    OS_CUDA(cudaEventCreate(&h->ev_stop));
    const size_t n = cells3(h.get());
    for (auto &f : h->field) OS_TRY(f.alloc(n));
    OS_TRY(h->mat.alloc(n));
    OS_TRY(h->rows.alloc(4 * ((size_t)g.nx + g.ny + g.nz)));
    OS_TRY(h->scratch.alloc(1));
    OS_TRY(h->err.alloc(1));
    OS_CUDA(cudaMemsetAsync(h->err.ptr, 0, sizeof(int32_t), h->stream));
    // x chunk: short runs of 24 planes per block (many more blocks than resident slots, so the last wave is a small
    // share of the launch; on 512^3 the step ran 37.9 G cell-updates/s at 256 planes, 48.6-50.4 at 12-32)
    h->x_chunk = std::min<int32_t>(g.nx, 24);
    OS_TRY(zero_state3(h.get()));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return OS_OK;
}

extern "C" int os_fdtd3d_destroy(OsFdtd3D *h) {
    if (!h) return OS_OK;
    cudaSetDevice(h->device);
    // only the handle's own stream: a caller's stream (os_fdtd3d_set_stream) may already be destroyed
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    cudaStream_t s = h->own_stream;
    delete h;
    if (s) cudaStreamDestroy(s);
    return OS_OK;
}

extern "C" int os_fdtd3d_set_rows(OsFdtd3D *h, const float *inv_e_x, const float *inv_e_y, const float *inv_e_z,
                                  const float *inv_h_x, const float *inv_h_y, const float *inv_h_z,
                                  const float *shares) {
    OS_CHECK(h && inv_e_x && inv_e_y && inv_e_z && inv_h_x && inv_h_y && inv_h_z && shares, OS_ERR_INVALID,
             "os_fdtd3d_set_rows: null argument");
    OS_TRY(bind3(h));
    const OsGrid3D &g = h->grid;
    std::vector<float> all;
    all.reserve(4 * ((size_t)g.nx + g.ny + g.nz));
    all.insert(all.end(), inv_e_x, inv_e_x + g.nx);
    all.insert(all.end(), inv_e_y, inv_e_y + g.ny);
    all.insert(all.end(), inv_e_z, inv_e_z + g.nz);
    all.insert(all.end(), inv_h_x, inv_h_x + g.nx);
    all.insert(all.end(), inv_h_y, inv_h_y + g.ny);
    all.insert(all.end(), inv_h_z, inv_h_z + g.nz);
    all.insert(all.end(), shares, shares + 2 * ((size_t)g.nx + g.ny + g.nz));
    OS_CUDA(cudaMemcpyAsync(h->rows.ptr, all.data(), all.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    h->same_ok = true;
    for (size_t q = 0; q < 2 * ((size_t)g.nx + g.ny + g.nz); ++q)
        if (shares[q] != 0.5f) h->same_ok = false;
    h->has_spacings = true;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_materials(OsFdtd3D *h, const uint16_t *material_id, int32_t n_ids, const float *t_ex,
                                       const float *t_ey, const float *t_ez, const float *t_sig, const float *t_mu,
                                       const float *t_sm, float dt) {
    OS_CHECK(h && material_id && t_ex && t_ey && t_ez && t_sig && t_mu && t_sm, OS_ERR_INVALID,
             "os_fdtd3d_set_materials: null argument");
    OS_CHECK(n_ids >= 1 && n_ids <= 65536, OS_ERR_INVALID, "os_fdtd3d_set_materials: %d material ids (1..65536)",
             n_ids);
    OS_CHECK(dt > 0.0f, OS_ERR_INVALID, "os_fdtd3d_set_materials: dt must be > 0");
    OS_TRY(bind3(h));
    const size_t n = cells3(h);
    OS_CUDA(cudaMemcpyAsync(h->mat.ptr, material_id, n * sizeof(uint16_t), cudaMemcpyHostToDevice, h->stream));
    OS_TRY(h->tables.alloc(6 * (size_t)n_ids));
    h->n_ids = n_ids;
    float *t = h->tables.ptr;
    OS_CUDA(cudaMemcpyAsync(t, t_ex, n_ids * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(t + n_ids, t_ey, n_ids * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(t + 2 * n_ids, t_ez, n_ids * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(t + 3 * n_ids, t_sig, n_ids * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    DeviceArray<float> mu, sm;
    OS_TRY(upload(mu, t_mu, (size_t)n_ids, h->stream));
    OS_TRY(upload(sm, t_sm, (size_t)n_ids, h->stream));
    em3d_h_tables_kernel<<<(n_ids + 255) / 256, 256, 0, h->stream>>>(mu.ptr, sm.ptr, n_ids, dt, t + 4 * n_ids,
                                                                    t + 5 * n_ids);
    OS_CUDA(cudaGetLastError());
    std::vector<float> dadb(2 * (size_t)n_ids);
    OS_CUDA(cudaMemcpyAsync(dadb.data(), t + 4 * n_ids, dadb.size() * sizeof(float), cudaMemcpyDeviceToHost,
                            h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    h->dt = dt;
    h->h_uniform = true;
    h->da_u = dadb[0];
    h->db_u = dadb[n_ids];
    for (int32_t m = 1; m < n_ids; ++m)
        if (dadb[m] != h->da_u || dadb[n_ids + m] != h->db_u) h->h_uniform = false;
    h->e_lossless = true;
    for (int32_t m = 0; m < n_ids; ++m)
        if (t_sig[m] != 0.0f) h->e_lossless = false;
    h->ca_one = h->e_lossless;   // a face between two perfect conductors has ca = 0
    for (int32_t m = 0; m < n_ids; ++m)
        if (t_ex[m] < 0.0f || t_ey[m] < 0.0f || t_ez[m] < 0.0f) h->ca_one = false;
    OS_TRY(h->same.alloc(6 * (size_t)n_ids));
    Em3DParams q = make_params3(h);
    em3d_same_tables_kernel<<<(n_ids + 255) / 256, 256, 0, h->stream>>>(q, h->same.ptr);
    OS_CUDA(cudaGetLastError());
    OS_CUDA(cudaStreamSynchronize(h->stream));
    h->has_materials = true;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_cpml_axis(OsFdtd3D *h, int32_t axis, int32_t n_rows, const int32_t *row_map_e,
                                       const float *b_e, const float *gain_e, const int32_t *row_map_h,
                                       const float *b_h, const float *gain_h) {
    OS_CHECK(h && axis >= 0 && axis < 3, OS_ERR_INVALID, "os_fdtd3d_set_cpml_axis: bad handle or axis %d", axis);
    OS_CHECK(n_rows >= 1 && row_map_e && b_e && gain_e && row_map_h && b_h && gain_h, OS_ERR_INVALID,
             "os_fdtd3d_set_cpml_axis: rows and row maps are required (n_rows %d)", n_rows);
    OS_CHECK(!h->grid.periodic[axis], OS_ERR_INVALID, "os_fdtd3d_set_cpml_axis: axis %d is periodic", axis);
    OS_TRY(bind3(h));
    const OsGrid3D &g = h->grid;
    const int n = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
    for (int r = 0; r < n; ++r) {
        OS_CHECK(row_map_e[r] >= -1 && row_map_e[r] < n_rows && row_map_h[r] >= -1 && row_map_h[r] < n_rows,
                 OS_ERR_INVALID, "os_fdtd3d_set_cpml_axis: row map entry %d out of [-1, %d)", r, n_rows);
    }

    auto &c = h->cpml[axis];
    c.nr = n_rows;
    OS_TRY(c.rm.alloc(2 * (size_t)n));
    OS_CUDA(cudaMemcpyAsync(c.rm.ptr, row_map_e, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(c.rm.ptr + n, row_map_h, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    OS_TRY(c.coef.alloc(4 * (size_t)n_rows));
    OS_CUDA(cudaMemcpyAsync(c.coef.ptr, b_e, n_rows * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(c.coef.ptr + n_rows, gain_e, n_rows * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(c.coef.ptr + 2 * n_rows, b_h, n_rows * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    OS_CUDA(cudaMemcpyAsync(c.coef.ptr + 3 * n_rows, gain_h, n_rows * sizeof(float), cudaMemcpyHostToDevice,
                            h->stream));
    const size_t other = axis == 0 ? (size_t)g.ny * g.nz : (axis == 1 ? (size_t)g.nx * g.nz : (size_t)g.nx * g.ny);
    c.psi_count = other * (size_t)n_rows;
    OS_TRY(c.psi.alloc(4 * c.psi_count));
    OS_CUDA(cudaMemsetAsync(c.psi.ptr, 0, c.psi.bytes(), h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_face_cb(OsFdtd3D *h, int32_t comp, int32_t i, int32_t j, int32_t k, float *cb) {
    OS_CHECK(h && cb && comp >= 0 && comp < 3, OS_ERR_INVALID, "os_fdtd3d_face_cb: bad argument");
    OS_CHECK(h->has_materials && h->has_spacings, OS_ERR_STATE, "os_fdtd3d_face_cb: materials and rows must be set");
    const OsGrid3D &g = h->grid;
    OS_CHECK(i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz, OS_ERR_INVALID,
             "os_fdtd3d_face_cb: cell (%d, %d, %d) outside the grid", i, j, k);
    OS_TRY(bind3(h));
    em3d_face_cb_kernel<<<1, 1, 0, h->stream>>>(make_params3(h), comp, i, j, k, h->scratch.ptr);
    OS_CUDA(cudaGetLastError());
    OS_CUDA(cudaMemcpyAsync(cb, h->scratch.ptr, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_add_dipole(OsFdtd3D *h, int32_t comp, int32_t i, int32_t j, int32_t k, float weight,
                                    int32_t *dipole_id) {
    OS_CHECK(h && comp >= 0 && comp < 3, OS_ERR_INVALID, "os_fdtd3d_add_dipole: bad handle or component %d", comp);
    const OsGrid3D &g = h->grid;
    OS_CHECK(i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz, OS_ERR_INVALID,
             "os_fdtd3d_add_dipole: cell (%d, %d, %d) outside the grid", i, j, k);
    OS_CHECK((int)h->dipoles.size() < EM3D_MAX_DIPOLES, OS_ERR_INVALID, "os_fdtd3d_add_dipole: at most %d dipoles",
             EM3D_MAX_DIPOLES);
    h->dipoles.push_back({comp, i, j * g.nz + k, weight});
    if (dipole_id) *dipole_id = (int32_t)h->dipoles.size() - 1;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_dipole_weight(OsFdtd3D *h, int32_t dipole_id, float weight) {
    OS_CHECK(h && dipole_id >= 0 && dipole_id < (int32_t)h->dipoles.size(), OS_ERR_INVALID,
             "os_fdtd3d_set_dipole_weight: no dipole %d", dipole_id);
    h->dipoles[dipole_id].weight = weight;
    return OS_OK;
}

extern "C" int os_fdtd3d_add_flux_monitor(OsFdtd3D *h, int32_t nf, int32_t *monitor_id) {
    OS_CHECK(h && nf >= 1 && monitor_id, OS_ERR_INVALID, "os_fdtd3d_add_flux_monitor: bad argument (nf %d)", nf);
    h->monitor_nf.push_back(nf);
    *monitor_id = (int32_t)h->monitor_nf.size() - 1;
    return OS_OK;
}

extern "C" int os_fdtd3d_add_flux_pair(OsFdtd3D *h, int32_t monitor_id, int32_t e_comp, int32_t h_comp,
                                       int32_t normal_axis, int32_t edge, const int32_t *origin,
                                       const int32_t *extent, int32_t *pair_id) {
    OS_CHECK(h && origin && extent && pair_id, OS_ERR_INVALID, "os_fdtd3d_add_flux_pair: null argument");
    OS_CHECK(monitor_id >= 0 && monitor_id < (int32_t)h->monitor_nf.size(), OS_ERR_INVALID,
             "os_fdtd3d_add_flux_pair: no monitor %d", monitor_id);
    OS_CHECK(e_comp >= 0 && e_comp < 3 && h_comp >= 0 && h_comp < 3 && normal_axis >= 0 && normal_axis < 3,
             OS_ERR_INVALID, "os_fdtd3d_add_flux_pair: components and axis must be 0, 1 or 2");
    const OsGrid3D &g = h->grid;
    const int dims[3] = {g.nx, g.ny, g.nz};
    OS_CHECK(edge >= 1 && edge <= dims[normal_axis] - 1, OS_ERR_INVALID,
             "os_fdtd3d_add_flux_pair: edge %d needs a cell on both sides (1..%d)", edge, dims[normal_axis] - 1);
    OS_CHECK(extent[normal_axis] == 1, OS_ERR_INVALID, "os_fdtd3d_add_flux_pair: extent along the normal must be 1");
    int64_t count = 1;
    for (int a = 0; a < 3; ++a) {
        if (a == normal_axis) continue;
        OS_CHECK(extent[a] >= 1 && origin[a] >= 0 && origin[a] + extent[a] <= dims[a], OS_ERR_INVALID,
                 "os_fdtd3d_add_flux_pair: samples [%d, %d) outside axis %d of %d cells", origin[a],
                 origin[a] + extent[a], a, dims[a]);
        count *= extent[a];
    }
    OS_CHECK(count <= ((int64_t)1 << 30), OS_ERR_INVALID, "os_fdtd3d_add_flux_pair: too many samples");
    OS_TRY(bind3(h));
    Em3DFluxPair q{};
    q.e_comp = e_comp;
    q.h_comp = h_comp;
    q.normal = normal_axis;
    q.edge = edge;
    for (int a = 0; a < 3; ++a) {
        q.o[a] = a == normal_axis ? 0 : origin[a];
        q.n[a] = extent[a];
    }
    q.nf = h->monitor_nf[monitor_id];
    int32_t offset = 0;
    for (int32_t m = 0; m < monitor_id; ++m) offset += 2 * h->monitor_nf[m];
    q.phase_offset = offset;
    auto acc = std::make_unique<DeviceArray<double>>();
    OS_TRY(acc->alloc(4 * (size_t)q.nf * (size_t)count));
    OS_CUDA(cudaMemsetAsync(acc->ptr, 0, acc->bytes(), h->stream));
    q.e_acc = acc->ptr;
    q.h_acc = acc->ptr + 2 * (size_t)q.nf * (size_t)count;
    h->acc.push_back(std::move(acc));
    h->pairs.push_back(q);
    h->max_pair_cells = std::max<int32_t>(h->max_pair_cells, (int32_t)count);
    h->pairs_dirty = true;
    *pair_id = (int32_t)h->pairs.size() - 1;
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_set_sample_interval(OsFdtd3D *h, int64_t sample_interval) {
    OS_CHECK(h && sample_interval >= 1, OS_ERR_INVALID, "sample interval must be >= 1");
    h->sample_interval = sample_interval;
    return OS_OK;
}

extern "C" int os_fdtd3d_advance(OsFdtd3D *h, int64_t n_steps, const float *dipole_values, int64_t first_sample,
                                 int64_t n_samples, const float *phases) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_advance: null handle");
    OS_CHECK(n_steps >= 0, OS_ERR_INVALID, "n_steps must be >= 0, got %lld", (long long)n_steps);
    OS_CHECK(h->has_materials && h->has_spacings, OS_ERR_STATE, "os_fdtd3d_advance: materials and rows must be set");
    h->launches = 0;
    if (n_steps == 0) return OS_OK;
    OS_CHECK(h->dipoles.empty() || dipole_values, OS_ERR_INVALID, "os_fdtd3d_advance: dipole_values is required");
    const int64_t m = h->sample_interval;
    const int64_t q_first = h->n_step / m + 1, q_last = (h->n_step + n_steps) / m;
    int32_t row_floats = 0;
    for (int32_t nf : h->monitor_nf) row_floats += 2 * nf;
    const bool sampling = !h->pairs.empty() && q_last >= q_first;
    if (sampling)
        OS_CHECK(phases && first_sample <= q_first && first_sample + n_samples - 1 >= q_last, OS_ERR_INVALID,
                 "os_fdtd3d_advance: the phase table covers samples [%lld, %lld), the chunk needs [%lld, %lld]",
                 (long long)first_sample, (long long)(first_sample + n_samples), (long long)q_first,
                 (long long)q_last);
    OS_TRY(bind3(h));
    if (!h->dipoles.empty()) OS_TRY(upload(h->values, dipole_values, h->dipoles.size() * (size_t)n_steps, h->stream));
    if (sampling) OS_TRY(upload(h->phases, phases, (size_t)n_samples * row_floats, h->stream));
    if (h->pairs_dirty) {
        OS_TRY(upload(h->pairs_dev, h->pairs.data(), h->pairs.size(), h->stream));
        h->pairs_dirty = false;
    }
    const bool fused = fused_active(h), staged = staged_active(h), lean = lean_active(h);
    if (fused) {
        for (auto &f : h->field2)
            if (!f.ptr) OS_TRY(f.alloc(cells3(h)));
        for (auto &c : h->cpml)
            if (c.nr && !c.psi2.ptr) OS_TRY(c.psi2.alloc(4 * c.psi_count));
    }
    Em3DParams p = make_params3(h);
    p.dip_values = h->values.ptr;
    p.values_stride = n_steps;
    Em3DParams pd = p;   // the lean form adds the dipoles after the step, in em3d_dipole_kernel
    if (lean) p.n_dip = 0;
    Em3DParams faces[3] = {p, p, p};
    if (fused)
        for (int f = 0; f < 3; ++f) face_boxes(h, faces[f], f);
    const Em3DBox in = lean ? lean_box(h) : fused_box(h);
    const bool z_faces = in.k0 > 0;   // the z faces need launches of their own
    const int ty = fused_rows(fused_cfg(h));
    const dim3 block(EM3D_BZ, EM3D_BY);
    const dim3 fused_grid((unsigned)((in.k1 - in.k0 + EM3D_FZ - 2) / (EM3D_FZ - 1)),
                          (unsigned)((in.j1 - in.j0 + ty - 2) / (ty - 1)),
                          (unsigned)((in.i1 - in.i0 + p.x_chunk - 1) / p.x_chunk));
    OS_CUDA(cudaEventRecord(h->ev_start, h->stream));
    for (int64_t k = 0; k < n_steps; ++k) {
        p.k_step = k;
        for (auto &f : faces) f.k_step = k;
        pd.k_step = k;
        if (fused) {
            const int a = h->cur, b = a ^ 1;
            // faces H: E^n, H^{n-1/2}, psi of set a -> H^{n+1/2}, psi' of set b
            point_sets(h, p, a, a, b, b);
            point_psi(h, p, a, b);
            for (auto &f : faces) {
                point_sets(h, f, a, a, b, b);
                point_psi(h, f, a, b);
            }
            h->launches += launch_faces(h, faces, false, z_faces);
            if (lean) OS_TRY(launch_lean(h, a, p, in, h->stream));
            else if (staged) OS_TRY(launch_staged(h, a, fused_grid, p, in, h->stream));
            else OS_TRY(launch_fused(fused_cfg(h), fused_grid, p, in, h->stream));
            // faces E: E^n and psi of set a, H^{n+1/2} of set b -> E^{n+1}, psi' of set b
            for (auto &f : faces) point_sets(h, f, a, b, b, b);
            h->launches += launch_faces(h, faces, true, z_faces) + 1;
            if (lean && pd.n_dip) {
                point_sets(h, pd, a, b, b, b);
                em3d_dipole_kernel<<<1, 1, 0, h->stream>>>(pd);
                h->launches += 1;
            }
            h->cur = b;
        } else {
            const dim3 grid = box_grid(p);
            em3d_h_kernel<EM3D_BZ, EM3D_BY><<<grid, block, 0, h->stream>>>(p);
            em3d_e_kernel<EM3D_BZ, EM3D_BY><<<grid, block, 0, h->stream>>>(p);
            h->launches += 2;
        }
        h->n_step += 1;
        if (!h->pairs.empty() && h->n_step % m == 0) {
            const int64_t q = h->n_step / m;
            const dim3 fgrid((unsigned)((h->max_pair_cells + 255) / 256), (unsigned)h->pairs.size());
            const int c = h->cur;
            em3d_flux_kernel<<<fgrid, 256, 0, h->stream>>>(h->pairs_dev.ptr, fset(h, c, 0), fset(h, c, 1),
                                                            fset(h, c, 2), fset(h, c, 3), fset(h, c, 4), fset(h, c, 5),
                                                            h->grid.ny, h->grid.nz,
                                                            h->phases.ptr + (size_t)(q - first_sample) * row_floats);
            h->launches += 1;
        }
    }
    OS_CUDA(cudaGetLastError());
    OS_CUDA(cudaEventRecord(h->ev_stop, h->stream));
    h->timed = true;
    return OS_OK;
}

extern "C" int os_fdtd3d_read_field(OsFdtd3D *h, int32_t component, float *out) {
    OS_CHECK(h && out && component >= 0 && component < 6, OS_ERR_INVALID, "os_fdtd3d_read_field: bad argument");
    OS_TRY(bind3(h));
    OS_CUDA(cudaMemcpyAsync(out, fset(h, h->cur, component), h->field[component].bytes(), cudaMemcpyDeviceToHost,
                            h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return check_err3(h);
}

extern "C" int os_fdtd3d_write_field(OsFdtd3D *h, int32_t component, const float *in) {
    OS_CHECK(h && in && component >= 0 && component < 6, OS_ERR_INVALID, "os_fdtd3d_write_field: bad argument");
    OS_TRY(bind3(h));
    OS_CUDA(cudaMemcpyAsync(fset(h, h->cur, component), in, h->field[component].bytes(), cudaMemcpyHostToDevice,
                            h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_read_flux_pair(OsFdtd3D *h, int32_t pair_id, double *e_spectra, double *h_spectra) {
    OS_CHECK(h && e_spectra && h_spectra && pair_id >= 0 && pair_id < (int32_t)h->pairs.size(), OS_ERR_INVALID,
             "os_fdtd3d_read_flux_pair: bad argument");
    OS_TRY(bind3(h));
    const Em3DFluxPair &q = h->pairs[pair_id];
    const size_t n = 2 * (size_t)q.nf * q.n[0] * q.n[1] * q.n[2];
    OS_CUDA(cudaMemcpyAsync(e_spectra, q.e_acc, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaMemcpyAsync(h_spectra, q.h_acc, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_reset(OsFdtd3D *h) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_reset: null handle");
    OS_TRY(bind3(h));
    OS_TRY(zero_state3(h));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return OS_OK;
}

extern "C" int os_fdtd3d_synchronize(OsFdtd3D *h) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_synchronize: null handle");
    OS_TRY(bind3(h));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    return check_err3(h);
}

extern "C" int os_fdtd3d_set_stream(OsFdtd3D *h, void *cuda_stream) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_set_stream: null handle");
    OS_TRY(bind3(h));
    OS_CUDA(cudaStreamSynchronize(h->stream));
    h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_x_chunk(OsFdtd3D *h, int32_t planes) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_set_x_chunk: null handle");
    OS_CHECK(planes >= 1, OS_ERR_INVALID, "x chunk must be >= 1 plane, got %d", planes);
    h->x_chunk = planes;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_variant(OsFdtd3D *h, int32_t variant) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_set_variant: null handle");
    OS_CHECK(variant >= 0 && variant <= 3, OS_ERR_INVALID,
             "variant must be 0 (two in-place kernels), 1 (fused, two field sets), 2 (fused with staged planes) or 3 "
             "(lean staged fused pass), got %d", variant);
    h->variant = variant;
    return OS_OK;
}

extern "C" int os_fdtd3d_set_fused_config(OsFdtd3D *h, int32_t config) {
    OS_CHECK(h, OS_ERR_INVALID, "os_fdtd3d_set_fused_config: null handle");
    OS_CHECK(config >= -1 && config < FUSED_CONFIGS, OS_ERR_INVALID,
             "fused kernel configuration must be in [-1, %d), got %d", FUSED_CONFIGS, config);
    h->fused_config = config;
    return OS_OK;
}

extern "C" int os_fdtd3d_interior(OsFdtd3D *h, int32_t *box6, int32_t *fused) {
    OS_CHECK(h && box6 && fused, OS_ERR_INVALID, "os_fdtd3d_interior: null argument");
    const Em3DBox b = lean_active(h) ? lean_box(h) : fused_box(h);
    const int32_t v[6] = {b.i0, b.i1, b.j0, b.j1, b.k0, b.k1};
    for (int q = 0; q < 6; ++q) box6[q] = v[q];
    *fused = fused_active(h) ? 1 : 0;
    return OS_OK;
}

extern "C" int os_fdtd3d_last_advance_ms(OsFdtd3D *h, float *ms) {
    OS_CHECK(h && ms, OS_ERR_INVALID, "os_fdtd3d_last_advance_ms: null argument");
    OS_CHECK(h->timed, OS_ERR_STATE, "os_fdtd3d_last_advance_ms: no advance recorded yet");
    OS_TRY(bind3(h));
    OS_CUDA(cudaEventSynchronize(h->ev_stop));
    OS_CUDA(cudaEventElapsedTime(ms, h->ev_start, h->ev_stop));
    return OS_OK;
}

extern "C" int os_fdtd3d_launch_count(OsFdtd3D *h, int64_t *launches) {
    OS_CHECK(h && launches, OS_ERR_INVALID, "os_fdtd3d_launch_count: null argument");
    *launches = h->launches;
    return OS_OK;
}

extern "C" int os_fdtd3d_step_count(OsFdtd3D *h, int64_t *n_step) {
    OS_CHECK(h && n_step, OS_ERR_INVALID, "os_fdtd3d_step_count: null argument");
    *n_step = h->n_step;
    return OS_OK;
}
