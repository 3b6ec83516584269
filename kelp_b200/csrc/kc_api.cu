// C ABI of the B200 time-stepping path (declared in include/kelp_cuda.h):
// context, resident mesh / snapshot ring / particle state, the step kernels'
// launchers and the batch nearest-node query.
#include <cstdio>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/block/block_scan.cuh>

#include "../../include/kelp_cuda.h"
#include "kc_host.h"
#include "kc_launch.h"
#include "kc_beach.cuh"
#include "kc_sample.cuh"
#include "kc_sigma.cuh"

namespace {

constexpr int kSlots = 8;
constexpr int kEvents = 16;
constexpr int kChunks = 64;   // most chunks of one host-buffer step


struct Slot {
    void* u = nullptr;
    void* v = nullptr;
    void* w = nullptr;
    void* az = nullptr;    // vertical diffusivity rows (K, N), same element type as u
    int az_rows = 0;
    size_t cap_az = 0;
    double* eta = nullptr; // free surface (N), float64 (sigma meshes)
    bool has_eta = false;
    long long cap_eta = 0;
    float* su = nullptr;   // per-row scales of half storage
    float* sv = nullptr;
    float* sw = nullptr;
    long long n = 0;
    int uv_rows = 0, w_rows = 0, dtype = -1;
    size_t cap_uv = 0, cap_w = 0, cap_su = 0, cap_sv = 0, cap_sw = 0;
    // kc_field_upload_async: the copy's completion on the copy stream, and
    // the last launch on the library's stream that read the slot
    cudaEvent_t ready = nullptr, used = nullptr;
    bool pending = false, has_used = false;
};

}  // namespace

struct kc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // kc_field_upload_async (created on first use)
    std::string err;
    // mesh
    bool has_mesh = false;
    long long N = 0, E = 0;
    double2* d_ll = nullptr;
    int4* d_en = nullptr;
    int* d_n2e_off = nullptr;
    int* d_n2e = nullptr;
    int* d_gh_off = nullptr;
    double4* d_gh_tab = nullptr;
    int* d_pw_off = nullptr;         // pruned windows of the nearest-node scan
    double4* d_pw_tab = nullptr;
    double* d_xyz = nullptr;
    double* d_depth = nullptr;
    double* d_zlev = nullptr;
    double2* d_nsc = nullptr;
    double2* d_ecos = nullptr;
    float4* d_ebox = nullptr;        // containment prefilter boxes
    double* d_sig_eta_s = nullptr;   // (N) the tracking layer's sigma surfaces set by kc_sigma_surfaces
    double* d_sig_eta_e = nullptr;
    bool sig_s_on = false, sig_e_on = false, sig_steady = false;
    double* d_beach_eta = nullptr;   // (N) beaching surfaces set by kc_beach_surface
    double* d_beach_dry = nullptr;
    bool beach_eta_on = false, beach_dry_on = false;
    double2* d_erec = nullptr;       // per-element mask vertex coordinates
    int* d_maxl = nullptr;
    double* d_dl_p = nullptr;
    int* d_dl_last = nullptr;
    double* d_dl_bed = nullptr;
    int4* d_enb = nullptr;   // edge neighbours of the compacted rings (kc_elem_neighbors_upload)
    double2* d_ec = nullptr;  // element centres (kc_elem_centers_upload)
    double* d_sigma = nullptr;   // sigma interfaces (kc_sigma_upload)
    // NEMO C-grid tables (kc_cgrid_upload)
    int4* d_cg_corners = nullptr;
    int* d_cg_cell = nullptr;
    int* d_cg_nlev = nullptr;
    int* d_cg_nlev_r = nullptr;
    double4* d_cg_L = nullptr;
    double *d_cg_e2u = nullptr, *d_cg_e1v = nullptr, *d_cg_area = nullptr, *d_cg_zw = nullptr, *d_cg_e3b = nullptr;
    double *d_cg_e3u = nullptr, *d_cg_e3v = nullptr;
    int *d_cg_kbu = nullptr, *d_cg_kbv = nullptr;
    int max_v = 0;
    int* d_err = nullptr;
    unsigned *d_rx_a_off = nullptr, *d_rx_b_off = nullptr;   // RNG exception tables (kc::DRngX)
    unsigned short *d_rx_a = nullptr, *d_rx_b = nullptr;
    kc::DMesh dm{};
    // snapshot ring
    Slot slots[kSlots];
    // particles
    long long P = 0, cap = 0;
    double *lon = nullptr, *lat = nullptr, *z = nullptr, *U = nullptr, *V = nullptr, *W = nullptr;
    int *status = nullptr, *nn = nullptr, *rs = nullptr;
    signed char* fr = nullptr;
    long long* pid = nullptr;
    bool has_pid = false, has_rs = false, has_rid = false, has_elem = false;
    int* rid = nullptr;   // per-particle realization ids (ensemble members in one array)
    int* elem = nullptr;  // carried containing elements (elem_search walk)
    int* el = nullptr;    // carried local containment scans (valid where nn_ok bit 1)
    int* wel = nullptr;
    // re-sort by grid-hash cell: upload slot of every resident particle, the
    // spare buffer of the gathers, radix-sort keys / indices and CUB's storage
    long long* orig = nullptr;
    void* spare = nullptr;
    // beaching: entry status of the last step, wet-step counters, coastal flags
    int* prev = nullptr;
    int* wet = nullptr;
    // 1 where nn holds the exact anchor of the particle's current position
    // (written by the step and beaching kernels; cleared by every upload)
    unsigned char* nn_ok = nullptr;
    bool has_beach = false;
    unsigned char* d_coastal = nullptr;
    bool sorted = false;
    unsigned* skey[2] = {nullptr, nullptr};
    int* sidx[2] = {nullptr, nullptr};
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    long long sort_cap = 0;
    // query scratch of kc_find_nearest
    double* q = nullptr;
    int* qout = nullptr;
    long long qcap = 0;
    cudaEvent_t ev[kEvents] = {};
    // the host-buffer step's copy streams and per-chunk events (created on first use)
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_in[kChunks] = {}, ev_k[kChunks] = {}, ev_start = nullptr;
    // L2 eviction buffer of kc_l2_flush
    char* flush = nullptr;
    // fused multi-step launches: per-call argument block (page-locked staging
    // and its device copy), the event after its upload, the cached graph
    void* fused_host = nullptr;
    void* fused_dev = nullptr;
    size_t fused_cap = 0;
    cudaEvent_t fused_ev = nullptr;
    bool fused_ev_pending = false;
    cudaGraphExec_t fused_exec = nullptr;
    std::string fused_key;
    unsigned long long mesh_gen = 0;
    int fused_block = 128;   // particles per block of the fused launch (kc_set_fused_block)
    // float staging buffer of the half-precision snapshot conversion
    float* stage = nullptr;
    size_t stage_cap = 0;
    long long flush_cap = 0;
    unsigned flush_val = 0;
};

namespace {

int fail(kc_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define KC_CUDA(c, call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail((c), KC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename P>
void dfree(P*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

template <typename T>
kc::DField<T> field_of(const Slot& s) {
    return kc::DField<T>{(const T*)s.u, (const T*)s.v, (const T*)s.w, s.su, s.sv, s.sw,
                         s.az_rows > 0 ? (const T*)s.az : nullptr, s.has_eta ? s.eta : nullptr};
}

kc::DState state_of(kc_ctx* c) {
    kc::DState st;
    st.lon = c->lon; st.lat = c->lat; st.z = c->z; st.status = c->status; st.nn = c->nn;
    st.U = c->U; st.V = c->V; st.W = c->W; st.fr = c->fr;
    st.pid = c->has_pid ? c->pid : nullptr;
    st.release_step = c->has_rs ? c->rs : nullptr;
    st.rid = c->has_rid ? c->rid : nullptr;
    st.prev = c->has_beach ? c->prev : nullptr;
    st.nn_ok = c->nn_ok;
    st.elem = c->has_elem ? c->elem : nullptr;
    st.el = c->el;
    st.wel = c->wel;
    st.P = c->P;
    return st;
}

kc::DStep step_of(const kc_step_args* a) {
    kc::DStep s;
    s.dt = a->dt; s.time_dir = a->time_dir;
    for (int k = 0; k < 4; ++k) s.ak[k] = a->alpha_k[k];
    s.w_code = a->w_code; s.kick = a->kick; s.uv_dl = a->uv_vertical;
    s.kh_x = a->kh_x; s.kh_y = a->kh_y;
    s.seed = a->seed; s.real_id = a->real_id; s.step_i = a->step_i; s.pid_offset = a->pid_offset;
    s.global_step = a->global_step;
    s.az_on = a->az_kick; s.az_field = a->az_field; s.az_const = a->az_const;
    s.Dmin = a->Dmin; s.z0b_min = a->z0b_min; s.alpha_end = a->alpha_end;
    s.eta_s = nullptr; s.eta_e = nullptr; s.sig_steady = 0;
    s.edge_bc = a->uv_lsq >= 2 ? a->uv_lsq - 2 : -1;
    return s;
}

// sampling.py:383-429 / :487-541: one particle per thread; dead particles
// and negative anchors give NaN.
__global__ void __launch_bounds__(kBlock) k_sample(const __grid_constant__ kc::DMesh m, const kc::DSample S,
                                                   const double* q, const double* z, const int* nn,
                                                   const unsigned char* alive, long long P, int method, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int a = nn[i];
    if ((alive && !alive[i]) || a < 0) {
        out[i] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    out[i] = kc::sample_point(m, S, q[i], q[P + i], z ? z[i] : 0.0, a, method);
}

// sampling.py:876-890: an interface-shaped (K, N) field through the W
// interpolation of the method (vertical.py:1330-1420 interp_w_spatial,
// time_dir +1): nearest = the anchor's column, leastsq / idw = the 1-ring,
// barycentric = the containing element's vertex columns.
__global__ void __launch_bounds__(kBlock) k_sample_iface(const __grid_constant__ kc::DMesh m,
                                                         const kc::DBlend<double> f, const double* q, const double* z,
                                                         const int* nn, const unsigned char* alive, long long P,
                                                         int method, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int a = nn[i];
    if ((alive && !alive[i]) || a < 0) {
        out[i] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const double lon = q[i], lat = q[P + i], zp = z[i];
    if (method == kc::S_NEAREST) out[i] = kc::w_linear<double>(m, f, 0.0, zp, a, 1.0);
    else if (method == kc::S_BARYCENTRIC) out[i] = kc::w_bary<double>(m, f, 0.0, lon, lat, zp, a, 1.0);
    else out[i] = kc::w_ring<double>(m, f, method == kc::S_LEASTSQ ? 2 : 3, 0.0, lon, lat, zp, a, 1.0);
}

// sampling.py:659-689 on a sigma mesh: an interface field (K, N) through the
// sigma W interpolation of the method (vertical_sigma.py:971-1031, the
// columns max(depth + eta, Dmin)); mid-layer fields take k_sample with the
// sigma columns in DSample.
__global__ void __launch_bounds__(kBlock) k_sample_iface_sigma(const __grid_constant__ kc::DMesh m,
                                                               const kc::DBlend<double> f,
                                                               const __grid_constant__ kc::DStep s, const double* q,
                                                               const double* z, const int* nn,
                                                               const unsigned char* alive, long long P, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int a = nn[i];
    if ((alive && !alive[i]) || a < 0) {
        out[i] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const double lon = q[i], lat = q[P + i];
    kc::SigSite site;
    kc::sigma_site<double>(m, f, s, 0, lon, lat, a, site);
    out[i] = kc::w_sig<double>(m, f, s, 0, lon, lat, z[i], a, site);
}

__global__ void __launch_bounds__(kBlock) k_nearest(const __grid_constant__ kc::DMesh m, const double* q, long long P, int* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    out[i] = kc::site_anchor(m, kc::make_site(q[i], q[P + i]));
}

// mesh.py:2631-2712 find_containing_elements_walk: the walk from start[i]
// with its fallbacks; the exact anchor of the heal is searched here.  out may
// alias start (each thread reads its own entry first).
__global__ void __launch_bounds__(kBlock) k_walk(const __grid_constant__ kc::DMesh m, const double* q, long long P,
                                                 const int* start, int* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const double lon = q[i], lat = q[P + i];
    const int s = start[i];
    const int nn = kc::site_anchor(m, kc::make_site(lon, lat));
    out[i] = kc::walk_locate(m, lon, lat, s, nn);
}

// mesh.py:2286-2324 find_containing_elements: the local 1-ring / 2-ring scan
// around nn[i] (null: the exact anchor of the point); -1 outside.
__global__ void __launch_bounds__(kBlock) k_contain(const __grid_constant__ kc::DMesh m, const double* q, long long P,
                                                    const int* nn, int* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const double lon = q[i], lat = q[P + i];
    const int a = nn ? nn[i] : kc::site_anchor(m, kc::make_site(lon, lat));
    out[i] = kc::contain_local(m, lon, lat, a);
}

__global__ void __launch_bounds__(kBlock) k_normals(const kc::DRngX x, long long P, unsigned long long seed,
                                                    unsigned long long real_id, unsigned long long step,
                                                    unsigned long long pid0, unsigned long long comp, double* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    double g1, g2;
    kc::normal_pair<true>(x, seed, real_id, (unsigned long long)i + pid0, step, comp, g1, g2);
    out[2 * i] = g1;
    out[2 * i + 1] = g2;
}

// Order-free digests over the whole Box-Muller input domain j = 0 .. 2^32-1:
// the sums of mix(mix(j) ^ bits(v)) of v = sqrt(-2 log u), cos(2 pi u) and
// sin(2 pi u) at u = (j + 1/2) 2^-32, each as normal_pair evaluates it (with
// the exception tables when x carries them).  out[0..2] += r, cos, sin.
__device__ __forceinline__ unsigned long long rng_mix(unsigned long long v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}

__global__ void __launch_bounds__(256) k_rng_domain(const kc::DRngX x, unsigned long long* out) {
    const double INV = 1.0 / 4294967296.0, HALF = 0.5 * INV, TWO_PI = 2.0 * 3.141592653589793;
    unsigned long long dr = 0, dc = 0, ds = 0;
    const unsigned long long n = 1ull << 32;
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const double u = (double)j * INV + HALF;
        double r = sqrt(-2.0 * kc::cr::log_cr(u));
        double sn, cs;
        kc::cr::sincos_cr(TWO_PI * u, &sn, &cs);
        if (x.a_off) {
            const unsigned ca = kc::rngx_code(x.a_off, x.a, (unsigned)j);
            if (ca) r = kc::rngx_bump(r, ca);
        }
        if (x.b_off) {
            const unsigned cb = kc::rngx_code(x.b_off, x.b, (unsigned)j);
            if (cb & 3u) cs = kc::rngx_bump(cs, cb & 3u);
            if (cb >> 2) sn = kc::rngx_bump(sn, cb >> 2);
        }
        const unsigned long long mj = rng_mix(j);
        dr += rng_mix(mj ^ (unsigned long long)__double_as_longlong(r));
        dc += rng_mix(mj ^ (unsigned long long)__double_as_longlong(cs));
        ds += rng_mix(mj ^ (unsigned long long)__double_as_longlong(sn));
    }
    for (int o = 16; o > 0; o >>= 1) {
        dr += __shfl_down_sync(0xFFFFFFFFu, dr, o);
        dc += __shfl_down_sync(0xFFFFFFFFu, dc, o);
        ds += __shfl_down_sync(0xFFFFFFFFu, ds, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], dr);
        atomicAdd(&out[1], dc);
        atomicAdd(&out[2], ds);
    }
}

// The grid hash's cell of every node (mesh.py:980-990 _gh_cell_index: the
// quotient by the cell size truncated toward zero, then clamped), and the
// per-cell node counts.
__global__ void __launch_bounds__(kBlock) k_hash_cells(const double* lon, const double* lat, long long N, double cell,
                                                       double lon_min, double lat_min, int nx, int ny, int wrap,
                                                       unsigned* key, int* val, int* counts) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    int ci = wrap ? (int)(lon[n] / cell) : (int)((lon[n] - lon_min) / cell);
    if (wrap) {
        if (ci > nx - 1) ci = nx - 1;
    } else {
        ci = ci < 0 ? 0 : (ci > nx - 1 ? nx - 1 : ci);
    }
    int cj = (int)((lat[n] - lat_min) / cell);
    cj = cj < 0 ? 0 : (cj > ny - 1 ? ny - 1 : cj);
    const unsigned k = (unsigned)cj * (unsigned)nx + (unsigned)ci;
    key[n] = k;
    val[n] = (int)n;
    atomicAdd(&counts[k], 1);
}

// One of the tracking layer's sigma surfaces from resident records, as
// tracking.py:3097-3133 _eta_at_time evaluates it: kind 1 a record's own eta,
// 2 the linear blend of two records (io.py:68-117 _blend), 3 the
// monotone-cubic value of a four-record stencil at time q
// (temporal_reconstruct.py:87-153 _pchip_blend4).
__global__ void __launch_bounds__(kBlock) k_surface(long long N, int kind, const double* e0, const double* e1,
                                                   const double* e2, const double* e3, double alpha, double t0,
                                                   double t1, double t2, double t3, double q, double* out) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    if (kind == 1) {
        out[n] = e0[n];
    } else if (kind == 2) {
        out[n] = (1.0 - alpha) * e0[n] + alpha * e1[n];
    } else {
        const double t[4] = {t0, t1, t2, t3};
        out[n] = kc::pchip4(e0[n], e1[n], e2[n], e3[n], t, q);
    }
}

// ---------------------------------------------------------------------------
// The occupancy rule's per-sample statistics of one candidate cell
// (mesh.py:384-461 _gh_sample_stats).  cum is the (ny + 1) x (nx + 1) 2-D
// prefix table of the candidate grid's node counts: cum[j][i] = nodes in rows
// < j and columns < i.
// ---------------------------------------------------------------------------

// The candidate cell of every node (the cell rule of k_hash_cells), counted
// into cum[cj + 1][ci + 1] before the prefix passes.
__global__ void __launch_bounds__(kBlock) k_cell_counts(const double* lon, const double2* ll, long long N, double cell,
                                                        double lon_min, double lat_min, int nx, int ny, int wrap,
                                                        int* cum) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    int ci = wrap ? (int)(lon[n] / cell) : (int)((lon[n] - lon_min) / cell);
    if (wrap) {
        if (ci > nx - 1) ci = nx - 1;
    } else {
        ci = ci < 0 ? 0 : (ci > nx - 1 ? nx - 1 : ci);
    }
    int cj = (int)((ll[n].y - lat_min) / cell);
    cj = cj < 0 ? 0 : (cj > ny - 1 ? ny - 1 : cj);
    atomicAdd(&cum[(long long)(cj + 1) * (nx + 1) + ci + 1], 1);
}

// Running sums along each row j = 1..ny of cum (one block per row, the row
// scanned in tiles of the block with a carry between them).
constexpr int kScanBlock = 256;
__global__ void __launch_bounds__(kScanBlock) k_prefix_rows(int* cum, int nx) {
    using Scan = cub::BlockScan<int, kScanBlock>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int carry;
    int* row = cum + (long long)(blockIdx.x + 1) * (nx + 1);
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 1; base <= nx; base += kScanBlock) {
        const int i = base + (int)threadIdx.x;
        const int v = i <= nx ? row[i] : 0;
        int incl, total;
        Scan(tmp).InclusiveSum(v, incl, total);
        if (i <= nx) row[i] = incl + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

// Running sums down each column i = 1..nx (adjacent threads read adjacent
// columns of a row).
__global__ void __launch_bounds__(kBlock) k_prefix_cols(int* cum, int nx, int ny) {
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) + 1;
    if (i > nx) return;
    int acc = 0;
    for (int j = 1; j <= ny; ++j) {
        const long long k = (long long)j * (nx + 1) + i;
        acc += cum[k];
        cum[k] = acc;
    }
}

// mesh.py:353-380 _gh_rect_sum: the nodes of the cells ci-rx..ci+rx x
// cj-ry..cj+ry, rows clipped, columns wrapped on a cyclic grid (one or two
// slices) and clipped otherwise.
__device__ __forceinline__ int rect_nodes(const int* cum, int nx, int ny, int wrap, int ci, int cj, int rx, int ry) {
    const long long W = nx + 1;
    const int j0 = cj - ry < 0 ? 0 : cj - ry;
    const int j1 = cj + ry + 1 > ny ? ny : cj + ry + 1;
    auto span = [&](int a, int b) {   // columns [a, b) of rows [j0, j1)
        return (cum[j1 * W + b] - cum[j0 * W + b]) - (cum[j1 * W + a] - cum[j0 * W + a]);
    };
    if (wrap && 2 * rx + 1 >= nx) return span(0, nx);
    int i0 = ci - rx, i1 = ci + rx + 1;
    if (wrap) {
        if (i0 < 0) return span(0, i1) + span(i0 + nx, nx);
        if (i1 > nx) return span(i0, nx) + span(0, i1 - nx);
    } else {
        if (i0 < 0) i0 = 0;
        if (i1 > nx) i1 = nx;
    }
    return span(i0, i1);
}

// Per sample: its exact nearest node on the resident hash (mr), then the 3x3
// occupancy, the outside-window flag, the certificate's verdict and the
// scan-cost proxy on the candidate grid (mc: the resident mesh's node tables
// with the candidate geometry).  Cost weights: a cell visit 1, a certificate
// evaluation 20 (mesh.py:348-349).
__global__ void __launch_bounds__(kBlock) k_cell_stats(const __grid_constant__ kc::DMesh mr,
                                                       const __grid_constant__ kc::DMesh mc, const int* cum,
                                                       const double* q, long long P, int* nn_out, int* occ_out,
                                                       double* cost_out, signed char* unprov_out,
                                                       signed char* approx_out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const double lon = q[i], lat = q[P + i];
    const kc::Site s = kc::make_site(lon, lat);
    const int n = kc::nearest_exact(mr, s);
    nn_out[i] = n;
    if (n < 0) {
        occ_out[i] = 0; cost_out[i] = 0.0; unprov_out[i] = 0; approx_out[i] = 0;
        return;
    }
    int ci, cj, cin, cjn;
    kc::gh_cell_of(mc, lon, lat, ci, cj);
    const int occ = rect_nodes(cum, mc.nx, mc.ny, mc.wrap, ci, cj, 1, 1);
    occ_out[i] = occ;
    const double2 nl = __ldg(&mc.ll[n]);
    kc::gh_cell_of(mc, nl.x, nl.y, cin, cjn);
    int di = abs(cin - ci);
    if (mc.wrap && mc.nx - di < di) di = mc.nx - di;
    const int dj = abs(cjn - cj);
    const int approx = (di > 1 || dj > 1) ? 1 : 0;
    approx_out[i] = (signed char)approx;
    double theta, ext;
    kc::cap_extents(mc, s, n, theta, ext);
    const bool provable = occ > 0 && !approx && kc::provable_code(mc, s, 1, 1, theta, ext) == 0;
    if (provable) {
        cost_out[i] = (double)occ + 9.0 + 20.0;
        unprov_out[i] = 0;
        return;
    }
    int ry = (int)ceil(theta / mc.cell);
    if (ry < 1) ry = 1;
    if (ry > mc.ny) ry = mc.ny;
    int rx;
    if (ext >= 1.0e29) {
        rx = mc.nx;
    } else {
        rx = (int)ceil(ext / mc.cell);
        if (rx < 1) rx = 1;
    }
    long long cells, iters;
    if (rx * 2LL + 1 >= mc.nx) {
        rx = mc.nx;
        cells = 9 + 2LL * ry;
        iters = ry;
    } else {
        cells = 9 + (long long)rx * (2LL * ry + 1) + 2LL * ry;
        iters = rx > ry ? rx : ry;
    }
    cost_out[i] = ((double)rect_nodes(cum, mc.nx, mc.ny, mc.wrap, ci, cj, rx, ry) + (double)cells) +
                  (double)(iters + 1) * 20.0;
    unprov_out[i] = 1;
}

__global__ void __launch_bounds__(kBlock) k_beach(const __grid_constant__ kc::DMesh m,
                                                  const __grid_constant__ kc::DState st,
                                                  const __grid_constant__ kc::DBeach b, long long N) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.P) return;
    kc::beach_particle(m, st, b, N, i);
}

// Per-row power-of-two scale of a (rows, n) float array for half storage:
// 2^(e - 15) with max|x| = m 2^e, m in [0.5, 1), so every scaled value is
// below 2^15 in magnitude; 1 for an all-zero or non-finite row.
__global__ void k_row_scale(const float* __restrict__ x, long long n, float* __restrict__ scale) {
    const long long row = blockIdx.x;
    float mx = 0.0f;
    for (long long j = threadIdx.x; j < n; j += blockDim.x) mx = fmaxf(mx, fabsf(x[row * n + j]));
    __shared__ float red[256];
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float m = red[0];
        int e = 0;
        float sc = 1.0f;
        if (m > 0.0f && isfinite(m)) {
            frexpf(m, &e);
            sc = ldexpf(1.0f, e - 15);
        }
        scale[row] = sc;
    }
}

__global__ void k_to_half(const float* __restrict__ x, long long n, long long total, const float* __restrict__ scale,
                          __half* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    out[i] = __float2half_rn(x[i] / scale[i / n]);
}

__global__ void k_iota64(long long* out, long long P) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) out[i] = i;
}

// ---- pruned windows of the 3x3 nearest-node scan --------------------------
//
// For each grid-hash cell, the nodes of its 3x3 window (mesh.py:1235-1303
// order) that can be the window's first minimum for some query landing in the
// cell.  A node n is dropped when, on each of kPwSub x kPwSub sub-rectangles
// of the cell (grown by kPwPad degrees for the rounding of the cell index),
// one window node m is closer to every point by more than kPwDelta in squared
// chord: |q-n|^2 - |q-m|^2 = |n|^2 - |m|^2 + 2 q.(m-n) > kPwDelta, with the
// minimum of q.(m-n) over the sub-rectangle bounded from below by
// rect_min_dot.  kPwDelta covers the rounding of the scan's own float64
// distances (|q|, |n|, |m| within 1e-15 of 1), so every dropped node is
// strictly farther than the kept winner in the scan's own arithmetic and the
// first minimum and its distance are unchanged.
constexpr int kPwCap = 256;          // window positions held per cell; a larger window is kept whole
constexpr int kPwSub = 4;            // sub-rectangles per cell side
constexpr double kPwPad = 1e-9;      // degrees added around the cell
constexpr double kPwDelta = 1e-12;   // required margin in squared chord

// min over the sphere points q(l, p) of [l0, l1] x [p0, p1] (spans < pi,
// p within [-pi/2, pi/2]) of q . v.  For fixed p, vx cos l + vy sin l is a
// sinusoid with at most one critical point on the span, a minimum exactly when
// its derivative goes from negative to positive; cos p >= 0 then leaves
// g cos p + vz sin p, reduced the same way.
__device__ double rect_min_dot(double vx, double vy, double vz, const double* cl, const double* sl,
                               const double* cp, const double* sp) {
    double g = fmin(vx * cl[0] + vy * sl[0], vx * cl[1] + vy * sl[1]);
    if (-vx * sl[0] + vy * cl[0] < 0.0 && -vx * sl[1] + vy * cl[1] > 0.0) g = -sqrt(vx * vx + vy * vy);
    double h = fmin(g * cp[0] + vz * sp[0], g * cp[1] + vz * sp[1]);
    if (-g * sp[0] + vz * cp[0] < 0.0 && -g * sp[1] + vz * cp[1] > 0.0) h = -sqrt(g * g + vz * vz);
    return h;
}

// One thread per cell.  counts[cell] = the kept records (pass 1,
// tab_out == null); pass 2 copies them to off[cell] in window order.
__global__ void __launch_bounds__(kBlock) k_elem_boxes(const __grid_constant__ kc::DMesh m, float4* out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < m.E) out[c] = kc::elem_box(m, (int)c);
}

__global__ void __launch_bounds__(kBlock) k_elem_records(const __grid_constant__ kc::DMesh m, double2* out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < m.E) kc::elem_record(m, (int)c, out + 4 * c);
}

__global__ void __launch_bounds__(kBlock) k_prune_windows(const __grid_constant__ kc::DMesh m, int* counts,
                                                          const int* off, double4* tab_out) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= (long long)m.nx * m.ny) return;
    const int ci = (int)(cell % m.nx), cj = (int)(cell / m.nx);
    int pos[kPwCap];
    unsigned keep[kPwCap / 32];
    int n = 0;
    bool whole = false;
    for (int dj = -1; dj <= 1; ++dj) {           // the window in nearest_3x3's order
        const int cj2 = cj + dj;
        if (cj2 < 0 || cj2 >= m.ny) continue;
        for (int di = -1; di <= 1; ++di) {
            int ci2 = ci + di;
            if (ci2 < 0) ci2 = m.wrap ? ci2 + m.nx : -1;
            else if (ci2 >= m.nx) ci2 = m.wrap ? ci2 - m.nx : -1;
            if (ci2 < 0) continue;
            const int c2 = cj2 * m.nx + ci2;
            for (int k = m.gh_off[c2]; k < m.gh_off[c2 + 1]; ++k) {
                if (n < kPwCap) pos[n] = k;
                else whole = true;
                ++n;
            }
        }
    }
    const double lo0 = m.lon_min + (double)ci * m.cell - kPwPad, lo1 = m.lon_min + (double)(ci + 1) * m.cell + kPwPad;
    const double la0 = m.lat_min + (double)cj * m.cell - kPwPad, la1 = m.lat_min + (double)(cj + 1) * m.cell + kPwPad;
    if (!(m.cell < 90.0) || la0 < -90.0 || la1 > 90.0) whole = true;
    for (int w = 0; w < kPwCap / 32; ++w) keep[w] = whole ? 0xFFFFFFFFu : 0u;
    if (!whole && n > 1) {
        const double wl = (lo1 - lo0) / kPwSub, wp = (la1 - la0) / kPwSub;
        for (int b = 0; b < kPwSub && !whole; ++b) {
            double cp[2], sp[2];
            const double p0 = la0 + b * wp, p1 = (b + 1 == kPwSub) ? la1 : la0 + (b + 1) * wp;
            sincos(p0 * kc::DEG2RAD, &sp[0], &cp[0]);
            sincos(p1 * kc::DEG2RAD, &sp[1], &cp[1]);
            const double pc = 0.5 * (p0 + p1);
            for (int a = 0; a < kPwSub && !whole; ++a) {
                double cl[2], sl[2];
                const double l0 = lo0 + a * wl, l1 = (a + 1 == kPwSub) ? lo1 : lo0 + (a + 1) * wl;
                sincos(l0 * kc::DEG2RAD, &sl[0], &cl[0]);
                sincos(l1 * kc::DEG2RAD, &sl[1], &cl[1]);
                double sa, ca, so, co;
                sincos(pc * kc::DEG2RAD, &sa, &ca);
                sincos(0.5 * (l0 + l1) * kc::DEG2RAD, &so, &co);
                const double qx = ca * co, qy = ca * so, qz = sa;
                int m1 = -1, m2 = -1;              // the two window nodes nearest the centre
                double d1 = 1e300, d2 = 1e300;
                for (int j = 0; j < n; ++j) {
                    const double4 t = m.gh_tab[pos[j]];
                    const double dx = t.x - qx, dy = t.y - qy, dz = t.z - qz;
                    const double d = dx * dx + dy * dy + dz * dz;
                    if (d < d1) { d2 = d1; m2 = m1; d1 = d; m1 = j; }
                    else if (d < d2) { d2 = d; m2 = j; }
                }
                if (m1 < 0) { whole = true; break; }   // non-finite table entries: keep the window
                const double4 t1 = m.gh_tab[pos[m1]];
                const double n1 = t1.x * t1.x + t1.y * t1.y + t1.z * t1.z;
                double4 t2 = t1;
                double n2 = n1;
                if (m2 >= 0) { t2 = m.gh_tab[pos[m2]]; n2 = t2.x * t2.x + t2.y * t2.y + t2.z * t2.z; }
                keep[m1 >> 5] |= 1u << (m1 & 31);
                for (int j = 0; j < n; ++j) {
                    if (keep[j >> 5] & (1u << (j & 31))) continue;
                    const double4 t = m.gh_tab[pos[j]];
                    const double nn = t.x * t.x + t.y * t.y + t.z * t.z;
                    bool dom = (nn - n1) + 2.0 * rect_min_dot(t1.x - t.x, t1.y - t.y, t1.z - t.z, cl, sl, cp, sp) >
                               kPwDelta;
                    if (!dom && m2 >= 0 && m2 != j)
                        dom = (nn - n2) + 2.0 * rect_min_dot(t2.x - t.x, t2.y - t.y, t2.z - t.z, cl, sl, cp, sp) >
                              kPwDelta;
                    if (!dom) keep[j >> 5] |= 1u << (j & 31);
                }
            }
        }
    } else if (n <= 1) {
        whole = true;
    }
    if (!tab_out) {
        int cnt = n;
        if (!whole) {
            cnt = 0;
            for (int w = 0; w < kPwCap / 32; ++w) cnt += __popc(keep[w]);
        }
        counts[cell] = cnt;
        return;
    }
    double4* out = tab_out + off[cell];
    int t = 0;
    if (whole) {                                 // the window as it stands, enumerated again
        for (int dj = -1; dj <= 1; ++dj) {
            const int cj2 = cj + dj;
            if (cj2 < 0 || cj2 >= m.ny) continue;
            for (int di = -1; di <= 1; ++di) {
                int ci2 = ci + di;
                if (ci2 < 0) ci2 = m.wrap ? ci2 + m.nx : -1;
                else if (ci2 >= m.nx) ci2 = m.wrap ? ci2 - m.nx : -1;
                if (ci2 < 0) continue;
                const int c2 = cj2 * m.nx + ci2;
                for (int k = m.gh_off[c2]; k < m.gh_off[c2 + 1]; ++k) out[t++] = m.gh_tab[k];
            }
        }
    } else {
        for (int j = 0; j < n; ++j)
            if (keep[j >> 5] & (1u << (j & 31))) out[t++] = m.gh_tab[pos[j]];
    }
}

// Sort key of the periodic re-sort: the grid-hash cell of the particle's
// position (mesh.py:1210-1232); particles that left the domain go last.
__global__ void __launch_bounds__(kBlock) k_sort_keys(const __grid_constant__ kc::DMesh m, const double* lon,
                                                      const double* lat, const int* status, long long P,
                                                      unsigned* key, int* idx) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    unsigned k = 0xFFFFFFFFu;
    if (status[i] != kc::OUTSIDE) {
        int ci, cj;
        kc::gh_cell_of(m, lon[i], lat[i], ci, cj);
        k = (unsigned)(cj * m.nx + ci);
    }
    key[i] = k;
    idx[i] = (int)i;
}

template <typename T>
__global__ void k_gather(const T* __restrict__ src, T* __restrict__ dst, const int* __restrict__ idx, long long P) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) dst[i] = src[idx[i]];
}

template <typename T>
__global__ void k_scatter(const T* __restrict__ src, T* __restrict__ dst, const long long* __restrict__ to,
                          long long P) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) dst[to[i]] = src[i];
}

unsigned grid_for(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// Gather one per-particle array into the spare buffer by the sort's index and
// swap the two buffers (all are sized 8 bytes per particle).
int regather(kc_ctx* c, void** arr, int es, const int* idx) {
    const long long P = c->P;
    unsigned g = grid_for(P);
    if (es == 8) k_gather<long long><<<g, kBlock, 0, c->stream>>>((const long long*)*arr, (long long*)c->spare, idx, P);
    else if (es == 4) k_gather<int><<<g, kBlock, 0, c->stream>>>((const int*)*arr, (int*)c->spare, idx, P);
    else k_gather<signed char><<<g, kBlock, 0, c->stream>>>((const signed char*)*arr, (signed char*)c->spare, idx, P);
    KC_CUDA(c, cudaGetLastError());
    std::swap(*arr, c->spare);
    return KC_OK;
}

// Copy one per-particle array to the host in upload order (scattered back
// through the upload slots after a re-sort).
int fetch(kc_ctx* c, void* host, const void* dev, int es) {
    if (!host) return KC_OK;
    const long long P = c->P;
    const void* src = dev;
    if (c->sorted) {
        unsigned g = grid_for(P);
        if (es == 8) k_scatter<long long><<<g, kBlock, 0, c->stream>>>((const long long*)dev, (long long*)c->spare, c->orig, P);
        else if (es == 4) k_scatter<int><<<g, kBlock, 0, c->stream>>>((const int*)dev, (int*)c->spare, c->orig, P);
        else k_scatter<signed char><<<g, kBlock, 0, c->stream>>>((const signed char*)dev, (signed char*)c->spare, c->orig, P);
        KC_CUDA(c, cudaGetLastError());
        src = c->spare;
    }
    KC_CUDA(c, cudaMemcpyAsync(host, src, (size_t)P * es, cudaMemcpyDeviceToHost, c->stream));
    if (c->sorted) KC_CUDA(c, cudaStreamSynchronize(c->stream));   // the spare buffer is reused next
    return KC_OK;
}

// Row stride of a step's snapshot slots: nodes; element-centre u/v in 2-D:
// elements; 3-D element-centre u/v (K-1, E) with node w (K, N): max(E, N).
long long lsq_stride(const kc_ctx* c, const kc_step_args* a) {
    if (!a->uv_lsq) return c->N;
    return a->dims == 3 ? std::max(c->E, c->N) : c->E;
}

template <typename T>
kc::DBlend<T> blend_of(kc_ctx* c, const kc_step_args* a) {
    kc::DBlend<T> f;
    f.a = field_of<T>(c->slots[a->slot_a]);
    f.b = field_of<T>(c->slots[a->slot_b]);
    f.t = field_of<T>(c->slots[a->slot_t]);
    f.alpha0 = a->alpha0;
    f.n = lsq_stride(c, a);
    f.pchip = a->pchip ? 1 : 0;
    f.d = a->pchip ? field_of<T>(c->slots[a->slot_d]) : kc::DField<T>{};
    for (int k = 0; k < 4; ++k) f.pt[k] = a->pchip ? a->pchip_t[k] : 0.0;
    return f;
}

}  // namespace

namespace {

// Slots of one step, and the ordering against kc_field_upload_async: the
// library's stream waits for a pending copy into a slot it reads, and
// records the slot's last read for the next copy into it to wait on.
int step_slots(const kc_step_args* a, int* sl) {
    sl[0] = a->slot_a; sl[1] = a->slot_b; sl[2] = a->slot_t;
    if (a->pchip) { sl[3] = a->slot_d; return 4; }
    return 3;
}

int wait_slots(kc_ctx* c, const int* sl, int n) {
    for (int k = 0; k < n; ++k) {
        Slot& s = c->slots[sl[k]];
        if (s.pending) {
            KC_CUDA(c, cudaStreamWaitEvent(c->stream, s.ready, 0));
            s.pending = false;
        }
    }
    return KC_OK;
}

int mark_slots_used(kc_ctx* c, const int* sl, int n) {
    if (!c->copy_stream) return KC_OK;
    for (int k = 0; k < n; ++k) {
        Slot& s = c->slots[sl[k]];
        if (!s.used) KC_CUDA(c, cudaEventCreateWithFlags(&s.used, cudaEventDisableTiming));
        KC_CUDA(c, cudaEventRecord(s.used, c->stream));
        s.has_used = true;
    }
    return KC_OK;
}

int launch_step_on(kc_ctx* c, const kc_step_args* a, const kc::DState& st, const kc::DStep& s) {
    int sl[4];
    const int nsl = step_slots(a, sl);
    int rc0 = wait_slots(c, sl, nsl);
    if (rc0) return rc0;
    const int dtype = c->slots[a->slot_a].dtype;
    if (c->dm.cg.on && a->precision == KC_MIXED) {   // the mixed form's 3-D C-grid step
        if (dtype == KC_F16) kc_launch_cgrid_mixed_f16(c->dm, blend_of<__half>(c, a), st, s, a->scheme, c->stream);
        else kc_launch_cgrid_mixed_f32(c->dm, blend_of<float>(c, a), st, s, a->scheme, c->stream);
    } else if (c->dm.cg.on) {   // NEMO C-grid meshes: the exact C-grid steps (plain form)
        if (dtype == KC_F32) kc_launch_cgrid_f32(c->dm, blend_of<float>(c, a), st, s, a->dims, a->scheme, c->stream);
        else kc_launch_cgrid_f64(c->dm, blend_of<double>(c, a), st, s, a->dims, a->scheme, c->stream);
    } else if (a->uv_lsq) {   // element-layout u/v: 2-D least squares (plain form)
        if (dtype == KC_F32) kc_launch_lsq_f32(c->dm, blend_of<float>(c, a), st, s, a->dims, a->scheme, c->stream);
        else kc_launch_lsq_f64(c->dm, blend_of<double>(c, a), st, s, a->dims, a->scheme, c->stream);
    } else if (c->dm.sig && a->dims == 3) {   // sigma meshes: the plain form's s = z / H_p step
        kc::DStep ss = s;
        ss.eta_s = c->sig_s_on ? c->d_sig_eta_s : nullptr;
        ss.eta_e = c->sig_e_on ? c->d_sig_eta_e : nullptr;
        ss.sig_steady = c->sig_steady ? 1 : 0;
        if (dtype == KC_F32) kc_launch_sigma_f32(c->dm, blend_of<float>(c, a), st, ss, a->scheme, c->stream);
        else kc_launch_sigma_f64(c->dm, blend_of<double>(c, a), st, ss, a->scheme, c->stream);
    } else if (a->precision == KC_MIXED) {
        if (dtype == KC_F16) kc_launch_mixed_f16(c->dm, blend_of<__half>(c, a), st, s, a->dims, a->scheme, c->stream);
        else kc_launch_mixed_f32(c->dm, blend_of<float>(c, a), st, s, a->dims, a->scheme, c->stream);
    } else if (dtype == KC_F32) {
        kc_launch_plain_f32(c->dm, blend_of<float>(c, a), st, s, a->dims, a->scheme, c->stream);
    } else {
        kc_launch_plain_f64(c->dm, blend_of<double>(c, a), st, s, a->dims, a->scheme, c->stream);
    }
    KC_CUDA(c, cudaGetLastError());
    return mark_slots_used(c, sl, nsl);
}

int launch_step(kc_ctx* c, const kc_step_args* a) {
    if (c->P == 0) return KC_OK;
    return launch_step_on(c, a, state_of(c), step_of(a));
}

int check_step(kc_ctx* c, const kc_step_args* a) {
    if (!a) return fail(c, KC_ERR_ARG, "kc_step: null args");
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_step: no mesh uploaded");
    if (!(a->scheme == KC_EULER || a->scheme == KC_RK2 || a->scheme == KC_RK4))
        return fail(c, KC_ERR_ARG, "kc_step: unknown scheme");
    if (!(a->dims == 2 || a->dims == 3)) return fail(c, KC_ERR_ARG, "kc_step: dims must be 2 or 3");
    if (!(a->dt > 0.0)) return fail(c, KC_ERR_ARG, "kc_step: dt must be > 0");
    if (!(a->time_dir == 1.0 || a->time_dir == -1.0)) return fail(c, KC_ERR_ARG, "kc_step: time_dir must be +-1");
    if (a->w_code < 0 || a->w_code > 3) return fail(c, KC_ERR_ARG, "kc_step: w_code must be 0..3");
    if (a->w_code >= 2 && (a->precision != KC_PLAIN || c->dm.cg.on))
        return fail(c, KC_ERR_ARG, "kc_step: least-squares / inverse-distance W run in the plain form");
    if (a->kick && !(a->kh_x >= 0.0 && a->kh_y >= 0.0)) return fail(c, KC_ERR_ARG, "kc_step: Kh must be >= 0");
    if (a->precision != KC_PLAIN && a->precision != KC_MIXED)
        return fail(c, KC_ERR_ARG, "kc_step: precision must be KC_PLAIN or KC_MIXED");
    if (a->uv_lsq) {
        if (a->uv_lsq < 1 || a->uv_lsq > 3) return fail(c, KC_ERR_ARG, "kc_step: uv_lsq must be 0..3");
        if (a->uv_lsq >= 2 && !c->dm.enb)
            return fail(c, KC_ERR_STATE, "kc_step: edge least-squares u/v needs kc_elem_neighbors_upload");
        if (a->dims == 3 && (a->uv_vertical != 0 || c->dm.sig))
            return fail(c, KC_ERR_ARG, "kc_step: 3-D least-squares u/v is built for layer fields on z-level meshes");
        if (a->precision != KC_PLAIN) return fail(c, KC_ERR_ARG, "kc_step: least-squares u/v runs in the plain form");
        if (c->dm.cg.on) return fail(c, KC_ERR_ARG, "kc_step: C-grid meshes read face velocities, not element centres");
        if (!c->dm.ec) return fail(c, KC_ERR_STATE, "kc_step: least-squares u/v needs kc_elem_centers_upload");
        if (c->has_elem) return fail(c, KC_ERR_ARG, "kc_step: least-squares u/v reads no element (no walk)");
    }
    if (a->pchip) {
        if (a->precision != KC_PLAIN) return fail(c, KC_ERR_ARG, "kc_step: PCHIP stages run in the plain form");
        if (a->az_kick) return fail(c, KC_ERR_ARG, "kc_step: the Az kick with PCHIP stages is not built");
        if (c->dm.cg.on) return fail(c, KC_ERR_ARG, "kc_step: PCHIP stages on C-grid meshes are not built");
        if (a->slot_d < 0 || a->slot_d >= kSlots) return fail(c, KC_ERR_ARG, "kc_step: slot out of range");
        const Slot& d = c->slots[a->slot_d];
        const Slot& s0 = c->slots[a->slot_a];
        if (d.dtype < 0 || d.dtype != s0.dtype || d.n != s0.n || d.uv_rows != s0.uv_rows || d.w_rows != s0.w_rows)
            return fail(c, KC_ERR_ARG, "kc_step: the fourth PCHIP record differs from the first in shape or type");
        if (c->dm.sig && a->dims == 3 && !d.has_eta)
            return fail(c, KC_ERR_STATE, "kc_step: sigma steps need eta in every snapshot slot (kc_field_upload_eta)");
        const double* t = a->pchip_t;
        if (!(t[0] < t[1] && t[1] < t[2] && t[2] < t[3]))
            return fail(c, KC_ERR_ARG, "kc_step: PCHIP times must increase strictly");
    }
    if (c->dm.cg.on) {
        if (a->precision == KC_MIXED && a->dims != 3)
            return fail(c, KC_ERR_ARG, "kc_step: the mixed form on C-grid meshes is the 3-D step");
        if (a->az_kick) return fail(c, KC_ERR_ARG, "kc_step: the Az kick on C-grid meshes is not built");
        if (a->dims == 3 && (a->kick || c->dm.cg.K < 1))
            return fail(c, KC_ERR_ARG, "kc_step: the 3-D C-grid step needs a 3-D C-grid mesh and takes no kick");
        const long long nynx = c->dm.cg.nynx;
        const int sl3[3] = {a->slot_a, a->slot_b, a->slot_t};
        for (int k = 0; k < 3; ++k) {
            if (sl3[k] < 0 || sl3[k] >= kSlots) return fail(c, KC_ERR_ARG, "kc_step: slot out of range");
            const Slot& s = c->slots[sl3[k]];
            if (s.dtype < 0) return fail(c, KC_ERR_STATE, "kc_step: snapshot slot " + std::to_string(sl3[k]) + " is empty");
            if (a->precision == KC_PLAIN && s.dtype == KC_F16)
                return fail(c, KC_ERR_ARG, "kc_step: the plain form reads float32 or float64 rasters");
            if (a->precision == KC_MIXED && s.dtype == KC_F64)
                return fail(c, KC_ERR_ARG, "kc_step: the mixed form reads float32 or float16 rasters");
            if (s.n != nynx) return fail(c, KC_ERR_ARG, "kc_step: C-grid snapshots are ny * nx face rasters");
            if (a->dims == 2 && s.uv_rows != 1 && s.uv_rows != c->dm.cg.K)
                return fail(c, KC_ERR_ARG, "kc_step: 2-D C-grid u/v need one row (or K, the surface read)");
            if (a->dims == 3 && (s.uv_rows != c->dm.cg.K || s.w_rows != c->dm.cg.K + 1))
                return fail(c, KC_ERR_ARG, "kc_step: 3-D C-grid fields need u/v (K, ny*nx) and w (K+1, ny*nx)");
        }
        if (c->P > 0 && !c->lon) return fail(c, KC_ERR_STATE, "kc_step: no particles uploaded");
        return KC_OK;
    }
    if (c->dm.sig && a->dims == 3) {
        if (a->precision != KC_PLAIN) return fail(c, KC_ERR_ARG, "kc_step: sigma meshes step in the plain form");
        if (a->az_kick && a->az_field)
            return fail(c, KC_ERR_ARG, "kc_step: sigma meshes take the constant Az source only");
        if (!(a->Dmin > 0.0) || !(a->z0b_min >= 0.0))
            return fail(c, KC_ERR_ARG, "kc_step: sigma steps need Dmin > 0 and z0b_min >= 0");
        if (!a->pchip && !(a->alpha_end >= 0.0 && a->alpha_end <= 1.0 + 1e-9))
            return fail(c, KC_ERR_ARG, "kc_step: alpha_end must be in [0, 1]");
        const int sl3[3] = {a->slot_a, a->slot_b, a->slot_t};
        for (int k = 0; k < 3; ++k)
            if (sl3[k] < 0 || sl3[k] >= kSlots || !c->slots[sl3[k]].has_eta)
                return fail(c, KC_ERR_STATE, "kc_step: sigma steps need eta in every snapshot slot (kc_field_upload_eta)");
    }
    if (a->az_kick) {
        if (a->dims != 3) return fail(c, KC_ERR_ARG, "kc_step: the Az kick needs a 3-D step");
        if (!(a->az_const >= 0.0)) return fail(c, KC_ERR_ARG, "kc_step: az_const must be >= 0");
        if (a->az_field) {
            const int need[2] = {a->slot_a, a->alpha0 != 0.0 ? a->slot_b : a->slot_a};
            for (int k = 0; k < 2; ++k) {
                if (need[k] < 0 || need[k] >= kSlots) return fail(c, KC_ERR_ARG, "kc_step: slot out of range");
                if (c->slots[need[k]].az_rows != c->dm.K)
                    return fail(c, KC_ERR_STATE, "kc_step: the Az field needs (K, N) az rows in the bracket slots");
            }
        }
    }
    int sl[3] = {a->slot_a, a->slot_b, a->slot_t};
    int dtype = -1;
    for (int k = 0; k < 3; ++k) {
        if (sl[k] < 0 || sl[k] >= kSlots) return fail(c, KC_ERR_ARG, "kc_step: slot out of range");
        const Slot& s = c->slots[sl[k]];
        if (s.dtype < 0) return fail(c, KC_ERR_STATE, "kc_step: snapshot slot " + std::to_string(sl[k]) + " is empty");
        if (s.n != lsq_stride(c, a))
            return fail(c, KC_ERR_ARG, a->uv_lsq ? "kc_step: least-squares u/v snapshots hold one value per element "
                                                   "(3-D: u/v and w rows of stride max(E, N))"
                                                 : "kc_step: snapshot node count differs from the mesh");
        if (dtype >= 0 && s.dtype != dtype) return fail(c, KC_ERR_ARG, "kc_step: snapshots of mixed element types");
        dtype = s.dtype;
        if (a->precision == KC_PLAIN && dtype == KC_F16)
            return fail(c, KC_ERR_ARG, "kc_step: the plain form reads float32 or float64 snapshots");
        if (a->precision == KC_MIXED && dtype == KC_F64)
            return fail(c, KC_ERR_ARG, "kc_step: the mixed form reads float32 or float16 snapshots");
        if (a->dims == 2 && s.uv_rows != 1) return fail(c, KC_ERR_ARG, "kc_step: 2-D step needs single-row u/v");
        if (a->dims == 3) {
            if (c->dm.K < 2) return fail(c, KC_ERR_STATE, "kc_step: 3-D step needs z-levels and depth");
            if (a->uv_vertical == 1) {
                if (!c->d_dl_p) return fail(c, KC_ERR_STATE, "kc_step: depth-linear u/v needs kc_depth_points_upload");
                if (s.uv_rows != c->dm.dl_M || s.w_rows != c->dm.K)
                    return fail(c, KC_ERR_ARG, "kc_step: depth-linear fields need u/v (M, N) and w (K, N)");
            } else if (a->uv_vertical == 0) {
                if (s.uv_rows != c->dm.K - 1 || s.w_rows != c->dm.K)
                    return fail(c, KC_ERR_ARG, "kc_step: 3-D layer fields need u/v (K-1, N) and w (K, N)");
            } else {
                return fail(c, KC_ERR_ARG, "kc_step: uv_vertical must be 0 (layer) or 1 (depth-linear)");
            }
        }
    }
    if (c->P > 0 && !c->lon) return fail(c, KC_ERR_STATE, "kc_step: no particles uploaded");
    return KC_OK;
}

int do_step(kc_ctx* c, const kc_step_args* a) {
    int rc = check_step(c, a);
    if (rc) return rc;
    return launch_step(c, a);
}

template <typename T>
int upload(kc_ctx* c, T** dst, const void* src, size_t count) {
    KC_CUDA(c, cudaMalloc((void**)dst, std::max<size_t>(count, 1) * sizeof(T)));
    if (count) KC_CUDA(c, cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return KC_OK;
}

void free_mesh(kc_ctx* c) {
    dfree(c->d_ll); dfree(c->d_en); dfree(c->d_n2e_off); dfree(c->d_n2e); dfree(c->d_gh_off);
    dfree(c->d_gh_tab); dfree(c->d_pw_off); dfree(c->d_pw_tab); dfree(c->d_xyz); dfree(c->d_depth); dfree(c->d_zlev);
    dfree(c->d_nsc); dfree(c->d_ecos); dfree(c->d_ebox); dfree(c->d_erec); dfree(c->d_maxl); dfree(c->d_coastal);
    c->dm.ebox = nullptr;
    c->dm.erec = nullptr;
    dfree(c->d_beach_eta); dfree(c->d_beach_dry);
    dfree(c->d_sig_eta_s); dfree(c->d_sig_eta_e);
    c->beach_eta_on = c->beach_dry_on = false;
    c->sig_s_on = c->sig_e_on = c->sig_steady = false;
    dfree(c->d_dl_p); dfree(c->d_dl_last); dfree(c->d_dl_bed); dfree(c->d_enb); dfree(c->d_sigma);
    dfree(c->d_cg_corners); dfree(c->d_cg_cell); dfree(c->d_cg_nlev); dfree(c->d_cg_nlev_r); dfree(c->d_cg_L);
    dfree(c->d_cg_e2u); dfree(c->d_cg_e1v); dfree(c->d_cg_area); dfree(c->d_cg_zw); dfree(c->d_cg_e3b);
    dfree(c->d_cg_e3u); dfree(c->d_cg_e3v); dfree(c->d_cg_kbu); dfree(c->d_cg_kbv);
    c->dm.cg = kc::DCgrid{};
    c->dm.dl_p = nullptr; c->dm.dl_last = nullptr; c->dm.dl_bed = nullptr; c->dm.dl_M = 0;
    c->dm.enb = nullptr;
    dfree(c->d_ec);
    c->dm.ec = nullptr;
    c->dm.pw_off = nullptr; c->dm.pw_tab = nullptr;
    c->dm.sigma = nullptr; c->dm.sig = 0;
    c->has_mesh = false;
}

void free_particles(kc_ctx* c) {
    dfree(c->lon); dfree(c->lat); dfree(c->z); dfree(c->U); dfree(c->V); dfree(c->W);
    dfree(c->status); dfree(c->nn); dfree(c->fr); dfree(c->pid); dfree(c->rs); dfree(c->rid); dfree(c->elem);
    dfree(c->el); dfree(c->wel);
    c->has_elem = false;
    dfree(c->orig); dfree(c->spare); dfree(c->prev); dfree(c->wet); dfree(c->nn_ok);
    c->has_beach = false;
    dfree(c->skey[0]); dfree(c->skey[1]); dfree(c->sidx[0]); dfree(c->sidx[1]); dfree(c->cub_tmp);
    c->P = c->cap = c->sort_cap = 0;
    c->sorted = false;
}

}  // namespace

extern "C" {

int kc_abi_version(void) { return KC_ABI_VERSION; }

int kc_create(int device, kc_ctx** out) {
    if (!out) return KC_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return KC_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return KC_ERR_CUDA;
    kc_ctx* c = new kc_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&c->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
        kc_destroy(c);
        return KC_ERR_CUDA;
    }
    for (int k = 0; k < kEvents; ++k) cudaEventCreate(&c->ev[k]);
    // the RNG's exception tables, resident for the context's life
    {
        kc_host::RngTables t;
        if (!kc_host::rng_exception_tables(t)) {
            kc_destroy(c);
            return KC_ERR_STATE;
        }
        auto put = [&](void** d, const void* h, size_t bytes) {
            return cudaMalloc(d, bytes > 0 ? bytes : 4) == cudaSuccess &&
                   (bytes == 0 || cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice) == cudaSuccess);
        };
        if (!put((void**)&c->d_rx_a_off, t.a_off, t.n_off * 4) || !put((void**)&c->d_rx_a, t.a, t.na * 2) ||
            !put((void**)&c->d_rx_b_off, t.b_off, t.n_off * 4) || !put((void**)&c->d_rx_b, t.b, t.nb * 2)) {
            kc_destroy(c);
            return KC_ERR_CUDA;
        }
        c->dm.rx = kc::DRngX{c->d_rx_a_off, c->d_rx_a, c->d_rx_b_off, c->d_rx_b};
    }
    *out = c;
    return KC_OK;
}

void kc_destroy(kc_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_mesh(c);
    free_particles(c);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (auto& s : c->slots) {
        dfree(s.u); dfree(s.v); dfree(s.w); dfree(s.su); dfree(s.sv); dfree(s.sw); dfree(s.az); dfree(s.eta);
        if (s.ready) cudaEventDestroy(s.ready);
        if (s.used) cudaEventDestroy(s.used);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    dfree(c->q); dfree(c->qout); dfree(c->d_err); dfree(c->flush); dfree(c->stage);
    dfree(c->d_rx_a_off); dfree(c->d_rx_a); dfree(c->d_rx_b_off); dfree(c->d_rx_b);
    for (int k = 0; k < kEvents; ++k) if (c->ev[k]) cudaEventDestroy(c->ev[k]);
    for (int k = 0; k < kChunks; ++k) {
        if (c->ev_in[k]) cudaEventDestroy(c->ev_in[k]);
        if (c->ev_k[k]) cudaEventDestroy(c->ev_k[k]);
    }
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->fused_exec) cudaGraphExecDestroy(c->fused_exec);
    if (c->fused_ev) cudaEventDestroy(c->fused_ev);
    if (c->fused_host) cudaFreeHost(c->fused_host);
    dfree(c->fused_dev);
    if (c->s_in) { cudaStreamSynchronize(c->s_in); cudaStreamDestroy(c->s_in); }
    if (c->s_out) { cudaStreamSynchronize(c->s_out); cudaStreamDestroy(c->s_out); }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int kc_last_error(const kc_ctx* c, char* buf, int buflen) {
    if (!c || !buf || buflen <= 0) return KC_ERR_ARG;
    std::snprintf(buf, (size_t)buflen, "%s", c->err.c_str());
    return KC_OK;
}

int kc_synchronize(kc_ctx* c) {
    if (!c) return KC_ERR_ARG;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->copy_stream) KC_CUDA(c, cudaStreamSynchronize(c->copy_stream));
    return KC_OK;
}

// The containment tables of the uploaded elements: the prefilter boxes
// (elem_box) and the mask vertex records (elem_record).  In the environment,
// KELP_B200_ELEM_BOXES=0 leaves out the boxes (every ring element then goes
// through the full test) and KELP_B200_ELEM_RECORDS=0 the records (vertices
// then read through the element's node ids).
int build_elem_boxes(kc_ctx* c) {
    kc::DMesh& m = c->dm;
    m.ebox = nullptr;
    m.erec = nullptr;
    const char* env = getenv("KELP_B200_ELEM_BOXES");
    if (!(env && env[0] == '0')) {
        KC_CUDA(c, cudaMalloc((void**)&c->d_ebox, (size_t)c->E * sizeof(float4)));
        k_elem_boxes<<<grid_for(c->E), kBlock, 0, c->stream>>>(m, c->d_ebox);
        KC_CUDA(c, cudaGetLastError());
    }
    env = getenv("KELP_B200_ELEM_RECORDS");
    if (!(env && env[0] == '0')) {
        KC_CUDA(c, cudaMalloc((void**)&c->d_erec, (size_t)c->E * 4 * sizeof(double2)));
        k_elem_records<<<grid_for(c->E), kBlock, 0, c->stream>>>(m, c->d_erec);
        KC_CUDA(c, cudaGetLastError());
    }
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    m.ebox = c->d_ebox;
    m.erec = c->d_erec;
    return KC_OK;
}

// The pruned windows of the uploaded grid hash (k_prune_windows): counts,
// offsets on the host, positions.  KELP_B200_PRUNED_WINDOWS=0 in the
// environment keeps the whole-window scan.
int build_pruned_windows(kc_ctx* c) {
    const char* env = getenv("KELP_B200_PRUNED_WINDOWS");
    if (env && env[0] == '0') return KC_OK;
    kc::DMesh& m = c->dm;
    const long long ncell = (long long)m.nx * m.ny;
    int* d_cnt = nullptr;
    KC_CUDA(c, cudaMalloc((void**)&d_cnt, (size_t)ncell * sizeof(int)));
    k_prune_windows<<<grid_for(ncell), kBlock, 0, c->stream>>>(m, d_cnt, nullptr, nullptr);
    std::vector<int> cnt((size_t)ncell);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), d_cnt, (size_t)ncell * sizeof(int), cudaMemcpyDeviceToHost,
                                              c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_cnt);
    KC_CUDA(c, e);
    std::vector<int> off((size_t)ncell + 1);
    long long total = 0;
    for (long long k = 0; k < ncell; ++k) {
        off[k] = (int)total;
        total += cnt[k];
        if (total > (long long)INT_MAX) return KC_OK;   // too large to index: whole windows
    }
    off[ncell] = (int)total;
    int rc;
    if ((rc = upload(c, &c->d_pw_off, off.data(), off.size()))) return rc;
    KC_CUDA(c, cudaMalloc((void**)&c->d_pw_tab, (size_t)std::max<long long>(total, 1) * sizeof(double4)));
    k_prune_windows<<<grid_for(ncell), kBlock, 0, c->stream>>>(m, nullptr, c->d_pw_off, c->d_pw_tab);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    m.pw_off = c->d_pw_off;
    m.pw_tab = c->d_pw_tab;
    return KC_OK;
}

int kc_mesh_upload(kc_ctx* c, const kc_mesh_desc* d) {
    if (!c || !d) return KC_ERR_ARG;
    if (d->n_nodes <= 0 || d->n_elems <= 0) return fail(c, KC_ERR_ARG, "kc_mesh_upload: empty mesh");
    if (d->max_v != 3 && d->max_v != 4) return fail(c, KC_ERR_ARG, "kc_mesh_upload: max_v must be 3 or 4");
    if (!d->nodes_lon || !d->nodes_lat || !d->elem_nodes || !d->node_to_elems || !d->node_to_elems_count ||
        !d->gh_offsets || !d->gh_node_ids || !d->node_xyz)
        return fail(c, KC_ERR_ARG, "kc_mesh_upload: missing array");
    if (d->gh_nx <= 0 || d->gh_ny <= 0 || !(d->gh_cell_size > 0.0))
        return fail(c, KC_ERR_ARG, "kc_mesh_upload: invalid grid-hash geometry");
    if (d->n_levels > 0 && (!d->z_levels || !d->depth))
        return fail(c, KC_ERR_ARG, "kc_mesh_upload: 3-D mesh needs z_levels and depth");
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    free_mesh(c);
    const long long N = d->n_nodes, E = d->n_elems;
    const long long ncell = (long long)d->gh_nx * d->gh_ny;
    // host-side validation of every index the kernels will follow
    for (long long e = 0; e < E * d->max_v; ++e)
        if (d->elem_nodes[e] >= N || d->elem_nodes[e] < -1)
            return fail(c, KC_ERR_ARG, "kc_mesh_upload: elem_nodes index out of range");
    if (d->gh_offsets[0] != 0 || d->gh_offsets[ncell] != N)
        return fail(c, KC_ERR_ARG, "kc_mesh_upload: grid-hash offsets do not cover the nodes");
    for (long long k = 0; k < ncell; ++k)
        if (d->gh_offsets[k + 1] < d->gh_offsets[k]) return fail(c, KC_ERR_ARG, "kc_mesh_upload: offsets not monotone");
    // repacked tables
    std::vector<double2> ll((size_t)N);
    for (long long i = 0; i < N; ++i) ll[i] = make_double2(d->nodes_lon[i], d->nodes_lat[i]);
    std::vector<int4> en((size_t)E);
    for (long long e = 0; e < E; ++e) {
        const int* r = d->elem_nodes + e * d->max_v;
        en[e] = make_int4(r[0], r[1], r[2], d->max_v == 4 ? r[3] : -1);
    }
    std::vector<int> off((size_t)N + 1);
    std::vector<int> ids;
    ids.reserve((size_t)N * 6);
    off[0] = 0;
    for (long long i = 0; i < N; ++i) {
        int cnt = d->node_to_elems_count[i];
        if (cnt < 0 || cnt > d->max_conn) return fail(c, KC_ERR_ARG, "kc_mesh_upload: node_to_elems_count out of range");
        for (int k = 0; k < cnt; ++k) {
            int el = d->node_to_elems[i * d->max_conn + k];
            if (el >= E) return fail(c, KC_ERR_ARG, "kc_mesh_upload: node_to_elems index out of range");
            if (el >= 0) ids.push_back(el);
        }
        off[i + 1] = (int)ids.size();
    }
    std::vector<double4> tab((size_t)N);
    for (long long k = 0; k < N; ++k) {
        int nd = d->gh_node_ids[k];
        if (nd < 0 || nd >= N) return fail(c, KC_ERR_ARG, "kc_mesh_upload: gh_node_ids out of range");
        tab[k] = make_double4(d->node_xyz[3 * (long long)nd], d->node_xyz[3 * (long long)nd + 1],
                              d->node_xyz[3 * (long long)nd + 2], (double)nd);
    }
    std::vector<double2> nsc((size_t)N), ecos((size_t)E);
    std::vector<int> maxl(d->n_levels >= 2 ? (size_t)N : 0);
    kc_host::mesh_tables(N, E, d->max_v, d->nodes_lat, d->elem_nodes, d->depth, d->z_levels, d->n_levels,
                         reinterpret_cast<double*>(nsc.data()), reinterpret_cast<double*>(ecos.data()),
                         maxl.empty() ? nullptr : maxl.data());
    int rc;
    if ((rc = upload(c, &c->d_nsc, nsc.data(), nsc.size()))) return rc;
    if ((rc = upload(c, &c->d_ecos, ecos.data(), ecos.size()))) return rc;
    if (!maxl.empty() && (rc = upload(c, &c->d_maxl, maxl.data(), maxl.size()))) return rc;
    if ((rc = upload(c, &c->d_ll, ll.data(), ll.size()))) return rc;
    if ((rc = upload(c, &c->d_en, en.data(), en.size()))) return rc;
    if ((rc = upload(c, &c->d_n2e_off, off.data(), off.size()))) return rc;
    if ((rc = upload(c, &c->d_n2e, ids.data(), ids.size()))) return rc;
    if ((rc = upload(c, &c->d_gh_off, d->gh_offsets, (size_t)ncell + 1))) return rc;
    if ((rc = upload(c, &c->d_gh_tab, tab.data(), tab.size()))) return rc;
    if ((rc = upload(c, &c->d_xyz, d->node_xyz, (size_t)N * 3))) return rc;
    if (d->depth && (rc = upload(c, &c->d_depth, d->depth, (size_t)N))) return rc;
    if (d->n_levels > 0 && (rc = upload(c, &c->d_zlev, d->z_levels, (size_t)d->n_levels))) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    kc::DMesh& m = c->dm;
    m.ll = c->d_ll; m.en = c->d_en; m.n2e_off = c->d_n2e_off; m.n2e = c->d_n2e;
    m.gh_off = c->d_gh_off; m.gh_tab = c->d_gh_tab; m.xyz = c->d_xyz;
    m.depth = c->d_depth; m.zlev = c->d_zlev;
    m.nsc = c->d_nsc; m.ecos = c->d_ecos; m.max_layer = c->d_maxl;
    m.cell = d->gh_cell_size; m.lon_min = d->gh_lon_min; m.lat_min = d->gh_lat_min; m.r_earth = d->r_earth;
    m.nx = d->gh_nx; m.ny = d->gh_ny; m.wrap = d->gh_wrap_lon ? 1 : 0; m.far_rows = d->gh_far_rows;
    m.K = d->n_levels; m.exact = d->exact_nearest ? 1 : 0;
    m.err = c->d_err;
    m.E = E;
    c->max_v = d->max_v;
    c->N = N; c->E = E;
    if ((rc = build_elem_boxes(c))) return rc;
    if ((rc = build_pruned_windows(c))) return rc;
    c->has_mesh = true;
    ++c->mesh_gen;
    return KC_OK;
}

int kc_coastal_upload(kc_ctx* c, const unsigned char* flags) {
    if (!c || !flags) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_coastal_upload: no mesh uploaded");
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_coastal);
    int rc = upload(c, &c->d_coastal, flags, (size_t)c->E);
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_cgrid_upload(kc_ctx* c, const kc_cgrid_desc* d) {
    if (!c || !d) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_cgrid_upload: no mesh uploaded");
    const long long E = c->E, N = c->N;
    if (d->ny < 2 || d->nx < 2 || d->K < 0) return fail(c, KC_ERR_ARG, "kc_cgrid_upload: raster shape");
    if (!d->corners || !d->elem_ji || !d->nlev || !d->nlev_raster)
        return fail(c, KC_ERR_ARG, "kc_cgrid_upload: missing cell tables");
    if ((d->e2u == nullptr) != (d->e1v == nullptr)) return fail(c, KC_ERR_ARG, "kc_cgrid_upload: e2u and e1v go together");
    if (d->K > 0 && (!d->area || !d->zw || !d->e3b || !d->kbu || !d->e3u || !d->kbv || !d->e3v))
        return fail(c, KC_ERR_ARG, "kc_cgrid_upload: a 3-D mesh needs area, zw, e3b and the face partial levels");
    const long long nynx = (long long)d->ny * d->nx;
    std::vector<int4> cr((size_t)E);
    std::vector<int> cell((size_t)E);
    for (long long e = 0; e < E; ++e) {
        const int* q = d->corners + 4 * e;
        for (int k = 0; k < 4; ++k)
            if (q[k] < 0 || q[k] >= N) return fail(c, KC_ERR_ARG, "kc_cgrid_upload: corner out of range");
        const long long j = d->elem_ji[2 * e], i = d->elem_ji[2 * e + 1];
        if (j < 1 || j >= d->ny || i < 1 || i >= d->nx) return fail(c, KC_ERR_ARG, "kc_cgrid_upload: cell (j, i) out of range");
        if (d->nlev[e] < 0 || (d->K > 0 && d->nlev[e] > d->K))
            return fail(c, KC_ERR_ARG, "kc_cgrid_upload: wet levels out of range");
        cr[e] = make_int4(q[0], q[1], q[2], q[3]);
        cell[e] = (int)(j * d->nx + i);
    }
    for (long long k = 0; k < nynx; ++k)
        if (d->nlev_raster[k] < 0 || (d->K > 0 && d->nlev_raster[k] > d->K))
            return fail(c, KC_ERR_ARG, "kc_cgrid_upload: raster wet levels out of range");
    if (d->K > 0) {
        for (long long k = 0; k < nynx; ++k)
            if (d->kbu[k] < -1 || d->kbu[k] >= d->K || d->kbv[k] < -1 || d->kbv[k] >= d->K)
                return fail(c, KC_ERR_ARG, "kc_cgrid_upload: face partial level out of range");
        for (int k = 0; k < d->K; ++k)
            if (!(d->zw[k + 1] > d->zw[k])) return fail(c, KC_ERR_ARG, "kc_cgrid_upload: zw must increase");
    }
    std::vector<double> L;
    if (!d->e2u) {
        std::vector<double2> ll((size_t)N);
        std::vector<double> lon((size_t)N), lat((size_t)N);
        KC_CUDA(c, cudaSetDevice(c->device));
        KC_CUDA(c, cudaMemcpy(ll.data(), c->d_ll, (size_t)N * 16, cudaMemcpyDeviceToHost));
        for (long long n = 0; n < N; ++n) { lon[n] = ll[n].x; lat[n] = ll[n].y; }
        L.resize((size_t)E * 4);
        kc_host::cgrid_edge_lengths(E, d->corners, lon.data(), lat.data(), L.data());
    }
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_cg_corners); dfree(c->d_cg_cell); dfree(c->d_cg_nlev); dfree(c->d_cg_nlev_r); dfree(c->d_cg_L);
    dfree(c->d_cg_e2u); dfree(c->d_cg_e1v); dfree(c->d_cg_area); dfree(c->d_cg_zw); dfree(c->d_cg_e3b);
    dfree(c->d_cg_e3u); dfree(c->d_cg_e3v); dfree(c->d_cg_kbu); dfree(c->d_cg_kbv);
    c->dm.cg = kc::DCgrid{};
    int rc;
    if ((rc = upload(c, &c->d_cg_corners, cr.data(), cr.size()))) return rc;
    if ((rc = upload(c, &c->d_cg_cell, cell.data(), cell.size()))) return rc;
    if ((rc = upload(c, &c->d_cg_nlev, d->nlev, (size_t)E))) return rc;
    if ((rc = upload(c, &c->d_cg_nlev_r, d->nlev_raster, (size_t)nynx))) return rc;
    if (!L.empty() && (rc = upload(c, &c->d_cg_L, L.data(), (size_t)E))) return rc;
    if (d->e2u) {
        if ((rc = upload(c, &c->d_cg_e2u, d->e2u, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_e1v, d->e1v, (size_t)nynx))) return rc;
    }
    if (d->K > 0) {
        if ((rc = upload(c, &c->d_cg_area, d->area, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_zw, d->zw, (size_t)d->K + 1))) return rc;
        if ((rc = upload(c, &c->d_cg_e3b, d->e3b, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_kbu, d->kbu, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_e3u, d->e3u, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_kbv, d->kbv, (size_t)nynx))) return rc;
        if ((rc = upload(c, &c->d_cg_e3v, d->e3v, (size_t)nynx))) return rc;
    }
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    kc::DCgrid& g = c->dm.cg;
    g.corners = c->d_cg_corners; g.cell = c->d_cg_cell; g.nlev = c->d_cg_nlev; g.nlev_r = c->d_cg_nlev_r;
    g.L = c->d_cg_L; g.e2u = c->d_cg_e2u; g.e1v = c->d_cg_e1v; g.area = c->d_cg_area; g.zw = c->d_cg_zw;
    g.e3b = c->d_cg_e3b; g.kbu = c->d_cg_kbu; g.e3u = c->d_cg_e3u; g.kbv = c->d_cg_kbv; g.e3v = c->d_cg_e3v;
    g.nynx = nynx; g.nx = d->nx; g.K = d->K; g.shrunk = d->partial_shrunk ? 1 : 0; g.has_e = d->e2u ? 1 : 0;
    g.on = 1;
    ++c->mesh_gen;
    return KC_OK;
}

int kc_sigma_upload(kc_ctx* c, int K, const double* sigma) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sigma_upload: no mesh uploaded");
    if (!c->d_depth) return fail(c, KC_ERR_STATE, "kc_sigma_upload: the mesh has no depth");
    if (c->dm.zlev) return fail(c, KC_ERR_STATE, "kc_sigma_upload: the mesh was uploaded with z-levels");
    if (K < 2 || !sigma) return fail(c, KC_ERR_ARG, "kc_sigma_upload: at least 2 interfaces");
    for (int k = 0; k < K; ++k)
        if (!(sigma[k] >= -1e9 && sigma[k] <= 1e9)) return fail(c, KC_ERR_ARG, "kc_sigma_upload: non-finite interface");
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_sigma);
    c->dm.sigma = nullptr;
    c->dm.sig = 0;
    int rc = upload(c, &c->d_sigma, sigma, (size_t)K);
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dm.sigma = c->d_sigma;
    c->dm.sig = 1;
    c->dm.K = K;
    ++c->mesh_gen;
    return KC_OK;
}

int kc_elem_neighbors_upload(kc_ctx* c, int max_v, const int* enb) {
    if (!c || !enb) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_elem_neighbors_upload: no mesh uploaded");
    if (max_v != c->max_v) return fail(c, KC_ERR_ARG, "kc_elem_neighbors_upload: max_v differs from the mesh's");
    const long long E = c->E;
    std::vector<int4> t((size_t)E);
    for (long long e = 0; e < E; ++e) {
        const int* r = enb + e * max_v;
        for (int k = 0; k < max_v; ++k)
            if (r[k] < -1 || r[k] >= E) return fail(c, KC_ERR_ARG, "kc_elem_neighbors_upload: index out of range");
        t[e] = make_int4(r[0], r[1], r[2], max_v == 4 ? r[3] : -1);
    }
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_enb);
    c->dm.enb = nullptr;
    int rc = upload(c, &c->d_enb, t.data(), t.size());
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dm.enb = c->d_enb;
    ++c->mesh_gen;
    return KC_OK;
}

int kc_elem_centers_upload(kc_ctx* c, const double* lon, const double* lat) {
    if (!c || !lon || !lat) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_elem_centers_upload: no mesh uploaded");
    const long long E = c->E;
    std::vector<double2> t((size_t)E);
    for (long long e = 0; e < E; ++e) t[e] = make_double2(lon[e], lat[e]);
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_ec);
    c->dm.ec = nullptr;
    int rc = upload(c, &c->d_ec, t.data(), t.size());
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dm.ec = c->d_ec;
    ++c->mesh_gen;
    return KC_OK;
}

int kc_particles_set_elem(kc_ctx* c, const int* elem) {
    if (!c) return KC_ERR_ARG;
    if (c->sorted) return fail(c, KC_ERR_STATE, "kc_particles_set_elem: set the elements before kc_sort");
    if (elem && !c->dm.enb) return fail(c, KC_ERR_STATE, "kc_particles_set_elem: upload the element neighbours first");
    KC_CUDA(c, cudaSetDevice(c->device));
    c->has_elem = false;
    if (!elem) return KC_OK;
    if (c->P > 0) KC_CUDA(c, cudaMemcpyAsync(c->elem, elem, (size_t)c->P * 4, cudaMemcpyHostToDevice, c->stream));
    c->has_elem = true;
    return KC_OK;
}

int kc_particles_get_elem(kc_ctx* c, long long P, int* elem) {
    if (!c || !elem) return KC_ERR_ARG;
    if (!c->has_elem) return fail(c, KC_ERR_STATE, "kc_particles_get_elem: no carried elements (kc_particles_set_elem)");
    if (P != c->P) return fail(c, KC_ERR_ARG, "kc_particles_get_elem: P differs from the resident count");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    int rc = fetch(c, elem, c->elem, 4);
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_particles_set_realization(kc_ctx* c, const int* real_id) {
    if (!c) return KC_ERR_ARG;
    if (c->sorted) return fail(c, KC_ERR_STATE, "kc_particles_set_realization: set the realizations before kc_sort");
    KC_CUDA(c, cudaSetDevice(c->device));
    c->has_rid = false;
    if (!real_id || c->P == 0) return KC_OK;
    KC_CUDA(c, cudaMemcpyAsync(c->rid, real_id, (size_t)c->P * 4, cudaMemcpyHostToDevice, c->stream));
    c->has_rid = true;
    return KC_OK;
}

int kc_beach_state_upload(kc_ctx* c, const int* prev_status, const int* wet_streak) {
    if (!c) return KC_ERR_ARG;
    if (c->P > 0 && !c->prev) return fail(c, KC_ERR_STATE, "kc_beach_state_upload: no particles uploaded");
    KC_CUDA(c, cudaSetDevice(c->device));
    if (c->sorted) return fail(c, KC_ERR_STATE, "kc_beach_state_upload: upload the beaching state before kc_sort");
    const size_t n = (size_t)c->P * 4;
    if (c->P > 0) {
        if (prev_status) KC_CUDA(c, cudaMemcpyAsync(c->prev, prev_status, n, cudaMemcpyHostToDevice, c->stream));
        else KC_CUDA(c, cudaMemcpyAsync(c->prev, c->status, n, cudaMemcpyDeviceToDevice, c->stream));
        if (wet_streak) KC_CUDA(c, cudaMemcpyAsync(c->wet, wet_streak, n, cudaMemcpyHostToDevice, c->stream));
        else KC_CUDA(c, cudaMemsetAsync(c->wet, 0, n, c->stream));
    }
    c->has_beach = true;
    return KC_OK;
}

int kc_beach_state_download(kc_ctx* c, int* wet_streak) {
    if (!c || !wet_streak) return KC_ERR_ARG;
    if (!c->has_beach) return fail(c, KC_ERR_STATE, "kc_beach_state_download: no beaching state");
    KC_CUDA(c, cudaSetDevice(c->device));
    int rc = fetch(c, wet_streak, c->wet, 4);
    if (rc) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

// Validate one hook call's arguments against the context and build the
// device-side argument block.
static int beach_of(kc_ctx* c, const kc_beach_args* a, kc::DBeach& b) {
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_beach: no mesh uploaded");
    if (c->dm.cg.on) return fail(c, KC_ERR_ARG, "kc_beach: the reference runs no beaching on C-grid meshes");
    if (!c->has_beach) return fail(c, KC_ERR_STATE, "kc_beach: call kc_beach_state_upload first");
    if (!c->d_depth) return fail(c, KC_ERR_STATE, "kc_beach: the mesh has no depth");
    if (a->resuspension < 0 || a->resuspension > 3) return fail(c, KC_ERR_ARG, "kc_beach: resuspension code");
    const bool need_topo = a->use_coastal || a->use_stochastic;
    if (need_topo && !c->d_coastal) return fail(c, KC_ERR_STATE, "kc_beach: coastal flags not uploaded");
    b.use_depth = a->use_depth; b.use_coastal = a->use_coastal; b.use_stochastic = a->use_stochastic;
    b.on_failure = a->on_failure; b.need_topo = need_topo ? 1 : 0; b.resuspension = a->resuspension;
    b.min_wet_steps = a->min_wet_steps;
    b.depth_min = a->depth_min; b.zone_depth = a->zone_depth;
    b.rewet_level = a->depth_min + a->rewet_hysteresis;
    b.p_beach = a->p_beach; b.p_resusp = a->p_resusp;
    b.seed = a->seed; b.real_id = a->real_id; b.step_i = a->step_i; b.pid_offset = a->pid_offset;
    b.coastal = need_topo ? c->d_coastal : nullptr;
    b.eta = c->beach_eta_on ? c->d_beach_eta : nullptr;
    b.dry = c->beach_dry_on ? c->d_beach_dry : nullptr;
    b.prev = c->prev;
    b.wet_streak = c->wet;
    return KC_OK;
}

// The RNG key of every resident particle stays the slot index it was uploaded
// with, whatever the order the re-sort leaves them in.
static int pin_pid(kc_ctx* c) {
    if (!c->has_pid && c->P > 0) {
        KC_CUDA(c, cudaMemcpyAsync(c->pid, c->orig, (size_t)c->P * 8, cudaMemcpyDeviceToDevice, c->stream));
        c->has_pid = true;
    }
    return KC_OK;
}

int kc_beach(kc_ctx* c, const kc_beach_args* a) {
    if (!c || !a) return KC_ERR_ARG;
    kc::DBeach b;
    int rc = beach_of(c, a, b);
    if (rc) return rc;
    if (c->P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    if ((rc = pin_pid(c))) return rc;
    kc::DState st = state_of(c);
    k_beach<<<grid_for(c->P), kBlock, 0, c->stream>>>(c->dm, st, b, c->N);
    KC_CUDA(c, cudaGetLastError());
    return KC_OK;
}

int kc_beach_surface(kc_ctx* c, const double* eta, const double* dry_mask) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_beach_surface: no mesh uploaded");
    KC_CUDA(c, cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->N * 8;
    if (eta) {
        if (!c->d_beach_eta) KC_CUDA(c, cudaMalloc((void**)&c->d_beach_eta, bytes));
        KC_CUDA(c, cudaMemcpyAsync(c->d_beach_eta, eta, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    if (dry_mask) {
        if (!c->d_beach_dry) KC_CUDA(c, cudaMalloc((void**)&c->d_beach_dry, bytes));
        KC_CUDA(c, cudaMemcpyAsync(c->d_beach_dry, dry_mask, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    if (eta || dry_mask) KC_CUDA(c, cudaStreamSynchronize(c->stream));   // the caller may free its arrays
    c->beach_eta_on = eta != nullptr;
    c->beach_dry_on = dry_mask != nullptr;
    return KC_OK;
}

int kc_sigma_surfaces(kc_ctx* c, const double* eta_start, const double* eta_end, int steady) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sigma_surfaces: no mesh uploaded");
    if (!c->dm.sig) return fail(c, KC_ERR_STATE, "kc_sigma_surfaces: the resident mesh is not a sigma mesh");
    if (steady != 0 && steady != 1) return fail(c, KC_ERR_ARG, "kc_sigma_surfaces: steady is 0 or 1");
    KC_CUDA(c, cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->N * 8;
    if (eta_start) {
        if (!c->d_sig_eta_s) KC_CUDA(c, cudaMalloc((void**)&c->d_sig_eta_s, bytes));
        KC_CUDA(c, cudaMemcpyAsync(c->d_sig_eta_s, eta_start, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    if (eta_end) {
        if (!c->d_sig_eta_e) KC_CUDA(c, cudaMalloc((void**)&c->d_sig_eta_e, bytes));
        KC_CUDA(c, cudaMemcpyAsync(c->d_sig_eta_e, eta_end, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    if (eta_start || eta_end) KC_CUDA(c, cudaStreamSynchronize(c->stream));   // the caller may free its arrays
    c->sig_s_on = eta_start != nullptr;
    c->sig_e_on = eta_end != nullptr;
    c->sig_steady = steady != 0;
    return KC_OK;
}

int kc_sigma_surface_slots(kc_ctx* c, int which, int kind, const int* slots, double alpha, const double* t, double q,
                           int steady) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sigma_surface_slots: no mesh uploaded");
    if (!c->dm.sig) return fail(c, KC_ERR_STATE, "kc_sigma_surface_slots: the resident mesh is not a sigma mesh");
    if ((which != 0 && which != 1) || kind < 0 || kind > 3 || (steady != 0 && steady != 1))
        return fail(c, KC_ERR_ARG, "kc_sigma_surface_slots: which 0 / 1, kind 0..3, steady 0 / 1");
    c->sig_steady = steady != 0;
    bool& on = which == 0 ? c->sig_s_on : c->sig_e_on;
    if (kind == 0) {
        on = false;
        return KC_OK;
    }
    const int n_rec = kind == 1 ? 1 : (kind == 2 ? 2 : 4);
    if (!slots || (kind == 3 && !t)) return fail(c, KC_ERR_ARG, "kc_sigma_surface_slots: slots / times");
    const double* e[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < n_rec; ++k) {
        if (slots[k] < 0 || slots[k] >= kSlots) return fail(c, KC_ERR_ARG, "kc_sigma_surface_slots: slot");
        const Slot& sl = c->slots[slots[k]];
        if (!sl.has_eta || sl.n != c->N)
            return fail(c, KC_ERR_STATE, "kc_sigma_surface_slots: a slot without this mesh's surface");
        e[k] = sl.eta;
    }
    if (kind == 3 && !(t[0] < t[1] && t[1] < t[2] && t[2] < t[3]))
        return fail(c, KC_ERR_ARG, "kc_sigma_surface_slots: stencil times must increase");
    KC_CUDA(c, cudaSetDevice(c->device));
    double*& buf = which == 0 ? c->d_sig_eta_s : c->d_sig_eta_e;
    if (!buf) KC_CUDA(c, cudaMalloc((void**)&buf, (size_t)c->N * 8));
    int rc = wait_slots(c, slots, n_rec);
    if (rc) return rc;
    k_surface<<<grid_for(c->N), kBlock, 0, c->stream>>>(c->N, kind, e[0], e[1], e[2], e[3], alpha,
                                                        kind == 3 ? t[0] : 0.0, kind == 3 ? t[1] : 0.0,
                                                        kind == 3 ? t[2] : 0.0, kind == 3 ? t[3] : 0.0, q, buf);
    KC_CUDA(c, cudaGetLastError());
    rc = mark_slots_used(c, slots, n_rec);
    if (rc) return rc;
    on = true;
    return KC_OK;
}

int kc_depth_points_upload(kc_ctx* c, int M, const double* p, const int* last, const double* bed) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_depth_points_upload: no mesh uploaded");
    if (M <= 0 || !p || !last || !bed) return fail(c, KC_ERR_ARG, "kc_depth_points_upload: empty table");
    for (long long i = 0; i < c->N; ++i)
        if (last[i] < 0 || last[i] >= M) return fail(c, KC_ERR_ARG, "kc_depth_points_upload: last out of range");
    for (int k = 1; k < M; ++k)
        if (!(p[k] >= p[k - 1])) return fail(c, KC_ERR_ARG, "kc_depth_points_upload: points not non-decreasing");
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    dfree(c->d_dl_p); dfree(c->d_dl_last); dfree(c->d_dl_bed);
    int rc;
    if ((rc = upload(c, &c->d_dl_p, p, (size_t)M))) return rc;
    if ((rc = upload(c, &c->d_dl_last, last, (size_t)c->N))) return rc;
    if ((rc = upload(c, &c->d_dl_bed, bed, (size_t)c->N))) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    c->dm.dl_p = c->d_dl_p;
    c->dm.dl_last = c->d_dl_last;
    c->dm.dl_bed = c->d_dl_bed;
    c->dm.dl_M = M;
    return KC_OK;
}

// One (rows, n) float array into half storage with per-row scales: staged
// through a float device buffer, scaled and rounded on the device.
static int upload_half(kc_ctx* c, const float* host, long long n, int rows, float** scale, size_t* scale_cap,
                       __half* out) {
    const size_t total = (size_t)n * rows;
    if (c->stage_cap < total) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        dfree(c->stage);
        KC_CUDA(c, cudaMalloc((void**)&c->stage, total * 4));
        c->stage_cap = total;
    }
    if (*scale == nullptr || *scale_cap < (size_t)rows) {
        dfree(*scale);
        KC_CUDA(c, cudaMalloc((void**)scale, (size_t)rows * 4));
        *scale_cap = rows;
    }
    KC_CUDA(c, cudaMemcpyAsync(c->stage, host, total * 4, cudaMemcpyHostToDevice, c->stream));
    k_row_scale<<<rows, 256, 0, c->stream>>>(c->stage, n, *scale);
    KC_CUDA(c, cudaGetLastError());
    k_to_half<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(c->stage, n, (long long)total, *scale, out);
    KC_CUDA(c, cudaGetLastError());
    // the staging buffer is reused by the next array
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_field_upload(kc_ctx* c, int slot, int dtype, long long n_nodes, int n_uv_rows, const void* u,
                    const void* v, int n_w_rows, const void* w) {
    if (!c) return KC_ERR_ARG;
    if (slot < 0 || slot >= kSlots) return fail(c, KC_ERR_ARG, "kc_field_upload: slot out of range");
    if (dtype != KC_F32 && dtype != KC_F64 && dtype != KC_F16) return fail(c, KC_ERR_ARG, "kc_field_upload: dtype");
    if (n_nodes <= 0 || n_uv_rows <= 0 || !u || !v) return fail(c, KC_ERR_ARG, "kc_field_upload: empty u/v");
    if (n_w_rows > 0 && !w) return fail(c, KC_ERR_ARG, "kc_field_upload: missing w");
    KC_CUDA(c, cudaSetDevice(c->device));
    Slot& s = c->slots[slot];
    if (c->copy_stream) {   // an asynchronous copy may still be writing the slot
        KC_CUDA(c, cudaStreamSynchronize(c->copy_stream));
        s.pending = false;
    }
    size_t es = dtype == KC_F32 ? 4 : (dtype == KC_F16 ? 2 : 8);
    size_t nuv = (size_t)n_nodes * n_uv_rows * es;
    size_t nw = (size_t)n_nodes * (n_w_rows > 0 ? n_w_rows : 0) * es;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    if (s.cap_uv < nuv) {
        dfree(s.u); dfree(s.v);
        KC_CUDA(c, cudaMalloc(&s.u, nuv));
        KC_CUDA(c, cudaMalloc(&s.v, nuv));
        s.cap_uv = nuv;
    }
    if (s.cap_w < nw) {
        dfree(s.w);
        KC_CUDA(c, cudaMalloc(&s.w, nw));
        s.cap_w = nw;
    }
    if (dtype == KC_F16) {
        int rc;
        if ((rc = upload_half(c, (const float*)u, n_nodes, n_uv_rows, &s.su, &s.cap_su, (__half*)s.u))) return rc;
        if ((rc = upload_half(c, (const float*)v, n_nodes, n_uv_rows, &s.sv, &s.cap_sv, (__half*)s.v))) return rc;
        if (nw && (rc = upload_half(c, (const float*)w, n_nodes, n_w_rows, &s.sw, &s.cap_sw, (__half*)s.w))) return rc;
    } else {
        KC_CUDA(c, cudaMemcpyAsync(s.u, u, nuv, cudaMemcpyHostToDevice, c->stream));
        KC_CUDA(c, cudaMemcpyAsync(s.v, v, nuv, cudaMemcpyHostToDevice, c->stream));
        if (nw) KC_CUDA(c, cudaMemcpyAsync(s.w, w, nw, cudaMemcpyHostToDevice, c->stream));
    }
    s.n = n_nodes; s.uv_rows = n_uv_rows; s.w_rows = n_w_rows > 0 ? n_w_rows : 0; s.dtype = dtype;
    s.az_rows = 0;   // a new snapshot carries no Az until kc_field_upload_az
    s.has_eta = false;   // nor a surface until kc_field_upload_eta
    return KC_OK;
}

int kc_field_upload_async(kc_ctx* c, int slot, int dtype, long long n_nodes, int n_uv_rows, const void* u,
                          const void* v, int n_w_rows, const void* w) {
    if (!c) return KC_ERR_ARG;
    if (slot < 0 || slot >= kSlots) return fail(c, KC_ERR_ARG, "kc_field_upload_async: slot out of range");
    if (dtype != KC_F32 && dtype != KC_F64)
        return fail(c, KC_ERR_ARG, "kc_field_upload_async: float32 or float64 (float16 storage converts synchronously)");
    if (n_nodes <= 0 || n_uv_rows <= 0 || !u || !v) return fail(c, KC_ERR_ARG, "kc_field_upload_async: empty u/v");
    if (n_w_rows > 0 && !w) return fail(c, KC_ERR_ARG, "kc_field_upload_async: missing w");
    KC_CUDA(c, cudaSetDevice(c->device));
    if (!c->copy_stream) KC_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    Slot& s = c->slots[slot];
    const size_t es = dtype == KC_F32 ? 4 : 8;
    const size_t nuv = (size_t)n_nodes * n_uv_rows * es;
    const size_t nw = (size_t)n_nodes * (n_w_rows > 0 ? n_w_rows : 0) * es;
    if (s.cap_uv < nuv || s.cap_w < nw) {   // growing the slot: let every use of it finish first
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        KC_CUDA(c, cudaStreamSynchronize(c->copy_stream));
        s.pending = false;
        if (s.cap_uv < nuv) {
            dfree(s.u); dfree(s.v);
            KC_CUDA(c, cudaMalloc(&s.u, nuv));
            KC_CUDA(c, cudaMalloc(&s.v, nuv));
            s.cap_uv = nuv;
        }
        if (s.cap_w < nw) {
            dfree(s.w);
            KC_CUDA(c, cudaMalloc(&s.w, nw));
            s.cap_w = nw;
        }
    }
    if (s.has_used) KC_CUDA(c, cudaStreamWaitEvent(c->copy_stream, s.used, 0));
    KC_CUDA(c, cudaMemcpyAsync(s.u, u, nuv, cudaMemcpyHostToDevice, c->copy_stream));
    KC_CUDA(c, cudaMemcpyAsync(s.v, v, nuv, cudaMemcpyHostToDevice, c->copy_stream));
    if (nw) KC_CUDA(c, cudaMemcpyAsync(s.w, w, nw, cudaMemcpyHostToDevice, c->copy_stream));
    if (!s.ready) KC_CUDA(c, cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
    KC_CUDA(c, cudaEventRecord(s.ready, c->copy_stream));
    s.pending = true;
    s.n = n_nodes; s.uv_rows = n_uv_rows; s.w_rows = n_w_rows > 0 ? n_w_rows : 0; s.dtype = dtype;
    s.az_rows = 0;
    s.has_eta = false;
    return KC_OK;
}

// Device particle buffers for at least P particles.
static int ensure_capacity(kc_ctx* c, long long P) {
    if (P <= c->cap) return KC_OK;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    free_particles(c);
    // every per-particle buffer holds 8 bytes per particle, so the re-sort
    // can gather any array into the spare buffer and swap the pointers
    size_t n = (size_t)P * 8;
    KC_CUDA(c, cudaMalloc((void**)&c->lon, n)); KC_CUDA(c, cudaMalloc((void**)&c->lat, n));
    KC_CUDA(c, cudaMalloc((void**)&c->z, n)); KC_CUDA(c, cudaMalloc((void**)&c->U, n));
    KC_CUDA(c, cudaMalloc((void**)&c->V, n)); KC_CUDA(c, cudaMalloc((void**)&c->W, n));
    KC_CUDA(c, cudaMalloc((void**)&c->status, n)); KC_CUDA(c, cudaMalloc((void**)&c->nn, n));
    KC_CUDA(c, cudaMalloc((void**)&c->fr, n)); KC_CUDA(c, cudaMalloc((void**)&c->pid, n));
    KC_CUDA(c, cudaMalloc((void**)&c->rs, n)); KC_CUDA(c, cudaMalloc((void**)&c->orig, n));
    KC_CUDA(c, cudaMalloc((void**)&c->rid, n));
    KC_CUDA(c, cudaMalloc((void**)&c->elem, n));
    KC_CUDA(c, cudaMalloc((void**)&c->el, n));
    KC_CUDA(c, cudaMalloc((void**)&c->wel, n));
    KC_CUDA(c, cudaMalloc((void**)&c->spare, n));
    KC_CUDA(c, cudaMalloc((void**)&c->prev, n)); KC_CUDA(c, cudaMalloc((void**)&c->wet, n));
    KC_CUDA(c, cudaMalloc((void**)&c->nn_ok, n));
    c->cap = P;
    return KC_OK;
}

int kc_field_upload_az(kc_ctx* c, int slot, int dtype, long long n_nodes, int n_rows, const void* az) {
    if (!c) return KC_ERR_ARG;
    if (slot < 0 || slot >= kSlots) return fail(c, KC_ERR_ARG, "kc_field_upload_az: slot out of range");
    Slot& s = c->slots[slot];
    if (s.dtype < 0) return fail(c, KC_ERR_STATE, "kc_field_upload_az: upload the snapshot first");
    if (dtype != s.dtype || dtype == KC_F16)
        return fail(c, KC_ERR_ARG, "kc_field_upload_az: Az takes the snapshot's element type, float32 or float64");
    if (n_nodes != s.n || n_rows <= 0 || !az) return fail(c, KC_ERR_ARG, "kc_field_upload_az: shape");
    KC_CUDA(c, cudaSetDevice(c->device));
    const size_t bytes = (size_t)n_nodes * n_rows * (dtype == KC_F32 ? 4 : 8);
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    if (s.cap_az < bytes) {
        dfree(s.az);
        KC_CUDA(c, cudaMalloc(&s.az, bytes));
        s.cap_az = bytes;
    }
    KC_CUDA(c, cudaMemcpyAsync(s.az, az, bytes, cudaMemcpyHostToDevice, c->stream));
    s.az_rows = n_rows;
    return KC_OK;
}

int kc_field_upload_eta(kc_ctx* c, int slot, long long n_nodes, const double* eta) {
    if (!c) return KC_ERR_ARG;
    if (slot < 0 || slot >= kSlots) return fail(c, KC_ERR_ARG, "kc_field_upload_eta: slot out of range");
    Slot& s = c->slots[slot];
    if (s.dtype < 0) return fail(c, KC_ERR_STATE, "kc_field_upload_eta: upload the snapshot first");
    if (n_nodes != s.n || !eta) return fail(c, KC_ERR_ARG, "kc_field_upload_eta: shape");
    KC_CUDA(c, cudaSetDevice(c->device));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    if (s.cap_eta < n_nodes) {
        dfree(s.eta);
        KC_CUDA(c, cudaMalloc((void**)&s.eta, (size_t)n_nodes * 8));
        s.cap_eta = n_nodes;
    }
    KC_CUDA(c, cudaMemcpyAsync(s.eta, eta, (size_t)n_nodes * 8, cudaMemcpyHostToDevice, c->stream));
    s.has_eta = true;
    return KC_OK;
}

int kc_particles_upload(kc_ctx* c, long long P, const double* lon, const double* lat, const double* z,
                        const int* status, const int* nn, const signed char* fr, const long long* pid,
                        const int* rs) {
    if (!c) return KC_ERR_ARG;
    if (P < 0 || (P > 0 && (!lon || !lat || !status || !nn)))
        return fail(c, KC_ERR_ARG, "kc_particles_upload: missing array");
    KC_CUDA(c, cudaSetDevice(c->device));
    int rc0 = ensure_capacity(c, P);
    if (rc0) return rc0;
    c->P = P;
    c->sorted = false;
    c->has_beach = false;   // the beaching state belongs to the particles it was uploaded with
    if (P == 0) return KC_OK;
    size_t n = (size_t)P;
    cudaStream_t s = c->stream;
    k_iota64<<<grid_for(P), kBlock, 0, s>>>(c->orig, P);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(c->lon, lon, n * 8, cudaMemcpyHostToDevice, s));
    KC_CUDA(c, cudaMemcpyAsync(c->lat, lat, n * 8, cudaMemcpyHostToDevice, s));
    if (z) KC_CUDA(c, cudaMemcpyAsync(c->z, z, n * 8, cudaMemcpyHostToDevice, s));
    else KC_CUDA(c, cudaMemsetAsync(c->z, 0, n * 8, s));
    KC_CUDA(c, cudaMemcpyAsync(c->status, status, n * 4, cudaMemcpyHostToDevice, s));
    KC_CUDA(c, cudaMemcpyAsync(c->nn, nn, n * 4, cudaMemcpyHostToDevice, s));
    if (fr) KC_CUDA(c, cudaMemcpyAsync(c->fr, fr, n, cudaMemcpyHostToDevice, s));
    else KC_CUDA(c, cudaMemsetAsync(c->fr, 0, n, s));
    c->has_pid = pid != nullptr;
    if (pid) KC_CUDA(c, cudaMemcpyAsync(c->pid, pid, n * 8, cudaMemcpyHostToDevice, s));
    c->has_rs = rs != nullptr;
    if (rs) KC_CUDA(c, cudaMemcpyAsync(c->rs, rs, n * 4, cudaMemcpyHostToDevice, s));
    c->has_rid = false;
    c->has_elem = false;
    KC_CUDA(c, cudaMemsetAsync(c->nn_ok, 0, n, s));   // uploaded anchors are not trusted
    KC_CUDA(c, cudaMemsetAsync(c->U, 0, n * 8, s));
    KC_CUDA(c, cudaMemsetAsync(c->V, 0, n * 8, s));
    KC_CUDA(c, cudaMemsetAsync(c->W, 0, n * 8, s));
    return KC_OK;
}

int kc_particles_download(kc_ctx* c, long long P, double* lon, double* lat, double* z, int* status, int* nn,
                          signed char* fr, double* u, double* v, double* w) {
    if (!c) return KC_ERR_ARG;
    if (P != c->P) return fail(c, KC_ERR_ARG, "kc_particles_download: P differs from the resident count");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    int rc;
    if ((rc = fetch(c, lon, c->lon, 8))) return rc;
    if ((rc = fetch(c, lat, c->lat, 8))) return rc;
    if ((rc = fetch(c, z, c->z, 8))) return rc;
    if ((rc = fetch(c, status, c->status, 4))) return rc;
    if ((rc = fetch(c, nn, c->nn, 4))) return rc;
    if ((rc = fetch(c, fr, c->fr, 1))) return rc;
    if ((rc = fetch(c, u, c->U, 8))) return rc;
    if ((rc = fetch(c, v, c->V, 8))) return rc;
    if ((rc = fetch(c, w, c->W, 8))) return rc;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_sort(kc_ctx* c) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sort: no mesh uploaded");
    const long long P = c->P;
    if (P <= 1) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    if (P > c->sort_cap) {
        KC_CUDA(c, cudaStreamSynchronize(s));
        dfree(c->skey[0]); dfree(c->skey[1]); dfree(c->sidx[0]); dfree(c->sidx[1]); dfree(c->cub_tmp);
        for (int k = 0; k < 2; ++k) {
            KC_CUDA(c, cudaMalloc((void**)&c->skey[k], (size_t)P * 4));
            KC_CUDA(c, cudaMalloc((void**)&c->sidx[k], (size_t)P * 4));
        }
        size_t tmp = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp, c->skey[0], c->skey[1], c->sidx[0], c->sidx[1], (int)P, 0, 32, s);
        KC_CUDA(c, cudaMalloc(&c->cub_tmp, tmp));
        c->cub_bytes = tmp;
        c->sort_cap = P;
    }
    if (!c->has_pid) {   // the RNG key stays the slot index the particles were uploaded with
        KC_CUDA(c, cudaMemcpyAsync(c->pid, c->orig, (size_t)P * 8, cudaMemcpyDeviceToDevice, s));
        c->has_pid = true;
    }
    const long long ncell = (long long)c->dm.nx * c->dm.ny;
    int bits = 1;
    while (bits < 32 && (1ll << bits) <= ncell) ++bits;
    k_sort_keys<<<grid_for(P), kBlock, 0, s>>>(c->dm, c->lon, c->lat, c->status, P, c->skey[0], c->sidx[0]);
    KC_CUDA(c, cudaGetLastError());
    size_t tmp = c->cub_bytes;
    KC_CUDA(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp, tmp, c->skey[0], c->skey[1], c->sidx[0], c->sidx[1],
                                               (int)P, 0, bits, s));
    const int* idx = c->sidx[1];
    int rc;
    if ((rc = regather(c, (void**)&c->lon, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->lat, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->z, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->U, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->V, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->W, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->pid, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->orig, 8, idx))) return rc;
    if ((rc = regather(c, (void**)&c->status, 4, idx))) return rc;
    if ((rc = regather(c, (void**)&c->nn, 4, idx))) return rc;
    if ((rc = regather(c, (void**)&c->fr, 1, idx))) return rc;
    if ((rc = regather(c, (void**)&c->nn_ok, 1, idx))) return rc;
    if ((rc = regather(c, (void**)&c->el, 4, idx))) return rc;
    if ((rc = regather(c, (void**)&c->wel, 4, idx))) return rc;
    if (c->has_rs && (rc = regather(c, (void**)&c->rs, 4, idx))) return rc;
    if (c->has_rid && (rc = regather(c, (void**)&c->rid, 4, idx))) return rc;
    if (c->has_elem && (rc = regather(c, (void**)&c->elem, 4, idx))) return rc;
    if (c->has_beach) {
        if ((rc = regather(c, (void**)&c->prev, 4, idx))) return rc;
        if ((rc = regather(c, (void**)&c->wet, 4, idx))) return rc;
    }
    c->sorted = true;
    return KC_OK;
}

int kc_step_host(kc_ctx* c, const kc_step_args* a, long long P, const kc_host_particles* in,
                 const kc_host_particles* out, long long chunk) {
    if (!c || !in || !out) return KC_ERR_ARG;
    if (P < 0) return fail(c, KC_ERR_ARG, "kc_step_host: P < 0");
    if (P > 0 && (!in->lon || !in->lat || !in->status || !in->nearest_node || !out->lon || !out->lat ||
                  !out->status || !out->nearest_node))
        return fail(c, KC_ERR_ARG, "kc_step_host: lon, lat, status and nearest_node are required in and out");
    if (out->elem && !in->elem) return fail(c, KC_ERR_ARG, "kc_step_host: out.elem needs in.elem (walk mode)");
    if (in->elem && !c->dm.enb) return fail(c, KC_ERR_STATE, "kc_step_host: upload the element neighbours first");
    KC_CUDA(c, cudaSetDevice(c->device));
    int rc = ensure_capacity(c, P);
    if (rc) return rc;
    c->P = P;
    c->sorted = false;
    c->has_pid = in->pid != nullptr;
    c->has_rs = in->release_step != nullptr;
    c->has_rid = in->real_id != nullptr;
    c->has_elem = in->elem != nullptr;
    c->has_beach = false;
    if ((rc = check_step(c, a))) return rc;
    if (P == 0) return KC_OK;
    if (!c->s_in) {
        KC_CUDA(c, cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
        KC_CUDA(c, cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
        for (int k = 0; k < kChunks; ++k) {
            KC_CUDA(c, cudaEventCreateWithFlags(&c->ev_in[k], cudaEventDisableTiming));
            KC_CUDA(c, cudaEventCreateWithFlags(&c->ev_k[k], cudaEventDisableTiming));
        }
        KC_CUDA(c, cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming));
    }
    // chunk: a multiple of the block size, at most kChunks chunks; by default
    // eight, but no smaller than 2^18 particles, so a small state is not cut
    // into pieces whose copies and launches cost more than they overlap
    long long ch = chunk > 0 ? chunk : std::max((P + 7) / 8, 1LL << 18);
    ch = std::max(ch, (P + kChunks - 1) / kChunks);
    ch = std::max<long long>(kBlock, (ch + kBlock - 1) / kBlock * kBlock);
    const int nch = (int)((P + ch - 1) / ch);
    // the copies start after everything queued on the library's stream
    KC_CUDA(c, cudaEventRecord(c->ev_start, c->stream));
    KC_CUDA(c, cudaStreamWaitEvent(c->s_in, c->ev_start, 0));
    const kc::DState full = state_of(c);
    const kc::DStep s0 = step_of(a);
    for (int k = 0; k < nch; ++k) {
        const long long b = (long long)k * ch, n = std::min(ch, P - b);
        cudaStream_t si = c->s_in;
        KC_CUDA(c, cudaMemcpyAsync(c->lon + b, in->lon + b, n * 8, cudaMemcpyHostToDevice, si));
        KC_CUDA(c, cudaMemcpyAsync(c->lat + b, in->lat + b, n * 8, cudaMemcpyHostToDevice, si));
        if (in->z) KC_CUDA(c, cudaMemcpyAsync(c->z + b, in->z + b, n * 8, cudaMemcpyHostToDevice, si));
        else KC_CUDA(c, cudaMemsetAsync(c->z + b, 0, n * 8, si));
        KC_CUDA(c, cudaMemcpyAsync(c->status + b, in->status + b, n * 4, cudaMemcpyHostToDevice, si));
        KC_CUDA(c, cudaMemcpyAsync(c->nn + b, in->nearest_node + b, n * 4, cudaMemcpyHostToDevice, si));
        if (in->failure_reason)
            KC_CUDA(c, cudaMemcpyAsync(c->fr + b, in->failure_reason + b, n, cudaMemcpyHostToDevice, si));
        else KC_CUDA(c, cudaMemsetAsync(c->fr + b, 0, n, si));
        if (in->pid) KC_CUDA(c, cudaMemcpyAsync(c->pid + b, in->pid + b, n * 8, cudaMemcpyHostToDevice, si));
        if (in->real_id) KC_CUDA(c, cudaMemcpyAsync(c->rid + b, in->real_id + b, n * 4, cudaMemcpyHostToDevice, si));
        if (in->release_step)
            KC_CUDA(c, cudaMemcpyAsync(c->rs + b, in->release_step + b, n * 4, cudaMemcpyHostToDevice, si));
        if (in->elem) KC_CUDA(c, cudaMemcpyAsync(c->elem + b, in->elem + b, n * 4, cudaMemcpyHostToDevice, si));
        KC_CUDA(c, cudaEventRecord(c->ev_in[k], si));
        // the chunk's particles as a state of their own: RNG keys stay the
        // global index (pid_offset + base + local index); carried anchors are
        // not trusted (nn_ok null), as for any upload
        kc::DState st = full;
        st.lon += b; st.lat += b; st.z += b; st.status += b; st.nn += b;
        st.U += b; st.V += b; st.W += b; st.fr += b;
        st.pid = in->pid ? c->pid + b : nullptr;
        st.rid = in->real_id ? c->rid + b : nullptr;
        st.release_step = in->release_step ? c->rs + b : nullptr;
        st.elem = in->elem ? c->elem + b : nullptr;
        st.prev = nullptr; st.nn_ok = nullptr; st.el = nullptr; st.wel = nullptr;
        st.P = n;
        kc::DStep sk = s0;
        if (!in->pid) sk.pid_offset = s0.pid_offset + (unsigned long long)b;
        KC_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_in[k], 0));
        if ((rc = launch_step_on(c, a, st, sk))) return rc;
        KC_CUDA(c, cudaEventRecord(c->ev_k[k], c->stream));
    }
    // downloads after every upload and step is queued: a copy into pageable
    // memory returns only when done, and must not hold back the queueing
    for (int k = 0; k < nch; ++k) {
        const long long b = (long long)k * ch, n = std::min(ch, P - b);
        cudaStream_t so = c->s_out;
        KC_CUDA(c, cudaStreamWaitEvent(so, c->ev_k[k], 0));
        KC_CUDA(c, cudaMemcpyAsync(out->lon + b, c->lon + b, n * 8, cudaMemcpyDeviceToHost, so));
        KC_CUDA(c, cudaMemcpyAsync(out->lat + b, c->lat + b, n * 8, cudaMemcpyDeviceToHost, so));
        if (out->z) KC_CUDA(c, cudaMemcpyAsync(out->z + b, c->z + b, n * 8, cudaMemcpyDeviceToHost, so));
        KC_CUDA(c, cudaMemcpyAsync(out->status + b, c->status + b, n * 4, cudaMemcpyDeviceToHost, so));
        KC_CUDA(c, cudaMemcpyAsync(out->nearest_node + b, c->nn + b, n * 4, cudaMemcpyDeviceToHost, so));
        if (out->failure_reason)
            KC_CUDA(c, cudaMemcpyAsync(out->failure_reason + b, c->fr + b, n, cudaMemcpyDeviceToHost, so));
        if (out->u) KC_CUDA(c, cudaMemcpyAsync(out->u + b, c->U + b, n * 8, cudaMemcpyDeviceToHost, so));
        if (out->v) KC_CUDA(c, cudaMemcpyAsync(out->v + b, c->V + b, n * 8, cudaMemcpyDeviceToHost, so));
        if (out->w) KC_CUDA(c, cudaMemcpyAsync(out->w + b, c->W + b, n * 8, cudaMemcpyDeviceToHost, so));
        if (out->elem) KC_CUDA(c, cudaMemcpyAsync(out->elem + b, c->elem + b, n * 4, cudaMemcpyDeviceToHost, so));
    }
    KC_CUDA(c, cudaStreamSynchronize(c->s_out));
    KC_CUDA(c, cudaMemsetAsync(c->nn_ok, 0, (size_t)P, c->stream));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

// A particle state view of [begin, begin + count) of st.
static kc::DState state_range(kc::DState st, long long begin, long long count) {
    st.lon += begin; st.lat += begin; st.z += begin; st.status += begin; st.nn += begin;
    st.U += begin; st.V += begin; st.W += begin; st.fr += begin;
    if (st.pid) st.pid += begin;
    if (st.rid) st.rid += begin;
    if (st.release_step) st.release_step += begin;
    if (st.prev) st.prev += begin;
    if (st.nn_ok) st.nn_ok += begin;
    if (st.elem) st.elem += begin;
    if (st.el) st.el += begin;
    if (st.wel) st.wel += begin;
    st.P = count;
    return st;
}

int kc_step_range(kc_ctx* c, const kc_step_args* a, long long begin, long long count) {
    if (!c) return KC_ERR_ARG;
    int rc = check_step(c, a);
    if (rc) return rc;
    if (begin < 0 || count < 0 || begin + count > c->P)
        return fail(c, KC_ERR_ARG, "kc_step_range: range outside the resident particles");
    if (count == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    const kc::DState st = state_range(state_of(c), begin, count);
    kc::DStep s = step_of(a);
    if (!st.pid) s.pid_offset += (unsigned long long)begin;   // keys stay the global index
    return launch_step_on(c, a, st, s);
}

extern "C++" {
template <typename T>
static void launch_multi(kc_ctx* c, int precision, int dtype, const MultiHead* dh, const void* dp, int dims,
                         int scheme) {
    if (precision == KC_MIXED) {
        if (dtype == KC_F16)
            kc_launch_multi_mixed_f16(c->dm, dh, (const StepPack<__half>*)dp, c->P, dims, scheme, c->fused_block,
                                      c->stream);
        else
            kc_launch_multi_mixed_f32(c->dm, dh, (const StepPack<float>*)dp, c->P, dims, scheme, c->fused_block,
                                      c->stream);
    } else if constexpr (std::is_same<T, double>::value) {   // the plain form never reads half storage
        kc_launch_multi_plain_f64(c->dm, dh, (const StepPack<double>*)dp, c->P, dims, scheme, c->fused_block,
                                  c->stream);
    } else if constexpr (std::is_same<T, float>::value) {
        kc_launch_multi_plain_f32(c->dm, dh, (const StepPack<float>*)dp, c->P, dims, scheme, c->fused_block,
                                  c->stream);
    }
}

template <typename T>
static int run_fused_t(kc_ctx* c, const kc_step_args* steps, int n, const kc_beach_args* beach, int use_graph) {
    const size_t head_bytes = (sizeof(MultiHead) + 255) / 256 * 256;
    const size_t bytes = head_bytes + sizeof(StepPack<T>) * (size_t)n;
    if (c->fused_ev_pending) {   // the previous call's upload has read the staging buffer
        KC_CUDA(c, cudaEventSynchronize(c->fused_ev));
        c->fused_ev_pending = false;
    }
    if (c->fused_cap < bytes) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        if (c->fused_exec) cudaGraphExecDestroy(c->fused_exec);
        c->fused_exec = nullptr;
        c->fused_key.clear();
        if (c->fused_host) cudaFreeHost(c->fused_host);
        c->fused_host = nullptr;
        dfree(c->fused_dev);
        c->fused_cap = 0;
        KC_CUDA(c, cudaHostAlloc(&c->fused_host, bytes, cudaHostAllocDefault));
        KC_CUDA(c, cudaMalloc(&c->fused_dev, bytes));
        c->fused_cap = bytes;
    }
    if (!c->fused_ev) KC_CUDA(c, cudaEventCreateWithFlags(&c->fused_ev, cudaEventDisableTiming));
    for (int j = 0; j < n; ++j) {   // pending asynchronous snapshot copies, waited on before any capture
        int sl[4];
        const int nsl = step_slots(&steps[j], sl);
        int rc = wait_slots(c, sl, nsl);
        if (rc) return rc;
    }
    MultiHead* h = (MultiHead*)c->fused_host;
    h->st = state_of(c);
    h->N = c->N;
    h->n_steps = n;
    StepPack<T>* pk = (StepPack<T>*)((char*)c->fused_host + head_bytes);
    for (int j = 0; j < n; ++j) {
        std::memset((void*)&pk[j], 0, sizeof(StepPack<T>));
        pk[j].f = blend_of<T>(c, &steps[j]);
        pk[j].s = step_of(&steps[j]);
        pk[j].beach = beach ? 1 : 0;
        if (beach) {
            if (c->beach_eta_on || c->beach_dry_on)   // one surface per call cannot follow several steps
                return fail(c, KC_ERR_ARG, "kc_run_fused: beaching surfaces are per step; use kc_step + kc_beach");
            int rc = beach_of(c, &beach[j], pk[j].b);
            if (rc) return rc;
        }
    }
    const MultiHead* dh = (const MultiHead*)c->fused_dev;
    const void* dp = (const char*)c->fused_dev + head_bytes;
    const int precision = steps[0].precision, dtype = c->slots[steps[0].slot_a].dtype;
    const int dims = steps[0].dims, scheme = steps[0].scheme;
    if (!use_graph) {
        KC_CUDA(c, cudaMemcpyAsync(c->fused_dev, c->fused_host, bytes, cudaMemcpyHostToDevice, c->stream));
        launch_multi<T>(c, precision, dtype, dh, dp, dims, scheme);
        KC_CUDA(c, cudaGetLastError());
    } else {
        const std::string key = std::to_string(precision) + "/" + std::to_string(dtype) + "/" + std::to_string(dims) +
                                "/" + std::to_string(scheme) + "/" + std::to_string(n) + "/" +
                                std::to_string(bytes) + "/" + std::to_string(c->P) + "/" +
                                std::to_string(c->mesh_gen) + "/" + std::to_string(c->fused_block) + "/" +
                                std::to_string((size_t)c->fused_dev) + "/" +
                                std::to_string((size_t)c->fused_host);
        if (key != c->fused_key || !c->fused_exec) {
            if (c->fused_exec) cudaGraphExecDestroy(c->fused_exec);
            c->fused_exec = nullptr;
            c->fused_key.clear();
            // the graph: upload the argument block from the staging buffer,
            // then the fused kernel; replays copy whatever the staging holds
            cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            cudaError_t e1 = cudaMemcpyAsync(c->fused_dev, c->fused_host, bytes, cudaMemcpyHostToDevice, c->stream);
            if (e1 == cudaSuccess) {
                launch_multi<T>(c, precision, dtype, dh, dp, dims, scheme);
                e1 = cudaGetLastError();
            }
            cudaGraph_t g = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e1 != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return fail(c, KC_ERR_CUDA, std::string("graph capture: ") +
                                                cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
            }
            e = cudaGraphInstantiate(&c->fused_exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                c->fused_exec = nullptr;
                return fail(c, KC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            }
            c->fused_key = key;
        }
        KC_CUDA(c, cudaGraphLaunch(c->fused_exec, c->stream));
    }
    KC_CUDA(c, cudaEventRecord(c->fused_ev, c->stream));
    c->fused_ev_pending = true;
    for (int j = 0; j < n; ++j) {
        int sl[4];
        const int nsl = step_slots(&steps[j], sl);
        int rc = mark_slots_used(c, sl, nsl);
        if (rc) return rc;
    }
    return KC_OK;
}

}  // extern "C++"

int kc_set_fused_block(kc_ctx* c, int block) {
    if (!c) return KC_ERR_ARG;
    if (block != 128 && block != 256) return fail(c, KC_ERR_ARG, "kc_set_fused_block: 128 or 256");
    c->fused_block = block;
    return KC_OK;
}

int kc_run_fused(kc_ctx* c, const kc_step_args* steps, int n_steps, const kc_beach_args* beach, int use_graph) {
    if (!c || !steps) return KC_ERR_ARG;
    if (n_steps < 1 || n_steps > 1024) return fail(c, KC_ERR_ARG, "kc_run_fused: n_steps must be in 1..1024");
    int rc;
    for (int j = 0; j < n_steps; ++j) {
        if ((rc = check_step(c, &steps[j]))) return rc;
        const kc_step_args& a = steps[j];
        const kc_step_args& a0 = steps[0];
        if (a.dims != a0.dims || a.scheme != a0.scheme || a.precision != a0.precision ||
            c->slots[a.slot_a].dtype != c->slots[a0.slot_a].dtype)
            return fail(c, KC_ERR_ARG, "kc_run_fused: every step needs the same dims, scheme, form and snapshot type");
    }
    if (c->has_elem)
        return fail(c, KC_ERR_STATE, "kc_run_fused: carried walk elements step through kc_step / kc_run");
    if (c->dm.sig && steps[0].dims == 3)
        return fail(c, KC_ERR_STATE, "kc_run_fused: sigma meshes step through kc_step / kc_run");
    if (c->dm.cg.on) return fail(c, KC_ERR_STATE, "kc_run_fused: C-grid meshes step through kc_step / kc_run");
    if (steps[0].uv_lsq) return fail(c, KC_ERR_STATE, "kc_run_fused: least-squares u/v steps through kc_step / kc_run");
    if (c->P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    if ((rc = pin_pid(c))) return rc;
    const int dtype = c->slots[steps[0].slot_a].dtype;
    if (dtype == KC_F64) return run_fused_t<double>(c, steps, n_steps, beach, use_graph);
    if (dtype == KC_F16) return run_fused_t<__half>(c, steps, n_steps, beach, use_graph);
    return run_fused_t<float>(c, steps, n_steps, beach, use_graph);
}

int kc_step(kc_ctx* c, const kc_step_args* a) {
    if (!c) return KC_ERR_ARG;
    return do_step(c, a);
}

int kc_run(kc_ctx* c, const kc_step_args* steps, int n_steps) {
    if (!c) return KC_ERR_ARG;
    if (n_steps < 0 || (n_steps > 0 && !steps)) return fail(c, KC_ERR_ARG, "kc_run: bad step list");
    for (int k = 0; k < n_steps; ++k) {
        int rc = check_step(c, &steps[k]);
        if (rc) return rc;
    }
    for (int k = 0; k < n_steps; ++k) {
        int rc = do_step(c, &steps[k]);
        if (rc) return rc;
    }
    return KC_OK;
}

int kc_find_nearest(kc_ctx* c, long long P, const double* lon, const double* lat, int* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_find_nearest: no mesh uploaded");
    if (P < 0 || (P > 0 && (!lon || !lat || !out))) return fail(c, KC_ERR_ARG, "kc_find_nearest: arrays");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    if (P > c->qcap) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        dfree(c->q); dfree(c->qout);
        KC_CUDA(c, cudaMalloc((void**)&c->q, (size_t)P * 16));
        KC_CUDA(c, cudaMalloc((void**)&c->qout, (size_t)P * 4));
        c->qcap = P;
    }
    KC_CUDA(c, cudaMemcpyAsync(c->q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    KC_CUDA(c, cudaMemcpyAsync(c->q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    k_nearest<<<grid_for(P), kBlock, 0, c->stream>>>(c->dm, c->q, P, c->qout);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(out, c->qout, (size_t)P * 4, cudaMemcpyDeviceToHost, c->stream));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

// One scratch allocation for a sampling call (values, depths, query,
// anchors, mask, results), freed before kc_sample_field returns.
static int sample_run(kc_ctx* c, char* buf, const double* values, size_t nvals, int rows, const double* z_mids,
                      long long P, const double* lon, const double* lat, const double* z, const int* nearest,
                      const unsigned char* alive, int method, double* out) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    double* d_vals = (double*)buf;
    double* d_zm = (double*)(buf + al(nvals * 8));
    double* d_q = (double*)((char*)d_zm + al((size_t)rows * 8));
    double* d_z = (double*)((char*)d_q + al((size_t)P * 16));
    double* d_out = (double*)((char*)d_z + al((size_t)P * 8));
    int* d_nn = (int*)((char*)d_out + al((size_t)P * 8));
    unsigned char* d_al = (unsigned char*)((char*)d_nn + al((size_t)P * 4));
    cudaStream_t st = c->stream;
    KC_CUDA(c, cudaMemcpyAsync(d_vals, values, nvals * 8, cudaMemcpyHostToDevice, st));
    if (rows > 0) {
        if (z_mids) KC_CUDA(c, cudaMemcpyAsync(d_zm, z_mids, (size_t)rows * 8, cudaMemcpyHostToDevice, st));
        KC_CUDA(c, cudaMemcpyAsync(d_z, z, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    }
    KC_CUDA(c, cudaMemcpyAsync(d_q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    KC_CUDA(c, cudaMemcpyAsync(d_q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    if (alive) KC_CUDA(c, cudaMemcpyAsync(d_al, alive, (size_t)P, cudaMemcpyHostToDevice, st));
    if (nearest) {
        KC_CUDA(c, cudaMemcpyAsync(d_nn, nearest, (size_t)P * 4, cudaMemcpyHostToDevice, st));
    } else {
        k_nearest<<<grid_for(P), kBlock, 0, st>>>(c->dm, d_q, P, d_nn);
        KC_CUDA(c, cudaGetLastError());
    }
    if (rows > 0 && !z_mids) {   // an interface field (K, N)
        kc::DBlend<double> f{};
        f.a.w = f.b.w = f.t.w = d_vals;
        f.alpha0 = 0.0;
        f.n = c->N;
        k_sample_iface<<<grid_for(P), kBlock, 0, st>>>(c->dm, f, d_q, d_z, d_nn, alive ? d_al : nullptr, P, method,
                                                       d_out);
    } else {
        kc::DSample S{};
        S.values = d_vals;
        S.zm = rows > 0 ? d_zm : nullptr;
        S.n = c->N;
        S.rows = rows;
        k_sample<<<grid_for(P), kBlock, 0, st>>>(c->dm, S, d_q, rows > 0 ? d_z : nullptr, d_nn,
                                               alive ? d_al : nullptr, P, method, d_out);
    }
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(out, d_out, (size_t)P * 8, cudaMemcpyDeviceToHost, st));
    KC_CUDA(c, cudaStreamSynchronize(st));
    return KC_OK;
}

int kc_sample_field(kc_ctx* c, const double* values, int rows, const double* z_mids, long long P, const double* lon,
                    const double* lat, const double* z, const int* nearest, const unsigned char* alive, int method,
                    double* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sample_field: no mesh uploaded");
    if (method < 0 || method > 3) return fail(c, KC_ERR_ARG, "kc_sample_field: method must be 0..3");
    if (rows < 0 || !values || P < 0 || (P > 0 && (!lon || !lat || !out)))
        return fail(c, KC_ERR_ARG, "kc_sample_field: arrays");
    if (rows > 0 && ((P > 0 && !z) || !c->d_depth))
        return fail(c, KC_ERR_ARG, "kc_sample_field: a 3-D field needs the depths and the mesh depth");
    if (rows > 0 && !z_mids && (rows != c->dm.K || c->dm.sig || !c->dm.zlev))
        return fail(c, KC_ERR_ARG, "kc_sample_field: without z_mids the field is an interface field of the mesh's "
                                   "K z-levels");
    if (nearest)
        for (long long i = 0; i < P; ++i)
            if (nearest[i] >= c->N) return fail(c, KC_ERR_ARG, "kc_sample_field: nearest node out of range");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    const size_t nvals = (size_t)(rows > 0 ? rows : 1) * (size_t)c->N;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t total = al(nvals * 8) + al((size_t)rows * 8) + al((size_t)P * 16) + 2 * al((size_t)P * 8) +
                         al((size_t)P * 4) + al((size_t)P);
    char* buf = nullptr;
    KC_CUDA(c, cudaMalloc((void**)&buf, total));
    const int rc = sample_run(c, buf, values, nvals, rows, z_mids, P, lon, lat, z, nearest, alive, method, out);
    cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    return rc;
}

int kc_sample_field_sigma(kc_ctx* c, const double* values, int rows, const double* eta, double Dmin, long long P,
                          const double* lon, const double* lat, const double* z, const int* nearest,
                          const unsigned char* alive, int method, double* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_sample_field_sigma: no mesh uploaded");
    if (!c->dm.sig || !c->d_sigma) return fail(c, KC_ERR_STATE, "kc_sample_field_sigma: the mesh is not a sigma mesh");
    if (method < 0 || method > 3 || method == kc::S_BARYCENTRIC)
        return fail(c, KC_ERR_ARG, "kc_sample_field_sigma: method must be 0 (nearest), 1 (leastsq) or 3 (idw)");
    const int K = c->dm.K;
    if ((rows != K && rows != K - 1) || K < 2 || !values || !eta || !(Dmin > 0.0) || P < 0 ||
        (P > 0 && (!lon || !lat || !z || !out)))
        return fail(c, KC_ERR_ARG, "kc_sample_field_sigma: a (K, N) or (K-1, N) field, eta, Dmin > 0, depths");
    if (nearest)
        for (long long i = 0; i < P; ++i)
            if (nearest[i] >= c->N) return fail(c, KC_ERR_ARG, "kc_sample_field_sigma: nearest node out of range");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t nvals = (size_t)rows * (size_t)c->N;
    const size_t total = al(nvals * 8) + al((size_t)c->N * 8) + al((size_t)P * 16) + 2 * al((size_t)P * 8) +
                         al((size_t)P * 4) + al((size_t)P);
    char* buf = nullptr;
    KC_CUDA(c, cudaMalloc((void**)&buf, total));
    double* d_vals = (double*)buf;
    double* d_eta = (double*)(buf + al(nvals * 8));
    double* d_q = (double*)((char*)d_eta + al((size_t)c->N * 8));
    double* d_z = (double*)((char*)d_q + al((size_t)P * 16));
    double* d_out = (double*)((char*)d_z + al((size_t)P * 8));
    int* d_nn = (int*)((char*)d_out + al((size_t)P * 8));
    unsigned char* d_al = (unsigned char*)((char*)d_nn + al((size_t)P * 4));
    cudaStream_t st = c->stream;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; return e == cudaSuccess; };
    ok(cudaMemcpyAsync(d_vals, values, nvals * 8, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(d_eta, eta, (size_t)c->N * 8, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(d_q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(d_q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(d_z, z, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    if (alive) ok(cudaMemcpyAsync(d_al, alive, (size_t)P, cudaMemcpyHostToDevice, st));
    if (nearest) {
        ok(cudaMemcpyAsync(d_nn, nearest, (size_t)P * 4, cudaMemcpyHostToDevice, st));
    } else if (e == cudaSuccess) {
        k_nearest<<<grid_for(P), kBlock, 0, st>>>(c->dm, d_q, P, d_nn);
        ok(cudaGetLastError());
    }
    if (e == cudaSuccess && rows == K) {
        kc::DBlend<double> f{};
        f.a.w = f.b.w = f.t.w = d_vals;
        f.a.eta = f.b.eta = f.t.eta = d_eta;
        f.alpha0 = 0.0;
        f.n = c->N;
        kc::DStep s{};
        s.dt = 1.0; s.time_dir = 1.0; s.Dmin = Dmin;
        s.w_code = method == kc::S_NEAREST ? 0 : method == kc::S_BARYCENTRIC ? 1 : method == kc::S_LEASTSQ ? 2 : 3;
        s.edge_bc = -1;
        k_sample_iface_sigma<<<grid_for(P), kBlock, 0, st>>>(c->dm, f, s, d_q, d_z, d_nn, alive ? d_al : nullptr, P,
                                                             d_out);
        ok(cudaGetLastError());
    } else if (e == cudaSuccess) {
        kc::DSample S{};
        S.values = d_vals;
        S.n = c->N;
        S.rows = rows;
        S.sig = c->d_sigma;
        S.eta = d_eta;
        S.Dmin = Dmin;
        k_sample<<<grid_for(P), kBlock, 0, st>>>(c->dm, S, d_q, d_z, d_nn, alive ? d_al : nullptr, P, method, d_out);
        ok(cudaGetLastError());
    }
    ok(cudaMemcpyAsync(out, d_out, (size_t)P * 8, cudaMemcpyDeviceToHost, st));
    ok(cudaStreamSynchronize(st));
    cudaFree(buf);
    if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("kc_sample_field_sigma: ") + cudaGetErrorString(e));
    return KC_OK;
}

int kc_find_elements(kc_ctx* c, long long P, const double* lon, const double* lat, const int* nn, int* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_find_elements: no mesh uploaded");
    if (P < 0 || (P > 0 && (!lon || !lat || !out))) return fail(c, KC_ERR_ARG, "kc_find_elements: arrays");
    if (nn)
        for (long long i = 0; i < P; ++i)
            if (nn[i] < 0 || nn[i] >= c->N) return fail(c, KC_ERR_ARG, "kc_find_elements: anchor out of range");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    if (P > c->qcap) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        dfree(c->q); dfree(c->qout);
        KC_CUDA(c, cudaMalloc((void**)&c->q, (size_t)P * 16));
        KC_CUDA(c, cudaMalloc((void**)&c->qout, (size_t)P * 4));
        c->qcap = P;
    }
    KC_CUDA(c, cudaMemcpyAsync(c->q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    KC_CUDA(c, cudaMemcpyAsync(c->q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    if (nn) KC_CUDA(c, cudaMemcpyAsync(c->qout, nn, (size_t)P * 4, cudaMemcpyHostToDevice, c->stream));
    k_contain<<<grid_for(P), kBlock, 0, c->stream>>>(c->dm, c->q, P, nn ? c->qout : nullptr, c->qout);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(out, c->qout, (size_t)P * 4, cudaMemcpyDeviceToHost, c->stream));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_find_elements_walk(kc_ctx* c, long long P, const double* lon, const double* lat, const int* start, int* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_find_elements_walk: no mesh uploaded");
    if (!c->dm.enb) return fail(c, KC_ERR_STATE, "kc_find_elements_walk: upload the element neighbours first");
    if (P < 0 || (P > 0 && (!lon || !lat || !start || !out)))
        return fail(c, KC_ERR_ARG, "kc_find_elements_walk: arrays");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    if (P > c->qcap) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        dfree(c->q); dfree(c->qout);
        KC_CUDA(c, cudaMalloc((void**)&c->q, (size_t)P * 16));
        KC_CUDA(c, cudaMalloc((void**)&c->qout, (size_t)P * 4));
        c->qcap = P;
    }
    KC_CUDA(c, cudaMemcpyAsync(c->q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    KC_CUDA(c, cudaMemcpyAsync(c->q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    KC_CUDA(c, cudaMemcpyAsync(c->qout, start, (size_t)P * 4, cudaMemcpyHostToDevice, c->stream));
    k_walk<<<grid_for(P), kBlock, 0, c->stream>>>(c->dm, c->q, P, c->qout, c->qout);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(out, c->qout, (size_t)P * 4, cudaMemcpyDeviceToHost, c->stream));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Nearest-node queries without any device allocation.
//
// kc_find_nearest grows a per-context staging buffer with cudaMalloc.  Some
// callers cannot allow that: cudaMalloc synchronises the whole device (a stall
// in a latency-bound loop that shares the GPU with other work), and it fails
// outright when the host application has already handed all free device
// memory to its own pool.  kc_find_nearest_noalloc stages the queries and
// results in this fixed array instead, which every GPU that loads the library
// holds until the process exits.  In host code `g_noalloc_scratch` names a
// host-side stand-in, not a device address: the device address is looked up
// once per device with cudaGetSymbolAddress and passed to the kernel.
// ---------------------------------------------------------------------------

constexpr long long kNoAllocMaxPoints = 65536;   // 64 Ki queries -> 1.25 MiB of device memory
constexpr int kNoAllocMaxDevices = 64;

// lon (P doubles), lat (P doubles) at byte P*8, results (P ints) at byte
// kNoAllocMaxPoints*16
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocMaxPoints * 20];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// The device address of the scratch array on the current device (set up on the
// first call per device; the device must be current).
int noalloc_scratch(kc_ctx* c, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (c->device < 0 || c->device >= kNoAllocMaxDevices)
        return fail(c, KC_ERR_ARG, "kc_find_nearest_noalloc: device index beyond the supported range");
    if (!g_noalloc_addr[c->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(c, KC_ERR_CUDA, std::string("kc_find_nearest_noalloc: cudaGetSymbolAddress: ") +
                                            cudaGetErrorString(e));
        g_noalloc_addr[c->device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[c->device]);
    return KC_OK;
}

}  // namespace

extern "C" {

int kc_find_nearest_noalloc(kc_ctx* c, long long P, const double* lon, const double* lat, int* out) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_find_nearest_noalloc: no mesh uploaded");
    if (P < 0 || (P > 0 && (!lon || !lat || !out))) return fail(c, KC_ERR_ARG, "kc_find_nearest_noalloc: arrays");
    if (P > kNoAllocMaxPoints)
        return fail(c, KC_ERR_ARG, "kc_find_nearest_noalloc: " + std::to_string(P) +
                                       " queries exceed the fixed scratch of " + std::to_string(kNoAllocMaxPoints) +
                                       "; split the batch or use kc_find_nearest");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    unsigned char* base = nullptr;
    int rc = noalloc_scratch(c, &base);
    if (rc) return rc;
    double* q = reinterpret_cast<double*>(base);
    int* res = reinterpret_cast<int*>(base + kNoAllocMaxPoints * 16);
    KC_CUDA(c, cudaMemcpyAsync(q, lon, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    KC_CUDA(c, cudaMemcpyAsync(q + P, lat, (size_t)P * 8, cudaMemcpyHostToDevice, c->stream));
    k_nearest<<<grid_for(P), kBlock, 0, c->stream>>>(c->dm, q, P, res);
    KC_CUDA(c, cudaGetLastError());
    KC_CUDA(c, cudaMemcpyAsync(out, res, (size_t)P * 4, cudaMemcpyDeviceToHost, c->stream));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_rng_normals(kc_ctx* c, long long P, unsigned long long seed, unsigned long long real_id,
                   unsigned long long step_i, unsigned long long pid_offset, unsigned long long comp, double* out) {
    if (!c) return KC_ERR_ARG;
    if (P < 0 || (P > 0 && !out)) return fail(c, KC_ERR_ARG, "kc_rng_normals: arrays");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    double* d = nullptr;
    KC_CUDA(c, cudaMallocAsync((void**)&d, (size_t)P * 16, c->stream));
    k_normals<<<grid_for(P), kBlock, 0, c->stream>>>(c->dm.rx, P, seed, real_id, step_i, pid_offset, comp, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t)P * 16, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("kc_rng_normals: ") + cudaGetErrorString(e));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_grid_hash_build(kc_ctx* c, long long n_nodes, const double* lon, const double* lat, double cell_size,
                       double lon_min, double lat_min, int nx, int ny, int wrap, int* offsets, int* node_ids) {
    if (!c) return KC_ERR_ARG;
    if (n_nodes <= 0 || n_nodes > INT_MAX || !lon || !lat || !offsets || !node_ids)
        return fail(c, KC_ERR_ARG, "kc_grid_hash_build: arrays");
    if (!(cell_size > 0.0) || nx <= 0 || ny <= 0 || (long long)nx * ny > 2000000000LL)
        return fail(c, KC_ERR_ARG, "kc_grid_hash_build: grid geometry");
    KC_CUDA(c, cudaSetDevice(c->device));
    const long long N = n_nodes, C = (long long)nx * ny;
    cudaStream_t s = c->stream;
    double *dlon = nullptr, *dlat = nullptr;
    unsigned *k0 = nullptr, *k1 = nullptr;
    int *v0 = nullptr, *v1 = nullptr, *cnt = nullptr, *off = nullptr;
    void* tmp = nullptr;
    size_t tsort = 0, tscan = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; return e == cudaSuccess; };
    ok(cudaMallocAsync((void**)&dlon, N * 8, s));
    ok(cudaMallocAsync((void**)&dlat, N * 8, s));
    ok(cudaMallocAsync((void**)&k0, N * 4, s));
    ok(cudaMallocAsync((void**)&k1, N * 4, s));
    ok(cudaMallocAsync((void**)&v0, N * 4, s));
    ok(cudaMallocAsync((void**)&v1, N * 4, s));
    ok(cudaMallocAsync((void**)&cnt, (C + 1) * 4, s));
    ok(cudaMallocAsync((void**)&off, (C + 1) * 4, s));
    ok(cudaMemcpyAsync(dlon, lon, N * 8, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(dlat, lat, N * 8, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(cnt, 0, (C + 1) * 4, s));
    if (e == cudaSuccess) {
        k_hash_cells<<<grid_for(N), kBlock, 0, s>>>(dlon, dlat, N, cell_size, lon_min, lat_min, nx, ny, wrap, k0, v0,
                                                    cnt);
        ok(cudaGetLastError());
    }
    // stable radix sort of the node ids by cell (the order of numpy's stable argsort)
    int bits = 1;
    while (bits < 32 && (1ull << bits) < (unsigned long long)C) ++bits;
    ok(cub::DeviceRadixSort::SortPairs(nullptr, tsort, k0, k1, v0, v1, (int)N, 0, bits, s));
    ok(cub::DeviceScan::ExclusiveSum(nullptr, tscan, cnt, off, (int)(C + 1), s));
    ok(cudaMallocAsync(&tmp, std::max(tsort, tscan), s));
    ok(cub::DeviceRadixSort::SortPairs(tmp, tsort, k0, k1, v0, v1, (int)N, 0, bits, s));
    ok(cub::DeviceScan::ExclusiveSum(tmp, tscan, cnt, off, (int)(C + 1), s));   // offsets[C] = N
    ok(cudaMemcpyAsync(node_ids, v1, N * 4, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(offsets, off, (C + 1) * 4, cudaMemcpyDeviceToHost, s));
    for (void* p : {(void*)dlon, (void*)dlat, (void*)k0, (void*)k1, (void*)v0, (void*)v1, (void*)cnt, (void*)off, tmp})
        if (p) cudaFreeAsync(p, s);
    if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("kc_grid_hash_build: ") + cudaGetErrorString(e));
    KC_CUDA(c, cudaStreamSynchronize(s));
    return KC_OK;
}

int kc_grid_cell_stats(kc_ctx* c, long long n_nodes, const double* lon_branch, double cell_size, double lon_min,
                       double lat_min, int nx, int ny, int wrap, long long P, const double* lon, const double* lat,
                       int* nn, int* occ, double* cost, signed char* unprov, signed char* approx) {
    if (!c) return KC_ERR_ARG;
    if (!c->has_mesh) return fail(c, KC_ERR_STATE, "kc_grid_cell_stats: no mesh uploaded");
    if (n_nodes != c->N || !lon_branch) return fail(c, KC_ERR_ARG, "kc_grid_cell_stats: node longitudes");
    if (!(cell_size > 0.0) || nx <= 0 || ny <= 0 || (long long)nx * ny > 2000000000LL)
        return fail(c, KC_ERR_ARG, "kc_grid_cell_stats: grid geometry");
    if (P < 0 || (P > 0 && (!lon || !lat || !nn || !occ || !cost || !unprov || !approx)))
        return fail(c, KC_ERR_ARG, "kc_grid_cell_stats: sample arrays");
    if (P == 0) return KC_OK;
    KC_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const long long N = n_nodes, T = (long long)(nx + 1) * (ny + 1);
    double *dlon = nullptr, *dq = nullptr, *dcost = nullptr;
    int *cum = nullptr, *dnn = nullptr, *docc = nullptr;
    signed char *dun = nullptr, *dap = nullptr;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; return e == cudaSuccess; };
    ok(cudaMallocAsync((void**)&dlon, N * 8, s));
    ok(cudaMallocAsync((void**)&cum, T * 4, s));
    ok(cudaMallocAsync((void**)&dq, P * 16, s));
    ok(cudaMallocAsync((void**)&dnn, P * 4, s));
    ok(cudaMallocAsync((void**)&docc, P * 4, s));
    ok(cudaMallocAsync((void**)&dcost, P * 8, s));
    ok(cudaMallocAsync((void**)&dun, P, s));
    ok(cudaMallocAsync((void**)&dap, P, s));
    ok(cudaMemcpyAsync(dlon, lon_branch, N * 8, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(dq, lon, P * 8, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(dq + P, lat, P * 8, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(cum, 0, T * 4, s));
    if (e == cudaSuccess) {
        k_cell_counts<<<grid_for(N), kBlock, 0, s>>>(dlon, c->dm.ll, N, cell_size, lon_min, lat_min, nx, ny, wrap, cum);
        ok(cudaGetLastError());
    }
    if (e == cudaSuccess) {
        k_prefix_rows<<<(unsigned)ny, kScanBlock, 0, s>>>(cum, nx);
        ok(cudaGetLastError());
    }
    if (e == cudaSuccess) {
        k_prefix_cols<<<grid_for(nx), kBlock, 0, s>>>(cum, nx, ny);
        ok(cudaGetLastError());
    }
    if (e == cudaSuccess) {
        kc::DMesh mr = c->dm, mc = c->dm;
        mc.cell = cell_size; mc.lon_min = lon_min; mc.lat_min = lat_min; mc.nx = nx; mc.ny = ny; mc.wrap = wrap ? 1 : 0;
        k_cell_stats<<<grid_for(P), kBlock, 0, s>>>(mr, mc, cum, dq, P, dnn, docc, dcost, dun, dap);
        ok(cudaGetLastError());
    }
    ok(cudaMemcpyAsync(nn, dnn, P * 4, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(occ, docc, P * 4, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(cost, dcost, P * 8, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(unprov, dun, P, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(approx, dap, P, cudaMemcpyDeviceToHost, s));
    for (void* p : {(void*)dlon, (void*)cum, (void*)dq, (void*)dnn, (void*)docc, (void*)dcost, (void*)dun, (void*)dap})
        if (p) cudaFreeAsync(p, s);
    if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("kc_grid_cell_stats: ") + cudaGetErrorString(e));
    KC_CUDA(c, cudaStreamSynchronize(s));
    return KC_OK;
}

int kc_rng_domain_digests(kc_ctx* c, int corrected, unsigned long long* out) {
    if (!c || !out) return KC_ERR_ARG;
    if (corrected != 0 && corrected != 1) return fail(c, KC_ERR_ARG, "kc_rng_domain_digests: corrected is 0 or 1");
    KC_CUDA(c, cudaSetDevice(c->device));
    unsigned long long* d = nullptr;
    KC_CUDA(c, cudaMallocAsync((void**)&d, 3 * sizeof(unsigned long long), c->stream));
    cudaError_t e = cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), c->stream);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const kc::DRngX x = corrected ? c->dm.rx : kc::DRngX{nullptr, nullptr, nullptr, nullptr};
    if (e == cudaSuccess) {
        k_rng_domain<<<(unsigned)sms * 8, 256, 0, c->stream>>>(x, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    if (e != cudaSuccess) return fail(c, KC_ERR_CUDA, std::string("kc_rng_domain_digests: ") + cudaGetErrorString(e));
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    return KC_OK;
}

int kc_device_errors(kc_ctx* c, int* word) {
    if (!c || !word) return KC_ERR_ARG;
    KC_CUDA(c, cudaStreamSynchronize(c->stream));
    KC_CUDA(c, cudaMemcpy(word, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    KC_CUDA(c, cudaMemset(c->d_err, 0, sizeof(int)));
    return KC_OK;
}

int kc_event_record(kc_ctx* c, int slot) {
    if (!c || slot < 0 || slot >= kEvents) return KC_ERR_ARG;
    KC_CUDA(c, cudaEventRecord(c->ev[slot], c->stream));
    return KC_OK;
}

int kc_event_elapsed(kc_ctx* c, int a, int b, float* ms) {
    if (!c || !ms || a < 0 || b < 0 || a >= kEvents || b >= kEvents) return KC_ERR_ARG;
    KC_CUDA(c, cudaEventSynchronize(c->ev[b]));
    KC_CUDA(c, cudaEventElapsedTime(ms, c->ev[a], c->ev[b]));
    return KC_OK;
}

int kc_l2_flush(kc_ctx* c, long long bytes) {
    if (!c || bytes <= 0) return KC_ERR_ARG;
    KC_CUDA(c, cudaSetDevice(c->device));
    if (bytes > c->flush_cap) {
        KC_CUDA(c, cudaStreamSynchronize(c->stream));
        dfree(c->flush);
        KC_CUDA(c, cudaMalloc((void**)&c->flush, (size_t)bytes));
        c->flush_cap = bytes;
    }
    KC_CUDA(c, cudaMemsetAsync(c->flush, (int)(++c->flush_val & 0xff), (size_t)bytes, c->stream));
    return KC_OK;
}

int kc_host_alloc(long long bytes, void** out) {
    if (!out || bytes < 0) return KC_ERR_ARG;
    return cudaMallocHost(out, (size_t)std::max<long long>(bytes, 1)) == cudaSuccess ? KC_OK : KC_ERR_CUDA;
}

int kc_host_free(void* p) {
    if (!p) return KC_OK;
    return cudaFreeHost(p) == cudaSuccess ? KC_OK : KC_ERR_CUDA;
}

}  // extern "C"
