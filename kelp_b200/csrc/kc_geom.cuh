// Device-side geometry of the KELP time-stepping path: Python-semantics
// modulo, grid-hash cell lookup, exact nearest-node search with its
// certificate, element containment and vertex weights.
//
// Every routine restates a KELP Numba function (file:line in its comment)
// with the same floating-point operation order.  This translation unit is
// compiled with -fmad=false: Numba emits no fused multiply-adds, so a
// contracted a*b+c here would round differently and could flip an anchor or
// a containment verdict.
//
// Trigonometric values that depend only on the mesh (sin/cos of a node's
// latitude, cos of an element's mean latitude) come from tables evaluated on
// the host with the C library -- the functions the reference's Numba code
// calls -- so they carry the reference's exact values.  Values that depend on
// a particle position are evaluated once per evaluation site with CUDA's
// double-precision functions and shared by every consumer at that site.
#pragma once
#include "kc_crmath.cuh"

// Inlining of the shared helpers of the step kernels (build options, -D):
// __noinline__ keeps a kernel's code footprint small under divergence;
// __forceinline__ lets the register allocator see across the call, without
// the saves and restores of the call boundary.
#ifndef KC_INL_SITE
#define KC_INL_SITE __noinline__          // make_site
#endif
#ifndef KC_INL_NEAREST
#define KC_INL_NEAREST __noinline__       // nearest_exact
#endif
#ifndef KC_INL_CONTAIN
#define KC_INL_CONTAIN __noinline__       // contain_local, contain_local_w, w_search_elem
#endif
#ifndef KC_INL_STAGE
#define KC_INL_STAGE __noinline__         // interp_uv_at, w_bary_at (plain form)
#endif
#ifndef KC_INL_KICK
#define KC_INL_KICK __noinline__          // apply_kick
#endif
#include <cstdint>
#include <cuda_runtime.h>

namespace kc {

constexpr double DEG2RAD = 0.017453292519943295;   // pi / 180
constexpr double RAD2DEG = 57.29577951308232;      // 180 / pi
constexpr double SLM = 111120.0;                   // metres per degree of latitude
constexpr double R_STD = 6371000.0;                // standard Earth radius
constexpr double BARY_EPS = -1e-6;                 // mesh.py:33
constexpr double AREA_TOL = 1e-10;                 // mesh.py:32
constexpr int SHORT_ROW_CELLS = 32;                // mesh.py:1608
constexpr int ALIVE = 1, BEACHED = 2, OUTSIDE = 3, NOT_RELEASED = 4;
constexpr int FR_INTERP = 1, FR_OOB = 2;

// device error word bits (read back by the host)
constexpr int ERR_SEARCH_CAP = 1;   // exact-search growth loop hit its cap
constexpr int ERR_BAD_ANCHOR = 2;   // a particle's nearest_node is outside [-N, N)

// The NEMO C-grid tables of a mesh built by readers/nemo/_mesh.py
// build_nemo_cgrid_mesh (nodes = F-points, elements = T-cells), or on = 0.
struct DCgrid {
    const int4* corners;      // (E) F-point corners SW, SE, NE, NW
    const int* cell;          // (E) flat T index j * nx + i (j, i >= 1)
    const int* nlev;          // (E) wet levels, 0 for the dry ring
    const int* nlev_r;        // (ny * nx) wet levels per column
    const double4* L;         // (E) plane edge lengths S, E, N, W (host C library) when has_e is 0
    const double* e2u;        // (ny * nx) model u-face widths (has_e)
    const double* e1v;        // (ny * nx) model v-face widths (has_e)
    const double* area;       // (ny * nx) T-cell areas (3-D)
    const double* zw;         // (K + 1) reference interfaces (3-D)
    const double* e3b;        // (ny * nx) bottom wet cell thickness (3-D)
    const int* kbu;           // (ny * nx) partial level of each u face, -1 none (3-D)
    const double* e3u;
    const int* kbv;
    const double* e3v;
    long long nynx;
    int nx, K, shrunk, has_e, on;
};

// Resident mesh: node table, element table, node->element CSR, grid hash and
// the host-evaluated trigonometric tables.
// Box-Muller exception tables (built from the whole-domain scan of
// gen_rng_exceptions.cpp): the uniforms' 32-bit indices j at which the host
// C library's r = sqrt(-2 log u1) (table a) or cos / sin (2 pi u2) (table b)
// differ from the correctly rounded values, bucketed by j >> 12:
// off[b] .. off[b+1] index 16-bit entries (j & 0xfff) << 4 | code,
// ascending.  Null pointers: the correctly rounded draws.
struct DRngX {
    const unsigned* a_off;
    const unsigned short* a;
    const unsigned* b_off;
    const unsigned short* b;
};

struct DMesh {
    const double2* ll;        // (N) node lon, lat in degrees
    const double2* nsc;       // (N) sin, cos of the node latitude (radians)
    const int4* en;           // (E) element nodes, -1 padded to 4
    const double2* ecos;      // (E) cos(mean vertex latitude): x containment set, y compacted set
    const int* n2e_off;       // (N+1) CSR offsets of the node->element table
    const int* n2e;           // element ids, per node in the reference order
    const float4* ebox;       // (E) containment prefilter boxes (elem_box), or null
    const double2* erec;      // (E, 4) mask vertex lon, lat per element (elem_record), or null
    const int* gh_off;        // (nx*ny+1) CSR offsets of the grid hash
    const double4* gh_tab;    // hash-ordered {x, y, z, node id} unit-sphere table
    const int* pw_off;        // (nx*ny+1) pruned windows: CSR offsets, or null
    const double4* pw_tab;    // each cell's pruned window: gh_tab records in window scan order
    const double2* ec;        // (E) element centre lon, lat (element-layout u/v), or null
    const double* xyz;        // (N, 3) unit-sphere table by node id
    const double* depth;      // (N) bottom depth, positive down (3-D)
    const int* max_layer;     // (N) deepest valid layer above the node's bottom (3-D)
    const double* zlev;       // (K) z-level interfaces, positive down (3-D)
    const double* dl_p;       // (M) depth-linear data points (uv_vertical level / layer_linear)
    const int* dl_last;       // (N) last usable data point per node
    const double* dl_bed;     // (N) bed depth per node for the wall test
    const int4* enb;          // (E) edge neighbours of the compacted ring (edge walk), or null
    const double* sigma;      // (K) sigma interfaces, 1 surface -> 0 bed (sigma meshes), or null
    int sig;                  // 1: sigma mesh (K counts its interfaces, zlev is null)
    DCgrid cg;                // NEMO C-grid tables (cg.on)
    long long E;
    double cell, lon_min, lat_min, r_earth;
    int nx, ny, wrap, far_rows, K, exact, dl_M;
    int* err;                 // device error word
    DRngX rx;                 // the RNG's exception tables (set by kc_create)
};

// Trigonometry of one evaluation site (a query position).
struct Site {
    double lon, lat;
    double xp, yp, zp;        // unit-sphere position
    double sin_lat, cos_lat;  // of lat * DEG2RAD
    double sin_lon, cos_lon;  // of lon * DEG2RAD
};

static __device__ KC_INL_SITE Site make_site(double lon, double lat) {
    Site s;
    s.lon = lon;
    s.lat = lat;
    cr::sincos_cr(lat * DEG2RAD, &s.sin_lat, &s.cos_lat);   // correctly rounded: the C library's values but
    cr::sincos_cr(lon * DEG2RAD, &s.sin_lon, &s.cos_lon);   // where it misrounds (kc_crmath.cuh)
    s.xp = s.cos_lat * s.cos_lon;
    s.yp = s.cos_lat * s.sin_lon;
    s.zp = s.sin_lat;
    return s;
}

// The same site with CUDA's sincos (within 2 ulp): the mixed form's sites,
// where last-place agreement with the C library is not the contract.
static __device__ KC_INL_SITE Site make_site_fast(double lon, double lat) {
    Site s;
    s.lon = lon;
    s.lat = lat;
    sincos(lat * DEG2RAD, &s.sin_lat, &s.cos_lat);
    sincos(lon * DEG2RAD, &s.sin_lon, &s.cos_lon);
    s.xp = s.cos_lat * s.cos_lon;
    s.yp = s.cos_lat * s.sin_lon;
    s.zp = s.sin_lat;
    return s;
}

// fmod(x, 360) for |x| < 2^40 * 360 without the general remainder loop:
// with n the integer part of |x| / 360 (corrected by one when the division
// rounded across an integer), |x| - n * 360 is exact (n * 360 is exact, and
// for n >= 1 Sterbenz's lemma applies: n*360/2 <= |x| <= 2 n*360), so the
// result equals C fmod bit for bit; larger or non-finite x take fmod itself.
static __device__ __noinline__ double fmod360_slow(double x) { return fmod(x, 360.0); }

__device__ __forceinline__ double fmod360(double x) {
    double a = fabs(x);
    if (!(a < 395824185999360.0)) return fmod360_slow(x);    // 2^40 * 360, and NaN
    double n = trunc(a * (1.0 / 360.0));
    double r = a - n * 360.0;
    if (r < 0.0) r = a - (n - 1.0) * 360.0;
    else if (r >= 360.0) r = a - (n + 1.0) * 360.0;
    return copysign(r, x);
}

// Python float modulo by 360 (CPython float_rem, Numba real_divmod): the
// remainder carries the divisor's sign, zero is +0.
__device__ __forceinline__ double pymod360(double x) {
    double r = fmod360(x);
    if (r != 0.0) {
        if (r < 0.0) r += 360.0;
    } else {
        r = 0.0;
    }
    return r;
}

// ((x + 180) % 360) - 180.  For 0 <= x + 180 < 360 the remainder is x + 180
// itself, so the common case is the two roundings alone.
__device__ __forceinline__ double wrap180(double x) {
    const double y = x + 180.0;
    if (y >= 0.0 && y < 360.0) return y - 180.0;
    return pymod360(y) - 180.0;
}

// Python integer modulo for a positive divisor.
__device__ __forceinline__ int imod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// mesh.py:1192-1207 _gh_fold_dlon
__device__ __forceinline__ double gh_fold_dlon(const DMesh& m, double lon_p) {
    double dlon = pymod360(lon_p - m.lon_min);
    if (!m.wrap) {
        double grid_span = (double)m.nx * m.cell;
        if (dlon > grid_span && (dlon - grid_span) > (360.0 - dlon)) dlon -= 360.0;
    }
    return dlon;
}

// mesh.py:1210-1232 _gh_cell_of (int() truncates toward zero)
__device__ __forceinline__ void gh_cell_of(const DMesh& m, double lon_p, double lat_p, int& ci, int& cj) {
    double dlon = gh_fold_dlon(m, lon_p);
    ci = (int)(dlon / m.cell);
    cj = (int)((lat_p - m.lat_min) / m.cell);
    if (ci < 0) ci = 0;
    if (ci >= m.nx) ci = m.nx - 1;
    if (cj < 0) cj = 0;
    if (cj >= m.ny) cj = m.ny - 1;
}

// Scan hash-table positions [s, e): strict '<' keeps the first node found
// on a tie, which makes the CSR order part of the contract (mesh.py:1290-1301).
__device__ __forceinline__ void scan_range(const double4* __restrict__ tab, int s, int e,
                                           double xp, double yp, double zp, int& best, double& bd2) {
    for (int k = s; k < e; ++k) {
        const double2* p = reinterpret_cast<const double2*>(tab + k);
        double2 t0 = __ldg(p), t1 = __ldg(p + 1);
        double dx = t0.x - xp, dy = t0.y - yp, dz = t1.x - zp;
        double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < bd2) { bd2 = d2; best = (int)t1.y; }
    }
}

__device__ __forceinline__ void scan_cell(const DMesh& m, int cell, double xp, double yp, double zp, int& best,
                                          double& bd2) {
    scan_range(m.gh_tab, __ldg(&m.gh_off[cell]), __ldg(&m.gh_off[cell + 1]), xp, yp, zp, best, bd2);
}

// mesh.py:1235-1303 _grid_hash_nearest_3x3.  Adjacent columns of one row are
// adjacent in the CSR, so an unclipped, unwrapped row is one contiguous slice
// (same nodes, same order as three cell scans).
//
// A query whose cell needs no clamping scans the cell's pruned window instead
// (built by k_prune_windows at mesh upload): the window's records in the same
// scan order minus those that another window node is provably closer to at
// every point of the cell, so the first minimum and its distance are the
// window's own.  The records are copies, one contiguous slice per cell.
__device__ __forceinline__ int nearest_3x3(const DMesh& m, const Site& q, double& bd2_out) {
    int best = -1;
    double bd2 = 1e30;
    if (m.pw_off) {
        const double dlon = gh_fold_dlon(m, q.lon), dlat = q.lat - m.lat_min;
        if (dlon >= 0.0 && dlat >= 0.0) {
            const int ti = (int)(dlon / m.cell), tj = (int)(dlat / m.cell);
            if (ti < m.nx && tj < m.ny) {
                const int cell = tj * m.nx + ti;
                scan_range(m.pw_tab, __ldg(&m.pw_off[cell]), __ldg(&m.pw_off[cell + 1]), q.xp, q.yp, q.zp, best,
                           bd2);
                bd2_out = bd2;
                return best;
            }
        }
    }
    int ci, cj;
    gh_cell_of(m, q.lon, q.lat, ci, cj);
    for (int dj = -1; dj <= 1; ++dj) {
        int cj2 = cj + dj;
        if (cj2 < 0 || cj2 >= m.ny) continue;
        int row = cj2 * m.nx;
        if (ci >= 1 && ci + 1 < m.nx) {
            scan_range(m.gh_tab, __ldg(&m.gh_off[row + ci - 1]), __ldg(&m.gh_off[row + ci + 2]), q.xp, q.yp, q.zp,
                       best, bd2);
        } else {
            for (int di = -1; di <= 1; ++di) {
                int ci2 = ci + di;
                if (ci2 < 0) ci2 = m.wrap ? ci2 + m.nx : -1;
                else if (ci2 >= m.nx) ci2 = m.wrap ? ci2 - m.nx : -1;
                if (ci2 < 0) continue;
                scan_cell(m, row + ci2, q.xp, q.yp, q.zp, best, bd2);
            }
        }
    }
    bd2_out = bd2;
    return best;
}

// mesh.py:1306-1328 _cap_extents -> (theta_deg, ext_lon_deg); the node's
// sin/cos(latitude) from the host table, the query's from the site.
__device__ __forceinline__ void cap_extents(const DMesh& m, const Site& q, int node, double& theta_deg, double& ext) {
    double2 nl = __ldg(&m.ll[node]);
    double2 sc = __ldg(&m.nsc[node]);
    double cosd = q.sin_lat * sc.x + q.cos_lat * sc.y * cos((q.lon - nl.x) * DEG2RAD);
    if (cosd > 1.0) cosd = 1.0;
    if (cosd < -1.0) cosd = -1.0;
    double theta = acos(cosd);
    if (theta <= 0.0) { theta_deg = 0.0; ext = 0.0; return; }
    theta_deg = theta * RAD2DEG;
    if (fabs(q.lat) + theta_deg >= 90.0) { ext = 1.0e30; return; }
    double r = sin(theta) / q.cos_lat;
    if (r >= 1.0) { ext = 1.0e30; return; }
    ext = asin(r) * RAD2DEG;
}

// The coverage tests of mesh.py:1475-1549 _anchor_provable_rect for given
// (theta_deg, ext_lon).  Every test is monotone in both, so upper bounds that
// pass prove that the reference's own values pass.
__device__ __forceinline__ int provable_code(const DMesh& m, const Site& q, int rx, int ry, double theta_deg,
                                             double ext_lon) {
    if (theta_deg <= 0.0) return 0;
    const double lon_p = q.lon, lat_p = q.lat;
    double dlon = gh_fold_dlon(m, lon_p);
    double lon_q = m.lon_min + dlon;
    int ci_raw = (int)floor(dlon / m.cell);
    int cj_raw = (int)floor((lat_p - m.lat_min) / m.cell);
    const double INF = 1.0e30;
    int cj = cj_raw;
    if (cj < 0) cj = 0;
    if (cj > m.ny - 1) cj = m.ny - 1;
    double cov_dn = (cj - ry >= 0) ? lat_p - (m.lat_min + (double)(cj - ry) * m.cell) : INF;
    double cov_up = (cj + ry <= m.ny - 1) ? (m.lat_min + (double)(cj + ry + 1) * m.cell) - lat_p : INF;
    int code = 0;
    if (theta_deg > cov_dn || theta_deg > cov_up) code |= 1;
    if (m.wrap) {
        if (2 * rx + 1 >= m.nx) return code;
        if (ext_lon >= INF) return code | 4;
        double w_last = 360.0 - (double)(m.nx - 1) * m.cell;
        int ci = imod(ci_raw, m.nx);
        double left = m.lon_min + (double)(ci - rx) * m.cell;
        if (ci - rx < 0) left += m.cell - w_last;
        double right = m.lon_min + (double)(ci + rx + 1) * m.cell;
        if (ci + rx >= m.nx - 1) right -= m.cell - w_last;
        if (ext_lon > lon_q - left || ext_lon > right - lon_q) code |= 2;
        return code;
    }
    int ci = ci_raw;
    if (ci < 0) ci = 0;
    if (ci > m.nx - 1) ci = m.nx - 1;
    double cov_l = (ci - rx >= 0) ? lon_q - (m.lon_min + (double)(ci - rx) * m.cell) : INF;
    double cov_r = (ci + rx <= m.nx - 1) ? (m.lon_min + (double)(ci + rx + 1) * m.cell) - lon_q : INF;
    if (cov_l >= INF && cov_r >= INF) return code;
    if (ext_lon >= INF) return code | 4;
    if (ext_lon > cov_l || ext_lon > cov_r) code |= 2;
    double n_lo = m.lon_min + m.cell;
    double n_hi = m.lon_min + (double)(m.nx - 1) * m.cell;
    for (int s = 0; s < 2; ++s) {
        double shift = s == 0 ? -360.0 : 360.0;
        double a = lon_q - ext_lon + shift;
        double b = lon_q + ext_lon + shift;
        if (b >= n_lo && a <= n_hi) return code | 4;
    }
    return code;
}

// mesh.py:1475-1549 _anchor_provable_rect with the reference's own extents.
static __device__ __noinline__ int anchor_provable_rect(const DMesh& m, const Site& q, int node, int rx, int ry) {
    double theta_deg, ext_lon;
    cap_extents(m, q, node, theta_deg, ext_lon);
    return provable_code(m, q, rx, ry, theta_deg, ext_lon);
}

// Fast sufficient test of the 3x3 certificate.  Upper bounds of the cap's
// angular radius -- from the scan's chord c: 2 asin(c/2) <= c (1 + c^2/16)
// for c <= 1, plus 1e-7 rad for the rounding of the reference's acos form --
// and of its longitude extent (sin t <= t; asin(r) <= r (1 + 0.2 r^2) for
// r <= 0.5).  True only when the bounds pass every coverage test, so the
// reference's certificate passes too; otherwise the caller evaluates it.
__device__ __forceinline__ bool provable_fast(const DMesh& m, const Site& q, double bd2) {
    double c = sqrt(bd2);
    if (!(c <= 0.5)) return false;
    double t = c * (1.0 + c * c * 0.0625) * (1.0 + 1e-12) + 1e-7;
    double tdeg = t * RAD2DEG * (1.0 + 1e-12);
    if (fabs(q.lat) + tdeg >= 89.0) return false;
    double r = t / q.cos_lat * (1.0 + 1e-12);
    if (!(r <= 0.5)) return false;
    double edeg = r * (1.0 + 0.2 * r * r) * RAD2DEG * (1.0 + 1e-12);
    return provable_code(m, q, 1, 1, tdeg, edeg) == 0;
}

// mesh.py:1331-1442 _grid_hash_nearest_widened: the 3x3 window, and on an
// empty window a ring-by-ring scan that stops one ring after the first hit.
static __device__ __noinline__ int nearest_widened(const DMesh& m, const Site& q) {
    double bd2;
    int best = nearest_3x3(m, q, bd2);
    if (best >= 0) return best;
    int ci, cj;
    gh_cell_of(m, q.lon, q.lat, ci, cj);
    bd2 = 1e30;
    int max_ring = m.nx > m.ny ? m.nx : m.ny;
    int found_ring = -1;
    for (int r = 2; r <= max_ring; ++r) {
        for (int dj = -r; dj <= r; ++dj) {
            int cj2 = cj + dj;
            if (cj2 < 0 || cj2 >= m.ny) continue;
            int di_step = (dj == -r || dj == r) ? 1 : 2 * r;
            for (int di = -r; di <= r; di += di_step) {
                int ci2 = ci + di;
                if (m.wrap) ci2 = imod(ci2, m.nx);
                else if (ci2 < 0 || ci2 >= m.nx) continue;
                scan_cell(m, cj2 * m.nx + ci2, q.xp, q.yp, q.zp, best, bd2);
            }
        }
        if (best >= 0) {
            if (found_ring < 0) found_ring = r;
            else if (r > found_ring) break;
        }
    }
    return best;
}

// mesh.py:1552-1605 row slices
__device__ __forceinline__ void scan_row_range(const DMesh& m, int cj2, int c_lo, int c_hi,
                                               double xp, double yp, double zp, int& best, double& bd2) {
    scan_range(m.gh_tab, __ldg(&m.gh_off[cj2 * m.nx + c_lo]), __ldg(&m.gh_off[cj2 * m.nx + c_hi + 1]), xp, yp, zp,
               best, bd2);
}

__device__ __forceinline__ void scan_row_window(const DMesh& m, int cj2, int ci, int rx,
                                                double xp, double yp, double zp, int& best, double& bd2) {
    if (m.wrap && 2 * rx + 1 >= m.nx) { scan_row_range(m, cj2, 0, m.nx - 1, xp, yp, zp, best, bd2); return; }
    int c_lo = ci - rx, c_hi = ci + rx;
    if (m.wrap) {
        if (c_lo < 0) {
            scan_row_range(m, cj2, c_lo + m.nx, m.nx - 1, xp, yp, zp, best, bd2);
            c_lo = 0;
        } else if (c_hi > m.nx - 1) {
            scan_row_range(m, cj2, 0, c_hi - m.nx, xp, yp, zp, best, bd2);
            c_hi = m.nx - 1;
        }
    } else {
        if (c_lo < 0) c_lo = 0;
        if (c_hi > m.nx - 1) c_hi = m.nx - 1;
    }
    scan_row_range(m, cj2, c_lo, c_hi, xp, yp, zp, best, bd2);
}

// The certificate-driven rectangle growth of mesh.py:1670-1859, entered when
// the 3x3 hit is not provable (or the window is empty).
static __device__ __noinline__ int nearest_exact_slow(const DMesh& m, const Site& q, int best, int code) {
    const double far = (double)m.far_rows * m.cell;
    const double lat_p = q.lat;
    if (best >= 0) {
        double theta_deg, ext;
        cap_extents(m, q, best, theta_deg, ext);
        if (theta_deg > far) return best;
    }
    int ci, cj;
    gh_cell_of(m, q.lon, q.lat, ci, cj);
    const double xp = q.xp, yp = q.yp, zp = q.zp, cos_lat_p = q.cos_lat;
    double best_d2 = 1.0e30;
    if (best >= 0) {
        double xn = m.xyz[3 * (long long)best], yn = m.xyz[3 * (long long)best + 1];
        double zn = m.xyz[3 * (long long)best + 2];
        double dx = xn - xp, dy = yn - yp, dz = zn - zp;
        best_d2 = dx * dx + dy * dy + dz * dz;
    }
    int rx = 1, ry = 1;
    bool short_row = 360.0 * cos_lat_p <= (double)SHORT_ROW_CELLS * m.cell;
    int rx_max;
    if (m.wrap) {
        rx_max = m.nx / 2;
        if (rx_max < 1) rx_max = 1;
    } else {
        rx_max = ci > m.nx - 1 - ci ? ci : m.nx - 1 - ci;
    }
    int ry_max = cj > m.ny - 1 - cj ? cj : m.ny - 1 - cj;
    double abs_lat = lat_p >= 0.0 ? lat_p : -lat_p;
    double dlon_q = gh_fold_dlon(m, q.lon);
    const double INF = 1.0e30;
    // each pass grows rx or ry by at least one, or returns
    const int cap = 4 * (m.nx + m.ny) + 16;
    for (int it = 0; it < cap; ++it) {
        if (best >= 0 && code == 0) {
            code = anchor_provable_rect(m, q, best, rx, ry);
            if (code == 0) return best;
        }
        if (best < 0 || 2.0 * asin(0.5 * sqrt(best_d2)) * RAD2DEG > far) {
            bool cols_full;
            if (m.wrap) cols_full = 2 * rx + 1 >= m.nx;
            else cols_full = ci - rx <= 0 && ci + rx >= m.nx - 1;
            double clear = ry >= ry_max ? INF : (double)ry * m.cell;
            if (!cols_full) {
                double lat_edge = abs_lat + (double)(ry + 1) * m.cell;
                double clear_lon;
                if (lat_edge >= 90.0) {
                    clear_lon = 0.0;
                } else {
                    double dl = (double)rx * m.cell;
                    if (!m.wrap) {
                        double x = dlon_q > 0.0 ? dlon_q : 0.0;
                        double w = (double)m.nx * m.cell;
                        if (x > w) x = w;
                        double near_edge = x < w - x ? x : w - x;
                        double dl_cut = 360.0 - w + near_edge;
                        if (dl_cut < dl) dl = dl_cut;
                    }
                    if (dl > 180.0) dl = 180.0;
                    clear_lon = asin(sin(dl * DEG2RAD) * cos(lat_edge * DEG2RAD)) * RAD2DEG;
                }
                if (clear_lon < clear) clear = clear_lon;
            }
            if (clear >= far) {
                if (best >= 0) return best;
                return nearest_widened(m, q);
            }
        }
        bool grow_x, grow_y, all_x;
        if (best >= 0) {
            grow_x = (code & 2) != 0;
            grow_y = (code & 1) != 0;
            all_x = (code & 4) != 0;
            code = 0;
        } else if (short_row) {
            grow_x = false; grow_y = true; all_x = true;
        } else {
            grow_x = true; grow_y = true; all_x = false;
        }
        if (rx >= rx_max) { grow_x = false; all_x = false; }
        if (ry >= ry_max) grow_y = false;
        if (!(grow_x || grow_y || all_x)) {
            if (best >= 0) return best;
            return nearest_widened(m, q);
        }
        int rx_new = all_x ? rx_max : (grow_x ? rx + 1 : rx);
        int ry_new = grow_y ? ry + 1 : ry;
        int j_lo = cj - ry > 0 ? cj - ry : 0;
        int j_hi = cj + ry < m.ny - 1 ? cj + ry : m.ny - 1;
        if (rx_new > rx) {
            if (m.wrap && 2 * rx_new + 1 >= m.nx && rx_new - rx > 1) {
                for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                    int c_lo = imod(ci + rx + 1, m.nx);
                    int c_hi = imod(ci - rx - 1, m.nx);
                    if (c_lo <= c_hi) {
                        scan_row_range(m, cj2, c_lo, c_hi, xp, yp, zp, best, best_d2);
                    } else {
                        scan_row_range(m, cj2, c_lo, m.nx - 1, xp, yp, zp, best, best_d2);
                        scan_row_range(m, cj2, 0, c_hi, xp, yp, zp, best, best_d2);
                    }
                }
            } else if (!m.wrap && rx_new - rx > 1) {
                for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                    if (ci - rx - 1 >= 0) {
                        int c_lo = ci - rx_new > 0 ? ci - rx_new : 0;
                        scan_row_range(m, cj2, c_lo, ci - rx - 1, xp, yp, zp, best, best_d2);
                    }
                    if (ci + rx + 1 <= m.nx - 1) {
                        int c_hi = ci + rx_new < m.nx - 1 ? ci + rx_new : m.nx - 1;
                        scan_row_range(m, cj2, ci + rx + 1, c_hi, xp, yp, zp, best, best_d2);
                    }
                }
            } else {
                for (int r = rx + 1; r <= rx_new; ++r) {
                    if (m.wrap) {
                        int c_left = imod(ci - r, m.nx);
                        bool two = 2 * r + 1 <= m.nx;
                        int c_right = imod(ci + r, m.nx);
                        for (int cj2 = j_lo; cj2 <= j_hi; ++cj2) {
                            scan_cell(m, cj2 * m.nx + c_left, xp, yp, zp, best, best_d2);
                            if (two) scan_cell(m, cj2 * m.nx + c_right, xp, yp, zp, best, best_d2);
                        }
                    } else {
                        for (int side = 0; side < 2; ++side) {
                            int c2 = side == 0 ? ci - r : ci + r;
                            if (c2 < 0 || c2 > m.nx - 1) continue;
                            for (int cj2 = j_lo; cj2 <= j_hi; ++cj2)
                                scan_cell(m, cj2 * m.nx + c2, xp, yp, zp, best, best_d2);
                        }
                    }
                }
            }
        }
        for (int r = ry + 1; r <= ry_new; ++r) {
            for (int side = 0; side < 2; ++side) {
                int cj2 = side == 0 ? cj - r : cj + r;
                if (cj2 < 0 || cj2 > m.ny - 1) continue;
                scan_row_window(m, cj2, ci, rx_new, xp, yp, zp, best, best_d2);
            }
        }
        rx = rx_new;
        ry = ry_new;
    }
    atomicOr(m.err, ERR_SEARCH_CAP);
    return best;
}

// mesh.py:1611-1859 _grid_hash_nearest_exact: the 3x3 window accepted when
// the certificate proves it (fast bound first, the reference's own
// certificate when the bound is inconclusive), else the rectangle growth.
static __device__ KC_INL_NEAREST int nearest_exact(const DMesh& m, const Site& q) {
    const double far = (double)m.far_rows * m.cell;
    if (q.lat < m.lat_min - far || q.lat > m.lat_min + (double)m.ny * m.cell + far) return nearest_widened(m, q);
    double bd2;
    int best = nearest_3x3(m, q, bd2);
    int code = 0;
    if (best >= 0) {
        if (provable_fast(m, q, bd2)) return best;
        code = anchor_provable_rect(m, q, best, 1, 1);
        if (code == 0) return best;
    }
    return nearest_exact_slow(m, q, best, code);
}

// The anchor of one evaluation site (integrators.py:1470-1487).
// A finite position always has a nearest node; a non-finite one (a NaN
// velocity upstream) gets node 0, so every table read stays in bounds while
// its containment test fails.
__device__ __forceinline__ int site_anchor(const DMesh& m, const Site& q) {
    const int r = m.exact ? nearest_exact(m, q) : nearest_widened(m, q);
    return r >= 0 ? r : 0;
}

// ---------------------------------------------------------------------------
// Containment and weights
// ---------------------------------------------------------------------------

__device__ __forceinline__ int elem_node(const int4& e, int k) {
    return k == 0 ? e.x : (k == 1 ? e.y : (k == 2 ? e.z : e.w));
}

// mesh.py:2054-2073 _barycentric_weights_tri; false on a degenerate triangle
// (the reference's [-1, -1, -1] sentinel).
__device__ __forceinline__ bool bary_tri(double px, double py, double ax, double ay, double bx, double by,
                                         double cx, double cy, double& w1, double& w2, double& w3) {
    double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
    if (fabs(denom) < AREA_TOL) { w1 = w2 = w3 = -1.0; return false; }
    w1 = ((by - cy) * (px - cx) + (cx - bx) * (py - cy)) / denom;
    w2 = ((cy - ay) * (px - cx) + (ax - cx) * (py - cy)) / denom;
    w3 = 1.0 - w1 - w2;
    return true;
}

// The containment verdict of bary_tri (all three weights >= BARY_EPS)
// without its divisions where the numerators decide it.  With s the sign of
// the denominator, a_k = s num_k and d = |denom|, the exact weights are
// a_k / d (a_3 = d - a_1 - a_2).  All a_k >= 0 (a_3 within its rounding)
// puts every rounded weight above -1e-15 > BARY_EPS: inside.  One a_k below
// -1.1e-6 d by more than its rounding puts that rounded weight below
// BARY_EPS: outside.  Only the band between runs the division itself.  (a3
// is within 4.4e-16 (d + |a1| + |a2|) of d - a1 - a2, and the rounded w3
// within 6.6e-16 (d + |a1| + |a2|) / d of the exact third weight.)
__device__ __forceinline__ bool bary_tri_inside(double px, double py, double ax, double ay, double bx, double by,
                                                double cx, double cy, bool& nondeg) {
    const double denom = (by - cy) * (ax - cx) + (cx - bx) * (ay - cy);
    if (fabs(denom) < AREA_TOL) { nondeg = false; return -1.0 >= BARY_EPS; }
    nondeg = true;
    const double n1 = (by - cy) * (px - cx) + (cx - bx) * (py - cy);
    const double n2 = (cy - ay) * (px - cx) + (ax - cx) * (py - cy);
    const double d = fabs(denom);
    const double a1 = denom > 0.0 ? n1 : -n1, a2 = denom > 0.0 ? n2 : -n2;
    const double a3 = (d - a1) - a2;
    const double r3 = 2e-15 * (d + fabs(a1) + fabs(a2));   // above the rounding of a3 plus that of w3
    if (a1 >= 0.0 && a2 >= 0.0 && a3 >= r3) return true;
    const double lim = 1.1e-6 * d;
    if (a1 < -lim || a2 < -lim || a3 < -lim - r3) return false;
    const double w1 = n1 / denom, w2 = n2 / denom, w3 = 1.0 - w1 - w2;
    return w1 >= BARY_EPS && w2 >= BARY_EPS && w3 >= BARY_EPS;
}

// mesh.py:2076-2116 _wachspress_weights_quad (product form)
__device__ __forceinline__ void wachspress_quad(double px, double py, const double* x, const double* y, double* out) {
    double A[4], C[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int i1 = (k + 1) & 3, im = (k + 3) & 3;
        A[k] = (x[k] - px) * (y[i1] - py) - (x[i1] - px) * (y[k] - py);
        C[k] = (x[k] - x[im]) * (y[i1] - y[im]) - (x[i1] - x[im]) * (y[k] - y[im]);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double w = C[k] * A[(k + 1) & 3] * A[(k + 2) & 3];
        out[k] = w;
        s += w;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = out[k] / s;
}

// The vertices of an element in the containment (mask) convention of
// mesh.py:2216-2236: drop -1 slots, and slot 3 when it repeats slot 0.
struct Poly {
    double ln[4], la[4];
    int n;
};

__device__ __forceinline__ void put_vertex(Poly& p, int n, double2 a) {
    if (n == 0) { p.ln[0] = a.x; p.la[0] = a.y; }
    else if (n == 1) { p.ln[1] = a.x; p.la[1] = a.y; }
    else if (n == 2) { p.ln[2] = a.x; p.la[2] = a.y; }
    else { p.ln[3] = a.x; p.la[3] = a.y; }
}

__device__ __forceinline__ void load_poly_mask(const DMesh& m, int4 e, Poly& p) {
    bool v3 = e.w >= 0 && !(e.w == e.x && e.x >= 0);
    int n = 0;
    if (e.x >= 0) put_vertex(p, n++, __ldg(&m.ll[e.x]));
    if (e.y >= 0) put_vertex(p, n++, __ldg(&m.ll[e.y]));
    if (e.z >= 0) put_vertex(p, n++, __ldg(&m.ll[e.z]));
    if (v3) put_vertex(p, n++, __ldg(&m.ll[e.w]));
    p.n = n;
}

// Verdicts of element_contains_t for the barycentric W search of
// vertical.py:744-881, which tests the same fan triangles in the same frame
// but without the bounding-box prefilter and with a 1e-14 degenerate
// tolerance: W_OUT when that search rejects the element too, W_UNSURE when
// it might accept it (bbox-rejected within the tolerance band, a fan
// triangle with |denominator| in [1e-14, 1e-10), or an element whose W
// vertex ring differs from the containment vertex set).
constexpr int W_OUT = 0, W_UNSURE = 2;

__device__ __forceinline__ bool w_ring_matches_mask(const int4& e) {
    // the W ring drops every later vertex equal to the first valid one, the
    // mask only slot 3 repeating slot 0: they agree unless another slot
    // repeats the first valid vertex
    const int first = e.x >= 0 ? e.x : (e.y >= 0 ? e.y : e.z);
    if (first < 0) return true;
    if (e.x >= 0 && e.y == first) return false;
    if ((e.x >= 0 || e.y >= 0) && e.z == first) return false;
    if (e.x < 0 && e.w == first) return false;
    if (e.x >= 0 && e.w == first && e.w != e.x) return false;
    return true;
}

// The verdict for a point outside the reference's bounding box (the running
// bounds of the wrapped longitudes around the first vertex, dmin..dmax, and
// of the latitudes): 0, or with W_INFO the class of the W search, which has no
// bbox and rejects the element for sure only beyond the margin of
// w_ring_rejects (same bound, same frame).
template <bool W_INFO>
__device__ __forceinline__ int outside_box_verdict(int miss, double dmin, double dmax, double lamin, double lamax,
                                                   double dlon_p, double lat_p) {
    if (!W_INFO) return 0;
    if (miss || !(dmax - dmin < 90.0)) return W_UNSURE;
    const double my = 1e-5 * (lamax - lamin) + 1e-9, mx = 1e-5 * (dmax - dmin) + 1e-9;
    if (lat_p < lamin - my || lat_p > lamax + my || dlon_p < dmin - mx || dlon_p > dmax + mx) return W_OUT;
    return W_UNSURE;
}

// Inside the box: the local projection with the raw-mean origin unless the
// element spans > 180 deg, then the fan triangles.  p holds the n mask
// vertices (slot 3 repeats slot 0 for a triangle).
template <bool W_INFO>
__device__ __forceinline__ int inside_box_verdict(const DMesh& m, int c, const Poly& p, int n, int miss, double lon_p,
                                                  double lat_p) {
    const double lon_ref = p.ln[0];
    const double d1 = wrap180(p.ln[1] - lon_ref), d2 = wrap180(p.ln[2] - lon_ref);
    const double d3 = n == 4 ? wrap180(p.ln[3] - lon_ref) : 0.0;
    double lmin = fmin(fmin(p.ln[0], p.ln[1]), p.ln[2]), lmax = fmax(fmax(p.ln[0], p.ln[1]), p.ln[2]);
    if (n == 4) { lmin = fmin(lmin, p.ln[3]); lmax = fmax(lmax, p.ln[3]); }
    double lon0;
    if (lmax - lmin > 180.0) {
        double dsum = 0.0 + d1;        // 0 + wrap180(ln[0] - ln[0]) + d1 + d2 (+ d3)
        dsum += d2;
        if (n == 4) dsum += d3;
        lon0 = lon_ref + dsum / (double)n;
    } else {
        double s = p.ln[0] + p.ln[1];
        s += p.ln[2];
        if (n == 4) s += p.ln[3];
        lon0 = s / (double)n;
    }
    double sl = p.la[0] + p.la[1];
    sl += p.la[2];
    if (n == 4) sl += p.la[3];
    const double lat0 = sl / (double)n;
    const double cos_lat0 = __ldg(&m.ecos[c]).x;
    const double x0 = wrap180(p.ln[0] - lon0) * DEG2RAD * R_STD * cos_lat0;
    const double x1 = wrap180(p.ln[1] - lon0) * DEG2RAD * R_STD * cos_lat0;
    const double x2 = wrap180(p.ln[2] - lon0) * DEG2RAD * R_STD * cos_lat0;
    const double y0 = (p.la[0] - lat0) * DEG2RAD * R_STD;
    const double y1 = (p.la[1] - lat0) * DEG2RAD * R_STD;
    const double y2 = (p.la[2] - lat0) * DEG2RAD * R_STD;
    const double px = wrap180(lon_p - lon0) * DEG2RAD * R_STD * cos_lat0;
    const double py = (lat_p - lat0) * DEG2RAD * R_STD;
    bool nondeg;
    if (bary_tri_inside(px, py, x0, y0, x1, y1, x2, y2, nondeg)) return 1;
    int verdict = (W_INFO && !nondeg) ? W_UNSURE : miss;
    if (n == 3) return verdict;
    const double x3 = wrap180(p.ln[3] - lon0) * DEG2RAD * R_STD * cos_lat0;
    const double y3 = (p.la[3] - lat0) * DEG2RAD * R_STD;
    if (bary_tri_inside(px, py, x0, y0, x2, y2, x3, y3, nondeg)) return 1;
    return (W_INFO && !nondeg) ? W_UNSURE : verdict;
}


// mesh.py:2210-2263 _element_contains with mesh.py:2006-2051
// _project_to_local_xy and mesh.py:2139-2168 _polygon_contains_bool; the
// cos of the mean vertex latitude comes from the host table.  Returns 1 when
// the element contains the point; otherwise 0, or with W_INFO the verdict
// class of the W search (W_OUT / W_UNSURE).
template <bool W_INFO>
__device__ __forceinline__ int element_contains_t(const DMesh& m, int c, double lon_p, double lat_p) {
    if (m.erec) {
        // the element's own record of its mask vertices (elem_record): one
        // read, no vertex-id indirection; the same values and arithmetic
        const double2* r = m.erec + 4 * (long long)c;
        const double2 r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2), r3 = __ldg(r + 3);
        if (!isnan(r0.x)) {
            const int n = isnan(r3.x) ? 3 : 4;
            Poly p;
            p.ln[0] = r0.x; p.la[0] = r0.y;
            p.ln[1] = r1.x; p.la[1] = r1.y;
            p.ln[2] = r2.x; p.la[2] = r2.y;
            p.ln[3] = n == 4 ? r3.x : r0.x; p.la[3] = n == 4 ? r3.y : r0.y;
            double dmin = 0.0, dmax = 0.0, lamin = r0.y, lamax = r0.y;
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                if (k < n) {
                    const double d = wrap180(p.ln[k] - p.ln[0]);
                    dmin = fmin(dmin, d);
                    dmax = fmax(dmax, d);
                    lamin = fmin(lamin, p.la[k]);
                    lamax = fmax(lamax, p.la[k]);
                }
            }
            const double dlon_p = wrap180(lon_p - p.ln[0]);
            if (dlon_p > dmax || dlon_p < dmin || lat_p > lamax || lat_p < lamin)
                return outside_box_verdict<W_INFO>(0, dmin, dmax, lamin, lamax, dlon_p, lat_p);
            return inside_box_verdict<W_INFO>(m, c, p, n, 0, lon_p, lat_p);
        }
    }
    const int4 e = __ldg(&m.en[c]);
    // the mask's vertex slots in order (-1 slots dropped, slot 3 dropped when
    // it repeats slot 0)
    const bool v3 = e.w >= 0 && !(e.w == e.x && e.x >= 0);
    int id0 = -1, id1 = -1, id2 = -1, id3 = -1;   // scalars: no dynamically indexed array
    int n = 0;
    auto push = [&](int v) {
        if (n == 0) id0 = v;
        else if (n == 1) id1 = v;
        else if (n == 2) id2 = v;
        else id3 = v;
        ++n;
    };
    if (e.x >= 0) push(e.x);
    if (e.y >= 0) push(e.y);
    if (e.z >= 0) push(e.z);
    if (v3) push(e.w);
    if (n < 3) return (W_INFO && !w_ring_matches_mask(e)) ? W_UNSURE : 0;
    auto vid = [&](int k) { return k == 1 ? id1 : (k == 2 ? id2 : id3); };
    const int miss = (W_INFO && !w_ring_matches_mask(e)) ? W_UNSURE : 0;
    // bbox prefilter in wrapped-delta space around the first valid vertex
    // (the first vertex's own delta is wrap180(0) == 0): running bounds only,
    // in the reference's order, so most rejected elements hold few registers
    const double2 a0 = __ldg(&m.ll[id0]);
    const double lon_ref = a0.x;
    double dmin = 0.0, dmax = 0.0, lamin = a0.y, lamax = a0.y;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        if (k < n) {
            const double2 a = __ldg(&m.ll[vid(k)]);
            const double d = wrap180(a.x - lon_ref);
            dmin = fmin(dmin, d);
            dmax = fmax(dmax, d);
            lamin = fmin(lamin, a.y);
            lamax = fmax(lamax, a.y);
        }
    }
    const double dlon_p = wrap180(lon_p - lon_ref);
    if (dlon_p > dmax || dlon_p < dmin || lat_p > lamax || lat_p < lamin)
        return outside_box_verdict<W_INFO>(miss, dmin, dmax, lamin, lamax, dlon_p, lat_p);
    // inside the box: the vertices again (cached)
    Poly p;
    p.ln[0] = a0.x;
    p.la[0] = a0.y;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        const double2 a = __ldg(&m.ll[k < n ? vid(k) : id0]);
        p.ln[k] = a.x;
        p.la[k] = a.y;
    }
    return inside_box_verdict<W_INFO>(m, c, p, n, miss, lon_p, lat_p);
}

// A box around each element that can only reject what the test above
// rejects too.  {centre longitude, half width in longitude, lowest and
// highest latitude}, in degrees, from the mask vertices: the half width and
// the latitudes are widened by the W search's margin (1e-5 of the extent
// plus 1e-9) and by kBoxSlack, then rounded outward to float.  A point
// outside it is outside the reference's bounding box by more than that
// margin, so element_contains_t returns 0 (W_OUT with W_INFO) for it.
// Elements whose verdict the box cannot give -- fewer than three vertices,
// a W ring unlike the mask, or an extent of 90 degrees or more -- get a
// negative half width and are never rejected by it.
constexpr double kBoxSlack = 1e-7;   // degrees, far above the double roundings of either test

__device__ __forceinline__ float4 elem_box(const DMesh& m, int c) {
    const float4 none = make_float4(0.0f, -1.0f, 0.0f, 0.0f);
    const int4 e = m.en[c];
    const bool v3 = e.w >= 0 && !(e.w == e.x && e.x >= 0);
    const int n = (e.x >= 0) + (e.y >= 0) + (e.z >= 0) + (v3 ? 1 : 0);
    if (n < 3 || !w_ring_matches_mask(e)) return none;
    const int ids[4] = {e.x, e.y, e.z, v3 ? e.w : -1};
    double lon_ref = 0.0, dmin = 0.0, dmax = 0.0, lamin = 0.0, lamax = 0.0;
    bool first = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (ids[k] < 0) continue;
        const double2 a = m.ll[ids[k]];
        if (first) {
            lon_ref = a.x; lamin = lamax = a.y; first = false;
            continue;
        }
        const double d = wrap180(a.x - lon_ref);
        dmin = fmin(dmin, d); dmax = fmax(dmax, d);
        lamin = fmin(lamin, a.y); lamax = fmax(lamax, a.y);
    }
    if (!(dmax - dmin < 90.0)) return none;
    const float cf = __double2float_rn(wrap180(lon_ref + 0.5 * (dmin + dmax)));
    double hw = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (ids[k] < 0) continue;
        hw = fmax(hw, fabs(wrap180(m.ll[ids[k]].x - (double)cf)));
    }
    const double mx = 1e-5 * (dmax - dmin) + 1e-9 + kBoxSlack, my = 1e-5 * (lamax - lamin) + 1e-9 + kBoxSlack;
    return make_float4(cf, __double2float_ru(hw + mx), __double2float_rd(lamin - my), __double2float_ru(lamax + my));
}

// The mask vertices of element c in the containment convention (-1 slots
// dropped, slot 3 dropped when it repeats slot 0), as element_contains_t
// reads them: lon, lat of each; slot 3 NaN for a triangle.  An element that
// needs its vertex ids for the verdict (fewer than three vertices, or a W
// ring unlike the mask) gets NaN in slot 0 and is tested from the ids.
__device__ __forceinline__ void elem_record(const DMesh& m, int c, double2* out) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const int4 e = m.en[c];
    const bool v3 = e.w >= 0 && !(e.w == e.x && e.x >= 0);
    const int n = (e.x >= 0) + (e.y >= 0) + (e.z >= 0) + (v3 ? 1 : 0);
    out[0] = out[1] = out[2] = out[3] = make_double2(nan, nan);
    if (n < 3 || !w_ring_matches_mask(e)) return;
    const int ids[4] = {e.x, e.y, e.z, v3 ? e.w : -1};
    int k = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (ids[j] >= 0) out[k++] = m.ll[ids[j]];
}

__device__ __forceinline__ bool box_rejects(float4 b, double lon_p, double lat_p) {
    if (b.y < 0.0f) return false;
    double dl = lon_p - (double)b.x;
    if (!(dl >= -180.0 && dl < 180.0)) dl -= 360.0 * floor((dl + 180.0) / 360.0);
    return fabs(dl) > (double)b.y || lat_p < (double)b.z || lat_p > (double)b.w;
}

// Which of ring positions k0 .. k0+3 (below e) survive their boxes, as bits;
// the element ids in c0..c3.  All four loads are issued before any test.
__device__ __forceinline__ unsigned ring_pass4(const DMesh& m, int k0, int e, double lon_p, double lat_p, int& c0,
                                               int& c1, int& c2, int& c3) {
    c0 = __ldg(&m.n2e[k0]);
    c1 = k0 + 1 < e ? __ldg(&m.n2e[k0 + 1]) : -1;
    c2 = k0 + 2 < e ? __ldg(&m.n2e[k0 + 2]) : -1;
    c3 = k0 + 3 < e ? __ldg(&m.n2e[k0 + 3]) : -1;
    const float4 reject = make_float4(0.0f, 0.0f, 1.0f, -1.0f);
    const float4 b0 = __ldg(&m.ebox[c0]);
    const float4 b1 = c1 >= 0 ? __ldg(&m.ebox[c1]) : reject;
    const float4 b2 = c2 >= 0 ? __ldg(&m.ebox[c2]) : reject;
    const float4 b3 = c3 >= 0 ? __ldg(&m.ebox[c3]) : reject;
    return (box_rejects(b0, lon_p, lat_p) ? 0u : 1u) | (box_rejects(b1, lon_p, lat_p) ? 0u : 2u) |
           (box_rejects(b2, lon_p, lat_p) ? 0u : 4u) | (box_rejects(b3, lon_p, lat_p) ? 0u : 8u);
}

__device__ __forceinline__ int pick4(int j, int c0, int c1, int c2, int c3) {
    return j == 0 ? c0 : (j == 1 ? c1 : (j == 2 ? c2 : c3));
}

__device__ __forceinline__ bool element_contains(const DMesh& m, int c, double lon_p, double lat_p) {
    if (m.ebox && box_rejects(__ldg(&m.ebox[c]), lon_p, lat_p)) return false;
    return element_contains_t<false>(m, c, lon_p, lat_p) == 1;
}

static __device__ __noinline__ int contain_two_ring(const DMesh& m, double lon_p, double lat_p, int nn);

// mesh.py:2392-2470 _find_containing_element_local: the 1-ring of the anchor,
// then its 2-ring; -1 when no element contains the point.
static __device__ KC_INL_CONTAIN int contain_local(const DMesh& m, double lon_p, double lat_p, int nn) {
    int s = __ldg(&m.n2e_off[nn]), e = __ldg(&m.n2e_off[nn + 1]);
    if (e == s) return -1;
    if (m.ebox) {
        // the ring's boxes four at a time; the survivors in ring order
        for (int k0 = s; k0 < e; k0 += 4) {
            int c0, c1, c2, c3;
            unsigned pass = ring_pass4(m, k0, e, lon_p, lat_p, c0, c1, c2, c3);
            while (pass) {
                const int c = pick4(__ffs(pass) - 1, c0, c1, c2, c3);
                pass &= pass - 1;
                if (element_contains_t<false>(m, c, lon_p, lat_p) == 1) return c;
            }
        }
        return contain_two_ring(m, lon_p, lat_p, nn);
    }
    for (int k = s; k < e; ++k) {
        int c = __ldg(&m.n2e[k]);
        if (element_contains(m, c, lon_p, lat_p)) return c;
    }
    return contain_two_ring(m, lon_p, lat_p, nn);
}

static __device__ __noinline__ int contain_two_ring(const DMesh& m, double lon_p, double lat_p, int nn) {
    int s = m.n2e_off[nn], e = m.n2e_off[nn + 1];
    for (int k = s; k < e; ++k) {
        int el = m.n2e[k];
        int4 en = m.en[el];
        for (int j = 0; j < 4; ++j) {
            int v = elem_node(en, j);
            if (v < 0 || v == nn) continue;
            int s2 = m.n2e_off[v], e2 = m.n2e_off[v + 1];
            for (int kk = s2; kk < e2; ++kk) {
                int c = m.n2e[kk];
                int4 ce = m.en[c];
                if (ce.x == nn || ce.y == nn || ce.z == nn || ce.w == nn) continue;
                if (element_contains(m, c, lon_p, lat_p)) return c;
            }
        }
    }
    return -1;
}

// contain_local, plus what its 1-ring scan implies for the barycentric W
// search of the same point and anchor (vertical.py:744-881): w_elem is the
// element that search returns (-1: its nodal fallback) unless w_unsure, when
// only running that search decides.
static __device__ KC_INL_CONTAIN int contain_local_w(const DMesh& m, double lon_p, double lat_p, int nn, int& w_elem,
                                                   bool& w_unsure) {
    w_elem = -1;
    w_unsure = false;
    int s = __ldg(&m.n2e_off[nn]), e = __ldg(&m.n2e_off[nn + 1]);
    if (e == s) return -1;
    if (m.ebox) {
        // a box rejection is a W_OUT verdict (elem_box)
        for (int k0 = s; k0 < e; k0 += 4) {
            int c0, c1, c2, c3;
            unsigned pass = ring_pass4(m, k0, e, lon_p, lat_p, c0, c1, c2, c3);
            while (pass) {
                const int c = pick4(__ffs(pass) - 1, c0, c1, c2, c3);
                pass &= pass - 1;
                const int v = element_contains_t<true>(m, c, lon_p, lat_p);
                if (v == 1) {
                    w_elem = c;
                    return c;
                }
                if (v == W_UNSURE) w_unsure = true;
            }
        }
        return contain_two_ring(m, lon_p, lat_p, nn);
    }
    for (int k = s; k < e; ++k) {
        const int c = __ldg(&m.n2e[k]);
        const int v = element_contains_t<true>(m, c, lon_p, lat_p);
        if (v == 1) {
            w_elem = c;
            return c;
        }
        if (v == W_UNSURE) w_unsure = true;
    }
    return contain_two_ring(m, lon_p, lat_p, nn);
}

}  // namespace kc
